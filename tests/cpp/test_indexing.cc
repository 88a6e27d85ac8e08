// hpgb::CFSimpleIndexer against the reference's cases
// (tests/CFIndexerUnitTests.cc:19-102), restated.
#include <cstdio>

#include "hpgb/indexing.hpp"

static int failures = 0;
#define CHECK(cond)                                                 \
  do {                                                              \
    if (!(cond)) {                                                  \
      std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
      ++failures;                                                   \
    }                                                               \
  } while (0)

int main() {
  using Ix = hpgb::CFSimpleIndexer;
  {
    const unsigned nb = 1, nt = 2, nw = 3, nf = 4, nm = 5;
    for (int bits = 0; bits < 16; ++bits) {
      const bool bv = bits & 1, tv = bits & 2, wv = bits & 4, fv = bits & 8;
      unsigned cube = 1, grp = 1;
      (bv ? grp : cube) *= nb;
      (tv ? grp : cube) *= nt;
      (wv ? grp : cube) *= nw;
      (fv ? grp : cube) *= nf;
      Ix ix({nb, bv}, {nt, tv}, {nw, wv}, {nf, fv}, nm);
      CHECK((ix.cf_extents() == Ix::cf_index_t{nm, cube, grp}));
    }
  }
  {
    const unsigned nw = 3, nf = 4;
    Ix ix({2, true}, {2, false}, {nw, true}, {nf, true}, 8);
    struct Case { hpgb::CFCellIndex c; Ix::cf_index_t i; };
    const Case cases[] = {
        {{0, 0, 0, 0, 0}, {0, 0, 0}},
        {{1, 0, 0, 0, 0}, {0, 0, nw * nf}},
        {{1, 0, 2, 0, 0}, {0, 0, nw * nf + 2 * nf}},
        {{1, 0, 2, 0, 1}, {1, 0, nw * nf + 2 * nf}},
        {{1, 1, 2, 0, 0}, {0, 1, nw * nf + 2 * nf}},
        {{1, 1, 2, 0, 1}, {1, 1, nw * nf + 2 * nf}},
        {{1, 1, 2, 3, 1}, {1, 1, nw * nf + 2 * nf + 3}}};
    for (const auto& k : cases) {
      CHECK(ix.cf_index(k.c) == k.i);
      CHECK(ix.cell_index(k.i) == k.c);
    }
  }
  if (failures == 0) std::printf("OK\n");
  return failures == 0 ? 0 : 1;
}
