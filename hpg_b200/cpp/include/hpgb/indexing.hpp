// indexing.hpp -- CF index bookkeeping, as the reference's CFSimpleIndexer
// (src/hpg_indexing.hpp:67-181): a CF cell (baseline class, time, w plane,
// frequency, Mueller element) maps to the (mueller, cube, group) triple of
// VisData::cf_index and the CF arrays.  Axes whose CF size may vary are
// linearised into the group index, the others into the cube index, in the
// order baseline class, time, w plane, frequency (first = most
// significant).
#pragma once

#include <array>
#include <utility>

namespace hpgb {

struct CFCellIndex {
  unsigned baseline_class = 0, time = 0, w_plane = 0, frequency = 0,
           mueller = 0;
  CFCellIndex() = default;
  CFCellIndex(unsigned b, unsigned t, unsigned w, unsigned f, unsigned m)
      : baseline_class(b), time(t), w_plane(w), frequency(f), mueller(m) {}
  bool operator==(const CFCellIndex& o) const {
    return baseline_class == o.baseline_class && time == o.time &&
           w_plane == o.w_plane && frequency == o.frequency &&
           mueller == o.mueller;
  }
};

class CFSimpleIndexer {
 public:
  using axis_desc_t = std::pair<unsigned, bool>;  // (length, variable size)
  using cf_index_t = std::array<unsigned, 3>;     // (mueller, cube, group)

  CFSimpleIndexer(const axis_desc_t& baseline_class, const axis_desc_t& time,
                  const axis_desc_t& w_plane, const axis_desc_t& frequency,
                  unsigned mueller)
      : m_axes{baseline_class, time, w_plane, frequency}, m_mueller(mueller) {}

  cf_index_t cf_index(const CFCellIndex& c) const {
    const unsigned idx[4] = {c.baseline_class, c.time, c.w_plane, c.frequency};
    cf_index_t r{c.mueller, 0, 0};
    for (int a = 0; a < 4; ++a) {
      unsigned& part = m_axes[a].second ? r[2] : r[1];
      part = part * m_axes[a].first + idx[a];
    }
    return r;
  }

  CFCellIndex cell_index(cf_index_t i) const {
    unsigned out[4];
    for (int a = 3; a >= 0; --a) {
      unsigned& part = m_axes[a].second ? i[2] : i[1];
      out[a] = part % m_axes[a].first;
      part /= m_axes[a].first;
    }
    return CFCellIndex(out[0], out[1], out[2], out[3], i[0]);
  }

  cf_index_t cf_extents() const {
    cf_index_t r{m_mueller, 1, 1};
    for (const auto& ax : m_axes) (ax.second ? r[2] : r[1]) *= ax.first;
    return r;
  }

  std::array<unsigned, 5> cell_extents() const {
    return {m_axes[0].first, m_axes[1].first, m_axes[2].first,
            m_axes[3].first, m_mueller};
  }

 private:
  std::array<axis_desc_t, 4> m_axes;
  unsigned m_mueller;
};

}  // namespace hpgb
