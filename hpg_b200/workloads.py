"""Seeded synthetic workloads with the shapes of the benchmark configurations.

There is no dataset: every input is generated from a fixed seed.  CFs are
separable products of 1-D factors (a Gaussian amplitude, optionally a
w-dependent quadratic phase) times a per-Mueller-element complex factor,
built in FP64 and rounded to complex64 in the CFArray logical order
(x, y, mueller, cube).  Visibilities are hpg::VisData<N> records with u, v
uniform in a disk of radius ``disk * grid extent`` cells around the grid
centre and w uniform in +-``w_frac`` of the maximum baseline.

Configurations (sizes from the benchmark definition):
  single_pol : 512x512x1x1, 1 group support 7 (os 20), 100k visibilities,
               Mueller {{0}}, Gaussian sigma 1 cell, w = 0
  full_pol   : 2048x2048x4x1, 8 w-plane groups with supports
               8,12,16,20,24,28,32,32 (os 128), dense 4x4 Mueller (16 terms:
               1 on the diagonal, complex N(0, 0.1) off-diagonal), 10M
               visibilities, complex128 N(0,1) model
"""
import math

import numpy as np

C_LIGHT = 299792458.0


def visdata_dtype(npol):
    from .abi import visdata_dtype as vd
    return vd(npol)


def cf_extent(support, oversampling, padding=2):
    """Extent of a CF of even support S: (S + 2*padding)*os, so that the
    reference's radius formula (src/hpg.hpp:687-694) gives S/2 and the CF has
    S + 1 taps; an odd support S gives radius (S-1)/2 and S taps."""
    return (support + 2 * padding) * oversampling


def cf_axis(ext, oversampling, sigma_cells, w_phase=0.0):
    """1-D factor over the fine axis: Gaussian of sigma_cells, times
    exp(i*pi*w_phase*u^2) with u in cells from the centre."""
    x = np.arange(ext, dtype=np.float64)
    u = (x - ext / 2.0) / oversampling
    amp = np.exp(-0.5 * (u / sigma_cells) ** 2)
    return amp * np.exp(1j * np.pi * w_phase * u * u)


def separable_cf(supports, oversampling, mueller_factors, sigma=None,
                 w_phases=None, ncube=1):
    """Extents and complex64 values (one array per group) of a separable CF.

    mueller_factors: complex array of the Mueller planes' scale factors."""
    mf = np.asarray(mueller_factors, np.complex128).reshape(-1)
    extents, values = [], []
    for g, s in enumerate(supports):
        ext = cf_extent(s, oversampling)
        sg = sigma if sigma is not None else max(s / 6.0, 0.5)
        wp = 0.0 if w_phases is None else w_phases[g]
        a = cf_axis(ext, oversampling, sg, wp)
        v = (a[:, None, None] * a[None, :, None] * mf[None, None, :])
        v = np.repeat(v[..., None], ncube, axis=3)
        values.append(v.astype(np.complex64))
        extents.append((ext, ext, len(mf), ncube))
    return extents, values


def separable_cf_torch(supports, oversampling, mueller_factors, device,
                       sigma=None, w_phases=None):
    """Same CF as separable_cf, generated on a CUDA device with torch (for
    CF tables of several GB)."""
    import torch
    mf = torch.tensor(np.asarray(mueller_factors, np.complex128).reshape(-1),
                      device=device)
    extents, values = [], []
    for g, s in enumerate(supports):
        ext = cf_extent(s, oversampling)
        sg = sigma if sigma is not None else max(s / 6.0, 0.5)
        wp = 0.0 if w_phases is None else w_phases[g]
        a = torch.tensor(cf_axis(ext, oversampling, sg, wp), device=device)
        v = (a[:, None, None] * a[None, :, None]).to(torch.complex64)
        v = v * mf.to(torch.complex64)[None, None, :]
        values.append(v.unsqueeze(-1).contiguous())
        extents.append((ext, ext, len(mf), 1))
        del a
    return extents, values


def dense_mueller(rng, npol=4, scale=0.1):
    """4x4 Mueller factors: 1 on the diagonal, complex N(0, scale) off it."""
    m = (rng.normal(0, scale, (npol, npol)) +
         1j * rng.normal(0, scale, (npol, npol)))
    np.fill_diagonal(m, 1.0)
    idx = [[r * npol + c for c in range(npol)] for r in range(npol)]
    return m.reshape(-1), idx


def visibilities(n, npol, grid_size, grid_scale, freq, rng, disk=0.45,
                 w_frac=0.0, ngroups=1, group_of_w=None, weights=(0.5, 1.5),
                 phase=0.0, grad=None, ncube_cf=1, gaussian_values=True):
    """n VisData<npol> records with u, v uniform in a disk of radius
    disk*min(nx, ny) cells (converted through grid_scale and freq).

    When w_frac > 0, w is uniform in +-w_frac * max baseline and the CF group
    is group_of_w(|w| / w_max) (default: linear bins over ngroups)."""
    nx, ny = grid_size[0], grid_size[1]
    inv_lambda = freq / C_LIGHT
    rmax_cells = disk * min(nx, ny)
    r = rmax_cells * np.sqrt(rng.random(n))
    th = 2 * np.pi * rng.random(n)
    u = r * np.cos(th) / (grid_scale[0] * inv_lambda)
    v = r * np.sin(th) / (grid_scale[1] * inv_lambda)
    bmax = rmax_cells / (abs(grid_scale[0]) * inv_lambda)
    out = np.zeros(n, visdata_dtype(npol))
    if gaussian_values:
        vals = (rng.standard_normal((n, npol)) +
                1j * rng.standard_normal((n, npol))).astype(np.complex64)
    else:
        vals = (rng.uniform(-1, 1, (n, npol)) +
                1j * rng.uniform(-1, 1, (n, npol))).astype(np.complex64)
    out["vis"] = vals
    lo, hi = weights
    out["weights"] = (hi - (hi - lo) * rng.random((n, npol))).astype(np.float32)
    out["freq"] = freq
    out["phase"] = phase
    out["uvw"][:, 0] = u
    out["uvw"][:, 1] = v
    if w_frac > 0:
        w = (2 * rng.random(n) - 1) * w_frac * bmax
        out["uvw"][:, 2] = w
        frac = np.abs(w) / (w_frac * bmax)
        if group_of_w is None:
            grp = np.minimum((frac * ngroups).astype(np.int64), ngroups - 1)
        else:
            grp = group_of_w(frac)
        out["cf_index"][:, 1] = grp
    else:
        out["cf_index"][:, 1] = rng.integers(0, ngroups, n) if ngroups > 1 else 0
    if ncube_cf > 1:
        out["cf_index"][:, 0] = rng.integers(0, ncube_cf, n)
    if grad is not None:
        out["cf_phase_gradient"] = rng.uniform(-grad, grad, (n, 2))
    return out


def single_pol_config(n=100_000, seed=20261203):
    """Plain gridding case: 512x512, 1 polarization, support 7 at os 20."""
    rng = np.random.default_rng(seed)
    grid_size = (512, 512, 1, 1)
    grid_scale = (0.0476591, 0.0476591)
    extents, values = separable_cf([7], 20, [1.0], sigma=1.0)
    vis = visibilities(n, 1, grid_size, grid_scale, 1.4e9, rng)
    return dict(grid_size=grid_size, grid_scale=grid_scale, mueller=[[0]],
                conj_mueller=[[0]], oversampling=20, cf_extents=extents,
                cf_values=values, vis=vis, model=None)


FULL_POL_SUPPORTS = (8, 12, 16, 20, 24, 28, 32, 32)


def full_pol_params(seed=20261204, supports=FULL_POL_SUPPORTS, oversampling=128):
    rng = np.random.default_rng(seed)
    mf, idx = dense_mueller(rng)
    w_phases = [0.02 * g for g in range(len(supports))]
    return dict(rng=rng, mueller_factors=mf, mueller=idx, conj_mueller=idx,
                supports=list(supports), oversampling=oversampling,
                w_phases=w_phases, grid_scale=(0.0476591, 0.0476591),
                freq=1.4e9)


def full_pol_config(n, grid=2048, seed=20261204, supports=FULL_POL_SUPPORTS,
                    oversampling=128, with_cf=True, grad=None):
    """Full-polarization round trip: grid x grid x 4 x 1, 8 w-plane groups,
    dense Mueller, n visibilities, complex128 N(0,1) model."""
    p = full_pol_params(seed, supports, oversampling)
    rng = p["rng"]
    grid_size = (grid, grid, 4, 1)
    vis = visibilities(n, 4, grid_size, p["grid_scale"], p["freq"], rng,
                       w_frac=0.3, ngroups=len(supports), grad=grad)
    model = (rng.standard_normal((1, 4, grid, grid)) +
             1j * rng.standard_normal((1, 4, grid, grid)))
    cfg = dict(grid_size=grid_size, grid_scale=p["grid_scale"],
               mueller=p["mueller"], conj_mueller=p["conj_mueller"],
               oversampling=oversampling, vis=vis, model=model,
               supports=list(supports), mueller_factors=p["mueller_factors"],
               w_phases=p["w_phases"])
    if with_cf:
        ext, vals = separable_cf(supports, oversampling, p["mueller_factors"],
                                 w_phases=p["w_phases"])
        cfg["cf_extents"], cfg["cf_values"] = ext, vals
    return cfg


def algorithmic_bytes(vis, npol, taps_by_group, mueller_planes, grid_elems,
                      c):
    """Algorithmic HBM bytes of one batch: per visibility its record plus
    its CF slice (taps^2 * planes * 8 B, read once), plus c passes over the
    complex128 grid (c = 2 gridding, 3 degrid+grid)."""
    grp = vis["cf_index"][:, 1].astype(np.int64)
    taps = np.asarray(taps_by_group, np.int64)[grp]
    rec = visdata_dtype(npol).itemsize
    return int(len(vis) * rec + (taps * taps).sum() * mueller_planes * 8 +
               c * grid_elems * 16)
