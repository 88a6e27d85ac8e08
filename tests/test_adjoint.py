"""Degridding / gridding as FP64 linear operators and their adjoint kernels.

  - dot-product tests <D x, y> = <x, D^H y> and <G u, g> = <u, G^H g> to
    1e-10 relative (FP64 throughout);
  - the operators agree with the gridder's own degridding and gridding
    (which round to complex<float> / use FP32 products): 1e-6;
  - D^H y equals the CPU oracle's grid_visibilities applied to the
    cotangent (values y * phasor / conj(den) / (phasor * w), the reference's
    gridding with the degridding normaliser): 1e-6 (FP32 products there);
  - torch.autograd through the binding: dL/dG of
    L = sum w |D(G) - V|^2 against central finite differences on random
    cells (L is quadratic, so the differences are exact up to rounding).
"""
import numpy as np
import pytest

from hpg_b200 import CFArray, Gridder, abi, workloads

pytestmark = pytest.mark.gpu


def setup(n=1500, grad=0.3, seed=21, model=True):
    import torch
    cfg = workloads.full_pol_config(n, grid=128, oversampling=16,
                                    supports=(4, 6, 8), seed=seed, grad=grad)
    g = Gridder.create(0, 0, n, None, cfg["grid_size"], cfg["grid_scale"],
                       cfg["mueller"], cfg["conj_mueller"])
    g.set_convolution_function(CFArray(cfg["oversampling"], cfg["cf_extents"],
                                       cfg["cf_values"]))
    dvis = torch.from_numpy(
        np.frombuffer(cfg["vis"].tobytes(), np.uint8).copy()).to("cuda:0")
    return cfg, g, dvis


def crandn(shape, gen, scale=1.0):
    import torch
    re = torch.randn(shape, generator=gen, dtype=torch.float64, device="cuda:0")
    im = torch.randn(shape, generator=gen, dtype=torch.float64, device="cuda:0")
    return torch.complex(re, im) * scale


def grid_shape(cfg):
    nx, ny, nr, nc = cfg["grid_size"]
    return (nc, nr, ny, nx)


def test_degrid_dot_product(gpu):
    import torch
    from hpg_b200 import autograd as ag
    cfg, g, dvis = setup()
    gen = torch.Generator(device="cuda:0").manual_seed(1)
    n = len(cfg["vis"])
    x = crandn(grid_shape(cfg), gen)
    y = crandn((n, 4), gen)
    dx = ag.Degrid.apply(x, g, dvis)
    x_req = x.clone().requires_grad_(True)
    out = ag.Degrid.apply(x_req, g, dvis)
    out.backward(y)
    dhy = x_req.grad
    lhs = torch.vdot(dx.flatten(), y.flatten())   # <D x, y>
    rhs = torch.vdot(x.flatten(), dhy.flatten())  # <x, D^H y>
    assert abs(lhs) > 0
    assert abs(lhs - rhs) / abs(lhs) <= 1e-10
    g.close()


def test_grid_dot_product(gpu):
    import torch
    from hpg_b200 import autograd as ag
    cfg, g, dvis = setup(seed=22)
    gen = torch.Generator(device="cuda:0").manual_seed(2)
    n = len(cfg["vis"])
    u = crandn((n, 4), gen)
    gg = crandn(grid_shape(cfg), gen)
    gu = ag.Grid.apply(u, g, dvis)
    u_req = u.clone().requires_grad_(True)
    ag.Grid.apply(u_req, g, dvis).backward(gg)
    ghg = u_req.grad
    lhs = torch.vdot(gu.flatten(), gg.flatten())
    rhs = torch.vdot(u.flatten(), ghg.flatten())
    assert abs(lhs) > 0
    assert abs(lhs - rhs) / abs(lhs) <= 1e-10
    g.close()


def test_operators_match_gridder(gpu):
    """D and G against the gridder's own degridding and gridding."""
    import torch
    from hpg_b200 import autograd as ag
    cfg, g, dvis = setup(seed=23)
    g.set_model(cfg["model"])
    fut = g.degrid_get_predicted_visibilities(cfg["vis"])
    g.fence()
    pred = fut.get()["vis"].astype(np.complex128)
    model = torch.from_numpy(np.ascontiguousarray(cfg["model"])).to("cuda:0")
    dx = ag.Degrid.apply(model, g, dvis).cpu().numpy()
    assert np.linalg.norm(dx - pred) / np.linalg.norm(pred) <= 1e-6
    g.reset_grid()
    g.grid_visibilities(cfg["vis"])
    g.fence()
    vals = torch.from_numpy(cfg["vis"]["vis"].astype(np.complex128)).to("cuda:0")
    gu = ag.Grid.apply(vals, g, dvis).cpu().numpy()
    ref = g.grid_values()
    assert np.linalg.norm(gu - ref) / np.linalg.norm(ref) <= 1e-6
    g.close()


def test_degrid_adjoint_is_oracle_gridding_of_cotangent(gpu, oracle_lib):
    """D^H y is the reference's gridding (mueller == conjugate mueller here)
    of the values y * phasor / conj(den) / (phasor * w)."""
    import torch
    from hpg_b200 import autograd as ag
    O = oracle_lib
    cfg, g, dvis = setup(n=800, seed=24)
    vis = cfg["vis"]
    n = len(vis)
    rng = np.random.default_rng(5)
    y = rng.standard_normal((n, 4)) + 1j * rng.standard_normal((n, 4))
    o = O.Oracle(cfg["grid_size"], cfg["grid_scale"], cfg["mueller"],
                 cfg["conj_mueller"], cfg["oversampling"], cfg["cf_extents"],
                 cfg["cf_values"])
    den = o.normalisers(vis)
    w = vis["weights"].astype(np.float64)
    # values whose gridding value (phasor * w * value) is phasor * y / conj(den)
    v2 = vis.copy()
    v2["vis"] = (y / np.conj(den) / w).astype(np.complex64)
    o.grid_visibilities(v2, update_weights=False)
    yt = torch.from_numpy(y).to("cuda:0")
    x_req = torch.zeros(grid_shape(cfg), dtype=torch.complex128,
                        device="cuda:0", requires_grad=True)
    ag.Degrid.apply(x_req, g, dvis).backward(yt)
    dhy = x_req.grad.cpu().numpy()
    assert np.linalg.norm(dhy - o.grid) / np.linalg.norm(o.grid) <= 1e-6
    g.close()


def test_loss_gradient_finite_differences(gpu):
    """dL/dG of L = sum w |D(G) - V|^2 through torch.autograd against
    central differences on random grid cells."""
    import torch
    from hpg_b200 import autograd as ag
    cfg, g, dvis = setup(n=600, seed=25)
    n = len(cfg["vis"])
    gen = torch.Generator(device="cuda:0").manual_seed(3)
    G0 = crandn(grid_shape(cfg), gen, 0.1)
    V = torch.from_numpy(cfg["vis"]["vis"].astype(np.complex128)).to("cuda:0")
    W = torch.from_numpy(cfg["vis"]["weights"].astype(np.float64)).to("cuda:0")

    def loss(G):
        r = ag.Degrid.apply(G, g, dvis) - V
        return (W * (r.real ** 2 + r.imag ** 2)).sum()

    Gr = G0.clone().requires_grad_(True)
    loss(Gr).backward()
    grad = Gr.grad
    # cells the footprints touch (the gradient is zero elsewhere)
    nz = torch.nonzero(grad.abs() > 0)
    assert len(nz) > 100
    pick = nz[torch.randperm(len(nz), generator=gen, device="cuda:0")[:20]]
    h = 1e-3
    for idx in pick.tolist():
        idx = tuple(idx)
        for unit in (1.0, 1j):
            Gp = G0.clone()
            Gp[idx] += h * unit
            Gm = G0.clone()
            Gm[idx] -= h * unit
            fd = (loss(Gp) - loss(Gm)).item() / (2 * h)
            an = grad[idx].real.item() if unit == 1.0 else grad[idx].imag.item()
            assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-3), (idx, unit, fd, an)
    g.close()


def test_operator_argument_errors(gpu):
    cfg, g, dvis = setup(n=10, seed=26)
    lib = abi.load()
    import ctypes
    rc = lib.hpgb_degrid_linear(g._h, ctypes.c_void_p(dvis.data_ptr()), 10, 2,
                                ctypes.c_void_p(1), ctypes.c_void_p(1))
    assert rc == 1 + abi.ERROR_TYPES.index("InvalidNumberPolarizations")
    rc = lib.hpgb_grid_adjoint(g._h, ctypes.c_void_p(dvis.data_ptr()), 11, 4,
                               ctypes.c_void_p(1), ctypes.c_void_p(1))
    assert rc == 1 + abi.ERROR_TYPES.index("ExcessiveNumberVisibilities")
    rc = lib.hpgb_grid_linear(g._h, ctypes.c_void_p(dvis.data_ptr()), 10, 4,
                              None, None)
    assert rc == 1 + abi.ERROR_TYPES.index("Other")
    g.close()
