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


KINDS = {"direct": abi.KERNEL_DIRECT, "tiled": abi.KERNEL_TILED}


@pytest.fixture(params=["tiled", "direct"])
def kind(request):
    """The operators on the tile sort of the batch (adjoint_tiled.cu) and
    the per-visibility kernels (adjoint.cu)."""
    return request.param


def setup(n=1500, grad=0.3, seed=21, model=True, kind="tiled"):
    import torch
    cfg = workloads.full_pol_config(n, grid=128, oversampling=16,
                                    supports=(4, 6, 8), seed=seed, grad=grad)
    g = Gridder.create(0, 0, n, None, cfg["grid_size"], cfg["grid_scale"],
                       cfg["mueller"], cfg["conj_mueller"])
    g.set_gridding_kernel(KINDS[kind])
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


def test_degrid_dot_product(gpu, kind):
    import torch
    from hpg_b200 import autograd as ag
    cfg, g, dvis = setup(kind=kind)
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


def test_grid_dot_product(gpu, kind):
    import torch
    from hpg_b200 import autograd as ag
    cfg, g, dvis = setup(seed=22, kind=kind)
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


def test_operators_match_gridder(gpu, kind):
    """D and G against the gridder's own degridding and gridding."""
    import torch
    from hpg_b200 import autograd as ag
    cfg, g, dvis = setup(seed=23, kind=kind)
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


def test_degrid_adjoint_is_oracle_gridding_of_cotangent(gpu, kind, oracle_lib):
    """D^H y is the reference's gridding (mueller == conjugate mueller here)
    of the values y * phasor / conj(den) / (phasor * w)."""
    import torch
    from hpg_b200 import autograd as ag
    O = oracle_lib
    cfg, g, dvis = setup(n=800, seed=24, kind=kind)
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


def test_loss_gradient_finite_differences(gpu, kind):
    """dL/dG of L = sum w |D(G) - V|^2 through torch.autograd against
    central differences on random grid cells."""
    import torch
    from hpg_b200 import autograd as ag
    cfg, g, dvis = setup(n=600, seed=25, kind=kind)
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


def test_tiled_operators_equal_direct(gpu):
    """The tile-sorted operators against the per-visibility ones: the same
    FP64 arithmetic in another summation order (1e-12)."""
    import torch
    from hpg_b200 import autograd as ag
    cfg, gt, dvis = setup(n=1200, seed=27, kind="tiled")
    _, gd, _ = setup(n=1200, seed=27, kind="direct")
    gen = torch.Generator(device="cuda:0").manual_seed(4)
    n = len(cfg["vis"])
    x = crandn(grid_shape(cfg), gen)
    y = crandn((n, 4), gen)
    for op in (ag.Degrid, ag.Grid):
        arg = x if op is ag.Degrid else y
        a = op.apply(arg, gt, dvis)
        b = op.apply(arg, gd, dvis)
        assert gt.last_gridding_kernel() == abi.KERNEL_TILED
        assert gd.last_gridding_kernel() == abi.KERNEL_DIRECT
        assert torch.linalg.norm(a - b) / torch.linalg.norm(b) <= 1e-12
        # adjoints
        cot = y if op is ag.Degrid else x
        ar = arg.clone().requires_grad_(True)
        op.apply(ar, gt, dvis).backward(cot)
        br = arg.clone().requires_grad_(True)
        op.apply(br, gd, dvis).backward(cot)
        assert (torch.linalg.norm(ar.grad - br.grad) /
                torch.linalg.norm(br.grad)) <= 1e-12
    gt.close()
    gd.close()


@pytest.mark.parametrize("grad", [0.2, None], ids=["screen", "no-screen"])
@pytest.mark.parametrize("npol,expect", [(1, abi.KERNEL_TILED),
                                         (2, abi.KERNEL_TILED),
                                         (4, abi.KERNEL_DIRECT)])
def test_wide_support_dot_products(gpu, npol, expect, grad):
    """Supports 8..64 (9..65 taps), diagonal Mueller, as in the
    differentiable workload: both dot-product identities, with phase screens
    and without (the workload's case: the operators' cell loops without a
    screen take more cells per lane).  One or two grid rows take the tiled
    operators; four rows of FP64 regions for 65 taps do not fit shared
    memory, and the automatic choice takes the per-visibility kernels."""
    import torch
    from hpg_b200 import autograd as ag
    rng = np.random.default_rng(50 + npol)
    gs = (256, 256, npol, 1)
    supports = (8, 24, 40, 64)
    ext, vals = workloads.separable_cf(supports, 8, np.ones(npol) +
                                       0.1j * rng.standard_normal(npol))
    mi = [[r if c == r else -1 for c in range(npol)] for r in range(npol)]
    vis = workloads.visibilities(2000, npol, gs, (0.05, 0.05), 1.4e9, rng,
                                 disk=0.3, w_frac=0.3, ngroups=len(supports),
                                 grad=grad)
    g = Gridder.create(0, 0, len(vis), None, gs, (0.05, 0.05), mi, mi)
    g.set_gridding_kernel(abi.KERNEL_AUTO)
    g.set_convolution_function(CFArray(8, ext, vals))
    dvis = torch.from_numpy(
        np.frombuffer(vis.tobytes(), np.uint8).copy()).to("cuda:0")
    gen = torch.Generator(device="cuda:0").manual_seed(6)
    x = crandn((1, npol, 256, 256), gen)
    y = crandn((len(vis), npol), gen)
    for op, arg, cot in ((ag.Degrid, x, y), (ag.Grid, y, x)):
        fx = op.apply(arg, g, dvis)
        ar = arg.clone().requires_grad_(True)
        op.apply(ar, g, dvis).backward(cot)
        lhs = torch.vdot(fx.flatten(), cot.flatten())
        rhs = torch.vdot(arg.flatten(), ar.grad.flatten())
        assert abs(lhs) > 0
        assert abs(lhs - rhs) / abs(lhs) <= 1e-10
        assert g.last_gridding_kernel() == expect
    if expect == abi.KERNEL_TILED:
        # the tiled operators and their adjoints against the per-visibility
        # kernels: the same FP64 arithmetic in another order (1e-12)
        gd = Gridder.create(0, 0, len(vis), None, gs, (0.05, 0.05), mi, mi)
        gd.set_gridding_kernel(abi.KERNEL_DIRECT)
        gd.set_convolution_function(CFArray(8, ext, vals))
        for op, arg, cot in ((ag.Degrid, x, y), (ag.Grid, y, x)):
            a = op.apply(arg, g, dvis)
            b = op.apply(arg, gd, dvis)
            assert torch.linalg.norm(a - b) / torch.linalg.norm(b) <= 1e-12
            ar = arg.clone().requires_grad_(True)
            op.apply(ar, g, dvis).backward(cot)
            br = arg.clone().requires_grad_(True)
            op.apply(br, gd, dvis).backward(cot)
            assert (torch.linalg.norm(ar.grad - br.grad) /
                    torch.linalg.norm(br.grad)) <= 1e-12
        assert g.last_gridding_kernel() == abi.KERNEL_TILED
        assert gd.last_gridding_kernel() == abi.KERNEL_DIRECT
        gd.close()
    g.close()
