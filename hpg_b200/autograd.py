"""torch.autograd binding of the FP64 degridding and gridding operators.

A thin test binding over the C ABI (hpgb_degrid_linear / hpgb_degrid_adjoint
/ hpgb_grid_linear / hpgb_grid_adjoint): the forward calls the operator, the
backward calls its hand-written adjoint kernel.  Nothing of the forward is
stored for the backward: both maps are linear, so the backward needs only
the visibility records (geometry), which the caller keeps on the device.

PyTorch's convention for a real loss L of complex tensors is that the
gradient of z is dL/dRe(z) + i dL/dIm(z); for a complex-linear map y = A x
that gradient is A^H applied to the gradient of y, which is what the
adjoint kernels compute.

Tensors: the model / grid is complex128 of shape (cube, mrow, ny, nx) (the
gridder's device grid layout), per-visibility values are complex128 of shape
(n, npol), all on the gridder's device.  The library works on the gridder's
stream; these functions wait for torch's current stream before a call and
for the gridder after it.
"""
import ctypes

import torch

from .abi import check, load


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _grid_shape(gridder):
    nx, ny, nr, nc = gridder.grid_size
    return (nc, nr, ny, nx)


def _check_records(dvis, gridder):
    from .abi import visdata_dtype
    rec = visdata_dtype(gridder.npol).itemsize
    if dvis.dtype != torch.uint8 or not dvis.is_cuda or not dvis.is_contiguous():
        raise ValueError("records must be a contiguous CUDA uint8 tensor")
    if dvis.numel() % rec:
        raise ValueError("record buffer is not a whole number of records")
    return dvis.numel() // rec


def _run(fn, gridder, dvis, n, src, dst):
    torch.cuda.current_stream(src.device).synchronize()
    check(fn(gridder._h, _p(dvis), n, gridder.npol, _p(src), _p(dst)))
    gridder.fence()


class Degrid(torch.autograd.Function):
    """values = D(model): the FP64 degridding prediction of every record."""

    @staticmethod
    def forward(ctx, model, gridder, dvis):
        n = _check_records(dvis, gridder)
        model = model.contiguous()
        if model.dtype != torch.complex128 or tuple(model.shape) != _grid_shape(gridder):
            raise ValueError("model must be complex128 of the grid's shape")
        out = torch.empty((n, gridder.npol), dtype=torch.complex128,
                          device=model.device)
        _run(load().hpgb_degrid_linear, gridder, dvis, n, model, out)
        ctx.gridder, ctx.dvis, ctx.n = gridder, dvis, n
        return out

    @staticmethod
    def backward(ctx, grad_values):
        g = grad_values.contiguous().to(torch.complex128)
        gin = torch.zeros(_grid_shape(ctx.gridder), dtype=torch.complex128,
                          device=g.device)
        _run(load().hpgb_degrid_adjoint, ctx.gridder, ctx.dvis, ctx.n, g, gin)
        return gin, None, None


class Grid(torch.autograd.Function):
    """grid = G(values): FP64 gridding of phasor * weight * values."""

    @staticmethod
    def forward(ctx, values, gridder, dvis):
        n = _check_records(dvis, gridder)
        values = values.contiguous()
        if values.dtype != torch.complex128 or tuple(values.shape) != (n, gridder.npol):
            raise ValueError("values must be complex128 of shape (n, npol)")
        out = torch.zeros(_grid_shape(gridder), dtype=torch.complex128,
                          device=values.device)
        _run(load().hpgb_grid_linear, gridder, dvis, n, values, out)
        ctx.gridder, ctx.dvis, ctx.n = gridder, dvis, n
        return out

    @staticmethod
    def backward(ctx, grad_grid):
        g = grad_grid.contiguous().to(torch.complex128)
        gin = torch.empty((ctx.n, ctx.gridder.npol), dtype=torch.complex128,
                          device=g.device)
        _run(load().hpgb_grid_adjoint, ctx.gridder, ctx.dvis, ctx.n, g, gin)
        return gin, None, None


def degrid(model, gridder, dvis):
    return Degrid.apply(model, gridder, dvis)


def grid(values, gridder, dvis):
    return Grid.apply(values, gridder, dvis)
