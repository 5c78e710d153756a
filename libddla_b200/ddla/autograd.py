"""Differentiable negative log marginal likelihood on the GPU handle.

    loss_b = 1/2 (y_b^T A_b^-1 y_b + log det A_b)

`chol_nll(A, y)` takes the matrices; `gp_nll(X, y, theta)` builds
A = K(theta) + sigma^2 I (squared-exponential kernel
K_ij = sigma_f^2 exp(-|x_i - x_j|^2 / (2 l^2)), theta = (l, sigma_f^2, sigma^2))
on the device.  Both are torch.autograd.Functions whose forward is the batched
factor + solve + log-determinant launch and whose backward is the hand-written
adjoint (ddla_?_chol_nll_grad_batched / ddla_?_gp_nll_grad_batched):
dloss/dA = 1/2 (A^-1 - alpha alpha^T), dloss/dy = alpha (alpha = A^-1 y), and
for gp_nll the adjoint contracted with dA/dtheta inside the kernel.

A is read as a symmetric matrix: only the triangle that column-major storage
calls lower (the upper triangle of a row-major torch tensor) is used, and the
gradient returned for A is the full symmetric dloss/dA, the convention of
torch.linalg for symmetric inputs.  Orders above 1024 take one problem at a
time.  No reference counterpart.
"""
from __future__ import annotations

import ctypes

from . import _c_api as C

_HANDLE = None


def default_handle():
    """A GPU handle shared by calls that do not pass one."""
    global _HANDLE
    if _HANDLE is None:
        from .backend import Backend, Handle
        _HANDLE = Handle(Backend.GPU)
    return _HANDLE


def _torch():
    import torch
    return torch


def _handle_stream(handle):
    torch = _torch()
    st = ctypes.c_void_p()
    C.check_status(C.ddla_c_get_stream(handle.ptr, ctypes.byref(st)), "ddla_c_get_stream")
    return torch.cuda.ExternalStream(st.value) if st.value else torch.cuda.default_stream()


class _OnHandleStream:
    """Orders the handle's stream after torch's current stream on entry and
    torch's after the handle's on exit.  The tensors are allocated on torch's
    stream, which waits for the library's work before anything that follows,
    so the caching allocator cannot hand their memory out while it is in use."""

    def __init__(self, handle, *tensors):
        self.handle = handle

    def __enter__(self):
        torch = _torch()
        self.hs = _handle_stream(self.handle)
        self.cur = torch.cuda.current_stream()
        self.hs.wait_stream(self.cur)
        return self

    def __exit__(self, *exc):
        self.cur.wait_stream(self.hs)


def _sfx(dtype) -> str:
    torch = _torch()
    if dtype == torch.float64:
        return "d"
    if dtype == torch.float32:
        return "s"
    raise TypeError(f"unsupported dtype {dtype} (float32 or float64)")


def _check_info(info):
    bad = (info != 0).nonzero()
    if bad.numel():
        b = int(bad[0, 0])
        raise RuntimeError(f"matrix {b} is not positive definite (leading minor {int(info[b])})")


def _make_functions():
    torch = _torch()

    class _CholNLL(torch.autograd.Function):
        @staticmethod
        def forward(ctx, A, y, handle):
            batch, n = y.shape
            if A.shape != (batch, n, n):
                raise ValueError("chol_nll: A must be (batch, n, n) and y (batch, n)")
            if A.dtype != y.dtype:
                raise TypeError("chol_nll: A and y must share a dtype")
            p = _sfx(A.dtype)
            L = A.detach().contiguous().clone()
            yc = y.detach().contiguous()
            alpha = torch.empty_like(yc)
            logdet = torch.empty(batch, dtype=torch.float64, device=A.device)
            quad = torch.empty_like(logdet)
            info = torch.empty(batch, dtype=torch.int32, device=A.device)
            with _OnHandleStream(handle, L, yc, alpha, logdet, quad, info):
                C.check_status(getattr(C, f"ddla_{p}_chol_nll_batched")(
                    handle.ptr, batch, n, L.data_ptr(), yc.data_ptr(), alpha.data_ptr(), logdet.data_ptr(),
                    quad.data_ptr(), info.data_ptr()), "chol_nll")
            _check_info(info.cpu())
            ctx.save_for_backward(L, alpha)
            ctx.handle = handle
            return (0.5 * (quad + logdet)).to(A.dtype)

        @staticmethod
        def backward(ctx, g):
            L, alpha = ctx.saved_tensors
            handle = ctx.handle
            batch, n = alpha.shape
            p = _sfx(L.dtype)
            W = torch.empty_like(L)
            G = torch.empty_like(L)
            with _OnHandleStream(handle, L, alpha, W, G):
                C.check_status(getattr(C, f"ddla_{p}_chol_nll_grad_batched")(
                    handle.ptr, batch, n, L.data_ptr(), alpha.data_ptr(), W.data_ptr(), G.data_ptr()),
                    "chol_nll backward")
            gd = g.to(L.dtype)
            dA = G * gd[:, None, None] if ctx.needs_input_grad[0] else None
            dy = alpha * gd[:, None] if ctx.needs_input_grad[1] else None
            return dA, dy, None

    class _GPNLL(torch.autograd.Function):
        @staticmethod
        def forward(ctx, X, y, theta, handle):
            batch, n = y.shape
            if X.dim() != 3 or X.shape[:2] != (batch, n):
                raise ValueError("gp_nll: X must be (batch, n, d) and y (batch, n)")
            if X.requires_grad:
                raise ValueError("gp_nll: gradients with respect to the points are not provided")
            p = _sfx(y.dtype)
            d = X.shape[2]
            th = theta.detach().to(torch.float64).contiguous()
            if th.shape == (3,):
                tstride = 0
            elif th.shape == (batch, 3):
                tstride = 3
            else:
                raise ValueError("gp_nll: theta must be (3,) or (batch, 3): (l, sigma_f^2, sigma^2)")
            Xc = X.detach().to(y.dtype).contiguous()
            yc = y.detach().contiguous()
            A = torch.empty(batch, n, n, dtype=y.dtype, device=y.device)
            alpha = torch.empty_like(yc)
            logdet = torch.empty(batch, dtype=torch.float64, device=y.device)
            quad = torch.empty_like(logdet)
            info = torch.empty(batch, dtype=torch.int32, device=y.device)
            with _OnHandleStream(handle, Xc, th, yc, A, alpha, logdet, quad, info):
                C.check_status(getattr(C, f"ddla_{p}_gp_nll_batched")(
                    handle.ptr, batch, n, d, Xc.data_ptr(), th.data_ptr(), tstride, yc.data_ptr(), A.data_ptr(),
                    alpha.data_ptr(), logdet.data_ptr(), quad.data_ptr(), info.data_ptr()), "gp_nll")
            _check_info(info.cpu())
            ctx.save_for_backward(Xc, th, A, alpha)
            ctx.tstride = tstride
            ctx.theta_dtype = theta.dtype
            ctx.handle = handle
            return (0.5 * (quad + logdet)).to(y.dtype)

        @staticmethod
        def backward(ctx, g):
            Xc, th, L, alpha = ctx.saved_tensors
            handle = ctx.handle
            batch, n = alpha.shape
            p = _sfx(L.dtype)
            dtheta = None
            if ctx.needs_input_grad[2]:
                W = torch.empty_like(L)
                grad = torch.empty(batch, 3, dtype=torch.float64, device=L.device)
                with _OnHandleStream(handle, Xc, th, L, alpha, W, grad):
                    C.check_status(getattr(C, f"ddla_{p}_gp_nll_grad_batched")(
                        handle.ptr, batch, n, Xc.shape[2], Xc.data_ptr(), th.data_ptr(), ctx.tstride, L.data_ptr(),
                        alpha.data_ptr(), W.data_ptr(), grad.data_ptr()), "gp_nll backward")
                gt = grad * g.to(torch.float64)[:, None]
                dtheta = (gt.sum(0) if ctx.tstride == 0 else gt).to(ctx.theta_dtype)
            dy = alpha * g.to(alpha.dtype)[:, None] if ctx.needs_input_grad[1] else None
            return None, dy, dtheta, None

    return _CholNLL, _GPNLL


_FUNCS = None


def _funcs():
    global _FUNCS
    if _FUNCS is None:
        _FUNCS = _make_functions()
    return _FUNCS


def chol_nll(A, y, handle=None):
    """Per-problem loss 1/2 (y^T A^-1 y + log det A); A (batch, n, n), y (batch, n), CUDA tensors."""
    return _funcs()[0].apply(A, y, handle or default_handle())


def gp_nll(X, y, theta, handle=None):
    """Per-problem GP loss with A = K(theta) + sigma^2 I built on the device.
    X (batch, n, d) points, y (batch, n), theta (3,) shared or (batch, 3)."""
    return _funcs()[1].apply(X, y, theta, handle or default_handle())
