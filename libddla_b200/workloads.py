"""Seeded synthetic inputs of the benchmark configurations (device side via torch, host side via NumPy).

No public dataset is involved; every matrix is defined by a formula and a seed:
  gram_plus_identity   A = G G^T / n + I, G iid N(0,1)                (plain ppotrf+ppotrs, n=2048)
  se_kernel            A = K + 1e-2 I, squared-exponential kernel on points in [0,1]^3,
                       complex variant K * exp(i k.(x-y)), k ~ N(0, I3) (pposv d/z, n=16384)
  householder_spd      A = U diag(s) U^T, U = H1 H2 H3 H4 Householder reflectors with
                       N(0,1) vectors, s geometric from 1 to 1/kappa     (mixed pposv, n=32768)
  batched_gram         A_i = G_i G_i^T / n_i + 0.1 I, n_i uniform in [16, 512]
  gp_points / se_gram  SE kernel on points in [0,1]^2 (lengthscale 0.3) + sigma^2 I (GP likelihood)
"""
from __future__ import annotations

import numpy as np

SEED_BASE = 0xDD1A0000


def _torch():
    import torch

    return torch


def gram_plus_identity(n: int, seed: int, device="cuda", dtype=None):
    torch = _torch()
    dtype = dtype or torch.float64
    g = torch.Generator(device=device).manual_seed(seed)
    G = torch.randn(n, n, generator=g, device=device, dtype=dtype)
    A = G @ G.T / n
    A.diagonal().add_(1.0)
    return A


def se_kernel(n: int, seed: int, lengthscale=0.2, nugget=1e-2, complex_=False, device="cuda"):
    torch = _torch()
    g = torch.Generator(device=device).manual_seed(seed)
    x = torch.rand(n, 3, generator=g, device=device, dtype=torch.float64)
    d2 = torch.cdist(x, x).square_()
    K = torch.exp(-d2 / (2 * lengthscale ** 2))
    del d2
    if complex_:
        k = torch.randn(3, generator=g, device=device, dtype=torch.float64)
        ph = x @ k
        K = K * torch.exp(1j * (ph[:, None] - ph[None, :]))
    K.diagonal().add_(nugget)
    return K


def householder_factors(n: int, kappa: float, seed: int, device="cuda"):
    """(s, [v1, v2, v3, v4]) of householder_spd: the spectrum and the reflector vectors."""
    torch = _torch()
    g = torch.Generator(device=device).manual_seed(seed)
    s = torch.pow(torch.tensor(float(kappa), dtype=torch.float64, device=device),
                  -torch.arange(n, device=device, dtype=torch.float64) / max(1, n - 1))
    vs = [torch.randn(n, generator=g, device=device, dtype=torch.float64) for _ in range(4)]
    return s, vs


def householder_solve(s, vs, B):
    """A^-1 B = U diag(1/s) U^T B for A = U diag(s) U^T, U = H1 H2 H3 H4 (each H = I - 2 v v^T / v^T v
    symmetric), applied reflector by reflector: O(n nrhs) work, the exact inverse up to rounding.
    B: n x nrhs (torch, float64)."""
    def refl(v, X):
        return X - (2.0 / float(v @ v)) * torch_outer(v, v @ X)

    torch_outer = lambda v, w: v[:, None] * w[None, :]
    Y = B
    for v in vs:  # U^T B = H4 H3 H2 H1 B: H1 first
        Y = refl(v, Y)
    Y = Y / s[:, None]
    for v in reversed(vs):  # U Y = H1 H2 H3 H4 Y: H4 first
        Y = refl(v, Y)
    return Y


def householder_spd(n: int, kappa: float, seed: int, device="cuda"):
    """A = H1 H2 H3 H4 diag(s) H4 H3 H2 H1 built in place with rank-one updates (torch.addr_)."""
    torch = _torch()
    s, vs = householder_factors(n, kappa, seed, device=device)
    A = torch.diag(s)
    for v in reversed(vs):
        beta = 2.0 / float(v @ v)
        w = A @ v
        c = float(v @ w)
        A.addr_(v, w, alpha=-beta)
        A.addr_(w, v, alpha=-beta)
        A.addr_(v, v, alpha=beta * beta * c)
    return A


def householder_spd_host(n: int, kappa: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    s = float(kappa) ** (-np.arange(n) / max(1, n - 1))
    A = np.diag(s)
    vs = [rng.standard_normal(n) for _ in range(4)]
    for v in reversed(vs):
        beta = 2.0 / (v @ v)
        w = A @ v
        c = v @ w
        A -= beta * (np.outer(v, w) + np.outer(w, v))
        A += beta * beta * c * np.outer(v, v)
    return A


def householder_spd_host_lower(n: int, kappa: float, seed: int) -> np.ndarray:
    """The same family as householder_spd_host, column-major, with only the lower triangle
    defined (the upper one is zero): each reflector is one symmetric matrix-vector product
    and one symmetric rank-2 update, H A H = A - beta (v w'^T + w' v^T) with w = A v and
    w' = w - (beta v^T w / 2) v, through the multithreaded BLAS, so that full-size
    matrices (n = 32768, 8.6 GB) take seconds and no n x n temporaries."""
    import scipy.linalg.blas as blas

    rng = np.random.default_rng(seed)
    s = float(kappa) ** (-np.arange(n) / max(1, n - 1))
    A = np.zeros((n, n), dtype=np.float64, order="F")
    A[np.arange(n), np.arange(n)] = s
    vs = [rng.standard_normal(n) for _ in range(4)]
    for v in reversed(vs):
        beta = 2.0 / float(v @ v)
        w = blas.dsymv(1.0, A, v, lower=1)
        w = w - (0.5 * beta * float(v @ w)) * v
        A = blas.dsyr2(-beta, v, w, lower=1, a=A, overwrite_a=1)
    return A


def batched_sizes(count: int, seed: int, lo=16, hi=512) -> np.ndarray:
    return np.random.default_rng(seed).integers(lo, hi + 1, size=count)


def gp_points(n: int, seed: int, device="cuda", dim=2):
    torch = _torch()
    g = torch.Generator(device=device).manual_seed(seed)
    return torch.rand(n, dim, generator=g, device=device, dtype=torch.float64)
