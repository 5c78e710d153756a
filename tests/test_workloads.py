"""The bench's seeded synthetic inputs have the properties their formulas state
(small sizes, torch on the CPU device): the Householder family A = U diag(s) U^T
is symmetric with exactly the geometric spectrum 1 ... 1/kappa (so kappa(A) =
kappa), the Gram and SE-kernel families are symmetric / Hermitian positive
definite with the stated lower bounds, and equal seeds give equal matrices."""
import numpy as np
import pytest

from libddla_b200 import workloads as W


@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
def test_householder_family_spectrum(kappa):
    n = 96
    s = np.sort(float(kappa) ** (-np.arange(n) / (n - 1)))
    for A in (W.householder_spd(n, kappa, 0xDD1A0003, device="cpu").numpy(),
              W.householder_spd_host(n, kappa, 0xDD1A0003)):
        assert np.allclose(A, A.T, rtol=0, atol=1e-15)
        ev = np.linalg.eigvalsh(A)
        assert np.allclose(ev, s, rtol=1e-9, atol=1e-13), (kappa, ev[:3], s[:3])
        assert abs(ev[-1] / ev[0] / kappa - 1) < 1e-4
    # the reference arm's full-size generator: the same matrix, lower triangle only
    Lw = W.householder_spd_host_lower(n, kappa, 0xDD1A0003)
    assert Lw.flags.f_contiguous and not np.triu(Lw, 1).any()
    Af = W.householder_spd_host(n, kappa, 0xDD1A0003)
    assert np.allclose(np.tril(Af), Lw, rtol=0, atol=1e-15)
    a = W.householder_spd(n, kappa, 7, device="cpu")
    assert bool((a == W.householder_spd(n, kappa, 7, device="cpu")).all())


def test_gram_and_kernel_families():
    import torch

    A = W.gram_plus_identity(64, 3, device="cpu").numpy()
    assert np.allclose(A, A.T) and np.linalg.eigvalsh(A).min() >= 1 - 1e-12
    K = W.se_kernel(80, 4, device="cpu").numpy()
    assert np.allclose(K, K.T) and np.linalg.eigvalsh(K).min() >= 1e-2 - 1e-10
    Kz = W.se_kernel(80, 4, complex_=True, device="cpu").numpy()
    assert np.allclose(Kz, np.conj(Kz).T) and np.linalg.eigvalsh(Kz).min() >= 1e-2 - 1e-10
    assert np.allclose(np.abs(Kz), K, atol=1e-12)  # the phase factor has modulus 1
    sizes = W.batched_sizes(4096, 0xDD1A0004)
    assert sizes.min() >= 16 and sizes.max() <= 512 and len(sizes) == 4096
    x = W.gp_points(10, 5, device="cpu")
    assert x.shape == (10, 2) and bool(((x >= 0) & (x <= 1)).all())
    assert torch.equal(x, W.gp_points(10, 5, device="cpu"))


@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
def test_householder_exact_inverse(kappa):
    """householder_solve applies A^-1 = U diag(1/s) U^T from the reflectors: it agrees with a dense
    solve of the generated A to the accuracy the conditioning allows, and A X reproduces B."""
    import torch

    n = 160
    A = W.householder_spd(n, kappa, 11, device="cpu")
    s, vs = W.householder_factors(n, kappa, 11, device="cpu")
    B = torch.randn(n, 4, generator=torch.Generator().manual_seed(2), dtype=torch.float64)
    X = W.householder_solve(s, vs, B)
    eps = np.finfo(np.float64).eps
    assert float((A @ X - B).abs().max()) <= 50 * n * eps * float(A.abs().sum(0).max()) * float(X.abs().max())
    Xd = torch.linalg.solve(A, B)
    assert float((X - Xd).abs().max() / X.abs().max()) <= 10 * kappa * n * eps
