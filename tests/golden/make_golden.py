"""Write the golden fixtures under tests/golden/ (run once; outputs are committed).

    python tests/golden/make_golden.py

Each fixture holds inputs and the known answers of the reference's own tests
(generators.py restates the formulas with file:line citations):
  kat.npz        A = L L^H from the analytic factor, for n in {1, 2, 17, 38, 129}, all four types
  real_spd.npz   spd_value A, X_true, B = A X_true (test_ppotrf_real.cpp), n in {16, 40}, s and d
  hpd.npz        hpd_value A, X_true, B (test_api_grid_ppotrf.cpp), n in {1, 24}, z
  logdet.npz     diag_logdet diagonals and the long-double-style expected result per case
  python.npz     the seeded cases of python/tests/test_cholesky.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import generators as G  # noqa: E402


def main():
    kat = {}
    for p, dt in G.DTYPES.items():
        for n in (1, 2, 17, 38, 129):
            kat[f"{p}_{n}_A"] = G.kat_matrix(n, dt)
            kat[f"{p}_{n}_L"] = G.kat_factor(n, dt)
    np.savez_compressed(HERE / "kat.npz", **kat)

    real = {}
    for p in "sd":
        dt = G.DTYPES[p]
        for n in (16, 40):
            A = G.spd_value(n, dt)
            X = G.x_value_real(n, 3, dt)
            real[f"{p}_{n}_A"] = A
            real[f"{p}_{n}_X"] = X
            real[f"{p}_{n}_B"] = G.rhs_sequential(A, X)
    np.savez_compressed(HERE / "real_spd.npz", **real)

    hpd = {}
    for n in (1, 24):
        A = G.hpd_value(n) if n > 1 else np.array([[4.0 + 0j]])
        X = G.x_value(n, 3)
        hpd[f"z_{n}_A"] = A
        hpd[f"z_{n}_X"] = X
        hpd[f"z_{n}_B"] = G.rhs_sequential(A, X)
    np.savez_compressed(HERE / "hpd.npz", **hpd)

    ld = {}
    for p, dt in G.DTYPES.items():
        for k, diag in enumerate(G.logdet_cases(dt)):
            d = np.array(diag, dtype=dt)
            ref = G.logdet_reference(diag)
            ld[f"{p}_{k}_diag"] = d
            ld[f"{p}_{k}_expect"] = (np.array([np.nan, np.nan]) if ref is None
                                     else np.array([ref.real, ref.imag]))
            ld[f"{p}_{k}_valid"] = np.array(ref is not None)
    np.savez_compressed(HERE / "logdet.npz", **ld)

    py = G.python_cases()
    out = {"ppotrf_ppotrs_A": py["ppotrf_ppotrs"][0], "ppotrf_ppotrs_X": py["ppotrf_ppotrs"][1],
           "pposv_A": py["pposv"][0], "pposv_X": py["pposv"][1]}
    for k, (ch, uplo, A, X, B) in enumerate(py["typed"]):
        out[f"typed_{k}_{ch}_{uplo}_A"] = A
        out[f"typed_{k}_{ch}_{uplo}_X"] = X
        out[f"typed_{k}_{ch}_{uplo}_B"] = B
    np.savez_compressed(HERE / "python.npz", **out)
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
