"""Generates dgtsv_cases.json: seeded tridiagonal systems solved by SciPy's
LAPACK dgtsv (the routine the reference links for Crank-Nicolson,
src/Diffusion.F90:881-890).  Solutions are stored as float.hex strings.

    python tests/golden/make_dgtsv_cases.py
"""
import json
import pathlib

import numpy as np
from scipy.linalg import lapack


def main():
    rng = np.random.default_rng(20240601)
    cases = []
    for t in range(16):
        n = int(rng.integers(2, 80))
        if t < 10:  # Crank-Nicolson shaped: D = 1 + 0.5(L+R), off-diagonals -0.5L / -0.5R
            L = rng.uniform(0, 3.0, n)
            R = rng.uniform(0, 3.0, n)
            d = 1.0 + 0.5 * (L + R)
            dl = -(0.5 * L[1:])
            du = -(0.5 * R[:-1])
        else:  # general: pivoting branch
            d = rng.uniform(-1, 1, n)
            dl = rng.uniform(-3, 3, n - 1)
            du = rng.uniform(-1, 1, n - 1)
        b = rng.uniform(-1, 1, n)
        _, _, _, x, info = lapack.dgtsv(dl.copy(), d.copy(), du.copy(), b.copy())
        cases.append(dict(name=f"case{t}", dl=dl.tolist(), d=d.tolist(), du=du.tolist(), b=b.tolist(),
                          info=int(info), x_hex=[float(v).hex() for v in x]))
    out = pathlib.Path(__file__).parent / "dgtsv_cases.json"
    out.write_text(json.dumps(cases))
    print(f"wrote {len(cases)} cases to {out}")


if __name__ == "__main__":
    main()
