"""Pins the oracle's tridiagonal solver (a restatement of LAPACK dgtsv, the
third-party routine on the Crank-Nicolson path, src/Diffusion.F90:881-890)
against SciPy's LAPACK dgtsv, on the committed fixtures and on fresh seeded
systems: diagonally dominant ones (the only kind the path produces) and
general ones that exercise the row-interchange branch."""
import json
import pathlib

import numpy as np
import pytest

GOLD = pathlib.Path(__file__).parent / "golden" / "dgtsv_cases.json"


def _scipy_dgtsv(dl, d, du, b):
    from scipy.linalg import lapack
    _, _, _, x, info = lapack.dgtsv(np.array(dl), np.array(d), np.array(du), np.array(b))
    return x, info


def test_golden_fixture_matches_oracle(oracle_mod):
    cases = json.loads(GOLD.read_text())
    assert len(cases) >= 10
    for c in cases:
        x, info = oracle_mod.dgtsv(c["dl"], c["d"], c["du"], c["b"])
        assert info == c["info"]
        want = np.array([float.fromhex(h) for h in c["x_hex"]])
        assert np.array_equal(x, want), c["name"]


@pytest.mark.parametrize("seed", range(20))
def test_diag_dominant_bitwise(oracle_mod, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 400))
    L = rng.uniform(0, 2.0, n)
    R = rng.uniform(0, 2.0, n)
    imp = 0.5
    d = 1.0 + imp * (L + R)
    dl = -(imp * L[1:])
    du = -(imp * R[:-1])
    b = rng.uniform(-1, 1, n) * 10.0 ** rng.uniform(-8, 3, n)
    x, info = oracle_mod.dgtsv(dl, d, du, b)
    xs, infos = _scipy_dgtsv(dl, d, du, b)
    assert info == 0 and infos == 0
    assert np.array_equal(x, xs)


@pytest.mark.parametrize("seed", range(10))
def test_general_with_pivoting(oracle_mod, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(2, 60))
    d = rng.uniform(-1, 1, n)
    dl = rng.uniform(-3, 3, n - 1)
    du = rng.uniform(-1, 1, n - 1)
    b = rng.uniform(-1, 1, n)
    x, info = oracle_mod.dgtsv(dl, d, du, b)
    xs, infos = _scipy_dgtsv(dl, d, du, b)
    assert info == infos
    if info == 0:
        assert np.array_equal(x, xs)


def test_edge_sizes(oracle_mod):
    x, info = oracle_mod.dgtsv([], [4.0], [], [2.0])
    assert info == 0 and x[0] == 0.5
    x, info = oracle_mod.dgtsv([], [], [], [])
    assert info == 0
    x, info = oracle_mod.dgtsv([1.0], [0.0, 1.0], [1.0], [1.0, 1.0])  # interchange at row 1
    xs, infos = _scipy_dgtsv([1.0], [0.0, 1.0], [1.0], [1.0, 1.0])
    assert info == infos
