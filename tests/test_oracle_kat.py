"""The oracle against the reference's own known-answer tests.

* penta_example_1/2, tri_example_1 (src/external/sparskit/penta.f90:376-481):
  systems whose exact solution is 1..n.
* test_random (penta.f90:508-581): random diagonally dominant band systems,
  checked through band_multiply against the known solution.
* rhotst (src/shyfem/eq_state.f90:60-110): UNESCO densities `rhoref`.
* coo_test (src/shyfem/coo_util.f90:246-285): the sorted node-neighbour
  pattern of a small mesh.
"""
import numpy as np
import pytest

import shyref

D = [1, 2, 3, -4, 5, 6, 7, -1, 1, 8]
U1 = [2, 2, 1, 5, -7, 3, -1, 4, 5, 0]
U2 = [1, 5, -2, 1, 5, 2, 4, -3, 0, 0]
L1 = [0, 3, 2, 1, 2, 1, 2, 1, -2, 4]
L2 = [0, 0, 1, 3, 1, 5, 2, 2, 2, -1]
R = [8, 33, 8, 24, 29, 98, 99, 17, 57, 108]
T = np.arange(1, 11, dtype=float)


@pytest.mark.parametrize("fast", [False, True])
def test_penta_example_2(fast):
    val = np.array([L2, L1, D, U1, U2], float).T       # val(-2:2, n) row-banded
    s = shyref.penta_solve(shyref.penta_fact(val, fast=fast), R)
    assert np.sqrt(np.mean((s - T) ** 2)) < 1e-12


def test_tri_example_1():
    v = np.array([[0, 1, 2], [3, 4, 0]], float)        # lower, centre, upper
    s = shyref.tria_multi(v, np.array([[5, 11]], float))
    assert np.allclose(s[0], [1, 2], atol=1e-14)


def band_multiply(val, s, m):
    n = len(s)
    r = np.zeros(n)
    for i in range(n):
        for j in range(max(-m, -i), min(m, n - 1 - i) + 1):
            r[i] += val[i, j + m] * s[i + j]
    return r


@pytest.mark.parametrize("m", [1, 2])
def test_random_band(m):
    rng = np.random.default_rng(7)
    ssmax = 0.0
    for _ in range(300):
        n = int(rng.integers(2 * m, 21))
        val = rng.uniform(-1, 1, (n, 2 * m + 1))
        val[:, m] = np.abs(val).sum(axis=1) * rng.choice([-1, 1], n)
        s = rng.uniform(-1, 1, n)
        r = band_multiply(val, s, m)
        if m == 2:
            x = shyref.penta_solve(shyref.penta_fact(val, fast=True), r)
        else:
            x = shyref.tria_multi(val, r[None, :])[0]
        ssmax = max(ssmax, np.sqrt(np.mean((x - s) ** 2)))
    assert ssmax < 1e-12


RHOREF = [999.96675, 1044.12802, 997.04796, 1037.90204,
          1027.67547, 1069.48914, 1023.34306, 1062.53817]


def test_rhotst():
    i = 0
    for s in (0.0, 35.0):
        for t in (5.0, 25.0):
            for p in (0.0, 1000.0):
                rho = shyref.sigma_stp(s, t, p) + 1000.0
                assert abs(rho - RHOREF[i]) < 2e-5, (s, t, p, rho)
                i += 1


def test_coo_pattern():
    # two triangles sharing an edge plus one more: rows are sorted neighbour
    # lists with the diagonal, ijp points every element entry at its slot
    case = dict(nkn=5, nel=3, nen3v=np.array([[1, 2, 3], [1, 3, 4], [3, 5, 4]], np.int32))
    ntg, icol, ijp = shyref.coo_init(case)
    rows = [list(icol[ntg[k]:ntg[k + 1]]) for k in range(5)]
    assert rows == [[0, 1, 2, 3], [0, 1, 2], [0, 1, 2, 3, 4], [0, 2, 3, 4], [2, 3, 4]]
    for ie in range(3):
        for i in range(3):
            for j in range(3):
                ki, kj = case["nen3v"][ie, i] - 1, case["nen3v"][ie, j] - 1
                slot = ijp[ie, i, j]
                assert ntg[ki] <= slot < ntg[ki + 1] and icol[slot] == kj
