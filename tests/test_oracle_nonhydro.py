"""The oracle's non-hydrostatic pressure (nohydro.f90: sp256wnh,
nonhydro_prepare_matrix, nonhydro_correct_uveta; the 3D system of
coo_matrix.f90 and simsys_spkaux.f90) pinned to the analytic dispersion of
surface gravity waves.

A standing wave of wavenumber k in water of depth H oscillates with
omega^2 = g k tanh(k H); the hydrostatic equations give omega = k sqrt(g H).
In a closed 50 m basin 25 m deep (k H = pi/2) the two periods are 8.36 s and
6.39 s.  The oracle's hydrostatic run keeps the shallow-water period within
0.5%; with inohyd = 1 the period moves to the non-hydrostatic one and
converges to it as the layers are refined (first order in the layer
thickness: 7.80, 8.07, 8.22 s at 5, 10 and 20 layers).  The 3D system is
checked against the reference's layout: the COO positions of loccoo3d, the
unit diagonals of coo_adjust_3d and a solution that satisfies the system.
"""
import math

import numpy as np
import pytest

import shyref
from shygpu import cases

G, H, L = 9.81, 25.0, 50.0
K = math.pi / L
T_HYDRO = 2 * math.pi / (K * math.sqrt(G * H))
T_NONHYDRO = 2 * math.pi / math.sqrt(G * K * math.tanh(K * H))


def seiche_period(case, nsteps=300):
    o = shyref.OracleModel(case)
    k0 = int(np.argmin(case["xgv"]))
    z = [float(case["znv"][k0])]
    for _ in range(nsteps):
        o.run(1)
        z.append(float(o.state()["znv"][k0]))
    z = np.array(z)
    dt = case["params"]["dt"]
    cross = [(i + z[i] / (z[i] - z[i + 1])) * dt for i in range(len(z) - 1) if z[i] * z[i + 1] < 0]
    assert len(cross) >= 4
    return 2 * float(np.mean(np.diff(cross))), o


def test_hydrostatic_seiche_has_the_shallow_water_period():
    T, _ = seiche_period(cases.seiche_case(inohyd=0))
    assert abs(T - T_HYDRO) <= 0.005 * T_HYDRO


def test_nonhydrostatic_seiche_converges_to_the_dispersion_relation():
    errs = []
    for nlv in (5, 10, 20):
        T, o = seiche_period(cases.seiche_case(inohyd=1, nlv=nlv))
        errs.append(abs(T - T_NONHYDRO) / T_NONHYDRO)
        q, w, (iters, r0, r) = o.nh()
        assert iters > 0 and r <= 1e-8 * r0 + 1e-8
        assert np.abs(q[:, 0]).max() == 0.0          # nonhydro_adjust zeroes the first layer
    assert errs[-1] <= 0.02
    assert errs[0] > errs[1] > errs[2]
    assert 1.6 <= errs[1] / errs[2] <= 2.5           # first order in the layer thickness
    assert abs(T - T_HYDRO) > 0.2 * T_HYDRO


def test_still_water_stays_still_nonhydrostatic():
    c = cases.seiche_case(inohyd=1, ampli=0.0)
    o = shyref.OracleModel(c)
    o.run(20)
    s = o.state()
    assert np.abs(s["znv"]).max() == 0.0
    assert np.abs(s["utlnv"]).max() == 0.0
    q, w, _ = o.nh()
    assert np.abs(q).max() == 0.0 and np.abs(w).max() == 0.0


def test_3d_system_layout_and_solution():
    """loccoo3d's positions, coo_adjust_3d's unit diagonals and the solve."""
    c = cases.seiche_case(nx=6, ny=3, nlv=4)
    nkn, nel, nlv = c["nkn"], c["nel"], c["nlv"]
    s = shyref.System3D(nkn, nel, nlv, c["nen3v"])
    rng = np.random.default_rng(3)
    ntg, icol, _ = shyref.coo_init(c)
    for ie in range(1, nel + 1):
        for l in range(1, nlv):                        # the last layer left out: adjust fills it
            m = np.zeros((3, 3, 3), np.float32)
            m[1] = -rng.uniform(0.1, 1.0, (3, 3))
            m[1] = 0.5 * (m[1] + m[1].T)
            for i in range(3):
                m[1, i, i] -= 3.0
                m[0, i, i] = rng.uniform(0.1, 0.5)
                m[2, i, i] = rng.uniform(0.1, 0.5)
            s.assemble(ie, l, m, rng.uniform(-1, 1, 3).astype(np.float32))
    s.adjust()
    ia, ja, val, rhs = s.matrix()
    n = (nlv + 2) * nkn
    assert ia[-1] == val.size == ntg[-1] * nlv + 2 * nlv * nkn + 2 * nkn
    for k in range(nkn):
        ng = ntg[k + 1] - ntg[k]
        r0 = k * (nlv + 2)
        assert ia[r0 + 1] - ia[r0] == 1 and val[ia[r0]] == 1.0            # padding rows
        assert ia[r0 + nlv + 2] - ia[r0 + nlv + 1] == 1 and val[ia[r0 + nlv + 1]] == 1.0
        for l in range(1, nlv + 1):
            row = ja[ia[r0 + l]:ia[r0 + l + 1]]
            assert row.size == ng + 2 and np.all(np.diff(row) > 0)
            diag = val[ia[r0 + l]:ia[r0 + l + 1]][list(row).index(r0 + l)]
            assert diag != 0.0
        last = val[ia[r0 + nlv]:ia[r0 + nlv + 1]][list(ja[ia[r0 + nlv]:ia[r0 + nlv + 1]]).index(r0 + nlv)]
        assert last == 1.0                              # no element reached layer nlv
    z, iters = s.solve(np.zeros((nkn, nlv)))
    A = np.zeros((n, n))
    for r in range(n):
        A[r, ja[ia[r]:ia[r + 1]]] += val[ia[r]:ia[r + 1]]
    x = np.zeros(n)
    for k in range(nkn):
        x[k * (nlv + 2) + 1:k * (nlv + 2) + nlv + 1] = z[k]
    assert np.linalg.norm(A @ x - rhs) <= 1e-8 * np.linalg.norm(rhs) + 1e-8
    assert np.allclose(x, np.linalg.solve(A, rhs), rtol=0, atol=1e-7 * np.abs(x).max())


def test_refused_with_wetting_and_drying():
    c = cases.seiche_case(inohyd=1)
    c["params"] = dict(c["params"], wetdry=1)
    with pytest.raises(RuntimeError, match="non-hydrostatic"):
        shyref.OracleModel(c)
