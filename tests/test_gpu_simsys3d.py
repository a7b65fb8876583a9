"""The 3D simsys interface (system_assemble_3d, system_adjust_matrix_3d,
system_solve_3d, system_get_3d; simsys_spkaux.f90:495-716) on the GPU
against the oracle's restatement of the reference's 3D COO: the assembled
FP64 matrix equals the reference's call-order sum bit for bit, entry for
entry in the order of c3coo (coo_init_new and loccoo3d, coo_matrix.f90), and
the solution matches the ILUT+BiCGStab solve of the same system to the
solver's tolerance.  The element blocks are those of a non-hydrostatic
pressure system: negative definite, symmetric, a horizontal Laplacian per
layer and couplings to the layers above and below."""
import numpy as np
import pytest

import shygpu
import shyref
from shygpu import cases

pytestmark = pytest.mark.gpu


def blocks(case, nlv, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for ie in range(case["nel"]):
        for l in range(1, nlv + 1):
            if rng.uniform() < 0.1:                    # some element layers left out
                continue
            m = np.zeros((3, 3, 3), np.float32)
            a = rng.uniform(0.1, 1.0, (3, 3))
            m[1] = -0.5 * (a + a.T)
            for i in range(3):
                m[1, i, i] = -3.0 - rng.uniform(0.0, 1.0)
                if l > 1:
                    m[0, i, i] = rng.uniform(0.1, 0.5)
                if l < nlv:
                    m[2, i, i] = rng.uniform(0.1, 0.5)
            out.append((ie + 1, l, m, rng.uniform(-1, 1, 3).astype(np.float32)))
    return out


@pytest.mark.parametrize("nlv", [1, 6])
def test_simsys_3d_assembly_and_solve(nlv):
    c = cases.seiche_case(nx=21, ny=9, nlv=nlv)
    nkn, nel = c["nkn"], c["nel"]
    S = shygpu.simsys
    S.register(nkn, nel, c["nen3v"])
    S.set_layers(nlv)
    S.system_initialize()
    S.system_init()
    o = shyref.System3D(nkn, nel, nlv, c["nen3v"])
    for ie, l, m, r in blocks(c, nlv):
        S.system_assemble_3d(ie, l, nlv, c["nen3v"][ie - 1], m, r)
        o.assemble(ie, l, m, r)
    S.system_adjust_matrix_3d()
    o.adjust()
    S.system_solve_3d(np.zeros((nkn, nlv), np.float32))
    z = S.system_get_3d(nkn, nlv)
    ia, ja, val, rhs = o.matrix()
    rowptr, col, gval, grhs = S.get_matrix_3d()
    assert np.array_equal(rowptr, ia) and np.array_equal(col, ja)
    assert np.array_equal(gval, val) and np.array_equal(grhs, rhs)
    zo, _ = o.solve(np.zeros((nkn, nlv)))
    assert np.abs(z - zo).max() <= 1e-5 * np.abs(zo).max()
    # the returned x meets the reference's stop test in FP64
    n = (nlv + 2) * nkn
    x = np.zeros(n)
    for k in range(nkn):
        x[k * (nlv + 2) + 1:k * (nlv + 2) + nlv + 1] = z[k]
    A = np.zeros((n, n))
    for r in range(n):
        A[r, ja[ia[r]:ia[r + 1]]] += val[ia[r]:ia[r + 1]]
    assert np.linalg.norm(A @ x - rhs) <= 1e-5 * np.linalg.norm(rhs)
    assert S.iterations() > 0
    # a second solve with the solution as the guess keeps it
    S.system_solve_3d(z)
    assert np.abs(S.system_get_3d(nkn, nlv) - zo).max() <= 1e-5 * np.abs(zo).max()
