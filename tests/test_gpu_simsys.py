"""The simsys drop-in (system_initialize ... system_get) against the oracle:
the assembled FP64 matrix equals the reference's element-order COO sum bit
for bit, and the solution matches the ILUT+BiCGStab solve of the same
system to the solver tolerance."""
import numpy as np
import pytest

import shygpu
import shyref

pytestmark = pytest.mark.gpu


def element_systems(case, seed=3):
    """Element matrices and rhs like hydro_zeta builds them (random layer
    sums and transports), with a few Dirichlet nodes, in single precision."""
    ev = shyref.set_ev(case)
    rng = np.random.default_rng(seed)
    nel = case["nel"]
    flag = shyref.FLAG
    dirich = np.full(case["nkn"], flag)
    dirich[case["bnd_index"] > 0] = 0.3
    hias, hiks = [], []
    for ie in range(nel):
        kn = case["nen3v"][ie] - 1
        hia = np.zeros(9)
        hik = np.zeros(3)
        shyref.lib.shyref_element_system(
            shyref.dptr(np.ascontiguousarray(ev[ie])), shyref.dptr(rng.uniform(-0.2, 0.2, 3)),
            rng.uniform(5, 15), 0.0, 0.0, rng.uniform(5, 15), rng.uniform(-1, 1), rng.uniform(-1, 1),
            shyref.dptr(np.ascontiguousarray(dirich[kn])), 60.0, 0.5, 0.5, 9.81,
            shyref.dptr(hia), shyref.dptr(hik))
        hias.append(hia.reshape(3, 3).T.astype(np.float32))      # hia[n, m]
        hiks.append(hik.astype(np.float32))
    return hias, hiks


def test_simsys_assembly_and_solve(channel):
    nkn, nel = channel["nkn"], channel["nel"]
    hias, hiks = element_systems(channel)
    S = shygpu.simsys
    S.register(nkn, nel, channel["nen3v"])
    S.system_initialize()
    S.system_init()
    for ie in range(nel):
        S.system_assemble(ie + 1, channel["nen3v"][ie], hias[ie], hiks[ie])
    rqv = np.zeros(nkn, np.float32)
    S.system_add_rhs(60.0, rqv)
    z0 = np.zeros(nkn, np.float32)
    S.system_solve(z0)
    z = S.system_get(nkn)
    ntg, icol, ijp = shyref.coo_init(channel)
    rowptr, col, val, rhs = S.get_matrix(nkn, int(ntg[-1]))
    assert np.array_equal(rowptr, ntg) and np.array_equal(col, icol)
    # the reference's serial assembly: c2coo(ijp) += hia(i,j), element order, FP64
    c2 = np.zeros(ntg[-1])
    rv = np.zeros(nkn)
    for ie in range(nel):
        for i in range(3):
            for j in range(3):
                c2[ijp[ie, i, j]] += np.float64(hias[ie][i, j])
            rv[channel["nen3v"][ie, i] - 1] += np.float64(hiks[ie][i])
    assert np.array_equal(val, c2)
    assert np.array_equal(rhs, rv)
    x, it, r0, r = shyref.spk_solve(ntg, icol, c2, rv, z0.astype(np.float64))
    assert np.abs(z - x).max() <= 1e-5 * max(1.0, np.abs(x).max())
