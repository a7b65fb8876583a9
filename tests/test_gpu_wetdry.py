"""Wetting and drying on the GPU against the oracle (wetdry.f90,
topo_update.f90, hydrodynamic.f90:374-404): a tidal flat through a full M2
cycle, in which the flat dries at low water and floods again.

The dry set is decided by thresholds on the solved levels (hzoff, hzmin,
hzon).  Levels agree to the solver tolerance (a few micrometres), so the
runs take the same decisions step for step until a vertex's total depth
lands within that distance of a threshold; there one run may take an
element out or back a step before the other.  The test follows both runs
step by step: up to the first differing decision the dry marks, their
counters and the node kinds must be equal and the levels within ZETA_TOL;
that first difference must sit at such a tie (a vertex within TIE of a
threshold).  One decision a step apart moves the flooding front and, over
the flat, the decisions after it: from there on the levels may differ by
centimetres at the front (FRONT_TOL) and a few dry marks (DRY_DIFF), while
the volume stays within 1e-4."""
import numpy as np
import pytest

import shygpu
import shyref
from shygpu import cases

pytestmark = pytest.mark.gpu

ZETA_TOL = 1.0e-3          # m, on nodes in the system in both runs
TIE = 1.0e-4               # m, a threshold tie: far above the solver tolerance
FRONT_TOL = 0.1            # m, after a tie: the front shifted by a step or more
DRY_DIFF = 0.02            # fraction of the elements whose dry mark may differ after a tie


def levels(g, o):
    return g.get_state(0)["znv"].astype(np.float64), o.state()["znv"]


def at_a_tie(c, e, zs):
    """Whether element e has a vertex (or, for the mean-depth rule, a mean)
    within TIE of hzoff, hzmin or hzon in any of the level sets zs."""
    p = cases_params(c)
    hm = c["hm3v"][e].astype(np.float64)
    kn = c["nen3v"][e] - 1
    thr = np.array([p["hzoff"], p["hzmin"], p["hzon"]])
    for z in zs:
        hz = z[kn] + hm
        d = np.abs(np.r_[hz, hz.mean()][:, None] - thr[None, :])
        if d.min() <= TIE:
            return True
    return False


def cases_params(c):
    p = dict(hzmin=0.01, hzoff=0.05, hzon=0.10)
    p.update({k: v for k, v in c.get("params", {}).items() if k in p})
    return p


@pytest.mark.parametrize("nlv", [1, 4])
def test_tidal_flat_dries_and_floods(nlv):
    """One M2 period (750 steps of 60 s), compared after every step."""
    c = cases.flat_case(nlv=nlv)
    g = shygpu.Model(c)
    g.set_state(0)
    o = shyref.OracleModel(c)
    gw, ow = g.wetdry(0), o.wetdry()
    np.testing.assert_array_equal(gw[0], ow[0])          # setweg(0) of the initial state
    np.testing.assert_array_equal(gw[1], ow[1])
    zg, zo = levels(g, o)
    first_tie, ndry = None, []
    for step in range(1, 751):
        zg0, zo0 = zg, zo
        g.run(1)
        o.run(1)
        gw, ow = g.wetdry(0), o.wetdry()
        zg, zo = levels(g, o)
        ndry.append(int((ow[0] > 0).sum()))
        wet = (gw[2] != -2) & (ow[2] != -2)
        dz = np.abs(zg - zo)[wet].max()
        differ = np.nonzero((gw[0] != ow[0]) | (gw[1] != ow[1]))[0]
        if first_tie is None and len(differ):
            for e in differ:
                assert at_a_tie(c, e, (zg0, zo0, zg, zo)), (step, e)
            first_tie = step
        if first_tie is None:
            np.testing.assert_array_equal(gw[2], ow[2])
            assert dz <= ZETA_TOL, (step, dz)
        else:
            assert ((gw[0] > 0) != (ow[0] > 0)).sum() <= DRY_DIFF * c["nel"], step
            assert dz <= FRONT_TOL, (step, dz)
    assert abs(g.info(0).volume / o.info().volume - 1.0) <= 1e-4
    assert min(ndry) == 0 and max(ndry) > 0.4 * c["nel"], ndry
    # the stretch before a tie holds the flooding of the flat and its drying
    # to the largest dry set of the cycle
    assert first_tie is None or first_tie > int(np.argmax(ndry)) + 1, (first_tie, ndry)


def test_tidal_flat_in_a_batch():
    """A wetting-and-drying basin batched with a channel without it: each
    member as it runs alone (the dry set of the flat bit for bit)."""
    flat, chan = cases.flat_case(), cases.channel_case()
    b = shygpu.Model([chan, flat])
    b.set_state_all()
    a = shygpu.Model(flat)
    a.set_state(0)
    b.run(200)
    a.run(200)
    for x, y in zip(b.wetdry(1), a.wetdry(0)):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(b.get_state(1)["znv"], a.get_state(0)["znv"])
    o = shyref.OracleModel(chan)
    o.run(200)
    assert np.abs(b.get_state(0)["znv"] - o.state()["znv"]).max() <= ZETA_TOL
    assert not b.wetdry(0)[0].any()
