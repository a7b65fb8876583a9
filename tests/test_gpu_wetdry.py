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
centimetres at the front (FRONT_TOL) and inside the wet domain (INNER_TOL)
and a few dry marks (DRY_DIFF), while the volume stays within 1e-4."""
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
INNER_TOL = 0.1            # m, after a tie: nodes inside the wet domain of both runs
# With momentum advection (ilin = 0) the upwind choices (inflow f > 0 at a
# node) switch discontinuously where the flow stagnates, and rounding picks
# the branch: the oracle against itself, with 1e-6 m of noise in the initial
# levels, first decides differently at step 319 of the cycle and then
# differs by 7 cm at the front.  The GPU's first tie comes earlier (its
# whole state carries FP32 rounding); after it the front nodes, whose level
# in a run where their elements are dry comes from the dry Laplacian, may
# differ by decimetres, so only nodes inside both wet domains are compared,
# and the volume within 1e-3.


def levels(g, o):
    return g.get_state(0)["znv"].astype(np.float64), o.state()["znv"]


def at_a_tie(c, e, was_dry, z_old, z_new):
    """Whether a decision on element e sits within TIE of its threshold in
    one of the runs: a wet element leaves on a vertex below hzoff at the old
    level (setweg 2) or below hzmin at the new one (setweg 1); a dry one
    comes back on its vertices, or their mean, reaching hzon at the old
    level (setweg 3), and may leave again at the new one."""
    p = cases_params(c)
    hm = c["hm3v"][e].astype(np.float64)
    kn = c["nen3v"][e] - 1

    def near(x, t):
        return float(np.min(np.abs(np.atleast_1d(x) - t))) <= TIE

    for z in z_old:
        hz = z[kn] + hm
        if was_dry and (near(hz, p["hzon"]) or near(hz.mean(), p["hzon"])):
            return True
        if not was_dry and near(hz, p["hzoff"]):
            return True
    return any(near(z[kn] + hm, p["hzmin"]) for z in z_new)


def cases_params(c):
    p = dict(hzmin=0.01, hzoff=0.05, hzon=0.10)
    p.update({k: v for k, v in c.get("params", {}).items() if k in p})
    return p


@pytest.mark.parametrize("nlv,ilin", [(1, 1), (4, 1), (1, 0)])
def test_tidal_flat_dries_and_floods(nlv, ilin):
    """One M2 period (750 steps of 60 s), compared after every step; with
    momentum advection (ilin = 0) the nodal velocities skip dry elements."""
    c = cases.flat_case(nlv=nlv)
    c["params"] = dict(c["params"], ilin=ilin)
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
        dry0 = gw[0] > 0
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
                assert at_a_tie(c, e, dry0[e], (zg0, zo0), (zg, zo)), (step, e)
            first_tie = step
        if first_tie is None:
            np.testing.assert_array_equal(gw[2], ow[2])
            assert dz <= ZETA_TOL, (step, dz)
        else:
            assert ((gw[0] > 0) != (ow[0] > 0)).sum() <= DRY_DIFF * c["nel"], step
            inner = (gw[2] == 0) & (ow[2] == 0)
            assert np.abs(zg - zo)[inner].max() <= INNER_TOL, step
            if ilin:
                assert dz <= FRONT_TOL, (step, dz)
    assert abs(g.info(0).volume / o.info().volume - 1.0) <= (1e-4 if ilin else 1e-3)
    assert min(ndry) == 0 and max(ndry) > 0.4 * c["nel"], ndry
    if ilin:
        # the stretch before a tie holds the flooding of the flat and its
        # drying to the largest dry set of the cycle
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
