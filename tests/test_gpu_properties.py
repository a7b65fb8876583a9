"""The analytic properties of the step on the GPU: still water stays still,
and a closed basin keeps its volume and every tracer's mass while wind
moves the water (FP32 state: to single-precision round-off)."""
import numpy as np
import pytest

import shygpu
from shygpu import cases

pytestmark = pytest.mark.gpu


def node_areas(c):
    import shyref
    ev = shyref.set_ev(c)
    areafv = 12.0 * ev[:, 9] / 3.0
    A = np.zeros((c["nkn"], c["nlv"]))
    for e in range(c["nel"]):
        for k in c["nen3v"][e] - 1:
            A[k, :c["ilhv"][e]] += areafv[e]
    return A


def test_still_water_stays_still():
    c = cases.channel_case()
    c["tide"] = np.zeros_like(c["tide"])
    g = shygpu.Model(c)
    g.set_state(0)
    g.run(100)
    s = g.get_state(0)
    assert np.abs(s["znv"]).max() == 0.0 and np.abs(s["utlnv"]).max() == 0.0


def test_closed_basin_conserves_volume_and_tracer_mass():
    c = cases.lagoon_case(nkn_target=900, nlv=12)
    c["bnd_index"] = np.zeros_like(c["bnd_index"])
    c["tide"] = np.zeros((0, 2, 4), np.float32)
    c["tauxnv"] = np.full(c["nkn"], 2e-4, np.float32)
    A = node_areas(c)

    def budget(s):
        h = s["hdknv"].astype(np.float64)
        return (h * A).sum(), [(s["conzv"][t].astype(np.float64) * h * A).sum() for t in range(s["conzv"].shape[0])]

    g = shygpu.Model(c)
    g.set_state(0)
    v0, m0 = budget(g.get_state(0))
    g.run(40)
    v1, m1 = budget(g.get_state(0))
    assert np.abs(g.get_state(0)["znv"]).max() > 0.01
    assert abs(v1 / v0 - 1.0) < 1e-6
    for a, b in zip(m0, m1):
        assert abs(b / a - 1.0) < 1e-5


@pytest.mark.parametrize("scheme", ["upwind", "tvd"])
def test_uniform_tracers_stay_uniform(scheme):
    """A uniform field stays uniform under any flow (constancy): the
    transport's update is the conservative one solved for the increment, so
    in FP32 its rounding scales with the increment, not with the value.
    Temperature 15 and salinity 35 everywhere on the 3D basin (wind, M2,
    strong vertical velocities), and three tracers of 10 on the sigma
    lagoon; with scheme "tvd" horizontal (itvd 1) and vertical (itvdv 1)
    TVD.  What remains over 120 steps (5e-6 relative) is the rounding of
    the stored FP32 vertical velocities against the flows they balance,
    which the reference's real arrays carry as well."""
    b3 = cases.basin3d_case(nkn_target=2000, nlv=12)
    b3["tempv"] = np.full_like(b3["tempv"], 15.0)
    b3["saltv"] = np.full_like(b3["saltv"], 35.0)
    lg = cases.lagoon_case(nkn_target=900, nlv=12)
    lg["conzv"] = np.full_like(lg["conzv"], 10.0)
    for c, fields, value in ((b3, ("tempv", "saltv"), (15.0, 35.0)), (lg, ("conzv",), (10.0,))):
        if scheme == "tvd":
            c["params"] = dict(c["params"], itvd=1, itvdv=1, aapar=0.0)
        g = shygpu.Model(c)
        g.set_state(0)
        g.run(120)
        s = g.get_state(0)
        act = np.arange(c["nlv"])[None, :] < c["ilhkv"][:, None]
        for f, v in zip(fields, value):
            a = s[f] if s[f].ndim == 2 else s[f].reshape(-1, c["nkn"], c["nlv"])
            m = act if a.ndim == 2 else np.broadcast_to(act, a.shape)
            dev = np.abs(a[m] - v).max()
            assert dev <= 5e-6 * v, (c["name"], f, dev)
        g.close()


def test_closed_basin_volume_budget_to_fp64_roundoff():
    """The FP64 volume budget (shy_step_info.volume_budget: the initial
    volume plus every step's dt times the element fluxes of the zeta
    equation into each node column) of a closed basin under wind stays at
    its initial value to FP64 round-off over 1200 steps, while the FP32
    state's own volume (vol_mass) moves at FP32 round-off; the two agree to
    FP32 accuracy."""
    c = cases.basin3d_case(nkn_target=2000, nlv=8, baroclinic=False, ts=False)
    c["bnd_index"] = np.zeros_like(c["bnd_index"])
    c["tide"] = np.zeros((0, 1, 4), np.float32)
    g = shygpu.Model(c)
    g.set_state(0)
    i0 = g.info(0)
    b0, v0 = i0.volume_budget, i0.volume
    assert b0 == v0
    g.run(1200)
    i1 = g.info(0)
    assert np.abs(g.get_state(0)["znv"]).max() > 0.01        # the wind has moved the water
    assert abs(i1.volume_budget / b0 - 1.0) <= 1e-12, i1.volume_budget / b0 - 1.0
    assert abs(i1.volume / v0 - 1.0) <= 1e-5
    assert abs(i1.volume / i1.volume_budget - 1.0) <= 1e-5
