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
