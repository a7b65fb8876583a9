"""The GPU step against the committed oracle fixtures
(tests/golden/oracle_states.npz) instead of a live oracle run: the 2D tidal
channel after 60 steps and the small 3D basin (12 z-layers, T/S,
baroclinic) after 20, through the C ABI.  Tolerances as in the parity
tests: water level within 1 mm, transports within 1e-3 of their largest
value, tracers within 1e-4 relative, layer thicknesses within 1e-4 m,
vertical velocities within 2e-3 of their largest value."""
import json
from pathlib import Path

import numpy as np
import pytest

import shygpu
from shygpu import cases

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "oracle_states.npz"


@pytest.mark.parametrize("which", [0, 1])
def test_gpu_matches_the_oracle_fixture(which):
    z = np.load(GOLDEN)
    m = json.loads(str(z["meta"]))[which]
    c = getattr(cases, m["ctor"])(**m["args"])
    g = shygpu.Model(c)
    g.set_state(0)
    g.run(m["steps"])
    sg = g.get_state(0)
    ref = {f: z[f"{m['name']}/{f}"].astype(np.float64) for f in m["fields"]}
    node = np.arange(c["nlv"])[None, :] < c["ilhkv"][:, None]
    elem = np.arange(c["nlv"])[None, :] < c["ilhv"][:, None]
    assert np.abs(sg["znv"] - ref["znv"]).max() <= 1.0e-3
    umax = max(np.abs(ref["utlnv"][elem]).max(), np.abs(ref["vtlnv"][elem]).max())
    for f in ("utlnv", "vtlnv"):
        assert np.abs(sg[f] - ref[f])[elem].max() <= 1e-3 * umax, f
    for f in ("tempv", "saltv"):
        if f in ref:
            assert np.abs(sg[f] - ref[f])[node].max() <= 1e-4 * np.abs(ref[f][node]).max(), f
    if "hdknv" in ref:
        assert np.abs(sg["hdknv"] - ref["hdknv"])[node].max() <= 1e-4
    if "wlnv" in ref:
        assert np.abs(sg["wlnv"] - ref["wlnv"]).max() <= 2e-3 * np.abs(ref["wlnv"]).max()
    g.close()
