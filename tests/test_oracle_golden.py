"""The FP64 oracle reproduces the committed fixtures of its own states
(tests/golden/oracle_states.npz, written by tests/golden/make_golden.py):
the 2D tidal channel after 60 steps and the small 3D basin after 20, to
FP32 resolution of each field's scale.  A change of the oracle that moves
its results shows here before it reaches a parity test."""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "oracle_states.npz"


def load():
    z = np.load(GOLDEN)
    return json.loads(str(z["meta"])), z


def test_fixture_covers_the_cases_of_the_script():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN.parent / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    meta, z = load()
    assert [m["name"] for m in meta] == [c[0] for c in mg.CASES]
    for m in meta:
        for f in m["fields"]:
            assert f"{m['name']}/{f}" in z.files


@pytest.mark.parametrize("which", [0, 1])
def test_oracle_reproduces_its_fixture(which):
    import shyref
    from shygpu import cases
    meta, z = load()
    m = meta[which]
    o = shyref.OracleModel(getattr(cases, m["ctor"])(**m["args"]))
    o.run(m["steps"])
    st = o.state()
    for f in m["fields"]:
        ref = z[f"{m['name']}/{f}"].astype(np.float64)
        scale = max(np.abs(ref).max(), 1e-30)
        assert np.abs(st[f] - ref).max() <= 2e-7 * scale, f
