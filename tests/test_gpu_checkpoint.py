"""Exact checkpoints (restart.f90:445-660): a model's device arrays saved to
host memory and loaded back, into the same model or into a new one made
from the same inputs, continue the run bit for bit."""
import numpy as np
import pytest

import shygpu
from shygpu import cases

pytestmark = pytest.mark.gpu

FIELDS = ("znv", "utlnv", "vtlnv", "hdknv", "wlnv", "tempv", "saltv", "conzv")


def same(a, b):
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), f


@pytest.mark.parametrize("shape", ["basin3d_ts", "flat_wetdry", "lagoon_tvd"])
def test_checkpoint_resume_is_exact(small3d, shape):
    if shape == "basin3d_ts":
        c = small3d
    elif shape == "flat_wetdry":
        c = cases.flat_case(nlv=4)
        c["params"] = dict(c["params"], ilin=0)
    else:
        c = cases.lagoon_case(nkn_target=900, nlv=12)
        c["params"] = dict(c["params"], itvd=2, itvdv=1, aapar=0.0)
    g = shygpu.Model(c)
    g.set_state(0)
    g.run(25)
    ck = g.checkpoint()
    g.run(15)
    a = g.get_state(0)
    g.restore(ck)                     # back in the same model
    g.run(15)
    same(a, g.get_state(0))
    h = shygpu.Model(c)               # and into a new model of the same inputs
    h.restore(ck)
    h.run(15)
    same(a, h.get_state(0))
    if c["params"].get("wetdry"):
        for x, y in zip(g.wetdry(0), h.wetdry(0)):
            assert np.array_equal(x, y)


def test_checkpoint_of_another_model_is_refused(small3d):
    g = shygpu.Model(small3d)
    g.set_state(0)
    ck = g.checkpoint()
    other = shygpu.Model(cases.channel_case())
    with pytest.raises(shygpu.ShyError, match="SHY_EARG"):
        other.restore(ck)
