"""Failure detection without a GPU fault: the device-wide zeta solver's
barrier is made to wait for an arrival that never comes (one CTA more than
the launch has).  Every wait runs out after its short poll limit, the
kernel returns, the step reports SHY_ECUDA through the status the host
reads, and the same context then runs correctly again."""
import numpy as np
import pytest

import shygpu

pytestmark = pytest.mark.gpu


def test_grid_barrier_timeout_is_reported_and_recoverable(small3d):
    # the reference run: one step, then the initial state again (set_state
    # keeps the model clock, which the failed step also advanced), 3 steps
    ref = shygpu.Model(small3d)
    ref.set_option("zeta_variant", 2)
    ref.set_state(0)
    ref.run(1)
    ref.set_state(0)
    ref.run(3)
    want = ref.get_state(0)["znv"]

    g = shygpu.Model(small3d)
    g.set_option("zeta_variant", 2)
    g.set_state(0)
    g.set_option("zeta_barrier_timeout_test", 1)
    with pytest.raises(shygpu.ShyError) as e:
        g.run(1)
    assert e.value.code == 2 and "ran out" in str(e.value)
    g.set_option("zeta_barrier_timeout_test", 0)
    g.set_state(0)
    g.run(3)
    assert np.array_equal(g.get_state(0)["znv"], want)
