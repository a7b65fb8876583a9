"""The serving loop on the GPU: requests of different kinds arrive while
others run, are admitted as slots and memory free up, run concurrently,
and each result is the same as the same run alone."""
import numpy as np
import pytest

import shygpu
from shygpu import cases

pytestmark = pytest.mark.gpu


def alone(case, nsteps):
    m = shygpu.Model(case)
    m.set_state(0)
    m.run(nsteps)
    out = m.get_state(0)
    m.close()
    return out


def test_results_same_alone_and_in_the_mix():
    c_chan = cases.channel_case()
    c_ts = cases.basin3d_case(nkn_target=1500, nlv=12, seed=31)                     # T/S, baroclinic
    c_big = cases.basin3d_case(nkn_target=50000, nlv=4, seed=32, baroclinic=False, ts=False)  # device-wide solver
    c_cor = cases.basin3d_case(nkn_target=900, nlv=6, seed=33, baroclinic=False, ts=False)
    c_cor["fcorv"] = np.full(c_cor["nel"], 1.0e-4, np.float32)                      # BiCGStab, complex columns
    reqs = [(c_chan, 40), (c_ts, 25), (c_big, 15), (c_cor, 30)]
    # room for about two runs at once: later arrivals wait for memory
    budget = shygpu.footprint([c_big]) + shygpu.footprint([c_ts]) + 1
    srv = shygpu.Server(budget, max_active=3, quantum_steps=7)
    ids = [srv.submit(c, n) for c, n in reqs[:2]]
    srv.progress()
    srv.progress()
    ids += [srv.submit(c, n) for c, n in reqs[2:]]
    saw_queue = False
    for _ in range(10000):
        act, queued, _ = srv.progress(block=True)
        saw_queue |= queued > 0 and act > 0
        if all(srv.status(i)[0] >= shygpu.Server.DONE for i in ids):
            break
    assert saw_queue
    for i, (c, n) in zip(ids, reqs):
        st, steps, ts, ta, td = srv.status(i)
        assert st == shygpu.Server.DONE and steps == n and ts <= ta <= td
        got, info = srv.result(i)
        ref = alone(c, n)
        assert info.status == 0
        for f in ("znv", "utlnv", "vtlnv"):
            assert np.array_equal(got[f], ref[f]), (i, f)
        if c["params"]["itemp"]:
            assert np.array_equal(got["tempv"], ref["tempv"]) and np.array_equal(got["saltv"], ref["saltv"])
    assert srv.used() == 0
    srv.close()


def test_preempted_run_resumes_exactly():
    """shygpu_serve_preempt: a long run is stopped to make room for an urgent
    one (one run fits at a time), then continues from its checkpoint; both
    results equal the runs alone, bit for bit."""
    c_long = cases.basin3d_case(nkn_target=1500, nlv=12, seed=41)       # T/S, baroclinic
    c_urgent = cases.channel_case()
    budget = max(shygpu.footprint([c_long]), shygpu.footprint([c_urgent])) + 1
    srv = shygpu.Server(budget, max_active=1, quantum_steps=5)
    a = srv.submit(c_long, 40)
    for _ in range(3):
        srv.progress(block=True)
    assert srv.status(a)[0] == shygpu.Server.ACTIVE
    b = srv.submit(c_urgent, 30)
    srv.preempt(a)                       # b, already waiting, goes first; a queues behind it
    assert srv.used() == 0
    for _ in range(10000):
        srv.progress(block=True)
        if all(srv.status(i)[0] >= shygpu.Server.DONE for i in (a, b)):
            break
    assert srv.status(b)[4] <= srv.status(a)[4]      # the urgent run finished first
    for i, (c, n) in ((a, (c_long, 40)), (b, (c_urgent, 30))):
        assert srv.status(i)[0] == shygpu.Server.DONE
        got, info = srv.result(i)
        ref = alone(c, n)
        for f in ("znv", "utlnv", "vtlnv"):
            assert np.array_equal(got[f], ref[f]), (i, f)
    srv.close()
