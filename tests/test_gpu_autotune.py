"""shygpu_autotune: the project's own tuner of launch shapes.

It times candidate options on the model's basins from their current state
and keeps the fastest.  The tuned model must meet the parity tolerances
against the oracle, be no slower than the default plan, continue from the
state it had before tuning (the trials start from a checkpoint), and a
second model of the same shape must take the cached choice without trials.
"""
import time

import numpy as np
import pytest

import shygpu
import shyref
from shygpu import cases

pytestmark = pytest.mark.gpu


def members():
    # eight members of the bench's ensemble: 8 basins of 5k..100k nodes
    return cases.ensemble_cases(64, only=[17, 35, 47, 3, 8, 21, 40, 60])


def device_ms(model, steps):
    import torch
    st = torch.cuda.ExternalStream(model.stream())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(st):
        a.record(st)
        shygpu.lib().shygpu_enqueue(model.h, steps)
        b.record(st)
    torch.cuda.synchronize()
    shygpu.check(shygpu.lib().shygpu_sync(model.h), "sync")
    return a.elapsed_time(b) / steps


def test_autotune_keeps_parity_speed_and_state():
    ens = members()
    g = shygpu.Model(ens)
    g.set_state_all()
    choice, ms = g.autotune(steps=4)
    assert g.get_option("tuned") == 1 and ms > 0
    for item in choice.split():
        name, value = item.split("=")
        if name not in ("zeta_variant", "zeta_stage"):    # those report the plan that resulted
            assert abs(g.get_option(name) - float(value)) < 1e-6, item
    # the tuner left the state as it was: the tuned model continues like a
    # model given the same options directly
    h = shygpu.Model(ens)
    h.set_state_all()
    for item in choice.split():
        name, value = item.split("=")
        h.set_option(name, float(value))
    g.run(10)
    h.run(10)
    for i in (0, 3, 7):
        a, b = g.get_state(i), h.get_state(i)
        for f in ("znv", "utlnv", "vtlnv", "wlnv"):
            assert np.array_equal(a[f], b[f]), (i, f)
    # parity: the tuned model against the oracle after 60 steps
    for i in (0, 2):
        c = ens[i]
        m = shygpu.Model(c)
        m.set_state(0)
        for item in choice.split():
            name, value = item.split("=")
            m.set_option(name, float(value))
        o = shyref.OracleModel(c)
        m.run(60)
        o.run(60)
        sg, so = m.get_state(0), o.state()
        assert np.abs(sg["znv"] - so["znv"]).max() <= 1e-3
        me = np.arange(c["nlv"])[None, :] < c["ilhv"][:, None]
        umax = max(np.abs(so["utlnv"][me]).max(), np.abs(so["vtlnv"][me]).max())
        assert np.abs(sg["utlnv"] - so["utlnv"])[me].max() <= 1e-3 * umax
    # no slower than the default plan (device time per step, best of three)
    d = shygpu.Model(ens)
    d.set_state_all()
    d.run(3)
    g.run(3)
    t_default = min(device_ms(d, 10) for _ in range(3))
    t_tuned = min(device_ms(g, 10) for _ in range(3))
    assert t_tuned <= 1.05 * t_default, (t_tuned, t_default, choice)


def test_autotune_cache_applies_the_choice_without_trials():
    ens = members()
    a = shygpu.Model(ens)
    a.set_state_all()
    ca, _ = a.autotune(steps=2)
    b = shygpu.Model(ens)
    b.set_state_all()
    t0 = time.perf_counter()
    cb, ms = b.autotune(steps=2)
    assert cb == ca and ms == -1.0
    assert time.perf_counter() - t0 < 2.0
