"""The non-hydrostatic pressure (nohydro.f90; inohyd = 1) on the GPU against
the FP64 oracle.

* A standing wave in a 25 m deep, 50 m long basin, where the pressure
  changes the period by a quarter: level, transports and pressure against
  the oracle after 300 steps of 0.1 s, with both column-kernel forms, and
  the GPU's period against the oracle's.
* A 300 m basin under wind with T and S, on sigma layers and on z-layers
  (with vertical and horizontal advection of w, ivwadv = 1, inhflx = 1):
  level within 1e-3 of its range, transports within 1e-3 of their largest
  value, tracers 1e-4 relative, the pressure within 1e-2 of its largest.
* Still water stays still; the CUDA-graph step equals the eager one; a
  checkpoint resumes bit for bit (the pressure is part of the state).
"""
import numpy as np
import pytest

import shygpu
import shyref
from shygpu import cases

pytestmark = pytest.mark.gpu


def run_both(case, nsteps, **opts):
    g = shygpu.Model(case)
    for k, v in opts.items():
        g.set_option(k, v)
    g.set_state(0)
    o = shyref.OracleModel(case)
    g.run(nsteps)
    o.run(nsteps)
    return g, o


def active(case, node=True):
    il = case["ilhkv"] if node else case["ilhv"]
    return np.arange(case["nlv"])[None, :] < il[:, None]


def crossings(z, dt):
    return [(i + z[i] / (z[i] - z[i + 1])) * dt for i in range(len(z) - 1) if z[i] * z[i + 1] < 0]


@pytest.mark.parametrize("column_threads", [1, 0])
def test_seiche_matches_the_oracle(column_threads):
    c = cases.seiche_case()
    g, o = run_both(c, 300, column_threads=column_threads)
    sg, so = g.get_state(0), o.state()
    amp = float(np.abs(c["znv"]).max())
    assert np.abs(sg["znv"] - so["znv"]).max() <= 1e-3 * amp
    me = active(c, node=False)
    umax = np.abs(so["utlnv"][me]).max()
    for f in ("utlnv", "vtlnv"):
        assert np.abs(sg[f] - so[f])[me].max() <= 1e-3 * umax, f
    qg, (it, rf, r0, r) = g.nh(0)
    qo, _, _ = o.nh()
    mk = active(c)
    assert np.abs(qg - qo)[mk].max() <= 2e-3 * np.abs(qo[mk]).max()
    assert np.all(qg[:, 0] == 0.0)
    assert it > 0 and r <= 1e-8 * r0 + 1e-8
    assert abs(g.info(0).volume - o.info().volume) <= 1e-6 * o.info().volume


def test_seiche_period_on_the_gpu():
    """The GPU's standing wave keeps the oracle's non-hydrostatic period."""
    c = cases.seiche_case()
    k0 = int(np.argmin(c["xgv"]))
    g = shygpu.Model(c)
    g.set_state(0)
    o = shyref.OracleModel(c)
    zg, zo = [float(c["znv"][k0])], [float(c["znv"][k0])]
    for _ in range(200):
        g.run(1)
        o.run(1)
        zg.append(float(g.get_state(0)["znv"][k0]))
        zo.append(float(o.state()["znv"][k0]))
    dt = c["params"]["dt"]
    tg, to = crossings(np.array(zg), dt), crossings(np.array(zo), dt)
    assert len(tg) == len(to) >= 4
    assert np.abs(np.array(tg) - np.array(to)).max() <= 0.005 * (to[1] - to[0])


@pytest.mark.parametrize("column_threads", [1, 0])
def test_sigma_basin_with_nonhydrostatic_pressure(column_threads):
    """A 300 m basin on sigma layers, 5 to 30 m deep, under wind, T and S
    transported, for 200 steps of 0.5 s."""
    c = cases.nh_basin_case(sigma=True)
    g, o = run_both(c, 200, column_threads=column_threads)
    check_state(c, g, o)


def test_z_layer_basin_with_nonhydrostatic_pressure():
    """The same basin on z-layers, with vertical and upwind horizontal
    advection of w (ivwadv = 1, inhflx = 1) and horizontal diffusion, over
    40 steps.  On these stepped bottoms both the oracle and the GPU grow
    unstable after about 60 steps (the pressure doubles every few steps
    from there), so the comparison stops before."""
    c = cases.nh_basin_case(sigma=False)
    c["params"] = dict(c["params"], ivwadv=1, inhflx=1, ahpar=0.2)
    g, o = run_both(c, 40)
    check_state(c, g, o)


def check_state(c, g, o):
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= 1e-3 * max(np.abs(so["znv"]).max(), 1e-3)
    me, mk = active(c, node=False), active(c)
    umax = max(np.abs(so["utlnv"][me]).max(), np.abs(so["vtlnv"][me]).max())
    for f in ("utlnv", "vtlnv"):
        assert np.abs(sg[f] - so[f])[me].max() <= 1e-3 * umax, f
    for f in ("tempv", "saltv"):
        rel = np.abs(sg[f] - so[f])[mk].max() / np.abs(so[f][mk]).max()
        assert rel <= 1e-4, (f, rel)
    qg, (it, rf, r0, r) = g.nh(0)
    qo, _, _ = o.nh()
    assert np.abs(qg - qo)[mk].max() <= 1e-2 * np.abs(qo[mk]).max()
    assert it > 0 and r <= 1e-8 * r0 + 1e-8
    assert abs(g.info(0).volume - o.info().volume) <= 1e-6 * o.info().volume


def test_still_water_stays_still():
    c = cases.seiche_case(ampli=0.0)
    g = shygpu.Model(c)
    g.set_state(0)
    g.run(20)
    s = g.get_state(0)
    assert np.abs(s["znv"]).max() == 0.0 and np.abs(s["utlnv"]).max() == 0.0
    q, _ = g.nh(0)
    assert np.abs(q).max() == 0.0


def test_graph_equals_eager_and_checkpoint_resumes():
    c = cases.seiche_case()
    a = shygpu.Model(c)
    a.set_state(0)
    a.run(30)
    b = shygpu.Model(c)
    b.set_option("use_graph", 0)
    b.set_state(0)
    b.run(30)
    sa, sb = a.get_state(0), b.get_state(0)
    for f in ("znv", "utlnv", "vtlnv", "wlnv"):
        assert np.array_equal(sa[f], sb[f]), f
    ck = a.checkpoint()
    a.run(20)
    ref, qref = a.get_state(0), a.nh(0)[0]
    a.restore(ck)
    a.run(20)
    s2, q2 = a.get_state(0), a.nh(0)[0]
    for f in ("znv", "utlnv", "vtlnv", "wlnv"):
        assert np.array_equal(ref[f], s2[f]), f
    assert np.array_equal(qref, q2)


def test_nonhydrostatic_refused_with_wetting_and_drying():
    c = cases.seiche_case()
    c["params"] = dict(c["params"], wetdry=1)
    with pytest.raises(RuntimeError, match="non-hydrostatic"):
        shygpu.Model(c)
