"""The timed workloads at their full sizes against the FP64 oracle.

* The bench's batched ensemble (64 basins, 5k..100k nodes, 10 z-layers):
  all 64 basins advance together on the GPU in one model, as the bench runs
  them, and its smallest, median and largest members are compared with the
  oracle's runs of those basins.
* The 3D baroclinic basin at its configured size (20k nodes, 20 z-layers,
  T and S transported, wind, M2).
* The sigma-layer lagoon at 25k nodes (30 sigma layers, M2 + S2, three
  passive tracers).

Tolerances are the step's targets: water level within 1 mm, tracers within
1e-4 of their largest magnitude, transports within 1e-3 of the largest
transport component, volume within 1e-6 relative.  The oracle runs in spawned worker processes while the
GPU steps, one basin per process.
"""
import numpy as np
import pytest

import oracle_pool as pool
import shygpu
from shygpu import cases

pytestmark = pytest.mark.gpu

ZETA_TOL = 1.0e-3
TRACER_RTOL = 1.0e-4
TRANSPORT_RTOL = 1.0e-3
VOLUME_RTOL = 1.0e-6


def active(case, node=True):
    il = case["ilhkv"] if node else case["ilhv"]
    return np.arange(case["nlv"])[None, :] < il[:, None]


def compare(case, sg, vol_g, o, scalars=()):
    so = o["state"]
    dz = float(np.abs(sg["znv"] - so["znv"]).max())
    assert dz <= ZETA_TOL, ("water level", case["name"], dz)
    me = active(case, node=False)
    # the scale of the transport vector: its largest component anywhere
    umax = max(np.abs(so["utlnv"][me]).max(), np.abs(so["vtlnv"][me]).max())
    for f in ("utlnv", "vtlnv"):
        du = np.abs(sg[f] - so[f])[me].max()
        assert du <= TRANSPORT_RTOL * umax, (f, case["name"], du / umax)
    mk = active(case)
    for f in scalars:
        a, b = sg[f], so[f]
        m = mk if a.ndim == 2 else np.broadcast_to(mk, a.shape)
        rel = np.abs(a - b)[m].max() / np.abs(b[m]).max()
        assert rel <= TRACER_RTOL, (f, case["name"], rel)
    assert abs(vol_g - o["volume"]) <= VOLUME_RTOL * o["volume"], (case["name"], vol_g, o["volume"])
    return dz


def ensemble_picks(n=64):
    """The smallest, the median and the largest member by drawn node count."""
    sizes = [d[0] for d in cases.ensemble_draws(n)]
    order = np.argsort(sizes, kind="stable")
    return [int(order[0]), int(order[n // 2]), int(order[-1])]


def test_bench_ensemble_members_match_the_oracle():
    nsteps = 120
    picks = ensemble_picks()
    specs = [("ensemble_cases", dict(n=64, seed=4, only=[i])) for i in picks]
    p, r = pool.run_states(specs, nsteps, fields=("znv", "utlnv", "vtlnv"), wait=False)
    try:
        ens = cases.ensemble_cases(64)
        assert sum(c["nkn"] for c in ens) > 2_000_000
        g = shygpu.Model(ens)
        g.set_state_all()
        g.run(nsteps)
        res = r.get()
    finally:
        p.close()
        p.join()
    sizes = [ens[i]["nkn"] for i in picks]
    assert sizes[0] < 6000 and sizes[2] > 80000
    for i, o in zip(picks, res):
        compare(ens[i], g.get_state(i, ("znv", "utlnv", "vtlnv")), g.info(i).volume, o)
    g.close()


def test_basin3d_full_size_two_hundred_forty_steps():
    """The 3D baroclinic basin at its configured size over 8 h (240 steps
    of 120 s): T and S transported, baroclinic pressure, wind, M2."""
    nsteps = 240
    spec = ("basin3d_case", dict(nkn_target=20000))
    p, r = pool.run_states([spec], nsteps, wait=False)
    try:
        c = pool.build_case(spec)
        assert c["nkn"] >= 20000 and c["nlv"] == 20
        g = shygpu.Model(c)
        g.set_state(0)
        g.run(nsteps)
        (o,) = r.get()
    finally:
        p.close()
        p.join()
    compare(c, g.get_state(0), g.info(0).volume, o, scalars=("tempv", "saltv"))
    g.close()


def test_lagoon_25k_sigma_layers_three_tracers():
    """The lagoon on 30 sigma layers at 25k nodes, three passive tracers,
    M2 + S2, dt 30 s, 120 steps."""
    nsteps = 120
    spec = ("lagoon_case", dict(nkn_target=25000, nlv=30))
    p, r = pool.run_states([spec], nsteps, wait=False)
    try:
        c = pool.build_case(spec)
        assert c["nkn"] >= 24000 and c["nlv"] == 30 and c["params"]["nconz"] == 3
        g = shygpu.Model(c)
        g.set_state(0)
        g.run(nsteps)
        (o,) = r.get()
    finally:
        p.close()
        p.join()
    compare(c, g.get_state(0), g.info(0).volume, o, scalars=("conzv",))
    g.close()
