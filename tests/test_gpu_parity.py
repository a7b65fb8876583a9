"""GPU step against the FP64 CPU oracle (parity tests proper).

Tolerances (the targets of the step): water level within 1 mm, tracers
within 1e-4 relative; transports within 1e-3 of their maximum magnitude;
layer thicknesses and vertical velocities to single-precision accuracy of
their scale.  Runs go through the C ABI (shygpu.Model over libshygpu.so).
"""
import numpy as np
import pytest

import shygpu
import shyref
from shygpu import cases

pytestmark = pytest.mark.gpu

ZETA_TOL = 1.0e-3          # m
TRACER_RTOL = 1.0e-4


def run_both(case, nsteps, **opts):
    g = shygpu.Model(case)
    for k, v in opts.items():
        g.set_option(k, v)
    g.set_state(0)
    o = shyref.OracleModel(case)
    g.run(nsteps)
    o.run(nsteps)
    return g, o


def active_mask(case, node=True):
    nlv = case["nlv"]
    il = case["ilhkv"] if node else case["ilhv"]
    return np.arange(nlv)[None, :] < il[:, None]


def test_channel_2d_one_day_tide(channel):
    """Config 1: 2D channel, M2 0.5 m, dt 60 s, one simulated day."""
    g, o = run_both(channel, 1440)
    sg, so = g.get_state(0), o.state()
    dz = np.abs(sg["znv"] - so["znv"]).max()
    assert dz <= ZETA_TOL, dz
    umax = np.abs(so["utlnv"]).max()
    assert np.abs(sg["utlnv"] - so["utlnv"]).max() <= 1e-3 * umax
    ig, io = g.info(0), o.info()
    assert abs(ig.dtime - io.dtime) < 1e-6
    assert abs(ig.volume - io.volume) <= 1e-6 * io.volume
    assert abs(ig.volume_budget - io.volume) <= 1e-6 * io.volume   # the FP64 budget, open boundary


@pytest.mark.parametrize("column_threads", [1, 0])
def test_basin3d_baroclinic_ts(small3d, column_threads):
    """Config 2 shape at test size: z-layers, wind, M2, T/S, baroclinic;
    the column kernel with one thread per column and with one warp segment
    per column."""
    g, o = run_both(small3d, 120, column_threads=column_threads)
    assert g.get_option("column_threads") == column_threads
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    m = active_mask(small3d)
    for f in ("tempv", "saltv"):
        rel = np.abs(sg[f] - so[f])[m].max() / np.abs(so[f][m]).max()
        assert rel <= TRACER_RTOL, (f, rel)
    me = active_mask(small3d, node=False)
    umax = np.abs(so["utlnv"][me]).max()
    assert np.abs(sg["utlnv"] - so["utlnv"])[me].max() <= 1e-3 * umax
    assert np.abs(sg["hdknv"] - so["hdknv"])[m].max() <= 1e-4
    wmax = np.abs(so["wlnv"]).max()
    assert np.abs(sg["wlnv"] - so["wlnv"]).max() <= 2e-3 * wmax
    assert np.abs(sg["rhov"] - so["rhov"])[m].max() <= 1e-3


def test_coriolis_column_solve():
    """Coriolis couples u and v (penta system, complex PCR on the GPU)."""
    c = cases.basin3d_case(nkn_target=800, nlv=8, baroclinic=False, ts=False)
    c["fcorv"] = np.full(c["nel"], 1.0e-4, np.float32)
    g, o = run_both(c, 60)
    assert g.get_option("column_threads") == 1
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    me = active_mask(c, node=False)
    umax = np.abs(so["vtlnv"][me]).max()
    assert np.abs(sg["vtlnv"] - so["vtlnv"])[me].max() <= 1e-3 * umax


def test_batch_equals_alone():
    """Basins advanced together give the same bits as each advanced alone."""
    cs = [cases.basin3d_case(nkn_target=n, nlv=nl, seed=s)
          for n, nl, s in ((600, 6, 11), (1100, 10, 12), (400, 10, 13))]
    gb = shygpu.Model(cs)
    gb.set_state_all()
    gb.run(20)
    for i, c in enumerate(cs):
        ga = shygpu.Model(c)
        ga.set_state(0)
        ga.run(20)
        a, b = ga.get_state(0), gb.get_state(i)
        for f in ("znv", "utlnv", "tempv", "saltv", "wlnv"):
            assert np.array_equal(a[f], b[f]), (i, f)


def test_graph_equals_eager_and_deterministic(small3d):
    runs = []
    for use_graph in (1, 0, 1):
        g = shygpu.Model(small3d)
        g.set_option("use_graph", use_graph)
        g.set_state(0)
        g.run(15)
        runs.append(g.get_state(0))
    for f in ("znv", "utlnv", "tempv", "wlnv", "rhov"):
        assert np.array_equal(runs[0][f], runs[1][f]), f
        assert np.array_equal(runs[0][f], runs[2][f]), f


def test_split_phases_equal_run(channel):
    a = shygpu.Model(channel)
    a.set_state(0)
    a.run(5)
    b = shygpu.Model(channel)
    b.set_state(0)
    for _ in range(5):
        b.hydro()
        b.scalar()
    assert np.array_equal(a.get_state(0)["znv"], b.get_state(0)["znv"])


def test_transport_substeps():
    """A long time step makes the transport sub-step (istot > 1, scal3sh);
    the device-driven sub-step loop (graph) and the eager loop both match."""
    c = cases.basin3d_case(nkn_target=900, nlv=10, dt=900.0, wind=20.0)
    o = shyref.OracleModel(c)
    o.run(12)
    assert o.info().istot > 1
    so = o.state()
    m = active_mask(c)
    for use_graph in (1, 0):
        g = shygpu.Model(c)
        g.set_option("use_graph", use_graph)
        g.set_state(0)
        g.run(12)
        assert g.info(0).istot == o.info().istot
        sg = g.get_state(0)
        assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
        for f in ("tempv", "saltv"):
            rel = np.abs(sg[f] - so[f])[m].max() / np.abs(so[f][m]).max()
            assert rel <= TRACER_RTOL, (use_graph, f, rel)


@pytest.mark.parametrize("zeta_stage", [1, 0])
def test_device_wide_zeta_solver(small3d, zeta_stage):
    """The cooperative device-wide zeta solver (the one large basins use),
    with its tiles staged into shared memory by TMA bulk copies and with
    plain global loads, against the oracle on the config-2-shaped basin."""
    g, o = run_both(small3d, 120, zeta_variant=2, zeta_stage=zeta_stage)
    assert g.get_option("zeta_variant") == 2
    assert g.get_option("zeta_stage") == zeta_stage
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    m = active_mask(small3d)
    for f in ("tempv", "saltv"):
        rel = np.abs(sg[f] - so[f])[m].max() / np.abs(so[f][m]).max()
        assert rel <= TRACER_RTOL, (f, rel)
    assert g.info(0).krylov_iters > 0


def test_large_basin_in_a_mix():
    """A basin too large for one cluster sends the whole batch to the
    device-wide solver; every member's result matches its run alone to the
    solver's tolerance."""
    cs = [cases.basin3d_case(nkn_target=n, nlv=4, seed=s, baroclinic=False, ts=False)
          for n, s in ((50000, 21), (700, 22), (3000, 23))]
    gb = shygpu.Model(cs)
    assert gb.get_option("zeta_variant") == 2
    gb.set_state_all()
    gb.run(20)
    for i, c in enumerate(cs):
        ga = shygpu.Model(c)
        ga.set_state(0)
        ga.run(20)
        a, b = ga.get_state(0), gb.get_state(i)
        assert np.abs(a["znv"] - b["znv"]).max() <= 1e-5, i
        umax = np.abs(a["utlnv"]).max()
        assert np.abs(a["utlnv"] - b["utlnv"]).max() <= 1e-4 * umax, i


@pytest.mark.parametrize("nlv", [12, 30])
def test_lagoon_sigma_layers_tracers(nlv):
    """The lagoon config's vertical grid at test size: pure sigma layers,
    M2 + S2 boundary, three passive tracers (12 layers: thread-per-column
    kernels; 30 layers: warp-segment kernels)."""
    c = cases.lagoon_case(nkn_target=900, nlv=nlv)
    g, o = run_both(c, 80)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    assert np.abs(sg["hdknv"] - so["hdknv"]).max() <= 1e-4 * np.abs(so["hdknv"]).max()
    umax = np.abs(so["utlnv"]).max()
    assert np.abs(sg["utlnv"] - so["utlnv"]).max() <= 1e-3 * umax
    cmax = np.abs(so["conzv"]).max()
    assert np.abs(sg["conzv"] - so["conzv"]).max() <= TRACER_RTOL * cmax
    wmax = np.abs(so["wlnv"]).max()
    assert np.abs(sg["wlnv"] - so["wlnv"]).max() <= 2e-3 * wmax
    assert abs(g.info(0).volume - o.info().volume) <= 1e-6 * o.info().volume


def with_params(case, **over):
    c = dict(case)
    c["params"] = dict(case["params"], **over)
    return c


@pytest.mark.parametrize("shape", ["channel", "basin3d_threads", "basin3d_segments", "lagoon30"])
def test_momentum_advection(small3d, shape):
    """ilin = 0: explicit upwind momentum advection (set_advective,
    explicit.f90:685-861) from the node momentum of the old level
    (set_momentum_flux :588-683, with the last step's nodal velocities),
    through the thread-per-column and warp-segment column kernels.

    The scheme switches discontinuously where the flow stagnates (a node
    with no inflow takes its velocity times its thickness instead of the
    inflow's momentum), so rounding can pick the other branch there: on a
    tidal flat with 1 m/s currents the oracle against itself, with 1e-7
    relative noise in its state, differs by 4e-3 of the largest transport
    within 10 steps.  These cases stay inside the parity tolerances over
    their horizons."""
    if shape == "channel":
        c, n, opts = with_params(cases.channel_case(), ilin=0), 720, {}
    elif shape == "lagoon30":
        c, n, opts = with_params(cases.lagoon_case(nkn_target=900, nlv=30), ilin=0), 80, {}
    else:
        c, n = with_params(small3d, ilin=0), 120
        opts = dict(column_threads=1 if shape == "basin3d_threads" else 0)
    g, o = run_both(c, n, **opts)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    me = active_mask(c, node=False)
    umax = np.abs(so["utlnv"][me]).max()
    assert np.abs(sg["utlnv"] - so["utlnv"])[me].max() <= 1e-3 * umax
    assert abs(g.info(0).volume - o.info().volume) <= 1e-6 * o.info().volume
    # the advective terms change the flow: the same run without them differs
    # by far more than the tolerance
    lin = shyref.OracleModel(with_params(c, ilin=1))
    lin.run(n)
    assert np.abs(lin.state()["utlnv"] - so["utlnv"])[me].max() > 10e-3 * umax


@pytest.mark.parametrize("itvd", [1, 2])
@pytest.mark.parametrize("shape", ["basin3d", "lagoon30"])
def test_tvd_transport(small3d, shape, itvd):
    """Horizontal TVD fluxes (tvd_fluxes, tvd_admin.f90:673-838): itvd 1
    with node gradients recomputed before every sub-step (tvd_grad_3d
    :478-550), itvd 2 with the value at the point beyond the upwind vertex
    (tvd_upwind_init_elem :361-476, tvd_get_upwind_c :608-671): temperature
    and salinity of the 3D basin, three tracers on the 30-layer sigma
    lagoon."""
    if shape == "basin3d":
        c, n, fields = with_params(small3d, itvd=itvd), 120, ("tempv", "saltv")
    else:
        c, n, fields = with_params(cases.lagoon_case(nkn_target=900, nlv=30), itvd=itvd), 80, ("conzv",)
    g, o = run_both(c, n)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    m = active_mask(c)
    for f in fields:
        a, r = sg[f], so[f]
        if f == "conzv":
            a, r = a[:, m], r[:, m]
        else:
            a, r = a[m], r[m]
        rel = np.abs(a - r).max() / np.abs(r).max()
        assert rel <= TRACER_RTOL, (f, rel)
    # the limiter changes the tracers by far more than the parity tolerance
    up = shyref.OracleModel(with_params(c, itvd=0))
    up.run(n)
    f = fields[-1]
    assert np.abs(up.state()[f] - so[f]).max() > 10 * TRACER_RTOL * np.abs(so[f]).max()


@pytest.mark.parametrize("shape", ["basin3d", "lagoon30"])
def test_vertical_tvd_transport(small3d, shape):
    """itvdv = 1 with aapar = 0: superbee-limited vertical fluxes
    (vertical_flux_ie, tvd_admin.f90:930-1019), the far-upwind layer taken
    from each element's column; on the lagoon together with horizontal TVD."""
    if shape == "basin3d":
        c, n, fields = with_params(small3d, itvdv=1, aapar=0.0), 120, ("tempv", "saltv")
    else:
        c = with_params(cases.lagoon_case(nkn_target=900, nlv=30), itvd=1, itvdv=1, aapar=0.0)
        n, fields = 80, ("conzv",)
    g, o = run_both(c, n)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    m = active_mask(c)
    for f in fields:
        a, r = (sg[f][:, m], so[f][:, m]) if f == "conzv" else (sg[f][m], so[f][m])
        rel = np.abs(a - r).max() / np.abs(r).max()
        assert rel <= TRACER_RTOL, (f, rel)
    # the limiter changes the tracers by far more than the parity tolerance
    up = shyref.OracleModel(with_params(c, itvdv=0))
    up.run(n)
    f = fields[0]
    assert np.abs(up.state()[f] - so[f]).max() > 10 * TRACER_RTOL * np.abs(so[f]).max()


def test_water_level_nudging(channel):
    """andgzv (hydrodynamic.f90:612, 677-679): a per-node nudging
    contribution in the element right-hand sides, set through
    shygpu_set_nudging after the model's step graph exists (the first call
    rebuilds it)."""
    c = channel
    andg = (2e-4 * np.sin(c["xgv"] / 1.5e3) * np.cos(c["ygv"] / 700.0)).astype(np.float32)
    g = shygpu.Model(c)
    g.set_state(0)
    g.run(10)
    o = shyref.OracleModel(c)
    o.run(10)
    g.set_nudging(0, andg)
    o.set_nudging(andg)
    g.run(1430)                      # to the day's end, as the channel test (not at slack water)
    o.run(1430)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    umax = np.abs(so["utlnv"]).max()
    assert np.abs(sg["utlnv"] - so["utlnv"]).max() <= 1e-3 * umax
    free = shyref.OracleModel(c)
    free.run(1440)
    assert np.abs(free.state()["znv"] - so["znv"]).max() > 5 * ZETA_TOL


@pytest.mark.parametrize("column_threads", [1, 0])
def test_hybrid_sigma_z_layers(column_threads):
    """Hybrid layers (setdepth, elems_dealing.f90:1010-1050, 1075-1105): six
    sigma layers down to hsigma = 8 m, 3 m z-layers below, flat-bottomed
    deep elements; three tracers; the thread-per-column and warp-segment
    kernels."""
    c = cases.hybrid_lagoon_case()
    g, o = run_both(c, 80, column_threads=column_threads)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    m = active_mask(c)
    assert np.abs(sg["hdknv"] - so["hdknv"])[m].max() <= 1e-4 * np.abs(so["hdknv"]).max()
    me = active_mask(c, node=False)
    assert np.abs(sg["hdenv"] - so["hdenv"])[me].max() <= 1e-4 * np.abs(so["hdenv"]).max()
    umax = np.abs(so["utlnv"]).max()
    assert np.abs(sg["utlnv"] - so["utlnv"]).max() <= 1e-3 * umax
    cmax = np.abs(so["conzv"]).max()
    assert np.abs(sg["conzv"] - so["conzv"]).max() <= TRACER_RTOL * cmax
    wmax = np.abs(so["wlnv"]).max()
    assert np.abs(sg["wlnv"] - so["wlnv"]).max() <= 2e-3 * wmax
    assert abs(g.info(0).volume - o.info().volume) <= 1e-6 * o.info().volume


@pytest.mark.parametrize("pinned", [False, True])
def test_whole_model_transfers(pinned):
    """shygpu_set_forcing_all / shygpu_enqueue / shygpu_get_levels (one copy
    for all basins on the transfer streams, nothing waited for until
    shygpu_sync) give, step for step, the bits of the per-basin calls with a
    wait after each; with pinned host buffers the copies overlap the steps."""
    cs = [cases.basin3d_case(nkn_target=n, nlv=6, seed=s, baroclinic=False, ts=False)
          for n, s in ((700, 21), (1200, 22))]
    rng = np.random.default_rng(3)
    winds = [[rng.normal(0, 1e-4, c["nkn"]).astype(np.float32) for c in cs] for _ in range(8)]
    a = shygpu.Model(cs)
    a.set_state_all()
    refs = []
    for w in winds:
        for b in range(len(cs)):
            a.set_forcing(b, tauxnv=w[b], tauynv=-w[b])
        a.run(1)
        refs.append(np.concatenate([a.get_state(b)["znv"] for b in range(len(cs))]))
    g = shygpu.Model(cs)
    g.set_state_all()
    lib = shygpu.lib()
    n = sum(c["nkn"] for c in cs)
    if pinned:
        import torch
        host = lambda a_: torch.from_numpy(np.ascontiguousarray(a_)).pin_memory()
        outs = [torch.zeros(n, dtype=torch.float32).pin_memory() for _ in winds]
        ptr = lambda t: t.data_ptr()
        get = lambda t: t.numpy()
    else:
        host = np.ascontiguousarray
        outs = [np.zeros(n, np.float32) for _ in winds]
        ptr = lambda t: t.ctypes.data
        get = lambda t: t
    keep = []
    for w, out in zip(winds, outs):
        tx = host(np.concatenate(w))
        ty = host(-np.concatenate(w))
        keep += [tx, ty]
        shygpu.check(lib.shygpu_set_forcing_all(g.h, ptr(tx), ptr(ty), None, None), "forcing")
        shygpu.check(lib.shygpu_enqueue(g.h, 1), "enqueue")
        shygpu.check(lib.shygpu_get_levels(g.h, ptr(out)), "levels")
    shygpu.check(lib.shygpu_sync(g.h), "sync")
    for out, ref in zip(outs, refs):
        assert np.array_equal(get(out), ref)
    # a state set afterwards and a checkpoint restored over pending copies
    # order with them
    ck = g.checkpoint()
    shygpu.check(lib.shygpu_enqueue(g.h, 1), "enqueue")
    shygpu.check(lib.shygpu_get_levels(g.h, ptr(outs[0])), "levels")
    g.restore(ck)
    shygpu.check(lib.shygpu_sync(g.h), "sync")
    assert np.array_equal(np.concatenate([g.get_state(b)["znv"] for b in range(len(cs))]), refs[-1])
    assert g.nbytes() > 0
    g.close()


def far_end_nodes(c, n=3):
    """Nodes at the basin's far end (largest x), mid-channel."""
    x, y = c["xgv"], c["ygv"]
    far = np.nonzero(x >= x.max() - 1.0)[0]
    return far[np.argsort(np.abs(y[far] - y.mean()))][:n]


def with_river(c, q_total, n=3):
    c = dict(c)
    rqv = np.zeros(c["nkn"], np.float32)
    rqv[far_end_nodes(c, n)] = q_total / n
    c["rqv"] = rqv
    return c


@pytest.mark.parametrize("shape", ["basin3d", "lagoon30"])
def test_river_discharge(small3d, shape):
    """A discharge at three nodes of the far end (set_mass_flux,
    bnd_routines.f90:1035-1140): it enters the zeta system, the vertical
    velocity through each layer's share (hydrodynamic.f90:1727) and the
    transport with the scalars' boundary values (concentration_omp.f90:
    805-813): a 5 degC fresh river into the baroclinic 3D basin (12 z-layers,
    thread-per-column kernels), a river of tracer 5 into the 30-layer
    lagoon (warp-segment kernels)."""
    if shape == "basin3d":
        c, n = with_river(small3d, 150.0), 120
        bounds = [(0, "tempv", 5.0), (1, "saltv", 0.0)]
    else:
        c, n = with_river(cases.lagoon_case(nkn_target=900, nlv=30), 80.0), 80
        bounds = [(2, "conzv", 5.0)]
    g = shygpu.Model(c)
    g.set_state(0)
    o = shyref.OracleModel(c)
    for what, f, v in bounds:
        for itr in range(3 if what == 2 else 1):
            b = np.full((c["nkn"], c["nlv"]), v, np.float32)
            g.set_bound_scalar(0, what, b, itr)
            o.set_bound_scalar(what, b, itr)
    g.run(n)
    o.run(n)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    me = active_mask(c, node=False)
    umax = max(np.abs(so["utlnv"][me]).max(), np.abs(so["vtlnv"][me]).max())
    assert np.abs(sg["utlnv"] - so["utlnv"])[me].max() <= 1e-3 * umax
    wmax = np.abs(so["wlnv"]).max()
    assert np.abs(sg["wlnv"] - so["wlnv"]).max() <= 2e-3 * wmax
    m = active_mask(c)
    for _, f, _ in bounds:
        a, b = sg[f], so[f]
        mm = m if a.ndim == 2 else np.broadcast_to(m, a.shape)
        rel = np.abs(a - b)[mm].max() / np.abs(b[mm]).max()
        assert rel <= TRACER_RTOL, (f, rel)
    assert abs(g.info(0).volume - o.info().volume) <= 1e-6 * o.info().volume
    # the river is felt: the water rose at its nodes, its tracer entered
    k = far_end_nodes(c)[0]
    f0 = bounds[0][1]
    now = so[f0][0] if f0 == "conzv" else so[f0]
    before = c[f0][0] if f0 == "conzv" else c[f0]
    assert abs(now[k, 0] - before[k, 0]) > 1e-3


@pytest.mark.parametrize("river", [False, True])
def test_conz3d_entry_reproduces_run_scalar(river):
    """shygpu_conz3d driven by the reference's scal3sh loop (clip, conz3d_omp,
    boundary values, per sub-step; concentration.f90:727-770) after
    shygpu_hydro gives the bits of the whole-phase shygpu_scalar; with a
    river, its cbound is what shygpu_set_bound_scalar gave the step."""
    c = cases.lagoon_case(nkn_target=900, nlv=12, ntracer=1)
    if river:
        c = with_river(c, 60.0)
    p = c["params"]
    m = shygpu.Model(c)
    m.set_state(0)
    cb = np.asarray(c["conzv"][0], np.float32)          # boundary values: the initial columns
    if river:
        cb = np.full_like(cb, 7.0)
        m.set_bound_scalar(0, 2, cb, 0)
    m.run(4)
    ck = m.checkpoint()
    m.hydro()
    m.scalar()
    ref = m.get_state(0)["conzv"][0]
    istot = m.info(0).istot
    m.restore(ck)
    cn = np.ascontiguousarray(m.get_state(0)["conzv"][0])
    m.hydro()
    lib = shygpu.lib()
    nlv = c["nlv"]
    difhv = np.ones((c["nel"], nlv), np.float32)
    difv = np.ascontiguousarray(c["difv"], np.float32)
    cbp = np.ascontiguousarray(cb).ctypes.data if river else None
    bnd = c["bnd_index"] > 0
    assert istot >= 1
    for isact in range(1, istot + 1):
        cn[cn < 1e-15] = 0.0
        shygpu.check(lib.shygpu_conz3d(
            m.h, 0, cn.ctypes.data, None, float(p["dt"]), float(p["chpar"]), difhv.ctypes.data,
            difv.ctypes.data, float(p["difmol"]), cbp, 0, 0, None, None, None, 0.0, None, 0.0, None,
            0.0, None, float(p["azpar"]), float(p["adpar"]), float(p["aapar"]), istot, isact, nlv, nlv),
            "conz3d")
        cn[bnd] = cb[bnd]
    assert np.array_equal(cn, ref)
    if river:
        assert cn[far_end_nodes(c)[0], 0] > 1e-3


def test_conz3d_entry_source_terms():
    """shygpu_conz3d with scalar nudging, settling and loading
    (concentration_omp.f90:496, 694-709; conz3d_nodes :816-833), driven by
    the scal3sh loop for one step of the lagoon, against the oracle's step
    with the same terms; the load that deposition took comes back in load."""
    from test_oracle_properties import node_areas
    c = cases.lagoon_case(nkn_target=900, nlv=12, ntracer=1)
    p = c["params"]
    nkn, nlv, dt = c["nkn"], c["nlv"], float(p["dt"])
    rng = np.random.default_rng(11)
    c0 = np.asarray(c["conzv"][0], np.float32)
    cobs = (c0 + rng.uniform(1.0, 5.0, c0.shape)).astype(np.float32)
    rtauv = np.full((nkn, nlv), 1.0 / 1800.0, np.float32)
    wsinkv = rng.uniform(0.0, 2e-4, (nkn, nlv + 1)).astype(np.float32)
    mass = node_areas(c) * float(c0.mean())
    load = (rng.uniform(-0.5, 0.01, (nkn, nlv)) * mass / dt).astype(np.float32)
    o = shyref.OracleModel(c)
    o.set_scalar_terms(0, cobs=cobs, robs=1.0, rtauv=rtauv, wsink=1.0, wsinkv=wsinkv, rload=1.0, load=load)
    o.run(1)
    so = o.state()["conzv"][0]
    m = shygpu.Model(c)
    m.set_state(0)
    ck = m.checkpoint()
    m.hydro()
    m.scalar()
    plain = m.get_state(0)["conzv"][0]
    istot = m.info(0).istot
    assert istot == o.info().istot
    m.restore(ck)
    m.hydro()
    lib = shygpu.lib()
    cn = c0.copy()                                  # c0 keeps the boundary values
    difhv = np.ones((c["nel"], nlv), np.float32)
    difv = np.ascontiguousarray(c["difv"], np.float32)
    bnd = c["bnd_index"] > 0
    gl = load.copy()
    for isact in range(1, istot + 1):
        cn[cn < 1e-15] = 0.0
        shygpu.check(lib.shygpu_conz3d(
            m.h, 0, cn.ctypes.data, None, dt, float(p["chpar"]), difhv.ctypes.data, difv.ctypes.data,
            float(p["difmol"]), None, 0, 0, None, None, cobs.ctypes.data, 1.0, rtauv.ctypes.data, 1.0,
            wsinkv.ctypes.data, 1.0, gl.ctypes.data, float(p["azpar"]), float(p["adpar"]),
            float(p["aapar"]), istot, isact, nlv, nlv), "conz3d")
        cn[bnd] = c0[bnd]
    cmax = np.abs(so).max()
    act = active_mask(c)
    assert np.abs(cn - so)[act].max() <= TRACER_RTOL * cmax
    assert np.abs(cn - plain)[act].max() > 10 * TRACER_RTOL * cmax
    lo = o.load()
    assert np.abs(gl - lo)[act].max() <= TRACER_RTOL * np.abs(load).max()
    assert np.abs(gl - load)[act].max() > 10 * TRACER_RTOL * np.abs(load).max()


@pytest.mark.parametrize("ihwadv", [1, 2])
@pytest.mark.parametrize("column_threads", [1, 0])
def test_vertical_momentum_advection(ihwadv, column_threads):
    """ilin = 0 with vertical advection of momentum (set_advective,
    explicit.f90:776-833): upwind (1) or centred (2) from the old w at the
    element's vertices, in the thread-per-column and warp-segment kernels."""
    c = with_params(cases.basin3d_case(nkn_target=1500, nlv=12, dt=60.0, wind=5.0), ilin=0, ihwadv=ihwadv)
    g, o = run_both(c, 120, column_threads=column_threads)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    me = active_mask(c, node=False)
    umax = np.abs(so["utlnv"][me]).max()
    assert np.abs(sg["utlnv"] - so["utlnv"])[me].max() <= 1e-3 * umax
    flat = shyref.OracleModel(with_params(c, ihwadv=0))
    flat.run(120)
    assert np.abs(flat.state()["utlnv"] - so["utlnv"])[me].max() > 10e-3 * umax


@pytest.mark.parametrize("shape", ["basin3d", "lagoon30"])
def test_horizontal_viscosity_and_diffusion(small3d, shape):
    """Horizontal viscosity of momentum (ahpar, set_diff_horizontal,
    explicit.f90:389-493) and horizontal diffusion of the scalars (thpar,
    shpar, chpar: the wdifhv terms of conz3d_element) against the oracle,
    through the thread-per-column kernels (12 z-layers) and the warp-segment
    kernels (30 sigma layers)."""
    if shape == "basin3d":
        c, n, fields = with_params(small3d, ahpar=50.0, thpar=20.0, shpar=20.0), 120, ("tempv", "saltv")
    else:
        c, n, fields = with_params(cases.lagoon_case(nkn_target=900, nlv=30), ahpar=20.0, chpar=10.0), 80, ("conzv",)
    g, o = run_both(c, n)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    me = active_mask(c, node=False)
    umax = max(np.abs(so["utlnv"][me]).max(), np.abs(so["vtlnv"][me]).max())
    for f in ("utlnv", "vtlnv"):
        assert np.abs(sg[f] - so[f])[me].max() <= 1e-3 * umax, f
    m = active_mask(c)
    for f in fields:
        a, b = sg[f], so[f]
        mm = m if a.ndim == 2 else np.broadcast_to(m, a.shape)
        rel = np.abs(a - b)[mm].max() / np.abs(b[mm]).max()
        assert rel <= TRACER_RTOL, (f, rel)
    # the terms act: the run differs from one without them
    c0 = with_params(c, ahpar=0.0, thpar=0.0, shpar=0.0, chpar=0.0)
    o0 = shyref.OracleModel(c0)
    o0.run(n)
    assert np.abs(o0.state()["utlnv"] - so["utlnv"])[me].max() > 1e-3 * umax
    s0 = o0.state()
    f = fields[0]
    assert np.abs(s0[f] - so[f]).max() > 1e-3 * np.abs(so[f]).max()


@pytest.mark.parametrize("ilin", [1, 0])
def test_staged_column_kernel_equals_in_place(small3d, ilin):
    """The thread-per-column kernel with its columns staged through shared
    memory (the default without Coriolis) against the same kernel reading
    its columns in place: the same arithmetic, so the same state up to the
    compiler's choice of fused multiply-adds in either instance."""
    c = dict(small3d)
    c["params"] = dict(c["params"], ilin=ilin)
    states = []
    for staged in (1, 0):
        g = shygpu.Model(c)
        g.set_option("column_staged", staged)
        assert g.get_option("column_staged") == staged
        g.set_state(0)
        g.run(60)
        states.append(g.get_state(0))
    for f in ("znv", "utlnv", "vtlnv", "tempv", "saltv"):
        a, b = states[0][f], states[1][f]
        assert np.abs(a - b).max() <= 1e-6 * max(np.abs(b).max(), 1e-6), f


@pytest.mark.parametrize("column_threads", [1, 0])
def test_sigma_baroclinic(column_threads):
    """Baroclinic pressure on sigma layers (set_barocl_new_interface with
    bsigadjust): a stratified basin over 5-60 m bumps under wind, with noise
    in the temperature, on both column-kernel forms."""
    c = cases.stratified_basin_case(sigma=True, wind=8.0, noise=0.2)
    g, o = run_both(c, 120, column_threads=column_threads)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    m, me = active_mask(c), active_mask(c, node=False)
    umax = max(np.abs(so["utlnv"][me]).max(), np.abs(so["vtlnv"][me]).max())
    for f in ("utlnv", "vtlnv"):
        assert np.abs(sg[f] - so[f])[me].max() <= 1e-3 * umax, f
    rel = np.abs(sg["tempv"] - so["tempv"])[m].max() / np.abs(so["tempv"][m]).max()
    assert rel <= TRACER_RTOL, rel
    assert np.abs(sg["rhov"] - so["rhov"])[m].max() <= 1e-3


def test_hybrid_baroclinic():
    """Hybrid layers (sigma layers down to hsigma, z-layers below) with T/S
    and the baroclinic pressure."""
    c = cases.hybrid_lagoon_case()
    nkn, nlv = c["nkn"], c["nlv"]
    rng = np.random.default_rng(21)
    c["tempv"] = (18.0 - 0.3 * np.arange(nlv)[None, :] + 0.1 * rng.standard_normal((nkn, nlv))).astype(np.float32)
    c["saltv"] = (34.0 + 0.1 * np.arange(nlv)[None, :] + 0.05 * rng.standard_normal((nkn, nlv))).astype(np.float32)
    c["params"] = dict(c["params"], ibarcl=1, itemp=1, isalt=1)
    g, o = run_both(c, 80)
    sg, so = g.get_state(0), o.state()
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    m, me = active_mask(c), active_mask(c, node=False)
    umax = max(np.abs(so["utlnv"][me]).max(), np.abs(so["vtlnv"][me]).max())
    assert np.abs(sg["utlnv"] - so["utlnv"])[me].max() <= 1e-3 * umax
    for f in ("tempv", "saltv"):
        rel = np.abs(sg[f] - so[f])[m].max() / np.abs(so[f][m]).max()
        assert rel <= TRACER_RTOL, (f, rel)
