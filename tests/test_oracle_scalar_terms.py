"""conz3d_omp's source terms in the oracle (concentration_omp.f90:92-98):
nudging to observations (:694-709), settling (:496) and loading
(conz3d_nodes :816-833), each pinned on a still, flat basin where the
transport reduces to a closed form."""
import numpy as np

import shyref
from shygpu import cases
from test_oracle_properties import node_areas


def still_case(nlv=4, H=8.0, c0=2.0):
    c = cases.lagoon_case(nkn_target=300, nlv=nlv, ntracer=1)
    c["hm3v"] = np.full_like(c["hm3v"], H)
    c["tide"] = np.zeros_like(c["tide"])
    c["tauxnv"] = np.zeros(c["nkn"], np.float32)
    c["difv"] = np.zeros((c["nkn"], nlv + 1), np.float32)
    c["conzv"] = np.full((1, c["nkn"], nlv), c0, np.float32)
    c["params"] = dict(c["params"], difmol=0.0, chpar=0.0, aapar=0.0, adpar=0.0)
    return c


def test_nudging_relaxes_explicitly_to_the_observations():
    c = still_case()
    nkn, nlv, dt, c0 = c["nkn"], c["nlv"], float(c["params"]["dt"]), 2.0
    tau = 3600.0
    cobs = np.full((nkn, nlv), 5.0, np.float32)
    rtauv = np.full((nkn, nlv), 1.0 / tau, np.float32)
    o = shyref.OracleModel(c)
    o.set_scalar_terms(0, cobs=cobs, robs=1.0, rtauv=rtauv)
    n = 10
    o.run(n)
    cn = o.state()["conzv"][0]
    inner = c["bnd_index"] <= 0
    # an = 0: c <- c + dt (cobs - c) / tau each step
    want = 5.0 + (c0 - 5.0) * (1.0 - dt * np.float32(1.0 / tau)) ** n
    assert np.abs(cn[inner] - want).max() < 1e-6 * abs(want)


def test_settling_moves_mass_down_and_keeps_it():
    c = still_case()
    nkn, nlv, dt, c0 = c["nkn"], c["nlv"], float(c["params"]["dt"]), 2.0
    ws = float(np.float32(1e-3))            # the oracle reads wsinkv in FP32
    wsinkv = np.full((nkn, nlv + 1), ws, np.float32)
    o = shyref.OracleModel(c)
    o.set_scalar_terms(0, wsink=1.0, wsinkv=wsinkv)
    o.run(1)
    cn = o.state()["conzv"][0]
    inner = c["bnd_index"] <= 0
    hl = 8.0 / nlv
    # explicit upwind (aapar = 0): the surface layer drains at ws, the bottom
    # layer fills at ws, the layers between pass on what they receive
    assert np.abs(cn[inner, 0] - c0 * (1 - dt * ws / hl)).max() < 1e-9
    assert np.abs(cn[inner, 1:-1] - c0).max() < 1e-9
    assert np.abs(cn[inner, -1] - c0 * (1 + dt * ws / hl)).max() < 1e-9
    A = node_areas(c)
    m0 = (A * hl * c0).sum()
    assert abs((A * hl * cn).sum() / m0 - 1.0) < 1e-9


def test_loading_adds_sources_and_decays_sinks():
    c = still_case()
    nkn, nlv, dt, c0 = c["nkn"], c["nlv"], float(c["params"]["dt"]), 2.0
    A = node_areas(c)
    hl = 8.0 / nlv
    M0 = A * hl * c0                                   # node-layer mass
    rng = np.random.default_rng(3)
    # sources up to 1% of the mass per step, sinks up to twice the mass
    frac = rng.uniform(-2.0, 0.01, (nkn, nlv))
    load = (frac * M0 / dt).astype(np.float32)
    o = shyref.OracleModel(c)
    o.set_scalar_terms(0, rload=1.0, load=load)
    o.run(1)
    cn = o.state()["conzv"][0]
    inner = c["bnd_index"] <= 0
    L = load.astype(np.float64)
    want = np.where(L >= 0, M0 + dt * L, M0 * np.exp(dt * L / M0)) / (A * hl)
    assert np.abs(cn - want)[inner].max() < 1e-9 * c0
    # the sinks' load is cut to the decay that was taken
    got = o.load()
    cut = np.where(L < 0, -M0 * (1 - np.exp(dt * L / M0)) / dt, L)
    assert np.abs(got - cut)[inner].max() < 1e-9 * np.abs(L).max()


def test_fast_settling_sub_steps_the_transport():
    """Settling enters the stability index (conzstab, concentration.f90:1860):
    a settling speed that crosses more than one surface layer per step
    splits the step into istot sub-steps, and the surface layer drains by
    (1 - dt ws / (istot h)) per sub-step."""
    c = still_case()
    nkn, nlv, dt, c0 = c["nkn"], c["nlv"], float(c["params"]["dt"]), 2.0
    ws = float(np.float32(0.15))
    o = shyref.OracleModel(c)
    o.set_scalar_terms(0, wsink=1.0, wsinkv=np.full((nkn, nlv + 1), ws, np.float32))
    o.run(1)
    istot = o.info().istot
    hl = 8.0 / nlv
    assert istot >= 1 + int(dt * ws / hl)
    cn = o.state()["conzv"][0]
    inner = c["bnd_index"] <= 0
    want = c0 * (1 - dt * ws / (istot * hl)) ** istot
    assert np.abs(cn[inner, 0] - want).max() < 1e-9


def test_strong_nudging_sub_steps_the_transport():
    """Nudging enters the stability index as a source flux (conzstab,
    concentration.f90:1985): a relaxation faster than the step splits it
    into istot sub-steps, each relaxing explicitly by dt rtau / istot."""
    c = still_case()
    nkn, nlv, dt, c0 = c["nkn"], c["nlv"], float(c["params"]["dt"]), 2.0
    r = float(np.float32(2.5 / dt))
    o = shyref.OracleModel(c)
    o.set_scalar_terms(0, cobs=np.full((nkn, nlv), 5.0, np.float32), robs=1.0,
                       rtauv=np.full((nkn, nlv), r, np.float32))
    o.run(1)
    istot = o.info().istot
    assert istot == 1 + int(dt * r)
    cn = o.state()["conzv"][0]
    inner = c["bnd_index"] <= 0
    want = 5.0 + (c0 - 5.0) * (1 - dt * r / istot) ** istot
    assert np.abs(cn[inner] - want).max() < 1e-9


def test_settling_keeps_tracer_mass_in_a_moving_closed_basin():
    """Settling only moves mass between layers: the surface and the bottom
    interfaces carry none (wl(0) unused, wl(ilevel) = 0,
    concentration_omp.f90:503-515), so a closed basin under wind keeps its
    tracer mass while the tracer settles."""
    c = cases.lagoon_case(nkn_target=900, nlv=8, ntracer=1)
    c["bnd_index"] = np.zeros_like(c["bnd_index"])
    c["tide"] = np.zeros((0, 2, 4), np.float32)
    c["tauxnv"] = np.full(c["nkn"], 2e-4, np.float32)
    nkn, nlv = c["nkn"], c["nlv"]
    A = node_areas(c)
    o = shyref.OracleModel(c)
    o.set_scalar_terms(0, wsink=1.0, wsinkv=np.full((nkn, nlv + 1), 1e-3, np.float32))

    def mass(s):
        return (s["conzv"][0] * s["hdknv"] * A).sum(), (s["conzv"][0][:, 0] * s["hdknv"][:, 0] * A[:, 0]).sum()

    m0, top0 = mass(o.state())
    o.run(40)
    m1, top1 = mass(o.state())
    assert abs(m1 / m0 - 1.0) < 1e-12
    assert top1 < 0.9 * top0                              # the surface layer has drained
