"""Flux boundaries and point sources in the oracle (set_mass_flux,
bnd_routines.f90:1035-1140): a discharge rqv at a node enters the zeta
system (system_add_rhs), is spread over the node's layers by their volume
(mfluxv) for the vertical velocity (hydrodynamic.f90:1727) and brings the
scalars' boundary values into the transport (concentration_omp.f90:805-813).
In a basin closed everywhere else the water gained is the volume discharged
and the tracer mass gained is that volume times the inflow concentration,
to FP64 round-off."""
import numpy as np
import pytest

import shyref
from shygpu import cases
from test_oracle_properties import node_areas


def river(c, q_total, nodes):
    c = dict(c)
    rqv = np.zeros(c["nkn"], np.float32)
    rqv[nodes] = q_total / len(nodes)
    c["rqv"] = rqv
    return c


def closed(c):
    c = dict(c)
    c["bnd_index"] = np.zeros_like(c["bnd_index"])
    c["tide"] = np.zeros((0, 1, 4), np.float32)
    return c


def far_end_nodes(c, n=3):
    """Interior-edge nodes at the basin's far end (largest x), mid-channel."""
    x, y = c["xgv"], c["ygv"]
    far = np.nonzero(x >= x.max() - 1.0)[0]
    return far[np.argsort(np.abs(y[far] - y.mean()))][:n]


@pytest.mark.parametrize("shape", ["lagoon_sigma", "basin3d_z"])
def test_discharge_fills_a_closed_basin_with_its_volume_and_mass(shape):
    if shape == "lagoon_sigma":
        c = closed(cases.lagoon_case(nkn_target=900, nlv=12))
        c["conzv"] = np.zeros_like(c["conzv"])
        what, field, cin = 2, "conzv", 5.0
    else:
        c = closed(cases.basin3d_case(nkn_target=1500, nlv=12, baroclinic=False))
        what, field, cin = 0, "tempv", 5.0
    q, steps = 80.0, 40
    c = river(c, q, far_end_nodes(c))
    A = node_areas(c)
    o = shyref.OracleModel(c)
    bound = np.full((c["nkn"], c["nlv"]), cin, np.float32)
    for itr in range(max(int(c["params"]["nconz"]), 1) if what == 2 else 1):
        o.set_bound_scalar(what, bound, itr)

    def budget(s):
        f = s[field] if field != "conzv" else s["conzv"][0]
        return (s["hdknv"] * A).sum(), (f * s["hdknv"] * A).sum()

    v0, m0 = budget(o.state())
    o.run(steps)
    s = o.state()
    v1, m1 = budget(s)
    dvol = float(c["rqv"].astype(np.float64).sum()) * c["params"]["dt"] * steps   # rqv is FP32
    # the layer fractions of sigma layers are FP32 (hldv = -1/nlv) and sum to 1
    # within 3e-8, so the layers hold the gained water to that accuracy
    assert abs((v1 - v0) - dvol) <= 1e-7 * dvol, (v1 - v0, dvol)
    assert abs((m1 - m0) - cin * dvol) <= 1e-10 * cin * dvol + 1e-12 * abs(m0), (m1 - m0, cin * dvol)
    # the discharge reaches the water column: w is not zero below the river nodes
    k = far_end_nodes(c)[0]
    assert np.abs(s["wlnv"][k, 1:c["ilhkv"][k]]).max() > 0.0
    assert s["znv"].max() > 0.0


def test_discharge_splits_over_layers_by_volume():
    """mfluxv(l,k) = rqv(k) * vol(l,k) / sum_l vol(l,k): on a still basin the
    vertical velocity at the node's interfaces carries the layers below
    their share of the inflow that rises through them."""
    c = closed(cases.lagoon_case(nkn_target=900, nlv=6))
    c["tauxnv"] = np.zeros(c["nkn"], np.float32)
    k = far_end_nodes(c, 1)
    c = river(c, 10.0, k)
    o = shyref.OracleModel(c)
    o.run(1)
    s = o.state()
    assert np.all(np.isfinite(s["wlnv"]))
    assert s["znv"][k[0]] > 0.0
