"""The oracle's horizontal TVD transport (itvd = 1: tvd_grad_3d and
tvd_fluxes, tvd_admin.f90:478-838, in conz3d_element,
concentration_omp.f90:675-686) against the properties the scheme is built
for, on the CPU: a uniform tracer stays uniform, extrema are not created,
and a tracer keeps more of its variance than with upwind fluxes."""
import numpy as np

import shyref
from shygpu import cases


def lagoon(itvd, conz=None):
    c = cases.lagoon_case(nkn_target=900, nlv=12)
    c["params"] = dict(c["params"], itvd=itvd)
    if conz is not None:
        c["conzv"] = np.full_like(c["conzv"], conz)
    return c


def test_uniform_tracer_stays_uniform():
    o = shyref.OracleModel(lagoon(1, conz=5.0))
    o.run(40)
    cz = o.state()["conzv"]
    act = np.arange(12)[None, :] < lagoon(1)["ilhkv"][:, None]
    # to the consistency of the transports with the volume change (the zeta
    # solve's tolerance, in FP32 state): upwind shows the same 3e-7
    assert np.abs(cz[:, act] - 5.0).max() <= 1e-6


def test_tvd_keeps_bounds_and_variance():
    c0, c1 = lagoon(0), lagoon(1)
    lo, hi = float(c1["conzv"].min()), float(c1["conzv"].max())
    out = {}
    for itvd, c in ((0, c0), (1, c1)):
        o = shyref.OracleModel(c)
        o.run(80)
        out[itvd] = o.state()["conzv"]
    act = np.arange(12)[None, :] < c1["ilhkv"][:, None]
    tol = 1e-3 * (hi - lo)
    assert out[1][:, act].min() >= lo - tol and out[1][:, act].max() <= hi + tol
    for t in range(out[1].shape[0]):
        assert np.var(out[1][t][act]) > np.var(out[0][t][act])
    # the fluxes differ from upwind by far more than rounding
    assert np.abs(out[1] - out[0]).max() > 1e-2 * (hi - lo)


def test_vertical_tvd_keeps_more_stratification():
    """itvdv = 1 (vertical_flux_ie, tvd_admin.f90:930-1019, with aapar = 0
    as the reference requires): a uniform tracer stays uniform, and on the
    wind-driven stratified basin the temperature and salinity columns keep
    more of their vertical variance than with upwind fluxes."""
    var = {}
    for itvdv in (0, 1):
        c = cases.basin3d_case(nkn_target=1500, nlv=12)
        c["params"] = dict(c["params"], itvdv=itvdv, aapar=0.0)
        o = shyref.OracleModel(c)
        o.run(200)
        s, il = o.state(), c["ilhkv"]
        var[itvdv] = [np.mean([np.var(s[f][k, :il[k]]) for k in range(c["nkn"]) if il[k] > 1])
                      for f in ("tempv", "saltv")]
    assert var[1][0] > 1.1 * var[0][0] and var[1][1] > 1.1 * var[0][1], var
    c = lagoon(0, conz=5.0)
    c["params"] = dict(c["params"], itvdv=1, aapar=0.0)
    o = shyref.OracleModel(c)
    o.run(40)
    act = np.arange(12)[None, :] < c["ilhkv"][:, None]
    assert np.abs(o.state()["conzv"][:, act] - 5.0).max() <= 1e-6


def test_upwind_point_tvd():
    """itvd = 2 (tvd_upwind_init_elem and tvd_get_upwind_c,
    tvd_admin.f90:361-476, 608-671): the limiter's upwind difference from
    the value at the point beyond the upwind vertex.  A uniform tracer stays
    uniform; the tracers keep more variance than with upwind fluxes and stay
    within their initial range."""
    c = lagoon(2, conz=5.0)
    o = shyref.OracleModel(c)
    o.run(40)
    act = np.arange(12)[None, :] < c["ilhkv"][:, None]
    assert np.abs(o.state()["conzv"][:, act] - 5.0).max() <= 1e-6
    out = {}
    for itvd in (0, 2):
        o = shyref.OracleModel(lagoon(itvd))
        o.run(80)
        out[itvd] = o.state()["conzv"]
    c2 = lagoon(2)
    lo, hi = float(c2["conzv"].min()), float(c2["conzv"].max())
    tol = 1e-3 * (hi - lo)
    assert out[2][:, act].min() >= lo - tol and out[2][:, act].max() <= hi + tol
    for t in range(out[2].shape[0]):
        assert np.var(out[2][t][act]) > np.var(out[0][t][act])
