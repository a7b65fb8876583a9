"""Analytic and size-independent properties of the oracle's step: still
water stays still; a closed basin keeps its volume and every tracer's mass
while wind moves the water; a standing tide, an inertial oscillation and
vertical diffusion follow their closed forms; upwind transport makes no
new extrema."""
import numpy as np
import pytest

import shyref
from shygpu import cases


def node_areas(c):
    ev = shyref.set_ev(c)
    areafv = 12.0 * ev[:, 9] / 3.0
    A = np.zeros((c["nkn"], c["nlv"]))
    for e in range(c["nel"]):
        for k in c["nen3v"][e] - 1:
            A[k, :c["ilhv"][e]] += areafv[e]
    return A


def test_still_water_stays_still():
    c = cases.channel_case()
    c["tide"] = np.zeros_like(c["tide"])
    o = shyref.OracleModel(c)
    o.run(100)
    s = o.state()
    assert np.abs(s["znv"]).max() == 0.0 and np.abs(s["utlnv"]).max() == 0.0


@pytest.mark.parametrize("itvd,itvdv", [(0, 0), (1, 0), (2, 1)])
def test_closed_basin_conserves_volume_and_tracer_mass(itvd, itvdv):
    """Every horizontal flux leaves one vertex and enters another, and every
    vertical flux is shared by the two layers of its interface, with the
    upwind scheme and with both TVD forms alike.  The gradient TVD form
    (itvd 1) undershoots below zero in places, and scal3sh's clip of
    concentrations below 1e-15 (concentration.f90:736-740) then adds a
    little mass: there the budget may only grow, by round-off sizes."""
    c = cases.lagoon_case(nkn_target=900, nlv=12)
    if itvd or itvdv:
        c["params"] = dict(c["params"], itvd=itvd, itvdv=itvdv, aapar=0.0)
    c["bnd_index"] = np.zeros_like(c["bnd_index"])
    c["tide"] = np.zeros((0, 2, 4), np.float32)
    c["tauxnv"] = np.full(c["nkn"], 2e-4, np.float32)
    A = node_areas(c)

    def budget(s):
        return (s["hdknv"] * A).sum(), [(s["conzv"][t] * s["hdknv"] * A).sum() for t in range(s["conzv"].shape[0])]

    o = shyref.OracleModel(c)
    v0, m0 = budget(o.state())
    o.run(40)
    v1, m1 = budget(o.state())
    assert np.abs(o.state()["znv"]).max() > 0.01          # the wind has moved the water
    assert abs(v1 / v0 - 1.0) < 1e-12
    for a, b in zip(m0, m1):
        if itvd == 1:
            assert -1e-12 < b / a - 1.0 < 1e-9
        else:
            assert abs(b / a - 1.0) < 1e-12


def test_tidal_channel_matches_the_standing_wave():
    """A closed channel of length L forced by a tide at its mouth holds the
    standing long wave z(x) = A cos(k (L - x)) / cos(k L), k = omega /
    sqrt(g H): with k L = 0.9 the tide at the closed end is 1/cos(0.9) = 1.61
    times the mouth's.  Bottom friction lowers that a little; the oracle
    must be within 5% after eight periods of spin-up."""
    import math
    H, A = 10.0, 0.1
    k = (2 * math.pi / cases.M2_PERIOD) / math.sqrt(9.81 * H)
    L = 0.9 / k
    c = cases.channel_case(nx=91, ny=4, lx=L, ly=3e3, ampli=A, depth=H, ddepth=0.0)
    c["params"] = dict(c["params"], dt=120.0)
    o = shyref.OracleModel(c)
    per = int(cases.M2_PERIOD / 120.0)
    o.run(8 * per)
    x = c["xgv"]
    far, near = x > 0.97 * L, x < 0.03 * L
    a_far = a_near = 0.0
    for _ in range(per):
        o.run(1)
        z = o.state()["znv"]
        a_far = max(a_far, float(np.abs(z[far]).max()))
        a_near = max(a_near, float(np.abs(z[near]).max()))
    ratio = a_far / a_near
    assert abs(ratio / (1.0 / math.cos(0.9)) - 1.0) < 0.05, ratio


def test_inertial_oscillation_with_quadratic_friction():
    """Coriolis and bottom friction (hydro_intern, chezy.f90 ireib 5) against
    their analytic solution: a uniform flow in the middle of a wide, flat
    basin turns clockwise at the inertial frequency f (pointing south,
    west, north a quarter, half and three quarters of 2 pi / f later) while
    quadratic friction slows it as |U|(t) = U0 / (1 + cd U0 t / h^2)."""
    import math
    f, h, u0 = 1.0e-4, 20.0, 0.1
    c = cases.channel_case(nx=31, ny=31, lx=2.0e6, ly=2.0e6, ampli=0.0, depth=h, ddepth=0.0)
    c["bnd_index"] = np.zeros_like(c["bnd_index"])
    c["tide"] = np.zeros((0, 1, 4), np.float32)
    c["fcorv"] = np.full(c["nel"], f, np.float32)
    c["utlnv"] = np.full((c["nel"], 1), u0 * h, np.float32)
    c["params"] = dict(c["params"], dt=60.0)
    cd = float(c["params"]["czdef"])
    xe = c["xgv"][c["nen3v"] - 1].mean(1)
    ye = c["ygv"][c["nen3v"] - 1].mean(1)
    mid = int(np.argmin((xe - 1.0e6) ** 2 + (ye - 1.0e6) ** 2))
    o = shyref.OracleModel(c)
    period = 2 * math.pi / f
    done = 0
    for q, angle in ((1, -90.0), (2, 180.0), (3, 90.0)):
        n = int(round(q * period / 4 / 60.0))
        o.run(n - done)
        done = n
        s = o.state()
        U, V = float(s["utlnv"][mid, 0]), float(s["vtlnv"][mid, 0])
        d = (math.degrees(math.atan2(V, U)) - angle + 180.0) % 360.0 - 180.0
        assert abs(d) < 1.0, (q, d)
        t = n * 60.0
        expect = u0 * h / (1.0 + cd * u0 * h * t / h ** 2)
        assert abs(math.hypot(U, V) / expect - 1.0) < 0.01, (q, math.hypot(U, V), expect)


def test_vertical_diffusion_spreads_as_the_heat_equation():
    """conz3d's implicit vertical diffusion (concentration_omp.f90:566-611,
    conz3d_nodes) on a still, flat column of 32 sigma layers: a Gaussian
    tracer's variance grows by 2 K t, as the diffusion equation says (the
    implicit scheme keeps that moment relation exactly on a uniform grid),
    and its mass stays."""
    nlv, H, K, s0, zc = 32, 16.0, 1e-3, 1.0, 8.0
    c = cases.lagoon_case(nkn_target=300, nlv=nlv, ntracer=1)
    c["hm3v"] = np.full_like(c["hm3v"], H)
    c["tide"] = np.zeros_like(c["tide"])
    c["tauxnv"] = np.zeros(c["nkn"], np.float32)
    c["difv"] = np.full((c["nkn"], nlv + 1), K, np.float32)
    dz = H / nlv
    zmid = (np.arange(nlv) + 0.5) * dz
    prof = np.exp(-(zmid - zc) ** 2 / (2 * s0 ** 2))
    c["conzv"] = np.repeat(prof[None, None, :], c["nkn"], axis=1).astype(np.float32)
    c["params"] = dict(c["params"], difmol=0.0, chpar=0.0)
    o = shyref.OracleModel(c)
    k = int(np.argmin(np.abs(c["xgv"] - c["xgv"].mean()) + np.abs(c["ygv"] - c["ygv"].mean())))

    def moments(col):
        m0 = col.sum()
        m1 = (col * zmid).sum() / m0
        return m0, (col * (zmid - m1) ** 2).sum() / m0

    m0a, v0 = moments(o.state()["conzv"][0][k])
    n = 40
    o.run(n)
    m0b, v1 = moments(o.state()["conzv"][0][k])
    t = n * float(c["params"]["dt"])
    assert abs((v1 - v0) / (2 * K * t) - 1.0) < 1e-3
    assert abs(m0b / m0a - 1.0) < 1e-9


@pytest.mark.parametrize("itvd", [0, 2])
def test_transport_makes_no_new_extrema(itvd):
    """Upwind transport (itvd 0) and the TVD scheme with the upwind point
    (itvd 2, tvd_get_upwind_c, tvd_admin.f90:608-671) keep a tracer inside
    its initial range over 600 steps of the tidal lagoon (no horizontal
    diffusion, whose weights are not positive on every triangle).  The
    gradient form (itvd 1) is not bounded in the reference either: its
    far-upwind value is the node gradient extrapolated along the side
    (tvd_fluxes :790-795), which can lie outside the local range."""
    c = cases.lagoon_case(nkn_target=900, nlv=6, ntracer=1)
    c["params"] = dict(c["params"], chpar=0.0, itvd=itvd)
    c0 = np.asarray(c["conzv"][0])
    lo, hi = c0.min(), c0.max()
    o = shyref.OracleModel(c)
    act = np.arange(c["nlv"])[None, :] < c["ilhkv"][:, None]
    moved = 0.0
    for _ in range(20):
        o.run(30)
        cn = o.state()["conzv"][0][act]
        assert cn.min() >= lo - 1e-12 * hi and cn.max() <= hi * (1 + 1e-12)
        moved = max(moved, np.abs(cn - c0[act]).max())
    assert moved > 0.1 * hi
