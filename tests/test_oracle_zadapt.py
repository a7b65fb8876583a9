"""The oracle's z-adaptive surface layers (nzadapt > 1; zadaptutil.f90
compute_rzmov_info, compute_nadapt_info, compute_zadaptive_info and their
use in setdepth, elems_dealing.f90:1014-1110) on a tidal shelf whose three
1 m surface layers the tide would empty, checked on the CPU:

* plain z-layers lose the first layer at low water (setdepth stops), the
  z-adaptive ones stretch and every layer keeps a positive thickness;
* an element's layers still add up to its total depth hev + zmed;
* layers below the deepest one the level can reach stay at their nominal
  thickness; with nzadapt = nlv every layer above the bottom one is its
  nominal thickness times the mean of (h + z) / h over the vertices (z-star);
* a closed, wind-driven basin keeps its volume and its tracer mass.
"""
import numpy as np
import pytest

import shyref
from shygpu import cases

from test_oracle_properties import node_areas

LOW_WATER = 200          # steps of 60 s: just past the quarter period of M2


def active(c, node=False):
    il = c["ilhkv"] if node else c["ilhv"]
    return np.arange(c["nlv"])[None, :] < il[:, None]


def test_plain_z_layers_lose_the_surface_layer():
    c = cases.shelf_case(nzadapt=0)
    o = shyref.OracleModel(c)
    with pytest.raises(RuntimeError, match="SHY_EDEPTH"):
        o.run(LOW_WATER)


@pytest.mark.parametrize("nzadapt", [2, 3, 9])
def test_layers_stretch_and_add_up_to_the_depth(nzadapt):
    c = cases.shelf_case(nzadapt=nzadapt)
    o = shyref.OracleModel(c)
    o.run(LOW_WATER)
    s = o.state()
    assert s["znv"].min() < -1.2                     # below the first layers' bottoms
    me, mk = active(c), active(c, node=True)
    assert (s["hdenv"][me] > 0).all() and (s["hdknv"][mk] > 0).all()
    assert (s["hdenv"][~me] == 0).all()
    hev = c["hm3v"].astype(np.float64).mean(axis=1)
    zmed = s["zenv"].mean(axis=1)
    np.testing.assert_allclose((s["hdenv"] * me).sum(axis=1), hev + zmed, rtol=1e-12)


def test_deep_layers_keep_their_nominal_thickness():
    """With nzadapt = 3 on layers 1, 1, 1, 2, 3, ... m the threshold factor
    is hlv(2) / (hlv(3) - hlv(2)) = 2 and layer l + 1 follows the level
    while z <= -hlv(l) + 2 (hlv(l) - hlv(l - 1)): for levels above -2 m at
    most the first five layers adapt.  The ones between them and the
    bottom layer keep hldv."""
    c = cases.shelf_case(nzadapt=3)
    o = shyref.OracleModel(c)
    o.run(LOW_WATER)
    s = o.state()
    assert s["zenv"].min() > -2.0
    hld = c["hldv"].astype(np.float64)
    for ie in range(c["nel"]):
        lmax = c["ilhv"][ie]
        for l in range(5, lmax - 1):
            assert s["hdenv"][ie, l] == hld[l], (ie, l)
    # and the first layer does stretch: thinner than nominal plus z would be
    # impossible (1 m + z < 0 at low water) yet it is positive everywhere
    assert s["hdenv"][:, 0].min() > 0.0


def test_z_star_scales_every_layer_with_the_column():
    c = cases.shelf_case(nzadapt=9)
    o = shyref.OracleModel(c)
    o.run(LOW_WATER)
    s = o.state()
    hm = c["hm3v"].astype(np.float64)
    fac = ((hm + s["zenv"]) / hm).mean(axis=1)
    hld = c["hldv"].astype(np.float64)
    for ie in range(0, c["nel"], 7):
        lmax = c["ilhv"][ie]
        np.testing.assert_allclose(s["hdenv"][ie, :lmax - 1], hld[:lmax - 1] * fac[ie], rtol=1e-12)


@pytest.mark.parametrize("nzadapt", [3, 9])
def test_closed_shelf_conserves_volume_and_tracer_mass(nzadapt):
    c = cases.shelf_case(nzadapt=nzadapt, closed=True, wind=15.0)
    c["tide"] = np.zeros((0, 1, 4), np.float32)
    A = node_areas(c)

    def budget(s):
        return (s["hdknv"] * A).sum(), (s["conzv"][0] * s["hdknv"] * A).sum()

    o = shyref.OracleModel(c)
    v0, m0 = budget(o.state())
    o.run(60)
    s = o.state()
    v1, m1 = budget(s)
    assert np.ptp(s["znv"]) > 0.01                    # the wind has tilted the surface
    assert abs(v1 / v0 - 1.0) < 1e-11                # round-off of 60 FP64 steps
    assert abs(m1 / m0 - 1.0) < 1e-11


def test_refused_with_sigma_layers():
    c = cases.lagoon_case(nkn_target=300, nlv=6)
    c["params"] = dict(c["params"], nzadapt=3)
    with pytest.raises(RuntimeError, match="z-adaptive"):
        shyref.OracleModel(c)
