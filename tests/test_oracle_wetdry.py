"""The oracle's wetting and drying (wetdry.f90 setweg/setuvd/setznv,
topo_update.f90 setnod, hydrodynamic.f90:374-404, 710-727) on a tidal flat:
the properties the reference's scheme guarantees, checked on the CPU."""
import numpy as np
import pytest

import shyref
from shygpu import cases


def run_cycle(c, nsteps=750, every=25):
    o = shyref.OracleModel(c)
    out = []
    for _ in range(nsteps // every):
        o.run(every)
        out.append((o.wetdry(), o.state(), o.info()))
    return o, out


@pytest.mark.parametrize("nlv", [1, 4])
def test_flat_dries_and_floods(nlv):
    c = cases.flat_case(nlv=nlv)
    hm = c["hm3v"].astype(np.float64)
    nen = c["nen3v"] - 1
    o, out = run_cycle(c)
    ndry = [int((w[0] > 0).sum()) for w, _, _ in out]
    assert min(ndry) == 0 and max(ndry) > 0.4 * c["nel"], ndry
    for (iweg, iwet, inod), s, info in out:
        dry = iweg > 0
        # counters: wet elements count up, dry ones down
        assert (iwet[~dry] > 0).all() and (iwet[dry] < 0).all()
        # node kinds from the elements around each node (setnod)
        nwet = np.bincount(nen[~dry].ravel(), minlength=c["nkn"])
        nall = np.bincount(nen.ravel(), minlength=c["nkn"])
        assert (inod[nwet == 0] == -2).all()
        assert (nwet[inod == 0] == nall[inod == 0]).all()
        assert ((inod == -1) <= ((nwet > 0) & (nwet <= nall))).all()
        # wet elements: vertex levels are the node levels (setzev), every
        # vertex at least hzmin deep
        zen = s["zenv"].reshape(-1, 3)
        np.testing.assert_array_equal(zen[~dry], s["znv"][nen[~dry]])
        assert (zen[~dry] + hm[~dry] >= 0.01 - 1e-9).all()
        # dry elements keep a film of at least hzmin (setuvd)
        assert (zen[dry] + hm[dry] >= 0.01 - 1e-5).all()
        # every layer has positive thickness
        assert (s["hdenv"][np.arange(c["nlv"])[None, :] < c["ilhv"][:, None]] > 0).all()


def test_flat_without_wetting_and_drying_stops():
    """The flat's land (negative depth) has no layer without setweg: the
    reference stops in setdepth (elems_dealing.f90:1108-1118)."""
    c = cases.flat_case()
    c["params"] = dict(c["params"], wetdry=0)
    with pytest.raises(RuntimeError, match="SHY_EDEPTH"):
        o = shyref.OracleModel(c)
        o.run(5)
