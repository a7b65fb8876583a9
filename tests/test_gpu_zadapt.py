"""z-adaptive surface layers (nzadapt > 1; zadaptutil.f90 with setdepth,
elems_dealing.f90:1014-1110) on the GPU against the FP64 oracle: a tidal
shelf whose three 1 m surface layers an M2 of 1.5 m would empty, run past
low water, with the thread-per-column and the warp-segment kernels, and
with nzadapt = 3 (the top layers follow the level as it falls) and
nzadapt = nlv (every layer stretches with the column, z-star).  Plain
z-layers stop there on the GPU as in the oracle.

Tolerances as in the other parity tests: water level within 1 mm, layer
thicknesses within 1e-4 of their largest value, transports within 1e-3 of
their largest component, tracers within 1e-4 of their largest magnitude,
volume within 1e-6 relative."""
import numpy as np
import pytest

import shygpu
import shyref
from shygpu import cases

pytestmark = pytest.mark.gpu

ZETA_TOL = 1.0e-3
NSTEPS = 240                 # steps of 60 s: past the low water of M2


def active(c, node=True):
    il = c["ilhkv"] if node else c["ilhv"]
    return np.arange(c["nlv"])[None, :] < il[:, None]


@pytest.mark.parametrize("column_threads", [1, 0])
@pytest.mark.parametrize("nzadapt", [3, 9])
def test_shelf_past_low_water(nzadapt, column_threads):
    c = cases.shelf_case(nzadapt=nzadapt)
    g = shygpu.Model(c)
    g.set_option("column_threads", column_threads)
    g.set_state(0)
    o = shyref.OracleModel(c)
    g.run(NSTEPS)
    o.run(NSTEPS)
    sg, so = g.get_state(0), o.state()
    assert so["znv"].min() < -1.2
    assert np.abs(sg["znv"] - so["znv"]).max() <= ZETA_TOL
    mk, me = active(c), active(c, node=False)
    assert np.abs(sg["hdknv"] - so["hdknv"])[mk].max() <= 1e-4 * np.abs(so["hdknv"]).max()
    assert np.abs(sg["hdenv"] - so["hdenv"])[me].max() <= 1e-4 * np.abs(so["hdenv"]).max()
    assert (sg["hdenv"][me] > 0).all() and (sg["hdknv"][mk] > 0).all()
    umax = max(np.abs(so["utlnv"][me]).max(), np.abs(so["vtlnv"][me]).max())
    for f in ("utlnv", "vtlnv"):
        assert np.abs(sg[f] - so[f])[me].max() <= 1e-3 * umax, f
    cmax = np.abs(so["conzv"]).max()
    assert np.abs(sg["conzv"] - so["conzv"]).max() <= 1e-4 * cmax
    wmax = np.abs(so["wlnv"]).max()
    assert np.abs(sg["wlnv"] - so["wlnv"]).max() <= 2e-3 * wmax
    assert abs(g.info(0).volume - o.info().volume) <= 1e-6 * o.info().volume
    g.close()


def test_plain_z_layers_stop_at_low_water():
    c = cases.shelf_case(nzadapt=0)
    g = shygpu.Model(c)
    g.set_state(0)
    with pytest.raises(RuntimeError, match="SHY_EDEPTH"):
        g.run(NSTEPS)
    g.close()


def test_refused_with_wetting_and_drying():
    c = cases.shelf_case(nzadapt=3)
    c["params"] = dict(c["params"], wetdry=1)
    with pytest.raises(RuntimeError, match="z-adaptive"):
        shygpu.Model(c)
