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
volume within 1e-6 relative.

The number of adapted layers at an element vertex is a threshold test on
the vertex level (compute_zadaptive_info).  A level that passes within FP32
round-off of a threshold can take the other branch on the GPU than in the
FP64 oracle; the layer thicknesses then jump by a different amount at that
vertex for a step and the tracers around it follow.  The test records each
vertex whose count differs between the two runs after any step, requires
that the oracle's level was then within 2e-5 m of the threshold (a tie, not
a wrong count), and checks the tracers of nodes within three element rings
of such a vertex to 1e-3 of their largest magnitude instead of 1e-4."""
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


def adapted_layers(c, nzadapt, zenv):
    """Per element vertex, the deepest adapted layer of compute_zadaptive_info
    (0 for none) and the distance of the level to the threshold that decides
    it, as the node and element thickness kernels evaluate them."""
    hlv = c["hlv"].astype(np.float64)
    lmax = np.asarray(c["ilhv"])[:, None].repeat(3, axis=1)
    rzmov = hlv[nzadapt - 2] / (hlv[nzadapt - 1] - hlv[nzadapt - 2])
    lev = np.zeros(zenv.shape, np.int64)
    margin = np.full(zenv.shape, np.inf)
    going = np.ones(zenv.shape, bool)
    for l in range(1, int(lmax.max())):
        hl, hp = hlv[l - 1], (hlv[l - 2] if l > 1 else 0.0)
        th = -hl + rzmov * (hl - hp)
        live = going & (l <= lmax - 1)
        margin[live] = np.minimum(margin[live], np.abs(zenv[live] - th))
        ok = live & (zenv <= th)
        lev[ok] = l + 1
        going = ok
    return lev, margin


def rings(c, mark, n):
    """Nodes within n element rings of a marked node."""
    nen = c["nen3v"] - 1
    m = mark.copy()
    for _ in range(n):
        m[nen[m[nen].any(axis=1)].ravel()] = True
    return m


@pytest.mark.parametrize("column_threads", [1, 0])
@pytest.mark.parametrize("nzadapt", [3, 9])
def test_shelf_past_low_water(nzadapt, column_threads):
    c = cases.shelf_case(nzadapt=nzadapt)
    g = shygpu.Model(c)
    g.set_option("column_threads", column_threads)
    g.set_state(0)
    o = shyref.OracleModel(c)
    tie = np.zeros(c["nkn"], bool)
    for _ in range(NSTEPS):
        g.run(1)
        o.run(1)
        if nzadapt < c["nlv"]:
            zg = g.get_state(0, fields=("zenv",))["zenv"].astype(np.float64)
            zo = o.state()["zenv"]
            lg, mg = adapted_layers(c, nzadapt, zg)
            lo, mo = adapted_layers(c, nzadapt, zo)
            differ = lg != lo
            assert (mo[differ] <= 2.0e-5).all(), "adapted layer count differs away from a threshold tie"
            tie[c["nen3v"][differ] - 1] = True
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
    near = rings(c, tie, 3)
    dc = np.abs(sg["conzv"] - so["conzv"]).max(axis=(0, 2))
    assert dc[~near].max() <= 1e-4 * cmax
    assert dc.max() <= 1e-3 * cmax
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
