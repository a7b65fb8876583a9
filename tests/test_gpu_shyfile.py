"""Hydro output in the reference's .shy format (shygpu_shy_open/write/close,
io_shy.f90:1550-1681): the header and every record read back, against the
model state at the same steps."""
import numpy as np
import pytest

import shygpu
from shygpu import cases
from shygpu.shyfile import read_hydro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", ["channel2d", "basin3d"])
def test_shy_hydro_output(tmp_path, shape):
    c = cases.channel_case() if shape == "channel2d" else cases.basin3d_case(nkn_target=900, nlv=8)
    g = shygpu.Model(c)
    g.set_state(0)
    path = tmp_path / "out.hydro.shy"
    f = g.shy_open(0, path, date=20240101, time=0, title=f"test {shape}")
    snaps = []
    for k in range(4):
        if k:
            g.run(5)
        g.shy_write(f)
        s = g.get_state(0, ("znv", "zenv", "utlnv", "vtlnv"))
        snaps.append((g.info(0).dtime, {k2: v.copy() for k2, v in s.items()}))
    g.shy_close(f)
    r = read_hydro(path)
    assert (r["idshy"], r["nvers"], r["ftype"], r["npr"], r["nvar"]) == (1617, 14, 1, 3, 4)
    assert (r["nkn"], r["nel"], r["nlv"]) == (c["nkn"], c["nel"], c["nlv"])
    assert r["date"] == 20240101 and r["title"] == f"test {shape}"
    np.testing.assert_array_equal(r["nen3v"], c["nen3v"])
    np.testing.assert_array_equal(r["xgv"], c["xgv"])
    np.testing.assert_array_equal(r["hm3v"], c["hm3v"])
    np.testing.assert_array_equal(r["ilhv"], c["ilhv"])
    np.testing.assert_array_equal(r["ilhkv"], c["ilhkv"])
    assert len(r["records"]) == 4
    act = np.arange(c["nlv"])[None, :] < np.asarray(c["ilhv"])[:, None]
    for rec, (dtime, s) in zip(r["records"], snaps):
        assert rec["dtime"] == dtime
        assert (rec["ivar_z"], rec["ivar_u"]) == (1, 3)
        np.testing.assert_array_equal(rec["z"], s["znv"])
        np.testing.assert_array_equal(rec["ze"], s["zenv"].reshape(-1, 3))
        np.testing.assert_array_equal(rec["u"][act], s["utlnv"][act])
        np.testing.assert_array_equal(rec["v"][act], s["vtlnv"][act])
