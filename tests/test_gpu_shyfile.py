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


def test_scalar_shy_output(tmp_path):
    """The ts.shy file (records 11 salinity, 12 temperature, 13 density) of
    the 3D basin and the conz.shy file (records 301..303) of the lagoon's
    three tracers, against the state at each write."""
    from shygpu.shyfile import read_scalar
    b3 = cases.basin3d_case(nkn_target=900, nlv=8)
    lg = cases.lagoon_case(nkn_target=900, nlv=12)
    for c, what, ids, fields in ((b3, 1, [11, 12, 13], ["saltv", "tempv", "rhov"]),
                                 (lg, 2, [301, 302, 303], ["conzv"])):
        g = shygpu.Model(c)
        g.set_state(0)
        path = tmp_path / f"out{what}.shy"
        f = g.shy_open_scalar(0, path, what, with_rho=True, date=20240102, title="scalars")
        snaps = []
        for k in range(3):
            if k:
                g.run(4)
            g.shy_write(f)
            snaps.append((g.info(0).dtime, {k2: v.copy() for k2, v in g.get_state(0).items()}))
        g.shy_close(f)
        r = read_scalar(path)
        assert (r["ftype"], r["npr"], r["nvar"], r["nlv"]) == (2, 1, len(ids), c["nlv"])
        np.testing.assert_array_equal(r["ilhkv"], c["ilhkv"])
        assert len(r["records"]) == 3 * len(ids)
        act = np.arange(c["nlv"])[None, :] < np.asarray(c["ilhkv"])[:, None]
        for t, (dtime, s) in enumerate(snaps):
            for i, ivar in enumerate(ids):
                rec = r["records"][t * len(ids) + i]
                assert rec["dtime"] == dtime and rec["ivar"] == ivar
                ref = s["conzv"][i] if fields[0] == "conzv" else s[fields[i]]
                np.testing.assert_array_equal(rec["values"][act], ref[act])


def test_ext_time_series(tmp_path):
    """The .ext file at four nodes of the 3D basin: the header, then per
    write the nodal barotropic velocities and level, the nodal velocity of
    each layer (area-weighted means of U/H and U/h over the node's
    elements), temperature, salinity and density, against the state."""
    from shygpu.shyfile import read_ext
    c = cases.basin3d_case(nkn_target=900, nlv=8)
    nodes = [5, 120, 333, 700]
    g = shygpu.Model(c)
    g.set_state(0)
    path = tmp_path / "out.ext"
    f = g.ext_open(0, path, nodes, names=["a", "b", "c", "d"], atime0=1000.0, with_rho=True, title="stations")
    snaps = []
    for k in range(3):
        if k:
            g.run(5)
        g.ext_write(f)
        snaps.append((g.info(0).dtime, {k2: v.copy() for k2, v in g.get_state(0).items()}))
    g.ext_close(f)
    r = read_ext(path)
    assert (r["ext_type"], r["nvers"], r["n"], r["lmax"], r["nvar"]) == (947336, 8, 4, c["nlv"], 5)
    np.testing.assert_array_equal(r["knaus"], nodes)
    np.testing.assert_array_equal(r["il"], c["ilhkv"][np.array(nodes) - 1])
    assert r["names"] == ["a", "b", "c", "d"] and r["title"] == "stations"
    assert len(r["records"]) == 3 * 5
    import shyref
    aj = shyref.set_ev(c)[:, 9]
    hev = c["hm3v"].astype(np.float64).mean(axis=1)
    for t, (dtime, s) in enumerate(snaps):
        recs = r["records"][5 * t: 5 * t + 5]
        assert [x["ivar"] for x in recs] == [1, 2, 12, 11, 13]
        assert all(x["atime"] == 1000.0 + dtime for x in recs)
        for j, k in enumerate(np.array(nodes) - 1):
            els = np.nonzero((c["nen3v"] - 1 == k).any(axis=1))[0]
            hm = hev[els] + s["zenv"].reshape(-1, 3)[els].astype(np.float64).mean(axis=1)
            u0 = (aj[els] * s["unv"][els] / hm).sum() / aj[els].sum()
            np.testing.assert_allclose(recs[0]["values"][0, j, 0], u0, rtol=1e-5, atol=1e-9)
            assert recs[0]["values"][2, j, 0] == s["znv"][k]
            for l in range(c["ilhkv"][k]):
                e = els[c["ilhv"][els] > l]
                ul = (aj[e] * s["utlnv"][e, l] / s["hdenv"][e, l]).sum() / aj[e].sum()
                np.testing.assert_allclose(recs[1]["values"][0, j, l], ul, rtol=1e-5, atol=1e-9)
                assert recs[2]["values"][0, j, l] == s["tempv"][k, l]
                assert recs[3]["values"][0, j, l] == s["saltv"][k, l]
                assert recs[4]["values"][0, j, l] == s["rhov"][k, l]
