"""The .shy reader (shygpu/shyfile.py) on a file framed as Fortran
unformatted sequential records (a 4-byte length before and after each),
laid out as io_shy.f90:1577-1598 (header) and 1628-1660 (records) write
it: a 2-element, 4-node mesh with 2 layers and one element of 1 layer."""
import numpy as np

from shygpu.shyfile import read_hydro


def rec(b):
    n = np.int32(len(b)).tobytes()
    return n + b + n


def test_reader_on_a_hand_made_file(tmp_path):
    nkn, nel, nlv = 4, 2, 2
    nen3v = np.array([[1, 2, 3], [2, 4, 3]], np.int32)
    ilhv = np.array([2, 1], np.int32)
    ilhkv = np.array([2, 2, 2, 1], np.int32)
    x = np.array([0, 1, 0, 1], np.float32)
    y = np.array([0, 0, 1, 1], np.float32)
    hm3v = np.arange(6, dtype=np.float32).reshape(2, 3) + 1
    hlv = np.array([1.0, 5.0], np.float32)
    title = b"hand made".ljust(80)
    head = [np.array([1617, 14], np.int32).tobytes(), np.int32(1).tobytes(),
            np.array([nkn, nel, 3, nlv, 4], np.int32).tobytes(), np.int32(0).tobytes(),
            np.array([20240101, 120000], np.int32).tobytes(), np.int32(4).tobytes(),
            np.array([0.01, 0.05, 0, 0], np.float32).tobytes(), title, b"v".ljust(80), b"",
            nen3v.tobytes(), np.arange(1, 3, dtype=np.int32).tobytes(), np.arange(1, 5, dtype=np.int32).tobytes(),
            np.zeros(2, np.int32).tobytes(), np.zeros(4, np.int32).tobytes(), x.tobytes(), y.tobytes(),
            hm3v.tobytes(), hlv.tobytes(), ilhv.tobytes(), ilhkv.tobytes(), b""]
    z = np.array([0.1, 0.2, 0.3, 0.4], np.float32)
    ze = np.arange(6, dtype=np.float32) / 10
    u = np.array([[1.0, 2.0], [3.0, 0.0]], np.float32)      # element 2 has one layer
    v = -u

    def h(ivar, n, m, lmax):
        return np.float64(3600.0).tobytes() + np.array([ivar, n, m, lmax], np.int32).tobytes()

    body = [h(1, nkn, 1, 1), z.tobytes(), h(1, nel, 3, 1), ze.tobytes(),
            h(3, nel, 1, nlv), np.array([1.0, 2.0, 3.0], np.float32).tobytes(),
            h(3, nel, 1, nlv), np.array([-1.0, -2.0, -3.0], np.float32).tobytes()]
    p = tmp_path / "t.hydro.shy"
    p.write_bytes(b"".join(rec(b) for b in head + body))
    r = read_hydro(p)
    assert (r["nkn"], r["nel"], r["nlv"], r["ftype"], r["date"], r["title"]) == (4, 2, 2, 1, 20240101, "hand made")
    np.testing.assert_array_equal(r["nen3v"], nen3v)
    np.testing.assert_array_equal(r["hm3v"], hm3v)
    (s,) = r["records"]
    assert s["dtime"] == 3600.0
    np.testing.assert_array_equal(s["z"], z)
    np.testing.assert_array_equal(s["ze"], ze.reshape(2, 3))
    np.testing.assert_array_equal(s["u"], u)
    np.testing.assert_array_equal(s["v"], v)


def test_ext_reader_on_a_hand_made_file(tmp_path):
    """The .ext reader on records laid out as io_ext.f90:468-575 writes them:
    two stations with 2 and 1 layers, one record of ivar 2 (m = 2)."""
    from shygpu.shyfile import read_ext
    n, lmax = 2, 2
    il = np.array([2, 1], np.int32)
    head = [np.array([947336, 8], np.int32).tobytes(), np.array([n, lmax, 2], np.int32).tobytes(),
            np.float64(50.0).tobytes(), np.array([0, 0.01, 0], np.float32).tobytes(),
            b"stations".ljust(80) + b"v".ljust(80),
            np.array([3, 7], np.int32).tobytes() + np.array([4.5, 2.0], np.float32).tobytes() + il.tobytes()
            + np.array([1, 2], np.float32).tobytes() + np.array([3, 4], np.float32).tobytes()
            + b"s1".ljust(80) + b"s2".ljust(80),
            np.array([1.0, 5.0], np.float32).tobytes()]
    lin = np.array([1, 2, 3, 4, 5, 6], np.float32)           # u: 1 2 | 3 ; v: 4 5 | 6
    body = [np.float64(110.0).tobytes() + np.array([2, 2, lmax, 6], np.int32).tobytes() + lin.tobytes()]
    p = tmp_path / "t.ext"
    p.write_bytes(b"".join(rec(b) for b in head + body))
    r = read_ext(p)
    assert (r["ext_type"], r["nvers"], r["n"], r["lmax"], r["nvar"], r["atime0"]) == (947336, 8, 2, 2, 2, 50.0)
    assert r["names"] == ["s1", "s2"] and r["title"] == "stations"
    np.testing.assert_array_equal(r["knaus"], [3, 7])
    (s,) = r["records"]
    assert (s["atime"], s["ivar"], s["m"]) == (110.0, 2, 2)
    np.testing.assert_array_equal(s["values"], [[[1, 2], [3, 0]], [[4, 5], [6, 0]]])
