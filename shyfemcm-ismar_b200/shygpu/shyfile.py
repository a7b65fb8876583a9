"""Reader of the reference's .shy output files (io_shy.f90:1550-1681):
Fortran unformatted sequential records, a 4-byte length before and after
each.  Reads what shygpu_shy_open/shygpu_shy_write write, and hydro files
of the reference itself: the header, then per output time the water level
at the nodes and at the element vertices (ivar 1) and the transports U, V
(ivar 3), 3D records holding the active layers of each element only."""
import numpy as np


def _records(raw):
    off = 0
    while off < len(raw):
        n = int(np.frombuffer(raw, np.int32, 1, off)[0])
        body = raw[off + 4: off + 4 + n]
        m = int(np.frombuffer(raw, np.int32, 1, off + 4 + n)[0])
        if m != n:
            raise ValueError(f"broken record at byte {off}: {n} != {m}")
        yield body
        off += 8 + n


def read_hydro(path):
    """dict(header fields, arrays, records=[dict(dtime, z, ze, u, v)])."""
    recs = list(_records(open(path, "rb").read()))
    i32 = lambda b: np.frombuffer(b, np.int32)
    f32 = lambda b: np.frombuffer(b, np.float32)
    idshy, nvers = i32(recs[0])
    ftype = int(i32(recs[1])[0])
    nkn, nel, npr, nlv, nvar = (int(v) for v in i32(recs[2]))
    out = dict(idshy=int(idshy), nvers=int(nvers), ftype=ftype, nkn=nkn, nel=nel, npr=npr, nlv=nlv, nvar=nvar,
               nfix=int(i32(recs[3])[0]), date=int(i32(recs[4])[0]), time=int(i32(recs[4])[1]),
               simpar=f32(recs[6]).copy(), title=recs[7].decode().rstrip(), femver=recs[8].decode().rstrip())
    assert len(recs[9]) == 0
    names = ("nen3v", "ipev", "ipv", "iarv", "iarnv", "xgv", "ygv", "hm3v", "hlv", "ilhv", "ilhkv")
    for k, b in zip(names, recs[10:21]):
        out[k] = (f32 if k in ("xgv", "ygv", "hm3v", "hlv") else i32)(b).copy()
    out["nen3v"] = out["nen3v"].reshape(nel, 3)
    out["hm3v"] = out["hm3v"].reshape(nel, 3)
    assert len(recs[21]) == 0
    ilhv = out["ilhv"]
    rows = []
    r = recs[22:]
    for t in range(0, len(r), 8):
        snap = {}
        for j, key in enumerate(("z", "ze", "u", "v")):
            h = r[t + 2 * j]
            dtime = float(np.frombuffer(h, np.float64, 1, 0)[0])
            ivar, n, m, lmax = (int(v) for v in np.frombuffer(h, np.int32, 4, 8))
            vals = f32(r[t + 2 * j + 1])
            if lmax > 1:                        # linear2vals: active layers per element
                full = np.zeros((n, lmax), np.float32)
                pos = 0
                for e in range(n):
                    k = min(lmax, int(ilhv[e]))
                    full[e, :k] = vals[pos:pos + k]
                    pos += k
                vals = full
            elif m > 1:
                vals = vals.reshape(n, m)
            else:
                vals = vals.reshape(n, 1) if key in ("u", "v") else vals.copy()
            snap[key] = vals
            snap.setdefault("ivar_" + key, ivar)
        snap["dtime"] = dtime
        rows.append(snap)
    out["records"] = rows
    return out


def _header(recs):
    i32 = lambda b: np.frombuffer(b, np.int32)
    f32 = lambda b: np.frombuffer(b, np.float32)
    idshy, nvers = i32(recs[0])
    ftype = int(i32(recs[1])[0])
    nkn, nel, npr, nlv, nvar = (int(v) for v in i32(recs[2]))
    out = dict(idshy=int(idshy), nvers=int(nvers), ftype=ftype, nkn=nkn, nel=nel, npr=npr, nlv=nlv, nvar=nvar,
               nfix=int(i32(recs[3])[0]), date=int(i32(recs[4])[0]), time=int(i32(recs[4])[1]),
               simpar=f32(recs[6]).copy(), title=recs[7].decode().rstrip(), femver=recs[8].decode().rstrip())
    names = ("nen3v", "ipev", "ipv", "iarv", "iarnv", "xgv", "ygv", "hm3v", "hlv", "ilhv", "ilhkv")
    for k, b in zip(names, recs[10:21]):
        out[k] = (f32 if k in ("xgv", "ygv", "hm3v", "hlv") else i32)(b).copy()
    out["nen3v"] = out["nen3v"].reshape(nel, 3)
    out["hm3v"] = out["hm3v"].reshape(nel, 3)
    return out


def read_scalar(path):
    """A scalar .shy file (ftype 2: T/S/density or tracers): the header and
    records=[dict(dtime, ivar, values (nkn, nlv) with zeros below each node's
    layers)]."""
    recs = list(_records(open(path, "rb").read()))
    out = _header(recs)
    assert out["ftype"] == 2 and out["npr"] == 1
    ilhkv = out["ilhkv"]
    rows = []
    r = recs[22:]
    for t in range(0, len(r), 2):
        h = r[t]
        dtime = float(np.frombuffer(h, np.float64, 1, 0)[0])
        ivar, n, m, lmax = (int(v) for v in np.frombuffer(h, np.int32, 4, 8))
        vals = np.frombuffer(r[t + 1], np.float32)
        full = np.zeros((n, lmax), np.float32)
        pos = 0
        for k in range(n):
            kk = min(lmax, int(ilhkv[k]))
            full[k, :kk] = vals[pos:pos + kk]
            pos += kk
        rows.append(dict(dtime=dtime, ivar=ivar, values=full))
    out["records"] = rows
    return out


def read_ext(path):
    """A .ext time-series file (io_ext.f90:468-575): the header (nodes,
    depths, layer counts, x, y, names, layer depths) and records=[dict(atime,
    ivar, m, values (m, n, lmax) with zeros below each node's layers)]."""
    recs = list(_records(open(path, "rb").read()))
    i32 = lambda b: np.frombuffer(b, np.int32)
    f32 = lambda b: np.frombuffer(b, np.float32)
    ext_type, nvers = (int(v) for v in i32(recs[0]))
    n, lmax, nvar = (int(v) for v in i32(recs[1]))
    atime0 = float(np.frombuffer(recs[2], np.float64)[0])
    href, hzmin, nzadapt = (float(v) for v in f32(recs[3]))
    title, femver = recs[4][:80].decode().rstrip(), recs[4][80:].decode().rstrip()
    b = recs[5]
    knaus = np.frombuffer(b, np.int32, n, 0)
    hdep = np.frombuffer(b, np.float32, n, 4 * n)
    il = np.frombuffer(b, np.int32, n, 8 * n)
    x = np.frombuffer(b, np.float32, n, 12 * n)
    y = np.frombuffer(b, np.float32, n, 16 * n)
    names = [b[20 * n + 80 * j: 20 * n + 80 * (j + 1)].decode().rstrip() for j in range(n)]
    hlv = f32(recs[6]).copy()
    rows = []
    for rb in recs[7:]:
        atime = float(np.frombuffer(rb, np.float64, 1, 0)[0])
        ivar, m, lm, nlin = (int(v) for v in np.frombuffer(rb, np.int32, 4, 8))
        lin = np.frombuffer(rb, np.float32, nlin, 24)
        vals = np.zeros((m, n, lm), np.float32)
        pos = 0
        for i in range(m):
            for j in range(n):
                k = min(lm, int(il[j]))
                vals[i, j, :k] = lin[pos:pos + k]
                pos += k
        rows.append(dict(atime=atime, ivar=ivar, m=m, values=vals))
    return dict(ext_type=ext_type, nvers=nvers, n=n, lmax=lmax, nvar=nvar, atime0=atime0, href=href, hzmin=hzmin,
                nzadapt=nzadapt, title=title, femver=femver, knaus=knaus.copy(), hdep=hdep.copy(), il=il.copy(),
                x=x.copy(), y=y.copy(), names=names, hlv=hlv, records=rows)
