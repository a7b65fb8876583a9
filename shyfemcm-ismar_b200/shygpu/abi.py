"""ctypes mirror of include/shygpu.h (structs and status codes).

The structs describe a basin, its parameters and views of its state with
the reference's Fortran layouts (see the header).  `BasinArgs` builds a
`shy_basin` from a case dict and keeps the numpy buffers alive for as long
as the struct is used.
"""
from __future__ import annotations

import ctypes as C
import numpy as np

SHY_EVDIM = 19
SHY_MAX_LAYERS = 32
SHY_MAX_TIDE = 4
SHY_MAX_CONZ = 8

STATUS = {
    0: "SHY_OK", 1: "SHY_EARG", 2: "SHY_ECUDA", 3: "SHY_ENOCONV", 4: "SHY_ESINGULAR",
    5: "SHY_EDEPTH", 6: "SHY_EISTOT", 7: "SHY_ENAN", 8: "SHY_ESTATE", 9: "SHY_ECAPACITY",
}

f32p = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int32)


class ShyBasin(C.Structure):
    _fields_ = [
        ("nkn", C.c_int32), ("nel", C.c_int32), ("nlv", C.c_int32),
        ("nen3v", i32p), ("xgv", f32p), ("ygv", f32p), ("hm3v", f32p),
        ("hlv", f32p), ("hldv", f32p), ("ilhv", i32p), ("ilhkv", i32p),
        ("czv", f32p), ("fcorv", f32p), ("visv", f32p), ("difv", f32p),
        ("tauxnv", f32p), ("tauynv", f32p), ("ppv", f32p), ("rqv", f32p),
        ("bnd_index", i32p), ("nbnd", C.c_int32), ("ntide", C.c_int32), ("tide", f32p),
    ]


class ShyParams(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("dtime0", C.c_double),
        ("azpar", C.c_float), ("ampar", C.c_float), ("afpar", C.c_float),
        ("atpar", C.c_float), ("adpar", C.c_float), ("aapar", C.c_float),
        ("grav", C.c_float), ("rowass", C.c_float),
        ("vismol", C.c_float), ("difmol", C.c_float),
        ("hzoff", C.c_float), ("ahpar", C.c_float), ("rstol", C.c_float),
        ("thpar", C.c_float), ("shpar", C.c_float), ("chpar", C.c_float),
        ("ireib", C.c_int32), ("ibarcl", C.c_int32), ("ilin", C.c_int32),
        ("itemp", C.c_int32), ("isalt", C.c_int32), ("nconz", C.c_int32),
        ("istot_max", C.c_int32),
        ("solver_rtol", C.c_float), ("solver_atol", C.c_float), ("solver_maxit", C.c_int32),
        ("nsigma", C.c_int32), ("hsigma", C.c_float),
        ("wetdry", C.c_int32), ("hzmin", C.c_float), ("hzon", C.c_float), ("volmin", C.c_float),
        ("rlin", C.c_float), ("itvd", C.c_int32), ("itvdv", C.c_int32),
        ("ihwadv", C.c_int32), ("nzadapt", C.c_int32),
        ("inohyd", C.c_int32), ("aqpar", C.c_float), ("ivwadv", C.c_int32), ("inhflx", C.c_int32),
    ]


class ShyState(C.Structure):
    _fields_ = [(n, f32p) for n in (
        "znv", "zenv", "utlnv", "vtlnv", "unv", "vnv", "hdknv", "hdenv", "wlnv",
        "tempv", "saltv", "rhov", "conzv")]


class ShyStepInfo(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("krylov_iters", C.c_int32), ("refinements", C.c_int32),
        ("istot", C.c_int32), ("resid0", C.c_double), ("resid", C.c_double),
        ("volume", C.c_double), ("dtime", C.c_double), ("volume_budget", C.c_double),
    ]


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def ptr(a, t=f32p):
    return a.ctypes.data_as(t) if a is not None else None


class BasinArgs:
    """Owns the numpy buffers behind one ShyBasin."""

    def __init__(self, case):
        nkn, nel, nlv = case["nkn"], case["nel"], case["nlv"]
        self.bufs = {}

        def keep(name, arr, conv=_f32):
            a = conv(arr)
            self.bufs[name] = a
            return a

        tide = np.asarray(case["tide"], np.float32)          # (nbnd, ntide, 4)
        nbnd, ntide = tide.shape[0], tide.shape[1]
        if ntide > SHY_MAX_TIDE:
            raise ValueError("too many tidal constituents")
        b = ShyBasin()
        b.nkn, b.nel, b.nlv = nkn, nel, nlv
        b.nen3v = ptr(keep("nen3v", case["nen3v"], _i32), i32p)
        b.xgv = ptr(keep("xgv", case["xgv"]))
        b.ygv = ptr(keep("ygv", case["ygv"]))
        b.hm3v = ptr(keep("hm3v", case["hm3v"]))
        b.hlv = ptr(keep("hlv", case["hlv"]))
        b.hldv = ptr(keep("hldv", case["hldv"]))
        b.ilhv = ptr(keep("ilhv", case["ilhv"], _i32), i32p)
        b.ilhkv = ptr(keep("ilhkv", case["ilhkv"], _i32), i32p)
        for name in ("czv", "fcorv", "visv", "difv", "tauxnv", "tauynv", "ppv", "rqv"):
            setattr(b, name, ptr(keep(name, case[name])))
        b.bnd_index = ptr(keep("bnd_index", case["bnd_index"], _i32), i32p)
        b.nbnd, b.ntide = nbnd, ntide
        b.tide = ptr(keep("tide", tide))
        self.struct = b


def make_params(case, **over):
    p = dict(case["params"])
    p.update(over)
    s = ShyParams()
    s.dt = float(p["dt"])
    s.dtime0 = float(p.get("dtime0", 0.0))
    for name in ("azpar", "ampar", "afpar", "atpar", "adpar", "aapar", "grav", "rowass",
                 "vismol", "difmol", "hzoff", "ahpar", "rstol", "thpar", "shpar", "chpar"):
        setattr(s, name, float(p[name]))
    for name in ("ireib", "ibarcl", "ilin", "itemp", "isalt", "nconz"):
        setattr(s, name, int(p[name]))
    s.istot_max = int(p.get("istot_max", 1000))
    s.solver_rtol = float(p.get("solver_rtol", 1e-8))
    s.solver_atol = float(p.get("solver_atol", 1e-8))
    s.solver_maxit = int(p.get("solver_maxit", 1000))
    s.nsigma = int(p.get("nsigma", 0))
    s.hsigma = float(p.get("hsigma", 10000.0))
    s.wetdry = int(p.get("wetdry", 0))
    s.hzmin = float(p.get("hzmin", 0.01))
    s.hzon = float(p.get("hzon", 0.10))
    s.volmin = float(p.get("volmin", 1.0))
    s.rlin = float(p.get("rlin", 1.0))
    s.itvd = int(p.get("itvd", 0))
    s.itvdv = int(p.get("itvdv", 0))
    s.ihwadv = int(p.get("ihwadv", 0))
    s.nzadapt = int(p.get("nzadapt", 0))
    s.inohyd = int(p.get("inohyd", 0))
    s.aqpar = float(p.get("aqpar", 0.5))
    s.ivwadv = int(p.get("ivwadv", 0))
    s.inhflx = int(p.get("inhflx", 0))
    return s


class StateBuffers:
    """Host buffers for a basin's state, reference layouts (float32)."""

    FIELDS = ("znv", "zenv", "utlnv", "vtlnv", "unv", "vnv", "hdknv", "hdenv", "wlnv",
              "tempv", "saltv", "rhov", "conzv")

    def __init__(self, case, fill_from_case=False):
        nkn, nel, nlv = case["nkn"], case["nel"], case["nlv"]
        nc = max(int(case["params"].get("nconz", 0)), 0)
        shapes = dict(znv=(nkn,), zenv=(nel, 3), utlnv=(nel, nlv), vtlnv=(nel, nlv),
                      unv=(nel,), vnv=(nel,), hdknv=(nkn, nlv), hdenv=(nel, nlv),
                      wlnv=(nkn, nlv + 1), tempv=(nkn, nlv), saltv=(nkn, nlv),
                      rhov=(nkn, nlv), conzv=(max(nc, 1), nkn, nlv))
        self.arrays = {k: np.zeros(v, np.float32) for k, v in shapes.items()}
        if fill_from_case:
            for k in ("znv", "utlnv", "vtlnv", "tempv", "saltv"):
                self.arrays[k][...] = case[k]
            if nc:
                self.arrays["conzv"][...] = case["conzv"]

    def struct(self, only=None):
        s = ShyState()
        for k in self.FIELDS:
            if only is None or k in only:
                setattr(s, k, ptr(self.arrays[k]))
        return s

    def __getitem__(self, k):
        return self.arrays[k]
