"""ctypes wrapper of the CPU oracle (oracle/_build/libshyref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference leg, never by the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libshyref.so"
sys.path.insert(0, str(HERE.parent / "shyfemcm-ismar_b200"))
from shygpu import abi  # noqa: E402

d_p = C.POINTER(C.c_double)
i_p = C.POINTER(C.c_int)


def build():
    subprocess.check_call(["make", "-s", "-C", str(HERE)])


def _lib():
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    lib.shyref_last_error.restype = C.c_char_p
    lib.shyref_sigma_stp.restype = C.c_double
    lib.shyref_sigma_stp.argtypes = [C.c_double] * 3
    lib.shyref_flag.restype = C.c_double
    lib.shyref_create.restype = C.c_void_p
    lib.shyref_create.argtypes = [C.POINTER(abi.ShyBasin), C.POINTER(abi.ShyParams)]
    lib.shyref_destroy.argtypes = [C.c_void_p]
    lib.shyref_set_state.argtypes = [C.c_void_p, C.POINTER(abi.ShyState)]
    lib.shyref_run.argtypes = [C.c_void_p, C.c_int]
    lib.shyref_set_nudging.argtypes = [C.c_void_p, C.c_void_p]
    lib.shyref_set_scalar_terms.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_float, C.c_void_p,
                                            C.c_float, C.c_void_p, C.c_float, C.c_void_p]
    lib.shyref_get_load.argtypes = [C.c_void_p, d_p]
    lib.shyref_set_bound_scalar.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    lib.shyref_step_info.argtypes = [C.c_void_p, C.POINTER(abi.ShyStepInfo)]
    lib.shyref_get_state64.argtypes = [C.c_void_p] + [d_p] * 11
    lib.shyref_last_system.argtypes = [C.c_void_p, i_p, d_p, d_p]
    lib.shyref_element_system.argtypes = [d_p, d_p] + [C.c_double] * 6 + [d_p] + [C.c_double] * 4 + [d_p, d_p]
    lib.shyref_spk_solve.argtypes = [C.c_int, i_p, i_p, d_p, d_p, d_p, C.c_double, C.c_double,
                                     C.c_int, i_p, d_p, d_p]
    lib.shyref_set_nh_distance.argtypes = [C.c_void_p, C.c_void_p]
    lib.shyref_get_nh.argtypes = [C.c_void_p, d_p, d_p]
    lib.shyref_nh_info.argtypes = [C.c_void_p, i_p, d_p, d_p]
    lib.shyref_sys3d_create.restype = C.c_void_p
    lib.shyref_sys3d_create.argtypes = [C.c_int, C.c_int, C.c_int, i_p]
    lib.shyref_sys3d_nnz.argtypes = [C.c_void_p]
    lib.shyref_sys3d_assemble.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    lib.shyref_sys3d_adjust.argtypes = [C.c_void_p]
    lib.shyref_sys3d_solve.argtypes = [C.c_void_p, d_p, i_p]
    lib.shyref_sys3d_get.argtypes = [C.c_void_p, d_p, d_p, i_p, i_p]
    lib.shyref_sys3d_destroy.argtypes = [C.c_void_p]
    return lib


lib = _lib()
FLAG = lib.shyref_flag()


def dptr(a):
    return a.ctypes.data_as(d_p)


def iptr(a):
    return a.ctypes.data_as(i_p)


def check(st, what):
    if st != 0:
        raise RuntimeError(f"{what}: {abi.STATUS.get(st, st)}: {lib.shyref_last_error().decode()}")


def set_ev(case):
    nkn, nel = case["nkn"], case["nel"]
    ev = np.zeros((nel, abi.SHY_EVDIM), np.float64)
    nen = np.ascontiguousarray(case["nen3v"], np.int32)
    x = np.ascontiguousarray(case["xgv"], np.float64)
    y = np.ascontiguousarray(case["ygv"], np.float64)
    check(lib.shyref_set_ev(nkn, nel, iptr(nen), dptr(x), dptr(y), dptr(ev)), "set_ev")
    return ev


def penta_fact(val, fast=False):
    v = np.ascontiguousarray(val, np.float64).copy()
    n = v.shape[0]
    f = lib.shyref_penta_factf if fast else lib.shyref_penta_fact
    check(f(n, dptr(v)), "penta_fact")
    return v


def penta_solve(val, r):
    v = np.ascontiguousarray(val, np.float64)
    r = np.ascontiguousarray(r, np.float64)
    s = np.zeros_like(r)
    lib.shyref_penta_solve(v.shape[0], dptr(v), dptr(r), dptr(s))
    return s


def tria_multi(v, r):
    """v: (n,3) lower/centre/upper; r: (m,n) right-hand sides."""
    v = np.ascontiguousarray(v, np.float64).copy()
    r = np.ascontiguousarray(r, np.float64).copy()
    m, n = r.shape
    s = np.zeros_like(r)
    lib.shyref_tria_multi(n, m, dptr(v), dptr(r), dptr(s))
    return s


def sigma_stp(s, t, p):
    return lib.shyref_sigma_stp(s, t, p)


def coo_init(case):
    nkn, nel = case["nkn"], case["nel"]
    cap = 8 * nkn + 64
    ntg = np.zeros(nkn + 1, np.int32)
    icol = np.zeros(cap, np.int32)
    ijp = np.zeros(9 * nel, np.int32)
    nen = np.ascontiguousarray(case["nen3v"], np.int32)
    check(lib.shyref_coo_init(nkn, nel, iptr(nen), iptr(ntg), iptr(icol), iptr(ijp), cap), "coo_init")
    return ntg, icol[: ntg[-1]].copy(), ijp.reshape(nel, 3, 3)


def spk_solve(ia, ja, a, b, x0, rtol=1e-8, atol=1e-8, maxmv=1000):
    x = np.ascontiguousarray(x0, np.float64).copy()
    it = C.c_int(0)
    r0 = C.c_double(0)
    r = C.c_double(0)
    ia = np.ascontiguousarray(ia, np.int32)
    ja = np.ascontiguousarray(ja, np.int32)
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    check(lib.shyref_spk_solve(len(ia) - 1, iptr(ia), iptr(ja), dptr(a), dptr(b), dptr(x),
                               rtol, atol, maxmv, C.byref(it), C.byref(r0), C.byref(r)), "spk_solve")
    return x, it.value, r0.value, r.value


class OracleModel:
    """One basin advanced by the FP64 CPU restatement."""

    def __init__(self, case, **param_over):
        self.case = case
        self.args = abi.BasinArgs(case)
        self.params = abi.make_params(case, **param_over)
        self.h = lib.shyref_create(C.byref(self.args.struct), C.byref(self.params))
        if not self.h:
            raise RuntimeError("shyref_create: " + lib.shyref_last_error().decode())
        st = abi.StateBuffers(case, fill_from_case=True)
        self._init = st
        check(lib.shyref_set_state(self.h, C.byref(st.struct(
            only=("znv", "utlnv", "vtlnv", "tempv", "saltv", "conzv")))), "set_state")

    def run(self, nsteps):
        check(lib.shyref_run(self.h, nsteps), "shyref_run")

    def info(self):
        i = abi.ShyStepInfo()
        lib.shyref_step_info(self.h, C.byref(i))
        return i

    def state(self):
        c = self.case
        nkn, nel, nlv = c["nkn"], c["nel"], c["nlv"]
        nc = max(int(c["params"].get("nconz", 0)), 0)
        out = dict(znv=np.zeros(nkn), utlnv=np.zeros((nel, nlv)), vtlnv=np.zeros((nel, nlv)),
                   hdknv=np.zeros((nkn, nlv)), wlnv=np.zeros((nkn, nlv + 1)),
                   tempv=np.zeros((nkn, nlv)), saltv=np.zeros((nkn, nlv)),
                   rhov=np.zeros((nkn, nlv)), conzv=np.zeros((max(nc, 1), nkn, nlv)),
                   zenv=np.zeros((nel, 3)), hdenv=np.zeros((nel, nlv)))
        order = ("znv", "utlnv", "vtlnv", "hdknv", "wlnv", "tempv", "saltv", "rhov", "conzv",
                 "zenv", "hdenv")
        check(lib.shyref_get_state64(self.h, *[dptr(out[k]) for k in order]), "get_state")
        return out

    def wetdry(self):
        """(iwegv, iwetv, inodv): dry-element marks, their counters, node kinds."""
        c = self.case
        iweg = np.zeros(c["nel"], np.int32)
        iwet = np.zeros(c["nel"], np.int32)
        inod = np.zeros(c["nkn"], np.int32)
        i32 = C.POINTER(C.c_int)
        lib.shyref_wetdry(self.h, iweg.ctypes.data_as(i32), iwet.ctypes.data_as(i32),
                          inod.ctypes.data_as(i32))
        return iweg, iwet, inod

    def set_nudging(self, andgzv):
        """The water-level nudging contribution per node (andgzv), or None."""
        a = None if andgzv is None else np.ascontiguousarray(andgzv, np.float32)
        self._andg = a
        check(lib.shyref_set_nudging(self.h, None if a is None else a.ctypes.data), "set_nudging")

    def set_scalar_terms(self, itr, cobs=None, robs=0.0, rtauv=None, wsink=0.0, wsinkv=None,
                         rload=0.0, load=None):
        """conz3d_omp's nudging (cobs, robs, rtauv), settling (wsink, wsinkv)
        and loading (rload, load) for tracer itr; arrays (nkn, nlv), wsinkv
        (nkn, nlv+1).  itr < 0 removes them."""
        f = lambda a: None if a is None else np.ascontiguousarray(a, np.float32)
        arrs = [f(cobs), f(rtauv), f(wsinkv), f(load)]
        p = [None if a is None else a.ctypes.data for a in arrs]
        check(lib.shyref_set_scalar_terms(self.h, itr, p[0], robs, p[1], wsink, p[2], rload, p[3]),
              "set_scalar_terms")

    def set_bound_scalar(self, what, values, itr=0):
        """Boundary values (nkn, nlv) of a scalar (what: 0 temperature, 1
        salinity, 2 tracer itr): imposed on level boundaries, brought in by
        inflows."""
        a = np.ascontiguousarray(values, np.float32)
        self._bound = a
        check(lib.shyref_set_bound_scalar(self.h, int(what), int(itr), a.ctypes.data), "set_bound_scalar")

    def load(self):
        """The loading array after deposition has cut it, (nkn, nlv)."""
        out = np.zeros((self.case["nkn"], self.case["nlv"]))
        check(lib.shyref_get_load(self.h, dptr(out)), "get_load")
        return out

    def set_nh_distance(self, qdist):
        """The weight of the non-hydrostatic pressure per node (qhdist)."""
        a = np.ascontiguousarray(qdist, np.float32)
        self._qdist = a
        check(lib.shyref_set_nh_distance(self.h, a.ctypes.data), "set_nh_distance")

    def nh(self):
        """(qpnv (nkn, nlv), wnh (nkn, nlv+1), (iters, resid0, resid)) of the last step."""
        c = self.case
        q = np.zeros((c["nkn"], c["nlv"]))
        w = np.zeros((c["nkn"], c["nlv"] + 1))
        check(lib.shyref_get_nh(self.h, dptr(q), dptr(w)), "get_nh")
        it, r0, r = C.c_int(0), C.c_double(0), C.c_double(0)
        lib.shyref_nh_info(self.h, C.byref(it), C.byref(r0), C.byref(r))
        return q, w, (it.value, r0.value, r.value)

    def last_system(self):
        nnz = C.c_int(0)
        lib.shyref_last_system(self.h, C.byref(nnz), None, None)
        val = np.zeros(nnz.value)
        rhs = np.zeros(self.case["nkn"])
        lib.shyref_last_system(self.h, C.byref(nnz), dptr(val), dptr(rhs))
        return val, rhs

    def __del__(self):
        if getattr(self, "h", None):
            lib.shyref_destroy(self.h)
            self.h = None


class System3D:
    """The reference's 3D simsys interface (system_assemble_3d,
    system_adjust_matrix_3d, system_solve_3d, system_get_3d) restated on the
    CPU over one mesh: the 3D COO of coo_init_new and loccoo3d."""

    def __init__(self, nkn, nel, nlv, nen3v):
        self.nkn, self.nel, self.nlv = nkn, nel, nlv
        nen = np.ascontiguousarray(nen3v, np.int32)
        self.h = lib.shyref_sys3d_create(nkn, nel, nlv, iptr(nen))
        if not self.h:
            raise RuntimeError("sys3d_create: " + lib.shyref_last_error().decode())

    def assemble(self, ie, l, mass, rhs):
        """mass (3, 3, 3) indexed [d+1, i, j] for the reference's mass(d, i, j)."""
        m = np.asfortranarray(np.asarray(mass, np.float32).transpose(0, 1, 2))
        r = np.ascontiguousarray(rhs, np.float32)
        check(lib.shyref_sys3d_assemble(self.h, ie, l, m.ctypes.data, r.ctypes.data), "sys3d_assemble")

    def adjust(self):
        lib.shyref_sys3d_adjust(self.h)

    def solve(self, z0):
        z = np.ascontiguousarray(z0, np.float64).copy()
        it = C.c_int(0)
        check(lib.shyref_sys3d_solve(self.h, dptr(z), C.byref(it)), "sys3d_solve")
        return z, it.value

    def matrix(self):
        nnz = lib.shyref_sys3d_nnz(self.h)
        n = (self.nlv + 2) * self.nkn
        val, rhs = np.zeros(nnz), np.zeros(n)
        ia, ja = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32)
        lib.shyref_sys3d_get(self.h, dptr(val), dptr(rhs), iptr(ia), iptr(ja))
        return ia, ja, val, rhs

    def __del__(self):
        if getattr(self, "h", None):
            lib.shyref_sys3d_destroy(self.h)
            self.h = None
