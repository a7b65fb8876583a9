"""shygpu: SHYFEM's semi-implicit time step on B200 (host side).

This package is the host-side mirror of the reference's interface for the
step, over the C ABI of `libshygpu.so` (include/shygpu.h):

* `Model`   -- many basins advanced together on one GPU with device-resident
               state: `run(nsteps)` is `shyfem_run`'s loop body
               (src/shyfem/shyfem_subs.f90:569-658), `hydro()` and `scalar()`
               are its `hydro` / `run_scalar` phases.
* `Shyfem`  -- shyfem_initialize / shyfem_run / shyfem_finalize for one basin
               (shyfem_subs.f90:285, 551, 668).
* `simsys`  -- the reference's linear-system interface (system_initialize,
               system_init, system_assemble, system_add_rhs, system_solve,
               system_get; simsys_spkaux.f90:85-722).

There is no CPU fallback: every compute call raises `ShyError` when the
CUDA library cannot run.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import abi, cases  # noqa: F401

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libshygpu.so"

_lib = None


class ShyError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{abi.STATUS.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Load libshygpu.so (building it first when the sources are newer)."""
    global _lib, LIB_PATH
    if _lib is not None:
        return _lib
    if os.environ.get("SHYGPU_LIB"):                # an alternative build of the same ABI
        LIB_PATH = Path(os.environ["SHYGPU_LIB"])
    elif os.environ.get("SHYGPU_NO_BUILD") != "1":
        try:
            from . import build as _build
            _build.build()
        except Exception as exc:                    # no nvcc: use what is there
            if not LIB_PATH.exists():
                raise ShyError(2, f"libshygpu.so missing and could not be built: {exc}")
    if not LIB_PATH.exists():
        raise ShyError(2, f"libshygpu.so not found at {LIB_PATH}")
    L = C.CDLL(str(LIB_PATH))
    L.shygpu_last_error.restype = C.c_char_p
    L.shygpu_launch_count.restype = C.c_int64
    L.shygpu_model_bytes.restype = C.c_int64
    L.shygpu_model_bytes.argtypes = [C.c_void_p]
    L.shygpu_footprint.restype = C.c_int64
    L.shygpu_footprint.argtypes = [C.c_int32, C.POINTER(abi.ShyBasin), C.POINTER(abi.ShyParams)]
    L.shygpu_create.argtypes = [C.c_int32, C.POINTER(abi.ShyBasin), C.POINTER(abi.ShyParams),
                                C.POINTER(C.c_void_p)]
    L.shygpu_destroy.argtypes = [C.c_void_p]
    L.shygpu_set_state.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.ShyState)]
    L.shygpu_get_state.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.ShyState)]
    L.shygpu_run.argtypes = [C.c_void_p, C.c_int32]
    L.shygpu_enqueue.argtypes = [C.c_void_p, C.c_int32]
    L.shygpu_sync.argtypes = [C.c_void_p]
    L.shygpu_hydro.argtypes = [C.c_void_p]
    L.shygpu_scalar.argtypes = [C.c_void_p]
    L.shygpu_new_step.argtypes = [C.c_void_p]
    L.shygpu_step_info.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.ShyStepInfo)]
    L.shygpu_get_wetdry.argtypes = [C.c_void_p, C.c_int32] + [C.c_void_p] * 3
    L.shygpu_set_nudging.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    L.shygpu_set_nh_distance.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    L.shygpu_get_nh_pressure.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
    L.shygpu_nh_info.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                 C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.shygpu_set_bound_scalar.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]
    L.shygpu_autotune.argtypes = [C.c_void_p, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(C.c_double)]
    L.shygpu_shy_open_scalar.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.ShyBasin), C.c_char_p, C.c_int32,
                                         C.c_int32, C.c_char_p, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.shygpu_ext_open.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.ShyBasin), C.c_char_p, C.c_int32,
                                  C.c_void_p, C.c_char_p, C.c_char_p, C.c_double, C.c_int32, C.POINTER(C.c_void_p)]
    L.shygpu_ext_write.argtypes = [C.c_void_p]
    L.shygpu_ext_close.argtypes = [C.c_void_p]
    L.shygpu_conz3d.argtypes = ([C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_double, C.c_float,
                                 C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_int32, C.c_int32,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_float,
                                 C.c_void_p, C.c_float, C.c_void_p, C.c_float, C.c_float, C.c_float,
                                 C.c_int32, C.c_int32, C.c_int32, C.c_int32])
    L.shygpu_shy_open.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.ShyBasin), C.c_char_p, C.c_int32,
                                  C.c_int32, C.c_char_p, C.POINTER(C.c_void_p)]
    L.shygpu_shy_write.argtypes = [C.c_void_p]
    L.shygpu_shy_close.argtypes = [C.c_void_p]
    L.shygpu_serve_preempt.argtypes = [C.c_void_p, C.c_int64]
    L.shygpu_set_forcing_all.argtypes = [C.c_void_p] + [C.c_void_p] * 4
    L.shygpu_get_levels.argtypes = [C.c_void_p, C.c_void_p]
    L.shygpu_checkpoint_bytes.argtypes = [C.c_void_p]
    L.shygpu_checkpoint_bytes.restype = C.c_int64
    L.shygpu_checkpoint_save.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    L.shygpu_checkpoint_load.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    L.shygpu_set_option.argtypes = [C.c_void_p, C.c_char_p, C.c_double]
    L.shygpu_get_option.argtypes = [C.c_void_p, C.c_char_p]
    L.shygpu_get_option.restype = C.c_double
    L.shygpu_set_ev.argtypes = [C.c_int32, C.c_int32, abi.i32p, abi.f32p, abi.f32p, abi.f32p]
    L.shygpu_simsys_register.argtypes = [C.c_int32, C.c_int32, abi.i32p]
    L.shygpu_simsys_set_tolerance.argtypes = [C.c_double, C.c_double, C.c_int32]
    L.shygpu_simsys_get_matrix.argtypes = [C.POINTER(C.c_int32), C.POINTER(C.c_int32)] + [C.c_void_p] * 4
    L.shygpu_simsys_set_layers.argtypes = [C.c_int32]
    L.shygpu_simsys_get_matrix_3d.argtypes = [C.POINTER(C.c_int32), C.POINTER(C.c_int32)] + [C.c_void_p] * 4
    L.system_assemble_3d_.argtypes = [C.POINTER(C.c_int32)] * 3 + [abi.i32p, C.c_void_p, abi.f32p]
    L.system_adjust_matrix_3d_.argtypes = []
    L.system_solve_3d_.argtypes = [C.POINTER(C.c_int32)] * 3 + [abi.f32p]
    L.system_get_3d_.argtypes = [C.POINTER(C.c_int32)] * 3 + [abi.f32p]
    L.shygpu_set_forcing.argtypes = [C.c_void_p, C.c_int32] + [C.c_void_p] * 4
    L.shygpu_model_stream.argtypes = [C.c_void_p]
    L.shygpu_model_stream.restype = C.c_void_p
    L.shygpu_profile_steps.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_int32)]
    L.shygpu_serve_create.argtypes = [C.c_int64, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.shygpu_serve_submit.argtypes = [C.c_void_p, C.POINTER(abi.ShyBasin), C.POINTER(abi.ShyParams),
                                      C.POINTER(abi.ShyState), C.c_int32, C.POINTER(C.c_int64)]
    L.shygpu_serve_progress.argtypes = [C.c_void_p, C.c_int32] + [C.POINTER(C.c_int32)] * 3
    L.shygpu_serve_status.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int32)] + \
        [C.POINTER(C.c_double)] * 3
    L.shygpu_serve_result.argtypes = [C.c_void_p, C.c_int64, C.POINTER(abi.ShyState), C.POINTER(abi.ShyStepInfo)]
    L.shygpu_serve_release.argtypes = [C.c_void_p, C.c_int64]
    L.shygpu_serve_used.argtypes = [C.c_void_p]
    L.shygpu_serve_used.restype = C.c_int64
    L.shygpu_serve_destroy.argtypes = [C.c_void_p]
    _lib = L
    return L


def check(code, what=""):
    if code != 0:
        msg = lib().shygpu_last_error().decode(errors="replace")
        raise ShyError(code, f"{what}: {msg}" if what else msg)


def set_ev(case):
    """Element geometry ev(19, nel) through the library (evgeom.f90 set_ev)."""
    nkn, nel = case["nkn"], case["nel"]
    ev = np.zeros((nel, abi.SHY_EVDIM), np.float32)
    nen = np.ascontiguousarray(case["nen3v"], np.int32)
    x = np.ascontiguousarray(case["xgv"], np.float32)
    y = np.ascontiguousarray(case["ygv"], np.float32)
    check(lib().shygpu_set_ev(nkn, nel, abi.ptr(nen, abi.i32p), abi.ptr(x), abi.ptr(y), abi.ptr(ev)),
          "set_ev")
    return ev


class Model:
    """Independent basins advanced together; state stays on the device."""

    def __init__(self, case_list, **param_over):
        if isinstance(case_list, dict):
            case_list = [case_list]
        self.cases = list(case_list)
        self._args = [abi.BasinArgs(c) for c in self.cases]
        n = len(self.cases)
        self._basins = (abi.ShyBasin * n)(*[a.struct for a in self._args])
        self._params = (abi.ShyParams * n)(*[abi.make_params(c, **param_over) for c in self.cases])
        h = C.c_void_p()
        check(lib().shygpu_create(n, self._basins, self._params, C.byref(h)), "shygpu_create")
        self.h = h
        self._closed = False

    # -- options ----------------------------------------------------------
    def set_option(self, name, value):
        check(lib().shygpu_set_option(self.h, name.encode(), float(value)), f"set_option {name}")

    def get_option(self, name):
        return lib().shygpu_get_option(self.h, name.encode())

    # -- state ------------------------------------------------------------
    def set_state(self, ib=0, case=None):
        case = case if case is not None else self.cases[ib]
        buf = abi.StateBuffers(case, fill_from_case=True)
        st = buf.struct(only=("znv", "utlnv", "vtlnv", "tempv", "saltv", "conzv"))
        check(lib().shygpu_set_state(self.h, ib, C.byref(st)), "set_state")

    def set_state_all(self):
        for i in range(len(self.cases)):
            self.set_state(i)

    def get_state(self, ib=0, fields=None):
        buf = abi.StateBuffers(self.cases[ib])
        st = buf.struct(only=fields)
        check(lib().shygpu_get_state(self.h, ib, C.byref(st)), "get_state")
        return {k: v for k, v in buf.arrays.items() if fields is None or k in fields}

    # -- time stepping ----------------------------------------------------
    def run(self, nsteps=1):
        check(lib().shygpu_run(self.h, int(nsteps)), "shygpu_run")

    def hydro(self):
        check(lib().shygpu_hydro(self.h), "shygpu_hydro")

    def scalar(self):
        check(lib().shygpu_scalar(self.h), "shygpu_scalar")

    def info(self, ib=0):
        i = abi.ShyStepInfo()
        check(lib().shygpu_step_info(self.h, ib, C.byref(i)), "step_info")
        return i

    def wetdry(self, ib=0):
        """(iwegv, iwetv, inodv) of basin ib: the element and node wet/dry
        state as the reference's mod_geom_dynamic holds it."""
        c = self.cases[ib]
        iweg = np.zeros(c["nel"], np.int32)
        iwet = np.zeros(c["nel"], np.int32)
        inod = np.zeros(c["nkn"], np.int32)
        check(lib().shygpu_get_wetdry(self.h, ib, iweg.ctypes.data, iwet.ctypes.data,
                                      inod.ctypes.data), "get_wetdry")
        return iweg, iwet, inod

    def nbytes(self):
        return lib().shygpu_model_bytes(self.h)

    def stream(self):
        """The model's cudaStream_t as an integer handle."""
        return lib().shygpu_model_stream(self.h)

    def set_forcing(self, ib, tauxnv=None, tauynv=None, ppv=None, rqv=None):
        """Queue per-step forcing (host arrays, pinned for overlap)."""
        def p(a):
            return None if a is None else a.ctypes.data
        for a in (tauxnv, tauynv, ppv, rqv):
            if a is not None and (a.dtype != np.float32 or not a.flags.c_contiguous):
                raise ValueError("forcing arrays must be contiguous float32")
        check(lib().shygpu_set_forcing(self.h, ib, p(tauxnv), p(tauynv), p(ppv), p(rqv)),
              "set_forcing")

    def set_nudging(self, ib, andgzv):
        """Water-level nudging contribution andgzv (per node, float32) of basin ib."""
        a = np.ascontiguousarray(andgzv, np.float32)
        check(lib().shygpu_set_nudging(self.h, ib, a.ctypes.data), "set_nudging")
        lib().shygpu_sync(self.h)

    def set_nh_distance(self, ib, qdist):
        """Weight of the non-hydrostatic pressure per node (qdistv, float32 in [0, 1])."""
        a = np.ascontiguousarray(qdist, np.float32)
        check(lib().shygpu_set_nh_distance(self.h, ib, a.ctypes.data), "set_nh_distance")

    def nh(self, ib=0):
        """(qpnv (nkn, nlv), (iters, refinements, resid0, resid)) of basin ib:
        the non-hydrostatic pressure the next step starts from and the last
        pressure solve."""
        c = self.cases[ib]
        q = np.zeros((c["nkn"], c["nlv"]), np.float32)
        check(lib().shygpu_get_nh_pressure(self.h, ib, q.ctypes.data), "get_nh_pressure")
        it, rf = C.c_int32(0), C.c_int32(0)
        r0, r = C.c_double(0), C.c_double(0)
        check(lib().shygpu_nh_info(self.h, ib, C.byref(it), C.byref(rf), C.byref(r0), C.byref(r)), "nh_info")
        return q, (it.value, rf.value, r0.value, r.value)

    def autotune(self, steps=5):
        """shygpu_autotune: time the candidate launch shapes on this model's
        basins from its current state and keep the fastest; returns (the
        chosen options as "name=value ...", ms per step of the winner or -1
        when the shape was cached)."""
        buf = C.create_string_buffer(512)
        ms = C.c_double(0.0)
        check(lib().shygpu_autotune(self.h, int(steps), buf, 512, C.byref(ms)), "autotune")
        return buf.value.decode(), ms.value

    def set_bound_scalar(self, ib, what, values, itr=0):
        """Boundary values (nkn, nlv) of a scalar of basin ib (what: 0
        temperature, 1 salinity, 2 tracer itr): imposed on level boundaries
        and brought in by inflows.  Call after set_state."""
        a = np.ascontiguousarray(values, np.float32)
        c = self.cases[ib]
        if a.shape != (c["nkn"], c["nlv"]):
            raise ValueError(f"set_bound_scalar: values must have shape {(c['nkn'], c['nlv'])}")
        check(lib().shygpu_set_bound_scalar(self.h, ib, int(what), int(itr), a.ctypes.data), "set_bound_scalar")
        lib().shygpu_sync(self.h)

    def conz3d(self, ib, cn1, ddt, rkpar, difhv, difv, difmol, azpar, adpar, aapar, istot, isact,
               itvd=0, itvdv=0, gradxv=None, gradyv=None, cobs=None, robs=0.0, rtauv=None,
               wsink=0.0, wsinkv=None, rload=0.0, load=None, cbound=None):
        """conz3d_omp (concentration_omp.f90:65-76): one transport sub-step
        (isact of istot) of one scalar of basin ib on the state hydro() made.
        cn1 is overwritten with the new concentration, and load where
        deposition took less than asked.  Arrays are C-contiguous float32 of
        shape (nkn, nlv), but difhv (nel, nlv) and difv, wsinkv (nkn, nlv+1);
        cbound is what inflows bring where the basin has a discharge (None:
        the node's own value); the open-boundary values stay to the caller,
        as in scal3sh."""
        c = self.cases[ib]
        nkn, nel, nlv = c["nkn"], c["nel"], c["nlv"]
        arrays = dict(cn1=(cn1, (nkn, nlv)), difhv=(difhv, (nel, nlv)), difv=(difv, (nkn, nlv + 1)),
                      gradxv=(gradxv, (nkn, nlv)), gradyv=(gradyv, (nkn, nlv)), cobs=(cobs, (nkn, nlv)),
                      rtauv=(rtauv, (nkn, nlv)), wsinkv=(wsinkv, (nkn, nlv + 1)), load=(load, (nkn, nlv)),
                      cbound=(cbound, (nkn, nlv)))
        for name, (a, shape) in arrays.items():
            if a is None:
                continue
            if not isinstance(a, np.ndarray) or a.dtype != np.float32 or not a.flags.c_contiguous \
                    or a.shape != shape:
                raise ValueError(f"conz3d: {name} must be a C-contiguous float32 array of shape {shape}")

        def p(a):
            return None if a is None else a.ctypes.data
        check(lib().shygpu_conz3d(self.h, ib, p(cn1), None, float(ddt), float(rkpar), p(difhv), p(difv),
                                  float(difmol), p(cbound), int(itvd), int(itvdv), p(gradxv), p(gradyv),
                                  p(cobs), float(robs), p(rtauv), float(wsink), p(wsinkv), float(rload),
                                  p(load), float(azpar), float(adpar), float(aapar), int(istot),
                                  int(isact), nlv, nlv), "conz3d")

    def shy_open(self, ib, path, date=0, time=0, title=""):
        """Hydro output of basin ib in the reference's .shy format; returns a
        handle for shy_write/shy_close."""
        h = C.c_void_p()
        check(lib().shygpu_shy_open(self.h, ib, C.byref(self._basins[ib]), str(path).encode(), date, time,
                                    title.encode(), C.byref(h)), "shy_open")
        return h

    def shy_open_scalar(self, ib, path, what, with_rho=False, date=0, time=0, title=""):
        """Scalar output of basin ib in the reference's .shy format: what 1
        temperature/salinity (and density), 2 the passive tracers; returns a
        handle for shy_write/shy_close."""
        h = C.c_void_p()
        check(lib().shygpu_shy_open_scalar(self.h, ib, C.byref(self._basins[ib]), str(path).encode(), date, time,
                                           title.encode(), int(what), int(bool(with_rho)), C.byref(h)),
              "shy_open_scalar")
        return h

    def ext_open(self, ib, path, nodes, names=None, atime0=0.0, with_rho=False, title=""):
        """Time series at the basin's nodes `nodes` (1-based) in the .ext
        format; returns a handle for ext_write/ext_close."""
        nd = np.ascontiguousarray(nodes, np.int32)
        nm = None
        if names is not None:
            nm = b"".join(str(x).encode()[:80].ljust(80) for x in names)
        h = C.c_void_p()
        check(lib().shygpu_ext_open(self.h, ib, C.byref(self._basins[ib]), str(path).encode(), nd.size,
                                    nd.ctypes.data, nm, title.encode(), float(atime0), int(bool(with_rho)),
                                    C.byref(h)), "ext_open")
        return h

    def ext_write(self, f):
        check(lib().shygpu_ext_write(f), "ext_write")

    def ext_close(self, f):
        check(lib().shygpu_ext_close(f), "ext_close")

    def shy_write(self, f):
        check(lib().shygpu_shy_write(f), "shy_write")

    def shy_close(self, f):
        check(lib().shygpu_shy_close(f), "shy_close")

    def checkpoint(self):
        """Every device array of the model, as a host byte array."""
        n = lib().shygpu_checkpoint_bytes(self.h)
        buf = np.empty(n, np.uint8)
        check(lib().shygpu_checkpoint_save(self.h, buf.ctypes.data, n), "checkpoint_save")
        return buf

    def restore(self, buf):
        """Load a checkpoint of this model or of one made from the same inputs."""
        b = np.ascontiguousarray(buf, np.uint8)
        check(lib().shygpu_checkpoint_load(self.h, b.ctypes.data, b.size), "checkpoint_load")

    KERNELS = ("column", "zeta", "final", "node", "stab", "reduce", "conz", "rho")

    def profile_steps(self, nsteps):
        """Per-kernel device time (ms, summed) and launch counts over nsteps."""
        ms = (C.c_double * 8)()
        cnt = (C.c_int32 * 8)()
        check(lib().shygpu_profile_steps(self.h, int(nsteps), ms, cnt), "profile_steps")
        return {k: (ms[i], cnt[i]) for i, k in enumerate(self.KERNELS)}

    def close(self):
        if not self._closed and getattr(self, "h", None):
            lib().shygpu_destroy(self.h)
            self._closed = True

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop (shygpu_serve_*): forecast runs are
    admitted by HBM footprint, run concurrently with their state resident
    on the device, and return their final state."""

    QUEUED, ACTIVE, DONE, FAILED = 0, 1, 2, 3

    def __init__(self, hbm_budget, max_active=8, quantum_steps=60):
        h = C.c_void_p()
        check(lib().shygpu_serve_create(int(hbm_budget), int(max_active), int(quantum_steps), C.byref(h)),
              "serve_create")
        self.h = h
        self._cases = {}
        self._closed = False

    def submit(self, case, nsteps, **param_over):
        """Queue a run of `nsteps` steps from the case's initial state."""
        args = abi.BasinArgs(case)
        params = abi.make_params(case, **param_over)
        buf = abi.StateBuffers(case, fill_from_case=True)
        st = buf.struct(only=("znv", "utlnv", "vtlnv", "tempv", "saltv", "conzv"))
        rid = C.c_int64()
        check(lib().shygpu_serve_submit(self.h, C.byref(args.struct), C.byref(params), C.byref(st),
                                        int(nsteps), C.byref(rid)), "serve_submit")
        self._cases[rid.value] = case
        return rid.value

    def progress(self, block=False):
        """One pass of the loop; returns (active, queued, finished now)."""
        a, q, f = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().shygpu_serve_progress(self.h, 1 if block else 0, C.byref(a), C.byref(q), C.byref(f)),
              "serve_progress")
        return a.value, q.value, f.value

    def status(self, rid):
        """(state, steps enqueued, t_submit, t_admit, t_done) in seconds."""
        st, n = C.c_int32(), C.c_int32()
        ts, ta, td = C.c_double(), C.c_double(), C.c_double()
        check(lib().shygpu_serve_status(self.h, rid, C.byref(st), C.byref(n), C.byref(ts), C.byref(ta),
                                        C.byref(td)), "serve_status")
        return st.value, n.value, ts.value, ta.value, td.value

    def result(self, rid, release=True):
        """Final state arrays (znv, utlnv, vtlnv and the scalars) and info."""
        case = self._cases[rid]
        buf = abi.StateBuffers(case)
        st = buf.struct(only=("znv", "utlnv", "vtlnv", "tempv", "saltv", "conzv"))
        info = abi.ShyStepInfo()
        check(lib().shygpu_serve_result(self.h, rid, C.byref(st), C.byref(info)), "serve_result")
        if release:
            check(lib().shygpu_serve_release(self.h, rid), "serve_release")
            del self._cases[rid]
        out = {k: buf.arrays[k] for k in ("znv", "utlnv", "vtlnv", "tempv", "saltv", "conzv")}
        return out, info

    def preempt(self, rid):
        """Stop a running request, keep its state in host memory, queue it behind
        the requests already waiting."""
        check(lib().shygpu_serve_preempt(self.h, rid), "serve_preempt")

    def used(self):
        return lib().shygpu_serve_used(self.h)

    def close(self):
        if not self._closed and getattr(self, "h", None):
            lib().shygpu_serve_destroy(self.h)
            self._closed = True

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(case_list, **param_over):
    """Device bytes a Model of these basins would hold (admission control)."""
    args = [abi.BasinArgs(c) for c in case_list]
    n = len(case_list)
    basins = (abi.ShyBasin * n)(*[a.struct for a in args])
    params = (abi.ShyParams * n)(*[abi.make_params(c, **param_over) for c in case_list])
    return lib().shygpu_footprint(n, basins, params)


class Shyfem:
    """shyfem_initialize / shyfem_run / shyfem_finalize for one basin."""

    def __init__(self):
        self.model = None
        self.case = None

    def initialize(self, case, **param_over):
        self.case = case
        self.model = Model([case], **param_over)
        self.model.set_state(0)
        return self

    def run(self, dtstep):
        """Advance by dtstep seconds (a whole number of time steps)."""
        dt = self.case["params"]["dt"]
        n = int(round(dtstep / dt))
        if abs(n * dt - dtstep) > 1e-6 * dt:
            raise ValueError("dtstep must be a multiple of dt")
        self.model.run(n)

    def finalize(self):
        if self.model is not None:
            self.model.close()
            self.model = None


class _Simsys:
    """The reference's system_* calls (simsys_spkaux.f90) on the GPU solver."""

    def register(self, nkn, nel, nen3v):
        nen = np.ascontiguousarray(nen3v, np.int32)
        self._nen = nen
        check(lib().shygpu_simsys_register(nkn, nel, abi.ptr(nen, abi.i32p)), "simsys_register")

    def set_tolerance(self, rtol=1e-8, atol=1e-8, maxit=1000):
        check(lib().shygpu_simsys_set_tolerance(rtol, atol, maxit), "simsys_set_tolerance")

    def system_initialize(self):
        lib().system_initialize_()

    def system_init(self):
        lib().system_init_()

    def system_set_explicit(self):
        lib().system_set_explicit_()

    def system_assemble(self, ie, kn, hia, hik):
        """kn(3) 1-based, hia(3,3) with hia[n,m] = hia(n+1,m+1), hik(3)."""
        zs = abi_zeta()
        zs.kn[:] = [int(k) for k in kn]
        zs.hia[:] = [float(v) for v in np.asarray(hia, np.float32).T.ravel()]   # column-major
        zs.hik[:] = [float(v) for v in hik]
        ie_c = C.c_int32(int(ie))
        lib().system_assemble_(C.byref(ie_c))

    def system_add_rhs(self, dt, array):
        a = np.ascontiguousarray(array, np.float32)
        dt_c, n_c = C.c_float(dt), C.c_int32(a.size)
        lib().system_add_rhs_(C.byref(dt_c), C.byref(n_c), abi.ptr(a))

    def system_solve(self, z):
        zz = np.ascontiguousarray(z, np.float32)
        n_c = C.c_int32(zz.size)
        lib().system_solve_(C.byref(n_c), abi.ptr(zz))

    def system_get(self, n):
        z = np.zeros(n, np.float32)
        n_c = C.c_int32(n)
        lib().system_get_(C.byref(n_c), abi.ptr(z))
        return z

    def get_matrix(self, n, nnz):
        rowptr = np.zeros(n + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz, np.float64)
        rhs = np.zeros(n, np.float64)
        nn, zz = C.c_int32(0), C.c_int32(0)
        check(lib().shygpu_simsys_get_matrix(C.byref(nn), C.byref(zz), rowptr.ctypes.data,
                                             col.ctypes.data, val.ctypes.data, rhs.ctypes.data),
              "simsys_get_matrix")
        return rowptr, col, val, rhs

    def iterations(self):
        return lib().shygpu_simsys_iterations()

    def set_layers(self, nlv):
        """Layers of the 3D system (0: none); before system_initialize."""
        check(lib().shygpu_simsys_set_layers(int(nlv)), "simsys_set_layers")

    def system_assemble_3d(self, ie, l, nlv, kn, mass, rhs):
        """mass (3, 3, 3) indexed [d+1, i, j] for the reference's mass(d, i, j)."""
        m = np.asfortranarray(np.asarray(mass, np.float32))
        r = np.ascontiguousarray(rhs, np.float32)
        k = np.ascontiguousarray(kn, np.int32)
        a = [C.c_int32(int(v)) for v in (ie, l, nlv)]
        lib().system_assemble_3d_(C.byref(a[0]), C.byref(a[1]), C.byref(a[2]), abi.ptr(k, abi.i32p),
                                  m.ctypes.data, abi.ptr(r))

    def system_adjust_matrix_3d(self):
        lib().system_adjust_matrix_3d_()

    def system_solve_3d(self, z):
        """z (n, nlv): the guess."""
        zz = np.ascontiguousarray(z, np.float32)
        n, nlv = zz.shape
        a = [C.c_int32(v) for v in (n, nlv, nlv)]
        lib().system_solve_3d_(C.byref(a[0]), C.byref(a[1]), C.byref(a[2]), abi.ptr(zz))

    def system_get_3d(self, n, nlv):
        z = np.zeros((n, nlv), np.float32)
        a = [C.c_int32(v) for v in (n, nlv, nlv)]
        lib().system_get_3d_(C.byref(a[0]), C.byref(a[1]), C.byref(a[2]), abi.ptr(z))
        return z

    def get_matrix_3d(self):
        n, nnz = C.c_int32(0), C.c_int32(0)
        check(lib().shygpu_simsys_get_matrix_3d(C.byref(n), C.byref(nnz), None, None, None, None),
              "simsys_get_matrix_3d")
        rowptr = np.zeros(n.value + 1, np.int32)
        col = np.zeros(nnz.value, np.int32)
        val = np.zeros(nnz.value, np.float64)
        rhs = np.zeros(n.value, np.float64)
        check(lib().shygpu_simsys_get_matrix_3d(C.byref(n), C.byref(nnz), rowptr.ctypes.data, col.ctypes.data,
                                                val.ctypes.data, rhs.ctypes.data), "simsys_get_matrix_3d")
        return rowptr, col, val, rhs


class ZetaSystem(C.Structure):
    _fields_ = [("kn", C.c_int32 * 3), ("hia", C.c_float * 9), ("hik", C.c_float * 3)]


def abi_zeta():
    return ZetaSystem.in_dll(lib(), "shy_zeta_system")


simsys = _Simsys()
