"""shygpu_csr_solve_static: the sparse solve that allocates no device memory.

It solves the CSR system that the simsys path (system_assemble_ ...
system_solve_) assembles and must agree with system_solve_'s answer to the
solver tolerance, on two calls in a row, with the device's free memory
unchanged between calls once the first call has done its set-up.  Kept in
the last-collected file so it also runs after every other GPU test."""
import ctypes as C

import numpy as np
import pytest

import shygpu
import shyref
from shygpu import cases

SHY_OK, SHY_ECAPACITY = 0, 9
MAX_ROWS, MAX_NNZ = 65536, 524288


def solve_fn():
    f = shygpu.lib().shygpu_csr_solve_static
    f.restype = C.c_int
    f.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_void_p,
                  C.POINTER(C.c_int32)]
    return f


def last_error():
    f = shygpu.lib().shygpu_last_error
    f.restype = C.c_char_p
    return f().decode()


def test_static_solve_refuses_oversize_systems():
    f = solve_fn()
    it = C.c_int32(-1)
    dummy = C.c_void_p(256)   # never dereferenced: the size check comes first
    for n, nnz in ((MAX_ROWS + 1, 7 * MAX_ROWS // 8), (1000, MAX_NNZ + 1)):
        rc = f(n, nnz, dummy, dummy, dummy, dummy, dummy, dummy, 1e-8, 1e-8, 100, 0, None, C.byref(it))
        assert rc == SHY_ECAPACITY
        assert "65536 rows" in last_error() and "524288 entries" in last_error()
    assert it.value == -1


def element_systems(case, seed):
    """Element matrices and right-hand sides like hydro_zeta's (random layer
    sums and transports, Dirichlet rows at the open boundary), FP32."""
    ev = shyref.set_ev(case)
    rng = np.random.default_rng(seed)
    dirich = np.full(case["nkn"], shyref.FLAG)
    dirich[case["bnd_index"] > 0] = 0.3
    hias, hiks = [], []
    for ie in range(case["nel"]):
        kn = case["nen3v"][ie] - 1
        hia, hik = np.zeros(9), np.zeros(3)
        shyref.lib.shyref_element_system(
            shyref.dptr(np.ascontiguousarray(ev[ie])), shyref.dptr(rng.uniform(-0.2, 0.2, 3)),
            rng.uniform(5, 15), 0.0, 0.0, rng.uniform(5, 15), rng.uniform(-1, 1), rng.uniform(-1, 1),
            shyref.dptr(np.ascontiguousarray(dirich[kn])), 60.0, 0.5, 0.5, 9.81,
            shyref.dptr(hia), shyref.dptr(hik))
        hias.append(hia.reshape(3, 3).T.astype(np.float32))
        hiks.append(hik.astype(np.float32))
    return hias, hiks


def simsys_reference(case, seed):
    """Solve through the existing entry points; return the CSR system and
    system_get_'s answer."""
    nkn, nel = case["nkn"], case["nel"]
    hias, hiks = element_systems(case, seed)
    S = shygpu.simsys
    S.register(nkn, nel, case["nen3v"])
    S.system_initialize()
    S.system_init()
    for ie in range(nel):
        S.system_assemble(ie + 1, case["nen3v"][ie], hias[ie], hiks[ie])
    S.system_add_rhs(60.0, np.zeros(nkn, np.float32))
    z0 = np.random.default_rng(seed + 1).uniform(-0.05, 0.05, nkn).astype(np.float32)
    S.system_solve(z0)
    z = S.system_get(nkn)
    ntg, _, _ = shyref.coo_init(case)
    rowptr, col, val, rhs = S.get_matrix(nkn, int(ntg[-1]))
    return rowptr, col, val, rhs, z0, z


@pytest.mark.gpu
@pytest.mark.parametrize("size", ["channel", "basin5k"])
def test_static_solve_matches_simsys_twice(size):
    import torch
    case = cases.channel_case() if size == "channel" else cases.basin3d_case(
        nkn_target=5000, nlv=1, baroclinic=False, ts=False)
    rowptr, col, val, rhs, z0, z_ref = simsys_reference(case, seed=5)
    n, nnz = len(rowptr) - 1, int(rowptr[-1])
    dev = torch.device("cuda:0")
    t_rowptr = torch.from_numpy(rowptr.astype(np.int32)).to(dev)
    t_col = torch.from_numpy(col.astype(np.int32)).to(dev)
    t_val = torch.from_numpy(val.astype(np.float64)).to(dev)
    t_rhs = torch.from_numpy(rhs.astype(np.float64)).to(dev)
    t_x0 = torch.from_numpy(z0).to(dev)
    outs = [torch.full((n,), float("nan"), dtype=torch.float32, device=dev) for _ in range(2)]
    torch.cuda.synchronize()
    f = solve_fn()
    free = []
    for x in outs:
        it = C.c_int32(-1)
        rc = f(n, nnz, t_rowptr.data_ptr(), t_col.data_ptr(), t_val.data_ptr(), t_rhs.data_ptr(),
               t_x0.data_ptr(), x.data_ptr(), 1e-8, 1e-8, 1000, 0, None, C.byref(it))
        assert rc == SHY_OK, last_error()
        assert it.value > 0
        free.append(torch.cuda.mem_get_info()[0])
    tol = 1e-5 * max(1.0, float(np.abs(z_ref).max()))   # as the simsys parity test
    for x in outs:
        xs = x.cpu().numpy()
        assert np.isfinite(xs).all()
        assert np.abs(xs - z_ref).max() <= tol
    assert torch.equal(outs[0], outs[1])          # the second call starts from clean scratch
    assert free[0] == free[1]                      # no device memory taken by the second call
