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

SHY_OK, SHY_EARG, SHY_ENOCONV, SHY_ECAPACITY = 0, 1, 3, 9
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


def laplacian_csr(nx, ny, shift):
    """The 5-point Laplacian of an nx x ny grid plus shift on the diagonal:
    symmetric positive definite, condition number about 8 / shift."""
    n = nx * ny
    rowptr, col, val = [0], [], []
    for j in range(ny):
        for i in range(nx):
            k = j * nx + i
            ent = {k: 4.0 + shift}
            for di, dj in ((-1, 0), (1, 0), (0, -1), (0, 1)):
                if 0 <= i + di < nx and 0 <= j + dj < ny:
                    ent[k + dj * nx + di] = -1.0
            for c in sorted(ent):
                col.append(c)
                val.append(ent[c])
            rowptr.append(len(col))
    return np.array(rowptr, np.int32), np.array(col, np.int32), np.array(val, np.float64), n


def device_system(rowptr, col, val, rhs, x0):
    import torch
    dev = torch.device("cuda:0")
    return (torch.from_numpy(rowptr).to(dev), torch.from_numpy(col).to(dev),
            torch.from_numpy(val).to(dev), torch.from_numpy(rhs).to(dev),
            torch.from_numpy(x0).to(dev))


@pytest.mark.gpu
def test_static_solve_symmetric_cg_twice():
    """symmetric != 0 takes the CG branch: a shifted 2D Laplacian solved
    twice, against a direct FP64 solve, with no device memory taken."""
    import torch
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    rowptr, col, val, n = laplacian_csr(96, 80, 0.05)
    rng = np.random.default_rng(11)
    rhs = rng.uniform(-1, 1, n)
    x_ref = sla.spsolve(sp.csr_matrix((val, col, rowptr), shape=(n, n)).tocsc(), rhs)
    t_rowptr, t_col, t_val, t_rhs, t_x0 = device_system(rowptr, col, val, rhs, np.zeros(n, np.float32))
    outs = [torch.full((n,), float("nan"), dtype=torch.float32, device="cuda:0") for _ in range(2)]
    torch.cuda.synchronize()
    f = solve_fn()
    free = []
    for x in outs:
        it = C.c_int32(-1)
        rc = f(n, len(col), t_rowptr.data_ptr(), t_col.data_ptr(), t_val.data_ptr(), t_rhs.data_ptr(),
               t_x0.data_ptr(), x.data_ptr(), 1e-8, 1e-8, 1000, 1, None, C.byref(it))
        assert rc == SHY_OK, last_error()
        assert 0 < it.value <= 1000
        free.append(torch.cuda.mem_get_info()[0])
    for x in outs:
        assert np.abs(x.cpu().numpy() - x_ref).max() <= 1e-5 * np.abs(x_ref).max()
    assert torch.equal(outs[0], outs[1])
    assert free[0] == free[1]


@pytest.mark.gpu
def test_static_solve_maxit_counts_the_whole_call():
    """maxit bounds the iterations of all refinement rounds together; a budget
    equal to the iterations an unbounded call took gives the same answer."""
    import torch
    rowptr, col, val, n = laplacian_csr(64, 64, 0.01)
    rhs = np.random.default_rng(12).uniform(-1, 1, n)
    t_rowptr, t_col, t_val, t_rhs, t_x0 = device_system(rowptr, col, val, rhs, np.zeros(n, np.float32))
    f = solve_fn()

    def run(maxit, sym):
        x = torch.zeros(n, dtype=torch.float32, device="cuda:0")
        it = C.c_int32(-1)
        rc = f(n, len(col), t_rowptr.data_ptr(), t_col.data_ptr(), t_val.data_ptr(), t_rhs.data_ptr(),
               t_x0.data_ptr(), x.data_ptr(), 1e-8, 1e-8, maxit, sym, None, C.byref(it))
        return rc, it.value, x

    for sym in (1, 0):
        rc, k, x_full = run(1000, sym)
        assert rc == SHY_OK, last_error()
        rc, k2, x_k = run(k, sym)
        assert rc == SHY_OK, last_error()
        assert k2 == k and torch.equal(x_k, x_full)
        rc, k3, _ = run(3, sym)
        assert rc == SHY_ENOCONV and k3 == 3


@pytest.mark.gpu
def test_static_solve_refuses_inconsistent_csr():
    """rowptr[n] must equal nnz and every column must lie in [0, n): the
    kernel checks before it writes, so the scratch array is never overrun."""
    import torch
    rowptr, col, val, n = laplacian_csr(20, 20, 0.1)
    rhs = np.ones(n)
    t_rowptr, t_col, t_val, t_rhs, t_x0 = device_system(rowptr, col, val, rhs, np.zeros(n, np.float32))
    f = solve_fn()
    x = torch.full((n,), 7.0, dtype=torch.float32, device="cuda:0")
    it = C.c_int32(-1)
    rc = f(n, len(col) - 1, t_rowptr.data_ptr(), t_col.data_ptr(), t_val.data_ptr(), t_rhs.data_ptr(),
           t_x0.data_ptr(), x.data_ptr(), 1e-8, 1e-8, 100, 1, None, C.byref(it))
    assert rc == SHY_EARG and "rowptr[n] = nnz" in last_error()
    bad_col = col.copy()
    bad_col[5] = n
    t_bad = torch.from_numpy(bad_col).to("cuda:0")
    rc = f(n, len(col), t_rowptr.data_ptr(), t_bad.data_ptr(), t_val.data_ptr(), t_rhs.data_ptr(),
           t_x0.data_ptr(), x.data_ptr(), 1e-8, 1e-8, 100, 1, None, C.byref(it))
    assert rc == SHY_EARG
    assert bool((x == 7.0).all())          # nothing written to the result
    rc = f(n, len(col), t_rowptr.data_ptr(), t_col.data_ptr(), t_val.data_ptr(), t_rhs.data_ptr(),
           t_x0.data_ptr(), x.data_ptr(), 1e-8, 1e-8, 1000, 1, None, C.byref(it))
    assert rc == SHY_OK, last_error()      # the next good call works
