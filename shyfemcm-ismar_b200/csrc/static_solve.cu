// static_solve.cu -- a sparse solve that allocates no device memory.
//
// shygpu_csr_solve_static solves one linear system A x = b given in CSR form
// in device memory with the Krylov solver of the zeta kernel in
// k_zeta_global.cuh (Jacobi-preconditioned CG or BiCGStab in FP32 inside
// FP64 residual refinement, one thread-block cluster, stop test
// ||r|| <= rtol*||r0|| + atol).  Its Krylov vectors, the FP32 copy of the
// matrix and the result record live in one fixed array in the library's
// device memory (g_static_scratch below) instead of memory the library
// allocates, so the call never runs cudaMalloc or cudaFree and never asks a
// library routine that does.
//
// Who needs it: a caller whose device memory is owned by someone else -- an
// ocean model embedded in a framework whose memory pool has reserved the
// GPU, or a server that admits work by an exact HBM budget -- cannot let a
// solver take device memory on its own, and a cudaMalloc or cudaFree in the
// middle of a time loop also waits for work on other streams to finish.
//
// Limits and rules of use:
//  * at most kStaticMaxRows rows and kStaticMaxNnz stored entries; larger
//    systems are refused with SHY_ECAPACITY before anything runs;
//  * CSR arrays that do not describe n rows and nnz entries (rowptr[n] !=
//    nnz, a decreasing rowptr, a column outside [0, n)) are refused with
//    SHY_EARG by the kernel before it writes anything;
//  * maxit counts Krylov iterations over all refinement rounds of a call;
//  * the first call on a device (with that device current) looks the scratch
//    array up with cudaGetSymbolAddress; make that first call before any
//    stream capture begins;
//  * there is one scratch array per device: calls that overlap on one device
//    (two host threads, or two streams without ordering between them) race
//    on it and corrupt each other's results.  Serialise them;
//  * the call is synchronous: it waits on `stream` for the result record.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/shygpu.h"

namespace cg = cooperative_groups;

namespace shy {
int external_fail(int code, const char *msg);   // host.cu: sets shygpu_last_error()
void external_count_launch();                   // host.cu: shygpu_launch_count()
}

namespace {

constexpr int kStaticMaxRows = 65536;
constexpr int kStaticMaxNnz = 524288;
constexpr size_t kSlice = 256;
constexpr size_t round_up(size_t b) { return (b + kSlice - 1) / kSlice * kSlice; }

// result record at the start of the scratch array; cleared before each solve
struct StaticOut {
  int status, iters, refinements, pad;
  double resid0, resid;
};

// byte offsets inside the scratch array
constexpr size_t kOffOut = 0;
constexpr size_t kOffX64 = round_up(sizeof(StaticOut));
constexpr size_t kOffVal = kOffX64 + round_up(sizeof(double) * kStaticMaxRows);
constexpr size_t kOffVec = kOffVal + round_up(sizeof(float) * kStaticMaxNnz);
constexpr int kNumVec = 10;   // dinv r p q z e s t rh v
constexpr size_t kVecBytes = round_up(sizeof(float) * kStaticMaxRows);
constexpr size_t kStaticScratchBytes = kOffVec + kNumVec * kVecBytes;   // 5.0 MiB

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct StaticArgs {
  int n, nnz;
  const int *rowptr, *col;
  const double *val, *rhs;
  const float *x0;
  float *x;
  double rtol, atol;
  int maxit, sym, max_outer;
  float inner_rtol;
  StaticOut *out;
  double *x64;
  float *val32;
  float *dinv, *r, *p, *q, *z, *e, *s, *t, *rh, *v;
};

// Sum of NV values over the cluster in a fixed order (lanes, warps, ranks):
// every CTA obtains the same bits.  One cluster barrier; two parity-indexed
// slot sets keep a fast CTA from overwriting slots a slow one still reads.
template <int NV>
__device__ __forceinline__ void csum(cg::cluster_group &cl, double (&v)[NV], double *wsum, double *slots,
                                     double *bc, int &par, int CL) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; i++) {
    double a = v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) wsum[i * 32 + warp] = a;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double a = lane < nw ? wsum[i * 32 + lane] : 0.;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (lane == 0) slots[par * 4 + i] = a;
    }
  }
  cl.sync();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double a = lane < CL ? *cl.map_shared_rank(&slots[par * 4 + i], lane) : 0.;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (lane == 0) bc[i] = a;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; i++) v[i] = bc[i];
  par ^= 1;
}

__device__ __forceinline__ float spmv_row(const StaticArgs &a, int i, const float *u) {
  float w = 0.f;
  for (int k = a.rowptr[i]; k < a.rowptr[i + 1]; k++) w += a.val32[k] * __ldcg(&u[a.col[k]]);
  return w;
}

// one cluster of CL CTAs; CTA `rank` owns rows [r0, r1)
__global__ void __launch_bounds__(1024) k_csr_static(StaticArgs a) {
  cg::cluster_group cl = cg::this_cluster();
  const int CL = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  __shared__ double wsum[4 * 32];
  __shared__ double slots[2 * 4];
  __shared__ double bc[4];
  int par = 0;
  const int chunk = (a.n + CL - 1) / CL;
  const int r0 = min(a.n, rank * chunk), r1 = min(a.n, r0 + chunk);
  const int tid = threadIdx.x, nth = blockDim.x;

  // The CSR arrays are checked before anything is written: rowptr starts at
  // 0 and ends at nnz, no row has a negative length or reaches past nnz, and
  // every column lies in [0, n).  Every CTA takes the same sum, so a bad
  // matrix ends every CTA here, before the FP32 copy below writes val32.
  {
    double bad[1] = {0.};
    if (rank == 0 && tid == 0 && (a.rowptr[0] != 0 || a.rowptr[a.n] != a.nnz)) bad[0] += 1.;
    for (int i = r0 + tid; i < r1; i += nth) {
      const int k0 = a.rowptr[i], k1 = a.rowptr[i + 1];
      if (k0 < 0 || k1 < k0 || k1 > a.nnz) { bad[0] += 1.; continue; }
      for (int k = k0; k < k1; k++)
        if ((unsigned)a.col[k] >= (unsigned)a.n) bad[0] += 1.;
    }
    csum<1>(cl, bad, wsum, slots, bc, par, CL);
    if (bad[0] != 0.) {
      if (rank == 0 && tid == 0) a.out->status = SHY_EARG;
      cl.sync();   // peers may still read this CTA's slots
      return;
    }
  }

  // FP32 copy of the matrix, Jacobi diagonal (FP64 inverse), FP64 start
  for (int i = r0 + tid; i < r1; i += nth) {
    double diag = 0.;
    for (int k = a.rowptr[i]; k < a.rowptr[i + 1]; k++) {
      const double w = a.val[k];
      a.val32[k] = (float)w;
      if (a.col[k] == i) diag += w;
    }
    a.dinv[i] = diag != 0. ? (float)(1. / diag) : 1.f;
    a.x64[i] = (double)a.x0[i];
  }
  cl.sync();

  double tol = 0., rn = 0.;
  int iters = 0, outer = 0;
  bool conv = false;
  // Each round computes the FP64 residual of x64, stops when it meets the
  // target, and otherwise solves for a correction.  The residual after the
  // last correction is computed too, so the status always describes the x
  // that is returned.  maxit bounds the Krylov iterations of the whole call.
  for (outer = 0;; outer++) {
    double acc[1] = {0.};
    for (int i = r0 + tid; i < r1; i += nth) {
      double res = a.rhs[i];
      for (int k = a.rowptr[i]; k < a.rowptr[i + 1]; k++) res -= a.val[k] * __ldcg(&a.x64[a.col[k]]);
      a.r[i] = (float)res;
      acc[0] += res * res;
    }
    csum<1>(cl, acc, wsum, slots, bc, par, CL);
    rn = sqrt(acc[0]);
    if (outer == 0) tol = a.rtol * rn + a.atol;
    if (outer == 0 && rank == 0 && tid == 0) a.out->resid0 = rn;
    if (rn <= tol) { conv = true; break; }
    if (outer == a.max_outer || iters >= a.maxit) break;
    const double itol = fmax((double)a.inner_rtol * rn, 0.25 * tol);
    if (a.sym) {
      // Chronopoulos-Gear CG on the correction e
      for (int i = r0 + tid; i < r1; i += nth) {
        a.z[i] = a.dinv[i] * a.r[i];
        a.e[i] = 0.f; a.p[i] = 0.f; a.s[i] = 0.f;
      }
      cl.sync();
      double g2[2] = {0., 0.};
      for (int i = r0 + tid; i < r1; i += nth) {
        const float w = spmv_row(a, i, a.z);
        a.t[i] = w;
        g2[0] += (double)a.r[i] * a.z[i];
        g2[1] += (double)w * a.z[i];
      }
      csum<2>(cl, g2, wsum, slots, bc, par, CL);
      double gamma = g2[0], alpha = gamma / g2[1], beta = 0.;
      while (iters < a.maxit) {
        const float fa = (float)alpha, fb = (float)beta;
        for (int i = r0 + tid; i < r1; i += nth) {
          const float pp = a.z[i] + fb * a.p[i];
          const float ss = a.t[i] + fb * a.s[i];
          a.p[i] = pp; a.s[i] = ss;
          a.e[i] += fa * pp;
          const float rr = a.r[i] - fa * ss;
          a.r[i] = rr;
          a.z[i] = a.dinv[i] * rr;
        }
        cl.sync();
        double g3[3] = {0., 0., 0.};
        for (int i = r0 + tid; i < r1; i += nth) {
          const float w = spmv_row(a, i, a.z);
          a.t[i] = w;
          const float rr = a.r[i], u = a.z[i];
          g3[0] += (double)rr * u;
          g3[1] += (double)w * u;
          g3[2] += (double)rr * rr;
        }
        csum<3>(cl, g3, wsum, slots, bc, par, CL);
        iters++;
        if (sqrt(g3[2]) <= itol || !(g3[0] == g3[0])) break;
        beta = g3[0] / gamma;
        alpha = g3[0] / (g3[1] - beta * g3[0] / alpha);
        gamma = g3[0];
      }
    } else {
      // BiCGStab, right Jacobi preconditioning, on the correction e
      double a1[1] = {0.};
      for (int i = r0 + tid; i < r1; i += nth) {
        const float rr = a.r[i];
        a.rh[i] = rr; a.p[i] = 0.f; a.v[i] = 0.f; a.e[i] = 0.f;
        a1[0] += (double)rr * rr;
      }
      csum<1>(cl, a1, wsum, slots, bc, par, CL);
      double rho = 1., alpha = 1., omega = 1.;
      while (iters < a.maxit) {
        double g1[1] = {0.};
        for (int i = r0 + tid; i < r1; i += nth) g1[0] += (double)a.rh[i] * a.r[i];
        csum<1>(cl, g1, wsum, slots, bc, par, CL);
        const double rho1 = g1[0];
        const double beta = (rho1 / rho) * (alpha / omega);
        rho = rho1;
        const float fb = (float)beta, fo = (float)omega;
        for (int i = r0 + tid; i < r1; i += nth) {
          const float pp = a.r[i] + fb * (a.p[i] - fo * a.v[i]);
          a.p[i] = pp;
          a.z[i] = a.dinv[i] * pp;
        }
        cl.sync();
        double g2[1] = {0.};
        for (int i = r0 + tid; i < r1; i += nth) {
          const float vv = spmv_row(a, i, a.z);
          a.v[i] = vv;
          g2[0] += (double)a.rh[i] * vv;
        }
        csum<1>(cl, g2, wsum, slots, bc, par, CL);
        alpha = rho / g2[0];
        const float fa = (float)alpha;
        for (int i = r0 + tid; i < r1; i += nth) {
          const float ss = a.r[i] - fa * a.v[i];
          a.s[i] = ss;
          a.q[i] = a.dinv[i] * ss;
        }
        cl.sync();
        double g3[2] = {0., 0.};
        for (int i = r0 + tid; i < r1; i += nth) {
          const float tt = spmv_row(a, i, a.q);
          a.t[i] = tt;
          g3[0] += (double)tt * a.s[i];
          g3[1] += (double)tt * tt;
        }
        csum<2>(cl, g3, wsum, slots, bc, par, CL);
        omega = g3[1] > 0. ? g3[0] / g3[1] : 0.;
        const float fw = (float)omega;
        double g4[1] = {0.};
        for (int i = r0 + tid; i < r1; i += nth) {
          a.e[i] += fa * a.z[i] + fw * a.q[i];
          const float rr = a.s[i] - fw * a.t[i];
          a.r[i] = rr;
          g4[0] += (double)rr * rr;
        }
        csum<1>(cl, g4, wsum, slots, bc, par, CL);
        iters++;
        if (sqrt(g4[0]) <= itol || omega == 0. || !(g4[0] == g4[0])) break;
      }
    }
    for (int i = r0 + tid; i < r1; i += nth) a.x64[i] += (double)a.e[i];
    cl.sync();
  }
  for (int i = r0 + tid; i < r1; i += nth) a.x[i] = (float)a.x64[i];
  if (rank == 0 && tid == 0) {
    a.out->iters = iters;
    a.out->refinements = outer;
    a.out->resid = rn;
    a.out->status = conv ? SHY_OK : SHY_ENOCONV;
  }
  // the last csum reads every rank's slots after its barrier: no CTA may
  // leave while a peer can still read its shared memory
  cl.sync();
}

// cluster shape by system size (portable sizes only, so no function
// attribute has to be set)
void static_shape(int n, int &CL, int &threads) {
  CL = n >= 16384 ? 8 : (n >= 4096 ? 4 : (n >= 1024 ? 2 : 1));
  threads = n >= 4096 ? 1024 : 512;
}

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

// once per device, with that device current: find the scratch array and
// check that every cluster shape this file launches fits the device
int static_setup(int dev, unsigned char **ptr) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (g_scratch_ptr[dev]) { *ptr = g_scratch_ptr[dev]; return SHY_OK; }
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if (e != cudaSuccess) {
    char msg[256];
    snprintf(msg, sizeof msg, "csr_solve_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    return shy::external_fail(SHY_ECUDA, msg);
  }
  for (int n : {1, 1024, 4096, 16384}) {
    int CL, th;
    static_shape(n, CL, th);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(CL, 1, 1);
    cfg.blockDim = dim3(th, 1, 1);
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nc = 0;
    e = cudaOccupancyMaxActiveClusters(&nc, (const void *)k_csr_static, &cfg);
    if (e != cudaSuccess || nc < 1) {
      char msg[256];
      snprintf(msg, sizeof msg, "csr_solve_static: a cluster of %d x %d threads does not fit: %s", CL, th,
               cudaGetErrorString(e));
      return shy::external_fail(SHY_ECUDA, msg);
    }
  }
  g_scratch_ptr[dev] = (unsigned char *)p;
  *ptr = g_scratch_ptr[dev];
  return SHY_OK;
}

}  // namespace

extern "C" int shygpu_csr_solve_static(int32_t n, int32_t nnz, const int32_t *rowptr, const int32_t *col,
                                       const double *val, const double *rhs, const float *x0, float *x,
                                       double rtol, double atol, int32_t maxit, int32_t symmetric,
                                       void *stream, int32_t *iterations) {
  char msg[256];
  if (n < 1 || nnz < 1 || !rowptr || !col || !val || !rhs || !x0 || !x)
    return shy::external_fail(SHY_EARG, "csr_solve_static: bad arguments");
  if (!(rtol > 0.) || !(atol >= 0.) || maxit < 1)
    return shy::external_fail(SHY_EARG, "csr_solve_static: rtol > 0, atol >= 0, maxit >= 1");
  if (n > kStaticMaxRows || nnz > kStaticMaxNnz) {
    snprintf(msg, sizeof msg,
             "csr_solve_static: %d rows / %d entries exceed the fixed scratch (at most %d rows and %d entries)",
             n, nnz, kStaticMaxRows, kStaticMaxNnz);
    return shy::external_fail(SHY_ECAPACITY, msg);
  }
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    snprintf(msg, sizeof msg, "csr_solve_static: no usable device (%s)", cudaGetErrorString(e));
    return shy::external_fail(SHY_ECUDA, msg);
  }
  unsigned char *base = nullptr;
  if (int st = static_setup(dev, &base)) return st;
  cudaStream_t st = (cudaStream_t)stream;

  StaticArgs a;
  a.n = n; a.nnz = nnz; a.rowptr = rowptr; a.col = col; a.val = val; a.rhs = rhs; a.x0 = x0; a.x = x;
  a.rtol = rtol; a.atol = atol; a.maxit = maxit; a.sym = symmetric != 0;
  a.max_outer = 12; a.inner_rtol = 1e-4f;
  a.out = (StaticOut *)(base + kOffOut);
  a.x64 = (double *)(base + kOffX64);
  a.val32 = (float *)(base + kOffVal);
  float **vec[kNumVec] = {&a.dinv, &a.r, &a.p, &a.q, &a.z, &a.e, &a.s, &a.t, &a.rh, &a.v};
  for (int k = 0; k < kNumVec; k++) *vec[k] = (float *)(base + kOffVec + k * kVecBytes);

  // the result record starts at zero; every vector is written before it is read
  e = cudaMemsetAsync(a.out, 0, sizeof(StaticOut), st);
  int CL, threads;
  static_shape(n, CL, threads);
  if (e == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(CL, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_csr_static, a);
    if (e == cudaSuccess) shy::external_count_launch();
  }
  StaticOut o = {};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&o, a.out, sizeof o, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    snprintf(msg, sizeof msg, "csr_solve_static: %s", cudaGetErrorString(e));
    return shy::external_fail(SHY_ECUDA, msg);
  }
  if (iterations) *iterations = o.iters;
  if (o.status == SHY_EARG) {
    snprintf(msg, sizeof msg,
             "csr_solve_static: rowptr/col are not a CSR matrix of %d rows and %d entries "
             "(rowptr[0] = 0, rowptr[n] = nnz, rows of non-negative length, columns in [0, n))", n, nnz);
    return shy::external_fail(SHY_EARG, msg);
  }
  if (o.status != SHY_OK) {
    snprintf(msg, sizeof msg, "csr_solve_static: no convergence (residual %.3g from %.3g after %d iterations)",
             o.resid, o.resid0, o.iters);
    return shy::external_fail(o.status, msg);
  }
  return SHY_OK;
}
