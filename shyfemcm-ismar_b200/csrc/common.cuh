// common.cuh -- device data model and warp-segment primitives.
//
// Layout.  Every basin of a model lives in one set of flat arrays: global
// element index e in [0,NEL), node index k in [0,NKN).  Column arrays keep
// the reference's Fortran layout with the layer index fastest and a common
// stride NLV (the largest nlv of the model's basins):
//   element-layer  a[e*NLV + l]        (utlnv, vtlnv, hdenv, ...)
//   node-layer     a[k*NLV + l]        (hdknv, tempv, saltv, rhov, ...)
//   interface      a[k*(NLV+1) + l]    (wlnv, visv, difv)
// One warp segment of S lanes (S = next power of two >= NLV, S | 32) owns
// one column: lane l is layer l.  A segment reads a column as one contiguous
// run, and vertical recurrences (tridiagonal solves, prefix sums over
// layers) run across lanes with shuffles.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define SHY_FLAGF 1.23456e+23f      // mkonst :: flag, "no value" for rzv
#define SHY_FLAGD 1.23456e+23

namespace shy {

constexpr int kMaxScal = 10;        // T, S and up to 8 passive tracers
constexpr int kMaxTide = 4;

// per-basin parameters (device memory)
struct BasinPar {
  double dt;
  double dtime0;
  float az, am, af, at, ad, aa;
  float grav, rowass, vismol, difmol, hzoff, ahpar, rstol;
  float rkpar[kMaxScal];      // horizontal diffusivity per scalar
  int ireib, ibarcl, nsc;     // nsc: scalars transported (T, S, tracers)
  int itemp, isalt;
  int istot_max;
  int k0, nk, e0, ne, nlv;    // node/element ranges
  int tide_off, ntide;        // tide table offset (floats) and constituents
  float rtol, atol;
  int maxit;
  int has_cor;
  int is_temp[kMaxScal];      // scalar s is temperature (no clipping at 1e-15)
  int nsigma;                 // sigma layers on top (0: z-layers; nlv: pure sigma; between: hybrid)
  float hsigma;               // depth limit of the sigma layers
  int wetdry;                 // wetting and drying of elements (z-layers)
  float hzmin, hzon, volmin;  // its thresholds
  int adv;                    // explicit momentum advection (ilin = 0)
  float rlin;                 // its strength
  int itvd;                   // horizontal transport: 0 upwind, 1 TVD with node gradients
  int itvdv;                  // vertical transport: 0 upwind, 1 TVD
  int ihwadv;                 // vertical momentum advection (with adv): 0 none, 1 upwind, 2 centred
  int nzadapt;                // z-layers with z-adaptive surface layers when > 1
  double rzmov;               // their threshold factor (compute_rzmov_info)
  int inohyd;                 // non-hydrostatic pressure (nohydro.f90)
  float aqpar;                // its semi-implicit weight
  int ivwadv, inhflx;         // vertical / horizontal advection of w in sp256wnh
};

// set_advective's vertical term (explicit.f90:776-833) of one layer from
// the old velocities U/h of the layer and its neighbours (um, up: above
// and below, 0 where absent) and the old w at its top and bottom (wt, wb:
// vertex means, 0 at the surface and at the element's bottom)
__device__ __forceinline__ float2 vert_momentum_adv(int ihwadv, float wt, float wb, bool has_up, bool has_dn,
                                                    float u, float v, float h, float um, float vm, float hm,
                                                    float up, float vp, float hp) {
  if (ihwadv == 1) {
    float zx = 0.f, zy = 0.f;
    if (wt > 0.f) { zx = wt * u; zy = wt * v; }
    else if (has_up) { zx = wt * um; zy = wt * vm; }
    if (wb > 0.f) { if (has_dn) { zx -= wb * up; zy -= wb * vp; } }
    else { zx -= wb * u; zy -= wb * v; }
    return make_float2(zx, zy);
  }
  float ut = 0.f, vt = 0.f, ub = 0.f, vb = 0.f;
  if (has_up) { ut = (um * hm + u * h) / (hm + h); vt = (vm * hm + v * h) / (hm + h); }
  if (has_dn) { ub = (u * h + up * hp) / (h + hp); vb = (v * h + vp * hp) / (h + hp); }
  const float wl = 0.5f * (wt + wb);
  return make_float2(wl * (ut - ub), wl * (vt - vb));
}

// per-basin results of the last step (device memory)
struct BasinOut {
  double dtime;
  double resid0, resid;
  double volume;
  double vbudget;             // FP64 volume budget summed over the nodes (k_reduce)
  int status;
  int iters, refinements;
  int istot;
  int steps;                  // steps completed since the state was set
  float stab[kMaxScal];       // stability index (as float bits, max-reduced)
  int nh_iters, nh_refinements;   // the last non-hydrostatic pressure solve
  double nh_resid0, nh_resid;
};

// everything a kernel needs, passed by value
struct Dev {
  int nbasin, NKN, NEL, NLV, S, nsc_max;
  int col_threads;              // column kernel: 1 one thread per column, 0 one warp segment
  int col_staged;               // thread-per-column kernel without Coriolis: 1 columns staged
                                // through shared memory in coalesced passes, 0 read in place
  int node_prefetch;            // thread-per-column node kernel: 1 each element's layers loaded
                                // at once, 0 layer by layer
  int any_wd;                   // some basin has wetting and drying (thread-per-column forms)
  int any_zad;                  // some basin has z-adaptive layers (nzadapt > 1)
  int any_xt;                   // some basin has horizontal viscosity, baroclinic or
                                // non-hydrostatic pressure (the column kernel's instance with them)
  float2 *mom;                  // (NKN*NLV) node momentum {momentxv, momentyv} when a basin advects
  int any_tvd;                  // some basin transports with TVD (a gradient pass per sub-step)
  int any_tvdv;                 // some basin transports with vertical TVD (itvdv = 1)
  float2 *tgrad;                // (nsc_max*NKN*NLV) node gradients {gx, gy} of the sub-step's scalars
  int4 *tvdup;                  // (6*NEL) itvd = 2: {element, xi0, xi1, xi2 as float bits} per vertex pair
  float *andg;                  // (NKN) water-level nudging contribution andgzv, or null (none set)
  // non-hydrostatic pressure of the basins with inohyd = 1 (null when no
  // basin has it): qp (NKN*NLV) the pressure of the last step as the next
  // one reads it (qpov), qdist (NKN) its weight per node (qdistv)
  float *qp, *qdist;
  int conz_free_bnd;            // 1: k_conz leaves open-boundary values to the caller (shygpu_conz3d)
  // shygpu_conz3d's source terms (k_conz<S, 1, true> only): nudging to
  // cz_obs at rate cz_robs*cz_tau, settling cz_wsink*cz_wsv (NKN*(NLV+1)),
  // loading cz_rload*cz_load, which deposition cuts in place
  const float *cz_obs, *cz_tau, *cz_wsv;
  float *cz_load;
  float cz_robs, cz_wsink, cz_rload;
  // the transport's element part, per element vertex and layer: cz_ef
  // [((3e + ii) * nsc_max + s) * NLV + l] = 4aj (3 fl - hdif) of scalar s on
  // concentrations shifted by vertex ii's, cz_ef1 [(3e + ii) * NLV + l] =
  // 4aj 3 fl of a unit field (the horizontal flow into the vertex)
  float *cz_ef, *cz_ef1;
  BasinPar *par;
  BasinOut *out;
  // mesh (static)
  int4 *enode;        // {k1,k2,k3,basin}, global node numbers
  float *ev8;         // [e*8]: b1 b2 b3 c1 c2 c3 aj(=area/24) dd-unused
  float4 *hm3v;       // {h1,h2,h3,hev}
  int *ilhv, *ilhkv;
  float *czv, *fcorv;
  int *ieltv;         // [e*3+ii] neighbour opposite vertex ii, global, -1 none
  float *wdif;        // [e*9 + ii*3+iii]
  float *difhv;       // [e*NLV+l]
  int *kbnd;          // [k] level-boundary number (basin-local, 1-based) or 0
  float *tide;        // [(b-1)*ntide*4 + c*4 + {ampli,period,phase,zref}] + tide_off
  float *visv, *difv; // [k*(NLV+1)+l]
  float *taux, *tauy, *ppv, *rqv;
  float *hlv, *hldv;  // [b*NLV + l]
  float *areakv;      // [k*NLV+l]
  float2 *avol;       // [k*NLV+l] transport weights: {sum aj4 of elements with layer
                      //  l+1, sum aj4 of elements whose bottom layer is l}
  // zeta system
  int *rowptr, *col;          // CSR over all nodes (block diagonal)
  int *slot_ptr, *slot_src;   // gather of element entries per CSR slot
  int *inc_ptr, *inc;         // node -> (e*3+ii) incidence, increasing e
  int4 *incx;                 // the same entries packed: {e, ii | ilhv(e) << 2,
                              //  node of the next vertex, node of the one after}
  double *val64, *rhs64, *x64;
  float *val32, *dinv32, *r32, *p32, *q32, *z32, *e32, *s32, *t32, *rh32, *v32;
  // wetting and drying: per element the number of dry vertices (0: in the
  // system) and the wet/dry step counter; per node its kind (0 internal,
  // > 0 open boundary, -1 boundary of the wet domain, -2 out of the system)
  // and whether its full fan of elements closes (360 degrees)
  int *iweg, *iwet, *inod;
  unsigned char *kfull;
  float4 *cg4[2];                 // device-wide CG: {r, w = A D^-1 r, s, 1/diag} per row, two generations
  float2 *cg2;                    // device-wide CG: {p, e} per row
  // element system written by the column kernel, 12 floats per element:
  // hia (3x3, row-major, [e*12 + 3i+j]) then hik ([e*12 + 9 + i])
  float *hia;
  // state, [0] = new, [1] = old (swapped per step)
  float *zn, *zo;             // [k]
  float *zen, *zeo;           // [e*3+ii]
  float *un, *vn, *uo, *vo;   // [e*NLV+l]
  float *hkn, *hko;           // [k*NLV+l]
  float *hen, *heo;           // [e*NLV+l]
  float *unv, *vnv;           // [e]
  float *usv, *vsv;           // [e*NLV+l] az*U^{n+1} + (1-az)*U^n of the step
  float *wl;                  // [k*(NLV+1)+l]
  float *rho;                 // [k*NLV+l]
  float *ddx, *ddxi;          // [e*NLV+l] A^-1 H (real / imaginary part with Coriolis)
  float *sc_in, *sc_out;      // [s*NKN*NLV + k*NLV + l] scalars at step start / end
  float *scr0, *scr1;         // intermediate transport sub-steps
  float *cbnd;                // boundary values of the scalars, same layout
  double *vol_node;           // [k]
  double *vbud_node;          // [k] FP64 volume budget: the initial volume plus dt times every
                              //     step's flow into the node column (element fluxes, discharge)
  float *stab_node;           // [s*NKN + k]
  int *imax;                  // largest transport sub-step count of the step (all basins)
  int *subj;                  // sub-step index of the device-driven sub-step loop
  unsigned long long *nsub_launched;   // transport launches made by that loop
};

// ---------------------------------------------------------------------------
// warp-segment helpers (width S is a power of two dividing 32)
// ---------------------------------------------------------------------------
// Shuffles name only the lanes of the calling segment, so segments of one
// warp may follow different control flow (they can belong to different
// basins); all lanes of a segment always execute a shuffle together.
template <int S>
__device__ __forceinline__ unsigned seg_mask() {
  if constexpr (S == 32) return 0xffffffffu;
  else return ((1u << S) - 1u) << ((threadIdx.x & 31) & ~(S - 1));
}
template <int S, typename T>
__device__ __forceinline__ T seg_up(T v, int d) {   // value from lane l-d (same segment)
  return __shfl_up_sync(seg_mask<S>(), v, d, S);
}
template <int S, typename T>
__device__ __forceinline__ T seg_down(T v, int d) { // value from lane l+d (same segment)
  return __shfl_down_sync(seg_mask<S>(), v, d, S);
}
template <int S, typename T>
__device__ __forceinline__ T seg_bcast(T v, int src) {
  return __shfl_sync(seg_mask<S>(), v, src, S);
}
template <int S, typename T>
__device__ __forceinline__ T seg_sum(T v) {         // sum over the segment, all lanes get it
#pragma unroll
  for (int d = S / 2; d > 0; d >>= 1) v += __shfl_xor_sync(seg_mask<S>(), v, d, S);
  return v;
}
template <int S>
__device__ __forceinline__ float seg_max(float v) {
#pragma unroll
  for (int d = S / 2; d > 0; d >>= 1) v = fmaxf(v, __shfl_xor_sync(seg_mask<S>(), v, d, S));
  return v;
}
// set_mass_flux (bnd_routines.f90:1035-1140): the discharge rqv of node k
// [m^3/s] spread over its layers by their volumes at the start of the step
// (volnode(l,k,+1) when set_mass_flux runs, before hydro, is the old
// thickness here) in FP32 like the reference's real volnode, the fractions in
// FP64; zero where the node is out of the system (adjust_mass_flux).  One
// lane per layer; `rq` is uniform over the segment, so the sum is taken by
// every lane of a segment together or by none.
template <int S, typename DevT>
__device__ __forceinline__ float mflux_layer(const DevT &d, int k, bool act, size_t o, bool wetdry) {
  const float rq = d.rqv[k];
  if (rq == 0.f || (wetdry && d.inod[k] == -2)) return 0.f;
  const float vol = act ? d.hko[o] * d.areakv[o] : 0.f;
  double tot = (double)vol;
#pragma unroll
  for (int dd = S / 2; dd > 0; dd >>= 1) tot += __shfl_xor_sync(seg_mask<S>(), tot, dd, S);
  return (act && tot > 0.) ? (float)((double)rq * ((double)vol / tot)) : 0.f;
}

// inclusive prefix sum from the top (lane 0) down
template <int S, typename T>
__device__ __forceinline__ T seg_scan_down(T v, int lane) {
#pragma unroll
  for (int d = 1; d < S; d <<= 1) {
    T o = __shfl_up_sync(seg_mask<S>(), v, d, S);
    if (lane >= d) v += o;
  }
  return v;
}
// inclusive suffix sum from the bottom (lane S-1) up
template <int S, typename T>
__device__ __forceinline__ T seg_scan_up(T v, int lane) {
#pragma unroll
  for (int d = 1; d < S; d <<= 1) {
    T o = __shfl_down_sync(seg_mask<S>(), v, d, S);
    if (lane + d < S) v += o;
  }
  return v;
}

// Parallel cyclic reduction of a tridiagonal system a x_{l-1} + b x_l + c x_{l+1}
// = d across the S lanes of a segment (Hockney 1965; Hockney & Jesshope).
// Lanes outside the system carry the identity row (a=c=d=0, b=1) and the
// last row of the system has c = 0, so no coupling leaks across the border.
// NR right-hand sides share the factorisation.
template <int S, int NR>
__device__ __forceinline__ void pcr_solve(double a, double b, double c, double (&d)[NR], int lane) {
#pragma unroll
  for (int s = 1; s < S; s <<= 1) {
    double am = seg_up<S>(a, s), bm = seg_up<S>(b, s), cm = seg_up<S>(c, s);
    double ap = seg_down<S>(a, s), bp = seg_down<S>(b, s), cp = seg_down<S>(c, s);
    double dm[NR], dp[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) { dm[r] = seg_up<S>(d[r], s); dp[r] = seg_down<S>(d[r], s); }
    bool hasm = lane >= s, hasp = lane + s < S;
    if (!hasm) { am = 0.; bm = 1.; cm = 0.; }
    if (!hasp) { ap = 0.; bp = 1.; cp = 0.; }
    double k1 = hasm ? a / bm : 0.;
    double k2 = hasp ? c / bp : 0.;
    double na = -am * k1, nc = -cp * k2;
    double nb = b - cm * k1 - ap * k2;
#pragma unroll
    for (int r = 0; r < NR; r++) d[r] = d[r] - (hasm ? dm[r] * k1 : 0.) - (hasp ? dp[r] * k2 : 0.);
    a = na; b = nb; c = nc;
  }
#pragma unroll
  for (int r = 0; r < NR; r++) d[r] = d[r] / b;
}

// PCR in single precision with NR right-hand sides (same scheme as pcr_solve)
template <int S, int NR>
__device__ __forceinline__ void pcr_solve_f(float a, float b, float c, float (&d)[NR], int lane) {
#pragma unroll
  for (int s = 1; s < S; s <<= 1) {
    float am = seg_up<S>(a, s), bm = seg_up<S>(b, s), cm = seg_up<S>(c, s);
    float ap = seg_down<S>(a, s), bp = seg_down<S>(b, s), cp = seg_down<S>(c, s);
    float dm[NR], dp[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) { dm[r] = seg_up<S>(d[r], s); dp[r] = seg_down<S>(d[r], s); }
    const bool hasm = lane >= s, hasp = lane + s < S;
    const float k1 = hasm ? __fdividef(a, bm) : 0.f;
    const float k2 = hasp ? __fdividef(c, bp) : 0.f;
    const float na = hasm ? -am * k1 : 0.f, nc = hasp ? -cp * k2 : 0.f;
    const float nb = b - (hasm ? cm * k1 : 0.f) - (hasp ? ap * k2 : 0.f);
#pragma unroll
    for (int r = 0; r < NR; r++) d[r] = d[r] - (hasm ? dm[r] * k1 : 0.f) - (hasp ? dp[r] * k2 : 0.f);
    a = na; b = nb; c = nc;
  }
  const float rb = 1.f / b;
#pragma unroll
  for (int r = 0; r < NR; r++) d[r] = d[r] * rb;
}

// complex single precision (x = real, y = imaginary)
__device__ __forceinline__ float2 cmulf(float2 p, float2 q) {
  return make_float2(p.x * q.x - p.y * q.y, p.x * q.y + p.y * q.x);
}
__device__ __forceinline__ float2 cdivf(float2 p, float2 q) {
  const float r = 1.f / (q.x * q.x + q.y * q.y);
  return make_float2((p.x * q.x + p.y * q.y) * r, (p.y * q.x - p.x * q.y) * r);
}
template <int S>
__device__ __forceinline__ float2 seg_up2f(float2 v, int d) {
  return make_float2(seg_up<S>(v.x, d), seg_up<S>(v.y, d));
}
template <int S>
__device__ __forceinline__ float2 seg_down2f(float2 v, int d) {
  return make_float2(seg_down<S>(v.x, d), seg_down<S>(v.y, d));
}

// single-precision PCR of the complex column system (Coriolis): real
// off-diagonals a, c, complex diagonal b, NR complex right-hand sides
template <int S, int NR>
__device__ __forceinline__ void pcr_solve_cf(float a, float2 b, float c, float2 (&d)[NR], int lane) {
  float2 A = make_float2(a, 0.f), C = make_float2(c, 0.f);
  const float2 z = make_float2(0.f, 0.f);
#pragma unroll
  for (int s = 1; s < S; s <<= 1) {
    float2 am = seg_up2f<S>(A, s), bm = seg_up2f<S>(b, s), cm = seg_up2f<S>(C, s);
    float2 ap = seg_down2f<S>(A, s), bp = seg_down2f<S>(b, s), cp = seg_down2f<S>(C, s);
    float2 dm[NR], dp[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) { dm[r] = seg_up2f<S>(d[r], s); dp[r] = seg_down2f<S>(d[r], s); }
    const bool hasm = lane >= s, hasp = lane + s < S;
    const float2 k1 = hasm ? cdivf(A, bm) : z;
    const float2 k2 = hasp ? cdivf(C, bp) : z;
    const float2 t1 = cmulf(am, k1), t2 = cmulf(cp, k2);
    const float2 na = hasm ? make_float2(-t1.x, -t1.y) : z;
    const float2 nc = hasp ? make_float2(-t2.x, -t2.y) : z;
    float2 nb = b;
    if (hasm) { const float2 t = cmulf(cm, k1); nb.x -= t.x; nb.y -= t.y; }
    if (hasp) { const float2 t = cmulf(ap, k2); nb.x -= t.x; nb.y -= t.y; }
#pragma unroll
    for (int r = 0; r < NR; r++) {
      if (hasm) { const float2 t = cmulf(dm[r], k1); d[r].x -= t.x; d[r].y -= t.y; }
      if (hasp) { const float2 t = cmulf(dp[r], k2); d[r].x -= t.x; d[r].y -= t.y; }
    }
    A = na; b = nb; C = nc;
  }
#pragma unroll
  for (int r = 0; r < NR; r++) d[r] = cdivf(d[r], b);
}

// complex arithmetic on double2 (x = real, y = imaginary)
__device__ __forceinline__ double2 cmul(double2 p, double2 q) {
  return make_double2(p.x * q.x - p.y * q.y, p.x * q.y + p.y * q.x);
}
__device__ __forceinline__ double2 cdiv(double2 p, double2 q) {
  double den = q.x * q.x + q.y * q.y;
  return make_double2((p.x * q.x + p.y * q.y) / den, (p.y * q.x - p.x * q.y) / den);
}
__device__ __forceinline__ double2 csub(double2 p, double2 q) { return make_double2(p.x - q.x, p.y - q.y); }
template <int S>
__device__ __forceinline__ double2 seg_up2(double2 v, int d) {
  return make_double2(seg_up<S>(v.x, d), seg_up<S>(v.y, d));
}
template <int S>
__device__ __forceinline__ double2 seg_down2(double2 v, int d) {
  return make_double2(seg_down<S>(v.x, d), seg_down<S>(v.y, d));
}

// PCR for a complex tridiagonal with real off-diagonals a, c and complex
// diagonal b (the u/v column system with Coriolis, where u + i v is the
// unknown): NR complex right-hand sides.
template <int S, int NR>
__device__ __forceinline__ void pcr_solve_c(double a, double2 b, double c, double2 (&d)[NR], int lane) {
  double2 A = make_double2(a, 0.), C = make_double2(c, 0.);
#pragma unroll
  for (int s = 1; s < S; s <<= 1) {
    double2 am = seg_up2<S>(A, s), bm = seg_up2<S>(b, s), cm = seg_up2<S>(C, s);
    double2 ap = seg_down2<S>(A, s), bp = seg_down2<S>(b, s), cp = seg_down2<S>(C, s);
    double2 dm[NR], dp[NR];
#pragma unroll
    for (int r = 0; r < NR; r++) { dm[r] = seg_up2<S>(d[r], s); dp[r] = seg_down2<S>(d[r], s); }
    bool hasm = lane >= s, hasp = lane + s < S;
    double2 z = make_double2(0., 0.), one = make_double2(1., 0.);
    if (!hasm) { am = z; bm = one; cm = z; }
    if (!hasp) { ap = z; bp = one; cp = z; }
    double2 k1 = hasm ? cdiv(A, bm) : z;
    double2 k2 = hasp ? cdiv(C, bp) : z;
    double2 na = make_double2(-(cmul(am, k1).x), -(cmul(am, k1).y));
    double2 nc = make_double2(-(cmul(cp, k2).x), -(cmul(cp, k2).y));
    double2 nb = csub(csub(b, cmul(cm, k1)), cmul(ap, k2));
#pragma unroll
    for (int r = 0; r < NR; r++) {
      if (hasm) d[r] = csub(d[r], cmul(dm[r], k1));
      if (hasp) d[r] = csub(d[r], cmul(dp[r], k2));
    }
    A = na; b = nb; C = nc;
  }
#pragma unroll
  for (int r = 0; r < NR; r++) d[r] = cdiv(d[r], b);
}

__device__ __forceinline__ void atomic_max_pos(float *addr, float v) {
  // v >= 0: the ordering of non-negative IEEE floats matches their int bits
  atomicMax(reinterpret_cast<int *>(addr), __float_as_int(v));
}

// the element system of element e in its 12-float record (three 16-byte
// stores): a row of zeta equations gathers it from one or two sectors
__device__ __forceinline__ void store_elem_system(const Dev &d, int e, const double (&hia)[3][3],
                                                  const double (&hik)[3]) {
  float4 *p = reinterpret_cast<float4 *>(d.hia + (size_t)e * 12);
  p[0] = make_float4((float)hia[0][0], (float)hia[0][1], (float)hia[0][2], (float)hia[1][0]);
  p[1] = make_float4((float)hia[1][1], (float)hia[1][2], (float)hia[2][0], (float)hia[2][1]);
  p[2] = make_float4((float)hia[2][2], (float)hik[0], (float)hik[1], (float)hik[2]);
}

}  // namespace shy
