// shyref -- CPU oracle for the SHYFEM semi-implicit step.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++ and in FP64,
// the reference's algorithm for the path the GPU library implements, so that
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg can check
// or time it.  Nothing in the product links or calls this code.
//
// Reference: georgu/shyfemcm-ismar (SHYFEM 8.x), Fortran 90.  The reference
// cannot be compiled here (no Fortran compiler), so parity of the whole step is
// anchored on this restatement plus the reference's own known-answer tests
// (penta.f90 examples, eq_state.f90 rhotst values, coo_util.f90 pattern),
// which tests/test_oracle_kat.py checks.
//
// Every routine cites the reference file:line it follows.  Arrays use the
// reference's Fortran layouts: a(l,ie) of (nlv,nel) is a[ie*nlv + (l-1)],
// a(l,k) of (0:nlv,nkn) is a[k*(nlv+1) + l], nen3v 0-based internally.

#include "../include/shygpu.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

const double kFlag = 1.23456e+23;   // mkonst :: flag ("no value" marker for rzv)
const double kPi = 3.141592653;     // bnd_admin.f90:1312 (single-precision literal)

std::string g_err;
int fail(int code, const std::string &msg) { g_err = msg; return code; }

// ---------------------------------------------------------------------------
// set_ev (src/utils/shyutil/evgeom.f90:167-320) and adjust_bc (:1007-1040)
// ---------------------------------------------------------------------------
void adjust_bc(double &v1, double &v2, double &v3) {
  double vv = v1 + v2 + v3;
  if (vv == 0.) return;
  if (v1 == 0.) { v2 = v2 - vv / 2.; v3 = -v2; }
  else if (v2 == 0.) { v3 = v3 - vv / 2.; v1 = -v3; }
  else if (v3 == 0.) { v1 = v1 - vv / 2.; v2 = -v1; }
  else { v1 = v1 - vv / 3.; v2 = v2 - vv / 3.; v3 = v3 - vv / 3.; v3 = -v1 - v2; }
}

int set_ev(int nkn, int nel, const int *nen3v /*0-based*/, const double *x, const double *y,
           double *ev) {
  const double rad = 180. / (4. * std::atan(1.));
  for (int ie = 0; ie < nel; ie++) {
    int k1 = nen3v[3 * ie], k2 = nen3v[3 * ie + 1], k3 = nen3v[3 * ie + 2];
    if (k1 < 0 || k2 < 0 || k3 < 0 || k1 >= nkn || k2 >= nkn || k3 >= nkn)
      return fail(SHY_EARG, "set_ev: node index out of range");
    double x1 = x[k1], y1 = y[k1], x2 = x[k2], y2 = y[k2], x3 = x[k3], y3 = y[k3];
    double a1 = x2 * y3 - x3 * y2, a2 = x3 * y1 - x1 * y3, a3 = x1 * y2 - x2 * y1;
    double aj = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
    if (aj <= 0) return fail(SHY_EARG, "set_ev: element with non-positive area");
    double aji = 1. / aj;
    double b1 = (y2 - y3) * aji, c1 = (x3 - x2) * aji;
    double b2 = (y3 - y1) * aji, c2 = (x1 - x3) * aji;
    double b3 = (y1 - y2) * aji, c3 = (x2 - x1) * aji;
    a1 *= aji; a2 *= aji; a3 *= aji;
    adjust_bc(b1, b2, b3);
    adjust_bc(c1, c2, c3);
    double ss1 = (x3 - x2) * (x3 - x2) + (y3 - y2) * (y3 - y2), s1 = std::sqrt(ss1);
    double ss2 = (x3 - x1) * (x3 - x1) + (y3 - y1) * (y3 - y1), s2 = std::sqrt(ss2);
    double ss3 = (x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1), s3 = std::sqrt(ss3);
    double d1 = std::acos((ss2 + ss3 - ss1) / (2. * s2 * s3)) * rad;
    double d2 = std::acos((ss1 + ss3 - ss2) / (2. * s1 * s3)) * rad;
    double d3 = std::acos((ss1 + ss2 - ss3) / (2. * s1 * s2)) * rad;
    double dd1 = aj * std::sqrt(b1 * b1 + c1 * c1);
    double dd2 = aj * std::sqrt(b2 * b2 + c2 * c2);
    double dd3 = aj * std::sqrt(b3 * b3 + c3 * c3);
    double *e = ev + (size_t)ie * SHY_EVDIM;
    e[0] = a1; e[1] = a2; e[2] = a3;
    e[3] = b1; e[4] = b2; e[5] = b3;
    e[6] = c1; e[7] = c2; e[8] = c3;
    e[9] = aj / 24.;
    e[10] = d1; e[11] = d2; e[12] = d3;
    e[13] = dd1; e[14] = dd2; e[15] = dd3;
    e[16] = s1; e[17] = s2; e[18] = s3;
  }
  return SHY_OK;
}

// ---------------------------------------------------------------------------
// Band solvers: src/external/sparskit/penta.f90
// val(-2:2,n) row-banded: val(j,i) is the entry (i, i+j); stored val[5*i + j+2].
// ---------------------------------------------------------------------------
int penta_fact(int n, double *val) {           // penta.f90:215-296
  if (n < 4) return fail(SHY_EARG, "penta_fact: n<4");
  auto V = [&](int j, int i) -> double & { return val[5 * (i - 1) + j + 2]; };
  std::vector<double> x(n + 2), y(n + 2), z(n + 2);
  z[1] = 0.;
  int i = 1;
  double xx = V(0, i);
  if (xx == 0.) return fail(SHY_ESINGULAR, "penta_fact: matrix singular");
  x[i] = xx; y[i] = V(1, i); z[i + 1] = V(-1, i + 1) / xx; V(-2, i + 2) = V(-2, i + 2) / xx;
  i = 2;
  xx = V(0, i) - y[i - 1] * z[i];
  if (xx == 0.) return fail(SHY_ESINGULAR, "penta_fact: matrix singular");
  x[i] = xx; y[i] = V(1, i) - z[i] * V(2, i - 1);
  z[i + 1] = (V(-1, i + 1) - V(-2, i + 1) * y[i - 1]) / xx;
  V(-2, i + 2) = V(-2, i + 2) / xx;
  for (i = 3; i <= n - 2; i++) {
    xx = V(0, i) - y[i - 1] * z[i] - V(-2, i) * V(2, i - 2);
    if (xx == 0.) return fail(SHY_ESINGULAR, "penta_fact: matrix singular");
    x[i] = xx; y[i] = V(1, i) - z[i] * V(2, i - 1);
    z[i + 1] = (V(-1, i + 1) - V(-2, i + 1) * y[i - 1]) / xx;
    V(-2, i + 2) = V(-2, i + 2) / xx;
  }
  i = n - 1;
  xx = V(0, i) - y[i - 1] * z[i] - V(-2, i) * V(2, i - 2);
  if (xx == 0.) return fail(SHY_ESINGULAR, "penta_fact: matrix singular");
  x[i] = xx; y[i] = V(1, i) - z[i] * V(2, i - 1);
  z[i + 1] = (V(-1, i + 1) - V(-2, i + 1) * y[i - 1]) / xx;
  i = n;
  xx = V(0, i) - y[i - 1] * z[i] - V(-2, i) * V(2, i - 2);
  if (xx == 0.) return fail(SHY_ESINGULAR, "penta_fact: matrix singular");
  x[i] = xx; y[i] = 0.;
  for (int k = 1; k <= n; k++) { V(0, k) = x[k]; V(1, k) = y[k]; V(-1, k) = z[k]; }
  return SHY_OK;
}

void penta_solve(int n, const double *val, const double *r, double *s) {  // penta.f90:104-138
  auto V = [&](int j, int i) { return val[5 * (i - 1) + j + 2]; };
  std::vector<double> g(n + 1);
  g[1] = r[0];
  g[2] = r[1] - V(-1, 2) * g[1];
  for (int i = 3; i <= n; i++) g[i] = r[i - 1] - V(-1, i) * g[i - 1] - V(-2, i) * g[i - 2];
  s[n - 1] = g[n] / V(0, n);
  s[n - 2] = (g[n - 1] - V(1, n - 1) * s[n - 1]) / V(0, n - 1);
  for (int i = n - 2; i >= 1; i--)
    s[i - 1] = (g[i] - V(1, i) * s[i] - V(2, i) * s[i + 1]) / V(0, i);
}

int penta_factf(int n, double *val) {          // penta.f90:142-211
  if (n < 4) return fail(SHY_EARG, "penta_factf: n<4");
  auto V = [&](int j, int i) -> double & { return val[5 * (i - 1) + j + 2]; };
  int i = 1;
  double xx = V(0, 1);
  if (xx == 0.) return fail(SHY_ESINGULAR, "penta_factf: matrix singular");
  V(-1, 2) = V(-1, 2) / xx;
  V(-2, 3) = V(-2, 3) / xx;
  i = 2;
  xx = V(0, 2) - V(1, 1) * V(-1, 2);
  if (xx == 0.) return fail(SHY_ESINGULAR, "penta_factf: matrix singular");
  V(0, 2) = xx;
  V(1, 2) = V(1, 2) - V(-1, 2) * V(2, 1);
  V(-1, 3) = (V(-1, 3) - V(-2, 3) * V(1, 1)) / xx;
  V(-2, 4) = V(-2, 4) / xx;
  for (i = 3; i <= n - 2; i++) {
    xx = V(0, i) - V(1, i - 1) * V(-1, i) - V(-2, i) * V(2, i - 2);
    if (xx == 0.) return fail(SHY_ESINGULAR, "penta_factf: matrix singular");
    V(0, i) = xx;
    V(1, i) = V(1, i) - V(-1, i) * V(2, i - 1);
    V(-1, i + 1) = (V(-1, i + 1) - V(-2, i + 1) * V(1, i - 1)) / xx;
    V(-2, i + 2) = V(-2, i + 2) / xx;
  }
  int n1 = n - 1, n2 = n - 2;
  xx = V(0, n1) - V(1, n2) * V(-1, n1) - V(-2, n1) * V(2, n - 3);
  if (xx == 0.) return fail(SHY_ESINGULAR, "penta_factf: matrix singular");
  V(0, n1) = xx;
  V(1, n1) = V(1, n1) - V(-1, n1) * V(2, n2);
  V(-1, n) = (V(-1, n) - V(-2, n) * V(1, n2)) / xx;
  xx = V(0, n) - V(1, n1) * V(-1, n) - V(-2, n) * V(2, n2);
  if (xx == 0.) return fail(SHY_ESINGULAR, "penta_factf: matrix singular");
  V(0, n) = xx;
  return SHY_OK;
}

// tria_multi (penta.f90:332-372): v(3,n) lower/centre/upper, m right-hand sides r(n,m)
void tria_multi(int n, int m, double *v, double *r, double *s) {
  for (int i = 2; i <= n; i++) {
    double aux = v[3 * (i - 1) + 0] / v[3 * (i - 2) + 1];
    v[3 * (i - 1) + 1] = v[3 * (i - 1) + 1] - aux * v[3 * (i - 2) + 2];
    for (int j = 0; j < m; j++) r[j * n + i - 1] = r[j * n + i - 1] - aux * r[j * n + i - 2];
  }
  for (int j = 0; j < m; j++) {
    s[j * n + n - 1] = r[j * n + n - 1] / v[3 * (n - 1) + 1];
    for (int i = n - 1; i >= 1; i--)
      s[j * n + i - 1] = (r[j * n + i - 1] - v[3 * (i - 1) + 2] * s[j * n + i]) / v[3 * (i - 1) + 1];
  }
}

// ---------------------------------------------------------------------------
// UNESCO 1981 equation of state (Millero & Poisson; Fofonoff & Millard 1983)
// as used by sigma_stp (src/shyfem/eq_state.f90:154-230): density at one
// atmosphere plus the secant bulk modulus; returns rho - 1000 [kg/m^3].
// p is the pressure in bar.
// ---------------------------------------------------------------------------
double sigma_stp(double s, double t, double p) {
  // density of pure water (SMOW) and its salinity terms at p = 0
  double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  double s32 = std::sqrt(s * s * s);
  double rw = 999.842594 + 6.793952e-2 * t - 9.095290e-3 * t2 + 1.001685e-4 * t3
              - 1.120083e-6 * t4 + 6.536332e-9 * t5;
  double a = 8.24493e-1 - 4.0899e-3 * t + 7.6438e-5 * t2 - 8.2467e-7 * t3 + 5.3875e-9 * t4;
  double b = -5.72466e-3 + 1.0227e-4 * t - 1.6546e-6 * t2;
  double c = 4.8314e-4;
  double rho0 = rw + a * s + b * s32 + c * s * s;
  // secant bulk modulus K(s,t,p)
  double kw = 19652.21 + 148.4206 * t - 2.327105 * t2 + 1.360477e-2 * t3 - 5.155288e-5 * t4;
  double aw = 3.239908 + 1.43713e-3 * t + 1.16092e-4 * t2 - 5.77905e-7 * t3;
  double bw = 8.50935e-5 - 6.12293e-6 * t + 5.2787e-8 * t2;
  double k0 = kw + (54.6746 - 0.603459 * t + 1.09987e-2 * t2 - 6.1670e-5 * t3) * s
              + (7.944e-2 + 1.6483e-2 * t - 5.3009e-4 * t2) * s32;
  double aa = aw + (2.2838e-3 - 1.0981e-5 * t - 1.6078e-6 * t2) * s + 1.91075e-4 * s32;
  double bb = bw + (-9.9348e-7 + 2.0816e-8 * t + 9.1697e-10 * t2) * s;
  double kk = k0 + aa * p + bb * p * p;
  return rho0 / (1. - p / kk) - 1000.;
}

// ---------------------------------------------------------------------------
// Sparse pattern: construct_node_list + coo_init_new (src/shyfem/coo_matrix.f90:51-185,
// 330-400).  Rows are nodes with their sorted neighbour lists (diagonal
// included); ijp_ie(i,j,ie) points each element entry to its slot.  The COO
// arrays are row-sorted, so they are a CSR with row pointer ntg.
// ---------------------------------------------------------------------------
int coo_init(int nkn, int nel, const int *nen3v, std::vector<int> &ntg, std::vector<int> &icol,
             std::vector<int> &ijp) {
  std::vector<std::vector<int>> nl(nkn);
  for (int ie = 0; ie < nel; ie++)
    for (int ii = 0; ii < 3; ii++) {
      int k1 = nen3v[3 * ie + ii], k2 = nen3v[3 * ie + (ii + 1) % 3];
      nl[k1].push_back(k2);
      nl[k2].push_back(k1);
    }
  ntg.assign(nkn + 1, 0);
  icol.clear();
  for (int k = 0; k < nkn; k++) {
    nl[k].push_back(k);
    std::sort(nl[k].begin(), nl[k].end());
    nl[k].erase(std::unique(nl[k].begin(), nl[k].end()), nl[k].end());
    ntg[k + 1] = ntg[k] + (int)nl[k].size();
    for (int j : nl[k]) icol.push_back(j);
  }
  ijp.assign((size_t)9 * nel, -1);
  for (int ie = 0; ie < nel; ie++)
    for (int i = 0; i < 3; i++) {
      int ki = nen3v[3 * ie + i];
      for (int j = 0; j < 3; j++) {
        int kj = nen3v[3 * ie + j];
        int m = -1;
        for (int p = ntg[ki]; p < ntg[ki + 1]; p++)
          if (icol[p] == kj) { m = p; break; }
        if (m < 0) return fail(SHY_EARG, "coo_init: internal error (2)");
        ijp[(size_t)9 * ie + 3 * i + j] = m;
      }
    }
  return SHY_OK;
}

// ---------------------------------------------------------------------------
// ILUT (Saad, "ILUT: a dual threshold incomplete LU factorization", 1994;
// Iterative Methods for Sparse Linear Systems, 2nd ed., Alg. 10.6) with the
// parameters of sparskit_admin.f90:226-251 (lfil = 5, droptol = 0.01):
// row-wise elimination in increasing column order, drop of multipliers and
// of updated entries below droptol * (mean |a_ij| of the row), then keep the
// lfil largest entries of the L and of the U part; a zero pivot is replaced
// by (1e-4 + droptol) * rownorm.  Stored as L (unit, strictly lower) and U
// with the inverted diagonal.
// ---------------------------------------------------------------------------
struct Ilu {
  int n = 0;
  std::vector<int> lptr, lcol, uptr, ucol;
  std::vector<double> lval, uval, dinv;
};

int ilut(int n, const int *ia, const int *ja, const double *a, int lfil, double droptol, Ilu &f) {
  f.n = n;
  f.lptr.assign(n + 1, 0); f.uptr.assign(n + 1, 0); f.dinv.assign(n, 0.);
  f.lcol.clear(); f.lval.clear(); f.ucol.clear(); f.uval.clear();
  std::vector<double> w(n, 0.);
  std::vector<int> pos(n, -1);         // position marker
  std::vector<int> lidx, uidx;
  for (int i = 0; i < n; i++) {
    double tnorm = 0.;
    for (int p = ia[i]; p < ia[i + 1]; p++) tnorm += std::fabs(a[p]);
    if (tnorm == 0.) return fail(SHY_ESINGULAR, "ilut: zero row");
    tnorm /= (double)(ia[i + 1] - ia[i]);
    lidx.clear(); uidx.clear();
    double wdiag = 0.;
    bool has_diag = false;
    for (int p = ia[i]; p < ia[i + 1]; p++) {
      int j = ja[p];
      if (j < i) { lidx.push_back(j); w[j] = a[p]; pos[j] = 1; }
      else if (j == i) { wdiag = a[p]; has_diag = true; }
      else { uidx.push_back(j); w[j] = a[p]; pos[j] = 1; }
    }
    (void)has_diag;
    std::vector<int> lkept;
    std::vector<double> lkeptv;
    // eliminate in increasing column order (fill-ins may add new lower columns)
    size_t done = 0;
    std::sort(lidx.begin(), lidx.end());
    while (done < lidx.size()) {
      // pick smallest remaining column
      size_t best = done;
      for (size_t q = done + 1; q < lidx.size(); q++)
        if (lidx[q] < lidx[best]) best = q;
      std::swap(lidx[done], lidx[best]);
      int jrow = lidx[done++];
      double fact = w[jrow] * f.dinv[jrow];
      w[jrow] = 0.; pos[jrow] = -1;
      if (std::fabs(fact) <= droptol * tnorm) continue;
      for (int p = f.uptr[jrow]; p < f.uptr[jrow + 1]; p++) {
        int j = f.ucol[p];
        double s = fact * f.uval[p];
        if (j == i) { wdiag -= s; continue; }
        if (pos[j] < 0) {
          pos[j] = 1; w[j] = -s;
          if (j < i) lidx.push_back(j); else uidx.push_back(j);
        } else {
          w[j] -= s;
        }
      }
      lkept.push_back(jrow); lkeptv.push_back(fact);
    }
    // L part: keep lfil largest multipliers
    std::vector<int> ord(lkept.size());
    for (size_t q = 0; q < ord.size(); q++) ord[q] = (int)q;
    std::stable_sort(ord.begin(), ord.end(),
                     [&](int x, int y) { return std::fabs(lkeptv[x]) > std::fabs(lkeptv[y]); });
    if ((int)ord.size() > lfil) ord.resize(lfil);
    std::sort(ord.begin(), ord.end(), [&](int x, int y) { return lkept[x] < lkept[y]; });
    for (int q : ord) { f.lcol.push_back(lkept[q]); f.lval.push_back(lkeptv[q]); }
    f.lptr[i + 1] = (int)f.lcol.size();
    // U part: drop small, keep lfil largest
    std::vector<int> uk;
    for (int j : uidx) {
      if (std::fabs(w[j]) > droptol * tnorm) uk.push_back(j);
    }
    std::stable_sort(uk.begin(), uk.end(),
                     [&](int x, int y) { return std::fabs(w[x]) > std::fabs(w[y]); });
    if ((int)uk.size() > lfil) uk.resize(lfil);
    std::sort(uk.begin(), uk.end());
    for (int j : uk) { f.ucol.push_back(j); f.uval.push_back(w[j]); }
    f.uptr[i + 1] = (int)f.ucol.size();
    for (int j : uidx) { w[j] = 0.; pos[j] = -1; }
    if (wdiag == 0.) wdiag = (0.0001 + droptol) * tnorm;
    f.dinv[i] = 1. / wdiag;
  }
  return SHY_OK;
}

void lusol(const Ilu &f, const double *y, double *x) {   // solve L U x = y
  int n = f.n;
  for (int i = 0; i < n; i++) {
    double s = y[i];
    for (int p = f.lptr[i]; p < f.lptr[i + 1]; p++) s -= f.lval[p] * x[f.lcol[p]];
    x[i] = s;
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = x[i];
    for (int p = f.uptr[i]; p < f.uptr[i + 1]; p++) s -= f.uval[p] * x[f.ucol[p]];
    x[i] = s * f.dinv[i];
  }
}

void amux(int n, const int *ia, const int *ja, const double *a, const double *x, double *y) {
  for (int i = 0; i < n; i++) {      // spk_matvec.f90:74 (CSR y = A x)
    double t = 0.;
    for (int p = ia[i]; p < ia[i + 1]; p++) t += a[p] * x[ja[p]];
    y[i] = t;
  }
}

double dot(int n, const double *x, const double *y) {
  double s = 0.;
  for (int i = 0; i < n; i++) s += x[i] * y[i];
  return s;
}

// BiCGStab (van der Vorst 1992) with right preconditioning, the solver the
// reference selects (itsol = 3, ipar(2) = 1, sparskit_admin.f90:234,268), with
// the stop test of stopbis (spk_iters.f90:3304-3360) under ipar(3) = 1:
// ||r|| <= rtol * ||r0|| + atol, and a limit of maxmv matrix-vector products.
int bcgstab(int n, const int *ia, const int *ja, const double *a, const Ilu &M, const double *b,
            double *x, double rtol, double atol, int maxmv, int *iters, double *r0n, double *rn) {
  std::vector<double> r(n), rh(n), p(n, 0.), v(n, 0.), ph(n), s(n), sh(n), t(n);
  amux(n, ia, ja, a, x, r.data());
  for (int i = 0; i < n; i++) r[i] = b[i] - r[i];
  rh = r;
  double norm0 = std::sqrt(dot(n, r.data(), r.data()));
  *r0n = norm0;
  double tol = rtol * norm0 + atol;
  int nmv = 1;
  *iters = 0;
  if (norm0 <= tol) { *rn = norm0; return SHY_OK; }
  double rho = 1., alpha = 1., omega = 1.;
  while (true) {
    double rho1 = dot(n, rh.data(), r.data());
    double beta = (rho1 / rho) * (alpha / omega);
    rho = rho1;
    for (int i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
    lusol(M, p.data(), ph.data());
    amux(n, ia, ja, a, ph.data(), v.data()); nmv++;
    alpha = rho / dot(n, rh.data(), v.data());
    for (int i = 0; i < n; i++) s[i] = r[i] - alpha * v[i];
    (*iters)++;
    double sn = std::sqrt(dot(n, s.data(), s.data()));
    if (sn <= tol) {
      for (int i = 0; i < n; i++) x[i] += alpha * ph[i];
      *rn = sn;
      return SHY_OK;
    }
    lusol(M, s.data(), sh.data());
    amux(n, ia, ja, a, sh.data(), t.data()); nmv++;
    double tt = dot(n, t.data(), t.data());
    omega = tt > 0 ? dot(n, t.data(), s.data()) / tt : 0.;
    for (int i = 0; i < n; i++) {
      x[i] += alpha * ph[i] + omega * sh[i];
      r[i] = s[i] - omega * t[i];
    }
    double nr = std::sqrt(dot(n, r.data(), r.data()));
    *rn = nr;
    if (!(nr > tol)) return SHY_OK;
    if (nmv >= maxmv) return fail(SHY_ENOCONV, "bcgstab: iteration limit reached");
    if (omega == 0.) return fail(SHY_ENOCONV, "bcgstab: breakdown");
  }
}

// ---------------------------------------------------------------------------
// The model (one basin, FP64 state)
// ---------------------------------------------------------------------------
struct Model {
  int nkn = 0, nel = 0, nlv = 0;
  shy_params p{};
  std::vector<int> nen3v, ilhv, ilhkv, bnd, ieltv;
  std::vector<double> ev, hm3v, hev, hlv, hldv, czv, fcorv, visv, difv, tauxnv, tauynv, ppv, rqv;
  std::vector<double> tide;
  int nbnd = 0, ntide = 0;
  std::vector<double> areakv, wdifhv, difhv;
  std::vector<int> ntg, icol, ijp;
  // state (reference layouts)
  std::vector<double> znv, zov, zenv, zeov, rzv;
  std::vector<double> utlnv, vtlnv, utlov, vtlov, unv, vnv;
  std::vector<double> hdknv, hdkov, hdenv, hdeov, wlnv;
  std::vector<double> tempv, saltv, rhov, conzv;
  std::vector<double> tbnd, sbnd, cbnd;     // scalar boundary values: imposed on level
                                            // boundaries, brought in by inflows
  std::vector<double> mfluxv;               // (nkn, nlv) discharge per node layer (set_mass_flux)
  std::vector<double> rfricv, fxv, fyv, ddxv, ddyv;
  std::vector<double> c2coo, rvec2d;
  double dtime = 0.;
  // wetting and drying (mod_geom_dynamic :: iwegv, iwetv, inodv)
  std::vector<int> iwegv, iwetv, inodv;
  std::vector<double> uov, vov;             // barotropic transports of the old level
  std::vector<double> uprv, vprv;           // nodal velocities (mod_hydro_print), make_prvel
  std::vector<double> andgzv;               // water-level nudging contribution per node (mod_nudging)
  // conz3d_omp's source terms for one tracer (concentration_omp.f90:92-98):
  // nudging to cobs at rate robs*rtauv, settling at wsink*wsinkv, loading
  // rload*load; all (nkn, nlv) rows but wsinkv (nkn, nlv+1), interfaces 0..nlv
  struct ScalarTerms {
    int itr = -1;
    double robs = 0., wsink = 0., rload = 0.;
    std::vector<double> cobs, rtauv, wsinkv, load;
  } sterm;
  // itvd = 2: per element and ordered vertex pair (c, d) the element holding
  // the point 2 x_c - x_d and its barycentric weights there (tvd_upwind_init_elem)
  std::vector<int> tvdup_e;                 // [6*ie + slot], -1 outside the basin
  std::vector<double> tvdup_xi;             // [3*(6*ie + slot) + i]
  double dtime_weg = -1.;                   // setweg's dtime_old
  // non-hydrostatic pressure (mod_nohyd): qpov, qpnv (nkn, nlv) rows,
  // qdistv (nkn) its weight near open boundaries (qhdist; 1 by default),
  // wlov the old vertical velocity (copy_uvz), wnh the non-hydrostatic w
  // of sp256wnh (nkn, nlv+1); the 3D system (coo_init_new's 3D part):
  // nt3g row-block offsets, c3coo/rvec3d its values and right-hand side
  std::vector<double> qpov, qpnv, qdistv, wlov, wnh;
  std::vector<int> nt3g;
  std::vector<double> c3coo, rvec3d;
  int nh_iters = 0;
  double nh_resid0 = 0., nh_resid = 0.;
  shy_step_info info{};
  // solver controls
  double rtol = 1e-8, atol = 1e-8;
  int maxmv = 1000;
};

inline double &A2(std::vector<double> &a, int n1, int i, int j) { return a[(size_t)j * n1 + i]; }

// set_area (elems_dealing.f90:658-705)
void set_area(Model &m) {
  m.areakv.assign((size_t)m.nlv * m.nkn, 0.);
  for (int ie = 0; ie < m.nel; ie++) {
    double areafv = 12. * m.ev[(size_t)ie * SHY_EVDIM + 9] / 3.;
    for (int ii = 0; ii < 3; ii++) {
      int k = m.nen3v[3 * ie + ii];
      for (int l = 0; l < m.ilhv[ie]; l++) m.areakv[(size_t)k * m.nlv + l] += areafv;
    }
  }
}

// diffweight (diffusion_admin.f90:178-330) with idtype = 2 (def_para.f90:1021)
void diffweight(Model &m) {
  m.wdifhv.assign((size_t)9 * m.nel, 0.);
  const double fact = 2. / 3.;
  for (int ie = 0; ie < m.nel; ie++) {
    double bc[3][3] = {{0}};
    const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
    for (int i = 0; i < 3; i++) {
      int ia = (i + 1) % 3, ib = (i + 2) % 3;
      double w = 1. / (e[13 + i] * e[13 + i]) * fact;
      bc[ia][ib] = -w; bc[ib][ia] = -w; bc[i][i] = 0.;
    }
    for (int ii = 0; ii < 3; ii++) {
      double w = 0.;
      for (int iii = 0; iii < 3; iii++) w += bc[ii][iii];
      bc[ii][ii] = -w;
    }
    for (int ii = 0; ii < 3; ii++)
      for (int iii = 0; iii < 3; iii++) m.wdifhv[(size_t)9 * ie + 3 * ii + iii] = bc[ii][iii];
  }
}

// element neighbours opposite each vertex (ieltv); -1 on the boundary
void set_ieltv(Model &m) {
  m.ieltv.assign((size_t)3 * m.nel, -1);
  std::vector<std::vector<int>> inc(m.nkn);
  for (int ie = 0; ie < m.nel; ie++)
    for (int ii = 0; ii < 3; ii++) inc[m.nen3v[3 * ie + ii]].push_back(ie);
  for (int ie = 0; ie < m.nel; ie++)
    for (int ii = 0; ii < 3; ii++) {
      int k1 = m.nen3v[3 * ie + (ii + 1) % 3], k2 = m.nen3v[3 * ie + (ii + 2) % 3];
      for (int je : inc[k1]) {
        if (je == ie) continue;
        bool has = false;
        for (int jj = 0; jj < 3; jj++) has |= m.nen3v[3 * je + jj] == k2;
        if (has) { m.ieltv[3 * ie + ii] = je; break; }
      }
    }
}

// z-adaptive (z-star) layers of z-layer basins with nzadapt > 1
// (zadaptutil.f90).  compute_rzmov_info (:100-117): the threshold factor.
double zad_rzmov(int nlv, int nzadapt, const std::vector<double> &hlv) {
  if (nzadapt <= 1) return 0.;
  if (nzadapt >= nlv) return 10000.;
  return hlv[nzadapt - 2] / (hlv[nzadapt - 1] - hlv[nzadapt - 2]);
}

// compute_nadapt_info (:212-240): the lowest layer that follows the level
// z (1-based; 0: none) in a column of lmax layers
int zad_levmax(double z, const std::vector<double> &hlv, int lmax, double rzmov) {
  int nad = 0;
  for (int l = 1; l <= lmax - 1; l++) {
    const double hl = hlv[l - 1], hp = l > 1 ? hlv[l - 2] : 0.;
    if (z <= -hl + rzmov * (hl - hp)) nad = l + 1;
    else break;
  }
  return nad;
}

// the thickness of layer l (1-based) at an element vertex of level z and
// depth htot (setdepth :1014-1055 with compute_zadaptive_info :321-380): the
// layers down to levmax share the column hzad = hadapt + z in proportion to
// their nominal thickness (the weights (hlv(l-1) - hlv(l)) / hadapt, with
// the surface at 0 and, when levmax is the bottom layer, hadapt = htot);
// below them z-layers, the first one plus z when no layer follows the level
double zad_vertex_h(int l, double z, double htot, int lmax, int levmax, const Model &m) {
  if (levmax > 0 && l <= levmax) {
    const double had = levmax == lmax ? htot : m.hlv[levmax - 1];
    const double htop = l == 1 ? 0. : m.hlv[l - 2], hbot = l == lmax ? htot : m.hlv[l - 1];
    return -(had + z) * ((htop - hbot) / had);
  }
  if (lmax == 1) return htot + z;
  if (l < lmax) return m.hldv[l - 1] + (levmax == 0 && l == 1 ? z : 0.);
  return htot - m.hlv[lmax - 2];
}

// setdepth (elems_dealing.f90:930-1160) for z-layers (nsigma = 0), pure
// sigma layers (nsigma = nlv) and hybrid layers (nsigma sigma layers down to
// hsigma, z-layers below), and z-layers with z-adaptive surface layers
// (nzadapt > 1, nsigma = 0; zad_vertex_h above; an element's layers down to
// the deepest levmax of its vertices are the means of the vertex values).
// Without nzadapt compute_zadaptive_info returns nadapt = ladapt = 0
// (zadaptutil.f90:321-324).  Sigma layers take
// the fraction -hldv(l) of the total depth min(h, hsigma) + z: at the nodes
// from each element's vertex values in element order, the last element
// writing (:1010-1025), at the elements from hev and the mean water level
// (:1075-1085).  z-layers take their nominal thickness, the first one (with
// no sigma layers above) plus z, the last one down to the bottom; at the
// nodes as area-weighted means over the elements (:1026-1050, 1129-1140).
int setdepth(Model &m, std::vector<double> &hdkn, std::vector<double> &hden,
             const std::vector<double> &zenv) {
  const int nlv = m.nlv, nsigma = m.p.nsigma;
  const double hsigma = (double)(float)(m.p.hsigma > 0.f ? m.p.hsigma : 10000.f);
  hdkn.assign((size_t)nlv * m.nkn, 0.);
  hden.assign((size_t)nlv * m.nel, 0.);
  if (m.p.nzadapt > 1 && nsigma == 0) {
    const double rzmov = zad_rzmov(nlv, m.p.nzadapt, m.hlv);
    for (int ie = 0; ie < m.nel; ie++) {
      const double areafv = 12. * m.ev[(size_t)ie * SHY_EVDIM + 9] / 3.;
      const int lmax = m.ilhv[ie];
      int lev[3];
      double zmed = 0.;
      for (int ii = 0; ii < 3; ii++) {
        const int k = m.nen3v[3 * ie + ii];
        const double z = zenv[3 * ie + ii], htot = m.hm3v[3 * ie + ii];
        zmed += z;
        lev[ii] = zad_levmax(z, m.hlv, lmax, rzmov);
        for (int l = 1; l <= lmax; l++) hdkn[(size_t)k * nlv + l - 1] += areafv * zad_vertex_h(l, z, htot, lmax, lev[ii], m);
      }
      zmed /= 3.;
      const int lad = std::max(lev[0], std::max(lev[1], lev[2]));
      const double htot = m.hev[ie];
      for (int l = 1; l <= lmax; l++) {
        double h;
        if (lad > 0 && l <= lad) {
          h = 0.;
          for (int ii = 0; ii < 3; ii++)
            h += zad_vertex_h(l, zenv[3 * ie + ii], m.hm3v[3 * ie + ii], lmax, lev[ii], m);
          h /= 3.;
        } else if (lmax == 1) h = htot + zmed;
        else if (l < lmax) h = m.hldv[l - 1] + (lad == 0 && l == 1 ? zmed : 0.);
        else h = htot - m.hlv[lmax - 2];
        if (!(h > 0.))
          return fail(SHY_EDEPTH, "setdepth: no layer depth in element " + std::to_string(ie + 1) +
                                      " layer " + std::to_string(l));
        hden[(size_t)ie * nlv + l - 1] = h;
      }
    }
  } else
  for (int ie = 0; ie < m.nel; ie++) {
    const double areafv = 12. * m.ev[(size_t)ie * SHY_EVDIM + 9] / 3.;
    const int lmax = m.ilhv[ie], lmin = 1;
    double zmed = 0.;
    for (int ii = 0; ii < 3; ii++) {
      const int k = m.nen3v[3 * ie + ii];
      const int lmink = 1;
      const double htot = m.hm3v[3 * ie + ii];
      const double z = zenv[3 * ie + ii];
      zmed += z;
      const double hsig = std::min(htot, hsigma) + z;
      for (int l = 1; l <= nsigma; l++) hdkn[(size_t)k * nlv + l - 1] = -hsig * m.hldv[l - 1];
      if (lmax <= nsigma) continue;
      if (lmax == lmin) {
        hdkn[(size_t)k * nlv + lmin - 1] += areafv * (htot + z);
      } else {
        const int levmin = nsigma + lmink;
        for (int l = levmin; l <= lmax - 1; l++) hdkn[(size_t)k * nlv + l - 1] += areafv * m.hldv[l - 1];
        if (levmin == lmink) hdkn[(size_t)k * nlv + lmink - 1] += areafv * z;
        const double hlast = htot - m.hlv[lmax - 2];
        if (hlast < 0.) return fail(SHY_EDEPTH, "setdepth: last layer negative");
        hdkn[(size_t)k * nlv + lmax - 1] += areafv * hlast;
      }
    }
    zmed /= 3.;
    const double htot = m.hev[ie];
    const double hsig = std::min(htot, hsigma) + zmed;
    for (int l = 1; l <= nsigma; l++) hden[(size_t)ie * nlv + l - 1] = -hsig * m.hldv[l - 1];
    if (lmax > nsigma) {
      if (lmax == lmin) {
        hden[(size_t)ie * nlv + lmin - 1] = htot + zmed;
      } else {
        const int levmin = nsigma + lmin;
        for (int l = levmin; l <= lmax - 1; l++) hden[(size_t)ie * nlv + l - 1] = m.hldv[l - 1];
        if (levmin == lmin) hden[(size_t)ie * nlv + lmin - 1] += zmed;
        const double hlast = htot - m.hlv[lmax - 2];
        if (hlast < 0.) return fail(SHY_EDEPTH, "setdepth: last layer negative");
        hden[(size_t)ie * nlv + lmax - 1] = hlast;
      }
    }
    for (int l = lmin; l <= lmax; l++)
      if (hden[(size_t)ie * nlv + l - 1] <= 0.)
        return fail(SHY_EDEPTH, "setdepth: no layer depth in element " + std::to_string(ie + 1) +
                                    " layer " + std::to_string(l));
  }
  for (int k = 0; k < m.nkn; k++) {
    for (int l = nsigma + 1; l <= m.ilhkv[k]; l++) {
      const double a = m.areakv[(size_t)k * nlv + l - 1];
      if (a > 0.) hdkn[(size_t)k * nlv + l - 1] /= a;
      else break;
    }
    for (int l = 1; l <= m.ilhkv[k]; l++)
      if (hdkn[(size_t)k * nlv + l - 1] <= 0.)
        return fail(SHY_EDEPTH, "setdepth: no layer depth in node");
  }
  return SHY_OK;
}

// rhoset (baroclinic.f90:654-710): one pass, pressure from the previous rho'
void rhoset(Model &m) {
  int nlv = m.nlv;
  double rho0 = m.p.rowass, sigma0 = rho0 - 1000.;
  for (int k = 0; k < m.nkn; k++) {
    double depth = 0., presbc = 0.;
    for (int l = 1; l <= m.ilhkv[k]; l++) {
      // sigma layers: the old thickness; z-layers: the nominal one
      double hlayer = l <= m.p.nsigma ? m.hdkov[(size_t)k * nlv + l - 1] : m.hldv[l - 1];
      double hh = 0.5 * hlayer;
      depth += hh;
      double rhop = m.rhov[(size_t)k * nlv + l - 1];
      double dpresc = rhop * m.p.grav * hh;
      presbc += dpresc;
      double presbt = rho0 * m.p.grav * depth;
      double pres = 1.e-5 * (presbt + presbc);
      double salt = std::max(0., m.saltv[(size_t)k * nlv + l - 1]);
      rhop = sigma_stp(salt, m.tempv[(size_t)k * nlv + l - 1], pres) - sigma0;
      m.rhov[(size_t)k * nlv + l - 1] = rhop;
      depth += hh;
      presbc += dpresc;
    }
  }
}

// tidal level boundary: sp111(2) -> get_oscil (bnd_admin.f90:1304-1320), the
// constituents of one boundary summed.
void set_rzv(Model &m) {
  m.rzv.assign(m.nkn, kFlag);
  for (int k = 0; k < m.nkn; k++) {
    int b = m.bnd[k];
    if (b <= 0) continue;
    double z = 0.;
    for (int c = 0; c < m.ntide; c++) {
      const double *t = &m.tide[((size_t)(b - 1) * m.ntide + c) * 4];
      double ampli = t[0], period = t[1], phase = t[2], zref = t[3];
      if (period == 0.) continue;
      z += zref + ampli * std::sin(2. * kPi * (m.dtime + phase) / period);
    }
    m.rzv[k] = z;
  }
}

// bottom_friction (chezy.f90:239-398), ireib = 0 and 5 (others: config error)
int bottom_friction(Model &m) {
  m.rfricv.assign(m.nel, 0.);
  for (int ie = 0; ie < m.nel; ie++) {
    int lmax = m.ilhv[ie];
    double uso = m.utlov[(size_t)ie * m.nlv + lmax - 1], vso = m.vtlov[(size_t)ie * m.nlv + lmax - 1];
    double uv = std::sqrt(uso * uso + vso * vso);
    double hzg = m.hdeov[(size_t)ie * m.nlv + lmax - 1];
    if (hzg < m.p.hzoff) hzg = m.p.hzoff;
    double rr;
    if (m.p.ireib == 0) rr = 0.;
    else if (m.p.ireib == 5) rr = m.czv[ie] * uv / (hzg * hzg);
    else return fail(SHY_EARG, "bottom_friction: ireib not supported");
    m.rfricv[ie] = rr;
  }
  return SHY_OK;
}

// set_explicit (explicit.f90:123-213): horizontal viscosity
// (set_diff_horizontal :389-493), the advective terms and the baroclinic
// pressure (set_barocl_new_interface :1226-1530; z, sigma and hybrid
// layers, no z-adaptation).
void set_explicit(Model &m) {
  int nlv = m.nlv;
  m.fxv.assign((size_t)nlv * m.nel, 0.);
  m.fyv.assign((size_t)nlv * m.nel, 0.);
  if (m.p.ahpar > 0) {
    for (int ie = 0; ie < m.nel; ie++) {
      int lmax = m.ilhv[ie];
      double area = 12. * m.ev[(size_t)ie * SHY_EVDIM + 9];
      double rdist = 1.;
      for (int ii = 0; ii < 3; ii++) {
        int iei = m.ieltv[3 * ie + ii];
        if (iei < 0) iei = ie;
        int lmaxi = m.ilhv[iei];
        double areai = 12. * m.ev[(size_t)iei * SHY_EVDIM + 9];
        for (int l = 1; l <= lmax; l++) {
          if (l > lmaxi) break;
          double u = m.utlov[(size_t)ie * nlv + l - 1], v = m.vtlov[(size_t)ie * nlv + l - 1];
          double ui = m.utlov[(size_t)iei * nlv + l - 1], vi = m.vtlov[(size_t)iei * nlv + l - 1];
          double anu = m.p.ahpar * m.difhv[(size_t)ie * nlv + l - 1];
          double ai = 2. * anu / (area + areai);
          m.fxv[(size_t)ie * nlv + l - 1] -= rdist * ai * (ui - u);
          m.fyv[(size_t)ie * nlv + l - 1] -= rdist * ai * (vi - v);
        }
      }
    }
  }
  if (m.p.ilin == 0) {
    // set_advective (explicit.f90:685-861) with itlin 0, ihwadv 0 (no
    // vertical momentum advection) and rdistv = rcomputev = 1 (nadist 0):
    // set_momentum_flux (:588-683) first gives every node layer the momentum
    // flowing into it, weighted by the inflow, or, with outflow only, its
    // velocity from the last step's nodal velocities (uprv) times its old
    // thickness; each element layer then takes the upwind difference over
    // the vertices it receives flow from
    const size_t nn = (size_t)nlv * m.nkn;
    std::vector<double> saux(nn, 0.), momx(nn, 0.), momy(nn, 0.);
    for (int ie = 0; ie < m.nel; ie++) {
      const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
      for (int l = 0; l < m.ilhv[ie]; l++) {
        const double ut = m.utlov[(size_t)ie * nlv + l], vt = m.vtlov[(size_t)ie * nlv + l];
        for (int ii = 0; ii < 3; ii++) {
          const size_t kl = (size_t)m.nen3v[3 * ie + ii] * nlv + l;
          const double f = ut * e[3 + ii] + vt * e[6 + ii];   // > 0: flux into the node
          if (f > 0.) { saux[kl] += f; momx[kl] += f * ut; momy[kl] += f * vt; }
        }
      }
    }
    for (int k = 0; k < m.nkn; k++)
      for (int l = 0; l < m.ilhkv[k]; l++) {
        const size_t kl = (size_t)k * nlv + l;
        if (saux[kl] > 0.) { momx[kl] /= saux[kl]; momy[kl] /= saux[kl]; }
        else { momx[kl] = m.uprv[kl] * m.hdkov[kl]; momy[kl] = m.vprv[kl] * m.hdkov[kl]; }
      }
    const double rlin = m.p.rlin;
    const int ihwadv = m.p.ihwadv;
    for (int ie = 0; ie < m.nel; ie++) {
      const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
      const int lmax = m.ilhv[ie];
      // old velocities of the column (ulov = utlov/hdeov, ttov)
      auto ul = [&](int l, bool y) {
        const size_t el = (size_t)ie * nlv + l;
        const double h = m.hdeov[el];
        return h > 0. ? (y ? m.vtlov[el] : m.utlov[el]) / h : 0.;
      };
      double wtop = 0.;
      for (int l = 0; l < lmax; l++) {
        const size_t el = (size_t)ie * nlv + l;
        const double h = m.hdeov[el], ut = m.utlov[el], vt = m.vtlov[el];
        const double uc = ut / h, vc = vt / h;
        double xadv = 0., yadv = 0., wbot = 0.;
        for (int ii = 0; ii < 3; ii++) {
          const int k = m.nen3v[3 * ie + ii];
          const size_t kl = (size_t)k * nlv + l;
          wbot += m.wlnv[(size_t)k * (nlv + 1) + l + 1];       // old w at the layer's bottom
          const double f = ut * e[3 + ii] + vt * e[6 + ii];
          if (f < 0.) {                        // flux out of the node, into the element
            xadv += f * (momx[kl] / h - uc);
            yadv += f * (momy[kl] / h - vc);
          }
        }
        // vertical advection of momentum (:776-833)
        double zxadv = 0., zyadv = 0.;
        if (ihwadv > 0) {
          wbot /= 3.;
          if (l == lmax - 1) wbot = 0.;
          if (ihwadv == 1) {                   // upwind
            const int lt = wtop > 0. ? l : l - 1;
            zxadv = lt >= 0 ? wtop * ul(lt, false) : 0.;
            zyadv = lt >= 0 ? wtop * ul(lt, true) : 0.;
            const int lb = wbot > 0. ? l + 1 : l;
            zxadv -= lb < lmax ? wbot * ul(lb, false) : 0.;
            zyadv -= lb < lmax ? wbot * ul(lb, true) : 0.;
          } else {                             // centred
            const double dz = m.hdeov[el];
            double utop = 0., ubot = 0., vtop = 0., vbot = 0.;
            if (l > 0) {
              const double dztt = m.hdeov[el - 1];
              utop = (ul(l - 1, false) * dztt + ul(l, false) * dz) / (dztt + dz);
              vtop = (ul(l - 1, true) * dztt + ul(l, true) * dz) / (dztt + dz);
            }
            if (l < lmax - 1) {
              const double dzbb = m.hdeov[el + 1];
              ubot = (ul(l, false) * dz + ul(l + 1, false) * dzbb) / (dz + dzbb);
              vbot = (ul(l, true) * dz + ul(l + 1, true) * dzbb) / (dz + dzbb);
            }
            const double wlay = 0.5 * (wtop + wbot);
            zxadv = wlay * (utop - ubot);
            zyadv = wlay * (vtop - vbot);
          }
          wtop = wbot;
        }
        m.fxv[el] += rlin * (xadv + zxadv);
        m.fyv[el] += rlin * (yadv + zyadv);
      }
    }
  }
  bool bbarcl = m.p.ibarcl > 0 && m.p.ibarcl != 3 && m.p.ibarcl != 5;
  if (bbarcl) {
    // set_barocl_new_interface with bsigadjust (explicit.f90:1226-1530): on
    // sigma layers (l <= nsigma) the interfaces move with the level, so the
    // density gradient at interface l-1 is taken on the horizontal surface
    // at the element's mean depth of that interface: at each vertex the
    // density interpolated between the mid-layer depths of the node's
    // column that bracket it (hkkom, from the old level and old node
    // thickness), with the cases of vertices above the surface and below
    // the bottom; on z-layers the mean of the layer gradients.
    const int nsigma = m.p.nsigma;
    double raux = m.p.grav / m.p.rowass;
    std::vector<double> hkko, hkkom;
    if (nsigma > 0) {
      hkko.assign((size_t)(nlv + 1) * m.nkn, 0.);
      hkkom.assign((size_t)(nlv + 1) * m.nkn, 0.);
      for (int k = 0; k < m.nkn; k++) {
        double hkk = -m.zov[k];
        hkko[(size_t)k * (nlv + 1)] = hkk;
        hkkom[(size_t)k * (nlv + 1)] = hkk;
        for (int l = 1; l <= m.ilhkv[k]; l++) {
          hkk += m.hdkov[(size_t)k * nlv + l - 1];
          hkko[(size_t)k * (nlv + 1) + l] = hkk;
          hkkom[(size_t)k * (nlv + 1) + l] = 0.5 * (hkko[(size_t)k * (nlv + 1) + l] + hkko[(size_t)k * (nlv + 1) + l - 1]);
        }
      }
    }
    auto HO = [&](int l, int k) { return hkko[(size_t)k * (nlv + 1) + l]; };
    auto HM = [&](int l, int k) { return hkkom[(size_t)k * (nlv + 1) + l]; };
    auto RH = [&](int l, int k) { return m.rhov[(size_t)k * nlv + l - 1]; };
    for (int ie = 0; ie < m.nel; ie++) {
      const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
      int lmax = m.ilhv[ie];
      double presbcx = 0., presbcy = 0., brup = 0., crup = 0., hhup = 0.;
      for (int l = 1; l <= lmax; l++) {
        const bool bsigma = l <= nsigma;
        double hlayer = bsigma ? m.hdeov[(size_t)ie * nlv + l - 1] : m.hldv[l - 1];
        double hh = 0.5 * hlayer;
        double hint = hh + hhup;
        int llup[3] = {0, 0, 0}, lldown[3] = {0, 0, 0};
        double helei = 0.;
        if (bsigma) {
          for (int ii = 0; ii < 3; ii++) helei += HO(l - 1, m.nen3v[3 * ie + ii]);
          helei /= 3.;
          for (int ii = 0; ii < 3; ii++) {
            const int k = m.nen3v[3 * ie + ii], lkmax = m.ilhkv[k];
            int ll;
            if (helei < HO(l - 1, k)) {                  // look upwards
              for (ll = l - 1; ll >= 1; ll--) if (helei > HO(ll - 1, k)) break;
              if (ll <= 0) ll = 1;
            } else if (helei > HO(l, k)) {             // look downwards
              for (ll = l + 1; ll <= lkmax; ll++) if (helei < HO(ll, k)) break;
              if (ll > lkmax) ll = lkmax;
            } else {
              ll = l;
            }
            if (helei < HM(ll, k)) { llup[ii] = ll == 1 ? 1 : ll - 1; lldown[ii] = ll; }
            else { llup[ii] = ll; lldown[ii] = ll == lkmax ? lkmax : ll + 1; }
          }
        }
        int nb = 0, nn = 0;
        double br = 0., cr = 0., brl = 0., crl = 0.;
        for (int ii = 0; ii < 3; ii++) {
          const int k = m.nen3v[3 * ie + ii], lkmax = m.ilhkv[k];
          double rhop = RH(l, k);
          if (l == nsigma) { brl += e[3 + ii] * rhop; crl += e[6 + ii] * rhop; }
          if (bsigma) {
            const int lu = llup[ii], ld = lldown[ii];
            if (ld == 1) rhop = RH(1, k);
            else if (lu >= lkmax) { nb++; nn += ii + 1; rhop = RH(lkmax, k); }
            else {
              const double hu = HM(lu, k), hd = HM(ld, k);
              const double alpha = (helei - hu) / (hd - hu);
              rhop = alpha * RH(ld, k) + (1. - alpha) * RH(lu, k);
            }
          }
          br += e[3 + ii] * rhop;
          cr += e[6 + ii] * rhop;
        }
        double brint, crint;
        if (bsigma) {
          if (nb == 2) { brint = brup; crint = crup; }
          else if (nb == 1) {                           // the gradient along the bottom side kept
            const double b3 = e[3 + nn - 1], c3 = e[6 + nn - 1];
            const double aux = 1. / (c3 * c3 + b3 * b3);
            const double bn = aux * (brup * b3 + crup * c3) * b3, cn = aux * (brup * b3 + crup * c3) * c3;
            const double bt = br - aux * (br * b3 + cr * c3) * b3, ct = cr - aux * (br * b3 + cr * c3) * c3;
            brint = bn + bt; crint = cn + ct;
          } else { brint = br; crint = cr; }
        } else if (l == 1) { brint = br; crint = cr; }
        else { brint = 0.5 * (br + brup); crint = 0.5 * (cr + crup); }
        brup = br; crup = cr;
        if (l == nsigma) { brup = brl; crup = crl; }
        hhup = hh;
        presbcx += hint * brint;
        presbcy += hint * crint;
        m.fxv[(size_t)ie * nlv + l - 1] += raux * hlayer * presbcx;
        m.fyv[(size_t)ie * nlv + l - 1] += raux * hlayer * presbcy;
      }
    }
  }
  // nonhydro_set_explicit (nohydro.f90:526-586): the gradient of the old
  // non-hydrostatic pressure times the old thickness, weight 1 - aqpar (the
  // new pressure is zero here: nonhydro_copy cleared it at the step start)
  if (m.p.inohyd) {
    const double aqt = 1. - m.p.aqpar;
    for (int ie = 0; ie < m.nel; ie++) {
      const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
      for (int l = 1; l <= m.ilhv[ie]; l++) {
        double qx = 0., qy = 0.;
        for (int ii = 0; ii < 3; ii++) {
          const int k = m.nen3v[3 * ie + ii];
          const double qpo = m.qdistv[k] * m.qpov[(size_t)k * nlv + l - 1];
          qx += e[3 + ii] * qpo;
          qy += e[6 + ii] * qpo;
        }
        const double hhio = m.hdeov[(size_t)ie * nlv + l - 1];
        m.fxv[(size_t)ie * nlv + l - 1] += aqt * hhio * qx;
        m.fyv[(size_t)ie * nlv + l - 1] += aqt * hhio * qy;
      }
    }
  }
}

// hydro_intern (hydrodynamic.f90:868-1416) for one element column
int hydro_intern(Model &m, int ie) {
  const int nlv = m.nlv;
  const double dt = m.p.dt, at = m.p.atpar, af = m.p.afpar, grav = m.p.grav;
  const double rowass = m.p.rowass;
  const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
  int ilevel = m.ilhv[ie], jlevel = 1;
  int ngl = 2 * ilevel;
  bool b2d = (ngl == 2);
  double rcomp = 1., ruseterm = 1.;
  double bz = 0., cz = 0., bpres = 0., cpres = 0., taux = 0., tauy = 0.;
  int kn[3];
  double b[3], c[3];
  for (int ii = 0; ii < 3; ii++) {
    int kk = m.nen3v[3 * ie + ii];
    kn[ii] = kk;
    b[ii] = e[3 + ii]; c[ii] = e[6 + ii];
    double zz = m.zeov[3 * ie + ii];    // zeqv = 0 (no equilibrium tide)
    bz += zz * b[ii]; cz += zz * c[ii];
    bpres += m.ppv[kk] * b[ii]; cpres += m.ppv[kk] * c[ii];
    taux += m.tauxnv[kk]; tauy += m.tauynv[kk];
  }
  const double drittl = 1. / 3.;
  taux = rcomp * taux * drittl;
  tauy = rcomp * tauy * drittl;
  double gammat = m.fcorv[ie] * ruseterm;
  double gamma = af * dt * gammat;

  std::vector<double> hact(nlv + 2, 0.), rhact(nlv + 2, 0.), alev(nlv + 1, 0.);
  std::vector<double> smat(5 * (size_t)ngl, 0.), rvec(3 * (size_t)ngl, 0.), solv(3 * (size_t)ngl, 0.);
  double s2dmat[6] = {0, 0, 0, 0, 0, 0};
  for (int l = 1; l <= ilevel; l++) hact[l] = m.hdeov[(size_t)ie * nlv + l - 1];
  for (int l = 0; l <= ilevel + 1; l++) rhact[l] = hact[l] <= 0. ? 0. : 1. / hact[l];
  for (int l = jlevel - 1; l <= ilevel; l++) {
    double vis = m.p.vismol;
    vis += (m.visv[(size_t)kn[0] * (nlv + 1) + l] + m.visv[(size_t)kn[1] * (nlv + 1) + l] +
            m.visv[(size_t)kn[2] * (nlv + 1) + l]) / 3.;
    alev[l] = vis;
  }
  auto S = [&](int j, int row) -> double & { return smat[5 * (size_t)(row - 1) + j + 2]; };
  for (int l = 1; l <= ilevel; l++) {
    bool bfirst = l == jlevel, blast = l == ilevel;
    int lp = std::min(l + 1, ilevel), lm = std::max(l - 1, jlevel);
    double uui = m.utlov[(size_t)ie * nlv + l - 1], uuip = m.utlov[(size_t)ie * nlv + lp - 1];
    double uuim = m.utlov[(size_t)ie * nlv + lm - 1];
    double vvi = m.vtlov[(size_t)ie * nlv + l - 1], vvip = m.vtlov[(size_t)ie * nlv + lp - 1];
    double vvim = m.vtlov[(size_t)ie * nlv + lm - 1];
    double hhi = hact[l], hhip = hact[l + 1], hhim = hact[l - 1];
    double rhp = 0., rhm = 0.;
    if (hhi > 0.) {
      if (hhip > 0.) rhp = 2.0 * alev[l] / (hhi + hhip);
      if (hhim > 0.) rhm = 2.0 * alev[l - 1] / (hhi + hhim);
    }
    double aus = 1., aux = dt * at;
    double aa = aux * rhact[l] * (rhm + rhp);
    double aat = aus * rhact[l] * (rhm + rhp);
    double bb = aux * rhact[l + 1] * rhp;
    double bbt = aus * rhact[l + 1] * rhp;
    double cc = aux * rhact[l - 1] * rhm;
    double cct = aus * rhact[l - 1] * rhm;
    double ppx = 0., ppy = 0.;
    if (bfirst) { ppx -= taux; ppy -= tauy; }
    if (blast) {
      double rfric = m.rfricv[ie];
      aa += dt * rfric;
      aat += rfric;
    }
    double xexpl = m.fxv[(size_t)ie * nlv + l - 1], yexpl = m.fyv[(size_t)ie * nlv + l - 1];
    double presx = rcomp * bpres, presy = rcomp * cpres;
    double gravx = rcomp * grav * hhi * bz, gravy = rcomp * grav * hhi * cz;
    double ppx_aux = aat * uui - bbt * uuip - cct * uuim - gammat * vvi + gravx +
                     (hhi / rowass) * presx + xexpl;
    double ppy_aux = aat * vvi - bbt * vvip - cct * vvim + gammat * uui + gravy +
                     (hhi / rowass) * presy + yexpl;
    ppx += ppx_aux;
    ppy += ppy_aux;
    int jv = l + l, ju = jv - 1;
    if (b2d) {
      s2dmat[3 * 0 + 1] = 1. + aa;       // s2dmat(0,ju)
      s2dmat[3 * 1 + 1] = 1. + aa;       // s2dmat(0,jv)
      s2dmat[3 * 1 + 0] = gamma;         // s2dmat(-1,jv)
      s2dmat[3 * 0 + 2] = -gamma;        // s2dmat(+1,ju)
    } else {
      S(0, ju) = 1. + aa;
      S(0, jv) = 1. + aa;
      S(-1, jv) = gamma;
      S(+1, ju) = -gamma;
      if (!blast) { S(+2, ju) = -bb; S(+2, jv) = -bb; }
      if (!bfirst) { S(-2, ju) = -cc; S(-2, jv) = -cc; }
    }
    rvec[ju - 1] = ppx;
    rvec[jv - 1] = ppy;
    rvec[ngl + ju - 1] = hhi;
    rvec[ngl + jv - 1] = 0.;
    rvec[2 * ngl + ju - 1] = 0.;
    rvec[2 * ngl + jv - 1] = hhi;
  }
  std::vector<double> rvecp = rvec;
  if (b2d) {
    tria_multi(ngl, 3, s2dmat, rvecp.data(), solv.data());
  } else {
    int st = penta_fact(ngl, smat.data());
    if (st) return st;
    penta_solve(ngl, smat.data(), rvecp.data(), solv.data());
    penta_solve(ngl, smat.data(), rvecp.data() + ngl, solv.data() + ngl);
    penta_solve(ngl, smat.data(), rvecp.data() + 2 * ngl, solv.data() + 2 * ngl);
  }
  double dtafix = dt;     // iuvfix = 0
  for (int l = jlevel; l <= ilevel; l++) {
    m.utlnv[(size_t)ie * nlv + l - 1] = m.utlov[(size_t)ie * nlv + l - 1] - dtafix * solv[2 * l - 2];
    m.vtlnv[(size_t)ie * nlv + l - 1] = m.vtlov[(size_t)ie * nlv + l - 1] - dtafix * solv[2 * l - 1];
  }
  for (int l = 1; l <= ngl; l++) {
    m.ddxv[(size_t)ie * 2 * nlv + l - 1] = solv[ngl + l - 1];
    m.ddyv[(size_t)ie * 2 * nlv + l - 1] = solv[2 * ngl + l - 1];
  }
  return SHY_OK;
}

// hydro_zeta (hydrodynamic.f90:488-754) + system_assemble (simsys_spkaux.f90:533-594)
// + system_add_rhs (:687-705), element order ie = 1..nel.
void element_system(Model &m, int ie, int kn[3], double hia[3][3], double hik[3]) {
  const int nlv = m.nlv;
  const double az = m.p.azpar, am = m.p.ampar, ddt = m.p.dt;
  const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
  double b[3], c[3], z[3], zndg[3];
  for (int i = 0; i < 3; i++) {
    kn[i] = m.nen3v[3 * ie + i];
    b[i] = e[3 + i]; c[i] = e[6 + i];
    z[i] = m.zeov[3 * ie + i];
    zndg[i] = m.andgzv.empty() ? 0. : m.andgzv[kn[i]];   // andgzv (nudge.f90:333)
  }
  int ilevel = m.ilhv[ie];
  double aj = e[9];
  double delta = ddt * ddt * az * am * m.p.grav;     // afix = 1
  double dbb = 0., dbc = 0., dcb = 0., dcc = 0.;
  for (int l = 1; l <= ilevel; l++) {
    int jv = l + l, ju = jv - 1;
    dbb += m.ddxv[(size_t)ie * 2 * nlv + ju - 1];
    dbc += m.ddyv[(size_t)ie * 2 * nlv + ju - 1];
    dcb += m.ddxv[(size_t)ie * 2 * nlv + jv - 1];
    dcc += m.ddyv[(size_t)ie * 2 * nlv + jv - 1];
  }
  double uold = 0., vold = 0., uhat = 0., vhat = 0.;
  for (int l = 1; l <= ilevel; l++) {
    uold += m.utlov[(size_t)ie * nlv + l - 1];
    vold += m.vtlov[(size_t)ie * nlv + l - 1];
    uhat += m.utlnv[(size_t)ie * nlv + l - 1];
    vhat += m.vtlnv[(size_t)ie * nlv + l - 1];
  }
  double ut = az * uhat + (1. - az) * uold;
  double vt = az * vhat + (1. - az) * vold;
  for (int n = 0; n < 3; n++) {
    for (int mm = 0; mm < 3; mm++) {
      double abn = b[n] * (b[mm] * dbb + c[mm] * dbc);
      double acn = c[n] * (b[mm] * dcb + c[mm] * dcc);
      double h11 = delta * (abn + acn);
      hia[n][mm] = aj * ((n == mm ? 4. : 0.) + 12. * h11);
    }
    double acu = hia[n][0] * z[0] + hia[n][1] * z[1] + hia[n][2] * z[2];
    double andg = 4. * aj * ddt * zndg[n];
    hik[n] = acu + andg + 12. * aj * ddt * (ut * b[n] + vt * c[n]);
  }
  for (int i = 0; i < 3; i++) {
    if (m.rzv[kn[i]] != kFlag) {
      double rw = m.rzv[kn[i]];
      int j1 = (i + 1) % 3, j2 = (i + 2) % 3;
      hik[j1] -= rw * hia[j1][i];
      hik[j2] -= rw * hia[j2][i];
      hia[i][j1] = 0.; hia[i][j2] = 0.; hia[j1][i] = 0.; hia[j2][i] = 0.;
      hik[i] = rw * hia[i][i];
    }
  }
  if (m.p.wetdry && m.iwegv[ie] != 0) {       // excluded (dry) element (:710-727)
    const double hh999 = aj * 12.;
    for (int n = 0; n < 3; n++) {
      for (int mm = 0; mm < 3; mm++) hia[n][mm] = hh999 * (b[n] * b[mm] + c[n] * c[mm]);
      hik[n] = 0.;
    }
    for (int n = 0; n < 3; n++) {
      const int in = m.inodv[kn[n]];
      if (in != 0 && in != -2) {              // iskbnd: boundary of the wet domain
        for (int mm = 0; mm < 3; mm++) hia[n][mm] = 0.;
        hik[n] = 0.;
      }
    }
  }
}

void hydro_zeta_assemble(Model &m) {
  m.c2coo.assign(m.ntg[m.nkn], 0.);
  m.rvec2d.assign(m.nkn, 0.);
  for (int ie = 0; ie < m.nel; ie++) {
    int kn[3];
    double hia[3][3], hik[3];
    element_system(m, ie, kn, hia, hik);
    for (int i = 0; i < 3; i++) {
      for (int j = 0; j < 3; j++) m.c2coo[m.ijp[(size_t)9 * ie + 3 * i + j]] += hia[i][j];
      m.rvec2d[kn[i]] += hik[i];
    }
  }
  for (int k = 0; k < m.nkn; k++)             // adjust_mass_flux: none out of the system
    if (!(m.p.wetdry && m.inodv[k] == -2)) m.rvec2d[k] += m.p.dt * m.rqv[k];
}

int zeta_solve(Model &m) {    // system_solve -> spk_solve_system (sparskit_admin.f90:115-334)
  Ilu M;
  int st = ilut(m.nkn, m.ntg.data(), m.icol.data(), m.c2coo.data(), 5, 0.01, M);
  if (st) return st;
  std::vector<double> x(m.znv.begin(), m.znv.end());   // guess = z (real)
  int it = 0;
  double r0 = 0., r = 0.;
  st = bcgstab(m.nkn, m.ntg.data(), m.icol.data(), m.c2coo.data(), M, m.rvec2d.data(), x.data(),
               m.rtol, m.atol, m.maxmv, &it, &r0, &r);
  m.info.krylov_iters = it;
  m.info.resid0 = r0;
  m.info.resid = r;
  if (st) return st;
  for (int k = 0; k < m.nkn; k++) m.znv[k] = x[k];     // system_get
  return SHY_OK;
}

// hydro_transports_final (hydrodynamic.f90:1468-1578)
void hydro_transports_final(Model &m) {
  int nlv = m.nlv;
  double beta = m.p.dt * m.p.grav * m.p.ampar;
  m.unv.assign(m.nel, 0.); m.vnv.assign(m.nel, 0.);
  for (int ie = 0; ie < m.nel; ie++) {
    const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
    int ilevel = m.ilhv[ie];
    double bz = 0., cz = 0.;
    for (int ii = 0; ii < 3; ii++) {
      int kk = m.nen3v[3 * ie + ii];
      double dz = m.znv[kk] - m.zeov[3 * ie + ii];
      bz += dz * e[3 + ii];
      cz += dz * e[6 + ii];
    }
    for (int l = 1; l <= ilevel; l++) {
      int jv = l + l, ju = jv - 1;
      double du = beta * (m.ddxv[(size_t)ie * 2 * nlv + ju - 1] * bz + m.ddyv[(size_t)ie * 2 * nlv + ju - 1] * cz);
      double dv = beta * (m.ddxv[(size_t)ie * 2 * nlv + jv - 1] * bz + m.ddyv[(size_t)ie * 2 * nlv + jv - 1] * cz);
      m.utlnv[(size_t)ie * nlv + l - 1] -= du;
      m.vtlnv[(size_t)ie * nlv + l - 1] -= dv;
    }
    double um = 0., vm = 0.;
    for (int l = 1; l <= ilevel; l++) {
      um += m.utlnv[(size_t)ie * nlv + l - 1];
      vm += m.vtlnv[(size_t)ie * nlv + l - 1];
    }
    m.unv[ie] = um; m.vnv[ie] = vm;
  }
}

// set_mass_flux (bnd_routines.f90:1035-1140) for nodes with a discharge
// rqv [m^3/s]: mfluxv(l,k) = rqv(k) times the layer's share of the node's
// volume at the start of the step (volnode(l,k,+1) when set_mass_flux runs,
// before hydro: the old thickness), over all the node's layers (the levmin
// and levmax of a boundary default to them); rqv itself stays the vertical
// sum.  Distributed sources (rain, rqdsv) are not part of this path.
void set_mass_flux(Model &m) {
  const int nlv = m.nlv;
  m.mfluxv.assign((size_t)nlv * m.nkn, 0.);
  for (int k = 0; k < m.nkn; k++) {
    if (m.rqv[k] == 0.) continue;
    const int lmax = m.ilhkv[k];
    double vtot = 0.;
    for (int l = 1; l <= lmax; l++) vtot += m.hdkov[(size_t)k * nlv + l - 1] * m.areakv[(size_t)k * nlv + l - 1];
    if (!(vtot > 0.)) continue;
    for (int l = 1; l <= lmax; l++)
      m.mfluxv[(size_t)k * nlv + l - 1] =
          m.rqv[k] * (m.hdkov[(size_t)k * nlv + l - 1] * m.areakv[(size_t)k * nlv + l - 1] / vtot);
  }
}

// adjust_mass_flux (bnd_routines.f90:1185-1210): no discharge at nodes out
// of the wet system
void adjust_mass_flux(Model &m) {
  for (int k = 0; k < m.nkn; k++)
    if (m.inodv[k] == -2)
      for (int l = 0; l < m.nlv; l++) m.mfluxv[(size_t)k * m.nlv + l] = 0.;
}

// hydro_vertical (hydrodynamic.f90:1582-1781), with the discharge mfluxv of
// each node layer (:1727)
void hydro_vertical(Model &m) {
  int nlv = m.nlv;
  m.wlnv.assign((size_t)(nlv + 1) * m.nkn, 0.);
  if (nlv == 1) return;
  double az = m.p.azpar, azt = 1. - az, dt = m.p.dt;
  std::vector<double> vf((size_t)nlv * m.nkn, 0.), va((size_t)nlv * m.nkn, 0.);
  for (int ie = 0; ie < m.nel; ie++) {
    const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
    double aj = 4. * e[9];
    for (int l = 1; l <= m.ilhv[ie]; l++)
      for (int ii = 0; ii < 3; ii++) {
        int kk = m.nen3v[3 * ie + ii];
        double b = e[3 + ii], c = e[6 + ii];
        double ffn = m.utlnv[(size_t)ie * nlv + l - 1] * b + m.vtlnv[(size_t)ie * nlv + l - 1] * c;
        double ffo = m.utlov[(size_t)ie * nlv + l - 1] * b + m.vtlov[(size_t)ie * nlv + l - 1] * c;
        double ff = ffn * az + ffo * azt;
        vf[(size_t)kk * nlv + l - 1] += 3. * aj * ff;
        va[(size_t)kk * nlv + l - 1] += aj;
      }
  }
  auto W = [&](int l, int k) -> double & { return m.wlnv[(size_t)k * (nlv + 1) + l]; };
  for (int k = 0; k < m.nkn; k++) {
    int lmax = m.ilhkv[k], lmin = 1;
    W(lmax, k) = 0.;
    for (int l = lmax; l >= lmin; l--) {
      double voln = m.hdknv[(size_t)k * nlv + l - 1] * m.areakv[(size_t)k * nlv + l - 1];
      double volo = m.hdkov[(size_t)k * nlv + l - 1] * m.areakv[(size_t)k * nlv + l - 1];
      double dvdt = (voln - volo) / dt;
      double q = m.mfluxv[(size_t)k * nlv + l - 1];
      double wdiv = vf[(size_t)k * nlv + l - 1] + q;
      W(l - 1, k) = W(l, k) + wdiv - dvdt;
    }
    W(lmin - 1, k) = 0.;
  }
  for (int k = 0; k < m.nkn; k++) {
    int lmax = m.ilhkv[k];
    for (int l = 2; l <= lmax; l++) {
      double atop = va[(size_t)k * nlv + l - 1];
      if (atop > 0.) W(l - 1, k) /= atop;
    }
  }
  for (int k = 0; k < m.nkn; k++)
    if (m.bnd[k] > 0)
      for (int l = 0; l <= nlv; l++) W(l, k) = 0.;
}

// ---------------------------------------------------------------------------
// Non-hydrostatic pressure: nohydro.f90 and the 3D system of coo_matrix.f90 /
// simsys_spkaux.f90.  The 3D unknowns are (nlv+2) per node, layer 0 and
// layer nlv+1 being padding rows: unknown u(k,l) = k*(nlv+2) + l.
// ---------------------------------------------------------------------------

// coo_init_new's 3D part (coo_matrix.f90:180-247): row block k holds the
// layer-0 diagonal, then per layer l the node's sorted neighbours at l with
// (k,l-1), (k,l), (k,l+1) in the diagonal's place, then the layer-(nlv+1)
// diagonal: ng*nlv + 2*nlv + 2 entries, row-sorted, so the COO is a CSR
void coo3d_init(int nkn, int nlv, const std::vector<int> &ntg, std::vector<int> &nt3g) {
  nt3g.assign(nkn + 1, 0);
  for (int k = 0; k < nkn; k++) {
    const int ng = ntg[k + 1] - ntg[k];
    nt3g[k + 1] = nt3g[k] + (ng - 1) * nlv + 2 + 3 * nlv;
  }
}

// loccoo3d (coo_matrix.f90:665-695), 0-based: the position of element entry
// (i, j) of layer l (1..nlv) in the 3D COO; for i == j the (k,l-1) and
// (k,l+1) couplings sit just before and after it
int loc3d(const Model &m, int ie, int i, int j, int l) {
  const int ki = m.nen3v[3 * ie + i];
  const int ng = m.ntg[ki + 1] - m.ntg[ki];
  const int mi = m.ijp[(size_t)9 * ie + 3 * i + i] - m.ntg[ki];   // diagonal's index in the row
  const int mj = m.ijp[(size_t)9 * ie + 3 * i + j] - m.ntg[ki];
  const int p3 = mj < mi ? mj : (mj == mi ? mi + 1 : mj + 2);
  return m.nt3g[ki] + 1 + (l - 1) * (ng + 2) + p3;
}

// the CSR row pointer and columns of the 3D COO (coocsr of its row-sorted
// entries), unknowns u(k,l) = k*(nlv+2) + l
void coo3d_csr(const Model &m, std::vector<int> &ia, std::vector<int> &ja) {
  const int nlv = m.nlv, n = (nlv + 2) * m.nkn;
  ia.assign(n + 1, 0);
  ja.assign(m.nt3g[m.nkn], 0);
  int r = 0, p = 0;
  for (int k = 0; k < m.nkn; k++) {
    const int ng = m.ntg[k + 1] - m.ntg[k];
    ia[r] = p; ja[p++] = k * (nlv + 2); r++;                     // layer 0
    for (int l = 1; l <= nlv; l++) {
      ia[r] = p;
      for (int q = 0; q < ng; q++) {
        const int kj = m.icol[m.ntg[k] + q];
        if (kj == k) { ja[p++] = k * (nlv + 2) + l - 1; ja[p++] = k * (nlv + 2) + l; ja[p++] = k * (nlv + 2) + l + 1; }
        else ja[p++] = kj * (nlv + 2) + l;
      }
      r++;
    }
    ia[r] = p; ja[p++] = k * (nlv + 2) + nlv + 1; r++;            // layer nlv+1
  }
  ia[r] = p;
}

// system_assemble_3d (simsys_spkaux.f90:597-635): mass(-1:1,3,3) as
// mass[(d+1)*9 + 3*i + j], the three couplings added at kk-1, kk, kk+1
void assemble_3d(Model &m, int ie, int l, const double *mass, const double *rhs) {
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) {
      const int kk = loc3d(m, ie, i, j, l);
      m.c3coo[kk - 1] += mass[0 * 9 + 3 * i + j];
      m.c3coo[kk] += mass[1 * 9 + 3 * i + j];
      m.c3coo[kk + 1] += mass[2 * 9 + 3 * i + j];
    }
    m.rvec3d[(size_t)(m.nlv + 2) * m.nen3v[3 * ie + i] + l] += rhs[i];
  }
}

// coo_adjust_3d (coo_matrix.f90:269-325): unit diagonal where no element
// layer reached it, and on the padding rows
void adjust_3d(Model &m) {
  for (int ie = 0; ie < m.nel; ie++)
    for (int i = 0; i < 3; i++)
      for (int l = 1; l <= m.nlv; l++) {
        const int kk = loc3d(m, ie, i, i, l);
        if (m.c3coo[kk] == 0.) m.c3coo[kk] = 1.;
      }
  for (int k = 0; k < m.nkn; k++) {
    m.c3coo[m.nt3g[k]] = 1.;
    m.c3coo[m.nt3g[k + 1] - 1] = 1.;
  }
}

// system_solve_3d + spk_solve_system (3D: the same ILUT(5, 0.01) and
// BiCGStab as the zeta system, sparskit_admin.f90:115-334) + system_get_3d:
// the guess is z(l,k) with zero padding rows; the solution goes back to z
int solve_3d(Model &m, std::vector<double> &z /* (nkn, nlv) rows */) {
  const int nlv = m.nlv, n = (nlv + 2) * m.nkn;
  std::vector<int> ia, ja;
  coo3d_csr(m, ia, ja);
  Ilu M;
  int st = ilut(n, ia.data(), ja.data(), m.c3coo.data(), 5, 0.01, M);
  if (st) return st;
  std::vector<double> x(n, 0.);
  for (int k = 0; k < m.nkn; k++)
    for (int l = 1; l <= nlv; l++) x[(size_t)k * (nlv + 2) + l] = z[(size_t)k * nlv + l - 1];
  st = bcgstab(n, ia.data(), ja.data(), m.c3coo.data(), M, m.rvec3d.data(), x.data(), m.rtol, m.atol, m.maxmv,
               &m.nh_iters, &m.nh_resid0, &m.nh_resid);
  if (st) return st;
  for (int k = 0; k < m.nkn; k++)
    for (int l = 1; l <= nlv; l++) z[(size_t)k * nlv + l - 1] = x[(size_t)k * (nlv + 2) + l];
  return SHY_OK;
}

// tridag (keps_util.f90:82-111): a sub-, b main, c super-diagonal
int tridag(const double *a, const double *b, const double *c, const double *r, double *u, int n) {
  std::vector<double> gam(n + 1);
  if (b[0] == 0.) return fail(SHY_ESINGULAR, "tridag: matrix singular");
  double bet = b[0];
  u[0] = r[0] / bet;
  for (int j = 1; j < n; j++) {
    gam[j] = c[j - 1] / bet;
    bet = b[j] - a[j] * gam[j];
    if (bet == 0.) return fail(SHY_ESINGULAR, "tridag: matrix singular");
    u[j] = (r[j] - a[j] * u[j - 1]) / bet;
  }
  for (int j = n - 2; j >= 0; j--) u[j] -= gam[j + 1] * u[j + 1];
  return SHY_OK;
}

// sp256wnh (nohydro.f90:205-524): the vertical velocity from the vertical
// momentum equation with the old non-hydrostatic pressure, horizontal
// diffusion, horizontal advection (averaged, or upwind fluxes with
// inhflx = 1), vertical advection (ivwadv 1 upwind, 2 centred) and implicit
// vertical viscosity: one tridiagonal system per node over the interfaces
// 1..lmax-1.  An element whose last layer is l makes interface l of its
// nodes an identity row, over whatever came before it in element order.
int sp256wnh(Model &m) {
  const int nlv = m.nlv, I = nlv + 1;
  const double dt = m.p.dt, aq = m.p.aqpar, aqt = 1. - aq, az = m.p.azpar, azt = 1. - az;
  std::vector<double> wrhs((size_t)I * m.nkn, 0.), wdiag((size_t)I * m.nkn, 0.),
      wdiagt((size_t)I * m.nkn, 0.), wdiagb((size_t)I * m.nkn, 0.);
  auto WO = [&](int l, int k) { return m.wlov[(size_t)k * I + l]; };
  for (int ie = 0; ie < m.nel; ie++) {
    const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
    const int ilevel = m.ilhv[ie];
    int kn[3];
    double b[3], c[3];
    for (int ii = 0; ii < 3; ii++) { kn[ii] = m.nen3v[3 * ie + ii]; b[ii] = e[3 + ii]; c[ii] = e[6 + ii]; }
    const double aj4 = 4. * e[9];
    for (int l = 1; l <= ilevel; l++) {
      const bool blast = l == ilevel;
      const size_t o = (size_t)ie * nlv + l - 1;
      const double hdn = m.hdenv[o], hdo = m.hdeov[o];
      const double utn = m.utlnv[o], uto = m.utlov[o], vtn = m.vtlnv[o], vto = m.vtlov[o];
      double hdpn = 0., hdpo = 0., ubn = 0., ubo = 0., vbn = 0., vbo = 0., anu;
      if (blast) anu = 0.5 * m.p.ahpar * m.difhv[o];
      else {
        hdpn = m.hdenv[o + 1]; hdpo = m.hdeov[o + 1];
        ubn = m.utlnv[o + 1]; ubo = m.utlov[o + 1]; vbn = m.vtlnv[o + 1]; vbo = m.vtlov[o + 1];
        anu = 0.5 * m.p.ahpar * (m.difhv[o] + m.difhv[o + 1]);
      }
      const double dzn = 0.5 * (hdn + hdpn), dzo = 0.5 * (hdo + hdpo);
      const double us = 0.5 * (az * (utn + ubn) / dzn + azt * (uto + ubo) / dzo);
      const double vs = 0.5 * (az * (vtn + vbn) / dzn + azt * (vto + vbo) / dzo);
      double wl[3], f[3], fl[3] = {0., 0., 0.}, wb = 0., wc = 0., wsum = 0.;
      int itot = 0, isum = 0;
      for (int ii = 0; ii < 3; ii++) {
        wl[ii] = WO(l, kn[ii]);
        f[ii] = us * b[ii] + vs * c[ii];
        if (f[ii] < 0.) { itot++; isum += ii + 1; }
        wb += b[ii] * wl[ii]; wc += c[ii] * wl[ii]; wsum += wl[ii];
      }
      if (m.p.inhflx == 1) {
        if (itot == 1) {
          for (int ii = 0; ii < 3; ii++) fl[ii] = f[ii] * wl[isum - 1];
        } else if (itot == 2) {
          const int iz = 6 - isum - 1;
          for (int ii = 0; ii < 3; ii++) fl[ii] = f[ii] * wl[ii];
          fl[iz] = 0.;
          fl[iz] = -(fl[0] + fl[1] + fl[2]);
        }
      }
      for (int ii = 0; ii < 3; ii++) {
        const int k = kn[ii];
        const size_t r = (size_t)k * I + l;
        const double wq = blast ? 0. : -aqt * m.qdistv[k] *
                                           (m.qpov[(size_t)k * nlv + l - 1] - m.qpov[(size_t)k * nlv + l]) / dzo;
        double wadvv = 0.;
        if (m.p.ivwadv == 1 && !blast) {
          const double wplus = 0.5 * (WO(l, k) + WO(l - 1, k)) / dzo;
          wadvv = wplus > 0. ? wplus * WO(l, k) : wplus * WO(l - 1, k);
          const double wminus = 0.5 * (WO(l, k) + WO(l + 1, k)) / dzo;
          wadvv -= wminus > 0. ? wminus * WO(l + 1, k) : wminus * WO(l, k);
        } else if (m.p.ivwadv >= 2 && !blast) {
          wadvv = 0.5 * WO(l, k) * (WO(l - 1, k) - WO(l + 1, k)) / dzo;
        }
        const double wdifh = -3. * anu * (wb * b[ii] + wc * c[ii]);
        const double wadvh = m.p.inhflx == 1 ? -3. * fl[ii] : -(b[ii] * us + c[ii] * vs) * wsum;
        const double wr = dzn * (WO(l, k) + dt * (wq + wdifh - wadvh - wadvv));
        wrhs[r] += aj4 * wr;
        if (blast) {
          wdiag[r] = 1.; wdiagt[r] = 0.; wdiagb[r] = 0.; wrhs[r] = 0.;
        } else {
          const double rnu = m.visv[r];
          wdiag[r] += dzn * aj4 + dt * aj4 * rnu * (1. / hdn + 1. / hdpn);
          wdiagt[r] -= dt * aj4 * rnu / hdn;
          wdiagb[r] -= dt * aj4 * rnu / hdpn;
        }
      }
    }
  }
  m.wnh.assign((size_t)I * m.nkn, 0.);
  std::vector<double> sol(nlv + 1);
  for (int k = 0; k < m.nkn; k++) {
    const int lmax = m.ilhkv[k];
    if (lmax > 2) {
      const size_t r = (size_t)k * I + 1;
      int st = tridag(&wdiagt[r], &wdiag[r], &wdiagb[r], &wrhs[r], sol.data(), lmax - 1);
      if (st) return st;
      for (int l = 1; l <= lmax - 1; l++) m.wnh[(size_t)k * I + l] = sol[l - 1];
    }
  }
  return SHY_OK;
}

// nonhydro_prepare_matrix (nohydro.f90:589-753): per element layer the
// Poisson element matrix of the non-hydrostatic pressure (horizontal
// Laplacian times the layer thickness, vertical second differences across
// the layer interfaces, the free-surface term on the first layer) and the
// divergence of the predicted flow, assembled with system_assemble_3d
void nh_prepare_matrix(Model &m) {
  const int nlv = m.nlv, I = nlv + 1;
  const double dt = m.p.dt, aq = m.p.aqpar, az = m.p.azpar, azt = 1. - az;
  m.c3coo.assign(m.nt3g[m.nkn], 0.);                      // system_init
  m.rvec3d.assign((size_t)(nlv + 2) * m.nkn, 0.);
  std::vector<double> hld(nlv + 2, 0.);
  double mass[27], rhs[3];
  for (int ie = 0; ie < m.nel; ie++) {
    const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
    for (int l = 1; l <= nlv; l++) hld[l] = m.hdenv[(size_t)ie * nlv + l - 1];
    const double aj = e[9], aj4 = 4. * aj, aj12 = 12. * aj;
    int kn[3];
    double b[3], c[3];
    for (int ii = 0; ii < 3; ii++) { kn[ii] = m.nen3v[3 * ie + ii]; b[ii] = e[3 + ii]; c[ii] = e[6 + ii]; }
    const int lmax = m.ilhv[ie];
    for (int l = 1; l <= lmax; l++) {
      for (double &v : mass) v = 0.;
      const double hd = hld[l], hdm = hld[l - 1], hdp = hld[l + 1];
      double rhm = 2. / (hd + hdm), rhp = 2. / (hd + hdp);
      if (l == 1) rhm = 0.;
      if (l == lmax) rhp = 0.;
      const double rhc = rhm + rhp;
      for (int n = 0; n < 3; n++) {
        for (int q = 0; q < 3; q++) {
          mass[9 + 3 * n + q] = -aj12 * hd * dt * aq * az * (b[n] * b[q] + c[n] * c[q]);
          if (n == q) {
            mass[9 + 3 * n + q] -= aj4 * dt * aq * rhc;
            mass[0 + 3 * n + q] = aj4 * dt * aq * rhm;
            mass[18 + 3 * n + q] = aj4 * dt * aq * rhp;
          }
        }
        const int k = kn[n];
        const size_t o = (size_t)ie * nlv + l - 1;
        const double fhn = m.utlnv[o] * b[n] + m.vtlnv[o] * c[n];
        const double fho = m.utlov[o] * b[n] + m.vtlov[o] * c[n];
        const double fvn = m.wnh[(size_t)k * I + l - 1] - m.wnh[(size_t)k * I + l];
        const double ffh = -(az * fhn + azt * fho);
        rhs[n] = aj4 * (3. * ffh + fvn);
      }
      if (l == 1)
        for (int i = 0; i < 3; i++) {
          const int k = kn[i];
          mass[9 + 4 * i] -= aj4 / (m.p.grav * dt);
          rhs[i] += aj4 * (m.znv[k] - m.zov[k]) / dt;
        }
      assemble_3d(m, ie, l, mass, rhs);
    }
  }
  adjust_3d(m);
}

// nonhydro_correct_uveta (nohydro.f90:761-829): the water level moves by the
// surface pressure over g, the transports by the pressure gradient times
// aqpar dt and the layer thickness
void nh_correct_uveta(Model &m) {
  const int nlv = m.nlv;
  const double aq = m.p.aqpar, dt = m.p.dt;
  for (int k = 0; k < m.nkn; k++) m.znv[k] += m.qdistv[k] * m.qpnv[(size_t)k * nlv] / m.p.grav;
  for (int ie = 0; ie < m.nel; ie++) {
    const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
    for (int l = 1; l <= m.ilhv[ie]; l++) {
      double uq = 0., vq = 0.;
      for (int ii = 0; ii < 3; ii++) {
        const int k = m.nen3v[3 * ie + ii];
        const double q = m.qdistv[k] * m.qpnv[(size_t)k * nlv + l - 1];
        uq += e[3 + ii] * q;
        vq += e[6 + ii] * q;
      }
      const size_t o = (size_t)ie * nlv + l - 1;
      m.utlnv[o] -= aq * dt * uq * m.hdenv[o];
      m.vtlnv[o] -= aq * dt * vq * m.hdenv[o];
    }
  }
}

// sp256wnh and nonhydro_adjust (nohydro.f90:109-183) with inhadj = 0: the
// pressure from the 3D system (guess: zero, the cleared qpnv), the
// correction of level and transports, setzev, make_new_depth, and the
// pressure's first layer set to zero (the loop qpnv(l,k) - qpnv(1,k) zeroes
// qpnv(1,k) first and then subtracts that zero from the layers below)
int nonhydro_adjust(Model &m) {
  int st = sp256wnh(m);
  if (st) return st;
  nh_prepare_matrix(m);
  st = solve_3d(m, m.qpnv);
  if (st) return st;
  nh_correct_uveta(m);
  for (int ie = 0; ie < m.nel; ie++)
    for (int ii = 0; ii < 3; ii++) m.zenv[3 * ie + ii] = m.znv[m.nen3v[3 * ie + ii]];
  st = setdepth(m, m.hdknv, m.hdenv, m.zenv);
  if (st) return st;
  for (int k = 0; k < m.nkn; k++) m.qpnv[(size_t)k * m.nlv] = 0.;
  return SHY_OK;
}

// masscont (elems_dealing.f90:1191-1223) -> total volume in FP64
double masscont(Model &m) {
  double total = 0.;
  for (int k = 0; k < m.nkn; k++)
    for (int l = 1; l <= m.ilhkv[k]; l++)
      total += m.hdknv[(size_t)k * m.nlv + l - 1] * m.areakv[(size_t)k * m.nlv + l - 1];
  return total;
}

// conzstab (concentration.f90:1573-2080): the transport stability index with
// ddt = 1, with the inflow of point sources (mfluxv > 0, :1801) and settling
// and nudging from tm (or none).
double conzstab(Model &m, double rkpar, const Model::ScalarTerms *tm = nullptr) {
  int nlv = m.nlv;
  double az = m.p.azpar, azt = 1. - az, ad = m.p.adpar, adt = 1. - ad, aa = m.p.aapar, aat = 1. - aa;
  const double dt = 1.;      // ddt = 1, istot = isact = 1 -> rso = 0, rsn = 1
  std::vector<double> cn((size_t)nlv * m.nkn, 0.), cdiag(cn.size(), 0.), clow(cn.size(), 0.),
      chigh(cn.size(), 0.), co(cn.size(), 0.);
  for (size_t q = 0; q < co.size(); q++)
    if (m.mfluxv[q] > 0.) co[q] = m.mfluxv[q];   // point sources
  for (int ie = 0; ie < m.nel; ie++) {
    const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
    int kn[3];
    double b[3], c[3];
    for (int ii = 0; ii < 3; ii++) { kn[ii] = m.nen3v[3 * ie + ii]; b[ii] = e[3 + ii]; c[ii] = e[6 + ii]; }
    double aj = e[9], aj4 = 4. * aj;
    int ilevel = m.ilhv[ie];
    std::vector<double> hdv(nlv + 2, 0.), present(nlv + 2, 0.);
    std::vector<double> hnew(3 * (size_t)(nlv + 2), 0.), hold(3 * (size_t)(nlv + 2), 0.), wl(3 * (size_t)(nlv + 2), 0.);
    auto H = [&](std::vector<double> &a, int l, int ii) -> double & { return a[(size_t)ii * (nlv + 2) + l]; };
    for (int l = 1; l <= ilevel; l++) {
      hdv[l] = m.hdeov[(size_t)ie * nlv + l - 1];
      present[l] = 1.;
      for (int ii = 0; ii < 3; ii++) {
        int k = kn[ii];
        double hn = m.hdknv[(size_t)k * nlv + l - 1], ho = m.hdkov[(size_t)k * nlv + l - 1];
        H(hold, l, ii) = ho;                 // rso = 0
        H(hnew, l, ii) = hn;                 // rsn = 1
        H(wl, l, ii) = m.wlnv[(size_t)k * (nlv + 1) + l];
        if (tm && tm->wsink != 0.)           // settling (concentration.f90:1860)
          H(wl, l, ii) -= tm->wsink * tm->wsinkv[(size_t)k * (nlv + 1) + l];
      }
    }
    for (int ii = 0; ii < 3; ii++) H(wl, ilevel, ii) = 0.;
    for (int l = 1; l <= ilevel; l++) {
      double us = az * m.utlnv[(size_t)ie * nlv + l - 1] + azt * m.utlov[(size_t)ie * nlv + l - 1];
      double vs = az * m.vtlnv[(size_t)ie * nlv + l - 1] + azt * m.vtlov[(size_t)ie * nlv + l - 1];
      double rk3 = 3. * rkpar * m.difhv[(size_t)ie * nlv + l - 1];
      double f[3], fwin[3], fwout[3], fd[3], wdiff[3];
      for (int ii = 0; ii < 3; ii++) {
        int k = kn[ii];
        wdiff[ii] = m.wdifhv[(size_t)9 * ie + 3 * ii + ii];
        f[ii] = us * b[ii] + vs * c[ii];
        fwin[ii] = 0.; fwout[ii] = 0.;
        double w = H(wl, l - 1, ii);
        if (w > 0.) fwout[ii] += aat * w; else fwin[ii] -= aat * w;
        w = H(wl, l, ii);
        if (w > 0.) fwin[ii] += aat * w; else fwout[ii] -= aat * w;
        double rvptop = m.difv[(size_t)k * (nlv + 1) + l - 1] + m.p.difmol;
        double rvpbot = m.difv[(size_t)k * (nlv + 1) + l] + m.p.difmol;
        double hmtop = 2. * rvptop * present[l - 1] / (hdv[l - 1] + hdv[l]);
        double hmbot = 2. * rvpbot * present[l + 1] / (hdv[l] + hdv[l + 1]);
        fd[ii] = adt * (hmtop + hmbot);
      }
      double coadv = 0., ciadv = 0.;
      for (int ii = 0; ii < 3; ii++) {
        int k = kn[ii];
        double hmed = H(hold, l, ii);
        double chdiff = dt * aj4 * rk3 * hmed * wdiff[ii];
        double cvdiff = dt * aj4 * fd[ii];
        double chadv = dt * aj4 * 3. * f[ii];
        double cviadv = dt * aj4 * fwin[ii];
        double cvoadv = dt * aj4 * fwout[ii];
        if (chadv < 0.) coadv = cvoadv - chadv;
        else ciadv = cviadv + chadv;
        double cadv = std::max(coadv, ciadv);
        chigh[(size_t)k * nlv + l - 1] += cadv;
        clow[(size_t)k * nlv + l - 1] += chdiff;
        cn[(size_t)k * nlv + l - 1] += cvdiff;
        if (tm && tm->robs != 0.)            // nudging (concentration.f90:1985)
          co[(size_t)k * nlv + l - 1] += dt * aj4 * hmed * tm->robs * tm->rtauv[(size_t)k * nlv + l - 1];
      }
    }
    for (int l = 1; l <= ilevel; l++)
      for (int ii = 0; ii < 3; ii++) {
        int k = kn[ii];
        double hmed = std::min(H(hold, l, ii), H(hnew, l, ii));
        cdiag[(size_t)k * nlv + l - 1] += aj4 * hmed;
      }
  }
  double stabind = 0.;
  for (int k = 0; k < m.nkn; k++) {
    if (m.bnd[k] > 0) continue;           // is_zeta_bound
    for (int l = 1; l <= m.ilhkv[k]; l++) {
      size_t q = (size_t)k * nlv + l - 1;
      double voltot = cdiag[q];
      double flxtot = chigh[q] + clow[q] + cn[q] + co[q];
      if (voltot > 0.) stabind = std::max(stabind, flxtot / voltot);
    }
  }
  return stabind / m.p.rstol;
}

// tvd_grad_3d (tvd_admin.f90:478-550): node gradients of a scalar, the
// area-weighted mean of the element gradients over the elements that have
// the layer (itvd = 1)
void tvd_grad_3d(const Model &m, const std::vector<double> &cc, std::vector<double> &gx,
                 std::vector<double> &gy) {
  const int nlv = m.nlv;
  const size_t nn = (size_t)nlv * m.nkn;
  gx.assign(nn, 0.); gy.assign(nn, 0.);
  std::vector<double> aux(nn, 0.);
  for (int ie = 0; ie < m.nel; ie++) {
    const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
    const double area = e[9];
    for (int l = 0; l < m.ilhv[ie]; l++) {
      double ggx = 0., ggy = 0.;
      for (int ii = 0; ii < 3; ii++) {
        const size_t kl = (size_t)m.nen3v[3 * ie + ii] * nlv + l;
        ggx += cc[kl] * e[3 + ii];
        ggy += cc[kl] * e[6 + ii];
        aux[kl] += area;
      }
      for (int ii = 0; ii < 3; ii++) {
        const size_t kl = (size_t)m.nen3v[3 * ie + ii] * nlv + l;
        gx[kl] += ggx * area;
        gy[kl] += ggy * area;
      }
    }
  }
  for (size_t q = 0; q < nn; q++)
    if (aux[q] > 0.) { gx[q] /= aux[q]; gy[q] /= aux[q]; }
}

// the slot of the ordered vertex pair (c, d), c != d, among an element's six
inline int tvd_slot(int c, int d) { return 2 * c + ((d - c + 3) % 3 - 1); }

// tvd_upwind_init_elem (tvd_admin.f90:361-476): for every element and
// ordered pair (c, d) of its vertices, the point beyond c opposite d,
// 2 x_c - x_d (kept in single precision as the reference's real x, y), the
// element that holds it (the lowest-numbered one where several touch it;
// none outside the basin) and the point's natural coordinates there
// (xy2xi/adjust_xi, evgeom.f90:531-660: clipped to [0,1], summing to 1).
// A brute-force search: the oracle runs on small meshes.
void tvd_upwind_init(Model &m, const std::vector<double> &x, const std::vector<double> &y) {
  m.tvdup_e.assign((size_t)6 * m.nel, -1);
  m.tvdup_xi.assign((size_t)18 * m.nel, 0.);
  for (int ie = 0; ie < m.nel; ie++)
    for (int c = 0; c < 3; c++)
      for (int d = 0; d < 3; d++) {
        if (d == c) continue;
        const int kc = m.nen3v[3 * ie + c], kd = m.nen3v[3 * ie + d];
        const double xu = (double)(float)(2. * x[kc] - x[kd]), yu = (double)(float)(2. * y[kc] - y[kd]);
        const int sl = 6 * ie + tvd_slot(c, d);
        for (int je = 0; je < m.nel; je++) {
          const int *k = &m.nen3v[3 * je];
          const double x1 = x[k[0]], y1 = y[k[0]], x2 = x[k[1]], y2 = y[k[1]], x3 = x[k[2]], y3 = y[k[2]];
          const double det = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
          double l[3];
          l[1] = ((xu - x1) * (y3 - y1) - (x3 - x1) * (yu - y1)) / det;
          l[2] = ((x2 - x1) * (yu - y1) - (xu - x1) * (y2 - y1)) / det;
          l[0] = 1. - l[1] - l[2];
          if (l[0] < -1e-9 || l[1] < -1e-9 || l[2] < -1e-9) continue;
          double sum = 0.;
          for (int i = 0; i < 3; i++) { l[i] = std::min(1., std::max(0., l[i])); sum += l[i]; }
          m.tvdup_e[sl] = je;
          for (int i = 0; i < 3; i++) m.tvdup_xi[(size_t)3 * sl + i] = l[i] / sum;
          break;
        }
      }
}

// tvd_fluxes (tvd_admin.f90:673-838), itvd 1 or 2: the horizontal fluxes
// fl(3) of element ie, layer l (1-based), from the concentrations cl of its
// vertices, the element velocity (ulnv = utlnv/hdenv of the new level) and
// either the node gradients gx, gy (itvd 1) or the value of cv at the point
// beyond the upwind vertex (itvd 2), limited by superbee.  itot/isum as conz3d_element's
// (number and index sum of the vertices with f < 0).
void tvd_fluxes(const Model &m, int ie, int l, int itot, int isum, double dt, const double cl[3],
                const std::vector<double> &gx, const std::vector<double> &gy, const double f[3],
                const std::vector<double> &cv, double fl[3]) {
  fl[0] = fl[1] = fl[2] = 0.;
  if (itot < 1 || itot > 2) return;
  const int nlv = m.nlv;
  const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
  const size_t el = (size_t)ie * nlv + l - 1;
  const double h = m.hdenv[el];
  const double u = h > 0. ? m.utlnv[el] / h : 0., v = h > 0. ? m.vtlnv[el] / h : 0.;
  const double aj = 24. * e[9];
  const int itot2 = itot - 1, itot1 = 2 - itot;
  const int ip = itot2 * (6 - isum) + itot1 * isum;
  for (int ii = 1; ii <= 3; ii++) {
    if (ii == ip) continue;
    const int ic = itot2 * ii + itot1 * ip, id = itot2 * ip + itot1 * ii;
    const double fact = -itot2 + itot1;
    const double conc = cl[ic - 1], cond = cl[id - 1];
    const int iop = 6 - (id + ic);                  // the vertex opposite side ic-id
    const int tet1 = 1 + iop % 3;
    double dx = aj * e[5 + iop];                    // ev(6+iop)
    if (tet1 == id) dx = -dx;
    double dy = aj * e[2 + iop];                    // ev(3+iop)
    if (tet1 == ic) dy = -dy;
    const double dis = e[15 + iop];                 // ev(16+iop): length of side ic-id
    const double vel = std::fabs(u * dx + v * dy) / dis;
    const double alfa = dt * vel / dis;
    double grad;
    if (m.p.itvd == 2) {
      // the value at the point beyond ic opposite id (tvd_get_upwind_c
      // :608-671), or cond where that point has no layer l
      double conu = cond;
      const int sl = 6 * ie + tvd_slot(ic - 1, id - 1);
      const int je = m.tvdup_e[sl];
      if (je >= 0 && m.ilhv[je] >= l) {
        conu = 0.;
        for (int i = 0; i < 3; i++)
          conu += m.tvdup_xi[(size_t)3 * sl + i] * cv[(size_t)m.nen3v[3 * je + i] * nlv + l - 1];
      }
      grad = cond - conu;
    } else {
      const size_t kc = (size_t)m.nen3v[3 * ie + ic - 1] * nlv + l - 1;
      grad = 2. * (gx[kc] * dx + gy[kc] * dy);
    }
    const double rf = std::fabs(conc - cond) < 1.e-8 ? -1. : grad / (cond - conc) - 1.;
    const double psi = std::max(0., std::max(std::min(1., 2. * rf), std::min(2., rf)));   // superbee
    const double conf = conc + 0.5 * psi * (cond - conc) * (1. - alfa);
    const double term = fact * conf * f[ii - 1];
    fl[ic - 1] -= term;
    fl[id - 1] += term;
  }
}

// conz3d_omp (concentration_omp.f90:65-350) with conz3d_element (:355-755),
// vertical_flux_ie (tvd_admin.f90:930-1019, itvdv 0 or 1) and
// conz3d_nodes (:757-888); itvd 0 or 1 (gx, gy: the node gradients of
// tvd_grad_3d).  cbound (nkn, nlv) is the concentration inflows bring at
// nodes with a discharge (mfluxv).  tm (or null) carries the nudging,
// settling and loading terms; its load is updated where deposition takes
// less than asked (conz3d_nodes :819-829).
void conz3d(Model &m, std::vector<double> &cn1, double ddt, double rkpar, int istot, int isact,
            const std::vector<double> &gx, const std::vector<double> &gy, const std::vector<double> &cbound,
            Model::ScalarTerms *tm = nullptr) {
  int nlv = m.nlv;
  double az = m.p.azpar, ad = m.p.adpar, aa = m.p.aapar;
  double azt = 1. - az, adt = 1. - ad, aat = 1. - aa;
  double rstot = istot;
  double rso = (isact - 1) / rstot, rsn = isact / rstot, rsot = 1. - rso, rsnt = 1. - rsn;
  double dt = ddt / rstot;
  size_t nn = (size_t)nlv * m.nkn;
  std::vector<double> cn(nn, 0.), cdiag(nn, 0.), clow(nn, 0.), chigh(nn, 0.);
  for (int ie = 0; ie < m.nel; ie++) {
    const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
    int kn[3];
    double b[3], c[3];
    for (int ii = 0; ii < 3; ii++) { kn[ii] = m.nen3v[3 * ie + ii]; b[ii] = e[3 + ii]; c[ii] = e[6 + ii]; }
    double aj = e[9], aj4 = 4. * aj;
    int ilevel = m.ilhv[ie], jlevel = 1;
    int L2 = nlv + 2;
    std::vector<double> haver(L2, 0.), presentl(L2, 0.);
    std::vector<double> hnew(3 * (size_t)L2, 0.), hold(3 * (size_t)L2, 0.), cl(3 * (size_t)L2, 0.),
        wl(3 * (size_t)L2, 0.), vflux(3 * (size_t)L2, 0.);
    std::vector<double> clc(3 * (size_t)L2, 0.), clm(3 * (size_t)L2, 0.), clp(3 * (size_t)L2, 0.);
    auto H = [&](std::vector<double> &a, int l, int ii) -> double & { return a[(size_t)ii * L2 + l]; };
    for (int l = jlevel; l <= ilevel; l++) {
      haver[l] = rso * m.hdenv[(size_t)ie * nlv + l - 1] + rsot * m.hdeov[(size_t)ie * nlv + l - 1];
      presentl[l] = 1.;
      for (int ii = 0; ii < 3; ii++) {
        int k = kn[ii];
        double hn = m.hdknv[(size_t)k * nlv + l - 1], ho = m.hdkov[(size_t)k * nlv + l - 1];
        H(hold, l, ii) = rso * hn + rsot * ho;
        H(hnew, l, ii) = rsn * hn + rsnt * ho;
        H(cl, l, ii) = cn1[(size_t)k * nlv + l - 1];
        H(wl, l, ii) = m.wlnv[(size_t)k * (nlv + 1) + l];
        if (tm && tm->wsink != 0.)                 // settling (:496)
          H(wl, l, ii) -= tm->wsink * tm->wsinkv[(size_t)k * (nlv + 1) + l];
      }
    }
    for (int ii = 0; ii < 3; ii++) H(wl, ilevel, ii) = 0.;
    // vertical_flux_ie (tvd_admin.f90:930-1019): upwind, or with itvdv the
    // superbee-limited value between the upwind and downwind layers, the
    // far-upwind layer of this element's column giving the gradient ratio
    for (int ii = 0; ii < 3; ii++) {
      for (int l = jlevel; l <= ilevel - 1; l++) {
        double w = H(wl, l, ii);
        double conc = w > 0. ? H(cl, l + 1, ii) : H(cl, l, ii);
        double conf = conc;
        if (m.p.itvdv > 0) {
          double cond, conu;
          if (w > 0.) {
            cond = H(cl, l, ii);
            conu = l + 2 <= ilevel ? H(cl, l + 2, ii) : cond;
          } else {
            cond = H(cl, l + 1, ii);
            conu = l - 1 >= jlevel ? H(cl, l - 1, ii) : cond;
          }
          const double hdis = 0.5 * (H(hold, l, ii) + H(hold, l + 1, ii));
          const double alfa = dt * std::fabs(w) / hdis;
          const double rf = std::fabs(conc - cond) < 1.e-8 ? -1. : (cond - conu) / (cond - conc) - 1.;
          const double psi = std::max(0., std::max(std::min(1., 2. * rf), std::min(2., rf)));
          conf = conc + 0.5 * psi * (cond - conc) * (1. - alfa);
        }
        H(vflux, l, ii) = w * conf;
      }
      H(vflux, jlevel - 1, ii) = 0.;
      H(vflux, ilevel, ii) = 0.;
    }
    for (int l = jlevel; l <= ilevel; l++) {
      double us = az * m.utlnv[(size_t)ie * nlv + l - 1] + azt * m.utlov[(size_t)ie * nlv + l - 1];
      double vs = az * m.vtlnv[(size_t)ie * nlv + l - 1] + azt * m.vtlov[(size_t)ie * nlv + l - 1];
      double rk3 = 3. * rkpar * m.difhv[(size_t)ie * nlv + l - 1];
      int itot = 0, isum = 0;
      double f[3], fw[3], fd[3], fl[3], wdiff[3];
      for (int ii = 0; ii < 3; ii++) {
        int k = kn[ii];
        f[ii] = us * b[ii] + vs * c[ii];
        if (f[ii] < 0.) { itot++; isum += ii + 1; }
        fw[ii] = 0.;
        double waux = 0.;
        for (int iii = 0; iii < 3; iii++) waux += m.wdifhv[(size_t)9 * ie + 3 * iii + ii] * H(cl, l, iii);
        wdiff[ii] = waux;
        double rvptop = m.difv[(size_t)k * (nlv + 1) + l - 1] + m.p.difmol;
        double rvpbot = m.difv[(size_t)k * (nlv + 1) + l] + m.p.difmol;
        double hmotop = 2. * rvptop * presentl[l - 1] / (H(hold, l - 1, ii) + H(hold, l, ii));
        double hmobot = 2. * rvpbot * presentl[l + 1] / (H(hold, l, ii) + H(hold, l + 1, ii));
        double hmntop = 2. * rvptop * presentl[l - 1] / (H(hnew, l - 1, ii) + H(hnew, l, ii));
        double hmnbot = 2. * rvpbot * presentl[l + 1] / (H(hnew, l, ii) + H(hnew, l + 1, ii));
        fd[ii] = adt * ((H(cl, l, ii) - H(cl, l + 1, ii)) * hmobot - (H(cl, l - 1, ii) - H(cl, l, ii)) * hmotop);
        H(clc, l, ii) += ad * (hmntop + hmnbot);
        H(clm, l, ii) -= ad * hmntop;
        H(clp, l, ii) -= ad * hmnbot;
        double w = H(wl, l - 1, ii);
        if (l == jlevel) w = 0.;
        if (w >= 0.) H(clc, l, ii) += aa * w;
        else H(clm, l, ii) += aa * w;
        w = H(wl, l, ii);
        if (l == ilevel) w = 0.;
        if (w > 0.) H(clp, l, ii) -= aa * w;
        else H(clc, l, ii) -= aa * w;
        fw[ii] = aat * (H(vflux, l - 1, ii) - H(vflux, l, ii));
      }
      if (itot == 1) {
        for (int ii = 0; ii < 3; ii++) fl[ii] = f[ii] * H(cl, l, isum - 1);
      } else if (itot == 2) {
        int is = 6 - isum;
        for (int ii = 0; ii < 3; ii++) fl[ii] = f[ii] * H(cl, l, ii);
        fl[is - 1] = 0.;
        fl[is - 1] = -(fl[0] + fl[1] + fl[2]);
      } else {
        fl[0] = fl[1] = fl[2] = 0.;
      }
      // horizontal TVD (:675-686): elements without an open-boundary vertex
      if (m.p.itvd > 0 && m.bnd[kn[0]] <= 0 && m.bnd[kn[1]] <= 0 && m.bnd[kn[2]] <= 0) {
        const double c3[3] = {H(cl, l, 0), H(cl, l, 1), H(cl, l, 2)};
        tvd_fluxes(m, ie, l, itot, isum, dt, c3, gx, gy, f, cn1, fl);
      }
      for (int ii = 0; ii < 3; ii++) {
        int k = kn[ii];
        double hmed = haver[l];
        // nudging (:694-698): an = 0, so the relaxation is explicit and
        // finu, the implicit part of the diagonal (:729), is zero
        double fnudge = 0.;
        if (tm && tm->robs != 0.) {
          size_t q = (size_t)k * nlv + l - 1;
          fnudge = tm->robs * tm->rtauv[q] * (tm->cobs[q] - H(cl, l, ii));
        }
        double cexpl = aj4 * (H(hold, l, ii) * H(cl, l, ii) +
                              dt * (H(hold, l, ii) * fnudge + 3. * fl[ii] - fw[ii] - rk3 * hmed * wdiff[ii] -
                                    fd[ii]));
        double alow = aj4 * dt * H(clm, l, ii);
        double ahigh = aj4 * dt * H(clp, l, ii);
        double adiag = aj4 * dt * H(clc, l, ii) + aj4 * H(hnew, l, ii);
        size_t q = (size_t)k * nlv + l - 1;
        cn[q] += cexpl; clow[q] += alow; chigh[q] += ahigh; cdiag[q] += adiag;
      }
    }
  }
  // conz3d_nodes
  for (int k = 0; k < m.nkn; k++) {
    int ilevel = m.ilhkv[k], jlevel = 1;
    double *cnk = &cn[(size_t)k * nlv];
    double *cd = &cdiag[(size_t)k * nlv], *clo = &clow[(size_t)k * nlv], *chi = &chigh[(size_t)k * nlv];
    // boundary mass flux (:805-813): an inflow brings cbound, an outflow at
    // a boundary node the node's own concentration
    if (m.rqv[k] != 0.)
      for (int l = jlevel; l <= ilevel; l++) {
        const size_t q = (size_t)k * nlv + l - 1;
        const double qflux = m.mfluxv[q];
        const double cconz = qflux < 0. ? cn1[q] : cbound[q];
        cnk[l - 1] += dt * qflux * cconz;
      }
    // loading (:816-833) on the assembled mass: a source adds dt*loading; a
    // sink removes at most what an exponential decay over dt leaves, and the
    // load is cut to what was taken.  cload <= cn holds by construction, so
    // the reference's check on it (:827) never fires.
    for (int l = jlevel; tm && tm->rload != 0. && l <= ilevel; l++) {
      double &load = tm->load[(size_t)k * nlv + l - 1];
      double loading = tm->rload * load;
      if (loading == 0.) continue;
      if (loading < 0.) {
        double cload = 0.;
        if (cnk[l - 1] > 0.) cload = cnk[l - 1] * (1. - std::exp(dt * loading / cnk[l - 1]));
        else if (cnk[l - 1] < 0.) cnk[l - 1] = 0.;
        loading = -cload / dt;
        if (tm->rload > 0.) load = loading / tm->rload;
      }
      cnk[l - 1] += dt * loading;
    }
    if ((aa == 0. && ad == 0.) || nlv == 1) {
      for (int l = jlevel; l <= ilevel; l++)
        if (cd[l - 1] != 0.) cnk[l - 1] = cnk[l - 1] / cd[l - 1];
    } else {
      double aux = 1. / cd[jlevel - 1];
      chi[jlevel - 1] *= aux;
      cnk[jlevel - 1] *= aux;
      for (int l = jlevel + 1; l <= ilevel; l++) {
        aux = 1. / (cd[l - 1] - clo[l - 1] * chi[l - 2]);
        chi[l - 1] *= aux;
        cnk[l - 1] = (cnk[l - 1] - clo[l - 1] * cnk[l - 2]) * aux;
      }
      for (int l = ilevel - 1; l >= jlevel; l--) cnk[l - 1] = cnk[l - 1] - cnk[l] * chi[l - 1];
    }
  }
  for (size_t q = 0; q < nn; q++) cn1[q] = cn[q];
}

// scal3sh (concentration.f90:565-812): sub-stepping by the stability index,
// then conz3d per sub-step.  Returns SHY_EISTOT above istot_max.
// bndo_impbc (bndo.f90:700-760): on level-boundary nodes the scalar is set
// to its boundary value rbc(l,k) after each sub-step.
void bndo_impbc(Model &m, std::vector<double> &cnv, const std::vector<double> &rbc) {
  for (int k = 0; k < m.nkn; k++) {
    if (m.bnd[k] <= 0) continue;
    for (int l = 1; l <= m.ilhkv[k]; l++) cnv[(size_t)k * m.nlv + l - 1] = rbc[(size_t)k * m.nlv + l - 1];
  }
}

int scal3sh(Model &m, std::vector<double> &cnv, double rkpar, bool is_temp,
            const std::vector<double> &rbc, int *istot_out, Model::ScalarTerms *tm = nullptr) {
  double sindex = conzstab(m, rkpar, tm);
  double rindex = m.p.dt * sindex;
  int istot = 1 + (int)rindex;
  *istot_out = istot;
  int istot_max = m.p.istot_max > 0 ? m.p.istot_max : 1000;
  if (istot > istot_max) return fail(SHY_EISTOT, "scal3sh: istot index too high");
  std::vector<double> gx, gy;
  for (int isact = 1; isact <= istot; isact++) {
    if (!is_temp)
      for (auto &v : cnv) if (v < 1.e-15) v = 0.;
    if (m.p.itvd == 1) tvd_grad_3d(m, cnv, gx, gy);        // (concentration.f90:744)
    conz3d(m, cnv, m.p.dt, rkpar, istot, isact, gx, gy, rbc, tm);
    bndo_impbc(m, cnv, rbc);
  }
  return SHY_OK;
}

// ---------------------------------------------------------------------------
// Wetting and drying of elements on z-layers (wetdry.f90, topo_update.f90,
// bnd_routines.f90), used when the basin asks for it (shy_params::wetdry).
// ---------------------------------------------------------------------------
// setweg (wetdry.f90:128-345): iweich 0 first call (sets the minimum depth),
// 1 take away below hzmin (the hydro loop repeats), 2 take away below hzoff,
// 3 add back where the depth reached hzon.  Returns the number of changes.
int setweg(Model &m, int iweich, double dtime) {
  const double hzmin = m.p.hzmin, hzoff = m.p.hzoff, hzon = m.p.hzon, volmin = m.p.volmin;
  const int iwait = 5;                       // :176
  const bool bsigma = m.p.nsigma > 0;
  const bool bnewtime = dtime != m.dtime_weg;
  int iwh = 0;
  if (bsigma && iweich >= 1) return 0;       // :220
  if (iweich == 0) {
    for (int ie = 0; ie < m.nel; ie++) {
      const double aomega = m.ev[(size_t)ie * SHY_EVDIM + 9];
      double zmin = hzmin + volmin / (4. * aomega);
      if (zmin > hzoff) zmin = hzmin + 0.5 * (hzmin + hzoff);
      int iweg = 0;
      for (int ii = 0; ii < 3; ii++) {
        const double hzg = m.zenv[3 * ie + ii] + m.hm3v[3 * ie + ii];
        if (hzg < hzoff) iweg++;
        if (hzg < zmin) {
          m.zenv[3 * ie + ii] = zmin - m.hm3v[3 * ie + ii];
          if (bsigma) m.znv[m.nen3v[3 * ie + ii]] = m.zenv[3 * ie + ii];
        }
      }
      if (bsigma) iweg = 0;
      m.iwegv[ie] = iweg;
      if (iweg == 0) m.iwetv[ie] = 1;
      if (iweg > 0) iwh++;
    }
  } else if (iweich == 1 || iweich == 2) {
    const double hzlim = iweich == 1 ? hzmin : hzoff;
    for (int ie = 0; ie < m.nel; ie++) {
      if (m.iwegv[ie] != 0) continue;
      int iweg = 0;
      for (int ii = 0; ii < 3; ii++)
        if (m.znv[m.nen3v[3 * ie + ii]] + m.hm3v[3 * ie + ii] < hzlim) iweg++;
      if (iweg > 0) {
        iwh++;
        m.iwetv[ie] = 0;
        m.iwegv[ie] = iweg;
      }
    }
  } else if (iweich == 3) {
    for (int ie = 0; ie < m.nel; ie++) {
      if (m.iwegv[ie] <= 0) continue;
      int iweg = 0;
      double hztot = 0.;
      for (int ii = 0; ii < 3; ii++) {
        const double hzg = m.znv[m.nen3v[3 * ie + ii]] + m.hm3v[3 * ie + ii];
        hztot += hzg;
        if (hzg < hzon) iweg++;
      }
      hztot /= 3.;
      if (hztot >= hzon && -m.iwetv[ie] > iwait) iweg = 0;     // new algorithm (:306-312)
      if (iweg == 0) {
        iwh++;
        m.iwetv[ie] = 0;
        m.iwegv[ie] = 0;
      }
    }
  }
  for (int ie = 0; ie < m.nel; ie++)          // :322-331
    if (bnewtime || m.iwetv[ie] == 0) m.iwetv[ie] += m.iwegv[ie] == 0 ? 1 : -1;
  m.dtime_weg = dtime;
  return iwh;
}

// setnod (topo_update.f90:166-260): 0 internal, > 0 open boundary, -1
// boundary of the wet domain, -2 out of the system; from the angles of the
// wet elements around each node
int setnod(Model &m) {
  std::vector<double> winkv(m.nkn, 0.);
  for (int ie = 0; ie < m.nel; ie++)
    if (m.iwegv[ie] == 0)
      for (int ii = 0; ii < 3; ii++) winkv[m.nen3v[3 * ie + ii]] += m.ev[(size_t)ie * SHY_EVDIM + 10 + ii];
  for (int k = 0; k < m.nkn; k++) {
    if (winkv[k] > 359.99) m.inodv[k] = 0;
    else if (winkv[k] == 0.) m.inodv[k] = -2;
    else m.inodv[k] = -1;
  }
  for (int k = 0; k < m.nkn; k++)            // level boundaries (ibtyp 1)
    if (m.bnd[k] > 0) {
      if (m.inodv[k] != -1) return fail(SHY_EDEPTH, "setnod: error for open boundary node (dry boundary)");
      m.inodv[k] = m.bnd[k];
    }
  return SHY_OK;
}

// setznv (wetdry.f90:619-712): nodal levels from the wet elements' vertex
// levels (the larger where they differ), area-weighted from the dry ones
// where a node has no wet element
void setznv(Model &m) {
  std::vector<double> v1(m.nkn, 0.), v2(m.nkn, 0.);
  std::vector<char> set(m.nkn, 0);
  for (int ie = 0; ie < m.nel; ie++) {
    if (m.iwegv[ie] == 0) {
      for (int ii = 0; ii < 3; ii++) {
        const int k = m.nen3v[3 * ie + ii];
        double z = m.zenv[3 * ie + ii];
        if (set[k] && m.znv[k] != z) z = std::max(z, m.znv[k]);
        m.znv[k] = z;
        set[k] = 1;
      }
    } else {
      const double area = 4. * m.ev[(size_t)ie * SHY_EVDIM + 9];
      for (int ii = 0; ii < 3; ii++) {
        const int k = m.nen3v[3 * ie + ii];
        v1[k] += m.zenv[3 * ie + ii] * area;
        v2[k] += area;
      }
    }
  }
  for (int k = 0; k < m.nkn; k++)
    if (!set[k]) m.znv[k] = v1[k] / v2[k];
}

// setuvd (wetdry.f90:350-590): level and barotropic transport of each dry
// element, the element's volume kept, no vertex below hzmin
int setuvd(Model &m) {
  const double dt = m.p.dt, hzmin = m.p.hzmin, az = m.p.azpar, azt = 1. - az, eps = 1.e-5;
  for (int ie = 0; ie < m.nel; ie++) {
    if (m.iwegv[ie] <= 0) continue;
    const double *e = &m.ev[(size_t)ie * SHY_EVDIM];
    const double uo = m.uov[ie], vo = m.vov[ie];
    const double axdt = 3. * dt, adt = 1. / axdt;
    double zn[3], b[3], c[3], z[3], h[3];
    double zm = 0.;
    for (int ii = 0; ii < 3; ii++) {
      zn[ii] = m.zenv[3 * ie + ii];
      zm += zn[ii];
      b[ii] = e[3 + ii]; c[ii] = e[6 + ii];
      h[ii] = m.hm3v[3 * ie + ii];
    }
    const double zmed = zm / 3.;
    int itot = 0, isum = 0;
    for (int ii = 0; ii < 3; ii++) {
      if (zmed + h[ii] < hzmin) { z[ii] = hzmin - h[ii]; itot++; isum += ii + 1; }
      else z[ii] = zmed;
      zm -= z[ii];
    }
    if (itot == 1) {
      const int i1 = isum % 3, i2 = (i1 + 1) % 3, is = isum - 1;    // 0-based mod(isum,3)+1 etc.
      if (z[i1] + zm * 0.5 + h[i1] < hzmin) {
        z[i1] = hzmin - h[i1];
        z[i2] = 3. * zmed - z[i1] - z[is];
      } else if (z[i2] + zm * 0.5 + h[i2] < hzmin) {
        z[i2] = hzmin - h[i2];
        z[i1] = 3. * zmed - z[i2] - z[is];
      } else {
        z[i1] += 0.5 * zm;
        z[i2] += 0.5 * zm;
      }
    } else if (itot == 2) {
      const int i1 = 6 - isum - 1;
      z[i1] += zm;
    } else if (itot == 3) {
      return fail(SHY_EDEPTH, "setuvd: z computation");
    }
    zm = 0.;
    for (int ii = 0; ii < 3; ii++) {
      zm += z[ii];
      if (z[ii] + h[ii] < hzmin - eps) return fail(SHY_EDEPTH, "setuvd: z computation");
    }
    if (std::fabs(zm - 3. * zmed) > eps) return fail(SHY_EDEPTH, "setuvd: z computation");
    double d1 = (z[0] - zn[0]) * adt - azt * (b[0] * uo + c[0] * vo);
    double d2 = (z[1] - zn[1]) * adt - azt * (b[1] * uo + c[1] * vo);
    double det = 1. / (b[0] * c[1] - b[1] * c[0]);
    double u = det * (c[1] * d1 - c[0] * d2);
    double v = det * (-b[1] * d1 + b[0] * d2);
    itot = 0;
    for (int ii = 0; ii < 3; ii++) {
      const double zz = axdt * (b[ii] * (azt * uo + az * u) + c[ii] * (azt * vo + az * v)) + zn[ii];
      if (zz + h[ii] < hzmin - eps) itot++;
    }
    if (itot > 0) {                          // a node is drying: the velocity that keeps z
      if (az == 0.) return fail(SHY_EARG, "setuvd: drying with az=0 not possible");
      d1 = (z[0] - zn[0]) * adt - azt * (b[0] * uo + c[0] * vo);
      d2 = (z[1] - zn[1]) * adt - azt * (b[1] * uo + c[1] * vo);
      det = 1. / (az * (b[0] * c[1] - b[1] * c[0]));
      u = det * (c[1] * d1 - c[0] * d2);
      v = det * (-b[1] * d1 + b[0] * d2);
    }
    itot = 0;
    zm = 0.;
    for (int ii = 0; ii < 3; ii++) {
      const double zz = axdt * (b[ii] * (azt * uo + az * u) + c[ii] * (azt * vo + az * v)) + zn[ii];
      if (zz + h[ii] < hzmin - eps) itot++;
      m.zenv[3 * ie + ii] = zz;
      zm += zz;
    }
    if (std::fabs(zm - 3. * zmed) > eps) return fail(SHY_EDEPTH, "setuvd: z computation");
    if (itot > 0) return fail(SHY_EDEPTH, "setuvd: u/v computation");
    m.unv[ie] = u;
    m.vnv[ie] = v;
  }
  return SHY_OK;
}

// baro2l (transforms.f90:437-480): the barotropic transport of each dry
// element spread over its layers by their thickness
void baro2l(Model &m) {
  if (m.p.nsigma > 0) return;
  for (int ie = 0; ie < m.nel; ie++) {
    if (m.iwegv[ie] <= 0) continue;
    const int ilevel = m.ilhv[ie];
    double htot = 0.;
    for (int l = 1; l <= ilevel; l++) htot += m.hdenv[(size_t)ie * m.nlv + l - 1];
    for (int l = 1; l <= ilevel; l++) {
      const double weight = m.hdenv[(size_t)ie * m.nlv + l - 1] / htot;
      m.utlnv[(size_t)ie * m.nlv + l - 1] = m.unv[ie] * weight;
      m.vtlnv[(size_t)ie * m.nlv + l - 1] = m.vnv[ie] * weight;
    }
  }
}

// uvtopr (transforms.f90:214-270), the part of make_prvel (:553-566) that
// the next step reads: nodal velocities as the area-weighted mean of the
// element velocities ulnv = utlnv/hdenv (ttov, :98-122) over the elements
// in the system
void uvtopr(Model &m) {
  const int nlv = m.nlv;
  const size_t nn = (size_t)nlv * m.nkn;
  m.uprv.assign(nn, 0.); m.vprv.assign(nn, 0.);
  std::vector<double> vv(nn, 0.);
  for (int ie = 0; ie < m.nel; ie++) {
    if (m.iwegv[ie] != 0) continue;
    const double aj = m.ev[(size_t)ie * SHY_EVDIM + 9];
    for (int l = 0; l < m.ilhv[ie]; l++) {
      const size_t el = (size_t)ie * nlv + l;
      const double h = m.hdenv[el];
      const double ul = h > 0. ? m.utlnv[el] / h : 0., vl = h > 0. ? m.vtlnv[el] / h : 0.;
      for (int ii = 0; ii < 3; ii++) {
        const size_t kl = (size_t)m.nen3v[3 * ie + ii] * nlv + l;
        vv[kl] += aj; m.uprv[kl] += aj * ul; m.vprv[kl] += aj * vl;
      }
    }
  }
  for (size_t i = 0; i < nn; i++)
    if (vv[i] > 0.) { m.uprv[i] /= vv[i]; m.vprv[i] /= vv[i]; }
}

int init_state(Model &m) {
  m.zenv.assign((size_t)3 * m.nel, 0.);
  for (int ie = 0; ie < m.nel; ie++)
    for (int ii = 0; ii < 3; ii++) m.zenv[3 * ie + ii] = m.znv[m.nen3v[3 * ie + ii]];
  m.iwegv.assign(m.nel, 0); m.iwetv.assign(m.nel, 0); m.inodv.assign(m.nkn, 0);
  m.dtime_weg = -1.;
  if (m.p.wetdry) {                          // sp111 init: setweg(0) and setznv (bnd_routines.f90:413-415)
    setweg(m, 0, m.dtime);
    setznv(m);
  }
  m.unv.assign(m.nel, 0.); m.vnv.assign(m.nel, 0.);
  for (int ie = 0; ie < m.nel; ie++)
    for (int l = 0; l < m.ilhv[ie]; l++) {
      m.unv[ie] += m.utlnv[(size_t)ie * m.nlv + l];
      m.vnv[ie] += m.vtlnv[(size_t)ie * m.nlv + l];
    }
  int st = setdepth(m, m.hdknv, m.hdenv, m.zenv);
  if (st) return st;
  m.zov = m.znv; m.zeov = m.zenv; m.utlov = m.utlnv; m.vtlov = m.vtlnv;
  m.hdkov = m.hdknv; m.hdeov = m.hdenv;
  m.wlnv.assign((size_t)(m.nlv + 1) * m.nkn, 0.);
  m.wlov = m.wlnv;
  m.qpov.assign((size_t)m.nlv * m.nkn, 0.);         // nonhydro_init
  m.qpnv.assign((size_t)m.nlv * m.nkn, 0.);
  m.rhov.assign((size_t)m.nlv * m.nkn, 0.);
  if (m.p.ibarcl > 0) for (int it = 0; it < 3; it++) rhoset(m);   // barocl(0): rhoset_shell(3)
  uvtopr(m);                                      // make_prvel (initialize.f90:1656)
  m.info.volume = masscont(m);
  m.info.volume_budget = m.info.volume;   // the FP64 state's own volume is its budget
  m.tbnd = m.tempv; m.sbnd = m.saltv; m.cbnd = m.conzv;   // boundary values: initial columns
  return SHY_OK;
}

int step(Model &m) {
  if (m.p.wetdry) {                          // set_dry (shyfem_subs.f90:578) at the old time
    setweg(m, 2, m.dtime);
    setweg(m, 3, m.dtime);
  }
  // copy_uvz + copy_depth (transforms.f90:523; shyfem_subs.f90:589-591)
  m.dtime += m.p.dt;
  m.zov = m.znv; m.zeov = m.zenv; m.utlov = m.utlnv; m.vtlov = m.vtlnv;
  m.uov = m.unv; m.vov = m.vnv;
  m.hdkov = m.hdknv; m.hdeov = m.hdenv;
  m.wlov = m.wlnv;
  if (m.p.inohyd) {                               // nonhydro_copy (shyfem_subs.f90:590)
    m.qpov = m.qpnv;
    std::fill(m.qpnv.begin(), m.qpnv.end(), 0.);
  }
  set_rzv(m);                                     // sp111(2)
  set_mass_flux(m);
  // hydro (hydrodynamic.f90:284-485)
  int st = bottom_friction(m);
  if (st) return st;
  set_explicit(m);
  m.ddxv.assign((size_t)2 * m.nlv * m.nel, 0.);
  m.ddyv.assign((size_t)2 * m.nlv * m.nel, 0.);
  for (int ie = 0; ie < m.nel; ie++) {
    st = hydro_intern(m, ie);
    if (st) return st;
  }
  int krylov = 0;
  for (;;) {                                      // the loop over a changing domain (:374-404)
    if (m.p.wetdry) {
      st = setnod(m);
      if (st) return st;
    }
    hydro_zeta_assemble(m);
    st = zeta_solve(m);
    if (st) return st;
    krylov += m.info.krylov_iters;
    if (!m.p.wetdry || setweg(m, 1, m.dtime) == 0) break;
  }
  m.info.krylov_iters = krylov;
  if (m.p.wetdry) adjust_mass_flux(m);            // after the last setnod of the loop (:384)
  hydro_transports_final(m);
  for (int ie = 0; ie < m.nel; ie++)              // setzev: elements in the system
    if (!m.p.wetdry || m.iwegv[ie] == 0)
      for (int ii = 0; ii < 3; ii++) m.zenv[3 * ie + ii] = m.znv[m.nen3v[3 * ie + ii]];
  if (m.p.wetdry) {
    st = setuvd(m);
    if (st) return st;
    baro2l(m);
  }
  st = setdepth(m, m.hdknv, m.hdenv, m.zenv);     // make_new_depth
  if (st) return st;
  if (m.p.inohyd) {                               // sp256wnh + nonhydro_adjust (:435-438)
    st = nonhydro_adjust(m);
    if (st) return st;
  }
  hydro_vertical(m);
  uvtopr(m);                                      // compute_velocities (hydrodynamic.f90:473)
  m.info.volume = masscont(m);                    // vol_mass(1)
  m.info.volume_budget = m.info.volume;           // the FP64 state's own volume is its budget
  // run_scalar (shyfem_subs.f90:975-1028): T and S, then rho, then tracers
  int istot = 1;
  if (m.p.itemp) { st = scal3sh(m, m.tempv, m.p.thpar, true, m.tbnd, &istot); if (st) return st; }
  if (m.p.isalt) { st = scal3sh(m, m.saltv, m.p.shpar, false, m.sbnd, &istot); if (st) return st; }
  if (m.p.ibarcl > 0) rhoset(m);                  // rhoset_shell(1)
  for (int ic = 0; ic < m.p.nconz; ic++) {
    std::vector<double> c(m.conzv.begin() + (size_t)ic * m.nlv * m.nkn,
                          m.conzv.begin() + (size_t)(ic + 1) * m.nlv * m.nkn);
    std::vector<double> cb(m.cbnd.begin() + (size_t)ic * m.nlv * m.nkn,
                           m.cbnd.begin() + (size_t)(ic + 1) * m.nlv * m.nkn);
    st = scal3sh(m, c, m.p.chpar, false, cb, &istot, m.sterm.itr == ic ? &m.sterm : nullptr);
    if (st) return st;
    std::copy(c.begin(), c.end(), m.conzv.begin() + (size_t)ic * m.nlv * m.nkn);
  }
  m.info.istot = istot;
  m.info.dtime = m.dtime;
  return SHY_OK;
}

template <typename T> std::vector<double> dv(const T *p, size_t n, double def = 0.) {
  std::vector<double> v(n, def);
  if (p) for (size_t i = 0; i < n; i++) v[i] = (double)p[i];
  return v;
}

}  // namespace

// ===========================================================================
// C interface (ctypes)
// ===========================================================================
extern "C" {

const char *shyref_last_error(void) { return g_err.c_str(); }

int shyref_set_ev(int nkn, int nel, const int *nen3v /*1-based*/, const double *xgv,
                  const double *ygv, double *ev) {
  std::vector<int> nv((size_t)3 * nel);
  for (size_t i = 0; i < nv.size(); i++) nv[i] = nen3v[i] - 1;
  return set_ev(nkn, nel, nv.data(), xgv, ygv, ev);
}

int shyref_penta_fact(int n, double *val) { return penta_fact(n, val); }
int shyref_penta_factf(int n, double *val) { return penta_factf(n, val); }
void shyref_penta_solve(int n, const double *val, const double *r, double *s) { penta_solve(n, val, r, s); }
void shyref_tria_multi(int n, int m, double *v, double *r, double *s) { tria_multi(n, m, v, r, s); }
double shyref_sigma_stp(double s, double t, double p) {
  // the reference's arguments are single precision (eq_state.f90:154-159)
  return sigma_stp((double)(float)s, (double)(float)t, (double)(float)p);
}

int shyref_coo_init(int nkn, int nel, const int *nen3v /*1-based*/, int *ntg /*nkn+1*/,
                    int *icol /*cap*/, int *ijp /*9*nel, 0-based slots*/, int cap) {
  std::vector<int> nv((size_t)3 * nel);
  for (size_t i = 0; i < nv.size(); i++) nv[i] = nen3v[i] - 1;
  std::vector<int> a, b, c;
  int st = coo_init(nkn, nel, nv.data(), a, b, c);
  if (st) return st;
  if ((int)b.size() > cap) return fail(SHY_EARG, "coo_init: capacity");
  std::copy(a.begin(), a.end(), ntg);
  std::copy(b.begin(), b.end(), icol);
  std::copy(c.begin(), c.end(), ijp);
  return (int)b.size() > 0 ? SHY_OK : SHY_EARG;
}

// ILUT(5, 0.01) + BiCGStab solve of a CSR system (x: guess in, solution out)
int shyref_spk_solve(int n, const int *ia, const int *ja, const double *a, const double *b, double *x,
                     double rtol, double atol, int maxmv, int *iters, double *r0, double *r) {
  Ilu M;
  int st = ilut(n, ia, ja, a, 5, 0.01, M);
  if (st) return st;
  return bcgstab(n, ia, ja, a, M, b, x, rtol, atol, maxmv, iters, r0, r);
}

// The element system of hydro_zeta for given element inputs (used by the
// simsys parity test): ev (EVDIM), zeov(3), layer sums, barotropic transports,
// Dirichlet values (kFlag = none).
void shyref_element_system(const double *ev, const double *zeov, double dbb, double dbc, double dcb,
                           double dcc, double ut, double vt, const double *rzv3, double dt,
                           double az, double am, double grav, double *hia /*(3,3) col-major*/,
                           double *hik) {
  double b[3], c[3];
  for (int i = 0; i < 3; i++) { b[i] = ev[3 + i]; c[i] = ev[6 + i]; }
  double aj = ev[9], delta = dt * dt * az * am * grav;
  double h[3][3], k[3];
  for (int n = 0; n < 3; n++) {
    for (int mm = 0; mm < 3; mm++) {
      double abn = b[n] * (b[mm] * dbb + c[mm] * dbc);
      double acn = c[n] * (b[mm] * dcb + c[mm] * dcc);
      h[n][mm] = aj * ((n == mm ? 4. : 0.) + 12. * delta * (abn + acn));
    }
    k[n] = h[n][0] * zeov[0] + h[n][1] * zeov[1] + h[n][2] * zeov[2] +
           12. * aj * dt * (ut * b[n] + vt * c[n]);
  }
  for (int i = 0; i < 3; i++)
    if (rzv3[i] != kFlag) {
      double rw = rzv3[i];
      int j1 = (i + 1) % 3, j2 = (i + 2) % 3;
      k[j1] -= rw * h[j1][i]; k[j2] -= rw * h[j2][i];
      h[i][j1] = h[i][j2] = h[j1][i] = h[j2][i] = 0.;
      k[i] = rw * h[i][i];
    }
  for (int n = 0; n < 3; n++) {
    for (int mm = 0; mm < 3; mm++) hia[mm * 3 + n] = h[n][mm];
    hik[n] = k[n];
  }
}

double shyref_flag(void) { return kFlag; }

// --- whole model ------------------------------------------------------------
void *shyref_create(const shy_basin *B, const shy_params *P) {
  Model *m = new Model();
  m->nkn = B->nkn; m->nel = B->nel; m->nlv = B->nlv; m->p = *P;
  int nkn = m->nkn, nel = m->nel, nlv = m->nlv;
  if (nlv < 1 || nlv > SHY_MAX_LAYERS) { fail(SHY_EARG, "shyref_create: nlv"); delete m; return nullptr; }
  if (P->nsigma < 0 || P->nsigma > nlv) { fail(SHY_EARG, "shyref_create: nsigma outside 0..nlv"); delete m; return nullptr; }
  if (P->nzadapt > 1 && (P->nsigma > 0 || P->ibarcl > 0 || P->wetdry)) {
    fail(SHY_EARG, "shyref_create: z-adaptive layers on z-layers without baroclinic terms or wetting and drying");
    delete m;
    return nullptr;
  }
  if (P->inohyd && (P->wetdry || P->nzadapt > 1 || !(P->aqpar > 0.f && P->aqpar <= 1.f))) {
    fail(SHY_EARG, "shyref_create: non-hydrostatic pressure needs 0 < aqpar <= 1, no wetting and drying and "
                   "no z-adaptive layers");
    delete m;
    return nullptr;
  }
  m->nen3v.resize((size_t)3 * nel);
  for (size_t i = 0; i < m->nen3v.size(); i++) m->nen3v[i] = B->nen3v[i] - 1;
  std::vector<double> x = dv(B->xgv, nkn), y = dv(B->ygv, nkn);
  m->ev.assign((size_t)SHY_EVDIM * nel, 0.);
  if (set_ev(nkn, nel, m->nen3v.data(), x.data(), y.data(), m->ev.data())) { delete m; return nullptr; }
  if (P->itvd == 2) tvd_upwind_init(*m, x, y);
  m->hm3v = dv(B->hm3v, (size_t)3 * nel);
  m->hev.assign(nel, 0.);
  for (int ie = 0; ie < nel; ie++)   // element depth: mean of vertex depths (hev)
    m->hev[ie] = (m->hm3v[3 * ie] + m->hm3v[3 * ie + 1] + m->hm3v[3 * ie + 2]) / 3.;
  m->hlv = dv(B->hlv, nlv); m->hldv = dv(B->hldv, nlv);
  m->ilhv.assign(B->ilhv, B->ilhv + nel); m->ilhkv.assign(B->ilhkv, B->ilhkv + nkn);
  m->czv = dv(B->czv, nel); m->fcorv = dv(B->fcorv, nel);
  m->visv = dv(B->visv, (size_t)(nlv + 1) * nkn); m->difv = dv(B->difv, (size_t)(nlv + 1) * nkn);
  m->tauxnv = dv(B->tauxnv, nkn); m->tauynv = dv(B->tauynv, nkn);
  m->ppv = dv(B->ppv, nkn); m->rqv = dv(B->rqv, nkn);
  m->mfluxv.assign((size_t)nkn * B->nlv, 0.);
  m->bnd.assign(nkn, 0);
  if (B->bnd_index) m->bnd.assign(B->bnd_index, B->bnd_index + nkn);
  m->nbnd = B->nbnd; m->ntide = B->ntide;
  m->tide = dv(B->tide, (size_t)4 * B->ntide * B->nbnd);
  m->difhv.assign((size_t)nlv * nel, 1.);     // set_diffusivity with idhtyp = 0
  set_area(*m);
  diffweight(*m);
  set_ieltv(*m);
  if (coo_init(nkn, nel, m->nen3v.data(), m->ntg, m->icol, m->ijp)) { delete m; return nullptr; }
  if (P->inohyd) coo3d_init(nkn, nlv, m->ntg, m->nt3g);
  m->qdistv.assign(nkn, 1.);                  // qhdist with nqdist = 0
  m->rtol = P->solver_rtol > 0 ? P->solver_rtol : 1e-8;
  m->atol = P->solver_atol > 0 ? P->solver_atol : 1e-8;
  m->maxmv = P->solver_maxit > 0 ? P->solver_maxit : 1000;
  m->dtime = P->dtime0;
  m->znv.assign(nkn, 0.); m->utlnv.assign((size_t)nlv * nel, 0.); m->vtlnv.assign((size_t)nlv * nel, 0.);
  m->tempv.assign((size_t)nlv * nkn, 0.); m->saltv.assign((size_t)nlv * nkn, 0.);
  m->conzv.assign((size_t)nlv * nkn * std::max(0, P->nconz), 0.);
  m->unv.assign(nel, 0.); m->vnv.assign(nel, 0.);
  return m;
}

void shyref_destroy(void *h) { delete (Model *)h; }

int shyref_set_state(void *h, const shy_state *s) {
  Model &m = *(Model *)h;
  size_t nel = m.nel, nkn = m.nkn, nlv = m.nlv;
  if (s->znv) m.znv = dv(s->znv, nkn);
  if (s->utlnv) m.utlnv = dv(s->utlnv, nlv * nel);
  if (s->vtlnv) m.vtlnv = dv(s->vtlnv, nlv * nel);
  if (s->tempv) m.tempv = dv(s->tempv, nlv * nkn);
  if (s->saltv) m.saltv = dv(s->saltv, nlv * nkn);
  if (s->conzv) m.conzv = dv(s->conzv, nlv * nkn * std::max(0, m.p.nconz));
  return init_state(m);
}

// state out as double (FP64 oracle)
int shyref_get_state64(void *h, double *znv, double *utlnv, double *vtlnv, double *hdknv,
                       double *wlnv, double *tempv, double *saltv, double *rhov, double *conzv,
                       double *zenv, double *hdenv) {
  Model &m = *(Model *)h;
  auto cp = [](const std::vector<double> &a, double *o) { if (o) std::copy(a.begin(), a.end(), o); };
  cp(m.znv, znv); cp(m.utlnv, utlnv); cp(m.vtlnv, vtlnv); cp(m.hdknv, hdknv); cp(m.wlnv, wlnv);
  cp(m.tempv, tempv); cp(m.saltv, saltv); cp(m.rhov, rhov); cp(m.conzv, conzv);
  cp(m.zenv, zenv); cp(m.hdenv, hdenv);
  return SHY_OK;
}

int shyref_run(void *h, int nsteps) {
  Model &m = *(Model *)h;
  for (int i = 0; i < nsteps; i++) {
    int st = step(m);
    if (st) return st;
  }
  return SHY_OK;
}

// wet/dry state: iwegv (nel), iwetv (nel), inodv (nkn); any may be NULL
int shyref_wetdry(void *h, int *iwegv, int *iwetv, int *inodv) {
  Model *m = (Model *)h;
  for (int ie = 0; ie < m->nel; ie++) {
    if (iwegv) iwegv[ie] = m->iwegv.empty() ? 0 : m->iwegv[ie];
    if (iwetv) iwetv[ie] = m->iwetv.empty() ? 0 : m->iwetv[ie];
  }
  if (inodv) for (int k = 0; k < m->nkn; k++) inodv[k] = m->inodv.empty() ? 0 : m->inodv[k];
  return SHY_OK;
}

// the nudging contribution andgzv per node (nudge_zeta, nudge.f90:300-338,
// computed by the caller from its observations); NULL clears it
int shyref_set_nudging(void *h, const float *andgzv) {
  Model &m = *(Model *)h;
  if (!andgzv) { m.andgzv.clear(); return SHY_OK; }
  m.andgzv.assign(andgzv, andgzv + m.nkn);
  return SHY_OK;
}

// conz3d_omp's source terms for tracer itr (itr < 0: none): arrays (nkn,
// nlv) but wsinkv (nkn, nlv+1); an array whose factor is zero is unused.
// load is read back with shyref_get_load after deposition has cut it.
int shyref_set_scalar_terms(void *h, int itr, const float *cobs, float robs, const float *rtauv, float wsink,
                            const float *wsinkv, float rload, const float *load) {
  Model &m = *(Model *)h;
  Model::ScalarTerms t;
  t.itr = itr;
  const size_t n = (size_t)m.nkn * m.nlv, n1 = (size_t)m.nkn * (m.nlv + 1);
  if (itr >= 0) {
    if ((robs != 0.f && (!cobs || !rtauv)) || (wsink != 0.f && !wsinkv) || (rload != 0.f && !load))
      return fail(SHY_EARG, "set_scalar_terms: a term without its array");
    t.robs = robs; t.wsink = wsink; t.rload = rload;
    if (robs != 0.f) { t.cobs.assign(cobs, cobs + n); t.rtauv.assign(rtauv, rtauv + n); }
    if (wsink != 0.f) t.wsinkv.assign(wsinkv, wsinkv + n1);
    if (rload != 0.f) t.load.assign(load, load + n);
  }
  m.sterm = std::move(t);
  return SHY_OK;
}

// boundary values of a scalar (what 0 temperature, 1 salinity, 2 tracer
// itr), (nkn, nlv): imposed on level boundaries after each sub-step and
// brought in by inflows (make_scal_flux's r3v, bnd_routines.f90:1215-1300)
int shyref_set_bound_scalar(void *h, int what, int itr, const float *values) {
  Model &m = *(Model *)h;
  const size_t n = (size_t)m.nkn * m.nlv;
  std::vector<double> *dst = nullptr;
  size_t off = 0;
  if (what == 0 && m.p.itemp) dst = &m.tbnd;
  else if (what == 1 && m.p.isalt) dst = &m.sbnd;
  else if (what == 2 && itr >= 0 && itr < m.p.nconz) { dst = &m.cbnd; off = (size_t)itr * n; }
  if (!dst || !values) return fail(SHY_EARG, "set_bound_scalar: no such scalar");
  for (size_t q = 0; q < n; q++) (*dst)[off + q] = values[q];
  return SHY_OK;
}

int shyref_get_load(void *h, double *load) {
  Model &m = *(Model *)h;
  std::copy(m.sterm.load.begin(), m.sterm.load.end(), load);
  return SHY_OK;
}

int shyref_step_info(void *h, shy_step_info *info) {
  Model &m = *(Model *)h;
  *info = m.info;
  info->dtime = m.dtime;
  return SHY_OK;
}

// the weight of the non-hydrostatic pressure per node (qhdist, nohydro.f90:
// 962-1040: 0 on open boundaries with nad > 0, rising to 1 inland)
int shyref_set_nh_distance(void *h, const float *qdist) {
  Model &m = *(Model *)h;
  if (!qdist) return fail(SHY_EARG, "set_nh_distance: no array");
  m.qdistv.assign(qdist, qdist + m.nkn);
  return SHY_OK;
}

// the non-hydrostatic pressure qpnv (nkn, nlv) after the last step and the
// w of sp256wnh (nkn, nlv+1); either may be NULL
int shyref_get_nh(void *h, double *qpnv, double *wnh) {
  Model &m = *(Model *)h;
  if (qpnv) std::copy(m.qpnv.begin(), m.qpnv.end(), qpnv);
  if (wnh) {
    if (m.wnh.empty()) std::fill(wnh, wnh + (size_t)(m.nlv + 1) * m.nkn, 0.);
    else std::copy(m.wnh.begin(), m.wnh.end(), wnh);
  }
  return SHY_OK;
}

// iterations and residuals of the last non-hydrostatic solve
int shyref_nh_info(void *h, int *iters, double *resid0, double *resid) {
  Model &m = *(Model *)h;
  if (iters) *iters = m.nh_iters;
  if (resid0) *resid0 = m.nh_resid0;
  if (resid) *resid = m.nh_resid;
  return SHY_OK;
}

// The 3D simsys interface on its own (system_assemble_3d, system_adjust_matrix_3d,
// system_solve_3d, system_get_3d; simsys_spkaux.f90:495-716) over a mesh
// of nkn nodes, nel elements (1-based nen3v) and nlv layers: the values of
// the 3D COO (nt3g[nkn] entries) and its right-hand side ((nlv+2)*nkn)
void *shyref_sys3d_create(int nkn, int nel, int nlv, const int *nen3v) {
  Model *m = new Model();
  m->nkn = nkn; m->nel = nel; m->nlv = nlv;
  m->nen3v.resize((size_t)3 * nel);
  for (size_t i = 0; i < m->nen3v.size(); i++) m->nen3v[i] = nen3v[i] - 1;
  if (coo_init(nkn, nel, m->nen3v.data(), m->ntg, m->icol, m->ijp)) { delete m; return nullptr; }
  coo3d_init(nkn, nlv, m->ntg, m->nt3g);
  m->c3coo.assign(m->nt3g[nkn], 0.);
  m->rvec3d.assign((size_t)(nlv + 2) * nkn, 0.);
  return m;
}

int shyref_sys3d_nnz(void *h) { return ((Model *)h)->nt3g[((Model *)h)->nkn]; }

// ie, l 1-based as the reference passes them; mass(-1:1,3,3) in Fortran order
int shyref_sys3d_assemble(void *h, int ie, int l, const float *mass, const float *rhs) {
  Model &m = *(Model *)h;
  if (ie < 1 || ie > m.nel || l < 1 || l > m.nlv) return fail(SHY_EARG, "sys3d_assemble: ie or l out of range");
  double ms[27], r[3];
  for (int d = 0; d < 3; d++)
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) ms[d * 9 + 3 * i + j] = mass[d + 3 * i + 9 * j];
  for (int i = 0; i < 3; i++) r[i] = rhs[i];
  assemble_3d(m, ie - 1, l, ms, r);
  return SHY_OK;
}

int shyref_sys3d_adjust(void *h) { adjust_3d(*(Model *)h); return SHY_OK; }

// z (nkn, nlv) rows: the guess in, the solution out
int shyref_sys3d_solve(void *h, double *z, int *iters) {
  Model &m = *(Model *)h;
  std::vector<double> zz(z, z + (size_t)m.nkn * m.nlv);
  int st = solve_3d(m, zz);
  if (iters) *iters = m.nh_iters;
  if (st) return st;
  std::copy(zz.begin(), zz.end(), z);
  return SHY_OK;
}

int shyref_sys3d_get(void *h, double *val, double *rhs, int *ia, int *ja) {
  Model &m = *(Model *)h;
  if (val) std::copy(m.c3coo.begin(), m.c3coo.end(), val);
  if (rhs) std::copy(m.rvec3d.begin(), m.rvec3d.end(), rhs);
  if (ia || ja) {
    std::vector<int> a, b;
    coo3d_csr(m, a, b);
    if (ia) std::copy(a.begin(), a.end(), ia);
    if (ja) std::copy(b.begin(), b.end(), ja);
  }
  return SHY_OK;
}

void shyref_sys3d_destroy(void *h) { delete (Model *)h; }

// matrix of the last assembly (for the assembly parity test)
int shyref_last_system(void *h, int *nnz, double *val, double *rhs) {
  Model &m = *(Model *)h;
  *nnz = (int)m.c2coo.size();
  if (val) std::copy(m.c2coo.begin(), m.c2coo.end(), val);
  if (rhs) std::copy(m.rvec2d.begin(), m.rvec2d.end(), rhs);
  return SHY_OK;
}

}  // extern "C"
