// host.cu -- the engine's C ABI: system set-up, walker state, dispatch.
//
// One warp owns one walker.  Walker state lives in HBM, walker-major:
//   x[w][e][3] (double), ainv[w][spin block][k][e] (double, reference-determinant inverse),
//   fso[w][i][j] (T, Jastrow pair table: i != j pair term incl. e-e-n, i == j e-n term),
//   ln|D|, sign, J per walker.
// Per-warp scratch (basis values, proposed orbital row, gradient accumulators) lives in
// shared memory; larger per-walker scratch (orbitals of all electrons, projected
// coefficients, pseudopotential task lists) in HBM.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/champ_b200.h"
#include <cub/cub.cuh>
#include <cublas_v2.h>

#include "ctx.h"

using namespace champ;

// The limits the header publishes are the ones the kernels are compiled for.
static_assert(CHAMP_MAX_CTYPE == MAXCT, "centre types");
static_assert(CHAMP_MAX_LCHAN == MAXLCH, "pseudopotential channels");
static_assert(CHAMP_MAX_QUAD == MAXQ, "quadrature points");

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
static thread_local std::string g_err;
int champ_fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

static int fail(int code, const std::string &msg) { return champ_fail(code, msg); }
static int quad_points(const champ_ctx *c) { return c->nquad > 0 ? c->nquad : 12; }


static double host_det(std::vector<double> a, int n) {
  double d = 1;
  for (int c = 0; c < n; c++) {
    int p = c;
    for (int i = c + 1; i < n; i++)
      if (std::fabs(a[i * n + c]) > std::fabs(a[p * n + c])) p = i;
    if (a[p * n + c] == 0) return 0;
    if (p != c) {
      d = -d;
      for (int j = 0; j < n; j++) std::swap(a[c * n + j], a[p * n + j]);
    }
    d *= a[c * n + c];
    for (int i = c + 1; i < n; i++) {
      double f = a[i * n + c] / a[c * n + c];
      for (int j = c; j < n; j++) a[i * n + j] -= f * a[c * n + j];
    }
  }
  return d;
}

static int build_multidet(const champ_system *d, MultiDet &md) {
  const int N = d->nelec, nup = d->nup;
  md.ndet = d->ndet;
  md.ciu.assign(d->ndet, 0);
  md.cid.assign(d->ndet, 0);
  md.ccoef.assign(d->ndet, 0.0);
  for (int icsf = 0, off = 0; icsf < d->ncsf; icsf++)
    for (int i = 0; i < d->csf_ndet[icsf]; i++, off++) {
      int I = d->csf_det[off];
      if (I < 0 || I >= d->ndet) return fail(CHAMP_EINVAL, "csf_det index out of range");
      md.ccoef[I] += d->csf_det_coef[off] * d->csf_coef[icsf];
    }
  uint64_t lcg = 88172645463325252ull;
  auto rnd = [&]() { lcg = lcg * 6364136223846793005ull + 1442695040888963407ull; return 0.5 + (double)(lcg >> 11) / 9007199254740992.0; };
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? N - nup : nup, o0 = sp ? nup : 0;
    std::vector<int> R(d->det_orb + o0, d->det_orb + o0 + n);
    std::vector<int> used;
    for (int I = 0; I < d->ndet; I++)
      for (int j = 0; j < n; j++) {
        int o = d->det_orb[I * N + o0 + j];
        if (o < 0 || o >= d->norb) return fail(CHAMP_EINVAL, "det_orb orbital index out of range");
        if (std::find(R.begin(), R.end(), o) == R.end() && std::find(used.begin(), used.end(), o) == used.end())
          used.push_back(o);
      }
    std::sort(used.begin(), used.end());
    md.occ[sp] = R;
    md.occ[sp].insert(md.occ[sp].end(), used.begin(), used.end());
    md.nocc[sp] = (int)md.occ[sp].size();
    md.nvirt[sp] = (int)used.size();
    const int no = md.nocc[sp];
    auto col = [&](int o) { return (int)(std::find(md.occ[sp].begin(), md.occ[sp].end(), o) - md.occ[sp].begin()); };
    // a random T with T[:, reference] = 1 fixes each determinant's sign relative to det(alpha)
    std::vector<double> Tr((size_t)n * std::max(no, 1));
    for (int k = 0; k < n; k++)
      for (int m = 0; m < no; m++) Tr[(size_t)k * no + m] = (m < n) ? (m == k ? 1.0 : 0.0) : rnd();
    std::vector<std::vector<int>> uniq;
    for (int I = 0; I < d->ndet; I++) {
      std::vector<int> L(d->det_orb + I * N + o0, d->det_orb + I * N + o0 + n);
      int u = -1;
      for (size_t q = 0; q < uniq.size(); q++)
        if (uniq[q] == L) { u = (int)q; break; }
      if (u < 0) {
        u = (int)uniq.size();
        uniq.push_back(L);
        std::vector<int> holes, parts;
        for (int k = 0; k < n; k++)
          if (std::find(L.begin(), L.end(), R[k]) == L.end()) holes.push_back(k);
        for (int j = 0; j < n; j++)
          if (col(L[j]) >= n) parts.push_back(col(L[j]) - n);
        for (int j = 0; j < n; j++)
          for (int j2 = j + 1; j2 < n; j2++)
            if (L[j] == L[j2]) return fail(CHAMP_EINVAL, "determinant with a repeated orbital");
        if (holes.size() != parts.size() || holes.size() > 4)
          return fail(CHAMP_EINVAL, "determinant more than 4 excitations away from the reference");
        int k = (int)holes.size();
        std::vector<double> M((size_t)n * n), a((size_t)k * k);
        for (int r = 0; r < n; r++)
          for (int j = 0; j < n; j++) M[(size_t)r * n + j] = Tr[(size_t)r * no + col(L[j])];
        for (int ia = 0; ia < k; ia++)
          for (int ib = 0; ib < k; ib++) a[(size_t)ia * k + ib] = Tr[(size_t)holes[ia] * no + n + parts[ib]];
        double dm = host_det(M, n), da = k ? host_det(a, k) : 1.0;
        double sg = dm / da;
        if (!(std::fabs(std::fabs(sg) - 1.0) < 1e-6)) return fail(CHAMP_EINVAL, "could not fix a determinant's sign");
        md.dk[sp].push_back(k);
        for (int i = 0; i < 4; i++) {
          md.dh[sp].push_back(i < k ? holes[i] : 0);
          md.dp[sp].push_back(i < k ? parts[i] : 0);
        }
        md.dsg[sp].push_back(sg > 0 ? 1.0 : -1.0);
      }
      (sp ? md.cid : md.ciu)[I] = u;
    }
    md.ndu[sp] = (int)uniq.size();
  }
  md.multidet = (d->ndet > 1 || md.nvirt[0] > 0 || md.nvirt[1] > 0) ? 1 : 0;
  if (!md.multidet && md.ccoef[0] == 0.0) return fail(CHAMP_EINVAL, "zero determinant coefficient");
  return CHAMP_OK;
}


template <class T>
static T *dalloc(champ_ctx *c, size_t n) {
  void *p = nullptr;
  if (cudaMalloc(&p, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
  cudaMemset(p, 0, sizeof(T) * (n ? n : 1));
  c->allocs.push_back(p);
  return (T *)p;
}

static double host_fact(int n) {
  double f = 1;
  for (int i = 2; i <= n; i++) f *= i;
  return f;
}
// basis_norm.f90:53-60 (with sqrt((2l+1)/4pi))
static double host_anorm(int kind, int n, int l, double z) {
  const double pi = 3.141592653589793;
  if (kind == 0) return std::sqrt(std::pow(2 * z, 2 * n + 1) * (2 * l + 1) / (host_fact(2 * n) * 4 * pi));
  double g = std::sqrt(pi);
  for (int i = 1; i <= n; i++) g *= (i - 0.5);
  return std::sqrt(2 * std::pow(2 * z, n + 0.5) * (2 * l + 1) / (g * 4 * pi));
}

// Numerical radial tables (read_bas_num.f90:213-378, spline2.f90): per table the grid
// parameters as splfit_bas uses them, a 5-point polynomial through the first grid points (its
// slope at the first point is the spline's left end condition), an exponential a0 exp(-ak r)
// matched at the last points (its slope is the right end condition), and the spline's second
// derivatives.  Grid 3 reads the last point as r0 and derives r0 = r_last / (h^(nr-1) - 1).
static int build_radial_tables(const champ_system *d, champ_ctx *c) {
  c->rad_tab.clear(); c->rad_par.clear(); c->rad_y.clear(); c->rad_y2.clear();
  c->rad_shell.assign(d->nshell, -1);
  bool any = false;
  for (int i = 0; i < d->nshell; i++)
    if (d->shell_kind[i] == 2) {
      if (d->nrad < 1 || !d->shell_rad || d->shell_rad[i] < 0 || d->shell_rad[i] >= d->nrad)
        return fail(CHAMP_EINVAL, "numerical shell without a valid radial table");
      if (d->shell_nprim[i] != 1) return fail(CHAMP_EINVAL, "a numerical shell has exactly one primitive");
      c->rad_shell[i] = d->shell_rad[i];
      any = true;
    }
  if (!any) return CHAMP_OK;
  if (!d->rad_igrid || !d->rad_nr || !d->rad_h || !d->rad_r0 || !d->rad_x || !d->rad_val)
    return fail(CHAMP_EINVAL, "numerical radial tables: null array");
  size_t off = 0;
  for (int t = 0; t < d->nrad; t++) {
    const int g = d->rad_igrid[t], nr = d->rad_nr[t];
    if (g < 1 || g > 3) return fail(CHAMP_EINVAL, "radial grid type must be 1, 2 or 3");
    if (nr < 6) return fail(CHAMP_EINVAL, "a radial table needs at least 6 points");
    const double *x = d->rad_x + off, *y = d->rad_val + off;
    double h = d->rad_h[t], r0 = d->rad_r0[t];
    if (g == 2 && h <= 1.0) h = x[1] / x[0];
    if (g == 3) r0 = r0 / (std::pow(h, nr - 1) - 1.0);
    if (g == 2 && (r0 <= 0.0 || h <= 0.0)) { r0 = x[0]; h = x[1] / x[0]; }
    // small r: y = c0 + c1 r + ... + c4 r^4 through the first 5 points (Gauss-Jordan, pivoting)
    double A[5][6];
    for (int i = 0; i < 5; i++) {
      double pw = 1.0;
      for (int j = 0; j < 5; j++) { A[i][j] = pw; pw *= x[i]; }
      A[i][5] = y[i];
    }
    for (int col = 0; col < 5; col++) {
      int pv = col;
      for (int i = col + 1; i < 5; i++)
        if (std::fabs(A[i][col]) > std::fabs(A[pv][col])) pv = i;
      if (A[pv][col] == 0.0) return fail(CHAMP_EINVAL, "radial table: singular small-r fit");
      for (int j = 0; j < 6; j++) std::swap(A[col][j], A[pv][j]);
      for (int i = 0; i < 5; i++) {
        if (i == col) continue;
        const double f = A[i][col] / A[col][col];
        for (int j = col; j < 6; j++) A[i][j] -= f * A[col][j];
      }
    }
    double ce[5];
    for (int i = 0; i < 5; i++) ce[i] = A[i][5] / A[i][i];
    double dwf1 = 0;
    for (int i = 1; i < 5; i++) dwf1 += i * ce[i] * std::pow(x[0], i - 1);
    // large r: a0 exp(-ak r) with ak from the last two points
    double ae1 = 0, ae2 = 0, dwfn = 0;
    const double wfm = 0.5 * (y[nr - 1] + y[nr - 2]), dwfm = (y[nr - 1] - y[nr - 2]) / (x[nr - 1] - x[nr - 2]);
    if (std::fabs(wfm) > 1e-99) {
      ae2 = (dwfm / wfm < 0) ? -dwfm / wfm : 0.1;
      ae1 = y[nr - 1] * std::exp(ae2 * x[nr - 1]);
      dwfn = -ae2 * y[nr - 1];
    }
    // cubic spline with those end slopes (tridiagonal solve)
    std::vector<double> y2(nr), u(nr);
    y2[0] = -0.5;
    u[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - dwf1);
    for (int i = 1; i < nr - 1; i++) {
      const double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]), pp = sig * y2[i - 1] + 2.0;
      y2[i] = (sig - 1.0) / pp;
      u[i] = (6.0 * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1])) / (x[i + 1] - x[i - 1]) -
              sig * u[i - 1]) / pp;
    }
    const double qn = 0.5, un = (3.0 / (x[nr - 1] - x[nr - 2])) * (dwfn - (y[nr - 1] - y[nr - 2]) / (x[nr - 1] - x[nr - 2]));
    y2[nr - 1] = (un - qn * u[nr - 2]) / (qn * y2[nr - 2] + 1.0);
    for (int k = nr - 2; k >= 0; k--) y2[k] = y2[k] * y2[k + 1] + u[k];
    c->rad_tab.push_back(make_int4(g, nr, (int)c->rad_y.size(), 0));
    const double par[10] = {r0, h, std::log(h), ce[0], ce[1], ce[2], ce[3], ce[4], ae1, ae2};
    c->rad_par.insert(c->rad_par.end(), par, par + 10);
    c->rad_y.insert(c->rad_y.end(), y, y + nr);
    c->rad_y2.insert(c->rad_y2.end(), y2.begin(), y2.end());
    off += nr;
  }
  return CHAMP_OK;
}

// Angular quadrature of the nonlocal integration (gesqua, qmc/vmc/rotqua.f90:1-618): the rule
// with the number of points closest to nq among 4, 6, 12, 18, 26, 32, 50, 24, 20, 86 (ties go to
// the first listed), points on the unit sphere and weights summing to one.  Returns the points.
static int quadrature_rule(int nq_in, double (*q)[3], double *w) {
  static const int iq[10] = {4, 6, 12, 18, 26, 32, 50, 24, 20, 86};
  int icase = 0;
  for (int i = 1; i < 10; i++)
    if (std::abs(nq_in - iq[i]) < std::abs(nq_in - iq[icase])) icase = i;
  const int nq = iq[icase];
  for (int j = 0; j < MAXQ; j++) q[j][0] = q[j][1] = q[j][2] = w[j] = 0.0;
  // weights per point type (rows: rule; columns: point type), then the types' point counts
  double ww[10][6] = {{0}};
  ww[0][0] = 1.0 / 4; ww[1][0] = 1.0 / 6; ww[2][0] = 1.0 / 12; ww[3][0] = 1.0 / 30; ww[4][0] = 1.0 / 21;
  ww[5][0] = 5.0 / 168; ww[6][0] = 4.0 / 315; ww[2][1] = 1.0 / 12; ww[3][1] = 1.0 / 15; ww[4][1] = 4.0 / 105;
  ww[5][1] = 5.0 / 168; ww[6][1] = 64.0 / 2835; ww[4][2] = 27.0 / 840; ww[5][2] = 27.0 / 840;
  ww[6][2] = 27.0 / 1280; ww[6][3] = 14641.0 / 725760; ww[7][0] = 1.0 / 24; ww[8][0] = 1.0 / 20;
  ww[9][0] = .0115440115441; ww[9][2] = .0119439090859; ww[9][3] = .0111105557106; ww[9][4] = .0118765012945;
  ww[9][5] = .0118123037469;
  static const int octa[6] = {6, 12, 8, 24, 0, 0}, icosa[6] = {2, 10, 20, 0, 0, 0}, tetr[6] = {4, 0, 0, 0, 0, 0},
                   n24[6] = {24, 0, 0, 0, 0, 0}, n20[6] = {20, 0, 0, 0, 0, 0}, n86[6] = {6, 0, 8, 24, 24, 24};
  const int *cnt = nq == 4 ? tetr : (nq == 12 || nq == 32) ? icosa : nq == 20 ? n20 : nq == 24 ? n24 : nq == 86 ? n86 : octa;
  for (int k = 0, jj = 0; k < (nq == 86 ? 6 : 4); k++)
    for (int j = 0; j < cnt[k]; j++, jj++)
      if (jj < nq) w[jj] = ww[icase][k];
  const double p = 1.0 / std::sqrt(2.0), qq = 1.0 / std::sqrt(3.0), r = 1.0 / std::sqrt(11.0), sv = 3.0 / std::sqrt(11.0);
  const double pi = 3.14159265359;
  if (nq == 4) {  // tetrahedron
    for (int j = 0; j < 4; j++) {
      q[j][0] = j < 2 ? qq : -qq;
      q[j][1] = (j == 1 || j == 3) ? -qq : qq;
      q[j][2] = (j == 1 || j == 2) ? -qq : qq;
    }
  } else if (nq == 6 || nq == 18 || nq == 26 || nq == 50) {  // octahedral symmetry
    int ip = 0, lp = 0;
    for (int ii = 0; ii < 2; ii++) {
      const double si = ii == 0 ? 1.0 : -1.0;
      q[ii][0] = si; q[2 + ii][1] = si; q[4 + ii][2] = si;
      if (nq <= 6) continue;
      for (int jj = 0; jj < 2; jj++) {
        const double sj = jj == 0 ? 1.0 : -1.0;
        q[6 + ip][0] = si * p; q[6 + ip][1] = sj * p;
        q[10 + ip][1] = si * p; q[10 + ip][2] = sj * p;
        q[14 + ip][2] = si * p; q[14 + ip][0] = sj * p;
        ip++;
        if (nq <= 18) continue;
        for (int kk = 0; kk < 2; kk++) {
          const double sk = kk == 0 ? 1.0 : -1.0;
          q[18 + lp][0] = si * qq; q[18 + lp][1] = sj * qq; q[18 + lp][2] = sk * qq;
          if (nq > 26) {
            q[26 + lp][0] = si * r; q[26 + lp][1] = sj * r; q[26 + lp][2] = sk * sv;
            q[34 + lp][0] = si * r; q[34 + lp][1] = sj * sv; q[34 + lp][2] = sk * r;
            q[42 + lp][0] = si * sv; q[42 + lp][1] = sj * r; q[42 + lp][2] = sk * r;
          }
          lp++;
        }
      }
    }
  } else if (nq == 12 || nq == 20 || nq == 32) {  // icosahedral symmetry
    q[0][2] = 1.0;
    q[1][2] = -1.0;
    const double fi0 = pi / 5.0, s5 = std::sqrt(5.0), cstha = 1.0 / s5, sntha = 2.0 / s5;
    const double den = std::sqrt(15.0 + 6.0 * s5), csth1 = (2.0 + s5) / den, snth1 = std::sqrt(1.0 - csth1 * csth1);
    const double csth2 = 1.0 / den, snth2 = std::sqrt(1.0 - csth2 * csth2);
    for (int j = 1; j <= 5; j++) {
      const double rk2 = 2.0 * (j - 1), rk21 = rk2 + 1.0;
      const double c2 = std::cos(rk2 * fi0), s2 = std::sin(rk2 * fi0), c21 = std::cos(rk21 * fi0), s21 = std::sin(rk21 * fi0);
      if (nq != 20) {
        q[j + 1][0] = sntha * c2; q[j + 1][1] = sntha * s2; q[j + 1][2] = cstha;
        q[j + 6][0] = sntha * c21; q[j + 6][1] = sntha * s21; q[j + 6][2] = -cstha;
      }
      if (nq > 12) {
        const int k0 = nq == 20 ? 0 : 12;
        const int k1 = j + k0 - 1, k2 = j + k0 + 4, k3 = j + k0 + 9, k4 = j + k0 + 14;
        q[k1][0] = snth1 * c21; q[k1][1] = snth1 * s21; q[k1][2] = csth1;
        q[k2][0] = snth2 * c21; q[k2][1] = snth2 * s21; q[k2][2] = csth2;
        q[k3][0] = snth1 * c2; q[k3][1] = snth1 * s2; q[k3][2] = -csth1;
        q[k4][0] = snth2 * c2; q[k4][1] = snth2 * s2; q[k4][2] = -csth2;
      }
    }
  } else if (nq == 24) {
    int lq = 0;
    double x = .8662468181078, y = .4225186537611, z = .2666354015167;
    for (int l = 0; l < 3; l++) {
      if (l == 1) { const double hold = y; y = x; x = z; z = hold; }
      if (l == 2) { const double hold = z; z = y; y = x; x = hold; }
      const double cp = std::cos(-pi / 2.0), sp = std::sin(-pi / 2.0);
      const double u = cp * x - sp * z, v = y, ww2 = sp * x + cp * z;
      for (int m = 0; m < 4; m++) {
        const double fi = pi * m / 2.0, cf = std::cos(fi), sf = std::sin(fi);
        q[lq][0] = x * cf - y * sf; q[lq][1] = x * sf + y * cf; q[lq][2] = z; lq++;
        q[lq][0] = u * cf - v * sf; q[lq][1] = u * sf + v * cf; q[lq][2] = ww2; lq++;
      }
    }
  } else {  // 86 points
    const double pp = .927330657151, q2 = .374243039090, rl1 = .369602846454, sm1 = .852518311701,
                 rl2 = .694354006603, sm2 = .189063552885;
    int ip = 0, lp = 0;
    for (int ii = 0; ii < 2; ii++) {
      const double si = ii == 0 ? 1.0 : -1.0;
      q[ii][0] = si; q[2 + ii][1] = si; q[4 + ii][2] = si;
      for (int jj = 0; jj < 2; jj++) {
        const double sj = jj == 0 ? 1.0 : -1.0;
        q[62 + ip][0] = si * pp; q[62 + ip][1] = sj * q2;
        q[66 + ip][0] = si * pp; q[66 + ip][2] = sj * q2;
        q[70 + ip][1] = si * pp; q[70 + ip][2] = sj * q2;
        q[74 + ip][0] = si * q2; q[74 + ip][1] = sj * pp;
        q[78 + ip][0] = si * q2; q[78 + ip][2] = sj * pp;
        q[82 + ip][1] = si * q2; q[82 + ip][2] = sj * pp;
        ip++;
        for (int kk = 0; kk < 2; kk++) {
          const double sk = kk == 0 ? 1.0 : -1.0;
          q[6 + lp][0] = si * qq; q[6 + lp][1] = sj * qq; q[6 + lp][2] = sk * qq;
          q[14 + lp][0] = si * rl1; q[14 + lp][1] = sj * rl1; q[14 + lp][2] = sk * sm1;
          q[22 + lp][0] = si * rl1; q[22 + lp][1] = sj * sm1; q[22 + lp][2] = sk * rl1;
          q[30 + lp][0] = si * sm1; q[30 + lp][1] = sj * rl1; q[30 + lp][2] = sk * rl1;
          q[38 + lp][0] = si * rl2; q[38 + lp][1] = sj * rl2; q[38 + lp][2] = sk * sm2;
          q[46 + lp][0] = si * rl2; q[46 + lp][1] = sj * sm2; q[46 + lp][2] = sk * rl2;
          q[54 + lp][0] = si * sm2; q[54 + lp][1] = sj * rl2; q[54 + lp][2] = sk * rl2;
          lp++;
        }
      }
    }
  }
  return nq;
}

// cuspinit4 + cuspexact4 (qmc/fit/cuspinit4.f90:1-60, qmc/fit/cuspexact4.f90:14-40)
static void host_een_cusp(int nordc, int nct, int nt, std::vector<double> &c, std::vector<int> *dependents) {
  if (nordc <= 1) return;
  int neq = 2 * (nordc - 1);
  std::vector<double> d((size_t)neq * nt, 0.0);
  std::vector<int> iwc(neq, 0);
  int i = 0;
  for (int n = 2; n <= nordc; n++)
    for (int k = n - 1; k >= 0; k--) {
      int l_hi = (k == 0) ? n - k - 2 : n - k;
      for (int l = l_hi; l >= 0; l--) {
        int m = (n - k - l) / 2;
        if (2 * m != n - k - l) continue;
        i++;
        if (k == 1 && iwc[n - 2] == 0) iwc[n - 2] = i;
        if (k == 0 && iwc[n + nordc - 3] == 0) iwc[n + nordc - 3] = i;
        int iord = l + 2 * m;
        d[(size_t)(iord - 1) * nt + i - 1] -= 2 * k;
        if (l + m > 0) { iord = nordc - 1 + k + m; d[(size_t)(iord - 1) * nt + i - 1] -= (l + m); }
        if (m > 0) { iord = nordc - 1 + k + l + m; d[(size_t)(iord - 1) * nt + i - 1] -= m; }
      }
    }
  if (dependents) {
    dependents->clear();
    for (int e = 0; e < neq; e++) dependents->push_back(iwc[e] - 1);
  }
  std::vector<int> order;
  for (int e = 1; e <= nordc - 1; e++) order.push_back(e);
  for (int e = nordc + 1; e <= neq; e++) order.push_back(e);
  order.push_back(nordc);
  for (int it = 0; it < nct; it++) {
    double *cc = c.data() + (size_t)it * nt;
    for (int e : order) {
      int jd = iwc[e - 1];
      double sum = 0;
      for (int j = 1; j <= nt; j++)
        if (j != jd) sum += d[(size_t)(e - 1) * nt + j - 1] * cc[j - 1];
      cc[jd - 1] = -sum / d[(size_t)(e - 1) * nt + jd - 1];
    }
  }
}

// Jastrow parameters of the kernels from the context's parameters, e-e-n coefficients with the cusp
// conditions applied (cfull) and the asymptotic values.
template <class T>
static void fill_jaspar(const champ_ctx *c, const std::vector<double> &cfull, const double *asymp_a,
                        const double *asymp_b, JasPar<T> &J) {
  const Params &q = c->par;
  memset(&J, 0, sizeof J);
  J.scalek = (T)q.scalek; J.norda = q.norda; J.nordb = q.nordb; J.nspin2b = q.nspin2b; J.nct = c->nct;
  const int nt = (int)(cfull.size() / std::max(1, c->nct));
  for (int it = 0; it < c->nct; it++) {
    for (int k = 0; k <= q.norda; k++) J.a4[it][k] = (T)q.a4[it * (q.norda + 1) + k];
    for (int k = 0; k < nt; k++) J.c[it][k] = (T)cfull[(size_t)it * nt + k];
    J.asymp_a[it] = (T)asymp_a[it];
  }
  for (int is = 0; is < q.nspin2b; is++)
    for (int k = 0; k <= q.nordb; k++) J.b[is][k] = (T)q.b[is * (q.nordb + 1) + k];
  J.asymp_b[0] = (T)asymp_b[0]; J.asymp_b[1] = (T)asymp_b[1];
}

// e-e-n coefficients with the cusp conditions applied, and the isc=4 asymptotic values
// (set_scale_dist, scale_dist.f90:147-225), from the context's parameters.
static void derive_jastrow(const champ_ctx *c, std::vector<double> &cfull, double *asa, double *asb) {
  const Params &q = c->par;
  const int nt = q.nterms;
  cfull.assign((size_t)c->nct * std::max(nt, 1), 0.0);
  if (nt) std::copy(q.c.begin(), q.c.end(), cfull.begin());
  if (q.een_cusp && nt) host_een_cusp(q.nordc, c->nct, nt, cfull, nullptr);
  if (nt == 0) cfull.assign(c->nct, 0.0);
  const double ar = 1.0 / q.scalek;
  for (int it = 0; it < MAXCT; it++) asa[it] = 0;
  for (int it = 0; it < c->nct; it++) {
    const double *a = q.a4.data() + it * (q.norda + 1);
    double v = a[0] * ar / (1 + a[1] * ar);
    for (int k = 2; k <= q.norda; k++) v += a[k] * std::pow(ar, k);
    asa[it] = v;
  }
  for (int i = 0; i < 2; i++) {
    double ss = (i == 1 && q.nspin2b == 1) ? 0.5 : 1.0;
    int isp = (i == 1) ? q.nspin2b - 1 : 0;
    const double *b = q.b.data() + isp * (q.nordb + 1);
    double v = ss * b[0] * ar / (1 + b[1] * ar);
    for (int k = 2; k <= q.nordb; k++) v += b[k] * std::pow(ar, k);
    asb[i] = v;
  }
}

template <class T>
static int build_sys(champ_ctx *c, const champ_system *d, const std::vector<double> &pcn, const std::vector<double> &cfull,
                     const double *asymp_a, const double *asymp_b, const EcpPar &ecp, double pecent, Sys<T> &s) {
  s.N = c->N; s.nup = c->nup; s.ndn = c->ndn; s.C = c->C; s.nct = c->nct; s.nshell = c->nshell;
  s.nbasis = c->nbasis; s.nmax = c->nmax; s.nloc = c->nloc; s.nordc = c->nordc; s.pecent = pecent;
  s.scalek = d->scalek;
  double *cent = dalloc<double>(c, 3 * c->C);
  int *ctype = dalloc<int>(c, c->C);
  double *zc = dalloc<double>(c, c->C);
  int4 *sh = dalloc<int4>(c, c->nshell);
  int2 *shp = dalloc<int2>(c, c->nshell);
  int *shb0 = dalloc<int>(c, c->nshell);
  int nprim = (int)pcn.size();
  T *pz = dalloc<T>(c, nprim), *pc = dalloc<T>(c, nprim);
  const MultiDet &md = c->md;
  T *cr0 = dalloc<T>(c, (size_t)c->nbasis * std::max(1, md.nocc[0]));
  T *cr1 = dalloc<T>(c, (size_t)c->nbasis * std::max(1, md.nocc[1]));
  T *ct0 = dalloc<T>(c, (size_t)c->nbasis * std::max(1, md.nocc[0]));
  T *ct1 = dalloc<T>(c, (size_t)c->nbasis * std::max(1, md.nocc[1]));
  JasPar<T> *jp = dalloc<JasPar<T>>(c, 1);
  EcpPar *ep = dalloc<EcpPar>(c, 1);
  QuadRule *qr = dalloc<QuadRule>(c, 1);
  if (!qr) return fail(CHAMP_ENOMEM, "device allocation of the quadrature rule failed");
  CK(cudaMemcpy(qr, &c->quad, sizeof(QuadRule), cudaMemcpyHostToDevice));
  s.quad = qr;
  if (!cent || !ctype || !zc || !sh || !shp || !shb0 || !pz || !pc || !cr0 || !cr1 || !ct0 || !ct1 || !jp || !ep)
    return fail(CHAMP_ENOMEM, "device allocation of the system data failed");
  std::vector<double> zcv(c->C);
  for (int i = 0; i < c->C; i++) zcv[i] = d->znuc[d->iwctype[i]];
  std::vector<int4> shv(c->nshell);
  std::vector<int2> shpv(c->nshell);
  // internal basis order: shells in input order, each shell's 2l+1 functions in
  // harmonic-slot order (slot(m) = 0, 2m-1 for m > 0, -2m for m < 0)
  std::vector<int> shb0v(c->nshell, 0), perm_b(c->nbasis, -1);
  {
    int b0 = 0;
    for (int i = 0; i < c->nshell; i++) { shb0v[i] = b0; b0 += 2 * d->shell_l[i] + 1; }
    if (b0 != c->nbasis) return fail(CHAMP_EINVAL, "nbasis differs from the sum over shells of 2l+1");
    for (int b = 0; b < c->nbasis; b++) {
      int m = d->basis_m[b], ish = d->basis_shell[b];
      if (ish < 0 || ish >= c->nshell || m < -d->shell_l[ish] || m > d->shell_l[ish])
        return fail(CHAMP_EINVAL, "basis function with bad shell or m");
      int ib = shb0v[ish] + (m > 0 ? 2 * m - 1 : -2 * m);
      if (perm_b[ib] >= 0) return fail(CHAMP_EINVAL, "two basis functions with the same shell and m");
      perm_b[ib] = b;  // internal index ib holds input basis function b
    }
    c->perm_b = perm_b;
  }
  int p0 = 0;
  for (int i = 0; i < c->nshell; i++) {
    shv[i] = make_int4(d->shell_cent[i], d->shell_n[i], d->shell_l[i], d->shell_kind[i]);
    shpv[i] = make_int2(p0, d->shell_nprim[i]);
    p0 += d->shell_nprim[i];
  }
  std::vector<T> pzv(nprim), pcv(nprim);
  for (int i = 0; i < nprim; i++) { pzv[i] = (T)d->prim_zeta[i]; pcv[i] = (T)pcn[i]; }
  std::vector<T> crv[2];
  for (int sp = 0; sp < 2; sp++) {
    int no = md.nocc[sp];
    crv[sp].assign((size_t)c->nbasis * std::max(1, no), T(0));
    for (int k = 0; k < no; k++) {
      int o = md.occ[sp][k];
      for (int b = 0; b < c->nbasis; b++) crv[sp][(size_t)b * no + k] = (T)d->coef[(size_t)o * c->nbasis + perm_b[b]];
    }
  }
  if constexpr (std::is_same<T, float>::value) {
    c->tc_coef[0] = crv[0];
    c->tc_coef[1] = crv[1];
    c->tc_shl.assign(d->shell_l, d->shell_l + c->nshell);
  }
  // determinant tables
  s.multidet = md.multidet;
  s.ndet = md.ndet;
  s.nomax = c->nomax;
  s.nvmax = std::max(md.nvirt[0], md.nvirt[1]);
  for (int sp = 0; sp < 2; sp++) {
    s.nocc[sp] = md.nocc[sp];
    s.nvirt[sp] = md.nvirt[sp];
    s.ndu[sp] = md.ndu[sp];
    int nd = std::max(1, md.ndu[sp]);
    int *dk = dalloc<int>(c, nd), *dh = dalloc<int>(c, 4 * nd), *dpp = dalloc<int>(c, 4 * nd);
    double *dsg = dalloc<double>(c, nd);
    if (!dk || !dh || !dpp || !dsg) return fail(CHAMP_ENOMEM, "device allocation of determinant tables failed");
    if (md.ndu[sp]) {
      CK(cudaMemcpy(dk, md.dk[sp].data(), sizeof(int) * md.ndu[sp], cudaMemcpyHostToDevice));
      CK(cudaMemcpy(dh, md.dh[sp].data(), sizeof(int) * 4 * md.ndu[sp], cudaMemcpyHostToDevice));
      CK(cudaMemcpy(dpp, md.dp[sp].data(), sizeof(int) * 4 * md.ndu[sp], cudaMemcpyHostToDevice));
      CK(cudaMemcpy(dsg, md.dsg[sp].data(), sizeof(double) * md.ndu[sp], cudaMemcpyHostToDevice));
    }
    s.dk[sp] = dk; s.dh[sp] = dh; s.dpart[sp] = dpp; s.dsg[sp] = dsg;
  }
  {
    int nd = std::max(1, md.ndet);
    int *ciu = dalloc<int>(c, nd), *cid = dalloc<int>(c, nd);
    double *cc = dalloc<double>(c, nd);
    if (!ciu || !cid || !cc) return fail(CHAMP_ENOMEM, "device allocation of determinant tables failed");
    CK(cudaMemcpy(ciu, md.ciu.data(), sizeof(int) * md.ndet, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(cid, md.cid.data(), sizeof(int) * md.ndet, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(cc, md.ccoef.data(), sizeof(double) * md.ndet, cudaMemcpyHostToDevice));
    s.ciu = ciu; s.cid = cid; s.ccoef = cc;
  }
  {
    s.ncfree = c->ncfree;
    // CSF and orbital-rotation parameter tables
    s.norb = d->norb;
    s.ncsf = d->ncsf;
    s.norbp = c->norbp;
    {
      T *ca = dalloc<T>(c, (size_t)c->nbasis * d->norb);
      std::vector<T> cav((size_t)c->nbasis * d->norb);
      for (int m = 0; m < d->norb; m++)
        for (int b = 0; b < c->nbasis; b++) cav[(size_t)b * d->norb + m] = (T)d->coef[(size_t)m * c->nbasis + perm_b[b]];
      std::vector<int> off(d->ncsf + 1, 0), cdet;
      std::vector<double> cd;
      for (int q = 0, t = 0; q < d->ncsf; q++) {
        for (int i = 0; i < d->csf_ndet[q]; i++, t++) { cdet.push_back(d->csf_det[t]); cd.push_back(d->csf_det_coef[t]); }
        off[q + 1] = (int)cdet.size();
      }
      int *co = dalloc<int>(c, off.size()), *cdt = dalloc<int>(c, std::max<size_t>(1, cdet.size()));
      double *cdd = dalloc<double>(c, std::max<size_t>(1, cd.size()));
      int4 *op = dalloc<int4>(c, std::max(1, c->norbp));
      int *rp0 = dalloc<int>(c, d->norb), *rp1 = dalloc<int>(c, d->norb);
      int *oo0 = dalloc<int>(c, std::max(1, md.nocc[0])), *oo1 = dalloc<int>(c, std::max(1, md.nocc[1]));
      if (!ca || !co || !cdt || !cdd || !op || !rp0 || !rp1 || !oo0 || !oo1) return fail(CHAMP_ENOMEM, "device allocation failed");
      CK(cudaMemcpy(ca, cav.data(), sizeof(T) * cav.size(), cudaMemcpyHostToDevice));
      {
        std::vector<double> cdv(cav.begin(), cav.end());
        c->call_d = dalloc<double>(c, cdv.size());
        if (!c->call_d) return fail(CHAMP_ENOMEM, "device allocation failed");
        CK(cudaMemcpy(c->call_d, cdv.data(), sizeof(double) * cdv.size(), cudaMemcpyHostToDevice));
      }
      CK(cudaMemcpy(co, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
      if (!cdet.empty()) {
        CK(cudaMemcpy(cdt, cdet.data(), sizeof(int) * cdet.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(cdd, cd.data(), sizeof(double) * cd.size(), cudaMemcpyHostToDevice));
      }
      if (c->norbp) CK(cudaMemcpy(op, c->orbp.data(), sizeof(int4) * c->norbp, cudaMemcpyHostToDevice));
      int *rp[2] = {rp0, rp1}, *oo[2] = {oo0, oo1};
      for (int sp = 0; sp < 2; sp++) {
        std::vector<int> rpv(d->norb, -1);
        for (int k = 0; k < md.nocc[sp]; k++) rpv[md.occ[sp][k]] = k;
        CK(cudaMemcpy(rp[sp], rpv.data(), sizeof(int) * d->norb, cudaMemcpyHostToDevice));
        if (md.nocc[sp]) CK(cudaMemcpy(oo[sp], md.occ[sp].data(), sizeof(int) * md.nocc[sp], cudaMemcpyHostToDevice));
        s.refpos[sp] = rp[sp];
        s.occo[sp] = oo[sp];
      }
      s.call = ca; s.csf_off = co; s.csf_det = cdt; s.csf_cd = cdd; s.orbp = op;
    }
    double *cp = dalloc<double>(c, std::max<size_t>(1, c->cproj.size()));
    if (!cp) return fail(CHAMP_ENOMEM, "device allocation failed");
    if (!c->cproj.empty()) CK(cudaMemcpy(cp, c->cproj.data(), sizeof(double) * c->cproj.size(), cudaMemcpyHostToDevice));
    s.cproj = cp;
  }
  JasPar<T> J;
  fill_jaspar<T>(c, cfull, asymp_a, asymp_b, J);
  std::vector<int> ctv(d->iwctype, d->iwctype + c->C);
  CK(cudaMemcpy(cent, d->cent, sizeof(double) * 3 * c->C, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctype, ctv.data(), sizeof(int) * c->C, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(zc, zcv.data(), sizeof(double) * c->C, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sh, shv.data(), sizeof(int4) * c->nshell, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(shp, shpv.data(), sizeof(int2) * c->nshell, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(shb0, shb0v.data(), sizeof(int) * c->nshell, cudaMemcpyHostToDevice));
  {
    // shells grouped by centre: first shell of each centre and the largest group
    std::vector<int> cs0(c->C + 1, 0);
    bool grouped = true;
    for (int i = 1; i < c->nshell; i++)
      if (d->shell_cent[i] < d->shell_cent[i - 1]) grouped = false;
    int nshc = 0;
    if (grouped) {
      for (int cc = 0, i = 0; cc <= c->C; cc++) {
        while (i < c->nshell && d->shell_cent[i] < cc) i++;
        cs0[cc] = i;
      }
      cs0[c->C] = c->nshell;
      for (int cc = 0; cc < c->C; cc++) nshc = std::max(nshc, cs0[cc + 1] - cs0[cc]);
    }
    int *cs = dalloc<int>(c, c->C + 1);
    if (!cs) return fail(CHAMP_ENOMEM, "device allocation failed");
    CK(cudaMemcpy(cs, cs0.data(), sizeof(int) * (c->C + 1), cudaMemcpyHostToDevice));
    s.cshell0 = cs;
    s.nshc = grouped ? nshc : 0;
  }
  CK(cudaMemcpy(pz, pzv.data(), sizeof(T) * nprim, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(pc, pcv.data(), sizeof(T) * nprim, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(cr0, crv[0].data(), sizeof(T) * crv[0].size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(cr1, crv[1].data(), sizeof(T) * crv[1].size(), cudaMemcpyHostToDevice));
  for (int sp = 0; sp < 2; sp++) {
    int no = std::max(1, md.nocc[sp]);
    std::vector<T> tv((size_t)c->nbasis * no);
    for (int b = 0; b < c->nbasis; b++)
      for (int k = 0; k < no; k++) tv[(size_t)k * c->nbasis + b] = crv[sp][(size_t)b * no + k];
    CK(cudaMemcpy(sp ? ct1 : ct0, tv.data(), sizeof(T) * tv.size(), cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(jp, &J, sizeof J, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ep, &ecp, sizeof ecp, cudaMemcpyHostToDevice));
  s.cent = cent; s.ctype = ctype; s.zc = zc; s.shell = sh; s.shprim = shp; s.shb0 = shb0;
  s.pz = pz; s.pc = pc; s.cocc[0] = cr0; s.cocc[1] = cr1; s.coccT[0] = ct0; s.coccT[1] = ct1; s.jas = jp; s.ecp = ep;
  {
    // numerical radial tables (kind-2 shells)
    const size_t nt = c->rad_tab.size(), ny = c->rad_y.size();
    int *shr = dalloc<int>(c, c->nshell);
    int4 *rt = dalloc<int4>(c, std::max<size_t>(nt, 1));
    double *rp = dalloc<double>(c, std::max<size_t>(10 * nt, 1));
    T *ry = dalloc<T>(c, std::max<size_t>(ny, 1)), *ry2 = dalloc<T>(c, std::max<size_t>(ny, 1));
    if (!shr || !rt || !rp || !ry || !ry2) return fail(CHAMP_ENOMEM, "device allocation of the radial tables failed");
    CK(cudaMemcpy(shr, c->rad_shell.data(), sizeof(int) * c->nshell, cudaMemcpyHostToDevice));
    if (nt) {
      std::vector<T> yv(c->rad_y.begin(), c->rad_y.end()), y2v(c->rad_y2.begin(), c->rad_y2.end());
      CK(cudaMemcpy(rt, c->rad_tab.data(), sizeof(int4) * nt, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(rp, c->rad_par.data(), sizeof(double) * 10 * nt, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(ry, yv.data(), sizeof(T) * ny, cudaMemcpyHostToDevice));
      CK(cudaMemcpy(ry2, y2v.data(), sizeof(T) * ny, cudaMemcpyHostToDevice));
    }
    s.shrad = shr; s.rtab = rt; s.rpar = rp; s.ry = ry; s.ry2 = ry2;
  }
  return CHAMP_OK;
}

template <class T>
static int build_state(champ_ctx *c, State<T> &st) {
  size_t W = c->wmax, N = c->N;
  st.W = 0;
  st.astride = c->nup * c->nup + c->ndn * c->ndn;
  const MultiDet &md = c->md;
  st.tvstride = std::max(1, c->nup * md.nvirt[0] + c->ndn * md.nvirt[1]);
  st.gstride = md.multidet ? md.nocc[0] * c->nup + md.nocc[1] * c->ndn : 1;
  st.wstride = md.multidet ? 2 * (md.ndu[0] + md.ndu[1]) : 1;
  st.x = dalloc<double>(c, W * N * 3);
  st.ainv = dalloc<double>(c, W * st.astride);
  st.fso = dalloc<T>(c, W * N * N);
  st.ren = dalloc<T>(c, W * N * c->C * 2);
  st.zq = dalloc<T>(c, W * N * ZQ);
  st.fsum = dalloc<double>(c, W); st.lnd = dalloc<double>(c, W); st.sgn = dalloc<double>(c, W);
  st.status = dalloc<uint32_t>(c, W);
  st.pf = dalloc<T>(c, W * N);
  st.pa = dalloc<double>(c, W * c->nomax);
  st.pdj = dalloc<double>(c, W); st.prho = dalloc<double>(c, W); st.pxn = dalloc<double>(c, 3 * W);
  st.piel = dalloc<int>(c, W);
  st.orb5 = dalloc<T>(c, W * N * 5 * c->nomax);
  st.tv = dalloc<double>(c, W * st.tvstride);
  st.gam = dalloc<double>(c, W * st.gstride);
  st.ymd = dalloc<double>(c, W * st.tvstride);
  st.wdet = dalloc<double>(c, W * st.wstride);
  if (!st.tv || !st.gam || !st.ymd || !st.wdet) return fail(CHAMP_ENOMEM, "device allocation of the walker state failed");
  st.gproj = c->nloc > 0 ? dalloc<T>(c, W * N * c->nbasis) : nullptr;
  st.nlt = c->nloc > 0 ? dalloc<double>(c, W * N * c->C * NLT) : nullptr;
  st.o_lnpsi = dalloc<double>(c, W); st.o_sign = dalloc<double>(c, W); st.o_psij = dalloc<double>(c, W);
  st.o_vel = dalloc<double>(c, W * N * 3); st.o_divv = dalloc<double>(c, W * N); st.o_d2 = dalloc<double>(c, W);
  st.o_pe = dalloc<double>(c, W); st.o_peee = dalloc<double>(c, W); st.o_penl = dalloc<double>(c, W);
  st.o_eloc = dalloc<double>(c, W);
  st.s_esum = dalloc<double>(c, W); st.s_e2sum = dalloc<double>(c, W); st.s_acc = dalloc<double>(c, W);
  st.s_elast = dalloc<double>(c, W);
  if (!st.x || !st.ainv || !st.fso || !st.ren || !st.zq || !st.orb5 || !st.s_elast || (c->nloc > 0 && (!st.gproj || !st.nlt)))
    return fail(CHAMP_ENOMEM, "device allocation of the walker state failed");
  return CHAMP_OK;
}

// The staged evaluation of an FP64 state in HBM (elstage.cuh): per-warp shared memory and warps
// per block of its parts (up to 4 warps, at most 96 KB a block), and its per-walker scratch.
static int setup_el_staged(champ_ctx *c) {
  const size_t bytes[3] = {el_jas_bytes(c->N), el_orb_bytes<double>(c->nbasis),
                           el_fin_bytes<double>(c->N, el_fin_scratch(c->N, c->C))};
  for (int k = 0; k < 3; k++) {
    int wpb = 4;
    while (wpb > 1 && bytes[k] * wpb > 96 * 1024) wpb >>= 1;
    if (bytes[k] * wpb > 200 * 1024) return CHAMP_OK;  // too large: the single-kernel evaluation
    c->el_wpb[k] = wpb;
    c->el_smem[k] = bytes[k] * wpb;
  }
  c->el_nscr = el_fin_scratch(c->N, c->C);
  // the orbital part's warps share the coefficient stream when a block's items are always of one
  // spin (N and nup multiples of its warps) and the orbitals take warp_orbitals' lane mapping (> 16)
  {
    const int wpb = c->el_wpb[1], n0 = c->sd.nocc[0], n1 = c->sd.nocc[1];
    if (wpb == 4 && c->N % wpb == 0 && c->nup % wpb == 0 && n0 > 16 && n1 > 16) {
      const size_t st_bytes = sizeof(double) * EL_ORB_STG * EL_ORB_KB * (size_t)std::max(n0, n1);
      const size_t off = align16(c->el_smem[1]);
      if (off + st_bytes <= 200 * 1024) {
        c->orb_stage = off;
        c->el_smem[1] = off + st_bytes;
        c->orb_coop_ok = c->orb_coop = 1;
      }
    }
  }
  const size_t W = c->wmax, N = c->N;
  State<double> &st = c->std_;
  st.el_vj = dalloc<double>(c, W * 4 * N);
  st.el_sc = dalloc<double>(c, W * 8);
  st.el_rt = dalloc<double>(c, W * 2 * c->C * N);
  if (!st.el_vj || !st.el_sc || !st.el_rt) return fail(CHAMP_ENOMEM, "allocation of the staged-evaluation scratch failed");
  c->el_staged = 1;
  return CHAMP_OK;
}

// Delayed inverse updates of the moves (struct Delay) for a walker state in HBM: room for up to
// DELAY_MAX pending terms per spin; option "delay_rank" picks how many are folded in at a time.
static constexpr int DELAY_MAX = 32, DELAY_DEFAULT = 4;
static int setup_delay(champ_ctx *c) {
  State<double> &st = c->std_;
  st.dly = dalloc<double>(c, (size_t)c->wmax * 4 * DELAY_MAX * c->nmax);
  if (!st.dly) return fail(CHAMP_ENOMEM, "allocation of the delayed-update buffer failed");
  st.dlk = DELAY_DEFAULT;
  st.dlk_max = DELAY_MAX;
  return CHAMP_OK;
}

// Mixed precision: the FP32 state of the single-electron moves shares every FP64 buffer with the
// FP64 state (positions, inverses, log-det, determinant tables, outputs, statistics) and owns
// only the FP32 Jastrow pair table, distances and power sums, which every FP64 full evaluation
// refreshes (State::m_fso, m_ren, m_zq).
static void link_move_state(State<double> &d, State<float> &f) {
  float *fso = f.fso, *ren = f.ren, *zq = f.zq, *pf = f.pf, *rtd = f.rtd;
  f.W = d.W;
  f.x = d.x; f.ainv = d.ainv; f.fsum = d.fsum; f.lnd = d.lnd; f.sgn = d.sgn; f.status = d.status;
  f.pa = d.pa; f.pdj = d.pdj; f.prho = d.prho; f.pxn = d.pxn; f.piel = d.piel;
  f.orb5 = nullptr; f.gproj = nullptr; f.nlt = nullptr;
  f.tv = d.tv; f.gam = d.gam; f.ymd = d.ymd; f.wdet = d.wdet;
  f.astride = d.astride; f.tvstride = d.tvstride; f.gstride = d.gstride; f.wstride = d.wstride;
  f.o_lnpsi = d.o_lnpsi; f.o_sign = d.o_sign; f.o_psij = d.o_psij; f.o_vel = d.o_vel; f.o_divv = d.o_divv;
  f.o_d2 = d.o_d2; f.o_pe = d.o_pe; f.o_peee = d.o_peee; f.o_penl = d.o_penl; f.o_eloc = d.o_eloc;
  f.s_esum = d.s_esum; f.s_e2sum = d.s_e2sum; f.s_acc = d.s_acc; f.s_elast = d.s_elast;
  f.fso = fso; f.ren = ren; f.zq = zq; f.pf = pf; f.rtd = rtd;
  f.m_fso = f.m_ren = f.m_zq = nullptr;
  d.m_fso = fso; d.m_ren = ren; d.m_zq = zq;
  f.m_rtd = nullptr;
  d.m_rtd = f.rtd;
  d.rtd = nullptr;
  f.dly = d.dly;
  f.dlk = d.dlk;
  f.dlk_max = d.dlk_max;
}

static int build_move_state(champ_ctx *c, State<double> &d, State<float> &f) {
  size_t W = c->wmax, N = c->N;
  memset(&f, 0, sizeof f);
  f.fso = dalloc<float>(c, W * N * N);
  f.ren = dalloc<float>(c, W * N * c->C * 2);
  f.zq = dalloc<float>(c, W * N * ZQ);
  f.pf = dalloc<float>(c, W * N);
  if (!f.fso || !f.ren || !f.zq || !f.pf) return fail(CHAMP_ENOMEM, "device allocation of the FP32 move tables failed");
  f.rtd = nullptr;
  if (!c->kd.lay.resident) {  // walker state in HBM: the transposed distances of the pair loads
    f.rtd = dalloc<float>(c, W * N * c->C);
    if (!f.rtd) return fail(CHAMP_ENOMEM, "device allocation of the FP32 move tables failed");
  }
  link_move_state(d, f);
  return CHAMP_OK;
}

// Phase timing: events recorded on the context's stream around a launch when "phase_timing" is on.
enum { PH_SWEEP = 0, PH_MOVES = 1, PH_EVAL = 2, PH_TC = 3, PH_N = 4 };
static int ev_mark(champ_ctx *c, int phase, bool start) {
  if (!c->ptime) return CHAMP_OK;
  size_t i;
  if (start) {
    i = c->ev_use.empty() ? 0 : (size_t)c->ev_use.back().second + 2;
    while (c->ev_pool.size() < i + 2) {
      cudaEvent_t e;
      CK(cudaEventCreate(&e));
      c->ev_pool.push_back((void *)e);
    }
    c->ev_use.push_back({phase, (int)i});
  } else {
    i = (size_t)c->ev_use.back().second + 1;
  }
  CK(cudaEventRecord((cudaEvent_t)c->ev_pool[i], c->stream));
  return CHAMP_OK;
}

static int launch(champ_ctx *c, Op op, const OpArgs &a = OpArgs()) {
  if (op == Op::Vmc && a.phase < 0 && c->prec == CHAMP_PREC_FP64 && c->el_staged) {
    // moves, then the staged E_L, per sweep (the E_L re-inverts the Slater matrices every sweep)
    const State<double> &st = c->std_;
    CK(cudaMemsetAsync(st.s_esum, 0, sizeof(double) * c->W, c->stream));
    CK(cudaMemsetAsync(st.s_e2sum, 0, sizeof(double) * c->W, c->stream));
    CK(cudaMemsetAsync(st.s_acc, 0, sizeof(double) * c->W, c->stream));
    OpArgs b = a;
    b.nsweep = 1;
    for (int isw = 0; isw < a.nsweep; isw++) {
      b.sweep0 = a.sweep0 + (uint64_t)isw;
      b.phase = 1;
      int rc = ev_mark(c, PH_MOVES, true);
      if (!rc) rc = launch_f64(c, op, b);
      if (!rc) rc = ev_mark(c, PH_MOVES, false);
      if (rc) return rc;
      b.phase = 3;
      rc = ev_mark(c, PH_EVAL, true);
      if (!rc) rc = launch_f64(c, op, b);
      if (!rc) rc = ev_mark(c, PH_EVAL, false);
      if (rc) return rc;
    }
    return CHAMP_OK;
  }
  if (op == Op::Vmc && a.phase < 0 && c->prec != CHAMP_PREC_MIXED && !c->tc_on) {
    // the fused sweep kernel: moves and E_L in one launch
    int rc = ev_mark(c, PH_SWEEP, true);
    if (!rc) rc = c->prec == CHAMP_PREC_FP64 ? launch_f64(c, op, a) : launch_f32(c, op, a);
    if (!rc) rc = ev_mark(c, PH_SWEEP, false);
    return rc;
  }
  if (c->prec == CHAMP_PREC_FP64) return launch_f64(c, op, a);
  if (c->prec == CHAMP_PREC_FP32) return launch_f32(c, op, a);
  // mixed precision: moves on the FP32 instantiation, full evaluations on the FP64 one
  switch (op) {
  case Op::Eval:
  case Op::EvalOut:
  case Op::PGrad:
    return launch_f64(c, op, a);
  case Op::Propose:
  case Op::ProposeGrad:
  case Op::Accept:
  case Op::Tmove:  // T-moves, like the other moves, on the FP32 tables
  case Op::DmcCopy:
  case Op::PGradBwd:  // the parameter derivatives' reverse sweep in FP32 (E_L stays FP64)
    return launch_f32(c, op, a);
  case Op::DmcMove: {
    OpArgs b = a;
    b.phase = 1;
    int rc = launch_f32(c, op, b);
    if (rc) return rc;
    b.phase = 2;
    return launch_f64(c, op, b);
  }
  case Op::Vmc: {
    if (a.phase >= 0) return fail(CHAMP_EINVAL, "internal: explicit VMC phase on a mixed context");
    const State<double> &st = c->std_;
    CK(cudaMemsetAsync(st.s_esum, 0, sizeof(double) * c->W, c->stream));
    CK(cudaMemsetAsync(st.s_e2sum, 0, sizeof(double) * c->W, c->stream));
    CK(cudaMemsetAsync(st.s_acc, 0, sizeof(double) * c->W, c->stream));
    OpArgs b = a;
    b.nsweep = 1;
    for (int isw = 0; isw < a.nsweep; isw++) {
      b.sweep0 = a.sweep0 + (uint64_t)isw;
      b.phase = 1;  // the sweep's moves, FP32
      int rc = ev_mark(c, PH_MOVES, true);
      if (!rc) rc = launch_f32(c, op, b);
      if (!rc) rc = ev_mark(c, PH_MOVES, false);
      if (rc) return rc;
      b.phase = 3;  // its E_L, FP64 from the positions
      rc = ev_mark(c, PH_EVAL, true);
      if (!rc) rc = launch_f64(c, op, b);
      if (!rc) rc = ev_mark(c, PH_EVAL, false);
      if (rc) return rc;
    }
    return CHAMP_OK;
  }
  }
  return fail(CHAMP_EINVAL, "internal: unknown operation");
}
// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
template <class T>
static int copy_eval_out(champ_ctx *c, const champ_eval_out *o) {
  State<T> &st = stof<T>(c);
  size_t W = c->W, N = c->N;
  struct { double *h; double *d; size_t n; } m[] = {
      {o->lnpsi, st.o_lnpsi, W}, {o->sign, st.o_sign, W}, {o->psij, st.o_psij, W}, {o->velocity, st.o_vel, W * N * 3},
      {o->div_v, st.o_divv, W * N}, {o->d2lnpsi, st.o_d2, W}, {o->pe, st.o_pe, W}, {o->pe_ee, st.o_peee, W},
      {o->pe_nonloc, st.o_penl, W}, {o->energy, st.o_eloc, W}};
  for (auto &e : m)
    if (e.h) CK(cudaMemcpyAsync(e.h, e.d, sizeof(double) * e.n, cudaMemcpyDeviceToHost, c->stream));
  return CHAMP_OK;
}

template <class T>
static int copy_stats(champ_ctx *c, const champ_vmc_stats *s) {
  State<T> &st = stof<T>(c);
  size_t W = c->W;
  if (s->esum) CK(cudaMemcpyAsync(s->esum, st.s_esum, sizeof(double) * W, cudaMemcpyDeviceToHost, c->stream));
  if (s->e2sum) CK(cudaMemcpyAsync(s->e2sum, st.s_e2sum, sizeof(double) * W, cudaMemcpyDeviceToHost, c->stream));
  if (s->accept) CK(cudaMemcpyAsync(s->accept, st.s_acc, sizeof(double) * W, cudaMemcpyDeviceToHost, c->stream));
  if (s->elast) CK(cudaMemcpyAsync(s->elast, st.s_elast, sizeof(double) * W, cudaMemcpyDeviceToHost, c->stream));
  return CHAMP_OK;
}

// ---- DMC
template <class T>
static int alloc_state_copy(champ_ctx *c, const State<T> &a, State<T> &b) {
  b = a;  // strides, scratch and output buffers are shared
  size_t W = c->wmax, N = c->N;
  b.x = dalloc<double>(c, W * N * 3);
  b.ainv = dalloc<double>(c, W * a.astride);
  b.fso = dalloc<T>(c, W * N * N);
  b.ren = dalloc<T>(c, W * N * c->C * 2);
  b.zq = dalloc<T>(c, W * N * ZQ);
  b.tv = dalloc<double>(c, W * a.tvstride);
  b.gam = dalloc<double>(c, W * a.gstride);
  b.fsum = dalloc<double>(c, W);
  b.lnd = dalloc<double>(c, W);
  b.sgn = dalloc<double>(c, W);
  if (!b.x || !b.ainv || !b.fso || !b.ren || !b.zq || !b.tv || !b.gam || !b.fsum || !b.lnd || !b.sgn)
    return fail(CHAMP_ENOMEM, "allocation of the DMC state buffer failed");
  if (a.rtd) {
    b.rtd = dalloc<T>(c, W * N * c->C);
    if (!b.rtd) return fail(CHAMP_ENOMEM, "allocation of the DMC state buffer failed");
  }
  return CHAMP_OK;
}

static const int DMC_STAT_CAP = 1 << 16;

// ---------------------------------------------------------------------------------------
// Evaluation without allocation.  Some callers cannot call cudaMalloc: host codes whose
// device memory is entirely owned by their own pool allocator, or that must not pay for an
// allocation (and its implicit synchronisation) inside a time-critical loop.  For them
// champ_eval_energy_noalloc takes the walkers and the output as device buffers the caller
// owns, and keeps every per-walker intermediate in the fixed array below.  The array is a
// file-scope device variable: every GPU that loads this library holds it until the process
// exits, and every call shares it.
// ---------------------------------------------------------------------------------------
static constexpr size_t NOALLOC_BYTES = (size_t)16 << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[256];  // device address of g_noalloc_scratch, per device ordinal

// Device address of the scratch array for the current device, looked up once per device.
static int noalloc_scratch(void **out) {
  int dev = -1;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) return fail(CHAMP_ECUDA, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(CHAMP_ECUDA, std::string("cudaGetSymbolAddress of the scratch array: ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return CHAMP_OK;
}

// Carves a State<T> for nw walkers out of the scratch array (256-byte aligned pieces).
// Returns the bytes used, or 0 if they do not fit.
template <class T>
static size_t noalloc_carve(const champ_ctx *c, const State<T> &ref, int nw, char *base, double *eloc, State<T> &st) {
  size_t o = 0;
  auto take = [&](size_t bytes) -> char * {
    char *p = base + o;
    o += (bytes + 255) & ~(size_t)255;
    return p;
  };
  const size_t W = nw, N = c->N, C = c->C, B = c->nbasis, nm = c->nomax;
  st = ref;
  st.x = (double *)take(sizeof(double) * W * N * 3);
  st.ainv = (double *)take(sizeof(double) * W * ref.astride);
  st.fso = (T *)take(sizeof(T) * W * N * N);
  st.ren = (T *)take(sizeof(T) * W * N * C * 2);
  st.zq = (T *)take(sizeof(T) * W * N * ZQ);
  st.fsum = (double *)take(sizeof(double) * W);
  st.lnd = (double *)take(sizeof(double) * W);
  st.sgn = (double *)take(sizeof(double) * W);
  st.status = (uint32_t *)take(sizeof(uint32_t) * W);
  st.pf = (T *)take(sizeof(T) * W * N);
  st.pa = (double *)take(sizeof(double) * W * nm);
  st.pdj = (double *)take(sizeof(double) * W);
  st.prho = (double *)take(sizeof(double) * W);
  st.pxn = (double *)take(sizeof(double) * W * 3);
  st.piel = (int *)take(sizeof(int) * W);
  st.orb5 = (T *)take(sizeof(T) * W * N * 5 * nm);
  st.gproj = c->nloc > 0 ? (T *)take(sizeof(T) * W * N * B) : nullptr;
  st.nlt = c->nloc > 0 ? (double *)take(sizeof(double) * W * N * C * NLT) : nullptr;
  st.tv = (double *)take(sizeof(double) * W * ref.tvstride);
  st.gam = (double *)take(sizeof(double) * W * ref.gstride);
  st.ymd = (double *)take(sizeof(double) * W * ref.tvstride);
  st.wdet = (double *)take(sizeof(double) * W * ref.wstride);
  st.o_lnpsi = (double *)take(sizeof(double) * W);
  st.o_sign = (double *)take(sizeof(double) * W);
  st.o_psij = (double *)take(sizeof(double) * W);
  st.o_vel = (double *)take(sizeof(double) * W * N * 3);
  st.o_divv = (double *)take(sizeof(double) * W * N);
  st.o_d2 = (double *)take(sizeof(double) * W);
  st.o_pe = (double *)take(sizeof(double) * W);
  st.o_peee = (double *)take(sizeof(double) * W);
  st.o_penl = (double *)take(sizeof(double) * W);
  st.o_eloc = eloc;  // written straight into the caller's buffer
  st.m_fso = st.m_ren = st.m_zq = nullptr;  // the context's own move tables stay untouched
  st.m_rtd = nullptr;
  st.rtd = nullptr;
  st.dly = nullptr;
  st.el_vj = st.el_sc = nullptr;
  st.el_rt = nullptr;
  return o <= NOALLOC_BYTES ? o : 0;
}

template <class T>
static int eval_noalloc_t(champ_ctx *c, const State<T> &ref, int32_t nw, const double *x, double *eloc) {
  void *scr = nullptr;
  int rc = noalloc_scratch(&scr);
  if (rc) return rc;
  State<T> st;
  if (!noalloc_carve<T>(c, ref, nw, (char *)scr, eloc, st)) {
    State<T> one;
    size_t per = noalloc_carve<T>(c, ref, 1, (char *)scr, eloc, one);
    return fail(CHAMP_EINVAL, "champ_eval_energy_noalloc: " + std::to_string(nw) + " walkers need more than the " +
                                  std::to_string(NOALLOC_BYTES >> 20) + " MiB scratch array (at most " +
                                  std::to_string(per ? NOALLOC_BYTES / per : 0) + " walkers of this system)");
  }
  // the kernel writes the walkers back after its shared-memory pass, so it works on a copy
  CK(cudaMemcpyAsync(st.x, x, sizeof(double) * (size_t)nw * c->N * 3, cudaMemcpyDeviceToDevice, c->stream));
  OpArgs a;
  a.st_override = &st;
  a.nw_override = nw;
  rc = launch(c, Op::EvalOut, a);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
}

// Tensor-core orbital contraction: padded sizes and split coefficients.  Fused (orbfused.cuh):
// basis functions formed in shared memory, K in a padded order in which no shell straddles a
// 16-function block; usable when 5 channels x the padded orbital count fit the 512 TMEM columns.
// Otherwise basis rows in HBM (k_basis_rows) and the streamed product (k_orb_tc), when the rows
// fit in memory.  Left off (CUDA-core contraction) where neither applies.
static int tc_alloc_rows(champ_ctx *c) {
  if (c->tc_phi) return CHAMP_OK;
  c->tc_phi = dalloc<float>(c, (size_t)c->wmax * c->N * 5 * c->tc_Kp);
  if (!c->tc_phi) {
    cudaGetLastError();
    return fail(CHAMP_ENOMEM, "no room for the basis rows of the unfused tensor-core contraction");
  }
  return CHAMP_OK;
}

// The occupied orbitals' coefficients split for the 3-term TF32 products: x = hi + lo with hi and
// lo rounded to TF32, in the layouts of the two tensor-core contractions (K padded to BK; and the
// fused kernel's blocks of whole shells).
static int tc_upload_split(champ_ctx *c) {
  const int B = c->nbasis, Kp = c->tc_Kp, Kq = c->tc_kq;
  for (int sp = 0; sp < 2; sp++) {
    const int no = c->md.nocc[sp], Np = c->tc_Np[sp];
    if (no == 0 || (sp ? c->ndn : c->nup) == 0 || !c->tc_b[sp][0]) continue;
    std::vector<float> hi((size_t)Np * Kp, 0.f), lo((size_t)Np * Kp, 0.f);
    std::vector<float> fhi((size_t)Np * Kq, 0.f), flo((size_t)Np * Kq, 0.f);
    for (int m = 0; m < no; m++) {
      for (int b = 0; b < B; b++) {
        float v = c->tc_coef[sp][(size_t)b * no + m], h = orbtc::tf32_hi(v);
        hi[(size_t)m * Kp + b] = h;
        lo[(size_t)m * Kp + b] = orbtc::tf32_lo(v, h);
      }
      for (int i = 0; i < c->nshell; i++)
        for (int sl = 0; sl < 2 * c->tc_shl[i] + 1; sl++) {
          float v = c->tc_coef[sp][(size_t)(c->tc_b0_h[i] + sl) * no + m], h = orbtc::tf32_hi(v);
          fhi[(size_t)m * Kq + c->tc_kpos_h[i] + sl] = h;
          flo[(size_t)m * Kq + c->tc_kpos_h[i] + sl] = orbtc::tf32_lo(v, h);
        }
    }
    CK(cudaMemcpy(c->tc_b[sp][0], hi.data(), sizeof(float) * hi.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->tc_b[sp][1], lo.data(), sizeof(float) * lo.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->tc_bf[sp][0], fhi.data(), sizeof(float) * fhi.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->tc_bf[sp][1], flo.data(), sizeof(float) * flo.size(), cudaMemcpyHostToDevice));
  }
  return CHAMP_OK;
}

static int tc_setup(champ_ctx *c) {
  c->tc_on = c->tc_ok = c->tc_fused_ok = c->tc_mode = 0;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev));
  if (c->prec != CHAMP_PREC_FP32 || c->kf.lay.resident) return CHAMP_OK;
  if (std::max(c->md.nocc[0], c->md.nocc[1]) < 16) return CHAMP_OK;
  const int B = c->nbasis, Kp = (B + orbtc::BK - 1) / orbtc::BK * orbtc::BK;
  c->tc_Kp = Kp;
  // padded order for the fused kernel: kpos[shell], blocks of BKF functions holding whole shells
  const int BKF = orbf::BKF;
  std::vector<int> kpos(c->nshell), b0(c->nshell);
  int pos = 0, bb = 0;
  for (int i = 0; i < c->nshell; i++) {
    const int nf = 2 * c->tc_shl[i] + 1;
    if (pos % BKF + nf > BKF) pos = (pos + BKF - 1) / BKF * BKF;
    kpos[i] = pos;
    b0[i] = bb;
    pos += nf;
    bb += nf;
  }
  const int Kq = (pos + BKF - 1) / BKF * BKF, nkb = Kq / BKF;
  std::vector<int> blk(nkb + 1, c->nshell);
  for (int kb = 0, i = 0; kb <= nkb; kb++) {
    while (i < c->nshell && kpos[i] < kb * BKF) i++;
    blk[kb] = i;
  }
  bool fused = true;
  for (int sp = 0; sp < 2; sp++) {
    const int no = c->md.nocc[sp];
    if (no == 0 || (sp ? c->ndn : c->nup) == 0) continue;
    const int Np = (std::max(no, 16) + 15) / 16 * 16;
    int nc = 32;
    while (nc < Np) nc <<= 1;
    c->tc_Np[sp] = Np;
    c->tc_ncols[sp] = nc;
    int fc = 32;
    while (fc < 5 * Np) fc <<= 1;
    c->tc_fcols[sp] = fc;
    if (5 * Np > 512) fused = false;
    c->tc_b[sp][0] = dalloc<float>(c, (size_t)Np * Kp);
    c->tc_b[sp][1] = dalloc<float>(c, (size_t)Np * Kp);
    c->tc_bf[sp][0] = dalloc<float>(c, (size_t)Np * Kq);
    c->tc_bf[sp][1] = dalloc<float>(c, (size_t)Np * Kq);
    if (!c->tc_b[sp][0] || !c->tc_b[sp][1] || !c->tc_bf[sp][0] || !c->tc_bf[sp][1])
      return fail(CHAMP_ENOMEM, "device allocation failed");
  }
  c->tc_kpos_h = kpos;
  c->tc_b0_h = b0;
  c->tc_kq = Kq;
  {
    int rc = tc_upload_split(c);
    if (rc) return rc;
  }
  c->tc_nkb = nkb;
  c->tc_blk_sh = dalloc<int>(c, nkb + 1);
  c->tc_kpos = dalloc<int>(c, c->nshell);
  c->tc_err = dalloc<int>(c, 1);
  if (!c->tc_blk_sh || !c->tc_kpos || !c->tc_err) return fail(CHAMP_ENOMEM, "device allocation failed");
  CK(cudaMemcpy(c->tc_blk_sh, blk.data(), sizeof(int) * (nkb + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->tc_kpos, kpos.data(), sizeof(int) * c->nshell, cudaMemcpyHostToDevice));
  c->tc_fused_ok = fused ? 1 : 0;
  if (fused) {
    c->tc_ok = c->tc_on = 1;
    c->tc_mode = 1;
    return CHAMP_OK;
  }
  if (tc_alloc_rows(c) != CHAMP_OK) return CHAMP_OK;  // the CUDA-core contraction stays in use
  c->tc_ok = c->tc_on = 1;
  c->tc_mode = 2;
  return CHAMP_OK;
}

// One DMC step (rundmc_mod.f90:17-422): drift-diffusion moves and E_L, weight sums, copy counts,
// their prefix sum, the branching copy into the other state buffer, population and E_T update;
// then the buffers swap roles.  Reads its step number from the device counter.
static int dmc_one_step(champ_ctx *c) {
  int rc;
  if (c->dpar.tmove && c->nloc > 0) {  // T-moves first (rundmc_mod.f90:137)
    OpArgs t;
    t.tau = c->dpar.tau;
    t.variant = c->dpar.tmove;
    t.seed = c->dpar.seed;
    t.dmc = true;
    rc = launch(c, Op::Tmove, t);
    if (rc) return rc;
  }
  rc = launch(c, Op::DmcMove);  // moves, E_L, reweighting, weight sums, copy counts
  if (rc) return rc;
  if (cub::DeviceScan::ExclusiveSum(c->scan_tmp, c->scan_bytes, c->dA.ncopy, c->dA.off, c->dpar.wmax, c->stream) !=
      cudaSuccess)
    return fail(CHAMP_ECUDA, "DMC scan failed");
  rc = launch(c, Op::DmcCopy);
  if (rc) return rc;
  k_dmc_finish<<<1, 32, 0, c->stream>>>(c->dA, c->dB, c->dpar);
  CK(cudaGetLastError());
  std::swap(c->std_, c->std2);
  std::swap(c->stf, c->stf2);
  std::swap(c->dA.wt, c->dB.wt);
  std::swap(c->dA.el, c->dB.el);
  return CHAMP_OK;
}

static void dmc_graph_release(champ_ctx *c) {
  if (c->dmc_exec) cudaGraphExecDestroy((cudaGraphExec_t)c->dmc_exec);
  if (c->dmc_graph) cudaGraphDestroy((cudaGraph_t)c->dmc_graph);
  c->dmc_exec = c->dmc_graph = nullptr;
}

// Captures two consecutive DMC steps (buffers A -> B -> A, so the host-side roles are unchanged
// afterwards) into a CUDA graph on a private stream; re-captured when the seed changes (the seed
// is a kernel parameter, the step number is read on the device).
static int dmc_graph_prepare(champ_ctx *c, uint64_t seed) {
  if (c->dmc_exec && c->dmc_graph_seed == seed) return CHAMP_OK;
  dmc_graph_release(c);
  if (!c->cap_stream) CK(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
  cudaStream_t saved = c->stream;
  c->stream = c->cap_stream;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = dmc_one_step(c);
  if (!rc) rc = dmc_one_step(c);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  c->stream = saved;
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(CHAMP_ECUDA, std::string("DMC step capture: ") + cudaGetErrorString(e));
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(CHAMP_ECUDA, std::string("DMC graph instantiation: ") + cudaGetErrorString(e));
  }
  c->dmc_graph = g;
  c->dmc_exec = x;
  c->dmc_graph_seed = seed;
  return CHAMP_OK;
}

static int cublas_handle(champ_ctx *c) {
  if (!c->cublas) {
    cublasHandle_t h;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return fail(CHAMP_ECUDA, "cublasCreate failed");
    c->cublas = h;
  }
  if (cublasSetStream((cublasHandle_t)c->cublas, c->stream) != CUBLAS_STATUS_SUCCESS)
    return fail(CHAMP_ECUDA, "cublasSetStream failed");
  return CHAMP_OK;
}

// Reports (once) a tensor-core orbital contraction that gave up waiting for its MMA groups since
// the last check, and clears the flag.  Synchronises the stream when the contraction is in use.
static int tc_check(champ_ctx *c) {
  if (!c->tc_err || !c->tc_on) return CHAMP_OK;
  int h = 0;
  CK(cudaMemcpyAsync(&h, c->tc_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (h) {
    CK(cudaMemsetAsync(c->tc_err, 0, sizeof(int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return fail(CHAMP_ECUDA, "tensor-core orbital contraction gave up waiting for its MMA groups; the orbitals, "
                             "and the energies of the call that reported it, are not valid");
  }
  return CHAMP_OK;
}

extern "C" {

const char *champ_last_error(void) { return g_err.c_str(); }
const char *champ_version(void) { return "champ_b200 0.1 (sm_100a)"; }

int champ_create(const champ_system *d, int32_t w_max, int32_t precision, void *stream, champ_ctx **out) {
  if (!d || !out || w_max <= 0) return fail(CHAMP_EINVAL, "null argument or w_max <= 0");
  *out = nullptr;
  if (d->nelec < 1 || d->nelec > CHAMP_MAX_ELEC) return fail(CHAMP_EINVAL, "nelec out of range");
  if (d->nup < 0 || d->nup > d->nelec) return fail(CHAMP_EINVAL, "nup out of range");
  if (d->nup > CHAMP_MAX_SPIN || d->nelec - d->nup > CHAMP_MAX_SPIN) return fail(CHAMP_EINVAL, "more than 64 electrons of one spin");
  if (d->nctype < 1 || d->nctype > MAXCT) return fail(CHAMP_EINVAL, "nctype must be 1..4");
  if (d->ncent < 1) return fail(CHAMP_EINVAL, "ncent < 1");
  if (d->ndet < 1 || d->ndet > 65536) return fail(CHAMP_EINVAL, "ndet out of range");
  if (d->norda > MAXORD - 1 || d->nordb > MAXORD - 1) return fail(CHAMP_EINVAL, "norda/nordb > 7");
  if (!(d->nordc == 0 || d->nordc == 1 || d->nordc == 4 || d->nordc == 5)) return fail(CHAMP_EINVAL, "nordc must be 0, 1, 4 or 5");
  if (d->nloc != 0 && d->nloc != 6) return fail(CHAMP_EINVAL, "nloc must be 0 or 6");
  if (d->nloc == 6 && (d->nquad < 1 || d->nquad > 1000)) return fail(CHAMP_EINVAL, "nquad out of range");
  if (d->nloc == 6 && d->mgauss > MG) return fail(CHAMP_EINVAL, "more than 4 Gaussian terms per channel");
  if (precision != CHAMP_PREC_FP64 && precision != CHAMP_PREC_MIXED && precision != CHAMP_PREC_FP32)
    return fail(CHAMP_EINVAL, "bad precision");
  for (int i = 0; i < d->nshell; i++) {
    if (d->shell_l[i] < 0 || d->shell_l[i] > CHAMP_MAX_L || d->shell_n[i] < 1) return fail(CHAMP_EINVAL, "shell with bad n or l");
    if (d->shell_kind[i] < 0 || d->shell_kind[i] > 2) return fail(CHAMP_EINVAL, "shell kind must be 0, 1 or 2");
  }
  champ_ctx *c = new champ_ctx();
  c->prec = precision;
  c->stream = (cudaStream_t)stream;
  c->wmax = w_max;
  c->N = d->nelec; c->nup = d->nup; c->ndn = d->nelec - d->nup; c->C = d->ncent; c->nct = d->nctype;
  c->nshell = d->nshell; c->nbasis = d->nbasis; c->nmax = std::max(1, std::max(c->nup, c->ndn));
  c->nordc = d->nordc; c->nloc = d->nloc;
  {
    int rc0 = build_multidet(d, c->md);
    if (rc0) { delete c; return rc0; }
    c->nomax = std::max(1, std::max(c->md.nocc[0], c->md.nocc[1]));
    // orbital rotations by orbital class (single_ex_wf_bld, deriv_orb_mod.f90:130-417).  One
    // determinant: closed (both spins) -> open (one spin), closed -> virtual, open -> virtual.
    // Several: closed (both spins in every determinant) -> active, closed -> virtual,
    // active i -> active j (i < j, antisymmetric), active -> virtual.
    c->orbp.clear();
    {
      const int no = d->norb, ne = d->nelec, nu = d->nup;
      std::vector<int> cnt_all(no, 0), any(no, 0);
      for (int K = 0; K < d->ndet; K++) {
        std::vector<int> inu(no, 0), ind(no, 0);
        for (int e = 0; e < ne; e++) (e < nu ? inu : ind)[d->det_orb[(size_t)K * ne + e]] = 1;
        for (int m = 0; m < no; m++) {
          if (inu[m] && ind[m]) cnt_all[m]++;
          if (inu[m] || ind[m]) any[m] = 1;
        }
      }
      std::vector<int> cls, mid, vir;  // closed, open/active, virtual
      for (int m = 0; m < no; m++) {
        if (cnt_all[m] == d->ndet) cls.push_back(m);
        else if (any[m]) mid.push_back(m);
        else vir.push_back(m);
      }
      for (int i : cls)
        for (int j : mid) c->orbp.push_back(make_int4(i, j, 0, 0));
      for (int i : cls)
        for (int j : vir) c->orbp.push_back(make_int4(i, j, 0, 0));
      if (c->md.multidet)
        for (size_t a = 0; a < mid.size(); a++)
          for (size_t b = a + 1; b < mid.size(); b++) c->orbp.push_back(make_int4(mid[a], mid[b], 1, 0));
      for (int i : mid)
        for (int j : vir) c->orbp.push_back(make_int4(i, j, 0, 0));
    }
    c->norbp = (int)c->orbp.size();
    c->norb = d->norb;
    c->ncsfp = c->md.multidet && d->ncsf > 1 ? d->ncsf - 1 : 0;
    if (c->nomax > 256) { delete c; return fail(CHAMP_EINVAL, "more than 256 occupied orbitals of one spin"); }
  }
  // normalised primitive weights (basis_norm; numerical radial functions take the angular factor
  // sqrt((2l+1)/4pi) only, basis_norm.f90:57-58)
  std::vector<double> pcn;
  for (int i = 0, p = 0; i < d->nshell; i++)
    for (int q = 0; q < d->shell_nprim[i]; q++, p++)
      pcn.push_back(d->prim_coef[p] * (d->shell_kind[i] == 2
                                           ? std::sqrt((2 * d->shell_l[i] + 1) / (4 * 3.141592653589793))
                                           : host_anorm(d->shell_kind[i], d->shell_n[i], d->shell_l[i], d->prim_zeta[p])));
  {
    int rc0 = build_radial_tables(d, c);
    if (rc0) { delete c; return rc0; }
  }
  // e-e-n terms; the optimisable parameters kept for later updates
  int nt = 0;
  for (int n = 2; n <= d->nordc; n++)
    for (int k = n - 1; k >= 0; k--) {
      int l_hi = (k == 0) ? n - k - 2 : n - k;
      for (int l = l_hi; l >= 0; l--) if (((n - k - l) & 1) == 0) nt++;
    }
  {
    Params &q = c->par;
    q.norda = d->norda; q.nordb = d->nordb; q.nordc = d->nordc; q.nspin2b = d->nspin2b; q.een_cusp = d->een_cusp;
    q.nterms = nt; q.scalek = d->scalek;
    q.a4.assign(d->a4, d->a4 + (size_t)d->nctype * (d->norda + 1));
    q.b.assign(d->b, d->b + (size_t)d->nspin2b * (d->nordb + 1));
    q.c.assign((size_t)d->nctype * nt, 0.0);
    if (nt) memcpy(q.c.data(), d->c, sizeof(double) * d->nctype * nt);
    q.csf.assign(d->csf_coef, d->csf_coef + d->ncsf);
    q.csf_ndet.assign(d->csf_ndet, d->csf_ndet + d->ncsf);
    size_t ncd = 0;
    for (int i = 0; i < d->ncsf; i++) ncd += d->csf_ndet[i];
    q.csf_det.assign(d->csf_det, d->csf_det + ncd);
    q.csf_det_coef.assign(d->csf_det_coef, d->csf_det_coef + ncd);
    q.coef.assign(d->coef, d->coef + (size_t)d->norb * d->nbasis);
  }
  std::vector<double> cfull;
  double asa[MAXCT] = {0}, asb[2] = {0, 0};
  derive_jastrow(c, cfull, asa, asb);
  // free e-e-n coefficients and d c / d c_free (the cusp map is linear, so unit vectors give
  // its columns exactly)
  {
    std::vector<int> dep;
    if (d->een_cusp && nt > 0) {
      std::vector<double> z(nt, 0.0);
      host_een_cusp(d->nordc, 1, nt, z, &dep);
    }
    std::vector<int> fr;
    for (int ll = 0; ll < nt; ll++)
      if (std::find(dep.begin(), dep.end(), ll) == dep.end()) fr.push_back(ll);
    c->ncfree = (d->nordc > 1) ? (int)fr.size() : 0;
    c->par.cfree = fr;
    c->cproj.assign((size_t)std::max(nt, 1) * std::max(c->ncfree, 1), 0.0);
    for (int f = 0; f < c->ncfree; f++) {
      std::vector<double> u(nt, 0.0);
      u[fr[f]] = 1.0;
      if (d->een_cusp) host_een_cusp(d->nordc, 1, nt, u, nullptr);
      for (int ll = 0; ll < nt; ll++) c->cproj[(size_t)ll * c->ncfree + f] = u[ll];
    }
    int na = d->nctype * std::max(0, d->norda - 1), nb = d->nspin2b * d->nordb;
    c->np_raw = na + nb + (d->nordc > 1 ? d->nctype * nt : 0);
    c->nparm_jas = na + nb + d->nctype * c->ncfree;
  }

  // pseudopotential and quadrature (rotqua.f90 icosahedral rule)
  EcpPar ecp;
  memset(&ecp, 0, sizeof ecp);
  for (int it = 0; it < d->nctype; it++) ecp.znuc[it] = d->znuc[it];
  if (d->nloc == 6) {
    for (int it = 0; it < d->nctype; it++) {
      ecp.npotd[it] = d->npotd[it];
      ecp.lpotp1[it] = d->lpotp1[it];
      if (d->npotd[it] < 1 || d->npotd[it] > MAXLCH || d->lpotp1[it] < 1 || d->lpotp1[it] > d->npotd[it]) {
        delete c;
        return fail(CHAMP_EINVAL, "bad npotd/lpotp1");
      }
      for (int l = 0; l < MAXLCH; l++) {
        int ntm = d->necp_term[it * MAXLCH + l];
        if (ntm > MG) { delete c; return fail(CHAMP_EINVAL, "too many ECP terms"); }
        ecp.nterm[it][l] = ntm;
        for (int i = 0; i < ntm; i++) {
          size_t o = ((size_t)it * MAXLCH + l) * d->mgauss + i;
          ecp.coef[it][l][i] = d->ecp_coef[o];
          ecp.expo[it][l][i] = d->ecp_exponent[o];
          ecp.pw[it][l][i] = d->necp_power[o];
        }
      }
    }
  }
  ecp.nquad = quadrature_rule(d->nloc == 6 ? d->nquad : 12, c->quad.q0, c->quad.wq);
  c->nquad = ecp.nquad;
  double pecent = 0;
  for (int i = 0; i < d->ncent; i++)
    for (int j = 0; j < i; j++) {
      double dx = d->cent[3 * i] - d->cent[3 * j], dy = d->cent[3 * i + 1] - d->cent[3 * j + 1],
             dz = d->cent[3 * i + 2] - d->cent[3 * j + 2];
      pecent += d->znuc[d->iwctype[i]] * d->znuc[d->iwctype[j]] / std::sqrt(dx * dx + dy * dy + dz * dz);
    }
  int rc = CHAMP_OK;
  const bool use64 = precision != CHAMP_PREC_FP32, use32 = precision != CHAMP_PREC_FP64;
  // warps per block: up to 4, keeping the block's dynamic shared memory under 96 KB
  auto finish_cfg = [&](KCfg &k) -> int {
    k.smem = k.lay.bytes;
    k.wpb = 4;  // 128-thread blocks (the kernels' launch bounds)
    while (k.wpb > 1 && k.smem * k.wpb > 96 * 1024) k.wpb >>= 1;
    if (k.smem * k.wpb > 200 * 1024) return fail(CHAMP_EINVAL, "system too large for the per-warp shared memory");
    k.smem *= k.wpb;
    return CHAMP_OK;
  };
  if (use64) {
    rc = build_sys<double>(c, d, pcn, cfull, asa, asb, ecp, pecent, c->sd);
    if (!rc) rc = build_state<double>(c, c->std_);
    c->kd.lay = make_layout<double>(c->N, c->C, c->nbasis, c->nmax, c->nomax, c->std_.astride, c->std_.tvstride,
                                    c->std_.gstride, c->std_.wstride, c->nloc > 0, RESIDENT_LIMIT);
    if (!rc) rc = finish_cfg(c->kd);
    // walker state in HBM: the full evaluation as the four kernels of elstage.cuh
    if (!rc && !c->kd.lay.resident) rc = setup_el_staged(c);
    if (!rc && !c->kd.lay.resident && !c->md.multidet) rc = setup_delay(c);
  }
  if (use32 && !rc) {
    rc = build_sys<float>(c, d, pcn, cfull, asa, asb, ecp, pecent, c->sf);
    if (!rc) rc = precision == CHAMP_PREC_MIXED ? build_move_state(c, c->std_, c->stf) : build_state<float>(c, c->stf);
    // the mixed move kernels need no orbital, projection or quadrature scratch
    c->kf.lay = make_layout<float>(c->N, c->C, c->nbasis, c->nmax, c->nomax, c->stf.astride, c->stf.tvstride,
                                   c->stf.gstride, c->stf.wstride, c->nloc > 0 && precision == CHAMP_PREC_FP32,
                                   RESIDENT_LIMIT);
    if (!rc) rc = finish_cfg(c->kf);
    // Gaussian moves of a state in HBM: a move-only layout (one basis channel) and the block's
    // warps sharing the proposals' coefficient stream (block_orbitals: more than 16 and at most 128
    // orbitals per spin, the lane mapping of warp_orbitals, so the sums are the same)
    const int no0 = c->sf.nocc[0], no1 = c->sf.nocc[1];
    if (!rc && !c->kf.lay.resident && !c->md.multidet && no0 > 16 && no1 > 16 && no0 <= 128 && no1 <= 128) {
      KCfg &m = c->kfm;
      m.lay = make_layout<float>(c->N, c->C, c->nbasis, c->nmax, c->nomax, c->stf.astride, c->stf.tvstride,
                                 c->stf.gstride, c->stf.wstride, false, RESIDENT_LIMIT, true);
      m.wpb = 4;
      m.lay.stage = align16(m.lay.bytes * m.wpb);
      m.smem = m.lay.stage + sizeof(float) * COOP_STAGES * COOP_KB * (size_t)std::max(no0, no1);
      m.lay.coop = 1;
      if (m.smem <= 200 * 1024) c->move_coop = 1;
      else m = KCfg{};
    }
  }
  if (rc) { champ_destroy(c); return rc; }
  c->nfree = c->ncsfp + c->norbp + c->nparm_jas;
  {
    // the derivative kernel (FP64 for FP64 and mixed contexts) adds its accumulators to the
    // always-shared part of the layout
    const Layout &lp = use64 ? c->kd.lay : c->kf.lay;
    size_t pgb = lp.base + align16(sizeof(double) * (4 * (size_t)c->N + 3 * (size_t)c->np_raw +
                                                     (size_t)c->N * c->np_raw));
    // per-lane NLPP parameter slots: always in FP32; in FP64 while the warp's share stays small
    c->pg_lanesum = (c->prec == CHAMP_PREC_FP32 || pgb <= 24 * 1024) ? 1 : 0;
    if (c->pg_lanesum) pgb += align16(sizeof(double) * 32 * (size_t)c->np_raw);
    c->wpb_pg = 4;
    while (c->wpb_pg > 1 && pgb * c->wpb_pg > 160 * 1024) c->wpb_pg >>= 1;
    c->smem_pg = pgb * c->wpb_pg;
    if (c->smem_pg > 220 * 1024) c->smem_pg = 0;  // parameter derivatives unavailable for this size
  }
  if (use64) rc = attrs_f64(c);
  if (use32 && !rc) rc = attrs_f32(c);
  if (!rc) rc = tc_setup(c);
  c->reinv_every = std::max(1, (100 + c->N - 1) / c->N);  // about every 100 single-electron moves
  if (rc) { champ_destroy(c); return rc; }
  c->d_in = dalloc<double>(c, (size_t)w_max * 3 * c->N);
  c->d_out = dalloc<double>(c, (size_t)w_max * 4 * c->N);
  c->d_mask = dalloc<uint8_t>(c, w_max);
  if (!c->d_in || !c->d_out || !c->d_mask) { champ_destroy(c); return fail(CHAMP_ENOMEM, "staging allocation failed"); }
  {
    size_t W = w_max, P = c->nfree, P1 = P + 1;
    c->pg_dl = dalloc<double>(c, W * std::max<size_t>(P, 1));
    c->pg_de = dalloc<double>(c, W * std::max<size_t>(P, 1));
    c->pg_el = dalloc<double>(c, W);
    c->pg_wt = dalloc<double>(c, W);
    c->oh_oa = dalloc<double>(c, W * P1);
    c->oh_ow = dalloc<double>(c, W * P1);
    c->oh_mb = dalloc<double>(c, W * P1);
    c->oh_s = dalloc<double>(c, P1 * P1);
    c->oh_h = dalloc<double>(c, P1 * P1);
    if (c->ncsfp + c->norbp > 0) {
      size_t N = c->N, B = c->nbasis, M = d->norb, nm = c->nmax;
      c->scr_stride = N * B + N * 5 * M + N * M + 4 * nm * M + nm * nm + (size_t)(c->md.ndu[0] + c->md.ndu[1]) + 1;
      if (c->md.multidet) {
        size_t no = c->nomax;
        c->scr_stride += 4 * no * M + 5 * no * nm + (size_t)(c->md.ndu[0] + c->md.ndu[1]);
      }
      c->pg_scr = dalloc<double>(c, W * c->scr_stride);
      if (!c->pg_scr) { champ_destroy(c); return fail(CHAMP_ENOMEM, "allocation of the derivative scratch failed"); }
    }
    c->pg_tv = dalloc<double>(c, W * 4 * (size_t)c->N);
    c->pg_tn = dalloc<int>(c, W);
    c->pg_tc = c->nloc > 0 ? dalloc<double>(c, W * (size_t)c->N * c->C * quad_points(c)) : nullptr;
    if (!c->pg_tv || !c->pg_tn || (c->nloc > 0 && !c->pg_tc)) {
      champ_destroy(c);
      return fail(CHAMP_ENOMEM, "allocation of the parameter-gradient tape failed");
    }
    if (!c->pg_dl || !c->pg_de || !c->pg_el || !c->pg_wt || !c->oh_oa || !c->oh_ow || !c->oh_mb || !c->oh_s || !c->oh_h) {
      champ_destroy(c);
      return fail(CHAMP_ENOMEM, "allocation of the parameter-derivative buffers failed");
    }
  }
  *out = c;
  return CHAMP_OK;
}

int champ_destroy(champ_ctx *c) {
  if (!c) return CHAMP_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  else cudaDeviceSynchronize();
  dmc_graph_release(c);
  for (void *e : c->ev_pool) cudaEventDestroy((cudaEvent_t)e);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  for (void *p : c->allocs) cudaFree(p);
  if (c->cublas) cublasDestroy((cublasHandle_t)c->cublas);
  delete c;
  return CHAMP_OK;
}

static OpArgs pg_args(champ_ctx *c, int part) {
  OpArgs a;
  a.pgout.dlnpsi = c->pg_dl;
  a.pgout.deloc = c->pg_de;
  a.pgout.eloc = c->pg_el;
  a.pgout.nfree = c->nfree;
  a.pgout.scr = c->pg_scr;
  a.pgout.scr_stride = c->scr_stride;
  a.pgout.part = part;
  a.pgout.lanesum = c->pg_lanesum;
  a.pgout.tape_v = c->pg_tv;
  a.pgout.tape_n = c->pg_tn;
  a.pgout.tape_nlt = c->prec == CHAMP_PREC_FP32 ? c->stf.nlt : c->std_.nlt;
  a.pgout.tape_c = c->pg_tc;
  return a;
}

// The nonlocal part of the orbital-resolved local energy for all walkers, then the CSF and
// orbital-rotation derivatives (part 2 of the derivative kernel).
static int pg_orbital_part(champ_ctx *c) {
  if (!c->pg_scr) return CHAMP_OK;
  // nonlocal part of B for all walkers at once: Bm[w] += phis[w] (N x B) coef (B x M), row-major,
  // as the column-major product Bm^T (M x N) += coef^T (M x B) phis^T (B x N)
  int rc = cublas_handle(c);
  if (rc) return rc;
  const int N = c->N, B = c->nbasis, M = c->norb;
  const double one = 1.0;
  if (cublasDgemmStridedBatched((cublasHandle_t)c->cublas, CUBLAS_OP_N, CUBLAS_OP_N, M, N, B, &one, c->call_d, M, 0,
                                c->pg_scr, B, (long long)c->scr_stride, &one,
                                c->pg_scr + (size_t)N * B + (size_t)N * 5 * M, M, (long long)c->scr_stride,
                                c->W) != CUBLAS_STATUS_SUCCESS)
    return fail(CHAMP_ECUDA, "cublasDgemmStridedBatched failed");
  OpArgs a = pg_args(c, 2);
  return launch(c, Op::PGrad, a);
}

int champ_param_grad_fwd(champ_ctx *c, double *eloc) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (!c->have_walkers) return fail(CHAMP_ESTATE, "no walkers set");
  if (c->smem_pg == 0) return fail(CHAMP_EINVAL, "parameter derivatives: system too large for the kernel's shared memory");
  OpArgs a = pg_args(c, 3);
  int rc = launch(c, Op::PGrad, a);
  if (rc) return rc;
  c->have_tape = true;
  c->have_pgrad = false;
  if (eloc) {
    CK(cudaMemcpyAsync(eloc, c->pg_el, sizeof(double) * c->W, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return CHAMP_OK;
}

int champ_param_grad_bwd(champ_ctx *c, double *dlnpsi, double *deloc) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (!c->have_tape) return fail(CHAMP_ESTATE, "call champ_param_grad_fwd first");
  OpArgs a = pg_args(c, 4);
  int rc = launch(c, Op::PGradBwd, a);
  if (!rc) rc = pg_orbital_part(c);
  if (rc) return rc;
  c->have_tape = false;
  size_t W = c->W, P = c->nfree;
  if (dlnpsi) CK(cudaMemcpyAsync(dlnpsi, c->pg_dl, sizeof(double) * W * P, cudaMemcpyDeviceToHost, c->stream));
  if (deloc) CK(cudaMemcpyAsync(deloc, c->pg_de, sizeof(double) * W * P, cudaMemcpyDeviceToHost, c->stream));
  if (dlnpsi || deloc) CK(cudaStreamSynchronize(c->stream));
  c->have_pgrad = true;
  return CHAMP_OK;
}

int champ_param_grad(champ_ctx *c, double *dlnpsi, double *deloc, double *eloc) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (!c->have_walkers) return fail(CHAMP_ESTATE, "no walkers set");
  if (c->smem_pg == 0) return fail(CHAMP_EINVAL, "parameter derivatives: system too large for the kernel's shared memory");
  if (c->pg_mode == 0) {
    int rc = champ_param_grad_fwd(c, nullptr);
    if (!rc) rc = champ_param_grad_bwd(c, nullptr, nullptr);
    if (rc) return rc;
    size_t W = c->W, P = c->nfree;
    if (dlnpsi) CK(cudaMemcpyAsync(dlnpsi, c->pg_dl, sizeof(double) * W * P, cudaMemcpyDeviceToHost, c->stream));
    if (deloc) CK(cudaMemcpyAsync(deloc, c->pg_de, sizeof(double) * W * P, cudaMemcpyDeviceToHost, c->stream));
    if (eloc) CK(cudaMemcpyAsync(eloc, c->pg_el, sizeof(double) * W, cudaMemcpyDeviceToHost, c->stream));
    if (dlnpsi || deloc || eloc) CK(cudaStreamSynchronize(c->stream));
    return CHAMP_OK;
  }
  // one pass: E_L and the Jastrow derivatives together (option "param_grad_mode" 1)
  OpArgs a = pg_args(c, 1);
  int rc = launch(c, Op::PGrad, a);
  if (rc) return rc;
  rc = pg_orbital_part(c);
  if (rc) return rc;
  size_t W = c->W, P = c->nfree;
  if (dlnpsi) CK(cudaMemcpyAsync(dlnpsi, c->pg_dl, sizeof(double) * W * P, cudaMemcpyDeviceToHost, c->stream));
  if (deloc) CK(cudaMemcpyAsync(deloc, c->pg_de, sizeof(double) * W * P, cudaMemcpyDeviceToHost, c->stream));
  if (eloc) CK(cudaMemcpyAsync(eloc, c->pg_el, sizeof(double) * W, cudaMemcpyDeviceToHost, c->stream));
  if (dlnpsi || deloc || eloc) CK(cudaStreamSynchronize(c->stream));
  c->have_pgrad = true;
  return CHAMP_OK;
}

}  // extern "C"

// Re-derives and uploads everything the kernels take from the optimisable parameters: the Jastrow
// parameters (cusp-fixed e-e-n coefficients, asymptotic values), the determinant coefficients with
// the CSF coefficients folded in, the orbital coefficients in every layout the kernels read, and
// the tensor-core splits.  Writes into the buffers champ_create allocated.
template <class T>
static int upload_params(champ_ctx *c, Sys<T> &s) {
  const Params &q = c->par;
  std::vector<double> cfull;
  double asa[MAXCT], asb[2];
  derive_jastrow(c, cfull, asa, asb);
  JasPar<T> J;
  fill_jaspar<T>(c, cfull, asa, asb, J);
  CK(cudaMemcpy((void *)s.jas, &J, sizeof J, cudaMemcpyHostToDevice));
  std::vector<double> cc(c->md.ndet, 0.0);
  for (size_t icsf = 0, off = 0; icsf < q.csf.size(); icsf++)
    for (int i = 0; i < q.csf_ndet[icsf]; i++, off++) cc[q.csf_det[off]] += q.csf_det_coef[off] * q.csf[icsf];
  if (!c->md.multidet && cc[0] == 0.0) return fail(CHAMP_EINVAL, "zero determinant coefficient");
  c->md.ccoef = cc;
  CK(cudaMemcpy((void *)s.ccoef, cc.data(), sizeof(double) * cc.size(), cudaMemcpyHostToDevice));
  const int B = c->nbasis, M = c->norb;
  for (int sp = 0; sp < 2; sp++) {
    const int no = c->md.nocc[sp];
    if (no == 0) continue;
    std::vector<T> cr((size_t)B * no), ct((size_t)no * B);
    for (int k = 0; k < no; k++)
      for (int b = 0; b < B; b++) {
        const T v = (T)q.coef[(size_t)c->md.occ[sp][k] * B + c->perm_b[b]];
        cr[(size_t)b * no + k] = v;
        ct[(size_t)k * B + b] = v;
      }
    CK(cudaMemcpy((void *)s.cocc[sp], cr.data(), sizeof(T) * cr.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((void *)s.coccT[sp], ct.data(), sizeof(T) * ct.size(), cudaMemcpyHostToDevice));
    if constexpr (std::is_same<T, float>::value) c->tc_coef[sp] = cr;
  }
  std::vector<T> ca((size_t)B * M);
  std::vector<double> cd((size_t)B * M);
  for (int m = 0; m < M; m++)
    for (int b = 0; b < B; b++) ca[(size_t)b * M + m] = (T)(cd[(size_t)b * M + m] = q.coef[(size_t)m * B + c->perm_b[b]]);
  CK(cudaMemcpy((void *)s.call, ca.data(), sizeof(T) * ca.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->call_d, cd.data(), sizeof(double) * cd.size(), cudaMemcpyHostToDevice));
  if constexpr (std::is_same<T, float>::value)
    if (c->tc_ok) return tc_upload_split(c);
  return CHAMP_OK;
}

static int reload_params(champ_ctx *c) {
  int rc = CHAMP_OK;
  if (c->prec != CHAMP_PREC_FP32) rc = upload_params<double>(c, c->sd);
  if (!rc && c->prec != CHAMP_PREC_FP64) rc = upload_params<float>(c, c->sf);
  if (rc) return rc;
  c->have_pgrad = c->have_tape = false;
  if (c->have_walkers) {  // the walkers' tables and inverses for the new wave function
    rc = launch(c, Op::Eval);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
  }
  return CHAMP_OK;
}

extern "C" {

int champ_set_params(champ_ctx *c, const double *a4, const double *b, const double *cc, const double *csf_coef,
                     const double *coef) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  c->orb5_valid = false;  // orbital rows of the old coefficients
  Params &q = c->par;
  if (a4) std::copy(a4, a4 + q.a4.size(), q.a4.begin());
  if (b) std::copy(b, b + q.b.size(), q.b.begin());
  if (cc) std::copy(cc, cc + q.c.size(), q.c.begin());
  if (csf_coef) std::copy(csf_coef, csf_coef + q.csf.size(), q.csf.begin());
  if (coef) std::copy(coef, coef + q.coef.size(), q.coef.begin());
  return reload_params(c);
}

int champ_get_params(const champ_ctx *c, double *a4, double *b, double *cc, double *csf_coef, double *coef) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  const Params &q = c->par;
  if (a4) std::copy(q.a4.begin(), q.a4.end(), a4);
  if (b) std::copy(q.b.begin(), q.b.end(), b);
  if (cc) {
    std::vector<double> cfull;
    double asa[MAXCT], asb[2];
    derive_jastrow(c, cfull, asa, asb);
    std::copy(cfull.begin(), cfull.begin() + q.c.size(), cc);
  }
  if (csf_coef) std::copy(q.csf.begin(), q.csf.end(), csf_coef);
  if (coef) std::copy(q.coef.begin(), q.coef.end(), coef);
  return CHAMP_OK;
}

int champ_apply_param_step(champ_ctx *c, const double *dp) {
  if (!c || !dp) return fail(CHAMP_EINVAL, "null argument");
  c->orb5_valid = false;
  Params &q = c->par;
  int k = 0;
  for (int i = 1; i <= c->ncsfp; i++) q.csf[i] += dp[k++];
  if (c->norbp) {
    const std::vector<double> old = q.coef;
    const int B = c->nbasis;
    for (int r = 0; r < c->norbp; r++) {
      const int4 o = c->orbp[r];
      const double d = dp[k++];
      for (int bb = 0; bb < B; bb++) {
        q.coef[(size_t)o.x * B + bb] += d * old[(size_t)o.y * B + bb];
        if (o.z) q.coef[(size_t)o.y * B + bb] -= d * old[(size_t)o.x * B + bb];
      }
    }
  }
  for (int it = 0; it < c->nct; it++)
    for (int kk = 2; kk <= q.norda; kk++) q.a4[(size_t)it * (q.norda + 1) + kk] += dp[k++];
  for (int is = 0; is < q.nspin2b; is++)
    for (int kk = 1; kk <= q.nordb; kk++) q.b[(size_t)is * (q.nordb + 1) + kk] += dp[k++];
  if (q.nordc > 1)
    for (int it = 0; it < c->nct; it++)
      for (int f = 0; f < c->ncfree; f++) q.c[(size_t)it * q.nterms + q.cfree[f]] += dp[k++];
  if (k != c->nfree) return fail(CHAMP_EINVAL, "internal: parameter count mismatch");
  return reload_params(c);
}

int champ_oh_buffers(const champ_ctx *c, const double **S, const double **H) {
  if (!c || !S || !H) return fail(CHAMP_EINVAL, "null argument");
  *S = c->oh_s;
  *H = c->oh_h;
  return CHAMP_OK;
}

int champ_accumulate_oh(champ_ctx *c, const double *weights, double *S, double *H) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (!c->have_pgrad) return fail(CHAMP_ESTATE, "call champ_param_grad first");
  const int W = c->W, P = c->nfree, P1 = P + 1;
  int rc = cublas_handle(c);
  if (rc) return rc;
  cublasHandle_t h = (cublasHandle_t)c->cublas;
  if (weights) CK(cudaMemcpyAsync(c->pg_wt, weights, sizeof(double) * W, cudaMemcpyHostToDevice, c->stream));
  k_pack_oh<<<592, 256, 0, c->stream>>>(W, P, c->pg_dl, c->pg_de, c->pg_el, weights ? c->pg_wt : nullptr, c->oh_oa,
                                        c->oh_ow, c->oh_mb);
  CK(cudaGetLastError());
  // S[a][b] = sum_w wt (1,O)_a (1,O)_b ;  H[a][b] = sum_w wt (1,O)_a (E_L, E_L O + dE)_b  (row-major)
  const double one = 1.0, zero = 0.0;
  if (cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, P1, P1, W, &one, c->oh_ow, P1, c->oh_oa, P1, &zero, c->oh_s, P1) !=
          CUBLAS_STATUS_SUCCESS ||
      cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, P1, P1, W, &one, c->oh_mb, P1, c->oh_oa, P1, &zero, c->oh_h, P1) !=
          CUBLAS_STATUS_SUCCESS)
    return fail(CHAMP_ECUDA, "cublasDgemm failed");
  if (S) CK(cudaMemcpyAsync(S, c->oh_s, sizeof(double) * P1 * P1, cudaMemcpyDeviceToHost, c->stream));
  if (H) CK(cudaMemcpyAsync(H, c->oh_h, sizeof(double) * P1 * P1, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
}


int champ_dmc_init(champ_ctx *c, int32_t w_target, double tau, double gpop) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (!c->have_walkers) return fail(CHAMP_ESTATE, "set the initial walkers first");
  if (w_target < 1 || tau <= 0 || gpop <= 0) return fail(CHAMP_EINVAL, "bad DMC parameters");
  if (!c->dmc_ready) {
    int rc;
    if (c->prec == CHAMP_PREC_FP64) rc = alloc_state_copy<double>(c, c->std_, c->std2);
    else if (c->prec == CHAMP_PREC_FP32) rc = alloc_state_copy<float>(c, c->stf, c->stf2);
    else {
      // the second buffer holds the FP32 move state; its FP64 twin shares the FP64 scratch
      rc = alloc_state_copy<float>(c, c->stf, c->stf2);
      if (!rc) {
        c->std2 = c->std_;
        State<double> &d2 = c->std2;
        const State<float> &f2 = c->stf2;
        d2.x = f2.x; d2.ainv = f2.ainv; d2.tv = f2.tv; d2.gam = f2.gam;
        d2.fsum = f2.fsum; d2.lnd = f2.lnd; d2.sgn = f2.sgn;
        d2.m_fso = f2.fso; d2.m_ren = f2.ren; d2.m_zq = f2.zq; d2.m_rtd = f2.rtd;
      }
    }
    if (rc) return rc;
    size_t W = c->wmax;
    int *nw = dalloc<int>(c, 1);
    double *sc = dalloc<double>(c, 12);
    int *nc = dalloc<int>(c, W), *off = dalloc<int>(c, W);
    double *stat = dalloc<double>(c, 4 * (size_t)DMC_STAT_CAP);
    double *w0 = dalloc<double>(c, W), *w1 = dalloc<double>(c, W), *e0 = dalloc<double>(c, W), *e1 = dalloc<double>(c, W);
    double *v0 = dalloc<double>(c, W), *v1 = dalloc<double>(c, W), *te = dalloc<double>(c, W);
    long long *ctr = dalloc<long long>(c, 2);
    int *nx = dalloc<int>(c, 2);
    if (!nw || !sc || !nc || !off || !stat || !w0 || !w1 || !e0 || !e1 || !v0 || !v1 || !te || !ctr || !nx)
      return fail(CHAMP_ENOMEM, "DMC allocation failed");
    c->dA.ctr = c->dB.ctr = ctr;
    c->dA.nw = c->dB.nw = nw;
    c->dA.et = c->dB.et = sc;
    c->dA.eest = c->dB.eest = sc + 1;
    c->dA.red = c->dB.red = sc + 2;
    c->dA.esg = c->dB.esg = sc + 5;
    c->dA.egr = c->dB.egr = sc + 9;
    c->dA.next = c->dB.next = nx;
    c->dA.teff = c->dB.teff = te;
    c->dA.v2 = v0; c->dB.v2 = v1;
    c->dA.ncopy = c->dB.ncopy = nc;
    c->dA.off = c->dB.off = off;
    c->dA.stat = c->dB.stat = stat;
    c->dA.wt = w0; c->dB.wt = w1;
    c->dA.el = e0; c->dB.el = e1;
    c->scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, c->scan_bytes, nc, off, (int)W, c->stream);
    c->scan_tmp = dalloc<char>(c, c->scan_bytes);
    if (!c->scan_tmp) return fail(CHAMP_ENOMEM, "DMC scan allocation failed");
    c->dmc_ready = true;
  }
  c->dpar.tau = tau;
  c->dpar.adrift = 0.5;  // adrift_default (control_mod.f90:16)
  c->dpar.gpop = gpop;
  c->dpar.rewt_limit = 10.0;  // limit_rewt_dmc (control_mod.f90:16)
  c->dpar.c_rewt = 3.5;       // c_rewt (control_mod.f90:16)
  c->dpar.ene_int = c->dmc_ene_int;
  c->dpar.wtarget = w_target;
  c->dpar.wmax = c->wmax;
  // initial population: the current walkers, weight 1, with their local energies
  int rc = launch(c, Op::EvalOut);
  if (rc) return rc;
  double *el = c->prec == CHAMP_PREC_FP32 ? c->stf.o_eloc : c->std_.o_eloc;
  double *vel = c->prec == CHAMP_PREC_FP32 ? c->stf.o_vel : c->std_.o_vel;
  std::vector<double> elh(c->W), one(c->W, 1.0), velh((size_t)c->W * c->N * 3), v2h(c->W, 0.0);
  CK(cudaMemcpyAsync(elh.data(), el, sizeof(double) * c->W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(velh.data(), vel, sizeof(double) * velh.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int w = 0; w < c->W; w++)
    for (int i = 0; i < 3 * c->N; i++) v2h[w] += velh[(size_t)w * 3 * c->N + i] * velh[(size_t)w * 3 * c->N + i];
  // the initial energy estimate: the median of the finite local energies (a mean would follow the
  // rare near-node outliers of a short equilibration)
  std::vector<double> fin;
  for (double e : elh)
    if (std::isfinite(e)) fin.push_back(e);
  double em = 0.0;
  if (!fin.empty()) {
    std::nth_element(fin.begin(), fin.begin() + fin.size() / 2, fin.end());
    em = fin[fin.size() / 2];
  }
  double sc[12] = {em, em, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, em, 0.0, 0.0};
  int nw = c->W;
  CK(cudaMemcpyAsync(c->dA.el, elh.data(), sizeof(double) * c->W, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->dA.v2, v2h.data(), sizeof(double) * c->W, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->dA.wt, one.data(), sizeof(double) * c->W, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->dA.et, sc, sizeof(double) * 12, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->dA.nw, &nw, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->dA.next, 0, 2 * sizeof(int), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->dmc_step = 0;
  dmc_graph_release(c);
  return CHAMP_OK;
}

int champ_dmc_steps(champ_ctx *c, int32_t nstep, uint64_t seed, double *stats) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (!c->dmc_ready) return fail(CHAMP_ESTATE, "call champ_dmc_init first");
  if (nstep < 0 || nstep > DMC_STAT_CAP) return fail(CHAMP_EINVAL, "nstep out of range");
  c->dpar.seed = seed;
  // step counter (random-number key) and statistics index live on the device
  const long long ctr[2] = {(long long)c->dmc_step, 0};
  CK(cudaMemcpyAsync(c->dA.ctr, ctr, sizeof(ctr), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int done = 0;
  if (c->dmc_graph_on && nstep >= 2) {
    int rc = dmc_graph_prepare(c, seed);
    if (rc) return rc;
    for (; done + 2 <= nstep; done += 2) CK(cudaGraphLaunch((cudaGraphExec_t)c->dmc_exec, c->stream));
  }
  for (; done < nstep; done++) {
    int rc = dmc_one_step(c);
    if (rc) return rc;
  }
  c->dmc_step += nstep;
  int nw = 0;
  CK(cudaMemcpyAsync(&nw, c->dA.nw, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  if (stats && nstep)
    CK(cudaMemcpyAsync(stats, c->dA.stat, sizeof(double) * 4 * nstep, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->W = nw;
  return CHAMP_OK;
}

int champ_nparam(const champ_ctx *c, int32_t *nj, int32_t *ncsf, int32_t *norb) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (nj) *nj = c->nparm_jas;
  if (ncsf) *ncsf = c->ncsfp;
  if (norb) *norb = c->norbp;
  return CHAMP_OK;
}

// buffers that an FP64 or mixed context keeps in its FP64 state and an FP32 context in its FP32 one
static State<double> *st64(champ_ctx *c) { return c->prec == CHAMP_PREC_FP32 ? nullptr : &c->std_; }
static double *state_x(champ_ctx *c) { return st64(c) ? c->std_.x : c->stf.x; }

int champ_set_walkers(champ_ctx *c, int32_t nw, const double *x) {
  if (!c || !x) return fail(CHAMP_EINVAL, "null argument");
  if (nw < 1 || nw > c->wmax) return fail(CHAMP_EINVAL, "nw out of range");
  c->W = nw;
  CK(cudaMemcpyAsync(state_x(c), x, sizeof(double) * nw * 3 * c->N, cudaMemcpyHostToDevice, c->stream));
  int *piel = st64(c) ? c->std_.piel : c->stf.piel;
  CK(cudaMemsetAsync(piel, 0xFF, sizeof(int) * nw, c->stream));
  int rc = launch(c, Op::Eval);
  if (rc) return rc;
  c->have_walkers = true;
  CK(cudaStreamSynchronize(c->stream));
  return tc_check(c);
}

int champ_get_walkers(champ_ctx *c, double *x) {
  if (!c || !x) return fail(CHAMP_EINVAL, "null argument");
  if (!c->have_walkers) return fail(CHAMP_ESTATE, "no walkers set");
  CK(cudaMemcpyAsync(x, state_x(c), sizeof(double) * c->W * 3 * c->N, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
}

int champ_set_quadrature_rotation(champ_ctx *c, const double *rot) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  static const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  memcpy(c->rot, rot ? rot : I, sizeof(double) * 9);
  return CHAMP_OK;
}


int champ_eval_full(champ_ctx *c, const champ_eval_out *o) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (!c->have_walkers) return fail(CHAMP_ESTATE, "no walkers set");
  int rc = launch(c, Op::EvalOut);
  if (rc) return rc;
  if (o) {
    rc = st64(c) ? copy_eval_out<double>(c, o) : copy_eval_out<float>(c, o);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  return tc_check(c);
}

int champ_propose_1e(champ_ctx *c, int32_t iel, const double *xnew, double *ratio, double *grad_new) {
  if (!c || !xnew || !ratio) return fail(CHAMP_EINVAL, "null argument");
  if (!c->have_walkers) return fail(CHAMP_ESTATE, "no walkers set");
  if (iel < 0 || iel >= c->N) return fail(CHAMP_EINVAL, "iel out of range");
  size_t W = c->W;
  CK(cudaMemcpyAsync(c->d_in, xnew, sizeof(double) * 3 * W, cudaMemcpyHostToDevice, c->stream));
  OpArgs a;
  a.e = iel;
  a.xnew = c->d_in;
  a.ratio = c->d_out;
  a.grad = c->d_out + W;
  int rc = launch(c, grad_new ? Op::ProposeGrad : Op::Propose, a);
  if (rc) return rc;
  CK(cudaMemcpyAsync(ratio, c->d_out, sizeof(double) * W, cudaMemcpyDeviceToHost, c->stream));
  if (grad_new) CK(cudaMemcpyAsync(grad_new, c->d_out + W, sizeof(double) * 3 * W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
}

int champ_accept_1e(champ_ctx *c, int32_t iel, const uint8_t *accept) {
  if (!c || !accept) return fail(CHAMP_EINVAL, "null argument");
  if (!c->have_walkers) return fail(CHAMP_ESTATE, "no walkers set");
  if (iel < 0 || iel >= c->N) return fail(CHAMP_EINVAL, "iel out of range");
  CK(cudaMemcpyAsync(c->d_mask, accept, c->W, cudaMemcpyHostToDevice, c->stream));
  OpArgs a;
  a.e = iel;
  a.mask = c->d_mask;
  int rc = launch(c, Op::Accept, a);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
}

int champ_grad_1e(champ_ctx *c, int32_t iel, double *grad) {
  if (!c || !grad) return fail(CHAMP_EINVAL, "null argument");
  if (!c->have_walkers) return fail(CHAMP_ESTATE, "no walkers set");
  if (iel < 0 || iel >= c->N) return fail(CHAMP_EINVAL, "iel out of range");
  // a proposal at the current position: ratio 1, gradient of the current configuration
  std::vector<double> x((size_t)c->W * 3 * c->N), xn((size_t)c->W * 3), r(c->W);
  int rc = champ_get_walkers(c, x.data());
  if (rc) return rc;
  for (int w = 0; w < c->W; w++)
    for (int k = 0; k < 3; k++) xn[3 * w + k] = x[((size_t)w * c->N + iel) * 3 + k];
  return champ_propose_1e(c, iel, xn.data(), r.data(), grad);
}


int champ_vmc_sweeps(champ_ctx *c, int32_t nsweep, uint64_t seed, uint64_t sweep0, double step,
                     const champ_vmc_stats *stats) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (!c->have_walkers) return fail(CHAMP_ESTATE, "no walkers set");
  if (nsweep < 0) return fail(CHAMP_EINVAL, "nsweep < 0");
  OpArgs a;
  a.nsweep = nsweep;
  a.seed = seed;
  a.sweep0 = sweep0;
  a.step = step;
  int rc = launch(c, Op::Vmc, a);
  if (rc) return rc;
  if (stats) {
    rc = st64(c) ? copy_stats<double>(c, stats) : copy_stats<float>(c, stats);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
  }
  return tc_check(c);
}

int champ_vmc_run_host(champ_ctx *c, int32_t nw, double *x, int32_t nsweep, uint64_t seed, uint64_t sweep0,
                       double step, double *eloc) {
  if (!c || !x || !eloc) return fail(CHAMP_EINVAL, "null argument");
  if (nw < 1 || nw > c->wmax) return fail(CHAMP_EINVAL, "nw out of range");
  c->W = nw;
  CK(cudaMemcpyAsync(state_x(c), x, sizeof(double) * nw * 3 * c->N, cudaMemcpyHostToDevice, c->stream));
  OpArgs rb;
  rb.rebuild = true;  // the sweeps need the inverses and move tables; their E_L comes after the moves
  int rc = launch(c, Op::Eval, rb);
  if (rc) return rc;
  c->have_walkers = true;
  champ_vmc_stats st = {nullptr, nullptr, nullptr, nullptr};  // champ_vmc_sweeps reports a tensor-core give-up
  rc = champ_vmc_sweeps(c, nsweep, seed, sweep0, step, &st);
  if (rc) return rc;
  double *el = st64(c) ? c->std_.s_elast : c->stf.s_elast;
  CK(cudaMemcpyAsync(eloc, el, sizeof(double) * nw, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(x, state_x(c), sizeof(double) * nw * 3 * c->N, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
}

int champ_walker_status(champ_ctx *c, uint32_t *flags) {
  if (!c || !flags) return fail(CHAMP_EINVAL, "null argument");
  uint32_t *s = st64(c) ? c->std_.status : c->stf.status;
  CK(cudaMemcpyAsync(flags, s, sizeof(uint32_t) * c->W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return tc_check(c);
}

int champ_tmoves(champ_ctx *c, uint64_t seed, uint64_t step, double tau, int32_t variant, int32_t *moved) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (!c->have_walkers) return fail(CHAMP_ESTATE, "no walkers set");
  if (variant != 1 && variant != 2) return fail(CHAMP_EINVAL, "T-move variant: 1 (casula1) or 2 (det_balance1)");
  if (!(tau > 0)) return fail(CHAMP_EINVAL, "tau must be positive");
  if (c->nloc == 0) return fail(CHAMP_EINVAL, "T-moves need a nonlocal pseudopotential");
  OpArgs t;
  t.tau = tau;
  t.variant = variant;
  t.seed = seed;
  t.sweep0 = step;
  t.moved = moved ? (int *)c->d_out : nullptr;  // the staging buffer holds [w_max][4 nelec] doubles
  int rc = launch(c, Op::Tmove, t);
  if (rc) return rc;
  if (moved) CK(cudaMemcpyAsync(moved, t.moved, sizeof(int) * c->W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
}

int champ_set_mover(champ_ctx *c, int32_t imetro, double deltar, double deltat, double fbias) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (imetro != 1 && imetro != 6) return fail(CHAMP_EINVAL, "imetro must be 1 or 6 (accelerated Metropolis)");
  // the reference's corrections of out-of-range values (control_mod.f90:375-385)
  if (!(deltar >= 1.0)) deltar = 2.0;
  if (!(deltat >= 0.0 && deltat <= 2.0)) deltat = 2.0;
  fbias = std::min(2.0, std::max(0.0, fbias));
  c->mover = Mover{imetro, deltar, deltat, fbias};
  return CHAMP_OK;
}

int champ_set_option(champ_ctx *c, const char *name, int64_t value) {
  if (!c || !name) return fail(CHAMP_EINVAL, "null argument");
  if (!strcmp(name, "orbital_tc")) {
    if (value < 0 || value > 2) return fail(CHAMP_EINVAL, "orbital_tc: 0, 1 or 2");
    if (value && !c->tc_ok)
      return fail(CHAMP_EINVAL, "orbital_tc: needs FP32 precision, walker state in HBM, >= 16 orbitals of a spin "
                                "and room for the basis rows");
    if (value == 1) c->tc_mode = c->tc_fused_ok ? 1 : 2;
    if (value == 2) {
      int rc = tc_alloc_rows(c);
      if (rc) return rc;
      c->tc_mode = 2;
    }
    c->tc_on = value ? 1 : 0;
    return CHAMP_OK;
  }
  if (!strcmp(name, "dmc_graph")) {
    c->dmc_graph_on = value ? 1 : 0;
    return CHAMP_OK;
  }
  if (!strcmp(name, "reinvert_every")) {
    if (value < 1 || value > (1 << 30)) return fail(CHAMP_EINVAL, "reinvert_every must be >= 1");
    c->reinv_every = (int)value;
    return CHAMP_OK;
  }
  if (!strcmp(name, "orbital_tc_chunk")) {
    if (value < 0 || value > (1 << 20)) return fail(CHAMP_EINVAL, "orbital_tc_chunk must be >= 0");
    c->tc_kchunk = (int)value;
    return CHAMP_OK;
  }
  if (!strcmp(name, "phase_timing")) {
    c->ptime = value ? 1 : 0;
    c->ev_use.clear();
    return CHAMP_OK;
  }
  if (!strcmp(name, "param_grad_mode")) {
    if (value < 0 || value > 1) return fail(CHAMP_EINVAL, "param_grad_mode: 0 or 1");
    c->pg_mode = (int)value;
    return CHAMP_OK;
  }
  if (!strcmp(name, "mover_cache")) {
    if (value < 0 || value > 1) return fail(CHAMP_EINVAL, "mover_cache: 0 or 1");
    c->mover_cache = (int)value;
    return CHAMP_OK;
  }
  if (!strcmp(name, "orb_coop")) {
    if (value < 0 || value > 1) return fail(CHAMP_EINVAL, "orb_coop: 0 or 1");
    if (value && !c->orb_coop_ok)
      return fail(CHAMP_EINVAL, "orb_coop: needs the staged evaluation with electrons and up electrons in multiples "
                                "of 4 and more than 16 orbitals per spin");
    c->orb_coop = (int)value;
    return CHAMP_OK;
  }
  if (!strcmp(name, "move_coop")) {
    if (value < 0 || value > 1) return fail(CHAMP_EINVAL, "move_coop: 0 or 1");
    if (value && !c->kfm.lay.coop)
      return fail(CHAMP_EINVAL, "move_coop: needs an FP32 or mixed single-determinant context whose walker state "
                                "lives in HBM, with 17 to 128 orbitals per spin");
    c->move_coop = (int)value;
    return CHAMP_OK;
  }
  if (!strcmp(name, "dmc_persistent")) {
    if (value < 0 || value > 1) return fail(CHAMP_EINVAL, "dmc_persistent: 0 or 1");
    c->dpar.persist = (int)value;
    dmc_graph_release(c);
    return CHAMP_OK;
  }
  if (!strcmp(name, "dmc_ene_int")) {
    if (value < 0 || value > 1) return fail(CHAMP_EINVAL, "dmc_ene_int: 0 (no_ene_int) or 1 (ene_int_v9)");
    c->dmc_ene_int = c->dpar.ene_int = (int)value;
    dmc_graph_release(c);
    return CHAMP_OK;
  }
  if (!strcmp(name, "tmoves")) {
    if (value < 0 || value > 2) return fail(CHAMP_EINVAL, "tmoves: 0 (off), 1 (casula1) or 2 (det_balance1)");
    c->dpar.tmove = (int)value;
    dmc_graph_release(c);  // the captured steps carry the old setting
    return CHAMP_OK;
  }
  if (!strcmp(name, "delay_rank")) {
    if (value < 0 || value > DELAY_MAX) return fail(CHAMP_EINVAL, "delay_rank: 0 .. 32");
    if (value > 1 && !c->std_.dly)
      return fail(CHAMP_EINVAL, "delay_rank: needs a single-determinant FP64 or mixed context whose walker state "
                                "lives in HBM");
    c->std_.dlk = c->stf.dlk = (int)value;
    return CHAMP_OK;
  }
  if (!strcmp(name, "staged_eval")) {
    if (value && !c->std_.el_vj)
      return fail(CHAMP_EINVAL, "staged_eval: needs an FP64 or mixed context whose walker state lives in HBM");
    c->el_staged = value ? 1 : 0;
    return CHAMP_OK;
  }
  return fail(CHAMP_EINVAL, std::string("unknown option: ") + name);
}

int champ_phase_times(champ_ctx *c, double *ms, int32_t *launches) {
  if (!c || !ms) return fail(CHAMP_EINVAL, "null argument");
  CK(cudaStreamSynchronize(c->stream));
  for (int p = 0; p < PH_N; p++) {
    ms[p] = 0;
    if (launches) launches[p] = 0;
  }
  for (const auto &u : c->ev_use) {
    float t = 0;
    CK(cudaEventElapsedTime(&t, (cudaEvent_t)c->ev_pool[u.second], (cudaEvent_t)c->ev_pool[u.second + 1]));
    ms[u.first] += t;
    if (launches) launches[u.first]++;
  }
  c->ev_use.clear();
  return CHAMP_OK;
}

int champ_get_option(const champ_ctx *c, const char *name, int64_t *value) {
  if (!c || !name || !value) return fail(CHAMP_EINVAL, "null argument");
  if (!strcmp(name, "orbital_tc")) { *value = c->tc_on ? c->tc_mode : 0; return CHAMP_OK; }
  if (!strcmp(name, "launches_per_sweep")) {
    int spins = (c->nup > 0) + (c->ndn > 0);
    *value = c->tc_on                                     ? 2 + spins + (c->tc_mode == 2 ? 1 : 0)
             : (c->el_staged && c->prec != CHAMP_PREC_FP32) ? 5
             : (c->prec == CHAMP_PREC_MIXED ? 2 : 1);
    return CHAMP_OK;
  }
  if (!strcmp(name, "reinvert_every")) { *value = c->reinv_every; return CHAMP_OK; }
  if (!strcmp(name, "dmc_graph")) { *value = c->dmc_graph_on; return CHAMP_OK; }
  if (!strcmp(name, "orbital_tc_chunk")) { *value = c->tc_kchunk; return CHAMP_OK; }
  if (!strcmp(name, "phase_timing")) { *value = c->ptime; return CHAMP_OK; }
  if (!strcmp(name, "param_grad_mode")) { *value = c->pg_mode; return CHAMP_OK; }
  if (!strcmp(name, "staged_eval")) { *value = c->el_staged; return CHAMP_OK; }
  if (!strcmp(name, "delay_rank")) { *value = c->std_.dly ? c->std_.dlk : 0; return CHAMP_OK; }
  if (!strcmp(name, "tmoves")) { *value = c->dpar.tmove; return CHAMP_OK; }
  if (!strcmp(name, "dmc_ene_int")) { *value = c->dmc_ene_int; return CHAMP_OK; }
  if (!strcmp(name, "dmc_persistent")) { *value = c->dpar.persist; return CHAMP_OK; }
  if (!strcmp(name, "move_coop")) { *value = c->move_coop; return CHAMP_OK; }
  if (!strcmp(name, "orb_coop")) { *value = c->orb_coop_ok ? c->orb_coop : 0; return CHAMP_OK; }
  if (!strcmp(name, "mover_cache")) { *value = c->mover_cache; return CHAMP_OK; }
  return fail(CHAMP_EINVAL, std::string("unknown option: ") + name);
}

int champ_eval_energy_noalloc(champ_ctx *c, int32_t nw, const double *x, double *eloc) {
  if (!c || !x || !eloc) return fail(CHAMP_EINVAL, "null argument");
  if (nw < 1) return fail(CHAMP_EINVAL, "nw < 1");
  return st64(c) ? eval_noalloc_t<double>(c, c->std_, nw, x, eloc) : eval_noalloc_t<float>(c, c->stf, nw, x, eloc);
}

int champ_num_walkers(const champ_ctx *c, int32_t *nw) {
  if (!c || !nw) return fail(CHAMP_EINVAL, "null argument");
  *nw = c->W;
  return CHAMP_OK;
}

int champ_synchronize(champ_ctx *c) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  CK(cudaStreamSynchronize(c->stream));
  return tc_check(c);
}

}  // extern "C"
