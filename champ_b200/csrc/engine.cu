// engine.cu -- walker-batched Slater-Jastrow engine: kernels and the C ABI.
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
#include <mutex>
#include <string>
#include <vector>

#include "../../include/champ_b200.h"
#include "device_math.cuh"

using namespace champ;

// ---------------------------------------------------------------------------------------
// state
// ---------------------------------------------------------------------------------------
template <class T>
struct State {
  int W;
  double *x;       // [W][N][3]
  double *ainv;    // [W][astride]; spin-up block at 0 (nup x nup), spin-down at nup*nup
  T *fso;          // [W][N][N]
  T *ren;          // [W][N][C][2]: r_en and 1/(1 + scalek r_en)
  double *fsum, *lnd, *sgn;
  uint32_t *status;
  T *pf;           // [W][N] proposed pair values
  double *pa;      // [W][nmax] proposed orbital row (reference orbitals)
  double *pdj, *prho, *pxn;  // [W], [W], [W][3]
  int *piel;       // [W]
  T *orb5;         // [W][N][5][nmax]
  T *gproj;        // [W][N][nbasis]
  double *nlt;     // [W][N*C][NLT]
  int astride;
  // outputs of a full evaluation
  double *o_lnpsi, *o_sign, *o_psij, *o_vel, *o_divv, *o_d2, *o_pe, *o_peee, *o_penl, *o_eloc;
  // VMC accumulators
  double *s_esum, *s_e2sum, *s_acc, *s_elast;
};
constexpr int NLT = 2 + MAXLCH;  // task record: (e*C+c), r, vps[0..MAXLCH-1]

// Per-warp shared-memory layout, computed on the host.  When `resident` is set the
// walker's whole state and scratch live in shared memory for the life of a kernel
// (small systems); otherwise they stay in HBM.
struct Layout {
  size_t phi, arow, xs, vacc, divj, colb, vb, perm, rnew;  // always in shared memory
  size_t ainv, fso, ren, pf, orb5, gproj, nlt;             // resident mode only
  size_t bytes;
  int resident;
};

// Per-walker view: where this walker's arrays live for the current kernel.
template <class T>
struct View {
  T *phi, *arow;
  double *xs, *vacc, *divj, *colb, *vb;
  int *perm;
  T *rnew;         // [C][2] proposed electron's distances to the centres
  double *ainv;
  T *fso, *ren, *pf, *orb5, *gproj;
  double *nlt;
};

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

template <class T>
static Layout make_layout(int N, int C, int nbasis, int nmax, int astride, bool nl, size_t resident_limit) {
  Layout L;
  size_t o = 0;
  auto take = [&](size_t b) { size_t r = o; o += align16(b); return r; };
  L.phi = take(sizeof(T) * nbasis * 5);
  L.arow = take(sizeof(T) * 5 * nmax);
  L.xs = take(sizeof(double) * N * 3);
  L.vacc = take(sizeof(double) * N * 3);
  L.divj = take(sizeof(double) * N);
  L.colb = take(sizeof(double) * nmax);
  L.vb = take(sizeof(double) * nmax);
  L.perm = take(sizeof(int) * nmax);
  L.rnew = take(sizeof(T) * C * 2);
  size_t base = o;
  L.ainv = take(sizeof(double) * astride);
  L.fso = take(sizeof(T) * N * N);
  L.ren = take(sizeof(T) * N * C * 2);
  L.pf = take(sizeof(T) * N);
  L.orb5 = take(sizeof(T) * N * 5 * nmax);
  L.gproj = nl ? take(sizeof(T) * N * nbasis) : 0;
  L.nlt = nl ? take(sizeof(double) * N * C * NLT) : 0;
  L.resident = (o <= resident_limit) ? 1 : 0;
  L.bytes = L.resident ? o : base;
  return L;
}

template <class T>
__device__ inline View<T> make_view(char *base, const Layout &L, const State<T> &st, int w, int N, int C, int nbasis,
                                    int nmax, bool resident) {
  View<T> v;
  v.phi = (T *)(base + L.phi);
  v.arow = (T *)(base + L.arow);
  v.xs = (double *)(base + L.xs);
  v.vacc = (double *)(base + L.vacc);
  v.divj = (double *)(base + L.divj);
  v.colb = (double *)(base + L.colb);
  v.vb = (double *)(base + L.vb);
  v.perm = (int *)(base + L.perm);
  v.rnew = (T *)(base + L.rnew);
  if (resident) {
    v.ainv = (double *)(base + L.ainv);
    v.fso = (T *)(base + L.fso);
    v.ren = (T *)(base + L.ren);
    v.pf = (T *)(base + L.pf);
    v.orb5 = (T *)(base + L.orb5);
    v.gproj = (T *)(base + L.gproj);
    v.nlt = (double *)(base + L.nlt);
  } else {
    v.ainv = st.ainv + (size_t)w * st.astride;
    v.fso = st.fso + (size_t)w * N * N;
    v.ren = st.ren + (size_t)w * N * C * 2;
    v.pf = st.pf + (size_t)w * N;
    v.orb5 = st.orb5 + (size_t)w * N * 5 * nmax;
    v.gproj = st.gproj ? st.gproj + (size_t)w * N * nbasis : nullptr;
    v.nlt = st.nlt ? st.nlt + (size_t)w * N * C * NLT : nullptr;
  }
  return v;
}

// Copy a walker's persistent state between HBM and its resident view.
template <class T>
__device__ inline void view_load(const View<T> &v, const State<T> &st, int w, int N, int C, int lane) {
  for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
  for (int i = lane; i < st.astride; i += 32) v.ainv[i] = st.ainv[(size_t)w * st.astride + i];
  for (int i = lane; i < N * N; i += 32) v.fso[i] = st.fso[(size_t)w * N * N + i];
  for (int i = lane; i < N * C * 2; i += 32) v.ren[i] = st.ren[(size_t)w * N * C * 2 + i];
  __syncwarp();
}
template <class T>
__device__ inline void view_store(const View<T> &v, const State<T> &st, int w, int N, int C, int lane) {
  __syncwarp();
  for (int i = lane; i < 3 * N; i += 32) st.x[(size_t)w * 3 * N + i] = v.xs[i];
  for (int i = lane; i < st.astride; i += 32) st.ainv[(size_t)w * st.astride + i] = v.ainv[i];
  for (int i = lane; i < N * N; i += 32) st.fso[(size_t)w * N * N + i] = v.fso[i];
  for (int i = lane; i < N * C * 2; i += 32) st.ren[(size_t)w * N * C * 2 + i] = v.ren[i];
  __syncwarp();
}

// ---------------------------------------------------------------------------------------
// warp Gauss-Jordan inversion with partial pivoting, in place (matinv, qmc/vmc/matinv.f90).
// A is row-major n x n (electron row, orbital column); on return it holds the inverse
// indexed [orbital][electron].  Returns false if a pivot is exactly zero.
// ---------------------------------------------------------------------------------------
__device__ bool warp_gj(double *A, int n, int *perm, double &lnd, double &sg, int lane) {
  lnd = 0;
  sg = 1;
  for (int k = 0; k < n; k++) {
    double best = -1.0;
    int bi = k;
    for (int i = k + lane; i < n; i += 32) {
      double v = fabs(A[i * n + k]);
      if (v > best) { best = v; bi = i; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(0xffffffffu, best, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (!(best > 0.0)) return false;
    if (bi != k) {
      for (int j = lane; j < n; j += 32) {
        double t = A[k * n + j];
        A[k * n + j] = A[bi * n + j];
        A[bi * n + j] = t;
      }
      sg = -sg;
    }
    if (lane == 0) perm[k] = bi;
    __syncwarp();
    double piv = A[k * n + k];
    lnd += log(fabs(piv));
    if (piv < 0) sg = -sg;
    double pinv = 1.0 / piv;
    __syncwarp();
    for (int j = lane; j < n; j += 32) A[k * n + j] = (j == k) ? pinv : A[k * n + j] * pinv;
    __syncwarp();
    for (int idx = lane; idx < n * n; idx += 32) {
      int i = idx / n, j = idx - i * n;
      if (i != k && j != k) A[idx] -= A[i * n + k] * A[k * n + j];
    }
    __syncwarp();
    for (int i = lane; i < n; i += 32)
      if (i != k) A[i * n + k] = -A[i * n + k] * pinv;
    __syncwarp();
  }
  for (int k = n - 1; k >= 0; k--) {
    int p = perm[k];
    if (p != k)
      for (int i = lane; i < n; i += 32) {
        double t = A[i * n + k];
        A[i * n + k] = A[i * n + p];
        A[i * n + p] = t;
      }
    __syncwarp();
  }
  return true;
}

// (2L+1) P_L(x) (yl0, qmc/vmc/nonloc.f90:249-274)
__device__ __forceinline__ double yl0(int L, double x) {
  if (L == 0) return 1.0;
  double p0 = 1, p1 = x;
  for (int n = 1; n < L; n++) {
    double p2 = ((2 * n + 1) * x * p1 - n * p0) / (n + 1);
    p0 = p1;
    p1 = p2;
  }
  return (2 * L + 1) * p1;
}

// Gaussian pseudopotential channels at r (getvps_gauss/gauss_pot, readps_gauss.f90:126-165)
__device__ __forceinline__ void ecp_vps(const EcpPar &E, int it, double r, double *vps) {
  r = r > 1e-10 ? r : 1e-10;
  double rsq = r * r;
  for (int l = 0; l < E.npotd[it]; l++) {
    double v = 0;
    for (int i = 0; i < E.nterm[it][l]; i++) {
      int pw = E.pw[it][l][i];
      double p = 1.0;
      if (pw != 2) p = pow(r, (double)(pw - 2));
      v += p * E.coef[it][l][i] * exp(-E.expo[it][l][i] * rsq);
    }
    if (l + 1 == E.lpotp1[it]) v -= E.znuc[it] / r;
    vps[l] = v;
  }
}

// distance of point p to centre c and 1/(1 + scalek r)
template <class T>
__device__ __forceinline__ void cen_dist(const Sys<T> &s, T sk, const double *p, int c, T &r, T &d) {
  const double *cc = s.cent + 3 * c;
  T a = T(p[0] - cc[0]), b = T(p[1] - cc[1]), e = T(p[2] - cc[2]);
  r = tsqrt(a * a + b * b + e * e);
  d = T(1) / (T(1) + sk * r);
}

// Jastrow pair term (e-e + e-e-n) for electron e at xe (distances re[c][2]) and
// electron j at xj (distances rj[c][2]); gradient wrt xe if GRAD.
template <class T, int NORD, bool GRAD>
__device__ __forceinline__ T pair_value(const Sys<T> &s, const JasPar<T> &J, int e, int j, const double *xe,
                                        const T *re, const double *xj, const T *rj, T *g) {
  int isb, ipar;
  T ss;
  pair_class(J, s.nup, e, j, isb, ss, ipar);
  T rv[3] = {T(xe[0] - xj[0]), T(xe[1] - xj[1]), T(xe[2] - xj[2])};
  T rij = tsqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
  T du = T(1) / (T(1) + J.scalek * rij);
  T fu = 0, fuu = 0;
  T f = jas_ee<T, GRAD>(J, isb, ss, ipar, rij, du, fu, fuu);
  if (GRAD) { g[0] = fu * rv[0]; g[1] = fu * rv[1]; g[2] = fu * rv[2]; }
  if (NORD > 1) {
    for (int c = 0; c < s.C; c++) {
      Een<T> o;
      jas_een<T, NORD, GRAD ? 1 : 0>(J, s.ctype[c], rij, du, re[2 * c], re[2 * c + 1], rj[2 * c], rj[2 * c + 1], o);
      f += o.fc;
      if (GRAD) {
        const double *cc = s.cent + 3 * c;
#pragma unroll
        for (int k = 0; k < 3; k++) g[k] += o.fi * T(xe[k] - cc[k]) + o.fu * rv[k];
      }
    }
  }
  return f;
}

// ---------------------------------------------------------------------------------------
// hpsi for one walker (qmc/vmc/hpsi.f90:2-381), warp-cooperative.
// ---------------------------------------------------------------------------------------
struct EvalRes {
  double lnpsi, sign, psij, d2lnpsi, pe, pe_ee, pe_nl, eloc;
  bool singular;
};

template <class T, int NORD>
__device__ void full_eval(const Sys<T> &s, const JasPar<T> &J, const EcpPar &E, const State<T> &st, int w,
                          const View<T> &v, const double *R, int lane, bool outputs, EvalRes &res) {
  const int N = s.N, C = s.C, nmax = s.nmax;
  const double *xs = v.xs;
  T *fso = v.fso;
  const T sk = J.scalek;
  // --- electron-nucleus distance table (distances.f90:16-27)
  for (int i = lane; i < N * C; i += 32) {
    int e = i / C, c = i - e * C;
    T r, d;
    cen_dist(s, sk, xs + 3 * e, c, r, d);
    v.ren[2 * i] = r;
    v.ren[2 * i + 1] = d;
  }
  for (int i = lane; i < 3 * N; i += 32) v.vacc[i] = 0;
  for (int i = lane; i < N; i += 32) v.divj[i] = 0;
  __syncwarp();
  // --- Jastrow (jastrow4.f90) and e-e Coulomb (distances.f90:131-158)
  double fsum = 0, d2j = 0, pe_ee = 0, pe_en = 0;
  const int npair = N * (N - 1) / 2;
  for (int p = lane; p < npair; p += 32) {
    int i = (int)((1.0 + sqrt(1.0 + 8.0 * (double)p)) * 0.5);
    while (i * (i - 1) / 2 > p) i--;
    while ((i + 1) * i / 2 <= p) i++;
    int j = p - i * (i - 1) / 2;
    const double *xi = xs + 3 * i, *xj = xs + 3 * j;
    int isb, ipar;
    T ss;
    pair_class(J, s.nup, i, j, isb, ss, ipar);
    double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
    double rijd = sqrt(dx * dx + dy * dy + dz * dz);
    pe_ee += 1.0 / rijd;
    T rv[3] = {T(dx), T(dy), T(dz)};
    T rij = tsqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
    T du = T(1) / (T(1) + sk * rij);
    T fu, fuu;
    T f = jas_ee<T, true>(J, isb, ss, ipar, rij, du, fu, fuu);
    T gi[3], gj[3];
#pragma unroll
    for (int k = 0; k < 3; k++) { gi[k] = fu * rv[k]; gj[k] = -fu * rv[k]; }
    T d2 = 2 * (fuu + 2 * fu);
    if (NORD > 1) {
      const T *ri_ = v.ren + 2 * C * i, *rj_ = v.ren + 2 * C * j;
      for (int c = 0; c < C; c++) {
        const double *cc = s.cent + 3 * c;
        T ri = ri_[2 * c], rj = rj_[2 * c];
        Een<T> o;
        jas_een<T, NORD, 2>(J, s.ctype[c], rij, du, ri, ri_[2 * c + 1], rj, rj_[2 * c + 1], o);
        f += o.fc;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          gi[k] += o.fi * T(xi[k] - cc[k]) + o.fu * rv[k];
          gj[k] += o.fj * T(xj[k] - cc[k]) - o.fu * rv[k];
        }
        T sp = ri + rj, tm = ri - rj;
        d2 += 2 * (2 * o.fu + o.fi + o.fj) + 2 * o.fuu + o.fii + o.fjj + o.fui * (rij * rij + sp * tm) / (ri * rij) +
              o.fuj * (rij * rij - sp * tm) / (rj * rij);
      }
    }
    fsum += (double)f;
    d2j += (double)d2;
#pragma unroll
    for (int k = 0; k < 3; k++) {
      atomicAdd(&v.vacc[3 * i + k], (double)gi[k]);
      atomicAdd(&v.vacc[3 * j + k], (double)gj[k]);
    }
    atomicAdd(&v.divj[i], 0.5 * (double)d2);
    atomicAdd(&v.divj[j], 0.5 * (double)d2);
    fso[i * N + j] = f;
    fso[j * N + i] = f;
  }
  __syncwarp();
  for (int i = lane; i < N; i += 32) {
    const double *xi = xs + 3 * i;
    T f = 0, d2 = 0, g[3] = {0, 0, 0};
    for (int c = 0; c < C; c++) {
      const double *cc = s.cent + 3 * c;
      T r = v.ren[2 * (i * C + c)], dn = v.ren[2 * (i * C + c) + 1];
      T fi, fii;
      f += jas_en<T, true>(J, s.ctype[c], r, dn, fi, fii);
#pragma unroll
      for (int k = 0; k < 3; k++) g[k] += fi * T(xi[k] - cc[k]);
      d2 += fii + 2 * fi;
      if (s.nloc == 0) {
        double rd = sqrt((xi[0] - cc[0]) * (xi[0] - cc[0]) + (xi[1] - cc[1]) * (xi[1] - cc[1]) +
                         (xi[2] - cc[2]) * (xi[2] - cc[2]));
        pe_en -= s.zc[c] / rd;
      }
    }
    fsum += (double)f;
    d2j += (double)d2;
#pragma unroll
    for (int k = 0; k < 3; k++) v.vacc[3 * i + k] += (double)g[k];
    v.divj[i] += (double)d2;
    fso[i * N + i] = f;
  }
  fsum = warp_sum(fsum);
  d2j = warp_sum(d2j);
  pe_ee = warp_sum(pe_ee);
  pe_en = warp_sum(pe_en);
  __syncwarp();

  // --- orbitals of every electron, Slater matrices (determinant.f90:36-42, t_bld)
  double *ainv = v.ainv;
  T *orb5 = v.orb5;
  for (int e = 0; e < N; e++) {
    int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup, eo = sp ? e - s.nup : e;
    double *A = ainv + (sp ? s.nup * s.nup : 0);
    warp_basis<T, 5>(s, xs + 3 * e, v.phi, lane);
    T *oe = orb5 + (size_t)e * 5 * nmax;
    warp_orbitals<T, 5>(v.phi, s.cref[sp], s.nbasis, n, oe, nmax, lane);
    for (int k = lane; k < n; k += 32) A[eo * n + k] = (double)oe[k];
  }
  __syncwarp();
  double lnd = 0, sgn = 1;
  bool ok = true;
  for (int sp = 0; sp < 2; sp++) {
    int n = sp ? s.ndn : s.nup;
    if (n == 0) continue;
    double l1, s1;
    bool o1 = warp_gj(ainv + (sp ? s.nup * s.nup : 0), n, v.perm, l1, s1, lane);
    ok = ok && o1;
    lnd += l1;
    sgn *= s1;
  }
  // --- grad ln D, lap D / D per electron (determinant.f90:96-150)
  double d2lnd = 0, v2 = 0;
  for (int e = 0; e < N; e++) {
    int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup, eo = sp ? e - s.nup : e;
    const double *A = ainv + (sp ? s.nup * s.nup : 0);
    const T *oe = orb5 + (size_t)e * 5 * nmax;
    double g0 = 0, g1 = 0, g2 = 0, lp = 0;
    for (int k = lane; k < n; k += 32) {
      double a = A[k * n + eo];
      g0 += a * (double)oe[nmax + k];
      g1 += a * (double)oe[2 * nmax + k];
      g2 += a * (double)oe[3 * nmax + k];
      lp += a * (double)oe[4 * nmax + k];
    }
    g0 = warp_sum(g0); g1 = warp_sum(g1); g2 = warp_sum(g2); lp = warp_sum(lp);
    double dvd = lp - (g0 * g0 + g1 * g1 + g2 * g2);
    d2lnd += dvd;
    double vx = v.vacc[3 * e] + g0, vy = v.vacc[3 * e + 1] + g1, vz = v.vacc[3 * e + 2] + g2;
    v2 += vx * vx + vy * vy + vz * vz;
    if (outputs && lane == 0) {
      double *ov = st.o_vel + ((size_t)w * N + e) * 3;
      ov[0] = vx; ov[1] = vy; ov[2] = vz;
      st.o_divv[(size_t)w * N + e] = v.divj[e] + dvd;
    }
  }

  // --- pseudopotential (nonloc_pot.f90, nonloc.f90), quadrature rotated by R
  double vloc = 0, vnl = 0;
  if (s.nloc > 0 && ok) {
    const int B = s.nbasis;
    T *gp = v.gproj;
    // G projected onto the basis: g_e[b] = sum_k coef[b][k] Ainv[k][e] (psp_nonloc_pot_bld)
    for (int e = 0; e < N; e++) {
      int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup, eo = sp ? e - s.nup : e;
      const double *A = ainv + (sp ? s.nup * s.nup : 0);
      const T *cr = s.cref[sp];
      for (int b = lane; b < B; b += 32) {
        double acc = 0;
        for (int k = 0; k < n; k++) acc += (double)cr[b * n + k] * A[k * n + eo];
        gp[(size_t)e * B + b] = (T)acc;
      }
    }
    double *tl = v.nlt;
    int ntask = 0;
    for (int base = 0; base < N * C; base += 32) {
      int idx = base + lane;
      bool nl = false;
      double vps[MAXLCH], r = 0;
      int c = 0;
      if (idx < N * C) {
        int e = idx / C;
        c = idx - e * C;
        const double *cc = s.cent + 3 * c, *xe = xs + 3 * e;
        r = sqrt((xe[0] - cc[0]) * (xe[0] - cc[0]) + (xe[1] - cc[1]) * (xe[1] - cc[1]) +
                 (xe[2] - cc[2]) * (xe[2] - cc[2]));
        int it = s.ctype[c];
        ecp_vps(E, it, r, vps);
        vloc += vps[E.lpotp1[it] - 1];
        for (int l = 0; l < E.npotd[it]; l++)
          if (l + 1 != E.lpotp1[it] && fabs(vps[l]) > 1e-4) nl = true;
      }
      unsigned m = __ballot_sync(0xffffffffu, nl);
      if (nl) {
        int pos = ntask + __popc(m & ((1u << lane) - 1u));
        double *rec = tl + (size_t)pos * NLT;
        rec[0] = (double)idx;
        rec[1] = r;
        for (int l = 0; l < MAXLCH; l++) rec[2 + l] = (l < E.npotd[s.ctype[c]]) ? vps[l] : 0.0;
      }
      ntask += __popc(m);
    }
    vloc = warp_sum(vloc);
    __syncwarp();
    const int nq = E.nquad;
    for (int t = lane; t < ntask * nq; t += 32) {
      int task = t / nq, q = t - task * nq;
      const double *rec = tl + (size_t)task * NLT;
      int idx = (int)rec[0], e = idx / C, c = idx - (idx / C) * C;
      double r = rec[1];
      const double *cc = s.cent + 3 * c, *xe = xs + 3 * e;
      double qv[3];
#pragma unroll
      for (int k = 0; k < 3; k++) qv[k] = R[3 * k] * E.q0[q][0] + R[3 * k + 1] * E.q0[q][1] + R[3 * k + 2] * E.q0[q][2];
      double costh = ((xe[0] - cc[0]) * qv[0] + (xe[1] - cc[1]) * qv[1] + (xe[2] - cc[2]) * qv[2]) / r;
      double xn[3] = {cc[0] + r * qv[0], cc[1] + r * qv[1], cc[2] + r * qv[2]};
      // determinant ratio: orbitals at the point contracted with G
      const T *ge = gp + (size_t)e * B;
      T dr = 0;
      for (int ish = 0; ish < s.nshell; ish++) dr += shell_dot<T>(s, ish, xn, ge);
      // Jastrow ratio (nonlocj, nonloc.f90:432-522)
      double dj = 0;
      for (int j = 0; j < N; j++) {
        if (j == e) continue;
        int isb, ipar;
        T ss;
        pair_class(J, s.nup, e, j, isb, ss, ipar);
        const double *xj = xs + 3 * j;
        T a0 = T(xn[0] - xj[0]), a1 = T(xn[1] - xj[1]), a2 = T(xn[2] - xj[2]);
        T rij = tsqrt(a0 * a0 + a1 * a1 + a2 * a2);
        T du = T(1) / (T(1) + sk * rij);
        T fu, fuu;
        T f = jas_ee<T, false>(J, isb, ss, ipar, rij, du, fu, fuu);
        if (NORD > 1) {
          const T *rj_ = v.ren + 2 * C * j;
          for (int c2 = 0; c2 < C; c2++) {
            T ri, di;
            cen_dist(s, sk, xn, c2, ri, di);
            Een<T> o;
            jas_een<T, NORD, 0>(J, s.ctype[c2], rij, du, ri, di, rj_[2 * c2], rj_[2 * c2 + 1], o);
            f += o.fc;
          }
        }
        dj += (double)f - (double)fso[e * N + j];
      }
      {
        T f = 0;
        for (int c2 = 0; c2 < C; c2++) {
          T ri, di, fi, fii;
          cen_dist(s, sk, xn, c2, ri, di);
          f += jas_en<T, false>(J, s.ctype[c2], ri, di, fi, fii);
        }
        dj += (double)f - (double)fso[e * N + e];
      }
      int it = s.ctype[c];
      double vp = 0;
      for (int l = 0; l < E.npotd[it]; l++)
        if (l + 1 != E.lpotp1[it]) vp += rec[2 + l] * yl0(l, costh);
      vnl += E.wq[q] * exp(dj) * vp * (double)dr;
    }
    vnl = warp_sum(vnl);
  }
  double pe = s.pecent + pe_ee + (s.nloc > 0 ? vloc + vnl : pe_en);
  double d2lnpsi = d2lnd + d2j;
  double eloc = pe - HB * (d2lnpsi + v2);
  if (!ok) eloc = nan("");
  res.lnpsi = lnd + fsum;
  res.sign = ok ? sgn : 0.0;
  res.psij = fsum;
  res.d2lnpsi = d2lnpsi;
  res.pe = pe;
  res.pe_ee = pe_ee;
  res.pe_nl = vnl;
  res.eloc = eloc;
  res.singular = !ok;
  if (lane == 0) {
    st.fsum[w] = fsum;
    st.lnd[w] = ok ? lnd : -INFINITY;
    st.sgn[w] = ok ? sgn : 0.0;
    uint32_t flag = 0;
    if (!ok) flag |= CHAMP_WS_SINGULAR;
    if (!isfinite(eloc) || !isfinite(lnd + fsum)) flag |= CHAMP_WS_NONFINITE;
    st.status[w] = flag;
    if (outputs) {
      st.o_lnpsi[w] = res.lnpsi;
      st.o_sign[w] = res.sign;
      st.o_psij[w] = fsum;
      st.o_d2[w] = d2lnpsi;
      st.o_pe[w] = pe;
      st.o_peee[w] = pe_ee;
      st.o_penl[w] = vnl;
      st.o_eloc[w] = eloc;
    }
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------------------
// single-electron proposal (hpsie, qmc/vmc/hpsie.f90) and acceptance (jassav/detsav)
// ---------------------------------------------------------------------------------------
template <class T, int NORD, bool GRAD>
__device__ void propose(const Sys<T> &s, const JasPar<T> &J, const State<T> &st, int w, const View<T> &v, int e,
                        const double *xn, int lane, double &rho, double &dj, double *grad) {
  const int N = s.N, C = s.C, nmax = s.nmax;
  int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup, eo = sp ? e - s.nup : e;
  const double *A = v.ainv + (sp ? s.nup * s.nup : 0);
  constexpr int NCH = GRAD ? 5 : 1;
  for (int c = lane; c < C; c += 32) {
    T r, d;
    cen_dist(s, J.scalek, xn, c, r, d);
    v.rnew[2 * c] = r;
    v.rnew[2 * c + 1] = d;
  }
  warp_basis<T, NCH>(s, xn, v.phi, lane);
  warp_orbitals<T, NCH>(v.phi, s.cref[sp], s.nbasis, n, v.arow, nmax, lane);
  double r0 = 0, g0 = 0, g1 = 0, g2 = 0;
  for (int k = lane; k < n; k += 32) {
    double a = A[k * n + eo];
    r0 += a * (double)v.arow[k];
    if (GRAD) {
      g0 += a * (double)v.arow[nmax + k];
      g1 += a * (double)v.arow[2 * nmax + k];
      g2 += a * (double)v.arow[3 * nmax + k];
    }
  }
  rho = warp_sum(r0);
  const T *fso = v.fso;
  T *pf = v.pf;
  double d = 0, gj0 = 0, gj1 = 0, gj2 = 0;
  for (int j = lane; j < N; j += 32) {
    if (j == e) continue;
    T g[3];
    T f = pair_value<T, NORD, GRAD>(s, J, e, j, xn, v.rnew, v.xs + 3 * j, v.ren + 2 * C * j, g);
    d += (double)f - (double)fso[e * N + j];
    pf[j] = f;
    if (GRAD) { gj0 += g[0]; gj1 += g[1]; gj2 += g[2]; }
  }
  T fen = 0;
  for (int c = lane; c < C; c += 32) {
    T fi = 0, fii = 0;
    fen += jas_en<T, GRAD>(J, s.ctype[c], v.rnew[2 * c], v.rnew[2 * c + 1], fi, fii);
    if (GRAD) {
      const double *cc = s.cent + 3 * c;
      gj0 += fi * T(xn[0] - cc[0]);
      gj1 += fi * T(xn[1] - cc[1]);
      gj2 += fi * T(xn[2] - cc[2]);
    }
  }
  double fent = warp_sum((double)fen);
  if (lane == 0) {
    pf[e] = (T)fent;
    d += fent - (double)fso[e * N + e];
  }
  dj = warp_sum(d);
  if (GRAD) {
    g0 = warp_sum(g0); g1 = warp_sum(g1); g2 = warp_sum(g2);
    gj0 = warp_sum(gj0); gj1 = warp_sum(gj1); gj2 = warp_sum(gj2);
    grad[0] = gj0 + g0 / rho;
    grad[1] = gj1 + g1 / rho;
    grad[2] = gj2 + g2 / rho;
  }
  __syncwarp();
}

// Sherman-Morrison update of the inverse and Jastrow tables after accepting electron e
// at xn (dete_update/detsav, qmc/dete_mod.f90:165-190; jassav.f90).  The proposed orbital
// row is v.arow (channel 0), the proposed pair values v.pf, distances v.rnew.
template <class T>
__device__ void accept_move(const Sys<T> &s, const State<T> &st, int w, const View<T> &v, int e, const double *xn,
                            double dj, double rho, int lane) {
  const int N = s.N, C = s.C;
  int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup, eo = sp ? e - s.nup : e;
  double *A = v.ainv + (sp ? s.nup * s.nup : 0);
  for (int k = lane; k < n; k += 32) v.colb[k] = A[k * n + eo];
  for (int j = lane; j < n; j += 32) {
    double a = 0;
    for (int k = 0; k < n; k++) a += (double)v.arow[k] * A[k * n + j];
    v.vb[j] = a - (j == eo ? 1.0 : 0.0);
  }
  __syncwarp();
  double rinv = 1.0 / (v.vb[eo] + 1.0);
  for (int idx = lane; idx < n * n; idx += 32) {
    int k = idx / n, j = idx - k * n;
    A[idx] -= v.colb[k] * v.vb[j] * rinv;
  }
  T *fso = v.fso;
  for (int j = lane; j < N; j += 32) {
    T f = v.pf[j];
    fso[e * N + j] = f;
    fso[j * N + e] = f;
  }
  for (int i = lane; i < 2 * C; i += 32) v.ren[2 * C * e + i] = v.rnew[i];
  if (lane < 3) v.xs[3 * e + lane] = xn[lane];
  if (lane == 0) {
    st.fsum[w] += dj;
    st.lnd[w] += log(fabs(rho));
    if (rho < 0) st.sgn[w] = -st.sgn[w];
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------------------
template <class T>
__device__ inline void load_params(const Sys<T> &s, JasPar<T> &J, EcpPar &E) {
  const int *src = (const int *)s.jas;
  int *dst = (int *)&J;
  for (int i = threadIdx.x; i < (int)(sizeof(JasPar<T>) / 4); i += blockDim.x) dst[i] = src[i];
  src = (const int *)s.ecp;
  dst = (int *)&E;
  for (int i = threadIdx.x; i < (int)(sizeof(EcpPar) / 4); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

template <class T, int NORD>
__global__ void __launch_bounds__(128, 4) k_eval(Sys<T> s, State<T> st, Layout L, double r0, double r1, double r2,
                                                 double r3, double r4, double r5, double r6, double r7, double r8,
                                                 int outputs) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const double R[9] = {r0, r1, r2, r3, r4, r5, r6, r7, r8};
  for (int w = blockIdx.x * wpb + wib; w < st.W; w += gridDim.x * wpb) {
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nmax, L.resident != 0);
    for (int i = lane; i < 3 * s.N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * s.N + i];
    __syncwarp();
    EvalRes res;
    full_eval<T, NORD>(s, J, E, st, w, v, R, lane, outputs != 0, res);
    if (L.resident) view_store(v, st, w, s.N, s.C, lane);
  }
}

// The per-call proposal/accept kernels always work on the HBM copy of the state.
template <class T, int NORD>
__global__ void __launch_bounds__(128, 4) k_propose(Sys<T> s, State<T> st, Layout L, int e, const double *xnew,
                                                    double *ratio, double *grad) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nmax = s.nmax;
  for (int w = blockIdx.x * wpb + wib; w < st.W; w += gridDim.x * wpb) {
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nmax, false);
    for (int i = lane; i < 3 * s.N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * s.N + i];
    __syncwarp();
    double xn[3] = {xnew[3 * w], xnew[3 * w + 1], xnew[3 * w + 2]};
    double rho, dj, g[3];
    if (grad)
      propose<T, NORD, true>(s, J, st, w, v, e, xn, lane, rho, dj, g);
    else
      propose<T, NORD, false>(s, J, st, w, v, e, xn, lane, rho, dj, g);
    int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup;
    for (int k = lane; k < n; k += 32) st.pa[(size_t)w * nmax + k] = (double)v.arow[k];
    if (lane == 0) {
      st.pdj[w] = dj;
      st.prho[w] = rho;
      st.piel[w] = e;
      st.pxn[3 * w] = xn[0]; st.pxn[3 * w + 1] = xn[1]; st.pxn[3 * w + 2] = xn[2];
      ratio[w] = rho * exp(dj);
      if (grad) { grad[3 * w] = g[0]; grad[3 * w + 1] = g[1]; grad[3 * w + 2] = g[2]; }
    }
    __syncwarp();
  }
}

template <class T>
__global__ void __launch_bounds__(128, 4) k_accept(Sys<T> s, State<T> st, Layout L, int e, const uint8_t *mask) {
  extern __shared__ __align__(16) char dsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nmax = s.nmax, C = s.C;
  for (int w = blockIdx.x * wpb + wib; w < st.W; w += gridDim.x * wpb) {
    if (!mask[w] || st.piel[w] != e) continue;
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nmax, false);
    int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup;
    for (int k = lane; k < n; k += 32) v.arow[k] = (T)st.pa[(size_t)w * nmax + k];
    for (int i = lane; i < 3 * s.N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * s.N + i];
    double xn[3] = {st.pxn[3 * w], st.pxn[3 * w + 1], st.pxn[3 * w + 2]};
    for (int c = lane; c < C; c += 32) {
      T r, d;
      const double *cc = s.cent + 3 * c;
      T a = T(xn[0] - cc[0]), b = T(xn[1] - cc[1]), z = T(xn[2] - cc[2]);
      r = tsqrt(a * a + b * b + z * z);
      d = T(1) / (T(1) + (T)s.scalek * r);
      v.rnew[2 * c] = r;
      v.rnew[2 * c + 1] = d;
    }
    __syncwarp();
    accept_move<T>(s, st, w, v, e, xn, st.pdj[w], st.prho[w], lane);
    if (lane < 3) st.x[(size_t)w * 3 * s.N + 3 * e + lane] = xn[lane];
    if (lane == 0) st.piel[w] = -1;
    __syncwarp();
  }
}

// Fused VMC: nsweep sweeps of single-electron Metropolis moves plus E_L after each sweep.
template <class T, int NORD>
__global__ void __launch_bounds__(128, 4) k_vmc(Sys<T> s, State<T> st, Layout L, int nsweep, uint64_t seed,
                                                uint64_t sweep0, double step) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int N = s.N;
  for (int w = blockIdx.x * wpb + wib; w < st.W; w += gridDim.x * wpb) {
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nmax, L.resident != 0);
    if (L.resident) {
      view_load(v, st, w, N, s.C, lane);
    } else {
      for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
      __syncwarp();
    }
    double es = 0, e2 = 0, acc = 0, el = 0;
    for (int isw = 0; isw < nsweep; isw++) {
      uint64_t sweep = sweep0 + (uint64_t)isw;
      for (int e = 0; e < N; e++) {
        double g[3], ua;
        move_randoms(seed, (uint32_t)w, sweep, (uint32_t)e, g, &ua);
        double xn[3] = {v.xs[3 * e] + step * g[0], v.xs[3 * e + 1] + step * g[1], v.xs[3 * e + 2] + step * g[2]};
        double rho, dj, gr[3];
        propose<T, NORD, false>(s, J, st, w, v, e, xn, lane, rho, dj, gr);
        double p = rho * rho * exp(2.0 * dj);
        if (ua < p) {
          accept_move<T>(s, st, w, v, e, xn, dj, rho, lane);
          acc += 1;
        }
      }
      double R[9];
      random_rotation(seed, (uint32_t)w, sweep, R);
      EvalRes res;
      full_eval<T, NORD>(s, J, E, st, w, v, R, lane, false, res);
      el = res.eloc;
      es += el;
      e2 += el * el;
    }
    if (L.resident) {
      view_store(v, st, w, N, s.C, lane);
    } else {
      for (int i = lane; i < 3 * N; i += 32) st.x[(size_t)w * 3 * N + i] = v.xs[i];
    }
    if (lane == 0) {
      st.s_esum[w] = es;
      st.s_e2sum[w] = e2;
      st.s_acc[w] = acc;
      st.s_elast[w] = el;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
static thread_local std::string g_err;
static int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}
#define CK(call)                                                                               \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return fail(CHAMP_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Largest per-warp shared-memory footprint for which a walker's state stays resident in
// shared memory inside the fused kernels (keeps >= 16 warps per SM).
constexpr size_t RESIDENT_LIMIT = 12 * 1024;

struct champ_ctx {
  int prec = 0;
  cudaStream_t stream = nullptr;
  int wmax = 0, W = 0;
  int N = 0, nup = 0, ndn = 0, C = 0, nct = 0, nshell = 0, nbasis = 0, nmax = 0, nordc = 0, nloc = 0;
  std::vector<void *> allocs;
  Sys<double> sd;
  Sys<float> sf;
  State<double> std_;
  State<float> stf;
  double rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  bool have_walkers = false;
  int wpb = 4;
  size_t smem = 0;
  Layout lay;
  // device staging for per-call host arrays
  double *d_in = nullptr, *d_out = nullptr;
  uint8_t *d_mask = nullptr;
  int nparm_jas = 0;
};

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

// cuspinit4 + cuspexact4 (qmc/fit/cuspinit4.f90:1-60, qmc/fit/cuspexact4.f90:14-40)
static void host_een_cusp(int nordc, int nct, int nt, std::vector<double> &c) {
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
  T *cr0 = dalloc<T>(c, (size_t)c->nbasis * std::max(1, c->nup));
  T *cr1 = dalloc<T>(c, (size_t)c->nbasis * std::max(1, c->ndn));
  JasPar<T> *jp = dalloc<JasPar<T>>(c, 1);
  EcpPar *ep = dalloc<EcpPar>(c, 1);
  if (!cent || !ctype || !zc || !sh || !shp || !shb0 || !pz || !pc || !cr0 || !cr1 || !jp || !ep)
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
    int n = sp ? c->ndn : c->nup, off = sp ? c->nup : 0;
    crv[sp].assign((size_t)c->nbasis * std::max(1, n), T(0));
    for (int k = 0; k < n; k++) {
      int o = d->det_orb[off + k];
      for (int b = 0; b < c->nbasis; b++) crv[sp][(size_t)b * n + k] = (T)d->coef[(size_t)o * c->nbasis + perm_b[b]];
    }
  }
  JasPar<T> J;
  memset(&J, 0, sizeof J);
  J.scalek = (T)d->scalek; J.norda = d->norda; J.nordb = d->nordb; J.nspin2b = d->nspin2b; J.nct = c->nct;
  int nt = (int)(cfull.size() / std::max(1, c->nct));
  for (int it = 0; it < c->nct; it++) {
    for (int k = 0; k <= d->norda; k++) J.a4[it][k] = (T)d->a4[it * (d->norda + 1) + k];
    for (int k = 0; k < nt; k++) J.c[it][k] = (T)cfull[(size_t)it * nt + k];
    J.asymp_a[it] = (T)asymp_a[it];
  }
  for (int is = 0; is < d->nspin2b; is++)
    for (int k = 0; k <= d->nordb; k++) J.b[is][k] = (T)d->b[is * (d->nordb + 1) + k];
  J.asymp_b[0] = (T)asymp_b[0]; J.asymp_b[1] = (T)asymp_b[1];
  std::vector<int> ctv(d->iwctype, d->iwctype + c->C);
  CK(cudaMemcpy(cent, d->cent, sizeof(double) * 3 * c->C, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctype, ctv.data(), sizeof(int) * c->C, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(zc, zcv.data(), sizeof(double) * c->C, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sh, shv.data(), sizeof(int4) * c->nshell, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(shp, shpv.data(), sizeof(int2) * c->nshell, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(shb0, shb0v.data(), sizeof(int) * c->nshell, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(pz, pzv.data(), sizeof(T) * nprim, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(pc, pcv.data(), sizeof(T) * nprim, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(cr0, crv[0].data(), sizeof(T) * crv[0].size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(cr1, crv[1].data(), sizeof(T) * crv[1].size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(jp, &J, sizeof J, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ep, &ecp, sizeof ecp, cudaMemcpyHostToDevice));
  s.cent = cent; s.ctype = ctype; s.zc = zc; s.shell = sh; s.shprim = shp; s.shb0 = shb0;
  s.pz = pz; s.pc = pc; s.cref[0] = cr0; s.cref[1] = cr1; s.jas = jp; s.ecp = ep;
  return CHAMP_OK;
}

template <class T>
static int build_state(champ_ctx *c, State<T> &st) {
  size_t W = c->wmax, N = c->N;
  st.W = 0;
  st.astride = c->nup * c->nup + c->ndn * c->ndn;
  st.x = dalloc<double>(c, W * N * 3);
  st.ainv = dalloc<double>(c, W * st.astride);
  st.fso = dalloc<T>(c, W * N * N);
  st.ren = dalloc<T>(c, W * N * c->C * 2);
  st.fsum = dalloc<double>(c, W); st.lnd = dalloc<double>(c, W); st.sgn = dalloc<double>(c, W);
  st.status = dalloc<uint32_t>(c, W);
  st.pf = dalloc<T>(c, W * N);
  st.pa = dalloc<double>(c, W * c->nmax);
  st.pdj = dalloc<double>(c, W); st.prho = dalloc<double>(c, W); st.pxn = dalloc<double>(c, 3 * W);
  st.piel = dalloc<int>(c, W);
  st.orb5 = dalloc<T>(c, W * N * 5 * c->nmax);
  st.gproj = c->nloc > 0 ? dalloc<T>(c, W * N * c->nbasis) : nullptr;
  st.nlt = c->nloc > 0 ? dalloc<double>(c, W * N * c->C * NLT) : nullptr;
  st.o_lnpsi = dalloc<double>(c, W); st.o_sign = dalloc<double>(c, W); st.o_psij = dalloc<double>(c, W);
  st.o_vel = dalloc<double>(c, W * N * 3); st.o_divv = dalloc<double>(c, W * N); st.o_d2 = dalloc<double>(c, W);
  st.o_pe = dalloc<double>(c, W); st.o_peee = dalloc<double>(c, W); st.o_penl = dalloc<double>(c, W);
  st.o_eloc = dalloc<double>(c, W);
  st.s_esum = dalloc<double>(c, W); st.s_e2sum = dalloc<double>(c, W); st.s_acc = dalloc<double>(c, W);
  st.s_elast = dalloc<double>(c, W);
  if (!st.x || !st.ainv || !st.fso || !st.ren || !st.orb5 || !st.s_elast || (c->nloc > 0 && (!st.gproj || !st.nlt)))
    return fail(CHAMP_ENOMEM, "device allocation of the walker state failed");
  return CHAMP_OK;
}

// ---- kernel dispatch over (precision, e-e-n order)
template <class T, int NORD>
static int set_smem_attrs(champ_ctx *c) {
  int sm = (int)c->smem;
  CK(cudaFuncSetAttribute(k_eval<T, NORD>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CK(cudaFuncSetAttribute(k_propose<T, NORD>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CK(cudaFuncSetAttribute(k_accept<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CK(cudaFuncSetAttribute(k_vmc<T, NORD>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  const int co = cudaSharedmemCarveoutMaxShared;
  CK(cudaFuncSetAttribute(k_eval<T, NORD>, cudaFuncAttributePreferredSharedMemoryCarveout, co));
  CK(cudaFuncSetAttribute(k_propose<T, NORD>, cudaFuncAttributePreferredSharedMemoryCarveout, co));
  CK(cudaFuncSetAttribute(k_accept<T>, cudaFuncAttributePreferredSharedMemoryCarveout, co));
  CK(cudaFuncSetAttribute(k_vmc<T, NORD>, cudaFuncAttributePreferredSharedMemoryCarveout, co));
  return CHAMP_OK;
}

template <class T>
static Sys<T> &sysof(champ_ctx *c);
template <>
Sys<double> &sysof<double>(champ_ctx *c) { return c->sd; }
template <>
Sys<float> &sysof<float>(champ_ctx *c) { return c->sf; }
template <class T>
static State<T> &stof(champ_ctx *c);
template <>
State<double> &stof<double>(champ_ctx *c) { return c->std_; }
template <>
State<float> &stof<float>(champ_ctx *c) { return c->stf; }

static int nblocks(champ_ctx *c) { return (c->W + c->wpb - 1) / c->wpb; }

enum class Op { Eval, EvalOut, Propose, ProposeGrad, Accept, Vmc };
struct OpArgs {
  int e = 0;
  const double *xnew = nullptr;
  double *ratio = nullptr, *grad = nullptr;
  const uint8_t *mask = nullptr;
  int nsweep = 0;
  uint64_t seed = 0, sweep0 = 0;
  double step = 0;
};

template <class T, int NORD>
static int launch_t(champ_ctx *c, Op op, const OpArgs &a) {
  Sys<T> &s = sysof<T>(c);
  State<T> st = stof<T>(c);
  st.W = c->W;
  dim3 grid(nblocks(c)), block(32 * c->wpb);
  const double *R = c->rot;
  switch (op) {
  case Op::Eval:
  case Op::EvalOut:
    k_eval<T, NORD><<<grid, block, c->smem, c->stream>>>(s, st, c->lay, R[0], R[1], R[2], R[3], R[4], R[5], R[6], R[7], R[8],
                                                       op == Op::EvalOut ? 1 : 0);
    break;
  case Op::Propose:
  case Op::ProposeGrad:
    k_propose<T, NORD><<<grid, block, c->smem, c->stream>>>(s, st, c->lay, a.e, a.xnew, a.ratio, op == Op::ProposeGrad ? a.grad : nullptr);
    break;
  case Op::Accept:
    k_accept<T><<<grid, block, c->smem, c->stream>>>(s, st, c->lay, a.e, a.mask);
    break;
  case Op::Vmc:
    k_vmc<T, NORD><<<grid, block, c->smem, c->stream>>>(s, st, c->lay, a.nsweep, a.seed, a.sweep0, a.step);
    break;
  }
  CK(cudaGetLastError());
  return CHAMP_OK;
}

template <class T>
static int launch_p(champ_ctx *c, Op op, const OpArgs &a) {
  switch (c->nordc) {
  case 0: case 1: return launch_t<T, 0>(c, op, a);
  case 4: return launch_t<T, 4>(c, op, a);
  case 5: return launch_t<T, 5>(c, op, a);
  default: return fail(CHAMP_EINVAL, "nordc must be 0, 1, 4 or 5");
  }
}
static int launch(champ_ctx *c, Op op, const OpArgs &a = OpArgs()) {
  return c->prec == CHAMP_PREC_FP64 ? launch_p<double>(c, op, a) : launch_p<float>(c, op, a);
}

template <class T>
static int attrs_p(champ_ctx *c) {
  switch (c->nordc) {
  case 0: case 1: return set_smem_attrs<T, 0>(c);
  case 4: return set_smem_attrs<T, 4>(c);
  case 5: return set_smem_attrs<T, 5>(c);
  default: return fail(CHAMP_EINVAL, "nordc must be 0, 1, 4 or 5");
  }
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
  if (d->ndet != 1) return fail(CHAMP_EINVAL, "this build evaluates single-determinant wave functions (ndet == 1)");
  if (d->norda > MAXORD - 1 || d->nordb > MAXORD - 1) return fail(CHAMP_EINVAL, "norda/nordb > 7");
  if (!(d->nordc == 0 || d->nordc == 1 || d->nordc == 4 || d->nordc == 5)) return fail(CHAMP_EINVAL, "nordc must be 0, 1, 4 or 5");
  if (d->nloc != 0 && d->nloc != 6) return fail(CHAMP_EINVAL, "nloc must be 0 or 6");
  if (d->nloc == 6 && d->nquad != 12) return fail(CHAMP_EINVAL, "nquad must be 12");
  if (d->nloc == 6 && d->mgauss > MG) return fail(CHAMP_EINVAL, "more than 4 Gaussian terms per channel");
  if (precision != CHAMP_PREC_FP64 && precision != CHAMP_PREC_MIXED) return fail(CHAMP_EINVAL, "bad precision");
  for (int i = 0; i < d->nshell; i++)
    if (d->shell_l[i] < 0 || d->shell_l[i] > CHAMP_MAX_L || d->shell_n[i] < 1) return fail(CHAMP_EINVAL, "shell with bad n or l");
  champ_ctx *c = new champ_ctx();
  c->prec = precision;
  c->stream = (cudaStream_t)stream;
  c->wmax = w_max;
  c->N = d->nelec; c->nup = d->nup; c->ndn = d->nelec - d->nup; c->C = d->ncent; c->nct = d->nctype;
  c->nshell = d->nshell; c->nbasis = d->nbasis; c->nmax = std::max(1, std::max(c->nup, c->ndn));
  c->nordc = d->nordc; c->nloc = d->nloc;
  // normalised primitive weights (basis_norm)
  std::vector<double> pcn;
  for (int i = 0, p = 0; i < d->nshell; i++)
    for (int q = 0; q < d->shell_nprim[i]; q++, p++)
      pcn.push_back(d->prim_coef[p] * host_anorm(d->shell_kind[i], d->shell_n[i], d->shell_l[i], d->prim_zeta[p]));
  // e-e-n coefficients with the cusp conditions applied
  int nt = 0;
  for (int n = 2; n <= d->nordc; n++)
    for (int k = n - 1; k >= 0; k--) {
      int l_hi = (k == 0) ? n - k - 2 : n - k;
      for (int l = l_hi; l >= 0; l--) if (((n - k - l) & 1) == 0) nt++;
    }
  std::vector<double> cfull((size_t)d->nctype * std::max(nt, 1), 0.0);
  if (nt) memcpy(cfull.data(), d->c, sizeof(double) * d->nctype * nt);
  if (d->een_cusp) host_een_cusp(d->nordc, d->nctype, nt, cfull);
  if (nt == 0) cfull.assign(d->nctype, 0.0);
  // asymptotic values for isc=4 (set_scale_dist, scale_dist.f90:147-225)
  double ar = 1.0 / d->scalek, asa[MAXCT] = {0}, asb[2] = {0, 0};
  for (int it = 0; it < d->nctype; it++) {
    const double *a = d->a4 + it * (d->norda + 1);
    double v = a[0] * ar / (1 + a[1] * ar);
    for (int k = 2; k <= d->norda; k++) v += a[k] * std::pow(ar, k);
    asa[it] = v;
  }
  for (int i = 0; i < 2; i++) {
    double ss = (i == 1 && d->nspin2b == 1) ? 0.5 : 1.0;
    int isp = (i == 1) ? d->nspin2b - 1 : 0;
    const double *b = d->b + isp * (d->nordb + 1);
    double v = ss * b[0] * ar / (1 + b[1] * ar);
    for (int k = 2; k <= d->nordb; k++) v += b[k] * std::pow(ar, k);
    asb[i] = v;
  }
  // pseudopotential and quadrature (rotqua.f90 icosahedral rule)
  EcpPar ecp;
  memset(&ecp, 0, sizeof ecp);
  ecp.nquad = 12;
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
  {
    const double pi = 3.141592653589793, zr = 1.0 / std::sqrt(5.0), rr = 2.0 / std::sqrt(5.0);
    ecp.q0[0][0] = 0; ecp.q0[0][1] = 0; ecp.q0[0][2] = 1;
    ecp.q0[1][0] = 0; ecp.q0[1][1] = 0; ecp.q0[1][2] = -1;
    for (int k = 0; k < 5; k++) {
      double a = 2 * pi * k / 5.0, b = a + pi / 5.0;
      ecp.q0[2 + k][0] = rr * std::cos(a); ecp.q0[2 + k][1] = rr * std::sin(a); ecp.q0[2 + k][2] = zr;
      ecp.q0[7 + k][0] = rr * std::cos(b); ecp.q0[7 + k][1] = rr * std::sin(b); ecp.q0[7 + k][2] = -zr;
    }
    for (int k = 0; k < 12; k++) ecp.wq[k] = 1.0 / 12.0;
  }
  double pecent = 0;
  for (int i = 0; i < d->ncent; i++)
    for (int j = 0; j < i; j++) {
      double dx = d->cent[3 * i] - d->cent[3 * j], dy = d->cent[3 * i + 1] - d->cent[3 * j + 1],
             dz = d->cent[3 * i + 2] - d->cent[3 * j + 2];
      pecent += d->znuc[d->iwctype[i]] * d->znuc[d->iwctype[j]] / std::sqrt(dx * dx + dy * dy + dz * dz);
    }
  int rc;
  if (precision == CHAMP_PREC_FP64) {
    rc = build_sys<double>(c, d, pcn, cfull, asa, asb, ecp, pecent, c->sd);
    if (!rc) rc = build_state<double>(c, c->std_);
    c->lay = make_layout<double>(c->N, c->C, c->nbasis, c->nmax, c->std_.astride, c->nloc > 0, RESIDENT_LIMIT);
    c->smem = c->lay.bytes;
  } else {
    rc = build_sys<float>(c, d, pcn, cfull, asa, asb, ecp, pecent, c->sf);
    if (!rc) rc = build_state<float>(c, c->stf);
    c->lay = make_layout<float>(c->N, c->C, c->nbasis, c->nmax, c->stf.astride, c->nloc > 0, RESIDENT_LIMIT);
    c->smem = c->lay.bytes;
  }
  if (rc) { champ_destroy(c); return rc; }
  // warps per block: up to 8, keeping the block's dynamic shared memory under 96 KB
  c->wpb = 4;  // 128-thread blocks (the kernels' launch bounds)
  while (c->wpb > 1 && c->smem * c->wpb > 96 * 1024) c->wpb >>= 1;
  if (c->smem * c->wpb > 200 * 1024) { champ_destroy(c); return fail(CHAMP_EINVAL, "system too large for the per-warp shared memory"); }
  c->smem *= c->wpb;
  rc = c->prec == CHAMP_PREC_FP64 ? attrs_p<double>(c) : attrs_p<float>(c);
  if (rc) { champ_destroy(c); return rc; }
  c->d_in = dalloc<double>(c, (size_t)w_max * 3 * c->N);
  c->d_out = dalloc<double>(c, (size_t)w_max * 4 * c->N);
  c->d_mask = dalloc<uint8_t>(c, w_max);
  if (!c->d_in || !c->d_out || !c->d_mask) { champ_destroy(c); return fail(CHAMP_ENOMEM, "staging allocation failed"); }
  *out = c;
  return CHAMP_OK;
}

int champ_destroy(champ_ctx *c) {
  if (!c) return CHAMP_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  else cudaDeviceSynchronize();
  for (void *p : c->allocs) cudaFree(p);
  delete c;
  return CHAMP_OK;
}

int champ_nparam(const champ_ctx *c, int32_t *nj, int32_t *ncsf, int32_t *norb) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  if (nj) *nj = c->nparm_jas;
  if (ncsf) *ncsf = 0;
  if (norb) *norb = 0;
  return CHAMP_OK;
}

static double *state_x(champ_ctx *c) { return c->prec == CHAMP_PREC_FP64 ? c->std_.x : c->stf.x; }

int champ_set_walkers(champ_ctx *c, int32_t nw, const double *x) {
  if (!c || !x) return fail(CHAMP_EINVAL, "null argument");
  if (nw < 1 || nw > c->wmax) return fail(CHAMP_EINVAL, "nw out of range");
  c->W = nw;
  CK(cudaMemcpyAsync(state_x(c), x, sizeof(double) * nw * 3 * c->N, cudaMemcpyHostToDevice, c->stream));
  int *piel = c->prec == CHAMP_PREC_FP64 ? c->std_.piel : c->stf.piel;
  CK(cudaMemsetAsync(piel, 0xFF, sizeof(int) * nw, c->stream));
  int rc = launch(c, Op::Eval);
  if (rc) return rc;
  c->have_walkers = true;
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
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
    rc = c->prec == CHAMP_PREC_FP64 ? copy_eval_out<double>(c, o) : copy_eval_out<float>(c, o);
    if (rc) return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
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
    rc = c->prec == CHAMP_PREC_FP64 ? copy_stats<double>(c, stats) : copy_stats<float>(c, stats);
    if (rc) return rc;
    CK(cudaStreamSynchronize(c->stream));
  }
  return CHAMP_OK;
}

int champ_vmc_run_host(champ_ctx *c, int32_t nw, double *x, int32_t nsweep, uint64_t seed, uint64_t sweep0,
                       double step, double *eloc) {
  if (!c || !x || !eloc) return fail(CHAMP_EINVAL, "null argument");
  if (nw < 1 || nw > c->wmax) return fail(CHAMP_EINVAL, "nw out of range");
  c->W = nw;
  CK(cudaMemcpyAsync(state_x(c), x, sizeof(double) * nw * 3 * c->N, cudaMemcpyHostToDevice, c->stream));
  int rc = launch(c, Op::Eval);
  if (rc) return rc;
  c->have_walkers = true;
  champ_vmc_stats st = {nullptr, nullptr, nullptr, nullptr};
  rc = champ_vmc_sweeps(c, nsweep, seed, sweep0, step, &st);
  if (rc) return rc;
  double *el = c->prec == CHAMP_PREC_FP64 ? c->std_.s_elast : c->stf.s_elast;
  CK(cudaMemcpyAsync(eloc, el, sizeof(double) * nw, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(x, state_x(c), sizeof(double) * nw * 3 * c->N, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
}

int champ_walker_status(champ_ctx *c, uint32_t *flags) {
  if (!c || !flags) return fail(CHAMP_EINVAL, "null argument");
  uint32_t *s = c->prec == CHAMP_PREC_FP64 ? c->std_.status : c->stf.status;
  CK(cudaMemcpyAsync(flags, s, sizeof(uint32_t) * c->W, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
}

int champ_synchronize(champ_ctx *c) {
  if (!c) return fail(CHAMP_EINVAL, "null context");
  CK(cudaStreamSynchronize(c->stream));
  return CHAMP_OK;
}

}  // extern "C"
