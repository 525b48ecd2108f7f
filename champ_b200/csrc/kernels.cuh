// kernels.cuh -- walker-batched Slater-Jastrow engine: state layout and kernels.
//
// One warp owns one walker.  Walker state lives in HBM, walker-major:
//   x[w][e][3] (double), ainv[w][spin block][k][e] (double, reference-determinant inverse),
//   fso[w][i][j] (T, Jastrow pair table: i != j pair term incl. e-e-n, i == j e-n term),
//   ln|D|, sign, J per walker.
// Per-warp scratch (basis values, proposed orbital row, gradient accumulators) lives in
// shared memory; larger per-walker scratch (orbitals of all electrons, projected
// coefficients, pseudopotential task lists) in HBM.
#pragma once
#include <type_traits>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
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
  // the FP64 state's orbital rows [W][N][5][nomax] (value, gradient, Laplacian at each electron's
  // position), current for the positions, for the accelerated mover's drift at the current
  // position (kept current by its accepted moves); null when not current
  double *orb_cache = nullptr;
  double *ainv;    // [W][astride]; spin-up block at 0 (nup x nup), spin-down at nup*nup
  T *fso;          // [W][N][N]
  T *ren;          // [W][N][C][2]: r_en and 1/(1 + scalek r_en)
  T *zq;           // [W][N][ZQ]: sum_c (1/(1 + scalek r_en))^q, q = 0..7
  double *fsum, *lnd, *sgn;
  uint32_t *status;
  T *pf;           // [W][N] proposed pair values
  double *pa;      // [W][nomax] proposed orbital row (occupied orbitals)
  double *pdj, *prho, *pxn;  // [W], [W], [W][3]
  int *piel;       // [W]
  T *orb5;         // [W][N][5][nomax]
  T *gproj;        // [W][N][nbasis]
  double *nlt;     // [W][N*C][NLT]
  double *tv;      // [W][tvstride] T = Ainv Atilde restricted to the virtual orbitals, per spin [k][p]
  double *gam;     // [W][gstride] G matrix per spin [m][e] (multi-determinant only)
  double *ymd;     // [W][tvstride] Y scratch [p][k]
  double *wdet;    // [W][2*(ndu0+ndu1)] alpha determinants, then determinant weights
  int astride, tvstride, gstride, wstride;
  // outputs of a full evaluation
  double *o_lnpsi, *o_sign, *o_psij, *o_vel, *o_divv, *o_d2, *o_pe, *o_peee, *o_penl, *o_eloc;
  // VMC accumulators
  double *s_esum, *s_e2sum, *s_acc, *s_elast;
  // mixed precision: the FP32 tables of the single-electron moves ([W][N][N], [W][N][C][2],
  // [W][N][ZQ]), refreshed from the FP64 tables by every full evaluation; null otherwise
  float *m_fso, *m_ren, *m_zq;
  // the moves' scaled e-n distances transposed, [W][C][N] (the pair loads of a proposal read
  // consecutive electrons), kept by the accepted moves; null when unused.  m_rtd: its FP32
  // mirror, refreshed by the full evaluation of a mixed-precision state
  T *rtd;
  float *m_rtd;
  // intermediates of the staged evaluation (elstage.cuh) of a state in HBM; null otherwise:
  // per walker grad ln J and div of the Jastrow velocity [4N], scalars [8] (J, its Laplacian
  // sum, e-e and e-n Coulomb energies, ln|D| and sign(D) of each spin), and the e-n distances
  // as [2][C][N] planes
  double *el_vj, *el_sc;
  T *el_rt;
  // delayed inverse updates of the moves (struct Delay): [W][2][2][dlk_max][nmax] pending terms,
  // dlk terms per flush; null / 0 when the updates are applied at once
  double *dly;
  int dlk, dlk_max;
};
constexpr int NLT = 2 + MAXLCH;  // task record: (e*C+c), r, vps[0..MAXLCH-1]
constexpr int ZQ = 8;            // stride of the per-electron power sums zq
constexpr int MAXC_NL = 64;      // centres for the value-only e-e-n fast path

// Per-warp shared-memory layout, computed on the host.  When `resident` is set the
// walker's whole state and scratch live in shared memory for the life of a kernel
// (small systems); otherwise they stay in HBM.
struct Layout {
  size_t phi, arow, xs, vacc, divj, colb, vb, perm, rnew, asum;  // always in shared memory
  size_t ainv, fso, ren, zq, pf, orb5, gproj, nlt, tv, gam, ymd, wdet;  // resident mode only
  size_t bytes, base;  // total bytes per warp; bytes of the always-shared part
  int resident;
  int coop;            // the FP32 move kernel's warps share the coefficient stream (block_orbitals)
  size_t stage;        // offset of that stream's double buffer in the block's shared memory
};

// Per-walker view: where this walker's arrays live for the current kernel.
template <class T>
struct View {
  T *phi, *arow;
  double *xs, *vacc, *divj, *colb, *vb;
  int *perm;
  T *rnew;         // [C][2] proposed electron's distances to the centres
  T *asum;         // [ZQ] power sums of the proposed electron
  double *ainv;
  T *fso, *ren, *zq, *pf, *orb5, *gproj;
  double *nlt, *tv, *gam, *ymd, *wdet;
  T *rtd;          // [C][N] transposed scaled e-n distances (State::rtd) or null
};

__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// Elements of the per-warp basis scratch: the 5 channels of every basis function, and at least
// 32 per centre (the pseudopotential points' distances to the centres reuse it).
__host__ __device__ inline int phi_count(int nbasis, int C) { return nbasis * 5 > 32 * C ? nbasis * 5 : 32 * C; }

template <class T>
static Layout make_layout(int N, int C, int nbasis, int nmax, int nomax, int astride, int tvstride, int gstride,
                          int wstride, bool nl, size_t resident_limit, bool moves_only = false) {
  // moves_only: the Gaussian single-electron moves of a state in HBM (one basis channel, no
  // velocities); vacc and divj then share phi's place and must not be used
  Layout L{};
  size_t o = 0;
  auto take = [&](size_t b) { size_t r = o; o += align16(b); return r; };
  L.phi = take(sizeof(T) * (moves_only ? (size_t)nbasis : (size_t)phi_count(nbasis, C)));
  L.arow = take(sizeof(T) * 5 * nomax);
  L.xs = take(sizeof(double) * N * 3);
  L.vacc = moves_only ? L.phi : take(sizeof(double) * N * 3);
  L.divj = moves_only ? L.phi : take(sizeof(double) * N);
  L.colb = take(sizeof(double) * nmax);
  L.vb = take(sizeof(double) * nmax);
  L.perm = take(sizeof(int) * nmax);
  L.rnew = take(sizeof(T) * C * 2);
  L.asum = take(sizeof(T) * ZQ);
  size_t base = o;
  L.ainv = take(sizeof(double) * astride);
  L.fso = take(sizeof(T) * N * N);
  L.ren = take(sizeof(T) * N * C * 2);
  L.zq = take(sizeof(T) * N * ZQ);
  L.pf = take(sizeof(T) * N);
  L.orb5 = take(sizeof(T) * N * 5 * nomax);
  L.gproj = nl ? take(sizeof(T) * N * nbasis) : 0;
  L.nlt = nl ? take(sizeof(double) * N * C * NLT) : 0;
  L.tv = take(sizeof(double) * tvstride);
  L.gam = take(sizeof(double) * gstride);
  L.ymd = take(sizeof(double) * tvstride);
  L.wdet = take(sizeof(double) * wstride);
  L.base = base;
  L.resident = (!moves_only && o <= resident_limit) ? 1 : 0;
  L.bytes = L.resident ? o : base;
  return L;
}

template <class T>
__device__ inline View<T> make_view(char *base, const Layout &L, const State<T> &st, int w, int N, int C, int nbasis,
                                    int nomax, bool resident) {
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
  v.asum = (T *)(base + L.asum);
  if (resident) {
    v.ainv = (double *)(base + L.ainv);
    v.fso = (T *)(base + L.fso);
    v.ren = (T *)(base + L.ren);
    v.zq = (T *)(base + L.zq);
    v.pf = (T *)(base + L.pf);
    v.orb5 = (T *)(base + L.orb5);
    v.gproj = (T *)(base + L.gproj);
    v.nlt = (double *)(base + L.nlt);
    v.tv = (double *)(base + L.tv);
    v.gam = (double *)(base + L.gam);
    v.ymd = (double *)(base + L.ymd);
    v.wdet = (double *)(base + L.wdet);
  } else {
    v.ainv = st.ainv + (size_t)w * st.astride;
    v.fso = st.fso + (size_t)w * N * N;
    v.ren = st.ren + (size_t)w * N * C * 2;
    v.zq = st.zq + (size_t)w * N * ZQ;
    v.pf = st.pf + (size_t)w * N;
    v.orb5 = st.orb5 + (size_t)w * N * 5 * nomax;
    v.gproj = st.gproj ? st.gproj + (size_t)w * N * nbasis : nullptr;
    v.nlt = st.nlt ? st.nlt + (size_t)w * N * C * NLT : nullptr;
    v.tv = st.tv + (size_t)w * st.tvstride;
    v.gam = st.gam + (size_t)w * st.gstride;
    v.ymd = st.ymd + (size_t)w * st.tvstride;
    v.wdet = st.wdet + (size_t)w * st.wstride;
  }
  v.rtd = (st.rtd && !resident) ? st.rtd + (size_t)w * C * N : nullptr;
  return v;
}

// Copy a walker's persistent state between HBM and its resident view.
template <class T>
__device__ inline void view_load(const View<T> &v, const State<T> &st, int w, int N, int C, int lane) {
  for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
  for (int i = lane; i < st.astride; i += 32) v.ainv[i] = st.ainv[(size_t)w * st.astride + i];
  for (int i = lane; i < N * N; i += 32) v.fso[i] = st.fso[(size_t)w * N * N + i];
  for (int i = lane; i < N * C * 2; i += 32) v.ren[i] = st.ren[(size_t)w * N * C * 2 + i];
  for (int i = lane; i < N * ZQ; i += 32) v.zq[i] = st.zq[(size_t)w * N * ZQ + i];
  for (int i = lane; i < st.tvstride; i += 32) v.tv[i] = st.tv[(size_t)w * st.tvstride + i];
  for (int i = lane; i < st.gstride; i += 32) v.gam[i] = st.gam[(size_t)w * st.gstride + i];
  __syncwarp();
}
// Mixed precision: after an FP64 full evaluation, the FP32 copies of the Jastrow pair table,
// the e-n distances and the power sums that the single-electron moves read.
template <class T>
__device__ inline void mirror_store(const View<T> &v, const State<T> &st, int w, int N, int C, int lane,
                                    const T *rt = nullptr) {
  if (!st.m_fso) return;
  __syncwarp();
  for (int i = lane; i < N * N; i += 32) st.m_fso[(size_t)w * N * N + i] = (float)v.fso[i];
  for (int i = lane; i < N * C * 2; i += 32) st.m_ren[(size_t)w * N * C * 2 + i] = (float)v.ren[i];
  for (int i = lane; i < N * ZQ; i += 32) st.m_zq[(size_t)w * N * ZQ + i] = (float)v.zq[i];
  if (st.m_rtd) {
    // from the transposed planes when the evaluation has them ([2][C][N], scaled plane second)
    float *m = st.m_rtd + (size_t)w * C * N;
    if (rt)
      for (int i = lane; i < N * C; i += 32) m[i] = (float)rt[(size_t)C * N + i];
    else
      for (int i = lane; i < N * C; i += 32) {
        const int c = i / N, e = i - c * N;
        m[i] = (float)v.ren[2 * (e * C + c) + 1];
      }
  }
  __syncwarp();
}
// The persistent state a full evaluation produces, from a resident view back to HBM: the FP64
// tables, or only their FP32 mirrors when the state has them.
template <class T>
__device__ inline void eval_store(const View<T> &v, const State<T> &st, int w, int N, int C, int lane) {
  __syncwarp();
  for (int i = lane; i < 3 * N; i += 32) st.x[(size_t)w * 3 * N + i] = v.xs[i];
  for (int i = lane; i < st.astride; i += 32) st.ainv[(size_t)w * st.astride + i] = v.ainv[i];
  if (!st.m_fso) {
    for (int i = lane; i < N * N; i += 32) st.fso[(size_t)w * N * N + i] = v.fso[i];
    for (int i = lane; i < N * C * 2; i += 32) st.ren[(size_t)w * N * C * 2 + i] = v.ren[i];
    for (int i = lane; i < N * ZQ; i += 32) st.zq[(size_t)w * N * ZQ + i] = v.zq[i];
  }
  for (int i = lane; i < st.tvstride; i += 32) st.tv[(size_t)w * st.tvstride + i] = v.tv[i];
  for (int i = lane; i < st.gstride; i += 32) st.gam[(size_t)w * st.gstride + i] = v.gam[i];
  __syncwarp();
  mirror_store(v, st, w, N, C, lane);
}
template <class T>
__device__ inline void view_store(const View<T> &v, const State<T> &st, int w, int N, int C, int lane) {
  __syncwarp();
  for (int i = lane; i < 3 * N; i += 32) st.x[(size_t)w * 3 * N + i] = v.xs[i];
  for (int i = lane; i < st.astride; i += 32) st.ainv[(size_t)w * st.astride + i] = v.ainv[i];
  for (int i = lane; i < N * N; i += 32) st.fso[(size_t)w * N * N + i] = v.fso[i];
  for (int i = lane; i < N * C * 2; i += 32) st.ren[(size_t)w * N * C * 2 + i] = v.ren[i];
  for (int i = lane; i < N * ZQ; i += 32) st.zq[(size_t)w * N * ZQ + i] = v.zq[i];
  for (int i = lane; i < st.tvstride; i += 32) st.tv[(size_t)w * st.tvstride + i] = v.tv[i];
  for (int i = lane; i < st.gstride; i += 32) st.gam[(size_t)w * st.gstride + i] = v.gam[i];
  __syncwarp();
}

// ---------------------------------------------------------------------------------------
// warp Gauss-Jordan inversion with partial pivoting, in place (matinv, qmc/vmc/matinv.f90).
// A is row-major n x n (electron row, orbital column); on return it holds the inverse
// indexed [orbital][electron].  Returns false if a pivot is exactly zero.
// ---------------------------------------------------------------------------------------
static __device__ bool warp_gj(double *A, int n, int *perm, double &lnd, double &sg, int lane) {
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
static __device__ __forceinline__ double yl0(int L, double x) {
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
static __device__ __forceinline__ void ecp_vps(const EcpPar &E, int it, double r, double *vps) {
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
                                        const T *re, const double *xj, const T *rj, T *g, const T *ae = nullptr,
                                        const T *zj = nullptr, const T *dj = nullptr, int sdj = 0) {
  int isb, ipar;
  T ss;
  pair_class(J, s.nup, e, j, isb, ss, ipar);
  T rv[3] = {T(xe[0] - xj[0]), T(xe[1] - xj[1]), T(xe[2] - xj[2])};
  T rij = tsqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
  T du = T(1) / (T(1) + J.scalek * rij);
  T fu = 0, fuu = 0;
  T f = jas_ee<T, GRAD>(J, isb, ss, ipar, rij, du, fu, fuu);
  if (GRAD) { g[0] = fu * rv[0]; g[1] = fu * rv[1]; g[2] = fu * rv[2]; }
  if (NORD > 1 && !GRAD && J.nct == 1 && s.C <= MAXC_NL) {
    // value only, one centre type: X sums (see een_xsums)
    T X[make_mixed(NORD).n > 0 ? make_mixed(NORD).n : 1];
    if (dj) een_xsums<T, NORD>(s.C, re + 1, 2, dj, sdj, X);
    else een_xsums<T, NORD>(s.C, re + 1, 2, rj + 1, 2, X);
    f += een_from_x<T, NORD>(J.c[0], du, ae, zj, X);
  } else if (NORD > 1) {
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
// multi-determinant G matrix (deriv_fast_mod.f90: alpha_bld :427, eval_y :545, g_bld :600)
// ---------------------------------------------------------------------------------------
// Determinant (and inverse, row-major, if inv != nullptr) of a k x k matrix, k <= 4.
static __device__ inline double small_det_inv(const double *a0, int k, double *inv) {
  double m[4][8];
  for (int i = 0; i < k; i++)
    for (int j = 0; j < k; j++) {
      m[i][j] = a0[i * k + j];
      m[i][k + j] = (i == j) ? 1.0 : 0.0;
    }
  double det = 1.0;
  for (int c = 0; c < k; c++) {
    int p = c;
    for (int i = c + 1; i < k; i++)
      if (fabs(m[i][c]) > fabs(m[p][c])) p = i;
    if (m[p][c] == 0.0) {
      if (inv)
        for (int i = 0; i < k * k; i++) inv[i] = 0.0;
      return 0.0;
    }
    if (p != c) {
      det = -det;
      for (int j = 0; j < 2 * k; j++) { double t = m[c][j]; m[c][j] = m[p][j]; m[p][j] = t; }
    }
    double pv = m[c][c];
    det *= pv;
    double pi = 1.0 / pv;
    for (int j = 0; j < 2 * k; j++) m[c][j] *= pi;
    for (int i = 0; i < k; i++) {
      if (i == c) continue;
      double f = m[i][c];
      if (f != 0.0)
        for (int j = 0; j < 2 * k; j++) m[i][j] -= f * m[c][j];
    }
  }
  if (inv)
    for (int i = 0; i < k; i++)
      for (int j = 0; j < k; j++) inv[i * k + j] = m[i][k + j];
  return det;
}

template <class T, bool MD>
__device__ __forceinline__ double *gam_ptr(const Sys<T> &s, const View<T> &v, int sp) {
  if (MD) return v.gam + (sp ? s.nocc[0] * s.nup : 0);
  return v.ainv + (sp ? s.nup * s.nup : 0);
}

// alpha_I = T[holes, particles] for unique determinant I of spin sp
template <class T>
__device__ __forceinline__ int load_alpha(const Sys<T> &s, const View<T> &v, int sp, int I, double *a) {
  const int nv = s.nvirt[sp];
  const double *Tv = v.tv + (sp ? s.nup * s.nvirt[0] : 0);
  int k = s.dk[sp][I];
  for (int ia = 0; ia < k; ia++)
    for (int ib = 0; ib < k; ib++) a[ia * k + ib] = Tv[s.dh[sp][4 * I + ia] * nv + s.dpart[sp][4 * I + ib]];
  return k;
}

// From the reference inverses (v.ainv) and T (v.tv): chi = sum_I c_I s_I det(alpha_I^up) det(alpha_I^dn),
// Y = sum_I (c_I s_I det det / chi) alpha_I^-1 scattered to (particle, hole), and
// G = [Ainv - T Y Ainv ; Y Ainv] for both spins.  Returns ln|chi| and sign(chi).
template <class T>
__device__ void build_gamma(const Sys<T> &s, const View<T> &v, int lane, double &lnchi, double &sgnchi) {
  const int nd0 = s.ndu[0], nd1 = s.ndu[1];
  double *wd = v.wdet, *wg = v.wdet + nd0 + nd1;
  for (int sp = 0; sp < 2; sp++)
    for (int I = lane; I < s.ndu[sp]; I += 32) {
      double a[16];
      int k = load_alpha(s, v, sp, I, a);
      wd[(sp ? nd0 : 0) + I] = s.dsg[sp][I] * (k ? small_det_inv(a, k, nullptr) : 1.0);
    }
  for (int i = lane; i < nd0 + nd1; i += 32) wg[i] = 0.0;
  __syncwarp();
  double chi = 0;
  for (int I = lane; I < s.ndet; I += 32) {
    int iu = s.ciu[I], id = s.cid[I];
    double t = s.ccoef[I] * wd[iu] * wd[nd0 + id];
    chi += t;
    atomicAdd(&wg[iu], t);
    atomicAdd(&wg[nd0 + id], t);
  }
  chi = warp_sum(chi);
  __syncwarp();
  double ichi = 1.0 / chi;
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? s.ndn : s.nup, nv = s.nvirt[sp];
    if (n == 0) continue;
    double *Y = v.ymd + (sp ? s.nup * s.nvirt[0] : 0);
    const double *A = v.ainv + (sp ? s.nup * s.nup : 0);
    const double *Tv = v.tv + (sp ? s.nup * s.nvirt[0] : 0);
    double *G = v.gam + (sp ? s.nocc[0] * s.nup : 0);
    for (int i = lane; i < nv * n; i += 32) Y[i] = 0.0;
    __syncwarp();
    for (int I = lane; I < s.ndu[sp]; I += 32) {
      double a[16], inv[16];
      int k = load_alpha(s, v, sp, I, a);
      double wI = wg[(sp ? nd0 : 0) + I] * ichi;
      if (k == 0 || wI == 0.0) continue;
      small_det_inv(a, k, inv);
      for (int ia = 0; ia < k; ia++)
        for (int ib = 0; ib < k; ib++)
          atomicAdd(&Y[s.dpart[sp][4 * I + ib] * n + s.dh[sp][4 * I + ia]], wI * inv[ib * k + ia]);
    }
    __syncwarp();
    for (int i = lane; i < nv * n; i += 32) {
      int p = i / n, e = i - p * n;
      double acc = 0;
      for (int k = 0; k < n; k++) acc += Y[p * n + k] * A[k * n + e];
      G[(n + p) * n + e] = acc;
    }
    __syncwarp();
    for (int i = lane; i < n * n; i += 32) {
      int k = i / n, e = i - k * n;
      double acc = A[i];
      for (int p = 0; p < nv; p++) acc -= Tv[k * nv + p] * G[(n + p) * n + e];
      G[k * n + e] = acc;
    }
    __syncwarp();
  }
  lnchi = log(fabs(chi));
  sgnchi = chi < 0 ? -1.0 : 1.0;
}

// ---------------------------------------------------------------------------------------
// hpsi for one walker (qmc/vmc/hpsi.f90:2-381), warp-cooperative.
// ---------------------------------------------------------------------------------------
struct EvalRes {
  double lnpsi, sign, psij, d2lnpsi, pe, pe_ee, pe_nl, eloc, d2j, vj2;
  double v2;  // |grad ln psi|^2 summed over the electrons
  bool singular;
  int ntask;  // (electron, centre) pairs inside the nonlocal range (task records in the view's nlt)
};

// Shared-memory accumulators of the Jastrow parameter derivatives of one walker.
// Raw parameters: a_k (k = 3..norda+1) per centre type, b_k (k = 2..nordb+1) per b set,
// all e-e-n c terms per centre type.
struct PGBuf {
  double *vt;    // [N*3] grad ln psi
  double *csum;  // [N] sum over the electron's quadrature points of w e^dJ v_l(r) P_l D-ratio
  double *dvn;   // [P] sum over points of that coefficient times the parameter's basis function
  double *G;     // [P] d ln psi / dp
  double *K;     // [P] sum_e (lap_e g_p + 2 v_e . grad_e g_p)
  double *old;   // [N][P] basis function of p summed over the terms involving electron e
  double *dvl;   // [P][32] each lane's part of dvn (summed into dvn after the quadrature loop)
  int P, na, nb;
  double *phis;  // [N][nbasis] or null: sum over the electron's quadrature points of
                 // w e^dJ v_l(r) P_l times each basis function (nonlocal part of B in basis space)
  double *tape;  // [N*C][nquad] or null: the forward pass of the parameter gradient stores each
                 // point's coefficient here (per task and point) instead of adding its parameter sums
};

template <class T, int NORD, bool SLOTS>
__device__ void point_param_values(const Sys<T> &s, const JasPar<T> &J, const View<T> &v, int e, const double *xn,
                                   double coeff, const PGBuf &pg, const T *tsum_pre);

// Multi-determinant tables of one walker from the inverses of the reference determinant:
// T = Ainv Atilde on the virtual columns (t_bld, deriv_fast_mod.f90:367-398), then Y and G
// (build_gamma).  Returns ln|chi| and sign(chi).
template <class T>
__device__ void md_tables(const Sys<T> &s, const View<T> &v, int lane, double &lc, double &sc) {
  const int nomax = s.nomax;
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? s.ndn : s.nup, nv = s.nvirt[sp], e0 = sp ? s.nup : 0;
    const double *A = v.ainv + (sp ? s.nup * s.nup : 0);
    double *Tv = v.tv + (sp ? s.nup * s.nvirt[0] : 0);
    for (int i = lane; i < n * nv; i += 32) {
      int k = i / nv, p = i - k * nv;
      double acc = 0;
      for (int e = 0; e < n; e++) acc += A[k * n + e] * (double)v.orb5[(size_t)(e0 + e) * 5 * nomax + n + p];
      Tv[i] = acc;
    }
  }
  __syncwarp();
  build_gamma(s, v, lane, lc, sc);
}

// Distances to the centres (ren, zq), the Jastrow factor with its gradient (v.vacc) and the
// divergence of its velocity (v.divj) per electron, the pair table fso (jastrow4.f90,
// distances.f90) and the e-e (and, all-electron, e-n) Coulomb energies of one walker.  TR: the
// e-n distances are also written to, and the pair and e-n terms read from, rt = [2][C][N]
// (distance plane, then scaled-distance plane; consecutive electrons adjacent).
// VO: values only -- the tables and the Jastrow sum without the gradient and Laplacian terms (v.vacc
// and v.divj stay zero), for rebuilding the state the moves start from.
template <class T, int NORD, bool TR, bool VO = false>
__device__ void jastrow_tables(const Sys<T> &s, const JasPar<T> &J, const View<T> &v, T *rt, int lane, double &fsum,
                               double &d2j, double &pe_ee, double &pe_en) {
  const int N = s.N, C = s.C;
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
    if (TR) {
      rt[c * N + e] = r;
      rt[(C + c) * N + e] = d;
    }
  }
  __syncwarp();
  for (int e = lane; e < N; e += 32) {
    T z[ZQ];
    z[0] = T(C);
    for (int q = 1; q < ZQ; q++) z[q] = T(0);
    for (int c = 0; c < C; c++) {
      T d = v.ren[2 * (e * C + c) + 1], p = d;
      for (int q = 1; q < ZQ; q++) { z[q] += p; p *= d; }
    }
    for (int q = 0; q < ZQ; q++) v.zq[e * ZQ + q] = z[q];
  }
  for (int i = lane; i < 3 * N; i += 32) v.vacc[i] = 0;
  for (int i = lane; i < N; i += 32) v.divj[i] = 0;
  __syncwarp();
  // --- Jastrow (jastrow4.f90) and e-e Coulomb (distances.f90:131-158)
  fsum = 0, d2j = 0, pe_ee = 0, pe_en = 0;
  // distance of electron e to centre c and its scaled form (TR: from the transposed planes)
  auto rof = [&](int e, int c) -> T { return TR ? rt[c * N + e] : v.ren[2 * (e * C + c)]; };
  auto dof = [&](int e, int c) -> T { return TR ? rt[(C + c) * N + e] : v.ren[2 * (e * C + c) + 1]; };
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
    T f = jas_ee<T, !VO>(J, isb, ss, ipar, rij, du, fu, fuu);
    T gi[3] = {0, 0, 0}, gj[3] = {0, 0, 0}, d2 = 0;
    if constexpr (!VO) {
#pragma unroll
      for (int k = 0; k < 3; k++) { gi[k] = fu * rv[k]; gj[k] = -fu * rv[k]; }
      d2 = 2 * (fuu + 2 * fu);
    }
    if (NORD > 1) {
      for (int c = 0; c < C; c++) {
        const double *cc = s.cent + 3 * c;
        T ri = rof(i, c), rj = rof(j, c);
        Een<T> o;
        jas_een<T, NORD, VO ? 0 : 2>(J, s.ctype[c], rij, du, ri, dof(i, c), rj, dof(j, c), o);
        f += o.fc;
        if constexpr (!VO) {
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
    }
    fsum += (double)f;
    if constexpr (!VO) {
      d2j += (double)d2;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        atomicAdd(&v.vacc[3 * i + k], (double)gi[k]);
        atomicAdd(&v.vacc[3 * j + k], (double)gj[k]);
      }
      atomicAdd(&v.divj[i], 0.5 * (double)d2);
      atomicAdd(&v.divj[j], 0.5 * (double)d2);
    }
    fso[i * N + j] = f;
    fso[j * N + i] = f;
  }
  __syncwarp();
  for (int i = lane; i < N; i += 32) {
    const double *xi = xs + 3 * i;
    T f = 0, d2 = 0, g[3] = {0, 0, 0};
    for (int c = 0; c < C; c++) {
      const double *cc = s.cent + 3 * c;
      T r = rof(i, c), dn = dof(i, c);
      T fi = 0, fii = 0;
      f += jas_en<T, !VO>(J, s.ctype[c], r, dn, fi, fii);
      if constexpr (!VO) {
#pragma unroll
        for (int k = 0; k < 3; k++) g[k] += fi * T(xi[k] - cc[k]);
        d2 += fii + 2 * fi;
      }
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
}

// grad ln D and lap D / D of every electron (determinant.f90:96-150) from G and the orbitals'
// gradients and Laplacians; with the Jastrow velocities in v.vacc gives the velocities, |v|^2
// and sum lap ln D.
template <class T, bool MD, bool PG>
__device__ void det_velocities(const Sys<T> &s, const State<T> &st, int w, const View<T> &v, int lane, bool outputs,
                               const PGBuf *pg, double &d2lnd_o, double &v2_o) {
  const int N = s.N, nomax = s.nomax;
  const T *orb5 = v.orb5;
  double d2lnd = 0, v2 = 0;
  for (int e = 0; e < N; e++) {
    int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup, eo = sp ? e - s.nup : e;
    const double *G = gam_ptr<T, MD>(s, v, sp);
    const T *oe = orb5 + (size_t)e * 5 * nomax;
    double g0 = 0, g1 = 0, g2 = 0, lp = 0;
    for (int k = lane; k < s.nocc[sp]; k += 32) {
      double a = G[k * n + eo];
      g0 += a * (double)oe[nomax + k];
      g1 += a * (double)oe[2 * nomax + k];
      g2 += a * (double)oe[3 * nomax + k];
      lp += a * (double)oe[4 * nomax + k];
    }
    g0 = warp_sum(g0); g1 = warp_sum(g1); g2 = warp_sum(g2); lp = warp_sum(lp);
    double dvd = lp - (g0 * g0 + g1 * g1 + g2 * g2);
    d2lnd += dvd;
    double vx = v.vacc[3 * e] + g0, vy = v.vacc[3 * e + 1] + g1, vz = v.vacc[3 * e + 2] + g2;
    v2 += vx * vx + vy * vy + vz * vz;
    if (PG && lane == 0) {
      pg->vt[3 * e] = vx; pg->vt[3 * e + 1] = vy; pg->vt[3 * e + 2] = vz;
    }
    if (outputs && lane == 0) {
      double *ov = st.o_vel + ((size_t)w * N + e) * 3;
      ov[0] = vx; ov[1] = vy; ov[2] = vz;
      st.o_divv[(size_t)w * N + e] = v.divj[e] + dvd;
    }
  }
  d2lnd_o = d2lnd;
  v2_o = v2;
}

// FP64 tensor-core product D += A B of one 8x8 tile with k = 4 (mma m8n8k4, one element of A and
// of B and two of D per lane: A[lane/4][lane%4], B[lane%4][lane/4], D[lane/4][2(lane%4) + 0, 1]).
__device__ __forceinline__ void dmma_884(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Jastrow ratio terms of 32 quadrature points (one per lane; act false for a lane without one):
// the sum over the other electrons j of the pair term at the point (e-e, and e-e-n from the X
// sums) minus the pair table entry u(e, j) (nonlocj, nonloc.f90:432-522).  The X sums
// X_pq(point, j) = sum_c d_c^p(point) d_c^q(j) of the round are FP64 tensor-core products over
// the centres (KS k-steps of 4 centres, 4 KS >= C): row tiles of 8 points, whose A fragments (the points'
// scaled distances to the centres) each lane forms in registers; column tiles of 8 electrons,
// B fragments from bd (element (c, j) at bd[c sbc + j sbj]).
template <int NORD, int KS>
__device__ double nl_pairs_mma(const Sys<double> &s, const JasPar<double> &J, const View<double> &v,
                               const double *bd, int sbc, int sbj, const double *asum, const double *xn, int e,
                               bool act, int lane) {
  constexpr MixedPQ mx = make_mixed(NORD);
  constexpr int NM = mx.n > 0 ? mx.n : 1;
  const int N = s.N, C = s.C;
  const double sk = J.scalek;
  const unsigned full = 0xffffffffu, am = __ballot_sync(full, act);
  const int kq = lane & 3, rr = lane >> 2;
  double mine = 0;
#pragma unroll 1
  for (int mt = 0; mt < 4; mt++) {
    if (((am >> (8 * mt)) & 0xffu) == 0u) continue;  // no point in this row tile (uniform)
    const int prow = mt * 8 + rr;  // the point (lane) of this lane's fragment row
    const double px = __shfl_sync(full, xn[0], prow), py = __shfl_sync(full, xn[1], prow),
                 pz = __shfl_sync(full, xn[2], prow);
    const int pe = __shfl_sync(full, e, prow);
    const bool pact = (am >> prow) & 1u;
    double pas[NORD + 1];
#pragma unroll
    for (int q = 0; q <= NORD; q++) pas[q] = __shfl_sync(full, asum[q], prow);
    double a1[KS];
#pragma unroll
    for (int ks = 0; ks < KS; ks++) {
      const int ck = 4 * ks + kq;
      a1[ks] = 0.0;
      if (ck < C) {
        const double *cc = s.cent + 3 * ck;
        const double dx = px - cc[0], dy = py - cc[1], dz = pz - cc[2];
        a1[ks] = 1.0 / (1.0 + sk * sqrt(dx * dx + dy * dy + dz * dz));
      }
    }
    double dsum = 0;
    for (int j0 = 0; j0 < N; j0 += 8) {
      const int jb = j0 + rr, ja = j0 + 2 * kq;
      double b1[KS];
#pragma unroll
      for (int ks = 0; ks < KS; ks++) {
        const int ck = 4 * ks + kq;
        b1[ks] = (ck < C && jb < N) ? bd[(size_t)ck * sbc + (size_t)jb * sbj] : 0.0;
      }
      double fo[2];
#pragma unroll
      for (int h = 0; h < 2; h++) fo[h] = (pact && ja + h < N) ? v.fso[pe * N + ja + h] : 0.0;
      double acc[NM][2];
#pragma unroll
      for (int i = 0; i < NM; i++) acc[i][0] = acc[i][1] = 0.0;
#pragma unroll
      for (int ks = 0; ks < KS; ks++) {
        double ap[NORD + 1], bp[NORD + 1];
        ap[0] = bp[0] = 1.0;
#pragma unroll
        for (int q = 1; q <= NORD; q++) { ap[q] = ap[q - 1] * a1[ks]; bp[q] = bp[q - 1] * b1[ks]; }
#pragma unroll
        for (int i = 0; i < mx.n; i++) dmma_884(acc[i][0], acc[i][1], ap[mx.p[i]], bp[mx.q[i]]);
      }
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int j = ja + h;
        if (!pact || j >= N || j == pe) continue;
        int isb, ipar;
        double ss;
        pair_class(J, s.nup, pe, j, isb, ss, ipar);
        const double *xj = v.xs + 3 * j;
        const double d0 = px - xj[0], d1 = py - xj[1], d2 = pz - xj[2];
        const double rij = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        const double du = 1.0 / (1.0 + sk * rij);
        double fu, fuu;
        double f = jas_ee<double, false>(J, isb, ss, ipar, rij, du, fu, fuu);
        double X[NM];
#pragma unroll
        for (int i = 0; i < NM; i++) X[i] = acc[i][h];
        f += een_from_x<double, NORD>(J.c[0], du, pas, v.zq + ZQ * j, X);
        dsum += f - fo[h];
      }
    }
    dsum += __shfl_xor_sync(full, dsum, 1);
    dsum += __shfl_xor_sync(full, dsum, 2);
    const double got = __shfl_sync(full, dsum, 4 * (lane & 7));
    if ((lane >> 3) == mt) mine = got;
  }
  return mine;
}

// Nonlocal pseudopotential energy of one walker (nonloc_pot.f90, nonloc.f90), quadrature rotated
// by R.  scr: nscr elements of per-warp shared scratch, holding the radial parts of the tasks'
// centres' shells and, on the one-centre-type path without the tensor cores, each lane's scaled
// point-centre distances (stored [centre][lane], 32 C elements at the end).  TC: the FP64 X sums
// may run on the tensor cores (compiled only into the staged evaluation, whose registers the
// single-kernel evaluation of small systems does not have to carry).  st_rt: the walker's e-n distance planes
// (State::el_rt) or null.  Returns the local and nonlocal parts and the number of (electron,
// centre) tasks.
template <class T, int NORD, bool MD, bool PG, bool TC = false>
__device__ void nlpp_energy(const Sys<T> &s, const JasPar<T> &J, const EcpPar &E, const View<T> &v, const double *R,
                            int lane, const PGBuf *pg, T *scr, int nscr, const T *st_rt, double &vloc_o, double &vnl_o,
                            int &ntask_o) {
  const int N = s.N, C = s.C, B = s.nbasis;
  const double *xs = v.xs;
  const T *fso = v.fso;
  const T sk = J.scalek;
  // FP64 with 16 to 32 centres and at least 16 electrons: the X sums on the tensor cores (whose
  // tiles of 8 electrons and k-steps of 4 centres smaller systems would mostly leave empty),
  // without the per-lane distances in shared memory; else in each lane from those distances
  // (scratch permitting)
  const bool mma = TC && std::is_same<T, double>::value && NORD > 1 && J.nct == 1 && C >= 16 && C <= 32 && N >= 16;
  const bool fast = mma || ((NORD > 1) && J.nct == 1 && C <= MAXC_NL && nscr >= 32 * C);
  const int nrown = nscr - (fast && !mma ? 32 * C : 0);
  T *const prs = fast && !mma ? scr + nrown + lane : nullptr;  // this lane's point-centre distances, stride 32
  double vloc = 0, vnl = 0;
  T *gp = v.gproj;
  // G projected onto the basis: g_e[b] = sum_k coef[b][k] G[k][e] (psp_nonloc_pot_bld), one
  // [nbasis x nocc] x [nocc x n] product per spin in compute precision: lanes along b over
  // rows of the transposed coefficients (coalesced), 4 electrons x 4 basis functions per lane.
  for (int sp = 0; sp < 2; sp++) {
    const int n = sp ? s.ndn : s.nup, e0 = sp ? s.nup : 0, no = s.nocc[sp];
    const double *G = gam_ptr<T, MD>(s, v, sp);
    const T *ct = s.coccT[sp];
    for (int eo0 = 0; eo0 < n; eo0 += 4) {
      const int ne = min(4, n - eo0);
      for (int b0 = 0; b0 < B; b0 += 128) {
        T acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] = T(0);
        for (int k = 0; k < no; k++) {
          T g[4];
#pragma unroll
          for (int i = 0; i < 4; i++) g[i] = (i < ne) ? (T)G[k * n + eo0 + i] : T(0);
          const T *row = ct + (size_t)k * B + b0 + lane;
#pragma unroll
          for (int j = 0; j < 4; j++) {
            T cf = (b0 + lane + 32 * j < B) ? row[32 * j] : T(0);
#pragma unroll
            for (int i = 0; i < 4; i++) acc[i][j] += cf * g[i];
          }
        }
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) {
            int b = b0 + lane + 32 * j;
            if (i < ne && b < B) gp[(size_t)(e0 + eo0 + i) * B + b] = acc[i][j];
          }
      }
    }
  }
  double *tl = v.nlt;
  int ntask = 0;
  // tasks in centre-major order, so that the points of one round of 32 lanes mostly share
  // their centre (and with it the shells whose radial parts are precomputed per task)
  for (int base = 0; base < N * C; base += 32) {
    const int j = base + lane;
    int idx = j;
    bool nl = false;
    double vps[MAXLCH], r = 0;
    int c = 0;
    if (j < N * C) {
      c = j / N;
      const int e = j - c * N;
      idx = e * C + c;
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
  ntask_o = ntask;
  __syncwarp();
  const int nq = E.nquad;
  // The points of an (electron, centre) task lie at the task's distance r from that centre, so
  // the radial parts of the centre's own shells are evaluated once per task (into the per-warp
  // basis scratch, unused in this phase) when the table fits there.
  const int nshc = (s.nshc > 0 && ntask * s.nshc <= nrown) ? s.nshc : 0;
  T *rown = scr;  // [ntask][nshc]
  if (nshc > 0) {
    for (int i = lane; i < ntask * nshc; i += 32) {
      const int tk = i / nshc, k = i - tk * nshc;
      const double *rc = tl + (size_t)tk * NLT;
      const int ci = (int)rc[0] % C, ish = s.cshell0[ci] + k;
      if (ish < s.cshell0[ci + 1]) {
        T R3[3];
        shell_radial<T, false>(s, ish, (T)rc[1], R3);
        rown[i] = R3[0];
      }
    }
    __syncwarp();
  }
  // rounds of 32 points, one per lane (lanes past the last point repeat the round's first point
  // in the parts that all lanes run together and skip the rest)
  const int npts = ntask * nq;
  for (int t0 = 0; t0 < npts; t0 += 32) {
    const bool act = t0 + lane < npts;
    const int t = act ? t0 + lane : t0;
    int task = t / nq, q = t - task * nq;
    const double *rec = tl + (size_t)task * NLT;
    int idx = (int)rec[0], e = idx / C, c = idx - (idx / C) * C;
    double r = rec[1];
    const double *cc = s.cent + 3 * c, *xe = xs + 3 * e;
    double qv[3];
#pragma unroll
    for (int k = 0; k < 3; k++) qv[k] = R[3 * k] * s.quad->q0[q][0] + R[3 * k + 1] * s.quad->q0[q][1] + R[3 * k + 2] * s.quad->q0[q][2];
    double costh = ((xe[0] - cc[0]) * qv[0] + (xe[1] - cc[1]) * qv[1] + (xe[2] - cc[2]) * qv[2]) / r;
    double xn[3] = {cc[0] + r * qv[0], cc[1] + r * qv[1], cc[2] + r * qv[2]};
    // determinant ratio: orbitals at the point contracted with G
    const T *ge = gp + (size_t)e * B;
    T dr = 0;
    const int c0 = nshc > 0 ? s.cshell0[c] : 0, c1 = nshc > 0 ? s.cshell0[c + 1] : 0;
    const T *ro = rown + task * nshc - c0;
    // with the nonlocal B-matrix sums wanted, the basis values at the point are formed once,
    // after the Jastrow ratio, for both the ratio and those sums
    const bool merged = PG && pg->phis != nullptr;
    if (!merged && act)
      for (int ish = 0; ish < s.nshell; ish++)
        dr += shell_dot_r<T>(s, ish, xn, ge, (ish >= c0 && ish < c1) ? ro + ish : nullptr);
    // Jastrow ratio (nonlocj, nonloc.f90:432-522): point-centre distances once per point
    double dj = 0;
    T asum[ZQ];
    {
      T f = 0;
      for (int q2 = 0; q2 < ZQ; q2++) asum[q2] = (q2 == 0) ? T(C) : T(0);
      for (int c2 = 0; c2 < C; c2++) {
        T ri, di, fi, fii;
        cen_dist(s, sk, xn, c2, ri, di);
        f += jas_en<T, false>(J, s.ctype[c2], ri, di, fi, fii);
        if (fast) {
          if (!mma) prs[32 * c2] = di;
          T p = di;
          for (int q2 = 1; q2 < ZQ; q2++) { asum[q2] += p; p *= di; }
        }
      }
      dj += (double)f - (double)fso[e * N + e];
    }
    // FP32 derivative run: the e-e-n parameter basis functions at the point, summed over the
    // other electrons from the same X sums as the value (handed to point_param_values).  The
    // FP64 run forms them there instead: 13 more FP64 registers here cost it more in spills.
    constexpr bool SHARE = PG && std::is_same<T, float>::value;
    constexpr int NT = make_terms(NORD).n > 0 ? make_terms(NORD).n : 1;
    T tsum[SHARE ? NT : 1];
    if (SHARE)
#pragma unroll
      for (int ll = 0; ll < NT; ll++) tsum[ll] = T(0);
    constexpr bool MMA = TC && std::is_same<T, double>::value && !SHARE;
    if (MMA && mma) {
      if constexpr (MMA) {
        const double *bd = st_rt ? st_rt + (size_t)C * N : v.ren + 1;
        const int sbc = st_rt ? N : 2, sbj = st_rt ? 1 : 2 * C;
        dj += nl_pairs_mma<NORD, 8>(s, J, v, bd, sbc, sbj, asum, xn, e, act, lane);
      }
    }
    for (int j = 0; j < N && act && !(MMA && mma); j++) {
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
      if (fast) {
        T X[make_mixed(NORD).n > 0 ? make_mixed(NORD).n : 1];
        een_xsums<T, NORD>(C, prs, 32, v.ren + 2 * C * j + 1, 2, X);
        if (SHARE) {
          constexpr Terms tl = make_terms(NORD);
          constexpr XIdx xi = make_xidx(NORD);
          const T *zj = v.zq + ZQ * j;
          T uu[NORD + 1];
          uu[0] = T(1);
#pragma unroll
          for (int q2 = 1; q2 <= NORD; q2++) uu[q2] = uu[q2 - 1] * du;
#pragma unroll
          for (int ll = 0; ll < tl.n; ll++) {
            const T t = uu[tl.k[ll]] * (xsel(xi.a1[ll], asum, zj, X) + xsel(xi.a2[ll], asum, zj, X));
            f += J.c[0][ll] * t;
            tsum[ll] += t;
          }
        } else {
          f += een_from_x<T, NORD>(J.c[0], du, asum, v.zq + ZQ * j, X);
        }
      } else if (NORD > 1) {
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
    if (!act) continue;
    int it = s.ctype[c];
    double vp = 0;
    for (int l = 0; l < E.npotd[it]; l++)
      if (l + 1 != E.lpotp1[it]) vp += rec[2 + l] * yl0(l, costh);
    if (merged) {
      const double c2 = s.quad->wq[q] * exp(dj) * vp;
      double *ph = pg->phis + (size_t)e * s.nbasis;
      for (int ish = 0; ish < s.nshell; ish++)
        dr += shell_dot_acc<T>(s, ish, xn, ge, (ish >= c0 && ish < c1) ? ro + ish : nullptr, c2, ph);
    }
    vnl += s.quad->wq[q] * exp(dj) * vp * (double)dr;
    if (PG) {
      double coeff = s.quad->wq[q] * exp(dj) * vp * (double)dr;
      atomicAdd(&pg->csum[e], coeff);
      if (pg->tape) {
        pg->tape[t] = coeff;  // the backward pass forms the parameter sums at this point
      } else {
        const T *ts = (SHARE && fast) ? tsum : nullptr;
        if (pg->dvl) point_param_values<T, NORD, true>(s, J, v, e, xn, coeff, *pg, ts);
        else point_param_values<T, NORD, false>(s, J, v, e, xn, coeff, *pg, ts);
      }
    }
  }
  vnl = warp_sum(vnl);
  if (PG && pg->dvl) {
    __syncwarp();
    for (int p = lane; p < pg->P; p += 32) {
      double a = 0;
      for (int l = 0; l < 32; l++) a += pg->dvl[p * 32 + l];
      pg->dvn[p] += a;
    }
    __syncwarp();
  }
  vloc_o = vloc;
  vnl_o = vnl;
}

// E_L and the outputs of one walker's full evaluation from its parts (hpsi.f90:336-344): the
// walker's log-determinant, Jastrow, status and, with outputs, the per-walker output arrays.
template <class T>
__device__ void finish_eval(const Sys<T> &s, const State<T> &st, int w, const View<T> &v, int lane, bool outputs,
                            bool ok, double lnd, double sgn, double fsum, double d2j, double pe_ee, double pe_en,
                            double d2lnd, double v2, double vloc, double vnl, int ntask_all, EvalRes &res) {
  const int N = s.N;
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
  res.d2j = d2j;
  res.v2 = v2;
  {
    double vj2 = 0;
    for (int i = lane; i < 3 * N; i += 32) vj2 += v.vacc[i] * v.vacc[i];
    res.vj2 = warp_sum(vj2);
  }
  res.singular = !ok;
  res.ntask = ntask_all;
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

template <class T, int NORD, bool MD, bool PG = false>
__device__ void full_eval(const Sys<T> &s, const JasPar<T> &J, const EcpPar &E, const State<T> &st, int w,
                          const View<T> &v, const double *R, int lane, bool outputs, EvalRes &res,
                          const PGBuf *pg = nullptr, bool orbs_ready = false, bool reinvert = true) {
  const int N = s.N, C = s.C, nomax = s.nomax;
  const double *xs = v.xs;
  double fsum, d2j, pe_ee, pe_en;
  jastrow_tables<T, NORD, false>(s, J, v, nullptr, lane, fsum, d2j, pe_ee, pe_en);

  // --- orbitals of every electron, Slater matrices (determinant.f90:36-42, t_bld); with
  // orbs_ready they were computed for all walkers by the tensor-core contraction
  double *ainv = v.ainv;
  T *orb5 = v.orb5;
  for (int e = 0; e < N; e++) {
    int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup, eo = sp ? e - s.nup : e;
    double *A = ainv + (sp ? s.nup * s.nup : 0);
    T *oe = orb5 + (size_t)e * 5 * nomax;
    if (!orbs_ready) {
      warp_basis<T, 5>(s, xs + 3 * e, v.phi, lane);
      warp_orbitals<T, 5>(v.phi, s.cocc[sp], s.nbasis, s.nocc[sp], oe, nomax, lane);
    }
    if (reinvert)
      for (int k = lane; k < n; k += 32) A[eo * n + k] = (double)oe[k];
  }
  __syncwarp();
  double lnd = 0, sgn = 1;
  bool ok = true;
  if (!reinvert) {
    // inverses, T and G as kept current by the accepted moves' updates; ln|psi_D| likewise
    lnd = st.lnd[w];
    sgn = st.sgn[w];
    ok = isfinite(lnd) && sgn != 0.0;
  }
  for (int sp = 0; sp < 2 && reinvert; sp++) {
    int n = sp ? s.ndn : s.nup;
    if (n == 0) continue;
    double l1, s1;
    bool o1 = warp_gj(ainv + (sp ? s.nup * s.nup : 0), n, v.perm, l1, s1, lane);
    ok = ok && o1;
    lnd += l1;
    sgn *= s1;
  }
  if (MD && ok && reinvert) {
    double lc, sc;
    md_tables(s, v, lane, lc, sc);
    lnd += lc;
    sgn *= sc;
  }
  double d2lnd = 0, v2 = 0;
  det_velocities<T, MD, PG>(s, st, w, v, lane, outputs, pg, d2lnd, v2);

  // --- pseudopotential (nonloc_pot.f90, nonloc.f90), quadrature rotated by R
  double vloc = 0, vnl = 0;
  int ntask_all = 0;
  if (s.nloc > 0 && ok)
    nlpp_energy<T, NORD, MD, PG>(s, J, E, v, R, lane, pg, v.phi, phi_count(s.nbasis, C), nullptr, vloc, vnl, ntask_all);
  finish_eval(s, st, w, v, lane, outputs, ok, lnd, sgn, fsum, d2j, pe_ee, pe_en, d2lnd, v2, vloc, vnl, ntask_all, res);
  __syncwarp();
}

// ---------------------------------------------------------------------------------------
// single-electron proposal (hpsie, qmc/vmc/hpsie.f90) and acceptance (jassav/detsav)
// ---------------------------------------------------------------------------------------
// Delayed Sherman-Morrison updates of the reference inverse (single determinant, walker state in
// HBM; dete_update, dete_mod.f90:165-190, applied lazily): the accepted moves of a spin are kept as
// rank-1 terms, A = A_0 - sum_i u_i w_i^T (u_i the inverse's column of the moved electron over the
// ratio, w_i the moved row times the inverse minus the unit row), and folded into A_0 as one
// rank-K product on the FP64 tensor cores every K accepted moves of the spin and at the end of the
// moves.  Proposals read the current column of A from A_0 and the pending terms.
struct Delay {
  double *buf;  // this walker's [2 spins][u rows, w rows][K][nmax]; null: updates applied at once
  int K, nmax;
  int m[2];     // pending terms per spin
  __device__ double *u(int sp, int i) const { return buf + ((size_t)(2 * sp) * K + i) * nmax; }
  __device__ double *wr(int sp, int i) const { return buf + ((size_t)(2 * sp + 1) * K + i) * nmax; }
};

// Column eo of the current inverse of spin sp into col[n].
__device__ inline void delay_column(const Delay &d, const double *A0, int n, int sp, int eo, double *col, int lane) {
  for (int k = lane; k < n; k += 32) {
    double a = A0[k * n + eo];
    for (int i = 0; i < d.m[sp]; i++) a -= d.u(sp, i)[k] * d.wr(sp, i)[eo];
    col[k] = a;
  }
  __syncwarp();
}

// A_0 -= sum_{i < m} u_i w_i^T for spin sp: 8 x 8 tiles of A_0, k-steps of 4 pending terms
// (mma m8n8k4, FP64; terms past m read as zero).
__device__ inline void delay_flush(Delay &d, double *A0, int n, int sp, int lane) {
  const int m = d.m[sp];
  if (m == 0) return;
  __syncwarp();
  const int r = lane >> 2, q = lane & 3;
  for (int k0 = 0; k0 < n; k0 += 8)
    for (int j0 = 0; j0 < n; j0 += 8) {
      const int kr = k0 + r, jc = j0 + 2 * q;
      double c0 = (kr < n && jc < n) ? A0[kr * n + jc] : 0.0;
      double c1 = (kr < n && jc + 1 < n) ? A0[kr * n + jc + 1] : 0.0;
      for (int i0 = 0; i0 < m; i0 += 4) {
        const int i = i0 + q;
        const double a = (i < m && kr < n) ? -d.u(sp, i)[kr] : 0.0;        // A[row k][col i]
        const double b = (i < m && j0 + r < n) ? d.wr(sp, i)[j0 + r] : 0.0;  // B[row i][col j]
        dmma_884(c0, c1, a, b);
      }
      if (kr < n && jc < n) A0[kr * n + jc] = c0;
      if (kr < n && jc + 1 < n) A0[kr * n + jc + 1] = c1;
    }
  d.m[sp] = 0;
  __syncwarp();
}

template <class T, int NORD, bool MD, bool GRAD>
__device__ void propose(const Sys<T> &s, const JasPar<T> &J, const State<T> &st, int w, const View<T> &v, int e,
                        const double *xn, int lane, double &rho, double &dj, double *grad, const Delay *dl = nullptr,
                        T *coop = nullptr, const double *orow = nullptr) {
  // orow (may be null): the electron's orbital row at xn ([5][nomax], FP64) when it is known
  // already (its current position): no basis functions or contraction then
  const int N = s.N, C = s.C, nomax = s.nomax;
  int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup, eo = sp ? e - s.nup : e;
  const double *A = gam_ptr<T, MD>(s, v, sp);
  // with delayed updates the column of the current inverse goes to v.colb (accept_move reuses it)
  const bool dcol = !MD && dl && dl->buf;
  if (dcol) delay_column(*dl, A, n, sp, eo, v.colb, lane);
  const int no = s.nocc[sp];
  constexpr int NCH = GRAD ? 5 : 1;
  for (int c = lane; c < C; c += 32) {
    T r, d;
    cen_dist(s, J.scalek, xn, c, r, d);
    v.rnew[2 * c] = r;
    v.rnew[2 * c + 1] = d;
  }
  __syncwarp();
  if (lane < ZQ) {
    T z = (lane == 0) ? T(C) : T(0);
    if (lane > 0)
      for (int c = 0; c < C; c++) z += ipow(v.rnew[2 * c + 1], lane);
    v.asum[lane] = z;
  }
  if (orow) {
    // the row is given
  } else if constexpr (!GRAD && sizeof(T) == 4) {
    warp_basis<T, NCH>(s, xn, v.phi, lane);
    if (coop) block_orbitals<T, 1, COOP_KB, COOP_STAGES>(v.phi, s.cocc[sp], s.nbasis, no, v.arow, nomax, lane, coop, true);
    else warp_orbitals<T, NCH>(v.phi, s.cocc[sp], s.nbasis, no, v.arow, nomax, lane);
  } else {
    warp_basis<T, NCH>(s, xn, v.phi, lane);
    warp_orbitals<T, NCH>(v.phi, s.cocc[sp], s.nbasis, no, v.arow, nomax, lane);
  }
  // the wave function is linear in the moved electron's orbital row: ratio = sum_m G[m][e] phi_m
  double r0 = 0, g0 = 0, g1 = 0, g2 = 0;
  for (int k = lane; k < no; k += 32) {
    double a = dcol ? v.colb[k] : A[k * n + eo];
    r0 += a * (orow ? orow[k] : (double)v.arow[k]);
    if (GRAD) {
      g0 += a * (orow ? orow[nomax + k] : (double)v.arow[nomax + k]);
      g1 += a * (orow ? orow[2 * nomax + k] : (double)v.arow[2 * nomax + k]);
      g2 += a * (orow ? orow[3 * nomax + k] : (double)v.arow[3 * nomax + k]);
    }
  }
  rho = warp_sum(r0);
  const T *fso = v.fso;
  T *pf = v.pf;
  double d = 0, gj0 = 0, gj1 = 0, gj2 = 0;
  for (int j = lane; j < N; j += 32) {
    if (j == e) continue;
    T g[3];
    T f = pair_value<T, NORD, GRAD>(s, J, e, j, xn, v.rnew, v.xs + 3 * j, v.ren + 2 * C * j, g, v.asum,
                                    v.zq + ZQ * j, v.rtd ? v.rtd + j : nullptr, N);
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
template <class T, bool MD>
__device__ void accept_move(const Sys<T> &s, const State<T> &st, int w, const View<T> &v, int e, const double *xn,
                            double dj, double rho, int lane, Delay *dl = nullptr) {
  const int N = s.N, C = s.C;
  int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup, eo = sp ? e - s.nup : e;
  double *A = v.ainv + (sp ? s.nup * s.nup : 0);
  const bool delayed = !MD && dl && dl->buf;
  if (!delayed)
    for (int k = lane; k < n; k += 32) v.colb[k] = A[k * n + eo];
  for (int j = lane; j < n; j += 32) {
    double a = 0;
    for (int k = 0; k < n; k++) a += (double)v.arow[k] * A[k * n + j];
    v.vb[j] = a - (j == eo ? 1.0 : 0.0);
  }
  if (delayed) {
    // the pending terms: vb -= sum_i (arow . u_i) w_i
    const int m = dl->m[sp];
    for (int i = 0; i < m; i++) {
      const double *ui = dl->u(sp, i);
      double p = 0;
      for (int k = lane; k < n; k += 32) p += (double)v.arow[k] * ui[k];
      p = warp_sum(p);
      const double *wi = dl->wr(sp, i);
      for (int j = lane; j < n; j += 32) v.vb[j] -= p * wi[j];
    }
  }
  __syncwarp();
  double rinv = 1.0 / (v.vb[eo] + 1.0);
  if (delayed) {
    const int m = dl->m[sp];
    double *um = dl->u(sp, m), *wm = dl->wr(sp, m);
    for (int k = lane; k < n; k += 32) {
      um[k] = v.colb[k] * rinv;
      wm[k] = v.vb[k];
    }
    dl->m[sp] = m + 1;
    if (m + 1 == dl->K) delay_flush(*dl, A, n, sp, lane);
  }
  if (MD) {
    // T update: T += Ainv[:,e] (atilde'_virt - a'^T T) / rho_ref (dete_update, dete_mod.f90:186-190)
    const int nv = s.nvirt[sp];
    double *Tv = v.tv + (sp ? s.nup * s.nvirt[0] : 0);
    double *wb = v.ymd;  // scratch
    for (int p = lane; p < nv; p += 32) {
      double a = (double)v.arow[n + p];
      for (int k = 0; k < n; k++) a -= (double)v.arow[k] * Tv[k * nv + p];
      wb[p] = a;
    }
    __syncwarp();
    for (int i = lane; i < n * nv; i += 32) {
      int k = i / nv, p = i - k * nv;
      Tv[i] += v.colb[k] * wb[p] * rinv;
    }
    __syncwarp();
  }
  if (!delayed)
    for (int idx = lane; idx < n * n; idx += 32) {
      int k = idx / n, j = idx - k * n;
      A[idx] -= v.colb[k] * v.vb[j] * rinv;
    }
  if (MD) {
    __syncwarp();
    double lc, sc;
    build_gamma(s, v, lane, lc, sc);
  }
  T *fso = v.fso;
  for (int j = lane; j < N; j += 32) {
    T f = v.pf[j];
    fso[e * N + j] = f;
    fso[j * N + e] = f;
  }
  for (int i = lane; i < 2 * C; i += 32) v.ren[2 * C * e + i] = v.rnew[i];
  if (v.rtd)
    for (int c = lane; c < C; c += 32) v.rtd[c * N + e] = v.rnew[2 * c + 1];
  for (int q = lane; q < ZQ; q += 32) v.zq[ZQ * e + q] = v.asum[q];
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

template <class T, int NORD, bool MD>
__global__ void __launch_bounds__(128, 4) k_eval(Sys<T> s, State<T> st, Layout L, double r0, double r1, double r2,
                                                 double r3, double r4, double r5, double r6, double r7, double r8,
                                                 int outputs, int orbs_ready) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const double R[9] = {r0, r1, r2, r3, r4, r5, r6, r7, r8};
  for (int w = blockIdx.x * wpb + wib; w < st.W; w += gridDim.x * wpb) {
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nomax, L.resident != 0);
    for (int i = lane; i < 3 * s.N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * s.N + i];
    __syncwarp();
    EvalRes res;
    full_eval<T, NORD, MD>(s, J, E, st, w, v, R, lane, outputs != 0, res, nullptr, orbs_ready != 0);
    if (L.resident) eval_store(v, st, w, s.N, s.C, lane);
    else mirror_store(v, st, w, s.N, s.C, lane);
  }
}

// The per-call proposal/accept kernels always work on the HBM copy of the state.
template <class T, int NORD, bool MD>
__global__ void __launch_bounds__(128, 4) k_propose(Sys<T> s, State<T> st, Layout L, int e, const double *xnew,
                                                    double *ratio, double *grad) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nomax = s.nomax;
  for (int w = blockIdx.x * wpb + wib; w < st.W; w += gridDim.x * wpb) {
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nomax, false);
    for (int i = lane; i < 3 * s.N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * s.N + i];
    __syncwarp();
    double xn[3] = {xnew[3 * w], xnew[3 * w + 1], xnew[3 * w + 2]};
    double rho, dj, g[3];
    if (grad)
      propose<T, NORD, MD, true>(s, J, st, w, v, e, xn, lane, rho, dj, g);
    else
      propose<T, NORD, MD, false>(s, J, st, w, v, e, xn, lane, rho, dj, g);
    int sp = e < s.nup ? 0 : 1;
    for (int k = lane; k < s.nocc[sp]; k += 32) st.pa[(size_t)w * nomax + k] = (double)v.arow[k];
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

template <class T, bool MD>
__global__ void __launch_bounds__(128, 4) k_accept(Sys<T> s, State<T> st, Layout L, int e, const uint8_t *mask) {
  extern __shared__ __align__(16) char dsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nomax = s.nomax, C = s.C;
  for (int w = blockIdx.x * wpb + wib; w < st.W; w += gridDim.x * wpb) {
    if (!mask[w] || st.piel[w] != e) continue;
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nomax, false);
    int sp = e < s.nup ? 0 : 1;
    for (int k = lane; k < s.nocc[sp]; k += 32) v.arow[k] = (T)st.pa[(size_t)w * nomax + k];
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
    if (lane < ZQ) {
      T z = (lane == 0) ? T(C) : T(0);
      if (lane > 0)
        for (int c = 0; c < C; c++) z += ipow(v.rnew[2 * c + 1], lane);
      v.asum[lane] = z;
    }
    __syncwarp();
    accept_move<T, MD>(s, st, w, v, e, xn, st.pdj[w], st.prho[w], lane);
    if (lane < 3) st.x[(size_t)w * 3 * s.N + 3 * e + lane] = xn[lane];
    if (lane == 0) st.piel[w] = -1;
    __syncwarp();
  }
}

// Fused VMC: nsweep sweeps of single-electron Metropolis moves plus E_L after each sweep
// (phase 0); the E_L re-inverts the Slater matrices every reinv_every sweeps.  Phase 1 runs only
// the moves and phase 2 only the E_L, from orbitals computed in between for all walkers
// (tensor-core contraction).  Phase 3 runs only the E_L, from the positions alone (re-inverting,
// and refreshing the FP32 move tables when the state has them): the FP64 half of a mixed-precision
// sweep whose moves ran in FP32.  Statistics are added to st.s_*.
// (One kernel per phase, PH, so that each holds only the code it runs; MV: the mover, 1 Gaussian
// displacements, 6 the accelerated Metropolis method.)
template <class T, int NORD, bool MD, int PH, int MV = 1>
__global__ void __launch_bounds__(128, 4) k_vmc(Sys<T> s, State<T> st, Layout L, int nsweep, uint64_t seed,
                                                uint64_t sweep0, double step, int reinv_every, Mover mv) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int N = s.N;
  constexpr int phase = PH;
  constexpr bool moves = phase == 0 || phase == 1, eval = phase != 1;
  // FP32 Gaussian moves of a state in HBM with L.coop: the block's warps move their walkers'
  // electrons in step and share the coefficient stream of the proposals (block_orbitals)
  T *coop = nullptr;
  if constexpr (PH == 1 && MV == 1 && sizeof(T) == 4)
    if (L.coop) coop = (T *)(dsm + L.stage);
  for (int wb = blockIdx.x * wpb; wb < st.W; wb += gridDim.x * wpb) {
    const int w = wb + wib;
    if (w >= st.W) {
      if constexpr (PH == 1 && MV == 1 && sizeof(T) == 4) {
        if (coop) {
          // no walker for this warp: take part in the block's coefficient stream, no sums
          for (int isw = 0; isw < nsweep; isw++)
            for (int e = 0; e < N; e++) {
              const int sp = e < s.nup ? 0 : 1;
              block_orbitals<T, 1, COOP_KB, COOP_STAGES>((const T *)nullptr, s.cocc[sp], s.nbasis, s.nocc[sp],
                                                         (T *)nullptr, 0, lane, coop, false);
            }
          continue;
        }
      }
      break;
    }
    View<T> v = make_view<T>(dsm + L.bytes * wib, L, st, w, s.N, s.C, s.nbasis, s.nomax, L.resident != 0);
    if (L.resident && phase != 3) {
      view_load(v, st, w, N, s.C, lane);
    } else {
      for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
      __syncwarp();
    }
    double es = 0, e2 = 0, acc = 0, el = 0;
    Delay dl{};
    dl.buf = (moves && !MD && !L.resident && st.dly && st.dlk > 1)
                 ? st.dly + (size_t)w * 4 * st.dlk_max * s.nmax : nullptr;
    dl.K = st.dlk;
    dl.nmax = s.nmax;
    for (int isw = 0; isw < nsweep; isw++) {
      uint64_t sweep = sweep0 + (uint64_t)isw;
      for (int e = 0; moves && e < N; e++) {
        if constexpr (MV == 6) {
          // accelerated Metropolis (metrop_slat_mov1.f90:82-546): the drift at the current position,
          // the spherical-polar proposal about the nearest nucleus, psi and the drift at the new
          // position, both transition probabilities
          const double xo[3] = {v.xs[3 * e], v.xs[3 * e + 1], v.xs[3 * e + 2]};
          double r0, d0, go[3];
          double *orow = st.orb_cache ? st.orb_cache + ((size_t)w * N + e) * 5 * s.nomax : nullptr;
          propose<T, NORD, MD, true>(s, J, st, w, v, e, xo, lane, r0, d0, go, &dl, nullptr, orow);
          MoveRng rng{seed, (uint32_t)w, (uint32_t)sweep, (uint32_t)(sweep >> 32), (uint32_t)e, 0u, {0.0, 0.0}, 0};
          double xn[3], fxop, areao, rtry;
          slat_forward(s, mv, xo, go, rng, xn, fxop, areao, rtry);
          SlatBack b;
          double p = 0, rho = 0, dj = 0;
          if (slat_geometry(s, mv, xo, xn, b)) {
            double gn[3], fxnp, arean;
            propose<T, NORD, MD, true>(s, J, st, w, v, e, xn, lane, rho, dj, gn, &dl);
            slat_reverse(s, mv, b, gn, fxnp, arean);
            const double rr = rtry / b.rminon;
            p = rr * rr * rho * rho * exp(2.0 * dj) * fabs((fxnp * areao) / (fxop * arean));
          }
          if (rng.next() < p) {
            if (orow) {  // the electron's new orbital row becomes its cached row
              for (int i = lane; i < 5 * s.nomax; i += 32) orow[i] = (double)v.arow[i];
              __syncwarp();
            }
            accept_move<T, MD>(s, st, w, v, e, xn, dj, rho, lane, &dl);
            acc += 1;
          }
          continue;
        } else {
        double g[3], ua;
        move_randoms(seed, (uint32_t)w, sweep, (uint32_t)e, g, &ua);
        double xn[3] = {v.xs[3 * e] + step * g[0], v.xs[3 * e + 1] + step * g[1], v.xs[3 * e + 2] + step * g[2]};
        double rho, dj, gr[3];
        propose<T, NORD, MD, false>(s, J, st, w, v, e, xn, lane, rho, dj, gr, &dl, coop);
        double p = rho * rho * exp(2.0 * dj);
        if (ua < p) {
          accept_move<T, MD>(s, st, w, v, e, xn, dj, rho, lane, &dl);
          acc += 1;
        }
        }
      }
      if (dl.buf) {  // the sweep's pending inverse updates, before anything else reads the inverse
        delay_flush(dl, v.ainv, s.nup, 0, lane);
        delay_flush(dl, v.ainv + s.nup * s.nup, s.ndn, 1, lane);
      }
      if constexpr (!eval) continue;
      double R[9];
      random_rotation(seed, (uint32_t)w, sweep, R);
      EvalRes res;
      // periodic FP64 re-inversion: every reinv_every sweeps, in between the updated inverses;
      // phase 3 evaluates from the positions alone and always re-inverts
      const bool reinv = phase == 3 || reinv_every <= 1 || sweep % (uint64_t)reinv_every == 0;
      full_eval<T, NORD, MD>(s, J, E, st, w, v, R, lane, false, res, nullptr, phase == 2, reinv);
      el = res.eloc;
      es += el;
      e2 += el * el;
    }
    if (phase == 3) {
      if (L.resident) eval_store(v, st, w, N, s.C, lane);
      else mirror_store(v, st, w, N, s.C, lane);
    } else if (L.resident) {
      view_store(v, st, w, N, s.C, lane);
    } else {
      for (int i = lane; i < 3 * N; i += 32) st.x[(size_t)w * 3 * N + i] = v.xs[i];
    }
    if (lane == 0) {
      st.s_esum[w] += es;
      st.s_e2sum[w] += e2;
      st.s_acc[w] += acc;
      if (eval) st.s_elast[w] = el;
    }
    __syncwarp();
  }
}

#include "elstage.cuh"
#include "pgrad.cuh"
#include "dmc.cuh"
#include "orbtc.cuh"
