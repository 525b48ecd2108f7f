// device_math.cuh -- per-walker wave-function arithmetic shared by the engine's kernels.
//
// Every function here is warp-cooperative (one warp owns one walker) or per-lane scalar.
// T is the compute type of basis functions, orbitals, Jastrow and the nonlocal
// quadrature (double in FP64 mode, float in mixed mode); inverses, log-determinants,
// the accepted-move Sherman-Morrison update and energy sums are always double.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace champ {

constexpr int MAXCT = 4;     // centre types
constexpr int MAXORD = 8;    // norda, nordb <= 7
constexpr int MAXT = 24;     // e-e-n terms (nordc <= 5)
constexpr int MG = 4;        // Gaussian terms per pseudopotential channel
constexpr int MAXLCH = 5;    // pseudopotential channels
constexpr int MAXQ = 86;     // quadrature points (rules of 4 ... 86 points)
constexpr double HB = 0.5;   // hbar^2 / 2m

// ---------------------------------------------------------------------------------------
// parameters (copied once per block into shared memory)
// ---------------------------------------------------------------------------------------
template <class T>
struct JasPar {
  T scalek;
  int norda, nordb, nspin2b, nct;
  T a4[MAXCT][MAXORD];
  T b[2][MAXORD];
  T c[MAXCT][MAXT];
  T asymp_a[MAXCT];
  T asymp_b[2];
};

struct EcpPar {
  int npotd[MAXCT], lpotp1[MAXCT], nterm[MAXCT][MAXLCH];
  double coef[MAXCT][MAXLCH][MG], expo[MAXCT][MAXLCH][MG];
  int pw[MAXCT][MAXLCH][MG];
  double znuc[MAXCT];
  int nquad;
};

// The quadrature rule (points and weights, [nquad][4]) lives in global memory, not in the
// per-block shared copy of EcpPar: the 86-point rule would cost every block 2.7 KB of shared memory.
struct QuadRule {
  double q0[MAXQ][3], wq[MAXQ];
};

// System data in device memory (pointers into one allocation).
template <class T>
struct Sys {
  int N, nup, ndn, C, nct, nshell, nbasis, nmax, nloc, nordc;
  double pecent, scalek;
  const double *cent;   // [C][3]
  const int *ctype;     // [C]
  const double *zc;     // [C] charge of centre
  const int4 *shell;    // [nshell]: centre, n, l, kind
  const int2 *shprim;   // [nshell]: first primitive, count
  const int *shb0;      // [nshell] first basis function
  const int *cshell0;   // [C+1] first shell of each centre (shells grouped by centre)
  int nshc;             // most shells on one centre; 0 when shells are not grouped by centre
  const T *pz, *pc;     // primitive exponent, normalised weight
  // numerical radial tables (shell kind 2): per table (grid type, points, first value, 0) and
  // (r0, h, log h, small-r polynomial c0..c4, large-r a0, ak); per point the value and its
  // spline second derivative
  const int *shrad;     // [nshell] table of a kind-2 shell
  const int4 *rtab;     // [nrad]
  const double *rpar;   // [nrad][10]
  const T *ry, *ry2;    // [sum nr]
  // occupied orbitals of each spin: det-0 (reference) orbitals in column order, then the
  // other orbitals any determinant of that spin uses ("virtuals"), ascending
  int nocc[2], nvirt[2], nomax, nvmax;
  const T *cocc[2];     // [nbasis][nocc_s] orbital coefficients; rows in the internal basis
                        // order (each shell's functions in harmonic-slot order m = 0, 1, -1, ...)
  const T *coccT[2];    // the same coefficients transposed, [nocc_s][nbasis]
  // multi-determinant tables (deriv_fast_mod.f90:261 excit_bld): unique determinants per
  // spin as excitations of the reference, and the (up, down, coefficient) combinations
  int multidet, ndet, ndu[2];
  const int *dk[2];       // [ndu_s] excitation order
  const int *dh[2];       // [ndu_s][4] hole: reference column
  const int *dpart[2];    // [ndu_s][4] particle: virtual index
  const double *dsg[2];   // [ndu_s] sign of det(T[:, L]) / det(alpha)
  const int *ciu, *cid;   // [ndet] unique up / down determinant of each determinant
  const double *ccoef;    // [ndet] determinant coefficient (csf coefficients folded in)
  // free e-e-n coefficients: d c_ll / d c_free (cusp dependences, checkdepend4 in
  // qmc/fit/cuspinit4.f90) as a [nterms][ncfree] matrix
  int ncfree;
  const double *cproj;
  // CSF and orbital-rotation parameters
  int norb, ncsf, norbp;
  const T *call;           // [nbasis][norb] all orbitals (internal basis order)
  const int *csf_off;      // [ncsf+1]
  const int *csf_det;      // determinant of each CSF entry
  const double *csf_cd;    // coefficient of each CSF entry
  const int4 *orbp;        // [norbp] (i, j, rev, 0): orbital i rotated towards orbital j (and j
                           // away from i when rev: both active, single_ex_wf_bld)
  const int *refpos[2];    // [norb] position of the orbital in the spin's orbital set (reference
                           // columns, then virtuals), or -1
  const int *occo[2];      // [nocc_s] orbital index of each occupied column
  const JasPar<T> *jas;
  const EcpPar *ecp;
  const QuadRule *quad;
};

// ---------------------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double texp(double x) { return exp(x); }
__device__ __forceinline__ float texp(float x) { return expf(x); }
__device__ __forceinline__ double tsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float tsqrt(float x) { return sqrtf(x); }

template <class V>
__device__ __forceinline__ V warp_sum(V v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <class T>
__device__ __forceinline__ T ipow(T r, int n) {
  T p = 1;
  for (int i = 0; i < n; i++) p *= r;
  return p;
}

// ---------------------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (Salmon et al., SC'11) and the draws the
// movers use: the same definition as the CPU checker.
// ---------------------------------------------------------------------------------------
__host__ __device__ inline void philox(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                       uint32_t *out) {
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
__host__ __device__ inline double u53(uint32_t a, uint32_t b) {
  return ((double)(((uint64_t)(a >> 5) << 26) | (b >> 6)) + 0.5) * (1.0 / 9007199254740992.0);
}
__host__ __device__ inline double u32d(uint32_t a) { return ((double)a + 0.5) * (1.0 / 4294967296.0); }

// Gaussian displacement (3) and accept uniform for (seed, walker, sweep, electron).
__device__ inline void move_randoms(uint64_t seed, uint32_t w, uint64_t sweep, uint32_t e, double *g, double *ua) {
  uint32_t a[4], b[4];
  philox(seed, w, (uint32_t)sweep, (uint32_t)(sweep >> 32), 2u * e, a);
  philox(seed, w, (uint32_t)sweep, (uint32_t)(sweep >> 32), 2u * e + 1u, b);
  const double tp = 6.283185307179586;
  double u1 = u53(a[0], a[1]), u2 = u53(a[2], a[3]);
  double u3 = u53(b[0], b[1]), u4 = u32d(b[2]);
  double r1 = sqrt(-2.0 * log(u1)), r2 = sqrt(-2.0 * log(u3));
  double s2, c2, s4, c4;
  sincos(tp * u2, &s2, &c2);
  sincos(tp * u4, &s4, &c4);
  g[0] = r1 * c2;
  g[1] = r1 * s2;
  g[2] = r2 * c4;
  *ua = u32d(b[3]);
}

// ---------------------------------------------------------------------------------------
// Accelerated Metropolis proposal (imetro = 6; metrop_slat_mov1.f90:82-546, Umrigar's
// accelerated Metropolis): the electron moves in spherical coordinates about its nearest
// nucleus -- the new radius drawn between r/deltar and r deltar from sqrt(r)|1 + co r| e^-zeta r,
// whose shape follows the radial drift and the cusp, the polar angle within a cone that narrows
// near the nucleus, the azimuth biased by the tangential drift -- and the forward and reverse
// transition probabilities enter the acceptance.  Scalar FP64 code that every lane of a warp runs
// alike on the same random numbers.
// ---------------------------------------------------------------------------------------
struct Mover {
  int kind;  // 1: Gaussian displacements of size step; 6: accelerated Metropolis
  double deltar, deltat, fbias;
};

// The uniforms of one accelerated move: Philox keyed by (walker, sweep) with the electron and a
// draw counter in the last counter word (bit 31 set, apart from the words of move_randoms and
// random_rotation); draws past 2^15 per move reuse the last pair.
struct MoveRng {
  uint64_t seed;
  uint32_t w, s0, s1, e, ctr;
  double u[2];
  int left;
  __host__ __device__ double next() {
    if (left == 0) {
      uint32_t o[4];
      philox(seed, w, s0, s1, 0x80000000u | (e << 15) | (ctr < 32767u ? ctr : 32767u), o);
      ctr++;
      u[0] = u53(o[0], o[1]);
      u[1] = u53(o[2], o[3]);
      left = 2;
    }
    return u[2 - left--];
  }
};

// Incomplete gamma function of order a at x times x^a e^-x / x^a e^-x supplied as xae (gammai.f90):
// the lower function by its series below a + 4 (iflag = 1), minus the upper one by its continued
// fraction above (iflag = -1), with the reference's iteration counts.
__host__ __device__ inline double slat_gammai(double a, double x, double xae, int &iflag) {
  if (x < a + 4) {
    iflag = 1;
    double ap = a, sum = 1 / a, del = sum;
    const int iter = (int)(21 + 3 * (x - a));
    for (int n = 1; n <= iter; n++) {
      ap += 1;
      del *= x / ap;
      sum += del;
    }
    return sum * xae;
  }
  iflag = -1;
  double a0 = 1, a1 = x, b0 = 0, b1 = 1, fac = 1, g = 0;
  const long na = lround(a - x);
  const int iter = (int)(20 + na > 7 ? 20 + na : 7);
  for (int n = 1; n <= iter; n++) {
    const double an = (double)n, ana = an - a;
    a0 = (a1 + a0 * ana) * fac;
    b0 = (b1 + b0 * ana) * fac;
    const double anf = an * fac;
    a1 = x * a0 + anf * a1;
    b1 = x * b0 + anf * b1;
    fac = 1 / a1;
    g = b1 * fac;
  }
  return -g * xae;
}

// Shape of the radial distribution about a nucleus at distance r with radial drift vr and cusp
// zcusp: zeta and co of sqrt(r)|1 + co r| e^-zeta r.
__host__ __device__ inline void slat_shape(double zcusp, double vr, double r, double &zeta, double &co) {
  const double eps = 1e-10;
  double root = (zcusp + vr) * (zcusp + vr - 4 / r);
  if (root >= 0) {
    root = sqrt(root);
    zeta = 0.5 * (zcusp - vr - root);
    if (zeta <= 0) zeta = 0.5 * (zcusp - vr + root);
    if (zeta <= 0) zeta = eps;
  } else {
    zeta = vr < 0 ? -vr - eps : 1.0;
  }
  co = (zeta + vr) / (1 - (zeta + vr) * r);
}

// Integral of that distribution over [rbot, rtop] divided by its value bot at the current radius.
__host__ __device__ inline double slat_area(double zeta, double co, double rbot, double rtop, double bot) {
  const double g5b2 = 1.329340388179137, d2b3 = 0.666666666666667;
  const double rzero = -1 / co, zrbot = zeta * rbot, zrtop = zeta * rtop;
  const double zebot = sqrt(zrbot * zrbot * zrbot) * exp(-zrbot), zetop = sqrt(zrtop * zrtop * zrtop) * exp(-zrtop);
  int fb, ft, fz;
  const double gbot = slat_gammai(2.5, zrbot, zrbot * zebot, fb), gtop = slat_gammai(2.5, zrtop, zrtop * zetop, ft);
  const double norm = bot * sqrt(zeta * zeta * zeta);
  if (rzero < rbot || rzero > rtop) {
    const double g52 = (fb * ft == 1) ? gtop - gbot : gtop - gbot + g5b2;
    const double g32 = d2b3 * (g52 + zetop - zebot);
    return fabs(g32 + co * g52 / zeta) / norm;
  }
  const double zrzer = zeta * rzero, zezer = sqrt(zrzer * zrzer * zrzer) * exp(-zrzer);
  const double gzer = slat_gammai(2.5, zrzer, zrzer * zezer, fz);
  const double g521 = (fb * fz == 1) ? gzer - gbot : gzer - gbot + g5b2;
  const double g321 = d2b3 * (g521 + zezer - zebot);
  const double g522 = (ft * fz == 1) ? gtop - gzer : gtop - gzer + g5b2;
  const double g322 = d2b3 * (g522 + zetop - zezer);
  return (fabs(g321 + co * g521 / zeta) + fabs(g322 + co * g522 / zeta)) / norm;
}

__host__ __device__ inline double slat_thetamx(const Mover &m, double r, double z) {
  return m.deltat + (2 - m.deltat) / (1 + (z * r) * (z * r));
}

// Nearest centre of point p and the vector from it.
template <class SysT>
__host__ __device__ inline int slat_nearest(const SysT &s, const double *p, double *rv, double &r) {
  int best = 0;
  double bd = 1e300;
  for (int c = 0; c < s.C; c++) {
    const double d0 = p[0] - s.cent[3 * c], d1 = p[1] - s.cent[3 * c + 1], d2 = p[2] - s.cent[3 * c + 2];
    const double d = d0 * d0 + d1 * d1 + d2 * d2;
    if (d < bd) { bd = d; best = c; }
  }
  for (int k = 0; k < 3; k++) rv[k] = p[k] - s.cent[3 * best + k];
  r = sqrt(bd);
  return best;
}

// Local frame about the direction zaxis with the component of v perpendicular to it as xaxis:
// returns that component's length (eps-regularised as the reference does).
__host__ __device__ inline double slat_frame(const double *v, const double *zaxis, double vr, double *xaxis) {
  const double eps = 1e-10;
  double vp = 0;
  for (int k = 0; k < 3; k++) {
    xaxis[k] = v[k] - vr * zaxis[k];
    vp += xaxis[k] * xaxis[k];
  }
  vp = sqrt(vp);
  if (vp < eps) {
    xaxis[0] = eps * (1 - zaxis[0] * zaxis[0]);
    xaxis[1] = eps * (-zaxis[0] * zaxis[1]);
    xaxis[2] = eps * (-zaxis[0] * zaxis[2]);
    vp = eps * sqrt(1 - zaxis[0] * zaxis[0]);
  }
  for (int k = 0; k < 3; k++) xaxis[k] /= vp;
  return vp;
}

// Forward half of an accelerated move of the electron at xo with drift vold: the new position
// xn, and the forward transition factors fxop (the sampled densities relative to the current
// point) and areao (their normalisations), the sampled radius rtry.
template <class SysT>
__host__ __device__ inline void slat_forward(const SysT &s, const Mover &m, const double *xo, const double *vold,
                                             MoveRng &rng, double *xn, double &fxop, double &areao, double &rtry) {
  double rv[3], r;
  const int near = slat_nearest(s, xo, rv, r);
  const double zn = s.zc[near], zcusp = s.nloc == 0 ? zn : 0.0;
  const double deltri = 1 / m.deltar, rbot = r * deltri, rtop = r * m.deltar;
  double zaxis[3], xaxis[3], yaxis[3];
  for (int k = 0; k < 3; k++) zaxis[k] = rv[k] / r;
  double vr = (vold[0] * rv[0] + vold[1] * rv[1] + vold[2] * rv[2]) / r;
  double vp = slat_frame(vold, zaxis, vr, xaxis);
  if (vr < -2 * zn) vr = -2 * zn;
  yaxis[0] = zaxis[1] * xaxis[2] - zaxis[2] * xaxis[1];
  yaxis[1] = zaxis[2] * xaxis[0] - zaxis[0] * xaxis[2];
  yaxis[2] = zaxis[0] * xaxis[1] - zaxis[1] * xaxis[0];
  vp *= m.fbias;
  double zeta, co;
  slat_shape(zcusp, vr, r, zeta, co);
  // maximum of the radial density on [rbot, rtop] for the rejection sampling
  const double root = sqrt((1.5 * co - zeta) * (1.5 * co - zeta) + 2 * zeta * co);
  double rmax1 = co != 0 ? (1.5 * co - zeta + root) / (2 * zeta * co) : rtop;
  rmax1 = rmax1 < rbot ? rbot : (rmax1 > rtop ? rtop : rmax1);
  double fmx = sqrt(rmax1) * fabs(1 + co * rmax1) * exp(-zeta * rmax1);
  if (co < 0) {
    double rmax2 = (1.5 * co - zeta - root) / (2 * zeta * co);
    rmax2 = rmax2 < rbot ? rbot : (rmax2 > rtop ? rtop : rmax2);
    const double f2 = sqrt(rmax2) * fabs(1 + co * rmax2) * exp(-zeta * rmax2);
    if (f2 > fmx) fmx = f2;
  }
  const double bot = sqrt(r) * fabs(1 + co * r) * exp(-zeta * r);
  double top = 0;
  for (int it = 0; it < 10000; it++) {  // bounded: the acceptance per try is far from zero
    rtry = ((m.deltar - deltri) * rng.next() + deltri) * r;
    top = sqrt(rtry) * fabs(1 + co * rtry) * exp(-zeta * rtry);
    if (top / fmx > rng.next()) break;
  }
  fxop = top / bot;
  areao = slat_area(zeta, co, rbot, rtop, bot);
  const double raver = 0.5 * (r + rtry), deltt = slat_thetamx(m, raver, zn);
  const double costht = 1 - deltt * rng.next(), zprime = rtry * costht, sintht = sqrt(1 - costht * costht);
  areao *= deltt;
  const double term = fmin(vp * raver * sintht, 1.0), fm = 1 + term;
  double phitry = 0, topp = 1;
  for (int it = 0; it < 10000; it++) {
    phitry = 3.141592653589793 * rng.next();
    topp = 1 + term * cos(phitry);
    if (topp > rng.next() * fm) break;
  }
  fxop *= topp;
  const double xprime = rtry * sintht * cos(phitry);
  double yprime = sqrt(fmax(0.0, rtry * rtry - xprime * xprime - zprime * zprime));
  if (rng.next() < 0.5) yprime = -yprime;
  for (int k = 0; k < 3; k++) xn[k] = xaxis[k] * xprime + yaxis[k] * yprime + zaxis[k] * zprime + s.cent[3 * near + k];
}

// The reverse geometry of a move xo -> xn about the new point's nearest centre; false when the
// reverse move could not be proposed (the move is rejected without evaluating psi).
struct SlatBack {
  int near;
  double rminn, rminon, costht, sintht, ravern, delttn, rvn[3], rvo[3];
};
template <class SysT>
__host__ __device__ inline bool slat_geometry(const SysT &s, const Mover &m, const double *xo, const double *xn,
                                              SlatBack &b) {
  b.near = slat_nearest(s, xn, b.rvn, b.rminn);
  double r2 = 0, dot = 0;
  for (int k = 0; k < 3; k++) {
    b.rvo[k] = xo[k] - s.cent[3 * b.near + k];
    r2 += b.rvo[k] * b.rvo[k];
    dot += b.rvn[k] * b.rvo[k];
  }
  b.rminon = sqrt(r2);
  dot /= b.rminn * b.rminon;
  b.costht = dot;
  b.sintht = sqrt(1 - dot * dot);
  b.ravern = 0.5 * (b.rminn + b.rminon);
  b.delttn = slat_thetamx(m, b.ravern, s.zc[b.near]);
  return !(b.rminon > b.rminn * m.deltar || dot < 1 - b.delttn);
}

// Reverse transition factors fxnp, arean of the move back from xn (drift vnew there) to xo.
template <class SysT>
__host__ __device__ inline void slat_reverse(const SysT &s, const Mover &m, const SlatBack &b, const double *vnew,
                                             double &fxnp, double &arean) {
  const double zn = s.zc[b.near], zcusp = s.nloc == 0 ? zn : 0.0;
  const double rbot = b.rminn / m.deltar, rtop = b.rminn * m.deltar;
  double zaxis[3], xaxis[3];
  for (int k = 0; k < 3; k++) zaxis[k] = b.rvn[k] / b.rminn;
  double vr = (vnew[0] * b.rvn[0] + vnew[1] * b.rvn[1] + vnew[2] * b.rvn[2]) / b.rminn;
  double vp = slat_frame(vnew, zaxis, vr, xaxis);
  if (vr < -2 * zn) vr = -2 * zn;
  vp *= m.fbias;
  double zeta, co;
  slat_shape(zcusp, vr, b.rminn, zeta, co);
  const double bot = sqrt(b.rminn) * fabs(1 + co * b.rminn) * exp(-zeta * b.rminn);
  const double top = sqrt(b.rminon) * fabs(1 + co * b.rminon) * exp(-zeta * b.rminon);
  fxnp = top / bot;
  arean = slat_area(zeta, co, rbot, rtop, bot) * b.delttn;
  const double term = fmin(vp * b.ravern * b.sintht, 1.0);
  double cosphi = 0, rnorm = 0;
  for (int k = 0; k < 3; k++) {
    const double t2 = b.rvo[k] / b.rminon - b.costht * b.rvn[k] / b.rminn;
    rnorm += t2 * t2;
    cosphi += t2 * xaxis[k];
  }
  cosphi /= sqrt(rnorm);
  fxnp *= 1 + term * cosphi;
}

// Uniform random rotation (Shoemake's quaternion method) for (seed, walker, sweep).
__device__ inline void random_rotation(uint64_t seed, uint32_t w, uint64_t sweep, double *R) {
  uint32_t o[4];
  philox(seed, w, (uint32_t)sweep, (uint32_t)(sweep >> 32), 0xFFFFFFFFu, o);
  double u1 = u53(o[0], o[1]), u2 = u32d(o[2]), u3 = u32d(o[3]);
  const double tp = 6.283185307179586;
  double s1 = sqrt(1.0 - u1), s2 = sqrt(u1);
  double sa, ca, sb, cb;
  sincos(tp * u2, &sa, &ca);
  sincos(tp * u3, &sb, &cb);
  double qx = s1 * sa, qy = s1 * ca, qz = s2 * sb, qw = s2 * cb;
  R[0] = 1 - 2 * (qy * qy + qz * qz); R[1] = 2 * (qx * qy - qz * qw); R[2] = 2 * (qx * qz + qy * qw);
  R[3] = 2 * (qx * qy + qz * qw); R[4] = 1 - 2 * (qx * qx + qz * qz); R[5] = 2 * (qy * qz - qx * qw);
  R[6] = 2 * (qx * qz - qy * qw); R[7] = 2 * (qy * qz + qx * qw); R[8] = 1 - 2 * (qx * qx + qy * qy);
}

// ---------------------------------------------------------------------------------------
// Basis functions: radial shell x real solid harmonic (basis_fns.f90:38-474)
// ---------------------------------------------------------------------------------------
// All 2l+1 solid harmonics of degree l at once, in slot order m = 0, 1, -1, 2, -2, ...
// (slot(m) = 0, 2m-1 for m > 0, -2m for m < 0), with gradients if GRAD.
template <class T, bool GRAD>
__device__ __forceinline__ void solid_all(int l, T x, T y, T z, T *S, T (*G)[3]) {
  T x2 = x * x, y2 = y * y, z2 = z * z, rho2 = x2 + y2;
  if (GRAD)
    for (int i = 0; i < 2 * l + 1; i++) G[i][0] = G[i][1] = G[i][2] = T(0);
  switch (l) {
  case 0:
    S[0] = T(1);
    return;
  case 1:
    S[0] = z; S[1] = x; S[2] = y;
    if (GRAD) { G[0][2] = 1; G[1][0] = 1; G[2][1] = 1; }
    return;
  case 2: {
    const T s3 = T(1.7320508075688772);
    S[0] = T(0.5) * (2 * z2 - rho2); S[1] = s3 * x * z; S[2] = s3 * y * z;
    S[3] = T(0.5) * s3 * (x2 - y2); S[4] = s3 * x * y;
    if (GRAD) {
      G[0][0] = -x; G[0][1] = -y; G[0][2] = 2 * z;
      G[1][0] = s3 * z; G[1][2] = s3 * x;
      G[2][1] = s3 * z; G[2][2] = s3 * y;
      G[3][0] = s3 * x; G[3][1] = -s3 * y;
      G[4][0] = s3 * y; G[4][1] = s3 * x;
    }
    return;
  }
  case 3: {
    const T c1 = T(0.61237243569579452), c2 = T(1.9364916731037085), c3 = T(0.79056941504209483);
    T q = 4 * z2 - rho2;
    S[0] = z * z2 - T(1.5) * z * rho2; S[1] = c1 * x * q; S[2] = c1 * y * q;
    S[3] = c2 * z * (x2 - y2); S[4] = 2 * c2 * x * y * z;
    S[5] = c3 * (x * x2 - 3 * x * y2); S[6] = c3 * (3 * x2 * y - y * y2);
    if (GRAD) {
      G[0][0] = -3 * x * z; G[0][1] = -3 * y * z; G[0][2] = 3 * z2 - T(1.5) * rho2;
      G[1][0] = c1 * (4 * z2 - 3 * x2 - y2); G[1][1] = -2 * c1 * x * y; G[1][2] = 8 * c1 * x * z;
      G[2][0] = -2 * c1 * x * y; G[2][1] = c1 * (4 * z2 - x2 - 3 * y2); G[2][2] = 8 * c1 * y * z;
      G[3][0] = 2 * c2 * x * z; G[3][1] = -2 * c2 * y * z; G[3][2] = c2 * (x2 - y2);
      G[4][0] = 2 * c2 * y * z; G[4][1] = 2 * c2 * x * z; G[4][2] = 2 * c2 * x * y;
      G[5][0] = 3 * c3 * (x2 - y2); G[5][1] = -6 * c3 * x * y;
      G[6][0] = 6 * c3 * x * y; G[6][1] = 3 * c3 * (x2 - y2);
    }
    return;
  }
  default: {
    const T c1 = T(0.79056941504209483), c2 = T(0.55901699437494742), c3 = T(2.0916500663351889),
            c4 = T(0.73950997288745201);
    T P = 6 * z2 - rho2, Q = x2 - y2, q = 4 * z2 - 3 * rho2;
    S[0] = z2 * z2 - 3 * rho2 * z2 + T(0.375) * rho2 * rho2;
    S[1] = c1 * x * z * q; S[2] = c1 * y * z * q;
    S[3] = c2 * P * Q; S[4] = 2 * c2 * P * x * y;
    S[5] = c3 * z * (x * x2 - 3 * x * y2); S[6] = c3 * z * (3 * x2 * y - y * y2);
    S[7] = c4 * (x2 * x2 - 6 * x2 * y2 + y2 * y2); S[8] = 4 * c4 * (x * x2 * y - x * y * y2);
    if (GRAD) {
      G[0][0] = -6 * x * z2 + T(1.5) * rho2 * x; G[0][1] = -6 * y * z2 + T(1.5) * rho2 * y;
      G[0][2] = 4 * z * z2 - 6 * rho2 * z;
      G[1][0] = c1 * (4 * z * z2 - 9 * x2 * z - 3 * y2 * z); G[1][1] = -6 * c1 * x * y * z;
      G[1][2] = c1 * (12 * x * z2 - 3 * x * x2 - 3 * x * y2);
      G[2][0] = -6 * c1 * x * y * z; G[2][1] = c1 * (4 * z * z2 - 3 * x2 * z - 9 * y2 * z);
      G[2][2] = c1 * (12 * y * z2 - 3 * x2 * y - 3 * y * y2);
      G[3][0] = 2 * c2 * x * (P - Q); G[3][1] = -2 * c2 * y * (P + Q); G[3][2] = 12 * c2 * z * Q;
      G[4][0] = 2 * c2 * y * (P - 2 * x2); G[4][1] = 2 * c2 * x * (P - 2 * y2); G[4][2] = 24 * c2 * x * y * z;
      G[5][0] = 3 * c3 * z * (x2 - y2); G[5][1] = -6 * c3 * x * y * z; G[5][2] = c3 * (x * x2 - 3 * x * y2);
      G[6][0] = 6 * c3 * x * y * z; G[6][1] = 3 * c3 * z * (x2 - y2); G[6][2] = c3 * (3 * x2 * y - y * y2);
      G[7][0] = c4 * (4 * x * x2 - 12 * x * y2); G[7][1] = c4 * (4 * y * y2 - 12 * x2 * y);
      G[8][0] = c4 * (12 * x2 * y - 4 * y * y2); G[8][1] = c4 * (4 * x * x2 - 12 * x * y2);
    }
    return;
  }
  }
}

// Numerical radial function f, f', f'' of table t at r (splfit_bas, qmc/vmc/splfit.f90): the
// grid interval from the grid's closed form, cubic-spline interpolation inside the grid, the
// small-r polynomial below its first point and the exponential beyond its last.
template <class T, bool DERIV>
__device__ __forceinline__ void table_radial(const Sys<T> &s, int t, T r, T *R) {
  const int4 tb = s.rtab[t];
  const double *p = s.rpar + 10 * t;
  const T r0 = (T)p[0], h = (T)p[1], lh = (T)p[2];
  int jx;
  T ref0, ref1;
  if (tb.x == 1) {
    jx = (int)((r - r0) / h + T(1));
    ref0 = r0 + h * T(jx - 1);
    ref1 = ref0 + h;
  } else if (tb.x == 2) {
    const T xr = log(r / r0) / lh + T(1);
    jx = xr < T(1) ? 0 : (int)xr;
    ref0 = r0 * pow(h, T(jx - 1));
    ref1 = ref0 * h;
  } else {
    jx = (int)(log((r + r0) / r0) / lh + T(1));
    ref0 = r0 * pow(h, T(jx - 1)) - r0;
    ref1 = (ref0 + r0) * h - r0;
  }
  if (jx < 1) {
    R[0] = (T)p[3];
    T rp = T(1);
    for (int i = 1; i < 5; i++) { rp *= r; R[0] += (T)p[3 + i] * rp; }
    if (DERIV) {
      R[1] = R[2] = T(0);
      T pm2 = T(0), pm1 = T(1);  // r^(i-2), r^(i-1)
      for (int i = 1; i < 5; i++) {
        R[1] += T(i) * (T)p[3 + i] * pm1;
        R[2] += T(i * (i - 1)) * (T)p[3 + i] * pm2;
        pm2 = pm1;
        pm1 *= r;
      }
    }
  } else if (jx >= tb.y) {
    const T ak = (T)p[9];
    R[0] = (T)p[8] * exp(-ak * r);
    if (DERIV) {
      R[1] = -ak * R[0];
      R[2] = -ak * R[1];
    }
  } else {
    const T *y = s.ry + tb.z + (jx - 1), *y2 = s.ry2 + tb.z + (jx - 1);
    const T delh = ref1 - ref0, bb = (r - ref0) / delh, aa = (ref1 - r) / delh;
    const T cc = aa * (aa * aa - T(1)) * delh * delh / T(6), dd = bb * (bb * bb - T(1)) * delh * delh / T(6);
    R[0] = aa * y[0] + bb * y[1] + cc * y2[0] + dd * y2[1];
    if (DERIV) {
      R[1] = (y[1] - y[0]) / delh + (-(T(3) * aa * aa - T(1)) * y2[0] + (T(3) * bb * bb - T(1)) * y2[1]) * delh / T(6);
      R[2] = aa * y2[0] + bb * y2[1];
    }
  }
}

// Radial function R, R', R'' of one shell at distance r (wfv(1..3), basis_fns.f90:118-157).
template <class T, bool DERIV>
__device__ __forceinline__ void shell_radial(const Sys<T> &s, int ish, T r, T *R) {
  int4 sh = s.shell[ish];
  int2 pr = s.shprim[ish];
  if (sh.w == 2) {
    table_radial<T, DERIV>(s, s.shrad[ish], r, R);
    const T w = s.pc[pr.x];
    R[0] *= w;
    if (DERIV) { R[1] *= w; R[2] *= w; }
    return;
  }
  int n = sh.y;
  T rn = T(n);
  T rm1 = ipow(r, n - 1);
  T ri = T(1) / r;
  T rm2 = rm1 * ri, rm3 = rm2 * ri;
  R[0] = R[1] = R[2] = T(0);
  for (int p = pr.x; p < pr.x + pr.y; p++) {
    T z = s.pz[p], w = s.pc[p];
    if (sh.w == 0) {
      T zr = z * r, ex = w * texp(-zr);
      R[0] += rm1 * ex;
      if (DERIV) {
        R[1] += rm2 * ((rn - 1) - zr) * ex;
        R[2] += rm3 * ((rn - 1) * (rn - 2 - zr) - (rn - 1 - zr) * zr) * ex;
      }
    } else {
      T zr = 2 * z * r * r, ex = w * texp(T(-0.5) * zr);
      R[0] += rm1 * ex;
      if (DERIV) {
        R[1] += rm2 * ((rn - 1) - zr) * ex;
        R[2] += rm3 * ((rn - 1) * (rn - 2) - (2 * rn - 1 - zr) * zr) * ex;
      }
    }
  }
}

// All basis functions of one shell at point pt, handed to put(slot, channel, value) as they are
// formed: NCH=1 values, NCH=5 value, gradient, Laplacian; slots in harmonic order
// m = 0, 1, -1, ... (the shell's basis functions are stored as b = b0 + slot).
template <class T, int NCH, class Put>
__device__ __forceinline__ void shell_eval_put(const Sys<T> &s, int ish, const double *pt, Put put) {
  int4 sh = s.shell[ish];
  int c = sh.x, l = sh.z;
  T d0 = T(pt[0] - s.cent[3 * c]), d1 = T(pt[1] - s.cent[3 * c + 1]), d2 = T(pt[2] - s.cent[3 * c + 2]);
  T r2 = d0 * d0 + d1 * d1 + d2 * d2;
  T r = tsqrt(r2);
  if (r == T(0)) { r = T(1e-30); d0 = r; }
  T R[3];
  shell_radial<T, NCH == 5>(s, ish, r, R);
  T ri = T(1) / r;
  T ril = ipow(ri, l);
  T S[9], G[9][3];
  solid_all<T, NCH == 5>(l, d0, d1, d2, S, G);
  const int nm = 2 * l + 1;
#pragma unroll
  for (int sl = 0; sl < 9; sl++) {
    if (sl < nm) {
      T Y = S[sl] * ril;
      put(sl, 0, Y * R[0]);
      if (NCH == 5) {
        T lr = T(l) * S[sl] * ril * ri * ri;
        put(sl, 1, Y * d0 * ri * R[1] + (G[sl][0] * ril - lr * d0) * R[0]);
        put(sl, 2, Y * d1 * ri * R[1] + (G[sl][1] * ril - lr * d1) * R[0]);
        put(sl, 3, Y * d2 * ri * R[1] + (G[sl][2] * ril - lr * d2) * R[0]);
        put(sl, 4, Y * (R[2] + 2 * ri * R[1] - T(l * (l + 1)) * ri * ri * R[0]));
      }
    }
  }
}

// All basis functions of one shell at point pt; NCH=1 values, NCH=5 value, grad, laplacian.
// out[b*NCH + ch] for the shell's basis functions b.
template <class T, int NCH>
__device__ __forceinline__ void shell_eval(const Sys<T> &s, int ish, const double *pt, T *out) {
  T *o = out + s.shb0[ish] * NCH;
  shell_eval_put<T, NCH>(s, ish, pt, [o](int sl, int ch, T v) { o[sl * NCH + ch] = v; });
}

// Values of all basis functions of one shell at pt contracted with g: sum_b phi_b(pt) g_b.
template <class T>
__device__ __forceinline__ T shell_dot(const Sys<T> &s, int ish, const double *pt, const T *g) {
  int4 sh = s.shell[ish];
  int c = sh.x, l = sh.z;
  T d0 = T(pt[0] - s.cent[3 * c]), d1 = T(pt[1] - s.cent[3 * c + 1]), d2 = T(pt[2] - s.cent[3 * c + 2]);
  T r = tsqrt(d0 * d0 + d1 * d1 + d2 * d2);
  if (r == T(0)) { r = T(1e-30); d0 = r; }
  T R[3];
  shell_radial<T, false>(s, ish, r, R);
  T S[9], G[9][3];
  solid_all<T, false>(l, d0, d1, d2, S, G);
  int b0 = s.shb0[ish];
  const int nm = 2 * l + 1;
  T acc = 0;
#pragma unroll
  for (int sl = 0; sl < 9; sl++)
    if (sl < nm) acc += S[sl] * g[b0 + sl];
  return acc * ipow(T(1) / r, l) * R[0];
}

// shell_dot with the radial value taken from *R0 when R0 is not null (the point's distance from
// the shell's centre known in advance).
template <class T>
__device__ __forceinline__ T shell_dot_r(const Sys<T> &s, int ish, const double *pt, const T *g, const T *R0) {
  int4 sh = s.shell[ish];
  int c = sh.x, l = sh.z;
  T d0 = T(pt[0] - s.cent[3 * c]), d1 = T(pt[1] - s.cent[3 * c + 1]), d2 = T(pt[2] - s.cent[3 * c + 2]);
  T r = tsqrt(d0 * d0 + d1 * d1 + d2 * d2);
  if (r == T(0)) { r = T(1e-30); d0 = r; }
  T R[3];
  if (R0) R[0] = *R0;
  else shell_radial<T, false>(s, ish, r, R);
  T S[9], G[9][3];
  solid_all<T, false>(l, d0, d1, d2, S, G);
  int b0 = s.shb0[ish];
  const int nm = 2 * l + 1;
  T acc = 0;
#pragma unroll
  for (int sl = 0; sl < 9; sl++)
    if (sl < nm) acc += S[sl] * g[b0 + sl];
  return acc * ipow(T(1) / r, l) * R[0];
}

// shell_dot_r that also adds c times every basis function of the shell into acc[b] (atomically),
// from the same values.
template <class T>
__device__ __forceinline__ T shell_dot_acc(const Sys<T> &s, int ish, const double *pt, const T *g, const T *R0,
                                           double cf, double *acc) {
  int4 sh = s.shell[ish];
  int c = sh.x, l = sh.z;
  T d0 = T(pt[0] - s.cent[3 * c]), d1 = T(pt[1] - s.cent[3 * c + 1]), d2 = T(pt[2] - s.cent[3 * c + 2]);
  T r = tsqrt(d0 * d0 + d1 * d1 + d2 * d2);
  if (r == T(0)) { r = T(1e-30); d0 = r; }
  T R[3];
  if (R0) R[0] = *R0;
  else shell_radial<T, false>(s, ish, r, R);
  T S[9], G[9][3];
  solid_all<T, false>(l, d0, d1, d2, S, G);
  int b0 = s.shb0[ish];
  const int nm = 2 * l + 1;
  const T rad = ipow(T(1) / r, l) * R[0];
  const double f = cf * (double)rad;
  T dot = 0;
#pragma unroll
  for (int sl = 0; sl < 9; sl++)
    if (sl < nm) {
      dot += S[sl] * g[b0 + sl];
      atomicAdd(&acc[b0 + sl], f * (double)S[sl]);
    }
  return dot * rad;
}

// Warp: all basis functions at pt into phi (shared memory).
template <class T, int NCH>
__device__ __forceinline__ void warp_basis(const Sys<T> &s, const double *pt, T *phi, int lane) {
  for (int ish = lane; ish < s.nshell; ish += 32) shell_eval<T, NCH>(s, ish, pt, phi);
  __syncwarp();
}

// Warp: orbitals o_m = sum_b coef[b][m] phi[b] for m < n (orbitals_loc_ana.f90:50-64).
// Lanes are split into LM lanes along m and 32/LM along b, reduced by shuffles.
// out[ch*ostride + m].
template <class T, int NCH, class O>
__device__ __forceinline__ void warp_orbitals(const T *phi, const T *coef, int nbasis, int n, O *out, int ostride,
                                              int lane) {
  if (n > 16) {
    // lanes along m, two orbitals per lane per pass (64 per pass); the coefficient rows of U
    // basis functions are loaded together so that the L2 latency of the coefficient stream is
    // paid once per U functions.  Each orbital is summed over b in order, as on the path below.
    constexpr int U = NCH == 1 ? 8 : 4;
    for (int m0 = 0; m0 < n; m0 += 64) {
      const int ma = m0 + lane, mb = m0 + 32 + lane;
      const bool ha = ma < n, hb = mb < n;
      T aa[NCH], ab[NCH];
#pragma unroll
      for (int ch = 0; ch < NCH; ch++) aa[ch] = ab[ch] = T(0);
      int b = 0;
      for (; b + U <= nbasis; b += U) {
        T ca[U], cb[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          ca[u] = ha ? coef[(size_t)(b + u) * n + ma] : T(0);
          cb[u] = hb ? coef[(size_t)(b + u) * n + mb] : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++)
#pragma unroll
          for (int ch = 0; ch < NCH; ch++) {
            T p = phi[(b + u) * NCH + ch];
            aa[ch] += ca[u] * p;
            ab[ch] += cb[u] * p;
          }
      }
      for (; b < nbasis; b++) {
        T ca = ha ? coef[(size_t)b * n + ma] : T(0), cb = hb ? coef[(size_t)b * n + mb] : T(0);
#pragma unroll
        for (int ch = 0; ch < NCH; ch++) {
          T p = phi[b * NCH + ch];
          aa[ch] += ca * p;
          ab[ch] += cb * p;
        }
      }
#pragma unroll
      for (int ch = 0; ch < NCH; ch++) {
        if (ha) out[ch * ostride + ma] = (O)aa[ch];
        if (hb) out[ch * ostride + mb] = (O)ab[ch];
      }
    }
    __syncwarp();
    return;
  }
  int LM = 1;
  while (LM < n && LM < 32) LM <<= 1;
  int LB = 32 / LM;
  int lm = lane & (LM - 1), lb = lane / LM;
  for (int m0 = 0; m0 < n; m0 += LM) {
    int m = m0 + lm;
    T acc[NCH];
#pragma unroll
    for (int ch = 0; ch < NCH; ch++) acc[ch] = T(0);
    if (m < n) {
      for (int b = lb; b < nbasis; b += LB) {
        T cf = coef[b * n + m];
#pragma unroll
        for (int ch = 0; ch < NCH; ch++) acc[ch] += cf * phi[b * NCH + ch];
      }
    }
    for (int o = LM; o < 32; o <<= 1)
#pragma unroll
      for (int ch = 0; ch < NCH; ch++) acc[ch] += __shfl_xor_sync(0xffffffffu, acc[ch], o);
    if (lb == 0 && m < n)
#pragma unroll
      for (int ch = 0; ch < NCH; ch++) out[ch * ostride + m] = (O)acc[ch];
  }
  __syncwarp();
}

// Block: the same contraction as warp_orbitals (n > 16), for every warp of the block at once, each
// with its own phi ([nbasis][NCH]), sharing the coefficient stream: chunks of KB coefficient rows
// (contiguous in [nbasis][n]) go through STG shared-memory buffers (stage, STG x KB x n elements)
// by cp.async, STG - 1 chunks in flight while one is summed.  Each orbital and channel is summed
// over b in order, as warp_orbitals does, so the results are the same.  Every warp of the block
// must make the call with the same n and coefficients (a warp without work passes active = false:
// it copies and waits, no sums).  Without 16-byte alignment the chunks are copied by plain loads.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int K>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(K) : "memory"); }

template <class T, int NCH, int KB, int STG, class O>
__device__ __forceinline__ void block_orbitals(const T *phi, const T *coef, int nbasis, int n, O *out, int ostride,
                                               int lane, T *stage, bool active) {
  static_assert(STG >= 2 && 16 % sizeof(T) == 0, "pipeline of at least two 16-byte-copyable buffers");
  constexpr int EV = 16 / sizeof(T);  // elements per 16-byte copy
  const int tid = threadIdx.x, nt = blockDim.x;
  const int nchunk = (nbasis + KB - 1) / KB;
  const bool vec = n % EV == 0 && (reinterpret_cast<uintptr_t>(coef) & 15) == 0;
  auto issue = [&](int k) {  // chunk k into buffer k % STG (this thread's share)
    if (k >= nchunk) return;
    const int len = min(KB, nbasis - k * KB) * n;
    const T *src = coef + (size_t)k * KB * n;
    T *dst = stage + (size_t)(k % STG) * KB * n;
    if (vec) {
      for (int q = tid; EV * q < len; q += nt) cp_async16(dst + EV * q, src + EV * q);
    } else {
      for (int i = tid; i < len; i += nt) dst[i] = src[i];
    }
  };
  for (int m0 = 0; m0 < n; m0 += 64) {
    const int ma = m0 + lane, mb = m0 + 32 + lane;
    const bool ha = ma < n, hb = mb < n;
    T aa[NCH], ab[NCH];
#pragma unroll
    for (int ch = 0; ch < NCH; ch++) aa[ch] = ab[ch] = T(0);
    __syncthreads();  // earlier readers of the buffers are done
#pragma unroll
    for (int k = 0; k < STG - 1; k++) {
      issue(k);
      cp_async_commit();
    }
    for (int k = 0; k < nchunk; k++) {
      cp_async_wait<STG - 2>();  // this thread's copies of chunk k have landed
      __syncthreads();           // everyone's have; chunk k - 1 is no longer read
      issue(k + STG - 1);        // into chunk k - 1's buffer
      cp_async_commit();
      if (active) {
        const T *cs = stage + (size_t)(k % STG) * KB * n;
        const int b0 = k * KB, kb = min(KB, nbasis - b0);
        for (int u = 0; u < kb; u++) {
          const T ca = ha ? cs[u * n + ma] : T(0), cb = hb ? cs[u * n + mb] : T(0);
#pragma unroll
          for (int ch = 0; ch < NCH; ch++) {
            const T p = phi[(b0 + u) * NCH + ch];
            aa[ch] += ca * p;
            ab[ch] += cb * p;
          }
        }
      }
    }
    cp_async_wait<0>();
    if (active) {
#pragma unroll
      for (int ch = 0; ch < NCH; ch++) {
        if (ha) out[ch * ostride + ma] = (O)aa[ch];
        if (hb) out[ch * ostride + mb] = (O)ab[ch];
      }
    }
  }
  __syncwarp();
}
// the FP32 single-electron moves' pipeline: 32-row chunks, three buffers
constexpr int COOP_KB = 32, COOP_STAGES = 3;

// ---------------------------------------------------------------------------------------
// Jastrow ijas=4, isc=4 (jastrow4.f90, scale_dist.f90:644-648, 857-884)
// ---------------------------------------------------------------------------------------
struct Terms {
  int n;
  int k[64], l[64], m[64];
};
__host__ __device__ constexpr Terms make_terms(int nord) {
  Terms t{};
  int i = 0;
  for (int n = 2; n <= nord; n++)
    for (int k = n - 1; k >= 0; k--) {
      int l_hi = (k == 0) ? n - k - 2 : n - k;
      for (int l = l_hi; l >= 0; l--) {
        int m = (n - k - l) / 2;
        if (2 * m == n - k - l) { t.k[i] = k; t.l[i] = l; t.m[i] = m; i++; }
      }
    }
  t.n = i;
  return t;
}

// The e-e-n value sum over centres, for one pair (i, j), rewritten as
//   sum_c sum_klm c_klm u^k (a_c^l + r_c^l)(a_c r_c)^m = sum_klm c_klm u^k [X(l+m, m) + X(m, l+m)],
//   X(p, q) = sum_c a_c^p r_c^q,  a_c = 1/(1+k r_ic), r_c = 1/(1+k r_jc)  (switched distances),
// with X(p, 0) depending only on electron i and X(0, q) only on electron j: per centre only the
// products with p, q >= 1 remain.  Valid when all centres share one type (one c set).
struct MixedPQ {
  int n;
  int p[40], q[40];
};
__host__ __device__ constexpr MixedPQ make_mixed(int nord) {
  MixedPQ x{};
  Terms t = make_terms(nord);
  for (int ll = 0; ll < t.n; ll++) {
    int l = t.l[ll], m = t.m[ll];
    int pp[2] = {l + m, m}, qq[2] = {m, l + m};
    for (int s2 = 0; s2 < 2; s2++) {
      if (pp[s2] == 0 || qq[s2] == 0) continue;
      bool seen = false;
      for (int i = 0; i < x.n; i++)
        if (x.p[i] == pp[s2] && x.q[i] == qq[s2]) seen = true;
      if (!seen) { x.p[x.n] = pp[s2]; x.q[x.n] = qq[s2]; x.n++; }
    }
  }
  return x;
}
__host__ __device__ constexpr int mixed_index(const MixedPQ &x, int p, int q) {
  for (int i = 0; i < x.n; i++)
    if (x.p[i] == p && x.q[i] == q) return i;
  return -1;
}

// X sums of one pair: a[sa c] = a_c, r[sr c] = r_c (the scaled e-n distances of the two
// electrons, strided); mixed products only.
template <class T, int NORD>
__device__ __forceinline__ void een_xsums(int C, const T *a, int sa, const T *r, int sr, T *X) {
  constexpr MixedPQ mx = make_mixed(NORD);
#pragma unroll
  for (int i = 0; i < mx.n; i++) X[i] = T(0);
  for (int c = 0; c < C; c++) {
    T ac = a[sa * c], rc = r[sr * c];
    T ap[NORD + 1], rp[NORD + 1];
    ap[0] = rp[0] = T(1);
#pragma unroll
    for (int q = 1; q <= NORD; q++) { ap[q] = ap[q - 1] * ac; rp[q] = rp[q - 1] * rc; }
#pragma unroll
    for (int i = 0; i < mx.n; i++) X[i] += ap[mx.p[i]] * rp[mx.q[i]];
  }
}

// Per term, where its two X factors come from: code < 100 -> mixed sum X[code],
// 100 + p -> ai[p] (sum over centres of a_c^p), 200 + q -> rj[q] (sum of r_c^q).
struct XIdx {
  int a1[64], a2[64];
};
__host__ __device__ constexpr XIdx make_xidx(int nord) {
  XIdx x{};
  Terms t = make_terms(nord);
  MixedPQ mx = make_mixed(nord);
  for (int ll = 0; ll < t.n; ll++) {
    int l = t.l[ll], m = t.m[ll];
    int pp[2] = {l + m, m}, qq[2] = {m, l + m};
    for (int s2 = 0; s2 < 2; s2++) {
      int code = 0;
      if (qq[s2] == 0) code = 100 + pp[s2];
      else if (pp[s2] == 0) code = 200 + qq[s2];
      else code = mixed_index(mx, pp[s2], qq[s2]);
      if (s2 == 0) x.a1[ll] = code; else x.a2[ll] = code;
    }
  }
  return x;
}

template <class T>
__device__ __forceinline__ T xsel(int code, const T *ai, const T *rj, const T *X) {
  return code >= 200 ? rj[code - 200] : (code >= 100 ? ai[code - 100] : X[code]);
}

// e-e-n value of one pair from its X sums (jastrow4.f90:211-257 summed over centres)
template <class T, int NORD>
__device__ __forceinline__ T een_from_x(const T *c, T du, const T *ai, const T *rj, const T *X) {
  constexpr Terms tl = make_terms(NORD);
  constexpr XIdx xi = make_xidx(NORD);
  T uu[NORD + 1];
  uu[0] = T(1);
#pragma unroll
  for (int q = 1; q <= NORD; q++) uu[q] = uu[q - 1] * du;
  T f = 0;
#pragma unroll
  for (int ll = 0; ll < tl.n; ll++)
    f += c[ll] * uu[tl.k[ll]] * (xsel(xi.a1[ll], ai, rj, X) + xsel(xi.a2[ll], ai, rj, X));
  return f;
}

// spin class of pair (i,j): parallel spins use b set 2 (nspin2b=2) or 1/2 on b1.
template <class T>
__device__ __forceinline__ void pair_class(const JasPar<T> &J, int nup, int i, int j, int &isb, T &ss, int &ipar) {
  bool par = (i < nup) == (j < nup);
  ipar = par ? 1 : 0;
  isb = (par && J.nspin2b == 2) ? 1 : 0;
  ss = (par && J.nspin2b == 1) ? T(0.5) : T(1);
}

// In all Jastrow terms d = 1/(1 + scalek r) is passed in: the isc=4 scaled distance is
// r d (scale_dist2, scale_dist.f90:644-648) and the switched one used by the e-e-n term
// is 1 - scalek r d = d (switch_scale2, scale_dist.f90:857-884).

// e-e term: f, f'/r, f'' (jastrow4.f90:63-156)
template <class T, bool DERIV>
__device__ __forceinline__ T jas_ee(const JasPar<T> &J, int isb, T ss, int ipar, T rij, T deni, T &fu, T &fuu) {
  T u = rij * deni;
  T b1 = J.b[isb][0], b2 = J.b[isb][1];
  T bot = T(1) + b2 * u;
  T f = ss * b1 * u / bot - J.asymp_b[ipar];
  T feeu = 0, feeuu = 0;
  if (DERIV) {
    feeu = ss * b1 / (bot * bot);
    feeuu = -2 * feeu * b2 / bot;
  }
  T up = u, upm1 = T(1), upm2 = T(0);
  for (int iord = 2; iord <= J.nordb; iord++) {
    upm2 = upm1; upm1 = up; up = up * u;
    T bb = J.b[isb][iord];
    f += bb * up;
    if (DERIV) {
      feeu += bb * iord * upm1;
      feeuu += bb * iord * (iord - 1) * upm2;
    }
  }
  if (DERIV) {
    T dd1 = deni * deni, dd2 = -2 * J.scalek * deni * dd1;
    fuu = feeuu * dd1 * dd1 + feeu * dd2;
    fu = feeu * dd1 / rij;
  }
  return f;
}

// e-n term: f, f'/r, f'' (jastrow4.f90:354-455)
template <class T, bool DERIV>
__device__ __forceinline__ T jas_en(const JasPar<T> &J, int it, T ri, T deni, T &fi, T &fii) {
  T rr = ri * deni;
  T a1 = J.a4[it][0], a2 = J.a4[it][1];
  T bot = T(1) + a2 * rr;
  T f = a1 * rr / bot - J.asymp_a[it];
  T feni = 0, fenii = 0;
  if (DERIV) {
    feni = a1 / (bot * bot);
    fenii = -2 * feni * a2 / bot;
  }
  T p = rr, pm1 = T(1), pm2 = T(0);
  for (int iord = 2; iord <= J.norda; iord++) {
    pm2 = pm1; pm1 = p; p = p * rr;
    T aa = J.a4[it][iord];
    f += aa * p;
    if (DERIV) {
      feni += aa * iord * pm1;
      fenii += aa * iord * (iord - 1) * pm2;
    }
  }
  if (DERIV) {
    T dd7 = deni * deni, dd9 = -2 * J.scalek * deni * dd7;
    fii = fenii * dd7 * dd7 + feni * dd9;
    fi = feni * dd7 / ri;
  }
  return f;
}

template <class T>
struct Een {
  T fc, fu, fuu, fi, fii, fj, fjj, fui, fuj;
};

// e-e-n term for one centre (jastrow4.f90:159-336).  LEVEL 0: value, 1: + first
// derivatives (fu, fi, fj), 2: everything.  Power tables carry two zero entries below 0.
template <class T, int NORD, int LEVEL>
__device__ __forceinline__ void jas_een(const JasPar<T> &J, int it, T rij, T du, T ri, T di, T rj, T dj,
                                        Een<T> &o) {
  constexpr Terms tl = make_terms(NORD);
  T sk = J.scalek;
  T u1 = du, ri1 = di, rj1 = dj;
  T uu[NORD + 3], rri[NORD + 3], rrj[NORD + 3], ssv[NORD + 3], ttv[NORD + 3];
  uu[0] = uu[1] = rri[0] = rri[1] = rrj[0] = rrj[1] = ssv[0] = ssv[1] = ttv[0] = ttv[1] = T(0);
  uu[2] = 1; ssv[2] = 2; ttv[2] = 1; rri[2] = 1; rrj[2] = 1;
#pragma unroll
  for (int i = 1; i <= NORD; i++) {
    uu[i + 2] = uu[i + 1] * u1;
    rri[i + 2] = rri[i + 1] * ri1;
    rrj[i + 2] = rrj[i + 1] * rj1;
    ssv[i + 2] = rri[i + 2] + rrj[i + 2];
    ttv[i + 2] = rri[i + 2] * rrj[i + 2];
  }
  T fc = 0, fu = 0, fuu = 0, fi = 0, fii = 0, fj = 0, fjj = 0, fui = 0, fuj = 0;
  const T *c = J.c[it];
#pragma unroll
  for (int ll = 0; ll < tl.n; ll++) {
    const int k = tl.k[ll], l = tl.l[ll], m = tl.m[ll];
    T cc = c[ll];
    T st = ssv[l + 2] * ttv[m + 2];
    fc += cc * uu[k + 2] * st;
    if (LEVEL >= 1) {
      T pi_ = T(l + m) * rri[l + m + 1] * rrj[m + 2] + T(m) * rri[m + 1] * rrj[l + m + 2];
      T pj_ = T(l + m) * rrj[l + m + 1] * rri[m + 2] + T(m) * rrj[m + 1] * rri[l + m + 2];
      fu += cc * T(k) * uu[k + 1] * st;
      fi += cc * uu[k + 2] * pi_;
      fj += cc * uu[k + 2] * pj_;
      if (LEVEL >= 2) {
        fuu += cc * T(k * (k - 1)) * uu[k] * st;
        fii += cc * uu[k + 2] * (T((l + m) * (l + m - 1)) * rri[l + m] * rrj[m + 2] + T(m * (m - 1)) * rri[m] * rrj[l + m + 2]);
        fjj += cc * uu[k + 2] * (T((l + m) * (l + m - 1)) * rrj[l + m] * rri[m + 2] + T(m * (m - 1)) * rrj[m] * rri[l + m + 2]);
        fui += cc * T(k) * uu[k + 1] * pi_;
        fuj += cc * T(k) * uu[k + 1] * pj_;
      }
    }
  }
  o.fc = fc;
  if (LEVEL >= 1) {
    // derivatives of the switched scaled distances: -k d^2 and 2 k^2 d^3
    T dd1 = -sk * du * du, dd7 = -sk * di * di, dd8 = -sk * dj * dj;
    if (LEVEL >= 2) {
      T dd2 = 2 * sk * sk * du * du * du, dd9 = 2 * sk * sk * di * di * di, dd10 = 2 * sk * sk * dj * dj * dj;
      o.fuu = fuu * dd1 * dd1 + fu * dd2;
      o.fui = fui * dd1 * dd7;
      o.fuj = fuj * dd1 * dd8;
      o.fii = fii * dd7 * dd7 + fi * dd9;
      o.fjj = fjj * dd8 * dd8 + fj * dd10;
    }
    o.fu = fu * dd1 / rij;
    o.fi = fi * dd7 / ri;
    o.fj = fj * dd8 / rj;
  }
}

}  // namespace champ
