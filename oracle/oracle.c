/*
 * oracle.c -- FP64 CPU restatement of CHAMP's Slater-Jastrow hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library.
 *
 * Each routine cites the reference routine whose arithmetic it restates
 * (paths relative to the CHAMP source tree).  The reference cannot be compiled
 * here (no Fortran compiler); parity of this restatement is pinned by the
 * reference's own finite-difference checks and by its example VMC energies.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXORD 8
#define MAXLCH CHAMP_MAX_LCHAN
#define HB 0.5 /* hbar^2/2m in Hartree atomic units (const_mod hb) */

/* ------------------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).                                    */
/* ------------------------------------------------------------------------------------ */
void orc_philox(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t *out) {
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
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

static double u53(uint32_t a, uint32_t b) {
  return ((double)(((uint64_t)(a >> 5) << 26) | (b >> 6)) + 0.5) * (1.0 / 9007199254740992.0);
}
static double u32d(uint32_t a) { return ((double)a + 0.5) * (1.0 / 4294967296.0); }

void orc_random_rotation(uint64_t seed, uint32_t walker, uint64_t sweep, double *R) {
  uint32_t o[4];
  orc_philox(seed, walker, (uint32_t)sweep, (uint32_t)(sweep >> 32), 0xFFFFFFFFu, o);
  double u1 = u53(o[0], o[1]), u2 = u32d(o[2]), u3 = u32d(o[3]);
  const double tp = 6.283185307179586;
  double s1 = sqrt(1.0 - u1), s2 = sqrt(u1);
  double qx = s1 * sin(tp * u2), qy = s1 * cos(tp * u2), qz = s2 * sin(tp * u3), qw = s2 * cos(tp * u3);
  R[0] = 1 - 2 * (qy * qy + qz * qz); R[1] = 2 * (qx * qy - qz * qw); R[2] = 2 * (qx * qz + qy * qw);
  R[3] = 2 * (qx * qy + qz * qw); R[4] = 1 - 2 * (qx * qx + qz * qz); R[5] = 2 * (qy * qz - qx * qw);
  R[6] = 2 * (qx * qz - qy * qw); R[7] = 2 * (qy * qz + qx * qw); R[8] = 1 - 2 * (qx * qx + qy * qy);
}

/* Gaussian proposal displacement and accept uniform for (seed, walker, sweep, electron). */
static void move_randoms(uint64_t seed, uint32_t w, uint64_t sweep, uint32_t e, double *g, double *ua) {
  uint32_t a[4], b[4];
  orc_philox(seed, w, (uint32_t)sweep, (uint32_t)(sweep >> 32), 2u * e, a);
  orc_philox(seed, w, (uint32_t)sweep, (uint32_t)(sweep >> 32), 2u * e + 1u, b);
  const double tp = 6.283185307179586;
  double u1 = u53(a[0], a[1]), u2 = u53(a[2], a[3]);
  double u3 = u53(b[0], b[1]), u4 = u32d(b[2]);
  double r1 = sqrt(-2.0 * log(u1)), r2 = sqrt(-2.0 * log(u3));
  g[0] = r1 * cos(tp * u2);
  g[1] = r1 * sin(tp * u2);
  g[2] = r2 * cos(tp * u4);
  *ua = u32d(b[3]);
}

/* ------------------------------------------------------------------------------------ */
/* System set-up                                                                         */
/* ------------------------------------------------------------------------------------ */
struct orc_sys {
  int N, nup, ndn, C, nct;
  double *cent;
  int *ctype;
  double *znuc;
  double pecent;
  int nshell, nprim, nbasis, norb;
  int *sh_cent, *sh_n, *sh_l, *sh_kind, *sh_np, *sh_p0;
  double *pz, *pc; /* primitive exponents and normalised weights */
  int *b_shell, *b_m;
  double *coef; /* [norb][nbasis] */
  int ndet;
  int *det_orb;
  double *cdet; /* combined det coefficient (cdet_in_wf) */
  int nocc[2];
  int occ[2][CHAMP_MAX_ELEC];
  /* Jastrow */
  double scalek;
  int norda, nordb, nordc, nspin2b, nterms;
  double a4[CHAMP_MAX_CTYPE][MAXORD + 1], b[2][MAXORD + 1];
  double *c; /* [nct][nterms] */
  int tk[64], tl[64], tm[64];
  double asymp_r, asymp_jasa[CHAMP_MAX_CTYPE], asymp_jasb[2];
  int een_cusp;
  /* pseudopotential */
  int nloc, nquad, mgauss;
  int npotd[CHAMP_MAX_CTYPE], lpotp1[CHAMP_MAX_CTYPE];
  int *necp_term, *necp_power;
  double *ecp_coef, *ecp_exp;
  double q0[86][3], wq[86], q[86][3];
  /* numerical radial tables (kind-2 shells): grid type, points, derived r0, h, the small-r
     polynomial, the large-r exponential, values and spline second derivatives */
  int nrad, *rad_of_shell;
  int *rt_grid, *rt_nr;
  double *rt_r0, *rt_h, (*rt_ce)[5], (*rt_ae)[2];
  double **rt_y, **rt_y2;
};

int orc_nterms4(int nord) {
  /* nterms4 (qmc/vmc/jastrow4.f90:495-516) */
  int i = 0;
  for (int n = 2; n <= nord; n++)
    for (int k = n - 1; k >= 0; k--) {
      int l_hi = (k == 0) ? n - k - 2 : n - k;
      for (int l = l_hi; l >= 0; l--) {
        int m = (n - k - l) / 2;
        if (2 * m == n - k - l) i++;
      }
    }
  return i;
}

static double fact(int n) {
  double f = 1;
  for (int i = 2; i <= n; i++) f *= i;
  return f;
}

/* Radial normalisation incl. sqrt((2l+1)/4pi) (qmc/vmc/basis_norm.f90:53-60). */
static double basis_anorm(int kind, int n, int l, double z) {
  const double pi = 3.141592653589793;
  if (kind == 0) return sqrt(pow(2 * z, 2 * n + 1) * (2 * l + 1) / (fact(2 * n) * 4 * pi));
  /* Gamma(n+1/2) (gamma1 in basis_norm.f90) */
  double g = sqrt(pi);
  for (int i = 1; i <= n; i++) g *= (i - 0.5);
  return sqrt(2 * pow(2 * z, n + 0.5) * (2 * l + 1) / (g * 4 * pi));
}

/* Cusp conditions on the e-e-n coefficients (qmc/fit/cuspinit4.f90:1-60 builds d and
   iwc4; qmc/fit/cuspexact4.f90:14-40 solves for the dependent coefficients). */
static void een_cusp(orc_sys *s, int *dep_out) {
  int nordc = s->nordc, nt = s->nterms;
  if (nordc <= 1) return;
  int neq = 2 * (nordc - 1);
  double d[2 * MAXORD][64];
  int iwc4[2 * MAXORD];
  memset(d, 0, sizeof d);
  for (int i = 0; i < neq; i++) iwc4[i] = 0;
  int i = 0;
  for (int n = 2; n <= nordc; n++)
    for (int k = n - 1; k >= 0; k--) {
      int l_hi = (k == 0) ? n - k - 2 : n - k;
      for (int l = l_hi; l >= 0; l--) {
        int m = (n - k - l) / 2;
        if (2 * m != n - k - l) continue;
        i++;
        if (k == 1 && iwc4[n - 2] == 0) iwc4[n - 2] = i;
        if (k == 0 && iwc4[n + nordc - 3] == 0) iwc4[n + nordc - 3] = i;
        int iord = l + 2 * m;
        d[iord - 1][i - 1] -= 2 * k;
        if (l + m > 0) { iord = nordc - 1 + k + m; d[iord - 1][i - 1] -= (l + m); }
        if (m > 0) { iord = nordc - 1 + k + l + m; d[iord - 1][i - 1] -= m; }
      }
    }
  if (dep_out)
    for (int e = 0; e < neq; e++) dep_out[e] = iwc4[e] - 1;
  for (int it = 0; it < s->nct; it++) {
    double *c = s->c + (size_t)it * nt;
    int order[2 * MAXORD], no = 0;
    for (int e = 1; e <= nordc - 1; e++) order[no++] = e;
    for (int e = nordc + 1; e <= neq; e++) order[no++] = e;
    order[no++] = nordc;
    for (int q = 0; q < no; q++) {
      int e = order[q];
      int jd = iwc4[e - 1];
      double sum = 0;
      for (int j = 1; j <= nt; j++)
        if (j != jd) sum += d[e - 1][j - 1] * c[j - 1];
      c[jd - 1] = -sum / d[e - 1][jd - 1];
    }
  }
}
static void apply_een_cusp(orc_sys *s) { een_cusp(s, NULL); }

/* asymptotic values of the e-n and e-e terms (set_scale_dist, qmc/vmc/scale_dist.f90:147-225,
   isc=4 branch) */
static void set_asymptotes(orc_sys *s) {
  s->asymp_r = 1.0 / s->scalek;
  double ar = s->asymp_r;
  for (int it = 0; it < s->nct; it++) {
    double v = s->a4[it][0] * ar / (1 + s->a4[it][1] * ar);
    for (int iord = 2; iord <= s->norda; iord++) v += s->a4[it][iord] * pow(ar, iord);
    s->asymp_jasa[it] = v;
  }
  for (int i = 0; i < 2; i++) {
    double sspinn = 1;
    int isp = 0;
    if (i == 1) {
      sspinn = (s->nspin2b == 1) ? 0.5 : 1.0;
      isp = s->nspin2b - 1;
    }
    double v = sspinn * s->b[isp][0] * ar / (1 + s->b[isp][1] * ar);
    for (int iord = 2; iord <= s->nordb; iord++) v += s->b[isp][iord] * pow(ar, iord);
    s->asymp_jasb[i] = v;
  }
}

static void *dupmem(const void *p, size_t n) {
  if (!p || n == 0) return calloc(1, n ? n : 1);
  void *q = malloc(n);
  memcpy(q, p, n);
  return q;
}

/* gesqua (qmc/vmc/rotqua.f90:1-618): of the rules with 4, 6, 12, 18, 26, 32, 50, 24, 20 and 86
   points the one closest to nq (first on ties).  Points are generated by symmetry type as the
   reference does; weights by point type.  Returns the number of points. */
static int gesqua(int nq_in, double q[][3], double *w) {
  static const int iq[10] = {4, 6, 12, 18, 26, 32, 50, 24, 20, 86};
  int best = 0;
  for (int i = 1; i < 10; i++)
    if (abs(nq_in - iq[i]) < abs(nq_in - iq[best])) best = i;
  int nq = iq[best];
  memset(q, 0, sizeof(double) * 3 * 86);
  memset(w, 0, sizeof(double) * 86);
  /* weight of each point type per rule (ww of the reference) and the types' sizes */
  double wt[10][6];
  memset(wt, 0, sizeof wt);
  wt[0][0] = 1.0 / 4.0;  wt[1][0] = 1.0 / 6.0;  wt[2][0] = 1.0 / 12.0; wt[2][1] = 1.0 / 12.0;
  wt[3][0] = 1.0 / 30.0; wt[3][1] = 1.0 / 15.0;
  wt[4][0] = 1.0 / 21.0; wt[4][1] = 4.0 / 105.0; wt[4][2] = 27.0 / 840.0;
  wt[5][0] = 5.0 / 168.0; wt[5][1] = 5.0 / 168.0; wt[5][2] = 27.0 / 840.0;
  wt[6][0] = 4.0 / 315.0; wt[6][1] = 64.0 / 2835.0; wt[6][2] = 27.0 / 1280.0; wt[6][3] = 14641.0 / 725760.0;
  wt[7][0] = 1.0 / 24.0; wt[8][0] = 1.0 / 20.0;
  wt[9][0] = .0115440115441; wt[9][2] = .0119439090859; wt[9][3] = .0111105557106;
  wt[9][4] = .0118765012945; wt[9][5] = .0118123037469;
  int sizes[6] = {6, 12, 8, 24, 0, 0}, ntyp = 4;
  if (nq == 4) { sizes[0] = 4; sizes[1] = sizes[2] = sizes[3] = 0; }
  if (nq == 12 || nq == 32) { sizes[0] = 2; sizes[1] = 10; sizes[2] = 20; sizes[3] = 0; }
  if (nq == 20) { sizes[0] = 20; sizes[1] = sizes[2] = sizes[3] = 0; }
  if (nq == 24) { sizes[0] = 24; sizes[1] = sizes[2] = sizes[3] = 0; }
  if (nq == 86) { int s86[6] = {6, 0, 8, 24, 24, 24}; memcpy(sizes, s86, sizeof s86); ntyp = 6; }
  for (int k = 0, j = 0; k < ntyp; k++)
    for (int i = 0; i < sizes[k]; i++, j++)
      if (j < nq) w[j] = wt[best][k];
  const double pi = 3.14159265359, a = 1.0 / sqrt(2.0), b = 1.0 / sqrt(3.0), c11 = 1.0 / sqrt(11.0),
               d11 = 3.0 / sqrt(11.0);
  if (nq == 4) {
    /* tetrahedron: (+,+,+) (+,-,-) (-,+,-) (-,-,+) scaled by 1/sqrt(3) */
    static const int sg[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
    for (int j = 0; j < 4; j++)
      for (int k = 0; k < 3; k++) q[j][k] = sg[j][k] * b;
  } else if (nq == 6 || nq == 18 || nq == 26 || nq == 50) {
    /* octahedral families: the 6 axis points; 12 edge midpoints; 8 cube corners; 24 (r,r,s) */
    int m = 6, n8 = 0;
    for (int k = 0; k < 3; k++) { q[2 * k][k] = 1; q[2 * k + 1][k] = -1; }
    if (nq > 6) {
      /* pairs in (x,y), (y,z), (z,x) planes, the reference's order: for each sign of the first
         coordinate and of the second */
      for (int s1 = 0; s1 < 2; s1++)
        for (int s2 = 0; s2 < 2; s2++) {
          double u = s1 ? -a : a, v = s2 ? -a : a;
          int i = 2 * s1 + s2;
          q[6 + i][0] = u;  q[6 + i][1] = v;
          q[10 + i][1] = u; q[10 + i][2] = v;
          q[14 + i][2] = u; q[14 + i][0] = v;
        }
      m = 18;
    }
    if (nq > 18) {
      for (int s1 = 0; s1 < 2; s1++)
        for (int s2 = 0; s2 < 2; s2++)
          for (int s3 = 0; s3 < 2; s3++, n8++) {
            double sx = s1 ? -1 : 1, sy = s2 ? -1 : 1, sz = s3 ? -1 : 1;
            q[18 + n8][0] = sx * b; q[18 + n8][1] = sy * b; q[18 + n8][2] = sz * b;
            if (nq > 26) {
              q[26 + n8][0] = sx * c11; q[26 + n8][1] = sy * c11; q[26 + n8][2] = sz * d11;
              q[34 + n8][0] = sx * c11; q[34 + n8][1] = sy * d11; q[34 + n8][2] = sz * c11;
              q[42 + n8][0] = sx * d11; q[42 + n8][1] = sy * c11; q[42 + n8][2] = sz * c11;
            }
          }
    }
    (void)m;
  } else if (nq == 12 || nq == 20 || nq == 32) {
    /* icosahedral families: poles + two rings of 5 at z = +-1/sqrt(5) (12); the 20 dodecahedron
       vertices (20, overwriting the poles); both (32) */
    double s5 = sqrt(5.0), den = sqrt(15.0 + 6.0 * s5);
    double ct = 1.0 / s5, st = 2.0 / s5, c1 = (2.0 + s5) / den, s1 = sqrt(1.0 - c1 * c1), c2 = 1.0 / den,
           s2 = sqrt(1.0 - c2 * c2);
    q[0][2] = 1.0; q[1][2] = -1.0;
    for (int j = 0; j < 5; j++) {
      double ph0 = 2.0 * j * pi / 5.0, ph1 = (2.0 * j + 1.0) * pi / 5.0;
      if (nq != 20) {
        q[2 + j][0] = st * cos(ph0); q[2 + j][1] = st * sin(ph0); q[2 + j][2] = ct;
        q[7 + j][0] = st * cos(ph1); q[7 + j][1] = st * sin(ph1); q[7 + j][2] = -ct;
      }
      if (nq > 12) {
        int k0 = nq == 20 ? 0 : 12;
        q[k0 + j][0] = s1 * cos(ph1);      q[k0 + j][1] = s1 * sin(ph1);      q[k0 + j][2] = c1;
        q[k0 + 5 + j][0] = s2 * cos(ph1);  q[k0 + 5 + j][1] = s2 * sin(ph1);  q[k0 + 5 + j][2] = c2;
        q[k0 + 10 + j][0] = s1 * cos(ph0); q[k0 + 10 + j][1] = s1 * sin(ph0); q[k0 + 10 + j][2] = -c1;
        q[k0 + 15 + j][0] = s2 * cos(ph0); q[k0 + 15 + j][1] = s2 * sin(ph0); q[k0 + 15 + j][2] = -c2;
      }
    }
  } else if (nq == 24) {
    /* one point, its images under the three cyclic coordinate shifts, each also turned by -90
       degrees about y, then all rotated about z in steps of 90 degrees */
    double p3[3] = {.8662468181078, .4225186537611, .2666354015167};
    int n = 0;
    for (int l = 0; l < 3; l++) {
      double x, y, z;
      if (l == 0) { x = p3[0]; y = p3[1]; z = p3[2]; }
      else if (l == 1) { x = p3[2]; y = p3[0]; z = p3[1]; }
      else { x = p3[1]; y = p3[2]; z = p3[0]; }
      double u = -z * sin(-pi / 2.0) + x * cos(-pi / 2.0), v = y, t = x * sin(-pi / 2.0) + z * cos(-pi / 2.0);
      for (int m = 0; m < 4; m++) {
        double f = pi * m / 2.0, cf = cos(f), sf = sin(f);
        q[n][0] = x * cf - y * sf; q[n][1] = x * sf + y * cf; q[n][2] = z; n++;
        q[n][0] = u * cf - v * sf; q[n][1] = u * sf + v * cf; q[n][2] = t; n++;
      }
    }
  } else {
    /* 86 points: axes; cube corners; three families of 24 (r,r,s); 24 (p,q,0) */
    double pp = .927330657151, qq = .374243039090, r1 = .369602846454, m1 = .852518311701,
           r2 = .694354006603, m2 = .189063552885;
    for (int k = 0; k < 3; k++) { q[2 * k][k] = 1; q[2 * k + 1][k] = -1; }
    for (int s1 = 0; s1 < 2; s1++)
      for (int s2 = 0; s2 < 2; s2++) {
        double u = s1 ? -1 : 1, v = s2 ? -1 : 1;
        int i = 2 * s1 + s2;
        q[62 + i][0] = u * pp; q[62 + i][1] = v * qq;
        q[66 + i][0] = u * pp; q[66 + i][2] = v * qq;
        q[70 + i][1] = u * pp; q[70 + i][2] = v * qq;
        q[74 + i][0] = u * qq; q[74 + i][1] = v * pp;
        q[78 + i][0] = u * qq; q[78 + i][2] = v * pp;
        q[82 + i][1] = u * qq; q[82 + i][2] = v * pp;
        for (int s3 = 0; s3 < 2; s3++) {
          double t = s3 ? -1 : 1;
          int k = 4 * s1 + 2 * s2 + s3;
          q[6 + k][0] = u * b;   q[6 + k][1] = v * b;   q[6 + k][2] = t * b;
          q[14 + k][0] = u * r1; q[14 + k][1] = v * r1; q[14 + k][2] = t * m1;
          q[22 + k][0] = u * r1; q[22 + k][1] = v * m1; q[22 + k][2] = t * r1;
          q[30 + k][0] = u * m1; q[30 + k][1] = v * r1; q[30 + k][2] = t * r1;
          q[38 + k][0] = u * r2; q[38 + k][1] = v * r2; q[38 + k][2] = t * m2;
          q[46 + k][0] = u * r2; q[46 + k][1] = v * m2; q[46 + k][2] = t * r2;
          q[54 + k][0] = u * m2; q[54 + k][1] = v * r2; q[54 + k][2] = t * r2;
        }
      }
  }
  return nq;
}

/* Numerical radial function tables (qmc/vmc/read_bas_num.f90:213-378): grid parameters as
   splfit_bas uses them; c_k of the polynomial through the first five grid points (ncoef = 5,
   the fit used with pseudopotentials); a0 exp(-ak r) from the last two points; the clamped
   cubic spline of spline2 (Numerical Recipes p. 88) with the polynomial's slope at the first
   point and the exponential's at the last. */
static void build_tables(orc_sys *s, const champ_system *d) {
  s->nrad = d->nrad;
  s->rad_of_shell = (int *)calloc(s->nshell, sizeof(int));
  for (int i = 0; i < s->nshell; i++) s->rad_of_shell[i] = (s->sh_kind[i] == 2 && d->shell_rad) ? d->shell_rad[i] : -1;
  if (s->nrad <= 0) return;
  int nt = s->nrad;
  s->rt_grid = (int *)calloc(nt, sizeof(int)); s->rt_nr = (int *)calloc(nt, sizeof(int));
  s->rt_r0 = (double *)calloc(nt, sizeof(double)); s->rt_h = (double *)calloc(nt, sizeof(double));
  s->rt_ce = (double(*)[5])calloc(nt, sizeof(double[5])); s->rt_ae = (double(*)[2])calloc(nt, sizeof(double[2]));
  s->rt_y = (double **)calloc(nt, sizeof(double *)); s->rt_y2 = (double **)calloc(nt, sizeof(double *));
  size_t off = 0;
  for (int t = 0; t < nt; t++) {
    int g = d->rad_igrid[t], n = d->rad_nr[t];
    const double *x = d->rad_x + off, *y = d->rad_val + off;
    double h = d->rad_h[t], r0 = d->rad_r0[t];
    if (g == 2 && h <= 1.0) h = x[1] / x[0];
    if (g == 3) r0 = r0 / (pow(h, n - 1) - 1.0);
    if (g == 2 && (r0 <= 0 || h <= 0)) { r0 = x[0]; h = x[1] / x[0]; }
    s->rt_grid[t] = g; s->rt_nr[t] = n; s->rt_r0[t] = r0; s->rt_h[t] = h;
    /* Vandermonde system of the first five points, Gaussian elimination with partial pivoting */
    double m[5][6];
    for (int i = 0; i < 5; i++) {
      for (int j = 0; j < 5; j++) m[i][j] = pow(x[i], j);
      m[i][5] = y[i];
    }
    for (int k = 0; k < 5; k++) {
      int pv = k;
      for (int i = k + 1; i < 5; i++) if (fabs(m[i][k]) > fabs(m[pv][k])) pv = i;
      for (int j = 0; j < 6; j++) { double tmp = m[k][j]; m[k][j] = m[pv][j]; m[pv][j] = tmp; }
      for (int i = k + 1; i < 5; i++) {
        double f = m[i][k] / m[k][k];
        for (int j = k; j < 6; j++) m[i][j] -= f * m[k][j];
      }
    }
    for (int i = 4; i >= 0; i--) {
      double acc = m[i][5];
      for (int j = i + 1; j < 5; j++) acc -= m[i][j] * s->rt_ce[t][j];
      s->rt_ce[t][i] = acc / m[i][i];
    }
    double yp1 = 0;
    for (int i = 1; i < 5; i++) yp1 += i * s->rt_ce[t][i] * pow(x[0], i - 1);
    double wfm = 0.5 * (y[n - 1] + y[n - 2]), dwfm = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]), ypn = 0;
    if (fabs(wfm) > 1e-99) {
      s->rt_ae[t][1] = dwfm / wfm < 0 ? -dwfm / wfm : 0.1;
      s->rt_ae[t][0] = y[n - 1] * exp(s->rt_ae[t][1] * x[n - 1]);
      ypn = -s->rt_ae[t][1] * y[n - 1];
    }
    double *y2 = (double *)calloc(n, sizeof(double)), *wk = (double *)calloc(n, sizeof(double));
    y2[0] = -0.5;
    wk[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1);
    for (int i = 1; i < n - 1; i++) {
      double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]), p = sig * y2[i - 1] + 2.0;
      y2[i] = (sig - 1.0) / p;
      wk[i] = (6.0 * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1])) /
                   (x[i + 1] - x[i - 1]) - sig * wk[i - 1]) / p;
    }
    double un = (3.0 / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]));
    y2[n - 1] = (un - 0.5 * wk[n - 2]) / (0.5 * y2[n - 2] + 1.0);
    for (int k = n - 2; k >= 0; k--) y2[k] = y2[k] * y2[k + 1] + wk[k];
    free(wk);
    s->rt_y2[t] = y2;
    s->rt_y[t] = (double *)dupmem(y, sizeof(double) * n);
    off += n;
  }
}

/* splfit_bas (qmc/vmc/splfit.f90): f, f', f'' of table t at r. */
static void table_fit(const orc_sys *s, int t, double r, double *f) {
  int g = s->rt_grid[t], n = s->rt_nr[t], jx;
  double r0 = s->rt_r0[t], h = s->rt_h[t], ref0, ref1;
  if (g == 1) {
    jx = (int)((r - r0) / h + 1);
    ref0 = r0 + h * (jx - 1); ref1 = ref0 + h;
  } else if (g == 2) {
    double xr = log(r / r0) / log(h) + 1;
    jx = xr < 1 ? 0 : (int)xr;
    ref0 = r0 * pow(h, jx - 1); ref1 = ref0 * h;
  } else {
    jx = (int)(log((r + r0) / r0) / log(h) + 1.0);
    ref0 = r0 * pow(h, jx - 1) - r0; ref1 = (ref0 + r0) * h - r0;
  }
  const double *ce = s->rt_ce[t];
  if (jx < 1) {
    f[0] = ce[0]; f[1] = 0; f[2] = 0;
    for (int i = 1; i < 5; i++) {
      f[0] += ce[i] * pow(r, i);
      f[1] += i * ce[i] * pow(r, i - 1);
      if (i >= 2) f[2] += i * (i - 1) * ce[i] * pow(r, i - 2);
    }
  } else if (jx >= n) {
    f[0] = s->rt_ae[t][0] * exp(-s->rt_ae[t][1] * r);
    f[1] = -s->rt_ae[t][1] * f[0];
    f[2] = -s->rt_ae[t][1] * f[1];
  } else {
    const double *y = s->rt_y[t] + jx - 1, *y2 = s->rt_y2[t] + jx - 1;
    double dh = ref1 - ref0, bb = (r - ref0) / dh, aa = (ref1 - r) / dh;
    double cc = aa * (aa * aa - 1) * dh * dh / 6, dd = bb * (bb * bb - 1) * dh * dh / 6;
    f[0] = aa * y[0] + bb * y[1] + cc * y2[0] + dd * y2[1];
    f[1] = (y[1] - y[0]) / dh + (-(3 * aa * aa - 1) * y2[0] + (3 * bb * bb - 1) * y2[1]) * dh / 6;
    f[2] = aa * y2[0] + bb * y2[1];
  }
}


orc_sys *orc_create(const champ_system *d) {
  orc_sys *s = (orc_sys *)calloc(1, sizeof(orc_sys));
  s->N = d->nelec; s->nup = d->nup; s->ndn = d->nelec - d->nup;
  s->C = d->ncent; s->nct = d->nctype;
  s->cent = (double *)dupmem(d->cent, sizeof(double) * 3 * s->C);
  s->ctype = (int *)dupmem(d->iwctype, sizeof(int) * s->C);
  s->znuc = (double *)dupmem(d->znuc, sizeof(double) * s->nct);
  /* nuclear repulsion pecent */
  s->pecent = 0;
  for (int i = 0; i < s->C; i++)
    for (int j = 0; j < i; j++) {
      double dx = s->cent[3 * i] - s->cent[3 * j], dy = s->cent[3 * i + 1] - s->cent[3 * j + 1],
             dz = s->cent[3 * i + 2] - s->cent[3 * j + 2];
      s->pecent += s->znuc[s->ctype[i]] * s->znuc[s->ctype[j]] / sqrt(dx * dx + dy * dy + dz * dz);
    }
  s->nshell = d->nshell;
  s->sh_cent = (int *)dupmem(d->shell_cent, sizeof(int) * s->nshell);
  s->sh_n = (int *)dupmem(d->shell_n, sizeof(int) * s->nshell);
  s->sh_l = (int *)dupmem(d->shell_l, sizeof(int) * s->nshell);
  s->sh_kind = (int *)dupmem(d->shell_kind, sizeof(int) * s->nshell);
  s->sh_np = (int *)dupmem(d->shell_nprim, sizeof(int) * s->nshell);
  s->sh_p0 = (int *)calloc(s->nshell + 1, sizeof(int));
  for (int i = 0; i < s->nshell; i++) s->sh_p0[i + 1] = s->sh_p0[i] + s->sh_np[i];
  s->nprim = s->sh_p0[s->nshell];
  s->pz = (double *)dupmem(d->prim_zeta, sizeof(double) * s->nprim);
  s->pc = (double *)dupmem(d->prim_coef, sizeof(double) * s->nprim);
  for (int i = 0; i < s->nshell; i++)
    for (int p = s->sh_p0[i]; p < s->sh_p0[i + 1]; p++)
      s->pc[p] *= s->sh_kind[i] == 2 ? sqrt((2 * s->sh_l[i] + 1) / (4 * 3.141592653589793))
                                     : basis_anorm(s->sh_kind[i], s->sh_n[i], s->sh_l[i], s->pz[p]);
  build_tables(s, d);
  s->nbasis = d->nbasis;
  s->b_shell = (int *)dupmem(d->basis_shell, sizeof(int) * s->nbasis);
  s->b_m = (int *)dupmem(d->basis_m, sizeof(int) * s->nbasis);
  s->norb = d->norb;
  s->coef = (double *)dupmem(d->coef, sizeof(double) * s->norb * s->nbasis);
  s->ndet = d->ndet;
  s->det_orb = (int *)dupmem(d->det_orb, sizeof(int) * s->ndet * s->N);
  /* cdet_in_wf (qmc/deriv_fast_mod.f90:144-172) */
  s->cdet = (double *)calloc(s->ndet, sizeof(double));
  {
    int off = 0;
    for (int icsf = 0; icsf < d->ncsf; icsf++) {
      for (int i = 0; i < d->csf_ndet[icsf]; i++, off++)
        s->cdet[d->csf_det[off]] += d->csf_det_coef[off] * d->csf_coef[icsf];
    }
  }
  /* occupied orbitals per spin (occ_bld, qmc/deriv_fast_mod.f90:211) */
  for (int sp = 0; sp < 2; sp++) {
    int n0 = sp ? s->nup : 0, n1 = sp ? s->N : s->nup;
    int used[4096] = {0};
    s->nocc[sp] = 0;
    for (int i = 0; i < s->ndet; i++)
      for (int e = n0; e < n1; e++) used[s->det_orb[i * s->N + e]] = 1;
    for (int o = 0; o < s->norb; o++)
      if (used[o]) s->occ[sp][s->nocc[sp]++] = o;
  }
  /* Jastrow */
  s->scalek = d->scalek;
  s->norda = d->norda; s->nordb = d->nordb; s->nordc = d->nordc; s->nspin2b = d->nspin2b;
  s->nterms = orc_nterms4(s->nordc);
  for (int it = 0; it < s->nct; it++)
    for (int k = 0; k <= s->norda; k++) s->a4[it][k] = d->a4[it * (s->norda + 1) + k];
  for (int is = 0; is < s->nspin2b; is++)
    for (int k = 0; k <= s->nordb; k++) s->b[is][k] = d->b[is * (s->nordb + 1) + k];
  s->c = (double *)calloc((size_t)s->nct * (s->nterms ? s->nterms : 1), sizeof(double));
  if (s->nterms) memcpy(s->c, d->c, sizeof(double) * s->nct * s->nterms);
  {
    int ll = 0;
    for (int n = 2; n <= s->nordc; n++)
      for (int k = n - 1; k >= 0; k--) {
        int l_hi = (k == 0) ? n - k - 2 : n - k;
        for (int l = l_hi; l >= 0; l--) {
          int m = (n - k - l) / 2;
          if (2 * m == n - k - l) { s->tk[ll] = k; s->tl[ll] = l; s->tm[ll] = m; ll++; }
        }
      }
  }
  s->een_cusp = d->een_cusp;
  if (d->een_cusp) apply_een_cusp(s);
  set_asymptotes(s);
  /* pseudopotential */
  s->nloc = d->nloc;
  s->nquad = d->nquad > 0 ? d->nquad : 12;
  s->mgauss = d->mgauss;
  if (s->nloc > 0) {
    size_t nt = (size_t)s->nct * MAXLCH;
    for (int it = 0; it < s->nct; it++) { s->npotd[it] = d->npotd[it]; s->lpotp1[it] = d->lpotp1[it]; }
    s->necp_term = (int *)dupmem(d->necp_term, sizeof(int) * nt);
    s->necp_power = (int *)dupmem(d->necp_power, sizeof(int) * nt * s->mgauss);
    s->ecp_coef = (double *)dupmem(d->ecp_coef, sizeof(double) * nt * s->mgauss);
    s->ecp_exp = (double *)dupmem(d->ecp_exponent, sizeof(double) * nt * s->mgauss);
  }
  s->nquad = gesqua(s->nloc > 0 ? s->nquad : 12, s->q0, s->wq);
  orc_set_rotation(s, NULL);
  return s;
}

void orc_destroy(orc_sys *s) {
  if (!s) return;
  free(s->cent); free(s->ctype); free(s->znuc);
  free(s->sh_cent); free(s->sh_n); free(s->sh_l); free(s->sh_kind); free(s->sh_np); free(s->sh_p0);
  free(s->pz); free(s->pc); free(s->b_shell); free(s->b_m); free(s->coef);
  free(s->det_orb); free(s->cdet); free(s->c);
  free(s->necp_term); free(s->necp_power); free(s->ecp_coef); free(s->ecp_exp);
  for (int t = 0; t < s->nrad && s->rt_y; t++) { free(s->rt_y[t]); free(s->rt_y2[t]); }
  free(s->rt_y); free(s->rt_y2); free(s->rt_grid); free(s->rt_nr); free(s->rt_r0); free(s->rt_h);
  free(s->rt_ce); free(s->rt_ae); free(s->rad_of_shell);
  free(s);
}

void orc_get_c(const orc_sys *s, double *c) {
  if (s->nterms) memcpy(c, s->c, sizeof(double) * s->nct * s->nterms);
}

void orc_set_rotation(orc_sys *s, const double *R) {
  /* rotqua (qmc/vmc/rotqua.f90:621-680): xq = R * xq0 */
  for (int iq = 0; iq < s->nquad; iq++)
    for (int k = 0; k < 3; k++) {
      if (!R) { s->q[iq][k] = s->q0[iq][k]; continue; }
      s->q[iq][k] = R[3 * k] * s->q0[iq][0] + R[3 * k + 1] * s->q0[iq][1] + R[3 * k + 2] * s->q0[iq][2];
    }
}

void orc_quadrature(const orc_sys *s, double *xyzw) {
  for (int iq = 0; iq < s->nquad; iq++) {
    xyzw[4 * iq] = s->q[iq][0]; xyzw[4 * iq + 1] = s->q[iq][1];
    xyzw[4 * iq + 2] = s->q[iq][2]; xyzw[4 * iq + 3] = s->wq[iq];
  }
}

/* ------------------------------------------------------------------------------------ */
/* Basis functions (qmc/vmc/basis_fns.f90:38-474)                                        */
/* ------------------------------------------------------------------------------------ */
/* Real solid harmonics S_lm(r) = r^l * C_lm(rhat), with the normalisation and sign of
   the th(l,|m|)*ph(m) products of basis_fns.f90:175-330, and their gradients. */
static void solid_harm(int l, int m, double x, double y, double z, double *S, double *g) {
  double x2 = x * x, y2 = y * y, z2 = z * z, rho2 = x2 + y2;
  g[0] = g[1] = g[2] = 0;
  switch (l) {
  case 0: *S = 1; return;
  case 1:
    if (m == 1) { *S = x; g[0] = 1; }
    else if (m == -1) { *S = y; g[1] = 1; }
    else { *S = z; g[2] = 1; }
    return;
  case 2: {
    const double s3 = sqrt(3.0);
    if (m == 0) { *S = 0.5 * (2 * z2 - rho2); g[0] = -x; g[1] = -y; g[2] = 2 * z; }
    else if (m == 1) { *S = s3 * x * z; g[0] = s3 * z; g[2] = s3 * x; }
    else if (m == -1) { *S = s3 * y * z; g[1] = s3 * z; g[2] = s3 * y; }
    else if (m == 2) { *S = 0.5 * s3 * (x2 - y2); g[0] = s3 * x; g[1] = -s3 * y; }
    else { *S = s3 * x * y; g[0] = s3 * y; g[1] = s3 * x; }
    return;
  }
  case 3: {
    const double c1 = sqrt(3.0 / 8.0), c2 = 0.5 * sqrt(15.0), c3 = sqrt(5.0 / 8.0);
    if (m == 0) { *S = z * z2 - 1.5 * z * rho2; g[0] = -3 * x * z; g[1] = -3 * y * z; g[2] = 3 * z2 - 1.5 * rho2; }
    else if (m == 1) { *S = c1 * x * (4 * z2 - rho2); g[0] = c1 * (4 * z2 - 3 * x2 - y2); g[1] = -2 * c1 * x * y; g[2] = 8 * c1 * x * z; }
    else if (m == -1) { *S = c1 * y * (4 * z2 - rho2); g[0] = -2 * c1 * x * y; g[1] = c1 * (4 * z2 - x2 - 3 * y2); g[2] = 8 * c1 * y * z; }
    else if (m == 2) { *S = c2 * z * (x2 - y2); g[0] = 2 * c2 * x * z; g[1] = -2 * c2 * y * z; g[2] = c2 * (x2 - y2); }
    else if (m == -2) { *S = 2 * c2 * x * y * z; g[0] = 2 * c2 * y * z; g[1] = 2 * c2 * x * z; g[2] = 2 * c2 * x * y; }
    else if (m == 3) { *S = c3 * (x * x2 - 3 * x * y2); g[0] = 3 * c3 * (x2 - y2); g[1] = -6 * c3 * x * y; }
    else { *S = c3 * (3 * x2 * y - y * y2); g[0] = 6 * c3 * x * y; g[1] = 3 * c3 * (x2 - y2); }
    return;
  }
  default: {
    const double c1 = 0.25 * sqrt(10.0), c2 = 0.25 * sqrt(5.0), c3 = 0.25 * sqrt(70.0), c4 = sqrt(35.0) / 8.0;
    if (m == 0) {
      *S = z2 * z2 - 3 * rho2 * z2 + 0.375 * rho2 * rho2;
      g[0] = -6 * x * z2 + 1.5 * rho2 * x; g[1] = -6 * y * z2 + 1.5 * rho2 * y; g[2] = 4 * z * z2 - 6 * rho2 * z;
    } else if (m == 1) {
      *S = c1 * x * z * (4 * z2 - 3 * rho2);
      g[0] = c1 * (4 * z * z2 - 9 * x2 * z - 3 * y2 * z); g[1] = -6 * c1 * x * y * z; g[2] = c1 * (12 * x * z2 - 3 * x * x2 - 3 * x * y2);
    } else if (m == -1) {
      *S = c1 * y * z * (4 * z2 - 3 * rho2);
      g[0] = -6 * c1 * x * y * z; g[1] = c1 * (4 * z * z2 - 3 * x2 * z - 9 * y2 * z); g[2] = c1 * (12 * y * z2 - 3 * x2 * y - 3 * y * y2);
    } else if (m == 2) {
      double P = 6 * z2 - rho2, Q = x2 - y2;
      *S = c2 * P * Q; g[0] = 2 * c2 * x * (P - Q); g[1] = -2 * c2 * y * (P + Q); g[2] = 12 * c2 * z * Q;
    } else if (m == -2) {
      double P = 6 * z2 - rho2;
      *S = 2 * c2 * P * x * y; g[0] = 2 * c2 * y * (P - 2 * x2); g[1] = 2 * c2 * x * (P - 2 * y2); g[2] = 24 * c2 * x * y * z;
    } else if (m == 3) {
      *S = c3 * z * (x * x2 - 3 * x * y2); g[0] = 3 * c3 * z * (x2 - y2); g[1] = -6 * c3 * x * y * z; g[2] = c3 * (x * x2 - 3 * x * y2);
    } else if (m == -3) {
      *S = c3 * z * (3 * x2 * y - y * y2); g[0] = 6 * c3 * x * y * z; g[1] = 3 * c3 * z * (x2 - y2); g[2] = c3 * (3 * x2 * y - y * y2);
    } else if (m == 4) {
      *S = c4 * (x2 * x2 - 6 * x2 * y2 + y2 * y2); g[0] = c4 * (4 * x * x2 - 12 * x * y2); g[1] = c4 * (4 * y * y2 - 12 * x2 * y);
    } else {
      *S = 4 * c4 * (x * x2 * y - x * y * y2); g[0] = c4 * (12 * x2 * y - 4 * y * y2); g[1] = c4 * (4 * x * x2 - 12 * x * y2);
    }
    return;
  }
  }
}

/* Radial function and its first two derivatives for one shell (wfv(1..3) of
   basis_fns.f90:118-157, summed over the contraction). */
static void radial(const orc_sys *s, int ish, double r, double *R) {
  if (s->sh_kind[ish] == 2) {
    table_fit(s, s->rad_of_shell[ish], r, R);
    double w = s->pc[s->sh_p0[ish]];
    R[0] *= w; R[1] *= w; R[2] *= w;
    return;
  }
  int n = s->sh_n[ish];
  double rn = n;
  R[0] = R[1] = R[2] = 0;
  double rm3 = pow(r, rn - 3), rm2 = rm3 * r, rm1 = rm2 * r;
  for (int p = s->sh_p0[ish]; p < s->sh_p0[ish + 1]; p++) {
    double z = s->pz[p], w = s->pc[p];
    if (s->sh_kind[ish] == 0) {
      double zr = z * r, ex = exp(-zr);
      R[0] += w * rm1 * ex;
      R[1] += w * rm2 * ((rn - 1) - zr) * ex;
      R[2] += w * rm3 * ((rn - 1) * (rn - 2 - zr) - (rn - 1 - zr) * zr) * ex;
    } else {
      double zr = 2 * z * r * r, ex = exp(-0.5 * zr);
      R[0] += w * rm1 * ex;
      R[1] += w * rm2 * ((rn - 1) - zr) * ex;
      R[2] += w * rm3 * ((rn - 1) * (rn - 2) - (2 * rn - 1 - zr) * zr) * ex;
    }
  }
}

void orc_basis(const orc_sys *s, const double *pt, double *phi) {
  int ish_prev = -1;
  double R[3] = {0, 0, 0}, d[3] = {0, 0, 0}, r = 0;
  for (int ib = 0; ib < s->nbasis; ib++) {
    int ish = s->b_shell[ib];
    if (ish != ish_prev) {
      int c = s->sh_cent[ish];
      for (int k = 0; k < 3; k++) d[k] = pt[k] - s->cent[3 * c + k];
      r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      if (r == 0) { r = 1e-99; d[0] = 1e-99; } /* basis_fns.f90:95-99 */
      radial(s, ish, r, R);
      ish_prev = ish;
    }
    int l = s->sh_l[ish];
    double S, g[3];
    solid_harm(l, s->b_m[ib], d[0], d[1], d[2], &S, g);
    double ri = 1 / r, ril = pow(ri, l);
    double Y = S * ril;
    double *o = phi + 5 * ib;
    o[0] = Y * R[0];
    for (int k = 0; k < 3; k++) {
      double dY = g[k] * ril - l * S * ril * ri * ri * d[k];
      o[1 + k] = Y * d[k] * ri * R[1] + dY * R[0];
    }
    o[4] = Y * (R[2] + 2 * ri * R[1] - l * (l + 1) * ri * ri * R[0]);
  }
}

/* Orbital contraction (qmc/vmc/orbitals_loc_ana.f90:50-64). */
void orc_orbitals(const orc_sys *s, const double *pt, double *orb) {
  double *phi = (double *)malloc(sizeof(double) * 5 * s->nbasis);
  orc_basis(s, pt, phi);
  for (int io = 0; io < s->norb; io++) {
    double a[5] = {0, 0, 0, 0, 0};
    const double *cf = s->coef + (size_t)io * s->nbasis;
    for (int ib = 0; ib < s->nbasis; ib++)
      for (int k = 0; k < 5; k++) a[k] += cf[ib] * phi[5 * ib + k];
    for (int k = 0; k < 5; k++) orb[5 * io + k] = a[k];
  }
  free(phi);
}

/* orbital values only, for occupied orbitals of one spin (orbitals_loc_anae) */
static void orbitals_val(const orc_sys *s, const double *pt, int sp, double *val, double *phi) {
  orc_basis(s, pt, phi);
  for (int j = 0; j < s->nocc[sp]; j++) {
    const double *cf = s->coef + (size_t)s->occ[sp][j] * s->nbasis;
    double a = 0;
    for (int ib = 0; ib < s->nbasis; ib++) a += cf[ib] * phi[5 * ib];
    val[j] = a;
  }
}

/* ------------------------------------------------------------------------------------ */
/* Jastrow ijas=4, isc=4 (qmc/vmc/jastrow4.f90, scale_dist.f90:585-884)                  */
/* ------------------------------------------------------------------------------------ */
/* scale_dist2 for isc=4 (scale_dist.f90:644-648) */
static void scale_dist2(double scalek, double r, double *rr, double *dd1, double *dd2) {
  double deni = 1 / (1 + scalek * r);
  *rr = r * deni;
  *dd1 = deni * deni;
  *dd2 = -2 * scalek * deni * (*dd1);
}
/* switch_scale2 for isc=4, c1_jas6=1 (scale_dist.f90:857-884) */
static void switch_scale2(double scalek, double *rr, double *dd1, double *dd2) {
  *rr = 1 - scalek * (*rr);
  *dd1 = -scalek * (*dd1);
  *dd2 = -scalek * (*dd2);
}

/* spin class of a pair: isb (b set), sspinn, ipar (jastrow4.f90:76-89) */
static void pair_spin(const orc_sys *s, int i, int j, int *isb, double *sspinn, int *ipar) {
  /* i > j */
  *isb = 0; *sspinn = 1; *ipar = 0;
  if (i < s->nup || j >= s->nup) {
    if (s->nspin2b == 2) *isb = 1;
    else *sspinn = 0.5;
    *ipar = 1;
  }
}

/* e-e pair: f, df/dr (already divided by r), and 2*(f'' + 2 f'/r) contribution to d2ijo */
static void jas_ee(const orc_sys *s, int i, int j, double rij, double *fee_o, double *feeu_o, double *feeuu_o) {
  int isb, ipar;
  double sspinn;
  pair_spin(s, i, j, &isb, &sspinn, &ipar);
  double u, dd1, dd2;
  scale_dist2(s->scalek, rij, &u, &dd1, &dd2);
  double top = sspinn * s->b[isb][0] * u, topu = sspinn * s->b[isb][0];
  double bot = 1 + s->b[isb][1] * u, botu = s->b[isb][1];
  double bot2 = bot * bot;
  double fee = top / bot, feeu = topu / bot2, feeuu = -2 * feeu * botu / bot;
  fee -= s->asymp_jasb[ipar];
  double uu[MAXORD + 2];
  uu[0] = 1; uu[1] = u;
  for (int iord = 2; iord <= s->nordb; iord++) {
    uu[iord] = u * uu[iord - 1];
    double bb = s->b[isb][iord];
    fee += bb * uu[iord];
    feeu += bb * iord * uu[iord - 1];
    feeuu += bb * iord * (iord - 1) * uu[iord - 2];
  }
  feeuu = feeuu * dd1 * dd1 + feeu * dd2;
  feeu = feeu * dd1 / rij;
  *fee_o = fee; *feeu_o = feeu; *feeuu_o = feeuu;
}

/* e-e-n term for pair (i,j) and one centre type with full derivatives
   (jastrow4.f90:159-336). Outputs the value fc and the chain-ruled derivatives. */
typedef struct { double fc, fu, fuu, fi, fii, fj, fjj, fui, fuj; } een_t;

static void jas_een(const orc_sys *s, int it, double rij, double ri, double rj, een_t *o) {
  int nordc = s->nordc;
  double u1, dd1, dd2, ri1, dd7, dd9, rj1, dd8, dd10;
  scale_dist2(s->scalek, rij, &u1, &dd1, &dd2);
  switch_scale2(s->scalek, &u1, &dd1, &dd2);
  scale_dist2(s->scalek, ri, &ri1, &dd7, &dd9);
  switch_scale2(s->scalek, &ri1, &dd7, &dd9);
  scale_dist2(s->scalek, rj, &rj1, &dd8, &dd10);
  switch_scale2(s->scalek, &rj1, &dd8, &dd10);
  /* power tables with two zero entries below index 0 (jastrow4.f90:45-56) */
  double uub[MAXORD + 3], rrib[MAXORD + 3], rrjb[MAXORD + 3], ssb[MAXORD + 3], ttb[MAXORD + 3];
  double *uu = uub + 2, *rri = rrib + 2, *rrj = rrjb + 2, *ss = ssb + 2, *tt = ttb + 2;
  for (int i = -2; i <= -1; i++) uu[i] = rri[i] = rrj[i] = ss[i] = tt[i] = 0;
  uu[0] = 1; ss[0] = 2; tt[0] = 1; rri[0] = 1; rrj[0] = 1;
  uu[1] = u1;
  for (int iord = 2; iord <= nordc; iord++) uu[iord] = u1 * uu[iord - 1];
  rri[1] = ri1; rrj[1] = rj1;
  for (int iord = 1; iord <= nordc; iord++) {
    rri[iord] = ri1 * rri[iord - 1];
    rrj[iord] = rj1 * rrj[iord - 1];
    ss[iord] = rri[iord] + rrj[iord];
    tt[iord] = rri[iord] * rrj[iord];
  }
  double fc = 0, fu = 0, fuu = 0, fi = 0, fii = 0, fj = 0, fjj = 0, fui = 0, fuj = 0;
  const double *c = s->c + (size_t)it * s->nterms;
  for (int ll = 0; ll < s->nterms; ll++) {
    int k = s->tk[ll], l = s->tl[ll], m = s->tm[ll];
    double cc = c[ll];
    double pi_ = (l + m) * rri[l + m - 1] * rrj[m] + m * rri[m - 1] * rrj[l + m];
    double pj_ = (l + m) * rrj[l + m - 1] * rri[m] + m * rrj[m - 1] * rri[l + m];
    fc += cc * uu[k] * ss[l] * tt[m];
    fu += cc * k * uu[k - 1] * ss[l] * tt[m];
    fuu += cc * k * (k - 1) * uu[k - 2] * ss[l] * tt[m];
    fi += cc * uu[k] * pi_;
    fii += cc * uu[k] * ((l + m) * (l + m - 1) * rri[l + m - 2] * rrj[m] + m * (m - 1) * rri[m - 2] * rrj[l + m]);
    fj += cc * uu[k] * pj_;
    fjj += cc * uu[k] * ((l + m) * (l + m - 1) * rrj[l + m - 2] * rri[m] + m * (m - 1) * rrj[m - 2] * rri[l + m]);
    fui += cc * k * uu[k - 1] * pi_;
    fuj += cc * k * uu[k - 1] * pj_;
  }
  fuu = fuu * dd1 * dd1 + fu * dd2;
  fu = fu * dd1 / rij;
  fui = fui * dd1 * dd7;
  fuj = fuj * dd1 * dd8;
  fii = fii * dd7 * dd7 + fi * dd9;
  fjj = fjj * dd8 * dd8 + fj * dd10;
  fi = fi * dd7 / ri;
  fj = fj * dd8 / rj;
  o->fc = fc; o->fu = fu; o->fuu = fuu; o->fi = fi; o->fii = fii;
  o->fj = fj; o->fjj = fjj; o->fui = fui; o->fuj = fuj;
}

/* e-n term (jastrow4.f90:354-455) */
static void jas_en(const orc_sys *s, int it, double ri, double *fen_o, double *feni_o, double *fenii_o) {
  double rr, dd7, dd9;
  scale_dist2(s->scalek, ri, &rr, &dd7, &dd9);
  double top = s->a4[it][0] * rr, topi = s->a4[it][0];
  double bot = 1 + s->a4[it][1] * rr, boti = s->a4[it][1];
  double bot2 = bot * bot;
  double fen = top / bot, feni = topi / bot2, fenii = -2 * feni * boti / bot;
  fen -= s->asymp_jasa[it];
  for (int iord = 2; iord <= s->norda; iord++) {
    double aa = s->a4[it][iord];
    fen += aa * pow(rr, iord);
    feni += aa * iord * pow(rr, iord - 1);
    fenii += aa * iord * (iord - 1) * pow(rr, iord - 2);
  }
  fenii = fenii * dd7 * dd7 + feni * dd9;
  feni = feni * dd7 / ri;
  *fen_o = fen; *feni_o = feni; *fenii_o = fenii;
}

/* Jastrow tables of one walker (jaso_mod: fso, fijo, d2ijo, fjo). */
typedef struct {
  double *fso;   /* [N][N] pair values (i != j symmetric), fso[i][i] e-n */
  double *fijo;  /* [N][N][3] grad wrt i of term (i,j) */
  double *fjo;   /* [N][3] */
  double fsumo;
} jtab_t;

/* jastrow4 (qmc/vmc/jastrow4.f90:1-492): full J, grad, laplacian for one walker. */
static double jastrow_full(const orc_sys *s, const double *x, double *v, double *d2o, double *div_vj, jtab_t *tab) {
  int N = s->N, C = s->C;
  double fsum = 0, d2 = 0;
  for (int i = 0; i < 3 * N; i++) v[i] = 0;
  if (div_vj) for (int i = 0; i < N; i++) div_vj[i] = 0;
  for (int i = 1; i < N; i++)
    for (int j = 0; j < i; j++) {
      double rv[3], rij = 0;
      for (int k = 0; k < 3; k++) { rv[k] = x[3 * i + k] - x[3 * j + k]; rij += rv[k] * rv[k]; }
      rij = sqrt(rij);
      double fee, feeu, feeuu;
      jas_ee(s, i, j, rij, &fee, &feeu, &feeuu);
      double fs = fee, fij[3], fji[3];
      for (int k = 0; k < 3; k++) { fij[k] = feeu * rv[k]; fji[k] = -feeu * rv[k]; }
      double d2ij = 2. * (feeuu + 2 * feeu);
      if (s->nordc > 1) {
        for (int ic = 0; ic < C; ic++) {
          int it = s->ctype[ic];
          double rvi[3], rvj[3], ri = 0, rj = 0;
          for (int k = 0; k < 3; k++) {
            rvi[k] = x[3 * i + k] - s->cent[3 * ic + k]; ri += rvi[k] * rvi[k];
            rvj[k] = x[3 * j + k] - s->cent[3 * ic + k]; rj += rvj[k] * rvj[k];
          }
          ri = sqrt(ri); rj = sqrt(rj);
          een_t e;
          jas_een(s, it, rij, ri, rj, &e);
          double ssum = ri + rj, t = ri - rj;
          double u2pst = rij * rij + ssum * t, u2mst = rij * rij - ssum * t;
          fs += e.fc;
          for (int k = 0; k < 3; k++) {
            fij[k] += e.fi * rvi[k] + e.fu * rv[k];
            fji[k] += e.fj * rvj[k] - e.fu * rv[k];
          }
          d2ij += 2 * (2 * e.fu + e.fi + e.fj) + 2 * e.fuu + e.fii + e.fjj + e.fui * u2pst / (ri * rij) +
                  e.fuj * u2mst / (rj * rij);
        }
      }
      fsum += fs;
      for (int k = 0; k < 3; k++) { v[3 * i + k] += fij[k]; v[3 * j + k] += fji[k]; }
      if (div_vj) { div_vj[i] += d2ij / 2; div_vj[j] += d2ij / 2; }
      d2 += d2ij;
      if (tab) {
        tab->fso[i * N + j] = tab->fso[j * N + i] = fs;
        for (int k = 0; k < 3; k++) { tab->fijo[(i * N + j) * 3 + k] = fij[k]; tab->fijo[(j * N + i) * 3 + k] = fji[k]; }
      }
    }
  for (int i = 0; i < N; i++) {
    double fs = 0, fg[3] = {0, 0, 0}, d2ii = 0;
    for (int ic = 0; ic < C; ic++) {
      int it = s->ctype[ic];
      double rv[3], ri = 0;
      for (int k = 0; k < 3; k++) { rv[k] = x[3 * i + k] - s->cent[3 * ic + k]; ri += rv[k] * rv[k]; }
      ri = sqrt(ri);
      double fen, feni, fenii;
      jas_en(s, it, ri, &fen, &feni, &fenii);
      fs += fen;
      for (int k = 0; k < 3; k++) fg[k] += feni * rv[k];
      d2ii += fenii + 2 * feni;
    }
    fsum += fs;
    for (int k = 0; k < 3; k++) v[3 * i + k] += fg[k];
    if (div_vj) div_vj[i] += d2ii;
    d2 += d2ii;
    if (tab) {
      tab->fso[i * N + i] = fs;
      for (int k = 0; k < 3; k++) tab->fijo[(i * N + i) * 3 + k] = fg[k];
    }
  }
  if (tab) {
    tab->fsumo = fsum;
    memcpy(tab->fjo, v, sizeof(double) * 3 * N);
  }
  *d2o = d2;
  return fsum;
}

double orc_jastrow(const orc_sys *s, const double *x, double *v, double *d2) {
  return jastrow_full(s, x, v, d2, NULL, NULL);
}

/* value and grad of the pair term (i,j) with electron i at xi, electron j at xj (the
   quantities jastrow4e.f90:66-232 accumulates into fsn/fijn). gi = grad wrt i, gj = grad wrt j. */
static double jas_pair_grad(const orc_sys *s, int i, int j, const double *xi, const double *xj, double *gi, double *gj) {
  int a = i > j ? i : j, bb = i > j ? j : i; /* spin class uses the ordered pair */
  double rv[3], rij = 0;
  for (int k = 0; k < 3; k++) { rv[k] = xi[k] - xj[k]; rij += rv[k] * rv[k]; }
  rij = sqrt(rij);
  double fee, feeu, feeuu;
  jas_ee(s, a, bb, rij, &fee, &feeu, &feeuu);
  double fs = fee;
  for (int k = 0; k < 3; k++) { gi[k] = feeu * rv[k]; gj[k] = -feeu * rv[k]; }
  if (s->nordc > 1)
    for (int ic = 0; ic < s->C; ic++) {
      int it = s->ctype[ic];
      double rvi[3], rvj[3], ri = 0, rj = 0;
      for (int k = 0; k < 3; k++) {
        rvi[k] = xi[k] - s->cent[3 * ic + k]; ri += rvi[k] * rvi[k];
        rvj[k] = xj[k] - s->cent[3 * ic + k]; rj += rvj[k] * rvj[k];
      }
      ri = sqrt(ri); rj = sqrt(rj);
      een_t e;
      jas_een(s, it, rij, ri, rj, &e);
      fs += e.fc;
      for (int k = 0; k < 3; k++) { gi[k] += e.fi * rvi[k] + e.fu * rv[k]; gj[k] += e.fj * rvj[k] - e.fu * rv[k]; }
    }
  return fs;
}

static double jas_en_grad(const orc_sys *s, const double *xi, double *g) {
  double fs = 0;
  g[0] = g[1] = g[2] = 0;
  for (int ic = 0; ic < s->C; ic++) {
    int it = s->ctype[ic];
    double rv[3], ri = 0;
    for (int k = 0; k < 3; k++) { rv[k] = xi[k] - s->cent[3 * ic + k]; ri += rv[k] * rv[k]; }
    ri = sqrt(ri);
    double fen, feni, fenii;
    jas_en(s, it, ri, &fen, &feni, &fenii);
    fs += fen;
    for (int k = 0; k < 3; k++) g[k] += feni * rv[k];
  }
  return fs;
}

/* jastrow4e (qmc/vmc/jastrow4e.f90:1-322): new J and grad of every electron after electron
   iel moved to xnew, from the old tables.  fsn/fijn receive the new row/column of iel. */
static double jastrow_1e(const orc_sys *s, const double *x, int iel, const double *xnew, const jtab_t *o,
                         double *fjn, double *fsn_row, double *fijn_row /* [N][2][3]: g_iel, g_j */) {
  int N = s->N;
  double fsumn = o->fsumo;
  memcpy(fjn, o->fjo, sizeof(double) * 3 * N);
  for (int jj = 0; jj < N; jj++) {
    if (jj == iel) continue;
    double gi[3], gj[3];
    double fs = jas_pair_grad(s, iel, jj, xnew, x + 3 * jj, gi, gj);
    fsumn += fs - o->fso[iel * N + jj];
    for (int k = 0; k < 3; k++) {
      fjn[3 * iel + k] += gi[k] - o->fijo[(iel * N + jj) * 3 + k];
      fjn[3 * jj + k] += gj[k] - o->fijo[(jj * N + iel) * 3 + k];
    }
    if (fsn_row) fsn_row[jj] = fs;
    if (fijn_row) for (int k = 0; k < 3; k++) { fijn_row[6 * jj + k] = gi[k]; fijn_row[6 * jj + 3 + k] = gj[k]; }
  }
  double g[3];
  double fs = jas_en_grad(s, xnew, g);
  fsumn += fs - o->fso[iel * N + iel];
  for (int k = 0; k < 3; k++) fjn[3 * iel + k] += g[k] - o->fijo[(iel * N + iel) * 3 + k];
  if (fsn_row) fsn_row[iel] = fs;
  if (fijn_row) for (int k = 0; k < 3; k++) { fijn_row[6 * iel + k] = g[k]; fijn_row[6 * iel + 3 + k] = 0; }
  return fsumn;
}

/* Value-only Jastrow change for the nonlocal quadrature (nonlocj, qmc/vmc/nonloc.f90:432-522,
   with psibnl/psinl/psianl of qmc/vmc/nonlpsi.f90). */
static double psibnl(const orc_sys *s, int i, int j, double rij) {
  int isb, ipar;
  double sspinn;
  pair_spin(s, i > j ? i : j, i > j ? j : i, &isb, &sspinn, &ipar);
  double u = rij / (1 + s->scalek * rij);
  double v = sspinn * s->b[isb][0] * u / (1 + s->b[isb][1] * u) - s->asymp_jasb[ipar];
  for (int k = 2; k <= s->nordb; k++) v += s->b[isb][k] * pow(u, k);
  return v;
}
static double psinl(const orc_sys *s, int it, double rij, double ri, double rj) {
  if (s->nordc <= 1) return 0;
  double uuu = 1 - s->scalek * (rij / (1 + s->scalek * rij));
  double rrri = 1 - s->scalek * (ri / (1 + s->scalek * ri));
  double rrrj = 1 - s->scalek * (rj / (1 + s->scalek * rj));
  double uu[MAXORD + 1], ss[MAXORD + 1], tt[MAXORD + 1];
  uu[0] = 1; ss[0] = 2; tt[0] = 1;
  double pi_ = 1, pj_ = 1;
  for (int jp = 1; jp <= s->nordc; jp++) {
    uu[jp] = uu[jp - 1] * uuu;
    pi_ *= rrri; pj_ *= rrrj;
    ss[jp] = pi_ + pj_;
    tt[jp] = pi_ * pj_;
  }
  const double *c = s->c + (size_t)it * s->nterms;
  double v = 0;
  for (int ll = 0; ll < s->nterms; ll++) v += c[ll] * uu[s->tk[ll]] * ss[s->tl[ll]] * tt[s->tm[ll]];
  return v;
}
static double psianl(const orc_sys *s, int it, double ri) {
  double rri = ri / (1 + s->scalek * ri);
  double v = s->a4[it][0] * rri / (1 + s->a4[it][1] * rri) - s->asymp_jasa[it];
  for (int i = 2; i <= s->norda; i++) v += s->a4[it][i] * pow(rri, i);
  return v;
}

/* J(new) - J(old) with electron iel at xn, old pair values from fso. */
static double nonlocj(const orc_sys *s, const double *x, int iel, const double *xn, const double *fso) {
  int N = s->N, C = s->C;
  double fsumn = 0;
  double ren[64];
  for (int ic = 0; ic < C && ic < 64; ic++) {
    double r2 = 0;
    for (int k = 0; k < 3; k++) { double d = xn[k] - s->cent[3 * ic + k]; r2 += d * d; }
    ren[ic] = sqrt(r2);
  }
  for (int jj = 0; jj < N; jj++) {
    if (jj == iel) continue;
    double r2 = 0;
    for (int k = 0; k < 3; k++) { double d = x[3 * jj + k] - xn[k]; r2 += d * d; }
    double rij = sqrt(r2);
    double f = psibnl(s, iel, jj, rij);
    for (int ic = 0; ic < C; ic++) {
      double rj2 = 0;
      for (int k = 0; k < 3; k++) { double d = x[3 * jj + k] - s->cent[3 * ic + k]; rj2 += d * d; }
      int a = iel > jj ? iel : jj;
      double ri = (a == iel) ? ren[ic] : sqrt(rj2), rj = (a == iel) ? sqrt(rj2) : ren[ic];
      f += psinl(s, s->ctype[ic], rij, ri, rj);
    }
    fsumn += f - fso[iel * N + jj];
  }
  double f = 0;
  for (int ic = 0; ic < C; ic++) f += psianl(s, s->ctype[ic], ren[ic]);
  fsumn += f - fso[iel * N + iel];
  return fsumn;
}

/* ------------------------------------------------------------------------------------ */
/* Determinants                                                                          */
/* ------------------------------------------------------------------------------------ */
/* LU with partial pivoting; replaces a (n x n, row-major) by its inverse.  Returns
   ln|det| and the sign; sign 0 means singular (matinv, qmc/vmc/matinv.f90). */
static double lu_inverse(double *a, int n, double *sign) {
  int piv[CHAMP_MAX_SPIN];
  double *lu = (double *)malloc(sizeof(double) * n * n);
  memcpy(lu, a, sizeof(double) * n * n);
  double lnd = 0, sg = 1;
  for (int k = 0; k < n; k++) {
    int p = k;
    double mx = fabs(lu[k * n + k]);
    for (int i = k + 1; i < n; i++)
      if (fabs(lu[i * n + k]) > mx) { mx = fabs(lu[i * n + k]); p = i; }
    piv[k] = p;
    if (mx == 0) { *sign = 0; free(lu); return -INFINITY; }
    if (p != k) {
      sg = -sg;
      for (int j = 0; j < n; j++) { double t = lu[k * n + j]; lu[k * n + j] = lu[p * n + j]; lu[p * n + j] = t; }
    }
    double d = lu[k * n + k];
    if (d < 0) sg = -sg;
    lnd += log(fabs(d));
    for (int i = k + 1; i < n; i++) {
      double f = lu[i * n + k] / d;
      lu[i * n + k] = f;
      for (int j = k + 1; j < n; j++) lu[i * n + j] -= f * lu[k * n + j];
    }
  }
  /* inverse: solve L U X = P I column by column */
  for (int col = 0; col < n; col++) {
    double *xcol = (double *)malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++) xcol[i] = (i == col) ? 1 : 0;
    /* apply row permutation to rhs: permute identity columns */
    for (int k = 0; k < n; k++) { int p = piv[k]; if (p != k) { double t = xcol[k]; xcol[k] = xcol[p]; xcol[p] = t; } }
    for (int i = 0; i < n; i++) { double sum = xcol[i]; for (int j = 0; j < i; j++) sum -= lu[i * n + j] * xcol[j]; xcol[i] = sum; }
    for (int i = n - 1; i >= 0; i--) { double sum = xcol[i]; for (int j = i + 1; j < n; j++) sum -= lu[i * n + j] * xcol[j]; xcol[i] = sum / lu[i * n + i]; }
    for (int i = 0; i < n; i++) a[i * n + col] = xcol[i];
    free(xcol);
  }
  free(lu);
  *sign = sg;
  return lnd;
}

/* Multi-determinant value and the G matrix of one spin pair.
   psi_D = sum_I cdet_I det(Atilde_up[:,L_I^up]) det(Atilde_dn[:,L_I^dn]).
   G[sp][m][e] = d ln psi_D / d Atilde_sp[e][m] (gup/gdn of qmc/deriv_fast_mod.f90:600-633,
   evaluated here by explicit LU of every determinant).  orbv[e][o] = orbital o at electron e. */
static int det_eval(const orc_sys *s, const double *orbv /* [N][norb] */, double *lnd, double *sgn,
                    double *G /* [2][norb][N] */, double *Ainv0 /* [2][n][n] ref inverse or NULL */) {
  int N = s->N, no = s->norb, D = s->ndet;
  int nsp[2] = {s->nup, s->ndn}, off[2] = {0, s->nup};
  double *lnI = (double *)malloc(sizeof(double) * 2 * D), *sI = (double *)malloc(sizeof(double) * 2 * D);
  int nmx = nsp[0] > nsp[1] ? nsp[0] : nsp[1];
  size_t st = (size_t)nmx * nmx;
  double *inv = (double *)malloc(sizeof(double) * (2 * D * st + 1));
  int singular = 0;
  for (int sp = 0; sp < 2; sp++) {
    int n = nsp[sp];
    for (int I = 0; I < D; I++) {
      double *a = inv + ((size_t)sp * D + I) * st;
      for (int e = 0; e < n; e++)
        for (int k = 0; k < n; k++) a[e * n + k] = orbv[(off[sp] + e) * no + s->det_orb[I * N + off[sp] + k]];
      if (n == 0) { lnI[sp * D + I] = 0; sI[sp * D + I] = 1; continue; }
      lnI[sp * D + I] = lu_inverse(a, n, &sI[sp * D + I]);  /* a := inverse, indexed [k][e] */
      if (sI[sp * D + I] == 0) singular = 1;
    }
  }
  if (singular) {
    /* reference convention: det = 0 */
    *lnd = -INFINITY; *sgn = 0;
    if (G) memset(G, 0, sizeof(double) * 2 * no * N);
    free(lnI); free(sI); free(inv);
    return 1;
  }
  /* weights relative to the largest term */
  double mx = -INFINITY;
  for (int I = 0; I < D; I++) {
    double l = lnI[I] + lnI[D + I];
    if (s->cdet[I] != 0 && l > mx) mx = l;
  }
  double chi = 0;
  double *wI = (double *)malloc(sizeof(double) * D);
  for (int I = 0; I < D; I++) {
    wI[I] = s->cdet[I] * sI[I] * sI[D + I] * exp(lnI[I] + lnI[D + I] - mx);
    chi += wI[I];
  }
  *lnd = mx + log(fabs(chi));
  *sgn = chi > 0 ? 1 : (chi < 0 ? -1 : 0);
  if (G) {
    memset(G, 0, sizeof(double) * 2 * no * N);
    for (int sp = 0; sp < 2; sp++) {
      int n = nsp[sp];
      for (int I = 0; I < D; I++) {
        double w = wI[I] / chi;
        if (w == 0) continue;
        const double *a = inv + ((size_t)sp * D + I) * st;
        for (int k = 0; k < n; k++) {
          int m = s->det_orb[I * N + off[sp] + k];
          for (int e = 0; e < n; e++) G[((size_t)sp * no + m) * N + off[sp] + e] += w * a[k * n + e];
        }
      }
    }
  }
  if (Ainv0)
    for (int sp = 0; sp < 2; sp++) {
      int n = nsp[sp];
      memcpy(Ainv0 + (size_t)sp * CHAMP_MAX_SPIN * CHAMP_MAX_SPIN, inv + ((size_t)sp * D) * st, sizeof(double) * n * n);
    }
  free(wI); free(lnI); free(sI); free(inv);
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Pseudopotential (qmc/vmc/readps_gauss.f90:126-165, nonloc_pot.f90, nonloc.f90)         */
/* ------------------------------------------------------------------------------------ */
void orc_vps(const orc_sys *s, int ict, double r, double *vps) {
  r = r > 1e-10 ? r : 1e-10;
  for (int l = 0; l < s->npotd[ict]; l++) {
    double v = 0, rsq = r * r;
    int nt = s->necp_term[ict * MAXLCH + l];
    for (int i = 0; i < nt; i++) {
      size_t o = ((size_t)ict * MAXLCH + l) * s->mgauss + i;
      int pw = s->necp_power[o];
      double p = (pw != 2) ? pow(r, pw - 2) : 1;
      v += p * s->ecp_coef[o] * exp(-s->ecp_exp[o] * rsq);
    }
    if (l + 1 == s->lpotp1[ict]) v -= s->znuc[ict] / r;
    vps[l] = v;
  }
}

/* (2L+1) P_L(x) for L = 0..4 (yl0, qmc/vmc/nonloc.f90:249-274, l = L+1) */
static double yl0(int L, double x) {
  double p0 = 1, p1 = x;
  if (L == 0) return 1;
  for (int n = 1; n < L; n++) { double p2 = ((2 * n + 1) * x * p1 - n * p0) / (n + 1); p0 = p1; p1 = p2; }
  return (2 * L + 1) * p1;
}

/* Local + nonlocal pseudopotential energy for one walker. G from det_eval, fso Jastrow
   pair table at x.  Returns V_local (sum of the local channel) in *vloc. */
static double nonloc_energy(const orc_sys *s, const double *x, const double *G, const double *fso, double *vloc) {
  int N = s->N, C = s->C, no = s->norb;
  double *phi = (double *)malloc(sizeof(double) * 5 * s->nbasis);
  double *ov = (double *)malloc(sizeof(double) * no);
  double vl = 0, vnl = 0;
  for (int i = 0; i < N; i++) {
    int sp = i < s->nup ? 0 : 1;
    for (int ic = 0; ic < C; ic++) {
      int ict = s->ctype[ic];
      double rv[3], r = 0;
      for (int k = 0; k < 3; k++) { rv[k] = x[3 * i + k] - s->cent[3 * ic + k]; r += rv[k] * rv[k]; }
      r = sqrt(r);
      double vps[MAXLCH];
      orc_vps(s, ict, r, vps);
      vl += vps[s->lpotp1[ict] - 1];
      int iskip = 1;
      for (int l = 0; l < s->npotd[ict]; l++)
        if (l + 1 != s->lpotp1[ict] && fabs(vps[l]) > 1e-4) iskip = 0;
      if (iskip) continue;
      double ri = 1 / r;
      for (int iq = 0; iq < s->nquad; iq++) {
        double costh = (rv[0] * s->q[iq][0] + rv[1] * s->q[iq][1] + rv[2] * s->q[iq][2]) * ri;
        double xn[3];
        for (int k = 0; k < 3; k++) xn[k] = r * s->q[iq][k] + s->cent[3 * ic + k];
        /* orbitals at the quadrature point, contracted with G: determinant ratio */
        orbitals_val(s, xn, sp, ov, phi);
        double dr = 0;
        for (int j = 0; j < s->nocc[sp]; j++) dr += G[((size_t)sp * no + s->occ[sp][j]) * N + i] * ov[j];
        double dj = nonlocj(s, x, i, xn, fso);
        double vp = 0;
        for (int l = 0; l < s->npotd[ict]; l++)
          if (l + 1 != s->lpotp1[ict]) vp += vps[l] * yl0(l, costh);
        vnl += s->wq[iq] * exp(dj) * vp * dr;
      }
    }
  }
  free(phi); free(ov);
  *vloc = vl;
  return vnl;
}

/* ------------------------------------------------------------------------------------ */
/* Full evaluation (qmc/vmc/hpsi.f90:2-381)                                              */
/* ------------------------------------------------------------------------------------ */
typedef struct {
  double *orb;   /* [N][norb][5] */
  double *orbv;  /* [N][norb] */
  double *G;     /* [2][norb][N] */
  double *Ainv;  /* [2][MAXS][MAXS] reference-determinant inverse [k][e] */
  jtab_t jt;
  double lnd, sgn, psij;
} wstate_t;

static void wstate_alloc(const orc_sys *s, wstate_t *w) {
  int N = s->N, no = s->norb;
  w->orb = (double *)malloc(sizeof(double) * N * no * 5);
  w->orbv = (double *)malloc(sizeof(double) * N * no);
  w->G = (double *)malloc(sizeof(double) * 2 * no * N);
  w->Ainv = (double *)malloc(sizeof(double) * 2 * CHAMP_MAX_SPIN * CHAMP_MAX_SPIN);
  w->jt.fso = (double *)malloc(sizeof(double) * N * N);
  w->jt.fijo = (double *)malloc(sizeof(double) * N * N * 3);
  w->jt.fjo = (double *)malloc(sizeof(double) * N * 3);
}
static void wstate_free(wstate_t *w) {
  free(w->orb); free(w->orbv); free(w->G); free(w->Ainv);
  free(w->jt.fso); free(w->jt.fijo); free(w->jt.fjo);
}

static int eval_full_ws(const orc_sys *s, const double *x, orc_eval *out, wstate_t *w) {
  int N = s->N, no = s->norb;
  /* e-e and nuclear Coulomb (distances, qmc/vmc/distances.f90:1-170) */
  double pe_ee = 0, pe_en = 0;
  for (int i = 1; i < N; i++)
    for (int j = 0; j < i; j++) {
      double r2 = 0;
      for (int k = 0; k < 3; k++) { double d = x[3 * i + k] - x[3 * j + k]; r2 += d * d; }
      pe_ee += 1 / sqrt(r2);
    }
  if (s->nloc == 0)
    for (int ic = 0; ic < s->C; ic++)
      for (int i = 0; i < N; i++) {
        double r2 = 0;
        for (int k = 0; k < 3; k++) { double d = x[3 * i + k] - s->cent[3 * ic + k]; r2 += d * d; }
        pe_en -= s->znuc[s->ctype[ic]] / sqrt(r2);
      }
  /* Jastrow */
  double vj[3 * CHAMP_MAX_ELEC], div_vj[CHAMP_MAX_ELEC], d2j;
  double psij = jastrow_full(s, x, vj, &d2j, div_vj, &w->jt);
  /* orbitals of every electron (determinant.f90:36-42 -> orbitals_loc_ana) */
  for (int i = 0; i < N; i++) {
    orc_orbitals(s, x + 3 * i, w->orb + (size_t)i * no * 5);
    for (int o = 0; o < no; o++) w->orbv[i * no + o] = w->orb[((size_t)i * no + o) * 5];
  }
  double lnd, sgn;
  int sing = det_eval(s, w->orbv, &lnd, &sgn, w->G, w->Ainv);
  /* ddet_det, div_vd (determinant.f90:96-150) */
  double vd[3 * CHAMP_MAX_ELEC], div_vd[CHAMP_MAX_ELEC], d2lnd = 0;
  for (int i = 0; i < N; i++) {
    int sp = i < s->nup ? 0 : 1;
    double g[3] = {0, 0, 0}, lap = 0;
    for (int j = 0; j < s->nocc[sp]; j++) {
      int m = s->occ[sp][j];
      double gg = w->G[((size_t)sp * no + m) * N + i];
      const double *o = w->orb + ((size_t)i * no + m) * 5;
      for (int k = 0; k < 3; k++) g[k] += gg * o[1 + k];
      lap += gg * o[4];
    }
    for (int k = 0; k < 3; k++) vd[3 * i + k] = g[k];
    div_vd[i] = lap - (g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    d2lnd += div_vd[i];
  }
  double pe = s->pecent + pe_en + pe_ee, vnl = 0, vloc = pe_en;
  if (s->nloc > 0 && !sing) {
    vnl = nonloc_energy(s, x, w->G, w->jt.fso, &vloc);
    pe += vloc + vnl;
  }
  double d2lnpsi = d2lnd + d2j, v2 = 0;
  for (int i = 0; i < 3 * N; i++) { double v = vj[i] + vd[i]; v2 += v * v; }
  double energy = pe - HB * (d2lnpsi + v2);
  w->lnd = lnd; w->sgn = sgn; w->psij = psij;
  if (out) {
    out->lnd = lnd; out->sign = sgn; out->psij = psij; out->lnpsi = lnd + psij;
    out->d2j = d2j; out->d2lnd = d2lnd; out->d2lnpsi = d2lnpsi;
    out->pe = pe; out->pe_ee = pe_ee; out->pe_local = vloc; out->pe_nonloc = vnl; out->pecent = s->pecent;
    out->energy = energy;
    for (int i = 0; i < N; i++)
      for (int k = 0; k < 3; k++) {
        if (out->vel) out->vel[3 * i + k] = vj[3 * i + k] + vd[3 * i + k];
        if (out->vj) out->vj[3 * i + k] = vj[3 * i + k];
        if (out->vd) out->vd[3 * i + k] = vd[3 * i + k];
      }
    if (out->div_v) for (int i = 0; i < N; i++) out->div_v[i] = div_vj[i] + div_vd[i];
  }
  return sing;
}

int orc_eval_full(const orc_sys *s, const double *x, orc_eval *out) {
  wstate_t w;
  wstate_alloc(s, &w);
  int r = eval_full_ws(s, x, out, &w);
  wstate_free(&w);
  return r;
}

/* ------------------------------------------------------------------------------------ */
/* Jastrow parameter derivatives (deriv_jastrow4, qmc/vmc/deriv_jastrow4.f90: gvalue, g, d2g;  */
/* the nonlocal part as deriv_nonloc_pot / deriv_nonloc, qmc/fit/deriv_nonloc_pot.f90)          */
/* ------------------------------------------------------------------------------------ */
/* The free Jastrow parameters in the engine's order: a_k (k = 2..norda) per centre type, b_k
   (k = 1..nordb, i.e. b_2 first) per spin set, then the e-e-n terms not fixed by the cusp
   conditions per centre type.  J is linear in all of them except b_2 (the Pade denominator), so
   the Jastrow of a system whose only non-zero free parameter is p = 1 (its dependent e-e-n terms
   solved from the cusp equations, the asymptotes recomputed) is dJ/dp with all its derivatives.
   Returns 0 for such a parameter (t set up), 1 for b_2 of spin set *isb, -1 past the last. */
static int unit_param_sys(const orc_sys *s, int p, orc_sys *t, double *cbuf, int *isb) {
  *t = *s;
  memset(t->a4, 0, sizeof t->a4);
  memset(t->b, 0, sizeof t->b);
  const int nt = s->nterms;
  t->c = cbuf;
  if (nt > 0) memset(cbuf, 0, sizeof(double) * s->nct * nt);
  const int na = s->nct * (s->norda > 1 ? s->norda - 1 : 0), nb = s->nspin2b * s->nordb;
  if (p < na) {
    t->a4[p / (s->norda - 1)][2 + p % (s->norda - 1)] = 1.0;
    set_asymptotes(t);
    return 0;
  }
  p -= na;
  if (p < nb) {
    const int is = p / s->nordb, k = 1 + p % s->nordb;
    if (k == 1) { *isb = is; return 1; }
    t->b[is][k] = 1.0;
    set_asymptotes(t);
    return 0;
  }
  p -= nb;
  if (s->nordc <= 1 || nt == 0) return -1;
  int dep[2 * MAXORD], ndep = 0, fr[64], nfr = 0;
  if (s->een_cusp) {
    orc_sys u = *s;
    double tmp[64];
    memset(tmp, 0, sizeof tmp);
    u.c = tmp;
    u.nct = 1;
    een_cusp(&u, dep);
    ndep = 2 * (s->nordc - 1);
  }
  for (int ll = 0; ll < nt; ll++) {
    int isdep = 0;
    for (int q = 0; q < ndep; q++) isdep |= dep[q] == ll;
    if (!isdep) fr[nfr++] = ll;
  }
  if (p >= s->nct * nfr) return -1;
  cbuf[(p / nfr) * nt + fr[p % nfr]] = 1.0;
  if (s->een_cusp) een_cusp(t, NULL);
  set_asymptotes(t);
  return 0;
}

/* d/d b_2 of the e-e term of pair (i, j) when it belongs to spin set isb_p: the value, its radial
   derivative divided by r and f'' + 2 f'/r's pieces in jas_ee's form. */
static void jas_ee_db2(const orc_sys *s, int i, int j, double rij, int isb_p, double *g, double *gu, double *guu) {
  int isb, ipar;
  double ss;
  pair_spin(s, i, j, &isb, &ss, &ipar);
  *g = *gu = *guu = 0;
  if (isb != isb_p) return;
  double u, dd1, dd2;
  scale_dist2(s->scalek, rij, &u, &dd1, &dd2);
  const double b1 = s->b[isb][0], b2 = s->b[isb][1], bot = 1 + b2 * u, ar = s->asymp_r, bota = 1 + b2 * ar;
  const double v = -ss * b1 * u * u / (bot * bot) + ss * b1 * ar * ar / (bota * bota);
  const double vu = -2 * ss * b1 * u / (bot * bot * bot);
  const double vuu = -2 * ss * b1 * (1 - 2 * b2 * u) / (bot * bot * bot * bot);
  *g = v;
  *guu = vuu * dd1 * dd1 + vu * dd2;
  *gu = vu * dd1 / rij;
}

/* Per free Jastrow parameter p at configuration x: gval[p] = dJ/dp and (when not NULL)
   gvel[p][N][3] = d grad_i J/dp, d2[p] = d sum_i lap_i J/dp.  Returns the parameter count. */
int orc_jastrow_pderiv(const orc_sys *s, const double *x, double *gval, double *gvel, double *d2) {
  const int N = s->N;
  double *cbuf = (double *)calloc((size_t)(s->nct * (s->nterms > 0 ? s->nterms : 1)), sizeof(double));
  double v[3 * CHAMP_MAX_ELEC];
  int p = 0;
  for (;; p++) {
    orc_sys t;
    int isb = 0;
    const int kind = unit_param_sys(s, p, &t, cbuf, &isb);
    if (kind < 0) break;
    double val = 0, dd = 0;
    if (kind == 0) {
      val = jastrow_full(&t, x, v, &dd, NULL, NULL);
    } else {
      for (int k = 0; k < 3 * N; k++) v[k] = 0;
      for (int i = 1; i < N; i++)
        for (int j = 0; j < i; j++) {
          double rv[3], rij = 0;
          for (int k = 0; k < 3; k++) { rv[k] = x[3 * i + k] - x[3 * j + k]; rij += rv[k] * rv[k]; }
          rij = sqrt(rij);
          double g, gu, guu;
          jas_ee_db2(s, i, j, rij, isb, &g, &gu, &guu);
          val += g;
          for (int k = 0; k < 3; k++) { v[3 * i + k] += gu * rv[k]; v[3 * j + k] -= gu * rv[k]; }
          dd += 2 * (guu + 2 * gu);
        }
    }
    gval[p] = val;
    if (gvel) memcpy(gvel + (size_t)p * 3 * N, v, sizeof(double) * 3 * N);
    if (d2) d2[p] = dd;
  }
  free(cbuf);
  return p;
}

/* d ln psi/dp and d E_L/dp of the free Jastrow parameters at x: the local part
   -1/2 (d2g_p + 2 v . g_p) (hpsi's kinetic energy differentiated), and for a pseudopotential each
   quadrature point's term w e^dJ v_l P_l (D'/D) times dJ(x with the electron at the point)/dp -
   dJ(x)/dp.  Returns the parameter count, or -1 for a singular configuration. */
int orc_jastrow_param_grad(const orc_sys *s, const double *x, double *dlnpsi, double *deloc) {
  const int N = s->N, C = s->C, no = s->norb;
  wstate_t w;
  wstate_alloc(s, &w);
  double vel[3 * CHAMP_MAX_ELEC];
  orc_eval e;
  memset(&e, 0, sizeof e);
  e.vel = vel;
  int sing = eval_full_ws(s, x, &e, &w);
  const int np = orc_jastrow_pderiv(s, x, dlnpsi, NULL, NULL);
  double *gvel = (double *)malloc(sizeof(double) * (size_t)(np > 0 ? np : 1) * 3 * N);
  double *d2 = (double *)malloc(sizeof(double) * (np > 0 ? np : 1));
  double *gq = (double *)malloc(sizeof(double) * (np > 0 ? np : 1));
  orc_jastrow_pderiv(s, x, dlnpsi, gvel, d2);
  for (int p = 0; p < np; p++) {
    double vg = 0;
    for (int k = 0; k < 3 * N; k++) vg += vel[k] * gvel[(size_t)p * 3 * N + k];
    deloc[p] = -HB * (d2[p] + 2 * vg);
  }
  if (s->nloc > 0 && !sing) {
    double *phi = (double *)malloc(sizeof(double) * 5 * s->nbasis);
    double *ov = (double *)malloc(sizeof(double) * no);
    double *xq = (double *)malloc(sizeof(double) * 3 * N);
    for (int i = 0; i < N; i++) {
      int sp = i < s->nup ? 0 : 1;
      for (int ic = 0; ic < C; ic++) {
        int ict = s->ctype[ic];
        double rv[3], r = 0;
        for (int k = 0; k < 3; k++) { rv[k] = x[3 * i + k] - s->cent[3 * ic + k]; r += rv[k] * rv[k]; }
        r = sqrt(r);
        double vps[MAXLCH];
        orc_vps(s, ict, r, vps);
        int iskip = 1;
        for (int l = 0; l < s->npotd[ict]; l++)
          if (l + 1 != s->lpotp1[ict] && fabs(vps[l]) > 1e-4) iskip = 0;
        if (iskip) continue;
        for (int iq = 0; iq < s->nquad; iq++) {
          double costh = (rv[0] * s->q[iq][0] + rv[1] * s->q[iq][1] + rv[2] * s->q[iq][2]) / r;
          double xn[3];
          for (int k = 0; k < 3; k++) xn[k] = r * s->q[iq][k] + s->cent[3 * ic + k];
          orbitals_val(s, xn, sp, ov, phi);
          double dr = 0;
          for (int j = 0; j < s->nocc[sp]; j++) dr += w.G[((size_t)sp * no + s->occ[sp][j]) * N + i] * ov[j];
          double dj = nonlocj(s, x, i, xn, w.jt.fso);
          double vp = 0;
          for (int l = 0; l < s->npotd[ict]; l++)
            if (l + 1 != s->lpotp1[ict]) vp += vps[l] * yl0(l, costh);
          const double tq = s->wq[iq] * exp(dj) * vp * dr;
          memcpy(xq, x, sizeof(double) * 3 * N);
          for (int k = 0; k < 3; k++) xq[3 * i + k] = xn[k];
          orc_jastrow_pderiv(s, xq, gq, NULL, NULL);
          for (int p = 0; p < np; p++) deloc[p] += tq * (gq[p] - dlnpsi[p]);
        }
      }
    }
    free(phi); free(ov); free(xq);
  }
  free(gvel); free(d2); free(gq);
  wstate_free(&w);
  return sing ? -1 : np;
}

/* ------------------------------------------------------------------------------------ */
/* Single-electron move (hpsie, qmc/vmc/hpsie.f90:1-71)                                  */
/* ------------------------------------------------------------------------------------ */
/* Determinant ratio and grad ln D at the new position from G (the multi-determinant
   wave function is linear in the row of Atilde of the moved electron). */
static double det_ratio_grad(const orc_sys *s, const double *G, int iel, const double *xnew, double *gd) {
  int N = s->N, no = s->norb, sp = iel < s->nup ? 0 : 1;
  double *orb = (double *)malloc(sizeof(double) * no * 5);
  orc_orbitals(s, xnew, orb);
  double rho = 0, g[3] = {0, 0, 0};
  for (int j = 0; j < s->nocc[sp]; j++) {
    int m = s->occ[sp][j];
    double gg = G[((size_t)sp * no + m) * N + iel];
    rho += gg * orb[5 * m];
    for (int k = 0; k < 3; k++) g[k] += gg * orb[5 * m + 1 + k];
  }
  free(orb);
  if (gd) for (int k = 0; k < 3; k++) gd[k] = g[k] / rho;
  return rho;
}

double orc_ratio_1e(const orc_sys *s, const double *x, int iel, const double *xnew, double *grad) {
  wstate_t w;
  wstate_alloc(s, &w);
  eval_full_ws(s, x, NULL, &w);
  int N = s->N;
  double *fjn = (double *)malloc(sizeof(double) * 3 * N);
  double fsumn = jastrow_1e(s, x, iel, xnew, &w.jt, fjn, NULL, NULL);
  double gd[3];
  double rho = det_ratio_grad(s, w.G, iel, xnew, gd);
  if (grad) for (int k = 0; k < 3; k++) grad[k] = fjn[3 * iel + k] + gd[k];
  double ratio = rho * exp(fsumn - w.jt.fsumo);
  free(fjn);
  wstate_free(&w);
  return ratio;
}

/* ------------------------------------------------------------------------------------ */
/* VMC driver (metrop_mov1 with a symmetric Gaussian proposal; vmc.f90:250-331)         */
/* ------------------------------------------------------------------------------------ */
/* Single-determinant SM update of the reference inverse after electron iel moved
   (dete_update/detsav, qmc/dete_mod.f90:165-190): Ainv[k][e]. */
static void sm_update(double *Ainv, int n, int e, const double *anew) {
  double v[CHAMP_MAX_SPIN], col[CHAMP_MAX_SPIN];
  for (int j = 0; j < n; j++) {
    double a = 0;
    for (int k = 0; k < n; k++) a += anew[k] * Ainv[k * n + j];
    v[j] = a;
  }
  double rho = v[e];
  for (int k = 0; k < n; k++) col[k] = Ainv[k * n + e];
  for (int k = 0; k < n; k++)
    for (int j = 0; j < n; j++) Ainv[k * n + j] -= col[k] * (v[j] - (j == e ? 1.0 : 0.0)) / rho;
}

int orc_vmc(const orc_sys *s, int nw, double *xall, int nsweep, uint64_t seed, uint64_t sweep0, double step,
            double *esum, double *e2sum, double *accept, double *elast, int nthreads) {
  int N = s->N;
  int single = (s->ndet == 1);
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int iw = 0; iw < nw; iw++) {
    orc_sys sl = *s; /* private copy: the quadrature rotation is per walker */
    double *x = xall + (size_t)iw * 3 * N;
    wstate_t w;
    wstate_alloc(s, &w);
    double *fjn = (double *)malloc(sizeof(double) * 3 * N);
    double *fsn = (double *)malloc(sizeof(double) * N);
    double *fijn = (double *)malloc(sizeof(double) * 6 * N);
    double *phi = (double *)malloc(sizeof(double) * 5 * s->nbasis);
    double anew[CHAMP_MAX_SPIN];
    double es = 0, e2 = 0, acc = 0, el = 0;
    eval_full_ws(&sl, x, NULL, &w);
    for (int isw = 0; isw < nsweep; isw++) {
      uint64_t sweep = sweep0 + (uint64_t)isw;
      for (int e = 0; e < N; e++) {
        double g[3], ua, xn[3];
        move_randoms(seed, (uint32_t)iw, sweep, (uint32_t)e, g, &ua);
        for (int k = 0; k < 3; k++) xn[k] = x[3 * e + k] + step * g[k];
        int sp = e < s->nup ? 0 : 1, eo = sp ? e - s->nup : e, n = sp ? s->ndn : s->nup;
        double fsumn = jastrow_1e(&sl, x, e, xn, &w.jt, fjn, fsn, fijn);
        double rho;
        if (single) {
          /* orbitals of the reference determinant at xn; ratio = a' . Ainv[:, e] */
          orbitals_val(&sl, xn, sp, anew, phi);
          double *Ai = w.Ainv + (size_t)sp * CHAMP_MAX_SPIN * CHAMP_MAX_SPIN;
          /* reorder to the determinant's column order */
          double a2[CHAMP_MAX_SPIN];
          for (int k = 0; k < n; k++) {
            int m = s->det_orb[(sp ? s->nup : 0) + k];
            int jj = 0;
            while (s->occ[sp][jj] != m) jj++;
            a2[k] = anew[jj];
          }
          rho = 0;
          for (int k = 0; k < n; k++) rho += a2[k] * Ai[k * n + eo];
          double p = rho * rho * exp(2 * (fsumn - w.jt.fsumo));
          if (ua < p) {
            sm_update(Ai, n, eo, a2);
            w.lnd += log(fabs(rho));
            if (rho < 0) w.sgn = -w.sgn;
            goto accepted;
          }
          continue;
        } else {
          double xsave[3];
          for (int k = 0; k < 3; k++) { xsave[k] = x[3 * e + k]; x[3 * e + k] = xn[k]; }
          for (int o = 0; o < s->norb; o++) w.orbv[e * s->norb + o] = 0;
          double *ov = (double *)malloc(sizeof(double) * s->norb * 5);
          orc_orbitals(&sl, xn, ov);
          double *oldrow = (double *)malloc(sizeof(double) * s->norb);
          for (int o = 0; o < s->norb; o++) { oldrow[o] = w.orbv[e * s->norb + o]; w.orbv[e * s->norb + o] = ov[5 * o]; }
          double lnd2, sg2;
          det_eval(&sl, w.orbv, &lnd2, &sg2, w.G, NULL);
          rho = sg2 * w.sgn * exp(lnd2 - w.lnd);
          double p = rho * rho * exp(2 * (fsumn - w.jt.fsumo));
          free(ov);
          if (ua < p) {
            w.lnd = lnd2; w.sgn = sg2;
            free(oldrow);
            for (int k = 0; k < 3; k++) x[3 * e + k] = xsave[k];
            goto accepted;
          }
          /* reject: restore */
          for (int k = 0; k < 3; k++) x[3 * e + k] = xsave[k];
          {
            double *orbx = (double *)malloc(sizeof(double) * s->norb * 5);
            orc_orbitals(&sl, x + 3 * e, orbx);
            for (int o = 0; o < s->norb; o++) w.orbv[e * s->norb + o] = orbx[5 * o];
            free(orbx);
            det_eval(&sl, w.orbv, &lnd2, &sg2, w.G, NULL);
          }
          free(oldrow);
          continue;
        }
      accepted:
        /* jassav: new row/column of the Jastrow tables */
        for (int j = 0; j < N; j++) {
          w.jt.fso[e * N + j] = w.jt.fso[j * N + e] = fsn[j];
          for (int k = 0; k < 3; k++) {
            w.jt.fijo[(e * N + j) * 3 + k] = fijn[6 * j + k];
            if (j != e) w.jt.fijo[(j * N + e) * 3 + k] = fijn[6 * j + 3 + k];
          }
        }
        memcpy(w.jt.fjo, fjn, sizeof(double) * 3 * N);
        w.jt.fsumo = fsumn;
        for (int k = 0; k < 3; k++) x[3 * e + k] = xn[k];
        acc += 1;
      }
      /* full E_L once per sweep (metrop_mov1.f90:296), quadrature rotated per sweep */
      double R[9];
      orc_random_rotation(seed, (uint32_t)iw, sweep, R);
      orc_set_rotation(&sl, R);
      orc_eval ev;
      memset(&ev, 0, sizeof ev);
      eval_full_ws(&sl, x, &ev, &w);
      el = ev.energy;
      es += el; e2 += el * el;
    }
    if (esum) esum[iw] = es;
    if (e2sum) e2sum[iw] = e2;
    if (accept) accept[iw] = acc;
    if (elast) elast[iw] = el;
    free(fjn); free(fsn); free(fijn); free(phi);
    wstate_free(&w);
  }
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Accelerated Metropolis VMC (imetro = 6, qmc/vmc/metrop_slat_mov1.f90:82-546; gammai.f90)   */
/* ------------------------------------------------------------------------------------ */
typedef struct { uint64_t seed; uint32_t w, s0, s1, e, ctr; double u[2]; int left; } mrng_t;
static double mrng_next(mrng_t *r) {
  if (r->left == 0) {
    uint32_t o[4];
    orc_philox(r->seed, r->w, r->s0, r->s1, 0x80000000u | (r->e << 15) | (r->ctr < 32767u ? r->ctr : 32767u), o);
    r->ctr++;
    r->u[0] = u53(o[0], o[1]);
    r->u[1] = u53(o[2], o[3]);
    r->left = 2;
  }
  return r->u[2 - r->left--];
}

/* gammai(a, x, xae, iflag) (gammai.f90:1-46): lower incomplete gamma by its series (x < a + 4,
   iflag 1), minus the upper one by its continued fraction (iflag -1), times xae = x^a e^-x */
static double gammai_ref(double a, double x, double xae, int *iflag) {
  if (x < a + 4) {
    *iflag = 1;
    double ap = a, sum = 1 / a, del = sum;
    int iter = (int)(21 + 3 * (x - a));
    for (int n = 1; n <= iter; n++) { ap += 1; del *= x / ap; sum += del; }
    return sum * xae;
  }
  *iflag = -1;
  double a0 = 1, a1 = x, b0 = 0, b1 = 1, fac = 1, g = 0;
  long na = lround(a - x);
  int iter = (int)(20 + na > 7 ? 20 + na : 7);
  for (int n = 1; n <= iter; n++) {
    double an = n, ana = an - a;
    a0 = (a1 + a0 * ana) * fac;
    b0 = (b1 + b0 * ana) * fac;
    double anf = an * fac;
    a1 = x * a0 + anf * a1;
    b1 = x * b0 + anf * b1;
    fac = 1 / a1;
    g = b1 * fac;
  }
  return -g * xae;
}

/* zeta and co of the radial density sqrt(r)|1 + co r| e^(-zeta r) (metrop_slat_mov1.f90:136-152) */
static void slat_zeta(double zcusp, double vr, double r, double *zeta, double *co) {
  const double eps = 1e-10;
  double root = (zcusp + vr) * (zcusp + vr - 4 / r);
  if (root >= 0) {
    root = sqrt(root);
    *zeta = 0.5 * (zcusp - vr - root);
    if (*zeta <= 0) *zeta = 0.5 * (zcusp - vr + root);
    if (*zeta <= 0) *zeta = eps;
  } else {
    *zeta = vr < 0 ? -vr - eps : 1.0;
  }
  *co = (*zeta + vr) / (1 - (*zeta + vr) * r);
}

/* normalisation of that density on [rbot, rtop] over its value bot (metrop_slat_mov1.f90:183-214) */
static double slat_norm(double zeta, double co, double rbot, double rtop, double bot) {
  const double g5b2 = 1.329340388179137, d2b3 = 0.666666666666667;
  double rzero = -1 / co, zrbot = zeta * rbot, zrtop = zeta * rtop;
  double zebot = sqrt(pow(zrbot, 3)) * exp(-zrbot), zetop = sqrt(pow(zrtop, 3)) * exp(-zrtop);
  int ib, it, iz;
  double g52bot = gammai_ref(2.5, zrbot, zrbot * zebot, &ib), g52top = gammai_ref(2.5, zrtop, zrtop * zetop, &it);
  if (rzero < rbot || rzero > rtop) {
    double g52dif = (ib * it == 1) ? g52top - g52bot : g52top - g52bot + g5b2;
    double g32dif = d2b3 * (g52dif + zetop - zebot);
    return fabs(g32dif + co * g52dif / zeta) / (bot * sqrt(pow(zeta, 3)));
  }
  double zrzer = zeta * rzero, zezer = sqrt(pow(zrzer, 3)) * exp(-zrzer);
  double g52zer = gammai_ref(2.5, zrzer, zrzer * zezer, &iz);
  double d1 = (ib * iz == 1) ? g52zer - g52bot : g52zer - g52bot + g5b2;
  double c1 = d2b3 * (d1 + zezer - zebot);
  double d2 = (it * iz == 1) ? g52top - g52zer : g52top - g52zer + g5b2;
  double c2 = d2b3 * (d2 + zetop - zezer);
  return (fabs(c1 + co * d1 / zeta) + fabs(c2 + co * d2 / zeta)) / (bot * sqrt(pow(zeta, 3)));
}

static int nearest_centre(const orc_sys *s, const double *p, double *rv, double *r) {
  int best = 0;
  double bd = 1e300;
  for (int c = 0; c < s->C; c++) {
    double d = 0;
    for (int k = 0; k < 3; k++) d += (p[k] - s->cent[3 * c + k]) * (p[k] - s->cent[3 * c + k]);
    if (d < bd) { bd = d; best = c; }
  }
  for (int k = 0; k < 3; k++) rv[k] = p[k] - s->cent[3 * best + k];
  *r = sqrt(bd);
  return best;
}

/* unit vector along the part of v perpendicular to the unit vector z; returns that part's length */
static double perp_axis(const double *v, const double *z, double vr, double *x) {
  const double eps = 1e-10;
  double vp = 0;
  for (int k = 0; k < 3; k++) { x[k] = v[k] - vr * z[k]; vp += x[k] * x[k]; }
  vp = sqrt(vp);
  if (vp < eps) {
    x[0] = eps * (1 - z[0] * z[0]); x[1] = eps * (-z[0] * z[1]); x[2] = eps * (-z[0] * z[2]);
    vp = eps * sqrt(1 - z[0] * z[0]);
  }
  for (int k = 0; k < 3; k++) x[k] /= vp;
  return vp;
}

static double thetamx(double deltat, double r, double z) { return deltat + (2 - deltat) / (1 + (z * r) * (z * r)); }

/* One accelerated Metropolis move of electron e (metrop_slat_mov1.f90:82-546); returns 1 if
   accepted (x updated). */
static int slat_move(const orc_sys *s, double *x, int e, uint64_t seed, uint32_t iw, uint64_t sweep,
                     double deltar, double deltat, double fbias) {
  mrng_t rng = {seed, iw, (uint32_t)sweep, (uint32_t)(sweep >> 32), (uint32_t)e, 0u, {0, 0}, 0};
  double xo[3] = {x[3 * e], x[3 * e + 1], x[3 * e + 2]}, vold[3];
  orc_ratio_1e(s, x, e, xo, vold);
  double rv[3], r;
  int near = nearest_centre(s, xo, rv, &r);
  double zn = s->znuc[s->ctype[near]], zcusp = s->nloc == 0 ? zn : 0.0;
  double deltri = 1 / deltar, rbot = r * deltri, rtop = r * deltar;
  double z[3], xa[3], ya[3];
  for (int k = 0; k < 3; k++) z[k] = rv[k] / r;
  double vr = (vold[0] * rv[0] + vold[1] * rv[1] + vold[2] * rv[2]) / r;
  double vp = perp_axis(vold, z, vr, xa);
  if (vr < -2 * zn) vr = -2 * zn;
  ya[0] = z[1] * xa[2] - z[2] * xa[1]; ya[1] = z[2] * xa[0] - z[0] * xa[2]; ya[2] = z[0] * xa[1] - z[1] * xa[0];
  vp *= fbias;
  double zeta, co;
  slat_zeta(zcusp, vr, r, &zeta, &co);
  double root = sqrt((1.5 * co - zeta) * (1.5 * co - zeta) + 2 * zeta * co);
  double rmax1 = co != 0 ? (1.5 * co - zeta + root) / (2 * zeta * co) : rtop;
  if (rmax1 < rbot) rmax1 = rbot;
  if (rmax1 > rtop) rmax1 = rtop;
  double fmx = sqrt(rmax1) * fabs(1 + co * rmax1) * exp(-zeta * rmax1);
  if (co < 0) {
    double rmax2 = (1.5 * co - zeta - root) / (2 * zeta * co);
    if (rmax2 < rbot) rmax2 = rbot;
    if (rmax2 > rtop) rmax2 = rtop;
    double f2 = sqrt(rmax2) * fabs(1 + co * rmax2) * exp(-zeta * rmax2);
    if (f2 > fmx) fmx = f2;
  }
  double bot = sqrt(r) * fabs(1 + co * r) * exp(-zeta * r), rtry = r, top = bot;
  for (int it = 0; it < 10000; it++) {
    rtry = ((deltar - deltri) * mrng_next(&rng) + deltri) * r;
    top = sqrt(rtry) * fabs(1 + co * rtry) * exp(-zeta * rtry);
    if (top / fmx > mrng_next(&rng)) break;
  }
  double fxop = top / bot, areao = slat_norm(zeta, co, rbot, rtop, bot);
  double raver = 0.5 * (r + rtry), deltt = thetamx(deltat, raver, zn);
  double costht = 1 - deltt * mrng_next(&rng), zprime = rtry * costht, sintht = sqrt(1 - costht * costht);
  areao *= deltt;
  double term = fmin(vp * raver * sintht, 1.0), fm = 1 + term, phitry = 0, tp = 1;
  for (int it = 0; it < 10000; it++) {
    phitry = 3.141592653589793 * mrng_next(&rng);
    tp = 1 + term * cos(phitry);
    if (tp > mrng_next(&rng) * fm) break;
  }
  fxop *= tp;
  double xprime = rtry * sintht * cos(phitry);
  double yprime = sqrt(fmax(0.0, rtry * rtry - xprime * xprime - zprime * zprime));
  if (mrng_next(&rng) < 0.5) yprime = -yprime;
  double xn[3];
  for (int k = 0; k < 3; k++) xn[k] = xa[k] * xprime + ya[k] * yprime + z[k] * zprime + s->cent[3 * near + k];
  /* the reverse move about the new point's nearest nucleus (metrop_slat_mov1.f90:216-250) */
  double rvn[3], rn;
  int nn = nearest_centre(s, xn, rvn, &rn);
  double rvo[3], ro = 0, dot = 0;
  for (int k = 0; k < 3; k++) { rvo[k] = xo[k] - s->cent[3 * nn + k]; ro += rvo[k] * rvo[k]; dot += rvn[k] * rvo[k]; }
  ro = sqrt(ro);
  dot /= rn * ro;
  double costn = dot, sintn = sqrt(1 - dot * dot), ravern = 0.5 * (rn + ro);
  double zn2 = s->znuc[s->ctype[nn]], delttn = thetamx(deltat, ravern, zn2);
  double p = 0;
  if (!(ro > rn * deltar || dot < 1 - delttn)) {
    double vnew[3];
    double ratio = orc_ratio_1e(s, x, e, xn, vnew);
    double zc2 = s->nloc == 0 ? zn2 : 0.0, rb2 = rn / deltar, rt2 = rn * deltar, zz[3], xb[3];
    for (int k = 0; k < 3; k++) zz[k] = rvn[k] / rn;
    double vnr = (vnew[0] * rvn[0] + vnew[1] * rvn[1] + vnew[2] * rvn[2]) / rn;
    double vnp = perp_axis(vnew, zz, vnr, xb);
    if (vnr < -2 * zn2) vnr = -2 * zn2;
    vnp *= fbias;
    double z2, c2;
    slat_zeta(zc2, vnr, rn, &z2, &c2);
    double bot2 = sqrt(rn) * fabs(1 + c2 * rn) * exp(-z2 * rn);
    double top2 = sqrt(ro) * fabs(1 + c2 * ro) * exp(-z2 * ro);
    double fxnp = top2 / bot2, arean = slat_norm(z2, c2, rb2, rt2, bot2) * delttn;
    double t2 = fmin(vnp * ravern * sintn, 1.0), cosphi = 0, rnorm = 0;
    for (int k = 0; k < 3; k++) {
      double q = rvo[k] / ro - costn * rvn[k] / rn;
      rnorm += q * q;
      cosphi += q * xb[k];
    }
    cosphi /= sqrt(rnorm);
    fxnp *= 1 + t2 * cosphi;
    double rr = rtry / ro;
    p = rr * rr * ratio * ratio * fabs((fxnp * areao) / (fxop * arean));
  }
  if (mrng_next(&rng) < p) {
    for (int k = 0; k < 3; k++) x[3 * e + k] = xn[k];
    return 1;
  }
  return 0;
}

/* VMC with the accelerated Metropolis mover: nsweep sweeps of moves of every electron, E_L after
   each sweep with the quadrature rotated per sweep, as orc_vmc. */
int orc_vmc_accel(const orc_sys *s, int nw, double *xall, int nsweep, uint64_t seed, uint64_t sweep0, double deltar,
                  double deltat, double fbias, double *esum, double *e2sum, double *accept, double *elast,
                  int nthreads) {
  int N = s->N;
  if (deltar < 1) deltar = 2;
  if (deltat < 0 || deltat > 2) deltat = 2;
  fbias = fmin(2.0, fmax(0.0, fbias));
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int iw = 0; iw < nw; iw++) {
    orc_sys sl = *s;
    double *x = xall + (size_t)iw * 3 * N;
    double es = 0, e2 = 0, acc = 0, el = 0;
    for (int isw = 0; isw < nsweep; isw++) {
      uint64_t sweep = sweep0 + (uint64_t)isw;
      for (int e = 0; e < N; e++) acc += slat_move(&sl, x, e, seed, (uint32_t)iw, sweep, deltar, deltat, fbias);
      double R[9];
      orc_random_rotation(seed, (uint32_t)iw, sweep, R);
      orc_set_rotation(&sl, R);
      orc_eval ev;
      memset(&ev, 0, sizeof ev);
      orc_eval_full(&sl, x, &ev);
      el = ev.energy;
      es += el; e2 += el * el;
    }
    if (esum) esum[iw] = es;
    if (e2sum) e2sum[iw] = e2;
    if (accept) accept[iw] = acc;
    if (elast) elast[iw] = el;
  }
  return 0;
}

/* ------------------------------------------------------------------------------------ */
/* T-moves (qmc/dmc/dmc_elec/tmove.f90:1-192; psi_utils_mod.f90:390 do_tmoves)            */
/* ------------------------------------------------------------------------------------ */
static void rotation_draws(mrng_t *r, double *R) {
  double u1 = mrng_next(r), u2 = mrng_next(r), u3 = mrng_next(r);
  const double tp = 6.283185307179586;
  double s1 = sqrt(1.0 - u1), s2 = sqrt(u1);
  double qx = s1 * sin(tp * u2), qy = s1 * cos(tp * u2), qz = s2 * sin(tp * u3), qw = s2 * cos(tp * u3);
  R[0] = 1 - 2 * (qy * qy + qz * qz); R[1] = 2 * (qx * qy - qz * qw); R[2] = 2 * (qx * qz + qy * qw);
  R[3] = 2 * (qx * qy + qz * qw); R[4] = 1 - 2 * (qx * qx + qz * qz); R[5] = 2 * (qy * qz - qx * qw);
  R[6] = 2 * (qx * qz - qy * qw); R[7] = 2 * (qy * qz + qx * qw); R[8] = 1 - 2 * (qx * qx + qy * qy);
}

/* the T-matrix element of one quadrature point: sum over the nonlocal channels of
   w_q (exp(-tau v_l) - 1) P_l(cos) times the wave-function ratio */
static double tmove_element(const orc_sys *s, int ict, const double *vps, double wq, double costh, double tau,
                            double ratio) {
  double g = 0;
  for (int l = 0; l < s->npotd[ict]; l++)
    if (l + 1 != s->lpotp1[ict]) g += wq * (exp(-tau * vps[l]) - 1) * yl0(l, costh) * ratio;
  return g;
}

/* T-moves of every electron of one walker at x (in place), with the draws of the engine's
   per-(walker, step, electron) streams; variant 1 casula1, 2 det_balance1.  Returns the number of
   accepted moves. */
int orc_tmoves(const orc_sys *s, double *x, uint64_t seed, uint32_t iw, uint64_t step, double tau, int variant) {
  int N = s->N, nmv = 0;
  for (int e = 0; e < N; e++) {
    mrng_t rng = {seed, iw, (uint32_t)step, (uint32_t)(step >> 32), 256u + (uint32_t)e, 0u, {0, 0}, 0};
    double R[9];
    rotation_draws(&rng, R);
    double xo[3] = {x[3 * e], x[3 * e + 1], x[3 * e + 2]};
    double S = 1.0, pratio = 0.0;
    int pc = -1, pq = -1;
    for (int c = 0; c < s->C; c++) {
      const double *cc = s->cent + 3 * c;
      double rv[3] = {xo[0] - cc[0], xo[1] - cc[1], xo[2] - cc[2]};
      double r = sqrt(rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
      int ict = s->ctype[c];
      double vps[MAXLCH];
      orc_vps(s, ict, r, vps);
      int skip = 1;
      for (int l = 0; l < s->npotd[ict]; l++)
        if (l + 1 != s->lpotp1[ict] && fabs(vps[l]) > 1e-4) skip = 0;
      if (skip) continue;
      for (int q = 0; q < s->nquad; q++) {
        double qv[3];
        for (int k = 0; k < 3; k++) qv[k] = R[3 * k] * s->q0[q][0] + R[3 * k + 1] * s->q0[q][1] + R[3 * k + 2] * s->q0[q][2];
        double costh = (rv[0] * qv[0] + rv[1] * qv[1] + rv[2] * qv[2]) / r;
        double xq[3] = {cc[0] + r * qv[0], cc[1] + r * qv[1], cc[2] + r * qv[2]};
        double ratio = orc_ratio_1e(s, x, e, xq, NULL);
        double g = tmove_element(s, ict, vps, s->wq[q], costh, tau, ratio);
        if (g > 0) {
          S += g;
          if (mrng_next(&rng) < g / S) { pc = c; pq = q; pratio = ratio; }
        }
      }
    }
    if (pc < 0) continue;
    const double *cc = s->cent + 3 * pc;
    double r = sqrt((xo[0] - cc[0]) * (xo[0] - cc[0]) + (xo[1] - cc[1]) * (xo[1] - cc[1]) + (xo[2] - cc[2]) * (xo[2] - cc[2]));
    double xn[3];
    for (int k = 0; k < 3; k++)
      xn[k] = cc[k] + r * (R[3 * k] * s->q0[pq][0] + R[3 * k + 1] * s->q0[pq][1] + R[3 * k + 2] * s->q0[pq][2]);
    double p = 1.0;
    if (variant == 2) {
      int ict = s->ctype[pc];
      double vps[MAXLCH], R2[9];
      orc_vps(s, ict, r, vps);
      rotation_draws(&rng, R2);
      double xe[3] = {xn[0] - cc[0], xn[1] - cc[1], xn[2] - cc[2]}, Sb = 1.0;
      for (int q = 0; q < s->nquad; q++) {
        double qv[3];
        for (int k = 0; k < 3; k++) qv[k] = R2[3 * k] * s->q0[q][0] + R2[3 * k + 1] * s->q0[q][1] + R2[3 * k + 2] * s->q0[q][2];
        double costh = (xe[0] * qv[0] + xe[1] * qv[1] + xe[2] * qv[2]) / r;
        double xq[3] = {cc[0] + r * qv[0], cc[1] + r * qv[1], cc[2] + r * qv[2]};
        double ratio = orc_ratio_1e(s, x, e, xq, NULL) / pratio;
        double g = tmove_element(s, ict, vps, s->wq[q], costh, tau, ratio);
        if (g > 0) Sb += g;
      }
      p = S / Sb < 1.0 ? S / Sb : 1.0;
    }
    if (mrng_next(&rng) >= p) continue;
    for (int k = 0; k < 3; k++) x[3 * e + k] = xn[k];
    nmv++;
  }
  return nmv;
}
