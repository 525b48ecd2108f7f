// elstage.cuh -- the full evaluation (hpsi) of walkers whose state lives in HBM, as four kernels
// that each run at the occupancy their own part allows:
//   k_el_jas  warp per walker: distances to the centres, Jastrow factor, its gradient and the
//             divergence of its velocity, pair table, Coulomb energies;
//   k_el_orb  warp per (walker, electron): basis functions and orbitals with their gradients and
//             Laplacians, and the Slater-matrix row;
//   k_el_inv  block per (walker, spin): Gauss-Jordan inversion of the Slater matrix in shared
//             memory, log-determinant and sign;
//   k_el_fin  warp per walker: multi-determinant tables, velocities, pseudopotential, E_L, and
//             the FP32 move tables of a mixed-precision state.
// The parts exchange per-walker intermediates through HBM (State::el_vj, el_sc, el_rt).  Each
// part runs the same device code as the single-kernel evaluation (full_eval), so both give the
// same results up to the order of floating-point sums.
#pragma once

// Per-warp dynamic shared memory of the parts (bytes).
__host__ __device__ inline size_t el_jas_bytes(int N) { return 2 * align16(sizeof(double) * 3 * N) + align16(sizeof(double) * N); }
template <class T>
__host__ __device__ inline size_t el_orb_bytes(int nbasis) { return align16(sizeof(T) * nbasis * 5); }
template <class T>
__host__ __device__ inline size_t el_fin_bytes(int N, int nscr) { return align16(sizeof(double) * 3 * N) + align16(sizeof(T) * nscr); }
// Scratch of the pseudopotential part (FP64): the radial table of the tasks' centres, as large as
// keeps a warp's shared memory within 13 KB (16 warps per SM) but at least 256 elements, and
// beyond 32 centres each lane's distances to the centres.
__host__ __device__ inline int el_fin_scratch(int N, int C) {
  const int room = (int)((13 * 1024 - align16(sizeof(double) * 3 * N)) / sizeof(double));
  return (room > 256 ? room : 256) + (C > 32 ? 32 * C : 0);
}

// VO: the tables and the Jastrow sum only (the rebuild of the state the moves start from)
template <class T, int NORD, bool VO = false>
__global__ void __launch_bounds__(128, 4) k_el_jas(Sys<T> s, State<T> st) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int N = s.N, C = s.C;
  char *base = dsm + el_jas_bytes(N) * wib;
  for (int w = blockIdx.x * wpb + wib; w < st.W; w += gridDim.x * wpb) {
    View<T> v{};
    v.xs = (double *)base;
    v.vacc = (double *)(base + align16(sizeof(double) * 3 * N));
    v.divj = (double *)(base + 2 * align16(sizeof(double) * 3 * N));
    v.ren = st.ren + (size_t)w * N * C * 2;
    v.zq = st.zq + (size_t)w * N * ZQ;
    v.fso = st.fso + (size_t)w * N * N;
    T *rt = st.el_rt + (size_t)w * 2 * C * N;
    for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
    __syncwarp();
    double fsum, d2j, pe_ee, pe_en;
    jastrow_tables<T, NORD, true, VO>(s, J, v, rt, lane, fsum, d2j, pe_ee, pe_en);
    double *vj = st.el_vj + (size_t)w * 4 * N;
    for (int i = lane; i < 3 * N; i += 32) vj[i] = v.vacc[i];
    for (int i = lane; i < N; i += 32) vj[3 * N + i] = v.divj[i];
    if (lane == 0) {
      double *sc = st.el_sc + (size_t)w * 8;
      sc[0] = fsum;
      sc[1] = d2j;
      sc[2] = pe_ee;
      sc[3] = pe_en;
    }
    __syncwarp();
  }
}

// Orbital coefficients shared by the block (coop): the block's warps take consecutive (walker,
// electron) items of one spin (the host checks that N and nup are multiples of the warps per
// block) and stream the coefficient rows through shared memory once for all of them
// (block_orbitals, 8-row chunks, two buffers at stage_off); otherwise every warp streams them.
constexpr int EL_ORB_KB = 8, EL_ORB_STG = 2;
template <class T>
__global__ void __launch_bounds__(128, 4) k_el_orb(Sys<T> s, State<T> st, int coop, size_t stage_off) {
  extern __shared__ __align__(16) char dsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int N = s.N, nomax = s.nomax;
  T *phi = (T *)(dsm + el_orb_bytes<T>(s.nbasis) * wib);
  T *stage = (T *)(dsm + stage_off);
  const long long items = (long long)st.W * N;
  for (long long ib = (long long)blockIdx.x * wpb; ib < items; ib += (long long)gridDim.x * wpb) {
    const long long it = ib + wib;
    if (it >= items) {
      if (!coop) break;
      // no item for this warp: take part in the block's coefficient stream
      const int e0 = (int)(ib % N), sp0 = e0 < s.nup ? 0 : 1;
      block_orbitals<T, 5, EL_ORB_KB, EL_ORB_STG>((const T *)nullptr, s.cocc[sp0], s.nbasis, s.nocc[sp0], (T *)nullptr,
                                                 0, lane, stage, false);
      continue;
    }
    const int w = (int)(it / N), e = (int)(it - (long long)w * N);
    const int sp = e < s.nup ? 0 : 1, n = sp ? s.ndn : s.nup, eo = sp ? e - s.nup : e;
    T *oe = st.orb5 + ((size_t)w * N + e) * 5 * nomax;
    warp_basis<T, 5>(s, st.x + ((size_t)w * N + e) * 3, phi, lane);
    if (coop)
      block_orbitals<T, 5, EL_ORB_KB, EL_ORB_STG>(phi, s.cocc[sp], s.nbasis, s.nocc[sp], oe, nomax, lane, stage, true);
    else
      warp_orbitals<T, 5>(phi, s.cocc[sp], s.nbasis, s.nocc[sp], oe, nomax, lane);
    __syncwarp();
    double *A = st.ainv + (size_t)w * st.astride + (sp ? s.nup * s.nup : 0);
    for (int k = lane; k < n; k += 32) A[eo * n + k] = (double)oe[k];
    __syncwarp();
  }
}

// Gauss-Jordan inversion with partial pivoting of one walker's Slater matrix of one spin by a
// block, in shared memory; the same steps, pivot choice and element updates as warp_gj (matinv,
// qmc/vmc/matinv.f90).  Writes the inverse ([orbital][electron]) back, and ln|D| and sign(D)
// (0 for a singular matrix) to sc[4 + 2 sp], sc[5 + 2 sp].
static __global__ void __launch_bounds__(128) k_el_inv(double *ainv, int astride, int nup, int ndn, int W, double *scr) {
  extern __shared__ __align__(16) double A[];
  __shared__ int perm[CHAMP_MAX_SPIN];
  __shared__ int s_piv, s_fail;
  const int w = blockIdx.x >> 1, sp = blockIdx.x & 1;
  if (w >= W) return;
  const int n = sp ? ndn : nup, tid = threadIdx.x, nt = blockDim.x;
  double *out = scr + (size_t)w * 8 + 4 + 2 * sp;
  if (n == 0) {
    if (tid == 0) { out[0] = 0.0; out[1] = 1.0; }
    return;
  }
  double *g = ainv + (size_t)w * astride + (sp ? nup * nup : 0);
  const int nn = n * n;
  for (int i = tid; i < nn; i += nt) A[i] = g[i];
  __syncthreads();
  // this thread's first element of the elimination and its step through the matrix
  const int i0 = tid / n, j0 = tid - i0 * n, di = nt / n, dj = nt - di * n;
  double lnd = 0, sg = 1;
  for (int k = 0; k < n; k++) {
    if (tid < 32) {
      double best = -1.0;
      int bi = k;
      for (int i = k + tid; i < n; i += 32) {
        const double v = fabs(A[i * n + k]);
        if (v > best) { best = v; bi = i; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (tid == 0) {
        s_piv = bi;
        s_fail = !(best > 0.0);
        perm[k] = bi;
      }
    }
    __syncthreads();
    if (s_fail) break;
    const int bi = s_piv;
    if (bi != k) {
      for (int j = tid; j < n; j += nt) {
        const double t = A[k * n + j];
        A[k * n + j] = A[bi * n + j];
        A[bi * n + j] = t;
      }
      sg = -sg;
    }
    __syncthreads();
    const double piv = A[k * n + k];
    lnd += log(fabs(piv));
    if (piv < 0) sg = -sg;
    const double pinv = 1.0 / piv;
    __syncthreads();
    for (int j = tid; j < n; j += nt) A[k * n + j] = (j == k) ? pinv : A[k * n + j] * pinv;
    __syncthreads();
    for (int idx = tid, i = i0, j = j0; idx < nn; idx += nt) {
      if (i != k && j != k) A[idx] -= A[i * n + k] * A[k * n + j];
      i += di;
      j += dj;
      if (j >= n) { j -= n; i++; }
    }
    __syncthreads();
    for (int i = tid; i < n; i += nt)
      if (i != k) A[i * n + k] = -A[i * n + k] * pinv;
    __syncthreads();
  }
  if (s_fail) {
    if (tid == 0) { out[0] = 0.0; out[1] = 0.0; }
    return;
  }
  for (int k = n - 1; k >= 0; k--) {
    const int p = perm[k];
    if (p != k)
      for (int i = tid; i < n; i += nt) {
        const double t = A[i * n + k];
        A[i * n + k] = A[i * n + p];
        A[i * n + p] = t;
      }
    __syncthreads();
  }
  for (int i = tid; i < nn; i += nt) g[i] = A[i];
  if (tid == 0) { out[0] = lnd; out[1] = sg; }
}

// Rotation of the quadrature grid: per walker and sweep (VMC) or one for all walkers.
struct ElRot {
  int random;
  uint64_t seed, sweep;
  double R[9];
};

template <class T, int NORD, bool MD>
// tables_only: the state the single-electron moves start from (log-determinant, sign, Jastrow sum,
// the FP32 move tables) without velocities, pseudopotential and E_L (the status flags then see
// no E_L; the next full evaluation sets them)
__global__ void __launch_bounds__(128, 4) k_el_fin(Sys<T> s, State<T> st, int nscr, int outputs, int stats, ElRot rot,
                                                   int tables_only) {
  __shared__ JasPar<T> J;
  __shared__ EcpPar E;
  extern __shared__ __align__(16) char dsm[];
  load_params(s, J, E);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int N = s.N, C = s.C;
  char *base = dsm + el_fin_bytes<T>(N, nscr) * wib;
  T *scr = (T *)(base + align16(sizeof(double) * 3 * N));
  for (int w = blockIdx.x * wpb + wib; w < st.W; w += gridDim.x * wpb) {
    View<T> v{};
    v.xs = (double *)base;
    v.phi = scr;
    v.vacc = st.el_vj + (size_t)w * 4 * N;
    v.divj = v.vacc + 3 * N;
    v.ainv = st.ainv + (size_t)w * st.astride;
    v.fso = st.fso + (size_t)w * N * N;
    v.ren = st.ren + (size_t)w * N * C * 2;
    v.zq = st.zq + (size_t)w * N * ZQ;
    v.orb5 = st.orb5 + (size_t)w * N * 5 * s.nomax;
    v.gproj = st.gproj ? st.gproj + (size_t)w * N * s.nbasis : nullptr;
    v.nlt = st.nlt ? st.nlt + (size_t)w * N * C * NLT : nullptr;
    v.tv = st.tv + (size_t)w * st.tvstride;
    v.gam = st.gam + (size_t)w * st.gstride;
    v.ymd = st.ymd + (size_t)w * st.tvstride;
    v.wdet = st.wdet + (size_t)w * st.wstride;
    for (int i = lane; i < 3 * N; i += 32) v.xs[i] = st.x[(size_t)w * 3 * N + i];
    __syncwarp();
    const double *sc = st.el_sc + (size_t)w * 8;
    const double fsum = sc[0], d2j = sc[1], pe_ee = sc[2], pe_en = sc[3];
    double lnd = sc[4] + sc[6], sgn = sc[5] * sc[7];
    const bool ok = sc[5] != 0.0 && sc[7] != 0.0;
    if (MD && ok) {
      double lc, sgc;
      md_tables(s, v, lane, lc, sgc);
      lnd += lc;
      sgn *= sgc;
    }
    double d2lnd = 0, v2 = 0;
    if (!tables_only) det_velocities<T, MD, false>(s, st, w, v, lane, outputs != 0, nullptr, d2lnd, v2);
    double vloc = 0, vnl = 0;
    int ntask = 0;
    if (s.nloc > 0 && ok && !tables_only) {
      double R[9];
      if (rot.random) random_rotation(rot.seed, (uint32_t)w, rot.sweep, R);
      else
        for (int i = 0; i < 9; i++) R[i] = rot.R[i];
      nlpp_energy<T, NORD, MD, false, true>(s, J, E, v, R, lane, nullptr, scr, nscr, st.el_rt + (size_t)w * 2 * C * N, vloc,
                                      vnl, ntask);
    }
    EvalRes res;
    finish_eval(s, st, w, v, lane, outputs != 0, ok, lnd, sgn, fsum, d2j, pe_ee, pe_en, d2lnd, v2, vloc, vnl, ntask,
                res);
    if (stats && lane == 0) {
      st.s_esum[w] += res.eloc;
      st.s_e2sum[w] += res.eloc * res.eloc;
      st.s_elast[w] = res.eloc;
    }
    mirror_store(v, st, w, N, C, lane, st.el_rt ? st.el_rt + (size_t)w * 2 * C * N : nullptr);
  }
}
