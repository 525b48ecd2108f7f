// orbfused.cuh -- basis functions and the basis-to-orbital contraction of the full evaluation in
// one tensor-core kernel: the basis rows are formed in shared memory and never reach HBM.
//
// Per spin, rows = electrons of that spin of all walkers, K = basis functions in a padded order
// in which no shell straddles a K-block of 16, N = orbitals of the spin.  Five products share the
// coefficients: one per channel (value, d/dx, d/dy, d/dz, Laplacian), accumulated in five TMEM
// column ranges.  Warps 0-3 evaluate the basis functions of one K-block for 128 electrons (one
// thread per electron, all lanes walk the same shells), split each value into its TF32 parts
// hi + lo (both rounded to nearest) and store both into the channel's A tile; warps 4-7 bring the split coefficients of
// the block with cp.async; one thread issues 5 x 2 x 3 tcgen05.mma (kind::tf32, hi.hi + hi.lo +
// lo.hi) per block and commits to the stage's mbarrier, so the evaluation of the next block
// overlaps the tensor cores.  All waits are bounded.
//
// Accumulation in chunks: the tensor core sums each MMA's products into the FP32 accumulator
// with truncation, so a long chain of MMAs into one accumulator shrinks it systematically
// (about half an ulp per MMA; over the 174 MMAs of a 416-function basis the E_L of a
// 128-electron walker moves by ~1e-6 relative).  The K-blocks are therefore taken in chunks of
// `kchunk`: after each chunk the accumulator is drained and added to the orbital rows in HBM
// with round-to-nearest FP32 adds (the first chunk stores), and the next chunk starts from zero.
#pragma once

namespace orbf {

using namespace orbtc;

constexpr int BKF = 16;   // basis functions per K-block (two MMA k-steps of 8)
constexpr int NTF = 256;  // threads: 0-127 one electron row each, 128-255 coefficient loads

struct FArgs {
  const double *x;          // walker positions [W][N][3]
  const float *bhi, *blo;   // [Np][Kq] split coefficients in the padded order (zero at pads)
  const int *blk_sh;        // [nkb+1] first shell of each K-block
  const int *kpos;          // [nshell] padded position of each shell's first function
  float *orb;               // orbital rows [(w*N + e)*5 + ch][nomax]
  int M;                    // rows: W * n
  int Kq, nkb, Np, ncols;   // padded K, K-blocks, padded N (multiple of 16, 5*Np <= 512), TMEM columns
  int n, N, e0, nomax, nocc;
  int kchunk;               // K-blocks per accumulation chunk (>= 1)
  int *err;
};

// One stage: 5 channels x (hi, lo) A tiles [128][16] and (hi, lo) B tiles [Np][16].
__host__ __device__ inline size_t fstage_bytes(int Np) {
  return 10 * (size_t)BM * BKF * 4 + 2 * (size_t)Np * BKF * 4;
}
__host__ __device__ inline size_t fsmem_bytes(int Np) { return 2 * fstage_bytes(Np) + 128; }

// byte offset of element (row r, k) of a [rows][BKF] tile in the no-swizzle K-major core-matrix
// layout: core matrices of 8 rows x 4 elements (128 B), BKF/4 of them along K per 8-row group
__device__ __forceinline__ uint32_t foff(int r, int k) {
  return (uint32_t)((((r >> 3) * (BKF / 4) + (k >> 2)) << 7) + ((r & 7) << 4) + ((k & 3) << 2));
}

static __global__ void __launch_bounds__(NTF, 1) k_orb_fused(Sys<float> s, FArgs a) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char *base = (unsigned char *)(((uintptr_t)sm + 127) & ~(uintptr_t)127);
  const uint32_t sA = BM * BKF * 4, sB = (uint32_t)a.Np * BKF * 4, stage = 10 * sA + 2 * sB;
  // both stages start at zero: a block's pad positions are never written and must stay finite
  for (uint32_t i = 16 * tid; i < 2 * stage; i += 16 * NTF) *(float4 *)(base + i) = make_float4(0.f, 0.f, 0.f, 0.f);
  if (tid == 0) {
    mbar_init(smem_u32(&mbar[0]), 1);
    mbar_init(smem_u32(&mbar[1]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tslot)), "r"(a.ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tbase = tslot;
  const uint32_t idesc = idesc_tf32(BM, a.Np);
  const int ntile = (a.M + BM - 1) / BM;
  const int cb = a.kchunk > 0 ? a.kchunk : a.nkb;
  const int quad = warp & 3, half = warp >> 2;
  const bool vec = (a.nomax & 3) == 0 && ((uintptr_t)a.orb & 15) == 0;  // rows and groups 16-byte aligned
  uint32_t it = 0;       // K-blocks started so far
  uint32_t ncommit = 0;  // K-blocks whose MMA group was committed (the same on every thread)
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntile && ok; tile += gridDim.x) {
    double pt[3] = {0, 0, 0};
    bool live = false;
    if (tid < BM) {
      const int r = tile * BM + tid;
      if (r < a.M) {
        const int w = r / a.n, eo = r - w * a.n;
        const double *p = a.x + ((size_t)w * a.N + a.e0 + eo) * 3;
        pt[0] = p[0]; pt[1] = p[1]; pt[2] = p[2];
        live = true;
      }
    }
    float *dst = nullptr;  // this thread's epilogue row
    {
      const int r = tile * BM + quad * 32 + lane;
      if (r < a.M) {
        const int w = r / a.n, eo = r - w * a.n;
        dst = a.orb + ((size_t)w * a.N + a.e0 + eo) * 5 * a.nomax;
      }
    }
    for (int kb = 0; kb < a.nkb; kb++, it++) {
      const int sg = it & 1;
      unsigned char *st = base + (size_t)sg * stage;
      // the stage is free once the MMAs committed two blocks ago have completed
      const bool got = it < 2 || mbar_wait(smem_u32(&mbar[sg]), ((it - 2) >> 1) & 1);
      if (tid < BM) {
        if (live) {
          const int k0 = kb * BKF;
          for (int ish = a.blk_sh[kb]; ish < a.blk_sh[kb + 1]; ish++) {
            const int kk = a.kpos[ish] - k0;
            shell_eval_put<float, 5>(s, ish, pt, [&](int sl, int ch, float v) {
              const float h = tf32_hi(v);
              const uint32_t o = foff(tid, kk + sl);
              *(float *)(st + (2 * ch) * sA + o) = h;
              *(float *)(st + (2 * ch + 1) * sA + o) = tf32_lo(v, h);
            });
          }
        }  // rows past the end keep finite stale values; their outputs are not stored
      } else {
        // coefficients of the block: 16-byte piece q lands at byte 16q (core-matrix order)
        const uint32_t ub = smem_u32(st + 10 * sA);
        for (int q = tid - BM; q < a.Np * (BKF / 4); q += NTF - BM) {
          const int cm = q >> 3, row = (cm / (BKF / 4)) * 8 + (q & 7), ck = cm % (BKF / 4);
          const size_t o = (size_t)row * a.Kq + (size_t)kb * BKF + 4 * ck;
          cp_async16(ub + 16 * q, a.bhi + o, 16);
          cp_async16(ub + sB + 16 * q, a.blo + o, 16);
        }
        cp_commit();
        cp_wait_all();
      }
      fence_async_smem();
      if (!__syncthreads_and(got)) { ok = false; break; }
      if (tid == BM) {
        fence_after();
        const uint32_t ua = smem_u32(st), ub = ua + 10 * sA;
#pragma unroll
        for (int ch = 0; ch < 5; ch++)
#pragma unroll
          for (int ks = 0; ks < BKF / 8; ks++) {
            const uint32_t ko = ks * 256;
            const uint64_t dah = sdesc(ua + 2 * ch * sA + ko, 128, (BKF / 4) * 128);
            const uint64_t dal = sdesc(ua + (2 * ch + 1) * sA + ko, 128, (BKF / 4) * 128);
            const uint64_t dbh = sdesc(ub + ko, 128, (BKF / 4) * 128), dbl = sdesc(ub + sB + ko, 128, (BKF / 4) * 128);
            const uint32_t d = tbase + (uint32_t)(ch * a.Np);
            mma_tf32(d, dal, dbh, idesc, (kb % cb > 0 || ks > 0) ? 1u : 0u);
            mma_tf32(d, dah, dbl, idesc, 1u);
            mma_tf32(d, dah, dbh, idesc, 1u);
          }
        mma_commit(smem_u32(&mbar[sg]));
      }
      ncommit = it + 1;
      if ((kb + 1) % cb != 0 && kb + 1 != a.nkb) continue;
      // end of a chunk: drain.  Warp q reads TMEM lanes 32(q mod 4)..+31; warps q and q+4 take
      // alternate groups of 16 columns of the 5 channel ranges (Np is a multiple of 16: a group
      // is in one channel).  Each thread adds into the row elements it stored itself.
      if (!__syncthreads_and(mbar_wait(smem_u32(&mbar[sg]), (it >> 1) & 1))) { ok = false; break; }
      fence_after();
      const bool first = kb < cb;
      for (int c0 = 16 * half; c0 < 5 * a.Np; c0 += 32) {
        float v[16];
        tmem_ld16(tbase + ((uint32_t)(quad * 32) << 16) + (uint32_t)c0, v);
        const int ch = c0 / a.Np, m0 = c0 - ch * a.Np;
        if (dst) {
          float *o = dst + ch * a.nomax + m0;
          if (vec && m0 + 16 <= a.nocc) {  // 16-byte aligned: four float4 per group
            float4 *o4 = (float4 *)o;
            if (first) {
#pragma unroll
              for (int k = 0; k < 4; k++) o4[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
            } else {
              float4 p[4];
#pragma unroll
              for (int k = 0; k < 4; k++) p[k] = o4[k];
#pragma unroll
              for (int k = 0; k < 4; k++)
                o4[k] = make_float4(p[k].x + v[4 * k], p[k].y + v[4 * k + 1], p[k].z + v[4 * k + 2], p[k].w + v[4 * k + 3]);
            }
          } else {
#pragma unroll
            for (int k = 0; k < 16; k++)
              if (m0 + k < a.nocc) o[k] = first ? v[k] : o[k] + v[k];
          }
        }
      }
      fence_before();
      __syncthreads();
    }
    if (!ok) break;
  }
  cp_wait_all();
  if (!ok) {
    if (a.err) atomicExch(a.err, 1);
    // let the committed MMA groups finish (bounded) before the accumulator is freed
    if (tid == 0)
      for (uint32_t u = ncommit > 2 ? ncommit - 2 : 0; u < ncommit; u++) mbar_wait(smem_u32(&mbar[u & 1]), (u >> 1) & 1);
  }
  __syncthreads();
  fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(a.ncols));
}

}  // namespace orbf
