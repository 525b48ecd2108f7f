// orbtc.cuh -- the basis-to-orbital contraction of the full evaluation on the tensor cores.
//
// orbitals_loc_ana (orbitals_loc_ana.f90:50-64) for every electron of every walker is one GEMM
// per spin: rows (walker, electron, channel) x K = basis functions x N = orbitals of that spin,
//   orb[w][e][ch][m] = sum_b phi[w][e][ch][b] coef[b][m],   ch = value, d/dx, d/dy, d/dz, lap.
// k_basis_rows writes phi (FP32, K-major rows padded to Kp) to HBM; k_orb_tc runs the product
// with tcgen05.mma kind::tf32 into a TMEM accumulator.  TF32 keeps 10 mantissa bits, so each
// operand is split as x = hi + lo + r with hi = x rounded to nearest TF32 and lo = (x - hi)
// rounded to nearest TF32 (both exact TF32 values, so the tensor core drops no bits of them),
// and the product is hi*hi + hi*lo + lo*hi: about FP32 accuracy (|r| <= 2^-22 |x|, lo*lo below
// 2^-22, FP32 accumulation), three tensor-core passes.  Rounding to nearest keeps the dropped
// parts of either sign; a truncating split would drop them all towards zero and shrink every
// product by ~1e-6 on average, a bias that accumulates in ln|D| over many rows.  Used by the
// mixed-precision engine only; the FP64 engine keeps the CUDA-core contraction.
#pragma once
#include <cstdint>

namespace orbtc {

constexpr int BM = 128;        // rows per tile (TMEM lanes)
constexpr int BK = 32;         // K (fp32 elements) per stage: 128 bytes per row
constexpr int NTHR = 256;      // 8 warps: all load and split, thread 0 issues, all drain TMEM
constexpr uint32_t WAIT_LIMIT = 1u << 24;  // bounded mbarrier polls before giving up

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major without swizzle: the operand is stored as core
// matrices of 8 rows x 16 bytes (128 contiguous bytes); lbo = bytes between core matrices
// adjacent along K, sbo = bytes between adjacent 8-row groups.  Bit 46 = descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// Instruction descriptor: D f32 (bits 4-5 = 1), A and B tf32 (bits 7-9, 10-12 = 2), both
// K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t dt, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dt),
      "l"(a), "l"(b), "r"(id), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for completion `parity` of the barrier; false after WAIT_LIMIT polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (uint32_t i = 0; i < WAIT_LIMIT; i++)
    if (mbar_try(mbar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// x rounded to the nearest TF32 value (ties away from zero), returned as an FP32 bit pattern
// with the low 13 mantissa bits zero
__host__ __device__ inline float tf32_rn(float x) {
#ifdef __CUDA_ARCH__
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
#else
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7F800000u) != 0x7F800000u) u += 0x1000u;  // half an ulp of TF32, carry into the exponent
  u &= 0xFFFFE000u;
  float h;
  memcpy(&h, &u, 4);
  return h;
#endif
}
// the two TF32 parts of x: hi = rn(x), lo = rn(x - hi)
__host__ __device__ inline float tf32_hi(float x) { return tf32_rn(x); }
__host__ __device__ inline float tf32_lo(float x, float hi) { return tf32_rn(x - hi); }

struct Args {
  const float *phi;          // [rows of all walkers][Kp]; row = (w*N + e)*5 + ch
  const float *bhi, *blo;    // [Np][Kp] coefficients of this spin, transposed, split, zero padded
  float *orb;                // [rows][nomax]
  int M;                     // rows of this spin: W * n * 5
  int Kp, Np, ncols;         // padded K (multiple of BK), padded N (multiple of 16), TMEM columns
  int n, N, e0, nomax, nocc; // electrons of the spin, all electrons, first electron, row stride, orbitals
  int kchunk;                // K-blocks per TMEM accumulation chunk (>= 1), drained into orb
  int *err;
};

// Bytes of one pipeline stage: A hi, A lo (BM x BK), B hi, B lo (Np x BK), core-matrix layout.
__host__ __device__ inline size_t stage_bytes(int Np) { return 2 * (size_t)BM * BK * 4 + 2 * (size_t)Np * BK * 4; }
__host__ __device__ inline size_t smem_bytes(int Np, int ns) { return ns * stage_bytes(Np) + 128; }
// Deepest pipeline (2..4 stages) that fits 200 KB of shared memory.
__host__ inline int stages_for(int Np) {
  int ns = 4;
  while (ns > 2 && smem_bytes(Np, ns) > 200 * 1024) ns--;
  return ns;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// One CTA streams tiles of BM rows through an NS-stage ring: cp.async brings the FP32 basis
// rows and the split coefficients of K-block i+NS-1 while the tensor cores work on block i.
// Each 16-byte piece q of a [rows][BK] tile lands at byte 16q, which is the core-matrix layout:
// q = (group*8 + k chunk)*8 + row in group.
template <int NS>
__global__ void __launch_bounds__(NTHR, 1) k_orb_tc(Args a) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar[NS];
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char *base = (unsigned char *)(((uintptr_t)sm + 127) & ~(uintptr_t)127);
  const uint32_t sA = BM * BK * 4, sB = (uint32_t)a.Np * BK * 4, stage = 2 * sA + 2 * sB;
  if (tid == 0) {
    for (int i = 0; i < NS; i++) mbar_init(smem_u32(&mbar[i]), 1);
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
  const int nkb = a.Kp / BK;
  const int ntile = (a.M + BM - 1) / BM;
  const int my_tiles = blockIdx.x < ntile ? (ntile - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  const int T = my_tiles * nkb;  // K-blocks this CTA runs
  const int nw_rows = a.n * 5;   // rows per walker of this spin
  const int cb = a.kchunk > 0 ? a.kchunk : nkb;
  const bool vec = (a.nomax & 3) == 0 && ((uintptr_t)a.orb & 15) == 0;

  // issue the copies of K-block i into its stage (an empty group past the end)
  auto issue = [&](int i) {
    if (i < T) {
      const int tile = (int)blockIdx.x + (i / nkb) * (int)gridDim.x, kb = i % nkb, k0 = kb * BK;
      const uint32_t st = smem_u32(base + (size_t)(i % NS) * stage);
      for (int q = tid; q < BM * (BK / 4); q += NTHR) {
        const int cm = q >> 3, r = ((cm >> 3) << 3) + (q & 7), ch = cm & 7, gr = tile * BM + r;
        const float *src = a.phi;
        uint32_t bytes = 0;
        if (gr < a.M) {
          const int w = gr / nw_rows, rem = gr - w * nw_rows;
          src = a.phi + ((long long)(w * a.N + a.e0) * 5 + rem) * a.Kp + k0 + 4 * ch;
          bytes = 16;
        }
        cp_async16(st + 16 * q, src, bytes);
      }
      for (int q = tid; q < a.Np * (BK / 4); q += NTHR) {
        const int cm = q >> 3, r = ((cm >> 3) << 3) + (q & 7), ch = cm & 7;
        const size_t o = (size_t)r * a.Kp + k0 + 4 * ch;
        cp_async16(st + 2 * sA + 16 * q, a.bhi + o, 16);
        cp_async16(st + 2 * sA + sB + 16 * q, a.blo + o, 16);
      }
    }
    cp_commit();
  };

  for (int i = 0; i < NS - 1; i++) issue(i);
  bool ok = true;
  int done = 0;  // K-blocks whose MMA group was committed
  for (int i = 0; i < T; i++) {
    const int s = i % NS, kb = i % nkb;
    unsigned char *st = base + (size_t)s * stage;
    cp_wait<NS - 2>();  // this thread's copies of block i have landed
    __syncthreads();
    // split A in place into its TF32 parts hi and lo
    for (int q = tid; q < BM * (BK / 4); q += NTHR) {
      float4 v = *(float4 *)(st + 16 * q);
      float4 h = make_float4(tf32_hi(v.x), tf32_hi(v.y), tf32_hi(v.z), tf32_hi(v.w));
      *(float4 *)(st + 16 * q) = h;
      *(float4 *)(st + sA + 16 * q) =
          make_float4(tf32_lo(v.x, h.x), tf32_lo(v.y, h.y), tf32_lo(v.z, h.z), tf32_lo(v.w, h.w));
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      const uint32_t uah = smem_u32(st), ual = uah + sA, ubh = uah + 2 * sA, ubl = ubh + sB;
#pragma unroll
      for (int ks = 0; ks < BK / 8; ks++) {
        // one instruction covers K = 8 (two core matrices along K)
        const uint32_t ko = ks * 256;
        uint64_t dah = sdesc(uah + ko, 128, (BK / 4) * 128), dal = sdesc(ual + ko, 128, (BK / 4) * 128);
        uint64_t dbh = sdesc(ubh + ko, 128, (BK / 4) * 128), dbl = sdesc(ubl + ko, 128, (BK / 4) * 128);
        mma_tf32(tbase, dal, dbh, idesc, (kb % cb > 0 || ks > 0) ? 1u : 0u);
        mma_tf32(tbase, dah, dbl, idesc, 1u);
        mma_tf32(tbase, dah, dbh, idesc, 1u);
      }
      mma_commit(smem_u32(&mbar[s]));
    }
    done = i + 1;
    // the stage of block i-1 is refilled with block i+NS-1 once block i-1's MMAs completed;
    // every thread polls, and the block agrees on the outcome
    bool got = true;
    if (i >= 1) got = mbar_wait(smem_u32(&mbar[(i - 1) % NS]), ((i - 1) / NS) & 1);
    if (!__syncthreads_and(got)) { ok = false; break; }
    issue(i + NS - 1);
    if ((kb + 1) % cb == 0 || kb == nkb - 1) {
      // end of an accumulation chunk: drain the accumulator and store it (first chunk of the
      // tile) or add it to the rows (round-to-nearest FP32; the tensor core's own accumulation
      // truncates, so chains stay short); warp q reads TMEM lanes 32(q mod 4)..+31 (the lanes a
      // warp may access), warps q and q+4 take alternate groups of 16 columns
      if (!__syncthreads_and(mbar_wait(smem_u32(&mbar[s]), (i / NS) & 1))) { ok = false; break; }
      const bool first = kb < cb;
      fence_after();
      const int tile = (int)blockIdx.x + (i / nkb) * (int)gridDim.x;
      const int quad = warp & 3, half = warp >> 2;
      const int gr = tile * BM + quad * 32 + lane;
      float *dst = nullptr;
      if (gr < a.M) {
        const int w = gr / nw_rows, rem = gr - w * nw_rows;
        dst = a.orb + ((long long)(w * a.N + a.e0) * 5 + rem) * a.nomax;
      }
      for (int c0 = 16 * half; c0 < a.Np; c0 += 32) {
        float v[16];
        tmem_ld16(tbase + ((uint32_t)(quad * 32) << 16) + (uint32_t)c0, v);
        if (!dst) continue;
        float *o = dst + c0;
        if (vec && c0 + 16 <= a.nocc) {  // 16-byte aligned: four float4 per group
          float4 *o4 = (float4 *)o;
          float4 p[4];
          if (!first)
#pragma unroll
            for (int k = 0; k < 4; k++) p[k] = o4[k];
#pragma unroll
          for (int k = 0; k < 4; k++)
            o4[k] = first ? make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3])
                          : make_float4(p[k].x + v[4 * k], p[k].y + v[4 * k + 1], p[k].z + v[4 * k + 2],
                                        p[k].w + v[4 * k + 3]);
        } else {
#pragma unroll
          for (int k = 0; k < 16; k++)
            if (c0 + k < a.nocc) o[k] = first ? v[k] : o[k] + v[k];
        }
      }
      fence_before();
      __syncthreads();
    }
  }
  cp_wait_all();
  if (!ok) {
    if (a.err) atomicExch(a.err, 1);
    // let the committed MMA groups finish (bounded) before the accumulator is freed
    if (tid == 0)
      for (int u = done > NS ? done - NS : 0; u < done; u++) mbar_wait(smem_u32(&mbar[u % NS]), (u / NS) & 1);
  }
  __syncthreads();
  fence_after();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(a.ncols));
}

}  // namespace orbtc

// Basis values (5 channels) of every electron of every walker as K-major FP32 rows:
// phi[((w*N + e)*5 + ch)*Kp + b], zero for nbasis <= b < Kp.  One warp per electron.
static __global__ void __launch_bounds__(128) k_basis_rows(Sys<float> s, const double *x, long long items, int Kp,
                                                    float *phi) {
  extern __shared__ __align__(16) float sphi[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float *ph = sphi + (size_t)wib * s.nbasis * 5;
  for (long long it = (long long)blockIdx.x * 4 + wib; it < items; it += (long long)gridDim.x * 4) {
    warp_basis<float, 5>(s, x + 3 * it, ph, lane);
    for (int ch = 0; ch < 5; ch++) {
      float *row = phi + (it * 5 + ch) * Kp;
      for (int b = lane; b < Kp; b += 32) row[b] = b < s.nbasis ? ph[b * 5 + ch] : 0.f;
    }
    __syncwarp();
  }
}

#include "orbfused.cuh"
