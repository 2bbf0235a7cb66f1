// Block low-rank correction on the 5th-generation tensor cores (tcgen05).
//
// For a block of NL complex64 right-hand sides x_q, the GeMSLR low-rank
// correction of one level (GemslrClass::SolveApplyLowRankLevel,
// gemslr.cpp:3681-3722; ParallelGemslrClass::SolveApplyLowRankLevel,
// parallel_gemslr.cpp:6627-6680) is two GEMMs:
//   Y = W^H X          (r x NL; W is m x r, X = [x_1 .. x_NL] is m x NL)
//   X' = X s + WH Y    (s: a per-vector scale, the lazy Krylov column scale)
// Each runs in real form on tcgen05.mma kind::tf32 with the accumulator in
// tensor memory (TMEM):
//   Y:  D = A B^T with A = [Re W, Im W]^T (2r x m) and B = [Re X, Im X]^T
//       (2NL x m), then Re Y = D11 + D22, Im Y = D12 - D21 (2x2 blocks);
//   X': D = A B^T with A = [Re WH | Im WH] (m x 2r) and
//       B = [[Re Y, -Im Y]; [Im Y, Re Y]]^T (2NL x 2r).
// A tf32 MMA reads the top 19 bits of each FP32 operand.  Every operand is
// split as a = hi + lo (hi: a with its 13 low mantissa bits cleared; lo: the
// exact remainder), and three MMAs (hi*hi, hi*lo, lo*hi) accumulate in FP32,
// which keeps the products to about FP32 accuracy ("3xTF32").
//
// Shared-memory operands use the K-major, non-swizzled canonical layout of
// the UMMA descriptors: core matrices of 8 rows x 16 bytes, the two 16-byte
// K halves of one MMA (K = 8 tf32) LBO = 128 bytes apart and consecutive
// 8-row groups SBO bytes apart.  One thread issues the MMAs; their completion
// is signalled by tcgen05.commit on an mbarrier whose waits are bounded.
#pragma once

#include "pgx_device.cuh"

namespace pgx {

constexpr int kUmmaThreads = 128;  // 4 warps: one per TMEM lane quarter (M = 128)
constexpr int kUmmaKT = 32;        // K rows staged per step of the W^H X kernel
constexpr int kUmmaMaxRank = 64;   // 2r <= 128 = M

// UMMA shared-memory matrix descriptor (K-major, no swizzle).
__device__ __forceinline__ uint64_t umma_desc(const void* smem, uint32_t lbo, uint32_t sbo) {
  const uint32_t a = smem_u32(smem);
  uint64_t d = 0;
  d |= (uint64_t)((a >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, layout type 0 (no swizzle)
}
// Instruction descriptor: D f32, A and B tf32, both K-major, M = 128, N.
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
// byte offset of element (row, k) in a K-major tile of KT columns
__device__ __forceinline__ int umma_off(int row, int k, int KT) {
  return (row >> 3) * (KT * 32) + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4;
}
__device__ __forceinline__ void tf32_split(float a, float& hi, float& lo) {
  hi = __int_as_float(__float_as_int(a) & (int)0xFFFFE000);
  lo = a - hi;
}
// Stage a rows x KT operand tile: value(row, k) for element e = (row, k) of the
// tile, split into its hi and lo tiles.  Each thread loads kStageBatch values
// before it stores any, so their global loads are in flight together.
constexpr int kStageBatch = 8;
template <typename F>
__device__ __forceinline__ void umma_stage(unsigned char* hi_tile, unsigned char* lo_tile, int rows, int KT,
                                           bool k_fastest, F value) {
  const int total = rows * KT;
  for (int base = threadIdx.x; base < total; base += kUmmaThreads * kStageBatch) {
    float v[kStageBatch];
#pragma unroll
    for (int u = 0; u < kStageBatch; u++) {
      const int e = base + u * kUmmaThreads;
      v[u] = 0.f;
      if (e < total) v[u] = k_fastest ? value(e / KT, e % KT) : value(e % rows, e / rows);
    }
#pragma unroll
    for (int u = 0; u < kStageBatch; u++) {
      const int e = base + u * kUmmaThreads;
      if (e < total) {
        const int row = k_fastest ? e / KT : e % rows, k = k_fastest ? e % KT : e / rows;
        float h, l;
        tf32_split(v[u], h, l);
        *(float*)(hi_tile + umma_off(row, k, KT)) = h;
        *(float*)(lo_tile + umma_off(row, k, KT)) = l;
      }
    }
  }
}

__device__ __forceinline__ void tmem_alloc32(uint32_t* slot) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_u32(slot)) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc32(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(taddr) : "memory");
}
__device__ __forceinline__ void umma_tf32(uint32_t taddr, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(taddr), "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 16 consecutive FP32 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __int_as_float((int)r[i]);
}

// Per-vector pointers of a block of NL complex64 right-hand sides.
template <int NL>
struct LrBlock {
  const cf32* in[NL];       // x_q (read)
  cf32* out[NL];            // x'_q (written; may equal in)
  const double* scale[NL];  // s_q, or null for 1
};

// Y = W^H X (with X scaled by s): split-K over the grid; every CTA keeps its
// partial 2r x 2NL product in global memory and the last CTA to finish sums
// them in CTA order (fixed, so the result does not depend on scheduling)
// into Y (r x NL, complex64, column q = vector q).
template <int NL>
__global__ void __launch_bounds__(kUmmaThreads) lr_wtx_umma_kernel(int m, int r, const cf32* __restrict__ W,
                                                                   LrBlock<NL> xb, float* __restrict__ partial,
                                                                   unsigned int* counter, cf32* __restrict__ Y,
                                                                   int* err, SkipR<NL> skip) {
  constexpr int N = 2 * NL;
  constexpr int KT = kUmmaKT;
  if (skip.on()) return;
  extern __shared__ __align__(128) unsigned char sm[];
  unsigned char* a_hi = sm;                    // 128 x KT
  unsigned char* a_lo = a_hi + 128 * KT * 4;
  unsigned char* b_hi = a_lo + 128 * KT * 4;   // N x KT
  unsigned char* b_lo = b_hi + N * KT * 4;
  __shared__ __align__(8) unsigned long long bar;
  __shared__ uint32_t s_taddr;
  __shared__ int s_last, s_fail;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int nchunks = (m + KT - 1) / KT;
  const int per = (nchunks + gridDim.x - 1) / gridDim.x;
  const int c0 = blockIdx.x * per, c1 = min(nchunks, c0 + per);
  if (tid == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
    s_fail = 0;
  }
  if (warp == 0) tmem_alloc32(&s_taddr);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = s_taddr;
  const uint32_t idesc = umma_idesc_tf32(N);
  unsigned phase = 0;
  bool issued = false;
  bool pending = false;  // a commit whose phase no thread has seen complete
  for (int ch = c0; ch < c1; ch++) {
    if (issued) {
      // the MMAs of the previous chunk have read the operands
      if (!mbar_wait(&bar, phase, err)) s_fail = 1;
      __syncthreads();
      if (s_fail) break;
      pending = false;
      phase ^= 1u;
    }
    const int k0 = ch * KT;
    // A = [Re W, Im W]^T, rows c and r + c; rows 2r..127 zero (staged once,
    // in the first chunk: the loop below only rewrites rows < 2r)
    umma_stage(a_hi, a_lo, ch == c0 ? 128 : 2 * r, KT, true, [&](int row, int k) -> float {
      if (row >= 2 * r || k0 + k >= m) return 0.f;
      const cf32 w = W[(size_t)(row % r) * m + k0 + k];
      return row < r ? w.x : w.y;
    });
    // B = [Re X, Im X]^T, rows q and NL + q, scaled by s_q
    umma_stage(b_hi, b_lo, N, KT, true, [&](int row, int k) -> float {
      if (k0 + k >= m) return 0.f;
      const int q = row % NL;
      cf32 x = xb.in[q][k0 + k];
      if (xb.scale[q]) x = x * (float)(*xb.scale[q]);
      return row < NL ? x.x : x.y;
    });
    proxy_fence_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < KT / 8; s++) {
        const uint32_t off = (uint32_t)s * 256;  // two 16-byte K halves of 8 tf32
        const uint64_t ah = umma_desc(a_hi + off, 128, KT * 32), al = umma_desc(a_lo + off, 128, KT * 32);
        const uint64_t bh = umma_desc(b_hi + off, 128, KT * 32), bl = umma_desc(b_lo + off, 128, KT * 32);
        const bool acc0 = ch > c0 || s > 0;
        umma_tf32(taddr, ah, bh, idesc, acc0);
        umma_tf32(taddr, ah, bl, idesc, true);
        umma_tf32(taddr, al, bh, idesc, true);
      }
      umma_commit(&bar);
    }
    issued = true;
    pending = true;
  }
  if (pending && !s_fail) {
    if (!mbar_wait(&bar, phase, err)) s_fail = 1;
    else
      pending = false;
  }
  __syncthreads();
  // a wait gave up: give the MMAs in flight one more bounded wait before the
  // tensor memory they write is released
  if (s_fail && pending) mbar_wait(&bar, phase, err);
  tc_fence_after();
  // this CTA's partial product (zero for a CTA without chunks)
  const int row = warp * 32 + (tid & 31);
  float d[N];
  if (issued && !s_fail) {
#pragma unroll
    for (int c = 0; c < N; c += 16) tmem_ld16(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, d + c);
  } else {
#pragma unroll
    for (int c = 0; c < N; c++) d[c] = 0.f;
  }
  if (row < 2 * r) {
#pragma unroll
    for (int c = 0; c < N; c++) partial[((size_t)blockIdx.x * 2 * r + row) * N + c] = d[c];
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc32(taddr);
  if (s_fail) return;
  __threadfence();
  if (tid == 0) s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // sum of the partial products in CTA order: each thread keeps its entries
  // (consecutive threads, consecutive entries) in registers, so every step
  // over the CTAs is one coalesced load per entry, all in flight together
  constexpr int PER = 2 * kUmmaMaxRank * N / kUmmaThreads;
  const int ne = 2 * r * N;
  float acc[PER];
#pragma unroll
  for (int u = 0; u < PER; u++) acc[u] = 0.f;
  for (int g = 0; g < (int)gridDim.x; g++) {
    const float* pg = partial + (size_t)g * ne;
#pragma unroll
    for (int u = 0; u < PER; u++) {
      const int e = tid + u * kUmmaThreads;
      if (e < ne) acc[u] += __ldcg(&pg[e]);
    }
  }
  float* red = (float*)sm;  // the operand buffers are free now
#pragma unroll
  for (int u = 0; u < PER; u++) {
    const int e = tid + u * kUmmaThreads;
    if (e < ne) red[e] = acc[u];
  }
  __syncthreads();
  // Y(c, q) = (D[c, q] + D[r + c, NL + q]) + i (D[c, NL + q] - D[r + c, q])
  for (int e = tid; e < r * NL; e += kUmmaThreads) {
    const int c = e % r, q = e / r;
    Y[(size_t)q * r + c] =
        cf32(red[c * N + q] + red[(r + c) * N + NL + q], red[c * N + NL + q] - red[(r + c) * N + q]);
  }
  if (tid == 0) *counter = 0u;
}

// X'_q = X_q s_q + WH Y_q for the 128-row tile of each CTA.
template <int NL>
__global__ void __launch_bounds__(kUmmaThreads) lr_update_umma_kernel(int m, int r, const cf32* __restrict__ WH,
                                                                      const cf32* __restrict__ Y, LrBlock<NL> xb,
                                                                      int* err, SkipR<NL> skip) {
  constexpr int N = 2 * NL;
  if (skip.on()) return;
  extern __shared__ __align__(128) unsigned char sm[];
  const int KT = (2 * r + 7) / 8 * 8;  // K = 2r, padded to whole MMAs
  unsigned char* a_hi = sm;            // 128 x KT
  unsigned char* a_lo = a_hi + 128 * KT * 4;
  unsigned char* b_hi = a_lo + 128 * KT * 4;  // N x KT
  unsigned char* b_lo = b_hi + N * KT * 4;
  __shared__ __align__(8) unsigned long long bar;
  __shared__ uint32_t s_taddr;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int i0 = blockIdx.x * 128;
  if (tid == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  if (warp == 0) tmem_alloc32(&s_taddr);
  // A = [Re WH | Im WH] rows i0..i0+127 (row fastest: coalesced along a
  // column of WH); K padding and rows past m zero
  umma_stage(a_hi, a_lo, 128, KT, false, [&](int row, int k) -> float {
    if (k >= 2 * r || i0 + row >= m) return 0.f;
    const cf32 w = WH[(size_t)(k % r) * m + i0 + row];
    return k < r ? w.x : w.y;
  });
  // B rows q: [Re Y_q, -Im Y_q]; rows NL + q: [Im Y_q, Re Y_q]
  umma_stage(b_hi, b_lo, N, KT, true, [&](int row, int k) -> float {
    if (k >= 2 * r) return 0.f;
    const int q = row % NL;
    const cf32 y = Y[(size_t)q * r + (k % r)];
    if (row < NL) return k < r ? y.x : -y.y;
    return k < r ? y.y : y.x;
  });
  proxy_fence_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t taddr = s_taddr;
  if (tid == 0) {
    const uint32_t idesc = umma_idesc_tf32(N);
    for (int s = 0; s < KT / 8; s++) {
      const uint32_t off = (uint32_t)s * 256;
      const uint64_t ah = umma_desc(a_hi + off, 128, KT * 32), al = umma_desc(a_lo + off, 128, KT * 32);
      const uint64_t bh = umma_desc(b_hi + off, 128, KT * 32), bl = umma_desc(b_lo + off, 128, KT * 32);
      umma_tf32(taddr, ah, bh, idesc, s > 0);
      umma_tf32(taddr, ah, bl, idesc, true);
      umma_tf32(taddr, al, bh, idesc, true);
    }
    umma_commit(&bar);
  }
  const bool ok = mbar_wait(&bar, 0, err);
  if (!ok) mbar_wait(&bar, 0, err);  // one more bounded wait before the TMEM is released
  tc_fence_after();
  const int row = warp * 32 + (tid & 31);
  float d[N];
  if (ok) {
#pragma unroll
    for (int c = 0; c < N; c += 16) tmem_ld16(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, d + c);
    const int i = i0 + row;
    if (i < m) {
#pragma unroll
      for (int q = 0; q < NL; q++) {
        cf32 x = xb.in[q][i];
        if (xb.scale[q]) x = x * (float)(*xb.scale[q]);
        xb.out[q][i] = x + cf32(d[q], d[NL + q]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc32(taddr);
}

// CTAs of the split-K W^H X: at least 8 K chunks each, at most one per SM,
// so the fixed-order sum of the partial products stays short
inline int lr_wtx_grid(int m) {
  const int nchunks = (m + kUmmaKT - 1) / kUmmaKT;
  return nchunks / 8 < 1 ? 1 : (nchunks / 8 > 148 ? 148 : nchunks / 8);
}

template <int NL>
constexpr size_t lr_wtx_smem() {
  return (size_t)2 * (128 + 2 * NL) * kUmmaKT * 4;
}
inline size_t lr_update_smem(int r, int NL) {
  const int KT = (2 * r + 7) / 8 * 8;
  return (size_t)2 * (128 + 2 * NL) * KT * 4;
}

}  // namespace pgx
