// Device-side building blocks of the GeMSLR-FGMRES solve phase (sm_100a).
//
// Every kernel takes a Skip descriptor: up to three device flags (the
// "cycle finished" / "solve finished" words of the enclosing FGMRES solves).
// A kernel whose flags are set returns at once, so a whole restart cycle can
// be enqueued (or captured in a CUDA graph) ahead of time and the iterations
// after convergence cost one launch each and no memory traffic.
#pragma once

#include <climits>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pgx {

constexpr int kWarp = 32;
constexpr int KMAX = 128;          // largest Krylov dimension a handle accepts
constexpr int kTsThreads = 512;    // block size of the tall-skinny kernels
constexpr int kTsMaxBlocks = 296;  // 2 blocks per SM on a 148-SM B200
constexpr int kSpinLimit = 1 << 21;  // bounded waits in the sync-free triangular solve

// status bits written by kernels into the handle's error word
constexpr int kErrTimeout = 1;
constexpr int kErrIndex = 2;

struct Skip {
  const int* f0;
  const int* f1;
  const int* f2;
  __device__ __forceinline__ bool on() const {
    return (f0 && *(const volatile int*)f0) || (f1 && *(const volatile int*)f1) ||
           (f2 && *(const volatile int*)f2);
  }
};

// Skip flags of R solves advancing together: a kernel shared by them returns
// only when every one of them is skipped.
template <int R>
struct SkipR {
  Skip s[R];
  __device__ __forceinline__ bool on() const {
#pragma unroll
    for (int r = 0; r < R; r++)
      if (!s[r].on()) return false;
    return true;
  }
};

// ---------------------------------------------------------------- FGMRES
// Device-resident state of one flexible GMRES solve (FlexGmresClass::Solve,
// ParGeMSLR SRC/solvers/fgmres.hpp:263-558).  H is column-major (KMAX+1) x KMAX.
struct FgmresDev {
  int done;        // solve finished (converged, max iterations or breakdown)
  int cycle_done;  // current restart cycle finished
  int breakdown;   // Givens breakdown: the reference skips the x update
  int converged;
  int iter;        // iterations so far (FlexGmresClass::_iter)
  int i;           // columns built in the current cycle
  int kdim;
  int maxits;
  double tolr;     // absolute threshold on the Givens residual estimate
  double tol;
  double normb;
  double normr;    // Givens residual estimate (reference: normr)
  double eps;      // numeric_limits<RealDataType>::epsilon() of the solver
  int absolute;
  int pad;
  double sc[KMAX + 1];     // V(:,c) = Vstored(:,c) * sc[c] (lazy normalisation)
  double hcol[KMAX + 1];   // column of H being built
  double coefA[KMAX + 1];  // first Gram-Schmidt coefficients
  double coefB[KMAX + 1];  // re-orthogonalisation coefficients
  double c[KMAX], s[KMAX], rs[KMAX + 1], y[KMAX];
  double H[(KMAX + 1) * KMAX];
};

template <typename T>
__device__ __forceinline__ T ldcg(const T* p) { return __ldcg(p); }

template <typename T>
__device__ __forceinline__ T group_reduce(T v, int S, int lane) {
  // sum over this lane's aligned group of S lanes; only that group's lanes
  // take part, so other groups of the warp may be elsewhere (spinning)
  const unsigned mask = S == 32 ? 0xffffffffu : (((1u << S) - 1u) << (lane & ~(S - 1)));
  for (int off = S >> 1; off > 0; off >>= 1) v += __shfl_xor_sync(mask, v, off);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_reduce(T v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// ------------------------------------------------------------ CSR SpMV
// y = alpha * (A1 x1) + alpha2 * (A2 x2) + beta * b, S lanes per row.
// A2 may be absent (rp2 == nullptr); b may be absent or alias y.
// Follows CsrMatrixPMatVecHostTemplate (ParGeMSLR SRC/matrices/matrixops.cpp:5139)
// for one matrix; the two-matrix form fuses the Schur operator
// C x - E (B^-1 F x) of GemslrClass::SchurMatVec (gemslr.cpp:3799-3960).
template <typename TA, typename TX, typename TY, typename TC, int S>
__global__ void __launch_bounds__(256) spmv_kernel(
    int nrows, const int* __restrict__ rp1, const int* __restrict__ cj1, const TA* __restrict__ va1,
    const TX* __restrict__ x1, TC alpha, const int* __restrict__ rp2, const int* __restrict__ cj2,
    const TA* __restrict__ va2, const TX* __restrict__ x2, TC alpha2, const TY* b, TC beta, TY* y,
    const double* __restrict__ xscale, Skip skip) {
  if (skip.on()) return;
  const int lane = threadIdx.x & (S - 1);
  const int wlane = threadIdx.x & 31;
  const int groups_per_block = blockDim.x / S;
  const TC xs = xscale ? (TC)(*xscale) : (TC)1;
  for (int row = blockIdx.x * groups_per_block + threadIdx.x / S; row < nrows;
       row += gridDim.x * groups_per_block) {
    TC acc = 0;
    const int k1 = rp1[row], k2 = rp1[row + 1];
    for (int k = k1 + lane; k < k2; k += S) acc += (TC)va1[k] * (TC)x1[cj1[k]];
    acc = group_reduce(acc, S, wlane);
    TC acc2 = 0;
    if (rp2) {
      const int q1 = rp2[row], q2 = rp2[row + 1];
      for (int k = q1 + lane; k < q2; k += S) acc2 += (TC)va2[k] * (TC)x2[cj2[k]];
      acc2 = group_reduce(acc2, S, wlane);
    }
    if (lane == 0) {
      TC v = alpha * (acc * xs);
      if (rp2) v += alpha2 * acc2;
      if (b) v += beta * (TC)b[row];
      y[row] = (TY)v;
    }
  }
}

// ----------------------------------------------- sync-free triangular solve
// One pass of the ILU solve of IluClass::SolveHost (ParGeMSLR
// SRC/preconditioners/ilu.cpp:3677-3790) over a whole level (all subdomains
// of the level concatenated block-diagonally):
//   lower:  y_r = rhs_r - sum_j L_rj y_j               (unit diagonal)
//   upper:  x_r = (y_r - sum_j U_rj x_j) * dinv_r     (dinv = inverse diagonal)
// Rows are stored in level-set order (IluClass::BuildLevels rule,
// ilu.cpp:832-1062), each level padded to whole groups of G = 32/S rows, so a
// group never holds two rows of which one depends on the other.
//
// Readiness is carried by the value itself: entries not yet computed hold a
// signalling-NaN sentinel that arithmetic never produces.  A row publishes
// its result with one relaxed store; a consumer polls the entry with relaxed
// loads until the sentinel is gone - one L2 round trip per dependency and no
// fences.  The lower pass writes y and sets x to the sentinel; the upper pass
// consumes y, writes x and puts the sentinel back into y, so each pass leaves
// the buffers ready for the next one.
//
// The grid is persistent and sized to the level width (few pollers, little
// L2 pressure).  Warps claim groups from a 64-bit ticket counter in schedule
// order; a row only waits on rows of earlier levels, whose groups were
// claimed earlier by warps that are running, so the waits always end.  The
// last warp to leave resets the counter (ticket[0]) and the exit count
// (ticket[1]) for the next launch, whatever the grid size.  Waits are
// bounded; on expiry the kernel records kErrTimeout and finishes.
template <typename T>
struct Sentinel;
template <>
struct Sentinel<double> {
  static __device__ __forceinline__ double value() { return __longlong_as_double(0xFFF4DEADBEEF0001LL); }
  static __device__ __forceinline__ bool is(double v) { return __double_as_longlong(v) == 0xFFF4DEADBEEF0001LL; }
  static __device__ __forceinline__ double load(const double* p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
  }
  static __device__ __forceinline__ void store(double* p, double v) {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
  }
};
template <>
struct Sentinel<float> {
  static __device__ __forceinline__ float value() { return __int_as_float((int)0xFFA0BEEFu); }
  static __device__ __forceinline__ bool is(float v) { return __float_as_int(v) == (int)0xFFA0BEEFu; }
  static __device__ __forceinline__ float load(const float* p) {
    float v;
    asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
  }
  static __device__ __forceinline__ void store(float* p, float v) {
    asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
  }
};

template <typename T>
__global__ void sentinel_fill_kernel(int n, T* p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = Sentinel<T>::value();
}

template <typename T, int S, bool UPPER>
__global__ void __launch_bounds__(256) trsv_kernel(
    int n, int ngroups, const int* __restrict__ ord, const int* __restrict__ rp, const int* __restrict__ cj,
    const T* __restrict__ va, const T* __restrict__ dinv, const T* __restrict__ rhs,
    const double* __restrict__ rhs_scale, T* y, T* x, unsigned long long* ticket, int* err, Skip skip) {
  constexpr int G = kWarp / S;  // rows per warp
  if (skip.on()) return;
  const int lane = threadIdx.x & (kWarp - 1);
  const int sl = lane & (S - 1);
  const double rs = rhs_scale ? *rhs_scale : 1.0;
  T* dep = UPPER ? x : y;  // the vector this pass polls
  while (true) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(&ticket[0], 1ULL);
    t = __shfl_sync(0xffffffffu, t, 0);
    const unsigned long long g = t;
    if (g >= (unsigned long long)ngroups) break;
    const int pos = (int)g * G + lane / S;
    const int r = ord[pos];  // -1 marks padding; uniform over the S-lane group
    if (r >= 0) {
      T acc = 0;
      const int k1 = rp[pos], k2 = rp[pos + 1];
      for (int k = k1 + sl; k < k2; k += S) {
        const int j = cj[k];
        if ((unsigned)j >= (unsigned)n) {
          atomicOr(err, kErrIndex);
          continue;
        }
        T v = Sentinel<T>::load(&dep[j]);
        if (Sentinel<T>::is(v)) {
          int spins = 0;
          do {
            if (++spins > kSpinLimit || (*(volatile int*)err & kErrTimeout)) {
              atomicOr(err, kErrTimeout);
              v = 0;
              break;
            }
            __nanosleep(20);
            v = Sentinel<T>::load(&dep[j]);
          } while (Sentinel<T>::is(v));
        }
        acc += va[k] * v;
      }
      acc = group_reduce(acc, S, lane);
      if (sl == 0) {
        if (UPPER) {
          const T yr = y[r];
          y[r] = Sentinel<T>::value();
          Sentinel<T>::store(&x[r], (yr - acc) * dinv[r]);
        } else {
          T b = rhs[r];
          if (rhs_scale) b = (T)((double)b * rs);
          x[r] = Sentinel<T>::value();
          Sentinel<T>::store(&y[r], b - acc);
        }
      }
    }
  }
  // the last warp to leave rewinds the counters for the next launch
  if (lane == 0) {
    __threadfence();
    const unsigned long long nw = (unsigned long long)gridDim.x * (blockDim.x / kWarp);
    if (atomicAdd(&ticket[1], 1ULL) == nw - 1) {
      ticket[0] = 0ULL;
      ticket[1] = 0ULL;
      __threadfence();
    }
  }
}

// ------------------------------------- segmented (CTA-local) triangular solve
// Same arithmetic as trsv_kernel, different schedule.  Each subdomain's rows,
// in level-set order, are cut into segments of at most kSegRows rows and
// kSegNnz nonzeros.  A CTA claims a segment (ticket order: by first level,
// then subdomain, so a segment only depends on segments claimed earlier),
// stages the segment's row list, row pointers, column indices and values into
// shared memory with cp.async, then sweeps the segment's levels with one
// __syncthreads per level.  Dependencies inside the segment are read from the
// shared-memory copy of the results (column index encoded as -(slot+1));
// dependencies on earlier segments are polled in global memory through the
// sentinel protocol of trsv_kernel.  Every result is also published to global
// memory for later segments and the next kernel.
constexpr int kSegThreads = 1024;
constexpr int kSegRows = 1024;
constexpr int kSegNnzF64 = 8192;    // staged cj + va + gathered operands: 160 KB (FP64)
constexpr int kSegNnzF32 = 12288;   // 144 KB (FP32)

template <typename T>
struct SegCfg {
  static constexpr int nnz = sizeof(T) == 8 ? kSegNnzF64 : kSegNnzF32;
  // smem layout: xs[kSegRows] T | sb[kSegRows] T | sd[kSegRows] T | va[nnz] T | ext[nnz] T |
  // cj[nnz] int | ord[kSegRows] int | rp[kSegRows+4] int | lvb[kSegRows+4] int; the host keeps
  // segments within kSegRows-4 rows and nnz-4 nonzeros
  static constexpr size_t bytes =
      sizeof(T) * (size_t)(3 * kSegRows + 2 * nnz) + sizeof(int) * (size_t)(nnz + kSegRows + 2 * (kSegRows + 4));
};

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// copy `bytes` (multiple of 16, both addresses 16-byte aligned) with cp.async
__device__ __forceinline__ void stage16(void* dst, const void* src, int bytes) {
  for (int o = threadIdx.x * 16; o < bytes; o += blockDim.x * 16) cp_async16((char*)dst + o, (const char*)src + o);
}

template <typename T, int S, bool UPPER>
__global__ void __launch_bounds__(kSegThreads) trsv_seg_kernel(
    int n, int nseg, const int* __restrict__ seg_row0,  // nseg+1: first slot in ord
    const int* __restrict__ seg_rp0,                     // nseg+1: first slot in rp (segment-relative values)
    const int* __restrict__ seg_nnz0,                    // nseg+1: first slot in cj / va
    const int* __restrict__ seg_lv0,                     // nseg+1: first slot in lvb
    const int* __restrict__ seg_nlvb,                    // nseg: number of level boundaries
    const int* __restrict__ ord, const int* __restrict__ rp,  // rp: segment-relative row pointers
    const int* __restrict__ cj, const T* __restrict__ va, const int* __restrict__ lvb,  // lvb: segment-relative
    const T* __restrict__ dinv, const T* __restrict__ rhs, const double* __restrict__ rhs_scale, T* y, T* x,
    unsigned long long* ticket, int* err, Skip skip) {
  if (skip.on()) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NNZ = SegCfg<T>::nnz;
  T* xs = (T*)smem_raw;
  T* sb = xs + kSegRows;  // rhs (lower) or y (upper) of the segment's rows
  T* sd = sb + kSegRows;  // dinv of the segment's rows (upper)
  T* sva = sd + kSegRows;
  T* sext = sva + NNZ;  // operands from earlier segments, gathered at staging
  int* scj = (int*)(sext + NNZ);
  int* sord = scj + NNZ;
  int* srp = sord + kSegRows;
  int* slvb = srp + kSegRows + 4;
  __shared__ unsigned long long s_t;
  const int tid = threadIdx.x, lane = tid & 31;
  const int sl = lane & (S - 1);
  const int group = tid / S, ngroups = kSegThreads / S;
  const double rs = rhs_scale ? *rhs_scale : 1.0;
  T* dep = UPPER ? x : y;
  while (true) {
    if (tid == 0) s_t = atomicAdd(&ticket[0], 1ULL);
    __syncthreads();
    const unsigned long long g = s_t;
    if (g >= (unsigned long long)nseg) break;
    const int sgi = (int)g;
    // every per-segment block starts 16-byte aligned and has a 16-byte
    // multiple length (padded on the host)
    const int r0 = seg_row0[sgi], r1 = seg_row0[sgi + 1];
    const int p0 = seg_rp0[sgi], p1 = seg_rp0[sgi + 1];
    const int z0 = seg_nnz0[sgi], z1 = seg_nnz0[sgi + 1];
    const int v0 = seg_lv0[sgi];
    const int nlvb = seg_nlvb[sgi];
    stage16(sva, va + z0, (z1 - z0) * (int)sizeof(T));
    stage16(scj, cj + z0, (z1 - z0) * 4);
    stage16(sord, ord + r0, (r1 - r0) * 4);
    stage16(srp, rp + p0, (p1 - p0) * 4);
    stage16(slvb, lvb + v0, (seg_lv0[sgi + 1] - v0) * 4);
    // gather the per-row operands while the copies are in flight (plain
    // loads: independent, so they overlap)
    for (int i = tid; i < r1 - r0; i += blockDim.x) {
      const int r = __ldg(&ord[r0 + i]);
      if (r < 0) continue;
      if (UPPER) {
        sb[i] = __ldcg(&y[r]);
        sd[i] = __ldg(&dinv[r]);
      } else {
        T bb = __ldg(&rhs[r]);
        if (rhs_scale) bb = (T)((double)bb * rs);
        sb[i] = bb;
      }
    }
    cp_async_wait_all();
    __syncthreads();
    // gather every operand owned by an earlier segment in one parallel sweep
    // through L2; most are final already, the rest still read the sentinel
    // and are polled in the sweep below.  Entries are written with single
    // 4/8-byte stores, so a load sees either the sentinel or the final value.
    for (int k = tid; k < z1 - z0; k += blockDim.x) {
      const int c = scj[k];
      if (c >= 0 && c < n) sext[k] = __ldcg(&dep[c]);
    }
    // this segment's rows: hand the buffers to the next pass
    for (int i = tid; i < r1 - r0; i += blockDim.x) {
      const int r = sord[i];
      if (r < 0) continue;
      if (UPPER)
        y[r] = Sentinel<T>::value();
      else
        x[r] = Sentinel<T>::value();
    }
    __syncthreads();
    for (int lv = 0; lv + 1 < nlvb; lv++) {
      const int a = slvb[lv], b = slvb[lv + 1];
      for (int i = a + group; i < b; i += ngroups) {
        const int r = sord[i];
        if (r < 0) continue;  // padding slot
        T acc = 0;
        const int k1 = srp[i], k2 = srp[i + 1];
        for (int k = k1 + sl; k < k2; k += S) {
          const int c = scj[k];
          T v;
          if (c < 0) {
            v = xs[-c - 1];
          } else {
            if ((unsigned)c >= (unsigned)n) {
              atomicOr(err, kErrIndex);
              continue;
            }
            v = sext[k];
            if (Sentinel<T>::is(v)) {
              v = Sentinel<T>::load(&dep[c]);
            }
            if (Sentinel<T>::is(v)) {
              int spins = 0;
              do {
                if (++spins > kSpinLimit || (*(volatile int*)err & kErrTimeout)) {
                  atomicOr(err, kErrTimeout);
                  v = 0;
                  break;
                }
                __nanosleep(20);
                v = Sentinel<T>::load(&dep[c]);
              } while (Sentinel<T>::is(v));
            }
          }
          acc += sva[k] * v;
        }
        acc = group_reduce(acc, S, lane);
        if (sl == 0) {
          T out;
          if (UPPER) {
            out = (sb[i] - acc) * sd[i];
            Sentinel<T>::store(&x[r], out);
          } else {
            out = sb[i] - acc;
            Sentinel<T>::store(&y[r], out);
          }
          xs[i] = out;
        }
      }
      __syncthreads();
    }
    __syncthreads();  // s_t and the staged arrays are reused by the next claim
  }
  // the last CTA to leave rewinds the counters for the next launch
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(&ticket[1], 1ULL) == (unsigned long long)gridDim.x - 1) {
      ticket[0] = 0ULL;
      ticket[1] = 0ULL;
      __threadfence();
    }
  }
}

// ----------------------------- one-CTA-per-subdomain triangular solve
// Same arithmetic as trsv_kernel.  In level-set order the dependencies of an
// ILU factor are short-range: for the RCM-ordered subdomains of a 3D problem
// the median distance between a row and the rows it needs is ~10^3
// positions and almost all are within 10^4.  So one CTA walks a whole
// subdomain (trsv_comp_kernel below).
#ifndef PGX_COMP_THREADS
#define PGX_COMP_THREADS 1024
#endif
// 1024 threads: one CTA per SM; 512 threads: two CTAs per SM (registers and
// shared memory sized for it), for many concurrent solves
constexpr int kCompThreads = PGX_COMP_THREADS;
constexpr int kCompMinBlocks = kCompThreads >= 1024 ? 1 : 2;
constexpr int kUnroll = 4;  // operands per lane loaded before any is used
// Operand indices into the ring are checked once on the host when the layout
// is built; the kernels clamp them into the shared array, so a damaged layout
// can give wrong values but never an access outside shared memory.
template <typename T>
struct CompCfg {
  static constexpr bool big = kCompThreads >= 1024;
  static constexpr int ring = big ? 8192 : 4096;              // 32/16 KB (f32), 64/32 KB (f64)
  static constexpr int far = big ? 1024 : 512;                // far operands per chunk (per buffer)
  static constexpr int nnz = sizeof(T) == 8 ? (big ? 4096 : 2048) : (big ? 8192 : 4096);  // per chunk buffer
  static constexpr int rows = sizeof(T) == 8 ? (big ? 768 : 384) : (big ? 1024 : 512);   // incl. padding
  // per buffer: va[nnz] T | sb[rows] T | sd[rows] T | cj[nnz] int | ord[rows] int | rp[rows+4] int | lvb[rows+4] int
  static constexpr size_t buf_bytes =
      sizeof(T) * (size_t)(nnz + 2 * rows) + sizeof(int) * (size_t)(nnz + rows + 2 * (rows + 4));
  // ring and the two far-operand buffers are one array: operand index -(c+1)
  static constexpr size_t bytes = sizeof(T) * (size_t)(ring + 2 * far) + 2 * buf_bytes;
  static_assert(bytes * kCompMinBlocks <= 227 * 1024, "per-subdomain solve exceeds the shared memory of an SM");
  static_assert(far <= kCompThreads && rows <= kCompThreads, "one gather per thread");
};

// Per-chunk metadata, two int4 per chunk: {row0, rp0, nnz0, lv0} and
// {pos0, far0, 0, 0}: first slot of the chunk in the row list, the row
// pointers, the nonzeros and the level boundaries; its first schedule
// position; its first far operand.  One record past the last chunk closes the
// ranges.
struct ChunkMeta {
  int row0, rp0, nnz0, lv0, pos0, far0;
};
__device__ __forceinline__ ChunkMeta load_meta(const int4* __restrict__ meta, int ch) {
  const int4 a = __ldg(&meta[2 * ch]), b = __ldg(&meta[2 * ch + 1]);
  ChunkMeta m;
  m.row0 = a.x;
  m.rp0 = a.y;
  m.nnz0 = a.z;
  m.lv0 = a.w;
  m.pos0 = b.x;
  m.far0 = b.y;
  return m;
}

__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem_src) : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src) {
  if (sizeof(T) == 8)
    cp_async8(dst, src);
  else
    cp_async4(dst, src);
}

template <typename T>
struct CompBuf {
  T *va, *sb, *sd;
  int *cj, *ord, *rp, *lvb;
};

template <typename T>
__device__ __forceinline__ CompBuf<T> comp_buf(unsigned char* base, int which) {
  using C = CompCfg<T>;
  unsigned char* b = base + sizeof(T) * (size_t)(C::ring + 2 * C::far) + (size_t)which * C::buf_bytes;
  CompBuf<T> o;
  o.va = (T*)b;
  o.sb = o.va + C::nnz;
  o.sd = o.sb + C::rows;
  o.cj = (int*)(o.sd + C::rows);
  o.ord = o.cj + C::nnz;
  o.rp = o.ord + C::rows;
  o.lvb = o.rp + C::rows + 4;
  return o;
}

struct CompArrays {
  const int4* meta;
  const int *ord, *rp, *cj, *lvb, *uslot, *far_col;
};

// all threads: issue the bulk copies of the chunk [m, me) into buffer b
template <typename T, bool UPPER>
__device__ __forceinline__ void comp_stage_bulk(const CompBuf<T>& b, const ChunkMeta& m, const ChunkMeta& me,
                                                const CompArrays& g, const T* __restrict__ va,
                                                const T* __restrict__ dslot, const T* yslot) {
  stage16(b.va, va + m.nnz0, (me.nnz0 - m.nnz0) * (int)sizeof(T));
  stage16(b.cj, g.cj + m.nnz0, (me.nnz0 - m.nnz0) * 4);
  stage16(b.ord, g.ord + m.row0, (me.row0 - m.row0) * 4);
  stage16(b.rp, g.rp + m.rp0, (me.rp0 - m.rp0) * 4);
  stage16(b.lvb, g.lvb + m.lv0, (me.lv0 - m.lv0) * 4);
  if (UPPER) {
    stage16(b.sd, dslot + m.row0, (me.row0 - m.row0) * (int)sizeof(T));
    stage16(b.sb, yslot + m.row0, (me.row0 - m.row0) * (int)sizeof(T));
  } else {
    stage16(b.sd, g.uslot + m.row0, (me.row0 - m.row0) * 4);  // upper-pass slot of each row (ints in sd)
  }
}

// One CTA per subdomain solves its rows level by level (the schedule of
// IluClass::BuildLevels, ilu.cpp:832-1062, restricted to the subdomain): a
// lower pass y = L^-1 rhs or an upper pass x = D U^-1 y.  Results live in a
// shared-memory ring indexed by schedule position, so a dependency on the
// last `ring` positions is a shared-memory read.  An older ("far") operand
// lies, by construction on the host, before the start of the previous chunk:
// it was published to global memory before that chunk began, so it is
// gathered into the far buffer while the previous chunk is being solved and
// is read from there.  Column indices are encoded as -(index + 1) into the
// ring-plus-far array.
//
// The subdomain's schedule is cut into chunks that fit a staging buffer;
// there are two buffers.  While the CTA sweeps the levels of chunk k (one
// barrier per level), the copies of chunk k+1 are in flight: the bulk
// arrays at once, and, after the first level, the far operands and (lower
// pass) the right-hand side gathered through the row list.  The chunk
// metadata is loaded three chunks ahead.  At a chunk boundary the CTA only
// publishes the chunk's results and waits for its copies.  No CTA waits on
// another: no tickets, no deadlock.
template <typename T, int S, bool UPPER>
__global__ void __launch_bounds__(kCompThreads, kCompMinBlocks) trsv_comp_kernel(
    int n, const int* __restrict__ comp_ch0,  // ncomp+1: chunk range of each subdomain
    CompArrays g, const T* __restrict__ va, const T* __restrict__ dslot, T* yslot, const T* rhs,
    const double* __restrict__ rhs_scale, T* y, T* x, int* err, Skip skip) {
  if (skip.on()) return;
  using C = CompCfg<T>;
  constexpr int RF = C::ring + 2 * C::far;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ring = (T*)smem_raw;  // ring, then far buffer 0, then far buffer 1
  const int tid = threadIdx.x, lane = tid & 31;
  const int c0 = comp_ch0[blockIdx.x], c1 = comp_ch0[blockIdx.x + 1];
  T* out = UPPER ? x : y;  // this pass's result, also the store of far operands
  const double rs = rhs_scale ? *rhs_scale : 1.0;
  if (c0 >= c1) return;
  ChunkMeta m0 = load_meta(g.meta, c0), m1 = load_meta(g.meta, c0 + 1);
  ChunkMeta m2 = c0 + 2 <= c1 ? load_meta(g.meta, c0 + 2) : m1;
  {
    // the first chunk of a subdomain has no far operands
    const CompBuf<T> b = comp_buf<T>(smem_raw, 0);
    comp_stage_bulk<T, UPPER>(b, m0, m1, g, va, dslot, yslot);
    if (!UPPER && tid < m1.row0 - m0.row0) {
      const int r = __ldg(&g.ord[m0.row0 + tid]);
      if (r >= 0) cp_async_elem(&b.sb[tid], &rhs[r]);
    }
    cp_async_wait_all();
    __syncthreads();
  }
  const int sl = tid & (S - 1), group = tid / S, ngroups = kCompThreads / S;
  for (int ch = c0; ch < c1; ch++) {
    const int bi = (ch - c0) & 1;
    const CompBuf<T> nb = comp_buf<T>(smem_raw, bi ^ 1);
    int rhs_row = -1, far_col = -1;
    if (ch + 1 < c1) {
      comp_stage_bulk<T, UPPER>(nb, m1, m2, g, va, dslot, yslot);
      if (!UPPER && tid < m2.row0 - m1.row0) rhs_row = __ldg(&g.ord[m1.row0 + tid]);
      if (tid < m2.far0 - m1.far0) far_col = __ldg(&g.far_col[m1.far0 + tid]);
    }
    const ChunkMeta m3 = ch + 3 <= c1 ? load_meta(g.meta, ch + 3) : m2;
    const CompBuf<T> b = comp_buf<T>(smem_raw, bi);
    const int pos0 = m0.pos0;
    const int nl = m1.lv0 - m0.lv0;
    bool gathered = false;
    int a = b.lvb[0], e = nl > 1 ? b.lvb[1] : a;
    for (int lv = 0; lv + 1 < nl; lv++) {
      if (a >= e) break;  // padding after the last boundary
      const int e_next = lv + 2 < nl ? b.lvb[lv + 2] : e;
      for (int i = a + group; i < e; i += ngroups) {
        const int k1 = b.rp[i], k2 = b.rp[i + 1];
        // up to kUnroll operands per lane with independent loads, then the rest
        T acc = 0;
        int q[kUnroll];
        T v[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
          const int k = k1 + sl + u * S;
          q[u] = k < k2 ? -b.cj[k] - 1 : 0;
          v[u] = k < k2 ? b.va[k] : T(0);
        }
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
          if (k1 + sl + u * S < k2) {  // never read an unwritten ring slot
            acc += v[u] * ring[min((unsigned)q[u], (unsigned)(RF - 1))];
          }
        }
        for (int k = k1 + sl + kUnroll * S; k < k2; k += S) {
          const int qq = -b.cj[k] - 1;
          acc += b.va[k] * ring[min((unsigned)qq, (unsigned)(RF - 1))];
        }
        acc = group_reduce(acc, S, lane);
        if (sl == 0) {
          // only the writing lane reads the row's right-hand side and inverse diagonal
          T o;
          if (UPPER) {
            o = (b.sb[i] - acc) * b.sd[i];
          } else {
            T bb = b.sb[i];
            if (rhs_scale) bb = (T)((double)bb * rs);
            o = bb - acc;
          }
          ring[(pos0 + i) & (C::ring - 1)] = o;
        }
      }
      __syncthreads();
      if (!gathered) {
        // the next chunk's gathers, once the loads of their indices had a level to land
        gathered = true;
        if (rhs_row >= 0) cp_async_elem(&nb.sb[tid], &rhs[rhs_row]);
        if (far_col >= 0) {
          if ((unsigned)far_col < (unsigned)n)
            cp_async_elem(&ring[C::ring + (bi ^ 1) * C::far + tid], &out[far_col]);
          else
            atomicOr(err, kErrIndex);
        }
      }
      a = e;
      e = e_next;
    }
    if (!gathered) {
      if (rhs_row >= 0) cp_async_elem(&nb.sb[tid], &rhs[rhs_row]);
      if (far_col >= 0 && (unsigned)far_col < (unsigned)n)
        cp_async_elem(&ring[C::ring + (bi ^ 1) * C::far + tid], &out[far_col]);
    }
    // publish the chunk's results from the ring: natural order (far operands
    // and the consumer) and, for the lower pass, the upper pass's slot order
    for (int i = tid; i < m1.row0 - m0.row0; i += blockDim.x) {
      const int r = b.ord[i];
      if (r < 0) continue;
      const T o = ring[(pos0 + i) & (C::ring - 1)];
      out[r] = o;
      if (!UPPER) yslot[((const int*)b.sd)[i]] = o;
    }
    if (ch + 1 < c1) {
      cp_async_wait_all();
      __syncthreads();
    }
    m0 = m1;
    m1 = m2;
    m2 = m3;
  }
}

// --------------------- per-subdomain triangular solve, several right-hand sides
// trsv_comp_batch_kernel: trsv_comp_kernel for R right-hand sides at once.
// The factor's rows, columns and values are staged and read once per chunk
// and applied to all R vectors; the ring holds R values per schedule
// position (one vector load per operand).  Shared-memory sizes shrink with R
// (CompCfgR), so the layout is built for the R it serves.
template <typename T, int R>
struct __align__(sizeof(T) * R <= 16 ? sizeof(T) * R : 16) VecR {
  T v[R];
};
template <typename T, int R>
struct PtrR {
  T* p[R];
};
template <typename T, int R>
struct CompCfgR {
  static constexpr bool d = sizeof(T) == 8;
  static constexpr int ring = R <= 1 ? CompCfg<T>::ring : (d ? (R == 2 ? 4096 : 2048) : (R == 2 ? 8192 : 4096));
  static constexpr int far = R <= 1 ? CompCfg<T>::far : (d ? (R == 2 ? 512 : 256) : (R == 2 ? 1024 : 512));
  static constexpr int nnz = R <= 1 ? CompCfg<T>::nnz : (d ? (R == 2 ? 3072 : 2048) : (R == 2 ? 5632 : 4096));
  static constexpr int rows = R <= 1 ? CompCfg<T>::rows : (d ? (R == 2 ? 768 : 512) : (R == 2 ? 1024 : 768));
  // per buffer: va[nnz] T | sb[R][rows] T | sd[rows] T | cj[nnz] int | ord[rows] int | rp[rows+4] int | lvb[rows+4] int
  static constexpr size_t buf_bytes =
      sizeof(T) * (size_t)(nnz + (R + 1) * rows) + sizeof(int) * (size_t)(nnz + rows + 2 * (rows + 4));
  static constexpr size_t bytes = sizeof(T) * R * (size_t)(ring + 2 * far) + 2 * buf_bytes;
  static_assert(bytes <= 227 * 1024, "batched per-subdomain solve exceeds the shared memory of one CTA");
  static_assert(far <= kCompThreads && rows <= kCompThreads, "one gather per thread");
};

template <typename T, int R>
struct CompBufR {
  T *va, *sb, *sd;  // sb: R arrays of `rows`
  int *cj, *ord, *rp, *lvb;
};
template <typename T, int R, typename C = CompCfgR<T, R>>
__device__ __forceinline__ CompBufR<T, R> comp_buf_r(unsigned char* base, int which) {
  unsigned char* b = base + sizeof(T) * R * (size_t)(C::ring + 2 * C::far) + (size_t)which * C::buf_bytes;
  CompBufR<T, R> o;
  o.va = (T*)b;
  o.sb = o.va + C::nnz;
  o.sd = o.sb + R * C::rows;
  o.cj = (int*)(o.sd + C::rows);
  o.ord = o.cj + C::nnz;
  o.rp = o.ord + C::rows;
  o.lvb = o.rp + C::rows + 4;
  return o;
}

template <typename T, int R, bool UPPER, typename C = CompCfgR<T, R>>
__device__ __forceinline__ void comp_stage_bulk_r(const CompBufR<T, R>& b, const ChunkMeta& m, const ChunkMeta& me,
                                                  const CompArrays& g, const T* __restrict__ va,
                                                  const T* __restrict__ dslot, const PtrR<T, R>& yslot) {
  stage16(b.va, va + m.nnz0, (me.nnz0 - m.nnz0) * (int)sizeof(T));
  stage16(b.cj, g.cj + m.nnz0, (me.nnz0 - m.nnz0) * 4);
  stage16(b.ord, g.ord + m.row0, (me.row0 - m.row0) * 4);
  stage16(b.rp, g.rp + m.rp0, (me.rp0 - m.rp0) * 4);
  stage16(b.lvb, g.lvb + m.lv0, (me.lv0 - m.lv0) * 4);
  if (UPPER) {
    stage16(b.sd, dslot + m.row0, (me.row0 - m.row0) * (int)sizeof(T));
#pragma unroll
    for (int r = 0; r < R; r++) stage16(b.sb + r * C::rows, yslot.p[r] + m.row0, (me.row0 - m.row0) * (int)sizeof(T));
  } else {
    stage16(b.sd, g.uslot + m.row0, (me.row0 - m.row0) * 4);
  }
}

template <typename T, int S, bool UPPER, int R, typename C = CompCfgR<T, R>>
__global__ void __launch_bounds__(kCompThreads, kCompMinBlocks) trsv_comp_batch_kernel(
    int n, const int* __restrict__ comp_ch0, CompArrays g, const T* __restrict__ va, const T* __restrict__ dslot,
    PtrR<T, R> yslot, PtrR<T, R> rhs, PtrR<T, R> y, PtrR<T, R> x, int* err, SkipR<R> skip) {
  if (skip.on()) return;
  using V = VecR<T, R>;
  constexpr int RF = C::ring + 2 * C::far;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* ring = (V*)smem_raw;  // ring, then far buffer 0, then far buffer 1
  const int tid = threadIdx.x, lane = tid & 31;
  const int c0 = comp_ch0[blockIdx.x], c1 = comp_ch0[blockIdx.x + 1];
  const PtrR<T, R> out = UPPER ? x : y;
  if (c0 >= c1) return;
  ChunkMeta m0 = load_meta(g.meta, c0), m1 = load_meta(g.meta, c0 + 1);
  ChunkMeta m2 = c0 + 2 <= c1 ? load_meta(g.meta, c0 + 2) : m1;
  {
    const CompBufR<T, R> b = comp_buf_r<T, R, C>(smem_raw, 0);
    comp_stage_bulk_r<T, R, UPPER, C>(b, m0, m1, g, va, dslot, yslot);
    if (!UPPER && tid < m1.row0 - m0.row0) {
      const int rr = __ldg(&g.ord[m0.row0 + tid]);
      if (rr >= 0) {
#pragma unroll
        for (int r = 0; r < R; r++) cp_async_elem(&b.sb[r * C::rows + tid], &rhs.p[r][rr]);
      }
    }
    cp_async_wait_all();
    __syncthreads();
  }
  const int sl = tid & (S - 1), group = tid / S, ngroups = kCompThreads / S;
  for (int ch = c0; ch < c1; ch++) {
    const int bi = (ch - c0) & 1;
    const CompBufR<T, R> nb = comp_buf_r<T, R, C>(smem_raw, bi ^ 1);
    int rhs_row = -1, far_col = -1;
    if (ch + 1 < c1) {
      comp_stage_bulk_r<T, R, UPPER, C>(nb, m1, m2, g, va, dslot, yslot);
      if (!UPPER && tid < m2.row0 - m1.row0) rhs_row = __ldg(&g.ord[m1.row0 + tid]);
      if (tid < m2.far0 - m1.far0) far_col = __ldg(&g.far_col[m1.far0 + tid]);
    }
    const ChunkMeta m3 = ch + 3 <= c1 ? load_meta(g.meta, ch + 3) : m2;
    const CompBufR<T, R> b = comp_buf_r<T, R, C>(smem_raw, bi);
    const int pos0 = m0.pos0;
    const int nl = m1.lv0 - m0.lv0;
    bool gathered = false;
    int a = b.lvb[0], e = nl > 1 ? b.lvb[1] : a;
    for (int lv = 0; lv + 1 < nl; lv++) {
      if (a >= e) break;
      const int e_next = lv + 2 < nl ? b.lvb[lv + 2] : e;
      for (int i = a + group; i < e; i += ngroups) {
        const int k1 = b.rp[i], k2 = b.rp[i + 1];
        T acc[R];
#pragma unroll
        for (int r = 0; r < R; r++) acc[r] = 0;
        int q[kUnroll];
        T v[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
          const int k = k1 + sl + u * S;
          q[u] = k < k2 ? -b.cj[k] - 1 : 0;
          v[u] = k < k2 ? b.va[k] : T(0);
        }
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
          if (k1 + sl + u * S < k2) {
            const V w = ring[min((unsigned)q[u], (unsigned)(RF - 1))];
#pragma unroll
            for (int r = 0; r < R; r++) acc[r] += v[u] * w.v[r];
          }
        }
        for (int k = k1 + sl + kUnroll * S; k < k2; k += S) {
          const int qq = -b.cj[k] - 1;
          const V w = ring[min((unsigned)qq, (unsigned)(RF - 1))];
          const T vv = b.va[k];
#pragma unroll
          for (int r = 0; r < R; r++) acc[r] += vv * w.v[r];
        }
        // sum over the group's lanes for every lane value: reduce-scatter
        // first (each step halves the values a lane carries), then a
        // butterfly on one value.  Every partial sum adds the same two
        // operands as group_reduce does, so the results are identical.
        const unsigned gmask = S == 32 ? 0xffffffffu : (((1u << S) - 1u) << (lane & ~(S - 1)));
        if (R == 4 && S >= 4) {
          const bool hb = (sl & (S >> 1)) != 0, qb = (sl & (S >> 2)) != 0;
          T k0 = hb ? acc[2] : acc[0], k1 = hb ? acc[3] : acc[1];
          const T s0 = hb ? acc[0] : acc[2], s1 = hb ? acc[1] : acc[3];
          k0 += __shfl_xor_sync(gmask, s0, S >> 1);
          k1 += __shfl_xor_sync(gmask, s1, S >> 1);
          T kk = qb ? k1 : k0;
          kk += __shfl_xor_sync(gmask, qb ? k0 : k1, S >> 2);
#pragma unroll
          for (int off = S >> 3; off > 0; off >>= 1) kk += __shfl_xor_sync(gmask, kk, off);
          if ((sl & ((S >> 2) - 1)) == 0) {
            const int r = (hb ? 2 : 0) + (qb ? 1 : 0);
            const T bb = b.sb[r * C::rows + i];
            ring[(pos0 + i) & (C::ring - 1)].v[r] = UPPER ? (bb - kk) * b.sd[i] : bb - kk;
          }
        } else if (R == 2 && S >= 2) {
          const bool hb = (sl & (S >> 1)) != 0;
          T kk = hb ? acc[1] : acc[0];
          kk += __shfl_xor_sync(gmask, hb ? acc[0] : acc[1], S >> 1);
#pragma unroll
          for (int off = S >> 2; off > 0; off >>= 1) kk += __shfl_xor_sync(gmask, kk, off);
          if ((sl & ((S >> 1) - 1)) == 0) {
            const int r = hb ? 1 : 0;
            const T bb = b.sb[r * C::rows + i];
            ring[(pos0 + i) & (C::ring - 1)].v[r] = UPPER ? (bb - kk) * b.sd[i] : bb - kk;
          }
        } else {
#pragma unroll
          for (int r = 0; r < R; r++) acc[r] = group_reduce(acc[r], S, lane);
          if (sl == 0) {
            V o;
            const T di_ = UPPER ? b.sd[i] : T(0);
#pragma unroll
            for (int r = 0; r < R; r++) {
              const T bb = b.sb[r * C::rows + i];
              o.v[r] = UPPER ? (bb - acc[r]) * di_ : bb - acc[r];
            }
            ring[(pos0 + i) & (C::ring - 1)] = o;
          }
        }
      }
      __syncthreads();
      if (!gathered) {
        gathered = true;
        if (rhs_row >= 0) {
#pragma unroll
          for (int r = 0; r < R; r++) cp_async_elem(&nb.sb[r * C::rows + tid], &rhs.p[r][rhs_row]);
        }
        if (far_col >= 0) {
          if ((unsigned)far_col < (unsigned)n) {
            V* fv = &ring[C::ring + (bi ^ 1) * C::far + tid];
#pragma unroll
            for (int r = 0; r < R; r++) cp_async_elem(&fv->v[r], &out.p[r][far_col]);
          } else {
            atomicOr(err, kErrIndex);
          }
        }
      }
      a = e;
      e = e_next;
    }
    if (!gathered) {
      if (rhs_row >= 0) {
#pragma unroll
        for (int r = 0; r < R; r++) cp_async_elem(&nb.sb[r * C::rows + tid], &rhs.p[r][rhs_row]);
      }
      if (far_col >= 0 && (unsigned)far_col < (unsigned)n) {
        V* fv = &ring[C::ring + (bi ^ 1) * C::far + tid];
#pragma unroll
        for (int r = 0; r < R; r++) cp_async_elem(&fv->v[r], &out.p[r][far_col]);
      }
    }
    for (int i = tid; i < m1.row0 - m0.row0; i += blockDim.x) {
      const int rr = b.ord[i];
      if (rr < 0) continue;
      const V o = ring[(pos0 + i) & (C::ring - 1)];
#pragma unroll
      for (int r = 0; r < R; r++) {
        out.p[r][rr] = o.v[r];
        if (!UPPER) yslot.p[r][((const int*)b.sd)[i]] = o.v[r];
      }
    }
    if (ch + 1 < c1) {
      cp_async_wait_all();
      __syncthreads();
    }
    m0 = m1;
    m1 = m2;
    m2 = m3;
  }
}

// ------------------------------------------------- tall-skinny kernels
// One kernel family covers every operation on a block of dense columns:
// the Gram-Schmidt passes of the Arnoldi step (PargemslrMgs / PargemslrCgs2,
// ParGeMSLR SRC/matrices/matrixops.cpp:10588-10806), the Woodbury low-rank
// correction W^T x then WH y (GemslrClass::SolveApplyLowRankLevel,
// gemslr.cpp:3681-3722) and the solution update x += Z y (fgmres.hpp:483-490).
//
//   TS_DOT          sums[c] = V(:,c) . w,            w = in * in_scale
//   TS_UPDATE       out = in * in_scale + sign * M coef'
//   TS_UPDATE_DOT   out = w' = (update above); sums[c] = V(:,c) . w'
//   TS_UPDATE_NORM  out = w' = (update above); sums[0] = w' . w'
//   TS_NORM_COPY    sums[0] = w . w; out = w (if out)
// with coef'[c] = coef[c] * msc[c] and msc the lazy column scales of M.
// Columns are column-major with leading dimension ld.  Each block walks
// 512-row tiles; per tile, thread t updates row t, then warp w reduces the
// columns c = w mod 16 over the tile (the tile is re-read from L1/L2, so DRAM
// sees each column once).  Block partials are combined by the last block to
// finish, in a fixed order, so results do not depend on block scheduling;
// that block then runs the epilogue (storing coefficients, or the Givens
// update of the Hessenberg column).
enum TsMode { TS_DOT = 0, TS_UPDATE = 1, TS_UPDATE_DOT = 2, TS_UPDATE_NORM = 3, TS_NORM_COPY = 4 };
enum EpiKind {
  EPI_NONE = 0,
  EPI_STORE = 1,       // dst[c] = sums[c] * vsc[c]
  EPI_CGS_FIRST = 2,   // hcol = coefA = sums * vsc
  EPI_CGS_SECOND = 3,  // coefB = sums * vsc; hcol += coefB
  EPI_GIVENS = 4,      // finish column j: norm, rotations, convergence, back-solve
  EPI_NORMB = 5,       // st->normb = sqrt(sums[0])
  EPI_INIT = 6,        // outer start of solve: normr, tolr, rs[0], sc[0]
  EPI_INIT_INNER = 7,  // inner solve from x0 = 0: normb = normr = ||rhs||
};

template <typename TV, typename TM, typename TW>
struct TsArgs {
  int n;
  int ncols;
  const int* ncols_dev;  // if set, the column count is read here (<= KMAX)
  const TV* V;
  long long ldv;
  const double* vsc;
  const TM* M;
  long long ldm;
  const double* msc;
  const double* coef;
  double sign;
  const TW* in;          // null: zero input
  const double* in_scale;
  TW* out;
  double* partial;       // [KMAX+1][gridDim.x]
  unsigned int* counter; // zero between launches
  int epi;
  FgmresDev* st;
  double* dst;
  int j;
  Skip skip;
};

__device__ inline void fgmres_givens(FgmresDev* st, int j, double t) {
  // H(:, j) from the Gram-Schmidt coefficients and ||w||
  // (PargemslrMgs sets H(0..k, k) and H(k+1, k), matrixops.cpp:10728-10806)
  const int ldh = KMAX + 1;
  double* H = st->H + (size_t)j * ldh;
  for (int c = 0; c <= j; c++) H[c] = st->hcol[c];
  H[j + 1] = t;
  st->sc[j + 1] = 1.0 / t;
  st->iter += 1;
  st->i = j + 1;
  // apply the previous rotations, then form the new one (fgmres.hpp:430-458)
  for (int k = 1; k <= j; k++) {
    double hii = H[k - 1];
    H[k - 1] = st->c[k - 1] * hii + st->s[k - 1] * H[k];
    H[k] = -st->s[k - 1] * hii + st->c[k - 1] * H[k];
  }
  double hii = H[j], hii1 = H[j + 1];
  double gam = sqrt(fabs(hii) * fabs(hii) + fabs(hii1) * fabs(hii1));
  if (fabs(gam) < st->eps) {
    // breakdown: the reference jumps past the solution update (fgmres.hpp:440-443)
    st->breakdown = 1;
    st->i = 0;
    st->cycle_done = 1;
    st->done = 1;
    return;
  }
  st->c[j] = hii / gam;
  st->s[j] = hii1 / gam;
  st->rs[j + 1] = -st->s[j] * st->rs[j];
  st->rs[j] = st->c[j] * st->rs[j];
  H[j] = st->c[j] * hii + st->s[j] * hii1;
  st->normr = fabs(st->rs[j + 1]);
  const bool conv = st->normr <= st->tolr;
  if (conv) st->converged = 1;
  if (conv || st->i >= st->kdim || st->iter >= st->maxits) {
    st->cycle_done = 1;
    if (conv || st->iter >= st->maxits) st->done = 1;
    // back substitution H y = rs, in place in rs (fgmres.hpp:471-480)
    const int i = st->i;
    double* rs = st->rs;
    rs[i - 1] /= st->H[(size_t)(i - 1) * ldh + (i - 1)];
    for (int k = i - 2; k >= 0; k--) {
      for (int jj = k + 1; jj < i; jj++) rs[k] -= st->H[(size_t)jj * ldh + k] * rs[jj];
      rs[k] /= st->H[(size_t)k * ldh + k];
    }
  }
}

template <typename TV, typename TM, typename TW>
__device__ inline void ts_epilogue(const TsArgs<TV, TM, TW>& a, const double* sums, int ncols) {
  FgmresDev* st = a.st;
  switch (a.epi) {
    case EPI_STORE:
      for (int c = 0; c < ncols; c++) a.dst[c] = sums[c] * (a.vsc ? a.vsc[c] : 1.0);
      break;
    case EPI_CGS_FIRST:
      for (int c = 0; c < ncols; c++) {
        double h = sums[c] * (a.vsc ? a.vsc[c] : 1.0);
        st->hcol[c] = h;
        st->coefA[c] = h;
      }
      break;
    case EPI_CGS_SECOND:
      for (int c = 0; c < ncols; c++) {
        double h = sums[c] * (a.vsc ? a.vsc[c] : 1.0);
        st->hcol[c] += h;
        st->coefB[c] = h;
      }
      break;
    case EPI_GIVENS:
      fgmres_givens(st, a.j, sqrt(sums[0]));
      break;
    case EPI_NORMB:
      st->normb = sqrt(sums[0]);
      if (st->normb < st->eps) {
        st->done = 1;
        st->cycle_done = 1;
        st->normr = 0.0;
        st->i = 0;
      }
      break;
    case EPI_INIT: {
      st->i = 0;
      st->iter = 0;
      st->converged = 0;
      st->breakdown = 0;
      if (st->done) break;  // zero right-hand side
      const double normr = sqrt(sums[0]);
      st->normr = normr;
      if (normr < st->eps) {
        st->done = 1;
        st->cycle_done = 1;
        st->converged = 1;
        break;
      }
      st->tolr = st->absolute ? st->tol : st->tol * st->normb;
      st->rs[0] = normr;
      st->sc[0] = 1.0 / normr;
      st->cycle_done = 0;
      break;
    }
    case EPI_INIT_INNER: {
      const double normb = sqrt(sums[0]);
      st->normb = normb;
      st->normr = normb;
      st->i = 0;
      st->iter = 0;
      st->converged = 0;
      st->breakdown = 0;
      st->done = 0;
      st->cycle_done = 0;
      if (normb < st->eps) {
        st->done = 1;
        st->cycle_done = 1;
        break;
      }
      st->tolr = st->absolute ? st->tol : st->tol * normb;
      st->rs[0] = normb;
      st->sc[0] = 1.0 / normb;
      break;
    }
    default:
      break;
  }
}

template <typename TV, typename TM, typename TW, int MODE>
__global__ void __launch_bounds__(kTsThreads) ts_kernel(TsArgs<TV, TM, TW> a) {
  if (a.skip.on()) return;
  __shared__ double scoef[KMAX + 1];
  __shared__ double sacc[KMAX + 1];
  __shared__ double swarp[kTsThreads / 32];
  __shared__ int s_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = kTsThreads / 32;
  const int ncols = a.ncols_dev ? min(*(const volatile int*)a.ncols_dev, KMAX + 1) : a.ncols;
  const bool update = MODE == TS_UPDATE || MODE == TS_UPDATE_DOT || MODE == TS_UPDATE_NORM;
  const bool reduce = MODE != TS_UPDATE;
  const int nred = (MODE == TS_DOT || MODE == TS_UPDATE_DOT) ? ncols : 1;
  if (MODE == TS_UPDATE && ncols == 0 && a.in == a.out) return;  // nothing to add
  const double in_s = a.in_scale ? *a.in_scale : 1.0;
  for (int c = tid; c <= KMAX; c += kTsThreads) {
    scoef[c] = (update && c < ncols) ? a.sign * a.coef[c] * (a.msc ? a.msc[c] : 1.0) : 0.0;
    sacc[c] = 0.0;
  }
  if (tid < NW) swarp[tid] = 0.0;
  __syncthreads();
  const int ntiles = (a.n + kTsThreads - 1) / kTsThreads;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * kTsThreads;
    const int row = r0 + tid;
    double wv = 0.0;
    if (row < a.n) {
      wv = a.in ? (double)a.in[row] * in_s : 0.0;
      if (update) {
        double acc = 0.0;
        const TM* m = a.M + row;
        for (int c = 0; c < ncols; c++) acc += (double)m[(long long)c * a.ldm] * scoef[c];
        wv += acc;
      }
      if (MODE != TS_DOT && a.out) a.out[row] = (TW)wv;
    }
    if (MODE == TS_UPDATE_NORM || MODE == TS_NORM_COPY) {
      double sq = (row < a.n) ? wv * wv : 0.0;
      if (MODE == TS_UPDATE_NORM) {
        // the norm of the stored (rounded) vector, as Norm2 of the reference
        TW stored = (TW)wv;
        sq = (row < a.n) ? (double)stored * (double)stored : 0.0;
      }
      sq = warp_reduce(sq);
      if (lane == 0) swarp[warp] += sq;  // one writer per slot: deterministic
    }
    if (MODE == TS_DOT || MODE == TS_UPDATE_DOT) {
      __syncthreads();  // out[] of this tile written by the whole block
      const int nrows_tile = min(kTsThreads, a.n - r0);
      for (int c = warp; c < ncols; c += NW) {
        const TV* v = a.V + (long long)c * a.ldv + r0;
        double acc = 0.0;
        for (int k = lane; k < nrows_tile; k += 32) {
          double w = (MODE == TS_DOT) ? (a.in ? (double)a.in[r0 + k] * in_s : 0.0)
                                      : (double)a.out[r0 + k];
          acc += (double)v[k] * w;
        }
        acc = warp_reduce(acc);
        if (lane == 0) sacc[c] += acc;
      }
      __syncthreads();
    }
  }
  if (!reduce) return;
  __syncthreads();
  if ((MODE == TS_UPDATE_NORM || MODE == TS_NORM_COPY) && tid == 0) {
    double t = 0.0;
    for (int w = 0; w < NW; w++) t += swarp[w];
    sacc[0] = t;
  }
  __syncthreads();
  // block partials -> global, column-major by block
  for (int c = tid; c < nred; c += kTsThreads) a.partial[(long long)c * gridDim.x + blockIdx.x] = sacc[c];
  __threadfence();
  __syncthreads();
  if (tid == 0) {
    unsigned int prev = atomicAdd(a.counter, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int c = warp; c < nred; c += NW) {
    double acc = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32) acc += __ldcg(&a.partial[(long long)c * gridDim.x + b]);
    acc = warp_reduce(acc);
    if (lane == 0) sacc[c] = acc;
  }
  __syncthreads();
  if (tid == 0) {
    ts_epilogue(a, sacc, nred);
    *a.counter = 0u;
    __threadfence();
  }
}

__global__ void fgmres_cycle_reset_kernel(FgmresDev* st, Skip skip) {
  if (skip.on()) return;
  st->i = 0;
  if (st->done) return;
  st->cycle_done = 0;
  st->rs[0] = st->normr;
  st->sc[0] = 1.0 / st->normr;
}

// --------------------------------------------------- permutation + convert
// out[i] = (TO)(in[perm[i]] * scale)  (IntVectorClass::GatherPerm, int_vector.cpp:668)
template <typename TI, typename TO>
__global__ void gather_kernel(int n, const int* __restrict__ perm, const TI* __restrict__ in,
                              const double* __restrict__ scale, TO* __restrict__ out, Skip skip) {
  if (skip.on()) return;
  const double s = scale ? *scale : 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int p = perm ? perm[i] : i;
    out[i] = scale ? (TO)((double)in[p] * s) : (TO)in[p];
  }
}

// out[perm[i]] = in[i]  (IntVectorClass::ScatterRperm, int_vector.cpp:629)
template <typename TI, typename TO>
__global__ void scatter_kernel(int n, const int* __restrict__ perm, const TI* __restrict__ in,
                               TO* __restrict__ out, Skip skip) {
  if (skip.on()) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int p = perm ? perm[i] : i;
    out[p] = (TO)in[i];
  }
}

template <typename T>
__global__ void fill_kernel(int n, T v, T* out, Skip skip) {
  if (skip.on()) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = v;
}

}  // namespace pgx
