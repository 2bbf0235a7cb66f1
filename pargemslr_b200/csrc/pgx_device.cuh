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

#include "pgx_complex.cuh"

namespace pgx {

using ::__shfl_xor_sync;  // the real forms beside the complex overload

constexpr int kWarp = 32;
constexpr int KMAX = 128;          // largest Krylov dimension a handle accepts
constexpr int kTsThreads = 512;    // block size of the tall-skinny kernels
constexpr int kTsMaxBlocks = 296;  // 2 blocks per SM on a 148-SM B200
constexpr int kSpinLimit = 1 << 21;  // default bound of the waits in the sync-free triangular solves

// status bits written by kernels into the handle's error word
constexpr int kErrTimeout = 1;  // a dependency wait of a cross-subdomain triangular solve gave up
constexpr int kErrIndex = 2;    // an index check failed
constexpr int kErrStage = 4;    // a staging wait of the per-subdomain triangular solve gave up

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
// S is the solver's scalar: double, or cf64 for a complex solve (Hessenberg,
// rotations and right-hand side of the least-squares problem complex; norms,
// tolerances and the lazy column scales real).  The header up to sc has the
// same layout for both.
template <typename S>
struct FgmresDevT {
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
  double normr0;   // ||r0|| at the start of the solve (first entry of the residual history)
  double eps;      // numeric_limits<RealDataType>::epsilon() of the solver
  int absolute;
  int pad;
  double sc[KMAX + 1];     // V(:,c) = Vstored(:,c) * sc[c] (lazy normalisation)
  double hist[KMAX];       // Givens estimate after each column of the current cycle (0 at a breakdown)
  S hcol[KMAX + 1];   // column of H being built
  S coefA[KMAX + 1];  // first Gram-Schmidt coefficients
  S coefB[KMAX + 1];  // re-orthogonalisation coefficients
  S c[KMAX], s[KMAX], rs[KMAX + 1], y[KMAX];
  S H[(KMAX + 1) * KMAX];
};
using FgmresDev = FgmresDevT<double>;

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }
template <>
__device__ __forceinline__ cf32 ldg<cf32>(const cf32* p) {
  const float2 v = __ldg((const float2*)p);
  return cf32(v.x, v.y);
}
template <>
__device__ __forceinline__ cf64 ldg<cf64>(const cf64* p) {
  const double2 v = __ldg((const double2*)p);
  return cf64(v.x, v.y);
}
template <typename T>
__device__ __forceinline__ T ldcg(const T* p) { return __ldcg(p); }
template <>
__device__ __forceinline__ cf32 ldcg<cf32>(const cf32* p) {
  const float2 v = __ldcg((const float2*)p);
  return cf32(v.x, v.y);
}
template <>
__device__ __forceinline__ cf64 ldcg<cf64>(const cf64* p) {
  const double2 v = __ldcg((const double2*)p);
  return cf64(v.x, v.y);
}

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
// Each lane issues the loads of its first kSpmvUnroll column indices, then
// of the x entries they name, before it multiplies: the gathers of x are in
// flight together.  A lane sums its entries in increasing order either way.
constexpr int kSpmvUnroll = 4;

template <typename TA, typename TX, typename TC, int S>
__device__ __forceinline__ TC row_dot(int k1, int k2, int lane, const int* __restrict__ cj, const TA* __restrict__ va,
                                      const TX* __restrict__ x, int xcols, bool& bad) {
  int c[kSpmvUnroll];
  TA v[kSpmvUnroll];
#pragma unroll
  for (int u = 0; u < kSpmvUnroll; u++) {
    const int k = k1 + lane + u * S;
    c[u] = k < k2 ? __ldg(&cj[k]) : -1;
    v[u] = k < k2 ? ldg(&va[k]) : TA(0);
    if (k < k2 && (unsigned)c[u] >= (unsigned)xcols) {
      bad = true;  // a column outside x: the entry is skipped
      c[u] = -1;
    }
  }
  TX xv[kSpmvUnroll];
#pragma unroll
  for (int u = 0; u < kSpmvUnroll; u++) xv[u] = c[u] >= 0 ? x[c[u]] : TX(0);
  TC acc = 0;
#pragma unroll
  for (int u = 0; u < kSpmvUnroll; u++)
    if (c[u] >= 0) acc += (TC)v[u] * (TC)xv[u];
  for (int k = k1 + lane + kSpmvUnroll * S; k < k2; k += S) {
    const int cc = __ldg(&cj[k]);
    if ((unsigned)cc < (unsigned)xcols)
      acc += (TC)ldg(&va[k]) * (TC)x[cc];
    else
      bad = true;
  }
  return acc;
}

// The same dot product with 128-bit loads: the row's entries [k1, k2) lie in
// the aligned 4-entry blocks k1/4 .. (k2+3)/4 - 1; the S lanes take the
// blocks in turn, each loading a block's column indices as one int4 and its
// values as one float4 or two double2, and mask the entries outside the row.
// Needs cj and va 16-byte aligned and padded to a whole last block (the
// library's own uploads are).  A lane sums its entries in increasing order.
template <typename TA>
__device__ __forceinline__ void load_block4(const TA* __restrict__ p, TA* v);
template <>
__device__ __forceinline__ void load_block4<float>(const float* __restrict__ p, float* v) {
  const float4 a = __ldg((const float4*)p);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = a.z;
  v[3] = a.w;
}
template <>
__device__ __forceinline__ void load_block4<double>(const double* __restrict__ p, double* v) {
  const double2 a = __ldg((const double2*)p), b = __ldg((const double2*)p + 1);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}

template <>
__device__ __forceinline__ void load_block4<cf32>(const cf32* __restrict__ p, cf32* v) {
  const float4 a = __ldg((const float4*)p), b = __ldg((const float4*)p + 1);
  v[0] = cf32(a.x, a.y);
  v[1] = cf32(a.z, a.w);
  v[2] = cf32(b.x, b.y);
  v[3] = cf32(b.z, b.w);
}
template <>
__device__ __forceinline__ void load_block4<cf64>(const cf64* __restrict__ p, cf64* v) {
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const double2 a = __ldg((const double2*)p + u);
    v[u] = cf64(a.x, a.y);
  }
}

template <typename TA, typename TX, typename TC, int S>
__device__ __forceinline__ TC row_dot_vec(int k1, int k2, int lane, const int* __restrict__ cj,
                                          const TA* __restrict__ va, const TX* __restrict__ x, int xcols, bool& bad) {
  TC acc = 0;
  const int b1 = (k2 + 3) >> 2;
  for (int bb = (k1 >> 2) + lane; bb < b1; bb += S) {
    const int kb = bb << 2;
    const int4 c4 = __ldg((const int4*)cj + bb);
    TA v[4];
    load_block4<TA>(va + kb, v);
    const int c[4] = {c4.x, c4.y, c4.z, c4.w};
    bool in[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      in[u] = kb + u >= k1 && kb + u < k2;
      if (in[u] && (unsigned)c[u] >= (unsigned)xcols) {
        bad = true;  // a column outside x: the entry is skipped
        in[u] = false;
      }
    }
    TX xv[4];
#pragma unroll
    for (int u = 0; u < 4; u++) xv[u] = in[u] ? x[c[u]] : TX(0);
#pragma unroll
    for (int u = 0; u < 4; u++)
      if (in[u]) acc += (TC)v[u] * (TC)xv[u];
  }
  return acc;
}

template <typename TA, typename TX, typename TY, typename TC, int S, bool VEC>
__global__ void __launch_bounds__(256) spmv_kernel(
    int nrows, const int* __restrict__ rp1, const int* __restrict__ cj1, const TA* __restrict__ va1,
    const TX* __restrict__ x1, int xcols1, TC alpha, const int* __restrict__ rp2, const int* __restrict__ cj2,
    const TA* __restrict__ va2, const TX* __restrict__ x2, int xcols2, TC alpha2, const TY* b, TC beta, TY* y,
    const double* __restrict__ xscale, int* err, Skip skip) {
  if (skip.on()) return;
  const int lane = threadIdx.x & (S - 1);
  const int wlane = threadIdx.x & 31;
  const int groups_per_block = blockDim.x / S;
  const TC xs = xscale ? (TC)(*xscale) : (TC)1;
  bool bad = false;
  for (int row = blockIdx.x * groups_per_block + threadIdx.x / S; row < nrows;
       row += gridDim.x * groups_per_block) {
    const int k1 = __ldg(&rp1[row]), k2 = __ldg(&rp1[row + 1]);
    TC acc = VEC ? row_dot_vec<TA, TX, TC, S>(k1, k2, lane, cj1, va1, x1, xcols1, bad)
                 : row_dot<TA, TX, TC, S>(k1, k2, lane, cj1, va1, x1, xcols1, bad);
    acc = group_reduce(acc, S, wlane);
    TC acc2 = 0;
    if (rp2) {
      const int q1 = __ldg(&rp2[row]), q2 = __ldg(&rp2[row + 1]);
      acc2 = VEC ? row_dot_vec<TA, TX, TC, S>(q1, q2, lane, cj2, va2, x2, xcols2, bad)
                 : row_dot<TA, TX, TC, S>(q1, q2, lane, cj2, va2, x2, xcols2, bad);
      acc2 = group_reduce(acc2, S, wlane);
    }
    if (lane == 0) {
      TC v = alpha * (acc * xs);
      if (rp2) v += alpha2 * acc2;
      if (b) v += beta * (TC)b[row];
      y[row] = (TY)v;
    }
  }
  if (bad && err) atomicOr(err, kErrIndex);
}

// ---------------------------------------------------- merge-path CSR SpMV
// For matrices whose row lengths are skewed (a few very long rows among
// short ones), the row-per-group kernel leaves most lanes idle on the short
// rows and serialises the long ones.  The merge-path SpMV (Merrill and
// Garland, "Merge-based parallel sparse matrix-vector multiplication", SC16)
// gives every thread the same number of merge items, where the items are
// the n row ends and the nnz nonzeros taken in merge order (a nonzero k of
// row r comes before the end of row r).  A thread finds its start on the
// merge path by a binary search on its diagonal, then consumes its items:
// rows that end in its range are written at once; the partial sum of the
// row it stops inside is its carry, added by merge_spmv_fixup_kernel.
// y = alpha * A x + beta * b (b may be absent or alias y).
constexpr int kMergeItems = 16;  // merge items per thread

__device__ __forceinline__ void merge_path_search(int diag, const int* __restrict__ rp, int nrows, int nnz, int* row,
                                                  int* k) {
  // the number of row ends among the first `diag` merge items: the largest i
  // with rp[i] (the end of row i-1) <= diag - i
  int lo = max(diag - nnz, 0), hi = min(diag, nrows);
  while (lo < hi) {
    const int pivot = (lo + hi) >> 1;
    if (__ldg(&rp[pivot + 1]) <= diag - pivot - 1)
      lo = pivot + 1;
    else
      hi = pivot;
  }
  *row = min(lo, nrows);
  *k = diag - *row;
}

template <typename TA, typename TX, typename TY, typename TC>
__global__ void __launch_bounds__(256) merge_spmv_kernel(
    int nrows, int nnz, const int* __restrict__ rp, const int* __restrict__ cj, const TA* __restrict__ va,
    const TX* __restrict__ x, TC alpha, const TY* b, TC beta, TY* y, int* __restrict__ carry_row,
    TC* __restrict__ carry_val, Skip skip) {
  if (skip.on()) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)nrows + nnz;
  const long long d0 = (long long)t * kMergeItems;
  if (d0 >= total) return;
  const int d1 = (int)min(d0 + kMergeItems, total);
  int r, k, r1, k1;
  merge_path_search((int)d0, rp, nrows, nnz, &r, &k);
  merge_path_search(d1, rp, nrows, nnz, &r1, &k1);
  TC acc = 0;
  int rend = r < nrows ? __ldg(&rp[r + 1]) : nnz;
  while (r < r1 || k < k1) {
    if (r < nrows && k < rend && k < k1) {
      acc += (TC)ldg(&va[k]) * (TC)x[__ldg(&cj[k])];
      k++;
    } else {
      // row r ends inside this range: its sum here plus the carries of the
      // threads before it that stopped inside the row
      TC v = alpha * acc;
      if (b) v += beta * (TC)b[r];
      y[r] = (TY)v;
      acc = 0;
      r++;
      rend = r < nrows ? __ldg(&rp[r + 1]) : nnz;
    }
  }
  carry_row[t] = r < nrows ? r : -1;
  carry_val[t] = acc;
}

// y[row] += alpha * (carries of that row, in thread order): one thread per
// run of equal rows, so the sum is deterministic
template <typename TY, typename TC>
__global__ void merge_spmv_fixup_kernel(int nthreads, const int* __restrict__ carry_row,
                                        const TC* __restrict__ carry_val, TC alpha, TY* y, Skip skip) {
  if (skip.on()) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nthreads; t += gridDim.x * blockDim.x) {
    const int row = carry_row[t];
    if (row < 0 || (t > 0 && carry_row[t - 1] == row)) continue;
    TC s = 0;
    for (int u = t; u < nthreads && carry_row[u] == row; u++) s += carry_val[u];
    y[row] = (TY)((TC)y[row] + alpha * s);
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
// bounded by spin_limit polls (kSpinLimit unless the handle sets another);
// on expiry the kernel records kErrTimeout and finishes.
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

// Complex values: the sentinel sits in the real part.  A complex64 value is
// published with one 8-byte store.  A complex128 value spans two 8-byte
// words: the imaginary part is stored first and the real part after it with
// release semantics, and a reader loads the real part with acquire semantics
// before the imaginary part, so a reader that sees a final real part also
// sees the imaginary part that belongs to it.
template <>
struct Sentinel<cf32> {
  static __device__ __forceinline__ cf32 value() { return cf32(Sentinel<float>::value(), 0.f); }
  static __device__ __forceinline__ bool is(const cf32& v) { return Sentinel<float>::is(v.x); }
  static __device__ __forceinline__ cf32 load(const cf32* p) {
    unsigned long long u;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(u) : "l"(p) : "memory");
    return cf32(__int_as_float((int)(u & 0xffffffffull)), __int_as_float((int)(u >> 32)));
  }
  static __device__ __forceinline__ void store(cf32* p, const cf32& v) {
    const unsigned long long u =
        (unsigned long long)(unsigned)__float_as_int(v.x) | ((unsigned long long)(unsigned)__float_as_int(v.y) << 32);
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(u) : "memory");
  }
};
template <>
struct Sentinel<cf64> {
  static __device__ __forceinline__ cf64 value() { return cf64(Sentinel<double>::value(), 0.0); }
  static __device__ __forceinline__ bool is(const cf64& v) { return Sentinel<double>::is(v.x); }
  static __device__ __forceinline__ cf64 load(const cf64* p) {
    double re, im;
    asm volatile("ld.acquire.gpu.global.f64 %0, [%1];" : "=d"(re) : "l"(&p->x) : "memory");
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(im) : "l"(&p->y) : "memory");
    return cf64(re, im);
  }
  static __device__ __forceinline__ void store(cf64* p, const cf64& v) {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(&p->y), "d"(v.y) : "memory");
    asm volatile("st.release.gpu.global.f64 [%0], %1;" ::"l"(&p->x), "d"(v.x) : "memory");
  }
};
// the segmented solve's operand prefetch: a complex128 operand goes through
// the acquire/release pair above
template <typename T>
__device__ __forceinline__ T ldcg_dep(const T* p) { return ldcg(p); }
template <>
__device__ __forceinline__ cf64 ldcg_dep<cf64>(const cf64* p) { return Sentinel<cf64>::load(p); }

template <typename T>
__global__ void sentinel_fill_kernel(int n, T* p) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = Sentinel<T>::value();
}

template <typename T, int S, bool UPPER>
__global__ void __launch_bounds__(256) trsv_kernel(
    int n, int ngroups, const int* __restrict__ ord, const int* __restrict__ rp, const int* __restrict__ cj,
    const T* __restrict__ va, const T* __restrict__ dinv, const T* __restrict__ rhs,
    const double* __restrict__ rhs_scale, T* y, T* x, unsigned long long* ticket, int* err, int spin_limit,
    Skip skip) {
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
            if (++spins > spin_limit || (*(volatile int*)err & kErrTimeout)) {
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
          if (rhs_scale) b = to<T>(to<typename Sc<T>::acc>(b) * rs);
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
constexpr int kSegNnzC128 = 4096;   // 192 KB (complex128)

template <typename T>
struct SegCfg {
  static constexpr int nnz = sizeof(T) == 16 ? kSegNnzC128 : sizeof(T) == 8 ? kSegNnzF64 : kSegNnzF32;
  // smem layout: xs[kSegRows] T | sb[kSegRows] T | sd[kSegRows] T | va[nnz] T | ext[nnz] T |
  // cj[nnz] int | ord[kSegRows] int | rp[kSegRows+4] int | lvb[kSegRows+4] int; the host keeps
  // segments within kSegRows-4 rows and nnz-4 nonzeros
  static constexpr size_t bytes =
      sizeof(T) * (size_t)(3 * kSegRows + 2 * nnz) + sizeof(int) * (size_t)(nnz + kSegRows + 2 * (kSegRows + 4));
  static_assert(bytes <= 227 * 1024, "segmented solve exceeds the shared memory of a CTA");
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
    unsigned long long* ticket, int* err, int spin_limit, Skip skip) {
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
        sb[i] = ldcg_dep(&y[r]);
        sd[i] = ldg(&dinv[r]);
      } else {
        T bb = ldg(&rhs[r]);
        if (rhs_scale) bb = to<T>(to<typename Sc<T>::acc>(bb) * rs);
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
      if (c >= 0 && c < n) sext[k] = ldcg_dep(&dep[c]);
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
                if (++spins > spin_limit || (*(volatile int*)err & kErrTimeout)) {
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
// subdomain (trsv_pipe_kernel below), for R right-hand sides at once.
#ifndef PGX_PIPE_THREADS
#define PGX_PIPE_THREADS 512
#endif
// one CTA per subdomain; the SM's other thread slots stay free for other kernels
constexpr int kPipeThreads = PGX_PIPE_THREADS;
constexpr int kPipeStages = 4;     // chunks in flight: the one being solved and three being staged
constexpr int kUnroll = 4;         // operands per lane loaded before any is used
constexpr long long kMbarWaitCycles = 1ll << 31;  // bound of a wait on a staging barrier: about 1 s

template <typename T, int R>
struct __align__(sizeof(T) * R <= 16 ? sizeof(T) * R : 16) VecR {
  T v[R];
};
template <typename T, int R>
struct PtrR {
  T* p[R];
};

// Shared-memory plan of the pipelined solve for value type T and R
// right-hand sides: a ring of the last `ring` results (R values per schedule
// position) followed by three far-operand buffers of `far` entries, then
// kPipeStages staging buffers of one chunk each (at most `nnz` nonzeros and
// `rows` rows, padding included).  Operand indices into the ring are checked
// once on the host when the layout is built; the kernel clamps them into the
// shared array, so a damaged layout can give wrong values but never an
// access outside shared memory.
template <typename T, int R>
struct PipeCfg {
  // sizes by value width: 4 bytes (FP32), 8 (FP64, complex64), 16 (complex128)
  static constexpr bool d = sizeof(T) == 8;
  static constexpr bool z = sizeof(T) == 16;
  static constexpr int ring = z ? (R == 1 ? 4096 : R == 2 ? 2048 : 1024)
                                : d ? (R == 1 ? 8192 : R == 2 ? 4096 : 2048) : (R == 4 ? 4096 : 8192);
  static constexpr int far = z ? 256 : d ? (R == 1 ? 512 : 256) : 512;
  static constexpr int nnz = z ? (R == 4 ? 768 : 1024)
                               : d ? (R == 4 ? 1536 : 2048) : (R == 1 ? 4096 : R == 2 ? 3072 : 2560);
  static constexpr int rows = z ? (R == 4 ? 128 : 192) : d ? 256 : (R == 1 ? 512 : R == 2 ? 384 : 320);
  // per stage: va[nnz] T | sb[R][rows] T | sd[rows] T | cj[nnz] | ord[rows] | rp[rows+4] | lvb[rows+4] | fc[far]
  static constexpr size_t buf_bytes =
      sizeof(T) * (size_t)(nnz + (R + 1) * rows) + sizeof(int) * (size_t)(nnz + rows + 2 * (rows + 4) + far);
  static constexpr size_t ring_bytes = sizeof(T) * R * (size_t)(ring + 3 * far);
  static constexpr size_t bytes = ring_bytes + kPipeStages * buf_bytes;
  static_assert(bytes <= 227 * 1024, "pipelined per-subdomain solve exceeds the shared memory of a CTA");
  static_assert(far <= kPipeThreads && rows <= kPipeThreads, "one gather per thread");
  static_assert((ring & (ring - 1)) == 0, "ring size must be a power of two");
  static_assert(nnz % 4 == 0 && rows % 4 == 0 && far % 4 == 0 && buf_bytes % 16 == 0 && ring_bytes % 16 == 0,
                "every staged array starts on a 16-byte boundary");
};

// Per-chunk metadata, two int4 per chunk: {row0, rp0, nnz0, lv0} and
// {pos0, far0, 0, 0}: first slot of the chunk in the row list, the row
// pointers, the nonzeros and the level boundaries; its first schedule
// position; its first far operand.  One record past the last chunk closes the
// ranges.  Every range starts on a 16-byte boundary and spans a multiple of
// 16 bytes (padded on the host), so each is one bulk copy.
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
  if (sizeof(T) == 16) {
    unsigned sd = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(sd), "l"(src) : "memory");
  } else if (sizeof(T) == 8) {
    cp_async8(dst, src);
  } else {
    cp_async4(dst, src);
  }
}

// mbarrier and bulk-copy (TMA, non-tensor) helpers.  The copies read this
// GPU's own global memory only.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false (and kErrStage recorded) if the phase did not
// complete within kMbarWaitCycles SM clocks
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (clock64() - t0 < kMbarWaitCycles)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(err, kErrStage);
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <typename T, int R>
struct PipeBuf {
  T *va, *sb, *sd;  // sb: R arrays of `rows`; sd: inverse diagonal (upper) or upper-pass slots (lower, as int)
  int *cj, *ord, *rp, *lvb, *fc;
};
template <typename T, int R, typename C = PipeCfg<T, R>>
__device__ __forceinline__ PipeBuf<T, R> pipe_buf(unsigned char* base, int stage) {
  unsigned char* b = base + C::ring_bytes + (size_t)stage * C::buf_bytes;
  PipeBuf<T, R> o;
  o.va = (T*)b;
  o.sb = o.va + C::nnz;
  o.sd = o.sb + R * C::rows;
  o.cj = (int*)(o.sd + C::rows);
  o.ord = o.cj + C::nnz;
  o.rp = o.ord + C::rows;
  o.lvb = o.rp + C::rows + 4;
  o.fc = o.lvb + C::rows + 4;
  return o;
}

struct CompArrays {
  const int4* meta;
  const int *ord, *rp, *cj, *lvb, *uslot, *far_col;
};

// one thread: stage chunk [m, me) into buffer b with bulk copies completing on
// bar (the byte count is announced first)
template <typename T, int R, bool UPPER>
__device__ __forceinline__ void pipe_issue(const PipeBuf<T, R>& b, const ChunkMeta& m, const ChunkMeta& me,
                                           const CompArrays& g, const T* __restrict__ va, const T* __restrict__ dslot,
                                           const PtrR<T, R>& yslot, unsigned long long* bar) {
  const unsigned nz = (unsigned)(me.nnz0 - m.nnz0), nr = (unsigned)(me.row0 - m.row0);
  const unsigned np = (unsigned)(me.rp0 - m.rp0), nv = (unsigned)(me.lv0 - m.lv0), nf = (unsigned)(me.far0 - m.far0);
  unsigned total = nz * (sizeof(T) + 4) + nr * 4 + np * 4 + nv * 4 + nf * 4 + nr * (UPPER ? sizeof(T) : 4);
  if (UPPER) total += R * nr * (unsigned)sizeof(T);
  mbar_arrive_expect_tx(bar, total);
  if (nz) {
    bulk_g2s(b.va, va + m.nnz0, nz * (unsigned)sizeof(T), bar);
    bulk_g2s(b.cj, g.cj + m.nnz0, nz * 4, bar);
  }
  bulk_g2s(b.ord, g.ord + m.row0, nr * 4, bar);
  bulk_g2s(b.rp, g.rp + m.rp0, np * 4, bar);
  bulk_g2s(b.lvb, g.lvb + m.lv0, nv * 4, bar);
  if (nf) bulk_g2s(b.fc, g.far_col + m.far0, nf * 4, bar);
  if (UPPER) {
    bulk_g2s(b.sd, dslot + m.row0, nr * (unsigned)sizeof(T), bar);
#pragma unroll
    for (int r = 0; r < R; r++) bulk_g2s(b.sb + r * PipeCfg<T, R>::rows, yslot.p[r] + m.row0, nr * (unsigned)sizeof(T), bar);
  } else {
    bulk_g2s(b.sd, g.uslot + m.row0, nr * 4, bar);
  }
}

// One CTA per subdomain solves its rows level by level (the schedule of
// IluClass::BuildLevels, ilu.cpp:832-1062, restricted to the subdomain),
// for R right-hand sides at once: a lower pass y = L^-1 rhs or an upper pass
// x = D U^-1 y.  Each staged factor entry is read once and applied to all R
// vectors.  Results live in a shared-memory ring indexed by schedule
// position, so a dependency on the last `ring` positions is a shared-memory
// read (one vector load for the R values).  An older ("far") operand lies,
// by construction on the host, before the start of the previous chunk: it
// was published to global memory before that chunk began, so it is gathered
// into the far buffer while the previous chunk is being solved.  Column
// indices are encoded as -(index + 1) into the ring-plus-far array.
//
// The subdomain's schedule is cut into chunks.  One thread stages chunk
// c + kPipeStages - 1 with bulk copies (completing on that stage's mbarrier)
// as soon as chunk c - 1 is done, so the factor streams in well ahead of the
// solve; at the start of chunk c the CTA gathers what needs an index (the
// lower pass's right-hand side through the row list, the far operands) for
// chunk c + 1.  A chunk's end coincides with the barrier of its last level:
// a chunk boundary costs no barrier of its own.  Each row's writing lanes
// publish its result to global memory at once (natural order, and the upper
// pass's slot order in the lower pass).  No CTA waits on another.
template <typename T, int S, bool UPPER, int R, typename C = PipeCfg<T, R>>
__global__ void __launch_bounds__(kPipeThreads, 1) trsv_pipe_kernel(
    int n, int nslots, const int* __restrict__ comp_ch0, CompArrays g, const T* __restrict__ va,
    const T* __restrict__ dslot, PtrR<T, R> yslot, PtrR<T, R> rhs, PtrR<T, R> y, PtrR<T, R> x, int* err,
    SkipR<R> skip) {
  // a wait of an earlier pass of this solve gave up: the solve reports the
  // timeout, and the passes after it do no work
  if (skip.on() || (*(volatile int*)err & (kErrTimeout | kErrStage))) return;
  using V = VecR<T, R>;
  constexpr int RF = C::ring + 3 * C::far;
  constexpr int D = kPipeStages;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long s_full[D];
  __shared__ ChunkMeta s_meta[D][2];  // {chunk, next chunk} of the chunk in each stage
  __shared__ int s_abort;
  V* ring = (V*)smem_raw;  // ring, then far buffers 0, 1, 2
  const int tid = threadIdx.x, lane = tid & 31;
  const int c0 = comp_ch0[blockIdx.x], c1 = comp_ch0[blockIdx.x + 1];
  const PtrR<T, R> out = UPPER ? x : y;
  if (c0 >= c1) return;
  // tid 0 keeps the metadata of the next chunk to stage and of the one after
  ChunkMeta ma{}, mb{};
  unsigned long long issued = 0, waited = 0;  // per-stage use counts, 16 bits each (tid 0), for the exit path
  if (tid == 0) {
    s_abort = 0;
    for (int s = 0; s < D; s++) mbar_init(&s_full[s], 1);
    mbar_fence_init();
    ma = load_meta(g.meta, c0);
    for (int k = 0; k < D && c0 + k < c1; k++) {
      mb = load_meta(g.meta, c0 + k + 1);
      s_meta[k][0] = ma;
      s_meta[k][1] = mb;
      pipe_issue<T, R, UPPER>(pipe_buf<T, R>(smem_raw, k), ma, mb, g, va, dslot, yslot, &s_full[k]);
      issued += 1ull << (16 * k);
      ma = mb;
    }
    mb = c0 + D + 1 <= c1 ? load_meta(g.meta, c0 + D + 1) : ma;
  }
  __syncthreads();
  const int sl = tid & (S - 1), group = tid / S;
  constexpr int NG = kPipeThreads / S;
  // What needs an index is gathered two chunks ahead, into chunk j's stage
  // (the lower pass's right-hand side through the row list) and into far
  // buffer j % 3 (the far operands, which the host placed before the start
  // of chunk j - 2, so they are published by then); each chunk's gathers are
  // one cp.async group.
  auto gather = [&](int j) {  // j: chunk index within the subdomain
    const int sj = j % D;
    if (!mbar_wait(&s_full[sj], (unsigned)((j / D) & 1), err)) {
      s_abort = 1;  // the staged indices are not there: gather nothing
      return;
    }
    if (tid == 0) waited += 1ull << (16 * sj);
    const PipeBuf<T, R> nb = pipe_buf<T, R>(smem_raw, sj);
    const ChunkMeta n0 = s_meta[sj][0], n1 = s_meta[sj][1];
    if (!UPPER && tid < n1.row0 - n0.row0) {
      const int rr = nb.ord[tid];
      if ((unsigned)rr < (unsigned)n) {
#pragma unroll
        for (int r = 0; r < R; r++) cp_async_elem(&nb.sb[r * C::rows + tid], &rhs.p[r][rr]);
      } else if (rr >= 0) {
        atomicOr(err, kErrIndex);
      }
    }
    if (tid < n1.far0 - n0.far0) {
      const int fcol = nb.fc[tid];
      if ((unsigned)fcol < (unsigned)n) {
        V* fv = &ring[C::ring + (j % 3) * C::far + tid];
#pragma unroll
        for (int r = 0; r < R; r++) cp_async_elem(&fv->v[r], &out.p[r][fcol]);
      } else if (fcol >= 0) {
        atomicOr(err, kErrIndex);
      }
    }
  };
  gather(0);
  asm volatile("cp.async.commit_group;" ::: "memory");
  if (c0 + 1 < c1) gather(1);
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 1;" ::: "memory");
  __syncthreads();
  for (int ch = c0; ch < c1; ch++) {
    if (s_abort) break;
    const int k = ch - c0;
    const int st = k % D;
    const PipeBuf<T, R> b = pipe_buf<T, R>(smem_raw, st);
    const ChunkMeta m0 = s_meta[st][0], m1 = s_meta[st][1];
    if (ch + 2 < c1) gather(k + 2);
    asm volatile("cp.async.commit_group;" ::: "memory");  // (empty near the end: keeps one group per chunk)
    const int pos0 = m0.pos0;
    const int nl = m1.lv0 - m0.lv0;
    // Every read of this chunk's stage happens before the barrier of its
    // last level: right after that barrier thread 0 reuses the stage for
    // the chunk kPipeStages ahead, so the boundary of the next level is read
    // before each barrier, and the last level ends the loop.
    int a = b.lvb[0];
    int e = nl > 1 ? b.lvb[1] : a;
    if (a >= e) {  // no level (the host never builds such a chunk): still land the gathers
      asm volatile("cp.async.wait_group 1;" ::: "memory");
      __syncthreads();
    }
    for (int lv = 0; a < e; lv++) {
      for (int i = a + group; i < e; i += NG) {
        // row pointers stay inside the staged nonzeros
        const int k1 = max(b.rp[i], 0), k2 = min(b.rp[i + 1], C::nnz);
        T acc[R];
#pragma unroll
        for (int r = 0; r < R; r++) acc[r] = 0;
        int q[kUnroll];
        T v[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
          const int kk = k1 + sl + u * S;
          q[u] = kk < k2 ? -b.cj[kk] - 1 : 0;
          v[u] = kk < k2 ? b.va[kk] : T(0);
        }
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
          if (k1 + sl + u * S < k2) {  // never read an unwritten ring slot
            const V w = ring[min((unsigned)q[u], (unsigned)(RF - 1))];
#pragma unroll
            for (int r = 0; r < R; r++) acc[r] += v[u] * w.v[r];
          }
        }
        for (int kk = k1 + sl + kUnroll * S; kk < k2; kk += S) {
          const int qq = -b.cj[kk] - 1;
          const V w = ring[min((unsigned)qq, (unsigned)(RF - 1))];
          const T vv = b.va[kk];
#pragma unroll
          for (int r = 0; r < R; r++) acc[r] += vv * w.v[r];
        }
        // sum over the group's lanes for every right-hand side: for R > 1 a
        // reduce-scatter first (each step halves the values a lane carries),
        // then a butterfly on one value.  Every partial sum adds the same two
        // operands as group_reduce does, so the results are identical to the
        // one-right-hand-side solve's.  Each result is written by one lane:
        // into the ring and, at once, to global memory.
        const unsigned gmask = S == 32 ? 0xffffffffu : (((1u << S) - 1u) << (lane & ~(S - 1)));
        auto put = [&](int r, T o) {
          const T bb = b.sb[r * C::rows + i];
          const T res = UPPER ? (bb - o) * b.sd[i] : bb - o;
          ring[(pos0 + i) & (C::ring - 1)].v[r] = res;
          // pick the lane's pointers by comparison: no dynamic index into a
          // parameter array (that would go through local memory)
          T* op = out.p[0];
          T* ys = yslot.p[0];
#pragma unroll
          for (int rr = 1; rr < R; rr++)
            if (rr == r) {
              op = out.p[rr];
              ys = yslot.p[rr];
            }
          const int orow = b.ord[i];
          if ((unsigned)orow < (unsigned)n)
            op[orow] = res;
          else
            atomicOr(err, kErrIndex);
          if (!UPPER) {
            const int us = ((const int*)b.sd)[i];
            if ((unsigned)us < (unsigned)nslots)
              ys[us] = res;
            else
              atomicOr(err, kErrIndex);
          }
        };
        if constexpr (R == 4 && S >= 4) {
          const bool hb = (sl & (S >> 1)) != 0, qb = (sl & (S >> 2)) != 0;
          T k0 = hb ? acc[2] : acc[0], kx = hb ? acc[3] : acc[1];
          const T s0 = hb ? acc[0] : acc[2], s1 = hb ? acc[1] : acc[3];
          k0 += __shfl_xor_sync(gmask, s0, S >> 1);
          kx += __shfl_xor_sync(gmask, s1, S >> 1);
          T kk = qb ? kx : k0;
          kk += __shfl_xor_sync(gmask, qb ? k0 : kx, S >> 2);
#pragma unroll
          for (int off = S >> 3; off > 0; off >>= 1) kk += __shfl_xor_sync(gmask, kk, off);
          if ((sl & ((S >> 2) - 1)) == 0) put((hb ? 2 : 0) + (qb ? 1 : 0), kk);
        } else if constexpr (R == 2 && S >= 2) {
          const bool hb = (sl & (S >> 1)) != 0;
          T kk = hb ? acc[1] : acc[0];
          kk += __shfl_xor_sync(gmask, hb ? acc[0] : acc[1], S >> 1);
#pragma unroll
          for (int off = S >> 2; off > 0; off >>= 1) kk += __shfl_xor_sync(gmask, kk, off);
          if ((sl & ((S >> 1) - 1)) == 0) put(hb ? 1 : 0, kk);
        } else {
#pragma unroll
          for (int r = 0; r < R; r++) acc[r] = group_reduce(acc[r], S, lane);
          if (sl == 0) {
#pragma unroll
            for (int r = 0; r < R; r++) put(r, acc[r]);
          }
        }
      }
      // the next boundary (the padding after the last one repeats it)
      const int e2 = lv + 2 < nl ? b.lvb[lv + 2] : e;
      // the last level of the chunk: the next chunk's gathers (all groups but
      // the newest) have landed before the barrier
      if (e2 <= e) asm volatile("cp.async.wait_group 1;" ::: "memory");
      __syncthreads();
      a = e;
      e = e2;
    }
    // chunk done: its stage is free for the chunk kPipeStages ahead
    if (tid == 0 && ch + D < c1) {
      s_meta[st][0] = ma;
      s_meta[st][1] = mb;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      pipe_issue<T, R, UPPER>(b, ma, mb, g, va, dslot, yslot, &s_full[st]);
      issued += 1ull << (16 * st);
      ma = mb;
      if (ch + D + 2 <= c1) mb = load_meta(g.meta, ch + D + 2);
    }
  }
  if (s_abort && tid == 0) {
    // a staging wait gave up: let the copies still in flight land (bounded)
    // before the CTA's shared memory is released
    for (int s = 0; s < D; s++) {
      const unsigned is = (unsigned)(issued >> (16 * s)) & 0xffffu, ws = (unsigned)(waited >> (16 * s)) & 0xffffu;
      for (unsigned u = ws; u < is; u++) mbar_wait(&s_full[s], u & 1u, err);
    }
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

// Reductions and coefficients are carried in TsAcc<TW>: double for a real
// solve, cf64 for a complex one (dots conjugate the basis column,
// V(:,c)^H w, as the reference's complex VectorDot does).
template <typename TW>
using TsAcc = typename Sc<TW>::acc;

template <typename TV, typename TM, typename TW>
struct TsArgs {
  using A = TsAcc<TW>;
  int n;
  int ncols;
  const int* ncols_dev;  // if set, the column count is read here (<= KMAX)
  const TV* V;
  long long ldv;
  const double* vsc;
  const TM* M;
  long long ldm;
  const double* msc;
  const A* coef;
  double sign;
  const TW* in;          // null: zero input
  const double* in_scale;
  TW* out;
  A* partial;            // [KMAX+1][gridDim.x]
  unsigned int* counter; // zero between launches
  int epi;
  FgmresDevT<A>* st;
  A* dst;
  int j;
  Skip skip;
};

template <typename S>
__device__ inline void fgmres_givens(FgmresDevT<S>* st, int j, double t) {
  // H(:, j) from the Gram-Schmidt coefficients and ||w||
  // (PargemslrMgs sets H(0..k, k) and H(k+1, k), matrixops.cpp:10728-10806)
  const int ldh = KMAX + 1;
  S* H = st->H + (size_t)j * ldh;
  for (int c = 0; c <= j; c++) H[c] = st->hcol[c];
  H[j + 1] = S(t);
  st->sc[j + 1] = 1.0 / t;
  st->iter += 1;
  st->i = j + 1;
  // apply the previous rotations, then form the new one (fgmres.hpp:430-458;
  // for complex values the rotation is conj(c), s as in the reference)
  for (int k = 1; k <= j; k++) {
    S hii = H[k - 1];
    H[k - 1] = conj(st->c[k - 1]) * hii + st->s[k - 1] * H[k];
    H[k] = -st->s[k - 1] * hii + st->c[k - 1] * H[k];
  }
  S hii = H[j], hii1 = H[j + 1];
  double gam = sqrt(cabs(hii) * cabs(hii) + cabs(hii1) * cabs(hii1));
  if (fabs(gam) < st->eps) {
    // breakdown: the reference jumps past the solution update (fgmres.hpp:440-443)
    // and records no residual for this iteration
    st->hist[j] = 0.0;
    st->breakdown = 1;
    st->i = 0;
    st->cycle_done = 1;
    st->done = 1;
    return;
  }
  st->c[j] = hii / gam;
  st->s[j] = hii1 / gam;
  st->rs[j + 1] = -st->s[j] * st->rs[j];
  st->rs[j] = conj(st->c[j]) * st->rs[j];
  H[j] = conj(st->c[j]) * hii + st->s[j] * hii1;
  st->normr = cabs(st->rs[j + 1]);
  st->hist[j] = st->normr;  // _rel_res_vector[_iter] = normr / normb (fgmres.hpp:450-452)
  const bool conv = st->normr <= st->tolr;
  if (conv) st->converged = 1;
  if (conv || st->i >= st->kdim || st->iter >= st->maxits) {
    st->cycle_done = 1;
    if (conv || st->iter >= st->maxits) st->done = 1;
    // back substitution H y = rs, in place in rs (fgmres.hpp:471-480)
    const int i = st->i;
    S* rs = st->rs;
    rs[i - 1] = rs[i - 1] / st->H[(size_t)(i - 1) * ldh + (i - 1)];
    for (int k = i - 2; k >= 0; k--) {
      for (int jj = k + 1; jj < i; jj++) rs[k] -= st->H[(size_t)jj * ldh + k] * rs[jj];
      rs[k] = rs[k] / st->H[(size_t)k * ldh + k];
    }
  }
}

template <typename TV, typename TM, typename TW>
__device__ inline void ts_epilogue(const TsArgs<TV, TM, TW>& a, const TsAcc<TW>* sums, int ncols) {
  using A = TsAcc<TW>;
  FgmresDevT<A>* st = a.st;
  switch (a.epi) {
    case EPI_STORE:
      for (int c = 0; c < ncols; c++) a.dst[c] = sums[c] * (a.vsc ? a.vsc[c] : 1.0);
      break;
    case EPI_CGS_FIRST:
      for (int c = 0; c < ncols; c++) {
        A h = sums[c] * (a.vsc ? a.vsc[c] : 1.0);
        st->hcol[c] = h;
        st->coefA[c] = h;
      }
      break;
    case EPI_CGS_SECOND:
      for (int c = 0; c < ncols; c++) {
        A h = sums[c] * (a.vsc ? a.vsc[c] : 1.0);
        st->hcol[c] += h;
        st->coefB[c] = h;
      }
      break;
    case EPI_GIVENS:
      fgmres_givens(st, a.j, sqrt(re(sums[0])));
      break;
    case EPI_NORMB:
      st->normb = sqrt(re(sums[0]));
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
      const double normr = sqrt(re(sums[0]));
      st->normr = normr;
      st->normr0 = normr;
      if (normr < st->eps) {
        st->done = 1;
        st->cycle_done = 1;
        st->converged = 1;
        break;
      }
      st->tolr = st->absolute ? st->tol : st->tol * st->normb;
      st->rs[0] = A(normr);
      st->sc[0] = 1.0 / normr;
      st->cycle_done = 0;
      break;
    }
    case EPI_INIT_INNER: {
      const double normb = sqrt(re(sums[0]));
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
      st->rs[0] = A(normb);
      st->sc[0] = 1.0 / normb;
      break;
    }
    default:
      break;
  }
}

template <typename TV, typename TM, typename TW, int MODE>
__global__ void __launch_bounds__(kTsThreads) ts_kernel(TsArgs<TV, TM, TW> a) {
  using A = TsAcc<TW>;
  if (a.skip.on()) return;
  __shared__ A scoef[KMAX + 1];
  __shared__ A sacc[KMAX + 1];
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
    scoef[c] = (update && c < ncols) ? a.sign * a.coef[c] * (a.msc ? a.msc[c] : 1.0) : A(0.0);
    sacc[c] = A(0.0);
  }
  if (tid < NW) swarp[tid] = 0.0;
  __syncthreads();
  const int ntiles = (a.n + kTsThreads - 1) / kTsThreads;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * kTsThreads;
    const int row = r0 + tid;
    A wv = A(0.0);
    if (row < a.n) {
      wv = a.in ? to<A>(a.in[row]) * in_s : A(0.0);
      if (update) {
        A acc = A(0.0);
        const TM* m = a.M + row;
        for (int c = 0; c < ncols; c++) acc += to<A>(m[(long long)c * a.ldm]) * scoef[c];
        wv += acc;
      }
      if (MODE != TS_DOT && a.out) a.out[row] = to<TW>(wv);
    }
    if (MODE == TS_UPDATE_NORM || MODE == TS_NORM_COPY) {
      double sq = (row < a.n) ? abs2(wv) : 0.0;
      if (MODE == TS_UPDATE_NORM) {
        // the norm of the stored (rounded) vector, as Norm2 of the reference
        TW stored = to<TW>(wv);
        sq = (row < a.n) ? abs2(to<A>(stored)) : 0.0;
      }
      sq = warp_reduce(sq);
      if (lane == 0) swarp[warp] += sq;  // one writer per slot: deterministic
    }
    if (MODE == TS_DOT || MODE == TS_UPDATE_DOT) {
      __syncthreads();  // out[] of this tile written by the whole block
      const int nrows_tile = min(kTsThreads, a.n - r0);
      for (int c = warp; c < ncols; c += NW) {
        const TV* v = a.V + (long long)c * a.ldv + r0;
        A acc = A(0.0);
        for (int k = lane; k < nrows_tile; k += 32) {
          A w = (MODE == TS_DOT) ? (a.in ? to<A>(a.in[r0 + k]) * in_s : A(0.0)) : to<A>(a.out[r0 + k]);
          acc += conj(to<A>(v[k])) * w;
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
    sacc[0] = A(t);
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
    A acc = A(0.0);
    for (int b = lane; b < (int)gridDim.x; b += 32) acc += ldcg(&a.partial[(long long)c * gridDim.x + b]);
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

template <typename S>
__global__ void fgmres_cycle_reset_kernel(FgmresDevT<S>* st, Skip skip) {
  if (skip.on()) return;
  st->i = 0;
  if (st->done) return;
  st->cycle_done = 0;
  st->rs[0] = S(st->normr);
  st->sc[0] = 1.0 / st->normr;
}

// --------------------------------------------------- permutation + convert
// out[i] = (TO)(in[perm[i]] * scale)  (IntVectorClass::GatherPerm, int_vector.cpp:668)
// Each thread handles kPermUnroll entries a block apart: it loads their
// permutation indices, then the values they name, then stores, so the
// dependent loads of several entries are in flight together.
constexpr int kPermUnroll = 4;
template <typename TI, typename TO>
__global__ void __launch_bounds__(256) gather_kernel(int n, const int* __restrict__ perm, const TI* __restrict__ in,
                                                     const double* __restrict__ scale, TO* __restrict__ out,
                                                     Skip skip) {
  if (skip.on()) return;
  const double s = scale ? *scale : 1.0;
  const int stride = gridDim.x * blockDim.x * kPermUnroll;
  for (int base = blockIdx.x * blockDim.x * kPermUnroll + threadIdx.x; base < n; base += stride) {
    int p[kPermUnroll];
#pragma unroll
    for (int u = 0; u < kPermUnroll; u++) {
      const int i = base + u * blockDim.x;
      p[u] = i < n ? (perm ? __ldg(&perm[i]) : i) : -1;
    }
    TI v[kPermUnroll];
#pragma unroll
    for (int u = 0; u < kPermUnroll; u++) v[u] = p[u] >= 0 ? in[p[u]] : TI(0);
#pragma unroll
    for (int u = 0; u < kPermUnroll; u++) {
      const int i = base + u * blockDim.x;
      if (i < n) out[i] = scale ? to<TO>(to<typename Sc<TI>::acc>(v[u]) * s) : to<TO>(v[u]);
    }
  }
}

// y += x  (the solution update of the multiplicative level solve)
template <typename T>
__global__ void __launch_bounds__(256) axpy_kernel(int n, const T* __restrict__ x, T* __restrict__ y, Skip skip) {
  if (skip.on()) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] += x[i];
}

// out[perm[i]] = in[i]  (IntVectorClass::ScatterRperm, int_vector.cpp:629)
template <typename TI, typename TO>
__global__ void __launch_bounds__(256) scatter_kernel(int n, const int* __restrict__ perm, const TI* __restrict__ in,
                                                      TO* __restrict__ out, Skip skip) {
  if (skip.on()) return;
  const int stride = gridDim.x * blockDim.x * kPermUnroll;
  for (int base = blockIdx.x * blockDim.x * kPermUnroll + threadIdx.x; base < n; base += stride) {
    int p[kPermUnroll];
    TI v[kPermUnroll];
#pragma unroll
    for (int u = 0; u < kPermUnroll; u++) {
      const int i = base + u * blockDim.x;
      p[u] = i < n ? (perm ? __ldg(&perm[i]) : i) : -1;
      v[u] = i < n ? in[i] : TI(0);
    }
#pragma unroll
    for (int u = 0; u < kPermUnroll; u++)
      if (p[u] >= 0) out[p[u]] = to<TO>(v[u]);
  }
}

template <typename T>
__global__ void fill_kernel(int n, T v, T* out, Skip skip) {
  if (skip.on()) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = v;
}

}  // namespace pgx
