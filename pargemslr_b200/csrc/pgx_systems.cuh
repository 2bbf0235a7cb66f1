// Many independent systems of uneven sizes solved by ONE persistent kernel
// launch: every CTA takes the next system of a packed work list (largest
// first) and runs its whole GeMSLR-preconditioned flexible GMRES on its own,
// restart cycles, level recursion and the level-0 inner Schur FGMRES
// included, then takes the next system.  The only synchronisation is
// __syncthreads inside a CTA, so no CTA ever waits on another.
//
// The arithmetic follows the per-system engine (and through it the
// reference):
//   FlexGmresClass::Solve, ParGeMSLR SRC/solvers/fgmres.hpp:263-558
//     (restarted right-preconditioned FGMRES, Givens rotations, the restart
//     residual b - A x and the Givens estimate carried into the next cycle);
//   GemslrClass::Solve / SolveLevel, gemslr.cpp:3431-3630 (gather by pperm,
//     block LU per level, scatter by qperm);
//   GemslrClass::SolveB, gemslr.cpp:3632-3678 with IluClass::SolveHost,
//     ilu.cpp:3677-3790 (unit lower L, strict upper U, inverse diagonal);
//   SolveApplyLowRankLevel, gemslr.cpp:3681-3722 (x += WH (W^T x));
//   the level-0 inner FlexGmres over GemslrSchurMatrixClass,
//     gemslr.cpp:294-330 and 1660-1674, with SchurMatVec, gemslr.cpp:3799-3960;
//   CGS2 orthogonalisation (PargemslrCgs2, matrixops.cpp:10588-10708);
//   the U solve option (gemslr.cpp:3527-3532: a level skips its block-L part).
// Krylov vectors, Givens rotations and the true residual are FP64; the
// preconditioner (factors, coupling blocks, low-rank bases and its vectors)
// is stored and accumulated in P (float for the mixed precision, double for
// FP64), with the low-rank and Gram-Schmidt coefficients reduced in FP64.
#pragma once

#include "pgx_device.cuh"

namespace pgx {

constexpr int kSysMaxThreads = 1024;
constexpr int kSysMaxLevels = 8;
constexpr int kSysDotCols = 8;   // dot products one pass over the rows accumulates

template <typename T>
struct SysCsr {
  int rows, cols;
  const int* rp;
  const int* cj;
  const T* va;
};

// A triangular factor with its rows stored level by level (IluClass level
// sets, ilu.cpp:832-1062): packed row k is row `row[k]`; levels are the
// ranges lvp[t]..lvp[t+1] of packed rows.  Column entries hold PACKED
// positions (pc[e] = position of column cj[e] in this order), so the solve
// keeps solved values in packed order; `span` is the farthest dependency
// (k - pc[e]) plus the widest level, the ring a pass needs.  The first
// kSysHead entries of every packed row are repeated in fixed-size heads
// (hpc, hva: kSysHead per row, zero-padded) so a row's data is addressed by
// its position alone; dst[k] is where the solved value of packed row k goes:
// the upper factor's packed position of that row (lower factor), or the row
// itself (upper factor).  Upper factors carry the inverse diagonal per
// packed row.
constexpr int kSysHead = 8;
template <typename P>
struct SysTri {
  int n, nlev, span;
  const int* lvp;
  const int* row;
  const int* rp;
  const int* pc;
  const P* va;
  const int* hpc;
  const P* hva;
  const int* dst;
  const P* dinv;
};

template <typename P>
struct SysLevel {
  int nl, m, rank;  // rows of B_l, rows below it, low-rank columns
  SysTri<P> L, U;
  SysCsr<P> E, F;   // E: m x nl, F: nl x m
  const P* W;       // m x rank, column-major
  const P* WH;
  P* z;             // nl + m: (zu | zl)
};

template <typename P>
struct SysDesc {
  int n, nlev;
  SysCsr<double> A;
  const int* pperm;
  const int* qperm;  // null: scatter by pperm
  SysLevel<P> lev[kSysMaxLevels];
  SysCsr<P> C0;      // level-0 C block (inner Schur FGMRES)
  int inner, inner_maxits;
  double inner_tol;
  int usolve;        // the U solve: a level's block-L part is skipped, z = rhs (gemslr.cpp:3527-3532)
  // work space
  double* V;   // n x (kdim + 1)
  P* Z;        // n x kdim
  P* rt;       // n: permuted right-hand side of the preconditioner
  P* xt;       // n: permuted preconditioner output
  P* y;        // n: packed scratch of the triangular passes whose span exceeds the shared ring
  P* yr;       // n: the lower pass's right-hand side in its packed order
  P* yu;       // n: the lower pass's result in the upper factor's packed order
  P* Vin;      // m0 x (inner_maxits + 1)
  P* Zin;      // m0 x inner_maxits
  P* xlr;      // m0
  P* s_zu;     // nl0
  P* s_wu;     // nl0
};

struct SysResult {
  int iters, converged, breakdown, pad;
  double normb, normr, true_r2;
  unsigned long long t0, t1;  // %globaltimer at the start and end of the system's solve (ns)
  unsigned long long tri_ns;  // of which in the triangular (B-block) solves
  int cta, pad2;
};

template <typename P>
struct SysArgs {
  const SysDesc<P>* sys;
  const int* order;  // work list
  int count;
  const double* const* b;
  double* const* x;
  int kdim, maxits, atol;
  double tol;
  int lanes;          // SpMV lanes per row (1, 2, 4 or 8)
  int scap;           // values of the dynamic shared-memory solve buffer
  int depth;          // levels the triangular passes fetch ahead (2 or 3)
  unsigned int* next;
  FgmresDev* st;      // per CTA: outer solve
  FgmresDev* st_in;   // per CTA: inner solve
  SysResult* res;
};

// shared memory of one CTA: reduction partials, coefficient vectors and the
// products an update applies
struct SysShared {
  double red[kSysDotCols * 32];
  void* sbuf;  // the CTA's triangular-solve buffer (dynamic shared memory)
  int scap;    // its capacity in values
  int depth;   // levels the triangular passes fetch ahead (2 or 3)
  unsigned long long tri_ns;  // time in the B-block solves of the current system (thread 0)
  double coef[KMAX + kSysDotCols];
  double coef2[KMAX + kSysDotCols];
  double prod[KMAX + kSysDotCols];
  double tmp[kSysDotCols];
  int sys;
};

__device__ __forceinline__ unsigned long long sys_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Block sums of NV per-thread values, combined in a fixed order (warp
// shuffles, then the warps in index order) into out[0..NV).  All threads
// call it; out is valid for all of them on return.
template <int NV>
__device__ __forceinline__ void sys_block_sum(double (&v)[NV], double* red, double* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int c = 0; c < NV; c++) {
    double t = v[c];
#pragma unroll
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    v[c] = t;
  }
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < NV; c++) red[c * 32 + warp] = v[c];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < nw; w++) s += red[threadIdx.x * 32 + w];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// out[c] = vsc[c] * isc * sum_i V(i, c) in(i), c < ncols (FP64 sums)
template <typename TV, typename TI>
__device__ void sys_multidot(int n, int ncols, const TV* V, long long ld, const double* vsc, const TI* in,
                             double isc, double* red, double* out) {
  for (int c0 = 0; c0 < ncols; c0 += kSysDotCols) {
    const int nc = min(kSysDotCols, ncols - c0);
    double acc[kSysDotCols];
#pragma unroll
    for (int c = 0; c < kSysDotCols; c++) acc[c] = 0.0;
    const TV* Vc = V + (long long)c0 * ld;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const double w = (double)in[i];
#pragma unroll
      for (int c = 0; c < kSysDotCols; c++)
        if (c < nc) acc[c] += (double)Vc[(long long)c * ld + i] * w;
    }
    sys_block_sum<kSysDotCols>(acc, red, out + c0);
    if (threadIdx.x < nc) out[c0 + threadIdx.x] *= (vsc ? vsc[c0 + threadIdx.x] : 1.0) * isc;
    __syncthreads();
  }
}

// out(i) = in(i) * isc + sign * sum_c M(i, c) msc[c] coef[c]  (in may be null:
// zero); returns the block sum of out(i)^2 when NORM.  coef may live in
// global or shared memory; the products sign * msc[c] * coef[c] are formed
// once in shared memory.
template <bool NORM, typename TM, typename TI, typename TO>
__device__ double sys_update(int n, int ncols, const TM* M, long long ld, const double* msc, const double* coef,
                             double sign, const TI* in, double isc, TO* out, SysShared& sh) {
  for (int c = threadIdx.x; c < ncols; c += blockDim.x) sh.prod[c] = sign * (msc ? msc[c] : 1.0) * coef[c];
  __syncthreads();
  double nrm[1] = {0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double u = in ? (double)in[i] * isc : 0.0;
    for (int c = 0; c < ncols; c++) u += (double)M[(long long)c * ld + i] * sh.prod[c];
    const TO o = (TO)u;
    out[i] = o;
    if (NORM) nrm[0] += (double)o * (double)o;
  }
  if (NORM) {
    sys_block_sum<1>(nrm, sh.red, sh.tmp);
    return sh.tmp[0];
  }
  __syncthreads();
  return 0.0;
}

// y(i) = alpha * sum_k M(i, k) x(k) + beta * yin(i)  (yin may alias y or be
// null), S lanes per row; every lane runs the same number of row rounds so
// the shuffles of a group see all of its lanes
template <typename TA, typename TM, typename TX, typename TY, typename TYI>
__device__ void sys_spmv(const SysCsr<TM>& M, const TX* x, TA alpha, const TYI* yin, TA beta, TY* y, int S) {
  const int g = threadIdx.x / S, l = threadIdx.x % S, ng = blockDim.x / S;
  for (int i0 = 0; i0 < M.rows; i0 += ng) {
    const int i = i0 + g;
    TA acc = TA(0);
    if (i < M.rows) {
      const int e1 = M.rp[i + 1];
      for (int e = M.rp[i] + l; e < e1; e += S) acc += (TA)M.va[e] * (TA)x[M.cj[e]];
    }
    for (int o = S >> 1; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (l == 0 && i < M.rows) y[i] = (TY)(alpha * acc + (yin ? beta * (TA)yin[i] : TA(0)));
  }
  __syncthreads();
}

// Level-scheduled triangular solve (IluClass::SolveHost, ilu.cpp:3677-3790):
// lower, unit diagonal: x_k = rhs_k - L(k,:) x;  upper: x_k = dinv_k (rhs_k -
// U(k,:) x), all in the factor's packed (level) order.  Rows of one level
// depend only on rows of earlier levels.  Solved values are kept in `buf`
// at position k & mask: a shared-memory ring when the factor's span fits it
// (a value is overwritten only after every row that reads it is done), else
// a global vector of the factor's length (mask all ones); each is also
// stored to out[dst[k]], off the dependency chain.
//
// A thread's first row of each level is fetched DEPTH levels ahead into
// registers: its right-hand side (already in packed order), destination,
// extent, head entries and inverse diagonal.  Every one of those loads is
// addressed by the row's packed position alone.  The registers rotate by
// slot, not by copy: slot d holds level t + d, is consumed there and
// refilled in place for level t + d + DEPTH (a register copy of a value
// still in flight would wait for it), and the level pointers each refill
// needs were loaded into the slot DEPTH levels before.  So no load is
// waited on before it has had DEPTH levels to arrive, and after a barrier
// only the ring reads (shared memory) remain on the chain.  DEPTH (2 or 3)
// is a schedule choice.
template <typename P>
struct SysRowPF {
  int k, kend, dst, e0, e1;
  P rhs, dg;
  int pc[kSysHead];
  P va[kSysHead];
};
template <bool UPPER, typename P>
__device__ __forceinline__ void sys_fetch_row(const SysTri<P>& T, const P* rhs, int lv0, int lv1, SysRowPF<P>& f) {
  f.k = lv0 + threadIdx.x;
  f.kend = lv1;
  f.dst = -1;
  const int k = f.k;
  if (k >= lv1) return;
  f.dst = T.dst[k];
  f.e0 = T.rp[k];
  f.e1 = T.rp[k + 1];
  f.rhs = rhs[k];
  f.dg = UPPER ? T.dinv[k] : P(1);
  const int4* hp = reinterpret_cast<const int4*>(T.hpc + (size_t)k * kSysHead);
#pragma unroll
  for (int u = 0; u < kSysHead / 4; u++) {
    const int4 q = hp[u];
    f.pc[4 * u] = q.x, f.pc[4 * u + 1] = q.y, f.pc[4 * u + 2] = q.z, f.pc[4 * u + 3] = q.w;
  }
#pragma unroll
  for (int u = 0; u < kSysHead; u++) f.va[u] = T.hva[(size_t)k * kSysHead + u];
}
// level pointer j, or n past the last level
template <typename P>
__device__ __forceinline__ int sys_lvp(const SysTri<P>& T, int j) {
  return j <= T.nlev ? T.lvp[j] : T.n;
}
template <bool UPPER, typename P>
__device__ __forceinline__ void sys_row_solve(const SysTri<P>& T, const SysRowPF<P>& a, const P* rhs, P* out, P* buf,
                                              unsigned mask) {
  if (a.dst < 0) return;
  P s = a.rhs;
#pragma unroll
  for (int u = 0; u < kSysHead; u++)
    if (a.e0 + u < a.e1) s -= a.va[u] * buf[(unsigned)a.pc[u] & mask];
  for (int e = a.e0 + kSysHead; e < a.e1; e++) s -= T.va[e] * buf[(unsigned)T.pc[e] & mask];
  const P x = a.dg * s;
  buf[(unsigned)a.k & mask] = x;
  out[a.dst] = x;
  // rows past the first blockDim of a wide level
  for (int kk = a.k + blockDim.x; kk < a.kend; kk += blockDim.x) {
    P q = rhs[kk];
    const int f1 = T.rp[kk + 1];
    for (int e = T.rp[kk]; e < f1; e++) q -= T.va[e] * buf[(unsigned)T.pc[e] & mask];
    const P y = UPPER ? T.dinv[kk] * q : q;
    buf[(unsigned)kk & mask] = y;
    out[T.dst[kk]] = y;
  }
}
// MAXT: the CTA-size bound of the calling kernel; each build gets its own
// copy, compiled with that build's register budget
template <bool UPPER, int DEPTH, int MAXT, typename P>
__device__ __noinline__ void sys_trsv(const SysTri<P>& T, const P* rhs, P* out, P* buf, unsigned mask) {
  if (T.nlev == 0) return;
  SysRowPF<P> pf[DEPTH];
  int la[DEPTH], lb[DEPTH];  // slot d: level pointers of the level its next refill fetches
#pragma unroll
  for (int d = 0; d < DEPTH; d++) {
    sys_fetch_row<UPPER>(T, rhs, sys_lvp(T, d), sys_lvp(T, d + 1), pf[d]);
    la[d] = sys_lvp(T, d + DEPTH);
    lb[d] = sys_lvp(T, d + DEPTH + 1);
  }
  for (int t = 0; t < T.nlev; t += DEPTH) {
#pragma unroll
    for (int d = 0; d < DEPTH; d++) {
      if (t + d < T.nlev) {
        sys_row_solve<UPPER>(T, pf[d], rhs, out, buf, mask);
        sys_fetch_row<UPPER>(T, rhs, la[d], lb[d], pf[d]);  // level t + d + DEPTH
        la[d] = sys_lvp(T, t + d + 2 * DEPTH);
        lb[d] = sys_lvp(T, t + d + 2 * DEPTH + 1);
        __syncthreads();
      }
    }
  }
}

// x = U^-1 L^-1 rhs of level l (GemslrClass::SolveB): rhs is gathered into
// the lower factor's packed order, the lower pass writes its result in the
// upper factor's packed order and the upper pass writes x in row order.
// Each pass keeps its solved values in the CTA's shared ring when the
// factor's span fits (ring = the largest power of two within the shared
// buffer), else in the system's packed scratch vector.
template <int MAXT, typename P>
__device__ void sys_solve_b(const SysDesc<P>& d, int l, const P* rhs, P* x, P* sbuf, int scap, int depth,
                            unsigned long long* tri_ns) {
  const unsigned long long t0 = threadIdx.x == 0 ? sys_clock() : 0ull;
  const SysLevel<P>& v = d.lev[l];
  const unsigned ring = scap > 0 ? 1u << (31 - __clz(scap)) : 0u;
  const bool lr = v.L.span < (int)ring, ur = v.U.span < (int)ring;
  constexpr int G = 4;  // gathers in flight per thread
  for (int k0 = threadIdx.x; k0 < v.nl; k0 += G * blockDim.x) {
    int r[G];
#pragma unroll
    for (int g = 0; g < G; g++) r[g] = k0 + g * (int)blockDim.x < v.nl ? v.L.row[k0 + g * blockDim.x] : -1;
    P q[G];
#pragma unroll
    for (int g = 0; g < G; g++) q[g] = r[g] >= 0 ? rhs[r[g]] : P(0);
#pragma unroll
    for (int g = 0; g < G; g++)
      if (r[g] >= 0) d.yr[k0 + g * blockDim.x] = q[g];
  }
  __syncthreads();
  if (depth == 3) {
    sys_trsv<false, 3, MAXT>(v.L, (const P*)d.yr, d.yu, lr ? sbuf : d.y, lr ? ring - 1 : 0xFFFFFFFFu);
    sys_trsv<true, 3, MAXT>(v.U, (const P*)d.yu, x, ur ? sbuf : d.y, ur ? ring - 1 : 0xFFFFFFFFu);
  } else {
    sys_trsv<false, 2, MAXT>(v.L, (const P*)d.yr, d.yu, lr ? sbuf : d.y, lr ? ring - 1 : 0xFFFFFFFFu);
    sys_trsv<true, 2, MAXT>(v.U, (const P*)d.yu, x, ur ? sbuf : d.y, ur ? ring - 1 : 0xFFFFFFFFu);
  }
  if (threadIdx.x == 0) *tri_ns += sys_clock() - t0;
}

// x += WH (W^T x) in place (SolveApplyLowRankLevel, gemslr.cpp:3585-3590)
template <typename P>
__device__ void sys_lowrank(const SysLevel<P>& v, P* x, SysShared& sh) {
  sys_multidot(v.m, v.rank, v.W, v.m, (const double*)nullptr, x, 1.0, sh.red, sh.coef);
  sys_update<false>(v.m, v.rank, v.WH, v.m, (const double*)nullptr, sh.coef, 1.0, x, 1.0, x, sh);
}

// Orthogonalise column j+1 of the basis against columns 0..j by CGS2, then
// finish the Hessenberg column with the Givens rotations (one thread).
template <typename TV>
__device__ void sys_arnoldi(TV* Vb, long long ld, int j, FgmresDev* st, int nrows, SysShared& sh) {
  TV* w = Vb + (long long)(j + 1) * ld;
  sys_multidot(nrows, j + 1, Vb, ld, st->sc, w, 1.0, sh.red, sh.coef);
  for (int c = threadIdx.x; c <= j; c += blockDim.x) {
    st->hcol[c] = sh.coef[c];
    st->coefA[c] = sh.coef[c];
  }
  sys_update<false>(nrows, j + 1, Vb, ld, st->sc, sh.coef, -1.0, w, 1.0, w, sh);
  sys_multidot(nrows, j + 1, Vb, ld, st->sc, w, 1.0, sh.red, sh.coef2);
  for (int c = threadIdx.x; c <= j; c += blockDim.x) {
    st->hcol[c] += sh.coef2[c];
    st->coefB[c] = sh.coef2[c];
  }
  const double t2 = sys_update<true>(nrows, j + 1, Vb, ld, st->sc, sh.coef2, -1.0, w, 1.0, w, sh);
  __syncthreads();
  if (threadIdx.x == 0) fgmres_givens(st, j, sqrt(t2));
  __syncthreads();
}

template <int MAXT, typename P>
__device__ void sys_inner_solve(const SysDesc<P>& d, P* xl, const P* zl, FgmresDev* st, int S, SysShared& sh);

// GemslrClass::SolveLevel from level l0 down (gemslr.cpp:3474-3630) with the
// recursion unrolled: the descent keeps each level's right-hand side, the
// ascent finishes the levels bottom up.  x and rhs hold the trailing
// n - lev_ptr[l0] unknowns.  With INNER, level 0 runs the inner Schur FGMRES
// in place of the low-rank correction and the lower levels.
template <bool INNER, int MAXT, typename P>
__device__ void sys_solve_from(const SysDesc<P>& d, int l0, P* x, const P* rhs, FgmresDev* st_in, int S,
                               SysShared& sh) {
  const P* rh[kSysMaxLevels];
  P* xs[kSysMaxLevels];
  int l = l0;
  const P* r = rhs;
  P* xv = x;
  bool stop_inner = false;
  for (; l < d.nlev - 1; l++) {
    const SysLevel<P>& v = d.lev[l];
    rh[l] = r;
    xs[l] = xv;
    P* zu = v.z;
    P* zl = v.z + v.nl;
    if (d.usolve) {                                                   // U solve: zl = rhs_l
      for (int i = threadIdx.x; i < v.m; i += blockDim.x) zl[i] = r[v.nl + i];
      __syncthreads();
    } else {
      sys_solve_b<MAXT>(d, l, r, zu, (P*)sh.sbuf, sh.scap, sh.depth, &sh.tri_ns);  // 1. zu = B^-1 rhs_u
      sys_spmv<P>(v.E, (const P*)zu, P(-1), r + v.nl, P(1), zl, S);   // 2-3. zl = rhs_l - E zu
    }
    if (INNER && l == 0 && d.inner) {
      sys_inner_solve<MAXT>(d, xv + v.nl, zl, st_in, S, sh);                // 4. inner FGMRES
      stop_inner = true;
      break;
    }
    if (v.rank > 0) sys_lowrank(v, zl, sh);                           // 4. low rank
    r = zl;
    xv = xv + v.nl;
  }
  int top;
  if (stop_inner) {
    top = l;
  } else {
    sys_solve_b<MAXT>(d, d.nlev - 1, r, xv, (P*)sh.sbuf, sh.scap, sh.depth, &sh.tri_ns);  // last level
    top = d.nlev - 2;
  }
  for (int t = top; t >= l0; t--) {
    const SysLevel<P>& v = d.lev[t];
    P* zu = v.z;
    sys_spmv<P>(v.F, (const P*)(xs[t] + v.nl), P(-1), rh[t], P(1), zu, S);  // 5-6. zu = rhs_u - F xl
    sys_solve_b<MAXT>(d, t, zu, xs[t], (P*)sh.sbuf, sh.scap, sh.depth, &sh.tri_ns);  // 7. xu = B^-1 zu
  }
}

// Level-0 inner flexible GMRES on S0 = C0 - E0 B0^-1 F0 from x0 = 0, one cycle
// of inner_maxits steps (gemslr.cpp:1660-1674, 3566-3572); its preconditioner
// is the low-rank correction followed by the level-1 recursion
// (GemslrSchurMatrixClass::Solve, gemslr.cpp:294-330).
template <int MAXT, typename P>
__device__ void sys_inner_solve(const SysDesc<P>& d, P* xl, const P* zl, FgmresDev* st, int S, SysShared& sh) {
  const SysLevel<P>& v0 = d.lev[0];
  const int m0 = v0.m;
  const long long ld = m0;
  {
    double nrm[1] = {0.0};
    for (int i = threadIdx.x; i < m0; i += blockDim.x) {
      const P z = zl[i];
      d.Vin[i] = z;
      nrm[0] += (double)z * (double)z;
    }
    sys_block_sum<1>(nrm, sh.red, sh.tmp);
    if (threadIdx.x == 0) {
      const double normb = sqrt(sh.tmp[0]);
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
      } else {
        st->tolr = st->absolute ? st->tol : st->tol * normb;
        st->rs[0] = normb;
        st->sc[0] = 1.0 / normb;
      }
    }
    __syncthreads();
  }
  for (int j = 0; j < d.inner_maxits; j++) {
    if (*(volatile int*)&st->cycle_done) break;
    P* vj = d.Vin + (long long)j * ld;
    P* zj = d.Zin + (long long)j * ld;
    P* wj = d.Vin + (long long)(j + 1) * ld;
    const double scj = st->sc[j];
    if (v0.rank > 0) sys_multidot(m0, v0.rank, v0.W, ld, (const double*)nullptr, vj, scj, sh.red, sh.coef);
    sys_update<false>(m0, v0.rank, v0.WH, ld, (const double*)nullptr, sh.coef, 1.0, vj, scj, d.xlr, sh);
    sys_solve_from<false, MAXT>(d, 1, zj, (const P*)d.xlr, st, S, sh);
    // w = S0 z (GemslrClass::SchurMatVec, gemslr.cpp:3799-3960)
    sys_spmv<P>(v0.F, (const P*)zj, P(1), (const P*)nullptr, P(0), d.s_zu, S);
    sys_solve_b<MAXT>(d, 0, d.s_zu, d.s_wu, (P*)sh.sbuf, sh.scap, sh.depth, &sh.tri_ns);
    sys_spmv<P>(d.C0, (const P*)zj, P(1), (const P*)nullptr, P(0), wj, S);
    sys_spmv<P>(v0.E, (const P*)d.s_wu, P(-1), (const P*)wj, P(1), wj, S);
    sys_arnoldi(d.Vin, ld, j, st, m0, sh);
  }
  const int ni = *(volatile int*)&st->i;
  sys_update<false>(m0, ni, d.Zin, ld, (const double*)nullptr, st->rs, 1.0, (const P*)nullptr, 1.0, xl, sh);
}

// GemslrClass::Solve (gemslr.cpp:3431-3472): z = Q^T M^-1 P v with v scaled
template <int MAXT, typename P>
__device__ void sys_precond(const SysDesc<P>& d, const double* v, double vsc, P* z, FgmresDev* st_in, int S,
                            SysShared& sh) {
  for (int i = threadIdx.x; i < d.n; i += blockDim.x) d.rt[i] = (P)(v[d.pperm[i]] * vsc);
  __syncthreads();
  sys_solve_from<true, MAXT>(d, 0, d.xt, (const P*)d.rt, st_in, S, sh);
  const int* q = d.qperm ? d.qperm : d.pperm;
  for (int i = threadIdx.x; i < d.n; i += blockDim.x) z[q[i]] = d.xt[i];
  __syncthreads();
}

// MAXT bounds the CTA size the kernel is compiled for: 1024 leaves 64
// registers per thread; 256, with two CTAs per SM, leaves 128 (the
// autotuner tries both).
template <typename P, int MAXT>
__global__ void __launch_bounds__(MAXT, MAXT <= 256 ? 2 : 1) systems_fgmres_kernel(SysArgs<P> a) {
  __shared__ SysShared sh;
  extern __shared__ __align__(16) unsigned char sys_dyn[];
  if (threadIdx.x == 0) {
    sh.sbuf = sys_dyn;
    sh.scap = a.scap;
    sh.depth = a.depth;
  }
  __syncthreads();
  FgmresDev* st = a.st + blockIdx.x;
  FgmresDev* st_in = a.st_in + blockIdx.x;
  const int S = a.lanes;
  for (;;) {
    if (threadIdx.x == 0) sh.sys = (int)atomicAdd(a.next, 1u);
    __syncthreads();
    const int w = sh.sys;
    __syncthreads();
    if (w >= a.count) return;
    const int s = a.order[w];
    const SysDesc<P>& d = a.sys[s];
    const double* b = a.b[s];
    double* x = a.x[s];
    const int n = d.n;
    const long long ld = n;
    const unsigned long long t0 = sys_clock();
    if (threadIdx.x == 0) {
      sh.tri_ns = 0ull;
      st->kdim = a.kdim;
      st->maxits = a.maxits;
      st->tol = a.tol;
      st->absolute = a.atol;
      st->eps = DBL_EPSILON;
      st->done = 0;
      st->cycle_done = 1;
      st->i = 0;
      st->iter = 0;
      st->converged = 0;
      st->breakdown = 0;
      st->normr = 0.0;
      st_in->kdim = d.inner_maxits;
      st_in->maxits = d.inner_maxits;
      st_in->tol = d.inner_tol;
      st_in->absolute = 0;
      st_in->eps = DBL_EPSILON;
    }
    // ||b||  (fgmres.hpp:319-329)
    {
      double nrm[1] = {0.0};
      for (int i = threadIdx.x; i < n; i += blockDim.x) nrm[0] += b[i] * b[i];
      sys_block_sum<1>(nrm, sh.red, sh.tmp);
      if (threadIdx.x == 0) {
        st->normb = sqrt(sh.tmp[0]);
        if (st->normb < st->eps) {
          st->done = 1;
          st->cycle_done = 1;
        }
      }
      __syncthreads();
    }
    const bool zero_b = *(volatile int*)&st->done;
    if (!zero_b) {
      // v = b - A x, ||v|| (fgmres.hpp:331-360)
      sys_spmv<double>(d.A, (const double*)x, -1.0, b, 1.0, d.V, S);
      double nrm[1] = {0.0};
      for (int i = threadIdx.x; i < n; i += blockDim.x) nrm[0] += d.V[i] * d.V[i];
      sys_block_sum<1>(nrm, sh.red, sh.tmp);
      if (threadIdx.x == 0) {
        const double normr = sqrt(sh.tmp[0]);
        st->normr = normr;
        st->normr0 = normr;
        if (normr < st->eps) {
          st->done = 1;
          st->cycle_done = 1;
          st->converged = 1;
        } else {
          st->tolr = st->absolute ? st->tol : st->tol * st->normb;
          st->rs[0] = normr;
          st->sc[0] = 1.0 / normr;
          st->cycle_done = 0;
        }
      }
      __syncthreads();
    }
    const int max_cycles = a.maxits > 0 ? a.maxits / a.kdim + 2 : 0;
    for (int cyc = 0; cyc < max_cycles; cyc++) {
      if (*(volatile int*)&st->done || *(volatile int*)&st->iter >= a.maxits) break;
      for (int j = 0; j < a.kdim; j++) {
        if (*(volatile int*)&st->cycle_done) break;
        P* zj = d.Z + (long long)j * ld;
        sys_precond<MAXT>(d, d.V + (long long)j * ld, st->sc[j], zj, st_in, S, sh);           // z = M^-1 v
        sys_spmv<double>(d.A, (const P*)zj, 1.0, (const double*)nullptr, 0.0, d.V + (long long)(j + 1) * ld, S);
        sys_arnoldi(d.V, ld, j, st, n, sh);
      }
      // x += Z y  (fgmres.hpp:471-490)
      const int ni = *(volatile int*)&st->i;
      sys_update<false>(n, ni, d.Z, ld, (const double*)nullptr, st->rs, 1.0, (const double*)x, 1.0, x, sh);
      if (!*(volatile int*)&st->done)
        sys_spmv<double>(d.A, (const double*)x, -1.0, b, 1.0, d.V, S);                 // restart residual
      if (threadIdx.x == 0) {
        st->i = 0;
        if (!st->done) {
          st->cycle_done = 0;
          st->rs[0] = st->normr;
          st->sc[0] = 1.0 / st->normr;
        }
      }
      __syncthreads();
    }
    if (zero_b) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) x[i] = 0.0;
      __syncthreads();
    }
    // FP64 true residual ||b - A x||
    sys_spmv<double>(d.A, (const double*)x, -1.0, b, 1.0, d.V, S);
    {
      double nrm[1] = {0.0};
      for (int i = threadIdx.x; i < n; i += blockDim.x) nrm[0] += d.V[i] * d.V[i];
      sys_block_sum<1>(nrm, sh.red, sh.tmp);
    }
    if (threadIdx.x == 0) {
      SysResult r;
      r.iters = st->iter;
      r.converged = st->converged;
      r.breakdown = st->breakdown;
      r.pad = 0;
      r.normb = st->normb;
      r.normr = st->normr;
      r.true_r2 = sh.tmp[0];
      r.t0 = t0;
      r.t1 = sys_clock();
      r.tri_ns = sh.tri_ns;
      r.cta = blockIdx.x;
      r.pad2 = 0;
      a.res[s] = r;
    }
    __syncthreads();
  }
}

}  // namespace pgx
