// pgx — B200-native solve phase of ParGeMSLR's GeMSLR-preconditioned FGMRES.
//
// Host side: import and validation of the post-setup GeMSLR structures,
// level-set schedules, device layout, and the enqueue logic that mirrors the
// reference's solve-phase call tree:
//
//   FlexGmresClass::Solve                 (ParGeMSLR SRC/solvers/fgmres.hpp:263-558)
//     GemslrClass::Solve                  (SRC/preconditioners/gemslr.cpp:3431-3472)
//       GemslrClass::SolveLevel           (gemslr.cpp:3474-3630)
//         SolveB -> IluClass::SolveHost   (gemslr.cpp:3632-3678, ilu.cpp:3677-3790)
//         E/F MatVec                      (gemslr.cpp:3551-3555, 3595-3599)
//         SolveApplyLowRankLevel          (gemslr.cpp:3681-3722)
//         level-0 inner FlexGmres over GemslrSchurMatrixClass
//                                         (gemslr.cpp:282-330, 3566-3572, 3799-3960)
//
// All of it runs on one GPU; the host only enqueues kernels and reads the
// FGMRES state word once per restart cycle.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstddef>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <array>
#include <deque>
#include <memory>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/pgx.h"
#include "pgx_device.cuh"
#include "pgx_internal.h"
#include "pgx_umma.cuh"
#include "pgx_systems.cuh"
#include "pgx_params.h"
#include "pgx_setup.h"

namespace pgx {

// ------------------------------------------------------------ error state
static thread_local std::string g_last_error;
static thread_local int g_device = 0;

// streaming multiprocessors of the current device (queried once per device)
static int num_sms() {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
  if (dev < 64) {
    const int c = cache[dev].load(std::memory_order_relaxed);
    if (c > 0) return c;
  }
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 148;
  if (dev < 64) cache[dev].store(n, std::memory_order_relaxed);
  return n;
}

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int set_error(int code, const char* msg) {
  g_last_error = msg;
  return code;
}

// Runs an entry point's body so that no C++ exception crosses the C ABI: a
// failed host allocation becomes PGX_ERROR_OOM, any other exception
// PGX_ERROR_FUNCTION_CALL, each with its message.
template <class F>
static int guarded(const char* what, F&& body) {
  try {
    return body();
  } catch (const std::bad_alloc&) {
    return fail(PGX_ERROR_OOM, "%s: host allocation failed", what);
  } catch (const std::exception& e) {
    return fail(PGX_ERROR_FUNCTION_CALL, "%s: %s", what, e.what());
  } catch (...) {
    return fail(PGX_ERROR_FUNCTION_CALL, "%s: unexpected exception", what);
  }
}

#define PGX_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(e_ == cudaErrorMemoryAllocation ? PGX_ERROR_OOM : PGX_ERROR_CUDA, "%s: %s", \
                  #call, cudaGetErrorString(e_));                                            \
  } while (0)

#define PGX_TRY(expr)              \
  do {                             \
    int rc_ = (expr);              \
    if (rc_ != PGX_SUCCESS) return rc_; \
  } while (0)

// ---------------------------------------------------------- host structures
// A host CSR matrix.  Values are doubles; a complex matrix keeps each value
// as two doubles {re, im} (va has 2 * nnz entries), as the C ABI passes them.
struct HostCsr {
  int rows = 0, cols = 0;
  std::vector<int> rp, cj;
  std::vector<double> va;
  long long nnz() const { return (long long)cj.size(); }
  bool empty() const { return rows == 0; }
};

// Value k of a host array of doubles as the device scalar T: a real T takes
// va[k], a complex T the pair {va[2k], va[2k+1]}.
template <typename T>
static inline T hval(const double* va, size_t k) {
  if constexpr (Sc<T>::complex)
    return T((typename Sc<T>::real)va[2 * k], (typename Sc<T>::real)va[2 * k + 1]);
  else
    return (T)va[k];
}
// the first `count` values of a host array as device scalars
template <typename T>
static std::vector<T> hvals(const std::vector<double>& va, size_t count) {
  std::vector<T> out(count);
  for (size_t k = 0; k < count; k++) out[k] = hval<T>(va.data(), k);
  return out;
}

// vw: doubles per value (1 real, 2 complex)
static int copy_csr(const pgx_csr* in, HostCsr& out, const char* what, int vw = 1) {
  out = HostCsr();
  if (!in || in->rows == 0) return PGX_SUCCESS;
  if (in->rows < 0 || in->cols < 0 || in->nnz < 0 || !in->rowptr)
    return fail(PGX_ERROR_INVALID_PARAM, "%s: bad CSR header", what);
  if (in->nnz > 0 && (!in->colidx || !in->values))
    return fail(PGX_ERROR_INVALID_PARAM, "%s: missing CSR arrays", what);
  if (in->nnz > INT32_MAX) return fail(PGX_ERROR_INVALID_PARAM, "%s: nnz exceeds 32-bit indices", what);
  out.rows = in->rows;
  out.cols = in->cols;
  out.rp.assign(in->rowptr, in->rowptr + in->rows + 1);
  out.cj.assign(in->colidx, in->colidx + in->nnz);
  out.va.assign(in->values, in->values + in->nnz * vw);
  if (out.rp[0] != 0 || out.rp[in->rows] != in->nnz)
    return fail(PGX_ERROR_INVALID_PARAM, "%s: row pointer does not span nnz", what);
  for (int r = 0; r < out.rows; r++)
    if (out.rp[r + 1] < out.rp[r]) return fail(PGX_ERROR_INVALID_PARAM, "%s: row pointer decreases", what);
  for (long long k = 0; k < in->nnz; k++)
    if (out.cj[k] < 0 || out.cj[k] >= out.cols)
      return fail(PGX_ERROR_INVALID_PARAM, "%s: column index %d out of range", what, out.cj[k]);
  return PGX_SUCCESS;
}

struct HostLevel {
  bool set = false;
  int ncomp = 0;
  std::vector<int> dom_ptr;
  HostCsr L, U, B, E, F;
  std::vector<double> dinv, W, WH;
  int rank = 0;
};

// ------------------------------------------- level sets (BuildLevels rule)
// level(i) = 1 + max level of the entries row i depends on (0 if none);
// rows ordered by level, then by index (IluClass::BuildLevels,
// ParGeMSLR SRC/preconditioners/ilu.cpp:832-1062).  Lower factors are swept
// from the first row, upper factors from the last.
static int build_levels(bool upper, int n, const int* rp, const int* cj, std::vector<int>& level_ptr,
                        std::vector<int>& order, std::vector<int>* lev_out = nullptr) {
  std::vector<int> lev(n, -1);
  int max_level = 0;
  for (int t = 0; t < n; t++) {
    int i = upper ? n - 1 - t : t;
    int l = -1;
    for (int k = rp[i]; k < rp[i + 1]; k++) {
      int j = cj[k];
      if (upper ? (j <= i) : (j >= i))
        return fail(PGX_ERROR_INVALID_PARAM, "%s factor is not strictly %s triangular (row %d, col %d)",
                    upper ? "U" : "L", upper ? "upper" : "lower", i, j);
      l = std::max(l, lev[j]);
    }
    lev[i] = l + 1;
    max_level = std::max(max_level, lev[i]);
  }
  int nlev = n > 0 ? max_level + 1 : 0;
  level_ptr.assign(nlev + 1, 0);
  for (int i = 0; i < n; i++) level_ptr[lev[i] + 1]++;
  for (int l = 0; l < nlev; l++) level_ptr[l + 1] += level_ptr[l];
  order.assign(n, 0);
  std::vector<int> pos(level_ptr.begin(), level_ptr.end() - (nlev > 0 ? 1 : 0));
  for (int i = 0; i < n; i++) order[pos[lev[i]]++] = i;
  if (lev_out) lev_out->swap(lev);
  return PGX_SUCCESS;
}

static int pick_lanes(long long nnz, long long rows) {
  double avg = rows > 0 ? (double)nnz / (double)rows : 0.0;
  if (avg > 16) return 32;
  if (avg > 8) return 16;
  if (avg > 4) return 8;
  if (avg > 2) return 4;
  return 2;
}

// true if every entry is finite (host memory; OpenMP over large vectors)
static bool all_finite(const double* b, long long n) {
  int bad = 0;
#pragma omp parallel for reduction(| : bad) schedule(static) if (n >= (1LL << 16))
  for (long long i = 0; i < n; i++) bad |= !std::isfinite(b[i]);
  return !bad;
}

// The SpMV variant of a matrix, picked from its row-length histogram:
//   lanes per row S: the 90th-percentile row fits in one unrolled load batch
//     of the S lanes (S * kSpmvUnroll entries), so nine rows in ten need no
//     second round of gathers;
//   merge path instead of S lanes per row when the rows are skewed: the
//     longest row is more than 16 batches long and rows longer than four
//     batches hold more than a tenth of the nonzeros (a group of lanes would
//     serialise them while the short rows leave lanes idle).
struct SpmvPlan {
  int S = 2;
  bool merge = false;
};
static SpmvPlan spmv_plan(int rows, const int* rp) {
  SpmvPlan p;
  if (rows <= 0) return p;
  std::vector<int> len(rows);
  long long nnz = 0;
  int mx = 0;
  for (int r = 0; r < rows; r++) {
    len[r] = rp[r + 1] - rp[r];
    nnz += len[r];
    mx = std::max(mx, len[r]);
  }
  std::vector<int> sorted(len);
  const size_t q = (size_t)std::min<long long>(rows - 1, (long long)std::ceil(0.9 * rows) - 1);
  std::nth_element(sorted.begin(), sorted.begin() + q, sorted.end());
  const int p90 = sorted[q];
  while (p.S < 32 && p.S * kSpmvUnroll < p90) p.S *= 2;
  const int batch = p.S * kSpmvUnroll;
  long long heavy = 0;
  for (int r = 0; r < rows; r++)
    if (len[r] > 4 * batch) heavy += len[r];
  p.merge = mx > 16 * batch && heavy * 10 > nnz;
  return p;
}

// merge-path threads (kMergeItems items each) for a rows x nnz matrix
static int merge_threads(long long rows, long long nnz) { return (int)((rows + nnz + kMergeItems - 1) / kMergeItems); }

// Lanes per row of the per-subdomain solve: about PGX_PIPE_NNZ_PER_LANE nonzeros
// per lane, so that a row's operand loads are issued at once (kUnroll deep)
// and a level of a few dozen rows needs one sweep of the CTA's groups.  The
// choice depends on the factor alone, so every slot and lane count of a
// handle sums each row in the same order.
#ifndef PGX_PIPE_NNZ_PER_LANE
#define PGX_PIPE_NNZ_PER_LANE 4
#endif
static int pipe_lanes(long long nnz, long long rows) {
  const double avg = rows > 0 ? (double)nnz / (double)rows : 0.0;
  int S = 2;
  while (S < 16 && avg > (double)PGX_PIPE_NNZ_PER_LANE * S) S *= 2;
  return S;
}

// -------------------------------------------------------- device memory
struct Arena {
  std::vector<void*> ptrs;
  size_t bytes = 0;
  ~Arena() { release(); }
  void release() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
    bytes = 0;
  }
  template <typename T>
  int alloc(T** out, size_t count) {
    *out = nullptr;
    if (count == 0) count = 1;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? PGX_ERROR_OOM : PGX_ERROR_CUDA, "cudaMalloc(%zu): %s",
                  count * sizeof(T), cudaGetErrorString(e));
    ptrs.push_back(p);
    bytes += count * sizeof(T);
    *out = (T*)p;
    return PGX_SUCCESS;
  }
  template <typename T, typename U>
  int upload(T** out, const U* src, size_t count, cudaStream_t s) {
    PGX_TRY(alloc(out, count));
    if (count == 0) return PGX_SUCCESS;
    std::vector<T> tmp(src, src + count);
    PGX_CUDA(cudaMemcpyAsync(*out, tmp.data(), count * sizeof(T), cudaMemcpyHostToDevice, s));
    PGX_CUDA(cudaStreamSynchronize(s));
    return PGX_SUCCESS;
  }
  template <typename T>
  int zeros(T** out, size_t count, cudaStream_t s) {
    PGX_TRY(alloc(out, count));
    PGX_CUDA(cudaMemsetAsync(*out, 0, std::max<size_t>(count, 1) * sizeof(T), s));
    return PGX_SUCCESS;
  }
};

template <typename T>
struct DCsr {
  int rows = 0, cols = 0, S = 8;
  bool merge = false;  // merge-path SpMV (skewed rows) instead of S lanes per row
  long long nnz = 0;
  int *rp = nullptr, *cj = nullptr;
  T* va = nullptr;
};

template <typename T>
static int upload_csr(Arena& ar, const HostCsr& h, DCsr<T>& d, cudaStream_t s) {
  d.rows = h.rows;
  d.cols = h.cols;
  d.nnz = h.nnz();
  if (h.rows == 0) return PGX_SUCCESS;
  const SpmvPlan plan = spmv_plan(h.rows, h.rp.data());
  d.S = plan.S;
  d.merge = plan.merge;
  PGX_TRY(ar.upload(&d.rp, h.rp.data(), h.rp.size(), s));
  // column indices and values padded to whole 4-entry blocks (column 0,
  // value 0) for the 128-bit loads of the SpMV
  const size_t padded = (h.cj.size() + 3) / 4 * 4;
  std::vector<int> cj(h.cj);
  std::vector<T> va = hvals<T>(h.va, h.cj.size());
  cj.resize(std::max<size_t>(padded, 4), 0);
  va.resize(std::max<size_t>(padded, 4), T(0.0));
  PGX_TRY(ar.upload(&d.cj, cj.data(), cj.size(), s));
  PGX_TRY(ar.upload(&d.va, va.data(), va.size(), s));
  return PGX_SUCCESS;
}

// A triangular factor stored in padded level-set order.
template <typename T>
struct DTri {
  int n = 0, S = 32, ngroups = 0, nlevels = 0, nblocks = 1;
  int *ord = nullptr, *rp = nullptr, *cj = nullptr;
  T* va = nullptr;
  unsigned long long* ticket = nullptr;
  // segmented schedule (trsv_seg_kernel); seg == false uses trsv_kernel
  bool seg = false;
  bool comp = false;  // one CTA per subdomain (trsv_pipe_kernel)
  int nseg = 0, ncomp = 1;
  int *comp_ch0 = nullptr, *cmeta = nullptr, *far_col = nullptr;  // one-CTA-per-subdomain schedule
  T* dslot = nullptr;   // upper pass: inverse diagonal in slot order
  int* uslot = nullptr; // lower pass: upper-pass slot of each row, in slot order
  int nslots = 0;       // length of the slot arrays (padded row list)
  int nslots_up = 0;    // lower pass: length of the yslot vector it fills (the upper layout's nslots)
  long long nnz_total = 0;  // nonzeros of the factor (without padding)
  int *seg_row0 = nullptr, *seg_rp0 = nullptr, *seg_nnz0 = nullptr, *seg_lv0 = nullptr, *seg_nlvb = nullptr,
      *lvb = nullptr;
};

// persistent grid of the triangular solve: a few warps per group of an
// average level keeps the frontier busy without flooding L2 with pollers
static int tri_blocks(int ngroups, int nlevels) {
  const int wpb = 256 / kWarp;
  double avg = nlevels > 0 ? (double)ngroups / nlevels : (double)ngroups;
  long long warps = (long long)std::ceil(8.0 * avg);
  warps = std::max<long long>(warps, 64);
  warps = std::min<long long>(warps, (long long)num_sms() * 32);
  warps = std::min<long long>(warps, ((long long)ngroups + wpb - 1) / wpb * wpb);
  return (int)std::max<long long>(1, (warps + wpb - 1) / wpb);
}

template <typename T>
static int upload_tri(Arena& ar, const HostCsr& h, bool upper, DTri<T>& d, cudaStream_t s) {
  d.n = h.rows;
  d.nnz_total = h.nnz();
  if (d.n == 0) return PGX_SUCCESS;
  std::vector<int> lptr, order;
  PGX_TRY(build_levels(upper, h.rows, h.rp.data(), h.cj.data(), lptr, order));
  d.nlevels = (int)lptr.size() - 1;
  d.S = pick_lanes(h.nnz(), h.rows);
  const int G = kWarp / d.S;
  // padded schedule: each level starts on a group boundary
  std::vector<int> ord, rp(1, 0), cj;
  std::vector<T> va;
  ord.reserve(h.rows + (size_t)d.nlevels * G);
  cj.reserve(h.nnz());
  va.reserve(h.nnz());
  for (int l = 0; l < d.nlevels; l++) {
    for (int p = lptr[l]; p < lptr[l + 1]; p++) {
      int r = order[p];
      ord.push_back(r);
      for (int k = h.rp[r]; k < h.rp[r + 1]; k++) {
        cj.push_back(h.cj[k]);
        va.push_back(hval<T>(h.va.data(), k));
      }
      rp.push_back((int)cj.size());
    }
    while (ord.size() % G) {
      ord.push_back(-1);
      rp.push_back((int)cj.size());
    }
  }
  d.ngroups = (int)(ord.size() / G);
  d.nblocks = tri_blocks(d.ngroups, d.nlevels);
  PGX_TRY(ar.upload(&d.ord, ord.data(), ord.size(), s));
  PGX_TRY(ar.upload(&d.rp, rp.data(), rp.size(), s));
  PGX_TRY(ar.upload(&d.cj, cj.data(), cj.size(), s));
  PGX_TRY(ar.upload(&d.va, va.data(), va.size(), s));
  PGX_TRY(ar.zeros(&d.ticket, 2, s));
  return PGX_SUCCESS;
}

// Segmented schedule for trsv_seg_kernel.  Rows of each subdomain, in
// level-set order, are cut into segments that fit the kernel's shared-memory
// staging; segments are ordered by (position in the subdomain, subdomain), so
// a segment depends only on segments before it.  Each per-segment block of
// the flat arrays starts 16-byte aligned and has a 16-byte multiple length.
template <typename T>
static int upload_tri_seg(Arena& ar, const HostCsr& h, bool upper, const std::vector<int>& dom, DTri<T>& d,
                          cudaStream_t s) {
  const int n = h.rows;
  d.n = n;
  d.seg = true;
  d.nnz_total = h.nnz();
  std::vector<int> lptr, order, lev;
  PGX_TRY(build_levels(upper, n, h.rp.data(), h.cj.data(), lptr, order, &lev));
  d.nlevels = (int)lptr.size() - 1;
  d.S = pick_lanes(h.nnz(), n);
  const int NNZCAP = SegCfg<T>::nnz - 4, ROWCAP = kSegRows - 4;
  std::vector<int> cuts = dom;
  bool cuts_ok = cuts.size() >= 2 && cuts.front() == 0 && cuts.back() == n;
  for (size_t c = 0; cuts_ok && c + 1 < cuts.size(); c++) cuts_ok = cuts[c] <= cuts[c + 1];
  if (!cuts_ok) cuts = {0, n};
  {
    // the factor must be block diagonal over the subdomains: a segment may only
    // wait on earlier segments of its own subdomain
    std::vector<int> comp_of(n);
    for (size_t c = 0; c + 1 < cuts.size(); c++)
      for (int r = cuts[c]; r < cuts[c + 1]; r++) comp_of[r] = (int)c;
    for (int r = 0; r < n; r++)
      for (int k = h.rp[r]; k < h.rp[r + 1]; k++)
        if (comp_of[h.cj[k]] != comp_of[r]) {
          cuts = {0, n};
          r = n;
          break;
        }
  }
  struct Seg {
    int first_level, comp, idx;
    std::vector<int> rows;
  };
  std::vector<Seg> segs;
  for (size_t c = 0; c + 1 < cuts.size(); c++) {
    // rows of the subdomain ordered by (level, index): filter the global order
    Seg cur{-1, (int)c, 0, {}};
    long long nnz = 0;
    int idx = 0;
    for (int p = 0; p < n; p++) {
      const int r = order[p];
      if (r < cuts[c] || r >= cuts[c + 1]) continue;
      const int rn = h.rp[r + 1] - h.rp[r];
      if (rn > NNZCAP) return fail(PGX_ERROR_INVALID_PARAM, "row %d of a factor has %d entries (> %d)", r, rn, NNZCAP);
      if ((int)cur.rows.size() == ROWCAP || nnz + rn > NNZCAP) {
        segs.push_back(std::move(cur));
        cur = Seg{-1, (int)c, ++idx, {}};
        nnz = 0;
      }
      if (cur.rows.empty()) cur.first_level = lev[r];
      cur.rows.push_back(r);
      nnz += rn;
    }
    if (!cur.rows.empty()) segs.push_back(std::move(cur));
  }
  // claim order: round robin over the subdomains by segment index, so every
  // subdomain's chain of segments advances at the same rate (ordering by
  // level would starve subdomains whose segments span many thin levels);
  // within a subdomain the order is the schedule order
  std::stable_sort(segs.begin(), segs.end(), [](const Seg& a, const Seg& b) {
    if (a.idx != b.idx) return a.idx < b.idx;
    return a.comp < b.comp;
  });
  d.nseg = (int)segs.size();
  std::vector<int> seg_of(n, -1), slot_of(n, -1);
  for (int q = 0; q < d.nseg; q++)
    for (size_t i = 0; i < segs[q].rows.size(); i++) {
      seg_of[segs[q].rows[i]] = q;
      slot_of[segs[q].rows[i]] = (int)i;
    }
  auto pad4 = [](std::vector<int>& v, int fill) {
    while (v.size() % 4) v.push_back(fill);
  };
  std::vector<int> ord, rp, cj, lvb, row0(1, 0), rp0(1, 0), nnz0(1, 0), lv0(1, 0), nlvb;
  std::vector<T> va;
  for (int q = 0; q < d.nseg; q++) {
    const Seg& g = segs[q];
    for (int r : g.rows) ord.push_back(r);
    pad4(ord, -1);
    row0.push_back((int)ord.size());
    int acc = 0;
    rp.push_back(0);
    for (int r : g.rows) {
      for (int k = h.rp[r]; k < h.rp[r + 1]; k++) {
        const int j = h.cj[k];
        cj.push_back(seg_of[j] == q ? -(slot_of[j] + 1) : j);
        va.push_back(hval<T>(h.va.data(), k));
      }
      acc += h.rp[r + 1] - h.rp[r];
      rp.push_back(acc);
    }
    pad4(rp, acc);
    rp0.push_back((int)rp.size());
    while (cj.size() % 4) {
      cj.push_back(0);
      va.push_back(T(0.0));
    }
    nnz0.push_back((int)cj.size());
    const int base = (int)lvb.size();
    lvb.push_back(0);
    for (size_t i = 1; i < g.rows.size(); i++)
      if (lev[g.rows[i]] != lev[g.rows[i - 1]]) lvb.push_back((int)i);
    lvb.push_back((int)g.rows.size());
    nlvb.push_back((int)lvb.size() - base);
    pad4(lvb, (int)g.rows.size());
    lv0.push_back((int)lvb.size());
  }
  d.ncomp = (int)cuts.size() - 1;
  d.nblocks = std::max(1, std::min(d.nseg, num_sms()));
  PGX_TRY(ar.upload(&d.ord, ord.data(), ord.size(), s));
  PGX_TRY(ar.upload(&d.rp, rp.data(), rp.size(), s));
  PGX_TRY(ar.upload(&d.cj, cj.data(), cj.size(), s));
  PGX_TRY(ar.upload(&d.va, va.data(), va.size(), s));
  PGX_TRY(ar.upload(&d.lvb, lvb.data(), lvb.size(), s));
  PGX_TRY(ar.upload(&d.seg_row0, row0.data(), row0.size(), s));
  PGX_TRY(ar.upload(&d.seg_rp0, rp0.data(), rp0.size(), s));
  PGX_TRY(ar.upload(&d.seg_nnz0, nnz0.data(), nnz0.size(), s));
  PGX_TRY(ar.upload(&d.seg_lv0, lv0.data(), lv0.size(), s));
  PGX_TRY(ar.upload(&d.seg_nlvb, nlvb.data(), nlvb.size(), s));
  PGX_TRY(ar.zeros(&d.ticket, 2, s));
  return PGX_SUCCESS;
}

// Chunked per-subdomain schedule for trsv_pipe_kernel: each subdomain's
// rows in level-set order, cut into chunks that fit the kernel's staging
// buffers, subdomain after subdomain.  A dependency is encoded as the
// negative ring slot -(q % ring + 1) when its schedule position q is close
// enough that no row of the consumer's level can have overwritten the slot
// (end of the consumer's level - q < ring); otherwise as the row index, read
// back from global memory.  Returns PGX_ERROR_INVALID_PARAM (and builds
// nothing) when the factor couples two subdomains.
template <typename T, typename CC>
static int upload_tri_sub(Arena& ar, const HostCsr& h, bool upper, const std::vector<int>& dom, DTri<T>& d,
                          cudaStream_t s, const std::vector<double>* dinv, std::vector<int>* slot_of_row,
                          const std::vector<int>* upper_slot_of_row);
template <typename T>
static int upload_tri_comp(Arena& ar, const HostCsr& h, bool upper, const std::vector<int>& dom, DTri<T>& d,
                           cudaStream_t s, const std::vector<double>* dinv, std::vector<int>* slot_of_row,
                           const std::vector<int>* upper_slot_of_row) {
  return upload_tri_sub<T, PipeCfg<T, 1>>(ar, h, upper, dom, d, s, dinv, slot_of_row, upper_slot_of_row);
}

// The layout for a per-subdomain kernel whose shared-memory sizes are CC's.
template <typename T, typename CC>
static int upload_tri_sub(Arena& ar, const HostCsr& h, bool upper, const std::vector<int>& dom, DTri<T>& d,
                          cudaStream_t s, const std::vector<double>* dinv, std::vector<int>* slot_of_row,
                          const std::vector<int>* upper_slot_of_row) {
  const int n = h.rows;
  std::vector<int> lptr, order, lev;
  PGX_TRY(build_levels(upper, n, h.rp.data(), h.cj.data(), lptr, order, &lev));
  std::vector<int> cuts = dom;
  bool ok = cuts.size() >= 2 && cuts.front() == 0 && cuts.back() == n;
  for (size_t c = 0; ok && c + 1 < cuts.size(); c++) ok = cuts[c] <= cuts[c + 1];
  if (!ok) cuts = {0, n};
  const int ncomp = (int)cuts.size() - 1;
  std::vector<int> comp_of(n);
  for (int c = 0; c < ncomp; c++)
    for (int r = cuts[c]; r < cuts[c + 1]; r++) comp_of[r] = c;
  for (int r = 0; r < n; r++)
    for (int k = h.rp[r]; k < h.rp[r + 1]; k++)
      if (comp_of[h.cj[k]] != comp_of[r]) return PGX_ERROR_INVALID_PARAM;
  for (int r = 0; r < n; r++)
    if (h.rp[r + 1] - h.rp[r] > CC::nnz - 4) return PGX_ERROR_INVALID_PARAM;
  // positions inside each subdomain, in level order
  std::vector<std::vector<int>> sched(ncomp);
  for (int p = 0; p < n; p++) sched[comp_of[order[p]]].push_back(order[p]);
  std::vector<int> posc(n), lvl_end(n);
  for (int c = 0; c < ncomp; c++) {
    auto& sc = sched[c];
    for (size_t p = 0; p < sc.size(); p++) posc[sc[p]] = (int)p;
    // end position (exclusive) of each row's level
    size_t a = 0;
    while (a < sc.size()) {
      size_t e = a;
      while (e < sc.size() && lev[sc[e]] == lev[sc[a]]) e++;
      for (size_t p = a; p < e; p++) lvl_end[sc[p]] = (int)e;
      a = e;
    }
  }
  auto pad4 = [](std::vector<int>& v, int fill) {
    while (v.size() % 4) v.push_back(fill);
  };
  const int ROWCAP = CC::rows - 4, NNZCAP = CC::nnz - 4;
  // near operands stay in the shared ring until the consumer reads them:
  // within `ring` positions of the end of the consumer's level
  auto is_near = [&](int r, int qj) { return lvl_end[r] - qj < CC::ring; };
  std::vector<int> nfar(n, 0);
  for (int r = 0; r < n; r++)
    for (int k = h.rp[r]; k < h.rp[r + 1]; k++)
      if (!is_near(r, posc[h.cj[k]])) nfar[r]++;
  for (int r = 0; r < n; r++)
    if (nfar[r] > CC::far) return PGX_ERROR_INVALID_PARAM;
  std::vector<int> ord, rp, cj, lvb, meta, comp_ch0(1, 0), far_col;
  std::vector<T> va;
  auto push_meta = [&](int pos0) {
    meta.insert(meta.end(), {(int)ord.size(), (int)rp.size(), (int)cj.size(), (int)lvb.size(), pos0,
                             (int)far_col.size(), 0, 0});
  };
  for (int c = 0; c < ncomp; c++) {
    const auto& sc = sched[c];
    size_t p = 0;
    // starts of the previous chunk and of the one before it: a chunk's far
    // operands are gathered while the chunk two before it is solved, so they
    // must lie before that chunk's start
    int prev_start = 0, prev2_start = 0, chunk_in_comp = 0;
    while (p < sc.size()) {
      // one chunk: consecutive positions within the row, nonzero and far caps
      size_t e = p;
      long long nz = 0;
      int nf = 0;
      while (e < sc.size() && (int)(e - p) < ROWCAP) {
        const int rn = h.rp[sc[e] + 1] - h.rp[sc[e]];
        if (nz + rn > NNZCAP || nf + nfar[sc[e]] > CC::far) break;
        nz += rn;
        nf += nfar[sc[e]];
        e++;
      }
      push_meta((int)p);
      const int far_base = CC::ring + (chunk_in_comp % 3) * CC::far;
      const int far0 = (int)far_col.size();
      rp.push_back(0);
      int acc = 0;
      for (size_t q = p; q < e; q++) {
        const int r = sc[q];
        ord.push_back(r);
        for (int k = h.rp[r]; k < h.rp[r + 1]; k++) {
          const int j = h.cj[k];
          const int qj = posc[j];
          if (is_near(r, qj)) {
            cj.push_back(-((qj & (CC::ring - 1)) + 1));
          } else {
            // far: gathered while the chunk two before is solved, so it
            // must have been published before that chunk began
            if (qj >= prev2_start) return PGX_ERROR_INVALID_PARAM;
            cj.push_back(-(far_base + ((int)far_col.size() - far0) + 1));
            far_col.push_back(j);
          }
          va.push_back(hval<T>(h.va.data(), k));
        }
        acc += h.rp[r + 1] - h.rp[r];
        rp.push_back(acc);
      }
      pad4(ord, -1);
      pad4(rp, acc);
      pad4(far_col, -1);
      while (cj.size() % 4) {
        cj.push_back(0);
        va.push_back(T(0.0));
      }
      lvb.push_back(0);
      for (size_t q = p + 1; q < e; q++)
        if (lev[sc[q]] != lev[sc[q - 1]]) lvb.push_back((int)(q - p));
      lvb.push_back((int)(e - p));
      pad4(lvb, (int)(e - p));
      prev2_start = prev_start;
      prev_start = (int)p;
      chunk_in_comp++;
      p = e;
    }
    comp_ch0.push_back((int)meta.size() / 8);
  }
  push_meta(0);  // closes the last chunk
  for (int c : cj)
    if (c >= 0 || -c - 1 >= CC::ring + 3 * CC::far)
      if (c != 0) return fail(PGX_ERROR_INVALID_PARAM, "per-subdomain layout: operand index out of range");
  // every chunk is staged by bulk copies: each range starts on a 16-byte
  // boundary, spans a multiple of 16 bytes and fits its staging buffer
  for (size_t ch = 0; ch + 1 < meta.size() / 8; ch++) {
    const int* m = &meta[ch * 8];
    const int* e = &meta[(ch + 1) * 8];
    const int nr = e[0] - m[0], np = e[1] - m[1], nz = e[2] - m[2], nv = e[3] - m[3], nf = e[5] - m[5];
    const bool aligned = (m[0] | m[1] | m[2] | m[3] | m[5] | nr | np | nz | nv | nf) % 4 == 0;
    const bool fits = nr > 0 && nr <= CC::rows && np <= CC::rows + 4 && nv <= CC::rows + 4 && nz <= CC::nnz &&
                      nf <= CC::far && np > 0 && nv > 0 && nz >= 0 && nf >= 0;
    if (!aligned || !fits)
      return fail(PGX_ERROR_INVALID_PARAM, "per-subdomain layout: chunk %zu breaks the staging rules", ch);
  }
  // slot of every row in the flat row list; the upper pass's slots index its
  // dinv and the y the lower pass leaves behind
  std::vector<int> slot(n, -1);
  for (size_t i = 0; i < ord.size(); i++)
    if (ord[i] >= 0) slot[ord[i]] = (int)i;
  std::vector<T> dsl;
  std::vector<int> usl;
  if (upper) {
    dsl.assign(ord.size(), T(0.0));
    for (size_t i = 0; i < ord.size(); i++)
      if (ord[i] >= 0) dsl[i] = hval<T>(dinv->data(), ord[i]);
  } else {
    usl.assign(ord.size(), 0);
    for (size_t i = 0; i < ord.size(); i++)
      if (ord[i] >= 0) usl[i] = (*upper_slot_of_row)[ord[i]];
  }
  if (slot_of_row) *slot_of_row = slot;
  d.n = n;
  d.comp = true;
  d.seg = false;
  d.ncomp = ncomp;
  d.nslots = (int)ord.size();
  d.nlevels = (int)lptr.size() - 1;
  d.nseg = (int)meta.size() / 8 - 1;
  d.nnz_total = h.nnz();
  d.S = pipe_lanes(h.nnz(), n);
  d.nblocks = ncomp;
  PGX_TRY(ar.upload(&d.ord, ord.data(), ord.size(), s));
  PGX_TRY(ar.upload(&d.rp, rp.data(), rp.size(), s));
  PGX_TRY(ar.upload(&d.cj, cj.data(), cj.size(), s));
  PGX_TRY(ar.upload(&d.va, va.data(), va.size(), s));
  PGX_TRY(ar.upload(&d.lvb, lvb.data(), lvb.size(), s));
  PGX_TRY(ar.upload(&d.cmeta, meta.data(), meta.size(), s));
  PGX_TRY(ar.upload(&d.comp_ch0, comp_ch0.data(), comp_ch0.size(), s));
  PGX_TRY(ar.upload(&d.far_col, far_col.data(), far_col.size(), s));
  if (upper)
    PGX_TRY(ar.upload(&d.dslot, dsl.data(), dsl.size(), s));
  else
    PGX_TRY(ar.upload(&d.uslot, usl.data(), usl.size(), s));
  return PGX_SUCCESS;
}

// the segmented schedule pays off when segments hold many rows
static bool want_segments(const HostCsr& h, int nnz_cap) {
  if (h.rows == 0) return false;
  int maxlen = 0;
  for (int r = 0; r < h.rows; r++) maxlen = std::max(maxlen, h.rp[r + 1] - h.rp[r]);
  const double avg = (double)h.nnz() / h.rows;
  return maxlen <= nnz_cap - 4 && avg * 32.0 <= (double)nnz_cap;
}

template <typename P>
struct DLevel {
  int start = 0, nl = 0, m = 0, rank = 0;
  DTri<P> L, U;
  P* dinv = nullptr;
  P* y = nullptr;  // lower-pass result, holds the sentinel between solves
  P* yslot = nullptr;  // lower-pass result in the upper pass's slot order (per-subdomain kernels)
  DCsr<P> E, F;
  DCsr<P> B;            // the level's unfactored blocks (multiplicative solve only)
  P* wmul = nullptr;    // nl: work vector of the multiplicative solve
  P *W = nullptr, *WH = nullptr;
  P *z = nullptr, *xlr = nullptr;
  TsAcc<P>* lrt = nullptr;  // low-rank coefficients W^H x
};

template <typename T>
static std::string describe_tri(const char* what, const DTri<T>& t) {
  char buf[256];
  if (t.n == 0) {
    snprintf(buf, sizeof(buf), "  %s: empty\n", what);
  } else if (t.comp) {
    snprintf(buf, sizeof(buf), "  %s: per-subdomain pipeline, %d CTAs, %d lanes per row, %d dependency levels, %d chunks, %lld nonzeros\n",
             what, t.ncomp, t.S, t.nlevels, t.nseg, t.nnz_total);
  } else if (t.seg) {
    snprintf(buf, sizeof(buf), "  %s: segmented, %d segments, %d CTAs, %d lanes per row, %d dependency levels\n", what,
             t.nseg, t.nblocks, t.S, t.nlevels);
  } else {
    snprintf(buf, sizeof(buf), "  %s: level-set, %d groups, %d CTAs, %d lanes per row, %d dependency levels\n", what,
             t.ngroups, t.nblocks, t.S, t.nlevels);
  }
  return buf;
}
template <typename T>
static std::string describe_csr(const char* what, const DCsr<T>& m) {
  char buf[192];
  if (m.rows == 0) return std::string();
  snprintf(buf, sizeof(buf), "  %s: %d x %d, %lld nonzeros, SpMV %s\n", what, m.rows, m.cols, m.nnz,
           m.merge ? "merge path" : (std::to_string(m.S) + " lanes per row").c_str());
  return buf;
}

static inline Skip mk_skip(const int* a = nullptr, const int* b = nullptr, const int* c = nullptr) {
  Skip s;
  s.f0 = a;
  s.f1 = b;
  s.f2 = c;
  return s;
}

static inline int grid_for(long long work, int per_block, int cap) {
  long long g = (work + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

// ---------------------------------------------------------------- engine
struct Import {
  int n = 0, precision = 0, nlev = 0;
  int vw = 1;  // doubles per value: 1 real, 2 complex
  HostCsr A;
  std::vector<int> pperm, qperm, lev_ptr;
  std::vector<HostLevel> levels;
  int inner_enable = 0, inner_maxits = 5;
  double inner_tol = 1e-2;
  // the solve option of GemslrClass (PARGEMSLR_IO_ADVANCED_GLOBAL_SOLVE,
  // gemslr.hpp:120-128): 0 the additive LU solve, 1 the U solve
  int solve_option = 0;
};

// The C block below level l, C_l (the operator of GemslrClass::SchurMatVec,
// gemslr.cpp:3799-3960): the B, E and F blocks of the levels after l,
// assembled over the trailing n - lev_ptr[l+1] unknowns.
static HostCsr host_c_block(const Import& im, int l) {
  const int base = im.lev_ptr[l + 1];
  const int m = im.n - base;
  const int vw = im.vw;
  // (column, value) with the value as {re, im} (im 0 for a real matrix)
  std::vector<std::vector<std::pair<int, std::pair<double, double>>>> rows(m);
  auto add = [&](const HostCsr& M, int roff, int coff) {
    for (int r = 0; r < M.rows; r++)
      for (int k = M.rp[r]; k < M.rp[r + 1]; k++)
        rows[roff + r].push_back({coff + M.cj[k], {M.va[(size_t)vw * k], vw == 2 ? M.va[(size_t)vw * k + 1] : 0.0}});
  };
  for (int j = l + 1; j < im.nlev; j++) {
    const HostLevel& h = im.levels[j];
    const int o = im.lev_ptr[j] - base, o1 = im.lev_ptr[j + 1] - base;
    add(h.B, o, o);
    if (j < im.nlev - 1) {
      add(h.F, o, o1);
      add(h.E, o1, o);
    }
  }
  HostCsr c;
  c.rows = c.cols = m;
  c.rp.assign(m + 1, 0);
  for (int r = 0; r < m; r++) {
    std::sort(rows[r].begin(), rows[r].end());
    for (auto& e : rows[r]) {
      c.cj.push_back(e.first);
      c.va.push_back(e.second.first);
      if (vw == 2) c.va.push_back(e.second.second);
    }
    c.rp[r + 1] = (int)c.cj.size();
  }
  return c;
}

struct EngineBase {
  virtual ~EngineBase() {}
  virtual int kernel_stats(int which, int level, int reps, double* avg_ms, double* bytes, int* launches) = 0;
  virtual int build_lowrank_level(Import& im, int l, int k, int its, unsigned long long seed) = 0;
  virtual int solve(double* x, const double* b, int location, int kdim, int maxits, double tol, int atol,
                    pgx_result* res) = 0;
  virtual int apply(double* z, const double* v, int location) = 0;
  virtual int64_t device_bytes(int kdim) const = 0;
  // a solve slot: begin() enqueues the start of a solve and its first
  // restart cycle, poll() advances it by at most one cycle
  virtual int64_t slot_bytes(int kdim) const = 0;
  // prechecked: a host b was already checked for NaN/Inf by the caller
  virtual int begin(double* x, const double* b, int location, int kdim, int maxits, double tol, int atol,
                    bool prechecked = false) = 0;
  virtual int poll(bool block, bool* finished, pgx_result* res) = 0;
  virtual int make_clone(std::unique_ptr<EngineBase>& out) = 0;
  virtual int solve_fixed_basis(double* x, const double* b, int location, int kdim, int maxits, double tol,
                                int atol, void* pool, size_t pool_bytes, pgx_result* res) = 0;
  // right-hand sides the slot advances together; poll() then fills lanes()
  // results
  virtual int lanes() const { return 1; }
  // device bytes of the multi-lane factor layouts this handle keeps, and their release
  virtual int64_t layout_bytes() const { return 0; }
  virtual void release_layouts() {}
  // another slot over the same factors advancing `lanes` right-hand sides together
  virtual int make_lanes_clone(Import& im, int lanes, std::unique_ptr<EngineBase>& out) {
    (void)im;
    (void)lanes;
    (void)out;
    return fail(PGX_ERROR_FUNCTION_CALL, "slots are cloned from the handle itself");
  }
  // polls before a triangular-solve dependency wait gives up; captured
  // restart cycles are rebuilt with the new bound
  virtual void set_wait_limit(int polls) = 0;
  // relative Givens residual estimates of the slot's last solve
  virtual std::vector<double> residual_history() const { return std::vector<double>(); }
  // one line per structure: which kernel and layout each pass and SpMV uses
  virtual std::string describe() const { return std::string(); }
  virtual int begin_many(int count, double* const* x, const double* const* b, int location, int kdim, int maxits,
                         double tol, int atol, bool prechecked = false) {
    if (count != 1) return fail(PGX_ERROR_INVALID_PARAM, "this slot solves one right-hand side at a time");
    return begin(x[0], b[0], location, kdim, maxits, tol, atol, prechecked);
  }
};


template <typename P>
struct Engine;
template <typename P>
int make_batch_slot(Engine<P>& own, Import& im, int lanes, std::unique_ptr<EngineBase>& out);
constexpr int kMaxLanes = 16;  // right-hand sides one slot advances together

template <typename P>
struct Engine : EngineBase {
  // F: the scalar of the outer FGMRES (double, or cf64 when the factors are
  // complex); SD: its device state.  The inner FGMRES accumulates in the same
  // type (TsAcc<P> == F for every P).
  using F = std::conditional_t<Sc<P>::complex, cf64, double>;
  using SD = FgmresDevT<F>;
  static constexpr int VW = Sc<P>::complex ? 2 : 1;  // doubles per value at the C ABI
  int n = 0, nlev = 0;
  std::vector<int> lev_ptr;
  cudaStream_t stream = nullptr;
  // ar: factors and operators, uploaded once by the owning slot and read by
  // every clone; wk: this slot's work vectors; krylov: this slot's basis
  Arena ar, wk, krylov;
  bool owner = true;
  int kdim_alloc = 0;
  DCsr<F> A;
  int *pperm = nullptr, *qperm = nullptr;
  std::vector<DLevel<P>> lv;
  // level-0 Schur-complement operator C0 x - E0 B0^-1 F0 x and its work space
  DCsr<P> C0;
  P *s_zu = nullptr, *s_wu = nullptr;
  // inner FGMRES on level 0
  int inner = 0, inner_maxits = 5;
  // U solve (GemslrClass::SolveLevel, gemslr.cpp:3527-3532): in the solve
  // phase a level skips its block-L part, z = rhs; the setup phase (the
  // low-rank build) always runs the LU sequence
  int usolve = 0;
  // multiplicative solve of ParallelGemslrClass (SolveLevelGemslrMul,
  // parallel_gemslr.cpp:5816-6050), its inner iteration on the RAP operator
  // (RAPMatVec, :7194); the inner preconditioner stays the additive level
  // solve (ParallelGemslrSchurMatrixClass::Solve, :370-410)
  int mul = 0;
  double inner_tol = 1e-2;
  P *Vin = nullptr, *Zin = nullptr;
  SD* st_in = nullptr;
  // outer FGMRES
  F* V = nullptr;
  P* Z = nullptr;
  SD* st = nullptr;
  F *bdev = nullptr, *xdev = nullptr, *rdev = nullptr, *scal = nullptr;
  P *rt = nullptr, *xt = nullptr;
  F* partial = nullptr;
  unsigned int* counter = nullptr;
  // merge-path SpMV carries of this slot (rows and partial sums, one per
  // thread of the largest merge-path matrix); null if no matrix uses it
  int* mcarry_row = nullptr;
  F* mcarry_val = nullptr;
  int* err = nullptr;
  int spin_limit = kSpinLimit;  // polls before a dependency wait gives up (pgx_gemslr_set_wait_limit)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_poll = nullptr;
  SD* hs_pin = nullptr;  // pinned copy of the FGMRES state header
  double* r2_pin = nullptr;     // pinned copy of the final residual norm
  double* hist_pin = nullptr;   // pinned copy of one cycle's residual estimates
  // Givens residual estimates of the last solve driven by begin()/poll() or
  // the static-basis solve: ||r0||, then one per iteration
  std::vector<double> history;
  int hist_iters = 0;
  double hist_normb = 0.0;
  // one FGMRES restart cycle captured as a CUDA graph, keyed by its arguments
  cudaGraphExec_t cycle_exec = nullptr;
  int cycle_nodes = 0;  // kernels in one captured cycle
  int g_kdim = -1;
  const void *g_x = nullptr, *g_b = nullptr;

  void drop_graph() {
    if (cycle_exec) cudaGraphExecDestroy(cycle_exec);
    cycle_exec = nullptr;
    g_kdim = -1;
  }

  ~Engine() override {
    if (stream) cudaStreamSynchronize(stream);
    drop_graph();
    ar.release();
    wk.release();
    krylov.release();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (ev_poll) cudaEventDestroy(ev_poll);
    if (hs_pin) cudaFreeHost(hs_pin);
    if (r2_pin) cudaFreeHost(r2_pin);
    if (hist_pin) cudaFreeHost(hist_pin);
    if (stream) cudaStreamDestroy(stream);
  }

  bool use_seg = true;

  // dynamic shared memory of the per-subdomain solve for R right-hand sides
  template <int R>
  static int set_pipe_smem() {
    const int bytes = (int)PipeCfg<P, R>::bytes;
#define PGX_PIPEATTR(SS)                                                                                     \
  PGX_CUDA(cudaFuncSetAttribute(trsv_pipe_kernel<P, SS, false, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                bytes));                                                                     \
  PGX_CUDA(cudaFuncSetAttribute(trsv_pipe_kernel<P, SS, true, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))
    PGX_PIPEATTR(2);
    PGX_PIPEATTR(4);
    PGX_PIPEATTR(8);
    PGX_PIPEATTR(16);
#undef PGX_PIPEATTR
    return PGX_SUCCESS;
  }

  // the per-subdomain solve of factor T for R right-hand sides
  template <int R>
  static void launch_pipe(const DTri<P>& T, bool upper, const PtrR<P, R>& yslot, const PtrR<P, R>& rhs,
                          const PtrR<P, R>& y, const PtrR<P, R>& x, int* err, const SkipR<R>& sk, cudaStream_t st) {
    const size_t bytes = PipeCfg<P, R>::bytes;
    CompArrays ca;
    ca.meta = (const int4*)T.cmeta;
    ca.ord = T.ord;
    ca.rp = T.rp;
    ca.cj = T.cj;
    ca.lvb = T.lvb;
    ca.uslot = T.uslot;
    ca.far_col = T.far_col;
#define PGX_PIPE(SS)                                                                                             \
  if (upper)                                                                                                     \
    trsv_pipe_kernel<P, SS, true, R><<<T.ncomp, kPipeThreads, bytes, st>>>(                                       \
        T.n, T.nslots_up, T.comp_ch0, ca, T.va, T.dslot, yslot, rhs, y, x, err, sk);                               \
  else                                                                                                           \
    trsv_pipe_kernel<P, SS, false, R><<<T.ncomp, kPipeThreads, bytes, st>>>(                                      \
        T.n, T.nslots_up, T.comp_ch0, ca, T.va, T.dslot, yslot, rhs, y, x, err, sk)
    switch (T.S) {
      case 2: PGX_PIPE(2); break;
      case 4: PGX_PIPE(4); break;
      case 8: PGX_PIPE(8); break;
      default: PGX_PIPE(16); break;
    }
#undef PGX_PIPE
  }

  int set_seg_smem() {
    const int bytes = (int)SegCfg<P>::bytes;
#define PGX_SEGATTR(SS)                                                                                     \
  PGX_CUDA(cudaFuncSetAttribute(trsv_seg_kernel<P, SS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)); \
  PGX_CUDA(cudaFuncSetAttribute(trsv_seg_kernel<P, SS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes))
    PGX_SEGATTR(2);
    PGX_SEGATTR(4);
    PGX_SEGATTR(8);
    PGX_SEGATTR(16);
    PGX_SEGATTR(32);
#undef PGX_SEGATTR
    PGX_TRY(set_pipe_smem<1>());
    return PGX_SUCCESS;
  }

  int64_t device_bytes(int kdim) const override { return (int64_t)ar.bytes + slot_bytes(kdim); }

  int64_t slot_bytes(int kdim) const override {
    return (int64_t)wk.bytes + (int64_t)n * (kdim + 1) * (sizeof(F) + sizeof(P));
  }

  // ------------------------------------------------------------ commit
  // The factors and operators are uploaded once; every solve slot (this
  // engine and its clones) adds its own stream and work space.
  int commit(Import& im) {
    PGX_TRY(set_seg_smem());
    PGX_TRY(init_stream());
    PGX_TRY(upload_factors(im));
    PGX_TRY(alloc_work());
    PGX_CUDA(cudaStreamSynchronize(stream));
    PGX_TRY(autotune());
    return PGX_SUCCESS;
  }

  int init_stream() {
    PGX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    PGX_CUDA(cudaEventCreate(&ev0));
    PGX_CUDA(cudaEventCreate(&ev1));
    PGX_CUDA(cudaEventCreateWithFlags(&ev_poll, cudaEventDisableTiming));
    PGX_CUDA(cudaMallocHost((void**)&hs_pin, sizeof(SD)));
    PGX_CUDA(cudaMallocHost((void**)&r2_pin, sizeof(double)));
    PGX_CUDA(cudaMallocHost((void**)&hist_pin, sizeof(double) * KMAX));
    memset(hs_pin, 0, sizeof(SD));
    *r2_pin = 0.0;
    return PGX_SUCCESS;
  }

  int upload_factors(Import& im) {
    n = im.n;
    nlev = im.nlev;
    lev_ptr = im.lev_ptr;
    PGX_TRY(upload_csr(ar, im.A, A, stream));
    PGX_TRY(ar.upload(&pperm, im.pperm.data(), im.pperm.size(), stream));
    if (!im.qperm.empty()) PGX_TRY(ar.upload(&qperm, im.qperm.data(), im.qperm.size(), stream));
    lv.resize(nlev);
    for (int l = 0; l < nlev; l++) {
      HostLevel& h = im.levels[l];
      DLevel<P>& d = lv[l];
      d.start = lev_ptr[l];
      d.nl = lev_ptr[l + 1] - lev_ptr[l];
      d.m = n - lev_ptr[l + 1];
      int rcL = PGX_ERROR_INVALID_PARAM, rcU = PGX_ERROR_INVALID_PARAM;
      if (h.L.rows > 0) {
        std::vector<int> uslot_of_row;
        rcU = upload_tri_comp(ar, h.U, true, h.dom_ptr, d.U, stream, &h.dinv, &uslot_of_row, nullptr);
        if (rcU == PGX_SUCCESS)
          rcL = upload_tri_comp(ar, h.L, false, h.dom_ptr, d.L, stream, nullptr, nullptr, &uslot_of_row);
        d.L.nslots_up = d.U.nslots_up = d.U.nslots;
      }
      if (rcL == PGX_SUCCESS && rcU == PGX_SUCCESS) {
        // one CTA per subdomain; y travels from the lower to the upper pass in slot order
      } else if (use_seg && want_segments(h.L, SegCfg<P>::nnz) && want_segments(h.U, SegCfg<P>::nnz)) {
        d.L = DTri<P>();
        d.U = DTri<P>();
        PGX_TRY(upload_tri_seg(ar, h.L, false, h.dom_ptr, d.L, stream));
        PGX_TRY(upload_tri_seg(ar, h.U, true, h.dom_ptr, d.U, stream));
      } else {
        d.L = DTri<P>();
        d.U = DTri<P>();
        PGX_TRY(upload_tri(ar, h.L, false, d.L, stream));
        PGX_TRY(upload_tri(ar, h.U, true, d.U, stream));
      }
      {
        const std::vector<P> dv = hvals<P>(h.dinv, (size_t)d.nl);
        PGX_TRY(ar.upload(&d.dinv, dv.data(), dv.size(), stream));
      }
      if (l < nlev - 1) {
        PGX_TRY(upload_csr(ar, h.E, d.E, stream));
        PGX_TRY(upload_csr(ar, h.F, d.F, stream));
        if (im.solve_option == 2) {
          if (h.B.rows != d.nl)
            return fail(PGX_ERROR_INVALID_PARAM, "the multiplicative solve needs the B blocks of level %d", l);
          PGX_TRY(upload_csr(ar, h.B, d.B, stream));
        }
        d.rank = h.rank;
        if (d.rank > 0) {
          const std::vector<P> w = hvals<P>(h.W, (size_t)d.m * d.rank), wh = hvals<P>(h.WH, (size_t)d.m * d.rank);
          PGX_TRY(ar.upload(&d.W, w.data(), w.size(), stream));
          PGX_TRY(ar.upload(&d.WH, wh.data(), wh.size(), stream));
        }
      }
    }
    inner = (im.inner_enable && nlev >= 2) ? 1 : 0;
    usolve = im.solve_option == 1 ? 1 : 0;
    mul = im.solve_option == 2 ? 1 : 0;
    inner_maxits = im.inner_maxits;
    inner_tol = im.inner_tol;
    if (inner) PGX_TRY(assemble_c0(im));
    return PGX_SUCCESS;
  }

  // the work space of one solve slot
  int alloc_work() {
    for (int l = 0; l < nlev; l++) {
      DLevel<P>& d = lv[l];
      if (d.L.comp) PGX_TRY(wk.zeros(&d.yslot, (size_t)d.U.nslots, stream));
      if (!owner) {
        // the level-set and segmented kernels count their CTAs per slot
        if (d.L.ticket) PGX_TRY(wk.zeros(&d.L.ticket, 2, stream));
        if (d.U.ticket) PGX_TRY(wk.zeros(&d.U.ticket, 2, stream));
      }
      PGX_TRY(wk.alloc(&d.y, (size_t)d.nl));
      sentinel_fill_kernel<P><<<grid_for(d.nl, 256, num_sms() * 8), 256, 0, stream>>>(d.nl, d.y);
      PGX_CUDA(cudaGetLastError());
      if (l < nlev - 1) {
        PGX_TRY(wk.zeros(&d.xlr, (size_t)d.m, stream));
        PGX_TRY(wk.zeros(&d.lrt, (size_t)KMAX + 1, stream));
      }
      PGX_TRY(wk.zeros(&d.z, (size_t)(n - d.start), stream));
      if (mul && l < nlev - 1) PGX_TRY(wk.zeros(&d.wmul, (size_t)d.nl, stream));
    }
    if (inner) {
      const int m0 = lv[0].m;
      PGX_TRY(wk.zeros(&s_zu, (size_t)lv[0].nl, stream));
      PGX_TRY(wk.zeros(&s_wu, (size_t)lv[0].nl, stream));
      PGX_TRY(wk.zeros(&Vin, (size_t)m0 * (inner_maxits + 1), stream));
      PGX_TRY(wk.zeros(&Zin, (size_t)m0 * (inner_maxits + 1), stream));
      PGX_TRY(wk.zeros(&st_in, 1, stream));
      SD h;
      memset(&h, 0, sizeof(h));
      h.kdim = inner_maxits;
      h.maxits = inner_maxits;
      h.tol = inner_tol;
      h.eps = std::is_same<typename Sc<P>::real, float>::value ? (double)FLT_EPSILON : DBL_EPSILON;
      *hs_pin = h;
      PGX_CUDA(cudaMemcpyAsync(st_in, hs_pin, sizeof(h), cudaMemcpyHostToDevice, stream));
      PGX_CUDA(cudaStreamSynchronize(stream));
    }
    PGX_TRY(wk.zeros(&st, 1, stream));
    PGX_TRY(wk.zeros(&bdev, (size_t)n, stream));
    PGX_TRY(wk.zeros(&xdev, (size_t)n, stream));
    PGX_TRY(wk.zeros(&rdev, (size_t)n, stream));
    PGX_TRY(wk.zeros(&scal, 8, stream));
    PGX_TRY(wk.zeros(&rt, (size_t)n, stream));
    PGX_TRY(wk.zeros(&xt, (size_t)n, stream));
    PGX_TRY(wk.zeros(&partial, (size_t)(KMAX + 1) * kTsMaxBlocks, stream));
    PGX_TRY(wk.zeros(&counter, 1, stream));
    PGX_TRY(wk.zeros(&err, 1, stream));
    int mthreads = 0;
    auto need = [&](const DCsr<P>& M) {
      if (M.merge) mthreads = std::max(mthreads, merge_threads(M.rows, M.nnz));
    };
    if (A.merge) mthreads = std::max(mthreads, merge_threads(A.rows, A.nnz));
    for (int l = 0; l < nlev; l++) {
      need(lv[l].E);
      need(lv[l].F);
    }
    need(C0);
    if (mthreads > 0) {
      PGX_TRY(wk.alloc(&mcarry_row, (size_t)mthreads));
      PGX_TRY(wk.alloc(&mcarry_val, (size_t)mthreads));
    }
    return PGX_SUCCESS;
  }

  // another solve slot over the same factors (the owner must outlive it)
  int clone_from(const Engine& s) {
    owner = false;
    n = s.n;
    nlev = s.nlev;
    lev_ptr = s.lev_ptr;
    A = s.A;
    pperm = s.pperm;
    qperm = s.qperm;
    lv = s.lv;  // factor pointers are shared, work pointers are replaced by alloc_work
    C0 = s.C0;
    inner = s.inner;
    usolve = s.usolve;
    mul = s.mul;
    inner_maxits = s.inner_maxits;
    inner_tol = s.inner_tol;
    use_seg = s.use_seg;
    spin_limit = s.spin_limit;
    PGX_TRY(init_stream());
    PGX_TRY(alloc_work());
    PGX_CUDA(cudaStreamSynchronize(stream));
    return PGX_SUCCESS;
  }

  // Autotuner: the persistent grid of each large segmented factor is picked
  // by timing the lower/upper pass pair at a few sizes (the number of
  // segments kept in flight per subdomain trades staging overlap against
  // idle CTAs holding shared memory).
  int autotune() {
    Skip sk = mk_skip();
    for (int l = 0; l < nlev; l++) {
      DLevel<P>& d = lv[l];
      if (!d.L.seg || !d.U.seg || d.nl < 32768) continue;  // one-CTA-per-subdomain kernels have no grid choice
      const int comps = std::max(d.L.ncomp, 1);
      std::vector<int> cand;
      const int sms = num_sms();
      for (int f : {2, 4, 8, 16}) cand.push_back(std::min(sms, comps * f));
      cand.push_back(sms);
      std::sort(cand.begin(), cand.end());
      cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
      int bestL = d.L.nblocks, bestU = d.U.nblocks;
      float tL = 1e30f, tU = 1e30f;
      for (int g : cand) {
        d.L.nblocks = std::min(g, d.L.nseg);
        d.U.nblocks = std::min(g, d.U.nseg);
        float mL = 0.f, mU = 0.f;
        for (int rep = 0; rep < 3; rep++) {
          PGX_CUDA(cudaEventRecord(ev0, stream));
          trsv(d.L, false, nullptr, rt + d.start, nullptr, d.y, xt + d.start, sk, d.yslot);
          PGX_CUDA(cudaEventRecord(ev1, stream));
          PGX_CUDA(cudaStreamSynchronize(stream));
          float a = 0.f;
          PGX_CUDA(cudaEventElapsedTime(&a, ev0, ev1));
          PGX_CUDA(cudaEventRecord(ev0, stream));
          trsv(d.U, true, d.dinv, nullptr, nullptr, d.y, xt + d.start, sk, d.yslot);
          PGX_CUDA(cudaEventRecord(ev1, stream));
          PGX_CUDA(cudaStreamSynchronize(stream));
          float b = 0.f;
          PGX_CUDA(cudaEventElapsedTime(&b, ev0, ev1));
          if (rep > 0) {
            mL += a;
            mU += b;
          }
        }
        if (mL < tL) {
          tL = mL;
          bestL = d.L.nblocks;
        }
        if (mU < tU) {
          tU = mU;
          bestU = d.U.nblocks;
        }
      }
      d.L.nblocks = bestL;
      d.U.nblocks = bestU;
    }
    return check_err();
  }

  // C_l = the matrix of GemslrClass::CMatVec(l) (gemslr.cpp:3962-4080): the
  // unfactored B_j blocks of levels j > l on the diagonal, E_j / F_j of the
  // non-last levels j > l off the diagonal, in the local numbering of the
  // trailing m_l unknowns.
  int assemble_c(Import& im, int l, DCsr<P>& out) { return upload_csr(ar, host_c_block(im, l), out, stream); }
  int assemble_c0(Import& im) { return assemble_c(im, 0, C0); }

  // replace the low-rank correction of level l
  int set_lowrank(int l, const std::vector<double>& W, const std::vector<double>& WH, int rank) {
    DLevel<P>& d = lv[l];
    d.rank = rank;
    if (rank > 0) {
      PGX_TRY(ar.upload(&d.W, W.data(), W.size(), stream));
      PGX_TRY(ar.upload(&d.WH, WH.data(), WH.size(), stream));
    }
    return PGX_SUCCESS;
  }

  // y = (I - C_l C~_l^-1) x + E_l B_l^-1 F_l C~_l^-1 x, the operator whose
  // dominant invariant subspace gives the level's low-rank correction
  // (GemslrClass::EBFCMatVec, gemslr.cpp:3737-3797).  C~_l^-1 is the
  // preconditioner of the lower levels, SolveLevel(l+1).
  void apply_ebfc(int l, const DCsr<P>& Cl, const P* x, P* y, P* tm, P* tu, P* tw) {
    DLevel<P>& d = lv[l];
    Skip sk = mk_skip();
    solve_level(l + 1, tm, x, sk);
    spmv<P, P, P, P>(Cl, tm, (P)-1, nullptr, nullptr, (P)0, x, (P)1, y, nullptr, sk);
    spmv<P, P, P, P>(d.F, tm, (P)1, nullptr, nullptr, (P)0, (const P*)nullptr, (P)0, tu, nullptr, sk);
    solve_b(l, tu, nullptr, tw, sk);
    spmv<P, P, P, P>(d.E, tw, (P)1, nullptr, nullptr, (P)0, y, (P)1, y, nullptr, sk);
  }

  // Low-rank correction of level l by subspace iteration
  // (PargemslrSubSpaceIteration, matrixops.cpp:8999-9180, kept-all branch of
  // SetupLowRankBuildLowRank, gemslr.cpp:3059-3150): Q = orth(B); B = G Q,
  // its times; then H = Q^T G Q, W = Q, WH = Q ((I - H)^-1 - I).
  int build_lowrank(Import& im, int l, int k, int its, unsigned long long seed, std::vector<double>& W,
                    std::vector<double>& WH, int& rank) {
    if constexpr (Sc<P>::complex) {
      (void)im, (void)l, (void)k, (void)its, (void)seed, (void)W, (void)WH, (void)rank;
      return fail(PGX_ERROR_INVALID_OPTION, "the low-rank build of the host setup is real only");
    } else {
      return build_lowrank_real(im, l, k, its, seed, W, WH, rank);
    }
  }
  int build_lowrank_real(Import& im, int l, int k, int its, unsigned long long seed, std::vector<double>& W,
                         std::vector<double>& WH, int& rank) {
    DLevel<P>& d = lv[l];
    const int m = d.m;
    rank = 0;
    k = std::min(k, m);
    if (k <= 0) return PGX_SUCCESS;
    DCsr<P> Cl;
    Arena tmp;
    P *Qd = nullptr, *Bd = nullptr, *tm = nullptr, *tu = nullptr, *tw = nullptr;
    {
      // C_l lives in the handle arena only for the duration of the build
      PGX_TRY(assemble_c(im, l, Cl));
    }
    PGX_TRY(tmp.alloc(&Qd, (size_t)m * k));
    PGX_TRY(tmp.alloc(&Bd, (size_t)m * k));
    PGX_TRY(tmp.alloc(&tm, (size_t)m));
    PGX_TRY(tmp.alloc(&tu, (size_t)d.nl));
    PGX_TRY(tmp.alloc(&tw, (size_t)d.nl));
    std::vector<double> B((size_t)m * k), Q((size_t)m * k);
    unsigned long long st = seed ? seed : 0x9E3779B97F4A7C15ULL;
    for (auto& v : B) {  // uniform [0, 1) from a 64-bit xorshift*
      st ^= st >> 12;
      st ^= st << 25;
      st ^= st >> 27;
      v = (double)((st * 0x2545F4914F6CDD1DULL) >> 11) * (1.0 / 9007199254740992.0);
    }
    std::vector<P> buf((size_t)m * k);
    int kk = k;
    for (int it = 0; it < std::max(its, 1); it++) {
      // Q = orth(B) by classical Gram-Schmidt with re-orthogonalisation
      Q = B;
      kk = k;
      for (int c = 0; c < kk; c++) {
        double* q = &Q[(size_t)c * m];
        for (int pass = 0; pass < 2; pass++)
          for (int p = 0; p < c; p++) {
            const double* qp = &Q[(size_t)p * m];
            double h = 0.0;
            for (int i = 0; i < m; i++) h += qp[i] * q[i];
            for (int i = 0; i < m; i++) q[i] -= h * qp[i];
          }
        double nr = 0.0;
        for (int i = 0; i < m; i++) nr += q[i] * q[i];
        nr = std::sqrt(nr);
        if (!(nr > 1e-13)) {  // numerically dependent: stop at this rank
          kk = c;
          break;
        }
        for (int i = 0; i < m; i++) q[i] /= nr;
      }
      if (kk == 0) return PGX_SUCCESS;
      for (size_t i = 0; i < (size_t)m * kk; i++) buf[i] = (P)Q[i];
      PGX_CUDA(cudaMemcpyAsync(Qd, buf.data(), sizeof(P) * (size_t)m * kk, cudaMemcpyHostToDevice, stream));
      for (int c = 0; c < kk; c++) apply_ebfc(l, Cl, Qd + (size_t)c * m, Bd + (size_t)c * m, tm, tu, tw);
      PGX_CUDA(cudaGetLastError());
      PGX_CUDA(cudaMemcpyAsync(buf.data(), Bd, sizeof(P) * (size_t)m * kk, cudaMemcpyDeviceToHost, stream));
      PGX_CUDA(cudaStreamSynchronize(stream));
      for (size_t i = 0; i < (size_t)m * kk; i++) B[i] = (double)buf[i];
      PGX_TRY(check_err());
    }
    // H = Q^T B; R = (I - H)^-1 - I via LU with partial pivoting
    std::vector<double> H((size_t)kk * kk), Rm((size_t)kk * kk), inv((size_t)kk * kk, 0.0);
    for (int a = 0; a < kk; a++)
      for (int b = 0; b < kk; b++) {
        double h = 0.0;
        for (int i = 0; i < m; i++) h += Q[(size_t)a * m + i] * B[(size_t)b * m + i];
        H[(size_t)b * kk + a] = h;  // column-major
      }
    for (int a = 0; a < kk; a++)
      for (int b = 0; b < kk; b++) Rm[(size_t)b * kk + a] = (a == b ? 1.0 : 0.0) - H[(size_t)b * kk + a];
    for (int a = 0; a < kk; a++) inv[(size_t)a * kk + a] = 1.0;
    for (int c = 0; c < kk; c++) {
      int piv = c;
      for (int r = c + 1; r < kk; r++)
        if (std::fabs(Rm[(size_t)c * kk + r]) > std::fabs(Rm[(size_t)c * kk + piv])) piv = r;
      if (Rm[(size_t)c * kk + piv] == 0.0) return fail(PGX_ERROR_FUNCTION_CALL, "low-rank: I - H is singular");
      if (piv != c)
        for (int b = 0; b < kk; b++) {
          std::swap(Rm[(size_t)b * kk + c], Rm[(size_t)b * kk + piv]);
          std::swap(inv[(size_t)b * kk + c], inv[(size_t)b * kk + piv]);
        }
      const double dv = Rm[(size_t)c * kk + c];
      for (int b = 0; b < kk; b++) {
        Rm[(size_t)b * kk + c] /= dv;
        inv[(size_t)b * kk + c] /= dv;
      }
      for (int r = 0; r < kk; r++) {
        if (r == c) continue;
        const double f = Rm[(size_t)c * kk + r];
        if (f == 0.0) continue;
        for (int b = 0; b < kk; b++) {
          Rm[(size_t)b * kk + r] -= f * Rm[(size_t)b * kk + c];
          inv[(size_t)b * kk + r] -= f * inv[(size_t)b * kk + c];
        }
      }
    }
    for (int a = 0; a < kk; a++) inv[(size_t)a * kk + a] -= 1.0;
    W.assign(Q.begin(), Q.begin() + (size_t)m * kk);
    WH.assign((size_t)m * kk, 0.0);
    for (int b = 0; b < kk; b++)
      for (int a = 0; a < kk; a++) {
        const double r = inv[(size_t)b * kk + a];
        if (r == 0.0) continue;
        const double* q = &Q[(size_t)a * m];
        double* w = &WH[(size_t)b * m];
        for (int i = 0; i < m; i++) w[i] += q[i] * r;
      }
    rank = kk;
    return PGX_SUCCESS;
  }

  int ensure_krylov(int kdim) {
    if (kdim <= kdim_alloc) return PGX_SUCCESS;
    PGX_CUDA(cudaStreamSynchronize(stream));
    drop_graph();
    krylov.release();
    PGX_TRY(krylov.zeros(&V, (size_t)n * (kdim + 1), stream));
    PGX_TRY(krylov.zeros(&Z, (size_t)n * (kdim + 1), stream));
    kdim_alloc = kdim;
    return PGX_SUCCESS;
  }

  // ---------------------------------------------------------- enqueues
  template <typename TA, typename TX, typename TY, typename TC>
  void spmv(const DCsr<TA>& M, const TX* x, TC alpha, const DCsr<TA>* M2, const TX* x2, TC alpha2,
            const TY* b, TC beta, TY* y, const double* xscale, Skip sk) {
    if (M.rows == 0) return;
    if (M.merge && !M2 && !xscale && mcarry_row) {
      const int nt = merge_threads(M.rows, M.nnz);
      merge_spmv_kernel<TA, TX, TY, TC><<<(nt + 255) / 256, 256, 0, stream>>>(
          M.rows, (int)M.nnz, M.rp, M.cj, M.va, x, alpha, b, beta, y, mcarry_row, (TC*)mcarry_val, sk);
      merge_spmv_fixup_kernel<TY, TC><<<grid_for(nt, 256, num_sms() * 8), 256, 0, stream>>>(nt, mcarry_row,
                                                                                     (const TC*)mcarry_val, alpha,
                                                                                     y, sk);
      return;
    }
    const int S = M.S;
    const int gpb = 256 / S;
    const int grid = grid_for(M.rows, gpb, num_sms() * 16);
    const int *rp2 = M2 ? M2->rp : nullptr, *cj2 = M2 ? M2->cj : nullptr;
    const TA* va2 = M2 ? M2->va : nullptr;
    const int xcols2 = M2 ? M2->cols : 0;
#define PGX_SPMV(SS)                                                                                            \
  spmv_kernel<TA, TX, TY, TC, SS, true><<<grid, 256, 0, stream>>>(M.rows, M.rp, M.cj, M.va, x, M.cols, alpha, rp2, \
                                                                  cj2, va2, x2, xcols2, alpha2, b, beta, y, xscale, \
                                                                  err, sk)
    switch (S) {
      case 2: PGX_SPMV(2); break;
      case 4: PGX_SPMV(4); break;
      case 8: PGX_SPMV(8); break;
      case 16: PGX_SPMV(16); break;
      default: PGX_SPMV(32); break;
    }
#undef PGX_SPMV
  }

  // one triangular pass; lower: y = L^-1 rhs (x set to the sentinel),
  // upper: x = D U^-1 y (y set back to the sentinel)
  void trsv(const DTri<P>& T, bool upper, const P* dinv, const P* rhs, const double* rhs_scale, P* y, P* x,
            Skip sk, P* yslot = nullptr) {
    if (T.n == 0) return;
    if (T.comp) {
      PtrR<P, 1> pys, prhs, py, px;
      pys.p[0] = yslot;
      prhs.p[0] = const_cast<P*>(rhs);
      py.p[0] = y;
      px.p[0] = x;
      SkipR<1> sr;
      sr.s[0] = sk;
      launch_pipe<1>(T, upper, pys, prhs, py, px, err, sr, stream);
      return;
    }
    if (T.seg) {
      const size_t bytes = SegCfg<P>::bytes;
#define PGX_TRSVSEG(SS)                                                                                       \
  if (upper)                                                                                                  \
    trsv_seg_kernel<P, SS, true><<<T.nblocks, kSegThreads, bytes, stream>>>(                                  \
        T.n, T.nseg, T.seg_row0, T.seg_rp0, T.seg_nnz0, T.seg_lv0, T.seg_nlvb, T.ord, T.rp, T.cj, T.va, T.lvb,  \
        dinv, rhs, rhs_scale, y, x, T.ticket, err, spin_limit, sk);                                           \
  else                                                                                                        \
    trsv_seg_kernel<P, SS, false><<<T.nblocks, kSegThreads, bytes, stream>>>(                                 \
        T.n, T.nseg, T.seg_row0, T.seg_rp0, T.seg_nnz0, T.seg_lv0, T.seg_nlvb, T.ord, T.rp, T.cj, T.va, T.lvb,  \
        dinv, rhs, rhs_scale, y, x, T.ticket, err, spin_limit, sk)
      switch (T.S) {
        case 2: PGX_TRSVSEG(2); break;
        case 4: PGX_TRSVSEG(4); break;
        case 8: PGX_TRSVSEG(8); break;
        case 16: PGX_TRSVSEG(16); break;
        default: PGX_TRSVSEG(32); break;
      }
#undef PGX_TRSVSEG
      return;
    }
#define PGX_TRSV(SS)                                                                                   \
  if (upper)                                                                                           \
    trsv_kernel<P, SS, true><<<T.nblocks, 256, 0, stream>>>(T.n, T.ngroups, T.ord, T.rp, T.cj, T.va,    \
                                                            dinv, rhs, rhs_scale, y, x, T.ticket, err,  \
                                                            spin_limit, sk);                            \
  else                                                                                                 \
    trsv_kernel<P, SS, false><<<T.nblocks, 256, 0, stream>>>(T.n, T.ngroups, T.ord, T.rp, T.cj, T.va,   \
                                                             dinv, rhs, rhs_scale, y, x, T.ticket, err, \
                                                             spin_limit, sk)
    switch (T.S) {
      case 2: PGX_TRSV(2); break;
      case 4: PGX_TRSV(4); break;
      case 8: PGX_TRSV(8); break;
      case 16: PGX_TRSV(16); break;
      default: PGX_TRSV(32); break;
    }
#undef PGX_TRSV
  }

  template <typename TV, typename TM, typename TW, int MODE>
  void ts(TsArgs<TV, TM, TW> a) {
    a.partial = partial;
    a.counter = counter;
    const int grid = grid_for(a.n, kTsThreads, kTsMaxBlocks);
    ts_kernel<TV, TM, TW, MODE><<<grid, kTsThreads, 0, stream>>>(a);
  }

  template <typename TV, typename TM, typename TW>
  static TsArgs<TV, TM, TW> ts_args(int nrows, Skip sk) {
    TsArgs<TV, TM, TW> a;
    memset(&a, 0, sizeof(a));
    a.n = nrows;
    a.sign = 1.0;
    a.skip = sk;
    return a;
  }

  // B-solve of level l: x = U^-1 L^-1 rhs  (GemslrClass::SolveB)
  void solve_b(int l, const P* rhs, const double* rhs_scale, P* x, Skip sk) {
    DLevel<P>& d = lv[l];
    trsv(d.L, false, nullptr, rhs, rhs_scale, d.y, x, sk, d.yslot);
    trsv(d.U, true, d.dinv, nullptr, nullptr, d.y, x, sk, d.yslot);
  }

  // x += WH (W^T x) in place  (SolveApplyLowRankLevel + Axpy, gemslr.cpp:3585-3590)
  void lowrank_inplace(int l, P* x, Skip sk) {
    DLevel<P>& d = lv[l];
    auto a = ts_args<P, P, P>(d.m, sk);
    a.ncols = d.rank;
    a.V = d.W;
    a.ldv = d.m;
    a.in = x;
    a.epi = EPI_STORE;
    a.dst = d.lrt;
    ts<P, P, P, TS_DOT>(a);
    auto u = ts_args<P, P, P>(d.m, sk);
    u.ncols = d.rank;
    u.M = d.WH;
    u.ldm = d.m;
    u.coef = d.lrt;
    u.in = x;
    u.out = x;
    ts<P, P, P, TS_UPDATE>(u);
  }

  // GemslrClass::SolveLevel (gemslr.cpp:3474-3630); x and rhs hold the
  // trailing n - lev_ptr[l] unknowns.  rhs may carry a lazy scale (level 0).
  void solve_level(int l, P* x, const P* rhs, Skip sk) {
    DLevel<P>& d = lv[l];
    if (l == nlev - 1) {
      solve_b(l, rhs, nullptr, x, sk);
      return;
    }
    P* zu = d.z;
    P* zl = d.z + d.nl;
    P* xl = x + d.nl;
    if (usolve) {                                                                  // U solve: zl = rhs_l
      gather_kernel<P, P><<<grid_for(d.m, 256 * kPermUnroll, num_sms() * 16), 256, 0, stream>>>(
          d.m, nullptr, rhs + d.nl, nullptr, zl, sk);
    } else {
      solve_b(l, rhs, nullptr, zu, sk);                                            // 1. zu = B^-1 rhs_u
      spmv<P, P, P, P>(d.E, zu, (P)-1, nullptr, nullptr, (P)0, rhs + d.nl, (P)1, zl, nullptr, sk);  // 2-3.
    }
    if (l == 0 && inner) {
      inner_solve(xl, zl, sk);                                                     // 4. inner FGMRES
    } else {
      if (d.rank > 0) lowrank_inplace(l, zl, sk);                                  // 4. low rank
      solve_level(l + 1, xl, zl, sk);                                              //    recursion
    }
    spmv<P, P, P, P>(d.F, xl, (P)-1, nullptr, nullptr, (P)0, rhs, (P)1, zu, nullptr, sk);  // 5-6.
    solve_b(l, zu, nullptr, x, sk);                                                // 7. xu = B^-1 zu
  }

  // ParallelGemslrClass::SolveLevelGemslrMul (parallel_gemslr.cpp:5816-6050):
  // the smoothing x_u = B^-1 b_u, the residual z = b - A [x_u; 0], its
  // restriction z_l - E B^-1 z_u, the Schur solve (the inner FGMRES on RAP at
  // level 0, else the low rank and the next level) and x_u += -B^-1 F x_l.
  void solve_level_mul(int l, P* x, const P* rhs, Skip sk) {
    DLevel<P>& d = lv[l];
    if (l == nlev - 1) {
      solve_b(l, rhs, nullptr, x, sk);
      return;
    }
    P* xu = x;
    P* xl = x + d.nl;
    P* zu = d.z;
    P* zl = d.z + d.nl;
    P* yu = d.wmul;
    solve_b(l, rhs, nullptr, xu, sk);                                                        // 1.
    spmv<P, P, P, P>(d.B, xu, (P)-1, nullptr, nullptr, (P)0, rhs, (P)1, zu, nullptr, sk);      // 2. z_u
    solve_b(l, zu, nullptr, yu, sk);                                                          // 3.
    spmv<P, P, P, P>(d.E, xu, (P)-1, &d.E, yu, (P)-1, rhs + d.nl, (P)1, zl, nullptr, sk);    // 2-3. z_l
    if (l == 0 && inner) {
      inner_solve(xl, zl, sk);                                                                // 4.
    } else {
      if (d.rank > 0) lowrank_inplace(l, zl, sk);
      solve_level_mul(l + 1, xl, zl, sk);
    }
    spmv<P, P, P, P>(d.F, xl, (P)-1, nullptr, nullptr, (P)0, (const P*)nullptr, (P)0, yu, nullptr, sk);  // 5.
    solve_b(l, yu, nullptr, zu, sk);
    axpy_kernel<P><<<grid_for(d.nl, 256, num_sms() * 16), 256, 0, stream>>>(d.nl, zu, xu, sk);
  }

  // Level-0 inner flexible GMRES on the Schur complement S0 = C0 - E0 B0^-1 F0,
  // from x0 = 0, one cycle of inner_maxits steps (gemslr.cpp:1660-1674, 3566-3572).
  void inner_solve(P* xl, const P* zl, Skip outer) {
    DLevel<P>& d0 = lv[0];
    const int m0 = d0.m;
    const long long ld = m0;
    Skip it = mk_skip(outer.f0, outer.f1, &st_in->cycle_done);
    {
      auto a = ts_args<P, P, P>(m0, outer);
      a.in = zl;
      a.out = Vin;
      a.epi = EPI_INIT_INNER;
      a.st = st_in;
      ts<P, P, P, TS_NORM_COPY>(a);
    }
    for (int j = 0; j < inner_maxits; j++) {
      P* vj = Vin + (long long)j * ld;
      P* zj = Zin + (long long)j * ld;
      P* wj = Vin + (long long)(j + 1) * ld;
      // Schur preconditioner (GemslrSchurMatrixClass::Solve, gemslr.cpp:294-330):
      // xlr = v + WH W^T v, then the level-1 recursion
      if (d0.rank > 0) {
        auto a = ts_args<P, P, P>(m0, it);
        a.ncols = d0.rank;
        a.V = d0.W;
        a.ldv = m0;
        a.in = vj;
        a.in_scale = &st_in->sc[j];
        a.epi = EPI_STORE;
        a.dst = d0.lrt;
        ts<P, P, P, TS_DOT>(a);
      }
      {
        auto u = ts_args<P, P, P>(m0, it);
        u.ncols = d0.rank;
        u.M = d0.WH;
        u.ldm = m0;
        u.coef = d0.lrt;
        u.in = vj;
        u.in_scale = &st_in->sc[j];
        u.out = d0.xlr;
        ts<P, P, P, TS_UPDATE>(u);
      }
      solve_level(1, zj, d0.xlr, it);
      if (mul) {
        // w = R A P z (RAPMatVec, parallel_gemslr.cpp:7194): P z = [-B^-1 F z; z],
        // A P z through B, F, E and C0, R = [-E B^-1, I]; xlr holds the lower part
        spmv<P, P, P, P>(d0.F, zj, (P)-1, nullptr, nullptr, (P)0, (const P*)nullptr, (P)0, s_zu, nullptr, it);
        solve_b(0, s_zu, nullptr, s_wu, it);
        spmv<P, P, P, P>(d0.B, s_wu, (P)1, &d0.F, zj, (P)1, (const P*)nullptr, (P)0, s_zu, nullptr, it);
        spmv<P, P, P, P>(d0.E, s_wu, (P)1, &C0, zj, (P)1, (const P*)nullptr, (P)0, d0.xlr, nullptr, it);
        solve_b(0, s_zu, nullptr, s_wu, it);
        spmv<P, P, P, P>(d0.E, s_wu, (P)-1, nullptr, nullptr, (P)0, (const P*)d0.xlr, (P)1, wj, nullptr, it);
      } else {
        // w = S0 z  (GemslrClass::SchurMatVec, gemslr.cpp:3799-3960)
        spmv<P, P, P, P>(d0.F, zj, (P)1, nullptr, nullptr, (P)0, (const P*)nullptr, (P)0, s_zu, nullptr, it);
        solve_b(0, s_zu, nullptr, s_wu, it);
        spmv<P, P, P, P>(C0, zj, (P)1, &d0.E, s_wu, (P)-1, (const P*)nullptr, (P)0, wj, nullptr, it);
      }
      arnoldi_step<P, P>(Vin, ld, j, st_in, m0, it);
    }
    {
      auto u = ts_args<P, P, P>(m0, outer);
      u.ncols_dev = &st_in->i;
      u.M = Zin;
      u.ldm = ld;
      u.coef = st_in->rs;
      u.in = nullptr;
      u.out = xl;
      ts<P, P, P, TS_UPDATE>(u);
    }
  }

  // Orthogonalise column j+1 of the basis against columns 0..j by classical
  // Gram-Schmidt with one re-orthogonalisation (CGS2, matrixops.cpp:10588-10708),
  // then finish the Hessenberg column with Givens rotations (fgmres.hpp:430-458).
  template <typename TV, typename TW>
  void arnoldi_step(TV* Vb, long long ld, int j, SD* s, int nrows, Skip sk) {
    TW* w = (TW*)(Vb + (long long)(j + 1) * ld);
    auto a = ts_args<TV, TV, TW>(nrows, sk);
    a.ncols = j + 1;
    a.V = Vb;
    a.ldv = ld;
    a.vsc = s->sc;
    a.in = w;
    a.epi = EPI_CGS_FIRST;
    a.st = s;
    ts<TV, TV, TW, TS_DOT>(a);
    auto b = a;
    b.M = Vb;
    b.ldm = ld;
    b.msc = s->sc;
    b.coef = s->coefA;
    b.sign = -1.0;
    b.out = w;
    b.epi = EPI_CGS_SECOND;
    ts<TV, TV, TW, TS_UPDATE_DOT>(b);
    auto c = b;
    c.coef = s->coefB;
    c.epi = EPI_GIVENS;
    c.j = j;
    ts<TV, TV, TW, TS_UPDATE_NORM>(c);
  }

  // GemslrClass::Solve (gemslr.cpp:3431-3472): gather by pperm, SolveLevel(0),
  // scatter by qperm (or pperm for symmetric reorderings).
  template <typename TO>
  void precond(const F* v, const double* v_scale, TO* z, Skip sk) {
    const int grid = grid_for(n, 256 * kPermUnroll, num_sms() * 16);  // gather / scatter
    gather_kernel<F, P><<<grid, 256, 0, stream>>>(n, pperm, v, v_scale, rt, sk);
    if (mul)
      solve_level_mul(0, xt, rt, sk);
    else
      solve_level(0, xt, rt, sk);
    scatter_kernel<P, TO><<<grid, 256, 0, stream>>>(n, qperm ? qperm : pperm, xt, z, sk);
  }

  int check_err() {
    int h = 0;
    PGX_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    PGX_CUDA(cudaStreamSynchronize(stream));
    if (h & kErrIndex) return fail(PGX_ERROR_INVALID_PARAM, "device index check failed");
    if (h & kErrTimeout) return fail(PGX_ERROR_TIMEOUT, "triangular-solve dependency wait timed out");
    if (h & kErrStage) return fail(PGX_ERROR_TIMEOUT, "triangular-solve staging wait timed out");
    return PGX_SUCCESS;
  }

  // Device time of one building block, measured with CUDA events on the
  // handle's stream over `reps` launches, and its algorithmic bytes per
  // launch (every operand read or written once):
  //   which 0: lower triangular pass of level `level`
  //   which 1: upper triangular pass of level `level`
  //   which 2: outer SpMV w = A z
  int kernel_stats(int which, int level, int reps, double* avg_ms, double* bytes, int* launches) override {
    if (reps < 1) reps = 1;
    if (which < 0 || which > 2) return fail(PGX_ERROR_INVALID_OPTION, "unknown kernel %d", which);
    if ((which <= 1) && (level < 0 || level >= nlev)) return fail(PGX_ERROR_INVALID_PARAM, "level out of range");
    PGX_TRY(ensure_krylov(1));
    Skip sk = mk_skip();
    const double vb = sizeof(P);
    float total = 0.f;
    if (which <= 1) {
      DLevel<P>& d = lv[level];
      const DTri<P>& T = which == 0 ? d.L : d.U;
      const double nnz = (double)(which == 0 ? d.L.nnz_total : d.U.nnz_total);
      *bytes = nnz * (vb + 4.0) + 4.0 * (d.nl + 1) + 4.0 * d.nl + 2.0 * vb * d.nl + (which == 1 ? vb * d.nl : 0.0);
      *launches = T.n > 0 ? 1 : 0;
      // lower and upper passes alternate so the sentinel protocol stays valid;
      // the events bracket only the pass being measured
      for (int r = 0; r < reps; r++) {
        if (which == 0) PGX_CUDA(cudaEventRecord(ev0, stream));
        trsv(d.L, false, nullptr, rt, nullptr, d.y, xt, sk, d.yslot);
        if (which == 0) PGX_CUDA(cudaEventRecord(ev1, stream));
        if (which == 1) PGX_CUDA(cudaEventRecord(ev0, stream));
        trsv(d.U, true, d.dinv, nullptr, nullptr, d.y, xt, sk, d.yslot);
        if (which == 1) PGX_CUDA(cudaEventRecord(ev1, stream));
        PGX_CUDA(cudaStreamSynchronize(stream));
        float ms = 0.f;
        PGX_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        total += ms;
      }
    } else {
      *bytes = (double)A.nnz * (sizeof(F) + 4.0) + 4.0 * (n + 1) + (double)n * (sizeof(P) + sizeof(F));
      *launches = 1;
      for (int r = 0; r < reps; r++) {
        PGX_CUDA(cudaEventRecord(ev0, stream));
        spmv<F, P, F, F>(A, Z, 1.0, nullptr, nullptr, 0.0, (const F*)nullptr, 0.0, V,
                                        nullptr, sk);
        PGX_CUDA(cudaEventRecord(ev1, stream));
        PGX_CUDA(cudaStreamSynchronize(stream));
        float ms = 0.f;
        PGX_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
        total += ms;
      }
    }
    PGX_TRY(check_err());
    *avg_ms = total / reps;
    return PGX_SUCCESS;
  }

  int build_lowrank_level(Import& im, int l, int k, int its, unsigned long long seed) override {
    std::vector<double> W, WH;
    int rank = 0;
    const int us = usolve, mu = mul;
    usolve = 0;  // the setup phase runs the LU sequence
    mul = 0;
    const int rc = build_lowrank(im, l, k, its, seed, W, WH, rank);
    usolve = us;
    mul = mu;
    PGX_TRY(rc);
    PGX_TRY(set_lowrank(l, W, WH, rank));
    im.levels[l].rank = rank;
    im.levels[l].W.swap(W);
    im.levels[l].WH.swap(WH);
    return PGX_SUCCESS;
  }

  int apply(double* z_, const double* v_, int location) override {
    F* z = (F*)z_;
    const F* v = (const F*)v_;
    const F* vin = v;
    F* zout = z;
    if (location == PGX_LOCATION_HOST) {
      PGX_CUDA(cudaMemcpyAsync(bdev, v, sizeof(F) * n, cudaMemcpyHostToDevice, stream));
      vin = bdev;
      zout = xdev;
    }
    PGX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), stream));
    precond<F>(vin, nullptr, zout, mk_skip());
    PGX_CUDA(cudaGetLastError());
    if (location == PGX_LOCATION_HOST)
      PGX_CUDA(cudaMemcpyAsync(z, xdev, sizeof(F) * n, cudaMemcpyDeviceToHost, stream));
    return check_err();
  }

  // One restart cycle of FlexGmresClass::Solve (fgmres.hpp:379-514): kdim
  // Arnoldi steps, the solution update, the restart residual and the cycle
  // reset.  Steps after convergence see the cycle flag and return at once.
  void enqueue_cycle(int kdim, F* xd, const F* bd) {
    const long long ld = n;
    Skip sk = mk_skip(&st->done, &st->cycle_done);
    for (int j = 0; j < kdim; j++) {
      F* vj = V + (long long)j * ld;
      P* zj = Z + (long long)j * ld;
      precond<P>(vj, &st->sc[j], zj, sk);                                            // z = M^-1 v
      spmv<F, P, F, F>(A, zj, 1.0, nullptr, nullptr, 0.0, (const F*)nullptr, 0.0,
                                      V + (long long)(j + 1) * ld, nullptr, sk);   // w = A z
      arnoldi_step<F, F>(V, ld, j, st, n, sk);
    }
    {
      auto u = ts_args<P, P, F>(n, mk_skip());
      u.ncols_dev = &st->i;
      u.M = Z;
      u.ldm = ld;
      u.coef = st->rs;
      u.in = xd;
      u.out = xd;
      ts<P, P, F, TS_UPDATE>(u);                                                // x += Z y
    }
    spmv<F, F, F, F>(A, xd, -1.0, nullptr, nullptr, 0.0, bd, 1.0, V, nullptr,
                                         mk_skip(&st->done));                        // restart residual
    fgmres_cycle_reset_kernel<<<1, 1, 0, stream>>>(st, mk_skip());
  }

  // FlexGmresClass::Solve (fgmres.hpp:263-558) with the basis, Hessenberg and
  // rotations on the device.  The solve is a small state machine so that one
  // host thread can drive many slots at once: begin() enqueues the start of
  // the solve and the first restart cycle, poll() looks at the state header
  // copied back after each cycle and enqueues either the next cycle or the
  // final residual check.
  enum { IDLE = 0, RUNNING = 1, FINISHING = 2 };
  int phase = IDLE;
  int s_cyc = 0, s_max_cycles = 0, s_maxits = 0, s_launches = 0, s_location = 0;
  F* s_xd = nullptr;
  const F* s_bd = nullptr;
  F* s_xuser = nullptr;

  int begin(double* x_, const double* b_, int location, int kdim, int maxits, double tol, int atol,
            bool prechecked = false) override {
    if (phase != IDLE) return fail(PGX_ERROR_FUNCTION_CALL, "slot busy");
    F* x = (F*)x_;
    const F* b = (const F*)b_;
    F* xd = nullptr;
    const F* bd = nullptr;
    PGX_TRY(begin_prologue(x, b, location, kdim, maxits, tol, atol, &xd, &bd, prechecked));
    s_max_cycles = maxits > 0 ? maxits / kdim + 2 : 0;
    if (s_max_cycles > 0 && (!cycle_exec || g_kdim != kdim || g_x != xd || g_b != bd)) {
      drop_graph();
      cudaGraph_t g = nullptr;
      PGX_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      enqueue_cycle(kdim, xd, bd);
      cudaError_t ce = cudaStreamEndCapture(stream, &g);
      if (ce != cudaSuccess) return fail(PGX_ERROR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
      size_t nodes = 0;
      cudaGraphGetNodes(g, nullptr, &nodes);
      cycle_nodes = (int)nodes;
      ce = cudaGraphInstantiate(&cycle_exec, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) {
        cycle_exec = nullptr;
        return fail(PGX_ERROR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
      }
      g_kdim = kdim;
      g_x = xd;
      g_b = bd;
    }
    s_cyc = 0;
    s_maxits = maxits;
    s_launches = 5;  // ||b||, residual, ||r0||, final residual and its norm
    s_location = location;
    history.clear();
    hist_iters = 0;
    s_xd = xd;
    s_bd = bd;
    s_xuser = x;
    phase = RUNNING;
    const int rc = launch_cycle_or_finish(false);
    if (rc != PGX_SUCCESS) phase = IDLE;
    return rc;
  }

  // The start of a solve up to the first restart cycle (fgmres.hpp:263-360):
  // inputs to the device, the FGMRES header, ||b||, r0 = b - A x0 and ||r0||.
  // *xd and *bd receive the device vectors the cycles work on.
  int begin_prologue(F* x, const F* b, int location, int kdim, int maxits, double tol, int atol,
                     F** xd_out, const F** bd_out, bool prechecked = false) {
    if (kdim < 1 || kdim > KMAX) return fail(PGX_ERROR_INVALID_PARAM, "kdim %d outside [1, %d]", kdim, KMAX);
    if (maxits < 0) return fail(PGX_ERROR_INVALID_PARAM, "maxits %d < 0", maxits);
    if (location == PGX_LOCATION_HOST && !prechecked && !all_finite((const double*)b, (long long)n * VW))
      return fail(PGX_ERROR_NOT_FINITE, "b is not finite");
    PGX_TRY(ensure_krylov(kdim));
    // The solve works on the slot's own b and x (copied in here, x copied
    // back when it finishes), from host or device memory alike: a captured
    // restart cycle is keyed by the vectors it reads and writes, so every
    // request of the slot reuses the same graph whatever its pointers.
    if (b != bdev)
      PGX_CUDA(cudaMemcpyAsync(bdev, b, sizeof(F) * n,
                               location == PGX_LOCATION_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                               stream));
    if (x != xdev)
      PGX_CUDA(cudaMemcpyAsync(xdev, x, sizeof(F) * n,
                               location == PGX_LOCATION_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                               stream));
    F* xd = xdev;
    const F* bd = bdev;
    SD h;
    memset(&h, 0, sizeof(h));
    h.kdim = kdim;
    h.maxits = maxits;
    h.tol = tol;
    h.absolute = atol;
    h.eps = DBL_EPSILON;
    h.cycle_done = 1;
    const size_t head = offsetof(SD, sc);
    *hs_pin = h;
    PGX_CUDA(cudaMemcpyAsync(st, hs_pin, head, cudaMemcpyHostToDevice, stream));
    PGX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), stream));
    PGX_CUDA(cudaEventRecord(ev0, stream));
    // ||b||, v = b - A x, ||v||  (fgmres.hpp:319-360)
    {
      auto a = ts_args<F, F, F>(n, mk_skip());
      a.in = bd;
      a.epi = EPI_NORMB;
      a.st = st;
      ts<F, F, F, TS_NORM_COPY>(a);
    }
    spmv<F, F, F, F>(A, xd, -1.0, nullptr, nullptr, 0.0, bd, 1.0, V, nullptr,
                                         mk_skip(&st->done));
    {
      auto a = ts_args<F, F, F>(n, mk_skip());
      a.in = V;
      a.epi = EPI_INIT;
      a.st = st;
      ts<F, F, F, TS_NORM_COPY>(a);
    }
    *xd_out = xd;
    *bd_out = bd;
    return PGX_SUCCESS;
  }

  // after a cycle: either the next cycle or the final FP64 residual check
  int launch_cycle_or_finish(bool last_done) {
    if (!last_done && s_cyc < s_max_cycles) {
      PGX_CUDA(cudaGraphLaunch(cycle_exec, stream));
      s_launches += cycle_nodes;
      s_cyc++;
      PGX_CUDA(cudaMemcpyAsync(hs_pin, st, offsetof(SD, sc), cudaMemcpyDeviceToHost, stream));
      PGX_CUDA(cudaMemcpyAsync(hist_pin, st->hist, sizeof(double) * g_kdim, cudaMemcpyDeviceToHost, stream));
      PGX_CUDA(cudaEventRecord(ev_poll, stream));
      return PGX_SUCCESS;
    }
    PGX_TRY(enqueue_finish());
    PGX_CUDA(cudaEventRecord(ev_poll, stream));
    phase = FINISHING;
    return PGX_SUCCESS;
  }

  // the FP64 true residual ||b - A x|| / ||b|| and the copies of the state
  // header and the residual norm back to the host
  int enqueue_finish() {
    spmv<F, F, F, F>(A, s_xd, -1.0, nullptr, nullptr, 0.0, s_bd, 1.0, rdev, nullptr, mk_skip());
    {
      auto a = ts_args<F, F, F>(n, mk_skip());
      a.in = rdev;
      a.epi = EPI_STORE;
      a.dst = scal;
      ts<F, F, F, TS_NORM_COPY>(a);
    }
    PGX_CUDA(cudaEventRecord(ev1, stream));
    PGX_CUDA(cudaMemcpyAsync(hs_pin, st, offsetof(SD, sc), cudaMemcpyDeviceToHost, stream));
    PGX_CUDA(cudaMemcpyAsync(r2_pin, scal, sizeof(double), cudaMemcpyDeviceToHost, stream));
    return PGX_SUCCESS;
  }

  int poll(bool block, bool* finished, pgx_result* res) override {
    *finished = false;
    if (phase == IDLE) {
      *finished = true;
      return PGX_SUCCESS;
    }
    if (block) {
      cudaError_t q = cudaEventSynchronize(ev_poll);
      if (q != cudaSuccess) {
        phase = IDLE;
        *finished = true;
        return fail(PGX_ERROR_CUDA, "cudaEventSynchronize: %s", cudaGetErrorString(q));
      }
    } else {
      cudaError_t q = cudaEventQuery(ev_poll);
      if (q == cudaErrorNotReady) return PGX_SUCCESS;
      if (q != cudaSuccess) {
        phase = IDLE;
        *finished = true;
        return fail(PGX_ERROR_CUDA, "cudaEventQuery: %s", cudaGetErrorString(q));
      }
    }
    if (phase == RUNNING) {
      const SD& hs = *hs_pin;
      absorb_history(hs);
      const bool over = hs.done || hs.iter >= s_maxits;
      const int rc = launch_cycle_or_finish(over);
      if (rc != PGX_SUCCESS) {
        phase = IDLE;
        *finished = true;
      }
      return rc;
    }
    // FINISHING: the state header and the residual norm are on the host
    phase = IDLE;
    *finished = true;
    return collect_result(res);
  }

  // the residual estimates of the cycle that just landed (hs: its state
  // header, hist_pin: its per-column estimates)
  void absorb_history(const SD& hs) {
    if (history.empty()) history.push_back(hs.normr0);
    const int fresh = std::min(hs.iter - hist_iters, KMAX);
    for (int j = 0; j < fresh; j++) history.push_back(hist_pin[j]);
    hist_iters = hs.iter;
    hist_normb = hs.normb;
  }

  // the relative residual history (FlexGmresClass::GetRelativeResidual,
  // fgmres.hpp:683): estimates over ||b||; a zero right-hand side gives [0]
  std::string describe() const override {
    std::string o;
    char buf[160];
    snprintf(buf, sizeof(buf), "n %d, %d levels, precision %s, inner Schur FGMRES %s\n", n, nlev,
             std::is_same<P, float>::value ? "mixed" : "fp64", inner ? "on" : "off");
    o += buf;
    o += describe_csr("A", A);
    for (int l = 0; l < nlev; l++) {
      const DLevel<P>& d = lv[l];
      snprintf(buf, sizeof(buf), "level %d: rows %d, trailing %d, rank %d\n", l, d.nl, d.m, d.rank);
      o += buf;
      o += describe_tri("L", d.L);
      o += describe_tri("U", d.U);
      o += describe_csr("E", d.E);
      o += describe_csr("F", d.F);
    }
    o += describe_csr("C0", C0);
    return o;
  }

  std::vector<double> residual_history() const override {
    std::vector<double> out;
    if (hist_normb < DBL_EPSILON || (history.size() == 1 && history[0] < DBL_EPSILON)) {
      // zero right-hand side, or x0 already the solution: the reference keeps [0]
      if (!history.empty()) out.push_back(0.0);
      return out;
    }
    for (double v : history) out.push_back(v / hist_normb);
    return out;
  }

  // after enqueue_finish has landed: zero right-hand side, x back to the
  // host, the outcome.  *res is always written: on a CUDA error before the
  // outcome is known it holds zeros and that error as its status.
  int collect_result(pgx_result* res) {
    if (res) memset(res, 0, sizeof(*res));
    const int out = collect_result_body(res);
    if (res && res->status == PGX_SUCCESS) res->status = out;
    return out;
  }

  int collect_result_body(pgx_result* res) {
    const SD hs = *hs_pin;
    const double r2 = *r2_pin;
    const int rc = check_err();
    float ms = 0.f;
    PGX_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    if (hs.normb < DBL_EPSILON) {
      // zero right-hand side: x = 0 (fgmres.hpp:321-329)
      PGX_CUDA(cudaMemsetAsync(s_xd, 0, sizeof(F) * n, stream));
    }
    if (s_xuser != s_xd)
      PGX_CUDA(cudaMemcpyAsync(s_xuser, s_xd, sizeof(F) * n,
                               s_location == PGX_LOCATION_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                               stream));
    PGX_CUDA(cudaStreamSynchronize(stream));
    int out = rc;
    if (out == PGX_SUCCESS && !(std::isfinite(hs.normr)))
      out = fail(PGX_ERROR_NOT_FINITE, "FGMRES residual is not finite");
    if (res) {
      res->status = out;
      res->iters = hs.iter;
      res->rel_res = hs.normb > 0 ? hs.normr / hs.normb : 0.0;
      res->true_rel_res = hs.normb > 0 ? sqrt(r2) / hs.normb : 0.0;
      res->solve_ms = ms;
      res->launches = s_launches;
    }
    return out;
  }

  int solve(double* x, const double* b, int location, int kdim, int maxits, double tol, int atol,
            pgx_result* res) override {
    PGX_TRY(begin(x, b, location, kdim, maxits, tol, atol));
    bool finished = false;
    while (!finished) PGX_TRY(poll(true, &finished, res));
    return PGX_SUCCESS;
  }

  int make_clone(std::unique_ptr<EngineBase>& out) override {
    auto* e = new Engine<P>();
    out.reset(e);
    return e->clone_from(*this);
  }

  void set_wait_limit(int polls) override {
    if (stream) cudaStreamSynchronize(stream);
    spin_limit = polls;
    drop_graph();
  }

  // batched factor layouts shared by this handle's multi-lane slots, by lane count
  std::shared_ptr<void> batch_layout[5];
  int64_t layout_bytes() const override;
  void release_layouts() override {
    for (auto& l : batch_layout) l.reset();
  }
  int make_lanes_clone(Import& im, int lanes, std::unique_ptr<EngineBase>& out) override {
    if (lanes == 1) return make_clone(out);
    return make_batch_slot<P>(*this, im, lanes, out);
  }

  // FGMRES with the Krylov basis in memory handed in by the caller (the
  // static pool of pgx_gemslr_solve_static) and every restart cycle enqueued
  // directly on the stream instead of through a captured graph: nothing is
  // allocated and no graph is instantiated.  The arithmetic and its order are
  // those of begin()/poll().
  int solve_fixed_basis(double* x, const double* b, int location, int kdim, int maxits, double tol, int atol,
                        void* pool, size_t pool_bytes, pgx_result* res) override {
    if (phase != IDLE) return fail(PGX_ERROR_FUNCTION_CALL, "slot busy");
    if (kdim < 1 || kdim > KMAX) return fail(PGX_ERROR_INVALID_PARAM, "kdim %d outside [1, %d]", kdim, KMAX);
    if (maxits < 0) return fail(PGX_ERROR_INVALID_PARAM, "maxits %d < 0", maxits);
    const size_t cols = (size_t)kdim + 1;
    const size_t vbytes = (sizeof(F) * (size_t)n * cols + 255) & ~(size_t)255;
    const size_t zbytes = sizeof(P) * (size_t)n * cols;
    if (vbytes + zbytes > pool_bytes)
      return fail(PGX_ERROR_INVALID_PARAM,
                  "n = %d with kdim = %d needs %zu bytes of Krylov basis; the static pool holds %zu", n, kdim,
                  vbytes + zbytes, pool_bytes);
    if (location == PGX_LOCATION_HOST) {
      for (long long i = 0; i < (long long)n * VW; i++)
        if (!std::isfinite(b[i])) return fail(PGX_ERROR_NOT_FINITE, "b[%lld] is not finite", i / VW);
    }
    F* own_V = V;
    P* own_Z = Z;
    V = (F*)pool;
    Z = (P*)((char*)pool + vbytes);
    const int rc = run_fixed_basis((F*)x, (const F*)b, location, kdim, maxits, tol, atol, vbytes, zbytes, res);
    V = own_V;
    Z = own_Z;
    return rc;
  }

  int run_fixed_basis(F* x, const F* b, int location, int kdim, int maxits, double tol, int atol,
                      size_t vbytes, size_t zbytes, pgx_result* res) {
    F* xd = x;
    const F* bd = b;
    if (location == PGX_LOCATION_HOST) {
      PGX_CUDA(cudaMemcpyAsync(bdev, b, sizeof(F) * n, cudaMemcpyHostToDevice, stream));
      PGX_CUDA(cudaMemcpyAsync(xdev, x, sizeof(F) * n, cudaMemcpyHostToDevice, stream));
      xd = xdev;
      bd = bdev;
    }
    // the pool keeps whatever the previous call left in it
    PGX_CUDA(cudaMemsetAsync(V, 0, vbytes, stream));
    PGX_CUDA(cudaMemsetAsync(Z, 0, zbytes, stream));
    SD h;
    memset(&h, 0, sizeof(h));
    h.kdim = kdim;
    h.maxits = maxits;
    h.tol = tol;
    h.absolute = atol;
    h.eps = DBL_EPSILON;
    h.cycle_done = 1;
    const size_t head = offsetof(SD, sc);
    *hs_pin = h;
    PGX_CUDA(cudaMemcpyAsync(st, hs_pin, head, cudaMemcpyHostToDevice, stream));
    PGX_CUDA(cudaMemsetAsync(err, 0, sizeof(int), stream));
    PGX_CUDA(cudaEventRecord(ev0, stream));
    {
      auto a = ts_args<F, F, F>(n, mk_skip());
      a.in = bd;
      a.epi = EPI_NORMB;
      a.st = st;
      ts<F, F, F, TS_NORM_COPY>(a);
    }
    spmv<F, F, F, F>(A, xd, -1.0, nullptr, nullptr, 0.0, bd, 1.0, V, nullptr,
                                         mk_skip(&st->done));
    {
      auto a = ts_args<F, F, F>(n, mk_skip());
      a.in = V;
      a.epi = EPI_INIT;
      a.st = st;
      ts<F, F, F, TS_NORM_COPY>(a);
    }
    const int max_cycles = maxits > 0 ? maxits / kdim + 2 : 0;
    history.clear();
    hist_iters = 0;
    hist_normb = 0.0;
    for (int cyc = 0; cyc < max_cycles; cyc++) {
      enqueue_cycle(kdim, xd, bd);
      PGX_CUDA(cudaGetLastError());
      PGX_CUDA(cudaMemcpyAsync(hs_pin, st, head, cudaMemcpyDeviceToHost, stream));
      PGX_CUDA(cudaMemcpyAsync(hist_pin, st->hist, sizeof(double) * kdim, cudaMemcpyDeviceToHost, stream));
      PGX_CUDA(cudaStreamSynchronize(stream));
      absorb_history(*hs_pin);
      if (hs_pin->done || hs_pin->iter >= maxits) break;
    }
    spmv<F, F, F, F>(A, xd, -1.0, nullptr, nullptr, 0.0, bd, 1.0, rdev, nullptr, mk_skip());
    {
      auto a = ts_args<F, F, F>(n, mk_skip());
      a.in = rdev;
      a.epi = EPI_STORE;
      a.dst = scal;
      ts<F, F, F, TS_NORM_COPY>(a);
    }
    PGX_CUDA(cudaEventRecord(ev1, stream));
    PGX_CUDA(cudaMemcpyAsync(hs_pin, st, head, cudaMemcpyDeviceToHost, stream));
    PGX_CUDA(cudaMemcpyAsync(r2_pin, scal, sizeof(double), cudaMemcpyDeviceToHost, stream));
    PGX_CUDA(cudaStreamSynchronize(stream));
    // the outcome exactly as pgx_gemslr_solve reports it
    s_xd = xd;
    s_location = location;
    s_xuser = x;
    s_launches = 0;  // kernels enqueued one by one are not counted here
    return collect_result(res);
  }
};

// Per-level layout of the triangular factors for R right-hand sides at once
// (the PipeCfg<P, R> chunking), built once per handle and read by every R-lane
// slot.  Levels whose factors do not fit that layout keep each lane's own
// single-right-hand-side kernels.
template <typename P, int R>
struct BatchLayout {
  Arena ar;
  std::vector<DTri<P>> L, U;
};

// A solve slot that advances R right-hand sides in lockstep: R lanes, each
// with its own FGMRES state and work vectors (clones of the owner), share one
// stream and one captured restart cycle.  The triangular passes of the
// preconditioner are merged over the lanes (trsv_pipe_kernel with R lanes: each
// factor entry is read once for R vectors); every other kernel runs once per
// lane exactly as in Engine, so each lane's arithmetic is that of a single
// solve and its result matches it bit for bit.
template <typename P, int R>
struct BatchEngine : EngineBase {
  // the triangular passes run in groups of G lanes (one merged launch per
  // group over the G-lane layout, shared with the handle's G-lane slots)
  static constexpr int G = R > 4 ? 4 : R;
  Engine<P>* owner = nullptr;
  std::shared_ptr<BatchLayout<P, G>> lay;
  std::unique_ptr<Engine<P>> lane[R];
  cudaStream_t stream = nullptr;
  Arena wk;
  std::vector<std::array<P*, R>> yslot;  // per level, in the R-layout's slot order
  int n = 0, nlev = 0;
  // Block low-rank correction on the tensor cores: complex64 slots of 8 or
  // 16 lanes apply W^H X and X + WH Y to all lanes in two tcgen05 GEMMs
  // (lr_wtx_umma_kernel, lr_update_umma_kernel) instead of one tall-skinny
  // kernel pair per lane.  Slots of 4 lanes or fewer keep the per-lane kernels,
  // so their results equal single solves bit for bit.
  static constexpr bool kTensorLowRank = std::is_same<P, cf32>::value && R >= 8;
  // groups of lanes beyond the first run their triangular passes on side
  // streams (fork/join through events; a captured cycle keeps them as
  // parallel branches), so the R / G merged launches of a pass overlap
  static constexpr int NSIDE = R / G - 1;
  cudaStream_t side[NSIDE > 0 ? NSIDE : 1] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[NSIDE > 0 ? NSIDE : 1] = {};
  static constexpr int kLrGrid = 148;  // CTAs of the split-K W^H X
  cf32* lr_y = nullptr;
  float* lr_partial = nullptr;
  unsigned int* lr_counter = nullptr;
  cudaGraphExec_t cycle_exec = nullptr;
  int cycle_nodes = 0, g_kdim = -1;
  std::array<const void*, R> g_x{}, g_b{};
  enum { IDLE = 0, RUNNING = 1, FINISHING = 2 };
  int phase = IDLE, count = 0, s_cyc = 0, s_max_cycles = 0, s_maxits = 0;

  ~BatchEngine() override {
    if (stream) cudaStreamSynchronize(stream);
    if (cycle_exec) cudaGraphExecDestroy(cycle_exec);
    for (int k = 0; k < NSIDE; k++) {
      if (side[k]) cudaStreamDestroy(side[k]);
      if (ev_join[k]) cudaEventDestroy(ev_join[k]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (int r = 1; r < R; r++)
      if (lane[r]) lane[r]->stream = nullptr;  // lane 0 owns the shared stream
  }

  int setup(Engine<P>& own, Import& im, std::shared_ptr<BatchLayout<P, G>> shared) {
    PGX_TRY(Engine<P>::template set_pipe_smem<G>());
    owner = &own;
    n = own.n;
    nlev = own.nlev;
    for (int r = 0; r < R; r++) {
      lane[r].reset(new Engine<P>());
      PGX_TRY(lane[r]->clone_from(own));
    }
    stream = lane[0]->stream;
    for (int r = 1; r < R; r++) {
      PGX_CUDA(cudaStreamSynchronize(lane[r]->stream));
      PGX_CUDA(cudaStreamDestroy(lane[r]->stream));
      lane[r]->stream = stream;
    }
    if (shared) {
      lay = shared;
    } else {
      lay = std::make_shared<BatchLayout<P, G>>();
      lay->L.resize(nlev);
      lay->U.resize(nlev);
      for (int l = 0; l < nlev; l++) {
        HostLevel& h = im.levels[l];
        if (h.L.rows == 0 || !own.lv[l].L.comp) continue;
        std::vector<int> uslot_of_row;
        using CC = PipeCfg<P, G>;
        int rc = upload_tri_sub<P, CC>(lay->ar, h.U, true, h.dom_ptr, lay->U[l], stream, &h.dinv, &uslot_of_row,
                                       nullptr);
        if (rc == PGX_SUCCESS)
          rc = upload_tri_sub<P, CC>(lay->ar, h.L, false, h.dom_ptr, lay->L[l], stream, nullptr, nullptr,
                                     &uslot_of_row);
        lay->L[l].nslots_up = lay->U[l].nslots_up = lay->U[l].nslots;
        if (rc != PGX_SUCCESS) {
          lay->L[l] = DTri<P>();
          lay->U[l] = DTri<P>();
        } else {
          // rows are summed as the handle's own slot sums them
          lay->L[l].S = own.lv[l].L.S;
          lay->U[l].S = own.lv[l].U.S;
        }
      }
    }
    yslot.resize(nlev);
    for (int l = 0; l < nlev; l++)
      for (int r = 0; r < R; r++) {
        yslot[l][r] = nullptr;
        if (lay->U[l].comp) PGX_TRY(wk.zeros(&yslot[l][r], (size_t)lay->U[l].nslots, stream));
      }
    for (int k = 0; k < NSIDE; k++) {
      PGX_CUDA(cudaStreamCreateWithFlags(&side[k], cudaStreamNonBlocking));
      PGX_CUDA(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
    }
    if (NSIDE > 0) PGX_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    if constexpr (kTensorLowRank) {
      PGX_TRY(wk.zeros(&lr_y, (size_t)kUmmaMaxRank * R, stream));
      PGX_TRY(wk.zeros(&lr_partial, (size_t)kLrGrid * 2 * kUmmaMaxRank * 2 * R, stream));
      PGX_TRY(wk.zeros(&lr_counter, 1, stream));
      PGX_CUDA(cudaFuncSetAttribute(lr_update_umma_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)lr_update_smem(kUmmaMaxRank, R)));
    }
    PGX_CUDA(cudaStreamSynchronize(stream));
    return PGX_SUCCESS;
  }

  // x'_q = x_q s_q + WH_l (W_l^H (x_q s_q)) for every lane on the tensor cores
  // (s_q: the lane's scale, or none)
  void lowrank_block(int l, const std::array<const P*, R>& in, const std::array<P*, R>& out,
                     const std::array<const double*, R>& scale, const std::array<Skip, R>& sk) {
    if constexpr (kTensorLowRank) {
      DLevel<P>& d = lane[0]->lv[l];
      LrBlock<R> xb;
      for (int r = 0; r < R; r++) {
        xb.in[r] = in[r];
        xb.out[r] = out[r];
        xb.scale[r] = scale[r];
      }
      const int grid = lr_wtx_grid(d.m);
      lr_wtx_umma_kernel<R><<<grid, kUmmaThreads, lr_wtx_smem<R>(), stream>>>(
          d.m, d.rank, d.W, xb, lr_partial, lr_counter, lr_y, lane[0]->err, all(sk));
      lr_update_umma_kernel<R><<<(d.m + 127) / 128, kUmmaThreads, lr_update_smem(d.rank, R), stream>>>(
          d.m, d.rank, d.WH, lr_y, xb, lane[0]->err, all(sk));
    } else {
      (void)l, (void)in, (void)out, (void)scale, (void)sk;
    }
  }
  bool use_lowrank_block(int l) const {
    return kTensorLowRank && lane[0]->lv[l].rank > 0 && lane[0]->lv[l].rank <= kUmmaMaxRank;
  }

  int lanes() const override { return R; }
  std::string describe() const override {
    std::string o = "slot of " + std::to_string(R) + " lanes\n";
    for (int l = 0; l < nlev; l++) {
      o += "level " + std::to_string(l) + ":\n";
      if (lay->L[l].comp) {
        o += describe_tri("L (merged over the lanes)", lay->L[l]);
        o += describe_tri("U (merged over the lanes)", lay->U[l]);
      } else {
        o += "  L, U: each lane's own passes\n";
      }
    }
    return o;
  }
  void set_wait_limit(int polls) override {
    if (stream) cudaStreamSynchronize(stream);
    for (int r = 0; r < R; r++) lane[r]->spin_limit = polls;
    if (cycle_exec) cudaGraphExecDestroy(cycle_exec);
    cycle_exec = nullptr;
    g_kdim = -1;
  }
  int64_t slot_bytes(int kdim) const override {
    int64_t b = (int64_t)wk.bytes;
    for (int r = 0; r < R; r++) b += lane[r]->slot_bytes(kdim);
    return b;
  }
  int64_t device_bytes(int kdim) const override { return slot_bytes(kdim); }

  static SkipR<R> all(const std::array<Skip, R>& s) {
    SkipR<R> o;
    for (int r = 0; r < R; r++) o.s[r] = s[r];
    return o;
  }

  // one triangular pass of level l for every lane
  void trsv_b(int l, bool upper, const std::array<const P*, R>& rhs, const std::array<P*, R>& y,
              const std::array<P*, R>& x, const std::array<Skip, R>& sk) {
    const DTri<P>& T = upper ? lay->U[l] : lay->L[l];
    if (!T.comp) {
      for (int r = 0; r < R; r++) {
        DLevel<P>& d = lane[r]->lv[l];
        lane[r]->trsv(upper ? d.U : d.L, upper, upper ? d.dinv : nullptr, rhs[r], nullptr, y[r], x[r], sk[r],
                      d.yslot);
      }
      return;
    }
    if (T.n == 0) return;
    if (NSIDE > 0) cudaEventRecord(ev_fork, stream);
    for (int g0 = 0; g0 < R; g0 += G) {
      const int k = g0 / G - 1;  // side stream of this group (-1: the slot's own)
      cudaStream_t sg_stream = k < 0 ? stream : side[k];
      if (k >= 0) cudaStreamWaitEvent(sg_stream, ev_fork, 0);
      PtrR<P, G> prhs, py, px, pys;
      SkipR<G> sg;
      for (int r = 0; r < G; r++) {
        prhs.p[r] = const_cast<P*>(rhs[g0 + r]);
        py.p[r] = y[g0 + r];
        px.p[r] = x[g0 + r];
        pys.p[r] = yslot[l][g0 + r];
        sg.s[r] = sk[g0 + r];
      }
      Engine<P>::template launch_pipe<G>(T, upper, pys, prhs, py, px, lane[0]->err, sg, sg_stream);
      if (k >= 0) cudaEventRecord(ev_join[k], sg_stream);
    }
    for (int k = 0; k < NSIDE; k++) cudaStreamWaitEvent(stream, ev_join[k], 0);
  }

  void solve_b_b(int l, const std::array<const P*, R>& rhs, const std::array<P*, R>& x,
                 const std::array<Skip, R>& sk) {
    std::array<P*, R> y;
    std::array<const P*, R> none;
    for (int r = 0; r < R; r++) {
      y[r] = lane[r]->lv[l].y;
      none[r] = nullptr;
    }
    trsv_b(l, false, rhs, y, x, sk);
    trsv_b(l, true, none, y, x, sk);
  }

  // Engine::solve_level for every lane
  void solve_level_b(int l, const std::array<P*, R>& x, const std::array<const P*, R>& rhs,
                     const std::array<Skip, R>& sk) {
    if (l == nlev - 1) {
      solve_b_b(l, rhs, x, sk);
      return;
    }
    const int nl = lane[0]->lv[l].nl;
    std::array<P*, R> zu, zl, xl;
    std::array<const P*, R> czu, czl;
    for (int r = 0; r < R; r++) {
      zu[r] = lane[r]->lv[l].z;
      zl[r] = zu[r] + nl;
      xl[r] = x[r] + nl;
      czu[r] = zu[r];
      czl[r] = zl[r];
    }
    if (lane[0]->usolve) {  // U solve: zl = rhs_l
      for (int r = 0; r < R; r++) {
        const int m = lane[r]->lv[l].m;
        gather_kernel<P, P><<<grid_for(m, 256 * kPermUnroll, num_sms() * 16), 256, 0, stream>>>(
            m, nullptr, rhs[r] + nl, nullptr, zl[r], sk[r]);
      }
    } else {
      solve_b_b(l, rhs, zu, sk);
      for (int r = 0; r < R; r++) {
        DLevel<P>& d = lane[r]->lv[l];
        lane[r]->template spmv<P, P, P, P>(d.E, zu[r], (P)-1, nullptr, nullptr, (P)0, rhs[r] + nl, (P)1, zl[r],
                                           nullptr, sk[r]);
      }
    }
    if (l == 0 && lane[0]->inner) {
      inner_solve_b(xl, czl, sk);
    } else {
      if (use_lowrank_block(l)) {
        std::array<const P*, R> czl2;
        std::array<const double*, R> none;
        for (int r = 0; r < R; r++) {
          czl2[r] = zl[r];
          none[r] = nullptr;
        }
        lowrank_block(l, czl2, zl, none, sk);
      } else {
        for (int r = 0; r < R; r++)
          if (lane[r]->lv[l].rank > 0) lane[r]->lowrank_inplace(l, zl[r], sk[r]);
      }
      solve_level_b(l + 1, xl, czl, sk);
    }
    for (int r = 0; r < R; r++) {
      DLevel<P>& d = lane[r]->lv[l];
      lane[r]->template spmv<P, P, P, P>(d.F, xl[r], (P)-1, nullptr, nullptr, (P)0, rhs[r], (P)1, zu[r], nullptr,
                                         sk[r]);
    }
    solve_b_b(l, czu, x, sk);
  }

  // Engine::inner_solve for every lane
  void inner_solve_b(const std::array<P*, R>& xl, const std::array<const P*, R>& zl,
                     const std::array<Skip, R>& outer) {
    const int m0 = lane[0]->lv[0].m;
    const long long ld = m0;
    const int kin = lane[0]->inner_maxits;
    for (int r = 0; r < R; r++) {
      Engine<P>& e = *lane[r];
      auto a = Engine<P>::template ts_args<P, P, P>(m0, outer[r]);
      a.in = zl[r];
      a.out = e.Vin;
      a.epi = EPI_INIT_INNER;
      a.st = e.st_in;
      e.template ts<P, P, P, TS_NORM_COPY>(a);
    }
    for (int j = 0; j < kin; j++) {
      std::array<Skip, R> it;
      std::array<P*, R> zj, xlr, szu, swu;
      std::array<const P*, R> cxlr, cszu;
      const bool block = use_lowrank_block(0);
      std::array<const P*, R> vjs;
      std::array<const double*, R> scs;
      for (int r = 0; r < R; r++) {
        Engine<P>& e = *lane[r];
        DLevel<P>& d0 = e.lv[0];
        it[r] = mk_skip(outer[r].f0, outer[r].f1, &e.st_in->cycle_done);
        P* vj = e.Vin + (long long)j * ld;
        zj[r] = e.Zin + (long long)j * ld;
        vjs[r] = vj;
        scs[r] = &e.st_in->sc[j];
        if (block) {
          // xlr = v + WH W^H v for all lanes below
        } else if (d0.rank > 0) {
          auto a = Engine<P>::template ts_args<P, P, P>(m0, it[r]);
          a.ncols = d0.rank;
          a.V = d0.W;
          a.ldv = m0;
          a.in = vj;
          a.in_scale = &e.st_in->sc[j];
          a.epi = EPI_STORE;
          a.dst = d0.lrt;
          e.template ts<P, P, P, TS_DOT>(a);
        }
        if (!block) {
          auto u = Engine<P>::template ts_args<P, P, P>(m0, it[r]);
          u.ncols = d0.rank;
          u.M = d0.WH;
          u.ldm = m0;
          u.coef = d0.lrt;
          u.in = vj;
          u.in_scale = &e.st_in->sc[j];
          u.out = d0.xlr;
          e.template ts<P, P, P, TS_UPDATE>(u);
        }
        xlr[r] = d0.xlr;
        cxlr[r] = d0.xlr;
        szu[r] = e.s_zu;
        swu[r] = e.s_wu;
        cszu[r] = e.s_zu;
      }
      if (block) lowrank_block(0, vjs, xlr, scs, it);
      solve_level_b(1, zj, cxlr, it);
      for (int r = 0; r < R; r++) {
        Engine<P>& e = *lane[r];
        e.template spmv<P, P, P, P>(e.lv[0].F, zj[r], (P)1, nullptr, nullptr, (P)0, (const P*)nullptr, (P)0, szu[r],
                                    nullptr, it[r]);
      }
      solve_b_b(0, cszu, swu, it);
      for (int r = 0; r < R; r++) {
        Engine<P>& e = *lane[r];
        P* wj = e.Vin + (long long)(j + 1) * ld;
        e.template spmv<P, P, P, P>(e.C0, zj[r], (P)1, &e.lv[0].E, swu[r], (P)-1, (const P*)nullptr, (P)0, wj,
                                    nullptr, it[r]);
        e.template arnoldi_step<P, P>(e.Vin, ld, j, e.st_in, m0, it[r]);
      }
    }
    for (int r = 0; r < R; r++) {
      Engine<P>& e = *lane[r];
      auto u = Engine<P>::template ts_args<P, P, P>(m0, outer[r]);
      u.ncols_dev = &e.st_in->i;
      u.M = e.Zin;
      u.ldm = ld;
      u.coef = e.st_in->rs;
      u.in = nullptr;
      u.out = xl[r];
      e.template ts<P, P, P, TS_UPDATE>(u);
    }
  }

  // Engine::enqueue_cycle for every lane, preconditioner applies merged
  using F = typename Engine<P>::F;
  void enqueue_cycle_b(int kdim, const std::array<F*, R>& xd, const std::array<const F*, R>& bd) {
    const long long ld = n;
    std::array<Skip, R> sk;
    for (int r = 0; r < R; r++) sk[r] = mk_skip(&lane[r]->st->done, &lane[r]->st->cycle_done);
    const int grid = grid_for(n, 256 * kPermUnroll, num_sms() * 16);  // gather / scatter
    for (int j = 0; j < kdim; j++) {
      std::array<P*, R> xt;
      std::array<const P*, R> rt;
      for (int r = 0; r < R; r++) {
        Engine<P>& e = *lane[r];
        gather_kernel<F, P><<<grid, 256, 0, stream>>>(n, e.pperm, e.V + (long long)j * ld, &e.st->sc[j], e.rt,
                                                           sk[r]);
        xt[r] = e.xt;
        rt[r] = e.rt;
      }
      solve_level_b(0, xt, rt, sk);
      for (int r = 0; r < R; r++) {
        Engine<P>& e = *lane[r];
        P* zj = e.Z + (long long)j * ld;
        scatter_kernel<P, P><<<grid, 256, 0, stream>>>(n, e.qperm ? e.qperm : e.pperm, e.xt, zj, sk[r]);
        e.template spmv<F, P, F, F>(e.A, zj, 1.0, nullptr, nullptr, 0.0, (const F*)nullptr, 0.0,
                                                   e.V + (long long)(j + 1) * ld, nullptr, sk[r]);
        e.template arnoldi_step<F, F>(e.V, ld, j, e.st, n, sk[r]);
      }
    }
    for (int r = 0; r < R; r++) {
      Engine<P>& e = *lane[r];
      auto u = Engine<P>::template ts_args<P, P, F>(n, mk_skip());
      u.ncols_dev = &e.st->i;
      u.M = e.Z;
      u.ldm = ld;
      u.coef = e.st->rs;
      u.in = xd[r];
      u.out = xd[r];
      e.template ts<P, P, F, TS_UPDATE>(u);
      e.template spmv<F, F, F, F>(e.A, xd[r], -1.0, nullptr, nullptr, 0.0, bd[r], 1.0, e.V,
                                                      nullptr, mk_skip(&e.st->done));
      fgmres_cycle_reset_kernel<<<1, 1, 0, stream>>>(e.st, mk_skip());
    }
  }

  int begin_many(int cnt, double* const* x, const double* const* b, int location, int kdim, int maxits, double tol,
                 int atol, bool prechecked = false) override {
    if (phase != IDLE) return fail(PGX_ERROR_FUNCTION_CALL, "slot busy");
    if (cnt < 1 || cnt > R) return fail(PGX_ERROR_INVALID_PARAM, "%d right-hand sides for a %d-lane slot", cnt, R);
    std::array<F*, R> xd;
    std::array<const F*, R> bd;
    for (int r = 0; r < R; r++) {
      Engine<P>& e = *lane[r];
      if (r < cnt) {
        PGX_TRY(e.begin_prologue((F*)x[r], (const F*)b[r], location, kdim, maxits, tol, atol, &xd[r], &bd[r],
                                 prechecked));
        e.s_location = location;
        e.s_xuser = (F*)x[r];
      } else {
        // an idle lane solves b = 0 (finished at once) on its own vectors
        PGX_CUDA(cudaMemsetAsync(e.bdev, 0, sizeof(F) * n, stream));
        PGX_CUDA(cudaMemsetAsync(e.xdev, 0, sizeof(F) * n, stream));
        PGX_TRY(e.begin_prologue(e.xdev, e.bdev, PGX_LOCATION_DEVICE, kdim, maxits, tol, atol, &xd[r], &bd[r]));
        e.s_location = PGX_LOCATION_DEVICE;
        e.s_xuser = e.xdev;
      }
      e.s_xd = xd[r];
      e.s_bd = bd[r];
      e.s_launches = 5;
    }
    s_max_cycles = maxits > 0 ? maxits / kdim + 2 : 0;
    bool same = cycle_exec && g_kdim == kdim;
    for (int r = 0; r < R; r++) same = same && g_x[r] == xd[r] && g_b[r] == bd[r];
    if (s_max_cycles > 0 && !same) {
      if (cycle_exec) cudaGraphExecDestroy(cycle_exec);
      cycle_exec = nullptr;
      cudaGraph_t g = nullptr;
      PGX_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      enqueue_cycle_b(kdim, xd, bd);
      cudaError_t ce = cudaStreamEndCapture(stream, &g);
      if (ce != cudaSuccess) return fail(PGX_ERROR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
      size_t nodes = 0;
      cudaGraphGetNodes(g, nullptr, &nodes);
      cycle_nodes = (int)nodes;
      ce = cudaGraphInstantiate(&cycle_exec, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) {
        cycle_exec = nullptr;
        return fail(PGX_ERROR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
      }
      g_kdim = kdim;
      for (int r = 0; r < R; r++) {
        g_x[r] = xd[r];
        g_b[r] = bd[r];
      }
    }
    count = cnt;
    s_cyc = 0;
    s_maxits = maxits;
    phase = RUNNING;
    const int rc = launch_cycle_or_finish(false);
    if (rc != PGX_SUCCESS) phase = IDLE;
    return rc;
  }

  int begin(double* x, const double* b, int location, int kdim, int maxits, double tol, int atol,
            bool prechecked = false) override {
    double* xs[1] = {x};
    const double* bs[1] = {b};
    return begin_many(1, xs, bs, location, kdim, maxits, tol, atol, prechecked);
  }

  int launch_cycle_or_finish(bool last_done) {
    cudaEvent_t evp = lane[0]->ev_poll;
    if (!last_done && s_cyc < s_max_cycles) {
      PGX_CUDA(cudaGraphLaunch(cycle_exec, stream));
      s_cyc++;
      for (int r = 0; r < R; r++) {
        lane[r]->s_launches += cycle_nodes / R;
        PGX_CUDA(cudaMemcpyAsync(lane[r]->hs_pin, lane[r]->st, offsetof(typename Engine<P>::SD, sc), cudaMemcpyDeviceToHost,
                                 stream));
      }
      PGX_CUDA(cudaEventRecord(evp, stream));
      return PGX_SUCCESS;
    }
    for (int r = 0; r < R; r++) PGX_TRY(lane[r]->enqueue_finish());
    PGX_CUDA(cudaEventRecord(evp, stream));
    phase = FINISHING;
    return PGX_SUCCESS;
  }

  int poll(bool block, bool* finished, pgx_result* res) override {
    *finished = false;
    if (phase == IDLE) {
      *finished = true;
      return PGX_SUCCESS;
    }
    cudaEvent_t evp = lane[0]->ev_poll;
    cudaError_t q = block ? cudaEventSynchronize(evp) : cudaEventQuery(evp);
    if (q == cudaErrorNotReady) return PGX_SUCCESS;
    if (q != cudaSuccess) {
      phase = IDLE;
      *finished = true;
      return fail(PGX_ERROR_CUDA, "cudaEventQuery: %s", cudaGetErrorString(q));
    }
    if (phase == RUNNING) {
      bool over = true;
      for (int r = 0; r < R; r++) {
        const auto& hs = *lane[r]->hs_pin;
        over = over && (hs.done || hs.iter >= s_maxits);
      }
      const int rc = launch_cycle_or_finish(over);
      if (rc != PGX_SUCCESS) {
        phase = IDLE;
        *finished = true;
      }
      return rc;
    }
    phase = IDLE;
    *finished = true;
    // each lane's outcome (a NaN in one right-hand side, say) is in its own
    // result; the return value is kept for failures of the slot as a whole
    // (a CUDA error: the lanes share one stream)
    int slot_rc = PGX_SUCCESS;
    for (int r = 0; r < R; r++) {
      pgx_result tmp;
      const int rc = lane[r]->collect_result(&tmp);
      if (r < count && res) res[r] = tmp;
      if ((rc == PGX_ERROR_CUDA || rc == PGX_ERROR_OOM) && slot_rc == PGX_SUCCESS) slot_rc = rc;
    }
    return slot_rc;
  }

  int solve(double* x, const double* b, int location, int kdim, int maxits, double tol, int atol,
            pgx_result* res) override {
    PGX_TRY(begin(x, b, location, kdim, maxits, tol, atol));
    bool finished = false;
    std::array<pgx_result, R> rr;
    while (!finished) PGX_TRY(poll(true, &finished, rr.data()));
    if (res) *res = rr[0];
    return PGX_SUCCESS;
  }

  // device time and algorithmic bytes of the merged lower (which 0) or upper
  // (which 1) pass of `level` over all R lanes; the factor is counted once,
  // the vectors once per lane
  int kernel_stats(int which, int level, int reps, double* avg_ms, double* bytes, int* launches) override {
    if (reps < 1) reps = 1;
    if (which < 0 || which > 1) return fail(PGX_ERROR_INVALID_OPTION, "unknown kernel %d", which);
    if (level < 0 || level >= nlev) return fail(PGX_ERROR_INVALID_PARAM, "level out of range");
    std::array<Skip, R> sk;
    std::array<const P*, R> rt, none;
    std::array<P*, R> y, xt;
    for (int r = 0; r < R; r++) {
      sk[r] = mk_skip();
      rt[r] = lane[r]->rt;
      none[r] = nullptr;
      y[r] = lane[r]->lv[level].y;
      xt[r] = lane[r]->xt;
    }
    const DTri<P>& T = which == 0 ? lay->L[level] : lay->U[level];
    const int nl = lane[0]->lv[level].nl;
    const double vb = sizeof(P);
    const double nnz = (double)(which == 0 ? lane[0]->lv[level].L.nnz_total : lane[0]->lv[level].U.nnz_total);
    *bytes = nnz * (vb + 4.0) + 4.0 * (nl + 1) + 4.0 * nl + R * 2.0 * vb * nl + (which == 1 ? vb * nl : 0.0);
    *launches = T.comp ? 1 : R;
    cudaEvent_t e0 = lane[0]->ev0, e1 = lane[0]->ev1;
    float total = 0.f;
    for (int rep = 0; rep < reps; rep++) {
      if (which == 0) PGX_CUDA(cudaEventRecord(e0, stream));
      trsv_b(level, false, rt, y, xt, sk);
      if (which == 0) PGX_CUDA(cudaEventRecord(e1, stream));
      if (which == 1) PGX_CUDA(cudaEventRecord(e0, stream));
      trsv_b(level, true, none, y, xt, sk);
      if (which == 1) PGX_CUDA(cudaEventRecord(e1, stream));
      PGX_CUDA(cudaStreamSynchronize(stream));
      float ms = 0.f;
      PGX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      total += ms;
    }
    PGX_TRY(lane[0]->check_err());
    *avg_ms = total / reps;
    return PGX_SUCCESS;
  }
  int build_lowrank_level(Import&, int, int, int, unsigned long long) override {
    return fail(PGX_ERROR_FUNCTION_CALL, "setup runs on the handle itself");
  }
  int apply(double*, const double*, int) override {
    return fail(PGX_ERROR_FUNCTION_CALL, "the preconditioner is applied on the handle itself");
  }
  int make_clone(std::unique_ptr<EngineBase>&) override {
    return fail(PGX_ERROR_FUNCTION_CALL, "slots are cloned from the handle itself");
  }
  int solve_fixed_basis(double*, const double*, int, int, int, double, int, void*, size_t, pgx_result*) override {
    return fail(PGX_ERROR_FUNCTION_CALL, "the static-basis solve runs on the handle itself");
  }
};

template <typename P, int R>
static int make_batch_slot_r(Engine<P>& own, Import& im, std::unique_ptr<EngineBase>& out) {
  auto* e = new BatchEngine<P, R>();
  out.reset(e);
  constexpr int G = BatchEngine<P, R>::G;
  auto shared = std::static_pointer_cast<BatchLayout<P, G>>(own.batch_layout[G]);
  PGX_TRY(e->setup(own, im, shared));
  if (!shared) own.batch_layout[G] = e->lay;
  return PGX_SUCCESS;
}

template <typename P>
int64_t Engine<P>::layout_bytes() const {
  int64_t b = 0;
  if (batch_layout[2]) b += (int64_t)std::static_pointer_cast<BatchLayout<P, 2>>(batch_layout[2])->ar.bytes;
  if (batch_layout[4]) b += (int64_t)std::static_pointer_cast<BatchLayout<P, 4>>(batch_layout[4])->ar.bytes;
  return b;
}

template <typename P>
int make_batch_slot(Engine<P>& own, Import& im, int lanes, std::unique_ptr<EngineBase>& out) {
  if (im.solve_option == 2)
    return fail(PGX_ERROR_INVALID_OPTION, "the multiplicative solve runs one right-hand side per slot");
  switch (lanes) {
    case 2: return make_batch_slot_r<P, 2>(own, im, out);
    case 4: return make_batch_slot_r<P, 4>(own, im, out);
    case 8: return make_batch_slot_r<P, 8>(own, im, out);
    case 16: return make_batch_slot_r<P, 16>(own, im, out);
    default: return fail(PGX_ERROR_INVALID_PARAM, "lanes %d: one of 1, 2, 4, 8, 16", lanes);
  }
}

}  // namespace pgx

// ===================================================================== C ABI
using namespace pgx;

// Krylov basis of pgx_gemslr_solve_static: a fixed pool in the module's
// global memory, so that solve needs no allocation.  Host code may not use
// the array's name as a device address; each device's address comes from
// cudaGetSymbolAddress on that device's first call.
static __device__ __align__(256) unsigned char g_static_basis[PGX_STATIC_BASIS_BYTES];
static void* g_static_basis_addr[64];
static std::mutex g_static_basis_mu;

static int static_basis(int device, void** out) {
  if (device < 0 || device >= 64) return fail(PGX_ERROR_INVALID_PARAM, "device %d outside [0, 64)", device);
  std::lock_guard<std::mutex> lock(g_static_basis_mu);
  if (!g_static_basis_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_basis);
    if (e != cudaSuccess)
      return fail(PGX_ERROR_CUDA, "cudaGetSymbolAddress(static Krylov pool): %s", cudaGetErrorString(e));
    g_static_basis_addr[device] = p;
  }
  *out = g_static_basis_addr[device];
  return PGX_SUCCESS;
}

struct pgx_gemslr_s {
  Import im;
  std::unique_ptr<EngineBase> eng;                 // slot 0: owns the factors
  std::vector<std::unique_ptr<EngineBase>> extra;  // slots 1..: borrow them
  int device = 0;
  int servers = 0;  // live pgx_server objects driving the slots
  int lanes = 1;    // right-hand sides each extra slot advances together
  int nslots() const { return eng ? 1 + (int)extra.size() : 0; }
  EngineBase* slot(int i) { return i == 0 ? eng.get() : extra[i - 1].get(); }
  ~pgx_gemslr_s() {
    extra.clear();  // clones first: they read the owner's factors
    eng.reset();
  }
};

// The serving loop of one handle: a FIFO of requests and the request each
// slot is working on.
struct pgx_server_s {
  pgx_handle h = nullptr;
  bool has_params = false;
  double params[180];
  struct Req {
    double* x;
    const double* b;
    int location;
    int64_t id;
  };
  std::deque<Req> queue;
  std::vector<std::vector<int64_t>> slot_ids;  // requests in each slot (one per lane), empty if free
  std::deque<std::pair<int64_t, pgx_result>> done;
  // the serving thread (pgx_server_start): mu guards the queue, the slots
  // and the finished list; the thread sleeps on cv while nothing is pending
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  std::atomic<bool> running{false};
  int worker_rc = 0;
  std::string worker_msg;
};

// the block low-rank correction for pgx_lowrank_block_apply_c64
template <int NL>
static int lowrank_block_apply(int m, int r, const cf32* W, const cf32* WH, cf32* X, int64_t ldx) {
  Arena tmp;
  cf32* y = nullptr;
  float* partial = nullptr;
  unsigned int* counter = nullptr;
  int* err = nullptr;
  const int grid = lr_wtx_grid(m);
  PGX_TRY(tmp.zeros(&y, (size_t)r * NL, nullptr));
  PGX_TRY(tmp.zeros(&partial, (size_t)grid * 2 * r * 2 * NL, nullptr));
  PGX_TRY(tmp.zeros(&counter, 1, nullptr));
  PGX_TRY(tmp.zeros(&err, 1, nullptr));
  LrBlock<NL> xb;
  for (int q = 0; q < NL; q++) {
    xb.in[q] = X + (size_t)q * ldx;
    xb.out[q] = X + (size_t)q * ldx;
    xb.scale[q] = nullptr;
  }
  SkipR<NL> sk;
  for (int q = 0; q < NL; q++) sk.s[q] = mk_skip();
  PGX_CUDA(cudaFuncSetAttribute(lr_update_umma_kernel<NL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)lr_update_smem(kUmmaMaxRank, NL)));
  lr_wtx_umma_kernel<NL><<<grid, kUmmaThreads, lr_wtx_smem<NL>()>>>(m, r, W, xb, partial, counter, y, err, sk);
  lr_update_umma_kernel<NL><<<(m + 127) / 128, kUmmaThreads, lr_update_smem(r, NL)>>>(m, r, WH, y, xb, err, sk);
  PGX_CUDA(cudaGetLastError());
  PGX_CUDA(cudaDeviceSynchronize());
  int h = 0;
  PGX_CUDA(cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) return fail(PGX_ERROR_TIMEOUT, "tensor-core wait gave up (error word %d)", h);
  return PGX_SUCCESS;
}

// ------------------------------------------------- many systems, one launch
// The systems of several committed handles packed for systems_fgmres_kernel:
// every structure of every system lives in three arenas (indices, P values,
// doubles), each array starting on a 64-element boundary, and one SysDesc
// per system holds its pointers.  The work list orders the systems by an
// estimate of their cost, largest first, so the CTAs that take the last
// systems take small ones.
struct SystemsBase {
  virtual ~SystemsBase() {}
  virtual int solve(double* const* x, const double* const* b, int location, int kdim, int maxits, double tol,
                    int atol, pgx_result* res) = 0;
  virtual int tune(const double* const* b, int location, int kdim, int maxits, double tol, int atol, int stride,
                   double* best_ms) = 0;
  virtual int64_t device_bytes() const = 0;
  int threads = 256, ctas_per_sm = 2, lanes = 2, depth = 2;
  double last_ms = 0.0;  // device time of the last solve's launch (CUDA events)
  std::vector<double> t_start, t_end;  // per system, ms from the launch's first system start
  std::vector<double> t_tri;           // per system, ms in its triangular (B-block) solves
  std::vector<std::array<double, 5>> tune_table;  // threads, ctas per SM, lanes, depth, ms
};

template <typename P>
struct Systems : SystemsBase {
  int count = 0, device = 0, nsm = 148;
  std::vector<int> n_of;             // unknowns per system
  std::vector<size_t> xoff;          // offsets of each system in the packed b and x
  size_t ntot = 0;
  std::vector<SysDesc<P>> desc;      // host copies (device pointers)
  std::vector<int> order;
  Arena ar, work;
  int *d_ints = nullptr, *d_order = nullptr;
  P* d_p = nullptr;
  double* d_d = nullptr;
  SysDesc<P>* d_desc = nullptr;
  double *d_bpack = nullptr, *d_xpack = nullptr;
  double *h_bpack = nullptr, *h_xpack = nullptr;  // pinned
  const double** d_bptr = nullptr;
  double** d_xptr = nullptr;
  std::vector<const double*> h_bptr_cur;
  std::vector<double*> h_xptr_cur;
  const double** h_bptr = nullptr;  // pinned staging of the pointer tables
  double** h_xptr = nullptr;
  unsigned int* d_next = nullptr;
  SysResult* d_res = nullptr;
  SysResult* h_res = nullptr;  // pinned
  FgmresDev *d_st = nullptr, *d_st_in = nullptr;
  int st_ctas = 0;
  int work_kdim = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;

  ~Systems() override {
    if (stream) cudaStreamSynchronize(stream);
    if (h_bpack) cudaFreeHost(h_bpack);
    if (h_xpack) cudaFreeHost(h_xpack);
    if (h_res) cudaFreeHost(h_res);
    if (h_bptr) cudaFreeHost(h_bptr);
    if (h_xptr) cudaFreeHost(h_xptr);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }

  struct Fix {
    void* field;
    int kind;  // 0 ints, 1 P values, 2 doubles
    size_t off;
  };
  std::vector<int> iv;
  std::vector<P> pv;
  std::vector<double> dv;
  std::vector<Fix> fix;
  static size_t padded(size_t n) { return (n + 63) / 64 * 64; }
  template <typename T, typename V>
  static size_t put(std::vector<T>& v, const V* src, size_t n) {
    const size_t off = v.size();
    v.resize(off + padded(n), T(0));
    for (size_t k = 0; k < n; k++) v[off + k] = (T)src[k];
    return off;
  }
  void ints(const int** field, const int* src, size_t n) { fix.push_back({field, 0, put(iv, src, n)}); }
  void vals(const P** field, const double* src, size_t n) { fix.push_back({field, 1, put(pv, src, n)}); }
  void dbls(const double** field, const double* src, size_t n) { fix.push_back({field, 2, put(dv, src, n)}); }
  // a rows x cols block; one given without entries (rows 0) becomes an
  // all-zero block of the expected shape, so its SpMV still writes y
  int csr_p(SysCsr<P>& c, const HostCsr& h, int rows, int cols, const char* what) {
    c.rows = rows;
    c.cols = cols;
    if (h.rows == 0) {
      const std::vector<int> rp(rows + 1, 0);
      ints(&c.rp, rp.data(), rp.size());
      return PGX_SUCCESS;
    }
    if (h.rows != rows || h.cols != cols)
      return fail(PGX_ERROR_INVALID_PARAM, "%s is %d x %d, expected %d x %d", what, h.rows, h.cols, rows, cols);
    ints(&c.rp, h.rp.data(), h.rp.size());
    ints(&c.cj, h.cj.data(), h.cj.size());
    vals(&c.va, h.va.data(), h.cj.size());
    return PGX_SUCCESS;
  }
  // rows in level order (IluClass::BuildLevels rule, ilu.cpp:832-1062)
  // dst_map: where the solved value of each row goes (null: the row itself);
  // pos_out receives each row's packed position
  int tri(SysTri<P>& t, const HostCsr& h_in, bool upper, const std::vector<double>* dinv, int nl,
          long long& levels, const std::vector<int>* dst_map, std::vector<int>* pos_out) {
    t.n = nl;
    t.nlev = 0;
    if (nl == 0) return PGX_SUCCESS;
    HostCsr none;  // a factor given without entries
    if (h_in.rows == 0) {
      none.rows = none.cols = nl;
      none.rp.assign(nl + 1, 0);
    }
    const HostCsr& h = h_in.rows == 0 ? none : h_in;
    if (h.rows != nl) return fail(PGX_ERROR_INVALID_PARAM, "triangular factor has %d rows, level has %d", h.rows, nl);
    if (upper && (!dinv || (int)dinv->size() < nl))
      return fail(PGX_ERROR_INVALID_PARAM, "inverse diagonal shorter than the level's %d rows", nl);
    std::vector<int> lvp, ord;
    PGX_TRY(build_levels(upper, nl, h.rp.data(), h.cj.data(), lvp, ord));
    t.nlev = (int)lvp.size() - 1;
    levels += t.nlev;
    std::vector<int> pos(nl);
    for (int k = 0; k < nl; k++) pos[ord[k]] = k;
    // columns as packed positions; the span is the farthest dependency plus
    // the widest level
    std::vector<int> rp(nl + 1, 0), pc;
    std::vector<double> va, di;
    pc.reserve(h.cj.size());
    va.reserve(h.cj.size());
    int far = 0, wide = 0;
    for (int lv = 0; lv < t.nlev; lv++) wide = std::max(wide, lvp[lv + 1] - lvp[lv]);
    for (int k = 0; k < nl; k++) {
      const int r = ord[k];
      for (int e = h.rp[r]; e < h.rp[r + 1]; e++) {
        const int q = pos[h.cj[e]];
        if (q >= k) return fail(PGX_ERROR_INVALID_PARAM, "triangular factor: row %d reads an unsolved entry", r);
        far = std::max(far, k - q);
        pc.push_back(q);
        va.push_back(h.va[e]);
      }
      rp[k + 1] = (int)pc.size();
      if (upper) di.push_back((*dinv)[r]);
    }
    t.span = far + wide;
    // fixed-size heads of every packed row and the destination of its value
    std::vector<int> hpc((size_t)nl * kSysHead, 0), dst(nl);
    std::vector<double> hva((size_t)nl * kSysHead, 0.0);
    for (int k = 0; k < nl; k++) {
      for (int e = rp[k], u = 0; e < rp[k + 1] && u < kSysHead; e++, u++) {
        hpc[(size_t)k * kSysHead + u] = pc[e];
        hva[(size_t)k * kSysHead + u] = va[e];
      }
      dst[k] = dst_map ? (*dst_map)[ord[k]] : ord[k];
    }
    ints(&t.lvp, lvp.data(), lvp.size());
    ints(&t.row, ord.data(), ord.size());
    ints(&t.rp, rp.data(), rp.size());
    ints(&t.pc, pc.data(), pc.size());
    vals(&t.va, va.data(), va.size());
    ints(&t.hpc, hpc.data(), hpc.size());
    vals(&t.hva, hva.data(), hva.size());
    ints(&t.dst, dst.data(), dst.size());
    if (upper) vals(&t.dinv, di.data(), di.size());
    if (pos_out) pos_out->swap(pos);
    return PGX_SUCCESS;
  }

  int create(const std::vector<const Import*>& ims, int dev) {
    device = dev;
    count = (int)ims.size();
    PGX_CUDA(cudaSetDevice(device));
    PGX_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    PGX_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    PGX_CUDA(cudaEventCreate(&ev0));
    PGX_CUDA(cudaEventCreate(&ev1));
    desc.assign(count, SysDesc<P>());
    std::memset((void*)desc.data(), 0, sizeof(SysDesc<P>) * count);
    n_of.resize(count);
    xoff.resize(count);
    std::vector<double> cost(count, 0.0);
    for (int s = 0; s < count; s++) {
      const Import& im = *ims[s];
      if (im.vw != 1) return fail(PGX_ERROR_INVALID_OPTION, "system %d: the systems solve is real only", s);
      if (im.solve_option == 2)
        return fail(PGX_ERROR_INVALID_OPTION, "system %d: the systems solve runs the LU and U solves only", s);
      if (im.nlev < 1 || im.nlev > kSysMaxLevels)
        return fail(PGX_ERROR_INVALID_PARAM, "system %d: %d levels (1..%d)", s, im.nlev, kSysMaxLevels);
      if (im.inner_enable && im.nlev >= 2 && im.inner_maxits > KMAX)
        return fail(PGX_ERROR_INVALID_PARAM, "system %d: inner maxits above %d", s, KMAX);
      SysDesc<P>& d = desc[s];
      const int n = im.n;
      d.n = n;
      d.nlev = im.nlev;
      n_of[s] = n;
      xoff[s] = ntot;
      ntot += padded(n);
      if (im.A.rows != n || im.A.cols != n) return fail(PGX_ERROR_INVALID_PARAM, "system %d: A is not %d x %d", s, n, n);
      if ((int)im.lev_ptr.size() != im.nlev + 1 || im.lev_ptr[0] != 0 || im.lev_ptr[im.nlev] != n)
        return fail(PGX_ERROR_INVALID_PARAM, "system %d: level pointer does not span n", s);
      d.A.rows = im.A.rows;
      d.A.cols = im.A.cols;
      ints(&d.A.rp, im.A.rp.data(), im.A.rp.size());
      ints(&d.A.cj, im.A.cj.data(), im.A.cj.size());
      dbls(&d.A.va, im.A.va.data(), im.A.cj.size());
      if ((int)im.pperm.size() != n) return fail(PGX_ERROR_INVALID_PARAM, "system %d: no permutation", s);
      ints(&d.pperm, im.pperm.data(), n);
      if (!im.qperm.empty()) ints(&d.qperm, im.qperm.data(), n);
      long long levels = 0, fnnz = 0;
      for (int l = 0; l < im.nlev; l++) {
        const HostLevel& h = im.levels[l];
        SysLevel<P>& v = d.lev[l];
        v.nl = im.lev_ptr[l + 1] - im.lev_ptr[l];
        v.m = n - im.lev_ptr[l + 1];
        // the upper factor's order first: the lower pass writes its result there
        std::vector<int> pos_u;
        PGX_TRY(tri(v.U, h.U, true, &h.dinv, v.nl, levels, nullptr, &pos_u));
        if (v.nl > 0 && (int)pos_u.size() != v.nl) {
          pos_u.resize(v.nl);
          for (int r = 0; r < v.nl; r++) pos_u[r] = r;
        }
        PGX_TRY(tri(v.L, h.L, false, nullptr, v.nl, levels, &pos_u, nullptr));
        fnnz += h.L.nnz() + h.U.nnz();
        if (l < im.nlev - 1) {
          PGX_TRY(csr_p(v.E, h.E, v.m, v.nl, "E"));
          PGX_TRY(csr_p(v.F, h.F, v.nl, v.m, "F"));
          v.rank = h.rank;
          if (h.rank > KMAX) return fail(PGX_ERROR_INVALID_PARAM, "system %d: rank %d above %d", s, h.rank, KMAX);
          if (h.rank > 0) {
            if (h.W.size() < (size_t)v.m * h.rank || h.WH.size() < (size_t)v.m * h.rank)
              return fail(PGX_ERROR_INVALID_PARAM, "system %d level %d: low-rank bases too short", s, l);
            vals(&v.W, h.W.data(), (size_t)v.m * h.rank);
            vals(&v.WH, h.WH.data(), (size_t)v.m * h.rank);
          }
        }
      }
      d.inner = (im.inner_enable && im.nlev >= 2) ? 1 : 0;
      d.usolve = im.solve_option == 1 ? 1 : 0;
      d.inner_maxits = im.inner_maxits;
      d.inner_tol = im.inner_tol;
      if (d.inner) PGX_TRY(csr_p(d.C0, host_c_block(im, 0), d.lev[0].m, d.lev[0].m, "C0"));
      const int sweeps = 2 + (d.inner ? 2 * d.inner_maxits : 0);
      cost[s] = (double)im.A.nnz() + (double)sweeps * ((double)fnnz + 1500.0 * (double)levels);
    }
    order.resize(count);
    for (int s = 0; s < count; s++) order[s] = s;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    PGX_TRY(ar.upload(&d_ints, iv.data(), iv.size(), stream));
    PGX_TRY(ar.upload(&d_p, pv.data(), pv.size(), stream));
    PGX_TRY(ar.upload(&d_d, dv.data(), dv.size(), stream));
    for (const Fix& f : fix) {
      void* p = f.kind == 0 ? (void*)(d_ints + f.off) : f.kind == 1 ? (void*)(d_p + f.off) : (void*)(d_d + f.off);
      *(void**)f.field = p;
    }
    iv.clear(), iv.shrink_to_fit();
    pv.clear(), pv.shrink_to_fit();
    dv.clear(), dv.shrink_to_fit();
    fix.clear();
    PGX_TRY(ar.upload(&d_order, order.data(), order.size(), stream));
    PGX_TRY(ar.zeros(&d_bpack, std::max<size_t>(ntot, 1), stream));
    PGX_TRY(ar.zeros(&d_xpack, std::max<size_t>(ntot, 1), stream));
    PGX_TRY(ar.alloc(&d_bptr, count));
    PGX_TRY(ar.alloc(&d_xptr, count));
    PGX_TRY(ar.zeros(&d_next, 1, stream));
    PGX_TRY(ar.zeros(&d_res, count, stream));
    PGX_TRY(ar.alloc(&d_desc, count));
    PGX_CUDA(cudaMallocHost(&h_bpack, sizeof(double) * std::max<size_t>(ntot, 1)));
    PGX_CUDA(cudaMallocHost(&h_xpack, sizeof(double) * std::max<size_t>(ntot, 1)));
    PGX_CUDA(cudaMallocHost(&h_res, sizeof(SysResult) * count));
    PGX_CUDA(cudaMallocHost(&h_bptr, sizeof(double*) * count));
    PGX_CUDA(cudaMallocHost(&h_xptr, sizeof(double*) * count));
    h_bptr_cur.assign(count, nullptr);
    h_xptr_cur.assign(count, nullptr);
    t_start.assign(count, 0.0);
    t_end.assign(count, 0.0);
    t_tri.assign(count, 0.0);
    PGX_CUDA(cudaStreamSynchronize(stream));
    return PGX_SUCCESS;
  }

  // work space for FGMRES(kdim): the Krylov bases and the preconditioner's vectors
  int ensure_work(int kdim) {
    if (kdim <= work_kdim) return PGX_SUCCESS;
    PGX_CUDA(cudaStreamSynchronize(stream));
    work.release();
    work_kdim = 0;
    size_t np = 0, nd = 0;
    for (int s = 0; s < count; s++) {
      const SysDesc<P>& d = desc[s];
      const size_t n = d.n, m0 = d.nlev > 1 ? d.lev[0].m : 0, nl0 = d.lev[0].nl;
      nd += padded(n * (kdim + 1));
      np += padded(n * kdim) + 5 * padded(n);
      size_t start = 0;
      for (int l = 0; l < d.nlev; l++) {
        np += padded(n - start);
        start += d.lev[l].nl;
      }
      if (d.inner) np += padded(m0 * (d.inner_maxits + 1)) + padded(m0 * d.inner_maxits) + padded(m0) + 2 * padded(nl0);
    }
    P* pw = nullptr;
    double* dw = nullptr;
    PGX_TRY(work.zeros(&pw, np, stream));
    PGX_TRY(work.zeros(&dw, nd, stream));
    size_t op = 0, od = 0;
    auto takep = [&](size_t k) {
      P* p = pw + op;
      op += padded(k);
      return p;
    };
    for (int s = 0; s < count; s++) {
      SysDesc<P>& d = desc[s];
      const size_t n = d.n, m0 = d.nlev > 1 ? d.lev[0].m : 0, nl0 = d.lev[0].nl;
      d.V = dw + od;
      od += padded(n * (kdim + 1));
      d.Z = takep(n * kdim);
      d.rt = takep(n);
      d.xt = takep(n);
      d.y = takep(n);
      d.yr = takep(n);
      d.yu = takep(n);
      size_t start = 0;
      for (int l = 0; l < d.nlev; l++) {
        d.lev[l].z = takep(n - start);
        start += d.lev[l].nl;
      }
      if (d.inner) {
        d.Vin = takep(m0 * (d.inner_maxits + 1));
        d.Zin = takep(m0 * d.inner_maxits);
        d.xlr = takep(m0);
        d.s_zu = takep(nl0);
        d.s_wu = takep(nl0);
      }
    }
    PGX_CUDA(cudaMemcpyAsync(d_desc, desc.data(), sizeof(SysDesc<P>) * count, cudaMemcpyHostToDevice, stream));
    PGX_CUDA(cudaStreamSynchronize(stream));
    work_kdim = kdim;
    return PGX_SUCCESS;
  }

  int ensure_states(int ctas) {
    if (ctas <= st_ctas) return PGX_SUCCESS;
    PGX_TRY(ar.zeros(&d_st, ctas, stream));
    PGX_TRY(ar.zeros(&d_st_in, ctas, stream));
    st_ctas = ctas;
    return PGX_SUCCESS;
  }

  int64_t device_bytes() const override { return (int64_t)(ar.bytes + work.bytes); }

  // the pointer tables the kernel reads b and x through
  int set_pointers(double* const* x, const double* const* b, int location) {
    bool changed = false;
    for (int s = 0; s < count; s++) {
      const double* bp = location == PGX_LOCATION_DEVICE ? b[s] : d_bpack + xoff[s];
      double* xp = location == PGX_LOCATION_DEVICE ? x[s] : d_xpack + xoff[s];
      if (bp != h_bptr_cur[s] || xp != h_xptr_cur[s]) changed = true;
      h_bptr_cur[s] = bp;
      h_xptr_cur[s] = xp;
    }
    if (!changed) return PGX_SUCCESS;
    PGX_CUDA(cudaStreamSynchronize(stream));
    std::memcpy(h_bptr, h_bptr_cur.data(), sizeof(double*) * count);
    std::memcpy(h_xptr, h_xptr_cur.data(), sizeof(double*) * count);
    PGX_CUDA(cudaMemcpyAsync(d_bptr, h_bptr, sizeof(double*) * count, cudaMemcpyHostToDevice, stream));
    PGX_CUDA(cudaMemcpyAsync(d_xptr, h_xptr, sizeof(double*) * count, cudaMemcpyHostToDevice, stream));
    return PGX_SUCCESS;
  }

  int launch(int kdim, int maxits, double tol, int atol, int th, int cps, int ln, int dp, const int* ord = nullptr,
             int nord = -1) {
    // CTAs of up to 256 threads use the build with 128 registers per thread
    void (*kern)(SysArgs<P>) = th <= 256 ? systems_fgmres_kernel<P, 256> : systems_fgmres_kernel<P, kSysMaxThreads>;
    int occ = 0;
    PGX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, th, 0));
    if (occ < 1) return fail(PGX_ERROR_INVALID_PARAM, "%d threads per CTA do not fit an SM", th);
    cps = std::min(cps, occ);
    // the rest of the SM's shared memory, split over its CTAs, holds the
    // triangular solves' vector for every block that fits
    size_t smem = 0;
    PGX_CUDA(cudaOccupancyAvailableDynamicSMemPerBlock(&smem, kern, cps, th));
    smem = smem / 256 * 256;
    PGX_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (!ord) {
      ord = d_order;
      nord = count;
    }
    const int grid = std::max(1, std::min(nord, nsm * cps));
    PGX_TRY(ensure_states(grid));
    SysArgs<P> a;
    a.sys = d_desc;
    a.order = ord;
    a.count = nord;
    a.b = d_bptr;
    a.x = d_xptr;
    a.kdim = kdim;
    a.maxits = maxits;
    a.atol = atol;
    a.tol = tol;
    a.lanes = ln;
    a.scap = (int)(smem / sizeof(P));
    a.depth = dp;
    a.next = d_next;
    a.st = d_st;
    a.st_in = d_st_in;
    a.res = d_res;
    PGX_CUDA(cudaMemsetAsync(d_next, 0, sizeof(unsigned int), stream));
    PGX_CUDA(cudaEventRecord(ev0, stream));
    kern<<<grid, th, smem, stream>>>(a);
    PGX_CUDA(cudaGetLastError());
    PGX_CUDA(cudaEventRecord(ev1, stream));
    return PGX_SUCCESS;
  }

  int check_params(int kdim, int maxits) {
    if (kdim < 1 || kdim > KMAX) return fail(PGX_ERROR_INVALID_PARAM, "kdim %d outside [1, %d]", kdim, KMAX);
    if (maxits < 0) return fail(PGX_ERROR_INVALID_PARAM, "maxits %d < 0", maxits);
    return PGX_SUCCESS;
  }

  int solve(double* const* x, const double* const* b, int location, int kdim, int maxits, double tol, int atol,
            pgx_result* res) override {
    PGX_TRY(check_params(kdim, maxits));
    PGX_CUDA(cudaSetDevice(device));
    for (int s = 0; s < count; s++)
      if (!x[s] || !b[s]) return fail(PGX_ERROR_INVALID_PARAM, "system %d: null x or b", s);
    if (location == PGX_LOCATION_HOST) {
      int bad = -1;
#pragma omp parallel for schedule(dynamic, 4)
      for (int s = 0; s < count; s++) {
        if (!all_finite(b[s], n_of[s])) {
#pragma omp critical
          bad = s;
        }
        std::memcpy(h_bpack + xoff[s], b[s], sizeof(double) * n_of[s]);
        std::memcpy(h_xpack + xoff[s], x[s], sizeof(double) * n_of[s]);
      }
      if (bad >= 0) return fail(PGX_ERROR_NOT_FINITE, "system %d: b is not finite", bad);
    } else if (location != PGX_LOCATION_DEVICE) {
      return fail(PGX_ERROR_MEMORY_LOCATION, "unknown location %d", location);
    }
    PGX_TRY(ensure_work(kdim));
    PGX_TRY(set_pointers(x, b, location));
    if (location == PGX_LOCATION_HOST) {
      PGX_CUDA(cudaMemcpyAsync(d_bpack, h_bpack, sizeof(double) * ntot, cudaMemcpyHostToDevice, stream));
      PGX_CUDA(cudaMemcpyAsync(d_xpack, h_xpack, sizeof(double) * ntot, cudaMemcpyHostToDevice, stream));
    }
    PGX_TRY(launch(kdim, maxits, tol, atol, threads, ctas_per_sm, lanes, depth));
    PGX_CUDA(cudaMemcpyAsync(h_res, d_res, sizeof(SysResult) * count, cudaMemcpyDeviceToHost, stream));
    if (location == PGX_LOCATION_HOST)
      PGX_CUDA(cudaMemcpyAsync(h_xpack, d_xpack, sizeof(double) * ntot, cudaMemcpyDeviceToHost, stream));
    PGX_CUDA(cudaStreamSynchronize(stream));
    if (location == PGX_LOCATION_HOST) {
#pragma omp parallel for schedule(dynamic, 4)
      for (int s = 0; s < count; s++) std::memcpy(x[s], h_xpack + xoff[s], sizeof(double) * n_of[s]);
    }
    float ms = 0.f;
    PGX_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    unsigned long long tmin = ~0ull;
    for (int s = 0; s < count; s++) tmin = std::min(tmin, h_res[s].t0);
    int out = PGX_SUCCESS;
    for (int s = 0; s < count; s++) {
      const SysResult& r = h_res[s];
      t_start[s] = (double)(r.t0 - tmin) * 1e-6;
      t_end[s] = (double)(r.t1 - tmin) * 1e-6;
      t_tri[s] = (double)r.tri_ns * 1e-6;
      int st = PGX_SUCCESS;
      if (!std::isfinite(r.normr) || !std::isfinite(r.true_r2)) {
        st = PGX_ERROR_NOT_FINITE;
        if (out == PGX_SUCCESS) out = fail(st, "system %d: FGMRES residual is not finite", s);
      }
      if (res) {
        res[s].status = st;
        res[s].iters = r.iters;
        res[s].rel_res = r.normb > 0 ? r.normr / r.normb : 0.0;
        res[s].true_rel_res = r.normb > 0 ? sqrt(r.true_r2) / r.normb : 0.0;
        res[s].solve_ms = t_end[s] - t_start[s];
        res[s].launches = 1;
      }
    }
    last_ms = ms;
    return out;
  }

  // The schedule autotuner: a sample of the batch (every stride-th system of
  // the work list past its largest sixteenth) solved once per candidate (threads
  // per CTA, CTAs per SM, SpMV lanes per row) from x0 = 0 into the library's
  // own x; the fastest by device time is kept.
  int tune(const double* const* b, int location, int kdim, int maxits, double tol, int atol, int stride,
           double* best_ms) override {
    PGX_TRY(check_params(kdim, maxits));
    if (stride < 1) return fail(PGX_ERROR_INVALID_PARAM, "stride %d < 1", stride);
    PGX_CUDA(cudaSetDevice(device));
    if (location == PGX_LOCATION_HOST) {
#pragma omp parallel for schedule(dynamic, 4)
      for (int s = 0; s < count; s++) std::memcpy(h_bpack + xoff[s], b[s], sizeof(double) * n_of[s]);
      PGX_CUDA(cudaMemcpyAsync(d_bpack, h_bpack, sizeof(double) * ntot, cudaMemcpyHostToDevice, stream));
    } else if (location == PGX_LOCATION_DEVICE) {
      for (int s = 0; s < count; s++)
        PGX_CUDA(cudaMemcpyAsync(d_bpack + xoff[s], b[s], sizeof(double) * n_of[s], cudaMemcpyDeviceToDevice,
                                 stream));
    } else {
      return fail(PGX_ERROR_MEMORY_LOCATION, "unknown location %d", location);
    }
    PGX_TRY(ensure_work(kdim));
    std::vector<double*> xs(count);
    std::vector<const double*> bs(count);
    PGX_TRY(set_pointers(xs.data(), bs.data(), PGX_LOCATION_HOST));
    // the largest sixteenth of the work list is left out of a sample (stride
    // > 1): every candidate would last as long as its largest system
    std::vector<int> sample;
    for (int w = stride > 1 ? count / 16 : 0; w < count; w += stride) sample.push_back(order[w]);
    Arena tmp;
    int* d_sample = nullptr;
    PGX_TRY(tmp.upload(&d_sample, sample.data(), sample.size(), stream));
    // coordinate descent: the CTA shape first, then the SpMV lanes, then the
    // levels the triangular passes fetch ahead
    tune_table.clear();
    double best = 1e300;
    int bt = 256, bc = 2, bl = 2, bd = 2;
    auto trial = [&](int th, int cps, int ln, int dp) -> int {
      PGX_CUDA(cudaMemsetAsync(d_xpack, 0, sizeof(double) * ntot, stream));
      PGX_TRY(launch(kdim, maxits, tol, atol, th, cps, ln, dp, d_sample, (int)sample.size()));
      PGX_CUDA(cudaStreamSynchronize(stream));
      float ms = 0.f;
      PGX_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
      tune_table.push_back({(double)th, (double)cps, (double)ln, (double)dp, (double)ms});
      if (ms < best) {
        best = ms;
        bt = th, bc = cps, bl = ln, bd = dp;
      }
      return PGX_SUCCESS;
    };
    static const int shapes[][2] = {{256, 2}, {512, 1}, {512, 2}, {1024, 1}};
    for (const auto& c : shapes) PGX_TRY(trial(c[0], c[1], 2, 2));
    const int st = bt, sc = bc;
    for (int ln : {4, 8}) PGX_TRY(trial(st, sc, ln, 2));
    PGX_TRY(trial(st, sc, bl, 3));
    threads = bt, ctas_per_sm = bc, lanes = bl, depth = bd;
    if (best_ms) *best_ms = best;
    return PGX_SUCCESS;
  }
};

extern "C" {

int pgx_init(int device) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return fail(PGX_ERROR_NO_DEVICE, "no CUDA device available");
  if (device < 0 || device >= count) return fail(PGX_ERROR_INVALID_PARAM, "device %d not in [0, %d)", device, count);
  PGX_CUDA(cudaSetDevice(device));
  g_device = device;
  return PGX_SUCCESS;
}

int pgx_finalize(void) { return PGX_SUCCESS; }

const char* pgx_last_error(void) { return g_last_error.c_str(); }

int pgx_version(void) { return 200; }  // 0.2.0: input readers, C++ front end, hypre interface, nnz

int pgx_gemslr_create(pgx_handle* handle, int32_t n, int32_t precision) {
  return guarded("pgx_gemslr_create", [&]() -> int {
    if (!handle) return fail(PGX_ERROR_INVALID_PARAM, "null handle pointer");
    *handle = nullptr;
    if (n <= 0) return fail(PGX_ERROR_INVALID_PARAM, "n must be positive");
    if (precision != PGX_PRECISION_FP64 && precision != PGX_PRECISION_MIXED &&
        precision != PGX_PRECISION_COMPLEX_FP64 && precision != PGX_PRECISION_COMPLEX_MIXED)
      return fail(PGX_ERROR_INVALID_OPTION, "unknown precision %d", precision);
    pgx_gemslr_s* h = new pgx_gemslr_s();
    h->im.n = n;
    h->im.precision = precision;
    h->im.vw = precision >= PGX_PRECISION_COMPLEX_FP64 ? 2 : 1;
    h->device = g_device;
    *handle = h;
    return PGX_SUCCESS;
  });
}

int pgx_gemslr_set_matrix(pgx_handle h, const pgx_csr* A) {
  return guarded("pgx_gemslr_set_matrix", [&]() -> int {
    if (!h || !A) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    if (A->rows != h->im.n || A->cols != h->im.n) return fail(PGX_ERROR_INVALID_PARAM, "A must be n x n");
    return copy_csr(A, h->im.A, "A", h->im.vw);
  });
}

static int check_perm(const int32_t* p, int n, const char* what) {
  std::vector<char> seen(n, 0);
  for (int i = 0; i < n; i++) {
    if (p[i] < 0 || p[i] >= n || seen[p[i]]) return fail(PGX_ERROR_INVALID_PARAM, "%s is not a permutation", what);
    seen[p[i]] = 1;
  }
  return PGX_SUCCESS;
}

int pgx_gemslr_set_perm(pgx_handle h, const int32_t* pperm, const int32_t* qperm) {
  return guarded("pgx_gemslr_set_perm", [&]() -> int {
    if (!h) return fail(PGX_ERROR_INVALID_PARAM, "null handle");
    const int n = h->im.n;
    if (pperm) {
      PGX_TRY(check_perm(pperm, n, "pperm"));
      h->im.pperm.assign(pperm, pperm + n);
    } else {
      h->im.pperm.resize(n);
      for (int i = 0; i < n; i++) h->im.pperm[i] = i;
    }
    h->im.qperm.clear();
    if (qperm) {
      PGX_TRY(check_perm(qperm, n, "qperm"));
      h->im.qperm.assign(qperm, qperm + n);
    }
    return PGX_SUCCESS;
  });
}

int pgx_gemslr_set_levels(pgx_handle h, int32_t nlev, const int32_t* lev_ptr) {
  return guarded("pgx_gemslr_set_levels", [&]() -> int {
    if (!h || !lev_ptr) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    if (nlev < 1) return fail(PGX_ERROR_INVALID_PARAM, "nlev must be >= 1");
    if (lev_ptr[0] != 0 || lev_ptr[nlev] != h->im.n) return fail(PGX_ERROR_INVALID_PARAM, "lev_ptr must span [0, n]");
    for (int l = 0; l < nlev; l++)
      if (lev_ptr[l + 1] <= lev_ptr[l]) return fail(PGX_ERROR_INVALID_PARAM, "level %d is empty", l);
    h->im.nlev = nlev;
    h->im.lev_ptr.assign(lev_ptr, lev_ptr + nlev + 1);
    h->im.levels.assign(nlev, HostLevel());
    return PGX_SUCCESS;
  });
}

int pgx_gemslr_set_level(pgx_handle h, int32_t level, const pgx_level* d) {
  return guarded("pgx_gemslr_set_level", [&]() -> int {
    if (!h || !d) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    Import& im = h->im;
    if (level < 0 || level >= im.nlev) return fail(PGX_ERROR_INVALID_PARAM, "level %d out of range", level);
    const int nl = im.lev_ptr[level + 1] - im.lev_ptr[level];
    const int m = im.n - im.lev_ptr[level + 1];
    const bool last = level == im.nlev - 1;
    HostLevel hl;
    hl.ncomp = d->ncomp;
    if (d->dom_ptr && d->ncomp > 0) hl.dom_ptr.assign(d->dom_ptr, d->dom_ptr + d->ncomp + 1);
    const int vw = im.vw;
    PGX_TRY(copy_csr(&d->L, hl.L, "L", vw));
    PGX_TRY(copy_csr(&d->U, hl.U, "U", vw));
    PGX_TRY(copy_csr(&d->B, hl.B, "B", vw));
    if (hl.L.rows != nl || hl.L.cols != nl || hl.U.rows != nl || hl.U.cols != nl)
      return fail(PGX_ERROR_INVALID_PARAM, "level %d: L/U must be %d x %d", level, nl, nl);
    if (!d->dinv) return fail(PGX_ERROR_INVALID_PARAM, "level %d: missing dinv", level);
    hl.dinv.assign(d->dinv, d->dinv + (size_t)nl * vw);
    if (!hl.B.empty() && (hl.B.rows != nl || hl.B.cols != nl))
      return fail(PGX_ERROR_INVALID_PARAM, "level %d: B must be %d x %d", level, nl, nl);
    if (!last) {
      PGX_TRY(copy_csr(&d->E, hl.E, "E", vw));
      PGX_TRY(copy_csr(&d->F, hl.F, "F", vw));
      if (hl.E.rows != m || hl.E.cols != nl) return fail(PGX_ERROR_INVALID_PARAM, "level %d: E must be %d x %d", level, m, nl);
      if (hl.F.rows != nl || hl.F.cols != m) return fail(PGX_ERROR_INVALID_PARAM, "level %d: F must be %d x %d", level, nl, m);
      if (d->rank < 0 || d->rank > KMAX) return fail(PGX_ERROR_INVALID_PARAM, "level %d: rank %d outside [0, %d]", level, d->rank, KMAX);
      hl.rank = d->rank;
      if (hl.rank > 0) {
        if (!d->W || !d->WH) return fail(PGX_ERROR_INVALID_PARAM, "level %d: missing W/WH", level);
        hl.W.assign(d->W, d->W + (size_t)m * hl.rank * vw);
        hl.WH.assign(d->WH, d->WH + (size_t)m * hl.rank * vw);
      }
    }
    hl.set = true;
    im.levels[level] = std::move(hl);
    return PGX_SUCCESS;
  });
}

int pgx_gemslr_set_inner(pgx_handle h, int32_t enable, int32_t maxits, double tol) {
  if (!h) return fail(PGX_ERROR_INVALID_PARAM, "null handle");
  if (enable && (maxits < 1 || maxits > KMAX)) return fail(PGX_ERROR_INVALID_PARAM, "inner maxits outside [1, %d]", KMAX);
  h->im.inner_enable = enable ? 1 : 0;
  h->im.inner_maxits = maxits;
  h->im.inner_tol = tol;
  return PGX_SUCCESS;
}

int pgx_gemslr_set_solve_option(pgx_handle h, int32_t option) {
  if (!h) return fail(PGX_ERROR_INVALID_PARAM, "null handle");
  if (h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "solve option set after commit");
  if (option < 0 || option > 2)
    return fail(PGX_ERROR_INVALID_OPTION, "solve option %d: 0 (LU), 1 (U) or 2 (multiplicative)", option);
  h->im.solve_option = option;
  return PGX_SUCCESS;
}

int pgx_gemslr_commit(pgx_handle h) {
  if (!h) return fail(PGX_ERROR_INVALID_PARAM, "null handle");
  Import& im = h->im;
  if (im.A.rows != im.n) return fail(PGX_ERROR_FUNCTION_CALL, "commit before set_matrix");
  if (im.nlev < 1) return fail(PGX_ERROR_FUNCTION_CALL, "commit before set_levels");
  if (im.pperm.empty()) PGX_TRY(pgx_gemslr_set_perm(h, nullptr, nullptr));
  for (int l = 0; l < im.nlev; l++)
    if (!im.levels[l].set) return fail(PGX_ERROR_FUNCTION_CALL, "level %d not set", l);
  if (im.inner_enable && im.nlev >= 2)
    for (int l = 1; l < im.nlev; l++)
      if (im.levels[l].B.empty()) return fail(PGX_ERROR_INVALID_PARAM, "inner iteration needs B of level %d", l);
  if (h->servers > 0) return fail(PGX_ERROR_FUNCTION_CALL, "commit while a server is live");
  PGX_CUDA(cudaSetDevice(h->device));
  h->extra.clear();
  h->eng.reset();
  switch (im.precision) {
    case PGX_PRECISION_MIXED: {
      auto* e = new Engine<float>();
      h->eng.reset(e);
      PGX_TRY(e->commit(im));
      break;
    }
    case PGX_PRECISION_COMPLEX_MIXED: {
      auto* e = new Engine<cf32>();
      h->eng.reset(e);
      PGX_TRY(e->commit(im));
      break;
    }
    case PGX_PRECISION_COMPLEX_FP64: {
      auto* e = new Engine<cf64>();
      h->eng.reset(e);
      PGX_TRY(e->commit(im));
      break;
    }
    default: {
      auto* e = new Engine<double>();
      h->eng.reset(e);
      PGX_TRY(e->commit(im));
    }
  }
  return PGX_SUCCESS;
}

// ------------------------------------------------------------ host setup
static void append_block(HostCsr& dst, const setup::Csr& b, int off) {
  for (int r = 0; r < b.rows; r++) {
    for (int k = b.rp[r]; k < b.rp[r + 1]; k++) {
      dst.cj.push_back(b.cj[k] + off);
      dst.va.push_back(b.va[k]);
    }
    dst.rp.push_back((int)dst.cj.size());
  }
}

static HostCsr to_host(const setup::Csr& b) {
  HostCsr h;
  h.rows = b.rows;
  h.cols = b.cols;
  h.rp = b.rp;
  h.cj = b.cj;
  h.va = b.va;
  return h;
}

int pgx_gemslr_setup(pgx_handle* handle, const pgx_csr* A, const double* params, int32_t precision) {
  return guarded("pgx_gemslr_setup", [&]() -> int {
    if (!handle || !A || !params) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    *handle = nullptr;
    if (A->rows != A->cols) return fail(PGX_ERROR_INVALID_PARAM, "A must be square");
    if (precision == PGX_PRECISION_COMPLEX_FP64 || precision == PGX_PRECISION_COMPLEX_MIXED)
      return fail(PGX_ERROR_INVALID_OPTION,
                  "the host setup is real; a complex preconditioner comes in through pgx_gemslr_set_*");
    pgx_handle h = nullptr;
    PGX_TRY(pgx_gemslr_create(&h, A->rows, precision));
    std::unique_ptr<pgx_gemslr_s> guard(h);
    Import& im = h->im;
    PGX_TRY(copy_csr(A, im.A, "A"));
    const int n = im.n;
    // parameters (PARGEMSLR_IO_* slots, SRC/utils/utils.hpp:77-297)
    const int nlev_req = std::max(1, (int)params[20]);
    const int perm_opt = (int)params[58];
    const double tolB = params[40], tolC = params[44];
    const int lfilB = std::max(1, (int)params[48]), lfilC = std::max(1, (int)params[50]);
    const int rank1 = std::max(0, (int)params[74]), rank2 = std::max(0, (int)params[75]);
    const double rfac1 = params[78] > 0 ? params[78] : 1.0, rfac2 = params[79] > 0 ? params[79] : 1.0;
    const int lr_its = std::max(1, (int)params[90]);
    im.inner_enable = params[130] != 0.0;
    im.solve_option = (int)params[141];
    if (im.solve_option != 0 && im.solve_option != 1)
      return fail(PGX_ERROR_INVALID_OPTION,
                  "solve option %d: this library's setup builds the LU and U solves only (the multiplicative solve "
                  "needs the reference's setup)", im.solve_option);
    im.inner_tol = params[131];
    im.inner_maxits = std::max(1, (int)params[132]);
    if (im.inner_maxits > KMAX) return fail(PGX_ERROR_INVALID_PARAM, "inner maxits above %d", KMAX);
    // 1. levels and ordering
    setup::Graph g = setup::symmetric_graph(n, im.A.rp.data(), im.A.cj.data());
    const setup::LocalOrder inside = perm_opt == 0                         ? setup::LocalOrder::kNone
                                     : perm_opt == PGX_REORDER_MULTICOLOR ? setup::LocalOrder::kMulticolor
                                                                          : setup::LocalOrder::kRcm;
    setup::Ordering ord = setup::gemslr_ordering(g, nlev_req, 10, inside);
    const int nlev = (int)ord.lev_ptr.size() - 1;
    std::vector<int> iperm(n);
    for (int i = 0; i < n; i++) iperm[ord.perm[i]] = i;
    im.pperm = ord.perm;
    im.qperm.clear();
    PGX_TRY(pgx_gemslr_set_levels(h, nlev, ord.lev_ptr.data()));
    // 2. blocks and ILUT factors per level (subdomains in parallel)
    for (int l = 0; l < nlev; l++) {
      HostLevel& hl = im.levels[l];
      const int start = ord.lev_ptr[l], end = ord.lev_ptr[l + 1], nl = end - start;
      const std::vector<int>& dom = ord.dom_ptr[l];
      const int ncomp = (int)dom.size() - 1;
      const bool last = l == nlev - 1;
      std::vector<setup::Csr> B(ncomp);
      std::vector<setup::Factor> F(ncomp);
      std::vector<int> rc(ncomp, 0);
  #pragma omp parallel for schedule(dynamic, 1)
      for (int c = 0; c < ncomp; c++) {
        const int r0 = start + dom[c], r1 = start + dom[c + 1];
        B[c] = setup::permuted_block(n, im.A.rp.data(), im.A.cj.data(), im.A.va.data(), ord.perm, iperm, r0, r1, r0, r1);
        rc[c] = setup::ilut(B[c].rows, B[c].rp.data(), B[c].cj.data(), B[c].va.data(), last ? tolC : tolB,
                            last ? lfilC : lfilB, F[c]);
      }
      for (int c = 0; c < ncomp; c++)
        if (rc[c]) return fail(PGX_ERROR_ILU_EMPTY_ROW, "ILUT met an empty row (level %d, subdomain %d)", l, c);
      hl.ncomp = ncomp;
      hl.dom_ptr = dom;
      hl.L = HostCsr();
      hl.U = HostCsr();
      hl.B = HostCsr();
      for (HostCsr* M : {&hl.L, &hl.U, &hl.B}) {
        M->rows = M->cols = nl;
        M->rp.assign(1, 0);
      }
      hl.dinv.clear();
      for (int c = 0; c < ncomp; c++) {
        append_block(hl.L, F[c].L, dom[c]);
        append_block(hl.U, F[c].U, dom[c]);
        append_block(hl.B, B[c], dom[c]);
        hl.dinv.insert(hl.dinv.end(), F[c].dinv.begin(), F[c].dinv.end());
      }
      if (!last) {
        hl.E = to_host(setup::permuted_block(n, im.A.rp.data(), im.A.cj.data(), im.A.va.data(), ord.perm, iperm, end,
                                             n, start, end));
        hl.F = to_host(setup::permuted_block(n, im.A.rp.data(), im.A.cj.data(), im.A.va.data(), ord.perm, iperm,
                                             start, end, end, n));
      }
      hl.rank = 0;
      hl.set = true;
    }
    // 3. low-rank corrections, bottom-up, on the GPU in FP64
    PGX_CUDA(cudaSetDevice(h->device));
    if (nlev >= 2 && (rank1 > 0 || rank2 > 0)) {
      const int inner = im.inner_enable;
      im.inner_enable = 0;
      auto* e = new Engine<double>();
      std::unique_ptr<EngineBase> eng(e);
      PGX_TRY(e->commit(im));
      for (int l = nlev - 2; l >= 0; l--) {
        const int k = (int)((l == 0 ? rank1 : rank2) * (l == 0 ? rfac1 : rfac2));
        PGX_TRY(e->build_lowrank_level(im, l, k, lr_its, 0x5EEDULL + (unsigned long long)l));
      }
      im.inner_enable = inner;
    }
    // 4. the solve engine in the requested precision
    PGX_TRY(pgx_gemslr_commit(h));
    *handle = guard.release();
    return PGX_SUCCESS;
  });
}

int pgx_gemslr_destroy(pgx_handle h) {
  if (!h) return PGX_SUCCESS;
  if (h->servers > 0) return fail(PGX_ERROR_FUNCTION_CALL, "destroy the handle's servers first");
  cudaSetDevice(h->device);
  delete h;
  return PGX_SUCCESS;
}

int pgx_gemslr_device_bytes(pgx_handle h, int32_t kdim, int64_t* bytes) {
  if (!h || !bytes) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "handle not committed");
  // factors and the handle's own slot, the other slots, the multi-lane layouts
  int64_t b = h->eng->device_bytes(kdim) + h->eng->layout_bytes();
  for (auto& e : h->extra) b += e->slot_bytes(kdim);
  *bytes = b;
  return PGX_SUCCESS;
}

// FlexGmres options of the reference's parameter array (PARGEMSLR_IO_SOLVER_*)
static void read_solver_params(const double* params, int& kdim, int& maxits, double& tol, int& atol) {
  kdim = 50;
  maxits = 100;
  tol = 1e-6;
  atol = 0;
  if (params) {
    kdim = (int)params[11];
    maxits = (int)params[12];
    tol = params[13];
    atol = params[14] != 0.0;
  }
}

int pgx_gemslr_solve(pgx_handle h, double* x, const double* b, int32_t location, const double* params,
                     pgx_result* result) {
  if (!h || !x || !b) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "solve before commit");
  if (location != PGX_LOCATION_HOST && location != PGX_LOCATION_DEVICE)
    return fail(PGX_ERROR_MEMORY_LOCATION, "unknown location %d", location);
  if (h->servers > 0) return fail(PGX_ERROR_FUNCTION_CALL, "solve while a server drives the slots");
  int kdim, maxits, atol;
  double tol;
  read_solver_params(params, kdim, maxits, tol, atol);
  PGX_CUDA(cudaSetDevice(h->device));
  return h->eng->solve(x, b, location, kdim, maxits, tol, atol, result);
}

int pgx_gemslr_precond_apply(pgx_handle h, double* z, const double* v, int32_t location) {
  if (!h || !z || !v) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "apply before commit");
  PGX_CUDA(cudaSetDevice(h->device));
  return h->eng->apply(z, v, location);
}

int pgx_gemslr_solve_static(pgx_handle h, double* x, const double* b, int32_t location, const double* params,
                            pgx_result* result) {
  if (!h || !x || !b) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "solve before commit");
  if (location != PGX_LOCATION_HOST && location != PGX_LOCATION_DEVICE)
    return fail(PGX_ERROR_MEMORY_LOCATION, "unknown location %d", location);
  if (h->servers > 0) return fail(PGX_ERROR_FUNCTION_CALL, "solve while a server drives the slots");
  int kdim, maxits, atol;
  double tol;
  read_solver_params(params, kdim, maxits, tol, atol);
  PGX_CUDA(cudaSetDevice(h->device));
  void* pool = nullptr;
  PGX_TRY(static_basis(h->device, &pool));
  return h->eng->solve_fixed_basis(x, b, location, kdim, maxits, tol, atol, pool, PGX_STATIC_BASIS_BYTES,
                                   result);
}

int pgx_gemslr_set_slots(pgx_handle h, int32_t nslots) {
  if (!h) return fail(PGX_ERROR_INVALID_PARAM, "null handle");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "handle not committed");
  if (nslots < 1 || nslots > 256) return fail(PGX_ERROR_INVALID_PARAM, "nslots %d outside [1, 256]", nslots);
  if (h->servers > 0) return fail(PGX_ERROR_FUNCTION_CALL, "slots cannot change while a server is live");
  PGX_CUDA(cudaSetDevice(h->device));
  while ((int)h->extra.size() > nslots - 1) h->extra.pop_back();
  while ((int)h->extra.size() < nslots - 1) {
    std::unique_ptr<EngineBase> e;
    const int rc = h->eng->make_lanes_clone(h->im, h->lanes, e);
    if (rc != PGX_SUCCESS) return rc;
    h->extra.push_back(std::move(e));
  }
  return PGX_SUCCESS;
}

int pgx_gemslr_set_lanes(pgx_handle h, int32_t lanes) {
  if (!h) return fail(PGX_ERROR_INVALID_PARAM, "null handle");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "handle not committed");
  if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16)
    return fail(PGX_ERROR_INVALID_PARAM, "lanes %d: one of 1, 2, 4, 8, 16", lanes);
  if (h->servers > 0) return fail(PGX_ERROR_FUNCTION_CALL, "lanes cannot change while a server is live");
  if (lanes == h->lanes) return PGX_SUCCESS;
  PGX_CUDA(cudaSetDevice(h->device));
  const int nslots = h->nslots();
  h->extra.clear();
  h->eng->release_layouts();  // rebuilt on demand for the new lane count
  h->lanes = lanes;
  return pgx_gemslr_set_slots(h, nslots);
}

int pgx_gemslr_slot_bytes(pgx_handle h, int32_t kdim, int64_t* bytes) {
  if (!h || !bytes) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "handle not committed");
  *bytes = h->extra.empty() ? h->eng->slot_bytes(kdim) : h->extra.back()->slot_bytes(kdim);
  return PGX_SUCCESS;
}

int pgx_gemslr_solve_batch(pgx_handle h, int32_t nrhs, double* X, int64_t ldx, const double* B, int64_t ldb,
                           int32_t location, const double* params, pgx_result* results) {
  if (!h || (nrhs > 0 && (!X || !B))) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "solve before commit");
  if (nrhs < 0 || ldx < h->im.n || ldb < h->im.n) return fail(PGX_ERROR_INVALID_PARAM, "bad batch shape");
  if (location != PGX_LOCATION_HOST && location != PGX_LOCATION_DEVICE)
    return fail(PGX_ERROR_MEMORY_LOCATION, "unknown location %d", location);
  if (h->servers > 0) return fail(PGX_ERROR_FUNCTION_CALL, "batch solve while a server drives the slots");
  int kdim, maxits, atol;
  double tol;
  read_solver_params(params, kdim, maxits, tol, atol);
  PGX_CUDA(cudaSetDevice(h->device));
  if (results) memset(results, 0, sizeof(pgx_result) * (size_t)nrhs);
  const int vw = h->im.vw;  // ldx, ldb count values; a complex value is two doubles
  // host columns are checked before any is assigned, so that a bad one does
  // not take the other lanes of its slot down with it
  std::vector<int> order;
  order.reserve((size_t)nrhs);
  int first_bad = -1;
  for (int r = 0; r < nrhs; r++) {
    const bool ok = location != PGX_LOCATION_HOST || all_finite(B + (size_t)r * ldb * vw, (long long)h->im.n * vw);
    if (ok) {
      order.push_back(r);
    } else {
      if (results) results[r].status = PGX_ERROR_NOT_FINITE;
      if (first_bad < 0) first_bad = r;
    }
  }
  const int ns = h->nslots();
  // busy[s]: the right-hand sides slot s is solving (one per lane)
  std::vector<std::vector<int>> busy(ns);
  int next = 0, remaining = nrhs, first_err = PGX_SUCCESS;
  std::string first_msg;
  auto note = [&](int rc) {
    if (rc != PGX_SUCCESS && first_err == PGX_SUCCESS) {
      first_err = rc;
      first_msg = g_last_error;
    }
  };
  std::vector<pgx_result> res(kMaxLanes);
  if (first_bad >= 0) {
    fail(PGX_ERROR_NOT_FINITE, "b(:, %d) is not finite", first_bad);
    note(PGX_ERROR_NOT_FINITE);
  }
  const int nok = (int)order.size();
  remaining = nok;
  while (remaining > 0) {
    bool progressed = false;
    // the additional (possibly multi-lane) slots first, the handle's own last
    for (int t = 0; t < ns; t++) {
      const int sidx = (t + 1) % ns;
      EngineBase* e = h->slot(sidx);
      if (busy[sidx].empty() && next < nok) {
        const int cnt = std::min(e->lanes(), nok - next);
        double* xs[kMaxLanes];
        const double* bs[kMaxLanes];
        for (int k = 0; k < cnt; k++) {
          xs[k] = X + (size_t)order[next + k] * ldx * vw;
          bs[k] = B + (size_t)order[next + k] * ldb * vw;
        }
        const int rc = e->begin_many(cnt, xs, bs, location, kdim, maxits, tol, atol, true);
        progressed = true;
        if (rc != PGX_SUCCESS) {
          for (int k = 0; k < cnt; k++)
            if (results) results[order[next + k]].status = rc;
          note(rc);
          next += cnt;
          remaining -= cnt;
          continue;
        }
        for (int k = 0; k < cnt; k++) busy[sidx].push_back(order[next + k]);
        next += cnt;
      }
      if (!busy[sidx].empty()) {
        bool fin = false;
        for (auto& r : res) memset(&r, 0, sizeof(r));
        const int rc = e->poll(false, &fin, res.data());
        if (rc != PGX_SUCCESS || fin) {
          for (size_t k = 0; k < busy[sidx].size(); k++) {
            if (rc != PGX_SUCCESS && res[k].status == PGX_SUCCESS) res[k].status = rc;
            if (results) results[busy[sidx][k]] = res[k];
            note(res[k].status);
          }
          remaining -= (int)busy[sidx].size();
          busy[sidx].clear();
          progressed = true;
        }
      }
    }
    if (!progressed) std::this_thread::yield();
  }
  if (first_err != PGX_SUCCESS) g_last_error = first_msg;
  return first_err;
}

int pgx_server_create(pgx_handle h, const double* params, pgx_server* out) {
  if (!h || !out) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "handle not committed");
  pgx_server_s* srv = new pgx_server_s();
  srv->h = h;
  srv->has_params = params != nullptr;
  if (params) memcpy(srv->params, params, sizeof(srv->params));
  srv->slot_ids.assign(h->nslots(), std::vector<int64_t>());
  h->servers++;
  *out = srv;
  return PGX_SUCCESS;
}

int pgx_server_submit(pgx_server srv, double* x, const double* b, int32_t location, int64_t request_id) {
  if (!srv || !x || !b) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (request_id < 0) return fail(PGX_ERROR_INVALID_PARAM, "request id %lld < 0", (long long)request_id);
  if (location != PGX_LOCATION_HOST && location != PGX_LOCATION_DEVICE)
    return fail(PGX_ERROR_MEMORY_LOCATION, "unknown location %d", location);
  if (location == PGX_LOCATION_HOST && !all_finite(b, (long long)srv->h->im.n * srv->h->im.vw))
    return fail(PGX_ERROR_NOT_FINITE, "b is not finite");
  {
    std::lock_guard<std::mutex> lock(srv->mu);
    srv->queue.push_back({x, b, location, request_id});
  }
  srv->cv.notify_one();
  return PGX_SUCCESS;
}

static int server_step_locked(pgx_server srv, int32_t* n_active, int32_t* n_queued) {
  pgx_handle h = srv->h;
  PGX_CUDA(cudaSetDevice(h->device));
  int kdim, maxits, atol;
  double tol;
  read_solver_params(srv->has_params ? srv->params : nullptr, kdim, maxits, tol, atol);
  int active = 0;
  pgx_result res[kMaxLanes];
  const int ns = h->nslots();
  // the additional (possibly multi-lane) slots first, the handle's own last
  for (int t = 0; t < ns; t++) {
    const int sidx = (t + 1) % ns;
    EngineBase* e = h->slot(sidx);
    std::vector<int64_t>& ids = srv->slot_ids[sidx];
    if (ids.empty() && !srv->queue.empty()) {
      // the oldest waiting requests (one per lane, same memory location) go to the free slot
      double* xs[kMaxLanes];
      const double* bs[kMaxLanes];
      const int loc = srv->queue.front().location;
      int cnt = 0;
      while (cnt < e->lanes() && !srv->queue.empty() && srv->queue.front().location == loc) {
        const pgx_server_s::Req r = srv->queue.front();
        srv->queue.pop_front();
        xs[cnt] = r.x;
        bs[cnt] = r.b;
        ids.push_back(r.id);
        cnt++;
      }
      const int rc = e->begin_many(cnt, xs, bs, loc, kdim, maxits, tol, atol, true);
      if (rc != PGX_SUCCESS) {
        for (int64_t id : ids) {
          pgx_result bad;
          memset(&bad, 0, sizeof(bad));
          bad.status = rc;
          srv->done.push_back({id, bad});
        }
        ids.clear();
        continue;
      }
    }
    if (!ids.empty()) {
      bool fin = false;
      memset(res, 0, sizeof(res));
      const int rc = e->poll(false, &fin, res);
      if (rc != PGX_SUCCESS || fin) {
        for (size_t k = 0; k < ids.size(); k++) {
          if (rc != PGX_SUCCESS && res[k].status == PGX_SUCCESS) res[k].status = rc;
          srv->done.push_back({ids[k], res[k]});
        }
        ids.clear();
      } else {
        active += (int)ids.size();
      }
    }
  }
  if (n_active) *n_active = active;
  if (n_queued) *n_queued = (int32_t)srv->queue.size();
  return PGX_SUCCESS;
}

int pgx_server_step(pgx_server srv, int32_t* n_active, int32_t* n_queued) {
  if (!srv) return fail(PGX_ERROR_INVALID_PARAM, "null server");
  if (srv->running) return fail(PGX_ERROR_FUNCTION_CALL, "the server steps on its own thread (pgx_server_stop first)");
  std::lock_guard<std::mutex> lock(srv->mu);
  return server_step_locked(srv, n_active, n_queued);
}

int pgx_server_start(pgx_server srv) {
  if (!srv) return fail(PGX_ERROR_INVALID_PARAM, "null server");
  if (srv->running) return fail(PGX_ERROR_FUNCTION_CALL, "the server thread is already running");
  srv->worker_rc = PGX_SUCCESS;
  srv->running = true;
  srv->worker = std::thread([srv]() {
    while (srv->running) {
      int32_t active = 0, queued = 0;
      {
        std::lock_guard<std::mutex> lock(srv->mu);
        const int rc = server_step_locked(srv, &active, &queued);
        if (rc != PGX_SUCCESS && srv->worker_rc == PGX_SUCCESS) {
          srv->worker_rc = rc;
          srv->worker_msg = g_last_error;
        }
      }
      if (active == 0 && queued == 0) {
        // idle: wait for a submission (or stop), waking now and then regardless
        std::unique_lock<std::mutex> lock(srv->mu);
        srv->cv.wait_for(lock, std::chrono::milliseconds(2),
                         [srv]() { return !srv->running || !srv->queue.empty(); });
      } else {
        // solves in flight: look again shortly without holding the lock
        std::this_thread::sleep_for(std::chrono::microseconds(50));
      }
    }
  });
  return PGX_SUCCESS;
}

int pgx_server_stop(pgx_server srv) {
  if (!srv) return fail(PGX_ERROR_INVALID_PARAM, "null server");
  if (!srv->running) return PGX_SUCCESS;
  srv->running = false;
  srv->cv.notify_all();
  if (srv->worker.joinable()) srv->worker.join();
  if (srv->worker_rc != PGX_SUCCESS) return fail(srv->worker_rc, "server thread: %s", srv->worker_msg.c_str());
  return PGX_SUCCESS;
}

int pgx_server_collect(pgx_server srv, int32_t max, int64_t* ids, pgx_result* results, int32_t* n) {
  if (!srv || !n) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  std::lock_guard<std::mutex> lock(srv->mu);
  int k = 0;
  while (k < max && !srv->done.empty()) {
    if (ids) ids[k] = srv->done.front().first;
    if (results) results[k] = srv->done.front().second;
    srv->done.pop_front();
    k++;
  }
  *n = k;
  return PGX_SUCCESS;
}

int pgx_server_destroy(pgx_server srv) {
  if (!srv) return PGX_SUCCESS;
  pgx_server_stop(srv);
  cudaSetDevice(srv->h->device);
  // finish the in-flight solves so that no slot is left in the middle of a cycle
  pgx_result res[kMaxLanes];
  for (int sidx = 0; sidx < srv->h->nslots(); sidx++) {
    if (srv->slot_ids[sidx].empty()) continue;
    bool fin = false;
    while (!fin)
      if (srv->h->slot(sidx)->poll(true, &fin, res) != PGX_SUCCESS) break;
  }
  srv->h->servers--;
  delete srv;
  return PGX_SUCCESS;
}

int pgx_gemslr_residual_history(pgx_handle h, int32_t capacity, double* hist, int32_t* count) {
  if (!h || !count) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "handle not committed");
  if (hist && capacity < 0) return fail(PGX_ERROR_INVALID_PARAM, "capacity %d < 0", capacity);
  const std::vector<double> r = h->eng->residual_history();
  *count = (int32_t)r.size();
  if (hist) std::copy(r.begin(), r.begin() + std::min<size_t>(r.size(), (size_t)capacity), hist);
  return PGX_SUCCESS;
}

int pgx_gemslr_describe(pgx_handle h, int32_t slot, char* buf, int32_t capacity, int32_t* length) {
  return guarded("pgx_gemslr_describe", [&]() -> int {
    if (!h || !length) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "handle not committed");
    if (slot < 0 || slot >= h->nslots()) return fail(PGX_ERROR_INVALID_PARAM, "slot %d outside [0, %d)", slot, h->nslots());
    const std::string d = h->slot(slot)->describe();
    *length = (int32_t)d.size();
    if (buf && capacity > 0) {
      const size_t k = std::min<size_t>(d.size(), (size_t)capacity - 1);
      memcpy(buf, d.data(), k);
      buf[k] = 0;
    }
    return PGX_SUCCESS;
  });
}

int pgx_gemslr_set_wait_limit(pgx_handle h, int64_t polls) {
  if (!h) return fail(PGX_ERROR_INVALID_PARAM, "null handle");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "handle not committed");
  if (polls < 1 || polls > INT32_MAX) return fail(PGX_ERROR_INVALID_PARAM, "wait limit %lld outside [1, 2^31)", (long long)polls);
  if (h->servers > 0) return fail(PGX_ERROR_FUNCTION_CALL, "the wait limit cannot change while a server is live");
  PGX_CUDA(cudaSetDevice(h->device));
  for (int i = 0; i < h->nslots(); i++) h->slot(i)->set_wait_limit((int)polls);
  return PGX_SUCCESS;
}

// A lower triangular pass of trsv_kernel over two rows in which row 1 depends
// on row 0 but only row 1 is scheduled: nothing ever publishes row 0, so the
// wait on it can only end by its bound.  Every index stays inside the arrays
// below (one group of 16 two-lane rows, one nonzero).
int pgx_wait_selfcheck(int64_t polls, int32_t* status, double* wait_ms) {
  if (!status) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (polls < 1 || polls > INT32_MAX) return fail(PGX_ERROR_INVALID_PARAM, "wait limit %lld outside [1, 2^31)", (long long)polls);
  PGX_CUDA(cudaSetDevice(g_device));
  constexpr int S = 2, G = kWarp / S;
  int ord[G], rp[G + 1], cj[1] = {0};
  double va[1] = {1.0}, rhs[2] = {1.0, 2.0};
  for (int i = 0; i < G; i++) ord[i] = i == 0 ? 1 : -1;
  for (int i = 0; i <= G; i++) rp[i] = i == 0 ? 0 : 1;
  Arena ar;
  int *d_ord = nullptr, *d_rp = nullptr, *d_cj = nullptr, *d_err = nullptr;
  double *d_va = nullptr, *d_rhs = nullptr, *d_y = nullptr, *d_x = nullptr;
  unsigned long long* d_ticket = nullptr;
  cudaStream_t s = nullptr;
  PGX_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{s};
  PGX_TRY(ar.upload(&d_ord, ord, G, s));
  PGX_TRY(ar.upload(&d_rp, rp, G + 1, s));
  PGX_TRY(ar.upload(&d_cj, cj, 1, s));
  PGX_TRY(ar.upload(&d_va, va, 1, s));
  PGX_TRY(ar.upload(&d_rhs, rhs, 2, s));
  PGX_TRY(ar.alloc(&d_y, 2));
  PGX_TRY(ar.alloc(&d_x, 2));
  PGX_TRY(ar.zeros(&d_ticket, 2, s));
  PGX_TRY(ar.zeros(&d_err, 1, s));
  sentinel_fill_kernel<double><<<1, 32, 0, s>>>(2, d_y);
  PGX_CUDA(cudaGetLastError());
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  PGX_CUDA(cudaEventCreate(&e0));
  PGX_CUDA(cudaEventCreate(&e1));
  PGX_CUDA(cudaEventRecord(e0, s));
  trsv_kernel<double, S, false><<<1, 256, 0, s>>>(2, 1, d_ord, d_rp, d_cj, d_va, nullptr, d_rhs, nullptr, d_y, d_x,
                                                  d_ticket, d_err, (int)polls, mk_skip());
  const cudaError_t le = cudaGetLastError();
  PGX_CUDA(cudaEventRecord(e1, s));
  const cudaError_t se = cudaStreamSynchronize(s);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (le != cudaSuccess) return fail(PGX_ERROR_CUDA, "wait self-check launch: %s", cudaGetErrorString(le));
  if (se != cudaSuccess) return fail(PGX_ERROR_CUDA, "wait self-check: %s", cudaGetErrorString(se));
  int herr = 0;
  PGX_CUDA(cudaMemcpy(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost));
  *status = (herr & kErrTimeout) ? PGX_ERROR_TIMEOUT : (herr & kErrIndex) ? PGX_ERROR_INVALID_PARAM : PGX_SUCCESS;
  if (wait_ms) *wait_ms = ms;
  return PGX_SUCCESS;
}

// --------------------------------------------------------------- serving pool
// Many resident preconditioned matrices served from one device-memory budget.
// Each member (a committed handle) keeps its factors resident; solve slots
// are created for a member when a request of it finds none idle and the
// budget has room for the slot's work space and Krylov basis, and idle slots
// of other members are released (least recently used first) when it has
// not.  Requests wait in one queue and are admitted first-fit in arrival
// order.
struct pgx_pool_s {
  struct Slot {
    std::unique_ptr<EngineBase> eng;  // null: the member's handle itself (slot 0)
    int64_t bytes = 0;                // counted against the budget (0 for slot 0, counted with the factors)
    int64_t req = -1;                 // request in flight, -1 when idle
    uint64_t last_used = 0;
    EngineBase* get(pgx_handle h) { return eng ? eng.get() : h->eng.get(); }
  };
  struct Member {
    pgx_handle h = nullptr;
    int64_t base_bytes = 0;  // factors, the handle's own slot and its basis
    int64_t slot_bytes = 0;  // one more slot, work space and basis
    std::vector<Slot> slots;
  };
  struct Req {
    int member;
    double* x;
    const double* b;
    int location;
    int64_t id;
  };
  int64_t budget = 0, in_use = 0, peak = 0;
  int kdim = 50, maxits = 100, atol = 0;
  double tol = 1e-6;
  int device = 0;
  uint64_t tick = 0;
  std::vector<Member> members;
  std::deque<Req> queue;
  std::deque<std::pair<int64_t, pgx_result>> done;
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  std::atomic<bool> running{false};
  int worker_rc = 0;
  std::string worker_msg;
};

static int pool_release_idle(pgx_pool p, int64_t need, int keep_member) {
  // free idle extra slots of other members, least recently used first, until
  // `need` more bytes fit the budget
  while (p->in_use + need > p->budget) {
    int bm = -1, bs = -1;
    uint64_t best = UINT64_MAX;
    for (int m = 0; m < (int)p->members.size(); m++) {
      if (m == keep_member) continue;
      auto& sl = p->members[m].slots;
      for (int i = 1; i < (int)sl.size(); i++)
        if (sl[i].req < 0 && sl[i].last_used < best) {
          best = sl[i].last_used;
          bm = m;
          bs = i;
        }
    }
    if (bm < 0) return 0;
    p->in_use -= p->members[bm].slots[bs].bytes;
    p->members[bm].slots.erase(p->members[bm].slots.begin() + bs);
  }
  return 1;
}

static int pool_step_locked(pgx_pool p, int32_t* n_active, int32_t* n_queued) {
  PGX_CUDA(cudaSetDevice(p->device));
  // 1. advance the slots in flight
  int active = 0;
  for (auto& m : p->members)
    for (auto& sl : m.slots) {
      if (sl.req < 0) continue;
      bool fin = false;
      pgx_result res;
      memset(&res, 0, sizeof(res));
      const int rc = sl.get(m.h)->poll(false, &fin, &res);
      if (rc != PGX_SUCCESS || fin) {
        if (rc != PGX_SUCCESS && res.status == PGX_SUCCESS) res.status = rc;
        p->done.push_back({sl.req, res});
        sl.req = -1;
        sl.last_used = ++p->tick;
      } else {
        active++;
      }
    }
  // 2. admit waiting requests, first fit in arrival order
  for (auto it = p->queue.begin(); it != p->queue.end();) {
    pgx_pool_s::Member& m = p->members[it->member];
    int slot = -1;
    for (int i = 0; i < (int)m.slots.size(); i++)
      if (m.slots[i].req < 0) {
        slot = i;
        break;
      }
    if (slot < 0 && pool_release_idle(p, m.slot_bytes, it->member)) {
      pgx_pool_s::Slot ns;
      const int rc = m.h->eng->make_lanes_clone(m.h->im, 1, ns.eng);
      if (rc == PGX_SUCCESS) {
        ns.bytes = m.slot_bytes;
        p->in_use += ns.bytes;
        p->peak = std::max(p->peak, p->in_use);
        m.slots.push_back(std::move(ns));
        slot = (int)m.slots.size() - 1;
      } else if (rc != PGX_ERROR_OOM) {
        return rc;
      }
    }
    if (slot < 0) {
      ++it;  // no room for this one now; a later, smaller one may fit
      continue;
    }
    pgx_pool_s::Slot& sl = m.slots[slot];
    const int rc = sl.get(m.h)->begin(it->x, it->b, it->location, p->kdim, p->maxits, p->tol, p->atol, true);
    if (rc != PGX_SUCCESS) {
      pgx_result bad;
      memset(&bad, 0, sizeof(bad));
      bad.status = rc;
      p->done.push_back({it->id, bad});
    } else {
      sl.req = it->id;
      active++;
    }
    it = p->queue.erase(it);
  }
  if (n_active) *n_active = active;
  if (n_queued) *n_queued = (int32_t)p->queue.size();
  return PGX_SUCCESS;
}

int pgx_pool_create(int64_t budget_bytes, const double* params, pgx_pool* out) {
  return guarded("pgx_pool_create", [&]() -> int {
    if (!out) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    *out = nullptr;
    if (budget_bytes <= 0) return fail(PGX_ERROR_INVALID_PARAM, "budget %lld <= 0", (long long)budget_bytes);
    pgx_pool_s* p = new pgx_pool_s();
    p->budget = budget_bytes;
    p->device = g_device;
    read_solver_params(params, p->kdim, p->maxits, p->tol, p->atol);
    if (p->kdim < 1 || p->kdim > KMAX) {
      delete p;
      return fail(PGX_ERROR_INVALID_PARAM, "kdim %d outside [1, %d]", p->kdim, KMAX);
    }
    *out = p;
    return PGX_SUCCESS;
  });
}

int pgx_pool_add(pgx_pool p, pgx_handle h, int32_t* index) {
  return guarded("pgx_pool_add", [&]() -> int {
    if (!p || !h || !index) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "handle not committed");
    if (h->servers > 0) return fail(PGX_ERROR_FUNCTION_CALL, "the handle is already served");
    if (h->device != p->device) return fail(PGX_ERROR_INVALID_PARAM, "handle and pool are on different devices");
    std::lock_guard<std::mutex> lock(p->mu);
    pgx_pool_s::Member m;
    m.h = h;
    m.base_bytes = h->eng->device_bytes(p->kdim) + h->eng->layout_bytes();
    for (auto& e : h->extra) m.base_bytes += e->slot_bytes(p->kdim);
    m.slot_bytes = h->eng->slot_bytes(p->kdim);
    if (p->in_use + m.base_bytes > p->budget)
      return fail(PGX_ERROR_OOM, "the handle needs %lld bytes; the pool has %lld of %lld left", (long long)m.base_bytes,
                  (long long)(p->budget - p->in_use), (long long)p->budget);
    m.slots.resize(1);  // the handle's own slot
    p->in_use += m.base_bytes;
    p->peak = std::max(p->peak, p->in_use);
    h->servers++;
    p->members.push_back(std::move(m));
    *index = (int32_t)p->members.size() - 1;
    return PGX_SUCCESS;
  });
}

int pgx_pool_submit(pgx_pool p, int32_t index, double* x, const double* b, int32_t location, int64_t request_id) {
  if (!p || !x || !b) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (request_id < 0) return fail(PGX_ERROR_INVALID_PARAM, "request id %lld < 0", (long long)request_id);
  if (location != PGX_LOCATION_HOST && location != PGX_LOCATION_DEVICE)
    return fail(PGX_ERROR_MEMORY_LOCATION, "unknown location %d", location);
  {
    std::lock_guard<std::mutex> lock(p->mu);
    if (index < 0 || index >= (int)p->members.size())
      return fail(PGX_ERROR_INVALID_PARAM, "member %d outside [0, %d)", index, (int)p->members.size());
    if (location == PGX_LOCATION_HOST &&
        !all_finite(b, (long long)p->members[index].h->im.n * p->members[index].h->im.vw))
      return fail(PGX_ERROR_NOT_FINITE, "b is not finite");
    p->queue.push_back({index, x, b, location, request_id});
  }
  p->cv.notify_one();
  return PGX_SUCCESS;
}

int pgx_pool_step(pgx_pool p, int32_t* n_active, int32_t* n_queued) {
  if (!p) return fail(PGX_ERROR_INVALID_PARAM, "null pool");
  if (p->running) return fail(PGX_ERROR_FUNCTION_CALL, "the pool steps on its own thread (pgx_pool_stop first)");
  std::lock_guard<std::mutex> lock(p->mu);
  return pool_step_locked(p, n_active, n_queued);
}

int pgx_pool_start(pgx_pool p) {
  if (!p) return fail(PGX_ERROR_INVALID_PARAM, "null pool");
  if (p->running) return fail(PGX_ERROR_FUNCTION_CALL, "the pool thread is already running");
  p->worker_rc = PGX_SUCCESS;
  p->running = true;
  p->worker = std::thread([p]() {
    while (p->running) {
      int32_t active = 0, queued = 0;
      {
        std::lock_guard<std::mutex> lock(p->mu);
        const int rc = pool_step_locked(p, &active, &queued);
        if (rc != PGX_SUCCESS && p->worker_rc == PGX_SUCCESS) {
          p->worker_rc = rc;
          p->worker_msg = g_last_error;
        }
      }
      if (active == 0 && queued == 0) {
        std::unique_lock<std::mutex> lock(p->mu);
        p->cv.wait_for(lock, std::chrono::milliseconds(2), [p]() { return !p->running || !p->queue.empty(); });
      } else {
        std::this_thread::sleep_for(std::chrono::microseconds(50));
      }
    }
  });
  return PGX_SUCCESS;
}

int pgx_pool_stop(pgx_pool p) {
  if (!p) return fail(PGX_ERROR_INVALID_PARAM, "null pool");
  if (!p->running) return PGX_SUCCESS;
  p->running = false;
  p->cv.notify_all();
  if (p->worker.joinable()) p->worker.join();
  if (p->worker_rc != PGX_SUCCESS) return fail(p->worker_rc, "pool thread: %s", p->worker_msg.c_str());
  return PGX_SUCCESS;
}

int pgx_pool_collect(pgx_pool p, int32_t max, int64_t* ids, pgx_result* results, int32_t* n) {
  if (!p || !n) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  std::lock_guard<std::mutex> lock(p->mu);
  int k = 0;
  while (k < max && !p->done.empty()) {
    if (ids) ids[k] = p->done.front().first;
    if (results) results[k] = p->done.front().second;
    p->done.pop_front();
    k++;
  }
  *n = k;
  return PGX_SUCCESS;
}

int pgx_pool_stats(pgx_pool p, int64_t* bytes_in_use, int64_t* peak_bytes, int32_t* slots) {
  if (!p) return fail(PGX_ERROR_INVALID_PARAM, "null pool");
  std::lock_guard<std::mutex> lock(p->mu);
  if (bytes_in_use) *bytes_in_use = p->in_use;
  if (peak_bytes) *peak_bytes = p->peak;
  if (slots) {
    int c = 0;
    for (auto& m : p->members) c += (int)m.slots.size();
    *slots = c;
  }
  return PGX_SUCCESS;
}

int pgx_pool_destroy(pgx_pool p) {
  if (!p) return PGX_SUCCESS;
  pgx_pool_stop(p);
  cudaSetDevice(p->device);
  for (auto& m : p->members) {
    for (auto& sl : m.slots) {
      if (sl.req < 0) continue;
      bool fin = false;
      pgx_result res;
      while (!fin)
        if (sl.get(m.h)->poll(true, &fin, &res) != PGX_SUCCESS) break;
    }
    m.slots.clear();  // the extra slots read the handle's factors: release them first
    m.h->servers--;
  }
  delete p;
  return PGX_SUCCESS;
}

int pgx_gemslr_kernel_stats(pgx_handle h, int32_t which, int32_t level, int32_t reps, double* avg_ms,
                            double* bytes) {
  if (!h || !avg_ms || !bytes) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (!h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "handle not committed");
  PGX_CUDA(cudaSetDevice(h->device));
  int launches = 0;
  if (which == 3 || which == 4) {
    // the merged passes of a multi-lane slot
    if (h->extra.empty() || h->extra.back()->lanes() < 2)
      return fail(PGX_ERROR_FUNCTION_CALL, "no multi-lane slot (pgx_gemslr_set_lanes, pgx_gemslr_set_slots)");
    return h->extra.back()->kernel_stats(which - 3, level, reps, avg_ms, bytes, &launches);
  }
  return h->eng->kernel_stats(which, level, reps, avg_ms, bytes, &launches);
}

int pgx_build_levels(char uplo, int32_t n, const int32_t* rowptr, const int32_t* colidx, int32_t* nlevels,
                     int32_t* level_ptr, int32_t* order) {
  return guarded("pgx_build_levels", [&]() -> int {
    if (n < 0 || (n > 0 && (!rowptr || !nlevels || !level_ptr || !order)))
      return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    if (uplo != 'L' && uplo != 'U') return fail(PGX_ERROR_INVALID_OPTION, "uplo must be 'L' or 'U'");
    for (int i = 0; i < n; i++)
      for (int k = rowptr[i]; k < rowptr[i + 1]; k++)
        if (colidx[k] < 0 || colidx[k] >= n) return fail(PGX_ERROR_INVALID_PARAM, "column index out of range");
    std::vector<int> lptr, ord;
    PGX_TRY(build_levels(uplo == 'U', n, rowptr, colidx, lptr, ord));
    *nlevels = (int)lptr.size() - 1;
    std::copy(lptr.begin(), lptr.end(), level_ptr);
    std::copy(ord.begin(), ord.end(), order);
    return PGX_SUCCESS;
  });
}

int pgx_csr_read_mm(const char* path, pgx_csr* A) {
  return guarded("pgx_csr_read_mm", [&]() -> int {
    if (!path || !A) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    memset(A, 0, sizeof(*A));
    setup::Csr c;
    std::string err;
    if (setup::read_matrix_market(path, c, err)) return fail(PGX_ERROR_IO, "%s: %s", path, err.c_str());
    const size_t nnz = c.cj.size();
    int32_t* rp = (int32_t*)malloc(sizeof(int32_t) * c.rp.size());
    int32_t* cj = (int32_t*)malloc(sizeof(int32_t) * std::max<size_t>(nnz, 1));
    double* va = (double*)malloc(sizeof(double) * std::max<size_t>(nnz, 1));
    if (!rp || !cj || !va) {
      free(rp);
      free(cj);
      free(va);
      return fail(PGX_ERROR_OOM, "host allocation for %zu nonzeros", nnz);
    }
    std::copy(c.rp.begin(), c.rp.end(), rp);
    std::copy(c.cj.begin(), c.cj.end(), cj);
    std::copy(c.va.begin(), c.va.end(), va);
    A->rows = c.rows;
    A->cols = c.cols;
    A->nnz = (int64_t)nnz;
    A->rowptr = rp;
    A->colidx = cj;
    A->values = va;
    return PGX_SUCCESS;
  });
}

int pgx_csr_free(pgx_csr* A) {
  if (!A) return PGX_SUCCESS;
  free((void*)A->rowptr);
  free((void*)A->colidx);
  free((void*)A->values);
  memset(A, 0, sizeof(*A));
  return PGX_SUCCESS;
}

int pgx_gemslr_nnz(pgx_handle h, int64_t* nnz_bsolver, int64_t* nnz_lr) {
  return guarded("pgx_gemslr_nnz", [&]() -> int {
    if (!h) return fail(PGX_ERROR_INVALID_PARAM, "null handle");
    const Import& im = h->im;
    if (im.nlev < 1) return fail(PGX_ERROR_FUNCTION_CALL, "levels not set");
    int64_t nb = 0, nl = 0;
    for (int l = 0; l < im.nlev; l++) {
      const HostLevel& hl = im.levels[l];
      if (!hl.set) return fail(PGX_ERROR_FUNCTION_CALL, "level %d not set", l);
      nb += (int64_t)(im.lev_ptr[l + 1] - im.lev_ptr[l]) + hl.L.nnz() + hl.U.nnz();
      nl += 2 * (int64_t)(im.n - im.lev_ptr[l + 1]) * hl.rank;
    }
    if (nnz_bsolver) *nnz_bsolver = nb;
    if (nnz_lr) *nnz_lr = nl;
    return PGX_SUCCESS;
  });
}

int pgx_vector_read_mm(const char* path, int32_t idxin, int32_t capacity, double* x, int32_t* n) {
  return guarded("pgx_vector_read_mm", [&]() -> int {
    if (!path || !n) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    std::vector<double> v;
    std::string err;
    if (setup::read_matrix_market_vector(path, idxin, v, err)) return fail(PGX_ERROR_IO, "%s: %s", path, err.c_str());
    *n = (int32_t)v.size();
    if (!x) return PGX_SUCCESS;
    if (capacity < *n) return fail(PGX_ERROR_INVALID_PARAM, "capacity %d below the vector's %d entries", capacity, *n);
    std::copy(v.begin(), v.end(), x);
    return PGX_SUCCESS;
  });
}

int pgx_params_default(double* params) {
  if (!params) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  params::set_defaults(params);
  return PGX_SUCCESS;
}

int pgx_params_read_file(const char* path, int32_t format, double* params) {
  return guarded("pgx_params_read_file", [&]() -> int {
    if (!path || !params) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    std::string err;
    const int rc = params::read_file(path, format, params, err);
    if (rc) return fail(rc, "%s", err.c_str());
    return PGX_SUCCESS;
  });
}

int pgx_params_read_args(int32_t argc, const char* const* argv, double* params) {
  return guarded("pgx_params_read_args", [&]() -> int {
    if (!params || argc < 0 || (argc > 0 && !argv)) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    params::read_args(argc, argv, params);
    return PGX_SUCCESS;
  });
}

int pgx_csr_spmv_plan(const pgx_csr* A, int32_t* lanes, int32_t* merge_path) {
  return guarded("pgx_csr_spmv_plan", [&]() -> int {
    if (!A || (A->rows > 0 && !A->rowptr)) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    if (A->rows < 0) return fail(PGX_ERROR_INVALID_PARAM, "rows %d < 0", A->rows);
    const SpmvPlan p = spmv_plan(A->rows, A->rowptr);
    if (lanes) *lanes = p.S;
    if (merge_path) *merge_path = p.merge ? 1 : 0;
    return PGX_SUCCESS;
  });
}

int pgx_csr_spmv_device_variant(const pgx_csr* Ad, int32_t variant, double alpha, const double* x, double beta,
                                double* y) {
  return guarded("pgx_csr_spmv_device_variant", [&]() -> int {
    if (!Ad || !x || !y) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    if (variant < 0 || variant > 2) return fail(PGX_ERROR_INVALID_OPTION, "unknown SpMV variant %d", variant);
    if (Ad->rows == 0) return PGX_SUCCESS;
    if (Ad->nnz > INT32_MAX || (long long)Ad->rows + Ad->nnz > INT32_MAX)
      return fail(PGX_ERROR_INVALID_PARAM, "matrix too large for 32-bit indices");
    // the plan needs the row pointer on the host
    std::vector<int> rp(Ad->rows + 1);
    PGX_CUDA(cudaMemcpy(rp.data(), Ad->rowptr, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost));
    const SpmvPlan p = spmv_plan(Ad->rows, rp.data());
    const bool merge = variant == 2 || (variant == 0 && p.merge);
    Skip sk = mk_skip();
    const double* b = beta != 0.0 ? y : nullptr;
    if (merge) {
      const int nt = merge_threads(Ad->rows, Ad->nnz);
      Arena tmp;
      int* crow = nullptr;
      double* cval = nullptr;
      PGX_TRY(tmp.alloc(&crow, (size_t)nt));
      PGX_TRY(tmp.alloc(&cval, (size_t)nt));
      merge_spmv_kernel<double, double, double, double><<<(nt + 255) / 256, 256>>>(
          Ad->rows, (int)Ad->nnz, Ad->rowptr, Ad->colidx, Ad->values, x, alpha, b, beta, y, crow, cval, sk);
      merge_spmv_fixup_kernel<double, double><<<grid_for(nt, 256, num_sms() * 8), 256>>>(nt, crow, cval, alpha, y, sk);
      PGX_CUDA(cudaGetLastError());
      PGX_CUDA(cudaDeviceSynchronize());
      return PGX_SUCCESS;
    }
    const int S = p.S;
    const int grid = grid_for(Ad->rows, 256 / S, num_sms() * 16);
    // caller-owned arrays: 128-bit loads only where both are 16-byte aligned
    // and the nonzeros fill whole 4-entry blocks
    const bool vec = ((uintptr_t)Ad->colidx % 16 == 0) && ((uintptr_t)Ad->values % 16 == 0) && Ad->nnz % 4 == 0;
#define PGX_SPMV1(SS)                                                                                             \
  if (vec)                                                                                                        \
    spmv_kernel<double, double, double, double, SS, true><<<grid, 256>>>(                                         \
        Ad->rows, Ad->rowptr, Ad->colidx, Ad->values, x, Ad->cols, alpha, nullptr, nullptr, nullptr, nullptr, 0, \
        0.0, b, beta, y, nullptr, nullptr, sk);                                                                   \
  else                                                                                                            \
    spmv_kernel<double, double, double, double, SS, false><<<grid, 256>>>(                                        \
        Ad->rows, Ad->rowptr, Ad->colidx, Ad->values, x, Ad->cols, alpha, nullptr, nullptr, nullptr, nullptr, 0, \
        0.0, b, beta, y, nullptr, nullptr, sk)
    switch (S) {
      case 2: PGX_SPMV1(2); break;
      case 4: PGX_SPMV1(4); break;
      case 8: PGX_SPMV1(8); break;
      case 16: PGX_SPMV1(16); break;
      default: PGX_SPMV1(32); break;
    }
#undef PGX_SPMV1
    PGX_CUDA(cudaGetLastError());
    PGX_CUDA(cudaDeviceSynchronize());
    return PGX_SUCCESS;
  });
}

int pgx_lowrank_block_apply_c64(int32_t m, int32_t r, int32_t nrhs, const void* W, const void* WH, void* X,
                                int64_t ldx) {
  return guarded("pgx_lowrank_block_apply_c64", [&]() -> int {
    if (!W || !WH || !X) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    if (m < 1 || r < 1 || r > kUmmaMaxRank || ldx < m)
      return fail(PGX_ERROR_INVALID_PARAM, "m %d, r %d (1..%d), ldx %lld", m, r, kUmmaMaxRank, (long long)ldx);
    switch (nrhs) {
      case 8: return lowrank_block_apply<8>(m, r, (const cf32*)W, (const cf32*)WH, (cf32*)X, ldx);
      case 16: return lowrank_block_apply<16>(m, r, (const cf32*)W, (const cf32*)WH, (cf32*)X, ldx);
      default: return fail(PGX_ERROR_INVALID_PARAM, "nrhs %d: 8 or 16", nrhs);
    }
  });
}

int pgx_csr_spmv_device(const pgx_csr* Ad, double alpha, const double* x, double beta, double* y) {
  return pgx_csr_spmv_device_variant(Ad, 0, alpha, x, beta, y);
}

// ------------------------------------------------- many systems, one launch
struct pgx_systems_s {
  std::unique_ptr<SystemsBase> impl;
  int device = 0;
  int count = 0;
};

int pgx_systems_create(pgx_systems* out, const pgx_handle* handles, int32_t count) {
  return guarded("pgx_systems_create", [&]() -> int {
    if (!out || !handles || count < 1) return fail(PGX_ERROR_INVALID_PARAM, "null argument or count %d", count);
    *out = nullptr;
    std::vector<const Import*> ims(count);
    int precision = -1, device = -1;
    for (int s = 0; s < count; s++) {
      pgx_handle h = handles[s];
      if (!h || !h->eng) return fail(PGX_ERROR_FUNCTION_CALL, "system %d: handle not committed", s);
      if (s == 0) {
        precision = h->im.precision;
        device = h->device;
      }
      if (h->im.precision != precision) return fail(PGX_ERROR_INVALID_PARAM, "system %d: precisions differ", s);
      if (h->device != device) return fail(PGX_ERROR_INVALID_PARAM, "system %d: devices differ", s);
      ims[s] = &h->im;
    }
    if (precision != PGX_PRECISION_MIXED && precision != PGX_PRECISION_FP64)
      return fail(PGX_ERROR_INVALID_OPTION, "the systems solve is real only (precision %d)", precision);
    std::unique_ptr<pgx_systems_s> o(new pgx_systems_s());
    o->device = device;
    o->count = count;
    if (precision == PGX_PRECISION_MIXED) {
      auto* sy = new Systems<float>();
      o->impl.reset(sy);
      PGX_TRY(sy->create(ims, device));
    } else {
      auto* sy = new Systems<double>();
      o->impl.reset(sy);
      PGX_TRY(sy->create(ims, device));
    }
    *out = o.release();
    return PGX_SUCCESS;
  });
}

int pgx_systems_solve(pgx_systems s, double* const* x, const double* const* b, int32_t location,
                      const double* params, pgx_result* results) {
  return guarded("pgx_systems_solve", [&]() -> int {
    if (!s || !x || !b) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    int kdim, maxits, atol;
    double tol;
    read_solver_params(params, kdim, maxits, tol, atol);
    return s->impl->solve(x, b, location, kdim, maxits, tol, atol, results);
  });
}

int pgx_systems_tune(pgx_systems s, const double* const* b, int32_t location, const double* params, int32_t stride,
                     double* best_ms) {
  return guarded("pgx_systems_tune", [&]() -> int {
    if (!s || !b) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
    int kdim, maxits, atol;
    double tol;
    read_solver_params(params, kdim, maxits, tol, atol);
    return s->impl->tune(b, location, kdim, maxits, tol, atol, stride, best_ms);
  });
}

int pgx_systems_tune_table(pgx_systems s, int32_t capacity, double* table, int32_t* rows) {
  if (!s) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  const auto& t = s->impl->tune_table;
  if (rows) *rows = (int32_t)t.size();
  if (table)
    for (int i = 0; i < (int)t.size() && i < capacity; i++)
      for (int k = 0; k < 5; k++) table[5 * i + k] = t[i][k];
  return PGX_SUCCESS;
}

int pgx_systems_set_schedule(pgx_systems s, int32_t threads, int32_t ctas_per_sm, int32_t lanes, int32_t depth) {
  if (!s) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (threads < 64 || threads > kSysMaxThreads || threads % 32)
    return fail(PGX_ERROR_INVALID_PARAM, "threads %d: a multiple of 32 in [64, %d]", threads, kSysMaxThreads);
  if (ctas_per_sm < 1 || ctas_per_sm > 32) return fail(PGX_ERROR_INVALID_PARAM, "ctas_per_sm %d", ctas_per_sm);
  if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
    return fail(PGX_ERROR_INVALID_PARAM, "lanes %d: a power of two up to 32", lanes);
  if (depth != 2 && depth != 3) return fail(PGX_ERROR_INVALID_PARAM, "depth %d: 2 or 3", depth);
  s->impl->threads = threads;
  s->impl->ctas_per_sm = ctas_per_sm;
  s->impl->lanes = lanes;
  s->impl->depth = depth;
  return PGX_SUCCESS;
}

int pgx_systems_get_schedule(pgx_systems s, int32_t* threads, int32_t* ctas_per_sm, int32_t* lanes, int32_t* depth) {
  if (!s) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  if (threads) *threads = s->impl->threads;
  if (ctas_per_sm) *ctas_per_sm = s->impl->ctas_per_sm;
  if (lanes) *lanes = s->impl->lanes;
  if (depth) *depth = s->impl->depth;
  return PGX_SUCCESS;
}

int pgx_systems_timing(pgx_systems s, int32_t capacity, double* start_ms, double* end_ms, double* tri_ms) {
  if (!s) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  const int k = std::min<int>(capacity, (int)s->impl->t_start.size());
  for (int i = 0; i < k; i++) {
    if (start_ms) start_ms[i] = s->impl->t_start[i];
    if (end_ms) end_ms[i] = s->impl->t_end[i];
    if (tri_ms) tri_ms[i] = s->impl->t_tri[i];
  }
  return PGX_SUCCESS;
}

int pgx_systems_last_ms(pgx_systems s, double* ms) {
  if (!s || !ms) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  *ms = s->impl->last_ms;
  return PGX_SUCCESS;
}

int pgx_systems_device_bytes(pgx_systems s, int64_t* bytes) {
  if (!s || !bytes) return fail(PGX_ERROR_INVALID_PARAM, "null argument");
  *bytes = s->impl->device_bytes();
  return PGX_SUCCESS;
}

int pgx_systems_destroy(pgx_systems s) {
  if (!s) return PGX_SUCCESS;
  cudaSetDevice(s->device);
  delete s;
  return PGX_SUCCESS;
}

}  // extern "C"
