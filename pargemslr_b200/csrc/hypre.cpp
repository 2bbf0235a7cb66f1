// The reference's hypre plugin interface (TESTS/hypre/pargemslr_hypre_interface.hpp)
// over this library's C ABI; the contract is in include/pgx_hypre.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/pgx_hypre.h"
#include "pgx_internal.h"

namespace {

struct HypreMatrix {
  int n = 0;
  int location = PGX_LOCATION_HOST;
  std::vector<int> rp, cj;
  std::vector<double> va;
};

struct HypreGemslr {
  double params[PGX_PARAMS_SIZE];
  int precision = PGX_PRECISION_FP64;
  int location = PGX_LOCATION_HOST;  // of the vectors, from the matrix given at Setup
  pgx_handle h = nullptr;
};

int err(int code, const std::string& msg) { return pgx::set_error(code, msg.c_str()); }

// count entries of src, on the host or the device, into dst
template <class T>
int fetch(std::vector<T>& dst, const T* src, size_t count, int location, const char* what) {
  dst.assign(count, T());
  if (count == 0) return PGX_SUCCESS;
  if (!src) return err(PGX_ERROR_INVALID_PARAM, std::string(what) + " is NULL");
  if (location == PGX_LOCATION_HOST) {
    std::copy(src, src + count, dst.begin());
    return PGX_SUCCESS;
  }
  const cudaError_t e = cudaMemcpy(dst.data(), src, sizeof(T) * count, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return err(PGX_ERROR_CUDA, std::string("copying ") + what + ": " + cudaGetErrorString(e));
  return PGX_SUCCESS;
}

int build_matrix(HypreMatrix& m, long int nrow_global, long int ncol_global, long int nrow_start, long int ncol_start,
                 int nrow_local, int ncol_local, const int* diag_i, const int* diag_j, const double* diag_data,
                 const int* offd_i, int n_offd_map, int location) {
  if (location != PGX_LOCATION_HOST && location != PGX_LOCATION_DEVICE)
    return err(PGX_ERROR_MEMORY_LOCATION, "data_location must be 0 (host) or 1 (device)");
  if (nrow_local <= 0 || nrow_local != ncol_local)
    return err(PGX_ERROR_INVALID_PARAM, "the local block must be square and non-empty");
  if (nrow_global != nrow_local || ncol_global != ncol_local || nrow_start != 0 || ncol_start != 0)
    return err(PGX_ERROR_INVALID_PARAM,
               "one rank only: rows " + std::to_string(nrow_start) + ".." + std::to_string(nrow_start + nrow_local) +
                   " of " + std::to_string(nrow_global) + " given, the whole system is needed");
  const int n = nrow_local;
  int rc = fetch(m.rp, diag_i, (size_t)n + 1, location, "diag_i");
  if (rc) return rc;
  if (m.rp[0] != 0) return err(PGX_ERROR_INVALID_PARAM, "diag_i[0] must be 0");
  for (int r = 0; r < n; r++)
    if (m.rp[r + 1] < m.rp[r]) return err(PGX_ERROR_INVALID_PARAM, "diag_i decreases at row " + std::to_string(r));
  const size_t nnz = (size_t)m.rp[n];
  if ((rc = fetch(m.cj, diag_j, nnz, location, "diag_j"))) return rc;
  if ((rc = fetch(m.va, diag_data, nnz, location, "diag_data"))) return rc;
  // the off-diagonal part couples to other ranks' rows: it must be empty here
  if (n_offd_map < 0) return err(PGX_ERROR_INVALID_PARAM, "n_offd_map is negative");
  if (offd_i) {
    std::vector<int> orp;
    if ((rc = fetch(orp, offd_i, (size_t)n + 1, location, "offd_i"))) return rc;
    if (orp[n] != orp[0]) return err(PGX_ERROR_INVALID_PARAM, "off-diagonal entries given: one rank only");
  }
  // columns in range and sorted within each row (hypre keeps the diagonal first)
  std::vector<int> order;
  std::vector<int> cj2;
  std::vector<double> va2;
  for (int r = 0; r < n; r++) {
    const int b = m.rp[r], e = m.rp[r + 1];
    for (int k = b; k < e; k++)
      if (m.cj[k] < 0 || m.cj[k] >= n)
        return err(PGX_ERROR_INVALID_PARAM, "column " + std::to_string(m.cj[k]) + " out of range in row " +
                                                std::to_string(r));
    if (std::is_sorted(m.cj.begin() + b, m.cj.begin() + e)) continue;
    order.resize(e - b);
    std::iota(order.begin(), order.end(), b);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return m.cj[x] < m.cj[y]; });
    cj2.resize(e - b);
    va2.resize(e - b);
    for (int t = 0; t < e - b; t++) {
      cj2[t] = m.cj[order[t]];
      va2[t] = m.va[order[t]];
    }
    std::copy(cj2.begin(), cj2.end(), m.cj.begin() + b);
    std::copy(va2.begin(), va2.end(), m.va.begin() + b);
  }
  m.n = n;
  m.location = location;
  return PGX_SUCCESS;
}

}  // namespace

extern "C" {

int pgx_hypre_init_gpu(int device) { return pgx_init(device); }

int pgx_hypre_finalize_gpu(void) { return pgx_finalize(); }

void* pgx_hypre_csr_matrix_create(long int nrow_global, long int ncol_global, long int nrow_start,
                                  long int ncol_start, int nrow_local, int ncol_local, int* diag_i, int* diag_j,
                                  double* diag_data, int* offd_i, int* /*offd_j*/, double* /*offd_data*/,
                                  int n_offd_map, long int* /*offd_map*/, int data_location) {
  try {
    std::unique_ptr<HypreMatrix> m(new HypreMatrix());
    if (build_matrix(*m, nrow_global, ncol_global, nrow_start, ncol_start, nrow_local, ncol_local, diag_i, diag_j,
                     diag_data, offd_i, n_offd_map, data_location))
      return nullptr;
    return m.release();
  } catch (const std::bad_alloc&) {
    err(PGX_ERROR_OOM, "host allocation for the matrix failed");
    return nullptr;
  }
}

int pgx_hypre_csr_matrix_destroy(void* matrix) {
  delete static_cast<HypreMatrix*>(matrix);
  return PGX_SUCCESS;
}

int pgx_hypre_csr_matrix_view(void* matrix, pgx_csr* A) {
  if (!matrix || !A) return err(PGX_ERROR_INVALID_PARAM, "null argument");
  const HypreMatrix& m = *static_cast<HypreMatrix*>(matrix);
  A->rows = A->cols = m.n;
  A->nnz = (int64_t)m.cj.size();
  A->rowptr = m.rp.data();
  A->colidx = m.cj.data();
  A->values = m.va.data();
  return PGX_SUCCESS;
}

void* pgx_hypre_gemslr_create(void) {
  HypreGemslr* g = new (std::nothrow) HypreGemslr();
  if (!g) {
    err(PGX_ERROR_OOM, "host allocation");
    return nullptr;
  }
  pgx_params_default(g->params);
  return g;
}

int pgx_hypre_gemslr_destroy(void* gemslr) {
  HypreGemslr* g = static_cast<HypreGemslr*>(gemslr);
  if (!g) return PGX_SUCCESS;
  if (g->h) pgx_gemslr_destroy(g->h);
  delete g;
  return PGX_SUCCESS;
}

int pgx_hypre_gemslr_set_params(void* gemslr, double* params) {
  if (!gemslr || !params) return err(PGX_ERROR_INVALID_PARAM, "null argument");
  std::memcpy(static_cast<HypreGemslr*>(gemslr)->params, params, sizeof(double) * PGX_PARAMS_SIZE);
  return PGX_SUCCESS;
}

int pgx_hypre_gemslr_set_precision(void* gemslr, int precision) {
  HypreGemslr* g = static_cast<HypreGemslr*>(gemslr);
  if (!g) return err(PGX_ERROR_INVALID_PARAM, "null argument");
  if (precision != PGX_PRECISION_FP64 && precision != PGX_PRECISION_MIXED)
    return err(PGX_ERROR_INVALID_OPTION, "unknown precision " + std::to_string(precision));
  if (g->h) return err(PGX_ERROR_FUNCTION_CALL, "precision set after setup");
  g->precision = precision;
  return PGX_SUCCESS;
}

int pgx_hypre_gemslr_setup(void* gemslr, void* matrix, double* /*x*/, double* /*rhs*/) {
  HypreGemslr* g = static_cast<HypreGemslr*>(gemslr);
  if (!g || !matrix) return err(PGX_ERROR_INVALID_PARAM, "null argument");
  if (g->h) return PGX_SUCCESS;
  const HypreMatrix& m = *static_cast<HypreMatrix*>(matrix);
  pgx_csr a;
  pgx_hypre_csr_matrix_view(matrix, &a);
  pgx_handle h = nullptr;
  const int rc = pgx_gemslr_setup(&h, &a, g->params, g->precision);
  if (rc) return rc;
  g->h = h;
  g->location = m.location;
  return PGX_SUCCESS;
}

int pgx_hypre_gemslr_solve(void* gemslr, void* /*matrix*/, double* x, double* rhs) {
  HypreGemslr* g = static_cast<HypreGemslr*>(gemslr);
  if (!g || !x || !rhs) return err(PGX_ERROR_INVALID_PARAM, "null argument");
  if (!g->h) return err(PGX_ERROR_FUNCTION_CALL, "solve before setup");
  return pgx_gemslr_precond_apply(g->h, x, rhs, g->location);
}

pgx_handle pgx_hypre_gemslr_handle(void* gemslr) { return gemslr ? static_cast<HypreGemslr*>(gemslr)->h : nullptr; }

double* pgx_hypre_params_from_file(const char* filename) {
  double* p = static_cast<double*>(malloc(sizeof(double) * PGX_PARAMS_SIZE));
  if (!p) {
    err(PGX_ERROR_OOM, "host allocation");
    return nullptr;
  }
  pgx_params_default(p);
  if (filename) pgx_params_read_file(filename, PGX_INPUTS_HYPRE, p);
  return p;
}

int pgx_hypre_params_destroy(double* params) {
  free(params);
  return PGX_SUCCESS;
}

}  // extern "C"
