/*
 * pgx_pargemslr.hpp — the reference's solver classes over the C ABI of pgx.h.
 *
 * A ParGeMSLR driver builds a matrix, a GeMSLR preconditioner and a flexible
 * GMRES solver, then calls Setup(x, b) and Solve(x, b) and reads the
 * iteration count and residual back
 * (TESTS/parallel/driver_laplacian_gemslr_par.cpp:379-425).  The classes here
 * keep those names, argument meanings and int status codes for one rank in
 * FP64, so such a driver moves its solve to the GPU by switching its types:
 *
 *   pargemslr::ParallelCsrMatrixClass<double>  -> pgx::ParallelCsrMatrixClass<double>
 *   pargemslr::ParallelVectorClass<double>     -> pgx::ParallelVectorClass<double>
 *   pargemslr::ParallelGemslrClass<M, V, double>  -> pgx::ParallelGemslrClass<M, V, double>
 *   pargemslr::FlexGmresClass<M, V, double>    -> pgx::FlexGmresClass<M, V, double>
 *
 * (M, V = ParallelCsrMatrixClass<double>, ParallelVectorClass<double>; the
 * reference's typedefs matrix_csr_par_double, vector_par_double,
 * precond_gemslr_csr_par_double and fgmres_csr_par_double exist here too).
 *
 * Setup runs this library's host setup (pgx_gemslr_setup) and moves the
 * preconditioner to the device; Solve runs FGMRES there (pgx_gemslr_solve).
 * Vectors may live on the host or on the device (kMemoryHost/kMemoryDevice).
 * What is not kept: MPI (one rank), complex and single-precision types, the
 * residual history GetRelativeResidual (only the final residual is recorded),
 * and unpreconditioned FGMRES.  Header-only; link with -lpgx.
 */
#ifndef PGX_PARGEMSLR_HPP
#define PGX_PARGEMSLR_HPP

#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#include "pgx.h"

namespace pgx {

/* the reference's memory locations (SRC/utils/memory.hpp:23-24) */
enum { kMemoryHost = PGX_LOCATION_HOST, kMemoryDevice = PGX_LOCATION_DEVICE };

/* ParallelVectorClass<double> on one rank (SRC/vectors/parallel_vector.hpp):
 * owns a host array after Setup, or borrows a host or device array after
 * SetupPtr/UpdatePtr. */
template <typename T>
class ParallelVectorClass {
  static_assert(std::is_same<T, double>::value, "the GPU solve path is FP64 at its boundary");

 public:
  ParallelVectorClass() {}
  ParallelVectorClass(const ParallelVectorClass&) = delete;
  ParallelVectorClass& operator=(const ParallelVectorClass&) = delete;

  int Setup(int n_local) {
    if (n_local < 0) return PGX_ERROR_INVALID_PARAM;
    own_.assign((size_t)n_local, 0.0);
    data_ = own_.data();
    n_ = n_local;
    location_ = kMemoryHost;
    return PGX_SUCCESS;
  }
  int SetupPtr(double* data, int n_local, int location) {
    if (n_local < 0 || (n_local > 0 && !data)) return PGX_ERROR_INVALID_PARAM;
    if (location != kMemoryHost && location != kMemoryDevice) return PGX_ERROR_MEMORY_LOCATION;
    own_.clear();
    data_ = data;
    n_ = n_local;
    location_ = location;
    return PGX_SUCCESS;
  }
  int UpdatePtr(double* data, int location) { return SetupPtr(data, n_, location); }
  /* host vectors only, like the host path of VectorClass::Fill */
  int Fill(double v) {
    if (location_ != kMemoryHost) return PGX_ERROR_MEMORY_LOCATION;
    for (int i = 0; i < n_; i++) data_[i] = v;
    return PGX_SUCCESS;
  }
  /* A vector in a coordinate Matrix Market file (SequentialVectorClass::
   * ReadFromMMFile, sequential_vector.hpp:572); idxin is the file's index
   * base.  The vector becomes an owned host vector. */
  int ReadFromMMFile(const char* vecfile, int idxin) {
    int32_t n = 0;
    int rc = pgx_vector_read_mm(vecfile, idxin, 0, nullptr, &n);
    if (rc) return rc;
    own_.assign((size_t)n, 0.0);
    rc = pgx_vector_read_mm(vecfile, idxin, n, own_.data(), &n);
    if (rc) return rc;
    data_ = own_.data();
    n_ = n;
    location_ = kMemoryHost;
    return PGX_SUCCESS;
  }
  double* GetData() const { return data_; }
  int GetLengthLocal() const { return n_; }
  long int GetLengthGlobal() const { return n_; }
  int GetDataLocation() const { return location_; }

 private:
  std::vector<double> own_;
  double* data_ = nullptr;
  int n_ = 0;
  int location_ = kMemoryHost;
};

/* ParallelCsrMatrixClass<double> on one rank: a host CSR matrix with 0-based
 * int32 indices (SRC/matrices/parallel_csr_matrix.hpp, csr_matrix.hpp). */
template <typename T>
class ParallelCsrMatrixClass {
  static_assert(std::is_same<T, double>::value, "the GPU solve path is FP64 at its boundary");

 public:
  /* nrows x ncols with room for nnz entries, row pointers zeroed; fill
   * GetI/GetJ/GetData afterwards */
  int Setup(int nrows, int ncols, int nnz) {
    if (nrows < 0 || ncols < 0 || nnz < 0) return PGX_ERROR_INVALID_PARAM;
    rows_ = nrows;
    cols_ = ncols;
    rp_.assign((size_t)nrows + 1, 0);
    cj_.assign((size_t)nnz, 0);
    va_.assign((size_t)nnz, 0.0);
    return PGX_SUCCESS;
  }
  int* GetI() { return rp_.data(); }
  int* GetJ() { return cj_.data(); }
  double* GetData() { return va_.data(); }
  int GetNumRowsLocal() const { return rows_; }
  int GetNumColsLocal() const { return cols_; }
  long int GetNumRowsGlobal() const { return rows_; }
  long int GetNumColsGlobal() const { return cols_; }
  long int GetNumNonzeros() const { return (long int)cj_.size(); }

  /* The reference's finite-difference stencil on an nx x ny x nz grid
   * (CsrMatrixClass::Laplacian, csr_matrix.hpp:639; stencil in
   * SRC/matrices/coo_matrix.cpp:519-614): off-diagonals -1 +/- alpha along each
   * axis, diagonal 6 - shift in 3D and 4 - shift when a dimension is 1, each
   * row's entries in the order z-, z+, y-, y+, x-, x+, diagonal, Dirichlet
   * boundaries by truncation. */
  int Laplacian(int nx, int ny, int nz, double alphax, double alphay, double alphaz, double shift) {
    if (nx <= 0 || ny <= 0 || nz <= 0) return PGX_ERROR_INVALID_PARAM;
    const long long nn = (long long)nx * ny * nz;
    if (nn > 0x7fffffffLL / 7) return PGX_ERROR_INVALID_PARAM;
    const int n = (int)nn, nxy = nx * ny;
    const double vd = ((nx == 1 || ny == 1 || nz == 1) ? 4.0 : 6.0) - shift;
    rows_ = cols_ = n;
    rp_.assign((size_t)n + 1, 0);
    cj_.clear();
    va_.clear();
    cj_.reserve((size_t)n * 7);
    va_.reserve((size_t)n * 7);
    for (int r = 0; r < n; r++) {
      const int k = r / nxy, i = (r - k * nxy) / nx, j = r - k * nxy - i * nx;
      if (k > 0) put(r - nxy, -1.0 + alphaz);
      if (k < nz - 1) put(r + nxy, -1.0 - alphaz);
      if (i > 0) put(r - nx, -1.0 + alphay);
      if (i < ny - 1) put(r + nx, -1.0 - alphay);
      if (j > 0) put(r - 1, -1.0 + alphax);
      if (j < nx - 1) put(r + 1, -1.0 - alphax);
      put(r, vd);
      rp_[(size_t)r + 1] = (int)cj_.size();
    }
    return PGX_SUCCESS;
  }

  /* A coordinate Matrix Market file (CsrMatrixClass::ReadFromMMFile,
   * csr_matrix.hpp:657).  Only 1-based files (idxin = 1, the format's own
   * convention) are read. */
  int ReadFromMMFile(const char* matfile, int idxin) {
    if (idxin != 1) return PGX_ERROR_INVALID_OPTION;
    pgx_csr c;
    const int rc = pgx_csr_read_mm(matfile, &c);
    if (rc) return rc;
    rows_ = c.rows;
    cols_ = c.cols;
    rp_.assign(c.rowptr, c.rowptr + c.rows + 1);
    cj_.assign(c.colidx, c.colidx + c.nnz);
    va_.assign(c.values, c.values + c.nnz);
    pgx_csr_free(&c);
    return PGX_SUCCESS;
  }

  /* y = alpha A x + beta y on host vectors, each row summed in stored order
   * (trans 'N' only). */
  int MatVec(char trans, double alpha, const ParallelVectorClass<T>& x, double beta, ParallelVectorClass<T>& y) const {
    if (trans != 'N' && trans != 'n') return PGX_ERROR_INVALID_OPTION;
    if (x.GetDataLocation() != kMemoryHost || y.GetDataLocation() != kMemoryHost) return PGX_ERROR_MEMORY_LOCATION;
    if (x.GetLengthLocal() != cols_ || y.GetLengthLocal() != rows_) return PGX_ERROR_INVALID_PARAM;
    const double* xd = x.GetData();
    double* yd = y.GetData();
    for (int r = 0; r < rows_; r++) {
      double s = 0.0;
      for (int k = rp_[(size_t)r]; k < rp_[(size_t)r + 1]; k++) s += va_[(size_t)k] * xd[cj_[(size_t)k]];
      yd[r] = beta == 0.0 ? alpha * s : alpha * s + beta * yd[r];
    }
    return PGX_SUCCESS;
  }

  /* the borrowed C-ABI view */
  pgx_csr View() const {
    pgx_csr c = {rows_, cols_, (int64_t)cj_.size(), rp_.data(), cj_.data(), va_.data()};
    return c;
  }

 private:
  void put(int col, double v) {
    cj_.push_back(col);
    va_.push_back(v);
  }
  int rows_ = 0, cols_ = 0;
  std::vector<int> rp_, cj_;
  std::vector<double> va_;
};

/* ParallelGemslrClass<..., double> (SRC/preconditioners/parallel_gemslr.hpp)
 * on one GPU.  Setup builds the multilevel preconditioner with this library's
 * host setup and moves it to the device; Solve applies it once, x = M^-1 rhs,
 * as the reference preconditioner's Solve does. */
template <class MatrixType, class VectorType, typename DataType>
class ParallelGemslrClass {
  static_assert(std::is_same<MatrixType, ParallelCsrMatrixClass<double>>::value &&
                    std::is_same<VectorType, ParallelVectorClass<double>>::value &&
                    std::is_same<DataType, double>::value,
                "one rank, FP64: ParallelCsrMatrixClass<double>, ParallelVectorClass<double>, double");

 public:
  ParallelGemslrClass() { pgx_params_default(params_); }
  ~ParallelGemslrClass() { Clear(); }
  ParallelGemslrClass(const ParallelGemslrClass&) = delete;
  ParallelGemslrClass& operator=(const ParallelGemslrClass&) = delete;

  int Clear() {
    if (h_) pgx_gemslr_destroy(h_);
    h_ = nullptr;
    return PGX_SUCCESS;
  }
  int SetMatrixP(MatrixType* A) {
    matrix_ = A;
    return PGX_SUCCESS;
  }
  MatrixType* GetMatrix() const { return matrix_; }
  int SetWithParameterArray(double* params) {
    if (!params) return PGX_ERROR_INVALID_PARAM;
    std::memcpy(params_, params, sizeof(params_));
    return PGX_SUCCESS;
  }
  /* Vectors carry their own location; this records the driver's choice only. */
  int SetSolveLocation(const int& location) {
    location_ = location;
    return PGX_SUCCESS;
  }
  /* PGX_PRECISION_FP64 (the default, the reference's arithmetic) or
   * PGX_PRECISION_MIXED (FP32 preconditioner inside FP64 FGMRES); before Setup. */
  int SetPrecision(int precision) {
    if (precision != PGX_PRECISION_FP64 && precision != PGX_PRECISION_MIXED) return PGX_ERROR_INVALID_OPTION;
    precision_ = precision;
    return PGX_SUCCESS;
  }
  /* Builds the preconditioner once; later calls return at once, as the
   * reference's do once the preconditioner is ready. */
  int Setup(VectorType& /*x*/, VectorType& /*rhs*/) {
    if (h_) return PGX_SUCCESS;
    if (!matrix_) return PGX_ERROR_FUNCTION_CALL;
    const pgx_csr a = matrix_->View();
    return pgx_gemslr_setup(&h_, &a, params_, precision_);
  }
  int Solve(VectorType& x, VectorType& rhs) {
    if (!h_) return PGX_ERROR_FUNCTION_CALL;
    if (x.GetDataLocation() != rhs.GetDataLocation()) return PGX_ERROR_MEMORY_LOCATION;
    return pgx_gemslr_precond_apply(h_, x.GetData(), rhs.GetData(), x.GetDataLocation());
  }
  /* nonzeros of the ILU factors and of the low-rank bases; returns their sum
   * (ParallelGemslrClass::GetNumNonzeros, parallel_gemslr.cpp:7609), or -1
   * before Setup */
  long int GetNumNonzeros(long int& nnz_bsolver, long int& nnz_lr) const {
    int64_t b = 0, l = 0;
    if (!h_ || pgx_gemslr_nnz(h_, &b, &l)) return -1;
    nnz_bsolver = (long int)b;
    nnz_lr = (long int)l;
    return (long int)(b + l);
  }
  long int GetNumNonzeros() const {
    long int b, l;
    return GetNumNonzeros(b, l);
  }
  /* the C-ABI handle, for the batch and serving calls of pgx.h */
  pgx_handle GetHandle() const { return h_; }

 private:
  double params_[PGX_PARAMS_SIZE];
  MatrixType* matrix_ = nullptr;
  pgx_handle h_ = nullptr;
  int precision_ = PGX_PRECISION_FP64;
  int location_ = kMemoryHost;
};

/* FlexGmresClass<ParallelCsrMatrixClass<double>, ParallelVectorClass<double>,
 * double> (SRC/solvers/fgmres.hpp), right-preconditioned by a
 * ParallelGemslrClass and run on the GPU.  The solver and its preconditioner
 * must share the matrix. */
template <class MatrixType, class VectorType, typename DataType>
class FlexGmresClass {
 public:
  typedef ParallelGemslrClass<MatrixType, VectorType, DataType> PrecondType;

  FlexGmresClass() {
    pgx_params_default(params_);
    std::memset(&result_, 0, sizeof(result_));
  }
  FlexGmresClass(const FlexGmresClass&) = delete;
  FlexGmresClass& operator=(const FlexGmresClass&) = delete;

  int SetMatrixP(MatrixType* A) {
    matrix_ = A;
    return PGX_SUCCESS;
  }
  int SetPreconditionerP(PrecondType* P) {
    precond_ = P;
    return PGX_SUCCESS;
  }
  /* the solver's slots only: tolerance, maximum iterations, Krylov dimension,
   * absolute tolerance and print level (fgmres.hpp:595-603) */
  int SetWithParameterArray(double* params) {
    if (!params) return PGX_ERROR_INVALID_PARAM;
    const int slots[] = {11, 12, 13, 14, 150};  // KDIM, MAXITS, TOL, ATOL, PRINT_LEVEL
    for (int s : slots) params_[s] = params[s];
    return PGX_SUCCESS;
  }
  template <typename T>
  int SetTolerance(T tol) {
    params_[13] = (double)tol;
    return PGX_SUCCESS;
  }
  int SetMaxNumberIterations(int maxits) {
    params_[12] = maxits;
    return PGX_SUCCESS;
  }
  int SetKrylovSubspaceDimension(int kdim) {
    params_[11] = kdim;
    return PGX_SUCCESS;
  }
  int SetAbsoluteTol(bool option) {
    params_[14] = option ? 1.0 : 0.0;
    return PGX_SUCCESS;
  }
  int SetSolveLocation(const int& location) {
    location_ = location;
    return PGX_SUCCESS;
  }
  /* sets the preconditioner up (once), as FlexGmresClass::Setup does
   * (fgmres.hpp:230-254) */
  int Setup(VectorType& x, VectorType& rhs) {
    if (ready_) return PGX_SUCCESS;
    if (!precond_) return PGX_ERROR_INVALID_PARAM;  // the GPU path is GeMSLR-preconditioned
    if (!matrix_) matrix_ = precond_->GetMatrix();
    if (!precond_->GetMatrix()) precond_->SetMatrixP(matrix_);
    if (precond_->GetMatrix() != matrix_) return PGX_ERROR_INVALID_PARAM;
    precond_->SetSolveLocation(location_);
    const int rc = precond_->Setup(x, rhs);
    if (rc) return rc;
    ready_ = true;
    return PGX_SUCCESS;
  }
  /* x holds the initial guess on entry and the solution on return */
  int Solve(VectorType& x, VectorType& rhs) {
    if (!ready_) return PGX_ERROR_FUNCTION_CALL;  // "Solve without setup." (fgmres.hpp:265-269)
    if (x.GetDataLocation() != rhs.GetDataLocation()) return PGX_ERROR_MEMORY_LOCATION;
    if (x.GetLengthLocal() != matrix_->GetNumRowsLocal() || rhs.GetLengthLocal() != matrix_->GetNumRowsLocal())
      return PGX_ERROR_INVALID_PARAM;
    const int rc = pgx_gemslr_solve(precond_->GetHandle(), x.GetData(), rhs.GetData(), x.GetDataLocation(),
                                    params_, &result_);
    return rc;
  }
  int GetNumberIterations() const { return result_.iters; }
  double GetFinalRelativeResidual() const { return result_.rel_res; }
  /* the whole outcome: status, FP64 true residual, device time, launches */
  const pgx_result& GetResult() const { return result_; }

 private:
  double params_[PGX_PARAMS_SIZE];
  MatrixType* matrix_ = nullptr;
  PrecondType* precond_ = nullptr;
  pgx_result result_;
  int location_ = kMemoryHost;
  bool ready_ = false;
};

typedef ParallelVectorClass<double> vector_par_double;
typedef ParallelCsrMatrixClass<double> matrix_csr_par_double;
typedef ParallelGemslrClass<matrix_csr_par_double, vector_par_double, double> precond_gemslr_csr_par_double;
typedef FlexGmresClass<matrix_csr_par_double, vector_par_double, double> fgmres_csr_par_double;

}  // namespace pgx

#endif /* PGX_PARGEMSLR_HPP */
