// A driver for the C++ front end (include/pgx_pargemslr.hpp), written the
// way the reference's parallel Laplacian driver writes its solve
// (TESTS/parallel/driver_laplacian_gemslr_par.cpp:379-425), with the pgx
// classes in place of pargemslr's.
//
//   frontend_driver NX NY NZ PARAMS_FILE FORMAT PRECISION OUT_DIR
//
// PARAMS_FILE is read with pgx_params_read_file in FORMAT (0 sequential,
// 1 parallel, 2 hypre) onto the defaults, or "-" for the defaults alone;
// PRECISION is 0 (FP64) or 1 (mixed).  b = A x_true with x_true from
// OUT_DIR/xtrue.bin (raw float64) when present, else all ones; x0 = 0.
// Writes the parameter array (params.bin), A (A_rp/A_cj/A_va.bin), b.bin and,
// after a solve, x.bin and z.bin (one preconditioner application) to OUT_DIR
// and prints key=value lines.  Without a CUDA device it checks the calls
// that need none and stops before Setup with "device=none".
#include <cstdio>
#include <string>
#include <vector>

#include "pgx_pargemslr.hpp"

using namespace pgx;

typedef ParallelCsrMatrixClass<double> Matrix;
typedef ParallelVectorClass<double> Vector;

static bool write_raw(const std::string& path, const void* p, size_t bytes) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = fwrite(p, 1, bytes, f) == bytes;
  fclose(f);
  return ok;
}

int main(int argc, char** argv) {
  if (argc != 8) {
    fprintf(stderr, "usage: %s NX NY NZ PARAMS_FILE FORMAT PRECISION OUT_DIR\n", argv[0]);
    return 2;
  }
  const int nx = atoi(argv[1]), ny = atoi(argv[2]), nz = atoi(argv[3]);
  const std::string params_file = argv[4], out = argv[7];
  const int format = atoi(argv[5]), precision = atoi(argv[6]);

  /* 1. parameters */
  double params[PGX_PARAMS_SIZE];
  pgx_params_default(params);
  if (params_file != "-") {
    const int rc = pgx_params_read_file(params_file.c_str(), format, params);
    printf("params=%d\n", rc);
    if (rc) {
      printf("error=%s\n", pgx_last_error());
      return 1;
    }
  }

  write_raw(out + "/params.bin", params, sizeof(params));

  /* 2. matrix, right-hand side, initial guess */
  Matrix* parcsr_mat = new Matrix();
  printf("laplacian=%d\n", parcsr_mat->Laplacian(nx, ny, nz, 0.0, 0.0, 0.0, 0.0));
  const int n = parcsr_mat->GetNumRowsLocal();
  const long int nnz = parcsr_mat->GetNumNonzeros();
  printf("n=%d nnzA=%ld\n", n, nnz);
  write_raw(out + "/A_rp.bin", parcsr_mat->GetI(), sizeof(int) * (n + 1));
  write_raw(out + "/A_cj.bin", parcsr_mat->GetJ(), sizeof(int) * nnz);
  write_raw(out + "/A_va.bin", parcsr_mat->GetData(), sizeof(double) * nnz);
  Vector x, b, xt;
  x.Setup(n);
  b.Setup(n);
  xt.Setup(n);
  xt.Fill(1.0);
  if (FILE* f = fopen((out + "/xtrue.bin").c_str(), "rb")) {
    const size_t got = fread(xt.GetData(), sizeof(double), n, f);
    fclose(f);
    if (got != (size_t)n) return 3;
  }
  b.Fill(0.0);
  printf("matvec=%d\n", parcsr_mat->MatVec('N', 1.0, xt, 0.0, b));
  write_raw(out + "/b.bin", b.GetData(), sizeof(double) * n);
  x.Fill(0.0);

  /* 3. solver and preconditioner, as the reference driver sets them */
  FlexGmresClass<Matrix, Vector, double>* solverp = new FlexGmresClass<Matrix, Vector, double>();
  ParallelGemslrClass<Matrix, Vector, double>* precondp = new ParallelGemslrClass<Matrix, Vector, double>();
  solverp->SetMatrixP(parcsr_mat);
  solverp->SetWithParameterArray(params);
  solverp->SetSolveLocation(kMemoryHost);
  precondp->SetMatrixP(parcsr_mat);
  precondp->SetWithParameterArray(params);
  precondp->SetSolveLocation(kMemoryHost);
  printf("precision=%d\n", precondp->SetPrecision(precision));
  solverp->SetPreconditionerP(precondp);

  /* calls that need no device: their status codes */
  printf("solve_before_setup=%d\n", solverp->Solve(x, b));
  printf("apply_before_setup=%d\n", precondp->Solve(x, b));
  printf("nnz_before_setup=%ld\n", precondp->GetNumNonzeros());
  printf("matvec_trans=%d\n", parcsr_mat->MatVec('T', 1.0, xt, 0.0, b));
  printf("mm_zero_based=%d\n", Matrix().ReadFromMMFile("unused.mtx", 0));

  if (pgx_init(0) != PGX_SUCCESS) {
    printf("device=none error=%s\n", pgx_last_error());
    delete solverp;
    delete precondp;
    delete parcsr_mat;
    return 0;
  }

  /* 4. setup and solve */
  int rc = solverp->Setup(x, b);
  printf("setup=%d\n", rc);
  if (rc) {
    printf("error=%s\n", pgx_last_error());
    return 1;
  }
  rc = solverp->Solve(x, b);
  printf("solve=%d\n", rc);
  if (rc) printf("error=%s\n", pgx_last_error());
  const pgx_result& r = solverp->GetResult();
  printf("iters=%d rel_res=%.17g true_rel_res=%.17g\n", solverp->GetNumberIterations(),
         solverp->GetFinalRelativeResidual(), r.true_rel_res);
  long int nnz_b = 0, nnz_lr = 0;
  const long int nnz_m = precondp->GetNumNonzeros(nnz_b, nnz_lr);
  printf("nnz_bsolver=%ld nnz_lr=%ld nnz_total=%ld\n", nnz_b, nnz_lr, nnz_m);
  write_raw(out + "/x.bin", x.GetData(), sizeof(double) * n);

  /* one preconditioner application z = M^-1 b through the preconditioner's Solve */
  Vector z;
  z.Setup(n);
  printf("apply=%d\n", precondp->Solve(z, b));
  write_raw(out + "/z.bin", z.GetData(), sizeof(double) * n);

  delete solverp;
  delete precondp;
  delete parcsr_mat;
  return rc ? 1 : 0;
}
