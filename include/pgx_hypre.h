/*
 * pgx_hypre.h — the reference's hypre plugin interface re-targeted at libpgx.
 *
 * The reference plugs GeMSLR into hypre as a preconditioner through
 * TESTS/hypre/pargemslr_hypre_interface.hpp:36-299: HYPRE_GEMSLRCreate /
 * Setup / Solve (TESTS/hypre/HYPRE_pargemslr.cpp) unpack a hypre ParCSR
 * matrix into diag/offd CSR arrays, hand them to
 * hypre_PargemslrParallelCsrMatrixDCreate, and call
 * hypre_PargemslrParallelGEMSLRD{Create,SetParams,Setup,Solve,Destroy}.
 * Each function below takes the arguments of the one it replaces, in the
 * same order and with the same meaning, so HYPRE_pargemslr.cpp switches by
 * renaming its calls; Solve applies the preconditioner once, x = M^-1 rhs,
 * on the GPU.
 *
 * Differences: one rank (the MPI_Comm argument is dropped and the matrix must
 * be the whole system, with an empty off-diagonal part); double precision
 * only (the S entry points are not provided; pgx_hypre_gemslr_set_precision
 * selects the FP32 preconditioner apply instead); and every call returns the
 * real status where the reference returns 0, with the message in
 * pgx_last_error().  The matrix is copied at create, its columns sorted
 * within each row (hypre stores the diagonal entry first).
 */
#ifndef PGX_HYPRE_H
#define PGX_HYPRE_H

#include "pgx.h"

#ifdef __cplusplus
extern "C" {
#endif

/* hypre_PargemslrInitGPU / hypre_PargemslrFinalizeGPU
 * (pargemslr_hypre_interface.hpp:51, 72): select and release the device. */
int pgx_hypre_init_gpu(int device);
int pgx_hypre_finalize_gpu(void);

/* hypre_PargemslrParallelCsrMatrixDCreate (pargemslr_hypre_interface.hpp:146-163).
 * data_location 0: the arrays are on the host; 1: on the device.  Returns
 * NULL on invalid input or on more than one rank's rows. */
void *pgx_hypre_csr_matrix_create(long int nrow_global, long int ncol_global, long int nrow_start,
                                  long int ncol_start, int nrow_local, int ncol_local, int *diag_i, int *diag_j,
                                  double *diag_data, int *offd_i, int *offd_j, double *offd_data, int n_offd_map,
                                  long int *offd_map, int data_location);
/* hypre_PargemslrParallelCsrMatrixDDestroy (…interface.hpp:91-92) */
int pgx_hypre_csr_matrix_destroy(void *matrix);
/* The stored matrix as a borrowed CSR view (valid until destroy). */
int pgx_hypre_csr_matrix_view(void *matrix, pgx_csr *A);

/* hypre_PargemslrParallelGEMSLRDCreate / Destroy / SetParams / Setup / Solve
 * (…interface.hpp:177-178, 195-196, 278-280, 224-228, 254-258).  Setup builds the
 * preconditioner for the matrix once (later calls return at once); x and rhs
 * are not read.  Solve computes x = M^-1 rhs with the matrix given at Setup;
 * x and rhs are on the host or the device as the matrix's data_location
 * says. */
void *pgx_hypre_gemslr_create(void);
int pgx_hypre_gemslr_destroy(void *gemslr);
int pgx_hypre_gemslr_set_params(void *gemslr, double *params);
int pgx_hypre_gemslr_set_precision(void *gemslr, int precision);
int pgx_hypre_gemslr_setup(void *gemslr, void *matrix, double *x, double *rhs);
int pgx_hypre_gemslr_solve(void *gemslr, void *matrix, double *x, double *rhs);
/* the C-ABI handle after Setup (NULL before), for the other pgx.h calls */
pgx_handle pgx_hypre_gemslr_handle(void *gemslr);

/* hypre_PargemslrCreateParameterArrayFromFile / DestroyParameterArray
 * (…interface.hpp:288-289, 297-298): the defaults overwritten by a hypre-format
 * parameter file (pgx_params_read_file, PGX_INPUTS_HYPRE).  As in the
 * reference the array comes back even when the file cannot be read or names
 * an unknown keyword, holding the defaults and the lines read before it
 * (pgx_last_error says what happened); NULL only when it cannot be allocated. */
double *pgx_hypre_params_from_file(const char *filename);
int pgx_hypre_params_destroy(double *params);

#ifdef __cplusplus
}
#endif

#endif /* PGX_HYPRE_H */
