"""The reference's parameter array, index for index.

ParGeMSLR drives every solver and preconditioner from one ``double
params[180]`` array whose slots are named ``PARGEMSLR_IO_*``
(ParGeMSLR SRC/utils/utils.hpp:77-297).  Drivers fill it with
``PargemslrSetDefaultParameterArray`` (SRC/utils/utils.cpp:30-126), then
overwrite slots from a positional text file (TESTS/sequential/io.cpp:336-725,
TESTS/parallel/io_par.cpp:359-819, TESTS/hypre/pargemslr_hypre_interface.cpp:391-820);
``read_inputs_file`` reads those files with the library's native reader.
The same array is accepted by this package's ``SetWithParameterArray`` and by
the C ABI, so a driver keeps its parameter handling unchanged.
"""
from __future__ import annotations

import math

import numpy as np

IO_SIZE = 180

PRECOND_GLOBAL_PRECOND = 0
PRECOND_LOCAL_REPCOND1 = 1
PRECOND_LOCAL_REPCOND1_LEVEL = 2
PRECOND_LOCAL_REPCOND2 = 3
PRECOND_LOCAL_REPCOND3 = 4
PRECOND_LOCAL_SMOOTHER1 = 5
SOLVER_OPTION = 10
SOLVER_KDIM = 11
SOLVER_MAXITS = 12
SOLVER_TOL = 13
SOLVER_ATOL = 14
PREPOSS_NLEV_GLOBAL = 20
PREPOSS_NLEV_LOCAL = 21
PREPOSS_NCOMP_GLOBAL = 22
PREPOSS_NCOMP_LOCAL = 23
PREPOSS_PARTITION_GLOBAL = 24
PREPOSS_PARTITION_LOCAL = 25
PREPOSS_MINSEP = 26
PREPOSS_KMIN_GLOBAL = 27
PREPOSS_KMIN_LOCAL = 28
PREPOSS_KFACTOR_GLOBAL = 29
PREPOSS_KFACTOR_LOCAL = 30
PREPOSS_VTXSEP_GLOBAL = 31
PREPOSS_VTXSEP_LOCAL = 32
PREPOSS_METIS_REFINE = 33
PREPOSS_GLOBAL_PARTITION = 34
ILU_DROPTOL_B_GLOBAL = 40
ILU_DROPTOL_B_LOCAL = 41
ILU_DROPTOL_EF_GLOBAL = 42
ILU_DROPTOL_EF_LOCAL = 43
ILU_DROPTOL_C_GLOBAL = 44
ILU_DROPTOL_C_LOCAL = 45
ILU_DROPTOL_S_GLOBAL = 46
ILU_DROPTOL_S_LOCAL = 47
ILU_ROWNNZ_B_GLOBAL = 48
ILU_ROWNNZ_B_LOCAL = 49
ILU_ROWNNZ_C_GLOBAL = 50
ILU_ROWNNZ_C_LOCAL = 51
ILU_LFIL_B_GLOBAL = 52
ILU_LFIL_B_LOCAL = 53
ILU_LFIL_C_GLOBAL = 54
ILU_LFIL_C_LOCAL = 55
ILU_ROWNNZ_S_GLOBAL = 56
ILU_ROWNNZ_S_LOCAL = 57
ILU_PERM_OPTION_GLOBAL = 58
ILU_PERM_OPTION_LOCAL = 59
ILU_OMP_OPTION_GLOBAL = 60
ILU_OMP_OPTION_LOCAL = 61
LR_ARNOLDI_OPTION1_GLOBAL = 70
LR_ARNOLDI_OPTION2_GLOBAL = 71
LR_ARNOLDI_OPTION1_LOCAL = 72
LR_ARNOLDI_OPTION2_LOCAL = 73
LR_RANK1_GLOBAL = 74
LR_RANK2_GLOBAL = 75
LR_RANK1_LOCAL = 76
LR_RANK2_LOCAL = 77
LR_RANK_FACTOR1_GLOBAL = 78
LR_RANK_FACTOR2_GLOBAL = 79
LR_RANK_FACTOR1_LOCAL = 80
LR_RANK_FACTOR2_LOCAL = 81
LR_ARNOLDI_FACTOR1_GLOBAL = 82
LR_ARNOLDI_FACTOR2_GLOBAL = 83
LR_ARNOLDI_FACTOR1_LOCAL = 84
LR_ARNOLDI_FACTOR2_LOCAL = 85
LR_TOL_EIG1_GLOBAL = 86
LR_TOL_EIG2_GLOBAL = 87
LR_TOL_EIG1_LOCAL = 88
LR_TOL_EIG2_LOCAL = 89
LR_MAXITS1_GLOBAL = 90
LR_MAXITS2_GLOBAL = 91
LR_MAXITS1_LOCAL = 92
LR_MAXITS2_LOCAL = 93
LR_TR_FACTOR = 94
LR_TOL_ORTH = 95
LR_TOL_REORTH = 96
LR_RAND_INIT_GUESS = 97
SCHUR_ENABLE = 130
SCHUR_ITER_TOL = 131
SCHUR_MAXITS = 132
ADVANCED_DIAG_SHIFT = 140
ADVANCED_GLOBAL_SOLVE = 141
ADVANCED_USE_COMPLEX_SHIFT = 142
ADVANCED_RESIDUAL_ITERS = 143
ADVANCED_GRAM_SCHMIDT = 144
GENERAL_PRINT_LEVEL = 150
POLY_ORDER = 160

# enum values used in the array (SRC/preconditioners/gemslr.hpp:30-60,
# SRC/preconditioners/ilu.hpp:90-100)
PARTITION_ND = 0
PARTITION_RKWAY = 1
REORDER_NO = 0
REORDER_RCM = 1
REORDER_AMD = 2
REORDER_MULTICOLOR = 6  # this library's greedy multicolor order inside subdomains (PGX_REORDER_MULTICOLOR)
LOWRANK_STD = 0
LOWRANK_TR = 1
LOWRANK_SUB = 2


def default_params() -> np.ndarray:
    """PargemslrSetDefaultParameterArray (SRC/utils/utils.cpp:30-126)."""
    p = np.zeros(IO_SIZE, dtype=np.float64)
    p[PRECOND_LOCAL_REPCOND1_LEVEL] = 1
    p[SOLVER_KDIM] = 50
    p[SOLVER_MAXITS] = 100
    p[SOLVER_TOL] = 1e-6
    p[PREPOSS_NLEV_GLOBAL] = 5
    p[PREPOSS_NLEV_LOCAL] = 5
    p[PREPOSS_NCOMP_GLOBAL] = 4
    p[PREPOSS_NCOMP_LOCAL] = 4
    p[PREPOSS_PARTITION_GLOBAL] = 1
    p[PREPOSS_PARTITION_LOCAL] = 0
    p[PREPOSS_MINSEP] = 10
    p[PREPOSS_KMIN_GLOBAL] = 1
    p[PREPOSS_KMIN_LOCAL] = 1
    p[PREPOSS_KFACTOR_GLOBAL] = 1
    p[PREPOSS_KFACTOR_LOCAL] = 1
    p[PREPOSS_VTXSEP_GLOBAL] = 1
    p[PREPOSS_VTXSEP_LOCAL] = 1
    p[ILU_DROPTOL_B_GLOBAL] = 1e-2
    p[ILU_DROPTOL_B_LOCAL] = 1e-2
    p[ILU_DROPTOL_EF_GLOBAL] = 1e-2
    p[ILU_DROPTOL_EF_LOCAL] = 1e-2
    p[ILU_DROPTOL_C_GLOBAL] = 1e-3
    p[ILU_DROPTOL_C_LOCAL] = 1e-3
    p[ILU_DROPTOL_S_GLOBAL] = 1e-3
    p[ILU_DROPTOL_S_LOCAL] = 1e-3
    p[ILU_ROWNNZ_B_GLOBAL] = 100
    p[ILU_ROWNNZ_B_LOCAL] = 100
    p[ILU_ROWNNZ_C_GLOBAL] = 200
    p[ILU_ROWNNZ_C_LOCAL] = 200
    p[ILU_ROWNNZ_S_GLOBAL] = 200
    p[ILU_ROWNNZ_S_LOCAL] = 200
    p[ILU_PERM_OPTION_GLOBAL] = 2
    p[ILU_PERM_OPTION_LOCAL] = 2
    p[LR_ARNOLDI_OPTION1_GLOBAL] = 1
    p[LR_ARNOLDI_OPTION2_GLOBAL] = 1
    p[LR_ARNOLDI_OPTION1_LOCAL] = 1
    p[LR_ARNOLDI_OPTION2_LOCAL] = 1
    p[LR_RANK1_GLOBAL] = 100
    p[LR_RANK1_LOCAL] = 100
    p[LR_RANK2_GLOBAL] = 50
    p[LR_RANK2_LOCAL] = 50
    for k in (LR_RANK_FACTOR1_GLOBAL, LR_RANK_FACTOR1_LOCAL, LR_RANK_FACTOR2_GLOBAL, LR_RANK_FACTOR2_LOCAL):
        p[k] = 1.0
    for k in (LR_ARNOLDI_FACTOR1_GLOBAL, LR_ARNOLDI_FACTOR1_LOCAL, LR_ARNOLDI_FACTOR2_GLOBAL,
              LR_ARNOLDI_FACTOR2_LOCAL):
        p[k] = 2.0
    for k in (LR_TOL_EIG1_GLOBAL, LR_TOL_EIG1_LOCAL, LR_TOL_EIG2_GLOBAL, LR_TOL_EIG2_LOCAL):
        p[k] = 1e-9
    for k in (LR_MAXITS1_GLOBAL, LR_MAXITS1_LOCAL, LR_MAXITS2_GLOBAL, LR_MAXITS2_LOCAL):
        p[k] = 3
    p[LR_TR_FACTOR] = 0.25
    p[LR_TOL_ORTH] = 1e-14
    p[LR_TOL_REORTH] = 1.0 / math.sqrt(2.0)
    p[LR_RAND_INIT_GUESS] = 1
    p[SCHUR_ENABLE] = 1
    p[SCHUR_ITER_TOL] = 1e-2
    p[SCHUR_MAXITS] = 5
    p[ADVANCED_RESIDUAL_ITERS] = 1
    p[GENERAL_PRINT_LEVEL] = 1
    p[POLY_ORDER] = 3
    return p


def sequential_inputs_params() -> np.ndarray:
    """Defaults overwritten by the reference's sequential parameter file.

    Mirrors what read_inputs_from_file (TESTS/sequential/io.cpp:336-560) does
    with TESTS/sequential/inputs:1-38, slot by slot (the LOCAL copies that the
    parser mirrors from the GLOBAL value are mirrored here too).
    """
    p = default_params()
    p[PRECOND_LOCAL_REPCOND1] = 0          # ILUT
    p[PRECOND_LOCAL_REPCOND1_LEVEL] = 1
    p[PRECOND_LOCAL_REPCOND2] = 0          # ILUT
    p[SOLVER_KDIM] = 50
    p[SOLVER_MAXITS] = 200
    p[SOLVER_TOL] = 1e-8
    p[SOLVER_ATOL] = 0
    p[PREPOSS_NLEV_GLOBAL] = 5
    p[PREPOSS_NLEV_LOCAL] = 2
    p[PREPOSS_NCOMP_GLOBAL] = 2
    p[PREPOSS_NCOMP_LOCAL] = 2
    p[PREPOSS_PARTITION_GLOBAL] = PARTITION_ND
    p[PREPOSS_PARTITION_LOCAL] = PARTITION_ND
    p[ILU_DROPTOL_B_GLOBAL] = p[ILU_DROPTOL_B_LOCAL] = 1e-3
    p[ILU_DROPTOL_C_GLOBAL] = p[ILU_DROPTOL_C_LOCAL] = 1e-3
    p[ILU_ROWNNZ_B_GLOBAL] = p[ILU_ROWNNZ_B_LOCAL] = 200
    p[ILU_ROWNNZ_C_GLOBAL] = p[ILU_ROWNNZ_C_LOCAL] = 200
    p[ILU_LFIL_B_GLOBAL] = 1
    p[ILU_LFIL_B_LOCAL] = p[ILU_ROWNNZ_B_GLOBAL]
    p[ILU_LFIL_C_GLOBAL] = 1
    p[ILU_LFIL_C_LOCAL] = p[ILU_ROWNNZ_C_GLOBAL]
    p[ILU_PERM_OPTION_GLOBAL] = p[ILU_PERM_OPTION_LOCAL] = REORDER_RCM
    p[LR_ARNOLDI_OPTION1_GLOBAL] = p[LR_ARNOLDI_OPTION1_LOCAL] = LOWRANK_TR
    p[LR_ARNOLDI_OPTION2_GLOBAL] = p[LR_ARNOLDI_OPTION2_LOCAL] = LOWRANK_TR
    p[LR_RANK1_GLOBAL] = p[LR_RANK1_LOCAL] = 32
    p[LR_RANK2_GLOBAL] = p[LR_RANK2_LOCAL] = 32
    p[LR_TOL_EIG1_GLOBAL] = p[LR_TOL_EIG1_LOCAL] = 1e-3
    p[LR_TOL_EIG2_GLOBAL] = p[LR_TOL_EIG2_LOCAL] = 1e-3
    p[LR_RANK_FACTOR1_GLOBAL] = p[LR_RANK_FACTOR1_LOCAL] = 1.0
    p[LR_RANK_FACTOR2_GLOBAL] = p[LR_RANK_FACTOR2_LOCAL] = 1.0
    p[LR_ARNOLDI_FACTOR1_GLOBAL] = p[LR_ARNOLDI_FACTOR1_LOCAL] = 2.0
    p[LR_ARNOLDI_FACTOR2_GLOBAL] = p[LR_ARNOLDI_FACTOR2_LOCAL] = 2.0
    p[LR_MAXITS1_GLOBAL] = p[LR_MAXITS1_LOCAL] = 10
    p[LR_MAXITS2_GLOBAL] = p[LR_MAXITS2_LOCAL] = 10
    p[SCHUR_ENABLE] = 1
    p[SCHUR_ITER_TOL] = 1e-2
    p[SCHUR_MAXITS] = 5
    p[ADVANCED_USE_COMPLEX_SHIFT] = 0
    p[ADVANCED_GLOBAL_SOLVE] = 0           # LU
    p[GENERAL_PRINT_LEVEL] = 1
    return p


def read_inputs_file(path: str, fmt: str = "sequential", base: np.ndarray | None = None) -> np.ndarray:
    """A driver parameter file read onto ``base`` (default: the defaults), as the reference driver of
    that format reads it; fmt is "sequential", "parallel" or "hypre" (pgx_params_read_file)."""
    from pargemslr_b200 import _abi
    return _abi.params_read_file(path, fmt, base)


def workload_params(name: str) -> np.ndarray:
    """Full parameter arrays for the named benchmark workloads.

    Every slot not named by the workload keeps the value of the reference's
    sequential parameter file; the inner Schur-complement FGMRES stays on with
    the file's settings (tol 1e-2, 5 iterations).
    """
    p = sequential_inputs_params()
    if name == "lap2d_256":
        # 2D 5-point Laplacian 256x256: 3 levels, ILUT 1e-2 / 20 per row, rank 8
        p[PREPOSS_NLEV_GLOBAL] = 3
        p[ILU_DROPTOL_B_GLOBAL] = p[ILU_DROPTOL_B_LOCAL] = 1e-2
        p[ILU_DROPTOL_C_GLOBAL] = p[ILU_DROPTOL_C_LOCAL] = 1e-2
        p[ILU_ROWNNZ_B_GLOBAL] = p[ILU_ROWNNZ_B_LOCAL] = 20
        p[ILU_ROWNNZ_C_GLOBAL] = p[ILU_ROWNNZ_C_LOCAL] = 20
        p[LR_RANK1_GLOBAL] = p[LR_RANK1_LOCAL] = 8
        p[LR_RANK2_GLOBAL] = p[LR_RANK2_LOCAL] = 8
    elif name == "lap3d_128":
        # 3D 7-point Laplacian 128^3: 4 levels, ILUT 1e-3, rank 16
        p[PREPOSS_NLEV_GLOBAL] = 4
        p[ILU_DROPTOL_B_GLOBAL] = p[ILU_DROPTOL_B_LOCAL] = 1e-3
        p[ILU_DROPTOL_C_GLOBAL] = p[ILU_DROPTOL_C_LOCAL] = 1e-3
        p[LR_RANK1_GLOBAL] = p[LR_RANK1_LOCAL] = 16
        p[LR_RANK2_GLOBAL] = p[LR_RANK2_LOCAL] = 16
    elif name == "serve":
        # random nonsymmetric sparse systems of the serving workload: 2 levels,
        # ILUT 1e-2 / 20 per row, rank 8, no inner Schur iteration, FGMRES(40)
        p[PREPOSS_NLEV_GLOBAL] = 2
        p[ILU_DROPTOL_B_GLOBAL] = p[ILU_DROPTOL_B_LOCAL] = 1e-2
        p[ILU_DROPTOL_C_GLOBAL] = p[ILU_DROPTOL_C_LOCAL] = 1e-2
        p[ILU_ROWNNZ_B_GLOBAL] = p[ILU_ROWNNZ_B_LOCAL] = 20
        p[ILU_ROWNNZ_C_GLOBAL] = p[ILU_ROWNNZ_C_LOCAL] = 20
        p[LR_RANK1_GLOBAL] = p[LR_RANK1_LOCAL] = 8
        p[LR_RANK2_GLOBAL] = p[LR_RANK2_LOCAL] = 8
        p[SCHUR_ENABLE] = 0
    elif name == "convdiff":
        # batched uneven upwind convection-diffusion systems: 2 levels, ILUT
        # 1e-2 / 20 per row, rank 8, inner Schur FGMRES on, FGMRES(30)
        p[PREPOSS_NLEV_GLOBAL] = 2
        p[ILU_DROPTOL_B_GLOBAL] = p[ILU_DROPTOL_B_LOCAL] = 1e-2
        p[ILU_DROPTOL_C_GLOBAL] = p[ILU_DROPTOL_C_LOCAL] = 1e-2
        p[ILU_ROWNNZ_B_GLOBAL] = p[ILU_ROWNNZ_B_LOCAL] = 20
        p[ILU_ROWNNZ_C_GLOBAL] = p[ILU_ROWNNZ_C_LOCAL] = 20
        p[LR_RANK1_GLOBAL] = p[LR_RANK1_LOCAL] = 8
        p[LR_RANK2_GLOBAL] = p[LR_RANK2_LOCAL] = 8
    elif name == "zlap3d_96":
        # complex shifted 3D Laplacian 96^3 (shift 0.05 + 0.01i): 5 levels,
        # ILUT 1e-3, rank 32, FGMRES(100)
        p[PREPOSS_NLEV_GLOBAL] = 5
        p[ILU_DROPTOL_B_GLOBAL] = p[ILU_DROPTOL_B_LOCAL] = 1e-3
        p[ILU_DROPTOL_C_GLOBAL] = p[ILU_DROPTOL_C_LOCAL] = 1e-3
        p[LR_RANK1_GLOBAL] = p[LR_RANK1_LOCAL] = 32
        p[LR_RANK2_GLOBAL] = p[LR_RANK2_LOCAL] = 32
    elif name == "zsmall":
        # complex test problems: the 5 levels and ILUT of zlap3d_96 with rank 8
        p[PREPOSS_NLEV_GLOBAL] = 5
        p[ILU_DROPTOL_B_GLOBAL] = p[ILU_DROPTOL_B_LOCAL] = 1e-3
        p[ILU_DROPTOL_C_GLOBAL] = p[ILU_DROPTOL_C_LOCAL] = 1e-3
        p[LR_RANK1_GLOBAL] = p[LR_RANK1_LOCAL] = 8
        p[LR_RANK2_GLOBAL] = p[LR_RANK2_LOCAL] = 8
    elif name == "small":
        # small problems for kernel-level checks
        p[PREPOSS_NLEV_GLOBAL] = 3
        p[ILU_DROPTOL_B_GLOBAL] = p[ILU_DROPTOL_B_LOCAL] = 1e-2
        p[ILU_DROPTOL_C_GLOBAL] = p[ILU_DROPTOL_C_LOCAL] = 1e-2
        p[ILU_ROWNNZ_B_GLOBAL] = p[ILU_ROWNNZ_B_LOCAL] = 20
        p[ILU_ROWNNZ_C_GLOBAL] = p[ILU_ROWNNZ_C_LOCAL] = 20
        p[LR_RANK1_GLOBAL] = p[LR_RANK1_LOCAL] = 4
        p[LR_RANK2_GLOBAL] = p[LR_RANK2_LOCAL] = 4
    else:
        raise ValueError(f"unknown workload {name!r}")
    p[SOLVER_KDIM] = {"serve": 40, "convdiff": 30, "zlap3d_96": 100, "zsmall": 100}.get(name, 50)
    p[SOLVER_TOL] = 1e-8
    return p
