// The double[180] parameter array of SetWithParameterArray: its defaults and
// the three plain-text parameter files the reference's drivers read.
//
//   defaults    PargemslrSetDefaultParameterArray   SRC/utils/utils.cpp:30-126
//   sequential  read_inputs_from_file  TESTS/sequential/io.cpp:336-725      (38 lines)
//   parallel    read_inputs_from_file  TESTS/parallel/io_par.cpp:359-819    (35 lines)
//   hypre       read_inputs_from_file  TESTS/hypre/pargemslr_hypre_interface.cpp:391-820 (31 lines)
//   arguments   read_inputs            TESTS/sequential/io.cpp:729-748
//
// A file is read line by line; line k has a fixed meaning in each format.  A
// numeric line fills its slots with the numbers found at its start, left to
// right, stopping at the first token that is not a number (slots without a
// number keep their value), then copies GLOBAL values into their LOCAL twins.
// A keyword line matches its first word, upper-cased, against the format's
// list for that line; an unknown keyword stops the read with the I/O error,
// the lines before it already applied.  Lines past the last one known to the
// format are ignored.  Lines are read in 1023-byte pieces as the reference's
// fgets buffer does, so a longer line counts as several.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "pgx_params.h"

namespace pgx {
namespace params {
namespace {

// slot indices (SRC/utils/utils.hpp:77-297)
enum : int {
  GLOBAL_PRECOND = 0, REPCOND1 = 1, REPCOND1_LEVEL = 2, REPCOND2 = 3, REPCOND3 = 4, SMOOTHER1 = 5,
  SOLVER_OPTION = 10, KDIM = 11, MAXITS = 12, TOL = 13, ATOL = 14,
  NLEV_G = 20, NLEV_L = 21, NCOMP_G = 22, NCOMP_L = 23, PART_G = 24, PART_L = 25, MINSEP = 26,
  KMIN_G = 27, KMIN_L = 28, KFACTOR_G = 29, KFACTOR_L = 30, VTXSEP_G = 31, VTXSEP_L = 32, METIS_REFINE = 33,
  GLOBAL_PARTITION = 34,
  DROP_B_G = 40, DROP_B_L = 41, DROP_EF_G = 42, DROP_EF_L = 43, DROP_C_G = 44, DROP_C_L = 45, DROP_S_G = 46,
  DROP_S_L = 47, NNZ_B_G = 48, NNZ_B_L = 49, NNZ_C_G = 50, NNZ_C_L = 51, LFIL_B_G = 52, LFIL_B_L = 53,
  LFIL_C_G = 54, LFIL_C_L = 55, NNZ_S_G = 56, NNZ_S_L = 57, PERM_G = 58, PERM_L = 59, OMP_G = 60, OMP_L = 61,
  ARN1_G = 70, ARN2_G = 71, ARN1_L = 72, ARN2_L = 73, RANK1_G = 74, RANK2_G = 75, RANK1_L = 76, RANK2_L = 77,
  RF1_G = 78, RF2_G = 79, RF1_L = 80, RF2_L = 81, AF1_G = 82, AF2_G = 83, AF1_L = 84, AF2_L = 85,
  EIG1_G = 86, EIG2_G = 87, EIG1_L = 88, EIG2_L = 89, LRIT1_G = 90, LRIT2_G = 91, LRIT1_L = 92, LRIT2_L = 93,
  TR_FACTOR = 94, TOL_ORTH = 95, TOL_REORTH = 96, RAND_INIT = 97, ARN_A = 99, RANK_A = 100, RF_A = 101,
  AF_A = 102, EIG_A = 103, LRIT_A = 104,
  SCHUR_ENABLE = 130, SCHUR_TOL = 131, SCHUR_MAXITS = 132,
  DIAG_SHIFT = 140, GLOBAL_SOLVE = 141, COMPLEX_SHIFT = 142, RESIDUAL_ITERS = 143, GRAM_SCHMIDT = 144,
  PRINT_LEVEL = 150, POLY_ORDER = 160,
  NPROC_X = 170, NPROC_Y = 171, NPROC_Z = 172, NDOM_X = 173, NDOM_Y = 174, NDOM_Z = 175,
  DROP = -1,  // a number that is read and thrown away
};

struct Keyword {
  const char* word;
  double value;
};
using Keywords = std::vector<Keyword>;

// enum values (SRC/preconditioners/gemslr.hpp:30-140, ilu.hpp:92-100)
const Keywords kBSolve = {{"ILUT", 0}, {"ILUK", 1}, {"GEMSLR", 2}};
const Keywords kCSolve4 = {{"ILUT", 0}, {"ILUK", 1}, {"BJILUT", 2}, {"BJILUK", 3}};
const Keywords kCSolve6 = {{"ILUT", 0}, {"ILUK", 1}, {"BJILUT", 2}, {"BJILUK", 3}, {"BJILUT2", 4}, {"BJILUK2", 5}};
const Keywords kGlobalPrecond = {{"BJ", 0}, {"ESCHUR", 1}, {"GEMSLR", 2}, {"PSLR", 3}};
const Keywords kPartition = {{"ND", 0}, {"RKWAY", 1}};
const Keywords kReordering = {{"NO", 0}, {"RCM", 1}, {"AMD", 2}, {"ND", 3}};
const Keywords kLowRank = {{"STD", 0}, {"TR", 1}, {"SUB", 2}};
const Keywords kSolve3 = {{"LU", 0}, {"U", 1}, {"MUL", 2}};
const Keywords kSolve2 = {{"LU", 0}, {"U", 1}};
const Keywords kSmoother = {{"MILU", 0}, {"ILU", 1}};

struct Line {
  std::vector<int> slots;                   // numbers, or the slots a keyword's value goes to
  std::vector<std::pair<int, int>> copies;  // then p[first] = p[second]
  const Keywords* keywords = nullptr;       // keyword line when set
};

Line num(std::vector<int> slots, std::vector<std::pair<int, int>> copies = {}) {
  Line l;
  l.slots = std::move(slots);
  l.copies = std::move(copies);
  return l;
}

Line kw(const Keywords& k, std::vector<int> slots) {
  Line l;
  l.slots = std::move(slots);
  l.keywords = &k;
  return l;
}

const std::vector<Line>& sequential_lines() {
  static const std::vector<Line> t = {
      kw(kBSolve, {REPCOND1}),                     // 1
      num({REPCOND1_LEVEL}),                       // 2
      kw(kBSolve, {REPCOND2}),                     // 3
      num({KDIM}),                                 // 4
      num({MAXITS}),                               // 5
      num({TOL}),                                  // 6
      num({ATOL}),                                 // 7
      num({NLEV_G}),                               // 8
      num({NLEV_L}),                               // 9
      num({NCOMP_G}),                              // 10
      num({NCOMP_L}),                              // 11
      kw(kPartition, {PART_G}),                    // 12
      kw(kPartition, {PART_L}),                    // 13
      num({DROP_B_G}, {{DROP_B_L, DROP_B_G}}),     // 14
      num({DROP_C_G}, {{DROP_C_L, DROP_C_G}}),     // 15
      num({NNZ_B_G}, {{NNZ_B_L, NNZ_B_G}}),        // 16
      num({NNZ_C_G}, {{NNZ_C_L, NNZ_C_G}}),        // 17
      // the LOCAL level of fill takes the GLOBAL row cap, as in io.cpp:512-523
      num({LFIL_B_G}, {{LFIL_B_L, NNZ_B_G}}),      // 18
      num({LFIL_C_G}, {{LFIL_C_L, NNZ_C_G}}),      // 19
      kw(kReordering, {PERM_G, PERM_L}),           // 20
      kw(kLowRank, {ARN1_G, ARN1_L}),              // 21
      kw(kLowRank, {ARN2_G, ARN2_L}),              // 22
      num({RANK1_G}, {{RANK1_L, RANK1_G}}),        // 23
      num({RANK2_G}, {{RANK2_L, RANK2_G}}),        // 24
      num({EIG1_G}, {{EIG1_L, EIG1_G}}),           // 25
      num({EIG2_G}, {{EIG2_L, EIG2_G}}),           // 26
      num({RF1_G}, {{RF1_L, RF1_G}}),              // 27
      num({RF2_G}, {{RF2_L, RF2_G}}),              // 28
      num({AF1_G}, {{AF1_L, AF1_G}}),              // 29
      num({AF2_G}, {{AF2_L, AF2_G}}),              // 30
      num({LRIT1_G}, {{LRIT1_L, LRIT1_G}}),        // 31
      num({LRIT2_G}, {{LRIT2_L, LRIT2_G}}),        // 32
      num({SCHUR_ENABLE}),                         // 33
      num({SCHUR_TOL}),                            // 34
      num({SCHUR_MAXITS}),                         // 35
      num({COMPLEX_SHIFT}),                        // 36
      kw(kSolve3, {GLOBAL_SOLVE}),                 // 37
      num({PRINT_LEVEL}),                          // 38
  };
  return t;
}

// lines 16-18 of the parallel file and 12-14 of the hypre file
const std::vector<std::pair<int, int>> kDropCopies = {
    {DROP_B_L, DROP_B_G}, {DROP_EF_L, DROP_EF_G}, {DROP_S_L, DROP_S_G}, {DROP_C_L, DROP_C_G}};
const std::vector<std::pair<int, int>> kNnzCopies = {{NNZ_B_L, NNZ_B_G}, {NNZ_S_L, NNZ_S_G}, {NNZ_C_L, NNZ_C_G}};
const std::vector<std::pair<int, int>> kLfilCopies = {{LFIL_B_L, LFIL_B_G}, {LFIL_C_L, LFIL_C_G}};

const std::vector<Line>& parallel_lines() {
  static const std::vector<Line> t = {
      kw(kGlobalPrecond, {GLOBAL_PRECOND}),                                      // 1
      num({GLOBAL_PARTITION}),                                                   // 2
      kw(kBSolve, {REPCOND1}),                                                   // 3
      num({REPCOND1_LEVEL}),                                                     // 4
      kw(kBSolve, {REPCOND2}),                                                   // 5
      kw(kCSolve6, {REPCOND3}),                                                  // 6
      num({POLY_ORDER}),                                                         // 7
      num({KDIM}),                                                               // 8
      num({MAXITS}),                                                             // 9
      num({TOL}),                                                                // 10
      num({ATOL}),                                                               // 11
      num({NLEV_G, NLEV_L}),                                                     // 12
      num({NCOMP_G, NCOMP_L}),                                                   // 13
      kw(kPartition, {PART_G}),                                                  // 14
      kw(kPartition, {PART_L}),                                                  // 15
      num({DROP_B_G, DROP_EF_G, DROP_S_G, DROP_C_G}, kDropCopies),               // 16
      num({NNZ_B_G, NNZ_S_G, NNZ_C_G}, kNnzCopies),                              // 17
      num({LFIL_B_G, DROP, LFIL_C_G}, kLfilCopies),                              // 18
      kw(kReordering, {PERM_G, PERM_L}),                                         // 19
      kw(kLowRank, {ARN1_G, ARN1_L}),                                            // 20
      kw(kLowRank, {ARN2_G, ARN2_L}),                                            // 21
      kw(kLowRank, {ARN_A}),                                                     // 22
      num({RANK1_G, RANK2_G, RANK_A}, {{RANK1_L, RANK1_G}, {RANK2_L, RANK2_G}}),  // 23
      num({EIG1_G, EIG2_G, EIG_A}, {{EIG1_L, EIG1_G}, {EIG2_L, EIG2_G}}),        // 24
      num({RF1_G, RF2_G, RF_A}, {{RF1_L, RF1_G}, {RF2_L, RF2_G}}),               // 25
      num({AF1_G, AF2_G, AF_A}, {{AF1_L, AF1_G}, {AF2_L, AF2_G}}),               // 26
      num({LRIT1_G, LRIT2_G, LRIT_A}, {{LRIT1_L, LRIT1_G}, {LRIT2_L, LRIT2_G}}), // 27
      num({SCHUR_ENABLE}),                                                       // 28
      num({SCHUR_TOL}),                                                          // 29
      num({SCHUR_MAXITS}),                                                       // 30
      num({COMPLEX_SHIFT}),                                                      // 31
      kw(kSolve3, {GLOBAL_SOLVE}),                                               // 32
      num({NPROC_X, NPROC_Y, NPROC_Z}),                                          // 33
      num({NDOM_X, NDOM_Y, NDOM_Z}),                                             // 34
      num({PRINT_LEVEL}),                                                        // 35
  };
  return t;
}

const std::vector<Line>& hypre_lines() {
  static const std::vector<Line> t = {
      kw(kGlobalPrecond, {GLOBAL_PRECOND}),                         // 1
      num({GLOBAL_PARTITION}),                                      // 2
      kw(kBSolve, {REPCOND1}),                                      // 3
      num({REPCOND1_LEVEL}),                                        // 4
      kw(kBSolve, {REPCOND2}),                                      // 5
      kw(kCSolve4, {REPCOND3}),                                     // 6
      num({POLY_ORDER}),                                            // 7
      num({NLEV_G, NLEV_L}),                                        // 8
      num({NCOMP_G, NCOMP_L}),                                      // 9
      kw(kPartition, {PART_G}),                                     // 10
      kw(kPartition, {PART_L}),                                     // 11
      num({DROP_B_G, DROP_EF_G, DROP_S_G, DROP_C_G}, kDropCopies),  // 12
      num({NNZ_B_G, NNZ_S_G, NNZ_C_G}, kNnzCopies),                 // 13
      num({LFIL_B_G, DROP, LFIL_C_G}, kLfilCopies),                 // 14
      kw(kReordering, {PERM_G, PERM_L}),                            // 15
      kw(kLowRank, {ARN1_G, ARN1_L}),                               // 16
      kw(kLowRank, {ARN2_G, ARN2_L}),                               // 17
      num({RANK1_G, RANK2_G}, {{RANK1_L, RANK1_G}, {RANK2_L, RANK2_G}}),  // 18
      num({EIG1_G, EIG2_G}, {{EIG1_L, EIG1_G}, {EIG2_L, EIG2_G}}),        // 19
      num({RF1_G, RF2_G}, {{RF1_L, RF1_G}, {RF2_L, RF2_G}}),              // 20
      num({AF1_G, AF2_G}, {{AF1_L, AF1_G}, {AF2_L, AF2_G}}),              // 21
      num({LRIT1_G, LRIT2_G}, {{LRIT1_L, LRIT1_G}, {LRIT2_L, LRIT2_G}}),  // 22
      num({SCHUR_ENABLE}),                                          // 23
      num({SCHUR_TOL}),                                             // 24
      num({SCHUR_MAXITS}),                                          // 25
      num({COMPLEX_SHIFT}),                                         // 26
      kw(kSolve2, {GLOBAL_SOLVE}),                                  // 27
      num({RESIDUAL_ITERS}),                                        // 28
      num({GRAM_SCHMIDT}),                                          // 29
      kw(kSmoother, {SMOOTHER1}),                                   // 30
      num({PRINT_LEVEL}),                                           // 31
  };
  return t;
}

// The first whitespace-delimited word of a line, upper-cased.
std::string first_word(const char* s) {
  while (*s && isspace((unsigned char)*s)) s++;
  std::string w;
  while (*s && !isspace((unsigned char)*s)) w.push_back((char)toupper((unsigned char)*s++));
  return w;
}

// Applies one line; false for an unknown keyword.
bool apply(const Line& l, const char* text, double* p) {
  if (l.keywords) {
    const std::string w = first_word(text);
    for (const Keyword& k : *l.keywords) {
      if (w == k.word) {
        for (int s : l.slots) p[s] = k.value;
        return true;
      }
    }
    return false;
  }
  const char* at = text;
  for (int s : l.slots) {
    char* end = nullptr;
    const double v = strtod(at, &end);
    if (end == at) break;
    if (s != DROP) p[s] = v;
    // The reference reads numbers with sscanf("%lf"); glibc's scanf also
    // consumes an exponent marker (and its sign) that no digit follows, when
    // the number has no exponent yet, so "1e 2" gives 1 then 2 where strtod
    // would stop at the 'e' ("1e5e 2" stops at the second 'e' in both).
    bool plain = isdigit((unsigned char)end[-1]) || end[-1] == '.';
    for (const char* c = at; c < end && plain; c++) plain = !strchr("xXeE", *c);
    if (plain && (*end == 'e' || *end == 'E')) {
      end++;
      if (*end == '+' || *end == '-') end++;
    }
    at = end;
  }
  for (const auto& c : l.copies) p[c.first] = p[c.second];
  return true;
}

}  // namespace

void set_defaults(double* p) {
  for (int i = 0; i < kSize; i++) p[i] = 0.0;
  p[REPCOND1_LEVEL] = 1;
  p[KDIM] = 50;
  p[MAXITS] = 100;
  p[TOL] = 1e-6;
  p[NLEV_G] = p[NLEV_L] = 5;
  p[NCOMP_G] = p[NCOMP_L] = 4;
  p[PART_G] = 1;
  p[MINSEP] = 10;
  p[KMIN_G] = p[KMIN_L] = 1;
  p[KFACTOR_G] = p[KFACTOR_L] = 1;
  p[VTXSEP_G] = p[VTXSEP_L] = 1;
  p[DROP_B_G] = p[DROP_B_L] = 1e-2;
  p[DROP_EF_G] = p[DROP_EF_L] = 1e-2;
  p[DROP_C_G] = p[DROP_C_L] = 1e-3;
  p[DROP_S_G] = p[DROP_S_L] = 1e-3;
  p[NNZ_B_G] = p[NNZ_B_L] = 100;
  p[NNZ_C_G] = p[NNZ_C_L] = 200;
  p[NNZ_S_G] = p[NNZ_S_L] = 200;
  p[PERM_G] = p[PERM_L] = 2;
  p[ARN1_G] = p[ARN2_G] = p[ARN1_L] = p[ARN2_L] = 1;
  p[RANK1_G] = p[RANK1_L] = 100;
  p[RANK2_G] = p[RANK2_L] = 50;
  p[RF1_G] = p[RF1_L] = p[RF2_G] = p[RF2_L] = 1.0;
  p[AF1_G] = p[AF1_L] = p[AF2_G] = p[AF2_L] = 2.0;
  p[EIG1_G] = p[EIG1_L] = p[EIG2_G] = p[EIG2_L] = 1e-9;
  p[LRIT1_G] = p[LRIT1_L] = p[LRIT2_G] = p[LRIT2_L] = 3;
  p[TR_FACTOR] = 0.25;
  p[TOL_ORTH] = 1e-14;
  p[TOL_REORTH] = 1.0 / std::sqrt(2.0);
  p[RAND_INIT] = 1;
  p[SCHUR_ENABLE] = 1;
  p[SCHUR_TOL] = 1e-2;
  p[SCHUR_MAXITS] = 5;
  p[RESIDUAL_ITERS] = 1;
  p[PRINT_LEVEL] = 1;
  p[POLY_ORDER] = 3;
}

// The command-line overrides of the drivers' read_inputs
// (TESTS/sequential/io.cpp:729-748, TESTS/parallel/io_par.cpp:822-843): "-tol
// V", "-kdim N", "-maxits N".  A flag counts when its next argument exists
// and does not start with '-'; the first such occurrence wins.  Values are
// read as atof / atoi read them (PargemslrReadInputArg, SRC/utils/utils.cpp:389-416).
void read_args(int argc, const char* const* argv, double* p) {
  struct Flag {
    const char* name;
    int slot;
    bool integer;
  };
  static const Flag flags[] = {{"tol", TOL, false}, {"kdim", KDIM, true}, {"maxits", MAXITS, true}};
  for (const Flag& f : flags) {
    for (int i = 0; i < argc; i++) {
      if (!argv[i] || argv[i][0] != '-' || strcmp(argv[i] + 1, f.name) != 0) continue;
      if (i + 1 >= argc || !argv[i + 1] || argv[i + 1][0] == '-') continue;
      p[f.slot] = f.integer ? (double)atoi(argv[i + 1]) : atof(argv[i + 1]);
      break;
    }
  }
}

int read_file(const char* path, int format, double* p, std::string& err) {
  const std::vector<Line>* lines = nullptr;
  switch (format) {
    case kSequential: lines = &sequential_lines(); break;
    case kParallel: lines = &parallel_lines(); break;
    case kHypre: lines = &hypre_lines(); break;
    default: err = "unknown parameter file format " + std::to_string(format); return 101;
  }
  FILE* f = fopen(path, "r");
  if (!f) {
    err = std::string("cannot open ") + path;
    return 102;
  }
  char buf[1024];
  size_t k = 0;
  while (fgets(buf, sizeof(buf), f)) {
    if (k < lines->size() && !apply((*lines)[k], buf, p)) {
      err = std::string(path) + ": unknown keyword '" + first_word(buf) + "' at line " + std::to_string(k + 1);
      fclose(f);
      return 102;
    }
    k++;
  }
  fclose(f);
  return 0;
}

}  // namespace params
}  // namespace pgx
