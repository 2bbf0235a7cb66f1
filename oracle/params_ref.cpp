// Test infrastructure (the oracle), not part of the library.
//
// Prints the parameter array that one of the reference's own parameter-file
// parsers builds.  The Makefile links this file with one of
//   TESTS/sequential/io.cpp                      -> _ref/params_ref_sequential
//   TESTS/parallel/io_par.cpp                    -> _ref/params_ref_parallel
//   TESTS/hypre/pargemslr_hypre_interface.cpp    -> _ref/params_ref_hypre
// each compiled where it lies, and with libpargemslr_ref.so for the defaults.
//
//   params_ref_<format> FILE [FILL]
//
// starts from PargemslrSetDefaultParameterArray (SRC/utils/utils.cpp:30-126),
// or from FILL in every slot when given (so a test sees exactly which slots
// the file writes), calls read_inputs_from_file(FILE, params) and prints
// "rc <code>" then "<slot> <value as %a>" for the 180 slots.
//
//   params_ref_<format> --args ARG...
//
// applies the driver's command-line reader read_inputs(params, argc, argv)
// to ARG... instead (sequential and parallel drivers only).
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace pargemslr {
double* PargemslrSetDefaultParameterArray(double* params);
}
int read_inputs_from_file(const char* filename, double* params);
#ifdef PGX_REF_HAS_READ_INPUTS
int read_inputs(double* input, int argc, char** argv);
#endif

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: %s FILE [FILL]\n", argv[0]);
    return 2;
  }
  double p[180];
  if (std::strcmp(argv[1], "--args") == 0) {
#ifdef PGX_REF_HAS_READ_INPUTS
    pargemslr::PargemslrSetDefaultParameterArray(p);
    const int rc = read_inputs(p, argc - 2, argv + 2);
    printf("rc %d\n", rc);
    for (int i = 0; i < 180; i++) printf("%d %a\n", i, p[i]);
    return 0;
#else
    fprintf(stderr, "this driver has no read_inputs\n");
    return 2;
#endif
  }
  if (argc > 2) {
    const double fill = strtod(argv[2], nullptr);
    for (int i = 0; i < 180; i++) p[i] = fill;
  } else {
    pargemslr::PargemslrSetDefaultParameterArray(p);
  }
  const int rc = read_inputs_from_file(argv[1], p);
  printf("rc %d\n", rc);
  for (int i = 0; i < 180; i++) printf("%d %a\n", i, p[i]);
  return 0;
}
