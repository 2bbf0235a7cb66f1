// Test infrastructure (the oracle), not part of the library.
//
// Prints the vector the reference's SequentialVectorClass::ReadFromMMFile
// (SRC/vectors/sequential_vector.cpp:1192, SequentialVectorReadFromFile in
// SRC/vectors/vectorops.cpp:1116-1180) reads from a coordinate Matrix Market
// file:
//
//   vector_ref FILE IDXIN
//
// prints "rc <code>", then "n <length>" and one "%a" value per line.
#include <cstdio>
#include <cstdlib>

#include "pargemslr.hpp"

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s FILE IDXIN\n", argv[0]);
    return 2;
  }
  pargemslr::SequentialVectorClass<double> v;
  const int rc = v.ReadFromMMFile(argv[1], atoi(argv[2]));
  printf("rc %d\n", rc);
  if (rc == 0) {
    printf("n %d\n", v.GetLengthLocal());
    for (int i = 0; i < v.GetLengthLocal(); i++) printf("%a\n", v[i]);
  }
  return 0;
}
