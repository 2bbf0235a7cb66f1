// The double[180] parameter array: defaults and the plain-text parameter
// files of the reference's drivers (see params.cpp).
#pragma once

#include <string>

namespace pgx {
namespace params {

constexpr int kSize = 180;

enum FileFormat { kSequential = 0, kParallel = 1, kHypre = 2 };

void set_defaults(double* p);
// Returns 0, or 102 (the reference's I/O error code) with a message in err;
// 101 for an unknown format.
int read_file(const char* path, int format, double* p, std::string& err);
// "-tol V", "-kdim N", "-maxits N" from a driver's command line.
void read_args(int argc, const char* const* argv, double* p);

}  // namespace params
}  // namespace pgx
