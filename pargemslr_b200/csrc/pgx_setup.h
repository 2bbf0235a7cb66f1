// Host setup of the GeMSLR structures (see setup.cpp).
#pragma once

#include <string>
#include <vector>

namespace pgx {
namespace setup {

struct Graph {
  int n = 0;
  std::vector<int> xadj, adj;
};

struct Csr {
  int rows = 0, cols = 0;
  std::vector<int> rp, cj;
  std::vector<double> va;
};

struct Factor {
  Csr L, U;
  std::vector<double> dinv;
};

// new position -> old index, level pointers and per-level subdomain pointers
// (relative to the level start)
struct Ordering {
  std::vector<int> perm;
  std::vector<int> lev_ptr;
  std::vector<std::vector<int>> dom_ptr;
};

Graph symmetric_graph(int n, const int* rp, const int* cj);
// order inside every subdomain: as found, reverse Cuthill-McKee, or greedy multicolor
enum class LocalOrder { kNone, kRcm, kMulticolor };
Ordering gemslr_ordering(const Graph& g, int nlev, int minsep, bool local_rcm);
Ordering gemslr_ordering(const Graph& g, int nlev, int minsep, LocalOrder local);
int ilut(int n, const int* rp, const int* cj, const double* va, double droptol, int lfil, Factor& f);
int read_matrix_market(const char* path, Csr& out, std::string& err);
int read_matrix_market_vector(const char* path, int idxin, std::vector<double>& x, std::string& err);
Csr permuted_block(int n, const int* rp, const int* cj, const double* va, const std::vector<int>& perm,
                   const std::vector<int>& iperm, int r0, int r1, int c0, int c1);

}  // namespace setup
}  // namespace pgx
