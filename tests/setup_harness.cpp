// Host checks of the GeMSLR setup routines (setup.cpp): the nested-
// dissection level structure, ILUT and the Matrix Market reader.  Built and
// run by tests/test_setup_host.py; prints "ok" lines and exits 0 on success.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../pargemslr_b200/csrc/pgx_setup.h"

using namespace pgx::setup;

static int failures = 0;
#define CHECK(cond, ...)                  \
  do {                                    \
    if (!(cond)) {                        \
      std::printf("FAIL: " __VA_ARGS__);  \
      std::printf("\n");                  \
      failures++;                         \
    }                                     \
  } while (0)

// 7-point Laplacian of an N^3 grid (x fastest), CSR with sorted columns
static void laplace3d(int N, std::vector<int>& rp, std::vector<int>& cj, std::vector<double>& va) {
  rp.assign(1, 0);
  cj.clear();
  va.clear();
  auto id = [&](int x, int y, int z) { return (z * N + y) * N + x; };
  for (int z = 0; z < N; z++)
    for (int y = 0; y < N; y++)
      for (int x = 0; x < N; x++) {
        const int cols[7] = {z > 0 ? id(x, y, z - 1) : -1, y > 0 ? id(x, y - 1, z) : -1, x > 0 ? id(x - 1, y, z) : -1,
                             id(x, y, z), x < N - 1 ? id(x + 1, y, z) : -1, y < N - 1 ? id(x, y + 1, z) : -1,
                             z < N - 1 ? id(x, y, z + 1) : -1};
        for (int c : cols)
          if (c >= 0) {
            cj.push_back(c);
            va.push_back(c == id(x, y, z) ? 6.0 : -1.0);
          }
        rp.push_back((int)cj.size());
      }
}

int main(int argc, char** argv) {
  const int N = 14, n = N * N * N;
  std::vector<int> rp, cj;
  std::vector<double> va;
  laplace3d(N, rp, cj, va);
  Graph g = symmetric_graph(n, rp.data(), cj.data());

  // 1. levels: a permutation; within a level, subdomains do not couple
  Ordering o = gemslr_ordering(g, 4, 10, true);
  std::vector<int> seen(n, 0), iperm(n);
  for (int i = 0; i < n; i++) {
    CHECK(o.perm[i] >= 0 && o.perm[i] < n, "perm entry out of range");
    seen[o.perm[i]]++;
    iperm[o.perm[i]] = i;
  }
  for (int i = 0; i < n; i++) CHECK(seen[i] == 1, "perm is not a permutation");
  const int nlev = (int)o.lev_ptr.size() - 1;
  CHECK(nlev >= 2 && o.lev_ptr[0] == 0 && o.lev_ptr[nlev] == n, "level pointers");
  int coupled = 0;
  for (int l = 0; l < nlev; l++) {
    const int s = o.lev_ptr[l], e = o.lev_ptr[l + 1];
    const std::vector<int>& dom = o.dom_ptr[l];
    CHECK(dom.front() == 0 && dom.back() == e - s, "domain pointers of level %d", l);
    std::vector<int> comp(e - s);
    for (size_t c = 0; c + 1 < dom.size(); c++)
      for (int r = dom[c]; r < dom[c + 1]; r++) comp[r] = (int)c;
    for (int r = s; r < e; r++) {
      const int old = o.perm[r];
      for (int k = rp[old]; k < rp[old + 1]; k++) {
        const int q = iperm[cj[k]];
        if (q >= s && q < e && comp[q - s] != comp[r - s]) coupled++;
      }
    }
  }
  CHECK(coupled == 0, "%d couplings between subdomains of one level", coupled);
  std::printf("ok levels: %d levels, level 0 has %zu subdomains\n", nlev, o.dom_ptr[0].size() - 1);

  // 2. ILUT with no dropping on a small block is the exact LU: (L + I) (U + D) reproduces B
  const int s0 = o.lev_ptr[0], c0e = s0 + o.dom_ptr[0][1];
  Csr B = permuted_block(n, rp.data(), cj.data(), va.data(), o.perm, iperm, s0, c0e, s0, c0e);
  Factor f;
  CHECK(ilut(B.rows, B.rp.data(), B.cj.data(), B.va.data(), 0.0, B.rows, f) == 0, "ilut failed");
  const int m = B.rows;
  std::vector<double> dense((size_t)m * m, 0.0);
  for (int i = 0; i < m; i++) {
    // row i of L+I times (U + D): sum_k L(i,k) Urow(k) + Urow(i)
    std::vector<double> row((size_t)m, 0.0);
    auto add_urow = [&](int k, double s) {
      row[k] += s / f.dinv[k];
      for (int t = f.U.rp[k]; t < f.U.rp[k + 1]; t++) row[f.U.cj[t]] += s * f.U.va[t];
    };
    add_urow(i, 1.0);
    for (int t = f.L.rp[i]; t < f.L.rp[i + 1]; t++) add_urow(f.L.cj[t], f.L.va[t]);
    for (int k = B.rp[i]; k < B.rp[i + 1]; k++) row[B.cj[k]] -= B.va[k];
    double err = 0.0;
    for (double v : row) err = std::fmax(err, std::fabs(v));
    CHECK(err < 1e-10, "row %d of LU - B: %g", i, err);
  }
  for (int i = 0; i < m; i++)
    for (int t = f.L.rp[i]; t < f.L.rp[i + 1]; t++) CHECK(f.L.cj[t] < i, "L not strictly lower");
  std::printf("ok ilut: exact LU of a %d-row subdomain block\n", m);

  // 3. with dropping, the factors keep at most lfil entries per row part
  Factor g2;
  CHECK(ilut(B.rows, B.rp.data(), B.cj.data(), B.va.data(), 1e-2, 5, g2) == 0, "ilut(1e-2, 5) failed");
  int longest = 0;
  for (int i = 0; i < m; i++) {
    longest = std::max(longest, g2.L.rp[i + 1] - g2.L.rp[i]);
    longest = std::max(longest, g2.U.rp[i + 1] - g2.U.rp[i]);
  }
  CHECK(longest <= 5, "row part with %d entries > lfil 5", longest);
  std::printf("ok ilut: fill limit respected (longest row part %d)\n", longest);

  // 4. Matrix Market: symmetric file mirrored, duplicates summed
  if (argc > 1) {
    Csr mm;
    std::string err;
    CHECK(read_matrix_market(argv[1], mm, err) == 0, "read_matrix_market: %s", err.c_str());
    CHECK(mm.rows == 3 && mm.cols == 3, "mm size");
    const std::vector<int> erp = {0, 2, 3, 5}, ecj = {0, 2, 1, 0, 2};
    const std::vector<double> eva = {3.5, -1.0, 2.0, -1.0, 4.0};
    CHECK(mm.rp == erp && mm.cj == ecj && mm.va == eva, "mm contents");
    std::printf("ok matrix market\n");
  }
  // 5. multicolor order inside subdomains: the same levels and subdomains as the RCM order; each level-0
  //    subdomain is a few uncoupled runs of rows (two on this grid); its ILUT factor has far fewer dependency levels
  {
    Ordering om = gemslr_ordering(g, 4, 10, LocalOrder::kMulticolor);
    std::vector<int> seen2(n, 0), iperm2(n);
    for (int i = 0; i < n; i++) {
      seen2[om.perm[i]]++;
      iperm2[om.perm[i]] = i;
    }
    bool perm_ok = true;
    for (int i = 0; i < n; i++) perm_ok = perm_ok && seen2[i] == 1;
    CHECK(perm_ok, "multicolor perm is not a permutation");
    CHECK(om.lev_ptr == o.lev_ptr && om.dom_ptr == o.dom_ptr, "multicolor changes the level structure");
    int most_runs = 0;
    const std::vector<int>& dom = om.dom_ptr[0];
    for (size_t c = 0; c + 1 < dom.size(); c++) {
      // count maximal runs of the subdomain's order in which no two rows couple
      std::vector<int> run_of(n, -1);
      int runs = 1;
      for (int r = dom[c]; r < dom[c + 1]; r++) {
        const int old = om.perm[r];
        bool clash = false;
        for (int k = rp[old]; k < rp[old + 1] && !clash; k++) clash = cj[k] != old && run_of[cj[k]] == runs;
        if (clash) runs++;
        run_of[old] = runs;
      }
      most_runs = std::max(most_runs, runs);
    }
    CHECK(most_runs <= 3, "a subdomain splits into %d uncoupled runs", most_runs);
    auto depth = [](const Csr& L) {
      std::vector<int> lev(L.rows, 0);
      int mx = 0;
      for (int i = 0; i < L.rows; i++) {
        for (int k = L.rp[i]; k < L.rp[i + 1]; k++) lev[i] = std::max(lev[i], lev[L.cj[k]] + 1);
        mx = std::max(mx, lev[i] + 1);
      }
      return mx;
    };
    const int e0 = dom[1];
    Csr Bm = permuted_block(n, rp.data(), cj.data(), va.data(), om.perm, iperm2, 0, e0, 0, e0);
    Csr Br = permuted_block(n, rp.data(), cj.data(), va.data(), o.perm, iperm, 0, e0, 0, e0);
    Factor fm, fr;
    CHECK(ilut(Bm.rows, Bm.rp.data(), Bm.cj.data(), Bm.va.data(), 1e-3, 200, fm) == 0, "ilut (multicolor)");
    CHECK(ilut(Br.rows, Br.rp.data(), Br.cj.data(), Br.va.data(), 1e-3, 200, fr) == 0, "ilut (RCM)");
    const int dm = depth(fm.L), dr = depth(fr.L);
    CHECK(2 * dm < dr, "multicolor factor depth %d not below half the RCM depth %d", dm, dr);
    std::printf("ok multicolor: at most %d uncoupled runs per subdomain; factor depth %d against %d (RCM)\n", most_runs,
                dm, dr);
  }

  // 6. the red-black split of a multicolor subdomain's factors: the leading (red) rows have empty L rows and U entries
  //    only into later colors, so L y = b is y_r = b_r, y_b = L_bb^-1 (b_b - L_br b_r), and (D + U) x = y is
  //    x_b = (D_b + U_bb)^-1 y_b, x_r = D_r^-1 (y_r - U_rb x_b); both equal the plain solves to rounding
  {
    Ordering om = gemslr_ordering(g, 4, 10, LocalOrder::kMulticolor);
    std::vector<int> iperm2(n);
    for (int i = 0; i < n; i++) iperm2[om.perm[i]] = i;
    const int e0 = om.dom_ptr[0][1];
    Csr Bm = permuted_block(n, rp.data(), cj.data(), va.data(), om.perm, iperm2, 0, e0, 0, e0);
    Factor fm;
    CHECK(ilut(Bm.rows, Bm.rp.data(), Bm.cj.data(), Bm.va.data(), 1e-3, 200, fm) == 0, "ilut (multicolor)");
    const int m = Bm.rows;
    int nred = 0;
    while (nred < m && fm.L.rp[nred + 1] == fm.L.rp[nred]) nred++;
    int red_red_u = 0;
    for (int r = 0; r < nred; r++)
      for (int k = fm.U.rp[r]; k < fm.U.rp[r + 1]; k++) red_red_u += fm.U.cj[k] < nred;
    CHECK(nred > m / 3 && red_red_u == 0, "red rows %d of %d, %d red-red U entries", nred, m, red_red_u);
    std::vector<double> b(m);
    for (int i = 0; i < m; i++) b[i] = std::sin(0.37 * i + 0.1);
    // plain solves
    std::vector<double> y(m), x(m);
    for (int i = 0; i < m; i++) {
      double s = b[i];
      for (int k = fm.L.rp[i]; k < fm.L.rp[i + 1]; k++) s -= fm.L.va[k] * y[fm.L.cj[k]];
      y[i] = s;
    }
    for (int i = m - 1; i >= 0; i--) {
      double s = y[i];
      for (int k = fm.U.rp[i]; k < fm.U.rp[i + 1]; k++) s -= fm.U.va[k] * x[fm.U.cj[k]];
      x[i] = s * fm.dinv[i];
    }
    // split solves
    std::vector<double> ys(m), xs(m);
    for (int i = 0; i < nred; i++) ys[i] = b[i];
    for (int i = nred; i < m; i++) {  // b_b - L_br b_r, then the black-only forward solve
      double s = b[i];
      for (int k = fm.L.rp[i]; k < fm.L.rp[i + 1]; k++)
        if (fm.L.cj[k] < nred) s -= fm.L.va[k] * b[fm.L.cj[k]];
      ys[i] = s;
    }
    for (int i = nred; i < m; i++) {
      double s = ys[i];
      for (int k = fm.L.rp[i]; k < fm.L.rp[i + 1]; k++)
        if (fm.L.cj[k] >= nred) s -= fm.L.va[k] * ys[fm.L.cj[k]];
      ys[i] = s;
    }
    for (int i = m - 1; i >= nred; i--) {  // the black-only backward solve
      double s = ys[i];
      for (int k = fm.U.rp[i]; k < fm.U.rp[i + 1]; k++) s -= fm.U.va[k] * xs[fm.U.cj[k]];
      xs[i] = s * fm.dinv[i];
    }
    for (int i = 0; i < nred; i++) {  // x_r = D_r^-1 (y_r - U_rb x_b)
      double s = ys[i];
      for (int k = fm.U.rp[i]; k < fm.U.rp[i + 1]; k++) s -= fm.U.va[k] * xs[fm.U.cj[k]];
      xs[i] = s * fm.dinv[i];
    }
    double dy = 0, dx = 0, ny = 0, nx = 0;
    for (int i = 0; i < m; i++) {
      dy = std::max(dy, std::fabs(ys[i] - y[i]));
      dx = std::max(dx, std::fabs(xs[i] - x[i]));
      ny = std::max(ny, std::fabs(y[i]));
      nx = std::max(nx, std::fabs(x[i]));
    }
    CHECK(dy <= 1e-13 * ny && dx <= 1e-13 * nx, "split solves differ: %.2e / %.2e", dy / ny, dx / nx);
    std::printf("ok red-black split: %d red rows of %d; split solves within %.1e / %.1e of the plain ones\n", nred, m,
                dy / ny, dx / nx);
  }
  return failures ? 1 : 0;
}
