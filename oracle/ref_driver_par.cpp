/*
 * pgx_ref_driver_par — project-written driver around the reference's
 * ParallelGemslrClass at one MPI rank (the oracle; test infrastructure only,
 * never shipped).
 *
 * It follows the reference's parallel Laplacian driver
 * (ParGeMSLR TESTS/parallel/driver_laplacian_gemslr_par.cpp): a
 * ParallelCsrMatrixClass Laplacian, FlexGmresClass + ParallelGemslrClass with
 * a parameter array, Setup, Solve.  The solve phase of ParallelGemslrClass
 * (parallel_gemslr.cpp:5496-5810) permutes each level's vector through the
 * level's CommunicationHelperClass before the level is solved and back after
 * it.  At one rank that transfer is a fixed permutation; this driver probes it
 * by transferring the index vector 0..N-1 and records the result:
 *
 *   --dump     DIR/setup_par.bin: n, nlev, lev_ptr, A, per level the
 *              subdomains' ILU factors (L, D^-1, U) and blocks B, the level's
 *              E and F (local parts), W, WH, the rank, and "perm" (perm[i] =
 *              the input index that lands at position i of the level's frame;
 *              identity when the level has no transfer); the rank of the
 *              global low-rank correction on A; the inner-FGMRES settings
 *   --solve    FlexGmresClass::Solve from x0 = 0 (DIR/solution.bin, result.txt)
 *   --apply K  ParallelGemslrClass::Solve on K seeded vectors (DIR/apply.bin)
 *
 * Matrix: --lap nx ny nz shift ax ay az (ParallelCsrMatrixClass::Laplacian
 * with one rank).  Right-hand side: --xtrue FILE (b = A x_true).
 *
 * The dump reads protected members of the reference classes; the access
 * specifiers are opened only inside this translation unit.
 */
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <random>
#include <sstream>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>
#include <omp.h>

#define private public
#define protected public
#include "pargemslr.hpp"
#undef private
#undef protected

using namespace pargemslr;

typedef ParallelCsrMatrixClass<double> PCsr;
typedef ParallelVectorClass<double> PVec;
typedef ParallelGemslrClass<PCsr, PVec, double> PGemslr;
typedef FlexGmresClass<PCsr, PVec, double> PFgmres;
typedef IluClass<CsrMatrixClass<double>, SequentialVectorClass<double>, double> Ilu;

enum { DT_I32 = 0, DT_F64 = 1 };

struct Writer {
   FILE *f;
   explicit Writer(const std::string &path)
   {
      f = std::fopen(path.c_str(), "wb");
      if (!f) { std::perror(path.c_str()); std::exit(2); }
      std::fwrite("PGXD", 1, 4, f);
   }
   ~Writer() { std::fclose(f); }
   void put(const std::string &name, int dt, const void *data, uint64_t count)
   {
      uint32_t len = (uint32_t)name.size();
      uint8_t d = (uint8_t)dt;
      std::fwrite(&len, 4, 1, f);
      std::fwrite(name.data(), 1, len, f);
      std::fwrite(&d, 1, 1, f);
      std::fwrite(&count, 8, 1, f);
      if (count) std::fwrite(data, dt == DT_I32 ? 4 : 8, count, f);
   }
   void i32(const std::string &n, const int *p, uint64_t c) { put(n, DT_I32, p, c); }
   void f64(const std::string &n, const double *p, uint64_t c) { put(n, DT_F64, p, c); }
   void scalar(const std::string &n, int v) { put(n, DT_I32, &v, 1); }
   void scalar(const std::string &n, double v) { put(n, DT_F64, &v, 1); }
};

static std::vector<double> read_f64(const std::string &path, const std::string &key)
{
   FILE *f = std::fopen(path.c_str(), "rb");
   if (!f) { std::perror(path.c_str()); std::exit(2); }
   char magic[4];
   if (std::fread(magic, 1, 4, f) != 4 || std::memcmp(magic, "PGXD", 4) != 0) std::exit(2);
   uint32_t len;
   std::vector<double> out;
   while (std::fread(&len, 4, 1, f) == 1)
   {
      std::string name(len, '\0');
      uint8_t d;
      uint64_t count;
      if (std::fread(&name[0], 1, len, f) != len || std::fread(&d, 1, 1, f) != 1 || std::fread(&count, 8, 1, f) != 1)
         std::exit(2);
      std::vector<char> bytes((d == DT_I32 ? 4 : 8) * count);
      if (count && std::fread(bytes.data(), 1, bytes.size(), f) != bytes.size()) std::exit(2);
      if (name == key && d == DT_F64)
      {
         out.resize(count);
         std::memcpy(out.data(), bytes.data(), bytes.size());
      }
   }
   std::fclose(f);
   return out;
}

/* a sequential CSR (or CSC, transposed into CSR) as name.i/.j/.a and its shape */
static void put_csr(Writer &w, const std::string &name, CsrMatrixClass<double> &A)
{
   int nr = A.GetNumRowsLocal(), nc = A.GetNumColsLocal();
   long nnz = A.GetNumNonzeros();
   int shape[2] = {nr, nc};
   w.i32(name + ".shape", shape, 2);
   if (nnz == 0 || A.GetI() == nullptr)
   {
      std::vector<int> ip(nr + 1, 0);
      w.i32(name + ".i", ip.data(), ip.size());
      w.i32(name + ".j", nullptr, 0);
      w.f64(name + ".a", nullptr, 0);
      return;
   }
   if (A.IsCsr())
   {
      w.i32(name + ".i", A.GetI(), nr + 1);
      w.i32(name + ".j", A.GetJ(), nnz);
      w.f64(name + ".a", A.GetData(), nnz);
      return;
   }
   const int *cp = A.GetI(), *ri = A.GetJ();
   const double *va = A.GetData();
   std::vector<int> ip(nr + 1, 0), jp(nnz);
   std::vector<double> ap(nnz);
   for (long k = 0; k < nnz; k++) ip[ri[k] + 1]++;
   for (int r = 0; r < nr; r++) ip[r + 1] += ip[r];
   std::vector<int> pos(ip.begin(), ip.end() - 1);
   for (int c = 0; c < nc; c++)
      for (int k = cp[c]; k < cp[c + 1]; k++)
      {
         int p = pos[ri[k]]++;
         jp[p] = c;
         ap[p] = va[k];
      }
   w.i32(name + ".i", ip.data(), ip.size());
   w.i32(name + ".j", jp.data(), jp.size());
   w.f64(name + ".a", ap.data(), ap.size());
}

static void put_dense(Writer &w, const std::string &name, DenseMatrixClass<double> &M)
{
   int nr = M.GetNumRowsLocal(), nc = M.GetNumColsLocal();
   int shape[2] = {nr, nc};
   w.i32(name + ".shape", shape, 2);
   std::vector<double> packed((size_t)nr * nc);
   if (nr * (size_t)nc > 0)
   {
      int ld = M.GetLeadingDimension();
      const double *d = M.GetData();
      for (int c = 0; c < nc; c++)
         for (int r = 0; r < nr; r++) packed[(size_t)c * nr + r] = d[(size_t)c * ld + r];
   }
   w.f64(name, packed.data(), packed.size());
}

/* the permutation the level's transfer applies: out[i] = in[perm[i]] */
static std::vector<int> probe_perm(CommunicationHelperClass &ch, int nloc)
{
   std::vector<int> perm(nloc);
   for (int i = 0; i < nloc; i++) perm[i] = i;
   if (!ch._is_ready) return perm;
   SequentialVectorClass<double> vin, vout;
   vin.Setup(nloc, kMemoryHost, false);
   vout.Setup(nloc, kMemoryHost, false);
   for (int i = 0; i < nloc; i++) vin[i] = (double)i;
   vout.Fill(-1.0);
   ch.DataTransfer(vin, vout, kMemoryHost, kMemoryHost);
   for (int i = 0; i < nloc; i++) perm[i] = (int)vout[i];
   return perm;
}

static void dump_setup(const std::string &path, PGemslr &P, PCsr &A)
{
   Writer w(path);
   int nlev = P._nlev_used;
   int n = A.GetNumRowsLocal();
   w.scalar("n", n);
   w.scalar("nlev", nlev);
   put_csr(w, "A", A.GetDiagMat());
   w.i32("lev_ptr", P._lev_ptr_v.GetData(), (uint64_t)nlev + 1);
   w.scalar("solve_option", P._gemslr_setups._solve_option_setup);
   w.scalar("global_precond", P._global_precond_option);
   w.scalar("inner.enable", (int)P._gemslr_setups._enable_inner_iters_setup);
   w.scalar("inner.maxits", P._gemslr_setups._inner_iters_maxits_setup);
   w.scalar("inner.tol", (double)P._gemslr_setups._inner_iters_tol_setup);
   w.scalar("lrcA", P._lev_A.empty() ? 0 : P._lev_A[0]._lrc);
   for (int l = 0; l < nlev; l++)
   {
      ParallelGemslrLevelClass<PCsr, PVec, double> &ls = P._levs_v[l];
      std::string pre = "L" + std::to_string(l) + ".";
      const int nloc = n - P._lev_ptr_v[l];
      std::vector<int> perm = probe_perm(ls._comm_helper, nloc);
      w.i32(pre + "perm", perm.data(), perm.size());
      w.scalar(pre + "ncomp", ls._ncomps);
      w.i32(pre + "dom_ptr", P._dom_ptr_v2[l].GetData(), (uint64_t)ls._ncomps + 1);
      for (int c = 0; c < ls._ncomps; c++)
      {
         std::string pc = pre + "B" + std::to_string(c) + ".";
         Ilu *ilu = (Ilu *)ls._B_solver[c];
         put_csr(w, pc + "A", ls._B_mat_v[c]);
         put_csr(w, pc + "L", ilu->_L);
         put_csr(w, pc + "U", ilu->_U);
         w.f64(pc + "D", ilu->_D.GetData(), (uint64_t)std::max(0, ilu->_D.GetLengthLocal()));
         w.scalar(pc + "perms", (int)(ilu->_row_perm_vec.GetLengthLocal() + ilu->_col_perm_vec.GetLengthLocal()));
      }
      if (l < nlev - 1)
      {
         put_csr(w, pre + "E", ls._E_mat.GetDiagMat());
         put_csr(w, pre + "F", ls._F_mat.GetDiagMat());
         w.scalar(pre + "lrc", ls._lrc);
         if (ls._lrc > 0)
         {
            put_dense(w, pre + "W", ls._Wk);
            put_dense(w, pre + "WH", ls._WHk);
         }
      }
   }
}

static double now_s()
{
   using namespace std::chrono;
   return duration<double>(steady_clock::now().time_since_epoch()).count();
}

static void usage()
{
   std::fprintf(stderr, "usage: pgx_ref_driver_par --out DIR --lap nx ny nz shift ax ay az [--xtrue FILE]\n"
                        "       [--param IDX=VAL]... [--dump] [--solve] [--apply K] [--threads T]\n");
   std::exit(2);
}

int main(int argc, char **argv)
{
   std::string out, xtrue_file;
   bool do_dump = false, do_solve = false, have_lap = false;
   int nx = 0, ny = 0, nz = 0, apply_k = 0, threads = 1;
   double shift = 0, ax = 0, ay = 0, az = 0;
   std::vector<std::pair<int, double>> overrides;
   for (int i = 1; i < argc; i++)
   {
      std::string a = argv[i];
      auto need = [&](int k) { if (i + k >= argc) usage(); };
      if (a == "--out") { need(1); out = argv[++i]; }
      else if (a == "--lap")
      {
         need(7);
         have_lap = true;
         nx = std::atoi(argv[++i]); ny = std::atoi(argv[++i]); nz = std::atoi(argv[++i]);
         shift = std::atof(argv[++i]); ax = std::atof(argv[++i]); ay = std::atof(argv[++i]); az = std::atof(argv[++i]);
      }
      else if (a == "--xtrue") { need(1); xtrue_file = argv[++i]; }
      else if (a == "--param")
      {
         need(1);
         std::string kv = argv[++i];
         size_t eq = kv.find('=');
         if (eq == std::string::npos) usage();
         overrides.push_back({std::atoi(kv.substr(0, eq).c_str()), std::atof(kv.substr(eq + 1).c_str())});
      }
      else if (a == "--dump") do_dump = true;
      else if (a == "--solve") do_solve = true;
      else if (a == "--apply") { need(1); apply_k = std::atoi(argv[++i]); }
      else if (a == "--threads") { need(1); threads = std::max(1, std::atoi(argv[++i])); }
      else usage();
   }
   if (out.empty() || !have_lap) usage();

   omp_set_num_threads(threads);
   PargemslrInit(&argc, &argv);
   PargemslrInitOpenMP(threads);
   double *params = pargemslr_global::_params;
   for (auto &kv : overrides)
   {
      if (kv.first < 0 || kv.first >= PARGEMSLR_IO_SIZE) usage();
      params[kv.first] = kv.second;
   }
   params[PARGEMSLR_IO_GENERAL_PRINT_LEVEL] = 0;

   pargemslr_global::_mersenne_twister_engine.seed(0);
   parallel_log parlog;
   PCsr A;
   A.Laplacian(nx, ny, nz, 1, 1, 1, ax, ay, az, shift, parlog, false);
   int n = A.GetNumRowsLocal();

   PVec x, b;
   x.Setup(n, 0, n, kMemoryHost, false, parlog);
   b.Setup(n, 0, n, kMemoryHost, false, parlog);
   if (!xtrue_file.empty())
   {
      std::vector<double> xt = read_f64(xtrue_file, "x_true");
      if ((int)xt.size() != n) usage();
      std::memcpy(x.GetData(), xt.data(), sizeof(double) * n);
   }
   else
   {
      x.Fill(1.0);
   }
   b.Fill(0.0);
   A.MatVec('N', 1.0, x, 0.0, b);
   x.Fill(0.0);
   {
      Writer w(out + "/problem.bin");
      put_csr(w, "A", A.GetDiagMat());
      w.f64("b", b.GetData(), n);
   }

   PFgmres solver;
   PGemslr precond;
   solver.SetMatrixP(&A);
   solver.SetWithParameterArray(params);
   solver.SetSolveLocation(kMemoryHost);
   precond.SetMatrixP(&A);
   precond.SetWithParameterArray(params);
   precond.SetSolveLocation(kMemoryHost);
   solver.SetPreconditionerP(&precond);
   double t0 = now_s();
   solver.Setup(x, b);
   double t_setup = now_s() - t0;
   if (do_dump) dump_setup(out + "/setup_par.bin", precond, A);

   FILE *res = std::fopen((out + "/result.txt").c_str(), "w");
   std::fprintf(res, "n=%d\nsetup_s=%.9g\nthreads=%d\nnlev=%d\n", n, t_setup, threads, precond._nlev_used);
   if (apply_k > 0)
   {
      std::mt19937_64 gen(20240501ULL);
      std::uniform_real_distribution<double> U(-1.0, 1.0);
      std::vector<double> vin((size_t)apply_k * n), vout((size_t)apply_k * n);
      PVec vi, vo;
      vi.Setup(n, 0, n, kMemoryHost, false, parlog);
      vo.Setup(n, 0, n, kMemoryHost, false, parlog);
      for (int k = 0; k < apply_k; k++)
      {
         for (int i = 0; i < n; i++) vin[(size_t)k * n + i] = U(gen);
         std::memcpy(vi.GetData(), &vin[(size_t)k * n], sizeof(double) * n);
         vo.Fill(0.0);
         precond.Solve(vo, vi);
         std::memcpy(&vout[(size_t)k * n], vo.GetData(), sizeof(double) * n);
      }
      Writer w(out + "/apply.bin");
      w.f64("in", vin.data(), vin.size());
      w.f64("out", vout.data(), vout.size());
      w.scalar("k", apply_k);
   }
   if (do_solve)
   {
      x.Fill(0.0);
      double ts = now_s();
      solver.Solve(x, b);
      double dt = now_s() - ts;
      PVec r;
      r.Setup(n, 0, n, kMemoryHost, false, parlog);
      std::memcpy(r.GetData(), b.GetData(), sizeof(double) * n);
      A.MatVec('N', -1.0, x, 1.0, r);
      double nr = 0.0, nb = 0.0;
      r.Norm2(nr);
      b.Norm2(nb);
      std::fprintf(res, "iters=%d\nrel_res=%.17g\ntrue_rel_res=%.17g\nsolve_s=%.9g\n", solver.GetNumberIterations(),
                   solver.GetFinalRelativeResidual(), nr / nb, dt);
      Writer w(out + "/solution.bin");
      w.f64("x", x.GetData(), n);
   }
   std::fclose(res);
   solver.Clear();
   precond.Clear();
   A.Clear();
   x.Clear();
   b.Clear();
   PargemslrFinalize();
   return 0;
}
