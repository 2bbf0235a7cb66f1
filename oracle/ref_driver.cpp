/*
 * pgx_ref_driver — project-written driver around the reference ParGeMSLR
 * CPU solver (the oracle; test infrastructure only, never shipped).
 *
 * It follows the reference's own sequential Laplacian driver
 * (ParGeMSLR TESTS/sequential/driver_laplacian_gemslr_seq.cpp:150-305):
 * PargemslrInit -> build CsrMatrixClass -> FlexGmresClass + GemslrClass with a
 * parameter array -> Setup -> Solve, and adds what the parity tests need:
 *
 *   --dump           write the post-setup GeMSLR structures (permutation,
 *                    level/domain pointers, per-domain ILU factors L, D^-1, U
 *                    and the reference's BuildLevels schedules, E, F, W, WH,
 *                    H, the inner Schur-FGMRES settings) to DIR/setup.bin
 *   --solve          run FlexGmresClass::Solve from x0 = 0 and write the
 *                    solution, the iteration count and the residual history
 *   --apply K        run the preconditioner GemslrClass::Solve on K seeded
 *                    vectors and write inputs/outputs (kernel-level checks)
 *
 * Matrix: --lap nx ny nz shift ax ay az (the reference's stencil,
 * CsrMatrixClass::Laplacian) or --csr FILE (PGXD container with
 * A.i, A.j, A.a).  Right-hand side: --xtrue FILE (b = A x_true computed by the
 * reference MatVec) or --rhs FILE.  Parameters: --param IDX=VALUE with the
 * reference's PARGEMSLR_IO_* indices (SRC/utils/utils.hpp:77-297).
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

typedef CsrMatrixClass<double> Csr;
typedef SequentialVectorClass<double> Vec;
typedef GemslrClass<Csr, Vec, double> Gemslr;
typedef FlexGmresClass<Csr, Vec, double> Fgmres;
typedef IluClass<Csr, Vec, double> Ilu;

/* ---------------------------------------------------------------- PGXD I/O */

enum { DT_I32 = 0, DT_F64 = 1, DT_I64 = 2, DT_F32 = 3 };

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
      size_t es = (dt == DT_I32 || dt == DT_F32) ? 4 : 8;
      if (count) std::fwrite(data, es, count, f);
   }
   void i32(const std::string &n, const int *p, uint64_t c) { put(n, DT_I32, p, c); }
   void f64(const std::string &n, const double *p, uint64_t c) { put(n, DT_F64, p, c); }
   void scalar(const std::string &n, int v) { put(n, DT_I32, &v, 1); }
   void scalar(const std::string &n, double v) { put(n, DT_F64, &v, 1); }
};

struct Record {
   int dt;
   std::vector<char> bytes;
};

static std::map<std::string, Record> read_pgxd(const std::string &path)
{
   std::map<std::string, Record> out;
   FILE *f = std::fopen(path.c_str(), "rb");
   if (!f) { std::perror(path.c_str()); std::exit(2); }
   char magic[4];
   if (std::fread(magic, 1, 4, f) != 4 || std::memcmp(magic, "PGXD", 4) != 0)
   {
      std::fprintf(stderr, "%s: not a PGXD file\n", path.c_str());
      std::exit(2);
   }
   uint32_t len;
   while (std::fread(&len, 4, 1, f) == 1)
   {
      std::string name(len, '\0');
      uint8_t d;
      uint64_t count;
      if (std::fread(&name[0], 1, len, f) != len || std::fread(&d, 1, 1, f) != 1 || std::fread(&count, 8, 1, f) != 1)
      {
         std::fprintf(stderr, "%s: truncated\n", path.c_str());
         std::exit(2);
      }
      size_t es = (d == DT_I32 || d == DT_F32) ? 4 : 8;
      Record r;
      r.dt = d;
      r.bytes.resize(es * count);
      if (count && std::fread(r.bytes.data(), es, count, f) != count)
      {
         std::fprintf(stderr, "%s: truncated data\n", path.c_str());
         std::exit(2);
      }
      out[name] = std::move(r);
   }
   std::fclose(f);
   return out;
}

/* ------------------------------------------------------------ dump helpers */

/* write a CSR matrix as name.i/.j/.a plus its shape; CSC storage is transposed
 * into CSR so that every dumped matrix has one layout */
static void put_csr(Writer &w, const std::string &name, Csr &A)
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
   /* CSC -> CSR */
   w.scalar(name + ".was_csc", 1);
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
   w.f64(name, packed.data(), packed.size()); /* column-major, ld = rows */
}

static void put_ivec(Writer &w, const std::string &name, IntVectorClass<int> &v)
{
   w.i32(name, v.GetData(), (uint64_t)std::max(0, v.GetLengthLocal()));
}

static void dump_setup(const std::string &path, Gemslr &P, Csr &A)
{
   Writer w(path);
   int nlev = P._nlev_used;
   w.scalar("n", P._n);
   w.scalar("nlev", nlev);
   put_csr(w, "A", A);
   put_ivec(w, "lev_ptr", P._lev_ptr_v);
   put_ivec(w, "pperm", P._pperm);
   put_ivec(w, "qperm", P._qperm);
   w.scalar("solve_option", P._gemslr_setups._solve_option_setup);
   w.scalar("inner.enable", (int)P._gemslr_setups._enable_inner_iters_setup);
   w.scalar("inner.maxits", P._gemslr_setups._inner_iters_maxits_setup);
   w.scalar("inner.tol", (double)P._gemslr_setups._inner_iters_tol_setup);
   for (int l = 0; l < nlev; l++)
   {
      GemslrLevelClass<Csr, Vec, double> &ls = P._levs_v[l];
      std::string pre = "L" + std::to_string(l) + ".";
      w.scalar(pre + "ncomp", ls._ncomps);
      put_ivec(w, pre + "dom_ptr", P._dom_ptr_v2[l]);
      for (int c = 0; c < ls._ncomps; c++)
      {
         std::string pc = pre + "B" + std::to_string(c) + ".";
         Ilu *ilu = (Ilu *)ls._B_solver[c];
         put_csr(w, pc + "A", ls._B_mat_v[c]);
         put_csr(w, pc + "L", ilu->_L);
         put_csr(w, pc + "U", ilu->_U);
         w.f64(pc + "D", ilu->_D.GetData(), (uint64_t)std::max(0, ilu->_D.GetLengthLocal()));
         put_ivec(w, pc + "rperm", ilu->_row_perm_vec);
         put_ivec(w, pc + "cperm", ilu->_col_perm_vec);
         /* the reference's level-set schedules (IluClass::BuildLevels) */
         if (ilu->_n > 0 && ilu->BuildLevels() == PARGEMSLR_SUCCESS)
         {
            put_ivec(w, pc + "lvl_ptr_l", ilu->_level_ptr_l);
            put_ivec(w, pc + "lvl_l", ilu->_levels_l);
            put_ivec(w, pc + "lvl_ptr_u", ilu->_level_ptr_u);
            put_ivec(w, pc + "lvl_u", ilu->_levels_u);
         }
      }
      if (l < nlev - 1)
      {
         put_csr(w, pre + "E", ls._E_mat);
         put_csr(w, pre + "F", ls._F_mat);
         w.scalar(pre + "lrc", ls._lrc);
         if (ls._lrc > 0)
         {
            put_dense(w, pre + "W", ls._Wk);
            put_dense(w, pre + "WH", ls._WHk);
            put_dense(w, pre + "H", ls._Hk);
         }
      }
   }
}

/* ----------------------------------------------------------------- driver */

static double now_s()
{
   using namespace std::chrono;
   return duration<double>(steady_clock::now().time_since_epoch()).count();
}

static void usage()
{
   std::fprintf(stderr,
      "usage: pgx_ref_driver --out DIR (--lap nx ny nz shift ax ay az | --csr FILE)\n"
      "       [--xtrue FILE | --rhs FILE] [--param IDX=VAL]... [--dump] [--solve]\n"
      "       [--apply K] [--repeat R] [--max-iters-timed M] [--threads T]\n");
   std::exit(2);
}

int main(int argc, char **argv)
{
   std::string out, csr_file, xtrue_file, rhs_file;
   bool lap = false, do_dump = false, do_solve = false, verbose = false, probe = false;
   int nx = 0, ny = 0, nz = 0, apply_k = 0, repeat = 1, threads = 1, timed_maxits = 0;
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
         lap = true;
         nx = std::atoi(argv[++i]); ny = std::atoi(argv[++i]); nz = std::atoi(argv[++i]);
         shift = std::atof(argv[++i]); ax = std::atof(argv[++i]); ay = std::atof(argv[++i]); az = std::atof(argv[++i]);
      }
      else if (a == "--csr") { need(1); csr_file = argv[++i]; }
      else if (a == "--xtrue") { need(1); xtrue_file = argv[++i]; }
      else if (a == "--rhs") { need(1); rhs_file = argv[++i]; }
      else if (a == "--param")
      {
         need(1);
         std::string kv = argv[++i];
         size_t eq = kv.find('=');
         if (eq == std::string::npos) usage();
         overrides.push_back({std::atoi(kv.substr(0, eq).c_str()), std::atof(kv.substr(eq + 1).c_str())});
      }
      else if (a == "--dump") do_dump = true;
      else if (a == "--verbose") verbose = true;
      else if (a == "--probe") probe = true;
      else if (a == "--solve") do_solve = true;
      else if (a == "--apply") { need(1); apply_k = std::atoi(argv[++i]); }
      else if (a == "--repeat") { need(1); repeat = std::max(1, std::atoi(argv[++i])); }
      else if (a == "--threads") { need(1); threads = std::max(1, std::atoi(argv[++i])); }
      else if (a == "--max-iters-timed") { need(1); timed_maxits = std::atoi(argv[++i]); }
      else usage();
   }
   if (out.empty() || (!lap && csr_file.empty())) usage();

   omp_set_num_threads(threads);
   PargemslrInit(&argc, &argv);
   PargemslrInitOpenMP(threads);

   double *params = pargemslr_global::_params;
   for (auto &kv : overrides)
   {
      if (kv.first < 0 || kv.first >= PARGEMSLR_IO_SIZE) usage();
      params[kv.first] = kv.second;
   }
   params[PARGEMSLR_IO_GENERAL_PRINT_LEVEL] = verbose ? 1 : 0;

   /* matrix */
   pargemslr_global::_mersenne_twister_engine.seed(0);
   Csr A;
   if (lap)
   {
      A.Laplacian(nx, ny, nz, ax, ay, az, shift, false);
   }
   else
   {
      auto rec = read_pgxd(csr_file);
      const auto &ri = rec.at("A.i"), &rj = rec.at("A.j"), &ra = rec.at("A.a");
      int n = (int)(ri.bytes.size() / 4) - 1;
      long nnz = (long)(rj.bytes.size() / 4);
      A.Setup(n, n, nnz, kMemoryHost, true);
      std::memcpy(A.GetI(), ri.bytes.data(), ri.bytes.size());
      std::memcpy(A.GetJ(), rj.bytes.data(), rj.bytes.size());
      std::memcpy(A.GetData(), ra.bytes.data(), ra.bytes.size());
      A.SetNumNonzeros();
   }
   int n = A.GetNumRowsLocal();

   Vec x, b;
   x.Setup(n, kMemoryHost, false);
   b.Setup(n, kMemoryHost, false);
   if (!rhs_file.empty())
   {
      auto rec = read_pgxd(rhs_file);
      std::memcpy(b.GetData(), rec.at("b").bytes.data(), sizeof(double) * n);
   }
   else if (!xtrue_file.empty())
   {
      auto rec = read_pgxd(xtrue_file);
      std::memcpy(x.GetData(), rec.at("x_true").bytes.data(), sizeof(double) * n);
      b.Fill(0.0);
      A.MatVec('N', 1.0, x, 0.0, b);
   }
   else
   {
      /* the reference driver's default: solution of ones (sol_opt 0) */
      x.Fill(1.0);
      b.Fill(0.0);
      A.MatVec('N', 1.0, x, 0.0, b);
   }
   x.Fill(0.0);

   {
      Writer w(out + "/problem.bin");
      put_csr(w, "A", A);
      w.f64("b", b.GetData(), n);
   }

   Fgmres solver;
   Gemslr precond;
   solver.SetMatrix(A);
   solver.SetWithParameterArray(params);
   solver.SetSolveLocation(kMemoryHost);
   precond.SetMatrix(A);
   precond.SetWithParameterArray(params);
   precond.SetSolveLocation(kMemoryHost);
   solver.SetPreconditioner(precond);

   double t0 = now_s();
   solver.Setup(x, b);
   double t_setup = now_s() - t0;

   if (do_dump) dump_setup(out + "/setup.bin", precond, A);

   FILE *res = std::fopen((out + "/result.txt").c_str(), "w");
   std::fprintf(res, "n=%d\nnnz=%ld\nsetup_s=%.9g\nthreads=%d\nnlev=%d\n", n, A.GetNumNonzeros(), t_setup, threads,
                precond._nlev_used);
   {
      /* the preconditioner's own nonzero count (GemslrClass::GetNumNonzeros, gemslr.cpp:4127) */
      long int nnz_bsolver = 0, nnz_lr = 0;
      precond.GetNumNonzeros(nnz_bsolver, nnz_lr);
      std::fprintf(res, "nnz_bsolver=%ld\nnnz_lr=%ld\n", nnz_bsolver, nnz_lr);
   }

   if (apply_k > 0)
   {
      /* preconditioner applications on seeded vectors */
      std::mt19937_64 gen(20240501ULL);
      std::uniform_real_distribution<double> U(-1.0, 1.0);
      std::vector<double> vin((size_t)apply_k * n), vout((size_t)apply_k * n);
      Vec vi, vo;
      vi.Setup(n, kMemoryHost, false);
      vo.Setup(n, kMemoryHost, false);
      double ta = now_s();
      for (int k = 0; k < apply_k; k++)
      {
         for (int i = 0; i < n; i++) vin[(size_t)k * n + i] = U(gen);
         std::memcpy(vi.GetData(), &vin[(size_t)k * n], sizeof(double) * n);
         precond.Solve(vo, vi);
         std::memcpy(&vout[(size_t)k * n], vo.GetData(), sizeof(double) * n);
      }
      double t_apply = (now_s() - ta) / apply_k;
      Writer w(out + "/apply.bin");
      w.f64("in", vin.data(), vin.size());
      w.f64("out", vout.data(), vout.size());
      w.scalar("k", apply_k);
      std::fprintf(res, "apply_s=%.9g\n", t_apply);
   }

   if (probe && precond._nlev_used >= 2)
   {
      /* pieces of the level-0 inner solve on seeded vectors: the Schur
       * operator, its preconditioner and the level-1 recursion */
      std::mt19937_64 gen(777ULL);
      std::uniform_real_distribution<double> U(-1.0, 1.0);
      int m0 = n - precond._lev_ptr_v[1];
      Vec xv, yv;
      xv.Setup(m0, kMemoryHost, false);
      yv.Setup(m0, kMemoryHost, false);
      for (int i = 0; i < m0; i++) xv[i] = U(gen);
      std::vector<double> xin(xv.GetData(), xv.GetData() + m0);
      precond.SchurMatVec(0, 'N', 1.0, xv, 0.0, yv);
      std::vector<double> schur(yv.GetData(), yv.GetData() + m0);
      precond._inner_iters_matrix.Solve(yv, xv);
      std::vector<double> ssolve(yv.GetData(), yv.GetData() + m0);
      precond.SolveLevel(yv, xv, 1);
      std::vector<double> lev1(yv.GetData(), yv.GetData() + m0);
      Writer w(out + "/probe.bin");
      w.f64("x", xin.data(), m0);
      w.f64("schur", schur.data(), m0);
      w.f64("schur_solve", ssolve.data(), m0);
      w.f64("level1", lev1.data(), m0);
   }

   if (do_solve)
   {
      if (timed_maxits > 0) solver.SetMaxNumberIterations(timed_maxits);
      double best = 1e300, total = 0.0;
      std::string times;
      for (int r = 0; r < repeat; r++)
      {
         x.Fill(0.0);
         double ts = now_s();
         solver.Solve(x, b);
         double dt = now_s() - ts;
         best = std::min(best, dt);
         total += dt;
         char buf[64];
         std::snprintf(buf, sizeof(buf), "%s%.9g", r ? "," : "", dt);
         times += buf;
      }
      std::fprintf(res, "solve_times=%s\n", times.c_str());
      /* true relative residual in FP64 */
      Vec r;
      r.Setup(n, kMemoryHost, false);
      std::memcpy(r.GetData(), b.GetData(), sizeof(double) * n);
      A.MatVec('N', -1.0, x, 1.0, r);
      double nr = 0.0, nb = 0.0;
      r.Norm2(nr);
      b.Norm2(nb);
      std::fprintf(res, "iters=%d\nrel_res=%.17g\ntrue_rel_res=%.17g\nsolve_s=%.9g\nsolve_s_mean=%.9g\nrepeat=%d\n",
                   solver.GetNumberIterations(), solver.GetFinalRelativeResidual(), nr / nb, best, total / repeat,
                   repeat);
      Writer w(out + "/solution.bin");
      w.f64("x", x.GetData(), n);
      SequentialVectorClass<double> &hist = solver.GetRelativeResidual();
      w.f64("rel_res_hist", hist.GetData(), (uint64_t)std::max(0, hist.GetLengthLocal()));
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
