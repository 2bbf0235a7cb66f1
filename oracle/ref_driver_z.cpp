/*
 * pgx_ref_driver_z — project-written driver around the reference ParGeMSLR
 * CPU solver for complex systems (the oracle; test infrastructure only,
 * never shipped).
 *
 * It follows the reference's own complex Laplacian driver
 * (ParGeMSLR TESTS/sequential/driver_laplacian_gemslrz_seq.cpp: FlexGmresClass
 * and GemslrClass over CsrMatrixClass<complexd>) and writes what the complex
 * parity tests need, in the same PGXD layout as pgx_ref_driver:
 *
 *   --dump       the post-setup GeMSLR structures (DIR/setup.bin); every
 *                value array holds complex values as interleaved {re, im}
 *                doubles, and the record "complex" = 1 says so
 *   --solve      FlexGmresClass::Solve of each right-hand side from x0 = 0
 *                (DIR/solution.bin: x<k>, rel_res_hist<k>; iterations and
 *                residuals in DIR/result.txt)
 *   --apply K    GemslrClass::Solve on K seeded complex vectors (DIR/apply.bin)
 *
 * Matrix: --lap nx ny nz shift_re shift_im ax ay az (CsrMatrixClass<complexd>
 * ::Laplacian with a complex shift: diagonal 6 - shift in 3D).  Right-hand
 * sides: --rhs FILE, a PGXD record "B" of nrhs * n complex values (row r is
 * right-hand side r) and "nrhs"; without it, b = A * ones.  Parameters:
 * --param IDX=VALUE with the reference's PARGEMSLR_IO_* indices.
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

typedef CsrMatrixClass<complexd> ZCsr;
typedef SequentialVectorClass<complexd> ZVec;
typedef GemslrClass<ZCsr, ZVec, complexd> ZGemslr;
typedef FlexGmresClass<ZCsr, ZVec, complexd> ZFgmres;
typedef IluClass<ZCsr, ZVec, complexd> ZIlu;

static_assert(sizeof(complexd) == 2 * sizeof(double), "complexd is {re, im}");

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
   /* c complex values as 2c doubles */
   void z(const std::string &n, const complexd *p, uint64_t c) { put(n, DT_F64, p, 2 * c); }
   void f64(const std::string &n, const double *p, uint64_t c) { put(n, DT_F64, p, c); }
   void scalar(const std::string &n, int v) { put(n, DT_I32, &v, 1); }
   void scalar(const std::string &n, double v) { put(n, DT_F64, &v, 1); }
};

static std::map<std::string, std::vector<char>> read_pgxd(const std::string &path)
{
   std::map<std::string, std::vector<char>> out;
   FILE *f = std::fopen(path.c_str(), "rb");
   if (!f) { std::perror(path.c_str()); std::exit(2); }
   char magic[4];
   if (std::fread(magic, 1, 4, f) != 4 || std::memcmp(magic, "PGXD", 4) != 0) std::exit(2);
   uint32_t len;
   while (std::fread(&len, 4, 1, f) == 1)
   {
      std::string name(len, '\0');
      uint8_t d;
      uint64_t count;
      if (std::fread(&name[0], 1, len, f) != len || std::fread(&d, 1, 1, f) != 1 || std::fread(&count, 8, 1, f) != 1)
         std::exit(2);
      std::vector<char> bytes((d == DT_I32 ? 4 : 8) * count);
      if (count && std::fread(bytes.data(), 1, bytes.size(), f) != bytes.size()) std::exit(2);
      out[name] = std::move(bytes);
   }
   std::fclose(f);
   return out;
}

/* CSR (CSC transposed) as name.i/.j/.a (complex values) plus the shape */
static void put_csr(Writer &w, const std::string &name, ZCsr &A)
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
      w.z(name + ".a", A.GetData(), nnz);
      return;
   }
   const int *cp = A.GetI(), *ri = A.GetJ();
   const complexd *va = A.GetData();
   std::vector<int> ip(nr + 1, 0), jp(nnz);
   std::vector<complexd> ap(nnz);
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
   w.z(name + ".a", ap.data(), ap.size());
}

static void put_dense(Writer &w, const std::string &name, DenseMatrixClass<complexd> &M)
{
   int nr = M.GetNumRowsLocal(), nc = M.GetNumColsLocal();
   int shape[2] = {nr, nc};
   w.i32(name + ".shape", shape, 2);
   std::vector<complexd> packed((size_t)nr * nc);
   if (nr * (size_t)nc > 0)
   {
      int ld = M.GetLeadingDimension();
      const complexd *d = M.GetData();
      for (int c = 0; c < nc; c++)
         for (int r = 0; r < nr; r++) packed[(size_t)c * nr + r] = d[(size_t)c * ld + r];
   }
   w.z(name, packed.data(), packed.size()); /* column-major, ld = rows */
}

static void put_ivec(Writer &w, const std::string &name, IntVectorClass<int> &v)
{
   w.i32(name, v.GetData(), (uint64_t)std::max(0, v.GetLengthLocal()));
}

static void dump_setup(const std::string &path, ZGemslr &P, ZCsr &A)
{
   Writer w(path);
   int nlev = P._nlev_used;
   w.scalar("complex", 1);
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
      GemslrLevelClass<ZCsr, ZVec, complexd> &ls = P._levs_v[l];
      std::string pre = "L" + std::to_string(l) + ".";
      w.scalar(pre + "ncomp", ls._ncomps);
      put_ivec(w, pre + "dom_ptr", P._dom_ptr_v2[l]);
      for (int c = 0; c < ls._ncomps; c++)
      {
         std::string pc = pre + "B" + std::to_string(c) + ".";
         ZIlu *ilu = (ZIlu *)ls._B_solver[c];
         put_csr(w, pc + "A", ls._B_mat_v[c]);
         put_csr(w, pc + "L", ilu->_L);
         put_csr(w, pc + "U", ilu->_U);
         w.z(pc + "D", ilu->_D.GetData(), (uint64_t)std::max(0, ilu->_D.GetLengthLocal()));
         put_ivec(w, pc + "rperm", ilu->_row_perm_vec);
         put_ivec(w, pc + "cperm", ilu->_col_perm_vec);
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
   std::fprintf(stderr,
      "usage: pgx_ref_driver_z --out DIR --lap nx ny nz shift_re shift_im ax ay az\n"
      "       [--rhs FILE] [--param IDX=VAL]... [--dump] [--solve] [--apply K] [--threads T]\n");
   std::exit(2);
}

int main(int argc, char **argv)
{
   std::string out, rhs_file;
   bool do_dump = false, do_solve = false, have_lap = false;
   int nx = 0, ny = 0, nz = 0, apply_k = 0, threads = 1;
   double sre = 0, sim = 0, ax = 0, ay = 0, az = 0;
   std::vector<std::pair<int, double>> overrides;
   for (int i = 1; i < argc; i++)
   {
      std::string a = argv[i];
      auto need = [&](int k) { if (i + k >= argc) usage(); };
      if (a == "--out") { need(1); out = argv[++i]; }
      else if (a == "--lap")
      {
         need(8);
         have_lap = true;
         nx = std::atoi(argv[++i]); ny = std::atoi(argv[++i]); nz = std::atoi(argv[++i]);
         sre = std::atof(argv[++i]); sim = std::atof(argv[++i]);
         ax = std::atof(argv[++i]); ay = std::atof(argv[++i]); az = std::atof(argv[++i]);
      }
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
   ZCsr A;
   A.Laplacian(nx, ny, nz, complexd(ax, 0.0), complexd(ay, 0.0), complexd(az, 0.0), complexd(sre, sim), false);
   int n = A.GetNumRowsLocal();

   /* right-hand sides */
   int nrhs = 1;
   std::vector<complexd> B;
   if (!rhs_file.empty())
   {
      auto rec = read_pgxd(rhs_file);
      nrhs = *(const int *)rec.at("nrhs").data();
      const std::vector<char> &bb = rec.at("B");
      if (bb.size() != sizeof(complexd) * (size_t)n * nrhs) usage();
      B.resize((size_t)n * nrhs);
      std::memcpy(B.data(), bb.data(), bb.size());
   }
   else
   {
      ZVec ones, b1;
      ones.Setup(n, kMemoryHost, false);
      b1.Setup(n, kMemoryHost, false);
      ones.Fill(complexd(1.0, 0.0));
      b1.Fill(complexd(0.0, 0.0));
      A.MatVec('N', complexd(1.0, 0.0), ones, complexd(0.0, 0.0), b1);
      B.assign(b1.GetData(), b1.GetData() + n);
   }

   ZVec x, b;
   x.Setup(n, kMemoryHost, false);
   b.Setup(n, kMemoryHost, false);
   std::memcpy(b.GetData(), B.data(), sizeof(complexd) * n);
   x.Fill(complexd(0.0, 0.0));
   {
      Writer w(out + "/problem.bin");
      w.scalar("complex", 1);
      put_csr(w, "A", A);
      w.z("B", B.data(), B.size());
      w.scalar("nrhs", nrhs);
   }

   ZFgmres solver;
   ZGemslr precond;
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
   std::fprintf(res, "n=%d\nnnz=%ld\nsetup_s=%.9g\nthreads=%d\nnlev=%d\nnrhs=%d\n", n, A.GetNumNonzeros(), t_setup,
                threads, precond._nlev_used, nrhs);

   if (apply_k > 0)
   {
      std::mt19937_64 gen(20240501ULL);
      std::uniform_real_distribution<double> U(-1.0, 1.0);
      std::vector<complexd> vin((size_t)apply_k * n), vout((size_t)apply_k * n);
      ZVec vi, vo;
      vi.Setup(n, kMemoryHost, false);
      vo.Setup(n, kMemoryHost, false);
      for (int k = 0; k < apply_k; k++)
      {
         for (int i = 0; i < n; i++)
         {
            const double re = U(gen);
            vin[(size_t)k * n + i] = complexd(re, U(gen));
         }
         std::memcpy(vi.GetData(), &vin[(size_t)k * n], sizeof(complexd) * n);
         precond.Solve(vo, vi);
         std::memcpy(&vout[(size_t)k * n], vo.GetData(), sizeof(complexd) * n);
      }
      Writer w(out + "/apply.bin");
      w.z("in", vin.data(), vin.size());
      w.z("out", vout.data(), vout.size());
      w.scalar("k", apply_k);
   }

   if (do_solve)
   {
      Writer w(out + "/solution.bin");
      std::string iters, rels, trues, times;
      for (int r = 0; r < nrhs; r++)
      {
         std::memcpy(b.GetData(), &B[(size_t)r * n], sizeof(complexd) * n);
         x.Fill(complexd(0.0, 0.0));
         double ts = now_s();
         solver.Solve(x, b);
         double dt = now_s() - ts;
         ZVec rv;
         rv.Setup(n, kMemoryHost, false);
         std::memcpy(rv.GetData(), b.GetData(), sizeof(complexd) * n);
         A.MatVec('N', complexd(-1.0, 0.0), x, complexd(1.0, 0.0), rv);
         double nr = 0.0, nb = 0.0;
         rv.Norm2(nr);
         b.Norm2(nb);
         char buf[96];
         std::snprintf(buf, sizeof(buf), "%s%d", r ? "," : "", solver.GetNumberIterations());
         iters += buf;
         std::snprintf(buf, sizeof(buf), "%s%.17g", r ? "," : "", (double)solver.GetFinalRelativeResidual());
         rels += buf;
         std::snprintf(buf, sizeof(buf), "%s%.17g", r ? "," : "", nr / nb);
         trues += buf;
         std::snprintf(buf, sizeof(buf), "%s%.9g", r ? "," : "", dt);
         times += buf;
         w.z("x" + std::to_string(r), x.GetData(), n);
         SequentialVectorClass<double> &hist = solver.GetRelativeResidual();
         w.f64("rel_res_hist" + std::to_string(r), hist.GetData(), (uint64_t)std::max(0, hist.GetLengthLocal()));
      }
      std::fprintf(res, "iters=%s\nrel_res=%s\ntrue_rel_res=%s\nsolve_times=%s\n", iters.c_str(), rels.c_str(),
                   trues.c_str(), times.c_str());
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
