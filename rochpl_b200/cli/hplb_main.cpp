// hplb: the HPL run driver at P = Q = 1 over the C ABI (include/hplb.h) --
// the native counterpart of rocHPL's xhpl (src/HPL_pddriver.cpp,
// src/HPL_pdinfo.cpp, src/HPL_pdtest.cpp) for the single-process solve.
//
//   hplb [-N n] [-NB nb] [-P p] [-Q q] [-p p] [-q q] [-f frac] [-it k] [-i HPL.dat]
//        [--progress] [--list] [--device d]
//
// Input: rocHPL's command-line flags (src/HPL_pdinfo.cpp:251-385; the
// command-line run fixes PFACT = R, NBMIN = 32, NDIV = 2, RFACT = R, DEPTH = 1,
// column-major process mapping, the 1-ring broadcast) or an HPL.dat with the
// reference's line layout, rejections and messages (src/HPL_pdinfo.cpp:590-1030).
// Run: the sweep in the reference's loop order (grids, N, NB, DEPTH, BCAST,
// RFACT, PFACT, NBMIN, NDIV; src/HPL_pddriver.cpp:120-212); per test a warm-up
// solve of at most 2 NB + 1 columns (the role of src/HPL_pdwarmup.cpp), then
// `-it` repetitions of generate, timed hplb_pdgesv, residual check.  Grids
// other than 1 x 1 are counted as skipped tests (the Python driver,
// rochpl_b200/driver.py under torchrun, runs P x Q grids).  Output: the reference's lines
// (src/HPL_pdtest.cpp:144-213 and :439-475, src/HPL_pddriver.cpp:226-283) and,
// with --progress, the per-step rows of src/pgesv/HPL_pdgesv.cpp:155-341.
// --list prints the sweep without touching a GPU.
//
// Exit status: 0 all checks passed, 1 bad input, 2 a residual check failed,
// 3 a library or CUDA error.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "hplb.h"

namespace {

constexpr int kMaxParam = 20;    // include/hpl_ptest.hpp:56
constexpr uint64_t kSeed = 100;  // include/hpl_ptest.hpp:57

struct InputError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct Config {
  std::vector<int> ns{45312}, nbs{384}, ps{1}, qs{1};
  double           thrsh = 16.0;
  std::vector<int> pfacts{2}, nbmins{32}, ndivs{2}, rfacts{2}, bcasts{0}, depths{1};
  int              l1notran = 0;
  int              pmap     = 1;  // 0 row-major, 1 column-major
  int              iters    = 1;
  double           frac     = 0.3;
  std::string      outfile;       // empty: stdout
};

// 0 left, 1 Crout, 2 right; anything else right (src/HPL_pdinfo.cpp:840-862).
int fact(int j) { return (j == 0 || j == 1 || j == 2) ? j : 2; }

bool parse_int(const std::string& s, int* v) {
  if(s.empty()) return false;
  char*      end = nullptr;
  const long x   = std::strtol(s.c_str(), &end, 10);
  if(*end != '\0') return false;
  *v = (int)x;
  return true;
}

std::vector<std::string> tokens(const std::string& line) {
  std::istringstream       in(line);
  std::vector<std::string> t;
  std::string              w;
  while(in >> w) t.push_back(w);
  return t;
}

// An HPL.dat: two free-text lines, then one value (or a list) per line.
struct DatReader {
  std::vector<std::string> lines;
  size_t                   pos = 2;

  explicit DatReader(const std::string& text) {
    std::istringstream in(text);
    std::string        l;
    while(std::getline(in, l)) lines.push_back(l);
  }
  const std::string& next() {
    if(pos >= lines.size()) throw InputError("Illegal input in file HPL.dat. Exiting ...");
    return lines[pos++];
  }
  int first_int() {
    const auto t = tokens(next());
    int        v = 0;
    return (!t.empty() && parse_int(t[0], &v)) ? v : 0;
  }
  std::vector<int> ints(int k) {
    auto             t = tokens(next());
    std::vector<int> v((size_t)k, 0);
    for(int i = 0; i < k && i < (int)t.size(); ++i)
      if(!parse_int(t[(size_t)i], &v[(size_t)i])) v[(size_t)i] = 0;
    return v;
  }
  int count(const char* what) {
    const int k = first_int();
    if(k < 1 || k > kMaxParam) {
      char m[160];
      std::snprintf(m, sizeof m, "Number of values of %s is less than 1 or greater than %d",
                    what, kMaxParam);
      throw InputError(m);
    }
    return k;
  }
};

bool any_below(const std::vector<int>& v, int lo) {
  for(int x : v)
    if(x < lo) return true;
  return false;
}

Config parse_dat(const std::string& text) {
  DatReader r(text);
  Config    c;
  const auto out = tokens(r.next());
  const int  dev = r.first_int();  // 6 stdout, 7 stderr, else the file named above
  c.ns = r.ints(r.count("N"));
  if(any_below(c.ns, 0)) throw InputError("Value of N less than 0");
  c.nbs = r.ints(r.count("NB"));
  if(any_below(c.nbs, 1)) throw InputError("Value of NB less than 1");
  c.pmap = r.first_int() == 1 ? 1 : 0;
  const int kg = r.count("grids");
  c.ps = r.ints(kg);
  c.qs = r.ints(kg);
  if(any_below(c.ps, 1)) throw InputError("Value of P less than 1");
  if(any_below(c.qs, 1)) throw InputError("Value of Q less than 1");
  {
    const auto t = tokens(r.next());
    c.thrsh      = t.empty() ? 16.0 : std::atof(t[0].c_str());
  }
  c.pfacts = r.ints(r.count("PFACT"));
  for(int& v : c.pfacts) v = fact(v);
  c.nbmins = r.ints(r.count("NBMIN"));
  if(any_below(c.nbmins, 1)) throw InputError("Value of NBMIN less than 1");
  c.ndivs = r.ints(r.count("NDIV"));
  if(any_below(c.ndivs, 2)) throw InputError("Value of NDIV less than 2");
  c.rfacts = r.ints(r.count("RFACT"));
  for(int& v : c.rfacts) v = fact(v);
  c.bcasts = r.ints(r.count("BCAST"));
  for(int& v : c.bcasts) v = (v >= 0 && v <= 4) ? v : 5;
  c.depths = r.ints(r.count("DEPTH"));
  if(any_below(c.depths, 0)) throw InputError("Value of DEPTH less than 0");
  for(int v : c.depths)
    if(v != 1) throw InputError("Value of DEPTH must be 1");
  if(r.first_int() != 1) throw InputError("Value of SWAP must be 1");
  r.next();  // swapping threshold
  const int l1 = r.first_int();
  c.l1notran   = (l1 == 0 || l1 == 1) ? l1 : 0;
  const int u  = r.first_int();
  if(u == 1) throw InputError("U  in no-transposed form unsupported");
  const int eq = r.first_int();
  if(eq != 0) throw InputError("Equilibration currently unsupported");
  if(dev != 6 && dev != 7 && !out.empty()) c.outfile = out[0];
  return c;
}

// The command line; *input receives the -i file, if any.
Config parse_cli(const std::vector<std::string>& args, std::string* input) {
  Config c;
  auto   val = [&](size_t i) -> std::string {
    return i + 1 < args.size() ? args[i + 1] : std::string();
  };
  auto num = [&](size_t i, const char* msg, int lo) {
    int v = 0;
    if(!parse_int(val(i), &v) || v < lo) throw InputError(msg);
    return v;
  };
  for(size_t i = 0; i < args.size(); ++i) {
    const std::string& a = args[i];
    if(a == "-P" || a == "--ranksP") {
      c.ps = {num(i, "Illegal value for P. Exiting ...", 1)};
      ++i;
    } else if(a == "-Q" || a == "--ranksQ") {
      c.qs = {num(i, "Illegal value for Q. Exiting ...", 1)};
      ++i;
    } else if(a == "-p" || a == "-q") {
      ++i;  // node-local grid: one process here
    } else if(a == "-N" || a == "--sizeN") {
      c.ns = {num(i, "Illegal value for N. Exiting ...", 1)};
      ++i;
    } else if(a == "-NB" || a == "--sizeNB") {
      c.nbs = {num(i, "Illegal value for NB. Exiting ...", 1)};
      ++i;
    } else if(a == "-f" || a == "--frac") {
      c.frac = std::atof(val(i).c_str());
      ++i;
    } else if(a == "-it") {
      c.iters = std::atoi(val(i).c_str());
      ++i;
    } else if(a == "-i" || a == "--input") {
      *input = val(i);
      ++i;
    }
  }
  return c;
}

// ---- output (the reference's lines) ----

const char* kRuleEq   = "================================================================================";
const char* kRuleDash = "--------------------------------------------------------------------------------";

struct Test {
  int       n, p, q, bcast;
  hplb_algo algo;
};

char fact_char(int f) { return f == 0 ? 'L' : (f == 1 ? 'C' : 'R'); }

// W, grid order, depth, broadcast, RFACT, NDIV, PFACT, NBMIN (src/HPL_pdtest.cpp:192-206).
std::string tv_code(const Test& t, int pmap) {
  char b[64];
  std::snprintf(b, sizeof b, "W%c%1d%c%c%1d%c%1d", pmap == 1 ? 'C' : 'R', t.algo.depth,
                (char)('0' + t.bcast), fact_char(t.algo.rfact), t.algo.ndiv,
                fact_char(t.algo.pfact), t.algo.nbmin);
  return b;
}

void table_header(FILE* f) {
  std::fprintf(f, "%s\n", kRuleEq);
  std::fprintf(f, "T/V                N    NB     P     Q               Time                 Gflops\n");
  std::fprintf(f, "%s\n", kRuleDash);
}

std::string ctime_str(std::time_t t) {
  char b[64];
  std::strftime(b, sizeof b, "%a %b %e %H:%M:%S %Y", std::localtime(&t));
  return b;
}

void result_lines(FILE* f, const Test& t, int pmap, double wtime, std::time_t t0, std::time_t t1) {
  if(wtime <= 0.0) return;
  const double n      = (double)t.n;
  const double gflops = (n / 1.0e9) * (n / wtime) * ((2.0 / 3.0) * n + 1.5);
  std::fprintf(f, "%s%12d %5d %5d %5d %18.2f     %18.3e\n", tv_code(t, pmap).c_str(), t.n,
               t.algo.nb, t.p, t.q, wtime, gflops);
  std::fprintf(f, "HPL_pdgesv() start time %s\n\n", ctime_str(t0).c_str());
  std::fprintf(f, "HPL_pdgesv() end time   %s\n\n", ctime_str(t1).c_str());
}

void residual_lines(FILE* f, const hplb_resid& r, double thrsh) {
  const bool ok = r.resid < thrsh;
  std::fprintf(f, "%s\n", kRuleDash);
  std::fprintf(f, "%s%16.7f%s%s\n", "||Ax-b||_oo/(eps*(||A||_oo*||x||_oo+||b||_oo)*N)= ", r.resid,
               " ...... ", ok ? "PASSED" : "FAILED");
  if(ok) return;
  const std::pair<const char*, double> rows[] = {
      {"||Ax-b||_oo  . . . . . . . . . . . . . . . . . = ", r.rnorm_inf},
      {"||A||_oo . . . . . . . . . . . . . . . . . . . = ", r.anorm_inf},
      {"||A||_1  . . . . . . . . . . . . . . . . . . . = ", r.anorm_1},
      {"||x||_oo . . . . . . . . . . . . . . . . . . . = ", r.xnorm_inf},
      {"||x||_1  . . . . . . . . . . . . . . . . . . . = ", r.xnorm_1},
      {"||b||_oo . . . . . . . . . . . . . . . . . . . = ", r.bnorm_inf}};
  for(const auto& row : rows) std::fprintf(f, "%s%18.6f\n", row.first, row.second);
}

void summary_lines(FILE* f, int kpass, int kfail, int kskip, double thrsh) {
  std::fprintf(f, "%s\n", kRuleEq);
  std::fprintf(f, "\n%s %6d %s\n", "Finished", kpass + kfail + kskip,
               "tests with the following results:");
  if(thrsh > 0.0) {
    std::fprintf(f, "         %6d %s\n", kpass, "tests completed and passed residual checks,");
    std::fprintf(f, "         %6d %s\n", kfail, "tests completed and failed residual checks,");
  } else {
    std::fprintf(f, "         %6d %s\n", kpass, "tests completed without checking,");
  }
  std::fprintf(f, "         %6d %s\n", kskip, "tests skipped because of illegal input values.");
  std::fprintf(f, "%s\n", kRuleDash);
  std::fprintf(f, "\nEnd of Tests.\n");
  std::fprintf(f, "%s\n", kRuleEq);
}

// Per-step rows: percent done, the step's first column, its time, and the
// rate so far counted as the reference does, (2/3 (N^3 - r^3) - 1/2 (N^2 - r^2)
// - 1/6 (N - r)) / t with r the columns still to factor.
void progress_lines(FILE* f, int n, const std::vector<int>& col, const std::vector<double>& ms) {
  std::fprintf(f, "---------------------------------------------------\n");
  std::fprintf(f, "   %%   | Column    | Step Time (s) | Overall GFLOPS\n");
  std::fprintf(f, "       |           |               |               \n");
  std::fprintf(f, "---------------------------------------------------\n");
  double total = 0.0;
  for(size_t i = 0; i < col.size(); ++i) {
    total += ms[i] * 1e-3;
    const double N = (double)n;
    const double r = (double)(n - (i + 1 < col.size() ? col[i + 1] : n));
    const double done = 2.0 / 3.0 * (N * N * N - r * r * r) - 0.5 * (N * N - r * r) - (N - r) / 6.0;
    std::fprintf(f, "%5.1f%% | %09d | ", n ? col[i] * 100.0 / n : 0.0, col[i]);
    std::fprintf(f, "   %9.7f  |", ms[i] * 1e-3);
    std::fprintf(f, "    %9.3e   \n", done / (total > 0.0 ? total : 1e-6) / 1e9);
  }
}

// The sweep in the reference's loop order.
std::vector<Test> sweep(const Config& c) {
  std::vector<Test> v;
  const size_t      ng = std::min(c.ps.size(), c.qs.size());
  for(size_t g = 0; g < ng; ++g)
    for(int n : c.ns)
      for(int nb : c.nbs)
        for(int depth : c.depths)
          for(int bc : c.bcasts)
            for(int rf : c.rfacts)
              for(int pf : c.pfacts)
                for(int nbm : c.nbmins)
                  for(int nd : c.ndivs)
                    v.push_back(Test{n, c.ps[g], c.qs[g], bc,
                                     hplb_algo{nb, nbm, nd, pf, rf, depth, c.l1notran}});
  return v;
}

// Grids beyond one process and values the library does not take.
bool skipped(const Test& t) {
  return t.p * t.q != 1 || t.algo.nbmin > 128 || t.algo.nb > 2048 || t.algo.depth != 1;
}

// ---- the run ----

struct LibError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void check(hplb_ctx* ctx, hplb_status s, const char* what) {
  if(s == HPLB_OK || s == HPLB_ERR_SINGULAR) return;
  std::string m = std::string(what) + ": " + hplb_status_string(s);
  if(ctx && hplb_last_error(ctx)) m += std::string(" (") + hplb_last_error(ctx) + ")";
  throw LibError(m);
}

void check_cuda(cudaError_t e, const char* what) {
  if(e != cudaSuccess) throw LibError(std::string(what) + ": " + cudaGetErrorString(e));
}

// Device [A|b] and x, reallocated when N changes.
struct Buffers {
  int     n  = -1;
  int64_t ld = 0;
  double* A  = nullptr;
  double* X  = nullptr;

  void ensure(int nn) {
    if(nn == n) return;
    release();
    ld = hplb_default_ld(nn);
    check_cuda(cudaMalloc(&A, (size_t)ld * (size_t)(nn + 1) * sizeof(double)), "cudaMalloc [A|b]");
    check_cuda(cudaMalloc(&X, (size_t)(nn > 1 ? nn : 1) * sizeof(double)), "cudaMalloc x");
    n = nn;
  }
  void release() {
    if(A) cudaFree(A);
    if(X) cudaFree(X);
    A = X = nullptr;
    n     = -1;
  }
  ~Buffers() { release(); }
};

int run(const Config& c, FILE* out, int device, bool progress) {
  hplb_status st  = HPLB_OK;
  hplb_ctx*   ctx = hplb_create(device, &st);
  if(!ctx) throw LibError(std::string("hplb_create: ") + hplb_status_string(st));
  Buffers buf;
  int     kpass = 0, kfail = 0, kskip = 0;
  bool    first = true;
  for(const Test& t : sweep(c)) {
    if(skipped(t)) {
      ++kskip;
      continue;
    }
    {  // warm-up: every kernel of the solve once, in buffers of its own
      Buffers w;
      const int m = std::min(t.n, 2 * t.algo.nb + 1);
      w.ensure(m);
      check(ctx, hplb_matgen(ctx, m, m + 1, t.algo.nb, kSeed, w.A, w.ld), "hplb_matgen");
      check(ctx, hplb_pdgesv(ctx, &t.algo, m, w.A, w.ld, w.X, nullptr, nullptr), "hplb_pdgesv");
    }
    buf.ensure(t.n);
    for(int it = 0; it < std::max(c.iters, 1); ++it) {
      check(ctx, hplb_matgen(ctx, t.n, t.n + 1, t.algo.nb, kSeed, buf.A, buf.ld), "hplb_matgen");
      check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
      const std::time_t t0 = std::time(nullptr);
      const auto        c0 = std::chrono::steady_clock::now();
      int               info = 0;
      check(ctx, hplb_pdgesv(ctx, &t.algo, t.n, buf.A, buf.ld, buf.X, nullptr, &info),
            "hplb_pdgesv");
      const double wtime =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
      const std::time_t t1 = std::time(nullptr);
      hplb_resid        r{};
      check(ctx, hplb_residual_lcg(ctx, t.n, kSeed, buf.X, &r), "hplb_residual_lcg");
      if(first) {  // before every checked result; once without checking
        table_header(out);
        if(c.thrsh <= 0.0) first = false;
      }
      if(progress) {
        int cnt = 0;
        check(ctx, hplb_last_steps(ctx, 0, &cnt, nullptr, nullptr), "hplb_last_steps");
        std::vector<int>    col((size_t)cnt);
        std::vector<double> ms((size_t)cnt);
        check(ctx, hplb_last_steps(ctx, cnt, &cnt, col.data(), ms.data()), "hplb_last_steps");
        progress_lines(out, t.n, col, ms);
      }
      result_lines(out, t, c.pmap, wtime, t0, t1);
      if(c.thrsh > 0.0) {
        (r.resid < c.thrsh ? kpass : kfail)++;
        residual_lines(out, r, c.thrsh);
      } else {
        ++kpass;
      }
      std::fflush(out);
    }
  }
  summary_lines(out, kpass, kfail, kskip, c.thrsh);
  std::fflush(out);
  buf.release();
  hplb_destroy(ctx);
  return kfail ? 2 : 0;
}

// --list: one line per test of the sweep, no GPU.
void list(const Config& c, FILE* out) {
  for(const Test& t : sweep(c))
    std::fprintf(out, "%s %d %d %d %d %s\n", tv_code(t, c.pmap).c_str(), t.n, t.algo.nb, t.p, t.q,
                 skipped(t) ? "skip" : "run");
  std::fprintf(out, "thrsh %g iters %d outfile %s\n", c.thrsh, std::max(c.iters, 1),
               c.outfile.empty() ? "-" : c.outfile.c_str());
}

}  // namespace

const char* kUsage =
    "usage: hplb [-N n] [-NB nb] [-P p] [-Q q] [-p p] [-q q] [-f frac] [-it k] [-i HPL.dat]\n"
    "            [--progress] [--list] [--device d]\n"
    "  -N, -NB        problem size and block size (default 45312, 384)\n"
    "  -P, -Q         process grid; this single process runs 1 x 1, other grids count as\n"
    "                 skipped tests (P x Q grids: python -m rochpl_b200.driver, one process\n"
    "                 per GPU under torchrun)\n"
    "  -p, -q, -f     accepted for compatibility (node-local grid, panel fraction)\n"
    "  -it k          timed repetitions of each test (after one warm-up)\n"
    "  -i HPL.dat     read the parameter sweep from an HPL.dat\n"
    "  --progress     per-step report (percent, column, step time, overall GFLOPS)\n"
    "  --list         print the tests the sweep contains; no GPU is touched\n"
    "  --device d     CUDA device (default 0)\n"
    "exit status: 0 all passed, 1 bad input, 2 a residual check failed, 3 a library error\n";

int main(int argc, char** argv) {
  std::vector<std::string> args(argv + 1, argv + argc);
  for(const auto& a : args)
    if(a == "-h" || a == "--help") {
      std::fputs(kUsage, stdout);
      return 0;
    }
  bool                     progress = false, only_list = false;
  int                      device = 0;
  std::vector<std::string> rest;
  for(size_t i = 0; i < args.size(); ++i) {
    if(args[i] == "--progress") {
      progress = true;
    } else if(args[i] == "--list") {
      only_list = true;
    } else if(args[i] == "--device" && i + 1 < args.size()) {
      device = std::atoi(args[++i].c_str());
    } else {
      rest.push_back(args[i]);
    }
  }
  Config c;
  try {
    std::string input;
    c = parse_cli(rest, &input);
    if(!input.empty()) {
      std::ifstream f(input);
      if(!f) throw InputError("cannot open " + input);
      std::stringstream ss;
      ss << f.rdbuf();
      const int iters = c.iters;
      c               = parse_dat(ss.str());
      c.iters         = iters;  // -it applies to an HPL.dat run too
    }
  } catch(const InputError& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  if(only_list) {
    list(c, stdout);
    return 0;
  }
  FILE* out = stdout;
  if(!c.outfile.empty()) {
    out = std::fopen(c.outfile.c_str(), "w");
    if(!out) {
      std::fprintf(stderr, "cannot open %s\n", c.outfile.c_str());
      return 1;
    }
  }
  int rc = 0;
  try {
    rc = run(c, out, device, progress);
  } catch(const LibError& e) {
    std::fprintf(stderr, "%s\n", e.what());
    rc = 3;
  }
  if(out != stdout) std::fclose(out);
  return rc;
}
