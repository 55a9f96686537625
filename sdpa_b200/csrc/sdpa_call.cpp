// class SDPA (include/sdpa_call.h): the reference's public C++ API
// (sdpa_call.h:91-267, sdpa_call.cpp) on top of the host-driven CUDA solver
// (solver.h), plus the SDPA file readers and the extern "C" handle API of
// include/sdpa_b200.h.  Input staging follows the reference: inputElement
// swaps i > j to the upper triangle (sdpa_call.cpp:330-332) and
// initializeUpperTriangle sorts the staged elements; .dat-s values are kept
// as written (F0 is negated to C inside the solver, sdpa_io.cpp:511).
#include "sdpa_call.h"

#include <ctype.h>
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "ipm_control.h"
#include "sdpa_b200.h"
#include "sdpab_internal.h"
#include "solver.h"

namespace sdpab {

struct SdpaImpl {
  Params prm = default_params(0);
  int ptype = 0;
  double kappa = 12.0;  // KAPPA (sdpa_call.cpp:41)
  FILE* display = nullptr;
  FILE* fpout = nullptr;
  bool isInitPoint = false;
  int numThreads = 0;
  char xPrint[32] = "%+8.3e", XPrint[32] = "%+8.3e", YPrint[32] = "%+8.3e", infPrint[32] = "%+10.16e";
  ProblemData prob;
  InitPoint init;
  bool initialized = false;
  bool solved = false;
  Solver solver;
  std::vector<double> xvec;
  std::vector<std::vector<double>> Xres, Yres;
  double file_read_seconds = 0.0;  // readInput / readInit / readParameter
  int err = 0;
  std::string errmsg;
  void fail(int code, const std::string& msg)
  {
    if (!err) {
      err = code;
      errmsg = msg;
    }
  }
  int nb() const { return (int)prob.blockStruct.size(); }
  bool isSdp(int l) const  // 0-based file block
  {
    const int s = prob.blockStruct[l];
    const int t = (l < (int)prob.blockType.size()) ? prob.blockType[l] : 0;
    return s >= 2 && t == 0;
  }
  int blockDim(int l) const { return std::abs(prob.blockStruct[l]); }
  void ensureInit()
  {
    const int nb_ = nb();
    if ((int)init.X.size() != nb_) {
      init.X.assign(nb_, {});
      init.Y.assign(nb_, {});
    }
    for (int l = 0; l < nb_; ++l) {
      const size_t need = isSdp(l) ? (size_t)blockDim(l) * blockDim(l) : (size_t)blockDim(l);
      if (init.X[l].size() != need) init.X[l].assign(need, 0.0);
      if (init.Y[l].size() != need) init.Y[l].assign(need, 0.0);
    }
    if ((int)init.xvec.size() != prob.m) init.xvec.assign(prob.m, 0.0);
  }
};

// Adds the lifetime of the object to a seconds counter (the reference's
// ComputeTime::FileRead).
struct ReadTimer {
  double& acc;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  explicit ReadTimer(double& a) : acc(a) {}
  ~ReadTimer() { acc += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

// ----------------------------------------------------------- text scanning
// Numbers are read out of any punctuation, like the reference's
// "%*[^0-9+-]" scans (sdpa_io.cpp:33-73).
struct Scanner {
  const char* p;
  const char* end;
  bool next(double& v)
  {
    while (p < end) {
      const char c = *p;
      if (isdigit((unsigned char)c) ||
          ((c == '+' || c == '-' || c == '.') && p + 1 < end &&
           (isdigit((unsigned char)p[1]) || (p[1] == '.' && p + 2 < end && isdigit((unsigned char)p[2]))))) {
        char* e = nullptr;
        v = strtod(p, &e);
        if (e == p) { ++p; continue; }
        p = e;
        return true;
      }
      ++p;
    }
    return false;
  }
  bool nextInt(int& v)
  {
    double d;
    if (!next(d)) return false;
    v = (int)d;
    return true;
  }
};

static bool slurp(const char* path, std::string& out)
{
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  char buf[1 << 16];
  size_t r;
  out.clear();
  while ((r = fread(buf, 1, sizeof(buf), f)) > 0) out.append(buf, r);
  fclose(f);
  return true;
}

// IO::read header + data (sdpa_io.cpp:33-73, :230-606): leading lines that
// start with '"' or '*' are title/comments; then m, nBlock, block struct, c,
// and either sparse "k l i j v" lines or dense block matrices F0..Fm.
int parse_sdpa(const std::string& text, bool sparse, ProblemData& P, std::string& why)
{
  size_t pos = 0;
  while (pos < text.size()) {
    const size_t eol = text.find('\n', pos);
    const size_t e = (eol == std::string::npos) ? text.size() : eol;
    if (e > pos && (text[pos] == '"' || text[pos] == '*')) { pos = e + 1; continue; }
    if (e == pos) { pos = e + 1; continue; }
    break;
  }
  Scanner S{text.c_str() + pos, text.c_str() + text.size()};
  int m, nb;
  if (!S.nextInt(m) || !S.nextInt(nb) || m < 1 || nb < 1) { why = "bad header (m, nBlock)"; return SDPAB_EIO; }
  P = ProblemData();
  P.m = m;
  P.blockStruct.resize(nb);
  P.blockType.assign(nb, 0);
  for (int l = 0; l < nb; ++l) {
    if (!S.nextInt(P.blockStruct[l]) || P.blockStruct[l] == 0) { why = "bad block struct"; return SDPAB_EIO; }
    if (P.blockStruct[l] < 0) P.blockType[l] = 2;
  }
  P.c.resize(m);
  for (int k = 0; k < m; ++k)
    if (!S.next(P.c[k])) { why = "short c vector"; return SDPAB_EIO; }
  if (sparse) {
    double v[5];
    while (true) {
      int got = 0;
      for (; got < 5; ++got)
        if (!S.next(v[got])) break;
      if (got < 5) break;
      Entry e{(int)v[0], (int)v[1], (int)v[2], (int)v[3], v[4]};
      if (e.k < 0 || e.k > m || e.l < 1 || e.l > nb) { why = "entry index out of range"; return SDPAB_EIO; }
      if (P.blockStruct[e.l - 1] < 0 && e.i != e.j) { why = "LP entry with i != j"; return SDPAB_EIO; }
      P.entries.push_back(e);
    }
  } else {
    for (int k = 0; k <= m; ++k) {
      for (int l = 0; l < nb; ++l) {
        const int s = P.blockStruct[l];
        if (s > 0) {
          for (int i = 0; i < s; ++i)
            for (int j = 0; j < s; ++j) {
              double v;
              if (!S.next(v)) { why = "short dense data"; return SDPAB_EIO; }
              if (v != 0.0 && i <= j) P.entries.push_back({k, l + 1, i + 1, j + 1, v});
            }
        } else {
          for (int i = 0; i < -s; ++i) {
            double v;
            if (!S.next(v)) { why = "short dense data"; return SDPAB_EIO; }
            if (v != 0.0) P.entries.push_back({k, l + 1, i + 1, i + 1, v});
          }
        }
      }
    }
  }
  return SDPAB_OK;
}

// Initial point file (IO::read of the init point, sdpa_io.cpp:75-227): the
// x vector, then "1 l i j v" (user X) / "2 l i j v" (user Y) lines (sparse)
// or the dense X and Y block matrices.
int parse_init(const std::string& text, bool sparse, SdpaImpl& I, std::string& why)
{
  I.ensureInit();
  Scanner S{text.c_str(), text.c_str() + text.size()};
  for (int k = 0; k < I.prob.m; ++k)
    if (!S.next(I.init.xvec[k])) { why = "short x vector"; return SDPAB_EIO; }
  auto put = [&](int target, int l, int i, int j, double v) -> bool {
    if (l < 1 || l > I.nb()) return false;
    std::vector<double>& M = (target == 1) ? I.init.X[l - 1] : I.init.Y[l - 1];
    const int n = I.blockDim(l - 1);
    if (i < 1 || j < 1 || i > n || j > n) return false;
    if (I.isSdp(l - 1)) {
      M[(i - 1) + (size_t)n * (j - 1)] = v;
      M[(j - 1) + (size_t)n * (i - 1)] = v;
    } else {
      if (i != j) return false;
      M[i - 1] = v;
    }
    return true;
  };
  if (sparse) {
    double v[5];
    while (true) {
      int got = 0;
      for (; got < 5; ++got)
        if (!S.next(v[got])) break;
      if (got < 5) break;
      if (v[4] == 0.0) continue;
      if (!put((int)v[0], (int)v[1], (int)v[2], (int)v[3], v[4])) { why = "bad init entry"; return SDPAB_EIO; }
    }
  } else {
    for (int target = 1; target <= 2; ++target)
      for (int l = 1; l <= I.nb(); ++l) {
        const int n = I.blockDim(l - 1);
        if (I.isSdp(l - 1)) {
          for (int i = 1; i <= n; ++i)
            for (int j = 1; j <= n; ++j) {
              double x;
              if (!S.next(x)) { why = "short dense init"; return SDPAB_EIO; }
              if (i <= j) put(target, l, i, j, x);
            }
        } else {
          for (int i = 1; i <= n; ++i) {
            double x;
            if (!S.next(x)) { why = "short dense init"; return SDPAB_EIO; }
            put(target, l, i, i, x);
          }
        }
      }
  }
  return SDPAB_OK;
}

}  // namespace sdpab

namespace sdpab {
static bool noprint(const char* fmt) { return strcmp(fmt, "NOPRINT") == 0; }

// Vector::display (sdpa_struct.cpp:82-123): "{v1,v2,...}"
static void print_vector(FILE* fp, const double* v, size_t n, const char* fmt)
{
  if (noprint(fmt)) { fprintf(fp, "NOPRINT\n"); return; }
  fprintf(fp, "{");
  for (size_t k = 0; k < n; ++k) {
    fprintf(fp, fmt, v[k]);
    fprintf(fp, (k + 1 < n) ? "," : "}\n");
  }
  if (n == 0) fprintf(fp, "  }\n");
}

// DenseMatrix::display (sdpa_struct.cpp:795-833): one brace group per row,
// the rows themselves in a brace group when n > 1.
static void print_dense(FILE* fp, const double* M, int n, const char* fmt)
{
  fprintf(fp, "{");
  for (int i = 0; i < n - 1; ++i) {
    fprintf(fp, i == 0 ? " {" : "  {");
    for (int j = 0; j < n; ++j) {
      fprintf(fp, fmt, M[i + (size_t)n * j]);
      if (j + 1 < n) fprintf(fp, ",");
    }
    fprintf(fp, " },\n");
  }
  if (n > 1) fprintf(fp, "  {");
  for (int j = 0; j < n; ++j) {
    fprintf(fp, fmt, M[(n - 1) + (size_t)n * j]);
    if (j + 1 < n) fprintf(fp, ",");
  }
  fprintf(fp, " }");
  fprintf(fp, n > 1 ? "   }\n" : "\n");
}

// DenseLinearSpace::displaySolution (sdpa_struct.cpp:1624-1661): the blocks in
// file order, SDP blocks as dense matrices, LP blocks as vectors.
static void print_blocks(SdpaImpl& I, std::vector<std::vector<double>>& M, const char* fmt, FILE* fp)
{
  if (noprint(fmt)) { fprintf(fp, "NOPRINT\n"); return; }
  fprintf(fp, "{\n");
  for (int l = 0; l < I.nb(); ++l) {
    const int n = I.blockDim(l);
    if (I.isSdp(l)) print_dense(fp, M[l].data(), n, fmt);
    else print_vector(fp, M[l].data(), (size_t)n, fmt);
  }
  fprintf(fp, "}\n");
}

// Parameter::display (sdpa_parts.cpp:266-310)
static void print_params(FILE* fp, const Params& p, const SdpaImpl& I, const char* fmt)
{
  if (noprint(fmt)) { fprintf(fp, "NOPRINT\n"); return; }
  fprintf(fp, "** Parameters **\n");
  fprintf(fp, "maxIteration = %d\n", p.maxIteration);
  const char* names[] = {"epsilonStar  = ", "lambdaStar   = ", "omegaStar    = ", "lowerBound   = ",
                         "upperBound   = ", "betaStar     = ", "betaBar      = ", "gammaStar    = ",
                         "epsilonDash  = "};
  const double vals[] = {p.epsilonStar, p.lambdaStar, p.omegaStar, p.lowerBound, p.upperBound,
                         p.betaStar,    p.betaBar,    p.gammaStar, p.epsilonDash};
  for (int q = 0; q < 9; ++q) {
    fprintf(fp, "%s", names[q]);
    fprintf(fp, fmt, vals[q]);
    fprintf(fp, "\n");
  }
  fprintf(fp, "xPrint       = %s \n", I.xPrint);
  fprintf(fp, "XPrint       = %s \n", I.XPrint);
  fprintf(fp, "YPrint       = %s \n", I.YPrint);
  fprintf(fp, "infPrint     = %s \n", I.infPrint);
}

// ComputeTime::display (sdpa_parts.cpp:78-164): the reference's table of
// rows; this solver times its own phases on the device (rMat+gVec, bMat,
// Cholesky, solves, dX/dZ, step length, update of X/Z and their inverses,
// residuals), which fill the matching rows; rows with no counterpart
// print 0.
static void print_times(FILE* fp, const SolveStats& s, double file_read)
{
  double ph[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (size_t q = 0; q < s.phase_seconds.size() && q < 8; ++q) ph[q] = s.phase_seconds[q];
  const double main_loop = s.solve_seconds;
  const double total = s.solve_seconds + file_read;
  const double div = (main_loop > 0.0) ? main_loop : 1.0;
  struct Row { const char* name; double v; };
  const double eig = ph[5];
  const Row rows[] = {
      {" Predictor time  =       ", 0.0}, {" Corrector time  =       ", 0.0},
      {" Make bMat time  =       ", ph[1]}, {" Make bDia time  =       ", 0.0},
      {" Make bF1  time  =       ", 0.0}, {" Make bF2  time  =       ", 0.0},
      {" Make bF3  time  =       ", 0.0}, {" Make bPRE time  =       ", 0.0},
      {" Make rMat time  =       ", ph[0]}, {" Make gVec Mul   =       ", 0.0},
      {" Make gVec time  =       ", 0.0}, {" Cholesky bMat   =       ", ph[2]},
      {" Ste Pre time    =       ", 0.0}, {" Ste Cor time    =       ", ph[5]},
      {" solve           =       ", ph[3]}, {" sumDz           =       ", 0.0},
      {" makedX          =       ", ph[4]}, {" symmetriseDx    =       ", 0.0},
      {" makedXdZ        =       ", 0.0}, {" xMatTime        =       ", 0.0},
      {" zMatTime        =       ", 0.0}, {" invzMatTime     =       ", 0.0},
      {" xMatzMatTime    =       ", ph[6]}, {" EigxMatTime     =       ", 0.0},
      {" EigzMatTime     =       ", 0.0}, {" EigxMatzMatTime =       ", 0.0},
      {" updateRes       =       ", ph[7]}, {" EigTime         =       ", eig},
      {" sub_total_bMat  =       ", main_loop - ph[1]}, {" Main Loop       =       ", main_loop},
      {" File Check      =       ", 0.0}, {" File Change     =       ", 0.0},
      {" File Read       =       ", file_read}, {" Total           =       ", total}};
  fprintf(fp, "\n");
  fprintf(fp, "                         Time(sec) ");
  fprintf(fp, " Ratio(%% : MainLoop) \n");
  for (const Row& r : rows) fprintf(fp, "%s%f,  %f\n", r.name, r.v, r.v / div * 100.0);
  fprintf(fp, "\n");
}

// IO::printOneIteration (sdpa_io.cpp:622-658) in the reference's reversed
// primal/dual form; r = mu, thetaP, thetaD, objP, objD, alphaP, alphaD, beta
// of the internal problem.
static void print_iteration(FILE* fp, int it, const double* r)
{
  fprintf(fp, "%2d %4.1e %4.1e %4.1e %+7.2e %+7.2e %4.1e %4.1e %4.2e\n", it, r[0], r[2], r[1], -r[4], -r[3],
          r[6], r[5], r[7]);
}
}  // namespace sdpab

using sdpab::SdpaImpl;

// SDPA_INT may be int64_t (the ILP64 build of this file): sizes and indices
// are checked against the int range the solver stores them in.
template <class T>
static bool in_int(T v)
{
  return (long long)v >= (long long)INT_MIN && (long long)v <= (long long)INT_MAX;
}

SDPA::SDPA() : impl_(new SdpaImpl()) {}
SDPA::~SDPA() { delete impl_; }

void SDPA::setParameterType(ParameterType type)
{
  impl_->ptype = (int)type;
  impl_->prm = sdpab::default_params((int)type);
}
void SDPA::setParameterMaxIteration(SDPA_INT v)
{
  if (!in_int(v)) return impl_->fail(SDPAB_EINVAL, "setParameterMaxIteration: value out of range");
  impl_->prm.maxIteration = (int)v;
}
void SDPA::setParameterEpsilonStar(double v) { impl_->prm.epsilonStar = v; }
void SDPA::setParameterLambdaStar(double v) { impl_->prm.lambdaStar = v; }
void SDPA::setParameterOmegaStar(double v) { impl_->prm.omegaStar = v; }
void SDPA::setParameterLowerBound(double v) { impl_->prm.lowerBound = v; }
void SDPA::setParameterUpperBound(double v) { impl_->prm.upperBound = v; }
void SDPA::setParameterBetaStar(double v) { impl_->prm.betaStar = v; }
void SDPA::setParameterBetaBar(double v) { impl_->prm.betaBar = v; }
void SDPA::setParameterGammaStar(double v) { impl_->prm.gammaStar = v; }
void SDPA::setParameterEpsilonDash(double v) { impl_->prm.epsilonDash = v; }
void SDPA::setParameterPrintXVec(char* s) { snprintf(impl_->xPrint, 32, "%s", s); }
void SDPA::setParameterPrintXMat(char* s) { snprintf(impl_->XPrint, 32, "%s", s); }
void SDPA::setParameterPrintYMat(char* s) { snprintf(impl_->YPrint, 32, "%s", s); }
void SDPA::setParameterPrintInformation(char* s) { snprintf(impl_->infPrint, 32, "%s", s); }
void SDPA::setDisplay(FILE* f) { impl_->display = f; }
void SDPA::setResultFile(FILE* f) { impl_->fpout = f; }
void SDPA::setInitPoint(bool b) { impl_->isInitPoint = b; }
// The solve runs on the GPU; the thread count is kept for getNumThreads and
// reported like Newton::setNumThreads (sdpa_newton.cpp:2127-2149): the given
// value, or OMP_NUM_THREADS, or 1.
void SDPA::setNumThreads(SDPA_INT n)
{
  if (!in_int(n)) return impl_->fail(SDPAB_EINVAL, "setNumThreads: value out of range");
  impl_->numThreads = (int)n;
  int nt = (int)n;
  if (nt == 0) {
    const char* env = getenv("OMP_NUM_THREADS");
    nt = env ? atoi(env) : 1;
  }
  for (FILE* f : {impl_->display, impl_->fpout})
    if (f) fprintf(f, "NumThreads  is set as %d\n", nt);
}

SDPA::ParameterType SDPA::getParameterType() { return (ParameterType)impl_->ptype; }
SDPA_INT SDPA::getParameterMaxIteration() { return impl_->prm.maxIteration; }
double SDPA::getParameterEpsilonStar() { return impl_->prm.epsilonStar; }
double SDPA::getParameterLambdaStar() { return impl_->prm.lambdaStar; }
double SDPA::getParameterOmegaStar() { return impl_->prm.omegaStar; }
double SDPA::getParameterLowerBound() { return impl_->prm.lowerBound; }
double SDPA::getParameterUpperBound() { return impl_->prm.upperBound; }
double SDPA::getParameterBetaStar() { return impl_->prm.betaStar; }
double SDPA::getParameterBetaBar() { return impl_->prm.betaBar; }
double SDPA::getParameterGammaStar() { return impl_->prm.gammaStar; }
double SDPA::getParameterEpsilonDash() { return impl_->prm.epsilonDash; }
char* SDPA::getParameterPrintXVec() { return impl_->xPrint; }
char* SDPA::getParameterPrintXMat() { return impl_->XPrint; }
char* SDPA::getParameterPrintYMat() { return impl_->YPrint; }
char* SDPA::getParameterPrintInformation() { return impl_->infPrint; }
FILE* SDPA::getDisplay() { return impl_->display; }
FILE* SDPA::getResultFile() { return impl_->fpout; }
bool SDPA::getInitPoint() { return impl_->isInitPoint; }
SDPA_INT SDPA::getNumThreads() { return impl_->numThreads; }

void SDPA::inputConstraintNumber(SDPA_INT m)
{
  if (m < 0 || !in_int(m)) return impl_->fail(SDPAB_EINVAL, "inputConstraintNumber: m out of range");
  impl_->prob.m = (int)m;
  impl_->prob.c.assign((size_t)m, 0.0);
}
void SDPA::inputBlockNumber(SDPA_INT nBlock)
{
  if (nBlock < 0 || !in_int(nBlock)) return impl_->fail(SDPAB_EINVAL, "inputBlockNumber: nBlock out of range");
  impl_->prob.blockStruct.assign((size_t)nBlock, 0);
  impl_->prob.blockType.assign((size_t)nBlock, 0);
}
void SDPA::inputBlockSize(SDPA_INT l, SDPA_INT size)
{
  if (l < 1 || l > impl_->nb()) return impl_->fail(SDPAB_EINVAL, "inputBlockSize: l out of range");
  if (!in_int(size)) return impl_->fail(SDPAB_EINVAL, "inputBlockSize: size out of range");
  impl_->prob.blockStruct[l - 1] = (int)size;
  if (size < 0) impl_->prob.blockType[l - 1] = 2;
}
void SDPA::inputBlockType(SDPA_INT l, ConeType t)
{
  if (l < 1 || l > impl_->nb()) return impl_->fail(SDPAB_EINVAL, "inputBlockType: l out of range");
  impl_->prob.blockType[l - 1] = (int)t;
}
void SDPA::inputCVec(SDPA_INT k, double v)
{
  if (k < 1 || k > impl_->prob.m) return impl_->fail(SDPAB_EINVAL, "inputCVec: k out of range");
  impl_->prob.c[k - 1] = v;
}
void SDPA::inputElement(SDPA_INT k, SDPA_INT l, SDPA_INT i, SDPA_INT j, double v, bool inputCheck)
{
  SdpaImpl& I = *impl_;
  if (inputCheck || true) {  // range errors are always reported (the reference may crash instead)
    if (k < 0 || k > I.prob.m) return I.fail(SDPAB_EINVAL, "inputElement: k out of range");
    if (l < 1 || l > I.nb()) return I.fail(SDPAB_EINVAL, "inputElement: l out of range");
    const int dim = I.blockDim(l - 1);
    if (i < 1 || j < 1 || i > dim || j > dim) return I.fail(SDPAB_EINVAL, "inputElement: i/j out of range");
    if (!I.isSdp(l - 1) && i != j) return I.fail(SDPAB_EINVAL, "inputElement: i != j in an LP block");
  }
  if (i > j) std::swap(i, j);
  I.prob.entries.push_back({(int)k, (int)l, (int)i, (int)j, v});
}
void SDPA::inputInitXVec(SDPA_INT k, double v)
{
  impl_->ensureInit();
  if (k < 1 || k > impl_->prob.m) return impl_->fail(SDPAB_EINVAL, "inputInitXVec: k out of range");
  impl_->init.xvec[k - 1] = v;
}
static void set_init(SdpaImpl& I, bool isX, long long l, long long i, long long j, double v)
{
  I.ensureInit();
  if (l < 1 || l > I.nb()) return I.fail(SDPAB_EINVAL, "inputInit: l out of range");
  const int n = I.blockDim((int)l - 1);
  if (i < 1 || j < 1 || i > n || j > n) return I.fail(SDPAB_EINVAL, "inputInit: i/j out of range");
  std::vector<double>& M = isX ? I.init.X[l - 1] : I.init.Y[l - 1];
  if (I.isSdp(l - 1)) {
    M[(i - 1) + (size_t)n * (j - 1)] = v;
    M[(j - 1) + (size_t)n * (i - 1)] = v;
  } else {
    if (i != j) return I.fail(SDPAB_EINVAL, "inputInit: i != j in an LP block");
    M[i - 1] = v;
  }
}
void SDPA::inputInitXMat(SDPA_INT l, SDPA_INT i, SDPA_INT j, double v) { set_init(*impl_, true, l, i, j, v); }
void SDPA::inputInitYMat(SDPA_INT l, SDPA_INT i, SDPA_INT j, double v) { set_init(*impl_, false, l, i, j, v); }

void SDPA::initializeUpperTriangleSpace()
{
  impl_->prob.entries.clear();
}
void SDPA::initializeUpperTriangle(bool inputTwiceCheck)
{
  // sortNonZeroElements / checkNonZeroElements (sdpa_call.cpp:446-501)
  std::vector<sdpab::Entry>& E = impl_->prob.entries;
  std::stable_sort(E.begin(), E.end(), [](const sdpab::Entry& a, const sdpab::Entry& b) {
    if (a.k != b.k) return a.k < b.k;
    if (a.l != b.l) return a.l < b.l;
    if (a.i != b.i) return a.i < b.i;
    return a.j < b.j;
  });
  if (inputTwiceCheck) {
    for (size_t q = 1; q < E.size(); ++q)
      if (E[q].k == E[q - 1].k && E[q].l == E[q - 1].l && E[q].i == E[q - 1].i && E[q].j == E[q - 1].j)
        return impl_->fail(SDPAB_EINVAL, "initializeUpperTriangle: element input twice");
  }
}
void SDPA::initializeSolve()
{
  SdpaImpl& I = *impl_;
  if (I.err) return;
  const int rc = I.solver.setup(I.prob, I.prm, I.kappa);
  if (rc != SDPAB_OK) return I.fail(rc, sdpab_last_error());
  // Newton::initialize_bMat's message (sdpa_newton.cpp:262-270): the Schur
  // path, always dense here
  for (FILE* f : {I.display, I.fpout})
    if (f) fprintf(f, "Schur computation : DENSE \n");
  I.initialized = true;
  I.solved = false;
}
void SDPA::resetParameters() {}
void SDPA::solve()
{
  SdpaImpl& I = *impl_;
  if (I.err) return;
  if (!I.initialized) return I.fail(SDPAB_ESTATE, "solve called before initializeSolve");
  if (I.isInitPoint) I.ensureInit();
  const int rc = I.solver.solve(I.isInitPoint ? &I.init : nullptr, &I.prm);
  if (rc != SDPAB_OK) return I.fail(rc, sdpab_last_error());
  I.solved = true;
  I.xvec = I.solver.xvec();
  I.Xres.assign(I.nb(), {});
  I.Yres.assign(I.nb(), {});
  for (int l = 1; l <= I.nb(); ++l) {
    I.Xres[l - 1] = I.solver.resultX(l);
    I.Yres[l - 1] = I.solver.resultY(l);
  }
  // the reference's output sequence of SDPA::solve (sdpa_solve.cpp:76, :164,
  // :212-231): header, one line per iteration, the last-iteration block,
  // parameters and times, the solution, and the time lines
  const sdpab::SolveStats& st = I.solver.stats();
  FILE* outs[2] = {I.fpout, I.display};
  const char* head = "   mu      thetaP  thetaD  objP      objD      alphaP  alphaD  beta \n";
  for (FILE* f : outs)
    if (f) fprintf(f, "%s", head);
  const size_t rows = st.trace.size() / 8;
  for (size_t q = 0; q < rows; ++q)
    for (FILE* f : outs)
      if (f) sdpab::print_iteration(f, (int)q, &st.trace[8 * q]);
  for (FILE* f : outs)
    if (f) sdpab::print_iteration(f, st.iterations, st.final_row);
  // IO::printLastInfo (sdpa_io.cpp:661-772)
  const double oP = st.objValPrimal, oD = st.objValDual;
  const double mean = (fabs(oP) + fabs(oD)) / 2.0, pdgap = fabs(oP - oD);
  const double relgap = (mean < 1.0) ? pdgap : pdgap / mean;
  const double gap = oP - oD;
  const double digits = -log10(fabs(pdgap / mean));
  char ph[32];
  getPhaseString(ph);
  for (FILE* f : {I.display, I.fpout}) {
    if (!f) continue;
    fprintf(f, "\n");
    fprintf(f, "phase.value  = %-10s\n", ph);
    fprintf(f, "   Iteration = %d\n", st.iterations);
    const char* labels[] = {"          mu = ", "relative gap = ", "        gap  = ", "     digits  = ",
                            "objValPrimal = ", "objValDual   = ", "p.feas.error = ", "d.feas.error = "};
    const double vals[] = {st.mu, relgap, gap, digits, -oD, -oP, st.primal_error, st.dual_error};
    for (int q = 0; q < 8; ++q) {
      fprintf(f, "%s", labels[q]);
      fprintf(f, I.infPrint, vals[q]);
      fprintf(f, "\n");
    }
    fprintf(f, "total time   = %.6f\n", st.solve_seconds + I.file_read_seconds);
  }
  if (I.fpout) {
    sdpab::print_params(I.fpout, I.prm, I, I.infPrint);
    sdpab::print_times(I.fpout, st, I.file_read_seconds);
    // IO::printSolution (sdpa_io.cpp:845-867)
    fprintf(I.fpout, "xVec = \n");
    printResultXVec(I.fpout);
    fprintf(I.fpout, "xMat = \n");
    printResultXMat(I.fpout);
    fprintf(I.fpout, "yMat = \n");
    printResultYMat(I.fpout);
  }
  const double tl[5] = {st.solve_seconds, st.solve_seconds + I.file_read_seconds, 0.0, 0.0, I.file_read_seconds};
  if (I.display) {
    const char* n[5] = {"  main loop time = ", "      total time = ", "file  check time = ", "file change time = ",
                        "file   read time = "};
    for (int q = 0; q < 5; ++q) fprintf(I.display, "%s%.6f\n", n[q], tl[q]);
  }
  if (I.fpout) {
    const char* n[5] = {"    main loop time = ", "        total time = ", "  file  check time = ",
                        "  file change time = ", "  file   read time = "};
    for (int q = 0; q < 5; ++q) fprintf(I.fpout, "%s%.6f\n", n[q], tl[q]);
  }
}

double* SDPA::getResultXVec() { return impl_->solved ? impl_->xvec.data() : nullptr; }
double* SDPA::getResultXMat(SDPA_INT l)
{
  if (!impl_->solved || l < 1 || l > impl_->nb()) return nullptr;
  return impl_->Xres[l - 1].data();
}
double* SDPA::getResultYMat(SDPA_INT l)
{
  if (!impl_->solved || l < 1 || l > impl_->nb()) return nullptr;
  return impl_->Yres[l - 1].data();
}
double SDPA::getPrimalObj() { return impl_->solver.stats().primal_obj; }
double SDPA::getDualObj() { return impl_->solver.stats().dual_obj; }
double SDPA::getPrimalError() { return impl_->solver.stats().primal_error; }
double SDPA::getDualError() { return impl_->solver.stats().dual_error; }
double SDPA::getDigits()
{
  const sdpab::SolveStats& s = impl_->solver.stats();
  const double mean = (fabs(s.objValPrimal) + fabs(s.objValDual)) / 2.0;
  return -log10(fabs(getDualityGap() / mean));
}
SDPA_INT SDPA::getIteration() { return impl_->solver.stats().iterations; }
double SDPA::getMu() { return impl_->solver.stats().mu; }
double SDPA::getDualityGap()
{
  const sdpab::SolveStats& s = impl_->solver.stats();
  return fabs(s.objValPrimal - s.objValDual);
}
SDPA::PhaseType SDPA::getPhaseValue() { return (PhaseType)impl_->solver.stats().phase; }
void SDPA::getPhaseString(char* str)
{
  static const char* names[] = {"noINFO    ", "pFEAS     ", "dFEAS     ", "pdFEAS    ", "pdINF     ",
                                "pFEAS_dINF", "pINF_dFEAS", "pdOPT     ", "pUNBD     ", "dUNBD     "};
  // SDPA::getPhaseString prints the internal (reversed) phase name (sdpa_call.cpp:788-803)
  int v = impl_->solver.stats().internal_phase;
  switch (v) {
    case 1: v = 2; break;
    case 2: v = 1; break;
    case 5: v = 6; break;
    case 6: v = 5; break;
    case 8: v = 9; break;
    case 9: v = 8; break;
  }
  strcpy(str, names[(v >= 0 && v < 10) ? v : 0]);
}
double SDPA::getSolveTime() { return impl_->solver.stats().solve_seconds; }
SDPA_INT SDPA::getConstraintNumber() { return impl_->prob.m; }
SDPA_INT SDPA::getBlockNumber() { return impl_->nb(); }
SDPA_INT SDPA::getBlockSize(SDPA_INT l)
{
  if (l < 1 || l > impl_->nb()) return 0;
  return impl_->blockDim(l - 1);
}
SDPA::ConeType SDPA::getBlockType(SDPA_INT l)
{
  if (l < 1 || l > impl_->nb()) return SDP;
  return impl_->isSdp(l - 1) ? SDP : LP;
}

// IO::computeDimacs (sdpa_io.cpp:775-813).  The input norms ||b||_1 and
// ||C||_1 (Lal::getOneNorm: largest absolute entry, sdpa_linear.cpp:184-235)
// come from the input data; the residual norms, X . Z and the minimum
// eigenvalues of X and Z are computed on the GPU from the final point.
void SDPA::getDimacsError(double* d)
{
  SdpaImpl& I = *impl_;
  for (int q = 0; q <= 6; ++q) d[q] = 0.0;
  if (!I.solved) return;
  double b1 = 0.0, c1 = 0.0;
  for (double v : I.prob.c) b1 = std::max(b1, fabs(v));
  for (const sdpab::Entry& e : I.prob.entries)
    if (e.k == 0) c1 = std::max(c1, fabs(e.v));
  double dev[5];
  const int rc = I.solver.dimacs(dev);
  if (rc != SDPAB_OK) {
    I.fail(rc, sdpab_last_error());
    return;
  }
  const sdpab::SolveStats& s = I.solver.stats();
  const double ctx = s.objValPrimal, bty = s.objValDual;
  d[1] = sqrt(dev[0]) / (1 + b1);
  d[2] = std::max(0.0, -dev[2] / (1 + b1));
  d[3] = sqrt(dev[1]) / (1 + c1);
  d[4] = std::max(0.0, -dev[3] / (1 + c1));
  d[5] = (ctx - bty) / (1 + fabs(ctx) + fabs(bty));
  d[6] = dev[4] / (1 + fabs(ctx) + fabs(bty));
}
void SDPA::printDimacsError(double* d, char* fmt, FILE* fp)
{
  if (!fp) return;
  static const char* what[] = {"", "[||Ax-b|| / (1+||b||_1)]", "[max(0, -lambda(x)/(1+||b||_1))]",
                               "[||A^Ty + z - c || / (1+||c||_1)]", "[max(0, -lambda(z)/(1+||c||_1))]",
                               "[(<c,x> - <b,y>) / (1 + |<c,x>| + |<b,y>|)]", "[<x,z> / (1 + |<c,x>| + |<b,y>|)]"};
  fprintf(fp, "\n* DIMACS_ERRORS * \n");
  for (int q = 1; q <= 6; ++q) {
    fprintf(fp, "err%d = ", q);
    fprintf(fp, fmt, d[q]);
    fprintf(fp, "  %s\n", what[q]);
  }
  fprintf(fp, "\n");
}

void SDPA::printResultXVec(FILE* fp)
{
  if (!fp || !impl_->solved) return;
  sdpab::print_vector(fp, impl_->xvec.data(), impl_->xvec.size(), impl_->xPrint);
}
void SDPA::printResultXMat(FILE* fp)
{
  if (fp && impl_->solved) sdpab::print_blocks(*impl_, impl_->Xres, impl_->XPrint, fp);
}
void SDPA::printResultYMat(FILE* fp)
{
  if (fp && impl_->solved) sdpab::print_blocks(*impl_, impl_->Yres, impl_->YPrint, fp);
}
void SDPA::printComputationTime(FILE* fp)
{
  if (fp) sdpab::print_times(fp, impl_->solver.stats(), impl_->file_read_seconds);
}
// Parameter::display with its default format "%+10.16e" (sdpa_parts.h:119)
void SDPA::printParameters(FILE* fp)
{
  if (fp) sdpab::print_params(fp, impl_->prm, *impl_, "%+10.16e");
}
void SDPA::printSDPAVersion(FILE* fp)
{
  if (fp) fprintf(fp, "%s\n", sdpab_version());
}

void SDPA::readInput(char* filename, FILE* fpout, SparseType type)
{
  const sdpab::ReadTimer timer_(impl_->file_read_seconds);
  SdpaImpl& I = *impl_;
  std::string txt, why;
  if (!filename || !sdpab::slurp(filename, txt)) return I.fail(SDPAB_EIO, "readInput: cannot open data file");
  bool sparse;
  if (type == AUTO) {
    const size_t len = strlen(filename);
    sparse = len >= 2 && filename[len - 1] == 's' && filename[len - 2] == '-';
  } else {
    sparse = (type == SPARSE);
  }
  if (fpout) {
    fprintf(fpout, "data   is %s  : %s\n", filename, sparse ? "sparse" : "dense");
    // the title / comment lines ahead of the data are echoed (IO::read, sdpa_io.cpp:33-45)
    size_t pos = 0;
    while (pos < txt.size() && (txt[pos] == '"' || txt[pos] == '*')) {
      const size_t eol = txt.find('\n', pos);
      const size_t e = (eol == std::string::npos) ? txt.size() : eol + 1;
      fwrite(txt.data() + pos, 1, e - pos, fpout);
      pos = e;
    }
  }
  const int rc = sdpab::parse_sdpa(txt, sparse, I.prob, why);
  if (rc != SDPAB_OK) return I.fail(rc, "readInput: " + why);
}
void SDPA::readInit(char* filename, FILE* fpout, SparseType type)
{
  const sdpab::ReadTimer timer_(impl_->file_read_seconds);
  SdpaImpl& I = *impl_;
  std::string txt, why;
  if (!filename || !sdpab::slurp(filename, txt)) return I.fail(SDPAB_EIO, "readInit: cannot open init file");
  bool sparse;
  if (type == AUTO) {
    const size_t len = strlen(filename);
    sparse = len >= 2 && filename[len - 1] == 's' && filename[len - 2] == '-';
  } else {
    sparse = (type == SPARSE);
  }
  if (fpout) fprintf(fpout, "initial is %s  : %s\n", filename, sparse ? "sparse" : "dense");
  const int rc = sdpab::parse_init(txt, sparse, I, why);
  if (rc != SDPAB_OK) return I.fail(rc, "readInit: " + why);
}
void SDPA::readParameter(char* filename, FILE* fpout)
{
  const sdpab::ReadTimer timer_(impl_->file_read_seconds);
  sdpab_params p;
  if (sdpab_read_params(filename, &p) != SDPAB_OK) return impl_->fail(SDPAB_EIO, "readParameter failed");
  memcpy(&impl_->prm, &p, sizeof(p));
  if (fpout) fprintf(fpout, "param  is %s \n", filename);
}
// SDPA::writeInputSparse (sdpa_call.cpp:1137-1197)
void SDPA::writeInputSparse(char* filename, char* fmt)
{
  SdpaImpl& I = *impl_;
  FILE* f = fopen(filename, "w");
  if (!f) return I.fail(SDPAB_EIO, "writeInputSparse: cannot open file");
  fprintf(f, "%d\n%d\n", I.prob.m, I.nb());
  for (int l = 0; l < I.nb(); ++l) fprintf(f, "%d ", I.prob.blockStruct[l]);
  fprintf(f, "\n");
  for (int k = 0; k < I.prob.m; ++k) {
    fprintf(f, fmt, I.prob.c[k]);
    fprintf(f, " ");
  }
  fprintf(f, "\n");
  std::vector<sdpab::Entry> E = I.prob.entries;
  std::stable_sort(E.begin(), E.end(), [](const sdpab::Entry& a, const sdpab::Entry& b) {
    return a.k != b.k ? a.k < b.k : a.l != b.l ? a.l < b.l : a.i != b.i ? a.i < b.i : a.j < b.j;
  });
  for (const sdpab::Entry& e : E) {
    fprintf(f, "%d %d %d %d ", e.k, e.l, e.i, e.j);
    fprintf(f, fmt, e.v);
    fprintf(f, "\n");
  }
  fclose(f);
}
// SDPA::writeInitSparse (sdpa_call.cpp:1199-1220): x, then user X (1) and Y (2)
void SDPA::writeInitSparse(char* filename, char* fmt)
{
  SdpaImpl& I = *impl_;
  if (!I.solved) return I.fail(SDPAB_ESTATE, "writeInitSparse: no solution");
  FILE* f = fopen(filename, "w");
  if (!f) return I.fail(SDPAB_EIO, "writeInitSparse: cannot open file");
  for (int k = 0; k < I.prob.m; ++k) {
    fprintf(f, fmt, I.xvec[k]);
    fprintf(f, " ");
  }
  fprintf(f, "\n");
  for (int target = 1; target <= 2; ++target)
    for (int l = 0; l < I.nb(); ++l) {
      const std::vector<double>& M = (target == 1) ? I.Xres[l] : I.Yres[l];
      const int n = I.blockDim(l);
      if (I.isSdp(l)) {
        for (int i = 0; i < n; ++i)
          for (int j = i; j < n; ++j) {
            const double v = M[i + (size_t)n * j];
            if (v == 0.0) continue;
            fprintf(f, "%d %d %d %d ", target, l + 1, i + 1, j + 1);
            fprintf(f, fmt, v);
            fprintf(f, "\n");
          }
      } else {
        for (int i = 0; i < n; ++i) {
          if (M[i] == 0.0) continue;
          fprintf(f, "%d %d %d %d ", target, l + 1, i + 1, i + 1);
          fprintf(f, fmt, M[i]);
          fprintf(f, "\n");
        }
      }
    }
  fclose(f);
}
void SDPA::terminate()
{
  impl_->solver.release();
  impl_->initialized = false;
  impl_->solved = false;
  impl_->xvec.clear();
  impl_->Xres.clear();
  impl_->Yres.clear();
}
// SDPA::copyCurrentToInit (sdpa_call.cpp:1238-1245): the last point becomes
// the initial point of the next solve.
void SDPA::copyCurrentToInit()
{
  SdpaImpl& I = *impl_;
  if (!I.solved) return;
  I.ensureInit();
  I.init.xvec = I.xvec;
  for (int l = 0; l < I.nb(); ++l) {
    I.init.X[l] = I.Xres[l];
    I.init.Y[l] = I.Yres[l];
  }
}
void SDPA::setKappa(double k) { impl_->kappa = k; }
void SDPA::setPrecision(int mode, double mu_switch) { impl_->solver.set_precision(mode, mu_switch); }
void SDPA::setTensorCoreWaitLimit(long long polls) { impl_->solver.set_tc_wait(polls); }
int SDPA::getErrorCode() { return impl_->err; }
const sdpab::SolveStats& SDPA::impl_solver_stats() { return impl_->solver.stats(); }
const char* SDPA::getErrorMessage() { return impl_->errmsg.c_str(); }

// ------------------------------------------------------------------ C ABI
extern "C" {

SDPAB_API sdpab_sdpa* sdpab_sdpa_new(void) { return (sdpab_sdpa*)new SDPA(); }
SDPAB_API void sdpab_sdpa_free(sdpab_sdpa* h) { delete (SDPA*)h; }

static int status_of(SDPA* p)
{
  const int e = p->getErrorCode();
  if (e) sdpab::set_error(e, p->getErrorMessage());
  return e;
}

SDPAB_API int sdpab_sdpa_set_params(sdpab_sdpa* h, const sdpab_params* prm)
{
  if (!h || !prm) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  SDPA* p = (SDPA*)h;
  p->setParameterMaxIteration(prm->maxIteration);
  p->setParameterEpsilonStar(prm->epsilonStar);
  p->setParameterLambdaStar(prm->lambdaStar);
  p->setParameterOmegaStar(prm->omegaStar);
  p->setParameterLowerBound(prm->lowerBound);
  p->setParameterUpperBound(prm->upperBound);
  p->setParameterBetaStar(prm->betaStar);
  p->setParameterBetaBar(prm->betaBar);
  p->setParameterGammaStar(prm->gammaStar);
  p->setParameterEpsilonDash(prm->epsilonDash);
  return SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_read_input(sdpab_sdpa* h, const char* path, int sparse_type)
{
  if (!h || !path) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  SDPA* p = (SDPA*)h;
  p->readInput((char*)path, NULL, (SDPA::SparseType)sparse_type);
  return status_of(p);
}
SDPAB_API int sdpab_sdpa_read_init(sdpab_sdpa* h, const char* path, int sparse_type)
{
  if (!h || !path) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  SDPA* p = (SDPA*)h;
  p->setInitPoint(true);
  p->readInit((char*)path, NULL, (SDPA::SparseType)sparse_type);
  return status_of(p);
}
SDPAB_API int sdpab_sdpa_read_param(sdpab_sdpa* h, const char* path)
{
  if (!h || !path) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  SDPA* p = (SDPA*)h;
  p->readParameter((char*)path, NULL);
  return status_of(p);
}
SDPAB_API int sdpab_sdpa_input_problem(sdpab_sdpa* h, int m, int nblock, const int* block_struct,
                                       const double* c, long long nnz, const int* k, const int* l,
                                       const int* i, const int* j, const double* v)
{
  if (!h || !block_struct || !c) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  SDPA* p = (SDPA*)h;
  p->inputConstraintNumber(m);
  p->inputBlockNumber(nblock);
  for (int b = 0; b < nblock; ++b) {
    p->inputBlockSize(b + 1, block_struct[b]);
    p->inputBlockType(b + 1, block_struct[b] < 0 ? SDPA::LP : SDPA::SDP);
  }
  p->initializeUpperTriangleSpace();
  for (int q = 0; q < m; ++q) p->inputCVec(q + 1, c[q]);
  for (long long e = 0; e < nnz; ++e) p->inputElement(k[e], l[e], i[e], j[e], v[e]);
  p->initializeUpperTriangle(false);
  return status_of(p);
}
SDPAB_API int sdpab_sdpa_set_init(sdpab_sdpa* h, const double* xvec, const double* const* X,
                                  const double* const* Y)
{
  if (!h || !xvec || !X || !Y) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  SDPA* p = (SDPA*)h;
  p->setInitPoint(true);
  const int m = p->getConstraintNumber(), nb = p->getBlockNumber();
  for (int k = 1; k <= m; ++k) p->inputInitXVec(k, xvec[k - 1]);
  for (int l = 1; l <= nb; ++l) {
    const int n = p->getBlockSize(l);
    const bool sdp = p->getBlockType(l) == SDPA::SDP;
    for (int i = 1; i <= n; ++i)
      for (int j = sdp ? i : i; j <= (sdp ? n : i); ++j) {
        const size_t off = sdp ? (size_t)(i - 1) + (size_t)n * (j - 1) : (size_t)(i - 1);
        p->inputInitXMat(l, i, j, X[l - 1][off]);
        p->inputInitYMat(l, i, j, Y[l - 1][off]);
      }
  }
  return status_of(p);
}
SDPAB_API int sdpab_sdpa_set_precision(sdpab_sdpa* h, int mode, double mu_switch)
{
  if (!h || (mode != SDPAB_PREC_FP64 && mode != SDPAB_PREC_MIXED))
    return sdpab::set_error(SDPAB_EINVAL, "set_precision: bad arguments");
  ((SDPA*)h)->setPrecision(mode, mu_switch);
  return SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_set_tc_wait(sdpab_sdpa* h, long long polls)
{
  if (!h) return sdpab::set_error(SDPAB_EINVAL, "set_tc_wait: null handle");
  ((SDPA*)h)->setTensorCoreWaitLimit(polls);
  return SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_tc_timeouts(sdpab_sdpa* h, int* out)
{
  if (!h || !out) return sdpab::set_error(SDPAB_EINVAL, "tc_timeouts: null argument");
  *out = ((SDPA*)h)->impl_solver_stats().tc_timeouts;
  return SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_solve(sdpab_sdpa* h)
{
  if (!h) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  SDPA* p = (SDPA*)h;
  p->initializeSolve();
  if (status_of(p)) return p->getErrorCode();
  p->solve();
  return status_of(p);
}
SDPAB_API int sdpab_sdpa_info(sdpab_sdpa* h, sdpab_sdpa_info_t* out)
{
  if (!h || !out) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  SDPA* p = (SDPA*)h;
  out->primal_obj = p->getPrimalObj();
  out->dual_obj = p->getDualObj();
  out->primal_error = p->getPrimalError();
  out->dual_error = p->getDualError();
  out->mu = p->getMu();
  out->duality_gap = p->getDualityGap();
  out->solve_seconds = p->getSolveTime();
  out->iterations = p->getIteration();
  out->phase = (int)p->getPhaseValue();
  out->m = p->getConstraintNumber();
  out->nblock = p->getBlockNumber();
  return SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_schur_pattern(sdpab_sdpa* h, int* sparse, long long* pairs)
{
  if (!h || !sparse || !pairs) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  const sdpab::SolveStats& s = ((SDPA*)h)->impl_solver_stats();
  *sparse = s.schur_sparse;
  pairs[0] = s.schur_sparse_pairs;
  pairs[1] = s.schur_dense_pairs;
  return SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_phase_times(sdpab_sdpa* h, double* out8)
{
  if (!h || !out8) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  const sdpab::SolveStats& s = ((SDPA*)h)->impl_solver_stats();
  for (int q = 0; q < 8; ++q) out8[q] = (q < (int)s.phase_seconds.size()) ? s.phase_seconds[q] : 0.0;
  return SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_get_xvec(sdpab_sdpa* h, double* out)
{
  SDPA* p = (SDPA*)h;
  const double* x = p ? p->getResultXVec() : nullptr;
  if (!x || !out) return sdpab::set_error(SDPAB_ESTATE, "no result");
  memcpy(out, x, sizeof(double) * p->getConstraintNumber());
  return SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_get_block(sdpab_sdpa* h, int l, int which, double* out)
{
  SDPA* p = (SDPA*)h;
  if (!p || !out || l < 1 || l > p->getBlockNumber()) return sdpab::set_error(SDPAB_EINVAL, "bad block");
  const double* M = (which == 0) ? p->getResultXMat(l) : p->getResultYMat(l);
  if (!M) return sdpab::set_error(SDPAB_ESTATE, "no result");
  const int n = p->getBlockSize(l);
  const size_t len = (p->getBlockType(l) == SDPA::SDP) ? (size_t)n * n : (size_t)n;
  memcpy(out, M, len * sizeof(double));
  return SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_block_size(sdpab_sdpa* h, int l, int* size, int* is_sdp)
{
  SDPA* p = (SDPA*)h;
  if (!p || l < 1 || l > p->getBlockNumber()) return sdpab::set_error(SDPAB_EINVAL, "bad block");
  *size = p->getBlockSize(l);
  *is_sdp = p->getBlockType(l) == SDPA::SDP;
  return SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_dimacs(sdpab_sdpa* h, double* err7)
{
  if (!h || !err7) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  SDPA* p = (SDPA*)h;
  const int before = p->getErrorCode();
  p->getDimacsError(err7);
  const int e = p->getErrorCode();
  return (e != before) ? e : SDPAB_OK;
}
SDPAB_API int sdpab_sdpa_write_init(sdpab_sdpa* h, const char* path)
{
  if (!h || !path) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  SDPA* p = (SDPA*)h;
  p->writeInitSparse((char*)path, (char*)"%+.17e");
  return status_of(p);
}
SDPAB_API int sdpab_sdpa_copy_current_to_init(sdpab_sdpa* h)
{
  if (!h) return sdpab::set_error(SDPAB_EINVAL, "null argument");
  ((SDPA*)h)->copyCurrentToInit();
  ((SDPA*)h)->setInitPoint(true);
  return SDPAB_OK;
}

}  // extern "C"
