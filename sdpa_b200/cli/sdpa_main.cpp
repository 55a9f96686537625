// sdpa — command-line driver of the B200 solver, a drop-in for the reference
// executable (sdpa_exe.cpp:81-343): the same two argument styles, the same
// start/end lines on stdout and in the result file, and the result file that
// SDPA::solve writes (iteration table, last-iteration block, parameters,
// times, xVec / xMat / yMat).
//
//   sdpa DataFile OutputFile [InitialPtFile] [-pt 0|1|2] [-dimacs] [-numThreads n]
//   sdpa [-dd|-ds DataFile] [-id|-is InitFile] -o OutputFile [-p ParamFile]
//        [-pt 0|1|2] [-k kappa] [-dimacs] [-numThreads n] [-mixed]
//
// Style 1 reads ./param.sdpa unless -pt is given; a data or init file name
// ending in "-s" is read as sparse.  -numThreads is accepted and ignored (the
// solve runs on the GPU).  -mixed (no reference counterpart) selects the
// mixed-precision mode.  Errors that the reference reports by exit() are
// reported here with the library's error message and exit status 1.
#include <sdpa_call.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>

namespace {

const char* kDefaultParam = "./param.sdpa";

void usage(const char* argv0)
{
  printf("\n*** Please assign data file and output file.***\n\n");
  printf("---- option type 1 ------------\n");
  printf("%s DataFile OutputFile [InitialPtFile] [-pt parameters] [-dimacs] [-numThreads numThreads]\n", argv0);
  printf("parameters = 0 default, 1 fast (unstable), 2 slow (stable)\n");
  printf("  -dimacs : printout dimacs information incurring additional computation cost \n");
  printf("  -numThreads: accepted for compatibility; the solve runs on the GPU\n\n");
  printf("---- option type 2 ------------\n");
  printf("%s [option filename]+ \n", argv0);
  printf("  -dd : data dense :: -ds : data sparse     \n");
  printf("  -id : init dense :: -is : init sparse     \n");
  printf("  -o  : output     :: -p  : parameter       \n");
  printf("  -k  : Kappa (RealValue)\n");
  printf("  -pt : parameters , 0 default, 1 fast (unstable)\n");
  printf("                     2 slow (stable)         \n");
  printf("  -dimacs : printout dimacs information incurring additional computation cost \n");
  printf("  -mixed : mixed precision (FP32 bulk products, FP64 refinement)\n");
  exit(1);
}

bool ends_sparse(const char* name)
{
  const size_t n = strlen(name);
  return n >= 2 && name[n - 1] == 's' && name[n - 2] == '-';
}

SDPA::ParameterType ptype_of(const char* s)
{
  switch (atoi(s)) {
    case 1: return SDPA::PARAMETER_UNSTABLE_BUT_FAST;
    case 2: return SDPA::PARAMETER_STABLE_BUT_SLOW;
    default: return SDPA::PARAMETER_DEFAULT;
  }
}

struct Args {
  const char* input = nullptr;
  const char* result = nullptr;
  const char* init = nullptr;
  const char* param = nullptr;
  SDPA::SparseType inputType = SDPA::DENSE;
  SDPA::SparseType initType = SDPA::DENSE;
  SDPA::ParameterType ptype = SDPA::PARAMETER_DEFAULT;
  bool dimacs = false;
  bool mixed = false;
  int numThreads = 0;
  double kappa = 0.0;
};

Args parse(int argc, char** argv)
{
  Args a;
  if (argc < 2) usage(argv[0]);
  if (argv[1][0] == '-') {  // option style
    for (int i = 1; i < argc; ++i) {
      const std::string o = argv[i];
      const bool has = i + 1 < argc;
      if (o == "-dd" && has) { a.input = argv[++i]; a.inputType = SDPA::DENSE; }
      else if (o == "-ds" && has) { a.input = argv[++i]; a.inputType = SDPA::SPARSE; }
      else if (o == "-id" && has) { a.init = argv[++i]; a.initType = SDPA::DENSE; }
      else if (o == "-is" && has) { a.init = argv[++i]; a.initType = SDPA::SPARSE; }
      else if (o == "-o" && has) a.result = argv[++i];
      else if (o == "-p" && has) a.param = argv[++i];
      else if (o == "-k" && has) a.kappa = atof(argv[++i]);
      else if (o == "-dimacs") a.dimacs = true;
      else if (o == "-mixed") a.mixed = true;
      else if (o == "-pt" && has) { a.ptype = ptype_of(argv[++i]); a.param = nullptr; }
      else if (o == "-numThreads" && has) a.numThreads = atoi(argv[++i]);
    }
  } else {  // positional style
    a.input = argv[1];
    if (ends_sparse(a.input)) a.inputType = SDPA::SPARSE;
    if (argc < 3) usage(argv[0]);
    a.result = argv[2];
    a.param = kDefaultParam;
    for (int i = 3; i < argc; ++i) {
      const std::string o = argv[i];
      if (o == "-dimacs") a.dimacs = true;
      else if (o == "-mixed") a.mixed = true;
      else if (o == "-numThreads" && i + 1 < argc) a.numThreads = atoi(argv[++i]);
      else if (o == "-pt" && i + 1 < argc) { a.ptype = ptype_of(argv[++i]); a.param = nullptr; }
      else {
        a.init = argv[i];
        if (ends_sparse(a.init)) a.initType = SDPA::SPARSE;
      }
    }
  }
  if (!a.input || !a.result) usage(argv[0]);
  return a;
}

std::string now_string()
{
  time_t t = time(nullptr);
  std::string s = ctime(&t);
  if (!s.empty() && s.back() == '\n') s.pop_back();
  return s;
}

int fail(SDPA& p, FILE* fres, const char* what)
{
  fprintf(stderr, "sdpa: %s: %s\n", what, p.getErrorMessage());
  if (fres) fprintf(fres, "sdpa: %s: %s\n", what, p.getErrorMessage());
  if (fres) fclose(fres);
  return 1;
}

}  // namespace

int main(int argc, char** argv)
{
  const auto t0 = std::chrono::steady_clock::now();
  const std::string start = now_string();
  printf("SDPA start at [%s]\n", start.c_str());
  setbuf(stdout, nullptr);
  Args a = parse(argc, argv);
  SDPA p;
  if (a.kappa > 0.0) {
    p.setKappa(a.kappa);
    printf("Kappa = %g\n", a.kappa);
  }
  p.setDisplay(stdout);
  FILE* fres = fopen(a.result, "w");
  if (!fres) {
    fprintf(stderr, "sdpa: cannot open result file %s\n", a.result);
    return 1;
  }
  fprintf(fres, "SDPA start at [%s]\n", start.c_str());
  p.setResultFile(fres);
  if (!a.param) {
    const char* names[] = {"DEFAULT", "UNSTABLE_BUT_FAST", "STABLE_BUT_SLOW"};
    printf("set   is %s\n", names[(int)a.ptype]);
    fprintf(fres, "set   is %s\n", names[(int)a.ptype]);
    p.setParameterType(a.ptype);
  } else {
    printf("param is %s\n", a.param);
    p.readParameter((char*)a.param, fres);
    if (p.getErrorCode()) return fail(p, fres, "cannot read the parameter file");
  }
  printf("data  is %s : %s\n", a.input, a.inputType == SDPA::SPARSE ? "sparse" : "dense");
  p.readInput((char*)a.input, fres, a.inputType);
  if (p.getErrorCode()) return fail(p, fres, "cannot read the data file");
  if (a.init) {
    p.setInitPoint(true);
    printf("init  is %s : %s\n", a.init, a.initType == SDPA::SPARSE ? "sparse" : "dense");
    p.readInit((char*)a.init, fres, a.initType);
    if (p.getErrorCode()) return fail(p, fres, "cannot read the initial point file");
  }
  printf("out   is %s\n", a.result);
  fprintf(fres, "out    is %s\n", a.result);
  if (a.dimacs) {
    printf("Dimacs information will be computed after the iteration.\n");
    fprintf(fres, "Dimacs information will be computed after the iteration.\n");
  }
  if (a.mixed) p.setPrecision(1);
  p.setNumThreads(a.numThreads);
  p.initializeSolve();
  if (p.getErrorCode()) return fail(p, fres, "initializeSolve");
  p.solve();
  if (p.getErrorCode()) return fail(p, fres, "solve");
  if (a.dimacs) {
    double d[7];
    p.getDimacsError(d);
    p.printDimacsError(d, p.getParameterPrintInformation(), stdout);
    p.printDimacsError(d, p.getParameterPrintInformation(), fres);
  }
  p.terminate();
  const std::string end = now_string();
  printf("SDPA end at [%s]\n", end.c_str());
  fprintf(fres, "SDPA end at [%s]\n", end.c_str());
  const double all = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  printf("ALL TIME = %.6f\n", all);
  fprintf(fres, "ALL TIME = %.6f\n", all);
  fclose(fres);
  return 0;
}
