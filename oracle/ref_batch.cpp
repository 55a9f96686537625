// Oracle driver (test infrastructure only): solves SDPA-format instances with
// the REFERENCE solver, linked from the reference sources by oracle/Makefile,
// through the reference's own public API (class SDPA of sdpa_call.h:91-267):
// readParameter / readInput / initializeSolve / solve / getters, the same
// sequence as the reference CLI main (sdpa_exe.cpp:224-343).
//
// Usage:
//   ref_batch [--param FILE] [--procs P] [--dump DIR] [--trace] [--xvec] FILE.dat-s ...
//
// One line per instance on stdout:
//   RESULT <file> <iterations> <phase> <primalObj> <dualObj> <solve_seconds>
// With --trace, each iteration's (mu, objP, objD, alphaP, alphaD, beta) line
// from the reference's own display output is echoed as
//   TRACE <file> <reference iteration line>
// With --xvec, the instance's xVec (getResultXVec) follows as
//   XVEC <file> <m> <x_1> ... <x_m>
// With --dump DIR, xVec (SDPA's x), and every block of X (getResultXMat) and
// Y (getResultYMat) are written as raw little-endian float64 files.
// --procs P forks P workers (instances dealt round-robin); the parent prints
//   WALL <seconds> <instances>
// where seconds is the longest worker's summed initializeSolve+solve time
// (file parsing excluded, as in the reference's own timing window).
#include <sdpa_call.h>
#include <sys/wait.h>
#include <unistd.h>
#include <sys/time.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

static double now_s()
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static const char* phase_name(SDPA::PhaseType p)
{
  switch (p) {
  case SDPA::noINFO: return "noINFO";
  case SDPA::pFEAS: return "pFEAS";
  case SDPA::dFEAS: return "dFEAS";
  case SDPA::pdFEAS: return "pdFEAS";
  case SDPA::pdINF: return "pdINF";
  case SDPA::pFEAS_dINF: return "pFEAS_dINF";
  case SDPA::pINF_dFEAS: return "pINF_dFEAS";
  case SDPA::pdOPT: return "pdOPT";
  case SDPA::pUNBD: return "pUNBD";
  case SDPA::dUNBD: return "dUNBD";
  }
  return "unknown";
}

static void dump(const std::string& path, const double* p, size_t n)
{
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) { perror(path.c_str()); exit(2); }
  fwrite(p, sizeof(double), n, f);
  fclose(f);
}

static std::string base_name(const std::string& f)
{
  size_t s = f.find_last_of('/');
  std::string b = (s == std::string::npos) ? f : f.substr(s + 1);
  size_t d = b.find(".dat");
  return d == std::string::npos ? b : b.substr(0, d);
}

// Solves one file; returns initializeSolve+solve seconds.
static double solve_one(const std::string& file, const char* param, const char* dumpdir,
                        bool trace, bool xvec, FILE* out)
{
  SDPA p;
  char tracefile[64] = {0};
  FILE* disp = NULL;
  if (trace) {
    snprintf(tracefile, sizeof(tracefile), "/tmp/ref_batch_trace_%d.txt", (int)getpid());
    disp = fopen(tracefile, "w+");
  }
  // The reference's printers and readParameter write to their FILE* without
  // NULL checks, so quiet output goes to /dev/null rather than NULL.
  static FILE* devnull = fopen("/dev/null", "w");
  p.setDisplay(disp ? disp : devnull);
  p.setResultFile(devnull);
  if (param) {
    p.readParameter((char*)param, devnull);
  } else {
    p.setParameterType(SDPA::PARAMETER_DEFAULT);
  }
  p.setNumThreads(0);
  p.readInput((char*)file.c_str(), devnull, SDPA::AUTO);
  double t0 = now_s();
  p.initializeSolve();
  p.solve();
  double t1 = now_s();
  fprintf(out, "RESULT %s %d %s %.17e %.17e %.9f\n", file.c_str(), (int)p.getIteration(),
          phase_name(p.getPhaseValue()), p.getPrimalObj(), p.getDualObj(), t1 - t0);
  if (xvec) {
    // one write per line: workers share the output pipe, and writes of up to
    // PIPE_BUF bytes (m up to about 160) do not interleave
    const int m = (int)p.getConstraintNumber();
    const double* x = p.getResultXVec();
    std::string line = "XVEC " + file + " " + std::to_string(m);
    char num[40];
    for (int k = 0; k < m; ++k) {
      snprintf(num, sizeof(num), " %.17e", x[k]);
      line += num;
    }
    line += "\n";
    fflush(out);
    fwrite(line.data(), 1, line.size(), out);
  }
  if (trace && disp) {
    fflush(disp);
    rewind(disp);
    char line[1024];
    while (fgets(line, sizeof(line), disp)) {
      fprintf(out, "TRACE %s %s", file.c_str(), line);
    }
    fclose(disp);
    unlink(tracefile);
  }
  if (dumpdir) {
    std::string b = std::string(dumpdir) + "/" + base_name(file);
    int m = (int)p.getConstraintNumber();
    dump(b + ".xvec.bin", p.getResultXVec(), (size_t)m);
    int nb = (int)p.getBlockNumber();
    for (int l = 1; l <= nb; ++l) {
      int sz = (int)p.getBlockSize(l);
      size_t n = (p.getBlockType(l) == SDPA::SDP) ? (size_t)sz * sz : (size_t)(sz < 0 ? -sz : sz);
      char sfx[64];
      snprintf(sfx, sizeof(sfx), ".X%d.bin", l);
      dump(b + sfx, p.getResultXMat(l), n);
      snprintf(sfx, sizeof(sfx), ".Y%d.bin", l);
      dump(b + sfx, p.getResultYMat(l), n);
    }
  }
  fflush(out);
  p.terminate();
  return t1 - t0;
}

int main(int argc, char** argv)
{
  const char* param = NULL;
  const char* dumpdir = NULL;
  bool trace = false, xvec = false;
  int procs = 1;
  std::vector<std::string> files;
  for (int a = 1; a < argc; ++a) {
    if (!strcmp(argv[a], "--param") && a + 1 < argc) param = argv[++a];
    else if (!strcmp(argv[a], "--dump") && a + 1 < argc) dumpdir = argv[++a];
    else if (!strcmp(argv[a], "--procs") && a + 1 < argc) procs = atoi(argv[++a]);
    else if (!strcmp(argv[a], "--trace")) trace = true;
    else if (!strcmp(argv[a], "--xvec")) xvec = true;
    else if (!strcmp(argv[a], "--list") && a + 1 < argc) {
      FILE* f = fopen(argv[++a], "r");
      if (!f) { perror(argv[a]); return 2; }
      char line[4096];
      while (fgets(line, sizeof(line), f)) {
        size_t l = strlen(line);
        while (l && (line[l - 1] == '\n' || line[l - 1] == '\r')) line[--l] = 0;
        if (l) files.push_back(line);
      }
      fclose(f);
    } else files.push_back(argv[a]);
  }
  if (files.empty()) {
    fprintf(stderr, "usage: ref_batch [--param F] [--procs P] [--dump DIR] [--trace] [--xvec] [--list F] FILE...\n");
    return 2;
  }
  if (procs <= 1) {
    double tot = 0.0;
    for (size_t i = 0; i < files.size(); ++i) tot += solve_one(files[i], param, dumpdir, trace, xvec, stdout);
    printf("WALL %.9f %zu\n", tot, files.size());
    return 0;
  }
  // Fork workers; each reports its summed solve time through a pipe.
  std::vector<int> rfd(procs);
  std::vector<pid_t> pid(procs);
  fflush(stdout);
  for (int r = 0; r < procs; ++r) {
    int fds[2];
    if (pipe(fds)) { perror("pipe"); return 2; }
    pid[r] = fork();
    if (pid[r] == 0) {
      close(fds[0]);
      double tot = 0.0;
      for (size_t i = r; i < files.size(); i += procs) tot += solve_one(files[i], param, dumpdir, trace, xvec, stdout);
      if (write(fds[1], &tot, sizeof(tot)) != (ssize_t)sizeof(tot)) _exit(3);
      close(fds[1]);
      fflush(stdout);
      _exit(0);
    }
    close(fds[1]);
    rfd[r] = fds[0];
  }
  double worst = 0.0;
  int rc = 0;
  for (int r = 0; r < procs; ++r) {
    double t = 0.0;
    if (read(rfd[r], &t, sizeof(t)) != (ssize_t)sizeof(t)) rc = 3;
    close(rfd[r]);
    int st = 0;
    waitpid(pid[r], &st, 0);
    if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) rc = 3;
    if (t > worst) worst = t;
  }
  printf("WALL %.9f %zu\n", worst, files.size());
  return rc;
}
