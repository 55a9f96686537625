// Host-driven solver for one SDPA problem with any block structure (SDP
// blocks + LP block), the engine behind the drop-in SDPA class.  Host C++
// runs the Mehrotra predictor-corrector control (ipm_control.h, the
// reference's sdpa_parts.cpp scalar logic); every vector/matrix step is a
// CUDA kernel on device-resident data.  No CPU fallback exists.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "ipm_control.h"

namespace sdpab {

// One nonzero of F_k (k = 0 is F0) exactly as a .dat-s line states it:
// 1-based block l, row i, column j (i <= j after staging), value v.
struct Entry {
  int k, l, i, j;
  double v;
};

// A problem in SDPA's input form (the .dat-s file / inputElement calls).
struct ProblemData {
  int m = 0;
  std::vector<int> blockStruct;   // signed block sizes (negative = LP)
  std::vector<int> blockType;     // 0 = SDP, 1 = SOCP (rejected), 2 = LP (SDPA::ConeType)
  std::vector<double> c;          // the m-vector c (b of the internal problem)
  std::vector<Entry> entries;
};

// Warm start in the user's terms (SDPA::inputInitXVec / XMat / YMat): dense
// column-major n x n per SDP block, a vector per LP block, in file block order.
struct InitPoint {
  std::vector<double> xvec;
  std::vector<std::vector<double>> X, Y;
};

struct SolveStats {
  int iterations = 0;
  int phase = 0;            // SDPA::PhaseType code (after reverse + getPhaseValue)
  int internal_phase = 0;
  double primal_obj = 0, dual_obj = 0;  // getPrimalObj / getDualObj
  double primal_error = 0, dual_error = 0;
  double mu = 0;
  double objValPrimal = 0, objValDual = 0;  // internal SolveInfo values
  double solve_seconds = 0;
  int cholesky_failed = 0;
  int warm_start_rejected = 0;
  int tc_timeouts = 0;      // tensor-core Schur updates abandoned (FP64 factor used instead)
  int schur_sparse = 0;     // 1: the Schur factorisation skipped the tile pairs its pattern leaves zero
  long long schur_sparse_pairs = 0, schur_dense_pairs = 0;  // trailing tile pairs: pattern / dense
  std::vector<double> trace;  // per iteration: mu, thetaP, thetaD, objP, objD, alphaP, alphaD, beta
  double final_row[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // the same quantities at loop exit
  // device seconds per phase: rMat+gVec, bMat, Cholesky, solves, dX/dZ,
  // step length, update (inverses), residuals
  std::vector<double> phase_seconds;
};

struct DevState;  // device buffers (single_engine.cu)

class Solver {
 public:
  Solver();
  ~Solver();
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;

  // SDPA::initializeSolve (sdpa_solve.cpp:10-43): block layout, constraint
  // index, formula choice (computeFormula_SDP), device upload.  Returns an
  // SDPAB_* status.  For problems of several SDP blocks the constraints are
  // first put in a fill-reducing order for the Schur factorisation (the
  // reference leaves that to MUMPS's own ordering); the results are given
  // back in the caller's order.
  int setup(const ProblemData& p, const Params& prm, double kappa);
  // The constraint order of the last setup: internal position -> caller's
  // constraint (0-based); empty when it is the caller's own order.
  const std::vector<int>& constraint_order() const { return perm_; }
  // SDPA::solve (sdpa_solve.cpp:59-233); init may be NULL.  `prm` are the
  // parameters in force at the call (the reference reads its Parameter
  // object at solve time, so changes after initializeSolve apply); NULL
  // keeps those given to setup.
  int solve(const InitPoint* init, const Params* prm = nullptr);
  void release();
  // SDPAB_PREC_FP64 (default) or SDPAB_PREC_MIXED: FP32 products and FP32
  // Schur factor with FP64 refinement while the relative complementarity
  // gap n*mu / max(1, mean |objective|) >= mu_switch (0 = 1e-2).
  void set_precision(int mode, double mu_switch)
  {
    precision_ = mode;
    mu_switch_ = mu_switch;
  }
  // polls per wait of the tensor-core pipelines (< 0: their default bound)
  void set_tc_wait(long long polls) { tc_wait_ = polls; }

  const SolveStats& stats() const { return stats_; }
  // Results in the reference getters' layout (file block order, 1-based l).
  const std::vector<double>& xvec() const { return xvec_; }
  const std::vector<double>& resultX(int l) const { return Xres_[l - 1]; }  // getResultXMat
  const std::vector<double>& resultY(int l) const { return Yres_[l - 1]; }  // getResultYMat
  int formula_count(int f) const;  // number of (constraint, block) pairs using F1/F2/F3
  // The device part of IO::computeDimacs (sdpa_io.cpp:775-813) for the last
  // solve: out = {||rp||^2, ||D||^2, lambda_min(X), lambda_min(Z), X . Z} of
  // the final point (internal X, Z; D and rp the final residuals).
  int dimacs(double* out);

 private:
  DevState* d_ = nullptr;
  int precision_ = 0;
  double mu_switch_ = 0.0;
  long long tc_wait_ = -1;
  SolveStats stats_;
  std::vector<double> xvec_;
  std::vector<int> perm_;  // internal constraint position -> caller's constraint
  int setup_ordered(const ProblemData& p, const Params& prm, double kappa);
  std::vector<std::vector<double>> Xres_, Yres_;
};

}  // namespace sdpab
