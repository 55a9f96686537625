/* sdpa_call.h — drop-in C++ interface of the B200 solver.
 *
 * Mirrors class SDPA of the reference (sdpa_call.h:91-267): the same enums,
 * method names, argument meanings, 1-based indices, upper-triangle staging of
 * inputElement, sign conventions (getResultXMat is the solver's internal Z,
 * getResultYMat its internal X, getPrimalObj = -objValDual), and result
 * pointers that stay valid until terminate() or destruction.  Differences:
 *  - no exit(): input errors set an error code (getErrorCode/getErrorMessage)
 *    and make initializeSolve/solve return without solving;
 *  - setNumThreads is accepted and ignored (the solve runs on the GPU);
 *  - SOCP is rejected as in the reference.
 * SDPA_INT is int by default (the reference's LP64 configuration,
 * LP64/sdpa_include.h:43-45), with sdpa_b200/_lib/libsdpa_b200.so.  Callers
 * built for the reference's ILP64 configuration (ILP64/sdpa_include.h:43-45,
 * SDPA_INT = int64_t) compile with -DSDPA_INT=int64_t and link
 * sdpa_b200/_lib/libsdpa_b200_ilp64.so, the same library with that integer
 * type in the class's signatures.  Sizes and indices beyond the int range
 * are rejected (the solver's dense Schur matrix limits m far below it).
 */
#ifndef SDPA_B200_SDPA_CALL_H
#define SDPA_B200_SDPA_CALL_H

#include <cstdint>
#include <cstdio>

#ifndef SDPA_INT
#define SDPA_INT int
#endif

#if defined(__GNUC__)
#define SDPAB_CLASS_API __attribute__((visibility("default")))
#else
#define SDPAB_CLASS_API
#endif

namespace sdpab {
struct SdpaImpl;
struct SolveStats;
}

class SDPAB_CLASS_API SDPA {
 public:
  enum PhaseType { noINFO, pFEAS, dFEAS, pdFEAS, pdINF, pFEAS_dINF, pINF_dFEAS, pdOPT, pUNBD, dUNBD };
  enum ParameterType { PARAMETER_DEFAULT, PARAMETER_UNSTABLE_BUT_FAST, PARAMETER_STABLE_BUT_SLOW };
  enum ConeType { SDP, SOCP, LP };
  enum SparseType { AUTO, SPARSE, DENSE };

  SDPA();
  ~SDPA();
  SDPA(const SDPA&) = delete;
  SDPA& operator=(const SDPA&) = delete;

  void setParameterType(ParameterType type = PARAMETER_DEFAULT);
  void setParameterMaxIteration(SDPA_INT maxIteration);
  void setParameterEpsilonStar(double epsilonStar);
  void setParameterLambdaStar(double lambdaStar);
  void setParameterOmegaStar(double omegaStar);
  void setParameterLowerBound(double lowerBound);
  void setParameterUpperBound(double upperBound);
  void setParameterBetaStar(double betaStar);
  void setParameterBetaBar(double betaBar);
  void setParameterGammaStar(double gammaStar);
  void setParameterEpsilonDash(double epsilonDash);
  void setParameterPrintXVec(char* xPrint);
  void setParameterPrintXMat(char* XPrint);
  void setParameterPrintYMat(char* YPrint);
  void setParameterPrintInformation(char* infPrint);
  void setDisplay(FILE* Display = stdout);
  void setResultFile(FILE* fpout = stdout);
  void setInitPoint(bool isInitPoint);
  void setNumThreads(SDPA_INT NumThreads = 0);

  ParameterType getParameterType();
  SDPA_INT getParameterMaxIteration();
  double getParameterEpsilonStar();
  double getParameterLambdaStar();
  double getParameterOmegaStar();
  double getParameterLowerBound();
  double getParameterUpperBound();
  double getParameterBetaStar();
  double getParameterBetaBar();
  double getParameterGammaStar();
  double getParameterEpsilonDash();
  char* getParameterPrintXVec();
  char* getParameterPrintXMat();
  char* getParameterPrintYMat();
  char* getParameterPrintInformation();
  FILE* getDisplay();
  FILE* getResultFile();
  bool getInitPoint();
  SDPA_INT getNumThreads();

  void inputConstraintNumber(SDPA_INT m);
  void inputBlockNumber(SDPA_INT nBlock);
  void inputBlockSize(SDPA_INT l, SDPA_INT size);
  void inputBlockType(SDPA_INT l, ConeType coneType);
  void inputCVec(SDPA_INT k, double value);
  void inputElement(SDPA_INT k, SDPA_INT l, SDPA_INT i, SDPA_INT j, double value, bool inputCheck = false);
  void inputInitXVec(SDPA_INT k, double value);
  void inputInitXMat(SDPA_INT l, SDPA_INT i, SDPA_INT j, double value);
  void inputInitYMat(SDPA_INT l, SDPA_INT i, SDPA_INT j, double value);

  void initializeUpperTriangleSpace();
  void initializeUpperTriangle(bool inputTwiceCheck = false);
  void initializeSolve();
  void resetParameters();
  void solve();

  double* getResultXVec();
  double* getResultXMat(SDPA_INT l);
  double* getResultYMat(SDPA_INT l);
  double getPrimalObj();
  double getDualObj();
  double getPrimalError();
  double getDualError();
  double getDigits();
  SDPA_INT getIteration();
  double getMu();
  double getDualityGap();
  PhaseType getPhaseValue();
  void getPhaseString(char* str);
  double getSolveTime();

  SDPA_INT getConstraintNumber();
  SDPA_INT getBlockNumber();
  SDPA_INT getBlockSize(SDPA_INT l);
  ConeType getBlockType(SDPA_INT l);

  void getDimacsError(double* DimacsError);
  void printDimacsError(double* DimacsError, char* printFormat, FILE* fp = stdout);
  void printResultXVec(FILE* fp = stdout);
  void printResultXMat(FILE* fp = stdout);
  void printResultYMat(FILE* fp = stdout);
  void printComputationTime(FILE* fp = stdout);
  void printParameters(FILE* fp = stdout);
  static void printSDPAVersion(FILE* fp = stdout);

  void readInput(char* filename, FILE* fpout = NULL, SparseType type = AUTO);
  void readInit(char* filename, FILE* fpout = NULL, SparseType type = AUTO);
  void readParameter(char* filename, FILE* fpout = NULL);
  void writeInputSparse(char* filename, char* printFormat);
  void writeInitSparse(char* filename, char* printFormat);

  void terminate();
  void copyCurrentToInit();
  void setKappa(double KAPPA);

  // not in the reference: precision mode (0 = FP64, 1 = mixed: FP32 bulk
  // products and FP32 Schur factor with FP64 refinement while the relative
  // complementarity gap n*mu / max(1, mean |objective|) >= mu_switch;
  // 0 = default 1e-2)
  void setPrecision(int mode, double mu_switch = 0.0);
  // not in the reference: bound on the polls of each wait of the mixed
  // mode's tensor-core pipelines (< 0: the default bound).  A pipeline that
  // gives up falls back to the FP64 factor / SIMT products for that
  // iteration; tests use a small bound to exercise that path.
  void setTensorCoreWaitLimit(long long polls);
  // not in the reference: the error channel that replaces its exit() calls
  int getErrorCode();
  const char* getErrorMessage();
  // not in the reference: per-phase solver statistics (device seconds)
  const sdpab::SolveStats& impl_solver_stats();

 private:
  sdpab::SdpaImpl* impl_;
};

#endif  // SDPA_B200_SDPA_CALL_H
