// Scalar control logic of SDPA's Mehrotra predictor-corrector loop, shared by
// the host-driven solver (sdpa_call.cpp) and the batched persistent kernel
// (batch_engine.cu).  Every function is a restatement of the reference's
// scalar code, cited by file:line (reference LP64/ tree).  Naming follows the
// reference's internal (REVERSE_PRIMAL_DUAL) convention: the internal problem
// is min C.X s.t. A_k.X = b_k, X psd; "X" is the user's Y, "Z" the user's X.
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define SDPAB_HD __host__ __device__ __forceinline__
#else
#define SDPAB_HD inline
#endif

namespace sdpab {

// Phase codes in the reference's SolveInfo enum order (sdpa_parts.h).
enum Phase { noINFO = 0, pFEAS, dFEAS, pdFEAS, pdINF, pFEAS_dINF, pINF_dFEAS, pdOPT, pUNBD, dUNBD };

struct Params {
  int maxIteration;
  double epsilonStar, lambdaStar, omegaStar, lowerBound, upperBound;
  double betaStar, betaBar, gammaStar, epsilonDash;
};

// Parameter::setDefaultParameter (sdpa_parts.cpp:182-224); type 0 = DEFAULT,
// 1 = UNSTABLE_BUT_FAST, 2 = STABLE_BUT_SLOW.
SDPAB_HD Params default_params(int type = 0)
{
  Params p;
  if (type == 2) {
    p.maxIteration = 1000; p.epsilonStar = 1.0e-7; p.lambdaStar = 1.0e4; p.omegaStar = 2.0;
    p.lowerBound = -1.0e5; p.upperBound = 1.0e5; p.betaStar = 0.1; p.betaBar = 0.3;
    p.gammaStar = 0.8; p.epsilonDash = 1.0e-7;
  } else if (type == 1) {
    p.maxIteration = 100; p.epsilonStar = 1.0e-7; p.lambdaStar = 1.0e2; p.omegaStar = 2.0;
    p.lowerBound = -1.0e5; p.upperBound = 1.0e5; p.betaStar = 0.01; p.betaBar = 0.02;
    p.gammaStar = 0.95; p.epsilonDash = 1.0e-7;
  } else {
    p.maxIteration = 100; p.epsilonStar = 1.0e-7; p.lambdaStar = 1.0e2; p.omegaStar = 2.0;
    p.lowerBound = -1.0e5; p.upperBound = 1.0e5; p.betaStar = 0.1; p.betaBar = 0.2;
    p.gammaStar = 0.9; p.epsilonDash = 1.0e-7;
  }
  return p;
}

// The scalar state the reference keeps in AverageComplementarity (mu),
// RatioInitResCurrentRes (theta), SolveInfo, Phase, Switch, DirectionParameter
// and StepLength.
struct Scalars {
  double mu0, mu;              // AverageComplementarity initial / current
  double thetaP, thetaD;       // RatioInitResCurrentRes
  double rho, etaP, etaD;      // SolveInfo
  double objP, objD;           // SolveInfo objValPrimal (C.X) / objValDual (b.y)
  double initNrp, initNrd;     // initRes.normPrimalVec / normDualMat
  double nrp, nrd;             // currentRes norms
  double beta;                 // DirectionParameter::value
  double alphaP, alphaD;       // StepLength primal / dual
  int phase;
  int centering;               // Switch: 1 = CENTERING, 0 = AFFINE
  int nDim;
};

// SolveInfo::initialize + RatioInitResCurrentRes::initialize (sdpa_parts.cpp:900-912, :838-852);
// mu0 from AverageComplementarity (:777-789).
SDPAB_HD void init_scalars(Scalars& s, const Params& p, int nDim, double mu0, double nrp,
                           double nrd, double objP, double objD)
{
  s.nDim = nDim;
  s.mu0 = s.mu = mu0;
  s.initNrp = s.nrp = nrp;
  s.initNrd = s.nrd = nrd;
  s.thetaP = (nrp < p.epsilonDash) ? 0.0 : 1.0;
  s.thetaD = (nrd < p.epsilonDash) ? 0.0 : 1.0;
  s.rho = 1.0;
  s.etaP = s.etaD = p.omegaStar * nDim * mu0;
  s.objP = objP;
  s.objD = objD;
  s.beta = p.betaStar;
  s.alphaP = s.alphaD = 0.0;
  s.phase = noINFO;
  s.centering = 1;
}

// Phase::updateCheck (sdpa_parts.cpp:1150-1242) with REVERSE_PRIMAL_DUAL.
// Returns true while the loop should continue.
SDPAB_HD bool update_check(Scalars& s, const Params& p)
{
  const double NONZERO = 1.0e-6;
  const double acc = p.epsilonDash;
  int v = noINFO;
  if (s.nrp <= acc) v = (s.nrd <= acc) ? pdFEAS : pFEAS;
  if (v == noINFO && s.nrd <= acc) v = dFEAS;
  s.phase = v;
  if (v == pdFEAS) {
    double mean = (fabs(s.objP) + fabs(s.objD)) / 2.0;
    double gap = fabs(s.objP - s.objD);
    double dom = (mean < 1.0) ? 1.0 : mean;
    if (gap / dom <= p.epsilonStar) { s.phase = pdOPT; return false; }
  }
  if (v == noINFO && s.rho > 1.0 + NONZERO) { s.phase = pdINF; return false; }
  if (v == pFEAS) {
    if (s.objP <= -p.upperBound) { s.phase = pUNBD; return false; }
    if (s.rho > 1.0 + NONZERO) { s.phase = pFEAS_dINF; return false; }
  }
  if (v == dFEAS) {
    if (s.objD >= -p.lowerBound) { s.phase = dUNBD; return false; }
    if (s.rho > 1.0 + NONZERO) { s.phase = pINF_dFEAS; return false; }
  }
  return true;
}

// Complementarity gap nDim * mu relative to the objective scale
// max(1, (|objP| + |objD|) / 2), the scale of the reference's gap test.  The
// mixed-precision modes run their FP32 products while this is at least the
// switch value (default 1e-2): the condition of X and Z grows like 1/mu, so
// the switch is tied to how far the iterate is from optimal, not to mu0
// (a warm start begins close to optimal).
SDPAB_HD double mixed_gap(const Scalars& s)
{
  const double mean = (fabs(s.objP) + fabs(s.objD)) / 2.0;
  return s.nDim * s.mu / (mean < 1.0 ? 1.0 : mean);
}

// Switch::MehrotraPredictor + DirectionParameter::MehrotraPredictor
// (sdpa_parts.cpp:733-743, :653-666).
SDPAB_HD void predictor_setup(Scalars& s, const Params& p)
{
  s.centering = (s.phase == noINFO || s.phase == pFEAS || s.phase == dFEAS) ? 1 : 0;
  if (s.phase == pdFEAS) s.beta = 0.0;
  else s.beta = s.centering ? p.betaBar : 2.0;
}

// The dual residual D enters the Newton system while the point is dual
// infeasible (Make_gVec / compute_DzMat, sdpa_newton.cpp:837-841, :2725).
SDPAB_HD bool dual_infeasible(const Scalars& s) { return s.phase == pFEAS || s.phase == noINFO; }

// Feasibility/effectiveness caps common to both step rules
// (sdpa_parts.cpp:454-490 and :521-557).  CdX = C.dX, bdy = b.dy.
SDPAB_HD void cap_steps(Scalars& s, double CdX, double bdy)
{
  if (s.phase == noINFO || s.phase == dFEAS) {
    if (s.alphaP > 1.0) s.alphaP = 1.0;
  } else if (CdX > 0.0) {
    if (s.alphaP > s.alphaD) s.alphaP = s.alphaD;
    if (s.alphaP > 1.0) s.alphaP = 1.0;
  }
  if (s.phase == noINFO || s.phase == pFEAS) {
    if (s.alphaD > 1.0) s.alphaD = 1.0;
  } else if (bdy < 0.0) {
    if (s.alphaD > s.alphaP) s.alphaD = s.alphaP;
    if (s.alphaD > 1.0) s.alphaD = 1.0;
  }
}

// StepLength::MehrotraPredictor (sdpa_parts.cpp:435-491): fixed 0.9 then caps.
SDPAB_HD void predictor_step(Scalars& s, double CdX, double bdy)
{
  s.alphaP = s.alphaD = 0.9;
  cap_steps(s, CdX, bdy);
}

// DirectionParameter::MehrotraCorrector (sdpa_parts.cpp:668-706).
// xdz = X.dZ, dxz = dX.Z, dxdz = dX.dZ of the predictor direction.
SDPAB_HD void corrector_beta(Scalars& s, const Params& p, double xdz, double dxz, double dxdz)
{
  double muT = s.mu + (s.alphaP * dxz + s.alphaD * xdz + s.alphaP * s.alphaD * dxdz) / s.nDim;
  double v = muT / s.mu;
  if (v < 1.0) v = v * v;
  if (s.phase == pdFEAS) {
    if (v < p.betaStar) v = p.betaStar;
    if (v > 1.0) v = 1.0;
  } else {
    if (v < p.betaBar) v = p.betaBar;
  }
  s.beta = v;
}

// StepLength::computeStepLength maps a minimum eigenvalue to a step bound
// (sdpa_parts.cpp:363-432, alphaBD = 100).
SDPAB_HD double step_from_min_eig(double minEig)
{
  const double alphaBD = 100.0;
  return (-minEig > 1.0 / alphaBD) ? -1.0 / minEig : alphaBD;
}

// StepLength::MehrotraCorrector (sdpa_parts.cpp:493-625).  minX / minZ are
// the minimum eigenvalues of L_X^-1 dX L_X^-T and L_Z^-1 dZ L_Z^-T; the inner
// products are of the corrector direction; objD_cur = b.y, objP_cur = C.X at
// the current point.
SDPAB_HD void corrector_step(Scalars& s, const Params& p, double minX, double minZ, double CdX,
                             double bdy, double xdz, double dxz, double dxdz, double objD_cur,
                             double objP_cur)
{
  const double xi = 3.0;
  s.alphaP = p.gammaStar * step_from_min_eig(minX);
  s.alphaD = p.gammaStar * step_from_min_eig(minZ);
  cap_steps(s, CdX, bdy);
  if (s.centering && (s.phase == noINFO || s.phase == pFEAS || s.phase == dFEAS)) {
    double thetaMax = fmax((1.0 - s.alphaP) * s.thetaP, (1.0 - s.alphaD) * s.thetaD);
    double muNew = s.mu + (s.alphaP * dxz + s.alphaD * xdz + s.alphaP * s.alphaD * dxdz) / s.nDim;
    // The reference loop ends once both steps fall below 1e-6 (each pass
    // shrinks the larger step by 0.95); the pass cap only bounds device code.
    for (int pass = 0; pass < 4096 && thetaMax * thetaMax * s.mu0 > xi * muNew; ++pass) {
      double alphaMax = 0.95 * fmax(s.alphaP, s.alphaD);
      s.alphaP = fmin(s.alphaP, alphaMax);
      s.alphaD = fmin(s.alphaD, alphaMax);
      thetaMax = fmax((1.0 - s.alphaP) * s.thetaP, (1.0 - s.alphaD) * s.thetaD);
      muNew = s.mu + (s.alphaP * dxz + s.alphaD * xdz + s.alphaP * s.alphaD * dxdz) / s.nDim;
      if (s.alphaP < 1.0e-6 && s.alphaD < 1.0e-6) break;
    }
  }
  if (s.phase == pdFEAS) {
    double incD = bdy * s.alphaD;
    double incP = CdX * s.alphaP;
    double maxRatio = (objD_cur - objP_cur) / (incP - incD);
    if (maxRatio > 0.0 && maxRatio < 1.0) {
      s.alphaP *= maxRatio;
      s.alphaD *= maxRatio;
    }
  }
}

// Solutions::update step-size test (sdpa_dataset.cpp:162-166).
SDPAB_HD bool cannot_move(const Scalars& s) { return s.alphaP < 1.0e-4 && s.alphaD < 1.0e-4; }

// After the point update: RatioInitResCurrentRes::update (sdpa_parts.cpp:854-863),
// AverageComplementarity::update (:785-790), update_exact (:865-882) and
// SolveInfo::update (:914-1060).  xz = X.Z; x0zM = X0.Z and xMz0 = X.Z0 (for
// the standard start these are lambda*tr(Z) and lambda*tr(X), :1003-1019).
SDPAB_HD void after_update(Scalars& s, const Params& p, double xz, double nrp, double nrd,
                           double objP, double objD, double x0zM, double xMz0)
{
  if (s.centering) {
    s.thetaP = fabs((1.0 - s.alphaP) * s.thetaP);
    s.thetaD = fabs((1.0 - s.alphaD) * s.thetaD);
  }
  s.mu = xz / s.nDim;
  s.nrp = nrp;
  s.nrd = nrd;
  s.thetaP = (s.initNrp > p.epsilonDash * 1.0e-2) ? nrp / s.initNrp : 0.0;
  s.thetaD = (s.initNrd > p.epsilonDash * 1.0e-2) ? nrd / s.initNrd : 0.0;
  s.objP = objP;
  s.objD = objD;
  const double th_p = s.thetaP, th_d = s.thetaD, om = p.omegaStar;
  const double x0z0 = s.nDim * s.mu0;
  const double xMzM = s.nDim * s.mu;
  const double acc = p.epsilonDash;
  s.rho = 0.0;
  if (nrp <= acc && xMz0 < s.etaP) s.etaP = xMz0;
  if (nrd <= acc && x0zM < s.etaD) s.etaD = x0zM;
  if (nrp > acc && nrd <= acc)
    s.rho = th_p * x0zM / ((th_p + (1.0 - th_p) * om) * s.etaD + xMzM);
  if (nrp <= acc && nrd > acc)
    s.rho = th_d * xMz0 / ((th_d + (1.0 - th_d) * om) * s.etaP + xMzM);
  if (nrp > acc && nrd > acc)
    s.rho = (th_d * xMz0 + th_p * x0zM) /
            ((th_p * th_d + om * (th_p * (1.0 - th_d) + (1.0 - th_p) * th_d)) * x0z0 + xMzM);
}

// Phase::reverse then SDPA::getPhaseValue (sdpa_parts.cpp:1244-1263,
// sdpa_call.cpp:769-786): the user-visible phase code (SDPA::PhaseType order).
SDPAB_HD int user_phase(int internal)
{
  int v = internal;
  switch (v) {  // Phase::reverse
    case pFEAS: v = dFEAS; break;
    case dFEAS: v = pFEAS; break;
    case pFEAS_dINF: v = pINF_dFEAS; break;
    case pINF_dFEAS: v = pFEAS_dINF; break;
    case pUNBD: v = dUNBD; break;
    case dUNBD: v = pUNBD; break;
    default: break;
  }
  switch (v) {  // getPhaseValue
    case pFEAS_dINF: return pINF_dFEAS;
    case pINF_dFEAS: return pFEAS_dINF;
    case pUNBD: return dUNBD;
    case dUNBD: return pUNBD;
    default: return v;
  }
}

}  // namespace sdpab
