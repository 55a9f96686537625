"""CPU oracle: a numpy restatement of the reference SDPA 7.4.4 interior-point
method for dense SDP blocks plus LP (diagonal) blocks.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg may import this module, and only as the checker.  The product
(sdpa_b200) never calls it: its solve path is the CUDA extension.

Parity pinning: this restatement is checked against the reference solver
itself, compiled from the reference sources by oracle/Makefile into
oracle/_ref/ (tests/test_oracle.py, tests/golden/), and against the known
answers the reference's manual prints for example1/example2.

Everything follows the reference's own operation sequence; each function cites
the reference file:line (paths relative to the reference's LP64/ tree).
Internal naming follows the reference (REVERSE_PRIMAL_DUAL, sdpa_tool.h:95):
the internal problem is  min C.X  s.t. A_k.X = b_k, X psd, with C = -F0,
A_k = F_k, b = c; internal X ("xMat") is the user's Y, internal Z ("zMat") is
the user's X, internal y is -x until the end of the solve.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field

import numpy as np

# Phase codes of SolveInfo (sdpa_parts.h) in the reference's enum order.
NOINFO, PFEAS, DFEAS, PDFEAS, PDINF, PFEAS_DINF, PINF_DFEAS, PDOPT, PUNBD, DUNBD = range(10)
PHASE_NAMES = ["noINFO", "pFEAS", "dFEAS", "pdFEAS", "pdINF", "pFEAS_dINF",
               "pINF_dFEAS", "pdOPT", "pUNBD", "dUNBD"]


@dataclass
class Params:
    """Parameter defaults: Parameter::setDefaultParameter (sdpa_parts.cpp:182-224)."""
    maxIteration: int = 100
    epsilonStar: float = 1.0e-7
    lambdaStar: float = 1.0e2
    omegaStar: float = 2.0
    lowerBound: float = -1.0e5
    upperBound: float = 1.0e5
    betaStar: float = 0.1
    betaBar: float = 0.2
    gammaStar: float = 0.9
    epsilonDash: float = 1.0e-7

    @staticmethod
    def read(path: str) -> "Params":
        """Parameter::readFile (sdpa_parts.cpp:231-263): 10 leading numbers, one per line."""
        vals = []
        with open(path) as f:
            for line in f:
                tok = line.split()
                if tok:
                    vals.append(tok[0])
                if len(vals) == 10:
                    break
        p = Params()
        p.maxIteration = int(float(vals[0]))
        (p.epsilonStar, p.lambdaStar, p.omegaStar, p.lowerBound, p.upperBound,
         p.betaStar, p.betaBar, p.gammaStar, p.epsilonDash) = map(float, vals[1:10])
        return p


@dataclass
class Problem:
    """An SDPA-format problem exactly as the .dat-s file states it.

    blocks: signed block sizes (negative = LP block, size 1 = LP too,
    sdpa_block.cpp:66-95).  c: the m-vector.  entries: list over k = 0..m of
    (l, i, j, v) tuples, 1-based, as in the file (k = 0 is F0).
    """
    m: int
    blocks: list
    c: np.ndarray
    entries: list = field(default_factory=list)


def parse_dats(text: str) -> Problem:
    """Sparse-format reader: IO::read (sdpa_io.cpp:33-73, :473-540).

    Comment lines start with '"' or '*'; numbers are pulled out of any
    punctuation, like the reference's '%*[^0-9+-]' scans."""
    lines = text.splitlines()
    pos = 0
    while pos < len(lines) and (not lines[pos].strip() or lines[pos].lstrip()[0] in '"*'):
        pos += 1
    rest = "\n".join(lines[pos:])
    num = re.compile(r"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eEdD][+-]?\d+)?")
    toks = [t.replace("D", "e").replace("d", "e") for t in num.findall(rest)]
    it = iter(toks)
    m = int(float(next(it)))
    nb = int(float(next(it)))
    blocks = [int(float(next(it))) for _ in range(nb)]
    c = np.array([float(next(it)) for _ in range(m)])
    entries = [[] for _ in range(m + 1)]
    rem = list(it)
    for q in range(0, len(rem) - 4, 5):
        k, l, i, j = (int(float(x)) for x in rem[q:q + 4])
        entries[k].append((l, i, j, float(rem[q + 4])))
    return Problem(m, blocks, c, entries)


class Internal:
    """Block layout after BlockStruct::makeInternalStructure (sdpa_block.cpp:66-95):
    SDP blocks (size >= 2) keep their order; LP blocks (negative size or size 1)
    are concatenated into one LP vector."""

    def __init__(self, prob: Problem):
        self.m = prob.m
        self.sdp_sizes = []
        self.map = []  # per file block: ("sdp", idx) or ("lp", offset)
        lp = 0
        for s in prob.blocks:
            if s >= 2:
                self.map.append(("sdp", len(self.sdp_sizes)))
                self.sdp_sizes.append(s)
            else:
                self.map.append(("lp", lp))
                lp += abs(s)
        self.nlp = lp
        self.nDim = sum(self.sdp_sizes) + self.nlp
        m = prob.m
        # dense copies: C = -F0, A_k = F_k (sdpa_io.cpp:511, :549)
        self.C = [np.zeros((n, n)) for n in self.sdp_sizes]
        self.Clp = np.zeros(self.nlp)
        self.A = [[np.zeros((n, n)) for n in self.sdp_sizes] for _ in range(m)]
        self.Alp = np.zeros((m, self.nlp))
        for k in range(m + 1):
            sign = -1.0 if k == 0 else 1.0
            for (l, i, j, v) in prob.entries[k]:
                kind, idx = self.map[l - 1]
                if kind == "sdp":
                    M = self.C[idx] if k == 0 else self.A[k - 1][idx]
                    M[i - 1, j - 1] += sign * v
                    if i != j:
                        M[j - 1, i - 1] += sign * v
                else:
                    if k == 0:
                        self.Clp[idx + i - 1] += sign * v
                    else:
                        self.Alp[k - 1, idx + i - 1] += v
        self.b = np.asarray(prob.c, dtype=float).copy()


# ----------------------------------------------------------------- block-space ops
def ip(As, Bs, alp=None, blp=None):
    """Frobenius inner product over all blocks (Lal::getInnerProduct, sdpa_linear.cpp:270-463)."""
    s = 0.0
    for a, b in zip(As, Bs):
        s += float(np.sum(a * b))
    if alp is not None:
        s += float(np.dot(alp, blp))
    return s


def A_dot(I: Internal, Xs, xlp):
    """multi_InnerProductToA: ret_k = A_k . X (sdpa_dataset.cpp:414-424)."""
    r = np.zeros(I.m)
    for k in range(I.m):
        r[k] = ip(I.A[k], Xs) + float(np.dot(I.Alp[k], xlp))
    return r


def A_sum(I: Internal, v):
    """multi_plusToA: sum_k A_k v_k (sdpa_dataset.cpp:427-433)."""
    out = [np.zeros((n, n)) for n in I.sdp_sizes]
    for k in range(I.m):
        for l in range(len(out)):
            out[l] += I.A[k][l] * v[k]
    lp = I.Alp.T @ v if I.nlp else np.zeros(0)
    return out, lp


def maxnorm(Ds, dlp):
    """Residuals::computeMaxNorm (sdpa_dataset.cpp:546-583)."""
    r = 0.0
    for d in Ds:
        if d.size:
            r = max(r, float(np.max(np.abs(d))))
    if dlp.size:
        r = max(r, float(np.max(np.abs(dlp))))
    return r


def chol_adjust(B):
    """Lower Cholesky with the reference's pivot rule: pivot < -1e-6 fails,
    pivot < 1e-14 is replaced by 1e100 (rATL_dpotrfL, sdpa_dpotrf.cpp:31-33,
    :218-265).  Plain right-looking column order; returns (L, ok)."""
    A = np.array(B, dtype=float, copy=True)
    n = A.shape[0]
    for j in range(n):
        d = A[j, j] - float(np.dot(A[j, :j], A[j, :j]))
        if d < -1.0e-6:
            return A, False
        if d < 1.0e-14:
            d = 1.0e100
        d = math.sqrt(d)
        A[j, j] = d
        if j + 1 < n:
            A[j + 1:, j] = (A[j + 1:, j] - A[j + 1:, :j] @ A[j, :j]) / d
    return np.tril(A), True


def chol_lapack(Xb):
    """dpotrf 'Lower' (Lal::getCholesky, sdpa_linear.cpp:465-515): fails on a
    non-positive pivot."""
    try:
        return np.linalg.cholesky(Xb), True
    except np.linalg.LinAlgError:
        return None, False


def lanczos_min_eig(L, X):
    """Lal::getMinEigen (sdpa_linear.cpp:29-143): Lanczos estimate of the
    minimum eigenvalue of L X L^T (L lower triangular), start vector all
    ones, stopping rule and error correction exactly as the reference."""
    n = X.shape[0]
    diag = np.full(n, 1.0e50)
    off = np.zeros(n)
    q = np.zeros(n)
    r = np.ones(n)
    beta = math.sqrt(n)
    mn, mn_old, err = 1.0e51, 1.0e52, 1.0e10
    k = kk = 0
    while (k < n and k < math.sqrt(n) + 10 and beta > 1.0e-16
           and (abs(mn - mn_old) > 1.0e-5 * abs(mn) + 1.0e-8
                or abs(err * beta) > 1.0e-2 * abs(mn) + 1.0e-4)):
        qold = q
        q = r * (1.0 / beta)
        w = L @ (X @ (L.T @ q))
        alpha = float(np.dot(q, w))
        diag[k] = alpha
        r = w - alpha * q
        r = r - beta * qold
        if kk >= math.sqrt(k) or k == n - 1 or k > math.sqrt(n + 9):
            kk = 0
            T = np.diag(diag[:k + 1]) + np.diag(off[:k], 1) + np.diag(off[:k], -1)
            ev, Q = np.linalg.eigh(T)
            mn_old = mn
            mn = float(ev[0])
            err = float(Q[k, 0])
        beta = math.sqrt(float(np.dot(r, r)))
        off[k] = beta
        k += 1
        kk += 1
    return mn - abs(err * beta)


def min_eig_block(Linv, D):
    """Jal::getMinEigen (sdpa_jordan.cpp:58-109): Lanczos for n > 20, otherwise
    all eigenvalues of L D L^T by dsyev on its lower triangle."""
    n = D.shape[0]
    if n > 20:
        return lanczos_min_eig(Linv, D)
    M = Linv @ (D @ Linv.T)
    return float(np.linalg.eigvalsh(M, UPLO="L")[0])


@dataclass
class Result:
    iterations: int
    phase: int            # SDPA::getPhaseValue() code
    primal_obj: float     # SDPA::getPrimalObj()
    dual_obj: float       # SDPA::getDualObj()
    xvec: np.ndarray      # SDPA::getResultXVec()
    Xmat: list            # getResultXMat per SDP block (internal Z)
    Ymat: list            # getResultYMat per SDP block (internal X)
    mu: float
    primal_error: float
    dual_error: float
    trace: list           # per iteration (mu, thetaP, thetaD, objP, objD, alphaP, alphaD, beta)


class State:
    pass


def solve(prob: Problem, param: Params | None = None, init=None, bmat_hook=None) -> Result:
    """SDPA::initializeSolve + SDPA::solve (sdpa_solve.cpp:10-43, :59-233).

    init: optional (xvec, Xmats, Ymats) warm start in USER terms (SDPA's
    inputInitXVec / inputInitXMat / inputInitYMat, sdpa_call.cpp:343-434).
    bmat_hook(iteration, B, g, dy): optional callback seeing the predictor's
    Schur matrix, right-hand side and direction (for per-iteration tests)."""
    P = param or Params()
    I = Internal(prob)
    m, nb = I.m, len(I.sdp_sizes)
    lam = P.lambdaStar
    S = State()
    if init is None:
        # Solutions::initialize (sdpa_dataset.cpp:47-74)
        X = [lam * np.eye(n) for n in I.sdp_sizes]
        Z = [lam * np.eye(n) for n in I.sdp_sizes]
        xlp = np.full(I.nlp, lam)
        zlp = np.full(I.nlp, lam)
        y = np.zeros(m)
    else:
        xv, Xu, Yu = init
        y = -np.asarray(xv, dtype=float)              # inputInitXVec stores -x
        Z = [np.array(a, dtype=float) for a in Xu[:nb]]   # user X -> internal Z
        X = [np.array(a, dtype=float) for a in Yu[:nb]]   # user Y -> internal X
        zlp = np.asarray(Xu[nb], dtype=float) if I.nlp else np.zeros(0)
        xlp = np.asarray(Yu[nb], dtype=float) if I.nlp else np.zeros(0)

    def compute_inverse():
        """Solutions::computeInverse (sdpa_dataset.cpp:117-142)."""
        ok = True
        LXi, LZi, Zi = [], [], []
        for l in range(nb):
            Lx, okx = chol_lapack(X[l])
            Lz, okz = chol_lapack(Z[l])
            if not okx or not okz:
                ok = False
                LXi.append(np.eye(X[l].shape[0])); LZi.append(np.eye(X[l].shape[0]))
                Zi.append(np.eye(X[l].shape[0]))
                continue
            lxi = np.linalg.solve(Lx, np.eye(Lx.shape[0]))
            lzi = np.linalg.solve(Lz, np.eye(Lz.shape[0]))
            LXi.append(np.tril(lxi)); LZi.append(np.tril(lzi))
            Zi.append(np.tril(lzi).T @ np.tril(lzi))
        if np.any(xlp < 0) or np.any(zlp < 0):
            ok = False
        with np.errstate(divide="ignore", invalid="ignore"):
            lxl = 1.0 / np.sqrt(xlp)
            lzl = 1.0 / np.sqrt(zlp)
            zil = 1.0 / zlp
        return ok, LXi, LZi, Zi, lxl, lzl, zil

    if init is None:
        LXi = [np.eye(n) / math.sqrt(lam) for n in I.sdp_sizes]
        LZi = [np.eye(n) / math.sqrt(lam) for n in I.sdp_sizes]
        Zi = [np.eye(n) / lam for n in I.sdp_sizes]
        lxl = np.full(I.nlp, 1.0 / math.sqrt(lam)); lzl = lxl.copy()
        zil = np.full(I.nlp, 1.0 / lam)
        mu0 = lam * lam                                   # AverageComplementarity (parts.cpp:777-781)
    else:
        mu0 = (ip(X, Z, xlp, zlp)) / I.nDim               # parts.cpp:783-789
        _, LXi, LZi, Zi, lxl, lzl, zil = compute_inverse()  # return value ignored (solve.cpp:63)
    X0 = [a.copy() for a in X]; Z0 = [a.copy() for a in Z]; x0lp = xlp.copy(); z0lp = zlp.copy()
    mu = mu0

    def residuals():
        """Residuals::compute (sdpa_dataset.cpp:585-608)."""
        rp = I.b - A_dot(I, X, xlp)
        sA, sAlp = A_sum(I, y)
        D = [I.C[l] - sA[l] - Z[l] for l in range(nb)]
        Dlp = I.Clp - sAlp - zlp
        return rp, D, Dlp, maxnorm([], rp), maxnorm(D, Dlp)

    rp, D, Dlp, nrp, nrd = residuals()
    init_nrp, init_nrd = nrp, nrd
    # RatioInitResCurrentRes::initialize (parts.cpp:838-852)
    thP = 0.0 if nrp < P.epsilonDash else 1.0
    thD = 0.0 if nrd < P.epsilonDash else 1.0
    # SolveInfo::initialize (parts.cpp:900-912)
    rho = 1.0
    etaP = etaD = P.omegaStar * I.nDim * mu0
    objP = ip(I.C, X, I.Clp, xlp)
    objD = float(np.dot(I.b, y))

    def update_check():
        """Phase::updateCheck (sdpa_parts.cpp:1150-1242)."""
        acc = P.epsilonDash
        ph = NOINFO
        if nrp <= acc:
            ph = PDFEAS if nrd <= acc else PFEAS
        if ph == NOINFO and nrd <= acc:
            ph = DFEAS
        if ph == PDFEAS:
            mean = (abs(objP) + abs(objD)) / 2.0
            gap = abs(objP - objD)
            dom = 1.0 if mean < 1.0 else mean
            if gap / dom <= P.epsilonStar:
                return PDOPT, False
        if ph == NOINFO and rho > 1.0 + 1.0e-6:
            return PDINF, False
        if ph == PFEAS:
            if objP <= -P.upperBound:
                return PUNBD, False
            if rho > 1.0 + 1.0e-6:
                return PFEAS_DINF, False
        if ph == DFEAS:
            if objD >= -P.lowerBound:
                return DUNBD, False
            if rho > 1.0 + 1.0e-6:
                return PINF_DFEAS, False
        return ph, True

    phase, _ = update_check()
    it = 0
    trace = []
    ap = ad = 0.0
    beta = P.betaStar
    while True:
        phase, cont = update_check()
        if not (cont and it < P.maxIteration):
            break
        # Switch::MehrotraPredictor (parts.cpp:733-743)
        centering = phase in (NOINFO, PFEAS, DFEAS)
        # DirectionParameter::MehrotraPredictor (parts.cpp:653-666)
        if phase == PDFEAS:
            beta = 0.0
        else:
            beta = 2.0 if not centering else P.betaBar
        dual_infeas = phase in (PFEAS, NOINFO)

        # ---- Newton::Mehrotra(PREDICTOR) (newton.cpp:2755-2809)
        # compute_rMat (newton.cpp:793-815)
        R = [beta * mu * Zi[l] - X[l] for l in range(nb)]
        Rlp = beta * mu * zil - xlp
        # Make_gVec (newton.cpp:817-883)
        if dual_infeas:
            XDZ = [X[l] @ D[l] @ Zi[l] for l in range(nb)]
            XDZlp = xlp * Dlp * zil
            W = [R[l] - XDZ[l] for l in range(nb)]
            Wlp = Rlp - XDZlp
        else:
            W, Wlp = R, Rlp
        g = -A_dot(I, W, Wlp) + rp
        # Make_bMat: B_ij = Tr(A_i X A_j Z^-1) over SDP blocks (F1/F2/F3 are
        # the same value, newton.cpp:885-1004, :1319-1403) + LP part (:2562-2602)
        B = np.zeros((m, m))
        for l in range(nb):
            G = [X[l] @ I.A[j][l] @ Zi[l] for j in range(m)]
            Af = np.stack([I.A[i][l].ravel() for i in range(m)])
            Gf = np.stack([G[j].T.ravel() for j in range(m)])
            B += Af @ Gf.T
        if I.nlp:
            B += (I.Alp * (xlp * zil)) @ I.Alp.T
        # compute_DyVec: choleskyFactorWithAdjust + solve (newton.cpp:2672-2716)
        Lb, ok = chol_adjust(B)
        if not ok:
            break
        dy = np.linalg.solve(Lb.T, np.linalg.solve(Lb, g))
        if bmat_hook is not None:
            bmat_hook(it, B, g, dy)

        def direction(R, Rlp, dy):
            # compute_DzMat (newton.cpp:2718-2732)
            sA, sAlp = A_sum(I, dy)
            dZ = [-sA[l] + (D[l] if dual_infeas else 0.0) for l in range(nb)]
            dzlp = -sAlp + (Dlp if dual_infeas else 0.0)
            # compute_DxMat (newton.cpp:2734-2752): dX = R - X dZ Z^-1, symmetrized
            dX = []
            for l in range(nb):
                t = R[l] - X[l] @ dZ[l] @ Zi[l]
                dX.append(0.5 * (t + t.T))
            dxlp = Rlp - xlp * dzlp * zil
            return dX, dxlp, dZ, dzlp

        dX, dxlp, dZ, dzlp = direction(R, Rlp, dy)

        # ---- StepLength::MehrotraPredictor (parts.cpp:435-491)
        ap = ad = 0.9
        if phase in (NOINFO, DFEAS):
            ap = min(ap, 1.0)
        else:
            if ip(I.C, dX, I.Clp, dxlp) > 0.0:
                ap = min(ap, ad)
                ap = min(ap, 1.0)
        if phase in (NOINFO, PFEAS):
            ad = min(ad, 1.0)
        else:
            if float(np.dot(I.b, dy)) < 0.0:
                ad = min(ad, ap)
                ad = min(ad, 1.0)

        # ---- DirectionParameter::MehrotraCorrector (parts.cpp:668-706)
        xv = ip(X, dZ, xlp, dzlp)
        uz = ip(dX, Z, dxlp, zlp)
        uv = ip(dX, dZ, dxlp, dzlp)
        muT = mu + (ap * uz + ad * xv + ap * ad * uv) / I.nDim
        beta = muT / mu
        if beta < 1.0:
            beta = beta * beta
        if phase == PDFEAS:
            beta = min(max(beta, P.betaStar), 1.0)
        else:
            beta = max(beta, P.betaBar)

        # ---- Newton::Mehrotra(CORRECTOR)
        R = [beta * mu * Zi[l] - X[l] - dX[l] @ dZ[l] @ Zi[l] for l in range(nb)]
        Rlp = beta * mu * zil - xlp - dxlp * dzlp * zil
        if dual_infeas:
            W = [R[l] - XDZ[l] for l in range(nb)]
            Wlp = Rlp - XDZlp
        else:
            W, Wlp = R, Rlp
        g = -A_dot(I, W, Wlp) + rp
        dy = np.linalg.solve(Lb.T, np.linalg.solve(Lb, g))
        dX, dxlp, dZ, dzlp = direction(R, Rlp, dy)

        # ---- StepLength::MehrotraCorrector (parts.cpp:493-625)
        # computeStepLength (parts.cpp:363-432)
        def step(Ls, Ds, llp, dlp):
            mn = 1.0e50
            for l in range(nb):
                mn = min(mn, min_eig_block(Ls[l], Ds[l]))
            for t in range(I.nlp):
                mn = min(mn, dlp[t] * llp[t] * llp[t])
            return -1.0 / mn if -mn > 1.0 / 100.0 else 100.0
        ap = step(LXi, dX, lxl, dxlp) * P.gammaStar
        ad = step(LZi, dZ, lzl, dzlp) * P.gammaStar
        if phase in (NOINFO, DFEAS):
            ap = min(ap, 1.0)
        else:
            if ip(I.C, dX, I.Clp, dxlp) > 0.0:
                ap = min(ap, ad)
                ap = min(ap, 1.0)
        if phase in (NOINFO, PFEAS):
            ad = min(ad, 1.0)
        else:
            if float(np.dot(I.b, dy)) < 0.0:
                ad = min(ad, ap)
                ad = min(ad, 1.0)
        if centering and phase in (NOINFO, PFEAS, DFEAS):
            xv = ip(X, dZ, xlp, dzlp)
            uz = ip(dX, Z, dxlp, zlp)
            uv = ip(dX, dZ, dxlp, dzlp)
            thmax = max((1.0 - ap) * thP, (1.0 - ad) * thD)
            muN = mu + (ap * uz + ad * xv + ap * ad * uv) / I.nDim
            while thmax * thmax * mu0 > 3.0 * muN:
                amax = 0.95 * max(ap, ad)
                ap = min(ap, amax)
                ad = min(ad, amax)
                thmax = max((1.0 - ap) * thP, (1.0 - ad) * thD)
                muN = mu + (ap * uz + ad * xv + ap * ad * uv) / I.nDim
                if ap < 1.0e-6 and ad < 1.0e-6:
                    break
        if phase == PDFEAS:
            oD = float(np.dot(I.b, y))
            oP = ip(I.C, X, I.Clp, xlp)
            incD = float(np.dot(I.b, dy)) * ad
            incP = ip(I.C, dX, I.Clp, dxlp) * ap
            with np.errstate(divide="ignore", invalid="ignore"):
                ratio = (oD - oP) / (incP - incD)
            if 0.0 < ratio < 1.0:
                ap *= ratio
                ad *= ratio

        trace.append((mu, thP, thD, objP, objD, ap, ad, beta))

        # ---- Solutions::update (sdpa_dataset.cpp:145-171)
        X = [X[l] + ap * dX[l] for l in range(nb)]
        xlp = xlp + ap * dxlp
        y = y + ad * dy
        Z = [Z[l] + ad * dZ[l] for l in range(nb)]
        zlp = zlp + ad * dzlp
        if ap < 1.0e-4 and ad < 1.0e-4:
            break
        ok, LXi, LZi, Zi, lxl, lzl, zil = compute_inverse()
        if not ok:
            break
        # RatioInitResCurrentRes::update (parts.cpp:854-863)
        if centering:
            thP = abs((1.0 - ap) * thP)
            thD = abs((1.0 - ad) * thD)
        mu = ip(X, Z, xlp, zlp) / I.nDim
        rp, D, Dlp, nrp, nrd = residuals()
        # update_exact (parts.cpp:865-882)
        thP = nrp / init_nrp if init_nrp > P.epsilonDash * 1.0e-2 else 0.0
        thD = nrd / init_nrd if init_nrd > P.epsilonDash * 1.0e-2 else 0.0
        # SolveInfo::update (parts.cpp:914-1060)
        objP = ip(I.C, X, I.Clp, xlp)
        objD = float(np.dot(I.b, y))
        x0z0 = I.nDim * mu0
        xz = I.nDim * mu
        if init is None:
            x0zM = lam * (sum(float(np.trace(a)) for a in Z) + float(np.sum(zlp)))
            xMz0 = lam * (sum(float(np.trace(a)) for a in X) + float(np.sum(xlp)))
        else:
            x0zM = ip(X0, Z, x0lp, zlp)
            xMz0 = ip(X, Z0, xlp, z0lp)
        acc = P.epsilonDash
        rho = 0.0
        if nrp <= acc and xMz0 < etaP:
            etaP = xMz0
        if nrd <= acc and x0zM < etaD:
            etaD = x0zM
        om = P.omegaStar
        if nrp > acc and nrd <= acc:
            rho = thP * x0zM / ((thP + (1.0 - thP) * om) * etaD + xz)
        if nrp <= acc and nrd > acc:
            rho = thD * xMz0 / ((thD + (1.0 - thD) * om) * etaP + xz)
        if nrp > acc and nrd > acc:
            rho = (thD * xMz0 + thP * x0zM) / ((thP * thD + om * (thP * (1.0 - thD) + (1.0 - thP) * thD)) * x0z0 + xz)
        it += 1

    # end of solve (sdpa_solve.cpp:199-211): final residuals, y -> -y, phase.reverse
    rp, D, Dlp, nrp, nrd = residuals()
    swap = {PFEAS: DFEAS, DFEAS: PFEAS, PFEAS_DINF: PINF_DFEAS, PINF_DFEAS: PFEAS_DINF,
            PUNBD: DUNBD, DUNBD: PUNBD}
    ph = swap.get(phase, phase)                          # Phase::reverse (parts.cpp:1244-1263)
    getmap = {PFEAS_DINF: PINF_DFEAS, PINF_DFEAS: PFEAS_DINF, PUNBD: DUNBD, DUNBD: PUNBD}
    ph = getmap.get(ph, ph)                              # SDPA::getPhaseValue (call.cpp:769-786)
    return Result(iterations=it, phase=ph, primal_obj=-objD, dual_obj=-objP,
                  xvec=-y, Xmat=Z, Ymat=X, mu=mu, primal_error=nrd, dual_error=nrp,
                  trace=trace)
