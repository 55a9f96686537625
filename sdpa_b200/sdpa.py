"""Python mirror of the drop-in SDPA class (include/sdpa_call.h) through the
whole-problem C ABI (sdpab_sdpa_*).  Method names follow the reference's
class SDPA (sdpa_call.h:91-267); indices are 1-based; errors raise
SolverError instead of exiting."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .instances import Instance

PHASES = N.PHASES


class SDPA:
    AUTO, SPARSE, DENSE = 0, 1, 2

    def __init__(self):
        self._lib = N.lib()
        self._h = self._lib.sdpab_sdpa_new()
        if not self._h:
            raise N.SolverError("sdpab_sdpa_new failed")
        self.params = N.default_params(0)

    def __del__(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            self._lib.sdpab_sdpa_free(h)

    # parameters (SDPA::setParameterType / setParameter* / readParameter)
    def setParameterType(self, kind: int = 0):
        self.params = N.default_params(kind)

    def setParameter(self, **kw):
        for k, v in kw.items():
            setattr(self.params, k, v)

    def setPrecision(self, mode: int, mu_switch: float = 0.0):
        """0 = FP64, 1 = mixed (FP32 products and Schur factor + FP64 refinement while
        the relative complementarity gap n*mu / max(1, mean |objective|) >= mu_switch;
        0 = default 1e-2)."""
        N.check(self._lib.sdpab_sdpa_set_precision(self._h, mode, mu_switch), "setPrecision")

    def setTensorCoreWaitLimit(self, polls: int):
        """Polls per wait of the mixed mode's tensor-core pipelines (< 0: the
        default bound); a pipeline that gives up falls back for that iteration."""
        N.check(self._lib.sdpab_sdpa_set_tc_wait(self._h, int(polls)), "setTensorCoreWaitLimit")

    def tensorCoreTimeouts(self) -> int:
        """Tensor-core pipelines that gave up during the last solve."""
        out = ctypes.c_int()
        N.check(self._lib.sdpab_sdpa_tc_timeouts(self._h, ctypes.byref(out)), "tensorCoreTimeouts")
        return out.value

    def readParameter(self, path: str):
        self.params = N.read_params(path)

    # input
    def readInput(self, path: str, sparse_type: int = 0):
        N.check(self._lib.sdpab_sdpa_read_input(self._h, path.encode(), sparse_type), "readInput")

    def readInit(self, path: str, sparse_type: int = 0):
        N.check(self._lib.sdpab_sdpa_read_init(self._h, path.encode(), sparse_type), "readInit")

    def inputProblem(self, inst: Instance):
        """inputConstraintNumber / inputBlockNumber / inputBlockSize / inputCVec /
        inputElement / initializeUpperTriangle for a whole Instance."""
        bs = np.ascontiguousarray(inst.blocks, np.int32)
        c = np.ascontiguousarray(inst.c, np.float64)
        arr = [np.ascontiguousarray(a, t) for a, t in ((inst.k, np.int32), (inst.l, np.int32),
                                                      (inst.i, np.int32), (inst.j, np.int32),
                                                      (inst.v, np.float64))]
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        N.check(self._lib.sdpab_sdpa_input_problem(self._h, inst.m, len(inst.blocks), p(bs), p(c),
                                                   arr[0].size, *[p(a) for a in arr]), "inputProblem")

    def setInitPoint(self, xvec, X, Y):
        """inputInitXVec / inputInitXMat / inputInitYMat: X[l], Y[l] dense per SDP block
        (user X and Y), vectors per LP block."""
        xv = np.ascontiguousarray(xvec, np.float64)
        Xs = [np.asfortranarray(np.asarray(a, np.float64)) for a in X]
        Ys = [np.asfortranarray(np.asarray(a, np.float64)) for a in Y]
        PX = (ctypes.c_void_p * len(Xs))(*[a.ctypes.data for a in Xs])
        PY = (ctypes.c_void_p * len(Ys))(*[a.ctypes.data for a in Ys])
        N.check(self._lib.sdpab_sdpa_set_init(self._h, xv.ctypes.data_as(ctypes.c_void_p), PX, PY),
                "setInitPoint")

    def copyCurrentToInit(self):
        N.check(self._lib.sdpab_sdpa_copy_current_to_init(self._h), "copyCurrentToInit")

    # solve (initializeSolve + solve)
    def solve(self):
        N.check(self._lib.sdpab_sdpa_set_params(self._h, ctypes.byref(self.params)), "setParameter")
        N.check(self._lib.sdpab_sdpa_solve(self._h), "solve")
        self._info = N.SdpaInfo()
        N.check(self._lib.sdpab_sdpa_info(self._h, ctypes.byref(self._info)), "info")

    # results
    def info(self) -> N.SdpaInfo:
        return self._info

    def getPrimalObj(self):
        return self._info.primal_obj

    def getDualObj(self):
        return self._info.dual_obj

    def getIteration(self):
        return self._info.iterations

    def getPhaseValue(self):
        return self._info.phase

    def getPhaseString(self):
        return PHASES[self._info.phase]

    def getResultXVec(self) -> np.ndarray:
        out = np.zeros(self._info.m)
        N.check(self._lib.sdpab_sdpa_get_xvec(self._h, out.ctypes.data_as(ctypes.c_void_p)), "getResultXVec")
        return out

    def _block(self, l: int, which: int) -> np.ndarray:
        n, sdp = ctypes.c_int(), ctypes.c_int()
        N.check(self._lib.sdpab_sdpa_block_size(self._h, l, ctypes.byref(n), ctypes.byref(sdp)), "block")
        size = n.value * n.value if sdp.value else n.value
        out = np.zeros(size)
        N.check(self._lib.sdpab_sdpa_get_block(self._h, l, which, out.ctypes.data_as(ctypes.c_void_p)),
                "getResult")
        return out.reshape(n.value, n.value, order="F") if sdp.value else out

    def getResultXMat(self, l: int) -> np.ndarray:
        return self._block(l, 0)

    def getResultYMat(self, l: int) -> np.ndarray:
        return self._block(l, 1)

    PHASE_NAMES = ["rMat+gVec", "bMat", "Cholesky", "solve", "dXdZ", "StepLength", "update", "residuals"]

    def schurPattern(self):
        """(sparse, pairs updated, pairs of the dense factorisation) of the
        last solve's Schur factorisation (tiles of 128 x 128)."""
        sp = ctypes.c_int(0)
        pr = np.zeros(2, np.int64)
        N.check(self._lib.sdpab_sdpa_schur_pattern(self._h, ctypes.byref(sp), pr.ctypes.data_as(ctypes.c_void_p)),
                "schurPattern")
        return bool(sp.value), int(pr[0]), int(pr[1])

    def phaseTimes(self) -> dict:
        """Device seconds per solver phase (ComputeTime categories)."""
        out = np.zeros(8)
        N.check(self._lib.sdpab_sdpa_phase_times(self._h, out.ctypes.data_as(ctypes.c_void_p)), "phaseTimes")
        return dict(zip(self.PHASE_NAMES, out.tolist()))

    def getDimacsError(self) -> np.ndarray:
        out = np.zeros(7)
        N.check(self._lib.sdpab_sdpa_dimacs(self._h, out.ctypes.data_as(ctypes.c_void_p)), "getDimacsError")
        return out

    def writeInitSparse(self, path: str):
        N.check(self._lib.sdpab_sdpa_write_init(self._h, path.encode()), "writeInitSparse")
