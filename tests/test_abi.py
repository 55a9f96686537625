"""The C ABI library loads and exports every function declared in include/*.h
(no compute calls: runs without a GPU)."""
import ctypes
import glob
import os
import re
import subprocess

from conftest import ROOT
from sdpa_b200 import _native as N


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names |= set(re.findall(r"SDPAB_API\s+[\w\s\*]+?\b(sdpab_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 8
    lib = ctypes.CDLL(N.LIB_PATH)
    for nm in sorted(names):
        assert hasattr(lib, nm), nm
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (sdpab_\w+)", out))
    assert names <= exported


def test_binding_covers_header():
    assert declared_functions() <= {s[0] for s in N.SIGNATURES}


def test_default_and_file_params(tmp_path):
    p = N.default_params(0)
    assert p.maxIteration == 100 and p.epsilonStar == 1e-7 and p.gammaStar == 0.9
    f = tmp_path / "param.sdpa"
    f.write_text("200 maxIteration\n1.0E-8 eps\n1.0E2 lambda\n2.0 omega\n-1.0E20 lb\n1.0E20 ub\n"
                 "0.1 betaStar\n0.2 betaBar\n0.9 gamma\n1.0E-8 epsDash\n%+10.16e\n%+10.16e\n%+10.16e\n%+10.16e\n")
    q = N.read_params(str(f))
    assert q.maxIteration == 200 and q.epsilonStar == 1e-8 and q.upperBound == 1e20


def test_errors_are_codes_not_exits():
    p = N.Params()
    assert N.lib().sdpab_default_params(7, ctypes.byref(p)) == N.EINVAL
    assert N.lib().sdpab_read_params(b"/nonexistent/param.sdpa", ctypes.byref(p)) == N.EIO
    assert b"cannot open" in N.lib().sdpab_last_error()
