"""The ILP64 build of class SDPA (libsdpa_b200_ilp64.so, SDPA_INT = int64_t,
as in the reference's ILP64 tree, ILP64/sdpa_include.h:43-45): a caller
compiled with -DSDPA_INT=int64_t links against it, and sizes or indices
beyond the int range the solver stores them in are rejected instead of
being truncated.  No device call is made."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "sdpa_b200", "_lib")

PROGRAM = r'''
#include "sdpa_call.h"
int main() {
  const int64_t big = (int64_t)1 << 33;
  { SDPA p; p.inputConstraintNumber(big); printf("m %d\n", p.getErrorCode()); }
  { SDPA p; p.setParameterMaxIteration(big); printf("maxit %d\n", p.getErrorCode()); }
  {
    SDPA p;
    p.inputConstraintNumber(2);
    p.inputBlockNumber(1);
    p.inputBlockSize(1, 3);
    p.inputBlockType(1, SDPA::SDP);
    p.inputElement(1, 1, 1, 2, 1.0);
    printf("ok %d m %lld n %lld\n", p.getErrorCode(), (long long)p.getConstraintNumber(),
           (long long)p.getBlockSize(1));
    p.inputElement(1, 1, 1, big + 2, 1.0);  /* would alias j = 2 if truncated */
    printf("j %d\n", p.getErrorCode());
  }
  { SDPA p; p.inputConstraintNumber(1); p.inputBlockNumber(1); p.inputBlockSize(1, big); printf("size %d\n", p.getErrorCode()); }
  return 0;
}
'''


def test_ilp64_library_links_and_rejects_out_of_range(tmp_path):
    lib = os.path.join(LIBDIR, "libsdpa_b200_ilp64.so")
    if not os.path.exists(lib):
        pytest.skip("libsdpa_b200_ilp64.so not built")
    src = tmp_path / "p.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "p"
    subprocess.run(["g++", "-O1", "-std=c++17", "-DSDPA_INT=int64_t", "-I" + os.path.join(ROOT, "include"),
                    str(src), "-L" + LIBDIR, "-lsdpa_b200_ilp64", "-Wl,-rpath," + LIBDIR, "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120, check=True).stdout
    lines = dict(ln.split(" ", 1) for ln in out.strip().splitlines())
    einval = "-1"
    assert lines["m"] == einval
    assert lines["maxit"] == einval
    assert lines["ok"] == "0 m 2 n 3"
    assert lines["j"] == einval
    assert lines["size"] == einval


def test_ilp64_library_exports_the_lp64_c_abi():
    """Both builds export the same C entry points (only class SDPA's
    signatures differ)."""
    lp, ilp = (os.path.join(LIBDIR, f) for f in ("libsdpa_b200.so", "libsdpa_b200_ilp64.so"))
    if not (os.path.exists(lp) and os.path.exists(ilp)):
        pytest.skip("libraries not built")
    syms = lambda p: {ln.split()[-1] for ln in subprocess.run(["nm", "-D", "--defined-only", p], capture_output=True,
                                                                text=True, check=True).stdout.splitlines()
                      if ln.split()[-1].startswith("sdpab_")}
    assert syms(lp) == syms(ilp) and len(syms(lp)) > 20
