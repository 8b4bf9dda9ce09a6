"""CPU tests of the boundary: the library builds, loads without a GPU and exports every
symbol include/happyray.h declares; the Python binding declares exactly those symbols."""
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "happyray.h"


def declared_symbols():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hr_[a-z0-9_]+)\s*\(", text)))


def test_header_parses():
    syms = declared_symbols()
    assert "hr_create" in syms and "hr_build" in syms and len(syms) >= 25


def test_library_exports_every_declared_symbol(hrlib):
    from happyray_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (hr_[a-z0-9_]+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for s in declared_symbols():
        assert hasattr(hrlib, s)


def test_fast_library_exports_the_same_symbols(hrlib):
    """libhappyray_b200_fast.so (the fast-arithmetic traversal) is a drop-in for the IEEE
    library: the same exported hr_* symbols."""
    from happyray_b200 import _lib
    from happyray_b200 import build as B
    if not B.OUT_FAST.exists():
        B.build(fast=True)

    def exported(p):
        out = subprocess.run(["nm", "-D", "--defined-only", str(p)], capture_output=True, text=True, check=True).stdout
        return set(re.findall(r"\bT (hr_[a-z0-9_]+)", out))

    assert exported(_lib.FAST_LIB_PATH) == exported(_lib.IEEE_LIB_PATH)
    assert set(declared_symbols()) <= exported(_lib.FAST_LIB_PATH)


def test_binding_matches_header():
    from happyray_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared_symbols()


def test_create_without_gpu_fails_cleanly(hrlib):
    """With no CUDA device hr_create returns a status, it never aborts the process."""
    from conftest import HAS_GPU
    if HAS_GPU:
        pytest.skip("a GPU is present")
    import ctypes as C
    ctx = C.c_void_p()
    st = hrlib.hr_create(C.byref(ctx), 0, None)
    assert st != 0 and not ctx.value


def test_c_header_compiles_standalone(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "happyray.h"\nint main(void){ hr_grid_info i; (void)i; return HR_OK; }\n')
    subprocess.run(["/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc", "-std=c99", "-Wall", "-Werror",
                    "-I", str(ROOT / "include"), "-c", str(src), "-o", str(tmp_path / "t.o")], check=True)


def test_probe_rejects_null_output(hrlib):
    """The L2 probe checks its output pointer before touching the device."""
    assert hrlib.hr_probe_l2_read(None, None) == 1   # HR_ERR_INVALID_ARG


@pytest.mark.gpu
def test_probe_l2_read_rate(hrlib):
    """The L2-resident read rate is a plausible bandwidth (below 500 GB/s the probe is broken)."""
    import ctypes as C
    out = C.c_double(0.0)
    assert hrlib.hr_probe_l2_read(None, C.byref(out)) == 0
    assert 500.0 < out.value < 100000.0
