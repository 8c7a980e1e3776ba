"""The C-ABI library: it loads, exports every entry point include/*.h declares,
and refuses to run without a GPU (there is no CPU fallback)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("orchard_b200.h", "orchard_b200_cases.h")]
LIB = os.path.join(ROOT, "solver_b200", "liborchard_b200.so")


def declared_symbols():
    names = set()
    for header in HEADERS:
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(of_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "solver_b200")])
    out = subprocess.check_output(["nm", "-D", "--defined-only", LIB]).decode()
    exported = set(re.findall(r"\bT (of_[a-z0-9_]+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    import solver_b200._capi as capi
    import solver_b200.cases as cases
    assert set(capi.EXPORTED_SYMBOLS) <= exported
    assert set(cases.CASE_SYMBOLS) <= exported
    assert set(declared_symbols()) <= set(capi.EXPORTED_SYMBOLS) | set(cases.CASE_SYMBOLS)


def test_library_loads_and_reports_abi_version():
    import solver_b200._capi as capi
    assert capi.load().of_abi_version() == 1


def test_no_cpu_fallback_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import solver_b200 as sb
    with pytest.raises(sb.OfError, match="no CUDA device"):
        sb.Context(sb.Grid(4, 4, 4, 1.0, 1.0, 1.0), [sb.PERIODIC] * 6)
    import solver_b200.cases as cases
    with pytest.raises(sb.OfError, match="no CUDA device"):
        cases.TaylorGreenCase(cases.TaylorGreenConfig(nx=8, ny=8))
