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


def _binom(n, k):
    from math import comb
    return comb(n, k) if 0 <= k <= n else 0


def _griewank_min_forward_steps(steps, checkpoints):
    """Least number of forward steps that reverse `steps` steps with
    `checkpoints` saved states, one of them the initial state (Griewank 1992,
    Griewank & Walther 2000): t*steps - binom(checkpoints + t, t - 1), t the
    smallest repetition number with binom(checkpoints + t, t) >= steps."""
    t = 0
    while _binom(checkpoints + t, t) < steps:
        t += 1
    return t * steps - _binom(checkpoints + t, t - 1)


def test_binomial_schedule_cost_is_the_published_minimum():
    """The C library's schedule (host-only call, no GPU) recomputes exactly the
    published minimum number of forward steps, and after a forward pass that
    placed its first snapshots, the recursion restated here."""
    import solver_b200 as sb
    for snaps in range(0, 9):
        for steps in range(1, 121):
            rev, _ = sb.adjoint_schedule_cost(steps, snaps)
            s = min(snaps, steps - 1)
            assert rev == (_griewank_min_forward_steps(steps, s + 1) if steps > 1 else 0), (steps, snaps)
    # after the forward pass: D(1,s)=0, D(n,0)=n(n-1)/2, D(n,s)=min_m D(n-m,s-1)+C(m,s)
    N, S = 60, 5
    C = [[0] * (S + 1) for _ in range(N + 1)]
    D = [[0] * (S + 1) for _ in range(N + 1)]
    for n in range(2, N + 1):
        C[n][0] = D[n][0] = n * (n - 1) // 2
        for s in range(1, S + 1):
            C[n][s] = min(m + C[n - m][s - 1] + C[m][s] for m in range(1, n))
            D[n][s] = min(D[n - m][s - 1] + C[m][s] for m in range(1, n))
    for n in range(1, N + 1):
        for s in range(0, S + 1):
            assert sb.adjoint_schedule_cost(n, s) == (C[n][min(s, n - 1)], D[n][min(s, n - 1)])
    # the adjoint workloads: 512^3 x 400 steps with 14 snapshots, 128^3 x 100 with 9
    assert sb.adjoint_schedule_cost(400, 14) == (1047, 650)
    assert sb.adjoint_schedule_cost(100, 9) == (222, 125)
    with pytest.raises(ValueError, match="1 to 4096 steps"):
        sb.adjoint_schedule_cost(4097, 3)
    with pytest.raises(ValueError, match="non-negative"):
        sb.adjoint_schedule_cost(10, -1)


def test_new_entry_points_reject_a_null_context_without_touching_a_device():
    """The host-state step and the binomial adjoint validate their context
    before any CUDA call, like every other entry point."""
    import ctypes as C
    import solver_b200._capi as capi
    lib = capi.load()
    prm = capi.OfStepParams(0.01, 0.01, 1.0, 10, 1e-10, 0, 1, b"Taylor-Green")
    hp = C.c_int(0)
    st = lib.of_step_host(None, C.byref(prm), *([None] * 7), C.byref(hp), None)
    assert st == 1 and lib.of_last_error().decode() == "null context"
    info = capi.OfAdjointInfo()
    st = lib.of_adjoint_gradient_binomial(None, C.byref(prm), 4, 0, *([None] * 6), C.byref(info))
    assert st == 1 and lib.of_last_error().decode() == "null context"
