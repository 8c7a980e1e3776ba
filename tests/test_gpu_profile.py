"""The coarse-level chain timing (of_profile_coarse_chain) on the GPU.

The bench times the V-cycle's coarse levels by replaying a CUDA graph of that
chain alone between steps.  Its contract: a positive time, the chain's launch
count, and no effect on later solves -- the replays rerun levels 1 ..
coarsest on the level-1 rhs of the last solve, and every value they write is
overwritten by the next solve's own V-cycles before it is read.  So a run
with replays between its steps must equal, bit for bit, the same run without
them.
"""
import numpy as np
import pytest

import solver_b200 as sb

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p")


def _run(n, precision, profile):
    h = 2 * np.pi / n
    ctx = sb.Context(sb.Grid(n, n, n, h, h, h), [sb.PERIODIC] * 6, precision=precision)
    try:
        dt = 0.5 / (3.0 / h)
        ctx.tg_init(1.0 / 1600, dt, 1)
        prm = sb.step_params(1.0 / 1600, dt, 400, 1e-12)
        ctx.run_steps(prm, 2)
        chain = sb.profile_coarse_chain(ctx, 20) if profile else None
        m = ctx.run_steps(prm, 2)
        return ctx.download_state(), m, chain
    finally:
        ctx.close()


@pytest.mark.parametrize("precision", [sb.OF_FP64, sb.OF_MIXED])
def test_coarse_chain_replays_leave_the_run_bitwise_unchanged(precision):
    ref, m_ref, _ = _run(64, precision, False)
    out, m, (us, launches) = _run(64, precision, True)
    assert us > 0.0 and launches >= 1
    assert m["pressure_iterations"] == m_ref["pressure_iterations"]
    for f in FIELDS:
        assert np.array_equal(np.asarray(out[f]), np.asarray(ref[f])), f
