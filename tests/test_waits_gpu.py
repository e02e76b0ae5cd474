"""GPU tests of the bounded device waits.

The fused passes (FF_PASSES=3) run z and y in one persistent launch in which
a consumer tile waits, with an iteration limit, for its plane's producer
tiles.  The test hook ff_plan_set_wait_limit shortens that limit and adds one
to the producer count each wait expects, a count that no producer ever
reaches, so every dependency wait runs out.  The kernels must return, the
plan must report FF_ERR_TIMEOUT once, and later solves must be correct again.
Nothing here faults or hangs a GPU: each wait gives up after its limit and
the block leaves without touching the plane it waited for.

The reference has no counterpart: its kernels never wait on one another and
its CHECK prints and exits (gpu.hpp:69-87).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("n", [(64, 64, 64), (30, 45, 50)])
def test_dependency_wait_runs_out_and_reports(torch_cuda, ff, oracle, n, monkeypatch):
    torch = torch_cuda
    monkeypatch.setenv("FF_PASSES", "3")
    plan = ff.Plan(n)
    assert plan.phases() == 3
    d = torch.empty(plan.nbytes // 8, dtype=torch.float64, device="cuda")
    p = torch.empty_like(d)
    N = n[0] * n[1] * n[2]
    # a target no producer reaches, and a short limit (about 0.1 ms per wait)
    plan.set_wait_limit(1024, 1)
    ff.init_field(n, d)
    with pytest.raises(ff.FFError) as e:
        plan.solve(d, p, timed=True)     # a timed solve checks the status word itself
    assert e.value.status == ff.FF_ERR_TIMEOUT
    plan.check()                         # the status word was cleared by that report
    # the same plan with the built-in limits: correct again
    plan.set_wait_limit(0, 0)
    ff.init_field(n, d)
    f = d[:N].cpu().numpy().reshape(n)
    plan.solve(d, p, timed=True)
    assert rel_l2(p[:N].cpu().numpy().reshape(n), oracle.solve(f)) <= FP64_TOL
    # and a fresh plan
    plan2 = ff.Plan(n)
    ff.init_field(n, d)
    plan2.solve(d, p)
    plan2.check()
    assert rel_l2(p[:N].cpu().numpy().reshape(n), oracle.solve(f)) <= FP64_TOL


def test_short_limit_without_a_missing_producer_is_harmless(torch_cuda, ff, oracle, monkeypatch):
    """A limit long enough for the producers that do exist: the waits end
    normally and the result is exact."""
    torch = torch_cuda
    monkeypatch.setenv("FF_PASSES", "3")
    n = (64, 48, 40)
    plan = ff.Plan(n)
    plan.set_wait_limit(1 << 22, 0)
    d = torch.empty(plan.nbytes // 8, dtype=torch.float64, device="cuda")
    p = torch.empty_like(d)
    N = n[0] * n[1] * n[2]
    ff.init_field(n, d)
    f = d[:N].cpu().numpy().reshape(n)
    plan.solve(d, p, timed=True)
    assert rel_l2(p[:N].cpu().numpy().reshape(n), oracle.solve(f)) <= FP64_TOL


def test_wait_limit_rejects_negative_arguments(ff):
    plan = ff.Plan((8, 8, 8))
    with pytest.raises(ff.FFError) as e:
        plan.set_wait_limit(-1, 0)
    assert e.value.status == ff.FF_ERR_INVALID
