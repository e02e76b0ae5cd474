"""GPU tests of the serving form (ff_server_*): results against the oracle,
the same alone as in a mix (continuous batching), admission under a tight
HBM budget, host and device inputs."""
import random
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def field(torch, ff, n, precision, seed, host=False):
    dt = torch.float64 if precision == 0 else torch.float32
    N = n[0] * n[1] * n[2]
    f = torch.empty(N, dtype=dt, device="cuda")
    ff.init_field(n, f, ff.modes_generate(seed, 16, 16, ff.alias_free_kaxis(n)), precision)
    if host:
        h = torch.empty(N, dtype=dt, pin_memory=True)
        h.copy_(f.cpu())
        return h
    return f


def solve_one(torch, ff, srv, n, precision, seed, host=False):
    f = field(torch, ff, n, precision, seed, host)
    rid = srv.submit(n, f, precision)
    srv.wait(rid)
    out = torch.empty_like(f, device="cuda")
    srv.fetch(rid, out)
    return f.double().cpu().numpy().reshape(n), out.double().cpu().numpy().reshape(n)


@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, FP32_TOL)])
@pytest.mark.parametrize("host", [False, True])
def test_server_single_request_parity(torch_cuda, ff, oracle, precision, tol, host):
    srv = ff.Server(1 << 30, max_active=16)
    try:
        for n in [(32, 48, 64), (36, 45, 50), (96, 80, 128)]:
            f, phi = solve_one(torch_cuda, ff, srv, n, precision, 5, host)
            assert rel_l2(phi, oracle.solve(f)) <= tol, n
        srv.check()
    finally:
        srv.close()


MIX = [(32, 32, 32), (48, 64, 80), (128, 96, 64), (36, 45, 50), (256, 64, 32), (60, 72, 90), (64, 64, 64),
       (512, 16, 24), (20, 30, 512), (100, 120, 81)]


def test_server_result_same_alone_and_in_mix(torch_cuda, ff):
    """Each request solved alone, then all together submitted from two threads
    at random intervals: results are bit-identical (the arithmetic of a
    request's tiles does not depend on what shares its launches)."""
    reqs = [(n, q % 2, 100 + q) for q, n in enumerate(MIX)]
    alone = []
    srv = ff.Server(1 << 31, max_active=64)
    try:
        for n, prec, seed in reqs:
            alone.append(solve_one(torch_cuda, ff, srv, n, prec, seed)[1])
        fields = [field(torch_cuda, ff, n, prec, seed) for n, prec, seed in reqs]
        torch_cuda.cuda.synchronize()
        ids = [None] * len(reqs)

        def client(part):
            rng = random.Random(part)
            for q in range(part, len(reqs), 2):
                time.sleep(rng.random() * 0.002)
                ids[q] = srv.submit(reqs[q][0], fields[q], reqs[q][1])

        th = [threading.Thread(target=client, args=(p,)) for p in (0, 1)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for q, (n, prec, seed) in enumerate(reqs):
            srv.wait(ids[q])
            out = torch_cuda.empty_like(fields[q])
            srv.fetch(ids[q], out)
            mixed = out.double().cpu().numpy().reshape(n)
            tol = FP64_TOL if prec == 0 else FP32_TOL
            assert rel_l2(mixed, alone[q]) <= tol, (q, n)
            assert np.array_equal(mixed, alone[q]), (q, n)
        st = srv.stats()
        assert st["completed"] == 2 * len(reqs)
        assert st["steps"] > 0 and st["launches"] >= st["steps"]
    finally:
        srv.close()


def test_server_admission_respects_budget(torch_cuda, ff, oracle):
    """A budget that holds two 64^3 FP64 requests (2 buffers each): ten queued
    requests all complete, never more than the budget in use."""
    n = (64, 64, 64)
    plan_bytes = 64 * 64 * 33 * 16
    budget = 2 * 2 * plan_bytes + 4096
    srv = ff.Server(budget, max_active=8)
    try:
        fields = [field(torch_cuda, ff, n, 0, s) for s in range(10)]
        ids = [srv.submit(n, f, 0) for f in fields]
        for q, rid in enumerate(ids):
            srv.wait(rid)
            out = torch_cuda.empty_like(fields[q])
            srv.fetch(rid, out)
            f = fields[q].cpu().numpy().reshape(n)
            assert rel_l2(out.cpu().numpy().reshape(n), oracle.solve(f)) <= FP64_TOL
        st = srv.stats()
        assert st["completed"] == 10
        assert st["peak_bytes"] <= budget
        assert st["max_active"] <= 2
    finally:
        srv.close()


def test_server_rejects_request_above_budget(torch_cuda, ff):
    srv = ff.Server(1 << 20, max_active=4)
    try:
        f = torch_cuda.zeros(64 * 64 * 64, dtype=torch_cuda.float64, device="cuda")
        with pytest.raises(ff.FFError) as e:
            srv.submit((64, 64, 64), f, 0)
        assert e.value.status == ff.FF_ERR_NOMEM
    finally:
        srv.close()


def test_server_wait_timeout_and_release(torch_cuda, ff):
    srv = ff.Server(1 << 28, max_active=4)
    try:
        n = (32, 32, 32)
        f = field(torch_cuda, ff, n, 1, 3)
        rid = srv.submit(n, f, 1)
        srv.wait(rid, timeout_ms=10000)
        srv.release(rid)
        with pytest.raises(ff.FFError):
            srv.wait(rid, timeout_ms=1)
    finally:
        srv.close()


def test_server_completion_queue_under_a_full_budget(torch_cuda, ff):
    """Requests taken in completion order (ff_server_next) and released at
    once: a budget that holds a few requests drains a queue of mixed sizes
    where waiting in submission order could hold memory with finished work."""
    sizes = [(128, 128, 128), (32, 32, 32), (64, 48, 40), (96, 96, 96), (40, 36, 45)] * 6
    budget = 2 * 2 * (128 * 128 * 65 * 16) + (1 << 20)
    srv = ff.Server(budget, max_active=16)
    try:
        fields = {n: field(torch_cuda, ff, n, 0, 9) for n in set(sizes)}
        ids = {srv.submit(n, fields[n], 0) for n in sizes}
        got = set()
        while len(got) < len(ids):
            rid, lat, queue, run = srv.next(timeout_ms=30000)
            assert rid in ids and rid not in got and lat >= run >= 0
            got.add(rid)
            srv.release(rid)
        st = srv.stats()
        assert st["completed"] == len(sizes) and st["peak_bytes"] <= budget
    finally:
        srv.close()


def test_server_large_requests_use_tma_tiles_and_match_oracle(torch_cuda, ff, oracle):
    """Lines of 256+ points on planes of many columns take the one-plane TMA
    tiles in the strided passes."""
    srv = ff.Server(1 << 31, max_active=8)
    try:
        for n, prec, tol in [((256, 64, 80), 0, FP64_TOL), ((40, 300, 160), 1, FP32_TOL),
                             ((270, 256, 90), 0, FP64_TOL)]:
            f, phi = solve_one(torch_cuda, ff, srv, n, prec, 21)
            assert rel_l2(phi, oracle.solve(f)) <= tol, n
    finally:
        srv.close()


@pytest.mark.parametrize("side_stream", [False, True])
def test_server_input_ordered_after_the_producing_stream(torch_cuda, ff, oracle, side_stream):
    """A device field whose last write is still queued (behind a long sleep
    kernel) when it is submitted: the server's input copy waits for it, on
    the legacy default stream by the submission's event, on another current
    stream by the wrapper's synchronisation."""
    torch = torch_cuda
    n = (64, 48, 40)
    src = field(torch, ff, n, 0, 21)
    torch.cuda.synchronize()
    srv = ff.Server(1 << 30, max_active=16)
    try:
        f = torch.zeros_like(src)
        s = torch.cuda.Stream() if side_stream else torch.cuda.default_stream()
        with torch.cuda.stream(s):
            torch.cuda._sleep(100_000_000)   # tens of milliseconds of device time
            f.copy_(src)
            rid = srv.submit(n, f, 0)
        srv.wait(rid)
        out = torch.empty_like(f)
        srv.fetch(rid, out)
        phi = out.double().cpu().numpy().reshape(n)
        ref = oracle.solve(src.double().cpu().numpy().reshape(n))
        assert rel_l2(phi, ref) <= FP64_TOL
    finally:
        srv.close()
