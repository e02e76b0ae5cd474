"""CPU tests of the multi-rank x-slab decomposition (fishfry_b200/slab.py).

The partition is checked against the reference's formulas for the task grid
(P, 1, 1) (ParisPencil.cpp:51-61, 142-258), and a whole solve runs as 2 and 3
gloo ranks: SlabPencil's orchestration and its all-to-all exchanges (the
product's host code) around a numpy stand-in for the three device phases
that uses the same buffer and block layouts as the sm_100a kernels (the
kernels themselves are checked on a GPU in test_slab_gpu.py).  The gathered
phi must match the oracle's single-grid solve.  The harness's reductions over
ranks (FishFry.hpp:153-154, :195-196, :205-228) run on gloo ranks too.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


class NumpySlabPhases:
    """The rank's three device phases on CPU tensors, with numpy's FFTs, in
    the kernels' layouts: the slab real field [i][j][k]; blocks [i - r*di]
    [j - p*djp][kh] of nhp complex values per row, block q at q * block."""

    def __init__(self, n, lo, hi, P, rank):
        from fishfry_b200.slab import SlabLayout
        self.lay = SlabLayout(n, P)
        self.rank = rank
        self.n = n
        self.dd = [2 * np.pi * (n[a] - 1) / (n[a] * (hi[a] - lo[a])) if n[a] > 1 else 0.0 for a in range(3)]

    def _blocks(self, t):
        lay = self.lay
        c = t.numpy()[:2 * lay.P * lay.block].view(np.complex128)
        return c.reshape(lay.P, lay.di, lay.djp, lay.nhp)

    def forward(self, density, potential, send, stream=None):
        lay, n = self.lay, self.n
        p0, p1 = lay.planes(self.rank)
        f = density.numpy()[:(p1 - p0) * n[1] * n[2]].reshape(p1 - p0, n[1], n[2])
        S = np.fft.fft(np.fft.rfft(f, axis=2), axis=1)
        out = self._blocks(send)
        for p in range(lay.P):
            j0, j1 = lay.rows(p)
            out[p, :p1 - p0, :j1 - j0, :lay.nh] = S[:, j0:j1, :]

    def xpass(self, pencils, send, stream=None):
        lay, n = self.lay, self.n
        j0, j1 = lay.rows(self.rank)
        pen = self._blocks(pencils).reshape(lay.P * lay.di, lay.djp, lay.nhp)[:n[0], :j1 - j0, :lay.nh]
        X = np.fft.fft(pen, axis=0)
        i = np.arange(n[0])
        j = np.arange(j0, j1)
        k = np.arange(lay.nh)
        i2 = (np.minimum(i, n[0] - i) * self.dd[0]) ** 2
        j2 = (np.minimum(j, n[1] - j) * self.dd[1]) ** 2
        k2 = (k * self.dd[2]) ** 2
        den = (i2[:, None, None] + j2[None, :, None]) + k2[None, None, :]
        with np.errstate(divide="ignore"):
            d = -1.0 / den / (n[0] * n[1] * n[2])
        d[den == 0] = 0.0
        X = np.fft.ifft(X * d, axis=0) * n[0]
        out = self._blocks(send)
        for q in range(lay.P):
            i0, i1 = lay.planes(q)
            out[q, :i1 - i0, :j1 - j0, :lay.nh] = X[i0:i1]

    def backward(self, packed, density, potential, stream=None):
        lay, n = self.lay, self.n
        p0, p1 = lay.planes(self.rank)
        pk = self._blocks(packed)
        S = np.empty((p1 - p0, n[1], lay.nh), dtype=np.complex128)
        for p in range(lay.P):
            j0, j1 = lay.rows(p)
            S[:, j0:j1, :] = pk[p, :p1 - p0, :j1 - j0, :lay.nh]
        S = np.fft.ifft(S, axis=1) * n[1]
        phi = np.fft.irfft(S, n=n[2], axis=2) * n[2]
        potential.numpy()[:phi.size] = phi.ravel()


def _solve_rank(rank, world, port, n, f_local, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from fishfry_b200.api import reference_domain
    from fishfry_b200.slab import SLAB_PHASES, SlabPencil
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        lo, hi, _, _ = reference_domain(n)
        sp = SlabPencil(n, lo, hi, (world, 1, 1), (rank, 0, 0),
                        kernels=NumpySlabPhases(n, lo, hi, world, rank))
        nb = sp.bytes()
        density = torch.zeros(nb // 8, dtype=torch.float64)
        potential = torch.zeros(nb // 8, dtype=torch.float64)
        density[:f_local.size] = torch.from_numpy(f_local.ravel())
        stamps = []
        sp.solve(nb, density, potential, stamps)
        assert [s[0] for s in stamps] == ["Total"] + SLAB_PHASES
        out.put((rank, potential[:f_local.size].numpy().reshape(f_local.shape).copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n,world", [((16, 12, 10), 2), ((30, 45, 50), 3), ((10, 9, 8), 3), ((7, 5, 6), 2)])
def test_slab_solve_on_gloo_ranks_matches_oracle(oracle, n, world):
    import torch.multiprocessing as mp

    from fishfry_b200.slab import SlabLayout
    lay = SlabLayout(n, world)
    rng = np.random.default_rng(3)
    f = rng.standard_normal(n)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = []
    for r in range(world):
        p0, p1 = lay.planes(r)
        procs.append(ctx.Process(target=_solve_rank, args=(r, world, port, n, f[p0:p1].copy(), q)))
    for p in procs:
        p.start()
    got = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    phi = np.concatenate([got[r] for r in range(world)], axis=0)
    ref = oracle.solve(f)
    assert np.linalg.norm(phi - ref) / np.linalg.norm(ref) <= 1e-12


def _reference_partition(n, P):
    """Planes and pencil rows per rank as ParisPencil.cpp computes them for the
    task grid (P, 1, 1): di (:54), djp (:61, mip = mi*mp = P), iLo/iHi (:145-147)
    and jLo/jHi (:262-263)."""
    ni, nj = n[0], n[1]
    di = (ni + P - 1) // P
    djp = (nj + P - 1) // P
    planes = [(min(r * di, ni), min(min(r * di, ni) + di, (r + 1) * di, ni)) for r in range(P)]
    rows = [(min(p * djp, nj), min(p * djp + djp, nj)) for p in range(P)]
    return di, djp, planes, rows


@pytest.mark.parametrize("n,P", [((512, 512, 512), 8), ((30, 45, 50), 4), ((10, 9, 8), 4), ((7, 7, 7), 7),
                                 ((1024, 512, 256), 3), ((100, 8, 8), 8)])
def test_partition_matches_reference_formulas(n, P):
    from fishfry_b200.slab import SlabLayout
    lay = SlabLayout(n, P)
    di, djp, planes, rows = _reference_partition(n, P)
    assert (lay.di, lay.djp) == (di, djp)
    assert [lay.planes(r) for r in range(P)] == planes
    assert [lay.rows(p) for p in range(P)] == rows
    # every plane and row is owned exactly once
    assert sum(b - a for a, b in planes) == n[0] and sum(b - a for a, b in rows) == n[1]
    # a block holds di x djp rows of nhp complex values (the reference's countI = 2*dip*djp*dhq doubles)
    assert lay.block == di * djp * (n[2] // 2 + 1)


def test_partition_refuses_too_many_ranks():
    from fishfry_b200 import FFError
    from fishfry_b200.slab import SlabLayout
    with pytest.raises(FFError):
        SlabLayout((8, 3, 8), 4)   # 3 rows cannot feed 4 ranks (main.cpp:20)


def _reduce_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from fishfry_b200.slab import phase_table_lines, reduce_phase_table, reduce_sums
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        s = reduce_sums([1.0 + rank, 10.0 * (rank + 1), [0.5, 0.25, 0.75][rank]])
        t = reduce_phase_table([2.0 + rank, 1.0 - 0.5 * rank])
        stamps = [("Total", 0.0), ("A", 1.0 + rank), ("B", 3.0)]
        lines = phase_table_lines(stamps, 2)
        out.put((rank, s, t, lines))
    finally:
        dist.destroy_process_group()


def test_harness_reductions_on_three_gloo_ranks():
    """Error sums: sum, sum, max (FishFry.hpp:153-154); phase table: min, avg,
    max over ranks (FishFry.hpp:220-222)."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 3
    procs = [ctx.Process(target=_reduce_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, s, t, lines in got:
        assert s == pytest.approx([6.0, 60.0, 0.75])
        assert t[0] == pytest.approx((2.0, 3.0, 4.0))
        assert t[1] == pytest.approx((0.0, 0.5, 1.0))
        # Total 1.5 per iteration on every rank; A = (1+rank)/2, B = (2-rank)/2 per iteration
        assert lines[1] == "Times Averaged across Iterations"
        assert lines[4].endswith("| Total") and "1.5000e+00 | 1.5000e+00 | 1.5000e+00 (100.0%)" in lines[4]
        assert "5.0000e-01 | 1.0000e+00 | 1.5000e+00 (100.0%) | A" in lines[5]
        assert "0.0000e+00 | 5.0000e-01 | 1.0000e+00 ( 66.7%) | B" in lines[6]
