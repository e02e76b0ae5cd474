"""Multi-rank solve: the x-slab decomposition, one rank per GPU.

The reference distributes the grid over an mi x mj x mk task grid of MPI ranks
and moves data between pencils with six MPI_Alltoall calls
(ParisPencil.cpp:23-75, :143-403).  On GPUs joined by NVSwitch every rank
reaches every other at full bandwidth, so this build uses the task grid
(P, 1, 1): the reference's decomposition with mi = P and mj = mk = 1
(ParisPencil.cpp:51-61), in which the z and y passes are local and only the
x pencils need an exchange:

  rank r holds planes i in [r*di, min((r+1)*di, n0)) of the real field,
      di = ceil(n0 / P)                                (ParisPencil.cpp:54)
  x pencils: rank p holds rows j in [p*djp, min((p+1)*djp, n1)) of the
      spectrum with every i, djp = ceil(n1 / P)        (ParisPencil.cpp:61)

A solve is three device phases and two all-to-all exchanges of equal blocks
of di x djp x nhp complex values (the reference's countI,
ParisPencil.cpp:236, :312):

  forward   z R2C and y forward on the rank's slab; the y pass stores each
            row j straight into the block for rank j // djp
  exchange  blocks to their ranks: each rank now holds x pencils
            S[i][j - p*djp][kh] for every i
  x         x forward, filter, x inverse (the filter uses the global j); the
            pass stores each row i straight into the block for rank i // di
  exchange  blocks back
  backward  y inverse (each row j read from the block of rank j // djp) and
            z C2R into potential

The device phases are the C-ABI's ff_slab_* calls; the exchanges are
torch.distributed all_to_all_single (NCCL between GPUs, gloo on the CPU for
tests).  The block pointers the device phases store into are explicit, so a
caller with peer-mapped memory can hand it the other ranks' receive buffers
and skip the exchanges.
"""
import ctypes
import math
import time

from . import _lib
from ._lib import FF_FP64, FFError, check, dbl3, int3, lib


class SlabLayout:
    """Partition of an n0 x n1 x n2 grid over P ranks (task grid (P, 1, 1))."""

    def __init__(self, n, nranks, precision=FF_FP64):
        n = tuple(int(x) for x in n)
        if nranks < 1:
            raise FFError(_lib.FF_ERR_INVALID, "slab: nranks = %d < 1" % nranks)
        if any(x < nranks for x in n[:2]):   # main.cpp:20 asserts n >= m per dimension
            raise FFError(_lib.FF_ERR_TASKS, "slab: %d x %d planes and rows cannot feed %d ranks" % (
                n[0], n[1], nranks))
        self.n = n
        self.P = int(nranks)
        self.precision = int(precision)
        self.nh = n[2] // 2 + 1
        # FP32 rows are padded to an even count (16-byte aligned rows), as the plan pads them
        self.nhp = self.nh if precision == FF_FP64 else (self.nh + 1) & ~1
        self.di = -(-n[0] // self.P)
        self.djp = -(-n[1] // self.P)
        self.esz = 8 if precision == FF_FP64 else 4
        self.block = self.di * self.djp * self.nhp          # complex values per (src, dst) block

    def planes(self, r):
        """Planes [lo, hi) of the real field on rank r."""
        lo = min(r * self.di, self.n[0])
        return lo, min(lo + self.di, self.n[0])

    def rows(self, p):
        """Rows [lo, hi) of the x pencils on rank p."""
        lo = min(p * self.djp, self.n[1])
        return lo, min(lo + self.djp, self.n[1])

    def local_grid(self, r):
        lo, hi = self.planes(r)
        return (hi - lo, self.n[1], self.n[2])

    def buffer_elems(self, r):
        """Real elements (FP64 or FP32) each of density and potential must hold on rank r."""
        ni, nj, nk = self.local_grid(r)
        return max(ni * nj * nk, 2 * ni * nj * self.nhp, 2 * self.P * self.block)

    def exchange_elems(self):
        """Real elements of one rank's side of an exchange (P blocks)."""
        return 2 * self.P * self.block


def exchange(send, recv, layout, group=None):
    """One all-to-all of equal blocks: recv[block q] on rank p = send[block p]
    on rank q.  send and recv are tensors of the field's real type; the first
    P blocks of each take part."""
    import torch.distributed as dist
    m = layout.exchange_elems()
    dist.all_to_all_single(recv[:m], send[:m], group=group)


# Phase names of a multi-rank solve: the reference's stamp names for the
# steps that remain with the task grid (P, 1, 1) (ParisPencil.cpp:142-424).
SLAB_PHASES = ["Real-to-complex FFT in Z + Forward FFT in Y", "Redistribute for X pencils", "X FFTs and filter",
               "Redistribute for Y pencils", "Backward FFT in Y + Complex-to-real FFT in Z"]


class SlabKernels:
    """The rank's device phases through the C ABI (ff_slab_*).  The phases
    store their blocks into a send buffer (block q at q * block_bytes), or,
    with the *_to forms, at explicit device addresses (another rank's receive
    buffer in peer memory)."""

    def __init__(self, n, lo, hi, precision, nranks, rank):
        h = ctypes.c_void_p()
        check(lib().ff_slab_create(int3(n), dbl3(lo), dbl3(hi), int(precision), int(nranks), int(rank),
                                   ctypes.byref(h)), "ff_slab_create")
        self._h = h
        self.P = nranks
        lay = (ctypes.c_int * 8)()
        nb, bb = ctypes.c_size_t(), ctypes.c_size_t()
        check(lib().ff_slab_layout(h, lay, ctypes.byref(nb), ctypes.byref(bb)), "ff_slab_layout")
        self.layout_ints = list(lay)
        self.nbytes = nb.value
        self.block_bytes = bb.value

    def _dst(self, ptrs):
        return (ctypes.c_void_p * self.P)(*[int(p) for p in ptrs])

    def _blocks(self, send):
        base = send.data_ptr()
        return [base + q * self.block_bytes for q in range(self.P)]

    def forward(self, density, potential, send, stream=None):
        self.forward_to(density, potential, self._blocks(send), stream)

    def forward_to(self, density, potential, dst, stream=None):
        check(lib().ff_slab_forward(self._h, _ptr(density), _ptr(potential), self._dst(dst), _stream(stream)),
              "ff_slab_forward")

    def xpass(self, pencils, send, stream=None):
        self.xpass_to(pencils, self._blocks(send), stream)

    def xpass_to(self, pencils, dst, stream=None):
        check(lib().ff_slab_xpass(self._h, _ptr(pencils), self._dst(dst), _stream(stream)), "ff_slab_xpass")

    def backward(self, packed, density, potential, stream=None):
        check(lib().ff_slab_backward(self._h, _ptr(packed), _ptr(density), _ptr(potential), _stream(stream)),
              "ff_slab_backward")

    def check(self, stream=None):
        check(lib().ff_slab_check(self._h, _stream(stream)), "ff_slab_check")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            check(lib().ff_slab_destroy(self._h), "ff_slab_destroy")
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(buf):
    if buf is None:
        return None
    return buf if isinstance(buf, int) else buf.data_ptr()


def _stream(stream):
    if stream is None:
        return None
    return stream if isinstance(stream, int) else stream.cuda_stream


class SlabPencil:
    """The reference's plugin interface (ParisPencil.hpp:23, :30, :44) for a
    task grid (P, 1, 1): rank id[0] of P = m[0] ranks of `group` (the default
    process group if None).  density and potential are this rank's buffers of
    at least bytes() bytes; density holds the rank's planes of f on entry
    (x slowest, as FishFry.hpp:43 indexes the local block) and potential
    receives the same planes of phi.  `kernels` supplies the device phases
    (default: the C ABI), with the same buffer layouts."""

    def __init__(self, n, lo, hi, m, id, precision=FF_FP64, group=None, kernels=None):
        import torch.distributed as dist
        m = tuple(int(x) for x in m)
        id = tuple(int(x) for x in id)
        if m[1] != 1 or m[2] != 1 or id[1] != 0 or id[2] != 0:
            raise FFError(_lib.FF_ERR_TASKS, "slab: the task grid must be (P, 1, 1); got %s" % (m,))
        P = m[0]
        if dist.is_initialized() and dist.get_world_size(group) != P:
            raise FFError(_lib.FF_ERR_TASKS, "slab: task grid %d != group size %d" % (P, dist.get_world_size(group)))
        if not 0 <= id[0] < P:
            raise FFError(_lib.FF_ERR_INVALID, "slab: rank %d outside 0..%d" % (id[0], P - 1))
        self.layout = SlabLayout(n, P, precision)
        self.rank = id[0]
        self.group = group
        self.kernels = kernels if kernels is not None else SlabKernels(n, lo, hi, precision, P, id[0])

    def bytes(self):
        return self.layout.buffer_elems(self.rank) * self.layout.esz

    def solve(self, nbytes, density, potential, stamps, stream=None):
        """One solve; stamps as the reference fills them (ParisPencil.cpp:97-424):
        ("Total", t0) and one (phase, t) per phase, host wall clock after each
        phase's device work has finished."""
        if nbytes < self.bytes():   # ParisPencil.cpp:101
            raise FFError(_lib.FF_ERR_BYTES, "slab: bytes %d < required %d" % (nbytes, self.bytes()))
        lay = self.layout
        k = self.kernels
        sync = (lambda: None) if not density.is_cuda else (lambda: _sync(density))
        stamps.clear()
        stamps.append(("Total", time.monotonic()))
        k.forward(density, potential, density, stream)
        sync()
        stamps.append((SLAB_PHASES[0], time.monotonic()))
        exchange(density, potential, lay, self.group)
        sync()
        stamps.append((SLAB_PHASES[1], time.monotonic()))
        k.xpass(potential, density, stream)
        sync()
        stamps.append((SLAB_PHASES[2], time.monotonic()))
        exchange(density, potential, lay, self.group)
        sync()
        stamps.append((SLAB_PHASES[3], time.monotonic()))
        k.backward(potential, density, potential, stream)
        sync()
        stamps.append((SLAB_PHASES[4], time.monotonic()))


def _sync(t):
    import torch
    torch.cuda.synchronize(t.device)


# ------------------------------------------------------------- harness
def reduce_sums(local, group=None):
    """The harness's reductions of the error sums to rank 0 (FishFry.hpp:153-154,
    :195-196): sum|d| and sum d^2 add, max|d| takes the maximum.  Returns the
    reduced triple on every rank (the reference's MPI_Reduce leaves it on
    rank 0 only; all ranks take the same steps here)."""
    import torch
    import torch.distributed as dist
    s = torch.tensor([float(local[0]), float(local[1])], dtype=torch.float64)
    mx = torch.tensor([float(local[2])], dtype=torch.float64)
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dev = _collective_device(group)
        s, mx = s.to(dev), mx.to(dev)
        dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(mx, op=dist.ReduceOp.MAX, group=group)
    return [float(s[0]), float(s[1]), float(mx[0])]


def reduce_phase_table(times, group=None):
    """Per-phase (min, avg, max) over ranks of the per-iteration phase times
    (FishFry.hpp:205-228: MPI_Reduce with MPI_MIN, MPI_SUM / size, MPI_MAX)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x) for x in times], dtype=torch.float64)
    lo, hi, tot = t.clone(), t.clone(), t.clone()
    size = 1
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        size = dist.get_world_size(group)
        dev = _collective_device(group)
        lo, hi, tot = lo.to(dev), hi.to(dev), tot.to(dev)
        dist.all_reduce(lo, op=dist.ReduceOp.MIN, group=group)
        dist.all_reduce(hi, op=dist.ReduceOp.MAX, group=group)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM, group=group)
    return [(float(lo[q]), float(tot[q]) / size, float(hi[q])) for q in range(len(times))]


def _collective_device(group):
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def phase_table_lines(stamps_sum, iters, group=None):
    """The harness's phase table (FishFry.hpp:201-228) from the per-rank sums
    of the stamps over the timed iterations: min / avg / max over ranks and
    the share of the total, in the reference's printf format."""
    dts = []
    for q in range(len(stamps_sum)):
        dt = stamps_sum[-1][1] - stamps_sum[0][1] if q == 0 else stamps_sum[q][1] - stamps_sum[q - 1][1]
        dts.append(dt / iters)
    rows = reduce_phase_table(dts, group)
    out = ["", "Times Averaged across Iterations", "Min Rank   | Avg Rank   | Max Rank   (%Total) | Phase",
           "--------------------------------------------------------"]
    percent = 100.0 / rows[0][2] if rows and rows[0][2] > 0 else 0.0
    for (lo, avg, hi), (name, _) in zip(rows, stamps_sum):
        out.append("%10.4e | %10.4e | %10.4e (%5.1f%%) | %s" % (lo, avg, hi, hi * percent, name))
    return out


def run_harness(solver_factory, n_tasks, n_points, iters, group=None, out=print, device=None):
    """FishFry<P>::run (FishFry.hpp:103-229) for the task grid (P, 1, 1) on
    this rank: f on the rank's planes of the reference domain, `iters` timed
    solves after one warm-up, the error norms reduced over ranks, and the
    phase table; rank 0 prints in the reference's formats.  solver_factory(n,
    lo, hi, m, id) makes the rank's solver (e.g. SlabPencil).  Returns the
    printed lines of rank 0 (empty elsewhere)."""
    import torch
    import torch.distributed as dist

    from .api import error_sums_at, init_field_at
    P = n_tasks[0]
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    n = tuple(n_points)
    dx = [2.0 * math.pi / n[a] for a in range(3)]
    lo = [-math.pi] * 3
    hi = [math.pi - dx[a] for a in range(3)]
    lines = []

    def emit(s):
        if rank == 0:
            lines.append(s)
            out(s)

    solver = solver_factory(n, lo, hi, tuple(n_tasks), (rank, 0, 0))
    lay = solver.layout
    p0, p1 = lay.planes(rank)
    local = (p1 - p0, n[1], n[2])
    xlo = [lo[0] + p0 * dx[0], lo[1], lo[2]]      # FishFry.hpp:137-139
    dev = device or torch.device("cuda", torch.cuda.current_device())
    dt = torch.float64
    nb = solver.bytes()
    f = torch.zeros(nb // 8, dtype=dt, device=dev)
    phi = torch.zeros(nb // 8, dtype=dt, device=dev)
    emit("FishFry<%s>: %dx%dx%d points over %dx%dx%d MPI processes" % (type(solver).__name__, *n, *n_tasks))
    scale = reduce_sums(error_sums_at(local, xlo, dx, None), group)
    scales = [1.0 / s if s else 0.0 for s in scale]
    total = None
    for it in range(iters + 1):
        init_field_at(local, xlo, dx, f)
        torch.cuda.synchronize(dev)
        if dist.is_initialized():
            dist.barrier(group)
        stamps = []
        solver.solve(nb, f, phi, stamps)
        t = stamps[-1][1] - stamps[0][1]
        if it == 0:
            total = [(name, 0.0) for name, _ in stamps]
        else:
            total = [(name, acc + v) for (name, acc), (_, v) in zip(total, stamps)]
        d = reduce_sums(error_sums_at(local, xlo, dx, phi), group)
        line = "%d: Time %10.4e Rate %10.4e L_1 %10.4e L_2 %10.4e L_\\inf %10.4e" % (
            it, t, n[0] * n[1] * n[2] / t, d[0] * scales[0], math.sqrt(d[1] * scales[1]), d[2] * scales[2])
        emit(line + (" (warmup, ignored)" if it == 0 else ""))
    for s in phase_table_lines(total, iters, group):
        emit(s)
    return lines
