"""Python mirror of the reference's solver plugin and harness interface.

`ParisPencil` keeps the reference constructor / bytes() / solve() contract
(ParisPencil.hpp:23, :30, :44); `Plan` is the thinner handle over the C ABI
with precision and stream control.  Device buffers are torch CUDA tensors (or
raw device addresses as ints); torch is only the allocator and stream owner.
"""
import ctypes
import math
import time

from . import _lib
from ._lib import FF_FP32, FF_FP64, FFError, check, dbl3, int3, lib, modes_array


def _ptr(buf):
    if buf is None:
        return None
    if isinstance(buf, int):
        return buf
    return buf.data_ptr()


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def reference_domain(n):
    """(lo, hi, xlo, dx) the harness uses for one task: x = -pi + i*2*pi/n
    (FishFry.hpp:109-111, :133-139)."""
    dx = [2.0 * math.pi / n[a] if n[a] > 0 else 0.0 for a in range(3)]
    lo = [-math.pi] * 3
    hi = [math.pi - dx[a] for a in range(3)]
    return lo, hi, list(lo), dx


def phase_names(plan):
    """Names of the plan's device launches (3 fused passes, or 5 passes)."""
    h = plan.handle if isinstance(plan, Plan) else plan._plan.handle
    return [lib().ff_phase_name(h, q).decode() for q in range(lib().ff_plan_phases(h))]


class Plan:
    """A planned solve of one grid: tables resident on the current device."""

    def __init__(self, n, lo=None, hi=None, precision=FF_FP64):
        n = [int(x) for x in n]
        if lo is None:
            lo, hi, _, _ = reference_domain(n)
        h = ctypes.c_void_p()
        check(lib().ff_plan_create(int3(n), dbl3(lo), dbl3(hi), int(precision), ctypes.byref(h)), "ff_plan_create")
        self._h = h
        self.n = tuple(n)
        self.precision = int(precision)
        b = ctypes.c_size_t()
        check(lib().ff_plan_bytes(h, ctypes.byref(b)), "ff_plan_bytes")
        self.nbytes = b.value

    @property
    def handle(self):
        return self._h

    def bytes(self):
        return self.nbytes

    def solve(self, density, potential, stream=None, nbytes=None, timed=False):
        """Enqueue the five passes; returns per-pass ms (and waits) if timed."""
        times = _lib.PhaseTimes() if timed else None
        nb = self.nbytes if nbytes is None else int(nbytes)
        check(lib().ff_solve(self._h, nb, _ptr(density), _ptr(potential), _stream(stream),
                             ctypes.byref(times) if timed else None), "ff_solve")
        if timed:
            return list(times.ms)[:times.count], times.total_ms
        return None

    def solve_passes(self, density, potential, passes, stream=None):
        """Enqueue only the first `passes` (1..5) passes (ff_solve_passes)."""
        check(lib().ff_solve_passes(self._h, self.nbytes, _ptr(density), _ptr(potential), _stream(stream),
                                    int(passes)), "ff_solve_passes")

    def phases(self):
        return lib().ff_plan_phases(self._h)

    def check(self, stream=None):
        """Raises FFError(FF_ERR_TIMEOUT) if a kernel's bounded wait gave up."""
        check(lib().ff_plan_check(self._h, _stream(stream)), "ff_plan_check")

    def set_wait_limit(self, iterations=0, target_extra=0):
        """Test hook (ff_plan_set_wait_limit): iteration limit of the bounded
        device waits (0: built-in) and an extra producer count added to the
        fused passes' dependency waits (1 makes them run out)."""
        check(lib().ff_plan_set_wait_limit(self._h, int(iterations), int(target_extra)), "ff_plan_set_wait_limit")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            check(lib().ff_plan_destroy(self._h), "ff_plan_destroy")
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent grids solved together: five persistent launches (one
    per pass) over the tiles of all grids, captured once in a CUDA graph.

    dims: list of (ni, nj, nk); lo/hi: per-grid bounds or None for the
    reference domain of each grid.
    """

    def __init__(self, dims, precision=FF_FP64, lo=None, hi=None):
        dims = [tuple(int(x) for x in d) for d in dims]
        cnt = len(dims)
        flat = (ctypes.c_int * (3 * cnt))(*[x for d in dims for x in d])
        lo_a = hi_a = None
        if lo is not None:
            lo_a = (ctypes.c_double * (3 * cnt))(*[float(x) for v in lo for x in v])
            hi_a = (ctypes.c_double * (3 * cnt))(*[float(x) for v in hi for x in v])
        h = ctypes.c_void_p()
        check(lib().ff_batch_create(cnt, flat, lo_a, hi_a, int(precision), ctypes.byref(h)), "ff_batch_create")
        self._h = h
        self.dims = dims
        self.precision = int(precision)
        self.nbytes = []
        for g in range(cnt):
            b = ctypes.c_size_t()
            check(lib().ff_batch_bytes(h, g, ctypes.byref(b)), "ff_batch_bytes")
            self.nbytes.append(b.value)

    def __len__(self):
        return len(self.dims)

    @staticmethod
    def _ptrs(bufs):
        return (ctypes.c_void_p * len(bufs))(*[_ptr(b) for b in bufs])

    def solve(self, density, potential, stream=None, timed=False):
        """Enqueue the batch solve; with timed, waits and returns (per-pass ms, total ms)."""
        times = _lib.PhaseTimes() if timed else None
        self._keep = (self._ptrs(density), self._ptrs(potential))
        check(lib().ff_batch_solve(self._h, self._keep[0], self._keep[1], _stream(stream),
                                   ctypes.byref(times) if timed else None), "ff_batch_solve")
        if timed:
            return list(times.ms)[:times.count], times.total_ms
        return None

    def tune(self, density, potential, stream=None, reps=3):
        """Autotune the tile shapes (overwrites the buffers)."""
        d, p = self._ptrs(density), self._ptrs(potential)
        check(lib().ff_batch_tune(self._h, d, p, _stream(stream), int(reps)), "ff_batch_tune")

    def shape(self, index, kind):
        """(W, ct, tma) of pass `kind` of grid `index`."""
        W, ct, tma = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().ff_batch_shape(self._h, int(index), int(kind), ctypes.byref(W), ctypes.byref(ct),
                                   ctypes.byref(tma)), "ff_batch_shape")
        return W.value, ct.value, tma.value

    def radices(self, index, axis):
        """Radix split (DIF stage order) of grid `index` on axis 0=x, 1=y, 2=z."""
        r = (ctypes.c_int * 16)()
        cnt = ctypes.c_int()
        check(lib().ff_batch_radices(self._h, int(index), int(axis), r, ctypes.byref(cnt)), "ff_batch_radices")
        return list(r)[:cnt.value]

    def check(self, stream=None):
        check(lib().ff_batch_check(self._h, _stream(stream)), "ff_batch_check")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            check(lib().ff_batch_destroy(self._h), "ff_batch_destroy")
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Request loop with continuous batching (ff_server_*): submit solves of
    mixed sizes and precisions; each result is ready after `wait`.

    hbm_budget: bytes of device memory for request buffers; max_active:
    requests on the device at once per precision.
    """

    def __init__(self, hbm_budget, max_active=1024):
        cfg = _lib.ServerConfig(int(hbm_budget), int(max_active))
        h = ctypes.c_void_p()
        check(lib().ff_server_create(ctypes.byref(cfg), ctypes.byref(h)), "ff_server_create")
        self._h = h
        self._inputs = {}

    def submit(self, n, f, precision=FF_FP64, on_host=None):
        """Queue a solve of field f (torch tensor on the device or pinned host
        tensor, or an int device address); returns the request id.  f is kept
        alive until the request is fetched or released.  The server's copy of f
        is ordered after the work on the legacy default stream; a tensor made
        on another current stream has that stream synchronised first."""
        if on_host is None:
            on_host = not isinstance(f, int) and not f.is_cuda
        if not isinstance(f, int) and f.is_cuda:
            import torch
            cs = torch.cuda.current_stream(f.device)
            if cs.cuda_stream != 0:
                cs.synchronize()
        rid = ctypes.c_uint64()
        check(lib().ff_server_submit(self._h, int3(n), int(precision), _ptr(f), int(bool(on_host)), ctypes.byref(rid)),
              "ff_server_submit")
        self._inputs[rid.value] = f
        return rid.value

    def wait(self, rid, timeout_ms=-1.0):
        """Blocks until request rid is done; returns (latency, queue, run) ms."""
        info = _lib.RequestInfo()
        check(lib().ff_server_wait(self._h, int(rid), float(timeout_ms), ctypes.byref(info)), "ff_server_wait")
        return info.latency_ms, info.queue_ms, info.run_ms

    def next(self, timeout_ms=-1.0):
        """(id, latency, queue, run ms) of the next finished request (completion order)."""
        rid = ctypes.c_uint64()
        info = _lib.RequestInfo()
        check(lib().ff_server_next(self._h, float(timeout_ms), ctypes.byref(rid), ctypes.byref(info)),
              "ff_server_next")
        return rid.value, info.latency_ms, info.queue_ms, info.run_ms

    def fetch(self, rid, out=None, on_host=None):
        """Copies the potential into `out` (device or host tensor; None: drop) and releases the request."""
        if on_host is None:
            on_host = out is not None and not isinstance(out, int) and not out.is_cuda
        check(lib().ff_server_fetch(self._h, int(rid), _ptr(out), int(bool(on_host))), "ff_server_fetch")
        self._inputs.pop(rid, None)

    def release(self, rid):
        check(lib().ff_server_release(self._h, int(rid)), "ff_server_release")
        self._inputs.pop(rid, None)

    def stats(self):
        r = _lib.ServerReport()
        check(lib().ff_server_stats(self._h, ctypes.byref(r)), "ff_server_stats")
        return {k: getattr(r, k) for k, _ in r._fields_}

    def reset_stats(self):
        check(lib().ff_server_reset_stats(self._h), "ff_server_reset_stats")

    def check(self):
        check(lib().ff_server_check(self._h), "ff_server_check")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            check(lib().ff_server_destroy(self._h), "ff_server_destroy")
            self._h = ctypes.c_void_p()
            self._inputs.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ParisPencil:
    """The reference plugin interface (ParisPencil.hpp:11-59) on one GPU.

    n: global points; lo/hi: physical bounds (hi one cell short of the period);
    m: task grid, must be (1,1,1); id: task coordinates, (0,0,0).
    """

    def __init__(self, n, lo, hi, m=(1, 1, 1), id=(0, 0, 0)):
        if tuple(m) != (1, 1, 1) or tuple(id) != (0, 0, 0):
            raise FFError(_lib.FF_ERR_TASKS, "ParisPencil: one task on one GPU (m must be 1x1x1)")
        self._plan = Plan(n, lo, hi, FF_FP64)

    def bytes(self):
        return self._plan.nbytes

    def solve(self, bytes, density, potential, stamps):
        """Overwrites `stamps` with [("Total", t0), (phase, t), ...]; blocks
        until done.  As in the reference (ParisPencil.cpp:98, :424) the last
        stamp minus the first is the host wall time of the whole solve; the
        phases in between are placed by their CUDA-event durations."""
        stamps.clear()
        t0 = time.monotonic()
        stamps.append(("Total", t0))
        ms, _ = self._plan.solve(density, potential, nbytes=bytes, timed=True)
        t1 = time.monotonic()
        t = t0
        names = phase_names(self._plan)
        for q, (name, dt) in enumerate(zip(names, ms)):
            t += 1e-3 * dt
            stamps.append((name, max(t, t1) if q + 1 == len(ms) else t))


def init_field_at(n, xlo, dx, f, modes=None, precision=FF_FP64, stream=None):
    """f on the device for the n points x = xlo + i*dx (per axis): one rank's
    block of the harness's field (FishFry.hpp:22-44, :137-139)."""
    nm, mp, keep = modes_array(modes)
    check(lib().ff_init_field(int3(n), dbl3(xlo), dbl3(dx), nm, mp, int(precision), _ptr(f), _stream(stream)),
          "ff_init_field")


def error_sums_at(n, xlo, dx, phi, modes=None, precision=FF_FP64, stream=None):
    """{sum|d|, sum d^2, max|d|} over the n points x = xlo + i*dx (one rank's
    block; FishFry.hpp:57-101)."""
    nm, mp, keep = modes_array(modes)
    out = (ctypes.c_double * 3)()
    check(lib().ff_error_sums(int3(n), dbl3(xlo), dbl3(dx), nm, mp, int(precision), _ptr(phi), out,
                              _stream(stream)), "ff_error_sums")
    return [out[0], out[1], out[2]]


def init_field(n, f, modes=None, precision=FF_FP64, stream=None):
    """f on the device: analytic right-hand side (FishFry.hpp:22-44) + modes."""
    _, _, xlo, dx = reference_domain(n)
    nm, mp, keep = modes_array(modes)
    check(lib().ff_init_field(int3(n), dbl3(xlo), dbl3(dx), nm, mp, int(precision), _ptr(f), _stream(stream)),
          "ff_init_field")


def error_sums(n, phi, modes=None, precision=FF_FP64, stream=None):
    """{sum|d|, sum d^2, max|d|} against the analytic phi (FishFry.hpp:57-101)."""
    _, _, xlo, dx = reference_domain(n)
    nm, mp, keep = modes_array(modes)
    out = (ctypes.c_double * 3)()
    check(lib().ff_error_sums(int3(n), dbl3(xlo), dbl3(dx), nm, mp, int(precision), _ptr(phi), out,
                              _stream(stream)), "ff_error_sums")
    return [out[0], out[1], out[2]]


def rel_norms(n, phi, modes=None, precision=FF_FP64, stream=None):
    """Relative L1, L2, Linf as the harness prints them (FishFry.hpp:156-158, :198)."""
    s = error_sums(n, None, modes, precision, stream)
    d = error_sums(n, phi, modes, precision, stream)
    return [d[0] / s[0], math.sqrt(d[1] / s[1]), d[2] / s[2]]


def modes_generate(seed, count, kmax=32, kaxis=(32, 32, 32), sigma=0.1):
    arr = (_lib.Mode * max(count, 1))()
    check(lib().ff_modes_generate(ctypes.c_uint64(seed), int(count), int(kmax), int3(kaxis), float(sigma),
                                  ctypes.cast(arr, ctypes.c_void_p)), "ff_modes_generate")
    return [(m.kx, m.ky, m.kz, m.a, m.theta) for m in arr[:count]]


def alias_free_kaxis(n, kmax=32):
    """Largest |k_axis| kept below n_axis/2 so the analytic comparison is alias-free."""
    return tuple(max(0, min(kmax, (int(x) - 1) // 2)) for x in n)
