"""GPU test of ff_error_sums_noalloc, the error-sum entry point for callers
that cannot allocate device memory.

Such callers (a host application whose pool allocator already owns the device
memory, a time-critical loop that cannot afford cudaMalloc's implicit device
synchronisation, a plug-in that may not call the CUDA allocator) get the same
three sums as ff_error_sums, computed with partials kept in a fixed array
inside the library instead of a buffer allocated per call.  The test calls
both entry points through the C ABI, twice in a row on different fields, and
also checks that grids beyond the fixed array are refused.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12   # the tolerance of the other error-sum parity tests


def noalloc_sums(ff, n, phi, modes=None, precision=0):
    from fishfry_b200 import _lib
    _, _, xlo, dx = ff.reference_domain(n)
    nm, mp, keep = _lib.modes_array(modes)
    out = (ctypes.c_double * 3)()
    ptr = None if phi is None else phi.data_ptr()
    _lib.check(ff.lib().ff_error_sums_noalloc(_lib.int3(n), _lib.dbl3(xlo), _lib.dbl3(dx), nm, mp, precision, ptr,
                                              out, None), "ff_error_sums_noalloc")
    return [out[0], out[1], out[2]]


def test_noalloc_sums_match_allocating_entry_point(torch_cuda, ff):
    torch = torch_cuda
    n = (96, 80, 72)
    N = n[0] * n[1] * n[2]
    rng = np.random.default_rng(7)
    for call in range(2):   # two calls in a row share (and reuse) the fixed array
        phi = torch.from_numpy(rng.standard_normal(N) * (call + 1)).cuda()
        want = ff.error_sums(n, phi)
        got = noalloc_sums(ff, n, phi)
        assert np.allclose(got[:2], want[:2], rtol=RTOL, atol=0), (call, got, want)
        assert got[2] == want[2], (call, got, want)


def test_noalloc_sums_match_oracle(torch_cuda, ff, oracle):
    """The same sums from the CPU oracle's restatement of the reference's diff
    kernel (FishFry.hpp:57-101), for two fields in a row and for the phi = 0
    pass.  The fields are O(1) away from the analytic phi, so the last-bit
    differences between the device's and the host's sin/cos/exp stay far below
    the tolerance."""
    torch = torch_cuda
    rng = np.random.default_rng(11)
    for n in [(64, 48, 40), (37, 20, 11)]:
        for call in range(2):
            phi = rng.standard_normal(n) * (call + 1)
            got = noalloc_sums(ff, n, torch.from_numpy(phi.ravel()).cuda())
            want = oracle.diff_sums(phi)
            assert np.allclose(got, want, rtol=RTOL, atol=0), (n, call, got, want)
        z = noalloc_sums(ff, n, None)
        assert np.allclose(z, oracle.diff_sums(np.zeros(n)), rtol=RTOL, atol=0), (n, z)


def test_noalloc_scale_pass_and_fp32(torch_cuda, ff):
    torch = torch_cuda
    n = (64, 48, 40)
    modes = ff.modes_generate(12345, 16, 32, ff.alias_free_kaxis(n))
    # phi = 0 pass (the relative-norm scales), then an FP32 field with modes
    assert np.allclose(noalloc_sums(ff, n, None, modes), ff.error_sums(n, None, modes), rtol=RTOL, atol=0)
    phi = torch.randn(n[0] * n[1] * n[2], dtype=torch.float32, device="cuda")
    got = noalloc_sums(ff, n, phi, modes, ff.FF_FP32)
    want = ff.error_sums(n, phi, modes, ff.FF_FP32)
    assert np.allclose(got[:2], want[:2], rtol=RTOL, atol=0)
    assert got[2] == want[2]


def test_noalloc_refuses_grids_beyond_the_fixed_array(ff):
    n = (1024, 1024, 1025)   # one plane more than 2^30 points; refused before any device work
    with pytest.raises(ff.FFError) as e:
        noalloc_sums(ff, n, None)
    assert e.value.status == ff.FF_ERR_UNSUPPORTED
