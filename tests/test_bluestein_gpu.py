"""GPU tests of axes whose length has a prime factor of 7 or above.

cuFFT, which the reference calls for its line transforms, accepts any length.
Here factors of 7 run direct radix-7 stages, and an axis with a prime factor
above 7 runs through the Bluestein passes (an M-point circular convolution,
M = 2^a 3^b 5^c 7^d >= 2n - 1).  Checked against the CPU oracle (its FFT
takes every length: a direct DFT for prime factors above 5), against
golden vectors the reference itself wrote on a B200 (tests/golden/), and
against exact single-mode solutions.

FP64 bar: 1e-12 relative L2; FP32 bar: 1e-5 relative L2 against the FP64 oracle.
"""
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def smooth235(n):
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def solve(torch, ff, f, precision=0, lo=None, hi=None):
    n = f.shape
    plan = ff.Plan(n, lo, hi, precision=precision) if lo is not None else ff.Plan(n, precision=precision)
    dt = torch.float64 if precision == 0 else torch.float32
    esz = 8 if precision == 0 else 4
    d = torch.zeros(plan.nbytes // esz, dtype=dt, device="cuda")
    p = torch.empty_like(d)
    d[:f.size] = torch.from_numpy(f.ravel()).to(dt).cuda()
    plan.solve(d, p)
    return p[:f.size].double().cpu().numpy().reshape(n)


# prime factors of 7 and above on one, two or three axes, with compile-time (64,
# 128, 256, 512), runtime and one-point axes beside them, and the largest
# padded length (1789 -> M = 3600)
SIZES = [(7, 8, 8), (8, 8, 11), (7, 11, 13), (14, 9, 22), (33, 34, 35), (127, 64, 64), (64, 127, 64),
         (64, 64, 127), (97, 60, 49), (1009, 4, 6), (4, 1789, 3), (5, 3, 1789), (49, 121, 26), (101, 256, 8),
         (8, 101, 512), (128, 12, 101), (1, 7, 1), (13, 1, 2), (2, 2, 17)]


@pytest.mark.parametrize("n", SIZES)
def test_fp64_parity_with_oracle(torch_cuda, ff, oracle, n):
    assert not all(smooth235(x) for x in n)
    rng = np.random.default_rng(sum(n))
    f = rng.standard_normal(n)
    phi = solve(torch_cuda, ff, f)
    assert rel_l2(phi, oracle.solve(f)) <= FP64_TOL, n


# 2^a 3^b 5^c 7^d axes (direct radix-7 stages), up to 1792 = 2^8 * 7 points
RADIX7 = [(448, 7, 12), (14, 343, 8), (28, 49, 196), (1792, 2, 4), (6, 5, 1792), (21, 35, 63), (112, 224, 56)]


@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, FP32_TOL)])
@pytest.mark.parametrize("n", RADIX7)
def test_radix7_axes_match_oracle(torch_cuda, ff, oracle, n, precision, tol):
    rng = np.random.default_rng(7 * sum(n) + precision)
    f = rng.standard_normal(n)
    if precision:
        f = f.astype(np.float32).astype(np.float64)
    phi = solve(torch_cuda, ff, f, precision=precision)
    assert rel_l2(phi, oracle.solve(f)) <= tol, n


@pytest.mark.parametrize("n", [(7, 11, 13), (97, 60, 49), (64, 127, 64), (4, 1789, 3), (33, 34, 35)])
def test_fp32_parity_with_oracle(torch_cuda, ff, oracle, n):
    rng = np.random.default_rng(3 * sum(n))
    f = rng.standard_normal(n).astype(np.float32).astype(np.float64)
    phi = solve(torch_cuda, ff, f, precision=1)
    assert rel_l2(phi, oracle.solve(f)) <= FP32_TOL, n


@pytest.mark.parametrize("n", [(31, 37, 41), (127, 64, 49), (17, 19, 23)])
def test_reference_field_norms_match_oracle(torch_cuda, ff, oracle, n):
    """The reference's analytic f (FishFry.hpp:22-44) and its error norms on
    grids of prime lengths: device norms equal the oracle's where the grid's
    truncation error sets them (17x19x23: 2e-8), and both are round-off
    (about 1e-15, where the two solves' rounding differs) on the finer grids."""
    plan = ff.Plan(n)
    d = torch_cuda.empty(plan.nbytes // 8, dtype=torch_cuda.float64, device="cuda")
    p = torch_cuda.empty_like(d)
    ff.init_field(n, d)
    N = n[0] * n[1] * n[2]
    f = d[:N].cpu().numpy().reshape(n)
    plan.solve(d, p)
    ref = oracle.solve(f)
    assert rel_l2(p[:N].cpu().numpy().reshape(n), ref) <= FP64_TOL
    got = ff.rel_norms(n, p)
    want = oracle.rel_norms(ref)
    assert all(abs(a - b) <= 1e-9 * b + 5e-15 for a, b in zip(got, want)), (got, want)


@pytest.mark.parametrize("n,L", [((7, 11, 13), (1.0, 2.0, 3.0)), ((97, 16, 49), (5.0, 0.5, 2.0))])
def test_single_mode_exact_solution(torch_cuda, ff, n, L):
    """f = cos(2*pi*(kx*x/Lx + ky*y/Ly + kz*z/Lz)) on a box other than the 2*pi
    cube: phi = -f / |2*pi*k/L|^2 to round-off."""
    lo = [0.0, -1.0, 2.5]
    hi = [lo[a] + L[a] * (n[a] - 1) / n[a] for a in range(3)]
    k = (2, 1, 3)
    x = [lo[a] + np.arange(n[a]) * L[a] / n[a] for a in range(3)]
    X, Y, Z = np.meshgrid(x[0], x[1], x[2], indexing="ij")
    f = np.cos(2 * np.pi * (k[0] * X / L[0] + k[1] * Y / L[1] + k[2] * Z / L[2]))
    k2 = sum((2 * np.pi * k[a] / L[a]) ** 2 for a in range(3))
    phi = solve(torch_cuda, ff, f, lo=lo, hi=hi)
    assert rel_l2(phi, -f / k2) <= 1e-12


def _golden_prime_files():
    out = []
    for path in sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz"))):
        n = tuple(int(x) for x in os.path.basename(path)[4:-4].split("x"))
        if not all(smooth235(x) for x in n):
            out.append(path)
    return out


@pytest.mark.parametrize("path", _golden_prime_files())
def test_matches_reference_golden(torch_cuda, ff, path):
    """phi of the reference itself (cuFFT on a B200, tests/golden/) on the
    reference's analytic f: this build's solve of the same f agrees."""
    g = np.load(path)
    n = tuple(int(x) for x in g["n"])
    plan = ff.Plan(n)
    d = torch_cuda.empty(plan.nbytes // 8, dtype=torch_cuda.float64, device="cuda")
    p = torch_cuda.empty_like(d)
    ff.init_field(n, d)
    N = n[0] * n[1] * n[2]
    f = d[:N].cpu().numpy().reshape(n)
    plan.solve(d, p)
    phi = p[:N].cpu().numpy().reshape(n)
    if "phi" in g.files:
        assert np.abs(f - g["f"]).max() <= 1e-14 * np.abs(g["f"]).max()
        assert rel_l2(phi, g["phi"]) <= FP64_TOL
    else:
        got = phi.ravel()[g["idx"]]
        assert np.abs(got - g["phi_samples"]).max() <= FP64_TOL * float(g["phi_l2"])
        assert abs(np.linalg.norm(phi) - float(g["phi_l2"])) <= FP64_TOL * float(g["phi_l2"])


def test_server_rejects_primes_above_7(torch_cuda, ff):
    """The serving form takes 2^a 3^b 5^c 7^d lengths only (its requests run in
    the batch kernels); a batch accepts any length, solving such grids by
    their own plans (tests/test_batch_gpu.py)."""
    srv = ff.Server(1 << 30, max_active=4)
    f = torch_cuda.zeros(8 * 8 * 11, dtype=torch_cuda.float64, device="cuda")
    with pytest.raises(ff.FFError) as e:
        srv.submit((8, 8, 11), f, ff.FF_FP64)
    assert e.value.status == ff.FF_ERR_UNSUPPORTED
    srv.close()


def test_batch_and_server_radix7_lengths(torch_cuda, ff, oracle):
    """2^a 3^b 5^c 7^d grids in a batch (default and tuned shapes) and through
    the server, FP64 and FP32, against the oracle."""
    dims = [(28, 49, 56), (112, 14, 21), (7, 8, 8), (35, 63, 98), (64, 7, 343)]
    for prec, tol in ((0, FP64_TOL), (1, FP32_TOL)):
        batch = ff.Batch(dims, precision=prec)
        dt = torch_cuda.float64 if prec == 0 else torch_cuda.float32
        esz = 8 if prec == 0 else 4
        d = [torch_cuda.zeros(nb // esz, dtype=dt, device="cuda") for nb in batch.nbytes]
        p = [torch_cuda.empty_like(x) for x in d]
        rng = np.random.default_rng(77 + prec)
        fs = [rng.standard_normal(n).astype(np.float32).astype(np.float64) for n in dims]
        for tuned in (False, True):
            for g, f in enumerate(fs):
                d[g][:f.size] = torch_cuda.from_numpy(f.ravel()).to(dt).cuda()
            if tuned:
                batch.tune(d, p, reps=1)
                for g, f in enumerate(fs):
                    d[g][:f.size] = torch_cuda.from_numpy(f.ravel()).to(dt).cuda()
            batch.solve(d, p)
            for g, f in enumerate(fs):
                phi = p[g][:f.size].double().cpu().numpy().reshape(dims[g])
                assert rel_l2(phi, oracle.solve(f)) <= tol, (prec, tuned, dims[g])
    srv = ff.Server(1 << 30, max_active=8)
    try:
        for q, n in enumerate(dims[:3]):
            f = torch_cuda.from_numpy(np.random.default_rng(q).standard_normal(n).ravel()).cuda()
            rid = srv.submit(n, f, 0)
            srv.wait(rid)
            out = torch_cuda.empty_like(f)
            srv.fetch(rid, out)
            ref = oracle.solve(f.cpu().numpy().reshape(n))
            assert rel_l2(out.cpu().numpy().reshape(n), ref) <= FP64_TOL, n
    finally:
        srv.close()


def test_plans_with_different_bluestein_tiles_coexist(torch_cuda, ff, oracle):
    """Two plans whose Bluestein passes need different shared memory, the
    larger one created first and solved after the smaller one was created
    (a kernel's shared-memory limit is shared by every plan)."""
    big, small = (1009, 4, 6), (11, 8, 8)
    rng = np.random.default_rng(4)
    fb = rng.standard_normal(big)
    fs = rng.standard_normal(small)
    pb = ff.Plan(big)
    ps = ff.Plan(small)
    for plan, f in ((pb, fb), (ps, fs), (pb, fb)):
        d = torch_cuda.zeros(plan.nbytes // 8, dtype=torch_cuda.float64, device="cuda")
        p = torch_cuda.empty_like(d)
        d[:f.size] = torch_cuda.from_numpy(f.ravel()).cuda()
        plan.solve(d, p)
        phi = p[:f.size].cpu().numpy().reshape(f.shape)
        assert rel_l2(phi, oracle.solve(f)) <= FP64_TOL
