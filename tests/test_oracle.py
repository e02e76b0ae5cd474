"""CPU tests of the oracle: its FFT and solve against numpy's pocketfft, the
known-answer relative norms of the reference grid, the seeded mode generator,
and the golden vectors written by the reference itself (tests/golden/)."""
import glob
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def numpy_solve(f, dd=(1.0, 1.0, 1.0)):
    """Independent statement of ParisPencil.cpp:263-285 + 406-421 with numpy's FFT."""
    ni, nj, nk = f.shape
    F = np.fft.rfftn(f)
    kx = np.minimum(np.arange(ni), ni - np.arange(ni)) * dd[0]
    ky = np.minimum(np.arange(nj), nj - np.arange(nj)) * dd[1]
    kz = np.arange(nk // 2 + 1) * dd[2]
    k2 = (kx[:, None, None] ** 2 + ky[None, :, None] ** 2) + kz[None, None, :] ** 2
    k2[0, 0, 0] = 1.0
    F = -F / k2
    F[0, 0, 0] = 0
    return np.fft.irfftn(F, s=f.shape, axes=(0, 1, 2))


# 2^a 3^b 5^c, 7-smooth (49, 343, 448, 1792) and prime (11, 13, 97, 127, 1789) lengths
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 8, 9, 11, 12, 13, 15, 16, 25, 27, 30, 45, 49, 64, 97, 120, 125, 127,
                               243, 343, 448, 512, 1000, 1789, 1792])
def test_fft1d_matches_numpy(oracle, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    scale = max(np.abs(ref).max(), 1e-300)
    assert np.abs(oracle.fft1d(x, -1) - ref).max() / scale < 1e-14
    assert np.abs(oracle.fft1d(x, +1) - np.fft.ifft(x) * n).max() / scale < 1e-14


@pytest.mark.parametrize("n", [(8, 8, 8), (16, 16, 16), (12, 10, 8), (5, 9, 6), (30, 45, 50), (7, 5, 9),
                               (1, 4, 6), (3, 1, 1), (2, 3, 5), (64, 48, 40), (7, 11, 13), (14, 9, 22), (49, 33, 17)])
def test_solve_matches_numpy(oracle, n):
    rng = np.random.default_rng(sum(n))
    f = rng.standard_normal(n)
    f -= f.mean()
    phi = oracle.solve(f)
    ref = numpy_solve(f)
    assert np.linalg.norm(phi - ref) <= 1e-13 * max(np.linalg.norm(ref), 1e-300)


def test_solve_domain_scale(oracle):
    # dd = 2*pi*(n-1)/(n*(hi-lo)) (ParisPencil.cpp:9-11) on a box of side 3 per axis
    n = (12, 10, 8)
    lo = [0.0, 0.0, 0.0]
    hi = [3.0 * (n[a] - 1) / n[a] for a in range(3)]
    dd = [2 * math.pi * (n[a] - 1) / (n[a] * (hi[a] - lo[a])) for a in range(3)]
    rng = np.random.default_rng(3)
    f = rng.standard_normal(n)
    phi = oracle.solve(f, lo, hi)
    ref = numpy_solve(f, dd)
    assert np.linalg.norm(phi - ref) <= 1e-13 * np.linalg.norm(ref)


# Known answers on the reference grid (lo = -pi, analytic f of FishFry.hpp:22-44):
# truncation dominated at 8^3 and 16^3, so they pin grid, filter and zero mode.
KATS = {
    (8, 8, 8): (5.7156e-3, 5.0619e-3, 4.6650e-3),
    (16, 16, 16): (8.2283e-8, 7.8372e-8, 9.6980e-8),
}


@pytest.mark.parametrize("n", list(KATS))
def test_known_answer_norms(oracle, n):
    phi = oracle.solve(oracle.init_f(n))
    got = oracle.rel_norms(phi)
    for g, want in zip(got, KATS[n]):
        assert abs(g - want) <= 1e-4 * want


@pytest.mark.parametrize("n", [(32, 32, 32), (64, 64, 64), (30, 45, 50)])
def test_roundoff_norms(oracle, n):
    phi = oracle.solve(oracle.init_f(n))
    assert max(oracle.rel_norms(phi)) < 1e-14


def test_modes_exact_solution(oracle):
    n = (32, 36, 40)
    kaxis = tuple((x - 1) // 2 for x in n)
    modes = oracle.modes_generate(12345, 64, 32, kaxis)
    assert len(modes) == 64
    for kx, ky, kz, a, th in modes:
        assert 0 < kx * kx + ky * ky + kz * kz <= 32 * 32
        assert abs(kx) <= kaxis[0] and abs(ky) <= kaxis[1] and abs(kz) <= kaxis[2]
        assert 0.0 <= th < 2 * math.pi
    phi = oracle.solve(oracle.init_f(n, modes))
    ex = oracle.phi_exact(n, modes)
    assert np.linalg.norm(phi - ex) / np.linalg.norm(ex) < 1e-13


def test_modes_zero_mean(oracle):
    n = (16, 16, 16)
    modes = oracle.modes_generate(7, 8, 32, (7, 7, 7))
    f = oracle.init_f(n, modes) - oracle.init_f(n)
    assert abs(f.mean()) < 1e-14


def test_norm_sums_match_numpy(oracle):
    n = (10, 12, 9)
    rng = np.random.default_rng(5)
    phi = rng.standard_normal(n)
    ex = oracle.phi_exact(n)
    d = np.abs(ex - phi)
    got = oracle.diff_sums(phi)
    assert np.allclose(got, [d.sum(), (d * d).sum(), d.max()], rtol=1e-13)


def _golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz")))


@pytest.mark.parametrize("path", _golden_files())
def test_oracle_matches_reference_golden(oracle, path):
    """Golden vectors produced by the reference's own ParisPencil + init kernel
    (oracle/ref/ref_dump, made by tests/golden/make_ref_golden.py on a B200)."""
    g = np.load(path)
    n = tuple(int(x) for x in g["n"])
    f = oracle.init_f(n)
    if "f" in g:   # reference f from its init kernel: same points, same formula
        assert np.abs(f - g["f"]).max() <= 1e-13 * np.abs(g["f"]).max()
        phi = oracle.solve(g["f"])
        assert np.linalg.norm(phi - g["phi"]) <= 1e-12 * np.linalg.norm(g["phi"])
    else:          # large grids: sampled points and norms of the reference phi
        phi = oracle.solve(f).ravel()
        idx = g["idx"]
        assert np.abs(phi[idx] - g["phi_samples"]).max() <= 1e-12 * np.abs(g["phi_samples"]).max()
        assert abs(np.linalg.norm(phi) - float(g["phi_l2"])) <= 1e-12 * float(g["phi_l2"])
    norms = oracle.rel_norms(oracle.solve(f))
    ref_norms = g["rel_norms"]
    for a, b in zip(norms, ref_norms):
        if b > 1e-10:        # truncation-dominated: equal up to the round-off in d
            assert abs(a - b) <= 1e-7 * b
        else:                # round-off level on both sides
            assert a < 1e-13 and b < 1e-13


def test_reference_printout_golden():
    """The reference benchmark's own printout (tests/golden/ref_printout_*.txt):
    its L1/L2/Linf at 8^3 and 16^3 equal the known answers above."""
    import re
    files = sorted(glob.glob(os.path.join(GOLDEN, "ref_printout_*.txt")))
    if not files:
        pytest.skip("no reference printout captured yet")
    seen = 0
    for p in files:
        text = open(p).read()
        m = re.search(r"FishFry<.*>: (\d+)x(\d+)x(\d+) points", text)
        n = tuple(int(x) for x in m.groups())
        runs = re.findall(r"L_1 (\S+) L_2 (\S+) L_\\inf (\S+)", text)
        assert runs
        if n in KATS:
            for r in runs:
                for g, want in zip(map(float, r), KATS[n]):
                    assert abs(g - want) <= 1e-4 * want
            seen += 1
    assert seen >= 1


def test_oracle_general_box_single_mode(oracle):
    """The oracle's wavenumber scale for a box of side L (hi one cell short):
    a single mode cos(2*pi*k*x/L) solves to -cos(...)/(2*pi*k/L)^2."""
    import numpy as np
    n = (24, 20, 16)
    L = (3.0, 10.0, 1.5)
    lo = [0.0, -1.0, 2.5]
    hi = [lo[a] + L[a] * (n[a] - 1) / n[a] for a in range(3)]
    k = (2, 1, 3)
    x = [lo[a] + np.arange(n[a]) * L[a] / n[a] for a in range(3)]
    X, Y, Z = np.meshgrid(x[0], x[1], x[2], indexing="ij")
    arg = 2 * np.pi * (k[0] * X / L[0] + k[1] * Y / L[1] + k[2] * Z / L[2])
    k2 = sum((2 * np.pi * k[a] / L[a]) ** 2 for a in range(3))
    phi = oracle.solve(np.cos(arg), lo, hi)
    assert np.abs(phi + np.cos(arg) / k2).max() <= 1e-13 * np.abs(np.cos(arg) / k2).max()
