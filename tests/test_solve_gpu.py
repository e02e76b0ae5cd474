"""GPU parity tests of the solve through the C ABI against the CPU oracle.

FP64 bar: phi within 1e-12 relative L2 of the oracle on the same f.
FP32 bar: phi within 1e-5 relative L2 of the FP64 oracle.
"""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FP64_TOL = 1e-12
FP32_TOL = 1e-5


def dev_field(torch, ff, n, modes=None, precision=0):
    plan = ff.Plan(n, precision=precision)
    dt = torch.float64 if precision == ff.FF_FP64 else torch.float32
    esz = 8 if precision == ff.FF_FP64 else 4
    count = plan.nbytes // esz
    d = torch.empty(count, dtype=dt, device="cuda")
    p = torch.empty(count, dtype=dt, device="cuda")
    ff.init_field(n, d, modes, precision)
    return plan, d, p


def run_solve(torch, ff, n, modes=None, precision=0):
    """(f, phi) as host arrays after one solve of the device-initialised f."""
    plan, d, p = dev_field(torch, ff, n, modes, precision)
    N = n[0] * n[1] * n[2]
    f = d[:N].double().cpu().numpy().reshape(n)
    plan.solve(d, p)
    torch.cuda.synchronize()
    phi = p[:N].double().cpu().numpy().reshape(n)
    return f, phi


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


PARITY_SIZES = [(8, 8, 8), (16, 16, 16), (12, 10, 8), (5, 9, 6), (2, 3, 5), (1, 4, 6), (3, 1, 1), (1, 1, 2),
                (30, 45, 50), (64, 48, 40), (64, 64, 64), (100, 36, 27), (96, 80, 75), (128, 128, 128),
                (45, 81, 125), (256, 96, 72), (1800, 2, 4), (4, 1800, 6), (6, 5, 1800), (243, 16, 10),
                (1024, 8, 10), (6, 960, 9), (1215, 4, 6), (3, 1125, 4), (1125, 3, 1215), (4, 1024, 6),
                (1024, 1024, 2), (30, 1024, 1024)]


@pytest.mark.parametrize("n", PARITY_SIZES)
def test_fp64_parity_with_oracle(torch_cuda, ff, oracle, n):
    f, phi = run_solve(torch_cuda, ff, n)
    ref = oracle.solve(f)
    assert rel_l2(phi, ref) <= FP64_TOL


# Axes longer than the 128-byte-row tiles hold (narrower strided tiles; one
# line pair per z tile), and lengths with a prime factor above 7 beyond 1800
# points (Bluestein convolutions of 4032 and 6048 points).
LONG_AXES = [(2048, 64, 64), (64, 2048, 32), (4096, 16, 16), (16, 4096, 8), (16, 16, 4096), (2048, 8, 2048),
             (2003, 8, 8), (8, 2003, 6), (6, 8, 2003), (3001, 4, 4)]


@pytest.mark.parametrize("n", LONG_AXES)
def test_long_axes_fp64_parity_with_oracle(torch_cuda, ff, oracle, n):
    f, phi = run_solve(torch_cuda, ff, n)
    assert rel_l2(phi, oracle.solve(f)) <= FP64_TOL


@pytest.mark.parametrize("n", [(4096, 16, 16), (16, 4096, 8), (16, 16, 4096), (2003, 8, 8)])
def test_long_axes_fp32_parity_with_oracle(torch_cuda, ff, oracle, n):
    modes = ff.modes_generate(5, 16, 16, ff.alias_free_kaxis(n))
    f64 = oracle.init_f(n, modes)
    plan = ff.Plan(n, precision=ff.FF_FP32)
    d = torch_cuda.zeros(plan.nbytes // 4, dtype=torch_cuda.float32, device="cuda")
    p = torch_cuda.empty_like(d)
    ff.init_field(n, d, modes, ff.FF_FP32)
    N = f64.size
    f32 = d[:N].double().cpu().numpy().reshape(n)
    plan.solve(d, p)
    phi = p[:N].double().cpu().numpy().reshape(n)
    assert rel_l2(phi, oracle.solve(f32)) <= FP32_TOL


@pytest.mark.parametrize("n", [(16, 16, 16), (30, 45, 50), (64, 64, 64)])
def test_fp64_parity_random_field(torch_cuda, ff, oracle, n):
    rng = np.random.default_rng(11)
    f = rng.standard_normal(n)
    plan = ff.Plan(n)
    d = torch_cuda.zeros(plan.nbytes // 8, dtype=torch_cuda.float64, device="cuda")
    p = torch_cuda.empty_like(d)
    N = f.size
    d[:N] = torch_cuda.from_numpy(f.ravel()).cuda()
    plan.solve(d, p)
    phi = p[:N].cpu().numpy().reshape(n)
    assert rel_l2(phi, oracle.solve(f)) <= FP64_TOL


def test_fp64_parity_with_modes(torch_cuda, ff, oracle):
    n = (64, 48, 80)
    modes = ff.modes_generate(12345, 64, 32, ff.alias_free_kaxis(n))
    f, phi = run_solve(torch_cuda, ff, n, modes)
    assert np.abs(f - oracle.init_f(n, modes)).max() <= 1e-13 * np.abs(f).max()
    assert rel_l2(phi, oracle.solve(f)) <= FP64_TOL
    assert rel_l2(phi, oracle.phi_exact(n, modes)) <= 1e-13


@pytest.mark.parametrize("n", [(8, 8, 8), (30, 45, 50), (64, 64, 64)])
def test_init_field_matches_oracle(torch_cuda, ff, oracle, n):
    _, d, _ = dev_field(torch_cuda, ff, n)
    N = n[0] * n[1] * n[2]
    f = d[:N].cpu().numpy().reshape(n)
    ref = oracle.init_f(n)
    assert np.abs(f - ref).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("n", [(8, 8, 8), (16, 16, 16)])
def test_known_answer_norms_on_device(torch_cuda, ff, oracle, n):
    from tests.test_oracle import KATS
    plan, d, p = dev_field(torch_cuda, ff, n)
    plan.solve(d, p)
    got = ff.rel_norms(n, p)
    for g, want in zip(got, KATS[n]):
        assert abs(g - want) <= 1e-4 * want


def test_error_sums_match_oracle(torch_cuda, ff, oracle):
    n = (30, 45, 50)
    rng = np.random.default_rng(2)
    phi = rng.standard_normal(n)
    t = torch_cuda.from_numpy(phi.ravel()).cuda()
    got = ff.error_sums(n, t)
    ref = oracle.diff_sums(phi)
    assert np.allclose(got, ref, rtol=1e-12, atol=0)
    z = ff.error_sums(n, None)
    assert np.allclose(z, oracle.diff_sums(np.zeros(n)), rtol=1e-12)


def test_solve_is_deterministic(torch_cuda, ff):
    n = (64, 48, 40)
    plan, d, p = dev_field(torch_cuda, ff, n)
    N = n[0] * n[1] * n[2]
    f0 = d.clone()
    plan.solve(d, p)
    a = p[:N].clone()
    d.copy_(f0)
    plan.solve(d, p)
    assert torch_cuda.equal(a, p[:N])


def test_rejects_small_buffers(torch_cuda, ff):
    n = (16, 16, 16)
    plan, d, p = dev_field(torch_cuda, ff, n)
    with pytest.raises(ff.FFError) as e:
        plan.solve(d, p, nbytes=plan.nbytes - 8)
    assert e.value.status == ff.FF_ERR_BYTES


def test_bytes_match_reference_formula(ff):
    # ParisPencil.cpp:65-75 at one task: 2*ni*nj*nh doubles
    for n in [(8, 8, 8), (30, 45, 50), (512, 512, 512), (1024, 512, 256)]:
        plan = ff.Plan(n)
        assert plan.nbytes == 2 * n[0] * n[1] * (n[2] // 2 + 1) * 8


def test_paris_pencil_drop_in(torch_cuda, ff, oracle):
    n = (32, 24, 40)
    lo, hi, _, _ = ff.reference_domain(n)
    pp = ff.ParisPencil(n, lo, hi, (1, 1, 1), (0, 0, 0))
    nb = max(pp.bytes(), 8 * n[0] * n[1] * n[2])
    d = torch_cuda.empty(nb // 8, dtype=torch_cuda.float64, device="cuda")
    p = torch_cuda.empty_like(d)
    ff.init_field(n, d)
    N = n[0] * n[1] * n[2]
    f = d[:N].cpu().numpy().reshape(n)
    stamps = []
    pp.solve(nb, d, p, stamps)
    names = ff.phase_names(pp)
    assert stamps[0][0] == "Total" and len(stamps) == 1 + len(names)
    assert [s[0] for s in stamps[1:]] == names
    assert "X FFTs and filter" in names
    assert stamps[-1][1] >= stamps[0][1]
    assert rel_l2(p[:N].cpu().numpy().reshape(n), oracle.solve(f)) <= FP64_TOL


@pytest.mark.parametrize("n", [(64, 64, 64), (128, 96, 80), (30, 45, 50), (1024, 24, 20), (16, 1024, 64)])
def test_fp32_precision_form(torch_cuda, ff, oracle, n):
    modes = ff.modes_generate(12345, 64, 32, ff.alias_free_kaxis(n))
    f64 = oracle.init_f(n, modes)
    ref = oracle.solve(f64)
    plan = ff.Plan(n, precision=ff.FF_FP32)
    d = torch_cuda.zeros(plan.nbytes // 4, dtype=torch_cuda.float32, device="cuda")
    p = torch_cuda.empty_like(d)
    N = f64.size
    ff.init_field(n, d, modes, ff.FF_FP32)
    plan.solve(d, p)
    phi = p[:N].double().cpu().numpy().reshape(n)
    assert rel_l2(phi, ref) <= FP32_TOL


def test_fishfry_driver_printout(ff):
    exe = os.path.join(ROOT, "fishfry_b200", "bin", "fishfry")
    r = subprocess.run([exe, "1", "1", "1", "64", "64", "64", "2"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    assert re.search(r"FishFry<\w*ParisPencil>: 64x64x64 points over 1x1x1 MPI processes", out)
    runs = re.findall(r"^(\d+): Time (\S+) Rate (\S+) L_1 (\S+) L_2 (\S+) L_\\inf (\S+)", out, re.M)
    assert [int(r_[0]) for r_ in runs] == [0, 1, 2]
    assert "(warmup, ignored)" in out.splitlines()[1]
    for r_ in runs:
        assert max(float(x) for x in r_[3:]) < 1e-14
    assert "Times Averaged across Iterations" in out
    for name in ["Total", "X FFTs and filter"]:
        assert re.search(r"\(\s*[\d.]+%\) \| " + re.escape(name) + "$", out, re.M)


def test_fishfry_driver_known_answer(ff):
    from tests.test_oracle import KATS
    exe = os.path.join(ROOT, "fishfry_b200", "bin", "fishfry")
    r = subprocess.run([exe, "1", "1", "1", "16", "16", "16"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    m = re.search(r"L_1 (\S+) L_2 (\S+) L_\\inf (\S+)", r.stdout)
    for g, want in zip(map(float, m.groups()), KATS[(16, 16, 16)]):
        assert abs(g - want) <= 1e-4 * want


# ------------------------------------------------------- full-size workloads
@pytest.mark.slow
@pytest.mark.parametrize("n", [(512, 512, 512), (1024, 512, 256)])
def test_full_size_fp64(torch_cuda, ff, oracle, n):
    """Size-independent properties at the headline sizes: analytic error at
    round-off, and parity with the oracle (OpenMP) on the same f."""
    plan, d, p = dev_field(torch_cuda, ff, n)
    N = n[0] * n[1] * n[2]
    f = d[:N].cpu().numpy().reshape(n)
    plan.solve(d, p)
    assert max(ff.rel_norms(n, p)) < 1e-13
    phi = p[:N].cpu().numpy().reshape(n)
    del d, p
    assert rel_l2(phi, oracle.solve(f)) <= FP64_TOL


@pytest.mark.slow
def test_full_size_fp32_1024(torch_cuda, ff):
    """1024^3 FP32 precision form with 64 random modes: relative L2 against the
    FP64 solve of the same f (the FP64 path is itself pinned to the oracle at
    1e-12 on the other sizes; the OpenMP oracle is too slow here), and against
    the analytic solution (exact to round-off for the alias-free modes)."""
    torch = torch_cuda
    n = (1024, 1024, 1024)
    N = n[0] * n[1] * n[2]
    modes = ff.modes_generate(12345, 64, 32, ff.alias_free_kaxis(n))
    plan64 = ff.Plan(n)
    d = torch.empty(plan64.nbytes // 8, dtype=torch.float64, device="cuda")
    p64 = torch.empty_like(d)
    ff.init_field(n, d, modes, ff.FF_FP64)
    f32 = d[:N].float()          # the FP32 solve sees f rounded once to FP32
    d[:N].copy_(f32.double())    # and the FP64 solve the same values
    plan64.solve(d, p64)
    phi64 = p64[:N].clone()
    del d, p64
    plan64.close()
    plan = ff.Plan(n, precision=ff.FF_FP32)
    d = torch.empty(plan.nbytes // 4, dtype=torch.float32, device="cuda")
    p = torch.empty_like(d)
    d[:N].copy_(f32)
    del f32
    plan.solve(d, p)
    phi32 = p[:N].double()
    rel = float(torch.linalg.vector_norm(phi32 - phi64) / torch.linalg.vector_norm(phi64))
    assert rel <= FP32_TOL, rel
    s0 = ff.error_sums(n, None, modes, ff.FF_FP32)
    s1 = ff.error_sums(n, p, modes, ff.FF_FP32)
    assert (s1[1] / s0[1]) ** 0.5 <= FP32_TOL


# ----------------------------------------- the reference itself (oracle/_ref)
REF_DUMP = os.path.join(ROOT, "oracle", "_ref", "ref_dump")


@pytest.mark.skipif(not os.path.exists(REF_DUMP), reason="reference not built (oracle/ref/Makefile)")
@pytest.mark.parametrize("n", [(8, 8, 8), (12, 10, 8), (30, 45, 50), (64, 64, 64), (100, 36, 27)])
def test_parity_with_reference_binary(torch_cuda, ff, n, tmp_path):
    out = tmp_path / "ref.bin"
    r = subprocess.run([REF_DUMP, str(n[0]), str(n[1]), str(n[2]), str(out)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(out, dtype=np.uint8)
    N = n[0] * n[1] * n[2]
    arr = raw[12:].view(np.float64)
    f_ref, phi_ref = arr[:N].reshape(n), arr[N:].reshape(n)
    plan = ff.Plan(n)
    d = torch_cuda.zeros(plan.nbytes // 8, dtype=torch_cuda.float64, device="cuda")
    p = torch_cuda.empty_like(d)
    d[:N] = torch_cuda.from_numpy(f_ref.ravel()).cuda()
    plan.solve(d, p)
    phi = p[:N].cpu().numpy().reshape(n)
    assert rel_l2(phi, phi_ref) <= FP64_TOL


# The reference's own harness (main.cpp, FishFry.hpp, gpu.hpp, TimeStamp.hpp,
# unchanged) compiled against include/ParisPencil.hpp and libfishfry.so by
# oracle/ref/Makefile: the drop-in boundary exercised by the code it replaces.
DROPIN = os.path.join(ROOT, "oracle", "_ref", "fishfry_dropin")
RUN_RE = re.compile(r"^(\d+): Time (\S+) Rate (\S+) L_1 (\S+) L_2 (\S+) L_\\inf (\S+)", re.M)


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in harness not built (oracle/ref/Makefile)")
@pytest.mark.parametrize("n", [(64, 64, 64), (256, 256, 256)])
def test_reference_harness_drives_dropin(ff, n):
    r = subprocess.run([DROPIN, "1", "1", "1", *map(str, n), "3"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = r.stdout
    assert re.search(r"FishFry<\w*ParisPencil>: %dx%dx%d points over 1x1x1 MPI processes" % n, out), out
    runs = RUN_RE.findall(out)
    assert [int(x[0]) for x in runs] == [0, 1, 2, 3], out
    golden = open(os.path.join(ROOT, "tests", "golden", "ref_printout_%dx%dx%d.txt" % n)).read()
    want = [float(x) for x in RUN_RE.findall(golden)[1][3:]]
    for run in runs:
        t, rate = float(run[1]), float(run[2])
        assert t > 0 and abs(rate * t / (n[0] * n[1] * n[2]) - 1) < 1e-3
        got = [float(x) for x in run[3:]]
        # the reference's own diff kernel and norms on this build's phi: round-off, as the reference's phi
        for g, w in zip(got, want):
            assert abs(g - w) <= 1e-14, (got, want)
    # the phase table: the reference's table code over this build's stamps
    assert "Times Averaged across Iterations" in out
    for name in ["Total"] + ff.phase_names(ff.Plan(n)):
        assert re.search(r"\(\s*[\d.]+%\) \| " + re.escape(name) + "$", out, re.M), name


@pytest.mark.parametrize("n", [(64, 64, 64), (30, 45, 50), (512, 16, 24), (16, 512, 512)])
def test_fused_passes_parity(torch_cuda, ff, oracle, n, monkeypatch):
    """Three-launch mode (z and y passes fused through L2, FF_PASSES=3) gives
    the same phi as the oracle."""
    monkeypatch.setenv("FF_PASSES", "3")
    plan = ff.Plan(n)
    assert plan.phases() == 3
    d = torch_cuda.empty(plan.nbytes // 8, dtype=torch_cuda.float64, device="cuda")
    p = torch_cuda.empty_like(d)
    ff.init_field(n, d)
    N = n[0] * n[1] * n[2]
    f = d[:N].cpu().numpy().reshape(n)
    plan.solve(d, p, timed=True)
    assert rel_l2(p[:N].cpu().numpy().reshape(n), oracle.solve(f)) <= FP64_TOL


def box_bounds(n, L, lo0=(0.0, -1.0, 2.5)):
    """Bounds of a periodic box of side L[a] sampled at n[a] points, with hi one
    cell short of the period as the reference's harness passes them
    (FishFry.hpp:133-134); the wavenumber scale is then 2*pi/L."""
    lo = [lo0[a] for a in range(3)]
    hi = [lo0[a] + L[a] * (n[a] - 1) / n[a] for a in range(3)]
    return lo, hi


@pytest.mark.parametrize("n,L", [((48, 40, 64), (3.0, 10.0, 1.5)), ((30, 45, 50), (1.0, 2.0, 7.0)),
                                 ((256, 8, 12), (0.5, 0.5, 0.5))])
def test_general_box_matches_oracle_and_mode_solution(torch_cuda, ff, oracle, n, L):
    """Boxes other than the reference's 2*pi cube (ParisPencil.cpp:9-11 derives
    the wavenumber scale from lo/hi): against the oracle on the same bounds,
    and against the exact solution of one Fourier mode,
    f = cos(2*pi*(kx*x/Lx + ky*y/Ly + kz*z/Lz)) -> phi = -f / |2*pi*k/L|^2."""
    lo, hi = box_bounds(n, L)
    k = (2, 1, 3)
    x = [lo[a] + np.arange(n[a]) * L[a] / n[a] for a in range(3)]
    X, Y, Z = np.meshgrid(x[0], x[1], x[2], indexing="ij")
    arg = 2 * np.pi * (k[0] * X / L[0] + k[1] * Y / L[1] + k[2] * Z / L[2])
    rng = np.random.default_rng(5)
    f = np.cos(arg) + 0.1 * rng.standard_normal(n)
    f -= f.mean()
    plan = ff.Plan(n, lo, hi)
    d = torch_cuda.zeros(plan.nbytes // 8, dtype=torch_cuda.float64, device="cuda")
    p = torch_cuda.empty_like(d)
    N = f.size
    d[:N] = torch_cuda.from_numpy(f.ravel()).cuda()
    plan.solve(d, p)
    phi = p[:N].cpu().numpy().reshape(n)
    assert rel_l2(phi, oracle.solve(f, lo, hi)) <= FP64_TOL
    # the single mode alone
    k2 = sum((2 * np.pi * k[a] / L[a]) ** 2 for a in range(3))
    d[:N] = torch_cuda.from_numpy(np.cos(arg).ravel()).cuda()
    plan.solve(d, p)
    phi1 = p[:N].cpu().numpy().reshape(n)
    assert rel_l2(phi1, -np.cos(arg) / k2) <= 1e-12


def test_general_box_in_a_batch(torch_cuda, ff, oracle):
    dims = [(48, 40, 64), (30, 45, 50)]
    Ls = [(3.0, 10.0, 1.5), (1.0, 2.0, 7.0)]
    bounds = [box_bounds(n, L) for n, L in zip(dims, Ls)]
    batch = ff.Batch(dims, lo=[b[0] for b in bounds], hi=[b[1] for b in bounds])
    rng = np.random.default_rng(8)
    fs = [rng.standard_normal(n) for n in dims]
    d = [torch_cuda.zeros(nb // 8, dtype=torch_cuda.float64, device="cuda") for nb in batch.nbytes]
    p = [torch_cuda.empty_like(x) for x in d]
    for g, f in enumerate(fs):
        d[g][:f.size] = torch_cuda.from_numpy(f.ravel()).cuda()
    batch.solve(d, p)
    for g, (f, (lo, hi)) in enumerate(zip(fs, bounds)):
        phi = p[g][:f.size].cpu().numpy().reshape(dims[g])
        assert rel_l2(phi, oracle.solve(f, lo, hi)) <= FP64_TOL, g


GUARD = 1 << 16
SENTINEL = 0xA5


@pytest.mark.parametrize("n,precision", [((64, 48, 512), 0), ((48, 64, 512), 1), ((40, 30, 256), 0), ((30, 40, 128), 1),
                                         ((24, 20, 1024), 0), ((20, 24, 64), 0), ((1024, 8, 10), 0), ((6, 1024, 9), 1),
                                         ((30, 45, 50), 0), ((97, 13, 30), 0), ((64, 64, 64), 1)])
def test_solve_writes_stay_inside_its_buffers(torch_cuda, ff, oracle, n, precision):
    """The single-grid passes write only the plan's two buffers: guard zones
    around them keep their sentinel bytes through a solve (compile-time z
    lengths with the fused last stages, 64-byte-row tiles, runtime and
    Bluestein lengths)."""
    torch = torch_cuda
    plan = ff.Plan(n, precision=precision)
    dt = torch.float64 if precision == ff.FF_FP64 else torch.float32
    esz = 8 if precision == ff.FF_FP64 else 4
    nb_al = (plan.nbytes + 255) // 256 * 256
    arenas = [torch.full((GUARD + nb_al + GUARD,), SENTINEL, dtype=torch.uint8, device="cuda") for _ in range(2)]
    d, p = [a[GUARD:GUARD + nb_al].view(dt)[:plan.nbytes // esz] for a in arenas]
    ff.init_field(n, d, None, precision)
    N = n[0] * n[1] * n[2]
    f = d[:N].double().cpu().numpy().reshape(n)
    plan.solve(d, p)
    torch.cuda.synchronize()
    for a in arenas:
        assert (a[:GUARD].cpu().numpy() == SENTINEL).all() and (a[GUARD + nb_al:].cpu().numpy() == SENTINEL).all()
    phi = p[:N].double().cpu().numpy().reshape(n)
    assert rel_l2(phi, oracle.solve(f)) <= (FP64_TOL if precision == 0 else FP32_TOL)


# z lengths with fused last stages (64 .. 1024), with line counts ni*nj that
# leave the last z tile partly empty (odd counts, a single line, fewer lines
# than one tile holds)
Z_FUSED = [(3, 5, 512), (1, 1, 512), (7, 3, 256), (5, 1, 128), (1, 3, 1024), (3, 1, 64), (9, 7, 32), (2, 3, 512)]


@pytest.mark.parametrize("n", Z_FUSED)
@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, FP32_TOL)])
def test_fused_z_lengths_with_partial_tiles(torch_cuda, ff, oracle, n, precision, tol):
    rng = np.random.default_rng(sum(n) + precision)
    f = rng.standard_normal(n)
    plan = ff.Plan(n, precision=precision)
    dt = torch_cuda.float64 if precision == 0 else torch_cuda.float32
    esz = 8 if precision == 0 else 4
    d = torch_cuda.zeros(plan.nbytes // esz, dtype=dt, device="cuda")
    p = torch_cuda.zeros_like(d)
    N = n[0] * n[1] * n[2]
    d[:N] = torch_cuda.from_numpy(f.ravel()).to(dt).cuda()
    fq = d[:N].double().cpu().numpy().reshape(n)
    plan.solve(d, p)
    torch_cuda.cuda.synchronize()
    phi = p[:N].double().cpu().numpy().reshape(n)
    assert rel_l2(phi, oracle.solve(fq)) <= tol
