"""GPU tests of the batched form (ff_batch_*) against the CPU oracle and the
single-grid solve.

FP64 bar: each grid's phi within 1e-12 relative L2 of the oracle on the same f.
FP32 bar: within 1e-5 relative L2 of the FP64 oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5

# compile-time lengths (32, 48, 64, 80, 96, 128, 256, 512), runtime-plan
# lengths (27, 30, 36, 45, 50, 60, 75, 100, 120) and one-point / tiny axes
MIXED = [(32, 48, 64), (80, 96, 128), (36, 45, 50), (64, 64, 64), (128, 32, 96), (27, 30, 25), (1, 8, 6),
         (60, 1, 100), (120, 75, 2), (16, 16, 16), (256, 8, 12), (6, 512, 4), (10, 12, 512)]


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def make_buffers(torch, batch, precision):
    dt = torch.float64 if precision == 0 else torch.float32
    esz = 8 if precision == 0 else 4
    d = [torch.empty(nb // esz, dtype=dt, device="cuda") for nb in batch.nbytes]
    p = [torch.empty(nb // esz, dtype=dt, device="cuda") for nb in batch.nbytes]
    return d, p


def init_all(ff, batch, d, modes_of, precision):
    fs = []
    for g, n in enumerate(batch.dims):
        ff.init_field(n, d[g], modes_of(n), precision)
        N = n[0] * n[1] * n[2]
        fs.append(d[g][:N].double().cpu().numpy().reshape(n))
    return fs


def results(batch, p):
    out = []
    for g, n in enumerate(batch.dims):
        N = n[0] * n[1] * n[2]
        out.append(p[g][:N].double().cpu().numpy().reshape(n))
    return out


def modes_for(ff, seed=12345):
    return lambda n: ff.modes_generate(seed, 64, 32, ff.alias_free_kaxis(n))


@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, FP32_TOL)])
def test_batch_parity_with_oracle(torch_cuda, ff, oracle, precision, tol):
    batch = ff.Batch(MIXED, precision=precision)
    d, p = make_buffers(torch_cuda, batch, precision)
    fs = init_all(ff, batch, d, modes_for(ff), precision)
    batch.solve(d, p)
    torch_cuda.cuda.synchronize()
    batch.check()
    for g, (f, phi) in enumerate(zip(fs, results(batch, p))):
        # the FP64 oracle solves the same (FP32-rounded, for FP32) f
        assert rel_l2(phi, oracle.solve(f)) <= tol, (g, batch.dims[g])


def test_batch_matches_single_grid_solve(torch_cuda, ff):
    batch = ff.Batch(MIXED)
    d, p = make_buffers(torch_cuda, batch, 0)
    init_all(ff, batch, d, modes_for(ff, 7), 0)
    batch.solve(d, p)
    got = results(batch, p)
    for g, n in enumerate(batch.dims):
        plan = ff.Plan(n)
        dd = torch_cuda.empty(plan.nbytes // 8, dtype=torch_cuda.float64, device="cuda")
        pp = torch_cuda.empty_like(dd)
        ff.init_field(n, dd, modes_for(ff, 7)(n), 0)
        plan.solve(dd, pp)
        N = n[0] * n[1] * n[2]
        ref = pp[:N].cpu().numpy().reshape(n)
        assert rel_l2(got[g], ref) <= 1e-14, (g, n)


def test_batch_graph_replay_is_repeatable(torch_cuda, ff):
    batch = ff.Batch(MIXED[:6])
    d, p = make_buffers(torch_cuda, batch, 0)
    runs = []
    for _ in range(3):
        init_all(ff, batch, d, modes_for(ff, 3), 0)
        ms, tot = batch.solve(d, p, timed=True)
        assert len(ms) == 5 and tot > 0 and all(x >= 0 for x in ms)
        runs.append(results(batch, p))
    for r in runs[1:]:
        for a, b in zip(runs[0], r):
            assert np.array_equal(a, b)


def test_batch_new_buffers_between_solves(torch_cuda, ff, oracle):
    batch = ff.Batch(MIXED[:5])
    for seed in (1, 2):
        d, p = make_buffers(torch_cuda, batch, 0)
        fs = init_all(ff, batch, d, modes_for(ff, seed), 0)
        batch.solve(d, p)
        for f, phi in zip(fs, results(batch, p)):
            assert rel_l2(phi, oracle.solve(f)) <= FP64_TOL


@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, FP32_TOL)])
def test_batch_tuned_shapes_keep_parity(torch_cuda, ff, oracle, precision, tol):
    batch = ff.Batch(MIXED, precision=precision)
    d, p = make_buffers(torch_cuda, batch, precision)
    batch.tune(d, p, reps=1)
    csz = 16 if precision == 0 else 8
    for g in range(len(batch)):
        for kind in range(5):
            W, ct, tma = batch.shape(g, kind)
            assert W >= 1 and ct in (0, 1) and tma in (0, 1)
            if kind in (1, 2, 3):
                assert (W * csz) % 128 == 0
    # the radix split of every axis is a reordering of the default one
    for g, n in enumerate(batch.dims):
        for axis in range(3):
            r = batch.radices(g, axis)
            assert sorted(r) == sorted(default_radices(n[axis])) and int(np.prod(r)) == n[axis], (g, axis, r)
    fs = init_all(ff, batch, d, modes_for(ff), precision)
    batch.solve(d, p)
    for g, (f, phi) in enumerate(zip(fs, results(batch, p))):
        assert rel_l2(phi, oracle.solve(f)) <= tol, (g, batch.dims[g])


def default_radices(n):
    """The default plan's radices: 8s while three factors of 2 remain, one 4 or
    2, then 5s, then 3s; a length of 1 is one stage of radix 1."""
    twos = fives = threes = 0
    m = n
    while m > 1 and m % 2 == 0:
        m //= 2
        twos += 1
    while m > 1 and m % 5 == 0:
        m //= 5
        fives += 1
    while m > 1 and m % 3 == 0:
        m //= 3
        threes += 1
    r = [8] * (twos // 3) + ([4] if twos % 3 == 2 else [2] if twos % 3 == 1 else []) + [5] * fives + [3] * threes
    return r or [1]


def test_batch_tuner_reorders_radices_of_runtime_lengths(torch_cuda, ff, oracle):
    """Lengths with mixed radices (runtime plans) get their radix order tuned;
    whatever order wins, results match the oracle."""
    dims = [(60, 90, 150), (150, 60, 90), (90, 150, 60), (45, 120, 100)]
    batch = ff.Batch(dims)
    d, p = make_buffers(torch_cuda, batch, 0)
    batch.tune(d, p, reps=1)
    for g, n in enumerate(dims):
        for axis in range(3):
            r = batch.radices(g, axis)
            assert sorted(r) == sorted(default_radices(n[axis])), (g, axis, r)
    fs = init_all(ff, batch, d, modes_for(ff, 31), 0)
    batch.solve(d, p)
    for g, (f, phi) in enumerate(zip(fs, results(batch, p))):
        assert rel_l2(phi, oracle.solve(f)) <= FP64_TOL, (g, dims[g])


def test_batch_of_256_seeded_grids(torch_cuda, ff, oracle):
    """The batched workload's shape: 256 grids, dims iid from
    {32, 48, 64, 80, 96, 128}; a sample of grids checked against the oracle,
    every grid against the analytic potential of its modes."""
    rng = np.random.default_rng(2024)
    choices = [32, 48, 64, 80, 96, 128]
    dims = [tuple(int(x) for x in rng.choice(choices, 3)) for _ in range(256)]
    batch = ff.Batch(dims)
    d, p = make_buffers(torch_cuda, batch, 0)
    fs = init_all(ff, batch, d, modes_for(ff, 99), 0)
    batch.solve(d, p)
    torch_cuda.cuda.synchronize()
    got = results(batch, p)
    for g in range(0, 256, 37):
        assert rel_l2(got[g], oracle.solve(fs[g])) <= FP64_TOL, (g, dims[g])
    for g in range(256):
        norms = ff.rel_norms(dims[g], p[g], modes_for(ff, 99)(dims[g]), 0)
        assert max(norms) < 1e-6, (g, dims[g], norms)


def test_batch_tma_tiles_for_long_lines(torch_cuda, ff, oracle):
    """Grids whose y or x lines have 256+ points and planes of 32+ columns use
    one-plane TMA tiles by default (compile-time 256/512 and runtime 300/270
    lengths)."""
    # lengths the tuning test above does not tune for these passes (tuned
    # shapes are remembered process-wide and would replace the defaults)
    dims = [(512, 64, 80), (64, 256, 72), (300, 270, 64), (320, 8, 100)]
    batch = ff.Batch(dims)
    assert batch.shape(0, 2) == (8, 1, 1) and batch.shape(1, 1) == (8, 1, 1) and batch.shape(1, 3) == (8, 1, 1)
    assert batch.shape(2, 2) == (8, 0, 1) and batch.shape(2, 1) == (8, 0, 1) and batch.shape(3, 2) == (8, 0, 1)
    d, p = make_buffers(torch_cuda, batch, 0)
    fs = init_all(ff, batch, d, modes_for(ff, 17), 0)
    batch.solve(d, p)
    for g, (f, phi) in enumerate(zip(fs, results(batch, p))):
        assert rel_l2(phi, oracle.solve(f)) <= FP64_TOL, (g, dims[g])


@pytest.mark.parametrize("precision,tol,want", [(0, FP64_TOL, [4, 5, 25]), (1, FP32_TOL, [8, 8, 25])])
def test_batch_z_tiles_of_long_lines(torch_cuda, ff, oracle, precision, tol, want):
    """Default z tiles: about 2048 points for short lines; lines of 256 and
    200 points take up to 32 KB of line pairs (at most 8), as the single-grid
    z passes do (FP32 8 pairs, where 2048 points would be 4 and 5)."""
    # z lengths no tuning test in this process tunes (tuned shapes would
    # replace the defaults)
    dims = [(64, 48, 256), (40, 36, 200), (50, 60, 40)]
    batch = ff.Batch(dims, precision=precision)
    for g, w in enumerate(want):
        assert batch.shape(g, 0)[0] == w and batch.shape(g, 4)[0] == w, (g, batch.shape(g, 0), batch.shape(g, 4))
    d, p = make_buffers(torch_cuda, batch, precision)
    fs = init_all(ff, batch, d, modes_for(ff, 29), precision)
    batch.solve(d, p)
    for g, (f, phi) in enumerate(zip(fs, results(batch, p))):
        assert rel_l2(phi, oracle.solve(f)) <= tol, (g, dims[g])


# Grids the batch kernels do not take (an axis with a prime factor above 7,
# or longer than their tiles) are solved by their own single-grid plans in
# the same ff_batch_solve.
WITH_SIDE = [(32, 48, 64), (97, 40, 36), (80, 96, 128), (36, 101, 50), (27, 30, 127), (600, 8, 12), (64, 64, 64)]


@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, FP32_TOL)])
def test_batch_with_prime_and_long_axes(torch_cuda, ff, oracle, precision, tol):
    batch = ff.Batch(WITH_SIDE, precision=precision)
    d, p = make_buffers(torch_cuda, batch, precision)
    batch.tune(d, p)   # tunes the batched grids only
    fs = init_all(ff, batch, d, modes_for(ff, 3), precision)
    ms, total = batch.solve(d, p, timed=True)
    assert total > 0 and len(ms) == 5
    batch.check()
    for g, (f, phi) in enumerate(zip(fs, results(batch, p))):
        assert rel_l2(phi, oracle.solve(f)) <= tol, (g, batch.dims[g])
    with pytest.raises(ff.FFError) as e:
        batch.shape(1, 0)
    assert e.value.status == ff.FF_ERR_UNSUPPORTED
    assert batch.shape(0, 0)[0] > 0


def test_batch_of_only_side_grids(torch_cuda, ff, oracle):
    dims = [(97, 8, 10), (11, 13, 17)]
    batch = ff.Batch(dims)
    d, p = make_buffers(torch_cuda, batch, 0)
    fs = init_all(ff, batch, d, lambda n: None, 0)
    batch.solve(d, p, timed=True)
    for g, (f, phi) in enumerate(zip(fs, results(batch, p))):
        assert rel_l2(phi, oracle.solve(f)) <= FP64_TOL, g


# the serving test mix plus MIXED: every tile shape the batch kernels choose
GUARD_DIMS = [(32, 32, 32), (48, 64, 80), (128, 96, 64), (36, 45, 50), (256, 64, 32), (60, 72, 90), (64, 64, 64),
              (512, 16, 24), (20, 30, 512), (100, 120, 81)] + MIXED
GUARD = 1 << 16
SENTINEL = 0xA5


def guarded_buffers(torch, sizes, dt):
    """One device arena per buffer, [guard | buffer | guard] with the guards
    filled with SENTINEL bytes; returns (arenas, typed views)."""
    arenas, views = [], []
    esz = torch.empty(0, dtype=dt).element_size()
    for nb in sizes:
        nb_al = (nb + 255) // 256 * 256
        a = torch.full((GUARD + nb_al + GUARD,), SENTINEL, dtype=torch.uint8, device="cuda")
        arenas.append((a, nb_al))
        views.append(a[GUARD:GUARD + nb_al].view(dt)[:nb // esz])
    return arenas, views


def guards_intact(torch, arenas):
    bad = []
    for q, (a, nb_al) in enumerate(arenas):
        lo = a[:GUARD].cpu().numpy()
        hi = a[GUARD + nb_al:].cpu().numpy()
        if (lo != SENTINEL).any() or (hi != SENTINEL).any():
            bad.append((q, int(np.flatnonzero(lo != SENTINEL).size), int(np.flatnonzero(hi != SENTINEL).size)))
    return bad


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("tuned", [False, True])
def test_batch_writes_stay_inside_each_grids_buffers(torch_cuda, ff, oracle, precision, tuned):
    """Every batch kernel writes only its own grid's buffers: guard zones
    around each density and potential buffer keep their sentinel bytes
    through a solve (and through the tuner's trial solves), with default and
    tuned tile shapes."""
    torch = torch_cuda
    batch = ff.Batch(GUARD_DIMS, precision=precision)
    dt = torch.float64 if precision == 0 else torch.float32
    ad, d = guarded_buffers(torch, batch.nbytes, dt)
    ap, p = guarded_buffers(torch, batch.nbytes, dt)
    if tuned:
        init_all(ff, batch, d, modes_for(ff), precision)
        batch.tune(d, p, reps=1)
        torch.cuda.synchronize()
        assert guards_intact(torch, ad) == [] and guards_intact(torch, ap) == []
    fs = init_all(ff, batch, d, modes_for(ff), precision)
    batch.solve(d, p)
    torch.cuda.synchronize()
    assert guards_intact(torch, ad) == [], "density guards"
    assert guards_intact(torch, ap) == [], "potential guards"
    tol = FP64_TOL if precision == 0 else FP32_TOL
    for g, (f, phi) in enumerate(zip(fs, results(batch, p))):
        assert rel_l2(phi, oracle.solve(f)) <= tol, g
