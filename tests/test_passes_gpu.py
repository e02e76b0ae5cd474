"""GPU tests of each of the five passes on its own (ff_solve_passes) against
numpy's FFTs of the same input: z R2C, y forward, x forward + filter + x
inverse, y inverse, z C2R.  The intermediates are the unnormalised
transforms in natural order, the filter -1/(k^2 N) with the zero mode 0
(ParisPencil.cpp:263-285, :406-421).

FP64 bar: 1e-12 relative L2 per pass; FP32: 1e-5.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def reference_passes(f, dd):
    """The five intermediates of the solve of f (numpy, FP64)."""
    ni, nj, nk = f.shape
    s1 = np.fft.rfft(f, axis=2)
    s2 = np.fft.fft(s1, axis=1)
    i = np.arange(ni)
    j = np.arange(nj)
    kh = np.arange(nk // 2 + 1)
    ki = (np.minimum(i, ni - i) * dd[0]) ** 2
    kj = (np.minimum(j, nj - j) * dd[1]) ** 2
    kk = (kh * dd[2]) ** 2
    k2 = ki[:, None, None] + kj[None, :, None] + kk[None, None, :]
    k2[0, 0, 0] = 1.0
    filt = -1.0 / (k2 * f.size)
    filt[0, 0, 0] = 0.0
    s3 = np.fft.ifft(np.fft.fft(s2, axis=0) * filt, axis=0) * ni
    s4 = np.fft.ifft(s3, axis=1) * nj
    phi = np.fft.irfft(s4, n=nk, axis=2) * nk
    return [s1, s2, s3, s4, phi]


SIZES = [(16, 16, 16), (30, 45, 50), (64, 48, 40), (12, 10, 9), (7, 11, 13), (97, 20, 33), (256, 8, 12)]


@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-5)])
@pytest.mark.parametrize("n", SIZES)
def test_each_pass_matches_numpy(torch_cuda, ff, n, precision, tol):
    torch = torch_cuda
    lo, hi, _, _ = ff.reference_domain(n)
    dd = [2 * np.pi * (n[a] - 1) / (n[a] * (hi[a] - lo[a])) if n[a] > 1 else 0.0 for a in range(3)]
    rng = np.random.default_rng(sum(n) + precision)
    f = rng.standard_normal(n)
    if precision:
        f = f.astype(np.float32).astype(np.float64)
    want = reference_passes(f, dd)
    plan = ff.Plan(n, precision=precision)
    rdt, cdt = (torch.float64, np.complex128) if precision == 0 else (torch.float32, np.complex64)
    esz = 8 if precision == 0 else 4
    nh = n[2] // 2 + 1
    nhp = nh if precision == 0 else (nh + 1) // 2 * 2
    N = f.size
    for passes in range(1, 6):
        d = torch.zeros(plan.nbytes // esz, dtype=rdt, device="cuda")
        p = torch.zeros_like(d)
        d[:N] = torch.from_numpy(f.ravel()).to(rdt).cuda()
        plan.solve_passes(d, p, passes)
        torch.cuda.synchronize()
        out = (d if passes == 4 else p).cpu().numpy()
        if passes == 5:
            got = out[:N].reshape(n)
        else:
            spec = out[:2 * n[0] * n[1] * nhp].view(cdt).reshape(n[0], n[1], nhp)
            got = spec[:, :, :nh]
        assert rel_l2(got, want[passes - 1]) <= tol, (n, passes)


def test_passes_argument_checks(torch_cuda, ff):
    plan = ff.Plan((8, 8, 8))
    d = torch_cuda.zeros(plan.nbytes // 8, dtype=torch_cuda.float64, device="cuda")
    p = torch_cuda.zeros_like(d)
    for bad in (0, 6):
        with pytest.raises(ff.FFError) as e:
            plan.solve_passes(d, p, bad)
        assert e.value.status == ff.FF_ERR_INVALID
