"""GPU tests of the multi-rank x-slab phases (ff_slab_*) through the C ABI.

All ranks of a task grid (P, 1, 1) run on one GPU, one after another, each
with its own buffers; nothing waits on another rank.  The exchanges are
device copies of blocks between the ranks' buffers (what an all-to-all
moves), or, in the direct form, each phase stores its blocks straight into
the receiving rank's buffer (as a rank with peer-mapped memory would).  The
gathered phi must match the oracle's single-grid solve: FP64 within 1e-12
relative L2, FP32 within 1e-5.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def run_ranks(torch, ff, n, P, precision, direct, f):
    from fishfry_b200.slab import SlabKernels, SlabLayout
    lo, hi, _, _ = ff.reference_domain(n)
    lay = SlabLayout(n, P, precision)
    dt = torch.float64 if precision == ff.FF_FP64 else torch.float32
    esz = 8 if precision == ff.FF_FP64 else 4
    ks = [SlabKernels(n, lo, hi, precision, P, r) for r in range(P)]
    for r, k in enumerate(ks):
        assert k.layout_ints == [P, r, lay.di, lay.djp, lay.planes(r)[0], lay.planes(r)[1] - lay.planes(r)[0],
                                 lay.rows(r)[0], lay.rows(r)[1] - lay.rows(r)[0]]
        assert k.nbytes == lay.buffer_elems(r) * esz
        assert k.block_bytes == lay.block * 2 * esz
    D = [torch.zeros(k.nbytes // esz, dtype=dt, device="cuda") for k in ks]
    Pt = [torch.zeros_like(x) for x in D]
    R = [torch.zeros_like(x) for x in D]
    for r in range(P):
        p0, p1 = lay.planes(r)
        D[r][:(p1 - p0) * n[1] * n[2]] = torch.from_numpy(f[p0:p1].ravel()).to(dt).cuda()
    bb = ks[0].block_bytes
    blk = bb // esz

    def addr(t, q):
        return t.data_ptr() + q * bb

    if not direct:
        for r in range(P):
            ks[r].forward(D[r], Pt[r], D[r])                    # send buffer: D
        for p in range(P):                                     # all-to-all: D -> Pt
            for r in range(P):
                Pt[p][r * blk:(r + 1) * blk].copy_(D[r][p * blk:(p + 1) * blk])
        for p in range(P):
            ks[p].xpass(Pt[p], D[p])
        for r in range(P):                                     # back: D -> Pt
            for p in range(P):
                Pt[r][p * blk:(p + 1) * blk].copy_(D[p][r * blk:(r + 1) * blk])
        for r in range(P):
            ks[r].backward(Pt[r], D[r], Pt[r])
    else:
        # stores straight into the receiving ranks' buffers: R receives the
        # pencils, D (free once its z pass has run) receives the blocks back
        for r in range(P):
            ks[r].forward_to(D[r], Pt[r], [addr(R[p], r) for p in range(P)])
        for p in range(P):
            ks[p].xpass_to(R[p], [addr(D[q], p) for q in range(P)])
        for r in range(P):
            ks[r].backward(D[r], R[r], Pt[r])
    torch.cuda.synchronize()
    for k in ks:
        k.check()
    out = []
    for r in range(P):
        p0, p1 = lay.planes(r)
        out.append(Pt[r][:(p1 - p0) * n[1] * n[2]].double().cpu().numpy().reshape(p1 - p0, n[1], n[2]))
    for k in ks:
        k.close()
    return np.concatenate(out, axis=0)


@pytest.mark.parametrize("direct", [False, True])
@pytest.mark.parametrize("n,P", [((64, 48, 40), 2), ((30, 45, 50), 4), ((10, 9, 8), 4), ((64, 64, 64), 1),
                                 ((128, 96, 80), 3), ((512, 64, 32), 8), ((96, 512, 36), 5), ((256, 256, 256), 4)])
def test_slab_ranks_fp64_match_oracle(torch_cuda, ff, oracle, n, P, direct):
    f = oracle.init_f(n, ff.modes_generate(7, 16, 16, ff.alias_free_kaxis(n)))
    phi = run_ranks(torch_cuda, ff, n, P, ff.FF_FP64, direct, f)
    assert rel_l2(phi, oracle.solve(f)) <= 1e-12


@pytest.mark.parametrize("n,P", [((64, 48, 40), 2), ((30, 45, 50), 3), ((128, 128, 128), 4)])
def test_slab_ranks_fp32_match_oracle(torch_cuda, ff, oracle, n, P):
    f = oracle.init_f(n, ff.modes_generate(9, 16, 16, ff.alias_free_kaxis(n)))
    phi = run_ranks(torch_cuda, ff, n, P, ff.FF_FP32, False, f.astype(np.float32).astype(np.float64))
    assert rel_l2(phi, oracle.solve(f.astype(np.float32).astype(np.float64))) <= 1e-5


def test_slab_rejects_bad_layouts(ff):
    from fishfry_b200.slab import SlabKernels
    lo, hi, _, _ = ff.reference_domain((8, 8, 8))
    for n, P, status in [((8, 3, 8), 4, ff.FF_ERR_TASKS), ((11, 8, 8), 2, ff.FF_ERR_UNSUPPORTED),
                         ((8, 8, 8), 65, ff.FF_ERR_TASKS)]:
        with pytest.raises(ff.FFError) as e:
            SlabKernels(n, lo, hi, ff.FF_FP64, P, 0)
        assert e.value.status == status, (n, P)


_NCCL_CHILD = r'''
import datetime, os, sys
import numpy as np
import torch
import torch.distributed as dist
sys.path.insert(0, sys.argv[1])
from fishfry_b200.api import FF_FP64, init_field, reference_domain
from fishfry_b200.slab import SLAB_PHASES, SlabPencil
os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=sys.argv[2], RANK="0", WORLD_SIZE="1")
torch.cuda.set_device(0)
dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
try:
    n = tuple(int(x) for x in sys.argv[3].split(","))
    N = n[0] * n[1] * n[2]
    lo, hi, _, _ = reference_domain(n)
    sp = SlabPencil(n, lo, hi, (1, 1, 1), (0, 0, 0))
    nb = sp.bytes()
    d = torch.zeros(nb // 8, dtype=torch.float64, device="cuda")
    p = torch.zeros_like(d)
    init_field(n, d[:N], None, FF_FP64)
    f = d[:N].cpu().numpy()
    stamps = []
    sp.solve(nb, d, p, stamps)
    assert [s[0] for s in stamps] == ["Total"] + SLAB_PHASES
    np.save(sys.argv[4], np.stack([f, p[:N].cpu().numpy()]))
finally:
    dist.destroy_process_group()
'''


@pytest.mark.parametrize("n", [(64, 48, 40), (30, 45, 50)])
def test_slab_pencil_over_nccl_on_one_rank(ff, oracle, n, tmp_path):
    """SlabPencil end to end on a GPU with its default device phases and the
    exchanges through NCCL's all-to-all (one rank, so each exchange is a copy
    within the GPU; ranks on several GPUs need a machine with several)."""
    import os
    import socket
    import subprocess
    import sys
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    out = tmp_path / "slab.npy"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _NCCL_CHILD, root, str(port), ",".join(map(str, n)), str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    f, phi = np.load(out)
    assert rel_l2(phi.reshape(n), oracle.solve(f.reshape(n))) <= 1e-12
