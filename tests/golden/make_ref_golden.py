"""Writes golden vectors from the reference itself, run on a GPU machine.

Needs oracle/_ref/ (built here by `make -C oracle/ref` from the reference's own
sources with the single-rank MPI stub).  For each grid it runs
oracle/_ref/ref_dump (reference ParisPencil + the reference init kernel) and
stores f, phi (small grids) or sampled phi values and the phi L2 norm (larger
grids), plus the relative norms of the reference phi against the analytic
solution.  It also captures the reference benchmark's own printout.

  python tests/golden/make_ref_golden.py OUTDIR [NIxNJxNK ...]   (only those grids)
"""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

REF = os.path.join(ROOT, "oracle", "_ref")
# the last two of FULL and of SAMPLED have axes with prime factors above 5
# (7, 11, 13, 17, 97, 127), which cuFFT transforms and this build runs
# through its Bluestein passes
FULL = [(8, 8, 8), (16, 16, 16), (12, 10, 8), (5, 9, 6), (2, 3, 5), (20, 15, 18), (7, 11, 13), (14, 9, 22)]
SAMPLED = [(30, 45, 50), (64, 64, 64), (100, 36, 27), (128, 96, 80), (256, 256, 256), (97, 60, 49),
           (127, 34, 64)]
PRINTOUT = [(8, 8, 8), (16, 16, 16), (64, 64, 64), (128, 128, 128), (256, 256, 256)]


def rel_norms(phi):
    from oracle import oracle as O
    return O.rel_norms(phi)


def run_dump(n, path):
    r = subprocess.run([os.path.join(REF, "ref_dump"), *map(str, n), path], capture_output=True, text=True,
                       timeout=600)
    if r.returncode:
        raise RuntimeError(r.stderr)
    raw = np.fromfile(path, dtype=np.uint8)
    N = n[0] * n[1] * n[2]
    arr = raw[12:].view(np.float64)
    return arr[:N].reshape(n), arr[N:].reshape(n), r.stdout.strip()


def main(out, only=None):
    os.makedirs(out, exist_ok=True)
    tmp = os.path.join(out, "_tmp.bin")
    for n in FULL + SAMPLED:
        if only and n not in only:
            continue
        f, phi, msg = run_dump(n, tmp)
        name = os.path.join(out, "ref_%dx%dx%d.npz" % n)
        norms = rel_norms(phi)
        if n in FULL:
            np.savez_compressed(name, n=np.array(n), f=f, phi=phi, rel_norms=np.array(norms))
        else:
            rng = np.random.default_rng(sum(n))
            idx = np.sort(rng.choice(phi.size, size=min(512, phi.size), replace=False))
            np.savez_compressed(name, n=np.array(n), idx=idx, phi_samples=phi.ravel()[idx],
                                phi_l2=np.linalg.norm(phi), rel_norms=np.array(norms))
        print(name, msg, norms, flush=True)
    os.remove(tmp)
    for n in PRINTOUT:
        if only and n not in only:
            continue
        r = subprocess.run([os.path.join(REF, "fishfry_ref"), "1", "1", "1", *map(str, n), "3"], capture_output=True,
                           text=True, timeout=600)
        with open(os.path.join(out, "ref_printout_%dx%dx%d.txt" % n), "w") as fh:
            fh.write("# oracle/_ref/fishfry_ref 1 1 1 %d %d %d 3 (exit %d)\n" % (*n, r.returncode))
            fh.write(r.stdout)
            if r.returncode:
                fh.write(r.stderr)
        print("printout", n, r.returncode, flush=True)


if __name__ == "__main__":
    sel = [tuple(int(x) for x in a.split("x")) for a in sys.argv[2:]]
    if len(sys.argv) < 2:
        sys.exit("usage: make_ref_golden.py OUT_DIR [NIxNJxNK ...]")
    main(sys.argv[1], sel or None)
