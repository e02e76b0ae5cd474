"""CPU tests of the native boundary: the C-ABI library loads and exports every
symbol include/fishfry.h declares, host-side argument checks return the
documented statuses without touching a GPU, the host mode generator matches
the oracle's restatement, and the C++ drop-in headers compile."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fishfry.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ff_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(ff):
    syms = declared_symbols()
    assert len(syms) >= 12
    L = ctypes.CDLL(ff.LIB_PATH)
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert sorted(ff.EXPORTS) == sorted(s for s in syms if s in ff.EXPORTS)
    assert set(syms) <= set(ff.EXPORTS), set(syms) - set(ff.EXPORTS)


def test_version_and_status_strings(ff):
    L = ff.lib()
    assert b"sm_100a" in L.ff_version()
    assert L.ff_status_string(ff.FF_ERR_UNSUPPORTED) == b"unsupported size"
    assert L.ff_phase_name(None, 0) == b""
    assert L.ff_plan_phases(None) == 0


# lengths up to FF_MAX_AXIS plan (prime factors above 7 through the
# Bluestein passes, where their convolution fits); longer axes and
# non-positive ones are refused before any device call
@pytest.mark.parametrize("n,status", [((4097, 7, 8), "FF_ERR_UNSUPPORTED"), ((8, 8, 4097), "FF_ERR_UNSUPPORTED"),
                                      ((0, 8, 8), "FF_ERR_INVALID"), ((8, -2, 8), "FF_ERR_INVALID"),
                                      ((8, 8, 8192), "FF_ERR_UNSUPPORTED"), ((8, 5000, 8), "FF_ERR_UNSUPPORTED")])
def test_plan_rejects_bad_sizes_before_any_device_call(ff, n, status):
    with pytest.raises(ff.FFError) as e:
        ff.Plan(n)
    assert e.value.status == getattr(ff, status)


def test_plan_rejects_bad_precision(ff):
    with pytest.raises(ff.FFError) as e:
        ff.Plan((8, 8, 8), precision=3)
    assert e.value.status == ff.FF_ERR_INVALID


def test_paris_pencil_rejects_task_grid(ff):
    lo, hi, _, _ = ff.reference_domain((8, 8, 8))
    with pytest.raises(ff.FFError) as e:
        ff.ParisPencil((8, 8, 8), lo, hi, m=(2, 1, 1), id=(0, 0, 0))
    assert e.value.status == ff.FF_ERR_TASKS


def test_modes_generator_matches_oracle(ff, oracle):
    for seed, count, kaxis in [(12345, 64, (32, 32, 32)), (1, 10, (15, 23, 7)), (99, 64, (0, 3, 0))]:
        a = ff.modes_generate(seed, count, 32, kaxis)
        b = oracle.modes_generate(seed, count, 32, kaxis)
        assert a == b


def test_alias_free_kaxis(ff):
    assert ff.alias_free_kaxis((32, 48, 128)) == (15, 23, 32)
    assert ff.alias_free_kaxis((1, 2, 3)) == (0, 0, 1)


def test_cpp_headers_compile(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "FishFry.hpp"\n#include "ParisPencil.hpp"\n'
                   "template class FishFry<ParisPencil>;\nint main() { return 0; }\n")
    cuda_inc = "/usr/local/cuda/include"
    r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"),
                        "-I" + cuda_inc, str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_driver_arguments_checked_on_host(ff):
    exe = os.path.join(ROOT, "fishfry_b200", "bin", "fishfry")
    if not os.path.exists(exe):
        pytest.skip("driver not built")
    r = subprocess.run([exe, "1", "1", "1"], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    r = subprocess.run([exe, "2", "1", "1", "8", "8", "8"], capture_output=True, text=True)
    assert r.returncode == ff.FF_ERR_TASKS
    r = subprocess.run([exe, "1", "1", "1", "8", "0", "8"], capture_output=True, text=True)
    assert r.returncode == 1


# (lengths the batch kernels do not take, e.g. 11 or 576, are accepted and
# solved by single-grid plans; see test_batch_gpu.py)
@pytest.mark.parametrize("dims,status", [([], "FF_ERR_INVALID"), ([(8, 8, 4097)], "FF_ERR_UNSUPPORTED"),
                                         ([(8, 8, 8), (0, 4, 4)], "FF_ERR_INVALID"),
                                         ([(5000, 8, 8)], "FF_ERR_UNSUPPORTED"), ([(8, -1, 8)], "FF_ERR_INVALID")])
def test_batch_rejects_bad_dims_before_any_device_call(ff, dims, status):
    with pytest.raises(ff.FFError) as e:
        ff.Batch(dims)
    assert e.value.status == getattr(ff, status)


def test_batch_rejects_bad_precision(ff):
    with pytest.raises(ff.FFError) as e:
        ff.Batch([(8, 8, 8)], precision=5)
    assert e.value.status == ff.FF_ERR_INVALID
