"""CPU: the C-ABI library loads and exports every entry point include/*.h declares; host
argument handling needs no GPU."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names |= set(re.findall(r"OIFT_API\s+[\w\s\*]+?\b(\w+)\s*\(", txt))
    return sorted(names)


def test_header_declares_entry_points():
    names = _declared()
    for must in ["oift_fmax_gpu_run", "oift_gpu_run", "oift_b200_create",
                 "oift_b200_run_device_i16", "oift_b200_run_host"]:
        assert must in names


def test_library_exports_every_declared_symbol(roift):
    lib = C.CDLL(roift.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", roift.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(_declared()) <= exported


def test_python_mirror_lists_all_exports(roift):
    assert set(roift.EXPORTS) == set(_declared())


def test_status_strings(roift):
    L = roift.lib()
    for code in roift.STATUS:
        assert L.oift_b200_status_string(code)


def test_weight_planes(roift):
    assert roift.weight_planes(6) == 3 and roift.weight_planes(4) == 3
    assert roift.weight_planes(26) == 13 and roift.weight_planes(8) == 13
    assert roift.weight_planes(5) == 0


def test_no_cpu_fallback_without_gpu(roift):
    """Without a CUDA device the library refuses loudly instead of computing on the CPU."""
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(roift.OiftError):
        roift.Context(0)
    lab = np.full(8, -1, np.int32)
    lab[0] = 1
    with pytest.raises(roift.OiftError):
        roift.oift_fmax_gpu_run(np.zeros(8, np.int32), lab, 2, 2, 2,
                                np.zeros(2, np.float32), np.array([0], np.int32))


def test_dropin_rejects_bad_arguments_before_touching_a_gpu(roift):
    L = roift.lib()
    img = np.zeros(8, np.int32)
    lab = np.full(8, -1, np.int32)
    pc = np.zeros(2, np.float32)
    sd = np.array([0], np.int32)
    # n inconsistent with the dimensions
    assert L.oift_fmax_gpu_run(img, lab, 9, 2, 2, 2, pc, 1, sd, 1) == -1
    assert L.oift_b200_last_status() == -1
    # additive cost mode is not provided
    assert L.oift_gpu_run(1, img, lab, 8, 2, 2, 2, pc, 1, sd, 1) == -1
    assert L.oift_b200_last_status() == -8


def test_boundary_seed_injection_is_host_logic(roift, oracle_lib):
    """The CLI's boundary seeds are computed on the host by the library itself; they match
    the restatement of oiftrelax.cpp:175-224 (pinned against the reference)."""
    import oracle as O
    rng = np.random.default_rng(11)
    for stride in (1, 2, 3):
        shape = (5, 9, 12)
        lab = rng.choice([-1, -1, 0, 1], size=5 * 9 * 12).astype(np.int32)
        exp_lab, exp_seeds = O.inject_boundary_seeds(lab, shape, stride)
        got = lab.copy()
        seeds = roift.inject_boundary_seeds(got, shape, stride)
        assert np.array_equal(seeds, exp_seeds) and np.array_equal(got, exp_lab)


def test_cli_text_inputs(roift, tmp_path):
    """Seeds and per-class polarity files as the CLI reads them (oiftrelax.cpp:280-352):
    negative labels become background, out-of-volume seeds are dropped, a later seed on the
    same voxel wins, polarities are stored x100 in float."""
    shape = (4, 5, 6)
    f = tmp_path / "seeds.txt"
    f.write_text("6\n1 2 3 0 1\n0 0 0 0 -2\n5 4 3 0 2\n6 0 0 0 1\n1 2 3 0 3\n2 1 0 7 1\n")
    lab = np.full(4 * 5 * 6, -1, np.int32)
    seeds = roift.read_seeds(str(f), shape, lab)
    addr = lambda x, y, z: x + y * 6 + z * 30
    assert list(seeds) == [addr(1, 2, 3), 0, addr(5, 4, 3), addr(1, 2, 3), addr(2, 1, 0)]
    assert lab[addr(1, 2, 3)] == 3 and lab[0] == 0 and lab[addr(5, 4, 3)] == 2
    assert (lab >= 0).sum() == 4
    pf = tmp_path / "pol.txt"
    pf.write_text("3\n-0.3 0.25 1\n")
    assert np.array_equal(roift.read_polarity(str(pf)),
                          np.array([np.float32(-0.3) * np.float32(100), 25.0, 100.0], np.float32))
    (tmp_path / "short.txt").write_text("3\n0.1 0.2\n")
    with pytest.raises(roift.OiftError):
        roift.read_polarity(str(tmp_path / "short.txt"))
