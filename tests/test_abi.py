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


# ------------------------------------------------------------------ volume files ----
import gzip  # noqa: E402
import struct  # noqa: E402

import oracle as O  # noqa: E402

_NII_TYPES = {"u1": 2, "i1": 256, "i2": 4, "u2": 512, "i4": 8, "f4": 16, "f8": 64}


def _nifti_bytes(vol, spacing, code, bo="<", onefile=True, vox_offset=352.0):
    """A NIfTI-1 file (or the .hdr of a pair) holding vol (Z, Y, X) with sample type code."""
    Z, Y, X = vol.shape
    h = bytearray(348)
    struct.pack_into(bo + "i", h, 0, 348)
    struct.pack_into(bo + "8h", h, 40, 3, X, Y, Z, 1, 1, 1, 1)
    dt = next(k for k, v in _NII_TYPES.items() if v == code)
    struct.pack_into(bo + "hh", h, 70, code, 8 * np.dtype(dt).itemsize)
    struct.pack_into(bo + "8f", h, 76, 1.0, *spacing, 0, 0, 0, 0)
    struct.pack_into(bo + "f", h, 108, vox_offset if onefile else 0.0)
    h[344:348] = b"n+1\0" if onefile else b"ni1\0"
    data = np.ascontiguousarray(vol.astype(np.dtype(dt).newbyteorder(bo))).tobytes()
    if onefile:
        return bytes(h) + b"\0" * (int(vox_offset) - 348) + data
    return bytes(h) + b"\0\0\0\0", data


def _vol(rng, shape, lo, hi):
    return rng.integers(lo, hi, shape).astype(np.int64)


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("hi", [200, 60000, 400000])
def test_scn_files_match_reference(roift, oracle_lib, tmp_path, hi):
    """.scn: the library's reader returns what Scene32::Read returns on the reference's own
    files, and its writer produces the same bytes as Scene32::Write (8 / 16 / 32-bit
    samples chosen by the maximum; negative values cast like the reference)."""
    rng = np.random.default_rng(hi)
    vol = _vol(rng, (5, 7, 9), -3 if hi < 256 else 0, hi).astype(np.int32)
    sp = (0.5, 1.25, 2.0)
    ref_path, our_path = str(tmp_path / "r.scn"), str(tmp_path / "o.scn")
    O.ref_write_volume(ref_path, vol, sp)
    roift.write_volume(our_path, vol, sp)
    assert open(ref_path, "rb").read() == open(our_path, "rb").read()
    got, gsp = roift.read_volume(ref_path)
    exp, esp = O.ref_read_volume(ref_path)
    assert np.array_equal(got, exp) and gsp == esp


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("ext", [".nii", ".hdr", ".img"])
def test_nifti_write_read_against_reference(roift, oracle_lib, tmp_path, ext):
    """NIfTI-1: files written by Scene32::Write read back identically through the library,
    and the library's files (single .nii and .hdr / .img pairs) read back identically
    through Scene32::Read."""
    rng = np.random.default_rng(5)
    vol = _vol(rng, (4, 6, 11), -70000, 70000).astype(np.int32)
    sp = (0.75, 0.75, 1.5)
    ref_path = str(tmp_path / ("r" + ext))
    O.ref_write_volume(ref_path, vol, sp)
    got, gsp = roift.read_volume(ref_path)
    assert np.array_equal(got, vol) and gsp == sp
    our_path = str(tmp_path / ("o" + ext))
    roift.write_volume(our_path, vol, sp)
    exp, esp = O.ref_read_volume(our_path)
    assert np.array_equal(exp, vol) and esp == sp


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("code", [2, 256, 4, 512, 8, 16])
@pytest.mark.parametrize("bo", ["<", ">"])
def test_nifti_sample_types_match_reference(roift, oracle_lib, tmp_path, code, bo):
    """ReadNifti1's conversions, both byte orders, one file and a pair: uint8, int8, int16,
    uint16 and int32 widened; float32 scaled by 10000 / max and rounded."""
    rng = np.random.default_rng(code)
    lo, hi = {2: (0, 256), 256: (-128, 128), 4: (-32768, 32768), 512: (0, 65536),
              8: (-2**31, 2**31 - 1), 16: (0, 1)}[code]
    shape = (3, 5, 7)
    if code == 16:
        vol = (rng.standard_normal(shape) * 40.0 + 10.0).astype(np.float32)
    else:
        vol = _vol(rng, shape, lo, hi)
    sp = (1.0, 0.5, 3.0)
    p1 = tmp_path / "a.nii"
    p1.write_bytes(_nifti_bytes(vol, sp, code, bo, vox_offset=400.0))
    hdr, img = _nifti_bytes(vol, sp, code, bo, onefile=False)
    (tmp_path / "b.hdr").write_bytes(hdr)
    (tmp_path / "b.img").write_bytes(img)
    for path in (str(p1), str(tmp_path / "b.hdr")):
        got, gsp = roift.read_volume(path)
        exp, esp = O.ref_read_volume(path)
        assert np.array_equal(got, exp) and gsp == esp


def test_volume_files_round_trip_and_errors(roift, tmp_path):
    """Round trips through every writable format (with .nii.gz read back compressed and a
    gzip copy of a plain file read the same), the dims-only query, and the errors."""
    rng = np.random.default_rng(9)
    vol = _vol(rng, (6, 5, 4), -1000, 1000).astype(np.int32)
    sp = (1.0, 2.0, 3.0)
    for name in ("v.nii", "v.nii.gz", "v.hdr", "w.img", "v.scn"):
        p = str(tmp_path / name)
        roift.write_volume(p, vol if name != "v.scn" else np.abs(vol), sp)
        got, gsp = roift.read_volume(p)
        assert np.array_equal(got, vol if name != "v.scn" else np.abs(vol)) and gsp == sp
    raw = (tmp_path / "v.nii").read_bytes()
    with gzip.open(tmp_path / "z.nii.gz", "wb") as f:
        f.write(raw)
    assert np.array_equal(roift.read_volume(str(tmp_path / "z.nii.gz"))[0], vol)
    dims, spc = (C.c_int * 3)(), (C.c_float * 3)()
    assert roift.lib().oift_b200_read_volume(os.fsencode(str(tmp_path / "v.nii")), None, 0,
                                             dims, spc) == 0
    assert tuple(dims) == (4, 5, 6)
    small = np.empty(10, np.int32)
    assert roift.lib().oift_b200_read_volume(os.fsencode(str(tmp_path / "v.nii")),
                                             small.ctypes.data, 10, dims, spc) == roift.E_RANGE
    (tmp_path / "d.nii").write_bytes(_nifti_bytes(vol.astype(np.float64), sp, 64))
    for bad, code in (("d.nii", roift.E_UNSUPPORTED), ("v.txt", roift.E_UNSUPPORTED),
                      ("missing.nii", roift.E_BAD_ARG)):
        with pytest.raises(roift.OiftError) as e:
            roift.read_volume(str(tmp_path / bad))
        assert e.value.status == code
