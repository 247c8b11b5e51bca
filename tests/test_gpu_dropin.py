"""Link-level drop-in: the reference's own CLI programs, compiled from their sources
unchanged, run on the GPU through this library.

  * oiftrelax.cpp linked with libgft_oift_b200.so ahead of the gft library: its calls of
    gft::ift::OIFT_Multi / ORelax_1_Multi (gft/include/gft_ift.h:108-122, 451-465) bind to the
    GPU drop-ins.  Its output equals the restated CLI chain (shift, Gaussian blur x2, OIFT,
    relaxation, conditional dilation; oiftrelax.cpp:227-414) with the lexicographic OIFT.
  * gpu/oiftrelax_fmax_gpu.cpp linked with liboift_b200.so for its extern "C"
    oift_fmax_gpu_run (gpu/oift_fmax_gpu.cu:139-149).  Its output equals R2 on the shifted,
    twice-blurred volume with the CLI's per-class table (-pol, +pol).

The programs are built by oracle/Makefile (`dropin`) where the reference tree is present and
travel prebuilt; the test is skipped without them.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import roift_b200 as rb
from roift_b200 import synth

pytestmark = pytest.mark.gpu

PROGS = O.dropin_programs()
needs_progs = pytest.mark.skipif(PROGS is None, reason="drop-in programs not built")


def _write_inputs(tmp_path, c):
    Z, Y, X = c.shape
    vol = os.path.join(tmp_path, "vol.nii")   # signed samples (a .scn file holds unsigned ones)
    rb.write_volume(vol, c.image.astype(np.int32), (1.0, 1.0, 1.0))
    seeds = os.path.join(tmp_path, "seeds.txt")
    with open(seeds, "w") as f:
        f.write(f"{len(c.seeds)}\n")
        for p, lb in zip(c.seeds, c.seed_labels):
            p = int(p)
            f.write(f"{p % X} {(p // X) % Y} {p // (X * Y)} 0 {int(lb)}\n")
    return vol, seeds


def _run(prog, vol, seeds, pol, niter, out, tmp_path):
    r = subprocess.run([prog, vol, seeds, f"{pol}", str(niter), "50", out, "0"],
                       cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    lab, _ = rb.read_volume(out)
    return lab.reshape(-1)


def _blurred(img):
    b = img.astype(np.int64)
    b = (b - min(0, int(b.min()))).astype(np.int32)
    return O.gaussian_blur(O.gaussian_blur(b).reshape(img.shape)).reshape(img.shape)


@needs_progs
@pytest.mark.parametrize("shape,pol,nl", [((20, 36, 44), -0.3, 1), ((16, 30, 70), 0.4, 2)])
def test_reference_cli_runs_on_gft_dropins(oracle_lib, tmp_path, shape, pol, nl):
    c = synth.small_case(seed=21, shape=shape, pol=pol, nlabels=nl, noise=100, contrast=500)
    c.image = (c.image.astype(np.int32) - 150).astype(np.int16)   # the CLI shifts it back
    vol, seeds = _write_inputs(str(tmp_path), c)
    out = os.path.join(str(tmp_path), "out.scn")
    niter = 6
    got = _run(PROGS[0], vol, seeds, pol, niter, out, str(tmp_path))
    exp, _ = O.oiftrelax_chain(c.image.astype(np.int32), pol, niter, 50.0, c.seeds,
                               c.seed_labels, oift="r2")
    assert np.array_equal(got, exp.reshape(-1)), f"{(got != exp.reshape(-1)).sum()} voxels differ"


@needs_progs
@pytest.mark.parametrize("shape,pol,nl", [((20, 36, 44), -0.3, 1), ((16, 30, 70), 0.4, 2)])
def test_reference_gpu_cli_runs_on_dropin_entry(oracle_lib, tmp_path, shape, pol, nl):
    c = synth.small_case(seed=22, shape=shape, pol=pol, nlabels=nl, noise=100, contrast=500)
    vol, seeds = _write_inputs(str(tmp_path), c)
    out = os.path.join(str(tmp_path), "out.scn")
    got = _run(PROGS[1], vol, seeds, pol, 0, out, str(tmp_path))
    f = _blurred(c.image.astype(np.int32))
    Z, Y, X = c.shape
    W, _ = O.build_weights(f, 6, "grad")
    per = float(np.float32(np.float32(-pol) * np.float32(100.0)))
    table = np.array([per] + [-per] * nl, np.float32)
    _, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), 6, c.seeds, c.seed_labels, per_class=table)
    assert np.array_equal(got, lab_r2), f"{(got != lab_r2).sum()} voxels differ"


@pytest.mark.parametrize("shape,pol,adj,nl", [((14, 22, 40), -0.3, 6, 1), ((1, 50, 61), 0.5, 4, 2),
                                              ((12, 18, 36), 0.2, 26, 2)])
def test_relax_host_relaxes_the_labels_it_is_given(roift, oracle_lib, shape, pol, adj, nl):
    """oift_b200_relax_host on labels that are not an OIFT result (the OIFT labels with a
    block flipped): membership bit-identical to the FP32 restatement of ORelax_1_Multi, labels
    equal to it and to the reference library."""
    c = synth.small_case(seed=23, shape=shape, pol=pol, adjacency=adj, nlabels=nl, noise=100,
                         contrast=400)
    img = c.image.astype(np.int32)
    Z, Y, X = c.shape
    W, _ = O.build_weights(img, adj, "grad")
    _, lab0, _ = O.oift_fmax(W, (X, Y, Z), adj, c.seeds, c.seed_labels, pol=pol)
    given = lab0.reshape(c.shape).copy()
    given[:, : Y // 3, : X // 3] = nl        # not an OIFT output any more
    given = given.reshape(-1)
    given[c.seeds] = c.seed_labels
    K = 5
    p = roift.make_params(c.shape, adjacency=adj, weight_mode="grad", pol=pol, sweeps=K)
    lab, memb, mask = roift._ctx().relax_host(p, img, given, c.seeds, want_membership=8,
                                              want_mask=True)
    lab32, m32, nc = O.relax(img, adj, c.seeds, given, K, pol=pol)
    assert np.array_equal(memb[: nc * c.n].view(np.uint32), m32.reshape(-1).view(np.uint32))
    assert np.array_equal(lab, lab32)
    assert np.array_equal(mask, (lab32 != 0).astype(np.uint8))
    if O.ref_available():
        assert np.array_equal(lab, O.ref_orelax_multi(img, adj, c.seeds, given, K, pol=pol))
