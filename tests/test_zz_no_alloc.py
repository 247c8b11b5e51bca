"""The allocation-free OIFT entry point (oift_b200_oift_noalloc).

It exists for callers that cannot let a library call cudaMalloc while they run (their own
memory pool already owns the GPU, or allocating would synchronise a pipeline that must not
stall).  It must give exactly the cost and label maps of the regular entry point, and keep
doing so on back-to-back calls that reuse its static device array.  This file is collected
last so that a run stopping at its first failure has already run every other test.
"""
import numpy as np
import pytest

import roift_b200 as rb
from roift_b200 import synth


def _device_case(c):
    import torch
    dev = torch.device("cuda:0")
    img = torch.from_numpy(c.image.astype(np.int16)).to(dev)
    seeds = torch.from_numpy(c.seeds).to(dev)
    labels = torch.from_numpy(c.seed_labels).to(dev)
    return img, seeds, labels


def _regular(c, img, seeds, labels, mode, per_class=None):
    import torch
    N = c.n
    cost = torch.empty(N, dtype=torch.int32, device=img.device)
    lab = torch.empty(N, dtype=torch.int32, device=img.device)
    p = rb.make_params(c.shape, adjacency=c.adjacency, weight_mode=mode, wq=4095,
                       pol=None if per_class is not None else c.pol, per_class=per_class,
                       sweeps=0)
    rb._ctx().run_device(p, img.data_ptr(), seeds.data_ptr(), labels.data_ptr(), len(c.seeds),
                         cost=cost.data_ptr(), oift_label=lab.data_ptr())
    torch.cuda.synchronize()
    return cost.cpu().numpy(), lab.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["ellipsoid64", "disc2d", "odd37", "perclass", "disc1024"])
def test_noalloc_matches_regular_entry_twice(roift, kind):
    """Full tiles (64^3, 256^2), partial tiles on every axis (37 x 41 x 29), a per-class
    polarity table with two object labels, and a 1024 x 1024 plane at the voxel limit."""
    import torch
    per_class = None
    if kind == "ellipsoid64":
        c, mode = synth.ellipsoid3d(seed=8, size=64, sweeps=0), "grad_q"
    elif kind == "disc2d":
        c, mode = synth.disc2d(seed=9), "grad"
    elif kind == "odd37":
        c, mode = synth.small_case(seed=12, shape=(29, 41, 37), pol=-0.4, nlabels=1), "grad_q"
    elif kind == "perclass":
        c, mode = synth.small_case(seed=13, shape=(20, 33, 47), pol=0.0, nlabels=2), "grad"
        per_class = np.array([-30.0, 25.0, -45.0], np.float32)
    else:
        c, mode = synth.disc2d(seed=10, size=1024), "grad"
    assert c.n <= 1 << 20
    img, seeds, labels = _device_case(c)
    cost_ref, lab_ref = _regular(c, img, seeds, labels, mode, per_class)
    for _ in range(2):  # two calls in a row share (and must reset) the static scratch
        cost = torch.full((c.n,), -7, dtype=torch.int32, device=img.device)
        lab = torch.full((c.n,), -7, dtype=torch.int32, device=img.device)
        rb.oift_noalloc(img.data_ptr(), c.shape, seeds.data_ptr(), labels.data_ptr(),
                        len(c.seeds), cost_ptr=cost.data_ptr(), label_ptr=lab.data_ptr(),
                        adjacency=c.adjacency, weight_mode=mode, wq=4095,
                        pol=None if per_class is not None else c.pol, per_class=per_class)
        torch.cuda.synchronize()
        assert np.array_equal(cost.cpu().numpy(), cost_ref)
        assert np.array_equal(lab.cpu().numpy(), lab_ref)


def test_noalloc_rejects_oversize_volume(roift):
    """More than OIFT_NOALLOC_MAX_VOXELS voxels: OIFT_E_RANGE before any device work."""
    L = rb.lib()
    rc = L.oift_b200_oift_noalloc(1, 1025, 1024, 1, 4, 1, 4095, 0.0, None, 0, 1, 1, 1, 1, 1,
                                  None)
    assert rc == -7
    assert L.oift_b200_noalloc_scratch_bytes() < 16 << 20
