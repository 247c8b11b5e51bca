"""GPU: exact weights wider than the 14-bit edge codes.

An image whose exact base weights exceed 16383 (|dI|, or |dI| + 1 on the image graph) used
to come back as OIFT_E_RANGE from the exact weight modes; the OIFT now runs with 64-bit keys and
evaluates every arc from the image (the face neighbours only for 6 / 4).  The bar is the
same as for the narrow path: cost map and labels equal the oracle's bit for bit (the
wide-range restatement of R2, pinned against the reference's IFT_fmax and OIFT_Multi in
the CPU tests; R2 on the image graph), and the relaxation after the OIFT equals the FP32
restatement of ORelax_1_Multi bit for bit.
"""
import numpy as np
import pytest

import oracle as O
from roift_b200 import synth

pytestmark = pytest.mark.gpu

CASES = [
    # shape (Z,Y,X), pol, adjacency, nlabels, intensity scale, costs beyond 32766 (a 15-bit
    # cost field would overflow; the others only exceed the 14-bit weight range)
    ((10, 14, 40), -0.3, 6, 1, 97, True),    # partial tiles on every axis
    ((16, 16, 64), 0.4, 6, 2, 131, True),    # full 32x4x4 tiles: 16-byte staging of 64-bit keys
    ((9, 21, 70), 0.4, 26, 2, 131, True),
    ((8, 12, 64), -0.5, 26, 1, 61, False),
    ((1, 45, 67), 0.5, 4, 1, 53, False),
    ((1, 40, 64), -0.2, 8, 2, 211, True),
]


def _wide_case(shape, pol, adj, nl, scale, seed=41):
    c = synth.small_case(seed=seed, shape=shape, pol=pol, adjacency=adj, nlabels=nl,
                         noise=150, contrast=300)
    img = (c.image.astype(np.int64) * scale).astype(np.int32)
    assert int(img.max()) - int(img.min()) > 16383
    return c, img


@pytest.mark.parametrize("shape,pol,adj,nl,scale,big", CASES)
def test_wide_range_oift_matches_oracle(roift, oracle_lib, shape, pol, adj, nl, scale, big):
    c, img = _wide_case(shape, pol, adj, nl, scale)
    ctx = roift._ctx()
    p = roift.make_params(shape, adjacency=adj, weight_mode="grad", pol=pol, sweeps=0)
    lab, cost, _, _, st = ctx.run_host(p, img, c.label_map(), c.seeds, want_cost=True)
    cost_r, lab_r = O.oift_fmax_wide(img.reshape(shape), adj, c.seeds, c.seed_labels, pol=pol)
    assert (int(cost_r.max()) > 32766) == big
    assert np.array_equal(cost, cost_r)
    assert np.array_equal(lab, lab_r)
    assert st.levels > 0


def test_wide_range_per_class_polarity_and_relaxation(roift, oracle_lib):
    """Per-class polarity on a range past 14 bits, then the relaxation.  The relaxation has
    its own bound, Wmax^8 * degree below FLT_MAX (Wmax = range * (1 + max|per| / 100), about
    51,500 for 6 neighbours; past it the reference's own sums overflow to inf / inf), so the
    range here, 29,600, lies between the two."""
    shape, adj = (10, 16, 40), 6
    c, img = _wide_case(shape, 0.0, adj, 3, 25)
    per_class = np.array([-30.0, 45.0, -10.0, 20.0], np.float32)
    ctx = roift._ctx()
    p = roift.make_params(shape, adjacency=adj, weight_mode="grad", per_class=per_class,
                          sweeps=0)
    lab, cost, _, _, _ = ctx.run_host(p, img, c.label_map(), c.seeds, want_cost=True)
    cost_r, lab_r = O.oift_fmax_wide(img.reshape(shape), adj, c.seeds, c.seed_labels,
                                     per_class=per_class)
    assert np.array_equal(cost, cost_r)
    assert np.array_equal(lab, lab_r)
    # 6 sweeps of the relaxation on the wide-range OIFT labels: FP32 restatement, bitwise
    p = roift.make_params(shape, adjacency=adj, weight_mode="grad", per_class=per_class,
                          sweeps=6)
    labk, _, memb, _, st = ctx.run_host(p, img, c.label_map(), c.seeds, want_membership=8)
    exp, m32, nc = O.relax(img.reshape(shape), adj, c.seeds, lab_r, 6, per_class=per_class)
    assert st.nclasses == nc
    assert np.array_equal(labk, exp)
    assert np.array_equal(memb.reshape(-1).view(np.uint32), m32.reshape(-1).view(np.uint32))


def test_wide_range_int16_device_entry(roift, oracle_lib):
    """The device entry with an int16 image whose range exceeds 16383."""
    import torch
    shape, adj, pol = (12, 20, 64), 6, -0.3
    c = synth.small_case(seed=43, shape=shape, pol=pol, adjacency=adj, nlabels=2,
                         noise=400, contrast=20000)
    img16 = c.image.astype(np.int16)
    assert int(img16.max()) - int(img16.min()) > 16383
    dev = torch.device("cuda", 0)
    d_img = torch.from_numpy(img16.reshape(-1).copy()).to(dev)
    d_sd = torch.from_numpy(c.seeds.astype(np.int32)).to(dev)
    d_sl = torch.from_numpy(c.seed_labels.astype(np.int32)).to(dev)
    d_cost = torch.empty(c.n, dtype=torch.int32, device=dev)
    d_lab = torch.empty(c.n, dtype=torch.int32, device=dev)
    ctx = roift._ctx()
    p = roift.make_params(shape, adjacency=adj, weight_mode="grad", pol=pol, sweeps=0)
    ctx.run_device(p, d_img.data_ptr(), d_sd.data_ptr(), d_sl.data_ptr(), len(c.seeds),
                   cost=d_cost.data_ptr(), oift_label=d_lab.data_ptr())
    torch.cuda.synchronize()
    cost_r, lab_r = O.oift_fmax_wide(img16.astype(np.int32), adj, c.seeds, c.seed_labels, pol=pol)
    assert np.array_equal(d_cost.cpu().numpy(), cost_r)
    assert np.array_equal(d_lab.cpu().numpy(), lab_r)


def test_wide_range_image_graph(roift, oracle_lib):
    """The 2D image graph (|dI| + 1, rounded orientation) past the 14-bit range."""
    shape, adj, pol = (1, 37, 70), 8, 0.2
    c, img = _wide_case(shape, pol, adj, 2, 113)
    img2 = img.reshape(shape[1:])
    ctx = roift._ctx()
    p = roift.make_params(shape, adjacency=adj, weight_mode="imagegraph", pol=pol, sweeps=0)
    lab, cost, _, _, _ = ctx.run_host(p, img, c.label_map(), c.seeds, want_cost=True)
    cost_r2, lab_r2, _ = O.oift_fmax_imagegraph(img2, adj, c.seeds, c.seed_labels, pol)
    assert int(cost_r2.max()) > 32766
    assert np.array_equal(cost, cost_r2)
    assert np.array_equal(lab, lab_r2)


def test_range_beyond_wide_keys_is_rejected(roift):
    """Exact weights above 2^30 - 1 still return OIFT_E_RANGE."""
    shape = (4, 8, 32)
    img = np.zeros(int(np.prod(shape)), np.int32)
    img[5] = 1 << 30
    lab = np.full(img.size, -1, np.int32)
    lab[0] = 1
    lab[img.size - 1] = 0
    seeds = np.array([0, img.size - 1], np.int32)
    ctx = roift._ctx()
    p = roift.make_params(shape, adjacency=6, weight_mode="grad", pol=0.3, sweeps=0)
    with pytest.raises(roift.OiftError) as e:
        ctx.run_host(p, img, lab, seeds)
    assert e.value.status == roift.E_RANGE


def test_wide_range_through_the_reference_entry(roift, oracle_lib):
    """oift_fmax_gpu_run (the reference's entry, gpu/oift_fmax_gpu.cu:139-149) on an int
    image whose neighbouring intensities differ by far more than 16383: the labels equal the
    wide-range R2's, and where the reference library is present, the reference OIFT_Multi
    labels have the same cut energy."""
    shape, adj = (12, 30, 40), 6
    c, img = _wide_case(shape, -0.4, adj, 2, 157)
    Z, Y, X = c.shape
    per_class = np.array([40.0, -40.0, -40.0], np.float32)
    lab = c.label_map()
    levels = roift.oift_fmax_gpu_run(img, lab, X, Y, Z, per_class, c.seeds)
    _, lab_r = O.oift_fmax_wide(img.reshape(shape), adj, c.seeds, c.seed_labels,
                                per_class=per_class)
    assert levels > 0
    assert np.array_equal(lab, lab_r)
    if O.ref_available():
        lab_ref = O.ref_oift_multi(img, adj, c.seeds, c.seed_labels, per_class=per_class)
        assert O.energy_wide(img.reshape(shape), adj, lab, per_class=per_class) == \
            O.energy_wide(img.reshape(shape), adj, lab_ref, per_class=per_class)
