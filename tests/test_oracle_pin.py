"""CPU: the oracle (C restatement) pinned against the reference itself.

Two anchors: the golden fixtures in tests/golden/ (produced by the reference library,
tests/golden/make_golden.py), and -- where oracle/_ref/libgft_ref.so is present -- the
live reference on fresh seeded inputs.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
from roift_b200 import synth

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _pol_args(d):
    pc = d["per_class"]
    if pc.size:
        return dict(pol=None, per_class=pc)
    return dict(pol=float(d["pol"]), per_class=None)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden(oracle_lib, path):
    d = np.load(path)
    img = d["image"]
    Z, Y, X = img.shape
    adj = int(d["adjacency"])
    seeds, sl = d["seeds"], d["seed_labels"]
    pa = _pol_args(d)
    W, ncl = O.build_weights(img, adj, "grad")
    assert ncl == 0
    # R1 (restated OIFT_Multi) reproduces the reference labels bit for bit
    lab_r1, val, pred, fmax = O.oift_prim(W, (X, Y, Z), adj, seeds, sl, **pa)
    assert np.array_equal(lab_r1, d["ref_oift_label"])
    # R2 (lexicographic f_max): same cut energy as the reference segmentation, and the
    # f_max derived along the reference forest equals the R2 cost map
    cost, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), adj, seeds, sl, **pa)
    nl = int(max(sl.max(), 0)) + 1
    e_ref, elb_ref = O.energy(W, (X, Y, Z), adj, d["ref_oift_label"], nl, **pa)
    e_r2, elb_r2 = O.energy(W, (X, Y, Z), adj, lab_r2, nl, **pa)
    assert e_ref == e_r2
    assert np.array_equal(fmax, cost)
    if "ref_ift_fmax_cost" in d.files:
        ns = np.ones(img.size, bool)
        ns[seeds] = False
        assert np.array_equal(d["ref_ift_fmax_cost"][ns] - 1, cost[ns])
    # R3 FP32 relaxation reproduces ORelax_1_Multi labels
    lab_rel, m32, nc = O.relax(img, adj, seeds, d["ref_oift_label"], int(d["sweeps"]), **pa)
    assert np.array_equal(lab_rel, d["ref_relax_label"])
    lab64, m64, _ = O.relax(img, adj, seeds, d["ref_oift_label"], int(d["sweeps"]), fp64=True, **pa)
    assert np.abs(m32.astype(np.float64) - m64).max() < 1e-5
    # blur restatement
    assert np.array_equal(O.gaussian_blur(img), d["ref_blur"])


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("seed,shape,pol,adj,nl", [
    (1, (14, 18, 22), -0.3, 6, 1), (2, (14, 18, 22), 0.4, 6, 2), (3, (8, 10, 14), 0.2, 26, 2),
    (4, (1, 50, 60), 0.5, 4, 1), (5, (1, 40, 44), -0.4, 8, 3)])
def test_oracle_matches_live_reference(oracle_lib, seed, shape, pol, adj, nl):
    c = synth.small_case(seed=seed, shape=shape, pol=pol, adjacency=adj, nlabels=nl,
                         noise=150, contrast=300)
    img = c.image.astype(np.int32)
    Z, Y, X = c.shape
    W, _ = O.build_weights(img, adj, "grad")
    lab_ref = O.ref_oift_multi(img, adj, c.seeds, c.seed_labels, pol=pol)
    lab_r1, _, _, fmax = O.oift_prim(W, (X, Y, Z), adj, c.seeds, c.seed_labels, pol=pol)
    assert np.array_equal(lab_r1, lab_ref)
    cost, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), adj, c.seeds, c.seed_labels, pol=pol)
    e1, _ = O.energy(W, (X, Y, Z), adj, lab_ref, nl + 1, pol=pol)
    e2, _ = O.energy(W, (X, Y, Z), adj, lab_r2, nl + 1, pol=pol)
    assert e1 == e2
    rel_ref = O.ref_orelax_multi(img, adj, c.seeds, lab_ref, 4, pol=pol)
    rel, _, _ = O.relax(img, adj, c.seeds, lab_ref, 4, pol=pol)
    assert np.array_equal(rel, rel_ref)


def test_oracle_planted_mistake_is_caught(oracle_lib):
    """A wrong polarity sign in the oracle input must change the labels or energy: the
    checker is sensitive to the orientation it is meant to pin."""
    c = synth.small_case(seed=9, shape=(12, 16, 20), pol=-0.5, nlabels=1, noise=150,
                         contrast=300)
    img = c.image.astype(np.int32)
    Z, Y, X = c.shape
    W, _ = O.build_weights(img, 6, "grad")
    c1, l1, _ = O.oift_fmax(W, (X, Y, Z), 6, c.seeds, c.seed_labels, pol=-0.5)
    c2, l2, _ = O.oift_fmax(W, (X, Y, Z), 6, c.seeds, c.seed_labels, pol=+0.5)
    assert not np.array_equal(c1, c2)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_tie_accounting_on_golden(oracle_lib, path):
    """R2 labels against the reference OIFT_Multi labels of the fixtures: every difference
    is an equal-cost tie, and a fixture without tie voxels has no difference."""
    d = np.load(path)
    img = d["image"]
    Z, Y, X = img.shape
    adj = int(d["adjacency"])
    seeds, sl = d["seeds"], d["seed_labels"]
    pa = _pol_args(d)
    W, _ = O.build_weights(img, adj, "grad")
    cost, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), adj, seeds, sl, **pa)
    ts = O.tie_stats(W, (X, Y, Z), adj, cost, lab_r2, d["ref_oift_label"], seeds, **pa)
    assert ts["diffs"] == int((lab_r2 != d["ref_oift_label"]).sum())
    assert ts["unexplained"] == 0, ts
    if ts["ties"] == 0:
        assert ts["diffs"] == 0


def test_tie_accounting_known_ties_and_planted_mistake(oracle_lib):
    """A flat image: every arc weighs 0, so both labels can reach every free voxel at cost
    0.  R2 gives all of them the smaller label (its tie voxels are the object seed's
    neighbours), the Prim order the label that arrives first; each difference is explained.  A label flipped on a tie-free
    volume (planted in the oracle's output, on the CPU) is reported as unexplained."""
    img = np.full((1, 6, 9), 50, np.int32)
    X, Y, Z = 9, 6, 1
    seeds = np.array([0, 8 + 5 * 9], np.int32)
    sl = np.array([1, 0], np.int32)
    W, _ = O.build_weights(img, 4, "grad")
    cost, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), 4, seeds, sl, pol=0.0)
    lab_r1 = O.oift_prim(W, (X, Y, Z), 4, seeds, sl, pol=0.0)[0]
    ts = O.tie_stats(W, (X, Y, Z), 4, cost, lab_r2, lab_r1, seeds, pol=0.0)
    assert ts["ties"] == 2
    assert ts["diffs"] > 0 and ts["unexplained"] == 0
    # tie-free volume (the 256^3 workload generator at 64^3): no tie, no difference, and a
    # flipped label is caught
    c = synth.ellipsoid3d(seed=2, size=64, sweeps=1)
    img = c.image.astype(np.int32)
    Z, Y, X = c.shape
    W, _ = O.build_weights(img, 6, "grad_q", wq=4095)
    cost, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), 6, c.seeds, c.seed_labels, pol=c.pol)
    lab_r1, _, _, fm = O.oift_prim(W, (X, Y, Z), 6, c.seeds, c.seed_labels, pol=c.pol)
    assert np.array_equal(fm, cost)
    assert O.tie_stats(W, (X, Y, Z), 6, cost, lab_r2, lab_r1, c.seeds, pol=c.pol) == \
        {"ties": 0, "diffs": 0, "explained": 0, "unexplained": 0}
    seeded = np.zeros(c.n, bool)
    seeded[c.seeds] = True
    p = int(np.flatnonzero(~seeded & (lab_r2 == 1))[0])
    bad = lab_r2.copy()
    bad[p] = 0
    ts = O.tie_stats(W, (X, Y, Z), 6, cost, bad, lab_r1, c.seeds, pol=c.pol)
    assert ts["diffs"] == 1 and ts["unexplained"] == 1


def test_weight_builder_modes(oracle_lib):
    img = np.array([[[0, 10, 5000, 4990]]], np.int32)
    W, ncl = O.build_weights(img, 6, "grad_q", wq=4095)
    # plane +x: |0-10| with I_p < I_q, |10-5000| clamped, |5000-4990| with I_p > I_q
    assert W[0] == (10 | 0x4000) and W[1] == (4095 | 0x4000) and W[2] == (10 | 0x8000)
    assert ncl == 1
    W, _ = O.build_weights(img, 6, "rbf_q", wq=4095, rbf_sigma=150.0)
    assert (W[1] & 0x3FFF) == 4095 and (W[0] & 0x3FFF) == round(4095 * (1 - np.exp(-100 / 45000)))


CLI_GOLDEN = [p for p in GOLDEN if "ref_chain_label" in np.load(p).files]


@pytest.mark.parametrize("path", CLI_GOLDEN, ids=[os.path.basename(p)[:-4] for p in CLI_GOLDEN])
def test_cli_steps_match_golden(oracle_lib, path):
    """Conditional dilation, boundary seeds and the whole CLI chain (shift, blur x2,
    OIFT_Multi, ORelax_1_Multi, dilation) restated against the reference's outputs."""
    d = np.load(path)
    img = d["image"]
    shape = img.shape
    seeds, sl = d["seeds"], d["seed_labels"]
    lab, n = O.conditional_dilation(d["ref_blur"].reshape(shape), d["ref_relax_label"], 1.0, 50.0)
    assert np.array_equal(lab, d["ref_dilated_p50"]) and n > 0
    chain_lab = np.full(img.size, -1, np.int32)
    chain_lab[seeds] = sl
    bl, bs = O.inject_boundary_seeds(chain_lab, shape, 2)
    assert np.array_equal(bl, d["ref_boundary_label"])
    assert np.array_equal(np.concatenate([seeds, bs]), d["ref_boundary_seeds"])
    out, _ = O.oiftrelax_chain(d["chain_image"], float(d["pol"]), int(d["sweeps"]), 50.0,
                               seeds, sl, oift="r1")
    assert np.array_equal(out, d["ref_chain_label"])


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("trial", range(24))
def test_dilation_and_boundary_seeds_match_live_reference(oracle_lib, trial):
    """Random label maps with NIL / 0 / 1, heavy ties in the intensities, several radii
    and percentiles (including the 0 and 100 ends and past 100)."""
    rng = np.random.default_rng(500 + trial)
    Z, Y, X = int(rng.integers(1, 9)), int(rng.integers(2, 14)), int(rng.integers(2, 14))
    img = rng.integers(0, 6 if trial % 2 else 3000, size=(Z, Y, X)).astype(np.int32)
    lab = rng.choice([-1, 0, 0, 0, 1], size=Z * Y * X).astype(np.int32)
    r = [1.0, 1.5, 2.0][trial % 3]
    pc = [0.0, 37.5, 50.0, 99.0, 100.0, 150.0][trial % 6]
    a, _ = O.conditional_dilation(img, lab, r, pc)
    assert np.array_equal(a, O.ref_dilation_conditional(img, lab, r, pc))
    stride = [1, 2, 3][trial % 3]
    la, sa = O.inject_boundary_seeds(lab, (Z, Y, X), stride)
    lb, sb = O.ref_inject_boundary_seeds(lab, (Z, Y, X), stride, np.zeros(0, np.int32))
    assert np.array_equal(la, lb) and np.array_equal(sa, sb)


C2F_GOLDEN = [p for p in GOLDEN if "ref_c2f_label" in np.load(p).files]


@pytest.mark.parametrize("path", C2F_GOLDEN, ids=[os.path.basename(p)[:-4] for p in C2F_GOLDEN])
def test_coarse_to_fine_matches_golden(oracle_lib, path):
    """The restated cascade (Subsampling, first-seed coarse map, coarse OIFT + relaxation,
    nearest ScaleLabel, NIL band, merge, all-labelled fine seeds, fine OIFT + relaxation,
    dilation) with OIFT_Multi's order reproduces the reference experiment's labels."""
    d = np.load(path)
    f = d["c2f_image"]
    seeds, sl = d["seeds"], d["seed_labels"]
    lab0 = np.full(f.size, -1, np.int32)
    lab0[seeds] = sl
    out = O.coarse_to_fine(f, int(d["adjacency"]), float(d["pol"]), int(d["sweeps"]), 50.0,
                           seeds, lab0, oift="r1")
    assert np.array_equal(out, d["ref_c2f_label"])


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("shape,adj,pol", [((12, 20, 26), 6, -0.3), ((11, 17, 23), 6, 0.5),
                                           ((10, 14, 18), 26, 0.2), ((1, 40, 52), 6, 0.4)])
def test_coarse_to_fine_matches_live_reference(oracle_lib, shape, adj, pol):
    c = synth.small_case(seed=40 + shape[1], shape=shape, pol=pol, adjacency=adj,
                         nlabels=2 if adj == 26 else 1, noise=120, contrast=400)
    img = c.image.astype(np.int32)
    f = O.gaussian_blur(O.gaussian_blur(img).reshape(shape)).reshape(shape)
    lab = np.full(img.size, -1, np.int32)
    lab[c.seeds] = c.seed_labels
    ref = O.ref_coarse_to_fine(f, adj, pol, 5, 50.0, c.seeds, lab)
    assert np.array_equal(O.coarse_to_fine(f, adj, pol, 5, 50.0, c.seeds, lab, oift="r1"), ref)


@pytest.mark.parametrize("kernel,adj", [("rbf", 6), ("pow8", 6), ("rbf", 26)])
def test_fp64_adjoint_matches_central_differences(kernel, adj):
    """The FP64 reverse-mode gradient of the relaxation (the checker of the CUDA adjoint)
    equals central differences of its own FP64 forward."""
    from oracle import adjoint as A
    rng = np.random.default_rng(0)
    Z, Y, X = 6, 9, 11
    img = rng.integers(0, 400, size=(Z, Y, X)).astype(float)
    img[2:5, 3:7, 3:9] += 600
    lab = np.zeros(Z * Y * X, np.int64)
    lab.reshape(Z, Y, X)[2:5, 3:7, 3:9] = 1
    seeds = np.array([0, 1, 2, np.ravel_multi_index((3, 5, 5), (Z, Y, X))])
    sl = np.array([0, 0, 0, 1])
    truth = lab.copy()
    truth.reshape(Z, Y, X)[2, 3, 3] = 0
    g = rng.integers(0, 300, size=(Z, Y, X)).astype(float)
    P = A.Problem(img, lab, seeds, sl, truth, adj=adj, grad=g, K=6, kernel=kernel)
    th = np.array([150.0, 0.3, 0.7])
    _, gr = P.gradient(*th)
    for i, h in enumerate([1e-3 * th[0], 1e-5, 1e-5]):
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fd = (P.forward(*tp)[0] - P.forward(*tm)[0]) / (2 * h)
        assert abs(gr[i] - fd) <= 1e-6 * max(abs(fd), 1e-9), (i, gr[i], fd)


BLEND_GOLDEN = [p for p in GOLDEN if "ref_blend_oift_label" in np.load(p).files]


@pytest.mark.parametrize("path", BLEND_GOLDEN, ids=[os.path.basename(p)[:-4] for p in BLEND_GOLDEN])
def test_blend_weights_match_golden(oracle_lib, path):
    """The Sobel gradient normalised to the image maximum, OIFT_Multi_GradWeight (R1 with
    blend weights) and ORelax_1_Multi_GradWeight restated against the reference experiment."""
    d = np.load(path)
    f = d["blend_image"]
    seeds, sl = d["seeds"], d["seed_labels"]
    pol, K, adj = float(d["pol"]), int(d["sweeps"]), int(d["adjacency"])
    g = O.sobel_normalized(f)
    assert np.array_equal(g, d["ref_sobel"])
    lab = O.oift_prim_blend(f, g, 0.6, adj, seeds, sl, pol=pol)
    assert np.array_equal(lab, d["ref_blend_oift_label"])
    out, _ = O.relax_blend(f, g, 0.6, adj, seeds, lab, K, pol)
    assert np.array_equal(out, d["ref_blend_relax_label"])


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("i,shape,pol,alpha", [(0, (12, 16, 20), -0.3, 0.6),
                                               (1, (10, 14, 18), 0.5, 0.3),
                                               (2, (9, 13, 25), 0.0, 1.0),
                                               (3, (8, 12, 16), 0.4, 0.0)])
def test_blend_weights_match_live_reference(oracle_lib, i, shape, pol, alpha):
    c = synth.small_case(seed=60 + i, shape=shape, pol=pol, adjacency=6,
                         nlabels=1 if i % 2 == 0 else 2, noise=120, contrast=400)
    img = c.image.astype(np.int32)
    f = O.gaussian_blur(O.gaussian_blur(img).reshape(shape)).reshape(shape)
    g = O.sobel_normalized(f)
    assert np.array_equal(g, O.ref_sobel_normalized(f))
    lr = O.ref_gradweight(f, g, alpha, c.seeds, c.seed_labels, pol, 0)
    assert np.array_equal(O.oift_prim_blend(f, g, alpha, 6, c.seeds, c.seed_labels, pol=pol), lr)
    out, _ = O.relax_blend(f, g, alpha, 6, c.seeds, lr, 7, pol)
    assert np.array_equal(out, O.ref_gradweight(f, g, alpha, c.seeds, c.seed_labels, pol, 7))


# --------------------------------------------------------- the 2D image graph ----
IG_GOLDEN = [p for p in GOLDEN if "ref_ig_oift_label" in np.load(p).files]


def _ig_inputs(d):
    shape = d["image"].shape
    return d["image"].reshape(shape[1:]), d["seeds"], d["seed_labels"]


@pytest.mark.parametrize("path", IG_GOLDEN, ids=[os.path.basename(p)[:-4] for p in IG_GOLDEN])
def test_imagegraph_matches_golden(oracle_lib, path):
    """OIFT(sImageGraph) and ORelax_1(sImageGraph) on ByEuclideanDistance + Orient2Digraph
    restated against the reference: R1 labels (every labelled pixel queued in address
    order, as S = NULL does), Wmax, the cut energy of R2's labels, the relaxed labels."""
    d = np.load(path)
    img, seeds, sl = _ig_inputs(d)
    pol, K, adj = float(d["pol"]), int(d["sweeps"]), int(d["adjacency"])
    order = np.argsort(seeds, kind="stable")
    assert O.imagegraph_wmax(img, adj, pol) == int(d["ref_ig_wmax"])
    lab, _, _, _ = O.oift_prim_imagegraph(img, adj, seeds[order], sl[order], pol)
    assert np.array_equal(lab, d["ref_ig_oift_label"])
    assert O.energy_imagegraph(img, adj, lab, pol) == int(d["ref_ig_energy"])
    _, lab_r2, _ = O.oift_fmax_imagegraph(img, adj, seeds, sl, pol)
    assert O.energy_imagegraph(img, adj, lab_r2, pol) == int(d["ref_ig_energy"])
    out, m = O.relax_imagegraph(img, adj, seeds, lab, K, pol)
    assert np.array_equal(out, d["ref_ig_relax_label"])
    assert np.array_equal(out, (~(m < 0.5)).astype(np.int32))


def _ig_random_case(rng, trial):
    adj = (4, 8)[trial % 2]
    Y, X = (int(v) for v in rng.integers(8, 40, 2))
    pol = float(rng.choice([-1.0, -0.5, -0.3, 0.0, 0.2, 0.5, 0.9, 1.0]))
    img = rng.integers(0, 60, (Y, X)).astype(np.int32)
    if trial % 3 == 0:  # a noisy disc, as the 2D CLI case
        yy, xx = np.mgrid[:Y, :X]
        disc = (yy - Y / 2) ** 2 + (xx - X / 2) ** 2 < (min(X, Y) / 3) ** 2
        img = np.clip(np.where(disc, 180, 60) + rng.normal(0, 12, (Y, X)), 0, 255).astype(np.int32)
    border = [p for p in range(X * Y) if p % X in (0, X - 1) or p // X in (0, Y - 1)]
    c = (Y // 2) * X + X // 2
    obj = {c, c + 1, c + X}
    seeds = np.array(sorted(set(border) | obj), np.int32)
    sl = np.array([1 if s in obj else 0 for s in seeds], np.int32)
    return img, adj, pol, seeds, sl, int(rng.integers(0, 12))


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
def test_imagegraph_matches_live_reference(oracle_lib):
    """60 random 2D cases, both neighbourhoods, alpha in [-1, 1]: R1 labels, Wmax and the
    relaxed labels equal the reference's; R2's labels have the reference's cut energy.
    (The f_max along the reference's Prim forest may differ from R2's cost on these
    oriented graphs, where a label's competition can block another's path; those pixels
    are counted, not required to be zero.)"""
    rng = np.random.default_rng(0)
    fmax_diff = 0
    for trial in range(60):
        img, adj, pol, seeds, sl, K = _ig_random_case(rng, trial)
        ref_lab, wmax = O.ref_imagegraph(img, adj, seeds, sl, pol, 0)
        assert wmax == O.imagegraph_wmax(img, adj, pol)
        r1, _, _, fm = O.oift_prim_imagegraph(img, adj, seeds, sl, pol)
        assert np.array_equal(r1, ref_lab), trial
        cost, r2, _ = O.oift_fmax_imagegraph(img, adj, seeds, sl, pol)
        fmax_diff += int((fm != cost).sum())
        e = O.ref_imagegraph_energy(img, adj, ref_lab, pol)
        assert O.energy_imagegraph(img, adj, ref_lab, pol) == e
        assert O.energy_imagegraph(img, adj, r2, pol) == e
        out, _ = O.relax_imagegraph(img, adj, seeds, ref_lab, K, pol)
        exp = O.ref_imagegraph(img, adj, seeds, sl, pol, K)[0] if K else None
        if K:
            assert np.array_equal(out, exp), trial
    print("pixels where the Prim-forest f_max differs from R2:", fmax_diff)


@pytest.mark.parametrize("adj,shape", [(6, (16, 20, 24)), (4, (1, 40, 52)), (26, (10, 14, 18))])
def test_bottleneck_arcs_carry_the_cost_and_gradient_is_exact(oracle_lib, adj, shape):
    """Restated bottleneck arcs: every reached non-seed voxel gets one; the arc's tail has the
    voxel's label and its integer oriented weight equals the voxel's f_max cost; the FP64
    cost-map loss has the gradient of its central differences."""
    from oracle import adjoint as AD
    c = synth.small_case(seed=44, shape=shape, pol=-0.3, adjacency=adj, nlabels=1, noise=120,
                         contrast=400)
    img = c.image.astype(np.int32)
    Z, Y, X = c.shape
    W, _ = O.build_weights(img, adj, "grad_q", wq=4095)
    cost, lab, _ = O.oift_fmax(W, (X, Y, Z), adj, c.seeds, c.seed_labels, pol=c.pol)
    arcs = AD.bottleneck_arcs(img.reshape(c.shape), cost, lab, c.seeds, adj, c.pol)
    assert not (arcs == -1).any()
    has = arcs >= 0
    offs = np.array(AD.offsets(adj))
    tail, d = arcs[has] >> 5, arcs[has] & 31
    head = (tail % X + offs[d, 0]) + ((tail // X) % Y + offs[d, 1]) * X + (tail // (X * Y) + offs[d, 2]) * X * Y
    assert np.array_equal(lab[tail], lab[has])
    I = img.reshape(-1).astype(np.int64)
    base = np.minimum(np.abs(I[tail] - I[head]), 4095)
    per = float(np.float32(c.pol * 100.0))
    pl = np.where(lab[tail] == 0, -per, per)
    f = np.where(I[tail] > I[head], 1.0 + pl / 100.0, np.where(I[tail] < I[head], 1.0 - pl / 100.0, 1.0))
    assert np.array_equal(np.floor(base * f).astype(np.int64), cost[has].astype(np.int64))
    truth = (img.reshape(-1) > 850).astype(np.uint8)
    th = np.array([160.0, 0.2, 0.9])
    g = np.abs(np.gradient(img.astype(np.float64), axis=-1))
    loss, grad = AD.cost_loss(img.reshape(c.shape), lab, arcs, truth, *th, adj=adj, g=g)
    h = 1e-3
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        fd = (AD.cost_loss(img.reshape(c.shape), lab, arcs, truth, *(th + e), adj=adj, g=g)[0] -
              AD.cost_loss(img.reshape(c.shape), lab, arcs, truth, *(th - e), adj=adj, g=g)[0]) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-6 * abs(grad[k]) + 1e-9


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("seed,shape,pol,adj,nl,scale", [
    (21, (10, 14, 18), -0.3, 6, 1, 97), (22, (8, 12, 16), 0.4, 26, 2, 131),
    (23, (1, 40, 44), 0.5, 4, 1, 53), (24, (1, 30, 36), -0.2, 8, 2, 211)])
def test_wide_range_oracle_matches_live_reference(oracle_lib, seed, shape, pol, adj, nl, scale):
    """The restatement for exact weights wider than the 14-bit edge codes: at polarity 0 its
    cost map plus one is the reference IFT_fmax cost map, and at any polarity the reference
    OIFT_Multi labels and its labels have the same oriented cut energy."""
    c = synth.small_case(seed=seed, shape=shape, pol=pol, adjacency=adj, nlabels=nl,
                         noise=150, contrast=300)
    img = (c.image.astype(np.int64) * scale).astype(np.int32)
    assert int(img.max()) - int(img.min()) > 16383
    ns = np.ones(img.size, bool)
    ns[c.seeds] = False
    cost0, _ = O.oift_fmax_wide(img, adj, c.seeds, c.seed_labels, pol=0.0)
    ref_cost, _ = O.ref_ift_fmax(img, adj, c.seeds, c.seed_labels)
    assert int(cost0.max()) > 16383
    assert np.array_equal(ref_cost[ns] - 1, cost0[ns])
    cost, lab = O.oift_fmax_wide(img, adj, c.seeds, c.seed_labels, pol=pol)
    lab_ref = O.ref_oift_multi(img, adj, c.seeds, c.seed_labels, pol=pol)
    assert O.energy_wide(img, adj, lab_ref, pol=pol) == O.energy_wide(img, adj, lab, pol=pol)


def test_wide_range_oracle_equals_code_oracle_on_narrow_ranges(oracle_lib):
    """Within the 14-bit range the wide restatement and R2 on edge codes agree exactly."""
    for seed, shape, pol, adj, nl in [(31, (9, 12, 20), -0.3, 6, 2), (32, (7, 9, 12), 0.5, 26, 3),
                                      (33, (1, 30, 40), 0.2, 8, 2)]:
        c = synth.small_case(seed=seed, shape=shape, pol=pol, adjacency=adj, nlabels=nl,
                             noise=150, contrast=300)
        img = c.image.astype(np.int32)
        Z, Y, X = c.shape
        W, _ = O.build_weights(img, adj, "grad")
        cost, lab, _ = O.oift_fmax(W, (X, Y, Z), adj, c.seeds, c.seed_labels, pol=pol)
        cw, lw = O.oift_fmax_wide(img, adj, c.seeds, c.seed_labels, pol=pol)
        assert np.array_equal(cost, cw)
        assert np.array_equal(lab, lw)
