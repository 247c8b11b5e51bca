"""GPU parity: the CUDA path (called through the C ABI) against the oracle and the
reference gft library on the same seeded inputs.

Bars (integer work bit-exact, FP32 relaxation bit-exact against the FP32 restatement
of ORelax_1_Multi and within 1e-5 of the FP64 oracle):
  * f_max cost map == R2 (lexicographic Dijkstra restatement) exactly;
  * OIFT labels == R2 labels exactly; oriented cut energy == energy of the reference
    OIFT_Multi labels exactly; label differences to OIFT_Multi only at equal-cost ties;
  * relaxed membership == R3-FP32 bitwise, |m - m64| <= 1e-5, labels == ORelax_1_Multi.
"""
import copy
import glob
import os

import numpy as np
import pytest

import oracle as O
from roift_b200 import synth

pytestmark = pytest.mark.gpu

CASES = [
    # shape (Z,Y,X), pol, adjacency, nlabels, weight mode
    ((16, 20, 24), -0.3, 6, 1, "grad"),
    ((16, 20, 24), 0.0, 6, 1, "grad"),
    ((16, 20, 24), 0.5, 6, 2, "grad"),
    ((9, 37, 70), -0.5, 6, 3, "grad"),
    ((1, 40, 48), 0.5, 4, 1, "grad"),
    ((1, 67, 45), -0.2, 4, 2, "grad"),
    ((20, 24, 64), -0.3, 6, 1, "grad_q"),
    ((12, 16, 40), 0.3, 6, 2, "rbf_q"),
    # full 3x3(x3) neighbourhoods: partial tiles along every axis, exact / quantised / RBF
    ((10, 14, 40), -0.3, 26, 1, "grad"),
    ((9, 21, 70), 0.4, 26, 2, "grad"),
    ((1, 45, 67), 0.5, 8, 1, "grad"),
    ((1, 40, 48), -0.2, 8, 2, "grad"),
    ((12, 16, 40), 0.3, 26, 2, "rbf_q"),
    ((8, 12, 64), -0.4, 26, 1, "grad_q"),
]


def _case(shape, pol, adj, nl, mode, seed=11):
    c = synth.small_case(seed=seed, shape=shape, pol=pol, adjacency=adj, nlabels=nl,
                         noise=120, contrast=400, weight_mode=mode)
    img = c.image.astype(np.int32)
    img -= min(0, int(img.min()))
    return c, img


def _run(roift, c, img, mode, sweeps, wq=4095, per_class=None):
    ctx = roift._ctx()
    shp = c.shape
    p = roift.make_params(shp, adjacency=c.adjacency, weight_mode=mode, wq=wq,
                          rbf_sigma=150.0, pol=c.pol if per_class is None else None,
                          per_class=per_class, sweeps=sweeps)
    lab = c.label_map()
    return ctx.run_host(p, img, lab, c.seeds, want_cost=True,
                        want_membership=8 if sweeps else 0, want_mask=bool(sweeps))


@pytest.mark.parametrize("shape,pol,adj,nl,mode", CASES)
def test_oift_cost_and_labels_match_oracle(roift, oracle_lib, shape, pol, adj, nl, mode):
    c, img = _case(shape, pol, adj, nl, mode)
    Z, Y, X = c.shape
    lab, cost, _, _, st = _run(roift, c, img, mode, sweeps=0, wq=4095 if mode != "grad" else 4095)
    W, ncl = O.build_weights(img, adj, mode, wq=4095, rbf_sigma=150.0)
    cost_r2, lab_r2, levels = O.oift_fmax(W, (X, Y, Z), adj, c.seeds, c.seed_labels, pol=c.pol)
    assert np.array_equal(cost, cost_r2), f"cost diffs {(cost != cost_r2).sum()}"
    assert np.array_equal(lab, lab_r2), f"label diffs {(lab != lab_r2).sum()}"
    # the GPU may also visit levels whose only entries went stale (a tile's pending key
    # was lowered afterwards); it never skips a populated one
    assert st.levels >= levels
    if mode == "grad" and O.ref_available():
        lab_ref = O.ref_oift_multi(img, adj, c.seeds, c.seed_labels, pol=c.pol)
        e_gpu, elb_gpu = O.energy(W, (X, Y, Z), adj, lab, nl + 1, pol=c.pol)
        e_ref, elb_ref = O.energy(W, (X, Y, Z), adj, lab_ref, nl + 1, pol=c.pol)
        assert e_gpu == e_ref
        # label differences to the reference Prim forest only where costs tie
        _, _, _, fm = O.oift_prim(W, (X, Y, Z), adj, c.seeds, c.seed_labels, pol=c.pol)
        assert np.array_equal(fm, cost), "f_max along the reference forest differs"
        # every differing voxel is an equal-cost tie: a neighbour labelled as in our map and
        # one labelled as in the reference's both reach it at exactly its cost; a volume
        # without tie voxels has no difference at all
        ts = O.tie_stats(W, (X, Y, Z), adj, cost, lab, lab_ref, c.seeds, pol=c.pol)
        assert ts["diffs"] == int((lab != lab_ref).sum())
        assert ts["unexplained"] == 0, ts
        if ts["ties"] == 0:
            assert ts["diffs"] == 0, ts


@pytest.mark.parametrize("shape,pol,adj,nl,mode", [CASES[0], CASES[2], CASES[3], CASES[4]])
def test_relax_bitexact(roift, oracle_lib, shape, pol, adj, nl, mode):
    c, img = _case(shape, pol, adj, nl, mode)
    Z, Y, X = c.shape
    K = 7
    lab, cost, memb, mask, st = _run(roift, c, img, mode, sweeps=K)
    W, _ = O.build_weights(img, adj, mode)
    _, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), adj, c.seeds, c.seed_labels, pol=c.pol)
    lab32, m32, nc = O.relax(img, adj, c.seeds, lab_r2, K, pol=c.pol)
    lab64, m64, _ = O.relax(img, adj, c.seeds, lab_r2, K, pol=c.pol, fp64=True)
    assert st.nclasses == nc
    assert np.array_equal(memb.view(np.uint32), m32.view(np.uint32)), \
        f"membership bit diffs {(memb != m32).sum()}"
    assert np.abs(memb.astype(np.float64) - m64).max() <= 1e-5
    assert np.array_equal(lab, lab32)
    assert np.array_equal(mask, (lab32 != 0).astype(np.uint8))
    if O.ref_available():
        lab_ref = O.ref_orelax_multi(img, adj, c.seeds, lab_r2, K, pol=c.pol)
        assert np.array_equal(lab, lab_ref)


def test_relax_perclass_bitexact(roift, oracle_lib):
    c, img = _case((10, 18, 33), 0.0, 6, 3, "grad")
    per_class = np.array([-30.0, 20.0, 45.0, -10.0], np.float32)
    K = 5
    lab, cost, memb, mask, st = _run(roift, c, img, "grad", sweeps=K, per_class=per_class)
    Z, Y, X = c.shape
    W, _ = O.build_weights(img, 6, "grad")
    cost_r2, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), 6, c.seeds, c.seed_labels,
                                     per_class=per_class)
    assert np.array_equal(cost, cost_r2)
    lab32, m32, nc = O.relax(img, 6, c.seeds, lab_r2, K, per_class=per_class)
    assert np.array_equal(memb.view(np.uint32), m32.view(np.uint32))
    assert np.array_equal(lab, lab32)
    if O.ref_available():
        lab_ref = O.ref_orelax_multi(img, 6, c.seeds, lab_r2, K, per_class=per_class)
        assert np.array_equal(lab, lab_ref)


def test_dropin_oift_fmax_gpu_run(roift, oracle_lib):
    c, img = _case((12, 30, 40), -0.4, 6, 2, "grad")
    Z, Y, X = c.shape
    per_class = np.array([40.0, -40.0, -40.0], np.float32)  # bg = -pol as the GPU CLI does
    lab = c.label_map()
    levels = roift.oift_fmax_gpu_run(img, lab, X, Y, Z, per_class, c.seeds)
    W, _ = O.build_weights(img, 6, "grad")
    _, lab_r2, lev = O.oift_fmax(W, (X, Y, Z), 6, c.seeds, c.seed_labels, per_class=per_class)
    assert np.array_equal(lab, lab_r2)
    assert levels >= lev
    if O.ref_available():
        lab_ref = O.ref_oift_multi(img, 6, c.seeds, c.seed_labels, per_class=per_class)
        e1, _ = O.energy(W, (X, Y, Z), 6, lab, 3, per_class=per_class)
        e2, _ = O.energy(W, (X, Y, Z), 6, lab_ref, 3, per_class=per_class)
        assert e1 == e2


def test_device_pipeline_ellipsoid(roift, oracle_lib):
    import torch
    c = synth.ellipsoid3d(seed=3, size=64, sweeps=6)
    Z, Y, X = c.shape
    dev = torch.device("cuda:0")
    img_t = torch.from_numpy(c.image.copy()).to(dev)
    s_t = torch.from_numpy(c.seeds).to(dev)
    l_t = torch.from_numpy(c.seed_labels).to(dev)
    N = c.n
    cost_t = torch.empty(N, dtype=torch.int32, device=dev)
    olab_t = torch.empty(N, dtype=torch.int32, device=dev)
    lab_t = torch.empty(N, dtype=torch.int32, device=dev)
    mask_t = torch.empty(N, dtype=torch.uint8, device=dev)
    memb_t = torch.empty(2 * N, dtype=torch.float32, device=dev)
    p = roift.make_params(c.shape, adjacency=6, weight_mode="grad_q", wq=4095, pol=c.pol,
                          sweeps=c.sweeps)
    ctx = roift._ctx()
    st = ctx.run_device(p, img_t.data_ptr(), s_t.data_ptr(), l_t.data_ptr(), len(c.seeds),
                        cost=cost_t.data_ptr(), oift_label=olab_t.data_ptr(),
                        label=lab_t.data_ptr(), mask=mask_t.data_ptr(),
                        membership=memb_t.data_ptr())
    torch.cuda.synchronize()
    img = c.image.astype(np.int32)
    W, ncl = O.build_weights(img, 6, "grad_q", wq=4095)
    assert ncl == st.clamped == 0
    cost_r2, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), 6, c.seeds, c.seed_labels, pol=c.pol)
    assert np.array_equal(cost_t.cpu().numpy(), cost_r2)
    assert np.array_equal(olab_t.cpu().numpy(), lab_r2)
    shifted = img - min(0, int(img.min()))
    lab32, m32, nc = O.relax(shifted, 6, c.seeds, lab_r2, c.sweeps, pol=c.pol)
    assert np.array_equal(memb_t.cpu().numpy().reshape(nc, N).view(np.uint32), m32.view(np.uint32))
    assert np.array_equal(lab_t.cpu().numpy(), lab32)


def test_div100_exhaustive(roift):
    """The sweeps' x/100 equals the IEEE FP32 quotient for every finite input."""
    bad, first = roift.selftest_div100()
    assert bad == 0, f"{bad} mismatches, first bit pattern {first:#010x}"


@pytest.mark.parametrize("size", [96])
def test_relax_tile_skipping_exact(roift, oracle_lib, size):
    """Clean ellipsoid boundary: early sweeps skip most tiles, membership stays bit-exact."""
    c = synth.ellipsoid3d(seed=4, size=size, sweeps=12)
    img = c.image.astype(np.int32)
    img -= min(0, int(img.min()))
    Z, Y, X = c.shape
    K = c.sweeps
    lab, cost, memb, mask, st = _run(roift, c, img, "grad_q", sweeps=K)
    W, _ = O.build_weights(img, 6, "grad_q")
    _, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), 6, c.seeds, c.seed_labels, pol=c.pol)
    lab32, m32, nc = O.relax(img, 6, c.seeds, lab_r2, K, pol=c.pol)
    assert np.array_equal(memb.view(np.uint32), m32.view(np.uint32))
    assert np.array_equal(lab, lab32)
    tiles = ((X + 31) // 32) * ((Y + 7) // 8) * ((Z + 3) // 4)
    assert st.relax_active_voxel_sweeps < 0.8 * K * tiles * 1024


def _batch_jobs(rb, cases, torch, dev, outs=None):
    """Job array over `cases`; outs[i] names the outputs of job i ("label", "mask", "cost").
    Cases that share an image object share one device image (one edge-code build)."""
    bufs, jobs = [], (rb.Job * len(cases))()
    imgs = {}
    for i, c in enumerate(cases):
        want = outs[i] if outs else ("label", "mask")
        if id(c.image) not in imgs:
            imgs[id(c.image)] = torch.from_numpy(c.image.astype(np.int16)).to(dev)
        img = imgs[id(c.image)]
        sd = torch.from_numpy(c.seeds).to(dev)
        sl = torch.from_numpy(c.seed_labels).to(dev)
        lab = torch.full((c.n,), -5, dtype=torch.int32, device=dev)
        mask = torch.zeros(c.n, dtype=torch.uint8, device=dev)
        cost = torch.full((c.n,), -5, dtype=torch.int32, device=dev)
        Z, Y, X = c.shape
        jobs[i] = rb.Job(img.data_ptr(), X, Y, Z, sd.data_ptr(), sl.data_ptr(), len(c.seeds),
                         float(np.float32(c.pol * 100.0)),
                         cost.data_ptr() if "cost" in want else None,
                         lab.data_ptr() if "label" in want else None,
                         mask.data_ptr() if "mask" in want else None, 0)
        bufs.append((img, sd, sl, lab, mask, cost))
    return jobs, bufs


def _batch_cases():
    """Uneven 3D volumes, a second seed set on one of them (shared image), a 2D slice."""
    cases = []
    for i, size in enumerate([40, 56, 48, 64, 40, 52]):
        cases.append(synth.ellipsoid3d(seed=20 + i, size=size, sweeps=6,
                                       pol=[-0.3, 0.2, 0.4][i % 3]))
    base = cases[1]
    rng = np.random.default_rng(3)
    keep = rng.random(len(base.seeds)) < 0.7
    alt = copy.copy(base)
    alt.seeds, alt.seed_labels = base.seeds[keep], base.seed_labels[keep]
    alt.pol = -0.45
    cases.append(alt)
    d = synth.disc2d(seed=9, size=96)
    d.image = d.image.astype(np.int16)
    cases.append(d)
    return cases


@pytest.mark.parametrize("teams,tile", [(1, 8), (3, 8), (16, 8), (0, 8), (3, 4), (16, 4)])
def test_batch_matches_single_runs(roift, teams, tile):
    """The team-batched OIFT (and the autotuner, teams=0) with either 3D warp tile (32x8x4,
    32x4x8) gives, per job, the labels, mask and costs of one-at-a-time runs, for every mix
    of requested outputs."""
    import torch
    dev = torch.device("cuda:0")
    cases = _batch_cases()
    outs = [("label", "mask"), ("label",), ("mask",), ("cost", "label"), ("cost",),
            ("label", "mask", "cost"), ("label", "mask"), ("label", "cost")]
    p = roift.make_params((1, 1, 1), adjacency=6, weight_mode="grad_q", wq=4095, sweeps=6)
    jobs, bufs = _batch_jobs(roift, cases, torch, dev, outs)
    ctx = roift.Context(0)
    ctx.set_batch_tile(tile)
    st = ctx.run_batch(p, jobs, teams=teams)
    torch.cuda.synchronize()
    assert st.jobs == len(cases) and st.teams >= 1
    if teams:
        assert st.tile_ty == tile
    for c, (img, sd, sl, lab, mask, cost), job, want in zip(cases, bufs, jobs, outs):
        assert job.status == 0
        single = roift.make_params(c.shape, adjacency=6, weight_mode="grad_q", wq=4095,
                                   pol=c.pol, sweeps=6)
        lab1 = torch.empty(c.n, dtype=torch.int32, device=dev)
        cost1 = torch.empty(c.n, dtype=torch.int32, device=dev)
        roift._ctx().run_device(single, img.data_ptr(), sd.data_ptr(), sl.data_ptr(),
                                len(c.seeds), label=lab1.data_ptr(), cost=cost1.data_ptr())
        torch.cuda.synchronize()
        if "label" in want:
            assert torch.equal(lab, lab1)
        if "mask" in want:
            assert torch.equal(mask, (lab1 != 0).to(torch.uint8))
        if "cost" in want:
            assert torch.equal(cost, cost1)
    ctx.close()


@pytest.mark.parametrize("teams", [3, 0])
def test_batch_graph_replays_match_batch(roift, teams):
    """A batch recorded into a CUDA graph gives, on two replays in a row, the labels, masks
    and costs of the direct batched call."""
    import torch
    dev = torch.device("cuda:0")
    cases = _batch_cases()
    outs = [("label", "mask"), ("label",), ("mask",), ("cost", "label"), ("cost",),
            ("label", "mask", "cost"), ("label", "mask"), ("label", "cost")]
    p = roift.make_params((1, 1, 1), adjacency=6, weight_mode="grad_q", wq=4095, sweeps=6)
    ref_jobs, ref_bufs = _batch_jobs(roift, cases, torch, dev, outs)
    ctx = roift.Context(0)
    ctx.run_batch(p, ref_jobs, teams=3)
    jobs, bufs = _batch_jobs(roift, cases, torch, dev, outs)
    g = ctx.batch_graph(p, jobs, teams=teams)
    for _ in range(2):
        for (_, _, _, lab, mask, cost) in bufs:
            lab.fill_(-7)
            mask.fill_(9)
            cost.fill_(-7)
        ms = g.launch()
        torch.cuda.synchronize()
        assert ms > 0.0
        for (_, _, _, lab, mask, cost), (_, _, _, rl, rm, rc), job, want in zip(bufs, ref_bufs,
                                                                                  jobs, outs):
            assert job.status == 0
            if "label" in want:
                assert torch.equal(lab, rl)
            if "mask" in want:
                assert torch.equal(mask, rm)
            if "cost" in want:
                assert torch.equal(cost, rc)
    g.close()
    ctx.close()


def test_batch_bad_seed_is_reported_per_job(roift):
    """A job whose seed lies outside its volume ends with OIFT_E_SEED_RANGE; the other
    jobs of the same launch still complete with the labels of single runs."""
    import torch
    dev = torch.device("cuda:0")
    cases = _batch_cases()[:4]
    bad = copy.copy(cases[2])
    bad.seeds = bad.seeds.copy()
    bad.seeds[len(bad.seeds) // 2] = bad.n + 5
    cases[2] = bad
    p = roift.make_params((1, 1, 1), adjacency=6, weight_mode="grad_q", wq=4095, sweeps=6)
    jobs, bufs = _batch_jobs(roift, cases, torch, dev)
    ctx = roift.Context(0)
    with pytest.raises(roift.OiftError):
        ctx.run_batch(p, jobs, teams=2)
    torch.cuda.synchronize()
    assert [j.status for j in jobs] == [0, 0, roift.E_SEED_RANGE, 0]
    for i in (0, 1, 3):
        c, (img, sd, sl, lab, mask, cost) = cases[i], bufs[i]
        single = roift.make_params(c.shape, adjacency=6, weight_mode="grad_q", wq=4095,
                                   pol=c.pol, sweeps=6)
        lab1 = torch.empty(c.n, dtype=torch.int32, device=dev)
        roift._ctx().run_device(single, img.data_ptr(), sd.data_ptr(), sl.data_ptr(),
                                len(c.seeds), label=lab1.data_ptr())
        torch.cuda.synchronize()
        assert torch.equal(lab, lab1)
    ctx.close()


# ------------------------------------------------------------ steps of the CLI ----
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_gaussian_blur_matches_reference(roift, path):
    """GPU blur == Scene32::GaussianBlur outputs (golden), and two passes == two oracle
    passes, on the image and on it shifted below zero."""
    import torch
    d = np.load(path)
    img = d["image"].astype(np.int32)
    dev = torch.device("cuda:0")
    ctx = roift._ctx()
    src = torch.from_numpy(img.reshape(-1).copy()).to(dev)
    out = torch.empty_like(src)
    ctx.gaussian_blur(src.data_ptr(), out.data_ptr(), img.shape, 1)
    assert np.array_equal(out.cpu().numpy(), d["ref_blur"])
    neg = (img - 700).astype(np.int32)
    src = torch.from_numpy(neg.reshape(-1).copy()).to(dev)
    ctx.gaussian_blur(src.data_ptr(), src.data_ptr(), img.shape, 2)   # in place
    exp = O.gaussian_blur(O.gaussian_blur(neg).reshape(img.shape))
    assert np.array_equal(src.cpu().numpy(), exp)


def test_gaussian_blur_large_matches_oracle(roift):
    import torch
    rng = np.random.default_rng(8)
    img = rng.integers(-30000, 30000, size=(37, 61, 130)).astype(np.int32)
    src = torch.from_numpy(img.reshape(-1).copy()).to("cuda:0")
    out = torch.empty_like(src)
    roift._ctx().gaussian_blur(src.data_ptr(), out.data_ptr(), img.shape, 1)
    assert np.array_equal(out.cpu().numpy(), O.gaussian_blur(img))


@pytest.mark.parametrize("trial", range(12))
def test_conditional_dilation_matches_oracle(roift, trial):
    """Border detection, percentile rank and address-order ties (few distinct values)."""
    import torch
    rng = np.random.default_rng(900 + trial)
    shape = [(1, 40, 52), (9, 23, 31), (24, 40, 70)][trial % 3]
    n = int(np.prod(shape))
    img = rng.integers(0, 4 if trial % 2 else 50000, size=shape).astype(np.int32) - 100
    lab = rng.choice([-1, 0, 0, 0, 1, 1], size=n).astype(np.int32)
    r = [1.0, 1.0, 1.5, 2.0][trial % 4]
    pc = [50.0, 0.0, 100.0, 37.5, 99.9, 150.0][trial % 6]
    exp, added = O.conditional_dilation(img, lab, r, pc)
    d_img = torch.from_numpy(img.reshape(-1).copy()).to("cuda:0")
    d_lab = torch.from_numpy(lab.copy()).to("cuda:0")
    got = roift._ctx().conditional_dilation(d_img.data_ptr(), d_lab.data_ptr(), shape, r, pc)
    assert got == added
    assert np.array_equal(d_lab.cpu().numpy(), exp)


CLI_GOLDEN = [p for p in GOLDEN if "ref_chain_label" in np.load(p).files]


@pytest.mark.parametrize("path", CLI_GOLDEN, ids=[os.path.basename(p)[:-4] for p in CLI_GOLDEN])
def test_cli_chain_matches_oracle_and_reference(roift, path):
    """run_cli_host (shift, blur x2, OIFT, relaxation, dilation) == the oracle chain on the
    lexicographic OIFT labels, bit for bit; == the reference chain wherever the oracle's
    OIFT_Multi restatement and the lexicographic labels agree (no equal-cost ties)."""
    d = np.load(path)
    img = d["chain_image"]
    seeds, sl = d["seeds"], d["seed_labels"]
    pol, K = float(d["pol"]), int(d["sweeps"])
    lab = np.full(img.size, -1, np.int32)
    lab[seeds] = sl
    adj = 4 if img.shape[0] == 1 else 6
    p = roift.make_params(img.shape, adjacency=adj, weight_mode="grad", pol=pol, sweeps=K)
    got, _ = roift._ctx().run_cli_host(p, img, lab.copy(), seeds, blur_passes=2, percentile=50.0)
    exp2, _ = O.oiftrelax_chain(img, pol, K, 50.0, seeds, sl, oift="r2")
    assert np.array_equal(got, exp2)
    exp1, _ = O.oiftrelax_chain(img, pol, K, 50.0, seeds, sl, oift="r1")
    if np.array_equal(exp1, exp2):
        assert np.array_equal(got, d["ref_chain_label"])


@pytest.mark.parametrize("adj", [26, 6])
def test_device_path_int16_full_neighbourhood(roift, oracle_lib, adj):
    """int16 device images through the full-neighbourhood kernel (and 6-adj beside it):
    three objects, RBF weights, cost and labels == R2."""
    import torch
    c = synth.three_ellipsoids(seed=31, shape=(40, 48, 56))
    dev = torch.device("cuda:0")
    img16 = c.image.astype(np.int16)
    Z, Y, X = c.shape
    p = roift.make_params(c.shape, adjacency=adj, weight_mode="rbf_q", wq=4095, rbf_sigma=150.0,
                          pol=c.pol, sweeps=0)
    d_img = torch.from_numpy(img16.reshape(-1).copy()).to(dev)
    sd = torch.from_numpy(c.seeds).to(dev)
    sl = torch.from_numpy(c.seed_labels).to(dev)
    cost = torch.empty(c.n, dtype=torch.int32, device=dev)
    lab = torch.empty(c.n, dtype=torch.int32, device=dev)
    roift._ctx().run_device(p, d_img.data_ptr(), sd.data_ptr(), sl.data_ptr(), len(c.seeds),
                            cost=cost.data_ptr(), oift_label=lab.data_ptr())
    W, _ = O.build_weights(img16.astype(np.int32), adj, "rbf_q", wq=4095, rbf_sigma=150.0)
    cost_r2, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), adj, c.seeds, c.seed_labels, pol=c.pol)
    assert np.array_equal(cost.cpu().numpy(), cost_r2)
    assert np.array_equal(lab.cpu().numpy(), lab_r2)


# ------------------------------------------------------ coarse-to-fine cascade ----
C2F_GOLDEN = [p for p in GOLDEN if "ref_c2f_label" in np.load(p).files]


def _c2f_expected(img, adj, pol, K, seeds, lab0, mode="grad", oift="r2"):
    b = np.asarray(img, np.int64)
    b = (b - min(0, int(b.min()))).astype(np.int32)
    f = O.gaussian_blur(O.gaussian_blur(b).reshape(img.shape)).reshape(img.shape)
    return O.coarse_to_fine(f, adj, pol, K, 50.0, seeds, lab0, mode=mode, oift=oift)


@pytest.mark.parametrize("path", C2F_GOLDEN, ids=[os.path.basename(p)[:-4] for p in C2F_GOLDEN])
def test_pyramid_matches_oracle_and_reference(roift, path):
    """run_pyramid_host == the restated cascade on the lexicographic OIFT bit for bit, and
    == the reference experiment where OIFT_Multi's order gives the same labels."""
    d = np.load(path)
    img = d["image"].astype(np.int32)
    seeds, sl = d["seeds"], d["seed_labels"]
    adj, pol, K = int(d["adjacency"]), float(d["pol"]), int(d["sweeps"])
    lab0 = np.full(img.size, -1, np.int32)
    lab0[seeds] = sl
    p = roift.make_params(img.shape, adjacency=adj, weight_mode="grad", pol=pol, sweeps=K)
    got, st = roift._ctx().run_pyramid_host(p, img, lab0.copy(), seeds, 2, 50.0)
    assert np.array_equal(got, _c2f_expected(img, adj, pol, K, seeds, lab0))
    if np.array_equal(_c2f_expected(img, adj, pol, K, seeds, lab0, oift="r1"),
                      _c2f_expected(img, adj, pol, K, seeds, lab0)):
        assert np.array_equal(got, d["ref_c2f_label"])


@pytest.mark.parametrize("adj,mode", [(26, "rbf_q"), (6, "grad_q")])
def test_pyramid_device_int16(roift, adj, mode):
    """Device flavour on an int16 volume with negative intensities, odd extents, three
    objects and a boundary shell (the configuration of the large three-object workload
    at a small size)."""
    import torch
    c = synth.three_ellipsoids(seed=7, shape=(37, 45, 51))
    img16 = (c.image.astype(np.int32) - 300).astype(np.int16)
    lab0 = np.full(c.n, -1, np.int32)
    lab0[c.seeds] = c.seed_labels
    dev = torch.device("cuda:0")
    d_img = torch.from_numpy(img16.reshape(-1).copy()).to(dev)
    d_lab = torch.from_numpy(lab0).to(dev)
    d_sd = torch.from_numpy(c.seeds).to(dev)
    out = torch.empty(c.n, dtype=torch.int32, device=dev)
    p = roift.make_params(c.shape, adjacency=adj, weight_mode=mode, wq=4095, rbf_sigma=150.0,
                          pol=0.2, sweeps=4)
    roift._ctx().run_pyramid_device(p, d_img.data_ptr(), d_lab.data_ptr(), d_sd.data_ptr(),
                                    len(c.seeds), out.data_ptr(), 2, 50.0)
    exp = _c2f_expected(img16.astype(np.int32), adj, 0.2, 4, c.seeds, lab0, mode=mode)
    assert np.array_equal(out.cpu().numpy(), exp)


# ------------------------------------------------------ gradient-blend weights ----
BLEND_CASES = [((14, 18, 40), -0.3, 6, 1, 0.6), ((9, 21, 70), 0.4, 6, 2, 0.3),
               ((1, 45, 67), 0.5, 4, 1, 0.8), ((12, 16, 40), 0.0, 6, 1, 1.0),
               ((10, 20, 36), 0.2, 6, 1, 0.0)]


@pytest.mark.parametrize("shape,pol,adj,nl,alpha", BLEND_CASES)
def test_blend_oift_and_relax_match_oracle(roift, oracle_lib, shape, pol, adj, nl, alpha):
    """BLEND_Q: the Sobel map normalised to the image maximum, OIFT with the float blend
    weights of OIFT_Multi_GradWeight (cost and labels == R2 with those weights), and the
    blend relaxation of ORelax_1_Multi_GradWeight (membership bit-identical)."""
    c, img = _case(shape, pol, adj, nl, "grad")
    X, Y, Z = shape[2], shape[1], shape[0]
    g = O.sobel_normalized(img.reshape(shape))
    p = roift.make_params(shape, adjacency=adj, weight_mode="blend_q", blend_a=alpha, pol=pol,
                          sweeps=0)
    lab, cost, _, _, _ = roift._ctx().run_host(p, img, c.label_map(), c.seeds, want_cost=True)
    cost_r2, lab_r2, _ = O.oift_fmax_blend(img.reshape(shape), g, alpha, adj, c.seeds,
                                           c.seed_labels, pol=pol)
    assert np.array_equal(cost, cost_r2)
    assert np.array_equal(lab, lab_r2)
    K = 6
    p = roift.make_params(shape, adjacency=adj, weight_mode="blend_q", blend_a=alpha, pol=pol,
                          sweeps=K)
    labk, _, memb, _, _ = roift._ctx().run_host(p, img, c.label_map(), c.seeds,
                                                want_membership=8)
    exp, m32 = O.relax_blend(img.reshape(shape), g, alpha, adj, c.seeds, lab_r2, K, pol)
    assert np.array_equal(labk, exp)
    assert np.array_equal(memb.view(np.uint32), m32.view(np.uint32))


BLEND_GOLDEN = [p for p in GOLDEN if "ref_blend_relax_label" in np.load(p).files]


@pytest.mark.parametrize("path", BLEND_GOLDEN, ids=[os.path.basename(p)[:-4] for p in BLEND_GOLDEN])
def test_blend_matches_reference_experiment(roift, oracle_lib, path):
    """On the reference experiment's inputs (twice-blurred image): the GPU blend OIFT +
    relaxation equals the reference's OIFT_Multi_GradWeight + ORelax_1_Multi_GradWeight
    wherever the lexicographic and the Prim-order OIFT agree."""
    d = np.load(path)
    f = d["blend_image"]
    seeds, sl = d["seeds"], d["seed_labels"]
    pol, K, adj = float(d["pol"]), int(d["sweeps"]), int(d["adjacency"])
    lab0 = np.full(f.size, -1, np.int32)
    lab0[seeds] = sl
    p = roift.make_params(f.shape, adjacency=adj, weight_mode="blend_q", blend_a=0.6, pol=pol,
                          sweeps=K)
    got, _, _, _, _ = roift._ctx().run_host(p, f.reshape(-1), lab0.copy(), seeds)
    g = O.sobel_normalized(f)
    _, lab_r2, _ = O.oift_fmax_blend(f, g, 0.6, adj, seeds, sl, pol=pol)
    exp, _ = O.relax_blend(f, g, 0.6, adj, seeds, lab_r2, K, pol)
    assert np.array_equal(got, exp)
    if np.array_equal(lab_r2, d["ref_blend_oift_label"]):
        assert np.array_equal(got, d["ref_blend_relax_label"])


# ------------------------------------------------------------ 2D image graph ----
IG_CASES = [((1, 40, 48), 0.5, 4, 7, 1), ((1, 45, 67), -0.3, 8, 5, 1), ((1, 64, 33), 0.0, 4, 0, 1),
            ((1, 31, 90), 1.0, 8, 3, 2), ((1, 50, 50), -1.0, 4, 4, 1), ((1, 37, 70), 0.2, 8, 9, 2)]


@pytest.mark.parametrize("shape,pol,adj,K,nl", IG_CASES)
def test_imagegraph_oift_and_relax_match_oracle(roift, oracle_lib, shape, pol, adj, K, nl):
    """OIFT_W_IMAGEGRAPH: cost and labels == R2 with the oriented image-graph weights
    (|dI| + 1, MAX(ROUND(w (1 +/- alpha)), 1)), the cut energy equals R1's (the reference
    order), and after K sweeps of ORelax_1(sImageGraph) the binary labels, mask and the
    single membership channel are bit-identical to the FP32 restatement."""
    c, img = _case(shape, pol, adj, nl, "grad")
    img2 = img.reshape(shape[1:])
    ctx = roift._ctx()
    p = roift.make_params(shape, adjacency=adj, weight_mode="imagegraph", pol=pol, sweeps=0)
    lab, cost, _, _, st = ctx.run_host(p, img, c.label_map(), c.seeds, want_cost=True)
    cost_r2, lab_r2, levels = O.oift_fmax_imagegraph(img2, adj, c.seeds, c.seed_labels, pol)
    assert np.array_equal(cost, cost_r2)
    assert np.array_equal(lab, lab_r2)
    assert st.levels >= levels
    order = np.argsort(c.seeds, kind="stable")
    r1, _, _, _ = O.oift_prim_imagegraph(img2, adj, c.seeds[order], c.seed_labels[order], pol)
    for lb in range(1, nl + 1):
        assert O.energy_imagegraph(img2, adj, lab, pol, lb) == O.energy_imagegraph(img2, adj, r1, pol, lb)
    p = roift.make_params(shape, adjacency=adj, weight_mode="imagegraph", pol=pol, sweeps=K)
    labk, _, memb, mask, st = ctx.run_host(p, img, c.label_map(), c.seeds, want_membership=1,
                                           want_mask=True)
    exp, m = O.relax_imagegraph(img2, adj, c.seeds, lab_r2, K, pol)
    assert st.nclasses == 1
    assert np.array_equal(labk, exp)
    assert np.array_equal(mask.astype(np.int32), exp)
    assert np.array_equal(memb.reshape(-1).view(np.uint32), m.view(np.uint32))


IG_GOLDEN = [p for p in GOLDEN if "ref_ig_oift_label" in np.load(p).files]


@pytest.mark.parametrize("path", IG_GOLDEN, ids=[os.path.basename(p)[:-4] for p in IG_GOLDEN])
def test_imagegraph_matches_reference_pipeline(roift, oracle_lib, path):
    """On the fixtures of the reference's own 2D pipeline: the GPU labels have the
    reference's cut energy; where R2 and the reference's Prim labels agree, the GPU's
    relaxed labels equal the reference's ORelax_1(sImageGraph) output."""
    d = np.load(path)
    shape = d["image"].shape
    img2 = d["image"].reshape(shape[1:])
    seeds, sl = d["seeds"], d["seed_labels"]
    pol, K, adj = float(d["pol"]), int(d["sweeps"]), int(d["adjacency"])
    lab0 = np.full(img2.size, -1, np.int32)
    lab0[seeds] = sl
    ctx = roift._ctx()
    p = roift.make_params(shape, adjacency=adj, weight_mode="imagegraph", pol=pol, sweeps=0)
    lab, _, _, _, _ = ctx.run_host(p, img2.reshape(-1), lab0.copy(), seeds)
    assert O.energy_imagegraph(img2, adj, lab, pol) == int(d["ref_ig_energy"])
    p = roift.make_params(shape, adjacency=adj, weight_mode="imagegraph", pol=pol, sweeps=K)
    labk, _, _, _, _ = ctx.run_host(p, img2.reshape(-1), lab0.copy(), seeds)
    exp, _ = O.relax_imagegraph(img2, adj, seeds, lab, K, pol)
    assert np.array_equal(labk, exp)
    if np.array_equal(lab, d["ref_ig_oift_label"]):
        assert np.array_equal(labk, d["ref_ig_relax_label"])


def test_imagegraph_rejections(roift):
    """The image graph is 2D with one global polarity; the batched driver and the cascade
    do not take it."""
    ctx = roift._ctx()
    img = np.zeros(4 * 5 * 6, np.int32)
    lab = np.full(img.size, -1, np.int32)
    lab[0] = 0
    seeds = np.array([0], np.int32)
    for shape, adj in (((4, 5, 6), 6), ((1, 20, 6), 6)):
        p = roift.make_params(shape, adjacency=adj, weight_mode="imagegraph", pol=0.3)
        with pytest.raises(roift.OiftError) as e:
            ctx.run_host(p, img[: int(np.prod(shape))], lab[: int(np.prod(shape))].copy(), seeds)
        assert e.value.status == roift.E_UNSUPPORTED
