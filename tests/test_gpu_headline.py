"""GPU parity at the sizes the throughput figures are quoted on, through the C ABI.

* 256^3 int16 ellipsoid (6-adjacency, uint16 [0,4095] gradient weights, alpha = -0.3,
  50 FP32 sweeps), through oift_b200_run_device_i16 exactly as the throughput bench calls
  it:
    - cost map == R2 (lexicographic-Dijkstra restatement) bit for bit;
    - OIFT labels == R2; oriented cut energy == the energy of gft::ift::OIFT_Multi's labels;
    - the f_max derived along OIFT_Multi's own forest == the cost map;
    - label differences against OIFT_Multi counted; each one must be an equal-cost tie
      (both labels reach the voxel at its cost), and with no tie voxel in the volume the
      count must be zero;
    - membership == R3-FP32 bitwise and within 1e-5 of R3-FP64; relaxed labels == R3 ==
      gft::ift::ORelax_1_Multi; mask == (labels != 0).
* 256^2 disc (4-adjacency |dI|, alpha = +0.5, 10 sweeps), through the host entry.
* A reduced three-object cascade (26-adjacency RBF weights, 2 levels, 30 sweeps).
* A 4-volume draw of the batch mix through the batched driver, job by job against R2 / R3.

Reference lines: gft/src/gft_ift.cpp:911-989 (OIFT_Multi), 287-319 (energy), 8655-8911
(ORelax_1_Multi).
"""
import numpy as np
import pytest

import oracle as O
from roift_b200 import synth

pytestmark = pytest.mark.gpu

TOL64 = 1e-5   # FP32 membership against the FP64 restatement


def _oift_checks(W, shape_xyz, adj, c, cost, olab, img_for_ref):
    """Cost / label / energy / forest / tie assertions shared by the headline cases;
    returns the tie statistics against the reference forest."""
    X, Y, Z = shape_xyz
    cost_r2, lab_r2, levels = O.oift_fmax(W, shape_xyz, adj, c.seeds, c.seed_labels, pol=c.pol)
    assert np.array_equal(cost, cost_r2), f"cost diffs {(cost != cost_r2).sum()}"
    assert np.array_equal(olab, lab_r2), f"label diffs {(olab != lab_r2).sum()}"
    # the reference forest (R1 restates OIFT_Multi; it is checked against the live library
    # below when that library is present)
    lab_r1, _, _, fm = O.oift_prim(W, shape_xyz, adj, c.seeds, c.seed_labels, pol=c.pol)
    assert np.array_equal(fm, cost), "f_max along the reference forest differs"
    nl = int(max(lab_r2.max(), lab_r1.max())) + 1
    e_gpu, _ = O.energy(W, shape_xyz, adj, olab, nl, pol=c.pol)
    e_r1, _ = O.energy(W, shape_xyz, adj, lab_r1, nl, pol=c.pol)
    assert e_gpu == e_r1
    if O.ref_available():
        lab_ref = O.ref_oift_multi(img_for_ref, adj, c.seeds, c.seed_labels, pol=c.pol)
        assert np.array_equal(lab_ref, lab_r1)
        e_ref, _ = O.energy(W, shape_xyz, adj, lab_ref, nl, pol=c.pol)
        assert e_gpu == e_ref
    ts = O.tie_stats(W, shape_xyz, adj, cost, olab, lab_r1, c.seeds, pol=c.pol)
    assert ts["unexplained"] == 0, ts
    if ts["ties"] == 0:
        assert ts["diffs"] == 0, ts
    return ts, lab_r2, levels


@pytest.fixture(scope="module")
def config2(roift):
    import torch
    c = synth.ellipsoid3d(seed=2, size=256, sweeps=50)
    Z, Y, X = c.shape
    N = c.n
    dev = torch.device("cuda:0")
    img_t = torch.from_numpy(c.image.copy()).to(dev)
    s_t = torch.from_numpy(c.seeds).to(dev)
    l_t = torch.from_numpy(c.seed_labels).to(dev)
    cost_t = torch.empty(N, dtype=torch.int32, device=dev)
    olab_t = torch.empty(N, dtype=torch.int32, device=dev)
    lab_t = torch.empty(N, dtype=torch.int32, device=dev)
    mask_t = torch.empty(N, dtype=torch.uint8, device=dev)
    memb_t = torch.empty(2 * N, dtype=torch.float32, device=dev)
    p = roift.make_params(c.shape, adjacency=6, weight_mode="grad_q", wq=4095, pol=c.pol,
                          sweeps=c.sweeps)
    ctx = roift.Context(0)
    st = ctx.run_device(p, img_t.data_ptr(), s_t.data_ptr(), l_t.data_ptr(), len(c.seeds),
                        cost=cost_t.data_ptr(), oift_label=olab_t.data_ptr(),
                        label=lab_t.data_ptr(), mask=mask_t.data_ptr(),
                        membership=memb_t.data_ptr())
    torch.cuda.synchronize()
    out = dict(case=c, stats=st, cost=cost_t.cpu().numpy(), olab=olab_t.cpu().numpy(),
               lab=lab_t.cpu().numpy(), mask=mask_t.cpu().numpy(),
               memb=memb_t.cpu().numpy()[: st.nclasses * N].reshape(st.nclasses, N))
    ctx.close()
    return out


def test_config2_oift_cost_labels_energy_ties(config2):
    c = config2["case"]
    Z, Y, X = c.shape
    img = c.image.astype(np.int32)
    W, ncl = O.build_weights(img, 6, "grad_q", wq=4095)
    assert ncl == config2["stats"].clamped == 0
    shifted = img - min(0, int(img.min()))   # the CLI's shift (oiftrelax.cpp:263-268)
    ts, _, levels = _oift_checks(W, (X, Y, Z), 6, c, config2["cost"], config2["olab"], shifted)
    assert config2["stats"].levels >= levels
    # this volume has no equal-cost tie, so the labels equal OIFT_Multi's everywhere
    assert ts == {"ties": 0, "diffs": 0, "explained": 0, "unexplained": 0}


def test_config2_relaxation_membership_and_mask(config2):
    c = config2["case"]
    N = c.n
    img = c.image.astype(np.int32)
    shifted = img - min(0, int(img.min()))
    olab = config2["olab"]
    lab32, m32, nc = O.relax(shifted, 6, c.seeds, olab, c.sweeps, pol=c.pol)
    memb = config2["memb"]
    assert config2["stats"].nclasses == nc == 2
    assert np.array_equal(memb.view(np.uint32), m32.view(np.uint32)), \
        f"membership bit diffs {(memb != m32).sum()}"
    del m32
    _, m64, _ = O.relax(shifted, 6, c.seeds, olab, c.sweeps, pol=c.pol, fp64=True)
    assert np.abs(memb.astype(np.float64) - m64).max() <= TOL64
    del m64
    assert np.array_equal(config2["lab"], lab32)
    assert np.array_equal(config2["mask"], (lab32 != 0).astype(np.uint8))
    if O.ref_available():
        lab_ref = O.ref_orelax_multi(shifted, 6, c.seeds, olab, c.sweeps, pol=c.pol)
        assert np.array_equal(config2["lab"], lab_ref)
    assert N == 256 ** 3


def test_config1_disc256(roift):
    c = synth.disc2d(seed=1, size=256)
    img = c.image.astype(np.int32)
    Z, Y, X = c.shape
    p = roift.make_params(c.shape, adjacency=4, weight_mode="grad", pol=c.pol, sweeps=c.sweeps)
    ctx = roift.Context(0)
    lab, cost, memb, mask, st = ctx.run_host(p, img, c.label_map(), c.seeds, want_cost=True,
                                             want_membership=2, want_mask=True)
    ctx.close()
    W, _ = O.build_weights(img, 4, "grad")
    p0 = roift.make_params(c.shape, adjacency=4, weight_mode="grad", pol=c.pol, sweeps=0)
    ctx = roift.Context(0)
    olab, cost0, _, _, _ = ctx.run_host(p0, img, c.label_map(), c.seeds, want_cost=True)
    ctx.close()
    assert np.array_equal(cost0, cost)
    _oift_checks(W, (X, Y, Z), 4, c, cost, olab, img)
    lab32, m32, nc = O.relax(img, 4, c.seeds, olab, c.sweeps, pol=c.pol)
    assert np.array_equal(memb.view(np.uint32), m32.view(np.uint32))
    _, m64, _ = O.relax(img, 4, c.seeds, olab, c.sweeps, pol=c.pol, fp64=True)
    assert np.abs(memb.astype(np.float64) - m64).max() <= TOL64
    assert np.array_equal(lab, lab32)
    assert np.array_equal(mask, (lab32 != 0).astype(np.uint8))
    if O.ref_available():
        assert np.array_equal(lab, O.ref_orelax_multi(img, 4, c.seeds, olab, c.sweeps,
                                                      pol=c.pol))


def test_config3_reduced_cascade(roift):
    """The three-object cascade at 128 x 128 x 96 (26-adjacency RBF weights sigma 150
    quantised to [0, 4095], 2 levels, 30 sweeps), through the device entry point, against
    the restated cascade (Subsampling, first-seed coarse map, nearest ScaleLabel, NIL band,
    fine pass) with R2 as the OIFT."""
    import torch
    c = synth.three_ellipsoids(seed=3, shape=(96, 128, 128), sweeps=30)
    lab0 = np.full(c.n, -1, np.int32)
    lab0[c.seeds] = c.seed_labels
    dev = torch.device("cuda:0")
    d_img = torch.from_numpy(c.image.reshape(-1).copy()).to(dev)
    d_lab = torch.from_numpy(lab0).to(dev)
    d_sd = torch.from_numpy(c.seeds).to(dev)
    out = torch.empty(c.n, dtype=torch.int32, device=dev)
    p = roift.make_params(c.shape, adjacency=26, weight_mode="rbf_q", wq=4095, rbf_sigma=150.0,
                          pol=c.pol, sweeps=c.sweeps)
    ctx = roift.Context(0)
    ctx.run_pyramid_device(p, d_img.data_ptr(), d_lab.data_ptr(), d_sd.data_ptr(),
                           len(c.seeds), out.data_ptr(), 2, 50.0)
    got = out.cpu().numpy()
    ctx.close()
    b = c.image.astype(np.int64)
    b = (b - min(0, int(b.min()))).astype(np.int32)
    f = O.gaussian_blur(O.gaussian_blur(b).reshape(c.shape)).reshape(c.shape)
    exp = O.coarse_to_fine(f, 26, c.pol, c.sweeps, 50.0, c.seeds, lab0, mode="rbf_q")
    assert np.array_equal(got, exp), f"label diffs {(got != exp).sum()}"
    assert set(np.unique(got)) == {0, 1, 2, 3}


def test_config4_batch_mix_draw(roift):
    """Four volumes of the batch mix (uneven axes from {96..256}, several seed sets each)
    through the batched driver with the autotuner: per job, the mask equals the mask of
    R2 followed by the FP32 relaxation restatement (20 sweeps), and the costs equal R2."""
    import torch
    dev = torch.device("cuda:0")
    mix = synth.batch_mix(seed=4, nvol=4, sweeps=20)
    jobs_py, keep = [], []
    for case, sets in mix:
        img = torch.from_numpy(case.image.copy()).to(dev)
        keep.append(img)
        for sd, sl in sets[:3]:
            st = torch.from_numpy(sd).to(dev)
            lt = torch.from_numpy(sl).to(dev)
            mask = torch.zeros(case.n, dtype=torch.uint8, device=dev)
            cost = torch.zeros(case.n, dtype=torch.int32, device=dev)
            keep += [st, lt, mask, cost]
            jobs_py.append((case, sd, sl, img, st, lt, mask, cost))
    jobs = (roift.Job * len(jobs_py))()
    for i, (case, sd, sl, img, st, lt, mask, cost) in enumerate(jobs_py):
        Z, Y, X = case.shape
        jobs[i] = roift.Job(img.data_ptr(), X, Y, Z, st.data_ptr(), lt.data_ptr(), len(sd),
                            float(np.float32(case.pol * 100.0)), cost.data_ptr(), None,
                            mask.data_ptr(), 0)
    common = roift.make_params((1, 1, 1), adjacency=6, weight_mode="grad_q", wq=4095, sweeps=20)
    ctx = roift.Context(0)
    ctx.run_batch(common, jobs, teams=0)
    torch.cuda.synchronize()
    for i, (case, sd, sl, img, st, lt, mask, cost) in enumerate(jobs_py):
        assert jobs[i].status == 0
        Z, Y, X = case.shape
        im = case.image.astype(np.int32)
        W, _ = O.build_weights(im, 6, "grad_q", wq=4095)
        cost_r2, lab_r2, _ = O.oift_fmax(W, (X, Y, Z), 6, sd, sl, pol=case.pol)
        assert np.array_equal(cost.cpu().numpy(), cost_r2), f"job {i} cost"
        shifted = im - min(0, int(im.min()))
        lab32, _, _ = O.relax(shifted, 6, sd, lab_r2, 20, pol=case.pol)
        assert np.array_equal(mask.cpu().numpy(), (lab32 != 0).astype(np.uint8)), f"job {i} mask"
    ctx.close()
