"""Bounded device waits of the persistent OIFT kernels, made to run out on purpose.

Every wait of the level loop (grid / team barrier, end of a level) gives up after a poll
limit, and a run that exceeds a level cap is declared runaway; either way every warp
leaves, the launch ends, and the call reports OIFT_E_NOT_CONVERGED with the context still
usable.  The limits are lowered through oift_b200_set_limits; nothing here faults, traps
or hangs the GPU.  The reference's own guard is its iteration cap
(gpu/oift_fmax_gpu.cu:197,240-242).
"""
import numpy as np
import pytest

import oracle as O
from roift_b200 import synth

pytestmark = pytest.mark.gpu


def _case():
    c = synth.small_case(seed=31, shape=(20, 24, 64), pol=-0.3, adjacency=6, nlabels=1,
                         noise=120, contrast=400, weight_mode="grad_q")
    img = c.image.astype(np.int32)
    return c, img


def _expected(c, img):
    Z, Y, X = c.shape
    W, _ = O.build_weights(img, 6, "grad_q", wq=4095)
    return O.oift_fmax(W, (X, Y, Z), 6, c.seeds, c.seed_labels, pol=c.pol)


@pytest.mark.parametrize("limits", [dict(max_levels=1), dict(max_levels=3),
                                    dict(spin_limit=1)])
def test_single_run_wait_limits_end_with_not_converged(roift, oracle_lib, limits):
    c, img = _case()
    p = roift.make_params(c.shape, adjacency=6, weight_mode="grad_q", wq=4095, pol=c.pol,
                          sweeps=4)
    ctx = roift.Context(0)
    ctx.set_limits(**limits)
    with pytest.raises(roift.OiftError) as e:
        ctx.run_host(p, img, c.label_map(), c.seeds, want_cost=True)
    assert e.value.status == roift.E_NOT_CONVERGED
    # the same context, default limits: a full run is bit-exact again
    ctx.set_limits()
    lab, cost, _, _, st = ctx.run_host(p, img, c.label_map(), c.seeds, want_cost=True)
    cost_r2, lab_r2, levels = _expected(c, img)
    assert np.array_equal(cost, cost_r2)
    assert st.levels >= levels > 3
    ctx.close()


def test_batch_level_cap_reports_per_job(roift, oracle_lib):
    """Batched driver with a level cap that the volumes exceed and a job that needs a
    single level (every voxel a seed): the capped jobs end with OIFT_E_NOT_CONVERGED, a job
    that ran to completion has the single-run result, and after the limits are restored the
    same batch is bit-exact."""
    import torch
    dev = torch.device("cuda:0")
    cases = [synth.ellipsoid3d(seed=40 + i, size=s, sweeps=3, pol=-0.2)
             for i, s in enumerate([48, 40, 56])]
    flat = synth.ellipsoid3d(seed=50, size=32, sweeps=3, pol=0.1)
    flat.seeds = np.arange(flat.n, dtype=np.int32)
    flat.seed_labels = np.zeros(flat.n, np.int32)
    cases.append(flat)
    keep, jobs = [], (roift.Job * len(cases))()
    for i, c in enumerate(cases):
        img = torch.from_numpy(c.image.copy()).to(dev)
        sd = torch.from_numpy(c.seeds).to(dev)
        sl = torch.from_numpy(c.seed_labels).to(dev)
        lab = torch.full((c.n,), -5, dtype=torch.int32, device=dev)
        keep.append((img, sd, sl, lab))
        Z, Y, X = c.shape
        jobs[i] = roift.Job(img.data_ptr(), X, Y, Z, sd.data_ptr(), sl.data_ptr(), len(c.seeds),
                            float(np.float32(c.pol * 100.0)), None, lab.data_ptr(), None, 0)
    p = roift.make_params((1, 1, 1), adjacency=6, weight_mode="grad_q", wq=4095, sweeps=3)
    ctx = roift.Context(0)
    ctx.set_limits(max_levels=2)
    with pytest.raises(roift.OiftError) as e:
        ctx.run_batch(p, jobs, teams=len(cases))
    torch.cuda.synchronize()
    assert e.value.status == roift.E_NOT_CONVERGED
    statuses = [j.status for j in jobs]
    assert all(s in (0, roift.E_NOT_CONVERGED) for s in statuses), statuses
    assert all(s == roift.E_NOT_CONVERGED for s in statuses[:3]), statuses

    def single(i):
        c, (img, sd, sl, _) = cases[i], keep[i]
        prm = roift.make_params(c.shape, adjacency=6, weight_mode="grad_q", wq=4095, pol=c.pol,
                                sweeps=3)
        out = torch.empty(c.n, dtype=torch.int32, device=dev)
        roift._ctx().run_device(prm, img.data_ptr(), sd.data_ptr(), sl.data_ptr(), len(c.seeds),
                                label=out.data_ptr())
        torch.cuda.synchronize()
        return out

    if statuses[3] == 0:
        assert torch.equal(keep[3][3], single(3))
    ctx.set_limits()
    for j in jobs:
        j.status = 0
    ctx.run_batch(p, jobs, teams=len(cases))
    torch.cuda.synchronize()
    for i in range(len(cases)):
        assert jobs[i].status == 0
        assert torch.equal(keep[i][3], single(i))
    ctx.close()
