"""GPU: the host entry oift_b200_run_host with a seed list long enough that its seed-label
gather is split over host threads (more than 65,536 seeds).

The labels it gathers decide the OIFT's result, so the cost map and labels must equal the
oracle's (R2, lexicographic Dijkstra f_max) bit for bit; a bad seed anywhere in the list
must give the error the first bad seed in list order gives, and the context must stay
usable after it.
"""
import numpy as np
import pytest

import oracle as O
from roift_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big_seed_case():
    c = synth.ellipsoid3d(seed=3, size=128, sweeps=5)
    assert len(c.seeds) > 65536, "the case must exercise the split gather"
    img = c.image.astype(np.int32)
    img -= min(0, int(img.min()))
    return c, img


def _params(roift, c, sweeps=0):
    return roift.make_params(c.shape, adjacency=6, weight_mode="grad_q", wq=4095, pol=c.pol,
                             sweeps=sweeps)


def test_host_entry_many_seeds_matches_oracle(roift, big_seed_case):
    c, img = big_seed_case
    Z, Y, X = c.shape
    ctx = roift._ctx()
    lab, cost, _, _, _ = ctx.run_host(_params(roift, c), img, c.label_map(), c.seeds,
                                      want_cost=True)
    W, _ = O.build_weights(img, 6, "grad_q", wq=4095)
    cost_r, lab_r, _ = O.oift_fmax(W, (X, Y, Z), 6, c.seeds, c.seed_labels, pol=c.pol)
    assert np.array_equal(cost, cost_r)
    assert np.array_equal(lab, lab_r)


def test_host_entry_bad_seed_late_in_a_long_list(roift, big_seed_case):
    c, img = big_seed_case
    ctx = roift._ctx()
    p = _params(roift, c)
    n = len(c.seeds)
    # an index outside the volume in the last part of the list
    seeds = c.seeds.astype(np.int32).copy()
    seeds[n - 3] = c.n
    with pytest.raises(roift.OiftError) as e:
        ctx.run_host(p, img, c.label_map(), seeds)
    assert e.value.status == roift.E_SEED_RANGE
    # a label above the largest label the keys hold, in the middle of the list
    lab = c.label_map()
    lab[c.seeds[n // 2]] = 40000
    with pytest.raises(roift.OiftError) as e:
        ctx.run_host(p, img, lab, c.seeds)
    assert e.value.status == roift.E_BAD_ARG
    # both: the first bad seed in list order (the label, at n // 3) decides
    lab = c.label_map()
    lab[c.seeds[n // 3]] = 40000
    with pytest.raises(roift.OiftError) as e:
        ctx.run_host(p, img, lab, seeds)
    assert e.value.status == roift.E_BAD_ARG
    # the context stays usable: a clean call gives the clean result
    lab_ok, cost_ok, _, _, _ = ctx.run_host(p, img, c.label_map(), c.seeds, want_cost=True)
    fresh = roift.Context(0)
    try:
        lab_ref, cost_ref, _, _, _ = fresh.run_host(p, img, c.label_map(), c.seeds, want_cost=True)
    finally:
        fresh.close()
    assert np.array_equal(cost_ok, cost_ref)
    assert np.array_equal(lab_ok, lab_ref)
