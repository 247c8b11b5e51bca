"""GPU: the adjoint of the relaxation (oift_b200_adjoint) against the FP64 reverse-mode
restatement in oracle/adjoint.py (itself checked against central differences on the CPU).

Bars: loss within 1e-5 relative of the FP64 forward; gradient within 1e-4 relative (plus
1e-7 of the largest component) of the FP64 gradient; the checkpoint interval does not
change the result beyond FP32 reduction order; a torch.autograd.Function wrapper (test
harness only) trains (sigma, alpha, beta) with Adam and lowers the loss.
"""
import numpy as np
import pytest

import oracle as O
from oracle import adjoint as A
from roift_b200 import synth

pytestmark = pytest.mark.gpu


def _problem(adj=6, shape=(18, 22, 26), seed=3):
    c = synth.small_case(seed=seed, shape=shape, pol=-0.3, adjacency=adj, nlabels=1,
                         noise=120, contrast=400)
    img = c.image.astype(np.int32)
    Z, Y, X = c.shape
    W, _ = O.build_weights(img, adj, "grad_q", wq=4095)
    _, lab, _ = O.oift_fmax(W, (X, Y, Z), adj, c.seeds, c.seed_labels, pol=c.pol)
    truth = (img.reshape(-1) > 850).astype(np.uint8)      # differs from the OIFT labels
    f = img.astype(np.float64)
    g = np.zeros_like(f)
    for ax in range(3):
        if f.shape[ax] > 2:
            g += np.gradient(f, axis=ax) ** 2
    g = np.sqrt(g).astype(np.float32)
    return c, img, lab.astype(np.int32), truth, g


def _gpu(roift, c, img, lab, truth, g, **kw):
    import torch
    dev = torch.device("cuda:0")
    t = dict(img=torch.from_numpy(img.astype(np.int16).reshape(-1).copy()).to(dev),
             lab=torch.from_numpy(lab).to(dev), sd=torch.from_numpy(c.seeds).to(dev),
             sl=torch.from_numpy(c.seed_labels).to(dev), tr=torch.from_numpy(truth).to(dev),
             g=torch.from_numpy(g.reshape(-1).copy()).to(dev))
    loss, grad = roift._ctx().adjoint(c.shape, t["img"].data_ptr(), t["lab"].data_ptr(),
                                      t["sd"].data_ptr(), t["sl"].data_ptr(), len(c.seeds),
                                      t["tr"].data_ptr(), grad_map_ptr=t["g"].data_ptr(), **kw)
    return loss, grad


@pytest.mark.parametrize("kernel,adj,shape", [("rbf", 6, (18, 22, 26)), ("pow8", 6, (18, 22, 26)),
                                              ("rbf", 26, (12, 16, 20)), ("rbf", 4, (1, 40, 52))])
def test_adjoint_matches_fp64(roift, oracle_lib, kernel, adj, shape):
    c, img, lab, truth, g = _problem(adj, shape)
    th = dict(sigma=180.0, alpha=0.25, beta=0.6)
    K = 9
    loss, grad = _gpu(roift, c, img, lab, truth, g, sweeps=K, checkpoint=3, kernel=kernel,
                      adjacency=adj, **th)
    P = A.Problem(img.reshape(c.shape), lab, c.seeds, c.seed_labels, truth, adj=adj,
                  grad=g.reshape(c.shape), K=K, kernel=kernel)
    loss64, grad64 = P.gradient(th["sigma"], th["alpha"], th["beta"])
    assert abs(loss - loss64) <= 1e-5 * abs(loss64)
    tol = 1e-4 * np.abs(grad64) + 1e-7 * np.abs(grad64).max()
    assert np.all(np.abs(grad - grad64) <= tol), (grad, grad64)


def test_adjoint_checkpoint_interval_invariant(roift, oracle_lib):
    c, img, lab, truth, g = _problem()
    ref = None
    for cp in (1, 2, 5, 12, 0):
        loss, grad = _gpu(roift, c, img, lab, truth, g, sweeps=12, checkpoint=cp, sigma=150.0,
                          alpha=-0.2, beta=0.8)
        if ref is None:
            ref = (loss, grad)
        assert abs(loss - ref[0]) <= 1e-12 * abs(ref[0])
        assert np.allclose(grad, ref[1], rtol=1e-6, atol=1e-12)


def test_adjoint_autograd_function_trains(roift, oracle_lib):
    """torch.autograd.Function over the C ABI (test harness only): backward gives the
    adjoint gradient, and Adam steps on (sigma, alpha, beta) lower the soft-Dice loss."""
    import torch
    c, img, lab, truth, g = _problem()

    class RelaxDice(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta):
            s, a, b = (float(v) for v in theta.detach().cpu())
            loss, grad = _gpu(roift, c, img, lab, truth, g, sweeps=10, sigma=s, alpha=a, beta=b)
            ctx.save_for_backward(torch.tensor(grad, dtype=torch.float64))
            return torch.tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            return gout * grad

    theta = torch.tensor([120.0, 0.1, 0.9], dtype=torch.float64, requires_grad=True)
    loss0 = RelaxDice.apply(theta)
    loss0.backward()
    _, direct = _gpu(roift, c, img, lab, truth, g, sweeps=10, sigma=120.0, alpha=0.1, beta=0.9)
    assert np.allclose(theta.grad.numpy(), direct)
    opt = torch.optim.Adam([theta], lr=0.02)
    first = None
    for _ in range(15):
        opt.zero_grad()
        loss = RelaxDice.apply(theta)
        loss.backward()
        opt.step()
        with torch.no_grad():
            theta[1].clamp_(-1.0, 1.0)
            theta[2].clamp_(0.0, 1.0)
        first = first if first is not None else float(loss)
    assert float(RelaxDice.apply(theta)) < first


# ---------------------------------------------------------- arc-weight-map term ----
@pytest.mark.parametrize("adj,shape,mode", [(6, (20, 24, 28), "grad_q"), (4, (1, 48, 56), "grad"),
                                            (26, (12, 16, 20), "grad_q")])
def test_cost_adjoint_matches_fp64_and_central_differences(roift, oracle_lib, adj, shape, mode):
    """Bottleneck arcs of the fixed OIFT forest (from the GPU's own integer OIFT result)
    equal the restatement's; the cost-map loss and its gradient equal the FP64
    restatement's; and the C-ABI gradient is within 1e-4 relative of central differences
    (h = 1e-3) of the GPU forward."""
    import torch
    c, img, lab, truth, g = _problem(adj, shape)
    dev = torch.device("cuda:0")
    N = c.n
    t_img = torch.from_numpy(img.astype(np.int16).reshape(-1).copy()).to(dev)
    t_sd = torch.from_numpy(c.seeds).to(dev)
    t_sl = torch.from_numpy(c.seed_labels).to(dev)
    cost = torch.empty(N, dtype=torch.int32, device=dev)
    olab = torch.empty(N, dtype=torch.int32, device=dev)
    arcs = torch.empty(N, dtype=torch.int64, device=dev)
    ctx = roift.Context(0)
    p = roift.make_params(c.shape, adjacency=adj, weight_mode=mode, wq=4095, pol=c.pol, sweeps=0)
    ctx.run_device(p, t_img.data_ptr(), t_sd.data_ptr(), t_sl.data_ptr(), len(c.seeds),
                   cost=cost.data_ptr(), oift_label=olab.data_ptr())
    ctx.bottleneck_arcs(p, t_img.data_ptr(), cost.data_ptr(), olab.data_ptr(), t_sd.data_ptr(),
                        len(c.seeds), arcs.data_ptr())
    torch.cuda.synchronize()
    cost_h, lab_h, arcs_h = cost.cpu().numpy(), olab.cpu().numpy(), arcs.cpu().numpy()
    arcs64 = A.bottleneck_arcs(img.reshape(c.shape), cost_h, lab_h, c.seeds, adj, c.pol, mode=mode)
    assert np.array_equal(arcs_h, arcs64)
    assert not (arcs_h == -1).any()
    t_lab = torch.from_numpy(lab_h).to(dev)
    t_tr = torch.from_numpy(truth).to(dev)
    t_g = torch.from_numpy(g.reshape(-1).copy()).to(dev)
    th = np.array([140.0, -0.25, 0.7])

    def gpu(theta, want_grad=True):
        return ctx.cost_adjoint(c.shape, t_img.data_ptr(), t_lab.data_ptr(), arcs.data_ptr(),
                                t_tr.data_ptr(), sigma=theta[0], alpha=theta[1], beta=theta[2],
                                adjacency=adj, grad_map_ptr=t_g.data_ptr(), want_grad=want_grad)

    loss, grad = gpu(th)
    # the C ABI takes float parameters: compare with FP64 at the same float values
    thf = np.array([np.float32(v) for v in th], np.float64)
    loss64, grad64 = A.cost_loss(img.reshape(c.shape), lab_h, arcs_h, truth, *thf, adj=adj,
                                 g=g.reshape(c.shape))
    assert abs(loss - loss64) <= 1e-9 * max(abs(loss64), 1e-12)
    assert np.allclose(grad, grad64, rtol=1e-8, atol=1e-12 * np.abs(grad64).max())
    h = 1e-3
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        # float parameters: difference the exact float points the GPU sees
        hi = np.array([np.float32(v) for v in th + e], np.float64)
        lo = np.array([np.float32(v) for v in th - e], np.float64)
        fd = (gpu(hi, False)[0] - gpu(lo, False)[0]) / (hi[k] - lo[k])
        assert abs(grad[k] - fd) <= 1e-4 * abs(grad[k]) + 1e-6 * np.abs(grad).max(), (k, grad, fd)
    ctx.close()
