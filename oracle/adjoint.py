"""TEST INFRASTRUCTURE ONLY: FP64 restatement of the differentiable relaxation and its
reverse-mode gradient, the checker of the CUDA adjoint (oift_b200_adjoint).

Parity unpinned: the reference has no gradient.  The forward model generalises the
relaxation sweep of ORelax_1_Multi (gft/src/gft_ift.cpp:8774-8833) with the weight
families of the reference experiments:

  d_pq    = beta * |I_p - I_q| + (1 - beta) * (g_p + g_q) / 2
            (gradient blend, experiments/exp_gradient_weight.cpp:244-247)
  w_or    = d_pq * (1 + s_pq * alpha * (2 m_bg(q) - 1)),  s_pq = sign(I_p - I_q)
            (soft polarity, gft_ift.cpp:8804-8811, per = 100 alpha)
  K(w)    = exp(-w^2 / sigma^2)                         (RBF, exp_gaussian_rbf_relax.cpp:343-345)
          or max(0, Wmax - w)^8, Wmax = max(I) (1 + |alpha|)   (gft_ift.cpp:8733-8734, 8812-8818)
  W_pq    = K(w_or) / Dpq   (each voxel's weights scaled by a common factor, below)
  m'(p)   = sum_q W_pq m(q) / sum_q W_pq on the growing mask (boundary of the OIFT labels
            dilated one ring per sweep), m'(p) = m(p) elsewhere or when the sum is 0,
            seeds one-hot.

The loss is the soft Dice of p_obj = 1 - m_bg against a binary truth:
L = 1 - (2 sum p t + eps) / (sum p + sum t + eps).  Gradients are with respect to
(sigma, alpha, beta); the OIFT labels are held fixed.
"""
from __future__ import annotations

import numpy as np

NIL = -1


def offsets(adj: int):
    """Spheric order without the centre (gft/src/gft_adjrel3.cpp:47-85)."""
    r2 = 3 if adj in (26, 8) else 1
    out = []
    for z in (-1, 0, 1):
        for y in (-1, 0, 1):
            for x in (-1, 0, 1):
                if (x, y, z) != (0, 0, 0) and x * x + y * y + z * z <= r2:
                    out.append((x, y, z))
    return out


def _shift(a, dx, dy, dz, fill=0.0):
    """b[z, y, x] = a[z + dz, y + dy, x + dx] (neighbour q = p + d), fill outside."""
    Z, Y, X = a.shape[-3:]
    b = np.full(a.shape, fill, dtype=a.dtype)
    zs, ys, xs = slice(max(0, -dz), Z - max(0, dz)), slice(max(0, -dy), Y - max(0, dy)), \
        slice(max(0, -dx), X - max(0, dx))
    zq, yq, xq = slice(max(0, dz), Z - max(0, -dz)), slice(max(0, dy), Y - max(0, -dy)), \
        slice(max(0, dx), X - max(0, -dx))
    b[..., zs, ys, xs] = a[..., zq, yq, xq]
    return b


def _unshift(a, dx, dy, dz):
    """Adjoint of _shift: the value held at p moves to q = p + d."""
    return _shift(a, -dx, -dy, -dz, 0.0)


class Problem:
    def __init__(self, img, labels0, seeds, seed_labels, truth, adj=6, grad=None, K=10,
                 kernel="rbf", eps=1.0):
        self.img = np.asarray(img, np.float64)
        self.shape = self.img.shape
        Z, Y, X = self.shape
        self.adj = adj if Z > 1 else (8 if adj in (26, 8) else 4)
        self.offs = [o for o in offsets(26 if adj in (26, 8) else 6) if Z > 1 or o[2] == 0]
        self.g = np.zeros(self.shape) if grad is None else np.asarray(grad, np.float64)
        self.K = K
        self.kernel = kernel
        self.eps = eps
        lab = np.asarray(labels0, np.int64).reshape(self.shape)
        seeds = np.asarray(seeds, np.int64)
        sl = np.asarray(seed_labels, np.int64)
        self.classes = sorted({0} | {int(v) for v in sl if v >= 0})
        C = len(self.classes)
        self.bg = self.classes.index(0)
        cls = np.full(self.shape, self.bg, np.int64)
        for k, l in enumerate(self.classes):
            cls[lab == l] = k
        self.m0 = np.zeros((C,) + self.shape)
        for k in range(C):
            self.m0[k][cls == k] = 1.0
        self.seed = np.zeros(self.shape, bool)
        self.seed_cls = np.full(self.shape, -1, np.int64)
        flat_seed, flat_sc = self.seed.reshape(-1), self.seed_cls.reshape(-1)
        for p, l in zip(seeds, sl):
            flat_seed[p] = True
            flat_sc[p] = self.classes.index(int(l) if l >= 0 else 0)
        # growing mask: rings around the voxels with a neighbour of another label
        valid = np.ones(self.shape, bool)
        bnd = np.zeros(self.shape, bool)
        for dx, dy, dz in self.offs:
            v = _shift(valid, dx, dy, dz, False)
            bnd |= v & (_shift(lab, dx, dy, dz, 0) != lab)
        dist = np.where(bnd, 0, 1 << 20)
        cur = bnd.copy()
        for t in range(1, K + 1):
            nxt = cur.copy()
            for dx, dy, dz in self.offs:
                nxt |= _shift(cur, dx, dy, dz, False)
            dist = np.where(nxt & ~cur, t, dist)
            cur = nxt
        self.dist = dist
        self.truth = np.asarray(truth, np.float64).reshape(self.shape)
        self.Imax = float(self.img.max())

    # ---- weights of every (p, q = p + d) pair ----
    # The sweep is invariant to a common factor on the weights of one voxel p, so each
    # voxel's weights are divided by its largest one (the neighbour with the smallest w):
    # no underflow, and the derivatives are taken with that factor held fixed (its own
    # derivative cancels in sum W (m_q - m'(p)) = 0).
    def weights(self, m, sigma, alpha, beta, want_grad=False):
        pre = []
        for dx, dy, dz in self.offs:
            valid = _shift(np.ones(self.shape, bool), dx, dy, dz, False)
            Iq = _shift(self.img, dx, dy, dz)
            gq = _shift(self.g, dx, dy, dz)
            mbg = _shift(m[self.bg], dx, dy, dz)
            diff = self.img - Iq
            s = np.sign(diff)
            dabs = np.abs(diff)
            gavg = 0.5 * (self.g + gq)
            dd = beta * dabs + (1.0 - beta) * gavg
            fac = 1.0 + s * alpha * (2.0 * mbg - 1.0)
            pre.append((valid, s, dabs, gavg, dd, fac, mbg, dd * fac))
        wmin = np.full(self.shape, np.inf)
        for valid, *_, w in pre:
            wmin = np.where(valid, np.minimum(wmin, w), wmin)
        wmin = np.where(np.isfinite(wmin), wmin, 0.0)
        Wmax = self.Imax * (1.0 + abs(alpha))
        out = []
        for (valid, s, dabs, gavg, dd, fac, mbg, w), (dx, dy, dz) in zip(pre, self.offs):
            Dpq = np.sqrt(dx * dx + dy * dy + dz * dz)
            if self.kernel == "rbf":
                Kw = np.exp(-(w * w - wmin * wmin) / (sigma * sigma))
                dK_dw = -2.0 * w / (sigma * sigma) * Kw
                dK_dsig = 2.0 * w * w / sigma ** 3 * Kw
                dK_dwmax = 0.0
            else:
                R = Wmax - wmin
                Rs = np.where(R > 0, R, 1.0)
                r = np.maximum(0.0, Wmax - w)
                Kw = np.where(R > 0, (r / Rs) ** 8, 0.0)
                dK_dw = np.where(R > 0, -8.0 * r ** 7 / Rs ** 8, 0.0)
                dK_dsig = 0.0 * Kw
                dK_dwmax = -dK_dw
            W = np.where(valid, Kw / Dpq, 0.0)
            if not want_grad:
                out.append(W)
                continue
            dW_dmbg = np.where(valid, dK_dw * dd * s * alpha * 2.0 / Dpq, 0.0)
            dW_dsig = np.where(valid, dK_dsig / Dpq, 0.0)
            dW_dalpha = dK_dw * dd * s * (2.0 * mbg - 1.0)
            if self.kernel != "rbf":
                dW_dalpha = dW_dalpha + dK_dwmax * self.Imax * np.sign(alpha)
            dW_dalpha = np.where(valid, dW_dalpha / Dpq, 0.0)
            dW_dbeta = np.where(valid, dK_dw * (dabs - gavg) * fac / Dpq, 0.0)
            out.append((W, dW_dmbg, dW_dsig, dW_dalpha, dW_dbeta))
        return out

    def sweep(self, m, t, sigma, alpha, beta):
        Ws = self.weights(m, sigma, alpha, beta)
        S = sum(Ws)
        num = np.zeros_like(m)
        for W, (dx, dy, dz) in zip(Ws, self.offs):
            num += W * _shift(m, dx, dy, dz)
        act = (self.dist <= t) & ~self.seed & (S > 0)
        mn = np.where(act, num / np.where(S > 0, S, 1.0), m)
        for k in range(m.shape[0]):
            mn[k][self.seed] = (self.seed_cls[self.seed] == k).astype(np.float64)
        return mn, S

    def forward(self, sigma, alpha, beta, keep=False):
        m = self.m0.copy()
        for k in range(m.shape[0]):
            m[k][self.seed] = (self.seed_cls[self.seed] == k).astype(np.float64)
        states = [m]
        for t in range(self.K):
            m, _ = self.sweep(m, t, sigma, alpha, beta)
            if keep:
                states.append(m)
        loss = self._loss(m)
        return (loss, m, states) if keep else (loss, m)

    def _loss(self, m):
        p = 1.0 - m[self.bg]
        I, P, T = (p * self.truth).sum(), p.sum(), self.truth.sum()
        return 1.0 - (2.0 * I + self.eps) / (P + T + self.eps)

    def gradient(self, sigma, alpha, beta):
        """Reverse mode through the K sweeps: (loss, [dL/dsigma, dL/dalpha, dL/dbeta])."""
        loss, mK, states = self.forward(sigma, alpha, beta, keep=True)
        p = 1.0 - mK[self.bg]
        I, P, T = (p * self.truth).sum(), p.sum(), self.truth.sum()
        den = P + T + self.eps
        dL_dp = -(2.0 * self.truth * den - (2.0 * I + self.eps)) / (den * den)
        lam = np.zeros_like(mK)
        lam[self.bg] = -dL_dp
        g = np.zeros(3)
        for t in range(self.K - 1, -1, -1):
            m, mn = states[t], states[t + 1]
            parts = self.weights(m, sigma, alpha, beta, want_grad=True)
            S = sum(pp[0] for pp in parts)
            act = (self.dist <= t) & ~self.seed & (S > 0)
            Ssafe = np.where(S > 0, S, 1.0)
            lam_act = np.where(act, lam, 0.0)
            new = np.where(act | self.seed, 0.0, lam)   # copied voxels pass lambda through
            for (W, dmbg, dsig, dal, dbe), (dx, dy, dz) in zip(parts, self.offs):
                mq = _shift(m, dx, dy, dz)
                a = (lam_act * (mq - mn)).sum(axis=0) / Ssafe
                new += _unshift(lam_act * W / Ssafe, dx, dy, dz)
                new[self.bg] += _unshift(dmbg * a, dx, dy, dz)
                g += [(dsig * a).sum(), (dal * a).sum(), (dbe * a).sum()]
            new[:, self.seed] = 0.0
            lam = new
        return loss, g


# ------------------------------------------------------- arc-weight-map term -------
# The cost map of a fixed OIFT forest as a function of (sigma, alpha, beta): each voxel's
# f_max cost is carried by one arc of its path (its bottleneck), read from the integer OIFT
# result; the continuous RBF weight of that arc gives a soft cost, the soft cost an object
# confidence, and the confidence a soft-Dice loss whose gradient is the bottleneck-arc
# subgradient of f_max (gft/src/gft_ift.cpp:965-981 with f_max; weights of
# experiments/exp_gaussian_rbf_relax.cpp:343-345 and exp_gradient_weight.cpp:244-247).

def _oriented_int(base, gt, lt, fgt, flt):
    """int(base * f) in double, truncated (gft_ift.cpp:965-973); base >= 0."""
    out = base.astype(np.int64).copy()
    out = np.where(gt, np.floor(base.astype(np.float64) * fgt).astype(np.int64), out)
    out = np.where(lt, np.floor(base.astype(np.float64) * flt).astype(np.int64), out)
    return out


def bottleneck_arcs(img, cost, label, seeds, adj, pol, mode="grad_q", wq=4095):
    """Restatement of oift_b200_bottleneck_arcs: int64 [N], tail * 32 + direction (Spheric
    order, tail -> tail + d), -2 at seeds, -3 unreached, -1 never assigned."""
    img = np.asarray(img, np.int64)
    Z, Y, X = img.shape
    N = X * Y * Z
    I = img.reshape(-1)
    cost = np.asarray(cost, np.int64).reshape(-1)
    label = np.asarray(label, np.int64).reshape(-1)
    seed = np.zeros(N, bool)
    seed[np.asarray(seeds, np.int64)] = True
    per = float(np.float32(pol * 100.0))
    fac = {0: (1.0 + (-per) / 100.0, 1.0 - (-per) / 100.0), 1: (1.0 + per / 100.0, 1.0 - per / 100.0)}
    offs = offsets(adj)
    n = len(offs)
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    z, y, x = z.reshape(-1), y.reshape(-1), x.reshape(-1)
    arcs = np.full(N, -1, np.int64)
    arcs[(cost == np.iinfo(np.int32).max) | (label < 0)] = -3
    arcs[seed] = -2

    def neighbour(i):
        dx, dy, dz = offs[i]
        qx, qy, qz = x + dx, y + dy, z + dz
        ok = (qx >= 0) & (qx < X) & (qy >= 0) & (qy < Y) & (qz >= 0) & (qz < Z)
        q = np.where(ok, qx + qy * X + qz * X * Y, 0)
        return q, ok

    def weight_to_p(q, lp):
        """Integer weight of the arc q -> p with the tail label lp (both labels equal)."""
        d = I[q] - I
        base = np.abs(d)
        if mode == "grad_q":
            base = np.minimum(base, wq)
        f0, f1 = fac[0], fac[1]
        fgt = np.where(lp == 0, f0[0], f1[0])
        flt = np.where(lp == 0, f0[1], f1[1])
        return _oriented_int(base, d > 0, d < 0, fgt, flt)

    unset = arcs == -1
    for i in range(n):
        q, ok = neighbour(i)
        cond = unset & (arcs == -1) & ok & (label[q] == label) & (seed[q] | (cost[q] < cost))
        cond &= weight_to_p(q, label) == cost
        arcs[cond] = q[cond] * 32 + (n - 1 - i)
    while True:
        old = arcs
        new = arcs.copy()
        done = np.zeros(N, bool)
        unset = old == -1
        for i in range(n):
            q, ok = neighbour(i)
            cond = unset & ~done & ok & (old[q] >= 0) & ~seed[q] & (label[q] == label)
            cond &= (cost[q] == cost) & (weight_to_p(q, label) <= cost)
            new[cond] = old[q][cond]
            done |= cond
        arcs = new
        if not done.any():
            break
    return arcs


def cost_loss(img, label, arcs, truth, sigma, alpha, beta, eps=1.0, adj=6, g=None):
    """FP64 soft-Dice loss of the cost-map confidence and its gradient (sigma, alpha, beta)."""
    img = np.asarray(img, np.float64)
    Z, Y, X = img.shape
    I = img.reshape(-1)
    G = None if g is None else np.asarray(g, np.float64).reshape(-1)
    label = np.asarray(label, np.int64).reshape(-1)
    arcs = np.asarray(arcs, np.int64).reshape(-1)
    t = (np.asarray(truth).reshape(-1) != 0).astype(np.float64)
    offs = np.array(offsets(adj), np.int64)
    has = arcs >= 0
    tail = np.where(has, arcs >> 5, 0)
    dirs = np.where(has, arcs & 31, 0)
    tx, ty, tz = tail % X, (tail // X) % Y, tail // (X * Y)
    head = (tx + offs[dirs, 0]) + (ty + offs[dirs, 1]) * X + (tz + offs[dirs, 2]) * X * Y
    head = np.where(has, head, 0)
    diff = I[tail] - I[head]
    s = np.sign(diff)
    dabs = np.abs(diff)
    gavg = 0.5 * (G[tail] + G[head]) if G is not None else np.zeros_like(diff)
    d = beta * dabs + (1.0 - beta) * gavg
    sl = np.where(label[tail] == 0, -1.0, 1.0)
    fac = 1.0 + s * sl * alpha
    c = d * fac
    e = np.exp(-0.5 * c * c / (sigma * sigma))
    w = 1.0 - e
    dw_dc = e * c / (sigma * sigma)
    dw = np.stack([-e * c * c / sigma ** 3, dw_dc * d * s * sl, dw_dc * (dabs - gavg) * fac])
    obj = label != 0
    u = np.where(has, np.where(obj, 1.0 - 0.5 * w, 0.5 * w),
                 np.where((arcs == -2) & obj, 1.0, 0.0))
    du = np.where(has, np.where(obj, -0.5, 0.5), 0.0)
    Isum, P, T = float((u * t).sum()), float(u.sum()), float(t.sum())
    den = P + T + eps
    loss = 1.0 - (2.0 * Isum + eps) / den
    dL_du = -2.0 * t / den + (2.0 * Isum + eps) / den ** 2
    grad = (dw * (dL_du * du)[None, :]).sum(axis=1)
    return loss, grad
