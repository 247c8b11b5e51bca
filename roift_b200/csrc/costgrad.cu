// costgrad.cu -- the arc-weight-map part of the adjoint: the f_max cost map of a fixed OIFT
// forest as a function of the weight parameters, a soft-Dice loss on it, and its gradient
// through the bottleneck arcs (row "differentiation"; the reference has no gradient).
//
// Bottleneck arcs.  On the OIFT forest a voxel's f_max cost is the largest arc weight on
// its path, C(p) = max(C(pred), w(pred -> p)) (gft/src/gft_ift.cpp:965-981 with f_max).  With
// the forest held fixed, dC(p)/dtheta is the derivative of that one arc, b(p).  The forest
// is read from the integer OIFT result (cost and label maps): in level (c, l) the entry
// voxels are those reached at exactly c from a voxel of label l conquered earlier (a seed,
// or cost < c) -- that arc weighs c and is b(p), the first such neighbour in the gft
// Spheric order (gft/src/gft_adjrel3.cpp:47-85); every other voxel of the level takes the
// bottleneck of a same-level neighbour that reaches it through an open arc (weight <= c),
// assigned by synchronous rounds from the entries outward (one round per voxel step, the
// first assigned neighbour in Spheric order winning).  The integer weights are the OIFT's
// own: base = |dI| (GRAD) or min(|dI|, wq) (GRAD_Q), oriented with the tail label's
// polarity in double and truncated (gft_ift.cpp:965-973).
//
// Differentiable cost.  The same arc with the continuous Gaussian-RBF weight of the
// weight parameters theta = (sigma, alpha, beta):
//   d   = beta |I_t - I_h| + (1 - beta) (g_t + g_h) / 2          (exp_gradient_weight.cpp:244-247)
//   c   = d (1 + s alpha_l),  s = sign(I_t - I_h),  alpha_l = -alpha (tail label 0) or +alpha
//                                                              (gft_ift.cpp:965-973, per = 100 alpha)
//   w   = 1 - exp(-c^2 / (2 sigma^2))                          (the RBF arc weight of the
//                                                              quantised OIFT, divided by wq)
// and the soft cost C~(p) = w(b(p)) (0 at seeds).  Object confidence u(p) = 1 - C~/2 for an
// object label, C~/2 for the background; L = 1 - (2 sum u t + eps) / (sum u + sum t + eps).
// dL/du(p) = A t(p) + B with A = -2 / (P + T + eps), B = (2 I + eps) / (P + T + eps)^2, so one
// pass accumulates I, P, T and the two theta-vectors sum t u' w' and sum u' w'.
#include <cmath>
#include <vector>

#include "kernels.cuh"

namespace oiftb {

constexpr long long BN_UNSET = -1;  // not yet assigned
constexpr long long BN_SEED = -2;   // a seed: cost 0, no arc
constexpr long long BN_NONE = -3;   // unreached voxel

struct BottleneckArgs {
    int X, Y, Z;
    size_t N;
    int nadj;
    int dx[26], dy[26], dz[26];
    const int16_t *img;
    const int32_t *cost, *label;
    const uint8_t *seed;  // 1 at seeds
    int wmode, wq;
    double fgt0, flt0, fgt1, flt1;  // oriented factors of label 0 and of every other label
};

// Integer oriented weight of the arc t -> h (h = t + d_i), the tail's label selecting the
// polarity, as the OIFT builds and orients it.
__device__ __forceinline__ int bn_weight(const BottleneckArgs &A, size_t t, size_t h, int lt) {
    const int it = A.img[t], ih = A.img[h];
    const int d = it - ih;
    int base = d < 0 ? -d : d;
    if (A.wmode == OIFT_W_GRAD_Q && base > A.wq) base = A.wq;
    const double fgt = lt == 0 ? A.fgt0 : A.fgt1, flt = lt == 0 ? A.flt0 : A.flt1;
    return oriented_weight((uint32_t)base, it > ih, it < ih, fgt, flt);
}

__global__ void bn_entry_kernel(BottleneckArgs A, long long *arcs) {
    const size_t XY = (size_t)A.X * A.Y;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < A.N;
         p += (size_t)gridDim.x * blockDim.x) {
        if (A.seed[p]) {
            arcs[p] = BN_SEED;
            continue;
        }
        const int c = A.cost[p], l = A.label[p];
        if (c == 0x7fffffff || l < 0) {
            arcs[p] = BN_NONE;
            continue;
        }
        const int x = (int)(p % A.X), y = (int)((p / A.X) % A.Y), z = (int)(p / XY);
        long long b = BN_UNSET;
        for (int i = 0; i < A.nadj && b == BN_UNSET; i++) {
            const int qx = x + A.dx[i], qy = y + A.dy[i], qz = z + A.dz[i];
            if (qx < 0 || qy < 0 || qz < 0 || qx >= A.X || qy >= A.Y || qz >= A.Z) continue;
            const size_t q = (size_t)qx + (size_t)qy * A.X + (size_t)qz * XY;
            if (A.label[q] != l || !(A.seed[q] || A.cost[q] < c)) continue;
            // the arc q -> p is direction nadj-1-i seen from q
            if (bn_weight(A, q, p, l) == c) b = (long long)q * 32 + (A.nadj - 1 - i);
        }
        arcs[p] = b;
    }
}

__global__ void bn_round_kernel(BottleneckArgs A, const long long *in, long long *out,
                                int *changed) {
    const size_t XY = (size_t)A.X * A.Y;
    int ch = 0;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < A.N;
         p += (size_t)gridDim.x * blockDim.x) {
        long long b = in[p];
        if (b == BN_UNSET) {
            const int c = A.cost[p], l = A.label[p];
            const int x = (int)(p % A.X), y = (int)((p / A.X) % A.Y), z = (int)(p / XY);
            for (int i = 0; i < A.nadj && b == BN_UNSET; i++) {
                const int qx = x + A.dx[i], qy = y + A.dy[i], qz = z + A.dz[i];
                if (qx < 0 || qy < 0 || qz < 0 || qx >= A.X || qy >= A.Y || qz >= A.Z) continue;
                const size_t q = (size_t)qx + (size_t)qy * A.X + (size_t)qz * XY;
                const long long bq = in[q];
                if (bq < 0 || A.seed[q] || A.label[q] != l || A.cost[q] != c) continue;
                if (bn_weight(A, q, p, l) <= c) b = bq;
            }
            if (b != BN_UNSET) ch = 1;
        }
        out[p] = b;
    }
    if (__syncthreads_or(ch) && threadIdx.x == 0) atomicExch(changed, 1);
}

struct CostGradArgs {
    int X, Y, Z;
    size_t N;
    int nadj;
    int dx[26], dy[26], dz[26];
    const int16_t *img;
    const float *g;  // gradient map of the blend (may be null: 0)
    const int32_t *label;
    const long long *arcs;
    const uint8_t *truth;
    double sigma, alpha, beta;
};

// Per-block sums: I, P, T, then sum t u' dw/dtheta (3) and sum u' dw/dtheta (3).
__global__ void cost_loss_kernel(CostGradArgs A, double *sums) {
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const size_t XY = (size_t)A.X * A.Y;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < A.N;
         p += (size_t)gridDim.x * blockDim.x) {
        const long long b = A.arcs[p];
        const int lp = A.label[p];
        const double t = A.truth[p] ? 1.0 : 0.0;
        double u, du = 0.0, dw[3] = {0, 0, 0};
        if (b >= 0) {
            const size_t tv = (size_t)(b >> 5);
            const int dir = (int)(b & 31);
            const int tx = (int)(tv % A.X), ty = (int)((tv / A.X) % A.Y), tz = (int)(tv / XY);
            const size_t hv = (size_t)(tx + A.dx[dir]) + (size_t)(ty + A.dy[dir]) * A.X +
                              (size_t)(tz + A.dz[dir]) * XY;
            const double diff = (double)A.img[tv] - (double)A.img[hv];
            const double s = diff > 0 ? 1.0 : (diff < 0 ? -1.0 : 0.0);
            const double dabs = fabs(diff);
            const double gavg = A.g ? 0.5 * ((double)A.g[tv] + (double)A.g[hv]) : 0.0;
            const double d = A.beta * dabs + (1.0 - A.beta) * gavg;
            const double sl = A.label[tv] == 0 ? -1.0 : 1.0;
            const double fac = 1.0 + s * sl * A.alpha;
            const double c = d * fac;
            const double is2 = 1.0 / (A.sigma * A.sigma);
            const double e = exp(-0.5 * c * c * is2);
            const double w = 1.0 - e;
            const double dw_dc = e * c * is2;
            dw[0] = -e * c * c * is2 / A.sigma;
            dw[1] = dw_dc * d * s * sl;
            dw[2] = dw_dc * (dabs - gavg) * fac;
            u = lp != 0 ? 1.0 - 0.5 * w : 0.5 * w;
            du = lp != 0 ? -0.5 : 0.5;
        } else {
            u = (b == BN_SEED && lp != 0) ? 1.0 : 0.0;  // a seed costs 0; an unreached voxel 0
        }
        acc[0] += u * t;
        acc[1] += u;
        acc[2] += t;
        for (int k = 0; k < 3; k++) {
            acc[3 + k] += t * du * dw[k];
            acc[6 + k] += du * dw[k];
        }
    }
    __shared__ double red[9][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 9; k++) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[k][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 9) {
        double v = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x][w];
        sums[(size_t)blockIdx.x * 9 + threadIdx.x] = v;
    }
}

__global__ void seed_flag_kernel(const int32_t *seeds, int nseeds, size_t N, uint8_t *flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nseeds && seeds[i] >= 0 && (size_t)seeds[i] < N) flag[seeds[i]] = 1;
}

int bottleneck_run(const BottleneckSetup &S, cudaStream_t s, int sms, long long *arcs,
                   long long *tmp, int *d_changed, int *h_changed, int *rounds_out) {
    BottleneckArgs A{};
    A.X = S.X;
    A.Y = S.Y;
    A.Z = S.Z;
    A.N = (size_t)S.X * S.Y * S.Z;
    const Adjacency adj = make_adjacency(S.adjacency == 4 ? 6 : (S.adjacency == 8 ? 26 : S.adjacency));
    A.nadj = adj.n;
    for (int i = 0; i < adj.n; i++) {
        A.dx[i] = adj.dx[i];
        A.dy[i] = adj.dy[i];
        A.dz[i] = adj.dz[i];
    }
    A.img = S.img;
    A.cost = S.cost;
    A.label = S.label;
    A.seed = S.seed;
    A.wmode = S.wmode;
    A.wq = S.wq;
    // label 0 takes -per, the others +per (gft_ift.cpp:968), evaluated as the OIFT does
    A.fgt0 = 1.0 + (double)(-S.per) / 100.0;
    A.flt0 = 1.0 - (double)(-S.per) / 100.0;
    A.fgt1 = 1.0 + (double)S.per / 100.0;
    A.flt1 = 1.0 - (double)S.per / 100.0;
    const int blocks = (int)std::min<size_t>((A.N + 255) / 256, (size_t)sms * 16);
    bn_entry_kernel<<<blocks, 256, 0, s>>>(A, arcs);
    long long *cur = arcs, *nxt = tmp;
    int rounds = 0;
    // one round per voxel step inside a level; a level cannot be deeper than the volume
    for (size_t r = 0; r <= A.N; r++) {
        if (cudaMemsetAsync(d_changed, 0, sizeof(int), s) != cudaSuccess) return OIFT_E_CUDA;
        bn_round_kernel<<<blocks, 256, 0, s>>>(A, cur, nxt, d_changed);
        if (cudaMemcpyAsync(h_changed, d_changed, sizeof(int), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return OIFT_E_CUDA;
        std::swap(cur, nxt);
        rounds++;
        if (!*h_changed) break;
    }
    if (cur != arcs &&
        cudaMemcpyAsync(arcs, cur, A.N * sizeof(long long), cudaMemcpyDeviceToDevice, s) !=
            cudaSuccess)
        return OIFT_E_CUDA;
    if (rounds_out) *rounds_out = rounds;
    return cudaGetLastError() == cudaSuccess ? OIFT_OK : OIFT_E_CUDA;
}

int cost_loss_run(const CostLossSetup &S, cudaStream_t s, int sms, double *d_sums,
                  int max_blocks, double *loss, double *grad) {
    CostGradArgs A{};
    A.X = S.X;
    A.Y = S.Y;
    A.Z = S.Z;
    A.N = (size_t)S.X * S.Y * S.Z;
    const Adjacency adj = make_adjacency(S.adjacency == 4 ? 6 : (S.adjacency == 8 ? 26 : S.adjacency));
    A.nadj = adj.n;
    for (int i = 0; i < adj.n; i++) {
        A.dx[i] = adj.dx[i];
        A.dy[i] = adj.dy[i];
        A.dz[i] = adj.dz[i];
    }
    A.img = S.img;
    A.g = S.g;
    A.label = S.label;
    A.arcs = S.arcs;
    A.truth = S.truth;
    A.sigma = S.sigma;
    A.alpha = S.alpha;
    A.beta = S.beta;
    const int blocks = (int)std::min<size_t>((A.N + 255) / 256, (size_t)std::min(max_blocks, sms * 8));
    cost_loss_kernel<<<blocks, 256, 0, s>>>(A, d_sums);
    std::vector<double> h((size_t)blocks * 9);
    if (cudaMemcpyAsync(h.data(), d_sums, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return OIFT_E_CUDA;
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < blocks; b++)  // fixed order: the sums do not depend on scheduling
        for (int k = 0; k < 9; k++) v[k] += h[(size_t)b * 9 + k];
    const double I = v[0], P = v[1], T = v[2], eps = S.eps;
    const double den = P + T + eps;
    *loss = 1.0 - (2.0 * I + eps) / den;
    if (grad) {
        const double Acoef = -2.0 / den, Bcoef = (2.0 * I + eps) / (den * den);
        for (int k = 0; k < 3; k++) grad[k] = Acoef * v[3 + k] + Bcoef * v[6 + k];
    }
    return OIFT_OK;
}

}  // namespace oiftb
