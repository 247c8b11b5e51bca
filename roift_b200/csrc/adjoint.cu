// adjoint.cu -- gradient of a soft-Dice loss through K relaxation sweeps with respect to the
// weight parameters (RBF sigma, polarity alpha, gradient-mix beta), OIFT labels held fixed.
//
// Forward model (FP32; one thread per voxel, planar [class][N] membership):
//   d_pq  = beta |I_p - I_q| + (1 - beta) (g_p + g_q) / 2     (exp_gradient_weight.cpp:244-247)
//   w_or  = d_pq (1 + s_pq alpha (2 m_bg(q) - 1)), s_pq = sign(I_p - I_q)   (gft_ift.cpp:8804-8811)
//   K     = exp(-w_or^2 / sigma^2)  (exp_gaussian_rbf_relax.cpp:343-345)
//           or max(0, Wmax - w_or)^8, Wmax = max(I) (1 + |alpha|)   (gft_ift.cpp:8733, 8812-8818)
//   W_pq  = K / Dpq (scaled per voxel, see pair_weight);  m'(p) = sum_q W_pq m(q) / sum_q W_pq
//           on the growing mask (OIFT label
//           boundary dilated one ring per sweep, gft_ift.cpp:8859-8886), else m(p); seeds one-hot.
// Loss: L = 1 - (2 sum p t + eps) / (sum p + sum t + eps), p = 1 - m_bg, t the binary truth.
//
// Reverse mode: the adjoint of one sweep is a gather over the voxels q whose neighbours p
// read them; for each pair (p, q) with p updated:
//   a_pq       = sum_k lam(p,k) (m(q,k) - m'(p,k)) / S_p
//   lam(q,k)  += lam(p,k) W_pq / S_p;   lam(q,bg) += dW_pq/dm_bg(q) a_pq
//   dL/dtheta += dW_pq/dtheta a_pq
// Copied voxels pass lam through; seeds, being constants, stop it.  States are kept every
// `checkpoint` sweeps and each segment is recomputed (with its weight sums S) on the way
// back, so memory is (K/c + c + 2) membership volumes instead of K.
#include <cmath>
#include <vector>

#include "kernels.cuh"

namespace oiftb {

constexpr int ADJ_MAX_CLASSES = 8;

struct AdjArgs {
    int X, Y, Z;
    size_t N;
    int noff;
    int dx[26], dy[26], dz[26];
    float inv_dpq[26];
    int C, bg;
    int kernel;  // 0 RBF, 1 POW8
    float sigma, alpha, beta, Wmax, Imax;
    const int16_t *img;
    const float *g;       // may be null (0)
    const uint16_t *dist; // sweep at which the voxel joins the mask
    const uint8_t *seedc; // class of a seed, 0xFF otherwise
};

struct PairW {
    float W, dmbg, dsig, dal, dbe;
};

// Oriented distance w of the pair (p updated, q its neighbour).
__device__ __forceinline__ float pair_dist(const AdjArgs &A, int ip, int iq, float gp, float gq,
                                           float mbg_q) {
    const float diff = (float)(ip - iq);
    const float s = diff > 0.0f ? 1.0f : (diff < 0.0f ? -1.0f : 0.0f);
    const float dd = A.beta * fabsf(diff) + (1.0f - A.beta) * (0.5f * (gp + gq));
    return dd * (1.0f + s * A.alpha * (2.0f * mbg_q - 1.0f));
}

// Weight of the pair and its partial derivatives.  The sweep is invariant to a common
// factor on the weights of one voxel, so p's weights are divided by its largest one (its
// neighbour with the smallest w, wmin): nothing underflows in FP32, and the derivatives are
// taken with that factor held fixed (its own derivative cancels in sum W (m_q - m'(p)) = 0).
__device__ __forceinline__ PairW pair_weight(const AdjArgs &A, int ip, int iq, float gp, float gq,
                                             float mbg_q, float inv_dpq, float wmin,
                                             bool want_grad) {
    const float diff = (float)(ip - iq);
    const float s = diff > 0.0f ? 1.0f : (diff < 0.0f ? -1.0f : 0.0f);
    const float dabs = fabsf(diff);
    const float gavg = 0.5f * (gp + gq);
    const float dd = A.beta * dabs + (1.0f - A.beta) * gavg;
    const float fac = 1.0f + s * A.alpha * (2.0f * mbg_q - 1.0f);
    const float w = dd * fac;
    PairW r;
    float K, dK_dw, dK_dsig = 0.0f, dK_dwmax = 0.0f;
    if (A.kernel == 0) {
        const float is2 = 1.0f / (A.sigma * A.sigma);
        K = expf(-(w - wmin) * (w + wmin) * is2);
        dK_dw = -2.0f * w * is2 * K;
        dK_dsig = 2.0f * w * w * is2 / A.sigma * K;
    } else {
        const float R = A.Wmax - wmin;
        if (R > 0.0f) {
            const float iR = 1.0f / R;
            const float rr = fmaxf(0.0f, A.Wmax - w) * iR;
            const float r2 = rr * rr, r4 = r2 * r2, r7 = r4 * r2 * rr;
            K = r4 * r4;
            dK_dw = -8.0f * r7 * iR;
        } else {
            K = 0.0f;
            dK_dw = 0.0f;
        }
        dK_dwmax = -dK_dw;
    }
    r.W = K * inv_dpq;
    if (want_grad) {
        r.dmbg = dK_dw * dd * s * A.alpha * 2.0f * inv_dpq;
        r.dsig = dK_dsig * inv_dpq;
        float dal = dK_dw * dd * s * (2.0f * mbg_q - 1.0f);
        if (A.kernel != 0)
            dal += dK_dwmax * A.Imax * (A.alpha > 0.0f ? 1.0f : (A.alpha < 0.0f ? -1.0f : 0.0f));
        r.dal = dal * inv_dpq;
        r.dbe = dK_dw * (dabs - gavg) * fac * inv_dpq;
    }
    return r;
}

__global__ void adj_init_kernel(AdjArgs A, const int32_t *__restrict__ lab, const int *__restrict__ l2c,
                                int maxl, float *m, uint16_t *dist) {
    const size_t XY = (size_t)A.X * A.Y;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < A.N;
         p += (size_t)gridDim.x * blockDim.x) {
        const int l = lab[p];
        int c = A.bg;
        if (l >= 0 && l <= maxl && l2c[l] >= 0) c = l2c[l];
        const uint8_t sc = A.seedc[p];
        if (sc != 0xFF) c = sc;
        for (int k = 0; k < A.C; k++) m[(size_t)k * A.N + p] = (k == c) ? 1.0f : 0.0f;
        const int x = (int)(p % A.X), y = (int)((p / A.X) % A.Y), z = (int)(p / XY);
        bool b = false;
        for (int i = 0; i < A.noff && !b; i++) {
            const int qx = x + A.dx[i], qy = y + A.dy[i], qz = z + A.dz[i];
            if (qx < 0 || qy < 0 || qz < 0 || qx >= A.X || qy >= A.Y || qz >= A.Z) continue;
            b = lab[(size_t)qx + (size_t)qy * A.X + (size_t)qz * XY] != l;
        }
        dist[p] = b ? 0 : 0xFFFF;
    }
}

// One ring of the growing mask: voxels next to ring t-1 join at sweep t.
__global__ void adj_ring_kernel(AdjArgs A, uint16_t *dist, int t) {
    const size_t XY = (size_t)A.X * A.Y;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < A.N;
         p += (size_t)gridDim.x * blockDim.x) {
        if (dist[p] != 0xFFFF) continue;
        const int x = (int)(p % A.X), y = (int)((p / A.X) % A.Y), z = (int)(p / XY);
        for (int i = 0; i < A.noff; i++) {
            const int qx = x + A.dx[i], qy = y + A.dy[i], qz = z + A.dz[i];
            if (qx < 0 || qy < 0 || qz < 0 || qx >= A.X || qy >= A.Y || qz >= A.Z) continue;
            if (dist[(size_t)qx + (size_t)qy * A.X + (size_t)qz * XY] == (uint16_t)(t - 1)) {
                dist[p] = (uint16_t)t;
                break;
            }
        }
    }
}

__global__ void adj_fwd_kernel(AdjArgs A, const float *__restrict__ m, float *__restrict__ mo,
                               float *__restrict__ S_out, float *__restrict__ wmin_out, int t) {
    const size_t XY = (size_t)A.X * A.Y, N = A.N;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        const uint8_t sc = A.seedc[p];
        float S = 0.0f;
        if (sc != 0xFF) {
            for (int k = 0; k < A.C; k++) mo[(size_t)k * N + p] = (k == sc) ? 1.0f : 0.0f;
        } else if (A.dist[p] > t) {
            for (int k = 0; k < A.C; k++) mo[(size_t)k * N + p] = m[(size_t)k * N + p];
        } else {
            const int x = (int)(p % A.X), y = (int)((p / A.X) % A.Y), z = (int)(p / XY);
            const int ip = A.img[p];
            const float gp = A.g ? A.g[p] : 0.0f;
            float num[ADJ_MAX_CLASSES];
            for (int k = 0; k < A.C; k++) num[k] = 0.0f;
            float wmin = 3.0e38f;
            for (int i = 0; i < A.noff; i++) {
                const int qx = x + A.dx[i], qy = y + A.dy[i], qz = z + A.dz[i];
                if (qx < 0 || qy < 0 || qz < 0 || qx >= A.X || qy >= A.Y || qz >= A.Z) continue;
                const size_t q = (size_t)qx + (size_t)qy * A.X + (size_t)qz * XY;
                wmin = fminf(wmin, pair_dist(A, ip, A.img[q], gp, A.g ? A.g[q] : 0.0f,
                                             m[(size_t)A.bg * N + q]));
            }
            if (wmin_out) wmin_out[p] = wmin;
            for (int i = 0; i < A.noff; i++) {
                const int qx = x + A.dx[i], qy = y + A.dy[i], qz = z + A.dz[i];
                if (qx < 0 || qy < 0 || qz < 0 || qx >= A.X || qy >= A.Y || qz >= A.Z) continue;
                const size_t q = (size_t)qx + (size_t)qy * A.X + (size_t)qz * XY;
                const PairW w = pair_weight(A, ip, A.img[q], gp, A.g ? A.g[q] : 0.0f,
                                            m[(size_t)A.bg * N + q], A.inv_dpq[i], wmin, false);
                S += w.W;
                for (int k = 0; k < A.C; k++) num[k] += w.W * m[(size_t)k * N + q];
            }
            for (int k = 0; k < A.C; k++)
                mo[(size_t)k * N + p] = S > 0.0f ? num[k] / S : m[(size_t)k * N + p];
        }
        if (S_out) S_out[p] = S;
    }
}

// Soft-Dice sums: I = sum p t, P = sum p, T = sum t (p = 1 - m_bg).
__global__ void adj_dice_kernel(AdjArgs A, const float *__restrict__ m, const uint8_t *__restrict__ truth,
                                double *sums) {
    double I = 0, P = 0, T = 0;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < A.N;
         p += (size_t)gridDim.x * blockDim.x) {
        const double pr = 1.0 - (double)m[(size_t)A.bg * A.N + p];
        const double tr = truth[p] ? 1.0 : 0.0;
        I += pr * tr;
        P += pr;
        T += tr;
    }
    for (int o = 16; o > 0; o >>= 1) {
        I += __shfl_down_sync(0xffffffffu, I, o);
        P += __shfl_down_sync(0xffffffffu, P, o);
        T += __shfl_down_sync(0xffffffffu, T, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sums[0], I);
        atomicAdd(&sums[1], P);
        atomicAdd(&sums[2], T);
    }
}

// lam_K(p, bg) = -dL/dp_p = (2 t_p den - (2 I + eps)) / den^2; other classes 0.
__global__ void adj_lambda_init_kernel(AdjArgs A, const uint8_t *__restrict__ truth, float *lam,
                                       double den, double num2) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < A.N;
         p += (size_t)gridDim.x * blockDim.x) {
        const double tr = truth[p] ? 1.0 : 0.0;
        for (int k = 0; k < A.C; k++)
            lam[(size_t)k * A.N + p] =
                k == A.bg ? (float)((2.0 * tr * den - num2) / (den * den)) : 0.0f;
    }
}

__global__ void adj_bwd_kernel(AdjArgs A, const float *__restrict__ lam1, float *__restrict__ lam0,
                               const float *__restrict__ m0, const float *__restrict__ m1,
                               const float *__restrict__ S, const float *__restrict__ wmin, int t,
                               double *gacc) {
    const size_t XY = (size_t)A.X * A.Y, N = A.N;
    double gs = 0.0, ga = 0.0, gb = 0.0;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < N;
         q += (size_t)gridDim.x * blockDim.x) {
        float lq[ADJ_MAX_CLASSES];
        const bool qseed = A.seedc[q] != 0xFF;
        const bool qcopy = !qseed && (A.dist[q] > t || !(S[q] > 0.0f));
        for (int k = 0; k < A.C; k++) lq[k] = qcopy ? lam1[(size_t)k * N + q] : 0.0f;
        {
            // seeds get no lambda, but the weights of the pairs that read them still
            // depend on the parameters
            const int x = (int)(q % A.X), y = (int)((q / A.X) % A.Y), z = (int)(q / XY);
            const int iq = A.img[q];
            const float gq = A.g ? A.g[q] : 0.0f;
            const float mbg_q = m0[(size_t)A.bg * N + q];
            for (int i = 0; i < A.noff; i++) {
                // p = q - d_i reads q as its neighbour d_i
                const int px = x - A.dx[i], py = y - A.dy[i], pz = z - A.dz[i];
                if (px < 0 || py < 0 || pz < 0 || px >= A.X || py >= A.Y || pz >= A.Z) continue;
                const size_t p = (size_t)px + (size_t)py * A.X + (size_t)pz * XY;
                if (A.seedc[p] != 0xFF || A.dist[p] > t) continue;
                const float Sp = S[p];
                if (!(Sp > 0.0f)) continue;
                const PairW w = pair_weight(A, A.img[p], iq, A.g ? A.g[p] : 0.0f, gq, mbg_q,
                                            A.inv_dpq[i], wmin[p], true);
                const float invS = 1.0f / Sp;
                float a = 0.0f;
                for (int k = 0; k < A.C; k++) {
                    const float lp = lam1[(size_t)k * N + p];
                    a += lp * (m0[(size_t)k * N + q] - m1[(size_t)k * N + p]);
                    if (!qseed) lq[k] += lp * w.W * invS;
                }
                a *= invS;
                if (!qseed) lq[A.bg] += w.dmbg * a;
                gs += (double)(w.dsig * a);
                ga += (double)(w.dal * a);
                gb += (double)(w.dbe * a);
            }
        }
        for (int k = 0; k < A.C; k++) lam0[(size_t)k * N + q] = lq[k];
    }
    for (int o = 16; o > 0; o >>= 1) {
        gs += __shfl_down_sync(0xffffffffu, gs, o);
        ga += __shfl_down_sync(0xffffffffu, ga, o);
        gb += __shfl_down_sync(0xffffffffu, gb, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&gacc[0], gs);
        atomicAdd(&gacc[1], ga);
        atomicAdd(&gacc[2], gb);
    }
}

// ------------------------------------------------------------------ host ----
int adjoint_run(const AdjointJob &J, cudaStream_t s, int sms, float *work, size_t work_floats,
                void *small, double *loss_out, double *grad_out) {
    const int X = J.X, Y = J.Y, Z = J.Z;
    const size_t N = (size_t)X * Y * Z;
    const int K = J.sweeps;
    const int c = J.checkpoint;
    const int C = J.C;
    AdjArgs A{};
    A.X = X;
    A.Y = Y;
    A.Z = Z;
    A.N = N;
    const Adjacency adj = make_adjacency(J.adjacency == 4 ? 6 : (J.adjacency == 8 ? 26 : J.adjacency));
    A.noff = 0;
    for (int i = 0; i < adj.n; i++) {
        if (Z == 1 && adj.dz[i] != 0) continue;
        A.dx[A.noff] = adj.dx[i];
        A.dy[A.noff] = adj.dy[i];
        A.dz[A.noff] = adj.dz[i];
        A.inv_dpq[A.noff] = 1.0f / sqrtf((float)(adj.dx[i] * adj.dx[i] + adj.dy[i] * adj.dy[i] +
                                                  adj.dz[i] * adj.dz[i]));
        A.noff++;
    }
    A.C = C;
    A.bg = J.bg;
    A.kernel = J.kernel;
    A.sigma = J.sigma;
    A.alpha = J.alpha;
    A.beta = J.beta;
    A.Imax = (float)J.imax;
    A.Wmax = (float)((double)J.imax * (1.0 + fabs((double)J.alpha)));
    A.img = J.img;
    A.g = J.g;
    A.dist = J.dist;
    A.seedc = J.seedc;
    const int nck = (K + c - 1) / c;
    const size_t vol = (size_t)C * N;
    // work: nck checkpoints + (c + 1) segment states + 2 lambdas (C*N each) + c weight sums
    // + c weight scales
    const size_t need = (size_t)(nck + c + 3) * vol + 2 * (size_t)c * N;
    if (work_floats < need) return OIFT_E_OOM;
    float *ck = work;
    float *seg = ck + (size_t)nck * vol;
    float *lam0 = seg + (size_t)(c + 1) * vol;
    float *lam1 = lam0 + vol;
    float *Sseg = lam1 + vol;
    float *Wseg = Sseg + (size_t)c * N;
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((N + 255) / 256, (size_t)sms * 16));
    double *d_sums = (double *)small;  // [0..2] dice sums, [3..5] gradient
    uint16_t *dist = const_cast<uint16_t *>(J.dist);
    // start state (one-hot OIFT labels, seeds one-hot in their class) and the growing mask
    adj_init_kernel<<<blocks, 256, 0, s>>>(A, J.labels0, J.l2c, J.maxl, ck, dist);
    for (int t = 1; t <= K; t++) adj_ring_kernel<<<blocks, 256, 0, s>>>(A, dist, t);
    // ---- forward, keeping every c-th state ----
    float *cur = seg, *nxt = seg + vol;
    if (cudaMemcpyAsync(cur, ck, vol * sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return OIFT_E_CUDA;
    for (int t = 0; t < K; t++) {
        if (t > 0 && t % c == 0 &&
            cudaMemcpyAsync(ck + (size_t)(t / c) * vol, cur, vol * sizeof(float),
                            cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return OIFT_E_CUDA;
        adj_fwd_kernel<<<blocks, 256, 0, s>>>(A, cur, nxt, nullptr, nullptr, t);
        std::swap(cur, nxt);
    }
    if (J.membership_out &&
        cudaMemcpyAsync(J.membership_out, cur, vol * sizeof(float), cudaMemcpyDeviceToDevice, s) !=
            cudaSuccess)
        return OIFT_E_CUDA;
    if (cudaMemsetAsync(d_sums, 0, 6 * sizeof(double), s) != cudaSuccess) return OIFT_E_CUDA;
    adj_dice_kernel<<<blocks, 256, 0, s>>>(A, cur, J.truth, d_sums);
    double hs[3];
    if (cudaMemcpyAsync(hs, d_sums, 3 * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return OIFT_E_CUDA;
    const double den = hs[1] + hs[2] + J.eps, num2 = 2.0 * hs[0] + J.eps;
    *loss_out = 1.0 - num2 / den;
    if (!grad_out) return OIFT_OK;
    // ---- backward, segment by segment ----
    adj_lambda_init_kernel<<<blocks, 256, 0, s>>>(A, J.truth, lam1, den, num2);
    for (int j = nck - 1; j >= 0; j--) {
        const int t0 = j * c, t1 = std::min(t0 + c, K);
        if (cudaMemcpyAsync(seg, ck + (size_t)j * vol, vol * sizeof(float),
                            cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return OIFT_E_CUDA;
        for (int t = t0; t < t1; t++)
            adj_fwd_kernel<<<blocks, 256, 0, s>>>(A, seg + (size_t)(t - t0) * vol,
                                                  seg + (size_t)(t - t0 + 1) * vol,
                                                  Sseg + (size_t)(t - t0) * N,
                                                  Wseg + (size_t)(t - t0) * N, t);
        for (int t = t1 - 1; t >= t0; t--) {
            adj_bwd_kernel<<<blocks, 256, 0, s>>>(A, lam1, lam0, seg + (size_t)(t - t0) * vol,
                                                  seg + (size_t)(t - t0 + 1) * vol,
                                                  Sseg + (size_t)(t - t0) * N,
                                                  Wseg + (size_t)(t - t0) * N, t, d_sums + 3);
            std::swap(lam0, lam1);
        }
    }
    if (cudaGetLastError() != cudaSuccess) return OIFT_E_CUDA;
    if (cudaMemcpyAsync(grad_out, d_sums + 3, 3 * sizeof(double), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return OIFT_E_CUDA;
    return OIFT_OK;
}

size_t adjoint_work_floats(size_t N, int C, int K, int c) {
    const int nck = (K + c - 1) / c;
    return (size_t)(nck + c + 3) * C * N + 2 * (size_t)c * N;
}

}  // namespace oiftb
