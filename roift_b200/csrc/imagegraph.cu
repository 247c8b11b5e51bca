// imagegraph.cu -- relaxation of the oriented 2D image graph (ORelax_1(sImageGraph),
// gft/src/gft_ift.cpp:7683-7847) after the OIFT of OIFT_W_IMAGEGRAPH.
//
// State: one FP32 membership per pixel (two buffers), a uint16 ring index per pixel and a
// seed flag.  The reference updates the mask M_t: the pixels with a differently-labelled
// neighbour, dilated once after every sweep but the last.  ring[p] = the sweep index at
// which p joins the mask minus one (0 for M_1, 0xFFFF while outside), so sweep t updates
// the pixels with ring <= t-1 and, when another sweep follows, marks their unmarked
// neighbours with t.  A pixel being marked is only ever read by the test ring <= t-1,
// which both its old value (0xFFFF) and its new one (t) fail, so marking in place is
// race-free.  Seeds keep label / Imax, the value the reference re-imposes after every
// sweep.
#include <algorithm>
#include <climits>
#include <cmath>

#include "kernels.cuh"

namespace oiftb {

// Circular(1.0) and Circular(1.5) offsets in the reference order (gft/src/gft_adjrel.cpp:
// 119-148): raster order over dy, then dx.
__constant__ int c_igdx[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
__constant__ int c_igdy[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
__constant__ int c_ig4[4] = {1, 3, 4, 6};  // the 4 face offsets among the 8

__device__ __forceinline__ int ig_offset(bool adj8, int i) { return adj8 ? i : c_ig4[i]; }

// n_link of the arc a -> b seen from a (Orient2Digraph, gft/src/gft_imagegraph.cpp:
// 981-1016), with fpos = 1.0 + alpha and fneg = 1.0 - alpha.
__device__ __forceinline__ int ig_link(int ia, int ib, double fpos, double fneg) {
    const uint32_t val = (uint32_t)abs(ia - ib) + 1u;
    if (ia > ib) return round_weight(val, fpos);
    if (ia < ib) return round_weight(val, fneg);
    return (int)val;
}

template <typename T>
__global__ void ig_edge_max_kernel(const T *__restrict__ img, int X, int Y, bool adj8,
                                   int *dmax) {
    const size_t N = (size_t)X * Y;
    int m = -1;  // -1: no in-image arc seen
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % X), y = (int)(p / X);
        const int ip = (int)img[p];
        for (int i = 0; i < (adj8 ? 8 : 4); i++) {
            const int o = ig_offset(adj8, i);
            const int qx = x + c_igdx[o], qy = y + c_igdy[o];
            if (qx < 0 || qx >= X || qy < 0 || qy >= Y) continue;
            const int d = abs(ip - (int)img[(size_t)qx + (size_t)qy * X]);
            m = d > m ? d : m;
        }
    }
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(dmax, m);
}

__global__ void ig_label_max_kernel(const int32_t *__restrict__ lab, size_t N, int *lmax) {
    int m = INT_MIN;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x)
        m = max(m, lab[p]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(lmax, m);
}

// m = label / Imax in float (gft_ift.cpp:7718); ring 0 where a neighbour's label differs
// (7719-7735).
__global__ void ig_init_kernel(const int32_t *__restrict__ lab, int X, int Y, bool adj8,
                               const int *__restrict__ d_lmax, float *__restrict__ m,
                               uint16_t *__restrict__ ring, uint8_t *__restrict__ seedf) {
    const size_t N = (size_t)X * Y;
    const float imax = (float)*d_lmax;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % X), y = (int)(p / X);
        const int lp = lab[p];
        m[p] = __fdiv_rn((float)lp, imax);
        uint16_t r = 0xFFFF;
        for (int i = 0; i < (adj8 ? 8 : 4); i++) {
            const int o = ig_offset(adj8, i);
            const int qx = x + c_igdx[o], qy = y + c_igdy[o];
            if (qx < 0 || qx >= X || qy < 0 || qy >= Y) continue;
            if (lab[(size_t)qx + (size_t)qy * X] != lp) {
                r = 0;
                break;
            }
        }
        ring[p] = r;
        seedf[p] = 0;
    }
}

__global__ void ig_seed_kernel(const int32_t *__restrict__ seeds, int nseeds, size_t N,
                               uint8_t *__restrict__ seedf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nseeds && seeds[i] >= 0 && (size_t)seeds[i] < N) seedf[seeds[i]] = 1;
}

// Sweep t (1-based), gft_ift.cpp:7737-7800: a mask pixel takes sum(w m_q) / sum(w) with
// w = (Wmax - n_link)^8, n_link = the arc p -> q when m_q < 0.5, else q -> p; every
// operation rounds to nearest in the C++ order.  grow: mark the next ring (7803-7833).
template <typename T>
__global__ void ig_sweep_kernel(const float *__restrict__ min_, float *__restrict__ mout,
                                const T *__restrict__ img, int X, int Y, bool adj8,
                                uint16_t *ring, const uint8_t *__restrict__ seedf, int t,
                                bool grow, float wmax, double fpos, double fneg) {
    const size_t N = (size_t)X * Y;
    const uint16_t tm1 = (uint16_t)(t - 1);
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % X), y = (int)(p / X);
        const uint16_t rp = ring[p];
        float out = min_[p];
        if (rp <= tm1 && !seedf[p]) {
            const int ip = (int)img[p];
            float acc = 0.0f, sw = 0.0f;
            for (int i = 0; i < (adj8 ? 8 : 4); i++) {
                const int o = ig_offset(adj8, i);
                const int qx = x + c_igdx[o], qy = y + c_igdy[o];
                if (qx < 0 || qx >= X || qy < 0 || qy >= Y) continue;
                const size_t q = (size_t)qx + (size_t)qy * X;
                const float mq = min_[q];
                const int iq = (int)img[q];
                const int nl = (mq < 0.5f) ? ig_link(ip, iq, fpos, fneg) : ig_link(iq, ip, fpos, fneg);
                float w = __fsub_rn(wmax, (float)nl);
                w = __fmul_rn(w, w);
                w = __fmul_rn(w, w);
                w = __fmul_rn(w, w);
                sw = __fadd_rn(sw, w);
                acc = __fadd_rn(acc, __fmul_rn(w, mq));
            }
            out = __fdiv_rn(acc, sw);
        }
        mout[p] = out;
        if (grow && rp == 0xFFFF) {
            for (int i = 0; i < (adj8 ? 8 : 4); i++) {
                const int o = ig_offset(adj8, i);
                const int qx = x + c_igdx[o], qy = y + c_igdy[o];
                if (qx < 0 || qx >= X || qy < 0 || qy >= Y) continue;
                if (ring[(size_t)qx + (size_t)qy * X] <= tm1) {
                    ring[p] = (uint16_t)t;
                    break;
                }
            }
        }
    }
}

// label = 0 where m < 0.5, else 1 (NaN included), gft_ift.cpp:7838-7844.
__global__ void ig_final_kernel(const float *__restrict__ m, size_t N, int32_t *label,
                                uint8_t *mask) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        const int l = (m[p] < 0.5f) ? 0 : 1;
        if (label) label[p] = l;
        if (mask) mask[p] = (uint8_t)l;
    }
}

double ig_wmax(int dmax, float per) {
    if (dmax < 0) return 0.0;  // no arcs
    if (dmax == 0) return 1.0;
    const float alpha = (float)((double)per / 100.0);
    const double f = 1.0 + (double)std::fabs(alpha);
    return (double)round_weight((uint32_t)dmax + 1u, f);
}

template <typename T>
int ig_relax_run(const IgRelax &R, const T *img, cudaStream_t s, int sms, int *kernels) {
    const int X = R.X, Y = R.Y;
    const size_t N = (size_t)X * Y;
    const bool adj8 = R.adjacency == 8;
    const int blocks = (int)std::min<size_t>((N + 255) / 256, (size_t)sms * 8);
    int init[2] = {-1, INT_MIN};
    if (cudaMemcpyAsync(R.small, init, sizeof(init), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return OIFT_E_CUDA;
    ig_edge_max_kernel<T><<<blocks, 256, 0, s>>>(img, X, Y, adj8, R.small);
    ig_label_max_kernel<<<blocks, 256, 0, s>>>(R.olabel, N, R.small + 1);
    int h[2];
    if (cudaMemcpyAsync(h, R.small, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return OIFT_E_CUDA;
    const float wmax = (float)ig_wmax(h[0], R.per);
    const float alpha = (float)((double)R.per / 100.0);
    const double fpos = 1.0 + (double)alpha, fneg = 1.0 - (double)alpha;
    float *m0 = R.m0, *m1 = R.m1;
    ig_init_kernel<<<blocks, 256, 0, s>>>(R.olabel, X, Y, adj8, R.small + 1, m0, R.ring, R.seedf);
    if (R.nseeds > 0)
        ig_seed_kernel<<<(R.nseeds + 255) / 256, 256, 0, s>>>(R.seeds, R.nseeds, N, R.seedf);
    if (R.ev_begin) cudaEventRecord(R.ev_begin, s);
    for (int t = 1; t <= R.sweeps; t++) {
        ig_sweep_kernel<T><<<blocks, 256, 0, s>>>(m0, m1, img, X, Y, adj8, R.ring, R.seedf, t,
                                                   t < R.sweeps, wmax, fpos, fneg);
        std::swap(m0, m1);
    }
    if (R.ev_end) cudaEventRecord(R.ev_end, s);
    if (R.label || R.mask) ig_final_kernel<<<blocks, 256, 0, s>>>(m0, N, R.label, R.mask);
    if (R.membership &&
        cudaMemcpyAsync(R.membership, m0, N * sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return OIFT_E_CUDA;
    if (kernels) *kernels = 4 + R.sweeps + ((R.label || R.mask) ? 1 : 0) + (R.nseeds > 0 ? 1 : 0);
    return cudaGetLastError() == cudaSuccess ? OIFT_OK : OIFT_E_CUDA;
}

template int ig_relax_run<int16_t>(const IgRelax &, const int16_t *, cudaStream_t, int, int *);
template int ig_relax_run<int32_t>(const IgRelax &, const int32_t *, cudaStream_t, int, int *);

}  // namespace oiftb
