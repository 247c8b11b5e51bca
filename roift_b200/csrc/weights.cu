// weights.cu -- arc-weight builder (row a1-a3) and intensity range reduction.
//
// One thread builds the P positive-direction edges of 8 consecutive voxels along x.
// Loads of I_p and of the +x/+y/+z neighbours are coalesced rows of the int16/int32
// image; each plane is written with 16-byte stores when the row allows it.
//
// Base weights (bits 0..13 of the edge code):
//   GRAD    |I_p - I_q|                          (gft/src/gft_ift.cpp:965, gft_graph.cpp:148)
//   GRAD_Q  min(|I_p - I_q|, wq), clamp counted  (uint16 [0,wq] quantiser of the workloads)
//   RBF_Q   lut[|I_p - I_q|], lut = floor(wq(1 - exp(-d^2/2s^2)) + 0.5) built on the host
//   BLEND_Q (int)(a|dI| + (1-a)(g_p + g_q)*0.5f) (experiments/exp_gradient_weight.cpp:244-247)
// Orientation bits: bit 15 = I_p > I_q, bit 14 = I_p < I_q.
#include "kernels.cuh"

namespace oiftb {


template <typename T>
__global__ void __launch_bounds__(256) build_weights_kernel(const T *__restrict__ img,
                                                            uint16_t *__restrict__ W,
                                                            BuildArgs a) {
    const int X = a.X, Y = a.Y, Z = a.Z;
    const size_t N = (size_t)X * Y * Z;
    const int xg = (X + 7) / 8;
    const size_t ngroups = (size_t)xg * Y * Z;
    unsigned long long nclamp = 0;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < ngroups;
         g += (size_t)gridDim.x * blockDim.x) {
        int x0 = (int)(g % xg) * 8;
        size_t rest = g / xg;
        int y = (int)(rest % Y), z = (int)(rest / Y);
        size_t prow = (size_t)y * X + (size_t)z * X * Y;
        int ip[8];
#pragma unroll
        for (int i = 0; i < 8; i++) ip[i] = (x0 + i < X) ? (int)img[prow + x0 + i] : 0;
        for (int k = 0; k < a.planes; k++) {
            int dx = a.dx[k], dy = a.dy[k], dz = a.dz[k];
            int qy = y + dy, qz = z + dz;
            bool rowok = qy >= 0 && qy < Y && qz >= 0 && qz < Z;
            size_t qrow = (size_t)qy * X + (size_t)qz * X * Y;
            uint16_t code[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                int x = x0 + i, qx = x + dx;
                code[i] = 0;
                if (x < X && rowok && qx >= 0 && qx < X) {
                    int iq = (int)img[qrow + qx];
                    int d = ip[i] - iq;
                    int ad = d < 0 ? -d : d;
                    int b;
                    if (a.mode == OIFT_W_RBF_Q) {
                        b = a.lut[ad < a.lut_len ? ad : a.lut_len - 1];
                    } else if (a.mode == OIFT_W_BLEND_Q) {
                        float gavg = (float)(a.grad[prow + x] + a.grad[qrow + qx]) * 0.5f;
                        float wf = __fadd_rn(__fmul_rn(a.blend_a, (float)ad),
                                             __fmul_rn(__fsub_rn(1.0f, a.blend_a), gavg));
                        b = (int)wf;
                        if (b < 0) b = 0;
                    } else if (a.mode == OIFT_W_IMAGEGRAPH) {
                        b = ad + 1;  // ByEuclideanDistance, gft_imagegraph.cpp:35
                    } else {
                        b = ad;
                    }
                    if (b > a.cap) {
                        b = a.cap;
                        nclamp++;
                    }
                    code[i] = (uint16_t)(b | (d > 0 ? 0x8000 : 0) | (d < 0 ? 0x4000 : 0));
                }
            }
            uint16_t *dst = W + (size_t)k * N + prow + x0;
            uint4 v;
            v.x = code[0] | ((uint32_t)code[1] << 16);
            v.y = code[2] | ((uint32_t)code[3] << 16);
            v.z = code[4] | ((uint32_t)code[5] << 16);
            v.w = code[6] | ((uint32_t)code[7] << 16);
            if (!a.planes_out) {
            } else if (x0 + 8 <= X && (((uintptr_t)dst) & 15) == 0) {
                *reinterpret_cast<uint4 *>(dst) = v;
            } else {
                for (int i = 0; i < 8 && x0 + i < X; i++) dst[i] = code[i];
            }
            if (a.Wt && k < 3) {  // the same 8 codes in the tile-major copy (16-byte aligned)
                const size_t t = (size_t)(x0 >> 5) + (size_t)(y / a.tty) * a.tntx +
                                 (size_t)(z / a.ttz) * a.tntx * a.tnty;
                const int r = (y % a.tty) + (z % a.ttz) * a.tty;
                *reinterpret_cast<uint4 *>(a.Wt + (t * 3 + k) * 1024 + r * 32 + (x0 & 31)) = v;
            }
        }
    }
    // warp-aggregated clamp count
    for (int o = 16; o > 0; o >>= 1) nclamp += __shfl_down_sync(0xffffffffu, nclamp, o);
    if ((threadIdx.x & 31) == 0 && nclamp) atomicAdd(a.clamped, nclamp);
}

template <typename T>
__global__ void minmax_kernel(const T *__restrict__ img, size_t n, int *mm) {
    int lo = 0x7fffffff, hi = (int)0x80000000;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        int v = (int)img[i];
        lo = min(lo, v);
        hi = max(hi, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_down_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_down_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&mm[0], lo);
        atomicMax(&mm[1], hi);
    }
}

template <typename T>
cudaError_t launch_build_weights(const T *img, uint16_t *W, const BuildArgs &a, int sms,
                                 cudaStream_t s) {
    size_t groups = (size_t)((a.X + 7) / 8) * a.Y * a.Z;
    int blocks = (int)((groups + 255) / 256);
    int cap = sms * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    build_weights_kernel<T><<<blocks, 256, 0, s>>>(img, W, a);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_minmax(const T *img, size_t n, int *mm, int sms, cudaStream_t s) {
    int blocks = (int)((n + 255) / 256);
    if (blocks > sms * 8) blocks = sms * 8;
    if (blocks < 1) blocks = 1;
    minmax_kernel<T><<<blocks, 256, 0, s>>>(img, n, mm);
    return cudaGetLastError();
}

template cudaError_t launch_build_weights<int16_t>(const int16_t *, uint16_t *,
                                                   const BuildArgs &, int, cudaStream_t);
template cudaError_t launch_build_weights<int32_t>(const int32_t *, uint16_t *,
                                                   const BuildArgs &, int, cudaStream_t);
template cudaError_t launch_minmax<int16_t>(const int16_t *, size_t, int *, int, cudaStream_t);
template cudaError_t launch_minmax<int32_t>(const int32_t *, size_t, int *, int, cudaStream_t);

}  // namespace oiftb
