// prepost.cu -- the device steps around OIFT + relaxation in the reference CLI
// (oiftrelax.cpp main): intensity shift, Gaussian blur, and the conditional dilation of
// a binary result.  All kernels are HBM-bound integer / FP32 stencils or scans.
#include "kernels.cuh"

namespace oiftb {

// ---------------------------------------------------------------- shift ----
// oiftrelax.cpp:263-268: when min(I) < 0 every voxel gets -min(I) added.
template <typename T>
__global__ void shift_to_i32_kernel(const T *__restrict__ in, int32_t *__restrict__ out,
                                    size_t n, const int *__restrict__ mm) {
    const int lo = mm[0];
    const int add = lo < 0 ? -lo : 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = (int32_t)in[i] + add;
}

template <typename T>
cudaError_t launch_shift_to_i32(const T *in, int32_t *out, size_t n, const int *d_mm, int sms,
                                cudaStream_t s) {
    int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)sms * 16);
    if (blocks < 1) blocks = 1;
    shift_to_i32_kernel<T><<<blocks, 256, 0, s>>>(in, out, n, d_mm);
    return cudaGetLastError();
}

// ----------------------------------------------------------------- blur ----
// Scene32::GaussianBlur (gft_filtering3.cpp:385-397): Convolution (321-346) with the
// normalised SphericalGaussian(R = 1, s = 10, f = 1) kernel (106-126, 72-83) over
// Spheric(1.0): the centre first, then -z, -y, -x, +x, +y, +z.  Neighbours outside the
// volume are skipped without renormalising; the sum is FP32 in that order with separate
// multiply and add; the result is ROUND (gft_common.h:120) evaluated in double.
// One thread per voxel, x fastest: the six neighbour reads of a warp are coalesced rows
// and the +-y / +-z rows are re-read from L2.
template <typename T>
__global__ void gaussian_blur_kernel(const T *__restrict__ in, int32_t *__restrict__ out,
                                     int X, int Y, int Z, float w0, float w1) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= X) return;
    const size_t XY = (size_t)X * Y;
    const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
    float conv = __fmul_rn((float)in[p], w0);
    if (z > 0) conv = __fadd_rn(conv, __fmul_rn((float)in[p - XY], w1));
    if (y > 0) conv = __fadd_rn(conv, __fmul_rn((float)in[p - X], w1));
    if (x > 0) conv = __fadd_rn(conv, __fmul_rn((float)in[p - 1], w1));
    if (x + 1 < X) conv = __fadd_rn(conv, __fmul_rn((float)in[p + 1], w1));
    if (y + 1 < Y) conv = __fadd_rn(conv, __fmul_rn((float)in[p + X], w1));
    if (z + 1 < Z) conv = __fadd_rn(conv, __fmul_rn((float)in[p + XY], w1));
    out[p] = conv < 0.0f ? (int32_t)((double)conv - 0.5) : (int32_t)((double)conv + 0.5);
}

template <typename T>
cudaError_t launch_gaussian_blur(const T *in, int32_t *out, int X, int Y, int Z, float w0,
                                 float w1, cudaStream_t s) {
    if (Y > 65535 || Z > 65535) return cudaErrorInvalidValue;
    dim3 grid((X + 127) / 128, Y, Z);
    gaussian_blur_kernel<T><<<grid, 128, 0, s>>>(in, out, X, Y, Z, w0, w1);
    return cudaGetLastError();
}

// ------------------------------------------------- conditional dilation ----
// oiftrelax.cpp:87-169.  The border is every voxel labelled 0 that has a voxel labelled 1
// within Spheric(radius); the border voxels whose blurred intensity ranks at or below the
// percentile index (ties in address order, as std::stable_sort keeps them) become 1.
//
// On the device: (1) border mask + a 65536-bin histogram of the high half of the
// order-preserving key (I ^ 0x80000000); (2) the host finds the bin of rank k; a second
// histogram of the low half inside that bin gives the exact value v and the count below
// it; (3) per-block counts of border voxels equal to v, (4) after a host prefix over the
// blocks, voxels below v, and the first ones equal to v in address order, are relabelled.

__device__ __forceinline__ uint32_t order_key(int v) { return (uint32_t)v ^ 0x80000000u; }

__global__ void dilation_border_kernel(const int32_t *__restrict__ label,
                                       const int32_t *__restrict__ img, uint8_t *border, int X,
                                       int Y, int Z, const int *__restrict__ off, int noff,
                                       unsigned *hist_hi, unsigned *count) {
    const size_t N = (size_t)X * Y * Z, XY = (size_t)X * Y;
    unsigned local = 0;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        uint8_t b = 0;
        if (label[p] == 0) {
            const int x = (int)(p % X), y = (int)((p / X) % Y), z = (int)(p / XY);
            for (int i = 0; i < noff; i++) {
                const int qx = x + off[3 * i], qy = y + off[3 * i + 1], qz = z + off[3 * i + 2];
                if (qx < 0 || qy < 0 || qz < 0 || qx >= X || qy >= Y || qz >= Z) continue;
                if (label[(size_t)qx + (size_t)qy * X + (size_t)qz * XY] == 1) {
                    b = 1;
                    break;
                }
            }
        }
        border[p] = b;
        if (b) {
            atomicAdd(&hist_hi[order_key(img[p]) >> 16], 1u);
            local++;
        }
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

__global__ void dilation_hist_lo_kernel(const uint8_t *__restrict__ border,
                                        const int32_t *__restrict__ img, size_t N,
                                        uint32_t hi, unsigned *hist_lo) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        if (!border[p]) continue;
        const uint32_t k = order_key(img[p]);
        if ((k >> 16) == hi) atomicAdd(&hist_lo[k & 0xffffu], 1u);
    }
}

// Count of border voxels equal to the pivot in each chunk of `chunk` addresses.
__global__ void dilation_tie_count_kernel(const uint8_t *__restrict__ border,
                                          const int32_t *__restrict__ img, size_t N,
                                          size_t chunk, uint32_t pivot, unsigned *counts) {
    const size_t b0 = (size_t)blockIdx.x * chunk;
    const size_t b1 = min(N, b0 + chunk);
    unsigned c = 0;
    for (size_t p = b0 + threadIdx.x; p < b1; p += blockDim.x)
        c += (border[p] && order_key(img[p]) == pivot) ? 1u : 0u;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    __shared__ unsigned ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += ws[w];
        counts[blockIdx.x] = t;
    }
}

// Relabel: border voxels below the pivot, and pivot-valued ones whose rank among equal
// values (address order) is below `take`.  tie_base[b] = pivot-valued border voxels in the
// chunks before b.  A block walks its chunk in rounds of blockDim addresses, ranking the
// pivot-valued voxels of each round with a block prefix sum.
__global__ void dilation_apply_kernel(const uint8_t *__restrict__ border,
                                      const int32_t *__restrict__ img, int32_t *label, size_t N,
                                      size_t chunk, uint32_t pivot,
                                      const unsigned *__restrict__ tie_base, unsigned take) {
    __shared__ unsigned ws[33];
    const size_t b0 = (size_t)blockIdx.x * chunk;
    const size_t b1 = min(N, b0 + chunk);
    unsigned base = tie_base[blockIdx.x];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (size_t r = b0; r < b1; r += blockDim.x) {
        const size_t p = r + threadIdx.x;
        bool eq = false, lt = false;
        if (p < b1 && border[p]) {
            const uint32_t k = order_key(img[p]);
            eq = k == pivot;
            lt = k < pivot;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, eq);
        if (lane == 0) ws[wid] = __popc(bal);
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned s = 0;
            for (int w = 0; w < nw; w++) {
                const unsigned v = ws[w];
                ws[w] = s;
                s += v;
            }
            ws[32] = s;
        }
        __syncthreads();
        const unsigned rank = base + ws[wid] + __popc(bal & ((1u << lane) - 1u));
        if (lt || (eq && rank < take)) label[p] = 1;
        base += ws[32];
        __syncthreads();
    }
}

template cudaError_t launch_shift_to_i32<int16_t>(const int16_t *, int32_t *, size_t,
                                                  const int *, int, cudaStream_t);
template cudaError_t launch_shift_to_i32<int32_t>(const int32_t *, int32_t *, size_t,
                                                  const int *, int, cudaStream_t);
template cudaError_t launch_gaussian_blur<int16_t>(const int16_t *, int32_t *, int, int, int,
                                                   float, float, cudaStream_t);
template cudaError_t launch_gaussian_blur<int32_t>(const int32_t *, int32_t *, int, int, int,
                                                   float, float, cudaStream_t);

}  // namespace oiftb

namespace oiftb {

// ------------------------------------------------------ coarse-to-fine cascade ----
// experiments/exp_coarse_to_fine.cpp:327-414 on the device.

// Scene32::Subsampling (gft_filtering3.cpp:445-476): coarse voxel v takes the fine voxel
// (v - c/2) * 2 + n/2 (integer halves) when it lies inside, else 0.
__global__ void pyr_subsample_kernel(const int32_t *__restrict__ fine, int32_t *__restrict__ coarse,
                                     int X, int Y, int Z, int cx, int cy, int cz) {
    const size_t cn = (size_t)cx * cy * cz;
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < cn;
         v += (size_t)gridDim.x * blockDim.x) {
        const int vx = (int)(v % cx), vy = (int)((v / cx) % cy), vz = (int)(v / ((size_t)cx * cy));
        const int ux = (vx - cx / 2) * 2 + X / 2, uy = (vy - cy / 2) * 2 + Y / 2,
                  uz = (vz - cz / 2) * 2 + Z / 2;
        const bool in = ux >= 0 && ux < X && uy >= 0 && uy < Y && uz >= 0 && uz < Z;
        coarse[v] = in ? fine[(size_t)ux + (size_t)uy * X + (size_t)uz * X * Y] : 0;
    }
}

// Seeds at (x/2, y/2, z/2); the first seed of the list that lands on a coarse voxel gives
// it its label (first[cq] = smallest seed index).
__global__ void pyr_coarse_first_kernel(const int32_t *__restrict__ seeds, int nseeds, int X,
                                        int Y, int Z, int cx, int cy, int cz, unsigned *first) {
    const size_t N = (size_t)X * Y * Z;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nseeds; i += gridDim.x * blockDim.x) {
        const int p = seeds[i];
        if (p < 0 || (size_t)p >= N) continue;
        const int x = p % X, y = (p / X) % Y, z = (int)(p / ((size_t)X * Y));
        const int qx = x / 2, qy = y / 2, qz = z / 2;
        if (qx >= cx || qy >= cy || qz >= cz) continue;
        atomicMin(&first[(size_t)qx + (size_t)qy * cx + (size_t)qz * cx * cy], (unsigned)i);
    }
}

__global__ void pyr_coarse_labels_kernel(const unsigned *__restrict__ first,
                                         const int32_t *__restrict__ seeds,
                                         const int32_t *__restrict__ fine_label, size_t cn,
                                         int32_t *__restrict__ clab) {
    for (size_t v = blockIdx.x * (size_t)blockDim.x + threadIdx.x; v < cn;
         v += (size_t)gridDim.x * blockDim.x) {
        const unsigned f = first[v];
        clab[v] = f == 0xFFFFFFFFu ? -1 : fine_label[seeds[f]];
    }
}

// Scene32::ScaleLabel(.., none) (gft_scene32.cpp:1145-1161, 1091-1120): fine voxel u takes
// coarse voxel (ix[x], iy[y], iz[z]); the per-axis tables are computed on the host with
// the reference's float / double expression.
__global__ void pyr_upscale_kernel(const int32_t *__restrict__ clab, int32_t *__restrict__ up,
                                   int X, int Y, int Z, int cx, int cy,
                                   const int *__restrict__ ix, const int *__restrict__ iy,
                                   const int *__restrict__ iz) {
    const size_t N = (size_t)X * Y * Z;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(p % X), y = (int)((p / X) % Y), z = (int)(p / ((size_t)X * Y));
        up[p] = clab[(size_t)ix[x] + (size_t)iy[y] * cx + (size_t)iz[z] * cx * cy];
    }
}

// mark_boundary_voxels_nil (exp_coarse_to_fine.cpp:216-249): a labelled voxel with a
// neighbour of another value (NIL included) becomes NIL; out-of-volume neighbours are
// ignored.  off: the adjacency without its centre.
__global__ void pyr_boundary_nil_kernel(const int32_t *__restrict__ lab, int32_t *__restrict__ out,
                                        int X, int Y, int Z, const int *__restrict__ off,
                                        int noff) {
    const size_t N = (size_t)X * Y * Z, XY = (size_t)X * Y;
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        const int l = lab[p];
        int o = l;
        if (l != -1) {
            const int x = (int)(p % X), y = (int)((p / X) % Y), z = (int)(p / XY);
            for (int i = 0; i < noff; i++) {
                const int qx = x + off[3 * i], qy = y + off[3 * i + 1], qz = z + off[3 * i + 2];
                if (qx < 0 || qy < 0 || qz < 0 || qx >= X || qy >= Y || qz >= Z) continue;
                if (lab[(size_t)qx + (size_t)qy * X + (size_t)qz * XY] != l) {
                    o = -1;
                    break;
                }
            }
        }
        out[p] = o;
    }
}

// Fine labels before the second pass: the caller's label where set, else the upscaled
// interior label (exp_coarse_to_fine.cpp:376-383).
__global__ void pyr_merge_kernel(const int32_t *__restrict__ label, const int32_t *__restrict__ up,
                                 int32_t *__restrict__ merged, size_t N) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        const int l = label[p];
        merged[p] = (l == -1) ? up[p] : l;
    }
}

// Every labelled voxel becomes a seed, in address order (build_seeds_from_label,
// exp_coarse_to_fine.cpp:197-212): per-chunk counts, then an ordered scatter.
__global__ void seeds_count_kernel(const int32_t *__restrict__ lab, size_t N, size_t chunk,
                                   unsigned *counts) {
    const size_t b0 = (size_t)blockIdx.x * chunk, b1 = min(N, b0 + chunk);
    unsigned c = 0;
    for (size_t p = b0 + threadIdx.x; p < b1; p += blockDim.x) c += lab[p] != -1;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    __shared__ unsigned ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += ws[w];
        counts[blockIdx.x] = t;
    }
}

__global__ void seeds_scatter_kernel(const int32_t *__restrict__ lab, size_t N, size_t chunk,
                                     const unsigned *__restrict__ base_of, int32_t *seeds,
                                     int32_t *seed_labels) {
    __shared__ unsigned ws[33];
    const size_t b0 = (size_t)blockIdx.x * chunk, b1 = min(N, b0 + chunk);
    unsigned base = base_of[blockIdx.x];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (size_t r = b0; r < b1; r += blockDim.x) {
        const size_t p = r + threadIdx.x;
        const int l = p < b1 ? lab[p] : -1;
        const unsigned bal = __ballot_sync(0xffffffffu, l != -1);
        if (lane == 0) ws[wid] = __popc(bal);
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned s = 0;
            for (int w = 0; w < nw; w++) {
                const unsigned v = ws[w];
                ws[w] = s;
                s += v;
            }
            ws[32] = s;
        }
        __syncthreads();
        if (l != -1) {
            const unsigned pos = base + ws[wid] + __popc(bal & ((1u << lane) - 1u));
            seeds[pos] = (int32_t)p;
            seed_labels[pos] = l < 0 ? 0 : l;
        }
        base += ws[32];
        __syncthreads();
    }
}

}  // namespace oiftb

namespace oiftb {

// ------------------------------------------------------------- Sobel gradient ----
// Scene32::SobelFilter (gft_filtering3.cpp:509-552) over the linear addresses
// [1 + X + XY, N - 1 - X - XY): neighbours by address arithmetic (rows and planes wrap as in
// the reference), three 3x3 difference stencils (1 2 1 / 2 4 2 / 1 2 1), each >> 4, then
// ROUND(sqrtf((a^2 + b^2 + c^2) / 3.0)) with the float sum, the double division and the
// float square root of the C++ expression; every other voxel 0.
template <typename T>
__global__ void sobel_kernel(const T *__restrict__ img, int32_t *__restrict__ out, long long N,
                             long long dy, long long dz) {
    const long long di = 1 + dy + dz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        if (i < di || i >= N - di) {
            out[i] = 0;
            continue;
        }
        int acc0 = 0, acc1 = 0, acc2 = 0;
#pragma unroll
        for (int m = 0; m < 9; m++) {
            const int n0 = m % 3 - 1, n1 = m / 3 - 1;
            const int we = (n0 == 0 ? 2 : 1) * (n1 == 0 ? 2 : 1);
            acc0 += we * ((int)img[i + dz + n0 + dy * n1] - (int)img[i - dz + n0 + dy * n1]);
            acc1 += we * ((int)img[i + 1 + dz * n0 + dy * n1] - (int)img[i - 1 + dz * n0 + dy * n1]);
            acc2 += we * ((int)img[i + dy + n0 + dz * n1] - (int)img[i - dy + n0 + dz * n1]);
        }
        acc0 >>= 4;
        acc1 >>= 4;
        acc2 >>= 4;
        const float f0 = (float)acc0, f1 = (float)acc1, f2 = (float)acc2;
        const float s = __fadd_rn(__fadd_rn(__fmul_rn(f0, f0), __fmul_rn(f1, f1)), __fmul_rn(f2, f2));
        const float q = __double2float_rn(__ddiv_rn((double)s, 3.0));
        const float r = __fsqrt_rn(q);
        out[i] = (int32_t)((double)r + 0.5);
    }
}

// g = g * max(I) / max(g) in 64-bit integers when both maxima are positive
// (exp_gradient_weight.cpp:600-608); mm_img / mm_g hold (min, max) of image and gradient.
__global__ void sobel_normalize_kernel(int32_t *g, long long N, const int *__restrict__ mm_img,
                                       const int *__restrict__ mm_g) {
    const long long wmax = mm_img[1], gmax = mm_g[1];
    if (!(gmax > 0 && wmax > 0)) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x)
        g[i] = (int32_t)((long long)g[i] * wmax / gmax);
}

template <typename T>
cudaError_t launch_sobel_normalized(const T *img, int32_t *g, int X, int Y, int Z,
                                    const int *d_mm_img, int *d_mm_g, int sms, cudaStream_t s) {
    const long long N = (long long)X * Y * Z;
    int blocks = (int)std::min<long long>((N + 255) / 256, (long long)sms * 16);
    if (blocks < 1) blocks = 1;
    sobel_kernel<T><<<blocks, 256, 0, s>>>(img, g, N, (long long)X, (long long)X * Y);
    const int mm_init[2] = {0x7fffffff, (int)0x80000000};
    cudaError_t e = cudaMemcpyAsync(d_mm_g, mm_init, sizeof(mm_init), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    e = launch_minmax<int32_t>(g, (size_t)N, d_mm_g, sms, s);
    if (e != cudaSuccess) return e;
    sobel_normalize_kernel<<<blocks, 256, 0, s>>>(g, N, d_mm_img, d_mm_g);
    return cudaGetLastError();
}

template cudaError_t launch_sobel_normalized<int16_t>(const int16_t *, int32_t *, int, int, int,
                                                      const int *, int *, int, cudaStream_t);
template cudaError_t launch_sobel_normalized<int32_t>(const int32_t *, int32_t *, int, int, int,
                                                      const int *, int *, int, cudaStream_t);

}  // namespace oiftb
