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

// Base weight of an edge with intensity difference d, capped at a.cap (the cap counted).
__device__ __forceinline__ int edge_base(const BuildArgs &a, int d, unsigned long long &nclamp) {
    const int ad = d < 0 ? -d : d;
    int b;
    if (a.mode == OIFT_W_RBF_Q)
        b = a.lut[ad < a.lut_len ? ad : a.lut_len - 1];
    else if (a.mode == OIFT_W_IMAGEGRAPH)
        b = ad + 1;  // ByEuclideanDistance, gft_imagegraph.cpp:35
    else
        b = ad;
    if (b > a.cap) {
        b = a.cap;
        nclamp++;
    }
    return b;
}

// The same builder for the 6 / 4 neighbourhoods with each OIFT tile's image box staged in
// shared memory by one TMA load: CTA t builds the +x / +y / +z edges of warp tile t
// (32 x TY x TZ voxels) from the box x0 .. x0+BX-1, y0 .. y0+TY, z0 .. z0+TZ (the tile and
// its one-voxel halo on the + sides; x0 is 16-byte aligned, BX rounds the 33 columns up to
// 16-byte rows).  Box positions outside the volume read as zero and are not used: an edge
// to a voxel outside the volume gets code 0, as in build_weights_kernel.  Writes the
// tile-major copy (one coalesced 64-byte row per warp and plane) and, when asked, the
// plane-major planes.  The image box lands on an mbarrier with a bounded wait; a box that
// does not land sets *a.tma_err and the CTA leaves after one more bounded wait.
template <typename T, int TY, int TZ>
__global__ void __launch_bounds__(256) build_weights_tma_kernel(const __grid_constant__ CUtensorMap imap,
                                                                uint16_t *__restrict__ W,
                                                                BuildArgs a) {
    constexpr int BX = sizeof(T) == 2 ? 40 : 36, BY = TY + 1, BZ = TZ + 1;
    static_assert(TY * TZ == 32, "a warp tile has 32 rows");
    __shared__ __align__(128) T sim[BZ][BY][BX];
    __shared__ __align__(8) unsigned long long mbar;
    const int t = blockIdx.x;
    const int tx = t % a.tntx, ty = (t / a.tntx) % a.tnty, tz = t / (a.tntx * a.tnty);
    const int x0 = tx * 32, y0 = ty * TY, z0 = tz * TZ;
    const int tid = threadIdx.x;
    const unsigned bar = (unsigned)__cvta_generic_to_shared(&mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
                     "r"((unsigned)sizeof(sim))
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"((unsigned)__cvta_generic_to_shared(&sim[0][0][0])),
            "l"(&imap), "r"(x0), "r"(y0), "r"(z0), "r"(bar)
            : "memory");
    }
    auto landed = [&]() -> bool {
        for (long long i = 0; i < (1ll << 24); i++) {  // about a second
            unsigned ok;
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                " selp.u32 %0, 1, 0, p;\n}\n"
                : "=r"(ok)
                : "r"(bar), "r"(0u)
                : "memory");
            if (ok) return true;
        }
        return false;
    };
    if (!landed()) {
        if (tid == 0) atomicExch(a.tma_err, 1);
        landed();
        return;
    }
    const int X = a.X, Y = a.Y, Z = a.Z;
    const size_t N = (size_t)X * Y * Z, XY = (size_t)X * Y;
    const int lx = tid & 31, w = tid >> 5;
    unsigned long long nclamp = 0;
#pragma unroll
    for (int rr = 0; rr < 4; rr++) {
        const int r = w + 8 * rr;
        const int yl = r % TY, zl = r / TY;
        const int x = x0 + lx, y = y0 + yl, z = z0 + zl;
        if (x >= X || y >= Y || z >= Z) continue;
        const int ip = (int)sim[zl][yl][lx];
        const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            if (k >= a.planes) break;
            const bool ok = k == 0 ? x + 1 < X : k == 1 ? y + 1 < Y : z + 1 < Z;
            uint16_t code = 0;
            if (ok) {
                const int iq = k == 0 ? (int)sim[zl][yl][lx + 1]
                                      : k == 1 ? (int)sim[zl][yl + 1][lx] : (int)sim[zl + 1][yl][lx];
                const int d = ip - iq;
                code = (uint16_t)(edge_base(a, d, nclamp) | (d > 0 ? 0x8000 : 0) | (d < 0 ? 0x4000 : 0));
            }
            if (a.planes_out) W[(size_t)k * N + p] = code;
            a.Wt[((size_t)t * 3 + k) * 1024 + r * 32 + lx] = code;
        }
    }
    for (int o = 16; o > 0; o >>= 1) nclamp += __shfl_down_sync(0xffffffffu, nclamp, o);
    if ((tid & 31) == 0 && nclamp) atomicAdd(a.clamped, nclamp);
}

template <typename T>
cudaError_t launch_build_weights(const T *img, uint16_t *W, const BuildArgs &a, int sms,
                                 cudaStream_t s) {
    // the tile-major copy of the 6 / 4 OIFT tiles, staged by TMA when the rows allow it
    const bool unit_offsets = a.planes >= 1 && a.planes <= 3 &&
                              (a.planes < 1 || (a.dx[0] == 1 && a.dy[0] == 0 && a.dz[0] == 0)) &&
                              (a.planes < 2 || (a.dx[1] == 0 && a.dy[1] == 1 && a.dz[1] == 0)) &&
                              (a.planes < 3 || (a.dx[2] == 0 && a.dy[2] == 0 && a.dz[2] == 1));
    const bool tile84 = a.tty == 8 && a.ttz == 4, tile321 = a.tty == 32 && a.ttz == 1;
    if (a.Wt && a.tma_err && unit_offsets && a.mode != OIFT_W_BLEND_Q && (tile84 || tile321)) {
        constexpr int BX = sizeof(T) == 2 ? 40 : 36;
        CUtensorMap imap;
        if (image_tma_encode(&imap, img, sizeof(T) == 4, a.X, a.Y, a.Z, BX, a.tty + 1, a.ttz + 1)) {
            const int ntiles = a.tntx * a.tnty * ((a.Z + a.ttz - 1) / a.ttz);
            if (tile84)
                build_weights_tma_kernel<T, 8, 4><<<ntiles, 256, 0, s>>>(imap, W, a);
            else
                build_weights_tma_kernel<T, 32, 1><<<ntiles, 256, 0, s>>>(imap, W, a);
            return cudaGetLastError();
        }
    }
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
