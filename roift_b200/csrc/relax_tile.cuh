// relax_tile.cuh -- device templates of the tile relaxation sweep (see relax.cu).
#pragma once
#include "kernels.cuh"

namespace oiftb {

// ------------------------------------------------------------------------------------
// Tile relaxation with exact skipping.
//
// The reference updates only the mask M_t = (voxels with a differently-labelled
// neighbour) dilated t-1 times (gft_ift.cpp:8757-8771, 8857-8886).  Every voxel outside
// M_t is unchanged by sweep t, so a 32x8x4 tile whose block distance to the tiles that
// hold M_1 exceeds t-1 is skipped: a voxel path of length L moves at most L tiles, so the
// block distance is a lower bound of the voxel distance (Manhattan blocks for 6/4-adj,
// Chebyshev blocks for 26/8-adj).  Skipped tiles keep their one-hot start in both
// ping-pong buffers.  Active tiles are staged with a one-voxel halo in shared memory.
constexpr int RT_X = 32, RT_Y = 8, RT_Z = 4;
constexpr int RH_X = RT_X + 2, RH_Y = RT_Y + 2, RH_Z = RT_Z + 2;
constexpr int RH_N = RH_X * RH_Y * RH_Z;

// Asynchronous 4-byte global -> shared copy (cp.async, cached in L1).
__device__ __forceinline__ void relax_cp_async4(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// Polarity factors of the arcs that end at q: (1 + per_pq / 100, 1 - per_pq / 100), with
// per_pq = per (2 m_bg(q) - 1) (gft_ift.cpp:8804-8811) or sum_k per_k m_k(q) per class
// (9076-9079).  They depend on q alone, so a tile computes them once per staged voxel.
template <int C, bool PERCLASS>
__device__ __forceinline__ float2 relax_polarity_factors(const RelaxArgs &a, const float *sm,
                                                         int i) {
    float per_pq;
    if (PERCLASS) {
        per_pq = 0.0f;
#pragma unroll
        for (int k = 0; k < C; k++) per_pq = __fadd_rn(per_pq, __fmul_rn(a.pcm[k], sm[k * RH_N + i]));
    } else {
        float pbg = sm[i];
#pragma unroll
        for (int k = 1; k < C; k++)
            if (k == a.bg) pbg = sm[k * RH_N + i];
        per_pq = __fmul_rn(a.per, __fsub_rn(__fmul_rn(2.0f, pbg), 1.0f));
    }
    const float d = div100_rn(per_pq);
    return make_float2(__fadd_rn(1.0f, d), __fsub_rn(1.0f, d));
}

// One arc p <- q of the sweep: w = ((Wmax - w_or)^8) / Dpq, in the C++ operation order.
template <int C, bool BLEND>
__device__ __forceinline__ void relax_accumulate(const RelaxArgs &a, int ip, int iq, int gp,
                                                 int gq, const float (&mq)[C], float2 fq,
                                                 float dpq, float &sw, float (&acc)[C]) {
    float w = fabsf((float)(ip - iq));
    if (BLEND)  // wf = alpha |dI| + (1 - alpha)(g_p + g_q) * 0.5f (exp_gradient_weight.cpp:403-405)
        w = __fadd_rn(__fmul_rn(a.alpha, w),
                      __fmul_rn(__fsub_rn(1.0f, a.alpha), __fmul_rn((float)(gp + gq), 0.5f)));
    if (ip > iq)
        w = __fmul_rn(w, fq.x);
    else if (ip < iq)
        w = __fmul_rn(w, fq.y);
    if (BLEND && w < 0.0f) w = 0.0f;
    w = __fsub_rn(a.Wmax, w);
    if (w < 0.0f) w = 0.0f;
    w = __fmul_rn(w, w);
    w = __fmul_rn(w, w);
    w = __fmul_rn(w, w);
    if (dpq != 1.0f) w = __fdiv_rn(w, dpq);
    sw = __fadd_rn(sw, w);
#pragma unroll
    for (int k = 0; k < C; k++) acc[k] = __fadd_rn(acc[k], __fmul_rn(w, mq[k]));
}


// Tiles holding a voxel with a differently-labelled neighbour get distance 0.
template <int C, typename T, bool PERCLASS, int ADJ, bool INTERIOR, bool BLEND>
__device__ __forceinline__ void relax_tile_voxels(const RelaxArgs &a, const float *sm,
                                                  const int *si, const int *sg, const float2 *sf,
                                                  float *__restrict__ mout,
                                                  const uint8_t *__restrict__ seedc, int x,
                                                  int y, int z0, int lx, int ly) {
    const int X = a.X, Y = a.Y, Z = a.Z;
    const size_t N = a.N, XY = (size_t)X * Y;
#pragma unroll
    for (int lz = 0; lz < RT_Z; lz++) {
        const int z = z0 + lz;
        if (z >= Z) break;
        const int hc = (lx + 1) + (ly + 1) * RH_X + (lz + 1) * RH_X * RH_Y;
        const int ip = si[hc];
        float acc[C];
#pragma unroll
        for (int k = 0; k < C; k++) acc[k] = 0.0f;
        float sw = 0.0f;
#pragma unroll
        for (int i = 0; i < (ADJ == 6 ? 6 : 26); i++) {
            int ddx, ddy, ddz;
            if (ADJ == 6) {
                ddx = (i == 2) ? -1 : (i == 3) ? 1 : 0;
                ddy = (i == 1) ? -1 : (i == 4) ? 1 : 0;
                ddz = (i == 0) ? -1 : (i == 5) ? 1 : 0;
            } else {
                const int j = i < 13 ? i : i + 1;  // the 3x3x3 cube without its centre
                ddx = j % 3 - 1;
                ddy = (j / 3) % 3 - 1;
                ddz = j / 9 - 1;
            }
            if (!INTERIOR) {
                const int qx = x + ddx, qy = y + ddy, qz = z + ddz;
                if (qx < 0 || qx >= X || qy < 0 || qy >= Y || qz < 0 || qz >= Z) continue;
            }
            const int hq = hc + ddx + ddy * RH_X + ddz * RH_X * RH_Y;
            float mq[C];
#pragma unroll
            for (int k = 0; k < C; k++) mq[k] = sm[k * RH_N + hq];
            const float dpq = (ADJ == 6) ? 1.0f : a.dpq[i];
            relax_accumulate<C, BLEND>(a, ip, si[hq], BLEND ? sg[hc] : 0, BLEND ? sg[hq] : 0, mq,
                                       sf[hq], dpq, sw, acc);
        }
        const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
        float out[C];
        if (sw > 0.0f) {
#pragma unroll
            for (int k = 0; k < C; k++) out[k] = __fdiv_rn(acc[k], sw);
        } else {
#pragma unroll
            for (int k = 0; k < C; k++) out[k] = sm[k * RH_N + hc];
        }
        const uint8_t sc = __ldg(&seedc[p]);
        if (sc != 0xFF) {
#pragma unroll
            for (int k = 0; k < C; k++) out[k] = (k == sc) ? 1.0f : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < C; k++) mout[(size_t)k * N + p] = out[k];
    }
}

// Blocks per SM the tile sweep is compiled for: with one or two classes (and no gradient
// halo) five blocks' shared memory fits an SM, and asking for them caps the kernel at 48
// registers without spills; larger variants are limited by shared memory first.
constexpr int relax_min_blocks(int classes, bool blend) { return (!blend && classes <= 2) ? 5 : 1; }

template <int C, typename T, bool PERCLASS, int ADJ, bool BLEND>
__global__ void __launch_bounds__(256, relax_min_blocks(C, BLEND)) relax_tile_kernel(const float *__restrict__ min_,
                                                         float *__restrict__ mout,
                                                         const T *__restrict__ img,
                                                         const uint8_t *__restrict__ seedc,
                                                         const uint16_t *__restrict__ tdist,
                                                         int sweep, RelaxArgs a, int ntx,
                                                         int nty) {
    const int t = blockIdx.x;
    if ((int)tdist[t] > sweep - 1) return;  // provably unchanged at this sweep
    extern __shared__ __align__(16) unsigned char rsm[];
    float *sm = reinterpret_cast<float *>(rsm);          // [C][RH_Z][RH_Y][RH_X]
    int *si = reinterpret_cast<int *>(sm + C * RH_N);    // [RH_Z][RH_Y][RH_X]
    int *sg = si + RH_N;                                 // gradient halo (BLEND only)
    float2 *sf = reinterpret_cast<float2 *>(si + (BLEND ? 2 : 1) * RH_N);  // polarity factors
    const int X = a.X, Y = a.Y, Z = a.Z;
    const size_t N = a.N, XY = (size_t)X * Y;
    const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
    const int x0 = tx * RT_X, y0 = ty * RT_Y, z0 = tz * RT_Z;
    const int tid = threadIdx.x + threadIdx.y * 32;
    // memberships (and the gradient) as asynchronous 4-byte copies, the image through
    // registers: every load of the halo is in flight before the first wait
    constexpr int NIT = (RH_N + 255) / 256;
    int iv[NIT];
#pragma unroll
    for (int j = 0; j < NIT; j++) {
        const int i = tid + 256 * j;
        const int hx = i % RH_X, hy = (i / RH_X) % RH_Y, hz = i / (RH_X * RH_Y);
        const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
        if (i < RH_N && gx >= 0 && gx < X && gy >= 0 && gy < Y && gz >= 0 && gz < Z) {
            const size_t g = (size_t)gx + (size_t)gy * X + (size_t)gz * XY;
#pragma unroll
            for (int k = 0; k < C; k++) relax_cp_async4(&sm[k * RH_N + i], &min_[(size_t)k * N + g]);
            if (BLEND) relax_cp_async4(&sg[i], &a.gmap[g]);
            iv[j] = (int)__ldg(&img[g]);
        }
    }
#pragma unroll
    for (int j = 0; j < NIT; j++) {
        const int i = tid + 256 * j;
        const int hx = i % RH_X, hy = (i / RH_X) % RH_Y, hz = i / (RH_X * RH_Y);
        const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
        if (i < RH_N && gx >= 0 && gx < X && gy >= 0 && gy < Y && gz >= 0 && gz < Z) si[i] = iv[j];
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    // each thread reads back only the staged voxels it wrote itself
    for (int i = tid; i < RH_N; i += 256) {
        const int hx = i % RH_X, hy = (i / RH_X) % RH_Y, hz = i / (RH_X * RH_Y);
        const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
        if (gx >= 0 && gx < X && gy >= 0 && gy < Y && gz >= 0 && gz < Z)
            sf[i] = relax_polarity_factors<C, PERCLASS>(a, sm, i);
    }
    __syncthreads();
    const int lx = threadIdx.x, ly = threadIdx.y;
    const int x = x0 + lx, y = y0 + ly;
    if (x >= X || y >= Y) return;
    // every neighbour of every voxel of an interior tile lies in the volume
    const bool interior = x0 >= 1 && x0 + RT_X < X && y0 >= 1 && y0 + RT_Y < Y && z0 >= 1 &&
                          z0 + RT_Z < Z;
    if (interior)
        relax_tile_voxels<C, T, PERCLASS, ADJ, true, BLEND>(a, sm, si, sg, sf, mout, seedc, x, y, z0,
                                                            lx, ly);
    else
        relax_tile_voxels<C, T, PERCLASS, ADJ, false, BLEND>(a, sm, si, sg, sf, mout, seedc, x, y, z0,
                                                             lx, ly);
}

// Launches the tile sweep for C classes; one explicit instantiation per translation unit.
template <int C>
cudaError_t launch_relax_tiles_c(const float *in, float *out, const void *img, bool img32,
                                 const uint8_t *seedc, const uint16_t *tdist, int sweep,
                                 const RelaxArgs &a, bool perclass, int ntiles, int ntx, int nty,
                                 cudaStream_t s);

}  // namespace oiftb
