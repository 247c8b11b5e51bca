// relax_tile.cuh -- device templates of the tile relaxation sweep (see relax.cu).
#pragma once
#include <cuda.h>

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
    if (BLEND) {
        if (ip > iq)
            w = __fmul_rn(w, fq.x);
        else if (ip < iq)
            w = __fmul_rn(w, fq.y);
    } else {
        // with equal intensities w is 0 and stays 0 (or -0) whatever the factor, and
        // Wmax - w below is then Wmax either way: one select instead of two tests
        w = __fmul_rn(w, ip > iq ? fq.x : fq.y);
    }
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

// ------------------------------------------------------------------------------------
// The same sweep with the tile's halo staged by the tensor-memory accelerator: one
// cp.async.bulk.tensor load brings the C membership planes of the halo box and one the
// image box, both completing on a shared-memory mbarrier, in place of one 4-byte copy per
// staged voxel and class with its address arithmetic.  A TMA box must start on a 16-byte
// boundary along x, so the membership box spans x0-4 .. x0+35 (40 floats) and the int16
// image box x0-8 .. x0+39 (48 values; int32: 40 from x0-4); y and z span the one-voxel halo.
// Box positions outside the volume read as zero and are never used.  Needs X % 8 == 0
// (int16) or X % 4 == 0 (int32) so every row of the planes starts 16-byte aligned.
constexpr int RB_X = 40, RB_Y = RT_Y + 2, RB_Z = RT_Z + 2;  // membership box
constexpr int RB_N = RB_X * RB_Y * RB_Z;
constexpr int RB_OFF = 4;                                     // x0 - RB_OFF is its first column
template <typename T>
struct RelaxImgBox {  // image box: 48 int16 or 40 int32 columns, aligned the same way
    static constexpr int X = sizeof(T) == 2 ? 48 : 40;
    static constexpr int OFF = sizeof(T) == 2 ? 8 : 4;
    static constexpr int N = X * RB_Y * RB_Z;
    static constexpr int BYTES = N * (int)sizeof(T);
};
// Polls of the mbarrier before the tile gives up (a TMA load that never lands): about a
// second; the tile then records the failure for the host and leaves.
constexpr long long RELAX_TMA_SPIN_LIMIT = 1ll << 24;

__device__ __forceinline__ unsigned relax_smem_addr(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ bool relax_mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(relax_smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool relax_mbar_wait_bounded(unsigned long long *bar, unsigned parity,
                                                        long long limit) {
    for (long long i = 0; i < limit; i++)
        if (relax_mbar_try_wait(bar, parity)) return true;
    return false;
}

// The polarity factors (1 + d, 1 - d), d = per_pq / 100, of a voxel with memberships mk
// (gft_ift.cpp:8800-8806; per-class form 9076-9079).
template <int C, bool PERCLASS>
__device__ __forceinline__ float2 relax_factor(const RelaxArgs &a, const float (&mk)[C]) {
    float per_pq;
    if (PERCLASS) {
        per_pq = 0.0f;
#pragma unroll
        for (int k = 0; k < C; k++) per_pq = __fadd_rn(per_pq, __fmul_rn(a.pcm[k], mk[k]));
    } else {
        float pbg = mk[0];
#pragma unroll
        for (int k = 1; k < C; k++)
            if (k == a.bg) pbg = mk[k];
        per_pq = __fmul_rn(a.per, __fsub_rn(__fmul_rn(2.0f, pbg), 1.0f));
    }
    const float d = div100_rn(per_pq);
    return make_float2(__fadd_rn(1.0f, d), __fsub_rn(1.0f, d));
}

// 6-neighbourhood sweep of one tile column (x, y, z0 .. z0+3) by its own thread, with the
// staged boxes already in shared memory.  The thread keeps the memberships, intensities
// and polarity factors of its column (z0-1 .. z0+4) in registers: it computes the factors of
// those six voxels itself, and the column supplies the -z / +z neighbours of each voxel, so
// only the four x / y neighbours come from shared memory.  The threads of the block also
// compute the factors of the x / y face halo; the caller synchronises the block between the
// two phases.  Neighbours are summed in the Spheric order (-z, -y, -x, +x, +y, +z).
template <int C, typename T, bool PERCLASS>
struct RelaxColumn6 {
    float cm[RB_Z][C];
    float2 cf[RB_Z];
    int ci[RB_Z];

    __device__ __forceinline__ void stage(const RelaxArgs &a, const float *sm, const T *si,
                                          float2 *sf, int x0, int y0, int z0, int lx, int ly,
                                          int tid) {
        using IB = RelaxImgBox<T>;
        const int X = a.X, Y = a.Y, Z = a.Z;
        const bool col_ok = x0 + lx < X && y0 + ly < Y;
#pragma unroll
        for (int bz = 0; bz < RB_Z; bz++) {
            const int gz = z0 - 1 + bz;
            const int j = (lx + RB_OFF) + (ly + 1) * RB_X + bz * RB_X * RB_Y;
#pragma unroll
            for (int k = 0; k < C; k++) cm[bz][k] = sm[k * RB_N + j];
            ci[bz] = (int)si[(lx + IB::OFF) + (ly + 1) * IB::X + bz * IB::X * RB_Y];
            cf[bz] = make_float2(0.0f, 0.0f);
            if (col_ok && gz >= 0 && gz < Z) {
                cf[bz] = relax_factor<C, PERCLASS>(a, cm[bz]);
                sf[j] = cf[bz];
            }
        }
        // the x faces (2 x RT_Y x RT_Z voxels) and y faces (2 x RT_X x RT_Z) of the halo
        for (int e = tid; e < 2 * RT_Y * RT_Z + 2 * RT_X * RT_Z; e += RT_X * RT_Y) {
            int bx, by, bz;
            if (e < 2 * RT_Y * RT_Z) {
                bx = (e & 1) ? RB_OFF + RT_X : RB_OFF - 1;
                by = 1 + ((e >> 1) % RT_Y);
                bz = 1 + (e >> 1) / RT_Y;
            } else {
                const int f = e - 2 * RT_Y * RT_Z;
                bx = RB_OFF + f % RT_X;
                by = ((f / RT_X) & 1) ? RT_Y + 1 : 0;
                bz = 1 + f / (2 * RT_X);
            }
            const int gx = x0 - RB_OFF + bx, gy = y0 - 1 + by, gz = z0 - 1 + bz;
            if (gx >= 0 && gx < X && gy >= 0 && gy < Y && gz < Z) {
                const int j = bx + by * RB_X + bz * RB_X * RB_Y;
                float mk[C];
#pragma unroll
                for (int k = 0; k < C; k++) mk[k] = sm[k * RB_N + j];
                sf[j] = relax_factor<C, PERCLASS>(a, mk);
            }
        }
    }

    template <bool INTERIOR>
    __device__ __forceinline__ void sweep(const RelaxArgs &a, const float *sm, const T *si,
                                          const float2 *sf, float *__restrict__ mout,
                                          const uint8_t *__restrict__ seedc, int x, int y,
                                          int z0, int lx, int ly) const {
        using IB = RelaxImgBox<T>;
        const int X = a.X, Y = a.Y, Z = a.Z;
        const size_t N = a.N, XY = (size_t)X * Y;
#pragma unroll
        for (int lz = 0; lz < RT_Z; lz++) {
            const int z = z0 + lz;
            if (z >= Z) break;
            const int bz = lz + 1;
            const int hc = (lx + RB_OFF) + (ly + 1) * RB_X + bz * RB_X * RB_Y;
            const int ic = (lx + IB::OFF) + (ly + 1) * IB::X + bz * IB::X * RB_Y;
            const int ip = ci[bz];
            float acc[C];
#pragma unroll
            for (int k = 0; k < C; k++) acc[k] = 0.0f;
            float sw = 0.0f;
            auto from_smem = [&](int dh, int di) {
                float mq[C];
#pragma unroll
                for (int k = 0; k < C; k++) mq[k] = sm[k * RB_N + hc + dh];
                relax_accumulate<C, false>(a, ip, (int)si[ic + di], 0, 0, mq, sf[hc + dh], 1.0f,
                                           sw, acc);
            };
            if (INTERIOR || z > 0)
                relax_accumulate<C, false>(a, ip, ci[bz - 1], 0, 0, cm[bz - 1], cf[bz - 1], 1.0f,
                                           sw, acc);
            if (INTERIOR || y > 0) from_smem(-RB_X, -IB::X);
            if (INTERIOR || x > 0) from_smem(-1, -1);
            if (INTERIOR || x + 1 < X) from_smem(1, 1);
            if (INTERIOR || y + 1 < Y) from_smem(RB_X, IB::X);
            if (INTERIOR || z + 1 < Z)
                relax_accumulate<C, false>(a, ip, ci[bz + 1], 0, 0, cm[bz + 1], cf[bz + 1], 1.0f,
                                           sw, acc);
            const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
            float out[C];
            if (sw > 0.0f) {
#pragma unroll
                for (int k = 0; k < C; k++) out[k] = __fdiv_rn(acc[k], sw);
            } else {
#pragma unroll
                for (int k = 0; k < C; k++) out[k] = cm[bz][k];
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
};

template <int C, typename T, bool PERCLASS, int ADJ, bool INTERIOR>
__device__ __forceinline__ void relax_tile_voxels_tma(const RelaxArgs &a, const float *sm,
                                                      const T *si, const float2 *sf,
                                                      float *__restrict__ mout,
                                                      const uint8_t *__restrict__ seedc, int x,
                                                      int y, int z0, int lx, int ly) {
    using IB = RelaxImgBox<T>;
    const int X = a.X, Y = a.Y, Z = a.Z;
    const size_t N = a.N, XY = (size_t)X * Y;
#pragma unroll
    for (int lz = 0; lz < RT_Z; lz++) {
        const int z = z0 + lz;
        if (z >= Z) break;
        const int hc = (lx + RB_OFF) + (ly + 1) * RB_X + (lz + 1) * RB_X * RB_Y;
        const int ic = (lx + IB::OFF) + (ly + 1) * IB::X + (lz + 1) * IB::X * RB_Y;
        const int ip = (int)si[ic];
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
            const int hq = hc + ddx + ddy * RB_X + ddz * RB_X * RB_Y;
            const int iq = ic + ddx + ddy * IB::X + ddz * IB::X * RB_Y;
            float mq[C];
#pragma unroll
            for (int k = 0; k < C; k++) mq[k] = sm[k * RB_N + hq];
            const float dpq = (ADJ == 6) ? 1.0f : a.dpq[i];
            relax_accumulate<C, false>(a, ip, (int)si[iq], 0, 0, mq, sf[hq], dpq, sw, acc);
        }
        const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
        float out[C];
        if (sw > 0.0f) {
#pragma unroll
            for (int k = 0; k < C; k++) out[k] = __fdiv_rn(acc[k], sw);
        } else {
#pragma unroll
            for (int k = 0; k < C; k++) out[k] = sm[k * RB_N + hc];
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

// mmap: the input membership buffer as a 4D tensor [C][Z][Y][X] of floats, box
// {RB_X, RB_Y, RB_Z, C}; imap: the image as a 3D tensor [Z][Y][X], box {IB::X, RB_Y, RB_Z}.
// No multicast: every load reads this GPU's own memory into this CTA's shared memory.
template <int C, typename T, bool PERCLASS, int ADJ>
__global__ void __launch_bounds__(256, relax_min_blocks(C, false))
    relax_tile_tma_kernel(const __grid_constant__ CUtensorMap mmap,
                          const __grid_constant__ CUtensorMap imap, float *__restrict__ mout,
                          const uint8_t *__restrict__ seedc, const uint16_t *__restrict__ tdist,
                          int sweep, RelaxArgs a, int ntx, int nty, int *__restrict__ tma_err) {
    using IB = RelaxImgBox<T>;
    const int t = blockIdx.x;
    if ((int)tdist[t] > sweep - 1) return;  // provably unchanged at this sweep
    // the block has no static shared memory, so the boxes start at the aligned base
    extern __shared__ __align__(128) unsigned char rtsm[];
    float *sm = reinterpret_cast<float *>(rtsm);                           // [C][RB_Z][RB_Y][RB_X]
    T *si = reinterpret_cast<T *>(rtsm + C * RB_N * 4);                    // [RB_Z][RB_Y][IB::X]
    float2 *sf = reinterpret_cast<float2 *>(rtsm + C * RB_N * 4 + IB::BYTES);  // [RB_N]
    unsigned long long &mbar =
        *reinterpret_cast<unsigned long long *>(rtsm + C * RB_N * 4 + IB::BYTES + RB_N * 8);
    const int X = a.X, Y = a.Y, Z = a.Z;
    const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
    const int x0 = tx * RT_X, y0 = ty * RT_Y, z0 = tz * RT_Z;
    const int tid = threadIdx.x + threadIdx.y * 32;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(relax_smem_addr(&mbar))
                     : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        const unsigned bar = relax_smem_addr(&mbar);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar),
                     "r"((unsigned)(C * RB_N * 4 + IB::BYTES))
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(relax_smem_addr(sm)),
            "l"(&mmap), "r"(x0 - RB_OFF), "r"(y0 - 1), "r"(z0 - 1), "r"(0), "r"(bar)
            : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
            " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(relax_smem_addr(si)),
            "l"(&imap), "r"(x0 - IB::OFF), "r"(y0 - 1), "r"(z0 - 1), "r"(bar)
            : "memory");
    }
    if (!relax_mbar_wait_bounded(&mbar, 0, RELAX_TMA_SPIN_LIMIT)) {
        // the loads did not land: record it, give the copies in flight one more bounded
        // wait before this CTA's shared memory is released, and leave
        if (tid == 0) atomicExch(tma_err, 1);
        relax_mbar_wait_bounded(&mbar, 0, RELAX_TMA_SPIN_LIMIT);
        return;
    }
    if constexpr (ADJ == 6) {
        RelaxColumn6<C, T, PERCLASS> col;
        col.stage(a, sm, si, sf, x0, y0, z0, threadIdx.x, threadIdx.y, tid);
        __syncthreads();
        const int x = x0 + (int)threadIdx.x, y = y0 + (int)threadIdx.y;
        if (x >= X || y >= Y) return;
        const bool interior = x0 >= 1 && x0 + RT_X < X && y0 >= 1 && y0 + RT_Y < Y &&
                              z0 >= 1 && z0 + RT_Z < Z;
        if (interior)
            col.template sweep<true>(a, sm, si, sf, mout, seedc, x, y, z0, threadIdx.x,
                                     threadIdx.y);
        else
            col.template sweep<false>(a, sm, si, sf, mout, seedc, x, y, z0, threadIdx.x,
                                      threadIdx.y);
    } else {
    // polarity factors of the staged voxels that neighbour the tile (box columns 3 .. 36)
    for (int j = tid; j < RB_N; j += 256) {
        const int bx = j % RB_X, row = j / RB_X;
        const int gx = x0 - RB_OFF + bx, gy = y0 - 1 + row % RB_Y, gz = z0 - 1 + row / RB_Y;
        if (bx >= RB_OFF - 1 && bx <= RB_OFF + RT_X && gx < X && gy >= 0 && gy < Y && gz >= 0 &&
            gz < Z && gx >= 0) {
            float mk[C];
#pragma unroll
            for (int k = 0; k < C; k++) mk[k] = sm[k * RB_N + j];
            float per_pq;
            if (PERCLASS) {
                per_pq = 0.0f;
#pragma unroll
                for (int k = 0; k < C; k++) per_pq = __fadd_rn(per_pq, __fmul_rn(a.pcm[k], mk[k]));
            } else {
                float pbg = mk[0];
#pragma unroll
                for (int k = 1; k < C; k++)
                    if (k == a.bg) pbg = mk[k];
                per_pq = __fmul_rn(a.per, __fsub_rn(__fmul_rn(2.0f, pbg), 1.0f));
            }
            const float d = div100_rn(per_pq);
            sf[j] = make_float2(__fadd_rn(1.0f, d), __fsub_rn(1.0f, d));
        }
    }
    __syncthreads();
    const int lx = threadIdx.x, ly = threadIdx.y;
    const int x = x0 + lx, y = y0 + ly;
    if (x >= X || y >= Y) return;
    const bool interior = x0 >= 1 && x0 + RT_X < X && y0 >= 1 && y0 + RT_Y < Y && z0 >= 1 &&
                          z0 + RT_Z < Z;
    if (interior)
        relax_tile_voxels_tma<C, T, PERCLASS, ADJ, true>(a, sm, si, sf, mout, seedc, x, y, z0, lx,
                                                         ly);
    else
        relax_tile_voxels_tma<C, T, PERCLASS, ADJ, false>(a, sm, si, sf, mout, seedc, x, y, z0,
                                                          lx, ly);
    }
}

template <int C, typename T>
constexpr size_t relax_tma_smem_bytes() {
    return (size_t)C * RB_N * 4 + RelaxImgBox<T>::BYTES + (size_t)RB_N * 8 + 8;
}

// Launches the tile sweep for C classes; one explicit instantiation per translation unit.
template <int C>
cudaError_t launch_relax_tiles_tma_c(const CUtensorMap &mmap, const CUtensorMap &imap, float *out,
                                     bool img32, const uint8_t *seedc, const uint16_t *tdist,
                                     int sweep, const RelaxArgs &a, bool perclass, int ntiles,
                                     int ntx, int nty, cudaStream_t s, int *err);
template <int C>
cudaError_t launch_relax_tiles_c(const float *in, float *out, const void *img, bool img32,
                                 const uint8_t *seedc, const uint16_t *tdist, int sweep,
                                 const RelaxArgs &a, bool perclass, int ntiles, int ntx, int nty,
                                 cudaStream_t s);

}  // namespace oiftb
