// relax.cu -- ROIFT fuzzy-membership relaxation sweeps (row a7) and argmax (row a10).
//
// Restates gft::ift::ORelax_1_Multi (gft/src/gft_ift.cpp:8655-8911) and
// ORelax_1_Multi_PerClass (gft_ift.cpp:8913-9187) in FP32 with the reference's exact
// operation order, so that memberships and labels are bit-identical to the CPU code:
//   w      = |I_p - I_q|                                   (8798)
//   per_pq = per * (2 p_bg(q) - 1)  or  sum_k per_k m_k(q)  (8800-8801, 9076-9079)
//   w     *= 1 +/- per_pq / 100                            (8803-8806)
//   w      = max(Wmax - w, 0)^8 / Dpq                      (8808-8815)
//   m'(p)  = sum_q w m(q) / sum_q w   (m(p) kept if sum w == 0)   (8817-8832)
//   seeds re-clamped one-hot after every sweep              (8839-8855)
// Every multiply/add/divide is an explicit round-to-nearest intrinsic: no FMA
// contraction, IEEE division, neighbours summed in the gft Spheric order.
//
// Dense update == masked update.  The reference updates only a "mask" that starts at
// voxels with a differently-labelled neighbour and dilates by one ring per sweep.  A
// voxel outside that mask at sweep t has only never-updated neighbours carrying its own
// one-hot class, so the dense formula gives sum(w*1)/sum(w) = 1 and 0 elsewhere --
// identical bits, provided sum(w) is finite (Wmax^8 * degree < FLT_MAX; the host
// rejects larger Wmax with OIFT_E_RANGE, where the reference itself would produce
// inf/inf = NaN).  So the sweep is a plain dense stencil with no mask state.
#include "kernels.cuh"

namespace oiftb {


// Contribution of one neighbour q to the sums of voxel p, in the reference order.
template <int C, bool PERCLASS>
__device__ __forceinline__ void relax_accumulate(const RelaxArgs &a, int ip, int iq,
                                                 const float (&mq)[C], float dpq, float &sw,
                                                 float (&acc)[C]) {
    float w = fabsf((float)(ip - iq));
    float per_pq;
    if (PERCLASS) {
        per_pq = 0.0f;
#pragma unroll
        for (int k = 0; k < C; k++) per_pq = __fadd_rn(per_pq, __fmul_rn(a.pcm[k], mq[k]));
    } else {
        float pbg = mq[0];
#pragma unroll
        for (int k = 1; k < C; k++)
            if (k == a.bg) pbg = mq[k];
        per_pq = __fmul_rn(a.per, __fsub_rn(__fmul_rn(2.0f, pbg), 1.0f));
    }
    if (ip > iq)
        w = __fmul_rn(w, __fadd_rn(1.0f, div100_rn(per_pq)));
    else if (ip < iq)
        w = __fmul_rn(w, __fsub_rn(1.0f, div100_rn(per_pq)));
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

template <int C, typename T, bool PERCLASS>
__device__ __forceinline__ void relax_finish(const RelaxArgs &a, const float *__restrict__ min_,
                                             float *__restrict__ mout,
                                             const uint8_t *__restrict__ seedc, size_t p,
                                             float sw, const float (&acc)[C]) {
    const size_t N = a.N;
    float out[C];
    if (sw > 0.0f) {
#pragma unroll
        for (int k = 0; k < C; k++) out[k] = __fdiv_rn(acc[k], sw);
    } else {
#pragma unroll
        for (int k = 0; k < C; k++) out[k] = __ldg(&min_[(size_t)k * N + p]);
    }
    const uint8_t sc = __ldg(&seedc[p]);
    if (sc != 0xFF) {
#pragma unroll
        for (int k = 0; k < C; k++) out[k] = (k == sc) ? 1.0f : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < C; k++) mout[(size_t)k * N + p] = out[k];
}

// 6-neighbourhood sweep: block (32, 8) threads over an x-y tile of one z plane.
// Neighbours in the Spheric order -z, -y, -x, +x, +y, +z (Dpq = 1).
template <int C, typename T, bool PERCLASS>
__global__ void __launch_bounds__(256) relax_sweep6_kernel(const float *__restrict__ min_,
                                                           float *__restrict__ mout,
                                                           const T *__restrict__ img,
                                                           const uint8_t *__restrict__ seedc,
                                                           RelaxArgs a) {
    const int X = a.X, Y = a.Y, Z = a.Z;
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= X || y >= Y) return;
    const size_t N = a.N, XY = (size_t)X * Y;
    const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
    const int ip = (int)__ldg(&img[p]);
    float acc[C];
#pragma unroll
    for (int k = 0; k < C; k++) acc[k] = 0.0f;
    float sw = 0.0f;
#pragma unroll
    for (int i = 0; i < 6; i++) {
        long long off;
        bool ok;
        switch (i) {
            case 0: ok = z > 0; off = -(long long)XY; break;
            case 1: ok = y > 0; off = -(long long)X; break;
            case 2: ok = x > 0; off = -1; break;
            case 3: ok = x + 1 < X; off = 1; break;
            case 4: ok = y + 1 < Y; off = X; break;
            default: ok = z + 1 < Z; off = (long long)XY; break;
        }
        if (!ok) continue;
        const size_t q = (size_t)((long long)p + off);
        float mq[C];
#pragma unroll
        for (int k = 0; k < C; k++) mq[k] = __ldg(&min_[(size_t)k * N + q]);
        relax_accumulate<C, PERCLASS>(a, ip, (int)__ldg(&img[q]), mq, 1.0f, sw, acc);
    }
    relax_finish<C, T, PERCLASS>(a, min_, mout, seedc, p, sw, acc);
}

// General neighbourhood (26 / 8 / 4): same arithmetic over the Spheric list.
template <int C, typename T, bool PERCLASS>
__global__ void __launch_bounds__(256) relax_sweep_kernel(const float *__restrict__ min_,
                                                          float *__restrict__ mout,
                                                          const T *__restrict__ img,
                                                          const uint8_t *__restrict__ seedc,
                                                          RelaxArgs a) {
    const int X = a.X, Y = a.Y, Z = a.Z;
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= X || y >= Y) return;
    const size_t N = a.N, XY = (size_t)X * Y;
    const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
    const int ip = (int)__ldg(&img[p]);
    float acc[C];
#pragma unroll
    for (int k = 0; k < C; k++) acc[k] = 0.0f;
    float sw = 0.0f;
    for (int i = 0; i < a.nadj; i++) {
        const int qx = x + a.dx[i], qy = y + a.dy[i], qz = z + a.dz[i];
        if (qx < 0 || qx >= X || qy < 0 || qy >= Y || qz < 0 || qz >= Z) continue;
        const size_t q = (size_t)qx + (size_t)qy * X + (size_t)qz * XY;
        float mq[C];
#pragma unroll
        for (int k = 0; k < C; k++) mq[k] = __ldg(&min_[(size_t)k * N + q]);
        relax_accumulate<C, PERCLASS>(a, ip, (int)__ldg(&img[q]), mq, a.dpq[i], sw, acc);
    }
    relax_finish<C, T, PERCLASS>(a, min_, mout, seedc, p, sw, acc);
}

// One-hot initial membership from the OIFT labels (gft_ift.cpp:8745-8752).
__global__ void relax_init_kernel(const int32_t *label, size_t N, int C, const int *l2c,
                                  int maxl, int bg, float *m) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        int lb = label[p], c = bg;
        if (lb >= 0 && lb <= maxl && l2c[lb] >= 0) c = l2c[lb];
        for (int k = 0; k < C; k++) m[(size_t)k * N + p] = (k == c) ? 1.0f : 0.0f;
    }
}

// Seed class map: 0xFF = not a seed, else the class of the seed's label.
__global__ void relax_seed_kernel(const int32_t *seeds, int nseeds, const int32_t *label,
                                  size_t N, const int *l2c, int maxl, int bg, uint8_t *seedc) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nseeds) return;
    int p = seeds[i];
    if (p < 0 || (size_t)p >= N) return;
    int lb = label[p], c = bg;
    if (lb >= 0 && lb <= maxl && l2c[lb] >= 0) c = l2c[lb];
    seedc[p] = (uint8_t)c;
}

// Labels present among the seeds (gft_ift.cpp:8684-8712): bitmap over label values,
// aggregated in shared memory so that a million seeds of two labels cost two global
// atomics per block.
__global__ void seed_presence_kernel(const int32_t *seed_labels, int nseeds, uint32_t *bits) {
    __shared__ uint32_t sb[1024];
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) sb[i] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nseeds; i += gridDim.x * blockDim.x) {
        int lb = seed_labels[i];
        if (lb < 0) lb = 0;
        if (lb > OIFT_MAX_LABEL) continue;
        const uint32_t bit = 1u << (lb & 31);
        if (!(sb[lb >> 5] & bit)) atomicOr(&sb[lb >> 5], bit);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 1024; i += blockDim.x)
        if (sb[i]) atomicOr(&bits[i], sb[i]);
}

// Argmax with strict '>' so the lowest class wins ties (gft_ift.cpp:8889-8904).
__global__ void relax_argmax_kernel(const float *m, size_t N, int C, const int *classes,
                                    int32_t *label, uint8_t *mask) {
    for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < N;
         p += (size_t)gridDim.x * blockDim.x) {
        int best = 0;
        float bv = m[p];
        for (int k = 1; k < C; k++) {
            float v = m[(size_t)k * N + p];
            if (v > bv) {
                bv = v;
                best = k;
            }
        }
        int lb = classes[best];
        if (label) label[p] = lb;
        if (mask) mask[p] = (uint8_t)(lb != 0);
    }
}

template <int C, typename T>
static cudaError_t launch_sweep_c(const float *in, float *out, const T *img,
                                  const uint8_t *seedc, const RelaxArgs &a, bool perclass,
                                  int sms, cudaStream_t s) {
    (void)sms;
    dim3 block(32, 8), grid((a.X + 31) / 32, (a.Y + 7) / 8, a.Z);
    const bool six = (a.nadj == 6);
    if (perclass) {
        if (six)
            relax_sweep6_kernel<C, T, true><<<grid, block, 0, s>>>(in, out, img, seedc, a);
        else
            relax_sweep_kernel<C, T, true><<<grid, block, 0, s>>>(in, out, img, seedc, a);
    } else {
        if (six)
            relax_sweep6_kernel<C, T, false><<<grid, block, 0, s>>>(in, out, img, seedc, a);
        else
            relax_sweep_kernel<C, T, false><<<grid, block, 0, s>>>(in, out, img, seedc, a);
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_relax_sweep(int C, const float *in, float *out, const T *img,
                               const uint8_t *seedc, const RelaxArgs &a, bool perclass,
                               int sms, cudaStream_t s) {
    switch (C) {
        case 1: return launch_sweep_c<1, T>(in, out, img, seedc, a, perclass, sms, s);
        case 2: return launch_sweep_c<2, T>(in, out, img, seedc, a, perclass, sms, s);
        case 3: return launch_sweep_c<3, T>(in, out, img, seedc, a, perclass, sms, s);
        case 4: return launch_sweep_c<4, T>(in, out, img, seedc, a, perclass, sms, s);
        case 5: return launch_sweep_c<5, T>(in, out, img, seedc, a, perclass, sms, s);
        case 6: return launch_sweep_c<6, T>(in, out, img, seedc, a, perclass, sms, s);
        case 7: return launch_sweep_c<7, T>(in, out, img, seedc, a, perclass, sms, s);
        case 8: return launch_sweep_c<8, T>(in, out, img, seedc, a, perclass, sms, s);
        default: return cudaErrorInvalidValue;
    }
}

template cudaError_t launch_relax_sweep<int16_t>(int, const float *, float *, const int16_t *,
                                                 const uint8_t *, const RelaxArgs &, bool, int,
                                                 cudaStream_t);
template cudaError_t launch_relax_sweep<int32_t>(int, const float *, float *, const int32_t *,
                                                 const uint8_t *, const RelaxArgs &, bool, int,
                                                 cudaStream_t);

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

// Tiles holding a voxel with a differently-labelled neighbour get distance 0.
__global__ void relax_boundary_tiles_kernel(const int32_t *__restrict__ label, int X, int Y,
                                            int Z, int nadj, RelaxArgs a, uint16_t *tdist,
                                            int ntx, int nty) {
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= X || y >= Y) return;
    const size_t XY = (size_t)X * Y;
    const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
    const int lp = label[p];
    bool edge = false;
    for (int i = 0; i < nadj && !edge; i++) {
        const int qx = x + a.dx[i], qy = y + a.dy[i], qz = z + a.dz[i];
        if (qx < 0 || qx >= X || qy < 0 || qy >= Y || qz < 0 || qz >= Z) continue;
        edge = label[(size_t)qx + (size_t)qy * X + (size_t)qz * XY] != lp;
    }
    if (edge) tdist[(x / RT_X) + (y / RT_Y) * ntx + (z / RT_Z) * ntx * nty] = 0;
}

// One pass of the tile-grid distance along axis `ax`: a gap of k >= 1 tiles of extent
// `dim` separates voxels by at least (k-1)*dim + 1 steps along that axis.  Three passes
// give min over boundary tiles of the sum (6/4-adj, Manhattan) or the max (26/8-adj,
// Chebyshev) of the per-axis gaps: a lower bound of the voxel distance to the mask.
__global__ void relax_tile_gap_pass_kernel(const uint16_t *__restrict__ din, uint16_t *dout,
                                           int ntx, int nty, int ntz, int ax, int dim,
                                           int cheb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nt = ntx * nty * ntz;
    if (t >= nt) return;
    const int c3[3] = {t % ntx, (t / ntx) % nty, t / (ntx * nty)};
    const int n = ax == 0 ? ntx : ax == 1 ? nty : ntz;
    const int stride = ax == 0 ? 1 : ax == 1 ? ntx : ntx * nty;
    const int i = c3[ax];
    const int base = t - i * stride;
    int best = 0xFFFF;
    for (int j = 0; j < n; j++) {
        const int v = din[base + j * stride];
        if (v == 0xFFFF) continue;
        const int k = i > j ? i - j : j - i;
        const int g = k == 0 ? 0 : (k - 1) * dim + 1;
        const int cmb = cheb ? (g > v ? g : v) : g + v;
        best = cmb < best ? cmb : best;
    }
    dout[t] = (uint16_t)(best > 0xFFFF ? 0xFFFF : best);
}

// One dilation step of the block distance: d' = min(d, min over neighbour tiles + 1).
__global__ void relax_tile_dilate_kernel(const uint16_t *__restrict__ din, uint16_t *dout,
                                         int ntx, int nty, int ntz, int cheb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nt = ntx * nty * ntz;
    if (t >= nt) return;
    const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
    int d = din[t];
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                const int man = (dx != 0) + (dy != 0) + (dz != 0);
                if (man == 0 || (!cheb && man > 1)) continue;
                const int qx = tx + dx, qy = ty + dy, qz = tz + dz;
                if (qx < 0 || qx >= ntx || qy < 0 || qy >= nty || qz < 0 || qz >= ntz) continue;
                const int v = din[qx + qy * ntx + qz * ntx * nty] + 1;
                d = v < d ? v : d;
            }
    dout[t] = (uint16_t)d;
}

// Number of tiles active at each sweep (for the algorithmic byte count).
__global__ void relax_tile_hist_kernel(const uint16_t *__restrict__ tdist, int nt, int K,
                                       unsigned int *hist) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int d = tdist[t];
    if (d < K) atomicAdd(&hist[d], 1u);
}

template <int C, typename T, bool PERCLASS, int ADJ, bool INTERIOR>
__device__ __forceinline__ void relax_tile_voxels(const RelaxArgs &a, const float *sm,
                                                  const int *si, float *__restrict__ mout,
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
            relax_accumulate<C, PERCLASS>(a, ip, si[hq], mq, dpq, sw, acc);
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

template <int C, typename T, bool PERCLASS, int ADJ>
__global__ void __launch_bounds__(256) relax_tile_kernel(const float *__restrict__ min_,
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
    const int X = a.X, Y = a.Y, Z = a.Z;
    const size_t N = a.N, XY = (size_t)X * Y;
    const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
    const int x0 = tx * RT_X, y0 = ty * RT_Y, z0 = tz * RT_Z;
    const int tid = threadIdx.x + threadIdx.y * 32;
    for (int i = tid; i < RH_N; i += 256) {
        const int hx = i % RH_X, hy = (i / RH_X) % RH_Y, hz = i / (RH_X * RH_Y);
        const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
        if (gx >= 0 && gx < X && gy >= 0 && gy < Y && gz >= 0 && gz < Z) {
            const size_t g = (size_t)gx + (size_t)gy * X + (size_t)gz * XY;
#pragma unroll
            for (int k = 0; k < C; k++) sm[k * RH_N + i] = __ldg(&min_[(size_t)k * N + g]);
            si[i] = (int)__ldg(&img[g]);
        }
    }
    __syncthreads();
    const int lx = threadIdx.x, ly = threadIdx.y;
    const int x = x0 + lx, y = y0 + ly;
    if (x >= X || y >= Y) return;
    // every neighbour of every voxel of an interior tile lies in the volume
    const bool interior = x0 >= 1 && x0 + RT_X < X && y0 >= 1 && y0 + RT_Y < Y && z0 >= 1 &&
                          z0 + RT_Z < Z;
    if (interior)
        relax_tile_voxels<C, T, PERCLASS, ADJ, true>(a, sm, si, mout, seedc, x, y, z0, lx, ly);
    else
        relax_tile_voxels<C, T, PERCLASS, ADJ, false>(a, sm, si, mout, seedc, x, y, z0, lx, ly);
}

template <int C, typename T, int ADJ>
static cudaError_t launch_tile_c(const float *in, float *out, const T *img, const uint8_t *seedc,
                                 const uint16_t *tdist, int sweep, const RelaxArgs &a,
                                 bool perclass, int ntiles, int ntx, int nty, cudaStream_t s) {
    const size_t smem = (size_t)(C + 1) * RH_N * 4;
    dim3 block(32, 8);
    if (perclass) {
        auto k = relax_tile_kernel<C, T, true, ADJ>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<ntiles, block, smem, s>>>(in, out, img, seedc, tdist, sweep, a, ntx, nty);
    } else {
        auto k = relax_tile_kernel<C, T, false, ADJ>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<ntiles, block, smem, s>>>(in, out, img, seedc, tdist, sweep, a, ntx, nty);
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_relax_tiles(int C, const float *in, float *out, const T *img,
                               const uint8_t *seedc, const uint16_t *tdist, int sweep,
                               const RelaxArgs &a, bool perclass, int ntiles, int ntx, int nty,
                               cudaStream_t s) {
    const bool six = (a.nadj == 6);
#define RELAX_TILE_CASE(CC)                                                                   \
    case CC:                                                                                  \
        return six ? launch_tile_c<CC, T, 6>(in, out, img, seedc, tdist, sweep, a, perclass,   \
                                             ntiles, ntx, nty, s)                             \
                   : launch_tile_c<CC, T, 26>(in, out, img, seedc, tdist, sweep, a, perclass,  \
                                              ntiles, ntx, nty, s);
    switch (C) {
        RELAX_TILE_CASE(1)
        RELAX_TILE_CASE(2)
        RELAX_TILE_CASE(3)
        RELAX_TILE_CASE(4)
        RELAX_TILE_CASE(5)
        RELAX_TILE_CASE(6)
        RELAX_TILE_CASE(7)
        RELAX_TILE_CASE(8)
        default: return cudaErrorInvalidValue;
    }
#undef RELAX_TILE_CASE
}

template cudaError_t launch_relax_tiles<int16_t>(int, const float *, float *, const int16_t *,
                                                 const uint8_t *, const uint16_t *, int,
                                                 const RelaxArgs &, bool, int, int, int,
                                                 cudaStream_t);
template cudaError_t launch_relax_tiles<int32_t>(int, const float *, float *, const int32_t *,
                                                 const uint8_t *, const uint16_t *, int,
                                                 const RelaxArgs &, bool, int, int, int,
                                                 cudaStream_t);

}  // namespace oiftb
