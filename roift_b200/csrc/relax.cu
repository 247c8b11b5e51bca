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
#include <cudaTypedefs.h>

#include "relax_tile.cuh"

namespace oiftb {

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

// Number of tiles active at each sweep (for the algorithmic byte count).
__global__ void relax_tile_hist_kernel(const uint16_t *__restrict__ tdist, int nt, int K,
                                       unsigned int *hist) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int d = tdist[t];
    if (d < K) atomicAdd(&hist[d], 1u);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    }
    return fn;
}

bool image_tma_encode(CUtensorMap *m, const void *img, bool img32, int X, int Y, int Z, int bx,
                      int by, int bz) {
    if (X % (img32 ? 4 : 8) != 0) return false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t esz = img32 ? 4 : 2;
    const cuuint64_t dim[3] = {(cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z};
    const cuuint64_t stride[2] = {(cuuint64_t)X * esz, (cuuint64_t)X * esz * (cuuint64_t)Y};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
    const cuuint32_t ones[3] = {1, 1, 1};
    return enc(m, img32 ? CU_TENSOR_MAP_DATA_TYPE_INT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16, 3,
               const_cast<void *>(img), dim, stride, box, ones, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool relax_tma_encode(RelaxTma *t, const float *m0, const float *m1, const void *img,
                      bool img32, int X, int Y, int Z, int C) {
    if (X % (img32 ? 4 : 8) != 0 || C < 1 || C > 8) return false;
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t row = (cuuint64_t)X * 4, plane = row * (cuuint64_t)Y;
    const cuuint64_t vol = plane * (cuuint64_t)Z;
    const cuuint64_t mdim[4] = {(cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z, (cuuint64_t)C};
    const cuuint64_t mstride[3] = {row, plane, vol};
    const cuuint32_t mbox[4] = {(cuuint32_t)RB_X, (cuuint32_t)RB_Y, (cuuint32_t)RB_Z,
                                (cuuint32_t)C};
    const cuuint32_t ones[4] = {1, 1, 1, 1};
    const float *bases[2] = {m0, m1};
    for (int i = 0; i < 2; i++) {
        if (enc(&t->memb[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)bases[i], mdim, mstride,
                mbox, ones, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
        t->base[i] = bases[i];
    }
    const cuuint64_t esz = img32 ? 4 : 2;
    const cuuint64_t idim[3] = {(cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z};
    const cuuint64_t istride[2] = {(cuuint64_t)X * esz, (cuuint64_t)X * esz * (cuuint64_t)Y};
    const cuuint32_t ibox[3] = {(cuuint32_t)(img32 ? RelaxImgBox<int32_t>::X : RelaxImgBox<int16_t>::X),
                                (cuuint32_t)RB_Y, (cuuint32_t)RB_Z};
    if (enc(&t->img, img32 ? CU_TENSOR_MAP_DATA_TYPE_INT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16, 3,
            (void *)img, idim, istride, ibox, ones, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    return true;
}

template <typename T>
cudaError_t launch_relax_tiles(int C, const float *in, float *out, const T *img,
                               const uint8_t *seedc, const uint16_t *tdist, int sweep,
                               const RelaxArgs &a, bool perclass, int ntiles, int ntx, int nty,
                               cudaStream_t s, const RelaxTma *tma) {
    const bool img32 = sizeof(T) == 4;
    // the TMA-staged sweep reads `in` through its tensor map (not with gradient blending)
    const CUtensorMap *mmap = nullptr;
    if (tma && !a.blend) mmap = tma->base[0] == in ? &tma->memb[0] : tma->base[1] == in ? &tma->memb[1] : nullptr;
#define RELAX_TILE_CASE(CC)                                                                  \
    case CC:                                                                                 \
        return mmap ? launch_relax_tiles_tma_c<CC>(*mmap, tma->img, out, img32, seedc, tdist,  \
                                                   sweep, a, perclass, ntiles, ntx, nty, s,   \
                                                   tma->err)                                  \
                    : launch_relax_tiles_c<CC>(in, out, img, img32, seedc, tdist, sweep, a,   \
                                               perclass, ntiles, ntx, nty, s);
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
                                                 cudaStream_t, const RelaxTma *);
template cudaError_t launch_relax_tiles<int32_t>(int, const float *, float *, const int32_t *,
                                                 const uint8_t *, const uint16_t *, int,
                                                 const RelaxArgs &, bool, int, int, int,
                                                 cudaStream_t, const RelaxTma *);

}  // namespace oiftb
