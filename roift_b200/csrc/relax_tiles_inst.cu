// relax_tiles_inst.cu -- the tile sweep for one class count, compiled once per value of
// RELAX_TILE_C (1..8) so that the instantiations build in parallel.
#include "relax_tile.cuh"

#ifndef RELAX_TILE_C
#error "compile with -DRELAX_TILE_C=<classes>"
#endif

namespace oiftb {

template <int C, typename T, int ADJ>
static cudaError_t launch_tile_c(const float *in, float *out, const T *img, const uint8_t *seedc,
                                 const uint16_t *tdist, int sweep, const RelaxArgs &a,
                                 bool perclass, int ntiles, int ntx, int nty, cudaStream_t s) {
    dim3 block(32, 8);
    if (a.blend) {  // gradient blend: 6 / 4 neighbourhood, global polarity
        if (ADJ != 6 || perclass) return cudaErrorInvalidValue;
        const size_t smem = (size_t)(C + 2) * RH_N * 4 + (size_t)RH_N * 8;
        auto k = relax_tile_kernel<C, T, false, 6, true>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k<<<ntiles, block, smem, s>>>(in, out, img, seedc, tdist, sweep, a, ntx, nty);
        return cudaGetLastError();
    }
    const size_t smem = (size_t)(C + 1) * RH_N * 4 + (size_t)RH_N * 8;
    if (perclass) {
        auto k = relax_tile_kernel<C, T, true, ADJ, false>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (relax_min_blocks(C, false) > 1)  // the shared-memory carve-out that holds them
            cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        k<<<ntiles, block, smem, s>>>(in, out, img, seedc, tdist, sweep, a, ntx, nty);
    } else {
        auto k = relax_tile_kernel<C, T, false, ADJ, false>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (relax_min_blocks(C, false) > 1)  // the shared-memory carve-out that holds them
            cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        k<<<ntiles, block, smem, s>>>(in, out, img, seedc, tdist, sweep, a, ntx, nty);
    }
    return cudaGetLastError();
}

template <int C, typename T, int ADJ>
static cudaError_t launch_tile_tma_c(const CUtensorMap &mmap, const CUtensorMap &imap, float *out,
                                     const uint8_t *seedc, const uint16_t *tdist, int sweep,
                                     const RelaxArgs &a, bool perclass, int ntiles, int ntx,
                                     int nty, cudaStream_t s, int *err) {
    dim3 block(32, 8);
    const size_t smem = relax_tma_smem_bytes<C, T>();
    auto launch = [&](auto k) {
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (relax_min_blocks(C, false) > 1)  // the shared-memory carve-out that holds them
            cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        k<<<ntiles, block, smem, s>>>(mmap, imap, out, seedc, tdist, sweep, a, ntx, nty, err);
        return cudaGetLastError();
    };
    return perclass ? launch(relax_tile_tma_kernel<C, T, true, ADJ>)
                    : launch(relax_tile_tma_kernel<C, T, false, ADJ>);
}

template <>
cudaError_t launch_relax_tiles_tma_c<RELAX_TILE_C>(const CUtensorMap &mmap, const CUtensorMap &imap,
                                                   float *out, bool img32, const uint8_t *seedc,
                                                   const uint16_t *tdist, int sweep,
                                                   const RelaxArgs &a, bool perclass, int ntiles,
                                                   int ntx, int nty, cudaStream_t s, int *err) {
    const bool six = (a.nadj == 6);
    if (img32)
        return six ? launch_tile_tma_c<RELAX_TILE_C, int32_t, 6>(mmap, imap, out, seedc, tdist, sweep,
                                                                 a, perclass, ntiles, ntx, nty, s, err)
                   : launch_tile_tma_c<RELAX_TILE_C, int32_t, 26>(mmap, imap, out, seedc, tdist, sweep,
                                                                  a, perclass, ntiles, ntx, nty, s, err);
    return six ? launch_tile_tma_c<RELAX_TILE_C, int16_t, 6>(mmap, imap, out, seedc, tdist, sweep, a,
                                                             perclass, ntiles, ntx, nty, s, err)
               : launch_tile_tma_c<RELAX_TILE_C, int16_t, 26>(mmap, imap, out, seedc, tdist, sweep, a,
                                                              perclass, ntiles, ntx, nty, s, err);
}

template <>
cudaError_t launch_relax_tiles_c<RELAX_TILE_C>(const float *in, float *out, const void *img,
                                               bool img32, const uint8_t *seedc,
                                               const uint16_t *tdist, int sweep,
                                               const RelaxArgs &a, bool perclass, int ntiles,
                                               int ntx, int nty, cudaStream_t s) {
    const bool six = (a.nadj == 6);
    if (img32)
        return six ? launch_tile_c<RELAX_TILE_C, int32_t, 6>(in, out, (const int32_t *)img, seedc,
                                                             tdist, sweep, a, perclass, ntiles, ntx, nty, s)
                   : launch_tile_c<RELAX_TILE_C, int32_t, 26>(in, out, (const int32_t *)img, seedc,
                                                              tdist, sweep, a, perclass, ntiles, ntx, nty, s);
    return six ? launch_tile_c<RELAX_TILE_C, int16_t, 6>(in, out, (const int16_t *)img, seedc, tdist,
                                                         sweep, a, perclass, ntiles, ntx, nty, s)
               : launch_tile_c<RELAX_TILE_C, int16_t, 26>(in, out, (const int16_t *)img, seedc, tdist,
                                                          sweep, a, perclass, ntiles, ntx, nty, s);
}

}  // namespace oiftb
