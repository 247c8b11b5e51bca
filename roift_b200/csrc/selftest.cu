// selftest.cu -- device self-tests of arithmetic shortcuts used by the kernels.
//
// div100_rn: correctly rounded x / 100 in FP32 by one residual correction of the
// product with the rounded reciprocal (the Newton/Markstein correction step: q0 = x*r,
// e = fma(-q0, 100, x) is exact, q1 = fma(e, r, q0)).  It is used by the relaxation
// sweeps in place of a full IEEE division; oift_b200_selftest_div100 compares it with
// the IEEE quotient for every one of the 2^32 FP32 bit patterns.
#include "kernels.cuh"

namespace oiftb {

__global__ void selftest_div100_kernel(unsigned long long *bad, unsigned int *first) {
    const unsigned long long total = 1ull << 32;
    unsigned long long nbad = 0;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
         i < total; i += (unsigned long long)gridDim.x * blockDim.x) {
        const float x = __uint_as_float((unsigned int)i);
        if (isnan(x) || isinf(x)) continue;
        const float a = div100_rn(x);
        const float b = __fdiv_rn(x, 100.0f);
        // signed zeros compare equal: the sweeps only use 1 +/- x/100
        if (a != b && !(isnan(a) && isnan(b))) {
            nbad++;
            atomicMin(first, (unsigned int)i);
        }
    }
    for (int o = 16; o > 0; o >>= 1) nbad += __shfl_down_sync(0xffffffffu, nbad, o);
    if ((threadIdx.x & 31) == 0 && nbad) atomicAdd(bad, nbad);
}

}  // namespace oiftb

using namespace oiftb;

extern "C" int oift_b200_selftest_div100(unsigned long long *mismatches, unsigned int *first_bad) {
    if (!mismatches) return OIFT_E_BAD_ARG;
    unsigned long long *d_bad = nullptr;
    unsigned int *d_first = nullptr;
    if (cudaMalloc(&d_bad, sizeof(unsigned long long)) != cudaSuccess) return OIFT_E_OOM;
    if (cudaMalloc(&d_first, sizeof(unsigned int)) != cudaSuccess) {
        cudaFree(d_bad);
        return OIFT_E_OOM;
    }
    cudaMemset(d_bad, 0, sizeof(unsigned long long));
    cudaMemset(d_first, 0xFF, sizeof(unsigned int));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    selftest_div100_kernel<<<sms * 8, 256>>>(d_bad, d_first);
    unsigned int hf = 0;
    cudaError_t e1 = cudaMemcpy(mismatches, d_bad, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaError_t e2 = cudaMemcpy(&hf, d_first, sizeof(unsigned int), cudaMemcpyDeviceToHost);
    if (first_bad) *first_bad = hf;
    cudaFree(d_bad);
    cudaFree(d_first);
    return (e1 == cudaSuccess && e2 == cudaSuccess) ? OIFT_OK : OIFT_E_CUDA;
}
