// common.cuh -- shared definitions of the sm_100a OIFT + relaxation kernels.
//
// Layout in HBM (one volume, N = X*Y*Z voxels, p = x + y*X + z*X*Y as in
// gft/include/gft_scene32.h:164-179):
//   image     int16 or int32 [N]
//   weights   uint16 [P][N]; plane k holds the edge {p, p + d_k} for the k-th "positive"
//             neighbour offset of the gft Spheric order (gft/src/gft_adjrel3.cpp:47-85):
//             6-adj: +x, +y, +z; 26-adj: the 13 offsets after the centre.  bits 0..13
//             base weight, bit 14 = (I_p < I_q), bit 15 = (I_p > I_q).
//   key       uint32 [N] OIFT state: field << 17 | label << 1 | U  (U = 1 not yet
//             expanded), 0xFFFFFFFF = unreached; field = 0 for a seed, cost + 1 for any
//             other voxel.  Integer order = (cost, label) order, seeds first.
//   membership float [C][N] planar relaxation state (two buffers).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/oift_b200.h"

#define OIFT_KEY_INF 0xFFFFFFFFu
#define OIFT_BASE_MASK 0x3FFFu
#define OIFT_MAX_BASE 16383
#define OIFT_MAX_COST 32766
#define OIFT_MAX_LABEL 32767

namespace oiftb {

// Neighbour offsets in gft Spheric order without the centre.  Entry i and entry
// n-1-i are opposite; the positive half is i >= n/2.
struct Adjacency {
    int n;
    int dx[26], dy[26], dz[26];
};

inline Adjacency make_adjacency(int adj) {
    Adjacency A;
    int r2 = (adj == 26 || adj == 8) ? 3 : 1;
    A.n = 0;
    for (int z = -1; z <= 1; z++)
        for (int y = -1; y <= 1; y++)
            for (int x = -1; x <= 1; x++) {
                if (x == 0 && y == 0 && z == 0) continue;
                if (x * x + y * y + z * z <= r2) {
                    A.dx[A.n] = x;
                    A.dy[A.n] = y;
                    A.dz[A.n] = z;
                    A.n++;
                }
            }
    return A;
}

// Keys.  A seed holds field 0 and every other voxel field cost + 1, so a seed's key lies
// below any key an arc can offer it: seeds keep their labels, as in OIFT_Multi, which
// gives the labelled voxels value 0 and conquers a voxel only when w < value[q]
// (gft/src/gft_ift.cpp:929-976).  The oriented cost is at most 2 * OIFT_MAX_BASE = 32766
// (|per| <= 100), so the field fits its 15 bits.
__host__ __device__ inline uint32_t make_key(int field, int label, int unexpanded) {
    return ((uint32_t)field << 17) | ((uint32_t)label << 1) | (uint32_t)unexpanded;
}
__host__ __device__ inline uint32_t seed_key(int label) { return make_key(0, label, 1); }
// Key offered at path cost nc (>= 0) with the label bits (label << 1 | U) of the tail.
__host__ __device__ inline uint32_t offer_key(int nc, uint32_t lab_bits) {
    return ((uint32_t)(nc + 1) << 17) | lab_bits;
}
// Path cost of a conquered voxel (0 for a seed).
__host__ __device__ inline int key_cost(uint32_t k) {
    const int f = (int)(k >> 17);
    return f > 0 ? f - 1 : 0;
}
// Cost at which a level floods: -1 on the seeds' own levels, where no arc opens.
__host__ __device__ inline int key_level_cost(uint32_t k) { return (int)(k >> 17) - 1; }
__host__ __device__ inline int key_label(uint32_t k) { return (int)((k >> 1) & 0xFFFFu); }

// The same keys in either width: uint32_t (costs up to OIFT_MAX_COST) or, for exact
// weights wider than 14 bits, unsigned long long with the same layout and a 32-bit field
// (costs up to 2^31 - 2).
template <typename K> __host__ __device__ constexpr K key_inf_t() { return ~(K)0; }
template <typename K> __host__ __device__ inline K seed_key_t(int label) {
    return ((K)(unsigned)label << 1) | (K)1;
}
template <typename K> __host__ __device__ inline K offer_key_t(int nc, K lab_bits) {
    return ((K)(unsigned)(nc + 1) << 17) | lab_bits;
}
template <typename K> __host__ __device__ inline int key_cost_t(K k) {
    const long long f = (long long)(k >> 17);
    return f > 0 ? (int)(f - 1) : 0;
}
template <typename K> __host__ __device__ inline int key_level_cost_t(K k) {
    return (int)((long long)(k >> 17) - 1);
}
template <typename K> __host__ __device__ inline int key_label_t(K k) {
    return (int)((k >> 1) & (K)0xFFFFu);
}
// Wide keys: exact base weights up to 2^30 - 1, so an oriented weight (|per| <= 100)
// stays below 2^31 - 1.
#define OIFT_WIDE_MAX_BASE 1073741823

// Oriented arc weight, gft/src/gft_ift.cpp:965-973: int w = |dI|; w *= (1 +/- per/100)
// evaluated in double and truncated.  fgt = 1.0 + per/100.0, flt = 1.0 - per/100.0 are
// computed once per label with the same double expression as the reference.
__host__ __device__ inline int oriented_weight(uint32_t base, bool tail_gt, bool tail_lt,
                                               double fgt, double flt) {
    if (tail_gt) return (int)((double)base * fgt);
    if (tail_lt) return (int)((double)base * flt);
    return (int)base;
}

// Largest base b in [0, OIFT_MAX_BASE] with (int)(b * f) <= c, -1 when c < 0; trunc(b*f)
// is monotone in b for f >= 0, so "oriented weight <= c" is "base <= threshold".
// maxb is the largest base weight of the run (OIFT_MAX_BASE, or OIFT_WIDE_MAX_BASE).
__host__ __device__ inline int max_base_for_cost(int c, double f, int maxb = OIFT_MAX_BASE) {
    if (c < 0) return -1;  // no arc weighs less than 0
    if (f <= 0.0) return maxb;
    double b = floor(((double)c + 1.0) / f);
    int bi = b > (double)maxb ? maxb : (b < 0.0 ? 0 : (int)b);
    while (bi > 0 && (int)((double)bi * f) > c) bi--;
    while (bi < maxb && (int)((double)(bi + 1) * f) <= c) bi++;
    return bi;
}

// Oriented arc weight of the 2D image graph (Orient2Digraph, gft/src/gft_imagegraph.cpp:
// 981-1016): base = |dI| + 1 becomes MAX(ROUND(base * f), 1) with ROUND(x) = (int)(x + 0.5)
// for x >= 0 (gft/include/gft_common.h:120), f = 1.0 +/- alpha and alpha = per/100.0 held in
// a float; equal intensities keep the base.  The product and the sum are rounded separately,
// as the C++ evaluates them.
__host__ __device__ inline int round_weight(uint32_t base, double f) {
#ifdef __CUDA_ARCH__
    const int w = (int)__dadd_rn(__dmul_rn((double)base, f), 0.5);
#else
    const int w = (int)((double)base * f + 0.5);
#endif
    return w > 1 ? w : 1;
}
__host__ __device__ inline int oriented_weight_round(uint32_t base, bool tail_gt, bool tail_lt,
                                                     double fgt, double flt) {
    if (tail_gt) return round_weight(base, fgt);
    if (tail_lt) return round_weight(base, flt);
    return (int)base;
}
// Largest base b in [0, OIFT_MAX_BASE] with MAX(ROUND(b f), 1) <= c (monotone in b for
// f >= 0); -1 when no base qualifies (c < 1).
__host__ __device__ inline int max_base_for_cost_round(int c, double f, int maxb = OIFT_MAX_BASE) {
    if (c < 1) return -1;
    if (f <= 0.0) return maxb;
    double b = floor(((double)c + 0.5) / f);
    int bi = b > (double)maxb ? maxb : (b < 0.0 ? 0 : (int)b);
    while (bi > 0 && round_weight((uint32_t)bi, f) > c) bi--;
    while (bi < maxb && round_weight((uint32_t)(bi + 1), f) <= c) bi++;
    return bi;
}

// x / 100 rounded to nearest-even in FP32, for all finite x (exhaustively checked against
// the IEEE quotient by oift_b200_selftest_div100): the product with r = RN(1/100) is
// corrected once by the exact FMA residual e = x - q*100 (Markstein's correction step).
// The residual is exact only while the quotient is a normal number, so |x| < 2^-100
// (never reached by the sweeps, whose |per_pq| is 0 or >= 2^-24 * |per|) takes the IEEE
// division.
__device__ __forceinline__ float div100_rn(float x) {
    if (fabsf(x) < 7.88860905e-31f) return __fdiv_rn(x, 100.0f);  // 2^-100
    const float r = 0.00999999977648258209228515625f;  // RN(1/100) = 0x3C23D70A
    const float q = __fmul_rn(x, r);
    const float e = __fmaf_rn(-q, 100.0f, x);
    return __fmaf_rn(e, r, q);
}

}  // namespace oiftb

// Kernel-side error codes written to a device flag (read by the host after a launch).
#define OIFT_DEV_OK 0
#define OIFT_DEV_TIMEOUT 1
#define OIFT_DEV_QUEUE 2
