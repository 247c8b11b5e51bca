// oift.cu -- oriented f_max Image Foresting Transform on sm_100a (rows a5-a6).
//
// Semantics (the restatement R2 of the oracle): keys (cost, label) are conquered in
// strictly increasing lexicographic order; a voxel p with key (c, l) offers its
// neighbour q the key (max(c, w_l(p->q)), l), where w_l is the oriented arc weight of
// gft/src/gft_ift.cpp:965-973 with the polarity of the TAIL's label (label 0 = -per in
// the global mode, gft_ift.cpp:968; per_class[l] otherwise, gft_ift.cpp:1055-1060).  The
// smaller label wins equal costs, as the reference GPU packing does
// (gpu/oift_fmax_gpu.cu:26-29,93-96).  Because a level (c, l) is a reachability closure,
// the result does not depend on the order inside a level: the map is deterministic and
// bit-exact against the oracle, unlike the arrival-order-dependent Bellman-Ford of the
// reference GPU path (gpu/oift_fmax_gpu.cu:33-107, 202-238).
//
// Execution: ONE persistent cooperative launch, OIFT_WARPS warps per SM.  The volume is cut
// into warp tiles of 32 (x) x TY (y) x TZ (z) voxels, TY*TZ = 32 rows: a lane owns one row
// as a 32-bit mask.  Tile t belongs to CTA t % #CTAs.  Per level (cost, label):
//   S  each CTA marks its tiles whose pending key equals the level as wanted and adds the
//      smallest pending key of its other tiles to the level's running minimum;
//   P  its warps claim wanted tiles one at a time: stage keys + edge codes of the tile,
//      flood the level inside the tile with row-mask operations (arc masks per row from a
//      per-level base-weight threshold), push across the tile faces and publish same-level
//      crossings to the owner CTAs' mailboxes, then give the in-tile heads the flood did
//      not reach their tentative keys; every pending-key update also lowers the running
//      minimum.
// The level ends when no tile is pending or in flight (the level's outstanding count); the
// running minimum is then the next level, so no grid barrier separates levels.
// Every wait (first-level barrier, level end, claims) is bounded; on expiry the kernel sets
// an error flag, every warp leaves, and the host reports OIFT_E_NOT_CONVERGED.
#include <cooperative_groups.h>

#include "kernels.cuh"

namespace oiftb {


// n / d for 0 <= n < 2^31 by a multiply-high, for divisors known only at run time: with
// s = floor(log2 d) and m = ceil(2^(32+s) / d) (m = 0 for a power of two, a shift alone),
// q = umulhi(n, m) >> s is exact on that range, since m exceeds 2^(32+s) / d by less than 1
// and 2^(32+s) / d >= 2^31.
struct FastDiv {
    uint32_t m, s;
};
__host__ __device__ inline FastDiv make_fastdiv(uint32_t d) {
    uint32_t s = 0;
    while ((d >> (s + 1)) != 0u) s++;
    FastDiv f;
    f.s = s;
    f.m = (d == (1u << s)) ? 0u
                           : (uint32_t)((((unsigned long long)1 << (32 + s)) + d - 1) / d);
    return f;
}
__device__ __forceinline__ uint32_t fast_div(uint32_t n, FastDiv f) {
    return (f.m ? __umulhi(n, f.m) : n) >> f.s;
}

struct OiftArgs {
    uint32_t *key;
    const uint16_t *W;
    uint32_t *tpend;
    // a wide-range run's 64-bit keys and pending keys (the full-neighbourhood kernel only)
    unsigned long long *key64;
    unsigned long long *tpend64;
    unsigned long long *mbox;  // [3][nctas][mbox_words] re-activation bitmasks, per level slot
    unsigned int *lprof;       // [lprof_cap][2]: per-level SM cycles and tile steps
    int lprof_cap;
    int mbox_words;
    int nwarps;
    int nctas;                 // CTAs of the grid (or team); tile t belongs to CTA t % nctas
    int X, Y, Z;
    size_t N;
    int ntx, nty, ntz, ntiles;
    FastDiv fd_ntx, fd_ntxy, fd_nctas;  // division by ntx, ntx * nty and nctas
    const float *pol_table;  // device, per label (x100)
    int npol;
    float pol_default;
    OiftGlobals *g;
    long long spin_limit;
    int max_levels;
    // 26 / 8 neighbourhoods: arc weights from the image on the fly (process_tile_full)
    const void *img;       // int16 or int32 [N]
    int wmode;             // OIFT_W_GRAD, OIFT_W_GRAD_Q or OIFT_W_RBF_Q
    int wcap;              // base weight ceiling (wq, or OIFT_MAX_BASE)
    const uint16_t *lut;   // RBF_Q table over |dI|
    int lut_len;
    // gradient blend (BLEND_Q, 6 / 4 neighbourhoods): normalised Sobel map and mix weight
    const int32_t *gmap;
    float alpha;
    // image-graph orientation (OIFT_W_IMAGEGRAPH): MAX(ROUND(base f), 1), f from a float alpha
    int ig;
    // tile-major copy of the code planes ([tile][plane][row][32]), or null
    const uint16_t *Wt;
    // set by the seeds kernel when a seed is out of range or has a bad label (or null)
    const int *seed_flag;
};

// Warps per CTA of the persistent kernels: 12 leaves each busy warp more issue slots than 16
// (32.3 against 33.3 ms on the 256^3 ellipsoid; 8 warps: 34.5 ms)
#ifndef OIFT_WARPS_OVERRIDE
constexpr int OIFT_WARPS = 12;
#else
constexpr int OIFT_WARPS = OIFT_WARPS_OVERRIDE;
#endif
constexpr int OIFT_SPARSE_MAX = 64;   // level voxels in a tile up to which it runs sparse
// Worklist rounds of a tile step before a flood that still runs finishes in bit mode.  With
// 0 (the default) every tile step floods in bit mode: the critical path of a level is its
// chain of flood layers, and a bit-mode layer costs a few row-mask operations where a
// worklist round costs a round of shared-memory traffic (256^3 ellipsoid: 45.8 -> 38.7 ms).
#ifndef OIFT_BIT_AFTER
#define OIFT_BIT_AFTER 0
#endif
// 1 (the default): a row's six families of arc masks are computed together the first time
// the frontier comes next to the row; 0: each family the first time the frontier reaches
// that side (32.8 against 36.3 ms on the 256^3 ellipsoid); 2: every row with open voxels at
// the first layer (39.7 ms)
// Order in which idle warps claim wanted tiles: 0 (the default) lowest slot first; 1 tiles
// re-activated through the mailbox first (33.5 against 32.2 ms on the 256^3 ellipsoid)
#ifndef OIFT_CLAIM_ORDER
#define OIFT_CLAIM_ORDER 0
#endif
// Longest sleep of an idle warp that does not watch the mailbox (ns): idle warps take issue
// slots from the warps that process tiles on the same SM (256^3 ellipsoid: 64 ns 32.28 ms,
// 512 ns 32.06 ms, 4096 ns 35.04 ms).
#ifndef OIFT_IDLE_NS_MAX
#define OIFT_IDLE_NS_MAX 512
#endif
#ifndef OIFT_MASK_ROWS
#define OIFT_MASK_ROWS 1
#endif
// Idle warps of a CTA that watch its mailbox and the level's count at the same time: with
// more than one, a re-activation is seen sooner after it lands (256^3 ellipsoid: 1 watcher
// 31.83 ms, 2 31.72 ms, 3 31.70 ms)
#ifndef OIFT_FETCHERS
#define OIFT_FETCHERS 3
#endif
constexpr int OIFT_WORKLIST = 256;    // per-warp voxel worklist of the sparse mode

__device__ __forceinline__ unsigned int vload(const volatile unsigned int *p) { return *p; }
__device__ __forceinline__ int vload(const volatile int *p) { return *p; }
__device__ __forceinline__ unsigned long long vload(const volatile unsigned long long *p) {
    return *p;
}

#ifndef OIFT_PROBE
#define OIFT_PROBE 0
#endif
// 1 (the default): the tile steps and the level loop sum their SM cycles per phase into the
// run's statistics; 0: those sums stay zero
#ifndef OIFT_CYCLES
#define OIFT_CYCLES 1
#endif
#define OIFT_CLOCK() (OIFT_CYCLES ? clock64() : 0ll)
#if OIFT_PROBE
// latency probes (globaltimer ns): [0,1] publish -> claim, [2,3] claim -> first publish,
// [4,5] claim -> end of step
__device__ unsigned long long g_probe[8];
__device__ unsigned long long g_hist[3][32];  // log2(ns) histograms of the three latencies
__device__ unsigned long long g_tpub[1 << 20];
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
#endif
// Release / acquire fence at GPU scope: orders this warp's earlier memory operations (and
// those of the lanes synchronised with it) before its later ones, without the total order
// of a sequentially consistent fence.
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;\n" ::: "memory"); }
// Exchange with acquire semantics at GPU scope: the writes released before the value that
// it takes are visible to this warp's later reads.
__device__ __forceinline__ unsigned long long exch_acquire_gpu(unsigned long long *p,
                                                               unsigned long long v) {
    unsigned long long old;
    asm volatile("atom.acquire.gpu.exch.b64 %0, [%1], %2;\n" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}

// Asynchronous global -> shared copies (cp.async): 16 bytes through L2 only, 4 bytes.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Barrier over the `nctas` CTAs that share `g` (the whole cooperative grid, or one team of
// the batched kernel), with a bounded wait.  Returns false, in every thread of the CTA, when
// the wait ended on an error flag or on the spin limit instead of the last arrival.
__device__ bool team_barrier(OiftGlobals *g, long long limit, unsigned int nctas) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned int gen = vload(&g->bar_gen);
        __threadfence();
        if (atomicAdd(&g->bar_count, 1u) == nctas - 1) {
            g->bar_count = 0;
            __threadfence();
            atomicAdd(&g->bar_gen, 1u);
        } else {
            long long spins = 0;
            while (vload(&g->bar_gen) == gen) {
                if (vload(&g->error)) {
                    ok = 0;
                    break;
                }
                if (++spins > limit) {
                    atomicCAS(&g->error, 0, OIFT_DEV_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Keys, pending keys and the level minima of a run, by key width.
template <typename K> __device__ __forceinline__ K *keys_of(const OiftArgs &A);
template <> __device__ __forceinline__ uint32_t *keys_of<uint32_t>(const OiftArgs &A) { return A.key; }
template <> __device__ __forceinline__ unsigned long long *keys_of<unsigned long long>(const OiftArgs &A) {
    return A.key64;
}
template <typename K> __device__ __forceinline__ K *tpend_of(const OiftArgs &A);
template <> __device__ __forceinline__ uint32_t *tpend_of<uint32_t>(const OiftArgs &A) { return A.tpend; }
template <> __device__ __forceinline__ unsigned long long *tpend_of<unsigned long long>(const OiftArgs &A) {
    return A.tpend64;
}
template <typename K> __device__ __forceinline__ K *runmin_of(OiftGlobals *g);
template <> __device__ __forceinline__ uint32_t *runmin_of<uint32_t>(OiftGlobals *g) { return g->runmin; }
template <> __device__ __forceinline__ unsigned long long *runmin_of<unsigned long long>(OiftGlobals *g) {
    return g->runmin64;
}
template <typename K> __device__ __forceinline__ K *first_of(OiftGlobals *g);
template <> __device__ __forceinline__ uint32_t *first_of<uint32_t>(OiftGlobals *g) { return &g->first; }
template <> __device__ __forceinline__ unsigned long long *first_of<unsigned long long>(OiftGlobals *g) {
    return &g->first64;
}

__device__ __forceinline__ float polarity_of(const OiftArgs &A, int l) {
    return (l < A.npol) ? A.pol_table[l] : A.pol_default;
}

// Arc feasibility at cost c: code is the edge code, tail_low = the tail is the voxel
// that stores the edge (so bit 15 means tail > head).
__device__ __forceinline__ bool arc_ok(uint32_t code, bool tail_low, int c, int bgt, int blt) {
    uint32_t base = code & OIFT_BASE_MASK;
    bool hi = (code >> 15) & 1, lo = (code >> 14) & 1;
    bool gt = tail_low ? hi : lo;
    bool lt = tail_low ? lo : hi;
    int thr = gt ? bgt : (lt ? blt : c);
    return (int)base <= thr;
}

// Re-activating a tile at the current level: tile t is owned by CTA t % nctas; each CTA has
// a bitmask mailbox in global memory (bit t / nctas).  The producer raises the level's
// outstanding count, then sets the bit; if the bit was already set the tile is already
// pending and the count is given back.  A warp of the owner CTA takes the bits with one
// exchange and hands them to the CTA's shared "wanted" set, from which any of its warps
// claims tiles one at a time.

template <int TY, int TZ>
__device__ __forceinline__ int tile_of(const OiftArgs &A, int x, int y, int z) {
    return (x >> 5) + (y / TY) * A.ntx + (z / TZ) * A.ntx * A.nty;
}

// Publishes the re-activations of a tile step; lane i names the tile it re-activates in
// tq (-1: none).  Tile tq belongs to CTA tq % nctas, bit tq / nctas of its mailbox for the
// level's slot `par` (a CTA still finishing the level before reads only that one's).  The
// level's outstanding count is raised first and the warp's key updates are released
// before the mailbox bits.  A tile that was marked already gives its count back in
// give_back_duplicates, which the tile step calls once it has nothing else to do, so that
// waiting for the mailbox update's reply does not delay the rest of the step.
__device__ __forceinline__ void publish_reactivations(const OiftArgs &A, int par, int tq,
                                                      unsigned long long &old,
                                                      unsigned long long &bit) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const uint32_t act = __ballot_sync(FULL, tq >= 0);
#if OIFT_PROBE
    if (tq >= 0) g_tpub[tq] = gtimer();
#endif
    if (lane == 0) atomicAdd(&A.g->outstanding[par], __popc(act));
    // every lane's key updates and the raised count precede the mailbox bits
    fence_acq_rel_gpu();
    __syncwarp();
    if (tq >= 0) {
        const int j = (int)fast_div((uint32_t)tq, A.fd_nctas), w = tq - j * A.nctas;
        const unsigned long long b = 1ull << (j & 63);
        old |= atomicOr(&A.mbox[((size_t)par * A.nctas + w) * A.mbox_words + (j >> 6)], b) & b;
        bit |= b;
    }
}
__device__ __forceinline__ void give_back_duplicates(const OiftArgs &A, int par,
                                                     unsigned long long old) {
    const uint32_t dups = __ballot_sync(0xffffffffu, old != 0ull);
    if ((threadIdx.x & 31) == 0 && dups) atomicSub(&A.g->outstanding[par], __popc(dups));
}

// Process one tile at level kk (cost c, label l).  All 32 lanes of the warp call it.
template <int TY, int TZ>
__device__ __forceinline__ void process_tile(const OiftArgs &A, int t, int par, uint32_t kk, int c, int l,
                             double fgt, double flt, int bgt, int blt, uint32_t *skey,
                             uint16_t *sw, uint16_t *shx, uint16_t *shy, uint16_t *shz,
                             uint32_t *wl, uint32_t *nfm, uint32_t *rmask, long long *cyc) {
    long long tc0 = OIFT_CLOCK();
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int X = A.X, Y = A.Y, Z = A.Z;
    const size_t XY = (size_t)X * Y, N = A.N;
    const int tyz = (int)fast_div((uint32_t)t, A.fd_ntx), tz = (int)fast_div((uint32_t)t, A.fd_ntxy);
    const int tx = t - tyz * A.ntx, ty = tyz - tz * A.nty;
    const int x0 = tx * 32, y0 = ty * TY, z0 = tz * TZ;
    const int x = x0 + lane;
    const bool has_z = (Z > 1);
    // per lane: a re-activation published by this step found its mailbox bit set already
    unsigned long long pub_old = 0ull, pub_bit = 0ull;
#if OIFT_PROBE
    const unsigned long long probe_t0 = gtimer();
    bool probe_pub = false;
    if (lane == 0) {
        const unsigned long long tp = atomicExch(&g_tpub[t], 0ull);
        if (tp && probe_t0 > tp) {
            atomicAdd(&g_probe[0], probe_t0 - tp);
            atomicAdd(&g_probe[1], 1ull);
            atomicAdd(&g_hist[0][63 - __clzll(probe_t0 - tp)], 1ull);
        }
    }
#endif

    const uint32_t kexp = kk - 1u;
    const uint32_t lab_bits = ((uint32_t)l << 1) | 1u;
    auto arc_key = [&](uint32_t code, bool tail_low) -> uint32_t {
        const bool hi = (code >> 15) & 1, lo = (code >> 14) & 1;
        const int w = A.ig ? oriented_weight_round(code & OIFT_BASE_MASK, tail_low ? hi : lo,
                                                   tail_low ? lo : hi, fgt, flt)
                           : oriented_weight(code & OIFT_BASE_MASK, tail_low ? hi : lo,
                                             tail_low ? lo : hi, fgt, flt);
        return offer_key(w > c ? w : c, lab_bits);
    };
    // A successful out-of-tile push either continues this level next door (the
    // face-neighbour tile is marked for re-activation; all marks of the tile step are
    // published together by flush_reactivations) or lowers the neighbour's pending key.
    // A push that only lowers a neighbour tile's pending key adds that key to the level's
    // running minimum at the end of the step (with the tile's own pending key, one update per
    // warp), not before the step's re-activations are published: every warp updates that one
    // word, and the publication's release fence would wait for the update
    // (256^3 ellipsoid: 30.33 -> 30.10 ms).
    uint32_t runmin_def = OIFT_KEY_INF;
    auto settle = [&](uint32_t nk, uint32_t old, int qx, int qy, int qz) {
        if (nk < old) {
            if (nk == kk) {
                const int face = qx < x0 ? 0 : qx >= x0 + 32 ? 1 : qy < y0 ? 2 : qy >= y0 + TY ? 3
                                 : qz < z0 ? 4 : 5;
                atomicOr(rmask, 1u << face);
            } else {
                atomicMin(&A.tpend[tile_of<TY, TZ>(A, qx, qy, qz)], nk);
                runmin_def = nk < runmin_def ? nk : runmin_def;
            }
        }
    };
    auto flush_reactivations = [&]() {
        __syncwarp();
        const uint32_t m = *(volatile uint32_t *)rmask;
        if (m == 0u) return;
        __syncwarp();
        if (lane == 0) *rmask = 0u;
        int tq = -1;
        if (lane < 6 && ((m >> lane) & 1u)) {
            const int nt = tx + (lane == 0 ? -1 : lane == 1 ? 1 : 0);
            const int ny = ty + (lane == 2 ? -1 : lane == 3 ? 1 : 0);
            const int nz = tz + (lane == 4 ? -1 : lane == 5 ? 1 : 0);
            tq = nt + ny * A.ntx + nz * A.ntx * A.nty;
        }
        publish_reactivations(A, par, tq, pub_old, pub_bit);
#if OIFT_PROBE
        {
            const unsigned long long now = gtimer();
            if (lane == 0 && !probe_pub) {
                atomicAdd(&g_probe[2], now - probe_t0);
                atomicAdd(&g_probe[3], 1ull);
                atomicAdd(&g_hist[1][63 - __clzll(now - probe_t0 + 1)], 1ull);
            }
            probe_pub = true;
        }
#endif
    };
    auto pending = [&]() {
        uint32_t m = OIFT_KEY_INF;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const uint4 v = reinterpret_cast<const uint4 *>(skey)[lane + 32 * i];
            if (v.x > kk && v.x < m) m = v.x;
            if (v.y > kk && v.y < m) m = v.y;
            if (v.z > kk && v.z < m) m = v.z;
            if (v.w > kk && v.w < m) m = v.w;
        }
        // the keys the step's pushes left pending next door join the level's minimum here
        uint32_t r = runmin_def < m ? runmin_def : m;
        for (int o = 16; o > 0; o >>= 1) {
            uint32_t v = __shfl_xor_sync(FULL, m, o);
            m = v < m ? v : m;
            v = __shfl_xor_sync(FULL, r, o);
            r = v < r ? v : r;
        }
        if (lane == 0 && m != OIFT_KEY_INF) atomicMin(&A.tpend[t], m);
        if (lane == 0 && r != OIFT_KEY_INF) atomicMin(&A.g->runmin[par], r);
    };
    // ---- stage keys, edge codes and the -x/-y/-z halo codes in shared memory ----
    // shx holds the -x halo as 32-bit pairs (codes of x0-2, x0-1): entry 2r+1 is row r's.
    const bool full = (x0 + 32 <= X) && (y0 + TY <= Y) && (z0 + TZ <= Z) && ((X & 7) == 0);
    if (full) {
        // one round trip: every lane queues its 16-byte chunks as asynchronous copies and
        // waits for all of them (rows start 16-byte aligned since X % 8 == 0, x0 % 32 == 0)
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const int j = lane + 32 * m, r = j >> 3, col = j & 7;
            const size_t p0 = (size_t)x0 + (size_t)(y0 + r % TY) * X + (size_t)(z0 + r / TY) * XY;
            cp_async16(reinterpret_cast<uint4 *>(skey) + j,
                       reinterpret_cast<const uint4 *>(A.key + p0) + col);
        }
        if (A.Wt) {  // the tile's 6 KB of codes in one contiguous run
            const uint4 *src = reinterpret_cast<const uint4 *>(A.Wt) + (size_t)t * 384;
#pragma unroll
            for (int m = 0; m < 12; m++) {
                const int j = lane + 32 * m, pl = j >> 7;
                if (pl < 2 || has_z)
                    cp_async16(reinterpret_cast<uint4 *>(sw) + j, src + j);
                else
                    reinterpret_cast<uint4 *>(sw)[j] = make_uint4(0, 0, 0, 0);
            }
        } else {
#pragma unroll
            for (int m = 0; m < 12; m++) {
                const int j = lane + 32 * m, pl = j >> 7, r = (j >> 2) & 31, col = j & 3;
                const size_t p0 = (size_t)x0 + (size_t)(y0 + r % TY) * X + (size_t)(z0 + r / TY) * XY;
                if (pl < 2 || has_z)
                    cp_async16(reinterpret_cast<uint4 *>(sw) + j,
                               reinterpret_cast<const uint4 *>(A.W + (size_t)pl * N + p0) + col);
                else
                    reinterpret_cast<uint4 *>(sw)[j] = make_uint4(0, 0, 0, 0);
            }
        }
        // halo codes of the -x / -y / -z neighbours: from the tile-major copy (the lower
        // neighbour tiles of a full tile are full), else from the planes
        {
            const int yr = y0 + (lane % TY), zr = z0 + (lane / TY);
            if (x0 > 0)
                cp_async4(shx + 2 * lane,
                          A.Wt ? A.Wt + ((size_t)(t - 1) * 3) * 1024 + lane * 32 + 30
                               : A.W + (size_t)(x0 - 2) + (size_t)yr * X + (size_t)zr * XY);
            else
                shx[2 * lane + 1] = 0;
        }
        if (lane < 4 * TZ) {
            const int zl = lane >> 2, col = lane & 3;
            if (y0 > 0)
                cp_async16(shy + zl * 32 + col * 8,
                           A.Wt ? A.Wt + ((size_t)(t - A.ntx) * 3 + 1) * 1024 + ((TY - 1) + zl * TY) * 32 + col * 8
                                : A.W + N + (size_t)(x0 + col * 8) + (size_t)(y0 - 1) * X + (size_t)(z0 + zl) * XY);
            else
                *reinterpret_cast<uint4 *>(shy + zl * 32 + col * 8) = make_uint4(0, 0, 0, 0);
        }
        if (TZ > 1 && (lane >> 2) < TY) {  // TY rows of four 16-byte chunks
            const int yl = lane >> 2, col = lane & 3;
            if (z0 > 0)
                cp_async16(shz + yl * 32 + col * 8,
                           A.Wt ? A.Wt + ((size_t)(t - A.ntx * A.nty) * 3 + 2) * 1024 + (yl + (TZ - 1) * TY) * 32 + col * 8
                                : A.W + 2 * N + (size_t)(x0 + col * 8) + (size_t)(y0 + yl) * X + (size_t)(z0 - 1) * XY);
            else
                *reinterpret_cast<uint4 *>(shz + yl * 32 + col * 8) = make_uint4(0, 0, 0, 0);
        }
        cp_async_wait_all();
    } else {
#pragma unroll 4
        for (int r = 0; r < 32; r++) {
            const int y = y0 + (r % TY), z = z0 + (r / TY);
            const bool valid = (x < X) && (y < Y) && (z < Z);
            skey[r * 32 + lane] =
                valid ? __ldcg(&A.key[(size_t)x + (size_t)y * X + (size_t)z * XY]) : 0u;
        }
        const int yr = y0 + (lane % TY), zr = z0 + (lane / TY);
        uint16_t hx = 0, hy[TZ], hz[TY];
        if (x0 > 0 && yr < Y && zr < Z)
            hx = __ldg(&A.W[(size_t)(x0 - 1) + (size_t)yr * X + (size_t)zr * XY]);
#pragma unroll
        for (int zl = 0; zl < TZ; zl++)
            hy[zl] = (y0 > 0 && x < X && z0 + zl < Z)
                ? __ldg(&A.W[N + (size_t)x + (size_t)(y0 - 1) * X + (size_t)(z0 + zl) * XY]) : 0;
#pragma unroll
        for (int yl = 0; yl < TY; yl++)
            hz[yl] = (TZ > 1 && has_z && z0 > 0 && x < X && y0 + yl < Y)
                ? __ldg(&A.W[2 * N + (size_t)x + (size_t)(y0 + yl) * X + (size_t)(z0 - 1) * XY]) : 0;
        for (int r = 0; r < 32; r++) {
            const int y = y0 + (r % TY), z = z0 + (r / TY);
            const bool valid = (x < X) && (y < Y) && (z < Z);
            const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
            sw[r * 32 + lane] = valid ? __ldg(&A.W[p]) : 0;
            sw[1024 + r * 32 + lane] = valid ? __ldg(&A.W[N + p]) : 0;
            sw[2048 + r * 32 + lane] = (valid && has_z) ? __ldg(&A.W[2 * N + p]) : 0;
        }
        shx[2 * lane + 1] = hx;
#pragma unroll
        for (int zl = 0; zl < TZ; zl++) shy[zl * 32 + lane] = hy[zl];
        if (TZ > 1) {
#pragma unroll
            for (int yl = 0; yl < TY; yl++) shz[yl * 32 + lane] = hz[yl];
        }
    }
    __syncwarp();
    // ---- level rows: lane r keeps row r's voxels at this level (rowF) and those at or
    // below it, i.e. at this level or expanded before (rowV) ----
    uint32_t rowF = 0, rowV = 0;
#pragma unroll 8
    for (int r = 0; r < 32; r++) {
        const uint32_t k = skey[r * 32 + lane];
        const uint32_t bF = __ballot_sync(FULL, k == kk);
        const uint32_t bV = __ballot_sync(FULL, k <= kk);
        if (lane == r) {
            rowF = bF;
            rowV = bV;
        }
    }
    int nf0 = __popc(rowF);
    for (int o = 16; o > 0; o >>= 1) nf0 += __shfl_xor_sync(FULL, nf0, o);
    const long long tcount = OIFT_CLOCK();
    cyc[0] += tcount - tc0;
    if (nf0 == 0) {  // stale activation: only the pending key is refreshed
        pending();
        cyc[3] += 1;
        return;
    }
    // Sparse rounds first: a voxel worklist expands up to 32 voxels per round.  A flood
    // that is still running after OIFT_BIT_AFTER rounds (or that starts with more than
    // OIFT_SPARSE_MAX level voxels) finishes in bit mode: the closure of the level inside
    // the tile advances one layer per step of row-mask operations, then every voxel it
    // reached is expanded from a compacted worklist.
    // Pushes across the tile faces from the expanded voxels wl[0, n), all lanes at once:
    // the global atomics of a batch share one round trip.
    auto push_out = [&](int n) {
        for (int base = 0; base < n; base += 32) {
            const int idx = base + lane;
            // one slot per axis: a voxel leaves the tile at most once along each axis
            uint32_t nk[3] = {OIFT_KEY_INF, OIFT_KEY_INF, OIFT_KEY_INF}, old[3] = {0, 0, 0};
            int qx[3] = {0, 0, 0}, qy[3] = {0, 0, 0}, qz[3] = {0, 0, 0};
            if (idx < n) {
                const uint32_t li = wl[idx];
                const int r = (int)(li >> 5), xl = (int)(li & 31);
                const int xg = x0 + xl, y = y0 + (r % TY), z = z0 + (r / TY);
                if (xl == 0 && xg > 0) {
                    nk[0] = arc_key(shx[2 * r + 1], false);
                    qx[0] = xg - 1; qy[0] = y; qz[0] = z;
                } else if (xl == 31 && xg + 1 < X) {
                    nk[0] = arc_key(sw[r * 32 + xl], true);
                    qx[0] = xg + 1; qy[0] = y; qz[0] = z;
                }
                if ((r % TY) == 0 && y > 0) {
                    nk[1] = arc_key(shy[(r / TY) * 32 + xl], false);
                    qx[1] = xg; qy[1] = y - 1; qz[1] = z;
                } else if ((r % TY) == TY - 1 && y + 1 < Y) {
                    nk[1] = arc_key(sw[1024 + r * 32 + xl], true);
                    qx[1] = xg; qy[1] = y + 1; qz[1] = z;
                }
                if (has_z) {
                    if (r < TY && z > 0) {
                        nk[2] = arc_key(TZ > 1 ? shz[(r % TY) * 32 + xl] : 0u, false);
                        qx[2] = xg; qy[2] = y; qz[2] = z - 1;
                    } else if (r + TY >= 32 && z + 1 < Z) {
                        nk[2] = arc_key(sw[2048 + r * 32 + xl], true);
                        qx[2] = xg; qy[2] = y; qz[2] = z + 1;
                    }
                }
#pragma unroll
                for (int a = 0; a < 3; a++)
                    if (nk[a] != OIFT_KEY_INF)
                        old[a] = atomicMin(&A.key[(size_t)qx[a] + (size_t)qy[a] * X +
                                                  (size_t)qz[a] * XY], nk[a]);
            }
#pragma unroll
            for (int a = 0; a < 3; a++)
                if (nk[a] != OIFT_KEY_INF) settle(nk[a], old[a], qx[a], qy[a], qz[a]);
        }
    };
    // The six arcs of worklist voxel li: in-tile head, its slot, the edge code and whether
    // the tail is the voxel that stores the edge.
    struct Arcs {
        bool in[6];
        int lq[6];
        uint32_t code[6];
    };
    auto arcs_of = [&](uint32_t li, Arcs &a) {
        const int r = (int)(li >> 5), xl = (int)(li & 31);
        const int xg = x0 + xl, y = y0 + (r % TY), z = z0 + (r / TY);
        a.in[0] = r >= TY;                              // -z
        a.lq[0] = li - 32 * TY;
        a.in[1] = (r % TY) > 0;                         // -y
        a.lq[1] = li - 32;
        a.in[2] = xl > 0;                               // -x
        a.lq[2] = li - 1;
        a.in[3] = xl < 31 && xg + 1 < X;                // +x
        a.lq[3] = li + 1;
        a.in[4] = (r % TY) < TY - 1 && y + 1 < Y;       // +y
        a.lq[4] = li + 32;
        a.in[5] = r + TY < 32 && has_z && z + 1 < Z;    // +z
        a.lq[5] = li + 32 * TY;
        a.code[0] = a.in[0] ? sw[2048 + a.lq[0]] : 0u;
        a.code[1] = a.in[1] ? sw[1024 + a.lq[1]] : 0u;
        a.code[2] = a.in[2] ? sw[a.lq[2]] : 0u;
        a.code[3] = sw[li];
        a.code[4] = sw[1024 + li];
        a.code[5] = sw[2048 + li];
    };
    const bool tail_low[6] = {false, false, false, true, true, true};
    int done = 0, cnt = 0, rounds = 0;
    bool bitmode = OIFT_BIT_AFTER == 0 || nf0 > OIFT_SPARSE_MAX;
    if (!bitmode) {
        // ---- sparse mode: flood and expand from a voxel worklist ----
        // append_rows(m, base): the voxels of row `lane` in m join the worklist after `base`
        // entries (a warp prefix sum places them) and are marked at this level; returns the
        // new count.  Entries past OIFT_WORKLIST are not stored: bit mode then finds them
        // through their key.
        auto append_rows = [&](uint32_t m, int base) -> int {
            const int n = __popc(m);
            int incl = n;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(FULL, incl, 31);
            int pos = base + incl - n;
            while (m) {
                const int b = __ffs(m) - 1;
                m &= m - 1;
                const uint32_t li = (uint32_t)(lane << 5 | b);
                if (pos < OIFT_WORKLIST) wl[pos] = li;
                skey[li] = kk;
                pos++;
            }
            return base + total;
        };
        const long long ts0 = OIFT_CLOCK();
        nfm[lane] = 0u;
        cnt = append_rows(rowF, 0);
        __syncwarp();
        const long long ts1 = OIFT_CLOCK();
        cyc[12] += ts1 - ts0;
        for (;;) {
            if (done >= cnt) break;
            if (cnt > OIFT_WORKLIST || rounds >= OIFT_BIT_AFTER) {
                bitmode = true;
                break;
            }
            // ---- one flood round: expand up to 32 worklist voxels, one per lane; open arcs
            // mark their in-tile heads in nfm, other arcs lower the heads' keys ----
            const int idx = done + lane;
            if (idx < cnt) {
                const uint32_t li = wl[idx];
                const int r = (int)(li >> 5), xl = (int)(li & 31);
                const size_t p = (size_t)(x0 + xl) + (size_t)(y0 + (r % TY)) * X +
                                 (size_t)(z0 + (r / TY)) * XY;
                // every head key is read before any update (keys only decrease, so an early
                // read costs at most a redundant push)
                Arcs a;
                arcs_of(li, a);
                uint32_t sk[6];
#pragma unroll
                for (int d = 0; d < 6; d++) sk[d] = a.in[d] ? skey[a.lq[d]] : 0u;
                A.key[p] = kexp;
                skey[li] = kexp;
                uint32_t same_row = 0u;  // open x-neighbours, marked with one update
#pragma unroll
                for (int d = 0; d < 6; d++) {
                    if (!a.in[d] || sk[d] <= kk) continue;  // across a face, at this level, or expanded
                    const int rq = a.lq[d] >> 5, xq = a.lq[d] & 31;
                    if (arc_ok(a.code[d], tail_low[d], c, bgt, blt)) {
                        if (rq == r)
                            same_row |= 1u << xq;
                        else
                            atomicOr(&nfm[rq], 1u << xq);
                    } else {
                        const uint32_t nk = arc_key(a.code[d], tail_low[d]);
                        if (nk < sk[d]) {
                            atomicMin(&skey[a.lq[d]], nk);
                            atomicMin(&A.key[(size_t)(x0 + xq) + (size_t)(y0 + rq % TY) * X +
                                             (size_t)(z0 + rq / TY) * XY], nk);
                        }
                    }
                }
                if (same_row) atomicOr(&nfm[r], same_row);
            }
            done = (done + 32 < cnt) ? done + 32 : cnt;
            rounds++;
            __syncwarp();
            // ---- the next flood layer: heads reached in this round and not visited ----
            const uint32_t m = nfm[lane] & ~rowV;
            nfm[lane] = 0u;
            rowV |= m;
            cnt = append_rows(m, cnt);
            __syncwarp();
        }
        __syncwarp();
        const long long ts2 = OIFT_CLOCK();
        push_out(done < OIFT_WORKLIST ? done : OIFT_WORKLIST);
        __syncwarp();
        const long long ts3 = OIFT_CLOCK();
        cyc[13] += ts2 - ts1;
        cyc[14] += ts3 - ts2;
        cyc[17] += rounds;
        cyc[18] += done;
        if (!bitmode) {
            cyc[19] += (*(volatile uint32_t *)rmask != 0u);
            flush_reactivations();
            give_back_duplicates(A, par, pub_old);
            const long long ts4 = OIFT_CLOCK();
            pending();
            const long long ts5 = OIFT_CLOCK();
            cyc[15] += ts4 - ts3;
            cyc[16] += ts5 - ts4;
            cyc[1] += ts5 - tcount;
            cyc[4] += 1;
            return;
        }
    }
    // ---- bit mode ----
    const long long tb0 = OIFT_CLOCK();
    // lane r: row r's flooded voxels not yet expanded (P) and its open voxels (Om: key above
    // the level, neither final nor flooded at this level).  Straight from the level rows
    // when no sparse round ran; rebuilt from the keys otherwise.
    uint32_t P, Om;
    if (done == 0 && cnt <= OIFT_WORKLIST) {
        P = rowF;
        Om = ~rowV;  // positions outside the volume were staged as key 0 (at or below)
    } else {
        P = 0u;
        Om = 0u;
#pragma unroll 8
        for (int r = 0; r < 32; r++) {
            const uint32_t k = skey[r * 32 + lane];
            const uint32_t bP = __ballot_sync(FULL, k == kk);
            const uint32_t bO = __ballot_sync(FULL, k > kk);
            if (lane == r) {
                P = bP;
                Om = bO;
            }
        }
    }
    // rows that have a y neighbour row inside the tile below / above them
    constexpr uint32_t ROWS_YM = []() constexpr {
        uint32_t m = 0;
        for (int r = 0; r < 32; r++) if (r % TY != 0) m |= 1u << r;
        return m;
    }();
    constexpr uint32_t ROWS_YP = []() constexpr {
        uint32_t m = 0;
        for (int r = 0; r < 32; r++) if (r % TY != TY - 1) m |= 1u << r;
        return m;
    }();
    // Closure of the level inside the tile.  Lane r keeps the pull masks of row r: bit x of
    // Mpx is "the arc (x-1 -> x) is open at this level", Mmx (x+1 -> x), Mym / Myp from the
    // rows y-1 / y+1, Mzm / Mzp from z-1 / z+1.  A family of masks of a row is computed the
    // first time the frontier reaches the row's neighbour on that side while the row still
    // has open voxels: one ballot with lane = x.
    uint32_t Fm = P, fr = P;
    uint32_t Mpx = 0u, Mmx = 0u, Mym = 0u, Myp = 0u, Mzm = 0u, Mzp = 0u;
    uint32_t rx = 0u;  // rows (families x) whose masks are computed
#if !OIFT_MASK_ROWS
    uint32_t rym = 0u, ryp = 0u, rzm = 0u, rzp = 0u;  // the other families, per row
#endif
    int biters = 0, mrows = 0;
    for (;;) {
        const uint32_t frows = __ballot_sync(FULL, fr != 0u);
        const uint32_t orows = __ballot_sync(FULL, (Om & ~Fm) != 0u);
#if OIFT_MASK_ROWS
        // every family of masks of a row the frontier reaches, computed together (2: of
        // every row with open voxels, at the first layer)
        uint32_t trows = frows | ((frows << 1) & ROWS_YM) | ((frows >> 1) & ROWS_YP);
        if constexpr (TZ > 1) trows |= (frows << TY) | (frows >> TY);
        if (OIFT_MASK_ROWS == 2) trows = FULL;
        uint32_t need = trows & orows & ~rx;
        rx |= need;
        while (need) {
            const int q = __ffs(need) - 1;
            need &= need - 1;
            mrows++;
            const uint32_t c0 = sw[q * 32 + lane];
            const uint32_t cym = (q % TY != 0) ? sw[1024 + (q - 1) * 32 + lane] : 0u;
            const uint32_t cyp = sw[1024 + q * 32 + lane];
            const uint32_t czm = (TZ > 1 && q >= TY) ? sw[2048 + (q - TY) * 32 + lane] : 0u;
            const uint32_t czp = sw[2048 + q * 32 + lane];
            const uint32_t c0m = __shfl_up_sync(FULL, c0, 1);
            const uint32_t bPX = __ballot_sync(FULL, lane > 0 && arc_ok(c0m, true, c, bgt, blt));
            const uint32_t bMX = __ballot_sync(FULL, lane < 31 && arc_ok(c0, false, c, bgt, blt));
            const uint32_t bYM = __ballot_sync(FULL, arc_ok(cym, true, c, bgt, blt));
            const uint32_t bYP = __ballot_sync(FULL, arc_ok(cyp, false, c, bgt, blt));
            const uint32_t bZM = __ballot_sync(FULL, arc_ok(czm, true, c, bgt, blt));
            const uint32_t bZP = __ballot_sync(FULL, arc_ok(czp, false, c, bgt, blt));
            if (lane == q) {
                Mpx = bPX;
                Mmx = bMX;
                Mym = (q % TY != 0) ? bYM : 0u;
                Myp = (q % TY != TY - 1) ? bYP : 0u;
                Mzm = (TZ > 1 && q >= TY) ? bZM : 0u;
                Mzp = (TZ > 1 && q + TY < 32) ? bZP : 0u;
            }
        }
#else
        uint32_t need = frows & orows & ~rx;
        rx |= need;
        while (need) {
            const int q = __ffs(need) - 1;
            need &= need - 1;
            mrows++;
            const uint32_t c0 = sw[q * 32 + lane];
            const uint32_t c0m = __shfl_up_sync(FULL, c0, 1);
            const uint32_t bPX = __ballot_sync(FULL, lane > 0 && arc_ok(c0m, true, c, bgt, blt));
            const uint32_t bMX = __ballot_sync(FULL, lane < 31 && arc_ok(c0, false, c, bgt, blt));
            if (lane == q) {
                Mpx = bPX;
                Mmx = bMX;
            }
        }
        need = (frows << 1) & ROWS_YM & orows & ~rym;
        rym |= need;
        while (need) {
            const int q = __ffs(need) - 1;
            need &= need - 1;
            mrows++;
            const uint32_t b = __ballot_sync(FULL, arc_ok(sw[1024 + (q - 1) * 32 + lane], true, c, bgt, blt));
            if (lane == q) Mym = b;
        }
        need = (frows >> 1) & ROWS_YP & orows & ~ryp;
        ryp |= need;
        while (need) {
            const int q = __ffs(need) - 1;
            need &= need - 1;
            mrows++;
            const uint32_t b = __ballot_sync(FULL, arc_ok(sw[1024 + q * 32 + lane], false, c, bgt, blt));
            if (lane == q) Myp = b;
        }
        if constexpr (TZ > 1) {
            need = (frows << TY) & orows & ~rzm;
            rzm |= need;
            while (need) {
                const int q = __ffs(need) - 1;
                need &= need - 1;
                mrows++;
                const uint32_t b = __ballot_sync(FULL, arc_ok(sw[2048 + (q - TY) * 32 + lane], true, c, bgt, blt));
                if (lane == q) Mzm = b;
            }
            need = (frows >> TY) & orows & ~rzp;
            rzp |= need;
            while (need) {
                const int q = __ffs(need) - 1;
                need &= need - 1;
                mrows++;
                const uint32_t b = __ballot_sync(FULL, arc_ok(sw[2048 + q * 32 + lane], false, c, bgt, blt));
                if (lane == q) Mzp = b;
            }
        }
#endif
        // one layer: the open, unflooded voxels next to the frontier through an open arc
        uint32_t g = ((fr << 1) & Mpx) | ((fr >> 1) & Mmx) |
                     (__shfl_up_sync(FULL, fr, 1) & Mym) | (__shfl_down_sync(FULL, fr, 1) & Myp);
        if constexpr (TZ > 1)
            g |= (__shfl_up_sync(FULL, fr, TY) & Mzm) | (__shfl_down_sync(FULL, fr, TY) & Mzp);
        g &= Om & ~Fm;
        biters++;
        if (!__any_sync(FULL, g != 0u)) break;
        Fm |= g;
        fr = g;
    }
    const long long tb1 = OIFT_CLOCK();
    // ---- expansion of the closure.  The voxels on the tile's faces go first: their arcs
    // across the faces are pushed and the tile's same-level crossings are published, so that
    // the flood continues next door while this tile marks its closure expanded in global
    // memory and gives its in-tile heads that the closure did not reach the arc's key (the
    // arc is closed there).  The face voxels are marked expanded only then, with the rest of
    // the closure: the publication's release fence does not wait for those stores, and a
    // neighbour's push that meets such a voxel before its mark re-activates this tile once
    // more, which finds nothing left (256^3 ellipsoid: 31.04 -> 30.30 ms).  Voxels join the
    // worklist OIFT_WORKLIST at a time ----
    nfm[lane] = Fm;
    // compact(m): the voxels of row `lane` in m join the worklist (up to OIFT_WORKLIST in all)
    // and leave m; returns how many joined
    auto compact = [&](uint32_t &m) -> int {
        const int n = __popc(m);
        int incl = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        int pos = incl - n;
        while (m && pos < OIFT_WORKLIST) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            wl[pos++] = (uint32_t)(lane << 5 | b);
        }
        __syncwarp();
        return total < OIFT_WORKLIST ? total : OIFT_WORKLIST;
    };
    constexpr uint32_t ROWS_FACE = []() constexpr {
        uint32_t m = 0;
        for (int r = 0; r < 32; r++)
            if (r % TY == 0 || r % TY == TY - 1 || (TZ > 1 && (r < TY || r >= 32 - TY))) m |= 1u << r;
        return m;
    }();
    int nexp = 0;
    {
        uint32_t frem = Fm & (((ROWS_FACE >> lane) & 1u) ? FULL : 0x80000001u);
        while (__any_sync(FULL, frem != 0u)) {
            const int nb = compact(frem);
            push_out(nb);
            __syncwarp();
        }
        const long long tf1 = OIFT_CLOCK();
        flush_reactivations();
        const long long tf2 = OIFT_CLOCK();
        cyc[16] += tf1 - tb1;
        cyc[17] += tf2 - tf1;
    }
    const long long tf3 = OIFT_CLOCK();
    uint32_t rem = Fm;
    while (__any_sync(FULL, rem != 0u)) {
        const int nb = compact(rem);
        nexp += nb;
        for (int base = 0; base < nb; base += 32) {
            const int idx = base + lane;
            if (idx < nb) {
                const uint32_t li = wl[idx];
                const int r = (int)(li >> 5), xl = (int)(li & 31);
                const size_t p = (size_t)(x0 + xl) + (size_t)(y0 + (r % TY)) * X +
                                 (size_t)(z0 + (r / TY)) * XY;
                Arcs a;
                arcs_of(li, a);
                uint32_t sk[6];
                bool tgt[6];
#pragma unroll
                for (int d = 0; d < 6; d++) {
                    tgt[d] = a.in[d] && !((nfm[a.lq[d] >> 5] >> (a.lq[d] & 31)) & 1u);
                    sk[d] = tgt[d] ? skey[a.lq[d]] : 0u;
                }
                A.key[p] = kexp;
                skey[li] = kexp;
#pragma unroll
                for (int d = 0; d < 6; d++) {
                    if (!tgt[d] || sk[d] <= kk) continue;
                    const uint32_t nk = arc_key(a.code[d], tail_low[d]);
                    if (nk < sk[d]) {
                        const int rq = a.lq[d] >> 5, xq = a.lq[d] & 31;
                        atomicMin(&skey[a.lq[d]], nk);
                        atomicMin(&A.key[(size_t)(x0 + xq) + (size_t)(y0 + rq % TY) * X +
                                         (size_t)(z0 + rq / TY) * XY], nk);
                    }
                }
            }
        }
        __syncwarp();
    }
    const long long tb2 = OIFT_CLOCK();
    cyc[18] += tb2 - tf3;
    // ---- pending key of this tile; published activations that merged give their counts back
    pending();
    give_back_duplicates(A, par, pub_old);
    const long long tb3 = OIFT_CLOCK();
#if OIFT_PROBE
    if (lane == 0) {
        const unsigned long long dt = gtimer() - probe_t0;
        atomicAdd(&g_probe[4], dt);
        atomicAdd(&g_probe[5], 1ull);
        atomicAdd(&g_hist[2][63 - __clzll(dt + 1)], 1ull);
    }
#endif
    cyc[6] += tb1 - tb0;
    cyc[7] += biters;
    cyc[8] += mrows;
    cyc[9] += tb2 - tb1;
    cyc[10] += nexp;
    cyc[11] += tb3 - tb2;
    cyc[2] += tb3 - tcount;
    cyc[5] += 1;
}


// ------------------------------------------------------ 26 / 8 neighbourhoods ----
// Tile step for the full 3x3(x3) neighbourhood (Spheric(1.75): 26 in 3D, 8 in 2D).  The
// 13 (4) edge planes of a tile would not fit in shared memory next to the keys, so the
// tile stages its intensities with a one-voxel halo instead and evaluates the base weight
// of every arc from |I_p - I_q| as the builder does (GRAD: |dI|, GRAD_Q: min(|dI|, wq),
// RBF_Q: lut[|dI|]); the orientation is the sign of I_tail - I_head.  Tiles are 32 x TY x TZ
// with TY * TZ <= 16 rows, the level's voxels are flooded in rounds from a worklist that
// holds every voxel of the tile (no overflow), and pushes across the 26 faces, edges and
// corners of the tile go out together after the flood.
template <typename TI>
__device__ __forceinline__ int gen_base(const OiftArgs &A, int ip, int iq) {
    const int d = ip - iq;
    const int ad = d < 0 ? -d : d;
    int b = ad;
    if (A.wmode == OIFT_W_RBF_Q) b = A.lut[ad < A.lut_len ? ad : A.lut_len - 1];
    else if (A.wmode == OIFT_W_IMAGEGRAPH) b = ad + 1;
    return b > A.wcap ? A.wcap : b;
}

template <int TY, int TZ, typename TI, bool BLEND, typename K = uint32_t, bool FACES = BLEND>
__device__ __forceinline__ void process_tile_full(const OiftArgs &A, int t, int par, K kk, int c, int l,
                                  double fgt, double flt, int bgt, int blt, K *skey,
                                  int32_t *simg, uint16_t *wl, uint32_t *nfm, uint32_t *rmask,
                                  long long *cyc) {
    constexpr int NR = TY * TZ;           // rows of 32 voxels
    constexpr int HY = TY + 2;
    constexpr int HZ = TZ > 1 ? TZ + 2 : 1;
    constexpr int ZO = TZ > 1 ? 1 : 0;    // halo offset along z
    static_assert(NR <= 16, "full-neighbourhood tiles hold at most 16 rows");
    long long tc0 = OIFT_CLOCK();
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int X = A.X, Y = A.Y, Z = A.Z;
    const size_t XY = (size_t)X * Y;
    const int tyz = (int)fast_div((uint32_t)t, A.fd_ntx), tz = (int)fast_div((uint32_t)t, A.fd_ntxy);
    const int tx = t - tyz * A.ntx, ty = tyz - tz * A.nty;
    const int x0 = tx * 32, y0 = ty * TY, z0 = tz * TZ;
    const int x = x0 + lane;
    const K kexp = kk - (K)1;
    const K lab_bits = ((K)(unsigned)l << 1) | (K)1;
    K *const keys = keys_of<K>(A);
    K *const tpend = tpend_of<K>(A);
    K *const runmin = runmin_of<K>(A.g);
    constexpr K KINF = key_inf_t<K>();
    const TI *img = static_cast<const TI *>(A.img);
    // staged halo: int32 intensities, or (BLEND) 16-bit intensities followed by 16-bit
    // gradients; both index by halo position
    constexpr int HN = 34 * HY * HZ;
    uint16_t *simg16 = reinterpret_cast<uint16_t *>(simg);
    auto hidx = [&](int xl, int yl, int zl) -> int {  // tile-local coordinates, -1 .. 32
        return (zl + ZO) * (HY * 34) + (yl + 1) * 34 + (xl + 1);
    };
    auto hval = [&](int h) -> int { return BLEND ? (int)simg16[h] : simg[h]; };
    // BLEND: per-label float factors of OIFT_Multi_GradWeight (exp_gradient_weight.cpp:249-252)
    float bgtf = 1.0f, bltf = 1.0f;
    if (BLEND) {
        const float q = __fdiv_rn(polarity_of(A, l), 100.0f);
        bgtf = __fadd_rn(1.0f, q);
        bltf = __fsub_rn(1.0f, q);
    }
    // oriented weight of the arc p -> q (halo positions hp, hq) with tail p
    auto arc_w = [&](int hp, int hq) -> int {
        const int ip = hval(hp), iq = hval(hq);
        if (BLEND) {
            // wf = alpha |dI| + (1 - alpha)(g_p + g_q) * 0.5f, (int)(wf * factor), >= 0
            const float idiff = (float)abs(ip - iq);
            const float gavg = __fmul_rn((float)((int)simg16[HN + hp] + (int)simg16[HN + hq]), 0.5f);
            const float wf = __fadd_rn(__fmul_rn(A.alpha, idiff),
                                       __fmul_rn(__fsub_rn(1.0f, A.alpha), gavg));
            const int w = ip > iq ? (int)__fmul_rn(wf, bgtf)
                                  : (ip < iq ? (int)__fmul_rn(wf, bltf) : (int)wf);
            return w < 0 ? 0 : w;
        }
        const uint32_t b = (uint32_t)gen_base<TI>(A, ip, iq);
        return A.ig ? oriented_weight_round(b, ip > iq, ip < iq, fgt, flt)
                    : oriented_weight(b, ip > iq, ip < iq, fgt, flt);
    };
    // arc p -> q with tail p: open at this cost, or the key it offers q
    auto arc_open = [&](int hp, int hq) -> bool {
        if (BLEND) return arc_w(hp, hq) <= c;
        const int ip = hval(hp), iq = hval(hq);
        const int b = gen_base<TI>(A, ip, iq);
        return ip > iq ? b <= bgt : (ip < iq ? b <= blt : b <= c);
    };
    auto arc_key = [&](int hp, int hq) -> K {
        const int w = arc_w(hp, hq);
        return offer_key_t<K>(w > c ? w : c, lab_bits);
    };
    auto pending = [&]() {
        K m = KINF;
        if constexpr (sizeof(K) == 4) {
#pragma unroll
            for (int i = 0; i < NR / 4; i++) {
                const uint4 v = reinterpret_cast<const uint4 *>(skey)[lane + 32 * i];
                if (v.x > kk && v.x < m) m = v.x;
                if (v.y > kk && v.y < m) m = v.y;
                if (v.z > kk && v.z < m) m = v.z;
                if (v.w > kk && v.w < m) m = v.w;
            }
        } else {
#pragma unroll
            for (int i = 0; i < NR / 2; i++) {
                const ulonglong2 v = reinterpret_cast<const ulonglong2 *>(skey)[lane + 32 * i];
                if (v.x > kk && v.x < m) m = v.x;
                if (v.y > kk && v.y < m) m = v.y;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const K v = __shfl_xor_sync(FULL, m, o);
            m = v < m ? v : m;
        }
        if (lane == 0 && m != KINF) {
            atomicMin(&tpend[t], m);
            atomicMin(&runmin[par], m);
        }
    };
    // ---- stage keys and the intensities with a one-voxel halo ----
    const bool full = (x0 + 32 <= X) && (y0 + TY <= Y) && (z0 + TZ <= Z) && ((X & 7) == 0);
    if (full) {
        // 16-byte chunks: CPR per row of 32 keys, NR * CPR / 32 per lane
        constexpr int CPR = 32 * (int)sizeof(K) / 16;
#pragma unroll
        for (int m = 0; m < NR * CPR / 32; m++) {
            const int j = lane + 32 * m, r = j / CPR, col = j % CPR;
            const size_t p0 = (size_t)x0 + (size_t)(y0 + r % TY) * X + (size_t)(z0 + r / TY) * XY;
            cp_async16(reinterpret_cast<uint4 *>(skey) + j,
                       reinterpret_cast<const uint4 *>(keys + p0) + col);
        }
    } else {
#pragma unroll 4
        for (int r = 0; r < NR; r++) {
            const int y = y0 + (r % TY), z = z0 + (r / TY);
            const bool valid = (x < X) && (y < Y) && (z < Z);
            skey[r * 32 + lane] =
                valid ? __ldcg(&keys[(size_t)x + (size_t)y * X + (size_t)z * XY]) : (K)0;
        }
    }
    for (int i = lane; i < HN; i += 32) {
        const int hx = i % 34, hy = (i / 34) % HY, hz = i / (34 * HY);
        const int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - ZO + hz;
        const bool ok = gx >= 0 && gx < X && gy >= 0 && gy < Y && gz >= 0 && gz < Z;
        const size_t g = (size_t)gx + (size_t)gy * X + (size_t)gz * XY;
        if (BLEND) {  // the host checked 0 <= I, g <= 65535
            simg16[i] = ok ? (uint16_t)__ldg(&img[g]) : (uint16_t)0;
            simg16[HN + i] = ok ? (uint16_t)__ldg(&A.gmap[g]) : (uint16_t)0;
        } else {
            simg[i] = ok ? (int32_t)__ldg(&img[g]) : 0;
        }
    }
    if (full) cp_async_wait_all();
    __syncwarp();
    // ---- level rows (lane r < NR keeps row r): at this level, at or below it ----
    uint32_t rowF = 0, rowV = 0;
#pragma unroll
    for (int r = 0; r < NR; r++) {
        const K k = skey[r * 32 + lane];
        const uint32_t bF = __ballot_sync(FULL, k == kk);
        const uint32_t bV = __ballot_sync(FULL, k <= kk);
        if (lane == r) {
            rowF = bF;
            rowV = bV;
        }
    }
    int nf0 = __popc(rowF);
    for (int o = 16; o > 0; o >>= 1) nf0 += __shfl_xor_sync(FULL, nf0, o);
    const long long tcount = OIFT_CLOCK();
    cyc[0] += tcount - tc0;
    if (nf0 == 0) {
        pending();
        cyc[3] += 1;
        return;
    }
    auto append_rows = [&](uint32_t m, int base) -> int {
        const int n = __popc(m);
        int incl = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        int pos = base + incl - n;
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            const int li = (lane << 5) | b;
            wl[pos++] = (uint16_t)li;
            skey[li] = kk;
        }
        return base + total;
    };
    if (lane < NR) nfm[lane] = 0u;
    int cnt = append_rows(rowF, 0);
    __syncwarp();
    int done = 0, rounds = 0;
    while (done < cnt) {
        // ---- one flood round over up to 32 worklist voxels ----
        const int idx = done + lane;
        if (idx < cnt) {
            const int li = wl[idx];
            const int r = li >> 5, xl = li & 31, yl = r % TY, zl = r / TY;
            const int xg = x0 + xl, y = y0 + yl, z = z0 + zl;
            keys[(size_t)xg + (size_t)y * X + (size_t)z * XY] = kexp;
            skey[li] = kexp;
            const int hp = hidx(xl, yl, zl);
#pragma unroll
            for (int dz = (TZ > 1 ? -1 : 0); dz <= (TZ > 1 ? 1 : 0); dz++)
#pragma unroll
                for (int dy = -1; dy <= 1; dy++)
#pragma unroll
                    for (int dx = -1; dx <= 1; dx++) {
                        if (dx == 0 && dy == 0 && dz == 0) continue;
                        // the blend weights and a wide-range 6 / 4 run: the face neighbours
                        if (FACES && (dx != 0) + (dy != 0) + (dz != 0) != 1) continue;
                        const int qxl = xl + dx, qyl = yl + dy, qzl = zl + dz;
                        if (qxl < 0 || qxl >= 32 || qyl < 0 || qyl >= TY || qzl < 0 || qzl >= TZ)
                            continue;  // across the tile boundary: after the flood
                        if (xg + dx >= X || y + dy >= Y || z + dz >= Z) continue;
                        const int lq = (qyl + TY * qzl) * 32 + qxl;
                        const K sk = skey[lq];
                        if (sk <= kk) continue;
                        const int hq = hidx(qxl, qyl, qzl);
                        if (arc_open(hp, hq)) {
                            atomicOr(&nfm[qyl + TY * qzl], 1u << qxl);
                        } else {
                            const K nk = arc_key(hp, hq);
                            if (nk < sk) {
                                atomicMin(&skey[lq], nk);
                                atomicMin(&keys[(size_t)(xg + dx) + (size_t)(y + dy) * X +
                                                (size_t)(z + dz) * XY], nk);
                            }
                        }
                    }
        }
        done = (done + 32 < cnt) ? done + 32 : cnt;
        rounds++;
        __syncwarp();
        uint32_t m = 0;
        if (lane < NR) {
            m = nfm[lane] & ~rowV;
            nfm[lane] = 0u;
            rowV |= m;
        }
        cnt = append_rows(m, cnt);
        __syncwarp();
    }
    // ---- pushes across the tile boundary from every voxel expanded in this step ----
    for (int base = 0; base < cnt; base += 32) {
        const int idx = base + lane;
        if (idx >= cnt) continue;
        const int li = wl[idx];
        const int r = li >> 5, xl = li & 31, yl = r % TY, zl = r / TY;
        const bool edge = xl == 0 || xl == 31 || yl == 0 || yl == TY - 1 ||
                          (TZ > 1 && (zl == 0 || zl == TZ - 1));
        if (!edge) continue;
        const int xg = x0 + xl, y = y0 + yl, z = z0 + zl;
        const int hp = hidx(xl, yl, zl);
#pragma unroll
        for (int dz = (TZ > 1 ? -1 : 0); dz <= (TZ > 1 ? 1 : 0); dz++) {
            K nk[9], old[9];
#pragma unroll
            for (int j = 0; j < 9; j++) {
                const int dy = j / 3 - 1, dx = j % 3 - 1;
                nk[j] = KINF;
                if (FACES && (dx != 0) + (dy != 0) + (dz != 0) != 1) continue;
                const int qxl = xl + dx, qyl = yl + dy, qzl = zl + dz;
                const bool out = qxl < 0 || qxl >= 32 || qyl < 0 || qyl >= TY || qzl < 0 || qzl >= TZ;
                const int qx = xg + dx, qy = y + dy, qz = z + dz;
                if (!out || qx < 0 || qy < 0 || qz < 0 || qx >= X || qy >= Y || qz >= Z) continue;
                nk[j] = arc_key(hp, hidx(qxl, qyl, qzl));
                old[j] = atomicMin(&keys[(size_t)qx + (size_t)qy * X + (size_t)qz * XY], nk[j]);
            }
#pragma unroll
            for (int j = 0; j < 9; j++) {
                if (nk[j] == KINF || !(nk[j] < old[j])) continue;
                const int dy = j / 3 - 1, dx = j % 3 - 1;
                const int qxl = xl + dx, qyl = yl + dy, qzl = zl + dz;
                const int ox = qxl < 0 ? -1 : (qxl >= 32 ? 1 : 0);
                const int oy = qyl < 0 ? -1 : (qyl >= TY ? 1 : 0);
                const int oz = qzl < 0 ? -1 : (qzl >= TZ ? 1 : 0);
                if (nk[j] == kk) {
                    atomicOr(rmask, 1u << ((oz + 1) * 9 + (oy + 1) * 3 + (ox + 1)));
                } else {
                    const int tq = (tx + ox) + (ty + oy) * A.ntx + (tz + oz) * A.ntx * A.nty;
                    atomicMin(&tpend[tq], nk[j]);
                    atomicMin(&runmin[par], nk[j]);
                }
            }
        }
    }
    __syncwarp();
    // ---- publish the same-level re-activations of the neighbour tiles ----
    {
        const uint32_t m = *(volatile uint32_t *)rmask;
        if (m != 0u) {
            __syncwarp();
            if (lane == 0) *rmask = 0u;
            int tq = -1;
            if (lane < 27 && ((m >> lane) & 1u)) {
                const int ox = lane % 3 - 1, oy = (lane / 3) % 3 - 1, oz = lane / 9 - 1;
                tq = (tx + ox) + (ty + oy) * A.ntx + (tz + oz) * A.ntx * A.nty;
            }
            unsigned long long o = 0ull, b = 0ull;
            publish_reactivations(A, par, tq, o, b);
            give_back_duplicates(A, par, o);
        }
    }
    __syncwarp();
    pending();
    cyc[1] += OIFT_CLOCK() - tcount;
    cyc[4] += 1;
    cyc[17] += rounds;
    cyc[18] += cnt;
}



// Re-activation bitmask words per CTA when `nctas` CTAs own `ntiles` tiles round-robin.
__host__ __device__ __forceinline__ int oift_mbox_words_for(int ntiles, int nctas) {
    return ((ntiles + nctas - 1) / nctas + 63) / 64;
}

// Shared-memory working set of one CTA of the persistent kernels.
struct OiftCtaSmem {
    // tiles of this CTA (bit j = tile team_cta + j * nctas) wanted at the current level, and
    // those a warp is processing; a tile is processed by one warp at a time
    unsigned long long want[OIFT_CTA_TILE_WORDS];
#if OIFT_CLAIM_ORDER == 1
    unsigned long long hot[OIFT_CTA_TILE_WORDS];  // wanted tiles that came through the mailbox
#endif
    unsigned long long run[OIFT_CTA_TILE_WORDS];
    int hits;
    int err;
    int fetcher;     // warps that watch the CTA's mailbox and the level's count
    int level_done;  // e + 1 once level e has ended
    unsigned long long blk_min[OIFT_WARPS];  // keys of either width
    unsigned long long level;
    uint32_t wl[OIFT_WARPS][OIFT_WORKLIST];
    uint32_t nfm[OIFT_WARPS][32];  // per row: voxels reached by open arcs in a flood round
    uint32_t rmask[OIFT_WARPS];
};

// The level loop of one OIFT job, run by the `team_ctas` CTAs starting at team CTA index
// `team_cta` (0 .. team_ctas-1).  A.nwarps must equal team_ctas * OIFT_WARPS.
template <int TY, int TZ, bool FULLN = false, typename TI = int16_t, bool BLEND = false,
          typename K = uint32_t, bool FACES = BLEND>
__device__ void oift_solve(const OiftArgs &A, int team_cta, int team_ctas, OiftCtaSmem &cs,
                           unsigned char *smem_raw) {
    const unsigned FULL = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *skey = reinterpret_cast<uint32_t *>(smem_raw) + warp * 1024;
    uint16_t *sw = reinterpret_cast<uint16_t *>(smem_raw + OIFT_WARPS * 4096) + warp * 3072;
    uint16_t *shx = reinterpret_cast<uint16_t *>(smem_raw + OIFT_WARPS * (4096 + 6144)) + warp * 448;
    uint16_t *shy = shx + 64;
    uint16_t *shz = shx + 64 + TZ * 32;  // 64 + 32 (TY + TZ) <= 448 halo codes per warp
    static_assert(FULLN || (TY * TZ == 32 && (TZ == 1 || TY + TZ <= 12)),
                  "the halo codes of a warp tile must fit their 448-entry region");
    static_assert(FULLN || sizeof(K) == 4, "64-bit keys run the full-neighbourhood tile step");
    constexpr K KINF = key_inf_t<K>();
    K *const tpend = tpend_of<K>(A);
    unsigned long long *blk_min = cs.blk_min;
    long long cyc_tile[20];
#pragma unroll
    for (int i = 0; i < 20; i++) cyc_tile[i] = 0;
    uint32_t *rmask = &cs.rmask[warp];
    if (lane == 0) *rmask = 0u;
    for (int i = threadIdx.x; i < OIFT_CTA_TILE_WORDS; i += blockDim.x) {
        cs.want[i] = 0ull;
        cs.run[i] = 0ull;
#if OIFT_CLAIM_ORDER == 1
        cs.hot[i] = 0ull;
#endif
    }
    if (threadIdx.x == 0) {
        cs.hits = 0;
        cs.fetcher = 0;
        cs.level_done = 0;
    }
    __syncthreads();
    uint32_t *wl = cs.wl[warp];
    uint32_t *nfm = cs.nfm[warp];
    OiftGlobals *g = A.g;
    const bool leader_cta = team_cta == 0;
    K prev_level = 0;
    long long lvl_t0 = 0;
    long long cyc_levelsync = 0, cyc_owner = 0, cyc_busy = 0, cyc_drain = 0;
    // ---- the first level: global minimum of the pending keys, one barrier.  Level e then
    // counts its outstanding work in g->outstanding[e % 3] and collects every pending key
    // above it in g->runmin[e % 3], whose value once the count is zero is level e + 1:
    // each CTA moves on as soon as it sees its level end, with no barrier between levels
    // (three slots, so a slot is reset only after every CTA has left the level that used
    // it before) ----
    {
        K m = KINF;
        for (int j = threadIdx.x; team_cta + j * team_ctas < A.ntiles; j += blockDim.x) {
            const K v = __ldcg(&tpend[team_cta + j * team_ctas]);
            m = v < m ? v : m;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const K v = __shfl_xor_sync(FULL, m, o);
            m = v < m ? v : m;
        }
        if (lane == 0) blk_min[warp] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            K bm = (K)blk_min[0];
            for (int w = 1; w < OIFT_WARPS; w++) bm = (K)blk_min[w] < bm ? (K)blk_min[w] : bm;
            if (bm != KINF) atomicMin(first_of<K>(g), bm);
            if (leader_cta) {
                g->outstanding[0] = team_ctas;  // one token per CTA for its scan
                runmin_of<K>(g)[0] = KINF;
            }
        }
        team_barrier(g, A.spin_limit, team_ctas);
        if (threadIdx.x == 0) {
            cs.level = vload(first_of<K>(g));
            cs.err = vload(&g->error);
        }
        __syncthreads();
    }
    for (int e = 0;; e++) {
        const int par = e % 3;
        const long long t_r0 = OIFT_CLOCK();
        if (leader_cta && threadIdx.x == 0 && A.lprof && e > 0 && e - 1 < A.lprof_cap) {
            const long long now = clock64();
            A.lprof[2 * (e - 1)] = (unsigned int)min(now - lvl_t0, 0xffffffffll);
            lvl_t0 = now;
        } else if (leader_cta && threadIdx.x == 0 && e == 0) {
            lvl_t0 = clock64();
        }
        // the level and the error flag were read once for the whole CTA: every warp leaves
        // the loop in the same iteration, so the CTA's barriers stay matched
        const K kk = (K)cs.level;
        if (kk == KINF || cs.err) break;
        // levels strictly increase; a repeat or a runaway level count is a fault
        if ((e > 0 && kk <= prev_level) || e >= A.max_levels) {
            if (threadIdx.x == 0) atomicCAS(&g->error, 0, OIFT_DEV_TIMEOUT);
            break;
        }
        prev_level = kk;
        if (leader_cta && threadIdx.x == 0) g->levels = e + 1;
        const int c = key_level_cost_t<K>(kk), l = key_label_t<K>(kk);
        // the largest base weight of the run bounds the per-level thresholds
        const int maxb = sizeof(K) == 8 ? A.wcap : OIFT_MAX_BASE;
        const double per = (double)polarity_of(A, l);
        double fgt, flt;
        int bgt, blt;
        if (A.ig) {  // Orient2Digraph: float alpha = per / 100.0, val * (1.0 +/- alpha)
            const float alpha = (float)(per / 100.0);
            fgt = 1.0 + (double)alpha;
            flt = 1.0 - (double)alpha;
            bgt = max_base_for_cost_round(c, fgt, maxb);
            blt = max_base_for_cost_round(c, flt, maxb);
        } else {
            fgt = 1.0 + per / 100.0;
            flt = 1.0 - per / 100.0;
            bgt = max_base_for_cost(c, fgt, maxb);
            blt = max_base_for_cost(c, flt, maxb);
        }
        // ---- S: the tiles of this CTA whose pending key equals the level become wanted; the
        // smallest pending key of its other tiles joins the level's running minimum ----
        unsigned long long steps = 0;
        const long long t_s0 = OIFT_CLOCK();
        cyc_levelsync += t_s0 - t_r0;
        {
            int h = 0;
            K m = KINF;
            for (int j = threadIdx.x; team_cta + j * team_ctas < A.ntiles; j += blockDim.x) {
                const int t = team_cta + j * team_ctas;
                const K v = __ldcg(&tpend[t]);
                if (v == kk) {
                    tpend[t] = KINF;
                    atomicOr(&cs.want[j >> 6], 1ull << (j & 63));
                    h++;
                } else if (v < m) {
                    m = v;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                h += __shfl_xor_sync(FULL, h, o);
                const K v = __shfl_xor_sync(FULL, m, o);
                m = v < m ? v : m;
            }
            if (lane == 0) {
                if (h) atomicAdd(&cs.hits, h);
                blk_min[warp] = m;
            }
            if (threadIdx.x == 0) cs.fetcher = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (leader_cta) {  // the slot of the next level, free since every CTA left e - 2
                g->outstanding[(e + 1) % 3] = team_ctas;
                runmin_of<K>(g)[(e + 1) % 3] = KINF;
            }
            K bm = (K)blk_min[0];
            for (int w = 1; w < OIFT_WARPS; w++) bm = (K)blk_min[w] < bm ? (K)blk_min[w] : bm;
            if (bm != KINF) atomicMin(&runmin_of<K>(g)[par], bm);
            // the resets and the running minimum precede any count of this CTA given back
            __threadfence();
            // the CTA's token of the level becomes one count per wanted tile, before any of
            // them can be claimed and counted off
            const int h = cs.hits;
            cs.hits = 0;
            if (h != 1) atomicAdd(&g->outstanding[par], h - 1);
        }
        __syncthreads();
        const long long t_p0 = OIFT_CLOCK();
        cyc_owner += t_p0 - t_s0;
        // ---- P: the CTA's warps claim its wanted tiles, one warp per tile, and fetch the
        // CTA's mailbox into the wanted set, until the level's outstanding count is zero ----
        unsigned long long *ctabox = A.mbox + ((size_t)par * team_ctas + team_cta) * A.mbox_words;
        const int words = A.mbox_words;
        long long spins = 0;
        int idle = 0;
        bool fetcher = false;
        unsigned nap = 64;  // sleep of an idle warp that does not watch, doubled while idle
        for (;;) {
            // claim: the first lane that sees a wanted tile no warp is processing takes it
            // with an atomic OR on the running set; a lost race looks again
            int j = -1;
#if OIFT_CLAIM_ORDER == 1
            // tiles re-activated through the mailbox first (the flood's continuation)
            for (int w0 = 0; w0 < words && j < 0; w0 += 32) {
                const int w = w0 + lane;
                const unsigned long long avail =
                    w < words ? (vload(&cs.hot[w]) & vload(&cs.want[w]) & ~vload(&cs.run[w])) : 0ull;
                const uint32_t have = __ballot_sync(FULL, avail != 0ull);
                if (!have) continue;
                const int src = __ffs(have) - 1;
                int got = -1;
                if (lane == src) {
                    const int b = __ffsll((long long)avail) - 1;
                    const unsigned long long bit = 1ull << b;
                    if (!(atomicOr(&cs.run[w], bit) & bit)) {
                        atomicAnd(&cs.want[w], ~bit);
                        atomicAnd(&cs.hot[w], ~bit);
                        got = w * 64 + b;
                    }
                }
                j = __shfl_sync(FULL, got, src);
            }
#endif
            for (int w0 = 0; w0 < words && j < 0;) {
                const int w = w0 + lane;
                const unsigned long long avail =
                    w < words ? (vload(&cs.want[w]) & ~vload(&cs.run[w])) : 0ull;
                const uint32_t have = __ballot_sync(FULL, avail != 0ull);
                if (!have) {
                    w0 += 32;
                    continue;
                }
                const int src = __ffs(have) - 1;
                int got = -1;
                if (lane == src) {
                    const int b = __ffsll((long long)avail) - 1;
                    const unsigned long long bit = 1ull << b;
                    if (!(atomicOr(&cs.run[w], bit) & bit)) {
                        atomicAnd(&cs.want[w], ~bit);
#if OIFT_CLAIM_ORDER == 1
                        atomicAnd(&cs.hot[w], ~bit);
#endif
                        got = w * 64 + b;
                    }
                }
                j = __shfl_sync(FULL, got, src);
            }
            if (j >= 0) {
                if (fetcher) {  // another idle warp takes over the watch while this one works
                    if (lane == 0) atomicSub(&cs.fetcher, 1);
                    fetcher = false;
                }
                // the activations merged into this claim precede the staging of the tile
                __threadfence_block();
                const long long tb = OIFT_CLOCK();
                const int t = team_cta + j * team_ctas;
                if constexpr (FULLN)
                    process_tile_full<TY, TZ, TI, BLEND, K, FACES>(
                        A, t, par, kk, c, l, fgt, flt, bgt, blt, reinterpret_cast<K *>(skey),
                        reinterpret_cast<int32_t *>(sw), reinterpret_cast<uint16_t *>(wl), nfm,
                        rmask, cyc_tile);
                else
                    process_tile<TY, TZ>(A, t, par, kk, c, l, fgt, flt, bgt, blt, skey, sw, shx,
                                         shy, shz, wl, nfm, rmask, cyc_tile);
                steps++;
                fence_acq_rel_gpu();  // the tile step's writes precede the release and count
                __syncwarp();
                if (lane == 0) {
                    atomicAnd(&cs.run[j >> 6], ~(1ull << (j & 63)));
                    atomicSub(&g->outstanding[par], 1);
                }
                cyc_busy += OIFT_CLOCK() - tb;
                spins = 0;
                idle = 0;
                nap = 64;
                continue;
            }
            // no wanted tile is free.  Up to OIFT_FETCHERS warps of the CTA at a time (the
            // fetchers) watch the CTA's mailbox and the level's outstanding count and publish
            // the level's end in shared memory; the others watch only the CTA's shared state.
            int done = 0;
            if (lane == 0) done = vload(&cs.level_done) == e + 1;
            done = __shfl_sync(FULL, done, 0);
            if (done) break;
            if (!fetcher) {
                int got = 0;
                if (lane == 0) {
                    const int f = vload(&cs.fetcher);
                    got = f < OIFT_FETCHERS && atomicCAS(&cs.fetcher, f, f + 1) == f;
                }
                fetcher = __shfl_sync(FULL, got, 0) != 0;
            }
            if (fetcher) {
                // fetch: the CTA's mailbox bits join the wanted set; bits already wanted merge
                // into the pending activation and give their count back.  The level's
                // outstanding count and the error flag are read in the same round trip.
                int outst = 1, errf = 0;
                if (lane == 0) {
                    outst = vload(&g->outstanding[par]);
                    errf = vload(&g->error);
                }
                bool fetched = false;
                for (int w0 = 0; w0 < words; w0 += 32) {
                    const int w = w0 + lane;
                    unsigned long long b = 0ull;
                    if (w < words) b = exch_acquire_gpu(&ctabox[w], 0ull);
                    if (b) {
                        __threadfence_block();
#if OIFT_CLAIM_ORDER == 1
                        atomicOr(&cs.hot[w], b);
#endif
                        const unsigned long long old = atomicOr(&cs.want[w], b);
                        const int dups = __popcll(old & b);
                        if (dups) atomicSub(&g->outstanding[par], dups);
                    }
                    fetched |= __any_sync(FULL, b != 0ull);
                }
                if (fetched) {
                    spins = 0;
                    idle = 0;
                    continue;
                }
                if (lane == 0) {
                    done = outst == 0 || errf != 0;
                    if (!done && ++spins > A.spin_limit) {
                        atomicCAS(&g->error, 0, OIFT_DEV_TIMEOUT);
                        done = 1;
                    }
                    if (done) {
                        // every key the level's tile steps left pending reached the running
                        // minimum before their counts were given back: it is the next level
                        fence_acq_rel_gpu();
                        cs.level = vload(&runmin_of<K>(g)[par]);
                        cs.err = vload(&g->error);
                        __threadfence_block();
                        *(volatile int *)&cs.level_done = e + 1;
                        atomicExch(&cs.fetcher, 0);
                    }
                }
            } else if (lane == 0 && ++spins > A.spin_limit) {
                atomicCAS(&g->error, 0, OIFT_DEV_TIMEOUT);
                done = 1;
            }
            idle++;
            done = __shfl_sync(FULL, done, 0);
            if (done) break;
            if (!fetcher) {
                __nanosleep(nap);
                nap = nap * 2 < OIFT_IDLE_NS_MAX ? nap * 2 : OIFT_IDLE_NS_MAX;
            }
        }
        if (lane == 0 && steps) atomicAdd(&g->tile_steps, steps);
        if (lane == 0 && steps && A.lprof && e < A.lprof_cap)
            atomicAdd(&A.lprof[2 * e + 1], (unsigned int)steps);
        cyc_drain += OIFT_CLOCK() - t_p0;
        // every warp has left the level; a warp whose own wait ran out has set the error
        // flag, which the watching warp reads before it ends the level
        __syncthreads();
    }
    if (lane == 0) {
        atomicAdd(&g->cycles[0], (unsigned long long)cyc_levelsync);
        atomicAdd(&g->cycles[1], (unsigned long long)cyc_owner);
        atomicAdd(&g->cycles[2], (unsigned long long)cyc_busy);
        atomicAdd(&g->cycles[3], (unsigned long long)cyc_drain);
        for (int i = 0; i < 20; i++) atomicAdd(&g->cycles[4 + i], (unsigned long long)cyc_tile[i]);
    }
}

template <int TY, int TZ, bool FULLN = false, typename TI = int16_t, bool BLEND = false,
          typename K = uint32_t, bool FACES = BLEND>
__global__ void __launch_bounds__(OIFT_WARPS * 32, 1) oift_persistent_kernel(OiftArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ OiftCtaSmem cs;
    __shared__ int s_bad;
    // a bad seed (flagged by the seeds kernel queued before) ends the launch at once; the
    // host reads the flag with the launch's outcome
    if (threadIdx.x == 0) s_bad = A.seed_flag ? *(volatile const int *)A.seed_flag : 0;
    __syncthreads();
    if (s_bad) return;
    oift_solve<TY, TZ, FULLN, TI, BLEND, K, FACES>(A, blockIdx.x, gridDim.x, cs, smem_raw);
}

// Batched OIFT: CTA b belongs to team b / team_ctas.  A team draws jobs from a shared
// counter until none is left; per job it clears its key / pending / mailbox arrays, places
// the seeds, runs the level loop of oift_solve over its own CTAs and writes cost and label.
// Five team barriers per job separate the phases.  An error inside the level loop (a
// bounded wait that expired, a worklist overflow) leaves the team's barrier state
// unusable, so the team records it in the job, sets the abort flag and stops; jobs that no
// team ended keep status OIFT_TEAM_NOT_RUN.
template <int TY, int TZ>
__global__ void __launch_bounds__(OIFT_WARPS * 32, 1)
    oift_team_kernel(OiftTeamJob *jobs, int njobs, int teams, OiftTeamScratch S,
                     long long spin_limit, int max_levels) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ OiftCtaSmem cs;
    __shared__ OiftArgs sA;
    __shared__ int s_job, s_bad;
    // team t owns CTAs [t*G/T, (t+1)*G/T): sizes differ by at most one CTA
    const unsigned G = gridDim.x, T = (unsigned)teams;
    const int team = (int)(((blockIdx.x + 1) * T - 1) / G);
    const int cta0 = (int)((unsigned long long)team * G / T);
    const int team_ctas = (int)((unsigned long long)(team + 1) * G / T) - cta0;
    const int tc = blockIdx.x - cta0;
    OiftGlobals *g = S.g + team;
    uint32_t *key = S.key + (size_t)team * S.key_stride;
    uint32_t *tpend = S.tpend + (size_t)team * S.tpend_stride;
    unsigned long long *mbox = S.mbox + (size_t)team * S.mbox_stride;
    const size_t tid = (size_t)tc * blockDim.x + threadIdx.x;
    const size_t nthr = (size_t)team_ctas * blockDim.x;
    const bool leader = tc == 0 && threadIdx.x == 0;
    for (;;) {
        // ---- the leader draws a job and clears the per-job globals ----
        if (leader) {
            g->job = vload(S.abort) ? njobs : (int)atomicAdd(S.next_job, 1u);
            g->first = OIFT_KEY_INF;
            g->levels = 0;
            g->tile_steps = 0;
            g->bad_seed = 0;
        }
        if (!team_barrier(g, spin_limit, team_ctas)) break;
        if (threadIdx.x == 0) s_job = vload(&g->job);
        __syncthreads();
        const int j = s_job;
        if (j >= njobs) break;
        OiftTeamJob *J = jobs + j;
        const int X = J->X, Y = J->Y, Z = J->Z, ntx = J->ntx, nty = J->nty;
        const int ntiles = J->ntiles;
        const int mbox_words = oift_mbox_words_for(ntiles, team_ctas);
        if (mbox_words > OIFT_CTA_TILE_WORDS) {  // the job needs a team of more CTAs
            if (leader) J->status = OIFT_E_UNSUPPORTED;
            continue;
        }
        const size_t N = (size_t)X * Y * Z;
        if (threadIdx.x == 0) {
            sA.key = key;
            sA.W = J->W;
            sA.tpend = tpend;
            sA.mbox = mbox;
            sA.lprof = nullptr;
            sA.lprof_cap = 0;
            sA.mbox_words = mbox_words;
            sA.nwarps = team_ctas * OIFT_WARPS;
            sA.nctas = team_ctas;
            sA.X = X;
            sA.Y = Y;
            sA.Z = Z;
            sA.N = N;
            sA.ntx = ntx;
            sA.fd_ntx = make_fastdiv((uint32_t)ntx);
            sA.fd_ntxy = make_fastdiv((uint32_t)(ntx * nty));
            sA.fd_nctas = make_fastdiv((uint32_t)team_ctas);
            sA.nty = nty;
            sA.ntz = J->ntz;
            sA.ntiles = ntiles;
            sA.pol_table = &J->pol0;
            sA.npol = 1;
            sA.pol_default = J->pol_default;
            sA.g = g;
            sA.spin_limit = spin_limit;
            sA.max_levels = max_levels;
            sA.ig = 0;
            sA.Wt = nullptr;
        }
        // ---- clear the team's state for this volume ----
        for (size_t i = tid; i < N; i += nthr) key[i] = OIFT_KEY_INF;
        for (size_t i = tid; i < (size_t)ntiles; i += nthr) tpend[i] = OIFT_KEY_INF;
        const size_t nmb = (size_t)3 * team_ctas * mbox_words;
        for (size_t i = tid; i < nmb; i += nthr) mbox[i] = 0ull;
        if (!team_barrier(g, spin_limit, team_ctas)) break;
        // ---- seeds (as oift_seed_kernel) ----
        for (size_t i = tid; i < (size_t)J->nseeds; i += nthr) {
            const int p = J->seeds[i];
            const int lb0 = J->seed_labels[i];
            const int lb = lb0 < 0 ? 0 : lb0;
            if (p < 0 || (size_t)p >= N) {
                atomicExch(&g->bad_seed, OIFT_E_SEED_RANGE);
                continue;
            }
            if (lb > OIFT_MAX_LABEL) {
                atomicExch(&g->bad_seed, OIFT_E_BAD_ARG);
                continue;
            }
            const uint32_t k = seed_key(lb);
            atomicMin(&key[p], k);
            const int x = p % X, y = (p / X) % Y, z = (int)(p / ((size_t)X * Y));
            atomicMin(&tpend[(x >> 5) + (y / TY) * ntx + (z / TZ) * ntx * nty], k);
        }
        if (!team_barrier(g, spin_limit, team_ctas)) break;
        if (threadIdx.x == 0) s_bad = vload(&g->bad_seed);
        __syncthreads();
        const int bad = s_bad;
        if (!bad) oift_solve<TY, TZ>(sA, tc, team_ctas, cs, smem_raw);
        const bool ok = team_barrier(g, spin_limit, team_ctas);
        const int err = vload(&g->error);
        if (!ok || err) {
            if (leader)
                J->status = err == OIFT_DEV_QUEUE ? OIFT_E_QUEUE_OVERFLOW : OIFT_E_NOT_CONVERGED;
            if (threadIdx.x == 0) atomicExch(S.abort, 1);
            break;
        }
        // ---- cost and label (as oift_finalize_kernel) ----
        if (!bad) {
            int32_t *cost = J->cost, *label = J->label;
            for (size_t i = tid; i < N; i += nthr) {
                const uint32_t k = __ldcg(&key[i]);
                if (cost) cost[i] = (k == OIFT_KEY_INF) ? 0x7fffffff : key_cost(k);
                if (label) label[i] = (k == OIFT_KEY_INF) ? -1 : key_label(k);
            }
        }
        if (leader) {
            J->levels = g->levels;
            J->steps = g->tile_steps;
            J->status = bad ? bad : OIFT_OK;
        }
    }
}

template <typename K>
__global__ void oift_seed_kernel(K *key, K *tpend, const int32_t *seeds,
                                 const int32_t *labels, int nseeds, int X, int Y, int Z,
                                 int ntx, int nty, int TY, int TZ, int *bad) {
    // every lane of the warp reaches the tile aggregation below (no early return)
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t N = (size_t)X * Y * Z;
    int t = -1;
    K k = key_inf_t<K>();
    if (i < nseeds) {
        const int p = seeds[i];
        const int lb = labels[i] < 0 ? 0 : labels[i];
        if (p < 0 || (size_t)p >= N) {
            atomicExch(bad, 1);
        } else if (lb > OIFT_MAX_LABEL) {
            atomicExch(bad, 2);
        } else {
            k = seed_key_t<K>(lb);
            atomicMin(&key[p], k);
            const int x = p % X, y = (p / X) % Y, z = (int)(p / ((size_t)X * Y));
            t = (x >> 5) + (y / TY) * ntx + (z / TZ) * ntx * nty;
        }
    }
    // seed lists in address order put many seeds of a warp in one tile: one pending-key
    // update per tile and warp (64-bit keys, which have no warp reduction: one per seed)
    if constexpr (sizeof(K) == 8) {
        if (t >= 0) atomicMin(&tpend[t], k);
        return;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, t);
    const K km = __reduce_min_sync(peers, (uint32_t)k);
    if (t >= 0 && (__ffs(peers) - 1) == (int)(threadIdx.x & 31)) atomicMin(&tpend[t], km);
}

template <typename K>
__global__ void oift_finalize_kernel(const K *key, size_t n, int32_t *cost, int32_t *label) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const K k = key[i];
        if (cost) cost[i] = (k == key_inf_t<K>()) ? 0x7fffffff : key_cost_t<K>(k);
        if (label) label[i] = (k == key_inf_t<K>()) ? -1 : key_label_t<K>(k);
    }
}

// ------------------------------------------------------------------ host side ----

OiftPlan oift_plan_full(int X, int Y, int Z) {
    OiftPlan P;
    if (Z == 1) {
        P.TY = 16;
        P.TZ = 1;
    } else {
        P.TY = 4;
        P.TZ = 4;
    }
    P.ntx = (X + 31) / 32;
    P.nty = (Y + P.TY - 1) / P.TY;
    P.ntz = (Z + P.TZ - 1) / P.TZ;
    P.ntiles = P.ntx * P.nty * P.ntz;
    P.qcap = 0;
    return P;
}

OiftPlan oift_plan(int X, int Y, int Z, int tile_ty) {
    OiftPlan P;
    if (Z == 1) {
        P.TY = 32;
        P.TZ = 1;
    } else if (tile_ty == 4) {
        P.TY = 4;
        P.TZ = 8;
    } else {
        P.TY = 8;
        P.TZ = 4;
    }
    P.ntx = (X + 31) / 32;
    P.nty = (Y + P.TY - 1) / P.TY;
    P.ntz = (Z + P.TZ - 1) / P.TZ;
    P.ntiles = P.ntx * P.nty * P.ntz;
    P.qcap = 0;
    return P;
}

size_t oift_smem_bytes() { return (size_t)OIFT_WARPS * (4096 + 6144 + 896); }


size_t oift_globals_bytes() { return sizeof(OiftGlobals); }
int oift_mbox_words(const OiftPlan &P, int ctas) {
    return oift_mbox_words_for(P.ntiles, ctas);
}
// one mailbox per CTA for each of the three level slots
size_t oift_mbox_bytes(const OiftPlan &P, int ctas) {
    return (size_t)3 * ctas * oift_mbox_words(P, ctas) * sizeof(unsigned long long);
}
int oift_min_ctas(const OiftPlan &P) {
    const int per = OIFT_CTA_TILE_WORDS * 64;
    int n = (P.ntiles + per - 1) / per;
    while (oift_mbox_words(P, n) > OIFT_CTA_TILE_WORDS) n++;
    return n;
}

// Queues the seeds kernel, the persistent kernel and (optionally) the finalize kernel with
// no host synchronisation: a bad seed stops the persistent kernel at its start.  The
// outcome is in the globals S.g and the seed flag d_flag, which oift_result interprets
// once they are on the host.
int oift_enqueue(const OiftPlan &P, const OiftScratch &S, const uint16_t *W, int X, int Y,
                 int Z, const int32_t *d_seeds, const int32_t *d_seed_labels, int nseeds,
                 const float *d_pol_table, int npol, float pol_default, int32_t *cost,
                 int32_t *label, int *d_flag, int sms, cudaStream_t st, cudaEvent_t ev_begin,
                 cudaEvent_t ev_end, const OiftFullN *fn, bool round_orient,
                 const uint16_t *Wt) {
    size_t N = (size_t)X * Y * Z;
    // a wide-range run keeps 64-bit keys and pending keys at the scratch addresses
    const bool wide = fn && fn->wide;
    const size_t ksz = wide ? sizeof(unsigned long long) : sizeof(uint32_t);
    unsigned long long *key64 = wide ? reinterpret_cast<unsigned long long *>(S.key) : nullptr;
    unsigned long long *tpend64 = wide ? reinterpret_cast<unsigned long long *>(S.tpend) : nullptr;
    cudaMemsetAsync(S.key, 0xFF, N * ksz, st);
    cudaMemsetAsync(S.tpend, 0xFF, (size_t)P.ntiles * ksz, st);
    cudaMemsetAsync(S.mbox, 0, oift_mbox_bytes(P, sms), st);
    cudaMemsetAsync(S.g, 0, sizeof(OiftGlobals), st);
    cudaMemsetAsync(&S.g->first, 0xFF, sizeof(S.g->first), st);
    cudaMemsetAsync(&S.g->first64, 0xFF, sizeof(S.g->first64), st);
    cudaMemsetAsync(d_flag, 0, sizeof(int), st);
    if (nseeds > 0) {
        if (wide)
            oift_seed_kernel<unsigned long long><<<(nseeds + 255) / 256, 256, 0, st>>>(
                key64, tpend64, d_seeds, d_seed_labels, nseeds, X, Y, Z, P.ntx, P.nty, P.TY, P.TZ,
                d_flag);
        else
            oift_seed_kernel<uint32_t><<<(nseeds + 255) / 256, 256, 0, st>>>(
                S.key, S.tpend, d_seeds, d_seed_labels, nseeds, X, Y, Z, P.ntx, P.nty, P.TY, P.TZ,
                d_flag);
    }

    OiftArgs A;
    A.key = S.key;
    A.W = W;
    A.tpend = S.tpend;
    A.key64 = key64;
    A.tpend64 = tpend64;
    A.mbox = S.mbox;
    A.lprof = S.lprof;
    A.lprof_cap = S.lprof_cap;
    if (S.lprof) cudaMemsetAsync(S.lprof, 0, (size_t)S.lprof_cap * 2 * sizeof(unsigned int), st);
    A.nwarps = sms * OIFT_WARPS;
    A.nctas = sms;
    A.mbox_words = oift_mbox_words(P, sms);
    if (A.mbox_words > OIFT_CTA_TILE_WORDS) return OIFT_E_UNSUPPORTED;
    A.X = X;
    A.Y = Y;
    A.Z = Z;
    A.N = N;
    A.ntx = P.ntx;
    A.nty = P.nty;
    A.ntz = P.ntz;
    A.ntiles = P.ntiles;
    A.fd_ntx = make_fastdiv((uint32_t)P.ntx);
    A.fd_ntxy = make_fastdiv((uint32_t)(P.ntx * P.nty));
    A.fd_nctas = make_fastdiv((uint32_t)sms);
    A.pol_table = d_pol_table;
    A.npol = npol;
    A.pol_default = pol_default;
    A.g = S.g;
    A.spin_limit = S.spin_limit;
    A.max_levels = S.max_levels;
    A.img = fn ? fn->img : nullptr;
    A.wmode = fn ? fn->wmode : 0;
    A.wcap = fn ? fn->wcap : OIFT_MAX_BASE;
    A.lut = fn ? fn->lut : nullptr;
    A.lut_len = fn ? fn->lut_len : 0;
    A.gmap = fn ? fn->gmap : nullptr;
    A.alpha = fn ? fn->alpha : 1.0f;
    A.ig = round_orient ? 1 : 0;
    A.Wt = fn ? nullptr : Wt;
    A.seed_flag = d_flag;
    size_t smem = oift_smem_bytes();
    void *args[] = {&A};
    cudaError_t err;
    if (ev_begin) cudaEventRecord(ev_begin, st);
    auto launch = [&](const void *kfn) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        return cudaLaunchCooperativeKernel(kfn, dim3(sms), dim3(OIFT_WARPS * 32), args, smem, st);
    };
    using u64 = unsigned long long;
    if (wide) {
        if (P.TZ == 1) {
            if (fn->faces)
                err = fn->img_i16 ? launch((const void *)oift_persistent_kernel<16, 1, true, int16_t, false, u64, true>)
                                  : launch((const void *)oift_persistent_kernel<16, 1, true, int32_t, false, u64, true>);
            else
                err = fn->img_i16 ? launch((const void *)oift_persistent_kernel<16, 1, true, int16_t, false, u64, false>)
                                  : launch((const void *)oift_persistent_kernel<16, 1, true, int32_t, false, u64, false>);
        } else {
            if (fn->faces)
                err = fn->img_i16 ? launch((const void *)oift_persistent_kernel<4, 4, true, int16_t, false, u64, true>)
                                  : launch((const void *)oift_persistent_kernel<4, 4, true, int32_t, false, u64, true>);
            else
                err = fn->img_i16 ? launch((const void *)oift_persistent_kernel<4, 4, true, int16_t, false, u64, false>)
                                  : launch((const void *)oift_persistent_kernel<4, 4, true, int32_t, false, u64, false>);
        }
    } else if (fn && fn->blend) {
        if (P.TZ == 1)
            err = fn->img_i16 ? launch((const void *)oift_persistent_kernel<16, 1, true, int16_t, true>)
                              : launch((const void *)oift_persistent_kernel<16, 1, true, int32_t, true>);
        else
            err = fn->img_i16 ? launch((const void *)oift_persistent_kernel<4, 4, true, int16_t, true>)
                              : launch((const void *)oift_persistent_kernel<4, 4, true, int32_t, true>);
    } else if (fn) {
        if (P.TZ == 1)
            err = fn->img_i16 ? launch((const void *)oift_persistent_kernel<16, 1, true, int16_t>)
                              : launch((const void *)oift_persistent_kernel<16, 1, true, int32_t>);
        else
            err = fn->img_i16 ? launch((const void *)oift_persistent_kernel<4, 4, true, int16_t>)
                              : launch((const void *)oift_persistent_kernel<4, 4, true, int32_t>);
    } else if (P.TZ == 1) {
        err = launch((const void *)oift_persistent_kernel<32, 1>);
    } else {
        err = launch((const void *)oift_persistent_kernel<8, 4>);
    }
    if (err != cudaSuccess) return OIFT_E_CUDA;
    if (ev_end) cudaEventRecord(ev_end, st);
    if (cost || label) {
        int blocks = (int)((N + 255) / 256);
        if (blocks > sms * 16) blocks = sms * 16;
        if (wide)
            oift_finalize_kernel<unsigned long long><<<blocks, 256, 0, st>>>(key64, N, cost, label);
        else
            oift_finalize_kernel<uint32_t><<<blocks, 256, 0, st>>>(S.key, N, cost, label);
    }
    return cudaGetLastError() == cudaSuccess ? OIFT_OK : OIFT_E_CUDA;
}

int oift_result(const OiftGlobals &hg, int seed_flag, int *levels_out, long long *steps_out,
                unsigned long long *cycles_out) {
    if (seed_flag == 1) return OIFT_E_SEED_RANGE;
    if (seed_flag == 2) return OIFT_E_BAD_ARG;
    if (levels_out) *levels_out = hg.levels;
    if (steps_out) *steps_out = (long long)hg.tile_steps;
    if (cycles_out)
        for (int i = 0; i < 24; i++) cycles_out[i] = hg.cycles[i];
    if (hg.error == OIFT_DEV_TIMEOUT) return OIFT_E_NOT_CONVERGED;
    if (hg.error == OIFT_DEV_QUEUE) return OIFT_E_QUEUE_OVERFLOW;
    return OIFT_OK;
}

// oift_enqueue, then a synchronous read of the outcome.
int oift_run(const OiftPlan &P, const OiftScratch &S, const uint16_t *W, int X, int Y, int Z,
             const int32_t *d_seeds, const int32_t *d_seed_labels, int nseeds,
             const float *d_pol_table, int npol, float pol_default, int32_t *cost,
             int32_t *label, int *d_flag, int sms, cudaStream_t st, int *levels_out,
             long long *steps_out, cudaEvent_t ev_begin, cudaEvent_t ev_end,
             unsigned long long *cycles_out, const OiftFullN *fn, bool round_orient,
             const uint16_t *Wt) {
    const int rc = oift_enqueue(P, S, W, X, Y, Z, d_seeds, d_seed_labels, nseeds, d_pol_table,
                                npol, pol_default, cost, label, d_flag, sms, st, ev_begin, ev_end,
                                fn, round_orient, Wt);
    if (rc != OIFT_OK) return rc;
    OiftGlobals hg;
    int hflag = 0;
    cudaMemcpyAsync(&hg, S.g, sizeof(OiftGlobals), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&hflag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return OIFT_E_CUDA;
    return oift_result(hg, hflag, levels_out, steps_out, cycles_out);
}

int oift_team_run(OiftTeamJob *d_jobs, int njobs, bool planar, int teams, int ctas,
                  const OiftTeamScratch &S, cudaStream_t st, int tile_ty) {
    if (njobs <= 0) return OIFT_OK;
    if (teams <= 0 || ctas < teams) return OIFT_E_BAD_ARG;
    if (cudaMemsetAsync(S.g, 0, (size_t)teams * sizeof(OiftGlobals), st) != cudaSuccess ||
        cudaMemsetAsync(S.next_job, 0, sizeof(unsigned int), st) != cudaSuccess ||
        cudaMemsetAsync(S.abort, 0, sizeof(int), st) != cudaSuccess) {
        cudaGetLastError();
        return OIFT_E_CUDA;
    }
    long long spin_limit = S.spin_limit;
    int max_levels = S.max_levels;
    int nt = teams;
    OiftTeamScratch sc = S;
    void *args[] = {&d_jobs, &njobs, &nt, &sc, &spin_limit, &max_levels};
    const size_t smem = oift_smem_bytes();
    // cooperative launch through the launch-attribute API, which a stream capture records as
    // a cooperative kernel node
    auto launch = [&](const void *kfn) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(ctas);
        cfg.blockDim = dim3(OIFT_WARPS * 32);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        return cudaLaunchKernelExC(&cfg, kfn, args);
    };
    cudaError_t err = planar ? launch((const void *)oift_team_kernel<32, 1>)
                      : tile_ty == 4 ? launch((const void *)oift_team_kernel<4, 8>)
                                     : launch((const void *)oift_team_kernel<8, 4>);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return OIFT_E_CUDA;
    }
    return OIFT_OK;
}

}  // namespace oiftb

#if OIFT_PROBE
extern "C" __attribute__((visibility("default"))) int oift_b200_probe_read(unsigned long long *out) {
    cudaMemcpyFromSymbol(out, oiftb::g_probe, sizeof(oiftb::g_probe));
    cudaMemcpyFromSymbol(out + 8, oiftb::g_hist, sizeof(oiftb::g_hist));
    static unsigned long long z[8 + 96];
    cudaMemcpyToSymbol(oiftb::g_hist, z, sizeof(oiftb::g_hist));
    return (int)cudaMemcpyToSymbol(oiftb::g_probe, z, sizeof(oiftb::g_probe));
}
#endif
