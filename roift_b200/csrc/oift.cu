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
// Execution: ONE persistent cooperative launch, 16 warps per SM.  The volume is cut into
// warp tiles of 32 (x) x TY (y) x TZ (z) voxels, TY*TZ = 32 rows: a lane owns one row as
// a 32-bit mask.  Per level:
//   R  every warp reduces its share of the per-tile pending minima -> global level key;
//      one grid barrier;
//   S  tiles whose pending key equals the level are queued (device work queue);
//   P  warps pop tiles: load keys + edge codes of the tile (coalesced rows), build the
//      "arc may be used at this level" masks with a per-level base-weight threshold,
//      flood the level inside the tile with bit operations and warp shuffles, then
//      expand the newly conquered voxels: in-tile neighbours get tentative keys, out-of-
//      tile neighbours are lowered with a 32-bit atomicMin; a same-level crossing
//      re-queues the neighbour tile, a higher one lowers its pending key.
// The level ends when the queue is empty and no tile is in flight (outstanding counter).
// Every wait (grid barrier, queue slot, level end) is bounded; on expiry the kernel sets
// an error flag, every warp leaves, and the host reports OIFT_E_NOT_CONVERGED.
#include <cooperative_groups.h>

#include "kernels.cuh"

namespace oiftb {


struct OiftArgs {
    uint32_t *key;
    const uint16_t *W;
    uint32_t *tpend;
    uint32_t *inq;
    uint32_t *queue;
    unsigned int qmask;
    int X, Y, Z;
    size_t N;
    int ntx, nty, ntz, ntiles;
    const float *pol_table;  // device, per label (x100)
    int npol;
    float pol_default;
    OiftGlobals *g;
    long long spin_limit;
    int max_levels;
};

constexpr int OIFT_WARPS = 16;
constexpr uint32_t QEMPTY = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned int vload(const volatile unsigned int *p) { return *p; }
__device__ __forceinline__ int vload(const volatile int *p) { return *p; }
__device__ __forceinline__ unsigned long long vload(const volatile unsigned long long *p) {
    return *p;
}

// Grid barrier for the cooperative launch, with a bounded wait.
__device__ bool grid_barrier(OiftGlobals *g, long long limit) {
    __syncthreads();
    bool ok = true;
    if (threadIdx.x == 0) {
        unsigned int gen = vload(&g->bar_gen);
        __threadfence();
        if (atomicAdd(&g->bar_count, 1u) == gridDim.x - 1) {
            g->bar_count = 0;
            __threadfence();
            atomicAdd(&g->bar_gen, 1u);
        } else {
            long long spins = 0;
            while (vload(&g->bar_gen) == gen) {
                if (vload(&g->error)) break;
                if (++spins > limit) {
                    atomicCAS(&g->error, 0, OIFT_DEV_TIMEOUT);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok;
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

__device__ __forceinline__ void enqueue_tile(const OiftArgs &A, int par, int t) {
    if (atomicExch(&A.inq[t], 1u) == 0u) {
        atomicAdd(&A.g->outstanding[par], 1);
        __threadfence();  // key updates that caused the queueing are visible first
        unsigned long long slot = atomicAdd(&A.g->qtail, 1ULL);
        atomicExch(&A.queue[slot & A.qmask], (uint32_t)t);
    }
}

template <int TY, int TZ>
__device__ __forceinline__ int tile_of(const OiftArgs &A, int x, int y, int z) {
    return (x >> 5) + (y / TY) * A.ntx + (z / TZ) * A.ntx * A.nty;
}

// Process one tile at level kk (cost c, label l).  All 32 lanes of the warp call it.
template <int TY, int TZ>
__device__ void process_tile(const OiftArgs &A, int t, int par, uint32_t kk, int c, int l,
                             double fgt, double flt, int bgt, int blt, uint32_t *skey,
                             uint16_t *sw, uint32_t &next_min) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int X = A.X, Y = A.Y, Z = A.Z;
    const size_t XY = (size_t)X * Y, N = A.N;
    const int tx = t % A.ntx, ty = (t / A.ntx) % A.nty, tz = t / (A.ntx * A.nty);
    const int x0 = tx * 32, y0 = ty * TY, z0 = tz * TZ;
    const int x = x0 + lane;
    const bool has_z = (Z > 1);

    uint32_t myF = 0, myOpen = 0, cpx = 0, cmx = 0, cpy = 0, cmy = 0, cpz = 0, cmz = 0;
    // ---- pass 1: rows -> shared memory, level masks (ballots) ----
#pragma unroll 4
    for (int r = 0; r < 32; r++) {
        const int y = y0 + (r % TY), z = z0 + (r / TY);
        const bool valid = (x < X) && (y < Y) && (z < Z);
        const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
        uint32_t k = 0;
        uint32_t cx = 0, cy = 0, cz = 0;
        if (valid) {
            k = __ldcg(&A.key[p]);
            cx = __ldg(&A.W[p]);
            cy = __ldg(&A.W[N + p]);
            if (has_z) cz = __ldg(&A.W[2 * N + p]);
        }
        skey[r * 32 + lane] = k;
        sw[r * 32 + lane] = (uint16_t)cx;
        sw[1024 + r * 32 + lane] = (uint16_t)cy;
        sw[2048 + r * 32 + lane] = (uint16_t)cz;
        const uint32_t bF = __ballot_sync(FULL, valid && k == kk);
        const uint32_t bO = __ballot_sync(FULL, valid && k > kk);
        const uint32_t cxm1 = __shfl_up_sync(FULL, cx, 1);
        const uint32_t bPX = __ballot_sync(FULL, lane > 0 && arc_ok(cxm1, true, c, bgt, blt));
        const uint32_t bMX = __ballot_sync(FULL, lane < 31 && arc_ok(cx, false, c, bgt, blt));
        const uint32_t bFY = __ballot_sync(FULL, arc_ok(cy, true, c, bgt, blt));
        const uint32_t bBY = __ballot_sync(FULL, arc_ok(cy, false, c, bgt, blt));
        const uint32_t bFZ = __ballot_sync(FULL, arc_ok(cz, true, c, bgt, blt));
        const uint32_t bBZ = __ballot_sync(FULL, arc_ok(cz, false, c, bgt, blt));
        if (lane == r) {
            myF = bF;
            myOpen = bO;
            cpx = bPX;
            cmx = bMX;
            cmy = ((r % TY) < TY - 1) ? bBY : 0u;
            cmz = (r + TY < 32) ? bBZ : 0u;
        }
        if (lane == r + 1 && ((r % TY) < TY - 1)) cpy = bFY;
        if (TZ > 1 && lane == r + TY) cpz = bFZ;
    }
    // ---- flood of the level inside the tile ----
    const bool ylo = (lane % TY) != 0, yhi = (lane % TY) != TY - 1;
    const bool zlo = lane >= TY, zhi = lane + TY < 32;
    uint32_t F = myF;
    for (int it = 0; it < 2048; it++) {
        uint32_t fym = __shfl_up_sync(FULL, F, 1);
        uint32_t fyp = __shfl_down_sync(FULL, F, 1);
        uint32_t fzm = __shfl_up_sync(FULL, F, TY);
        uint32_t fzp = __shfl_down_sync(FULL, F, TY);
        uint32_t grow = ((F << 1) & cpx) | ((F >> 1) & cmx) | (ylo ? (fym & cpy) : 0u) |
                        (yhi ? (fyp & cmy) : 0u) | (zlo ? (fzm & cpz) : 0u) |
                        (zhi ? (fzp & cmz) : 0u);
        uint32_t nF = F | (grow & myOpen);
        if (!__any_sync(FULL, nF != F)) break;
        F = nF;
    }
    __syncwarp();
    // ---- pass 2: expand every voxel conquered at this level ----
    const uint32_t kexp = kk - 1u;
    const int lo_shift = 17;
    for (int r = 0; r < 32; r++) {
        const uint32_t ne = __shfl_sync(FULL, F, r);
        if (ne == 0u) continue;
        const int y = y0 + (r % TY), z = z0 + (r / TY);
        if ((ne >> lane) & 1u) {
            const size_t p = (size_t)x + (size_t)y * X + (size_t)z * XY;
            A.key[p] = kexp;
            skey[r * 32 + lane] = kexp;
            // six neighbours: -z,-y,-x,+x,+y,+z
#pragma unroll
            for (int d = 0; d < 6; d++) {
                int qx = x, qy = y, qz = z;
                uint32_t code;
                bool tail_low;
                bool in_tile;
                int rq = r, xq = lane;
                if (d == 0) {  // -z
                    if (!has_z || z == 0) continue;
                    qz = z - 1;
                    tail_low = false;
                    in_tile = (r >= TY);
                    rq = r - TY;
                    code = in_tile ? sw[2048 + rq * 32 + lane] : __ldg(&A.W[2 * N + p - XY]);
                } else if (d == 1) {  // -y
                    if (y == 0) continue;
                    qy = y - 1;
                    tail_low = false;
                    in_tile = (r % TY) > 0;
                    rq = r - 1;
                    code = in_tile ? sw[1024 + rq * 32 + lane] : __ldg(&A.W[N + p - X]);
                } else if (d == 2) {  // -x
                    if (x == 0) continue;
                    qx = x - 1;
                    tail_low = false;
                    in_tile = lane > 0;
                    xq = lane - 1;
                    code = in_tile ? sw[r * 32 + lane - 1] : __ldg(&A.W[p - 1]);
                } else if (d == 3) {  // +x
                    if (x + 1 >= X) continue;
                    qx = x + 1;
                    tail_low = true;
                    in_tile = lane < 31;
                    xq = lane + 1;
                    code = sw[r * 32 + lane];
                } else if (d == 4) {  // +y
                    if (y + 1 >= Y) continue;
                    qy = y + 1;
                    tail_low = true;
                    in_tile = (r % TY) < TY - 1;
                    rq = r + 1;
                    code = sw[1024 + r * 32 + lane];
                } else {  // +z
                    if (!has_z || z + 1 >= Z) continue;
                    qz = z + 1;
                    tail_low = true;
                    in_tile = (r + TY) < 32;
                    rq = r + TY;
                    code = sw[2048 + r * 32 + lane];
                }
                const bool hi = (code >> 15) & 1, lo = (code >> 14) & 1;
                const int w = oriented_weight(code & OIFT_BASE_MASK, tail_low ? hi : lo,
                                              tail_low ? lo : hi, fgt, flt);
                const int nc = w > c ? w : c;
                const uint32_t nk = ((uint32_t)nc << lo_shift) | ((uint32_t)l << 1) | 1u;
                const size_t q = (size_t)qx + (size_t)qy * X + (size_t)qz * XY;
                if (in_tile) {
                    uint32_t sk = skey[rq * 32 + xq];
                    if (nk < sk) {
                        atomicMin(&skey[rq * 32 + xq], nk);
                        atomicMin(&A.key[q], nk);
                    }
                } else {
                    uint32_t gk = __ldcg(&A.key[q]);
                    if (nk < gk) {
                        uint32_t old = atomicMin(&A.key[q], nk);
                        if (nk < old) {
                            int tq = tile_of<TY, TZ>(A, qx, qy, qz);
                            if (nk == kk) {
                                enqueue_tile(A, par, tq);
                            } else {
                                atomicMin(&A.tpend[tq], nk);
                                next_min = nk < next_min ? nk : next_min;
                            }
                        }
                    }
                }
            }
        }
    }
    __syncwarp();
    // ---- pass 3: pending key of this tile ----
    uint32_t m = OIFT_KEY_INF;
#pragma unroll 8
    for (int r = 0; r < 32; r++) {
        uint32_t v = skey[r * 32 + lane];
        if (v > kk && v < m) m = v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        uint32_t v = __shfl_xor_sync(FULL, m, o);
        m = v < m ? v : m;
    }
    if (lane == 0 && m != OIFT_KEY_INF) atomicMin(&A.tpend[t], m);
    if (m < next_min) next_min = m;
}

template <int TY, int TZ>
__global__ void __launch_bounds__(OIFT_WARPS * 32, 1) oift_persistent_kernel(OiftArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const unsigned FULL = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *skey = reinterpret_cast<uint32_t *>(smem_raw) + warp * 1024;
    uint16_t *sw = reinterpret_cast<uint16_t *>(smem_raw + OIFT_WARPS * 4096) + warp * 3072;
    __shared__ uint32_t blk_min[OIFT_WARPS];
    __shared__ uint32_t s_level;
    OiftGlobals *g = A.g;
    const int gwarp = blockIdx.x * OIFT_WARPS + warp;
    const int nwarps = gridDim.x * OIFT_WARPS;

    uint32_t prev_level = 0;
    for (int e = 0;; e++) {
        const int par = e & 1;
        // ---- R: global minimum of the pending keys ----
        uint32_t m = OIFT_KEY_INF;
        for (int t = gwarp * 32 + lane; t < A.ntiles; t += nwarps * 32) {
            uint32_t v = __ldcg(&A.tpend[t]);
            m = v < m ? v : m;
        }
        for (int o = 16; o > 0; o >>= 1) {
            uint32_t v = __shfl_xor_sync(FULL, m, o);
            m = v < m ? v : m;
        }
        if (lane == 0) blk_min[warp] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t bm = blk_min[0];
            for (int w = 1; w < OIFT_WARPS; w++) bm = blk_min[w] < bm ? blk_min[w] : bm;
            if (bm != OIFT_KEY_INF) atomicMin(&g->nextmin[par], bm);
            if (blockIdx.x == 0) {
                g->outstanding[par] = nwarps;
                g->nextmin[par ^ 1] = OIFT_KEY_INF;
            }
        }
        grid_barrier(g, A.spin_limit);
        if (threadIdx.x == 0) s_level = vload(&g->nextmin[par]);
        __syncthreads();
        const uint32_t kk = s_level;
        if (kk == OIFT_KEY_INF || vload(&g->error)) break;
        // levels strictly increase; a repeat or a runaway level count is a fault
        if ((e > 0 && kk <= prev_level) || e >= A.max_levels) {
            if (threadIdx.x == 0) atomicCAS(&g->error, 0, OIFT_DEV_TIMEOUT);
            break;
        }
        prev_level = kk;
        if (blockIdx.x == 0 && threadIdx.x == 0) g->levels = e + 1;
        const int c = key_cost(kk), l = key_label(kk);
        const double per = (double)polarity_of(A, l);
        const double fgt = 1.0 + per / 100.0, flt = 1.0 - per / 100.0;
        const int bgt = max_base_for_cost(c, fgt), blt = max_base_for_cost(c, flt);
        // ---- S: queue the tiles of this level ----
        for (int t0 = gwarp * 32; t0 < A.ntiles; t0 += nwarps * 32) {
            int t = t0 + lane;
            bool hit = t < A.ntiles && __ldcg(&A.tpend[t]) == kk;
            if (hit) {
                A.tpend[t] = OIFT_KEY_INF;
                enqueue_tile(A, par, t);
            }
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicSub(&g->outstanding[par], 1);
        // ---- P: drain the level ----
        uint32_t next_min = OIFT_KEY_INF;
        long long spins = 0;
        unsigned long long steps = 0;
        for (;;) {
            int t = -1;
            if (lane == 0) {
                unsigned long long h = vload(&g->qhead), tl = vload(&g->qtail);
                if (h < tl) {
                    if (atomicCAS(&g->qhead, h, h + 1) == h) {
                        uint32_t v = QEMPTY;
                        long long ws = 0;
                        while ((v = atomicExch(&A.queue[h & A.qmask], QEMPTY)) == QEMPTY) {
                            if (++ws > A.spin_limit || vload(&g->error)) {
                                atomicCAS(&g->error, 0, OIFT_DEV_TIMEOUT);
                                break;
                            }
                        }
                        if (v != QEMPTY) {
                            atomicExch(&A.inq[v], 0u);
                            t = (int)v;
                        }
                    } else {
                        t = -2;
                    }
                }
            }
            t = __shfl_sync(FULL, t, 0);
            if (t >= 0) {
                process_tile<TY, TZ>(A, t, par, kk, c, l, fgt, flt, bgt, blt, skey, sw,
                                     next_min);
                steps++;
                __threadfence();
                __syncwarp();
                if (lane == 0) atomicSub(&g->outstanding[par], 1);
                spins = 0;
                continue;
            }
            if (t == -2) continue;
            int done = 0;
            if (lane == 0) {
                done = vload(&g->outstanding[par]) == 0 || vload(&g->error) != 0;
                if (!done && ++spins > A.spin_limit) {
                    atomicCAS(&g->error, 0, OIFT_DEV_TIMEOUT);
                    done = 1;
                }
            }
            done = __shfl_sync(FULL, done, 0);
            if (done) break;
            __nanosleep(32);
        }
        if (lane == 0 && steps) atomicAdd(&g->tile_steps, steps);
        (void)next_min;
    }
}

__global__ void oift_seed_kernel(uint32_t *key, uint32_t *tpend, const int32_t *seeds,
                                 const int32_t *labels, int nseeds, int X, int Y, int Z,
                                 int ntx, int nty, int TY, int TZ, int *bad) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nseeds) return;
    int p = seeds[i];
    size_t N = (size_t)X * Y * Z;
    if (p < 0 || (size_t)p >= N) {
        atomicExch(bad, 1);
        return;
    }
    int lb = labels[i] < 0 ? 0 : labels[i];
    if (lb > OIFT_MAX_LABEL) {
        atomicExch(bad, 2);
        return;
    }
    uint32_t k = make_key(0, lb, 1);
    atomicMin(&key[p], k);
    int x = p % X, y = (p / X) % Y, z = (int)(p / ((size_t)X * Y));
    int t = (x >> 5) + (y / TY) * ntx + (z / TZ) * ntx * nty;
    atomicMin(&tpend[t], k);
}

__global__ void oift_finalize_kernel(const uint32_t *key, size_t n, int32_t *cost,
                                     int32_t *label) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        uint32_t k = key[i];
        if (cost) cost[i] = (k == OIFT_KEY_INF) ? 0x7fffffff : key_cost(k);
        if (label) label[i] = (k == OIFT_KEY_INF) ? -1 : key_label(k);
    }
}

// ------------------------------------------------------------------ host side ----

OiftPlan oift_plan(int X, int Y, int Z) {
    OiftPlan P;
    if (Z == 1) {
        P.TY = 32;
        P.TZ = 1;
    } else {
        P.TY = 8;
        P.TZ = 4;
    }
    P.ntx = (X + 31) / 32;
    P.nty = (Y + P.TY - 1) / P.TY;
    P.ntz = (Z + P.TZ - 1) / P.TZ;
    P.ntiles = P.ntx * P.nty * P.ntz;
    unsigned int q = 1024;
    while (q < (unsigned int)P.ntiles + 64) q <<= 1;
    P.qcap = q;
    return P;
}

size_t oift_smem_bytes() { return (size_t)OIFT_WARPS * (4096 + 6144); }


size_t oift_globals_bytes() { return sizeof(OiftGlobals); }

// Runs the seeds kernel, the persistent kernel and (optionally) the finalize kernel.
int oift_run(const OiftPlan &P, const OiftScratch &S, const uint16_t *W, int X, int Y, int Z,
             const int32_t *d_seeds, const int32_t *d_seed_labels, int nseeds,
             const float *d_pol_table, int npol, float pol_default, int32_t *cost,
             int32_t *label, int *d_flag, int sms, cudaStream_t st, int *levels_out,
             long long *steps_out, cudaEvent_t ev_begin, cudaEvent_t ev_end) {
    size_t N = (size_t)X * Y * Z;
    cudaMemsetAsync(S.key, 0xFF, N * sizeof(uint32_t), st);
    cudaMemsetAsync(S.tpend, 0xFF, (size_t)P.ntiles * sizeof(uint32_t), st);
    cudaMemsetAsync(S.inq, 0, (size_t)P.ntiles * sizeof(uint32_t), st);
    cudaMemsetAsync(S.queue, 0xFF, (size_t)P.qcap * sizeof(uint32_t), st);
    cudaMemsetAsync(S.g, 0, sizeof(OiftGlobals), st);
    OiftGlobals init{};
    init.nextmin[0] = init.nextmin[1] = OIFT_KEY_INF;
    cudaMemcpyAsync(S.g, &init, sizeof(OiftGlobals), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(d_flag, 0, sizeof(int), st);
    if (nseeds > 0)
        oift_seed_kernel<<<(nseeds + 255) / 256, 256, 0, st>>>(S.key, S.tpend, d_seeds,
                                                               d_seed_labels, nseeds, X, Y,
                                                               Z, P.ntx, P.nty, P.TY, P.TZ,
                                                               d_flag);
    int hflag = 0;
    cudaMemcpyAsync(&hflag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return OIFT_E_CUDA;
    if (hflag == 1) return OIFT_E_SEED_RANGE;
    if (hflag == 2) return OIFT_E_BAD_ARG;

    OiftArgs A;
    A.key = S.key;
    A.W = W;
    A.tpend = S.tpend;
    A.inq = S.inq;
    A.queue = S.queue;
    A.qmask = P.qcap - 1;
    A.X = X;
    A.Y = Y;
    A.Z = Z;
    A.N = N;
    A.ntx = P.ntx;
    A.nty = P.nty;
    A.ntz = P.ntz;
    A.ntiles = P.ntiles;
    A.pol_table = d_pol_table;
    A.npol = npol;
    A.pol_default = pol_default;
    A.g = S.g;
    A.spin_limit = 20000000LL;  // ~1-2 s of polling at ~64 ns per spin
    A.max_levels = 4000000;
    size_t smem = oift_smem_bytes();
    void *args[] = {&A};
    cudaError_t err;
    if (ev_begin) cudaEventRecord(ev_begin, st);
    if (P.TZ == 1) {
        auto kfn = oift_persistent_kernel<32, 1>;
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        err = cudaLaunchCooperativeKernel((void *)kfn, dim3(sms), dim3(OIFT_WARPS * 32), args,
                                          smem, st);
    } else {
        auto kfn = oift_persistent_kernel<8, 4>;
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        err = cudaLaunchCooperativeKernel((void *)kfn, dim3(sms), dim3(OIFT_WARPS * 32), args,
                                          smem, st);
    }
    if (err != cudaSuccess) return OIFT_E_CUDA;
    if (ev_end) cudaEventRecord(ev_end, st);
    if (cost || label) {
        int blocks = (int)((N + 255) / 256);
        if (blocks > sms * 16) blocks = sms * 16;
        oift_finalize_kernel<<<blocks, 256, 0, st>>>(S.key, N, cost, label);
    }
    OiftGlobals hg;
    cudaMemcpyAsync(&hg, S.g, sizeof(OiftGlobals), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return OIFT_E_CUDA;
    if (levels_out) *levels_out = hg.levels;
    if (steps_out) *steps_out = (long long)hg.tile_steps;
    if (hg.error == OIFT_DEV_TIMEOUT) return OIFT_E_NOT_CONVERGED;
    if (hg.error == OIFT_DEV_QUEUE) return OIFT_E_QUEUE_OVERFLOW;
    return OIFT_OK;
}

}  // namespace oiftb
