// api.cu -- C ABI of liboift_b200 (include/oift_b200.h): context, device scratch,
// pipeline orchestration and the reference-compatible entry points.
//
// Pipeline of one job (all on the context's stream):
//   minmax(image) -> build_weights -> OIFT (persistent kernel) -> finalize labels/cost
//   -> relax init -> K sweeps (ping-pong membership) -> argmax labels + mask.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "kernels.cuh"

using namespace oiftb;

// Host-side trace ranges (NVTX, header-only): the entry points and the stages they queue
// show on a profiler's timeline beside the kernels; a few nanoseconds each with no tool
// attached.
// Scoped ranges mark the entry points (balanced on every return path); instant marks the
// stages the pipeline queues.
struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

struct oift_b200_ctx {
    int device = 0;
    int sms = 148;
    int oift_ctas = 0;  // CTAs of the persistent OIFT grid (0 = one per SM)
    // bounds of the OIFT kernels' waits (oift_b200_set_limits)
    long long spin_limit = OIFT_DEFAULT_SPIN_LIMIT;
    int max_levels = OIFT_DEFAULT_MAX_LEVELS;
    std::vector<oift_b200_ctx *> lanes;  // sub-contexts (relaxation streams) of the batched driver
    // batch autotuner: candidate (teams, warp-tile shape) with its measured rate (< 0 untried)
    struct TuneCand {
        int teams, tile_ty;
        double rate;
    };
    std::vector<TuneCand> tune_cands;
    int batch_tile_ty = 8;  // warp tile of explicit team counts: 8 (32x8x4) or 4 (32x4x8)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // ev[10]: the early readback of one pipeline call has landed; ev[11]: the host entry's
    // copy of the pinned seed labels has ended
    cudaEvent_t ev[12];
    // scratch (grow-only)
    DevBuf img32, img16, W, key, tpend, inq, queue, glob, flag, minmax, seeds, slabels, cost,
        olabel, flabel, memb, seedc, l2c, classes, pol, presence, lut, mask8, ctaq, lprof, rtdist;
    // batched driver: job descriptors, per-image min/max + clamp counters, per-team OIFT
    // state, job counter + abort flag, OIFT labels of jobs that only want a mask
    DevBuf bjobs, bmm, bkey, btpend, bmbox, bglob, bctl, bolab;
    // CLI steps: shifted / blurred images, dilation border, histograms and tie counts
    DevBuf cimg0, cimg1, dborder, dhist, daux, dlabel;
    // coarse-to-fine cascade: coarse image / labels / seeds, first-seed map, upscaled and
    // merged labels, fine seeds, axis tables and chunk counts
    DevBuf yimg, ylab, yseeds, yslab, yfirst, yup, ymerge, yfseeds, yfslab, yaux;
    // adjoint: checkpoints / segment / lambdas / weight sums, mask rings, seed classes, sums
    DevBuf awork, adist, aseedc, asmall, al2c;
    DevBuf gmap;  // normalised Sobel gradient of the gradient-blend weights
    DevBuf igring, igsmall;  // image-graph relaxation: ring index per pixel, reductions
    DevBuf Wt;  // tile-major copy of the OIFT code planes
    // pinned host staging of the seed labels of the host entry
    int32_t *hslab = nullptr;
    size_t hslab_n = 0;
    // pinned host copies of the small device results a call reads at its end (a copy into
    // pageable memory would wait for the stream)
    struct HostMirror {
        OiftGlobals g;
        int flag[4];
        int mm[2];
        int mm_init[2];
        unsigned long long clamp;
        uint32_t presence[1024];
    } *hm = nullptr;
    unsigned *hhist = nullptr;  // per-sweep tile histogram of the relaxation
    size_t hhist_n = 0;
    // Gaussian-RBF table on the device, built for (lut_sigma, lut_wq); lut_len 0 = none
    float lut_sigma = -1.0f;
    int lut_wq = -1, lut_len = 0;
    DevBuf hmemb;  // membership of the host entry
    DevBuf bseed, barcs, csums;  // arc-weight-map adjoint: seed flags, arcs, block sums
    bool relax_tma = false;  // the last relax_launch staged its tiles with TMA
    size_t total = 0;
    unsigned long long oift_cycles[24] = {0};
};

static thread_local int g_last_status = OIFT_OK;

static int grow(oift_b200_ctx *c, DevBuf &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return OIFT_OK;
    if (b.p) {
        cudaFree(b.p);
        c->total -= b.bytes;
        b.p = nullptr;
        b.bytes = 0;
    }
    if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return OIFT_E_OOM;
    }
    b.bytes = bytes;
    c->total += bytes;
    return OIFT_OK;
}

#define TRY(x)                        \
    do {                              \
        int _s = (x);                 \
        if (_s != OIFT_OK) return _s; \
    } while (0)
#define CU(x)                                  \
    do {                                       \
        if ((x) != cudaSuccess) {              \
            cudaGetLastError();                \
            return OIFT_E_CUDA;                \
        }                                      \
    } while (0)

extern "C" {

const char *oift_b200_status_string(int s) {
    switch (s) {
        case OIFT_OK: return "ok";
        case OIFT_E_BAD_ARG: return "bad argument";
        case OIFT_E_NO_SEEDS: return "no seeds";
        case OIFT_E_OOM: return "device allocation failed";
        case OIFT_E_NOT_CONVERGED: return "bounded wait expired (not converged)";
        case OIFT_E_QUEUE_OVERFLOW: return "device work queue overflow";
        case OIFT_E_CUDA: return "CUDA runtime error";
        case OIFT_E_RANGE: return "weight or intensity out of supported range";
        case OIFT_E_UNSUPPORTED: return "unsupported option";
        case OIFT_E_SEED_RANGE: return "seed address outside the volume";
        default: return "unknown status";
    }
}

int oift_b200_create(oift_b200_ctx **out, int device) {
    if (!out) return OIFT_E_BAD_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return OIFT_E_CUDA;
    }
    CU(cudaSetDevice(device));
    oift_b200_ctx *c = new oift_b200_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    if (!coop) {
        delete c;
        return OIFT_E_UNSUPPORTED;
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return OIFT_E_CUDA;
    }
    c->own_stream = true;
    for (auto &e : c->ev) cudaEventCreate(&e);
    if (cudaHostAlloc((void **)&c->hm, sizeof(oift_b200_ctx::HostMirror), cudaHostAllocDefault) !=
        cudaSuccess) {
        cudaGetLastError();
        oift_b200_destroy(c);
        return OIFT_E_OOM;
    }
    *out = c;
    return OIFT_OK;
}

int oift_b200_destroy(oift_b200_ctx *c) {
    if (!c) return OIFT_E_BAD_ARG;
    for (oift_b200_ctx *l : c->lanes) oift_b200_destroy(l);
    c->lanes.clear();
    cudaSetDevice(c->device);
    DevBuf *bufs[] = {&c->img32, &c->img16,  &c->W,      &c->key,     &c->tpend,   &c->inq,
                      &c->queue, &c->glob,   &c->flag,   &c->minmax,  &c->seeds,   &c->slabels,
                      &c->cost,  &c->olabel, &c->flabel, &c->memb,    &c->seedc,   &c->l2c,
                      &c->classes, &c->pol,  &c->presence, &c->lut,   &c->mask8, &c->ctaq,
                      &c->lprof, &c->rtdist, &c->bjobs, &c->bmm,  &c->bkey,  &c->btpend,
                      &c->bmbox, &c->bglob, &c->bctl, &c->bolab, &c->cimg0, &c->cimg1,
                      &c->dborder, &c->dhist, &c->daux, &c->dlabel, &c->yimg, &c->ylab,
                      &c->yseeds, &c->yslab, &c->yfirst, &c->yup, &c->ymerge, &c->yfseeds,
                      &c->yfslab, &c->yaux, &c->awork, &c->adist, &c->aseedc, &c->asmall,
                      &c->al2c, &c->gmap, &c->igring, &c->igsmall, &c->Wt, &c->hmemb,
                      &c->bseed, &c->barcs, &c->csums};
    for (DevBuf *b : bufs)
        if (b->p) cudaFree(b->p);
    if (c->hslab) cudaFreeHost(c->hslab);
    if (c->hm) cudaFreeHost(c->hm);
    if (c->hhist) cudaFreeHost(c->hhist);
    for (auto &e : c->ev) cudaEventDestroy(e);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return OIFT_OK;
}

size_t oift_b200_scratch_bytes(const oift_b200_ctx *c) {
    if (!c) return 0;
    size_t t = c->total;
    for (const oift_b200_ctx *l : c->lanes) t += l->total;
    return t;
}

int oift_b200_set_batch_tile(oift_b200_ctx *c, int tile_ty) {
    if (!c || (tile_ty != 8 && tile_ty != 4)) return OIFT_E_BAD_ARG;
    c->batch_tile_ty = tile_ty;
    return OIFT_OK;
}

int oift_b200_set_oift_grid(oift_b200_ctx *c, int ctas) {
    if (!c || ctas < 0) return OIFT_E_BAD_ARG;
    c->oift_ctas = ctas;
    return OIFT_OK;
}

int oift_b200_set_limits(oift_b200_ctx *c, long long spin_limit, int max_levels) {
    if (!c) return OIFT_E_BAD_ARG;
    c->spin_limit = spin_limit > 0 ? spin_limit : OIFT_DEFAULT_SPIN_LIMIT;
    c->max_levels = max_levels > 0 ? max_levels : OIFT_DEFAULT_MAX_LEVELS;
    for (oift_b200_ctx *l : c->lanes) {
        l->spin_limit = c->spin_limit;
        l->max_levels = c->max_levels;
    }
    return OIFT_OK;
}

int oift_b200_set_stream(oift_b200_ctx *c, void *stream) {
    if (!c) return OIFT_E_BAD_ARG;
    if (c->own_stream) cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    return OIFT_OK;
}

int oift_b200_level_profile(oift_b200_ctx *c, unsigned int *cycles_steps, int cap) {
    if (!c || !cycles_steps || cap < 0) return OIFT_E_BAD_ARG;
    if (!c->lprof.p) return 0;
    int n = cap < 8192 ? cap : 8192;
    if (cudaMemcpy(cycles_steps, c->lprof.p, (size_t)n * 2 * sizeof(unsigned int),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
        return OIFT_E_CUDA;
    return n;
}

int oift_b200_weight_planes(int adjacency) {
    if (adjacency == 6 || adjacency == 4) return 3;
    if (adjacency == 26 || adjacency == 8) return 13;
    return 0;
}

}  // extern "C"

// ------------------------------------------------------------------ helpers ----
static int check_params(const oift_b200_params *p) {
    if (!p) return OIFT_E_BAD_ARG;
    if (p->xsize <= 0 || p->ysize <= 0 || p->zsize <= 0) return OIFT_E_BAD_ARG;
    if ((size_t)p->xsize * p->ysize * p->zsize > 0x7fffffffULL) return OIFT_E_BAD_ARG;
    if (p->adjacency == 4 || p->adjacency == 8) {
        if (p->zsize != 1) return OIFT_E_BAD_ARG;
    } else if (p->adjacency != 6 && p->adjacency != 26) {
        return OIFT_E_BAD_ARG;
    }
    if (p->weight_mode < 0 || p->weight_mode > OIFT_W_IMAGEGRAPH) return OIFT_E_BAD_ARG;
    if ((p->weight_mode == OIFT_W_GRAD_Q || p->weight_mode == OIFT_W_RBF_Q) &&
        (p->wq <= 0 || p->wq > OIFT_MAX_BASE))
        return OIFT_E_BAD_ARG;
    if (p->relax_sweeps < 0) return OIFT_E_BAD_ARG;
    if (p->per_class) {
        if (p->max_label < 0 || p->max_label > OIFT_MAX_LABEL) return OIFT_E_BAD_ARG;
        for (int i = 0; i <= p->max_label; i++)
            if (!(std::fabs(p->per_class[i]) <= 100.0f)) return OIFT_E_BAD_ARG;
    } else if (!(std::fabs(p->per) <= 100.0f)) {
        return OIFT_E_BAD_ARG;
    }
    if (p->weight_mode == OIFT_W_BLEND_Q) {
        // the blend weights of exp_gradient_weight.cpp: face neighbourhood, global polarity,
        // a mix weight in [0, 1]
        if (p->adjacency != 6 && p->adjacency != 4) return OIFT_E_UNSUPPORTED;
        if (p->per_class) return OIFT_E_UNSUPPORTED;
        if (!(p->blend_a >= 0.0f && p->blend_a <= 1.0f)) return OIFT_E_BAD_ARG;
    }
    if (p->weight_mode == OIFT_W_IMAGEGRAPH) {
        // the 2D image graph of gft_imagegraph.cpp: Circular(1.0) / Circular(1.5), one
        // global polarity, ring indices of the relaxation in 16 bits
        if (p->zsize != 1 || (p->adjacency != 4 && p->adjacency != 8)) return OIFT_E_UNSUPPORTED;
        if (p->per_class) return OIFT_E_UNSUPPORTED;
        if (p->relax_sweeps >= 0xFFFF) return OIFT_E_BAD_ARG;
    }
    if (p->weight_mode == OIFT_W_RBF_Q && !(p->rbf_sigma > 0.0f)) return OIFT_E_BAD_ARG;
    return OIFT_OK;
}

// Polarity table of the OIFT: global mode -> [ -per ] with default +per
// (gft_ift.cpp:968); per-class mode -> per_class[0..max_label], default 0.
static int upload_polarity(oift_b200_ctx *c, const oift_b200_params *p, int *npol,
                           float *dflt) {
    std::vector<float> t;
    if (p->per_class) {
        t.assign(p->per_class, p->per_class + p->max_label + 1);
        *dflt = 0.0f;
    } else {
        t.push_back(-p->per);
        *dflt = p->per;
    }
    TRY(grow(c, c->pol, t.size() * sizeof(float)));
    CU(cudaMemcpyAsync(c->pol.p, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice,
                       c->stream));
    *npol = (int)t.size();
    return OIFT_OK;
}

struct RelaxResult {
    int nclasses = 0;
    long long active_voxel_sweeps = 0;
    int dilations = 0;
};

// Class set and sweep constants of one relaxation: classes = 0 and the labels present among
// the seeds (gft_ift.cpp:8684-8712, read back to the host); Wmax (8733-8734) from hmm.
struct RelaxPlan {
    int nclasses = 0, maxl = 0, bg = 0;
    std::vector<int> classes, l2c;
    RelaxArgs ra{};
};

// Queues the scan of the labels present among the seeds and its copy to the context's
// pinned mirror (hm->presence); relax_plan_finish reads it once the copy has completed.
static int relax_classes_launch(oift_b200_ctx *c, const int32_t *d_slabels, int nseeds) {
    cudaStream_t s = c->stream;
    TRY(grow(c, c->presence, 1024 * sizeof(uint32_t)));
    CU(cudaMemsetAsync(c->presence.p, 0, 1024 * sizeof(uint32_t), s));
    if (nseeds > 0)
        seed_presence_kernel<<<std::min((nseeds + 255) / 256, c->sms * 4), 256, 0, s>>>(
            d_slabels, nseeds, (uint32_t *)c->presence.p);
    CU(cudaMemcpyAsync(c->hm->presence, c->presence.p, 1024 * sizeof(uint32_t),
                       cudaMemcpyDeviceToHost, s));
    return OIFT_OK;
}

static int relax_plan_finish(oift_b200_ctx *c, const oift_b200_params *p, const int hmm[2],
                             RelaxPlan *pl);

static int relax_plan(oift_b200_ctx *c, const oift_b200_params *p, const int32_t *d_slabels,
                      int nseeds, const int hmm[2], RelaxPlan *pl) {
    TRY(relax_classes_launch(c, d_slabels, nseeds));
    CU(cudaStreamSynchronize(c->stream));
    return relax_plan_finish(c, p, hmm, pl);
}

static int relax_plan_finish(oift_b200_ctx *c, const oift_b200_params *p, const int hmm[2],
                             RelaxPlan *pl) {
    const int X = p->xsize, Y = p->ysize, Z = p->zsize;
    const size_t N = (size_t)X * Y * Z;
    Adjacency adj = make_adjacency(p->adjacency == 4 ? 6 : (p->adjacency == 8 ? 26 : p->adjacency));
    std::vector<uint32_t> bits(c->hm->presence, c->hm->presence + 1024);
    bits[0] |= 1u;
    pl->classes.clear();
    for (int l = 0; l <= OIFT_MAX_LABEL; l++)
        if ((bits[l >> 5] >> (l & 31)) & 1u) pl->classes.push_back(l);
    const int nclasses = (int)pl->classes.size();
    if (nclasses > 8) return OIFT_E_UNSUPPORTED;
    pl->nclasses = nclasses;
    pl->maxl = pl->classes.back();
    pl->l2c.assign(pl->maxl + 1, -1);
    for (int k = 0; k < nclasses; k++) pl->l2c[pl->classes[k]] = k;
    pl->bg = pl->l2c[0] < 0 ? 0 : pl->l2c[0];
    // Wmax (gft_ift.cpp:8733-8734) on the image shifted to >= 0 as the CLI does
    float max_abs_per = 0.0f;
    std::vector<float> pcm(nclasses, 0.0f);
    if (p->per_class) {
        for (int k = 0; k < nclasses; k++) {
            float v = (pl->classes[k] <= p->max_label) ? p->per_class[pl->classes[k]] : 0.0f;
            pcm[k] = v;
            if (std::fabs(v) > max_abs_per) max_abs_per = std::fabs(v);
        }
    } else {
        max_abs_per = std::fabs(p->per);
    }
    long long imax = hmm[1], imin = hmm[0];
    long long shifted_max = imin < 0 ? imax - imin : imax;
    float Wmax = (float)shifted_max;
    const bool blend = p->weight_mode == OIFT_W_BLEND_Q;
    if (blend)  // exp_gradient_weight.cpp:338-339, in float
        Wmax *= (1.0f + std::fabs(p->per) / 100.0f);
    else
        Wmax = (float)((double)Wmax * (1.0 + (double)max_abs_per / 100.0));
    double deg = (p->adjacency == 26) ? 26 : (p->adjacency == 8 ? 8 : (p->adjacency == 6 ? 6 : 4));
    if ((double)Wmax > std::pow(3.0e38 / deg, 0.125)) return OIFT_E_RANGE;

    RelaxArgs &ra = pl->ra;
    ra.X = X;
    ra.Y = Y;
    ra.Z = Z;
    ra.N = N;
    ra.nadj = adj.n;
    for (int i = 0; i < adj.n; i++) {
        ra.dx[i] = adj.dx[i];
        ra.dy[i] = adj.dy[i];
        ra.dz[i] = adj.dz[i];
        // Dpq = sqrtf(dx^2 + dy^2 + dz^2) / dmin with unit spacing (gft_ift.cpp:8723-8731)
        ra.dpq[i] = sqrtf((float)(adj.dx[i] * adj.dx[i]) + (float)(adj.dy[i] * adj.dy[i]) +
                          (float)(adj.dz[i] * adj.dz[i])) /
                    1.0f;
    }
    ra.Wmax = Wmax;
    ra.per = p->per;
    ra.bg = pl->bg;
    ra.blend = blend ? 1 : 0;
    ra.alpha = p->blend_a;
    ra.gmap = blend ? (const int32_t *)c->gmap.p : nullptr;
    for (int k = 0; k < 8; k++) ra.pcm[k] = k < nclasses ? pcm[k] : 0.0f;
    return OIFT_OK;
}

// Scratch a relaxation of N voxels with C classes and K sweeps needs in the context.
static int relax_reserve(oift_b200_ctx *c, size_t N, int C, int maxl, int X, int Y, int Z, int K) {
    TRY(grow(c, c->memb, 2 * (size_t)C * N * sizeof(float)));
    TRY(grow(c, c->seedc, N));
    TRY(grow(c, c->l2c, (maxl + 1) * sizeof(int)));
    TRY(grow(c, c->classes, C * sizeof(int)));
    const size_t rnt = (size_t)((X + 31) / 32) * ((Y + 7) / 8) * ((Z + 3) / 4);
    TRY(grow(c, c->rtdist, 2 * rnt * sizeof(uint16_t) + (size_t)(K + 1) * sizeof(unsigned)));
    return OIFT_OK;
}

// The sweeps of one planned relaxation: kernel launches and device-side memsets only (the
// context's scratch must already be reserved), so the sequence can also be captured in a
// CUDA graph.  With `active` true the sweep histogram is copied to the context's pinned
// c->hhist (count it with relax_active_sweeps once the stream has reached that copy), and
// the sweep loop is bracketed by the context's events.
template <typename T>
static int relax_launch(oift_b200_ctx *c, const oift_b200_params *p, const T *d_img,
                        const int32_t *d_seeds, int nseeds, const int32_t *d_olab,
                        const RelaxPlan &pl, const int *d_l2c, const int *d_classes,
                        const oift_b200_outputs *out, bool active, bool use_tma = true) {
    cudaStream_t s = c->stream;
    const int X = p->xsize, Y = p->ysize, Z = p->zsize;
    const size_t N = (size_t)X * Y * Z;
    const int K = p->relax_sweeps;
    const int nclasses = pl.nclasses, maxl = pl.maxl, bg = pl.bg;
    const RelaxArgs &ra = pl.ra;
    TRY(relax_reserve(c, N, nclasses, maxl, X, Y, Z, K));
    float *m0 = (float *)c->memb.p, *m1 = m0 + (size_t)nclasses * N;
    int blocks = (int)std::min<size_t>((N + 255) / 256, (size_t)c->sms * 16);
    // both ping-pong buffers start one-hot: tiles skipped at a sweep keep that value
    relax_init_kernel<<<blocks, 256, 0, s>>>(d_olab, N, nclasses, d_l2c, maxl, bg, m0);
    relax_init_kernel<<<blocks, 256, 0, s>>>(d_olab, N, nclasses, d_l2c, maxl, bg, m1);
    CU(cudaMemsetAsync(c->seedc.p, 0xFF, N, s));
    if (nseeds > 0)
        relax_seed_kernel<<<(nseeds + 255) / 256, 256, 0, s>>>(d_seeds, nseeds, d_olab, N,
                                                               d_l2c, maxl, bg,
                                                               (uint8_t *)c->seedc.p);
    // block distance of every relaxation tile to the label boundary (exact skipping)
    const int rtx = (X + 31) / 32, rty = (Y + 7) / 8, rtz = (Z + 3) / 4;
    const int rnt = rtx * rty * rtz;
    uint16_t *td0 = (uint16_t *)c->rtdist.p, *td1 = td0 + rnt;
    unsigned *hist = (unsigned *)(td1 + rnt);  // byte offset 4 * rnt
    CU(cudaMemsetAsync(td0, 0xFF, 2 * (size_t)rnt * sizeof(uint16_t), s));
    relax_boundary_tiles_kernel<<<dim3((X + 31) / 32, (Y + 7) / 8, Z), dim3(32, 8), 0, s>>>(
        d_olab, X, Y, Z, ra.nadj, ra, td0, rtx, rty);
    const int cheb = (ra.nadj == 26);
    // exact lower bound of the voxel distance to the mask: three separable passes
    relax_tile_gap_pass_kernel<<<(rnt + 255) / 256, 256, 0, s>>>(td0, td1, rtx, rty, rtz, 0, 32, cheb);
    relax_tile_gap_pass_kernel<<<(rnt + 255) / 256, 256, 0, s>>>(td1, td0, rtx, rty, rtz, 1, 8, cheb);
    relax_tile_gap_pass_kernel<<<(rnt + 255) / 256, 256, 0, s>>>(td0, td1, rtx, rty, rtz, 2, 4, cheb);
    std::swap(td0, td1);
    if (K > 0 && active) {
        CU(cudaMemsetAsync(hist, 0, (size_t)(K + 1) * sizeof(unsigned), s));
        relax_tile_hist_kernel<<<(rnt + 255) / 256, 256, 0, s>>>(td0, rnt, K, hist);
    }
    float *cur = m0, *nxt = m1;
    // TMA boxes for the tiles' halos when the extents allow them; a tile whose loads do not
    // land sets flag[1], read back with the sweeps (relax_tma_status)
    RelaxTma tma;
    if (use_tma) TRY(grow(c, c->flag, 4 * sizeof(int)));
    c->relax_tma = use_tma && relax_tma_encode(&tma, m0, m1, d_img, sizeof(T) == 4, X, Y, Z,
                                               nclasses);
    if (c->relax_tma) {
        tma.err = (int *)c->flag.p + 1;
        CU(cudaMemsetAsync(tma.err, 0, sizeof(int), s));
    }
    if (active) cudaEventRecord(c->ev[6], s);
    for (int it = 0; it < K; it++) {
        CU(launch_relax_tiles<T>(nclasses, cur, nxt, d_img, (const uint8_t *)c->seedc.p, td0,
                                 it + 1, ra, p->per_class != nullptr, rnt, rtx, rty, s,
                                 c->relax_tma ? &tma : nullptr));
        std::swap(cur, nxt);
    }
    if (c->relax_tma)
        CU(cudaMemcpyAsync(&c->hm->flag[1], tma.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (K > 0 && active) {
        if (c->hhist_n < (size_t)K) {
            if (c->hhist) cudaFreeHost(c->hhist);
            c->hhist = nullptr;
            c->hhist_n = 0;
            CU(cudaHostAlloc((void **)&c->hhist, (size_t)K * sizeof(unsigned), cudaHostAllocDefault));
            c->hhist_n = (size_t)K;
        }
        CU(cudaMemcpyAsync(c->hhist, hist, K * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    }
    if (active) cudaEventRecord(c->ev[7], s);
    relax_argmax_kernel<<<(int)std::min<size_t>((N + 255) / 256, (size_t)c->sms * 16), 256, 0, s>>>(
        cur, N, nclasses, d_classes, out->label, out->mask);
    if (out->membership)
        CU(cudaMemcpyAsync(out->membership, cur, (size_t)nclasses * N * sizeof(float),
                           cudaMemcpyDeviceToDevice, s));
    return OIFT_OK;
}

// Outcome of the TMA loads of the last relax_launch, once the stream has passed it.
static int relax_tma_status(const oift_b200_ctx *c) {
    return (c->relax_tma && c->hm->flag[1]) ? OIFT_E_CUDA : OIFT_OK;
}

// Voxel-sweeps computed by the last relax_launch with `active` (its histogram copy must have
// completed): tiles at block distance <= t-1 from the label boundary run at sweep t.
static long long relax_active_sweeps(const oift_b200_ctx *c, int K) {
    long long run = 0, active_vs = 0;
    for (int t = 1; t <= K && (size_t)t <= c->hhist_n; t++) {
        run += c->hhist[t - 1];
        active_vs += run * 1024;
    }
    return active_vs;
}

// Relaxation of one job on the context's stream: classes from the seed labels, one-hot
// start from the OIFT labels d_olab, K tile sweeps, argmax into out->label / out->mask (and
// the membership copy).  hmm = intensity min / max of the image.  d_olab is not read after
// the argmax kernel starts, so it may alias out->label.
template <typename T>
static int relax_stage(oift_b200_ctx *c, const oift_b200_params *p, const T *d_img,
                       const int32_t *d_seeds, const int32_t *d_slabels, int nseeds,
                       const int32_t *d_olab, const int hmm[2], const oift_b200_outputs *out,
                       RelaxResult *rr) {
    RelaxPlan pl;
    TRY(relax_plan(c, p, d_slabels, nseeds, hmm, &pl));
    const int X = p->xsize, Y = p->ysize, Z = p->zsize;
    TRY(relax_reserve(c, (size_t)X * Y * Z, pl.nclasses, pl.maxl, X, Y, Z, p->relax_sweeps));
    CU(cudaMemcpyAsync(c->l2c.p, pl.l2c.data(), (pl.maxl + 1) * sizeof(int),
                       cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemcpyAsync(c->classes.p, pl.classes.data(), pl.nclasses * sizeof(int),
                       cudaMemcpyHostToDevice, c->stream));
    TRY(relax_launch<T>(c, p, d_img, d_seeds, nseeds, d_olab, pl, (const int *)c->l2c.p,
                        (const int *)c->classes.p, out, true));
    CU(cudaStreamSynchronize(c->stream));
    TRY(relax_tma_status(c));
    rr->nclasses = pl.nclasses;
    rr->active_voxel_sweeps = relax_active_sweeps(c, p->relax_sweeps);
    rr->dilations = 3;
    return OIFT_OK;
}

// Gaussian-RBF base weights over |dI| = d: lut[d] = floor(wq (1 - exp(-d^2 / (2 sigma^2))) +
// 0.5), clamped to [0, wq].  The values rise to wq and stay there, so the table ends at its
// first wq entry (a larger |dI| reads the last entry) and does not depend on the image's
// range; it is built once per (sigma, wq) and kept on the device.  A sigma so wide that the
// table has not reached wq by 2^20 entries takes one entry per value of the image's range
// (`need_range` waits for the range readback).
template <typename F>
static int rbf_table(oift_b200_ctx *c, const oift_b200_params *p, F &&need_range,
                     const uint16_t **lut_out, int *len_out) {
    if (c->lut_len > 0 && c->lut_sigma == p->rbf_sigma && c->lut_wq == p->wq) {
        *lut_out = (const uint16_t *)c->lut.p;
        *len_out = c->lut_len;
        return OIFT_OK;
    }
    const double sg = p->rbf_sigma;
    auto value = [&](long long d) -> uint16_t {
        double a = std::exp(-((double)d * (double)d) / (2.0 * sg * sg));
        double v = std::floor((double)p->wq * (1.0 - a) + 0.5);
        if (v < 0) v = 0;
        if (v > p->wq) v = p->wq;
        return (uint16_t)v;
    };
    std::vector<uint16_t> lut;
    bool saturated = false;
    for (long long d = 0; d < (1 << 20) && !saturated; d++) {
        lut.push_back(value(d));
        saturated = lut.back() == p->wq;
    }
    if (!saturated) {
        TRY(need_range());
        const long long len = (long long)c->hm->mm[1] - (long long)c->hm->mm[0] + 1;
        if (len > (1ll << 24)) return OIFT_E_RANGE;
        for (long long d = (long long)lut.size(); d < len; d++) lut.push_back(value(d));
    }
    const int len = (int)lut.size();
    TRY(grow(c, c->lut, len * sizeof(uint16_t)));
    CU(cudaMemcpyAsync(c->lut.p, lut.data(), len * sizeof(uint16_t), cudaMemcpyHostToDevice,
                       c->stream));
    c->lut_len = saturated ? len : 0;  // a range-sized table is rebuilt for the next image
    c->lut_sigma = p->rbf_sigma;
    c->lut_wq = p->wq;
    *lut_out = (const uint16_t *)c->lut.p;
    *len_out = len;
    return OIFT_OK;
}

template <typename T>
static int run_pipeline(oift_b200_ctx *c, const oift_b200_params *p, const T *d_img,
                        const int32_t *d_seeds, const int32_t *d_slabels, int nseeds,
                        const oift_b200_outputs *out, oift_b200_stats *st) {
    TraceRange trace_("oift_b200 pipeline");
    cudaStream_t s = c->stream;
    const int X = p->xsize, Y = p->ysize, Z = p->zsize;
    const size_t N = (size_t)X * Y * Z;
    const int planes = oift_b200_weight_planes(p->adjacency);
    Adjacency adj = make_adjacency(p->adjacency == 4 ? 6 : (p->adjacency == 8 ? 26 : p->adjacency));
    // 26 / 8: the full-neighbourhood OIFT evaluates arc weights from the image itself
    const bool blend = p->weight_mode == OIFT_W_BLEND_Q;
    const bool ig = p->weight_mode == OIFT_W_IMAGEGRAPH;
    // exact base weights (|dI|, or |dI| + 1 on the image graph) must fit 14 bits
    const bool exact = p->weight_mode == OIFT_W_GRAD || ig;
    bool fulln = p->adjacency == 26 || p->adjacency == 8 || blend;
    OiftPlan plan = fulln ? oift_plan_full(X, Y, Z) : oift_plan(X, Y, Z);

    // with every OIFT tile full, the tile step reads only the tile-major code copy
    const bool all_full = !fulln && X % 32 == 0 && Y % plan.TY == 0 && Z % plan.TZ == 0;
    if (!fulln && !all_full) TRY(grow(c, c->W, (size_t)planes * N * sizeof(uint16_t)));
    TRY(grow(c, c->key, N * sizeof(uint32_t)));
    TRY(grow(c, c->tpend, (size_t)plan.ntiles * sizeof(uint32_t)));
    auto oift_ctas_for = [&](const OiftPlan &pl) {
        return std::max((c->oift_ctas > 0 && c->oift_ctas < c->sms) ? c->oift_ctas : c->sms,
                        std::min(c->sms, oift_min_ctas(pl)));
    };
    int octas = oift_ctas_for(plan);
    TRY(grow(c, c->queue, oift_mbox_bytes(plan, octas)));
    TRY(grow(c, c->glob, oift_globals_bytes()));
    TRY(grow(c, c->flag, 4 * sizeof(int)));
    TRY(grow(c, c->minmax, 2 * sizeof(unsigned long long) + 2 * sizeof(int)));
    TRY(grow(c, c->olabel, N * sizeof(int32_t)));
    TRY(grow(c, c->presence, 1024 * sizeof(uint32_t)));

    bool want_relax = out && (out->label || out->mask || out->membership);
    const bool tile_relax = want_relax && !ig;
    cudaEventRecord(c->ev[0], s);
    // ---- intensity range (Wmax of the relaxation) and the labels among the seeds (the
    // relaxation's classes): read back while the weights and the OIFT run, so the host
    // waits for them only when it queues the relaxation ----
    int *d_mm = (int *)c->minmax.p;
    unsigned long long *d_clamp = (unsigned long long *)((char *)c->minmax.p + 2 * sizeof(int) + 8);
    // the previous call ended with the stream idle, so the pinned mirror is free to reuse
    c->hm->mm_init[0] = 0x7fffffff;
    c->hm->mm_init[1] = (int)0x80000000;
    CU(cudaMemcpyAsync(d_mm, c->hm->mm_init, 2 * sizeof(int), cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(d_clamp, 0, sizeof(unsigned long long), s));
    CU(launch_minmax<T>(d_img, N, d_mm, c->sms, s));
    CU(cudaMemcpyAsync(c->hm->mm, d_mm, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (tile_relax) TRY(relax_classes_launch(c, d_slabels, nseeds));
    cudaEventRecord(c->ev[10], s);
    const int *hmm = c->hm->mm;
    bool have_range = false;
    auto need_range = [&]() -> int {
        if (!have_range && cudaEventSynchronize(c->ev[10]) != cudaSuccess) return OIFT_E_CUDA;
        have_range = true;
        return OIFT_OK;
    };

    // ---- exact base weights wider than 14 bits (|dI| above 16383, or |dI| + 1 on the image
    // graph): the OIFT runs with 64-bit keys and evaluates each arc from the image, as the
    // full-neighbourhood tile step does (on the face neighbours for 6 / 4), instead of
    // returning OIFT_E_RANGE; ranges above 2^30 - 1 still do ----
    bool wide = false;
    if (exact && !blend) {
        TRY(need_range());
        const long long span = (long long)hmm[1] - (long long)hmm[0] + (ig ? 1 : 0);
        if (span > OIFT_MAX_BASE) {
            if (span > OIFT_WIDE_MAX_BASE) return OIFT_E_RANGE;
            wide = true;
            fulln = true;
            plan = oift_plan_full(X, Y, Z);
            octas = oift_ctas_for(plan);
            TRY(grow(c, c->key, N * sizeof(unsigned long long)));
            TRY(grow(c, c->tpend, (size_t)plan.ntiles * sizeof(unsigned long long)));
            TRY(grow(c, c->queue, oift_mbox_bytes(plan, octas)));
        }
    }

    // ---- arc weights ----
    nvtxMarkA("oift_b200 weights");
    BuildArgs ba;
    ba.X = X;
    ba.Y = Y;
    ba.Z = Z;
    ba.planes = planes;
    ba.mode = p->weight_mode;
    ba.cap = wide ? OIFT_WIDE_MAX_BASE : (exact ? OIFT_MAX_BASE : p->wq);
    for (int k = 0; k < planes; k++) {
        int i = adj.n / 2 + k;
        ba.dx[k] = adj.dx[i];
        ba.dy[k] = adj.dy[i];
        ba.dz[k] = adj.dz[i];
    }
    ba.lut = nullptr;
    ba.lut_len = 0;
    ba.grad = nullptr;
    ba.blend_a = p->blend_a;
    ba.clamped = d_clamp;
    if (p->weight_mode == OIFT_W_RBF_Q) TRY(rbf_table(c, p, need_range, &ba.lut, &ba.lut_len));
    if (!fulln) {
        // tile-major copy of the codes: a tile step stages its 6 KB in one contiguous run
        TRY(grow(c, c->Wt, (size_t)plan.ntiles * 3 * 1024 * sizeof(uint16_t)));
        ba.Wt = (uint16_t *)c->Wt.p;
        ba.tty = plan.TY;
        ba.ttz = plan.TZ;
        ba.tntx = plan.ntx;
        ba.tnty = plan.nty;
        ba.planes_out = !all_full;
        // the TMA-staged builder reports an image box that did not land in flag[3]
        ba.tma_err = (int *)c->flag.p + 3;
        CU(cudaMemsetAsync(ba.tma_err, 0, sizeof(int), s));
        CU(launch_build_weights<T>(d_img, (uint16_t *)c->W.p, ba, c->sms, s));
    }
    OiftFullN fn{};
    fn.img = d_img;
    fn.img_i16 = sizeof(T) == 2;
    fn.wmode = p->weight_mode;
    fn.wcap = ba.cap;
    fn.lut = ba.lut;
    fn.lut_len = ba.lut_len;
    fn.wide = wide;
    fn.faces = wide && (p->adjacency == 6 || p->adjacency == 4);
    if (blend) {
        // blend weights (exp_gradient_weight.cpp:244-254) from the image and its Sobel
        // gradient normalised to the image maximum (596-608).  The tile stages both as 16-bit
        // values, and an oriented weight must fit the 15-bit cost: wf <= max(I), so
        // max(I) (1 + |per| / 100) must stay below 32767.
        TRY(need_range());
        if (hmm[0] < 0 || hmm[1] > 65535 ||
            (double)hmm[1] * (1.0 + std::fabs((double)p->per) / 100.0) >= 32767.0)
            return OIFT_E_RANGE;
        TRY(grow(c, c->gmap, N * sizeof(int32_t)));
        int *d_mm_g = (int *)((char *)c->minmax.p + 2 * sizeof(int));
        CU(launch_sobel_normalized<T>(d_img, (int32_t *)c->gmap.p, X, Y, Z, d_mm, d_mm_g, c->sms, s));
        fn.blend = true;
        fn.gmap = (const int32_t *)c->gmap.p;
        fn.alpha = p->blend_a;
    }
    cudaEventRecord(c->ev[1], s);

    // ---- OIFT (queued; its outcome is read at the end) ----
    nvtxMarkA("oift_b200 oift");
    int npol = 0;
    float dflt = 0.0f;
    TRY(upload_polarity(c, p, &npol, &dflt));
    OiftScratch S;
    S.spin_limit = c->spin_limit;
    S.max_levels = c->max_levels;
    S.key = (uint32_t *)c->key.p;
    S.tpend = (uint32_t *)c->tpend.p;
    S.mbox = (unsigned long long *)c->queue.p;
    S.g = (OiftGlobals *)c->glob.p;
    TRY(grow(c, c->lprof, 8192 * 2 * sizeof(unsigned int)));
    S.lprof = (unsigned int *)c->lprof.p;
    S.lprof_cap = 8192;
    int32_t *d_cost = out ? out->cost : nullptr;
    int32_t *d_olab = (out && out->oift_label) ? out->oift_label : (int32_t *)c->olabel.p;
    TRY(oift_enqueue(plan, S, (const uint16_t *)c->W.p, X, Y, Z, d_seeds, d_slabels, nseeds,
                     (const float *)c->pol.p, npol, dflt, d_cost, d_olab, (int *)c->flag.p,
                     octas, s, c->ev[4], c->ev[5], fulln ? &fn : nullptr, ig,
                     fulln ? nullptr : ba.Wt));
    CU(cudaMemcpyAsync(&c->hm->g, S.g, sizeof(OiftGlobals), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(c->hm->flag, c->flag.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&c->hm->clamp, d_clamp, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    cudaEventRecord(c->ev[2], s);

    // ---- relaxation ----
    nvtxMarkA("oift_b200 relaxation");
    const int K = p->relax_sweeps;
    RelaxResult rr;
    int ig_kernels = 0;
    if (want_relax && ig) {
        // ORelax_1(sImageGraph): one membership channel, binary labels
        TRY(grow(c, c->memb, 2 * N * sizeof(float)));
        TRY(grow(c, c->igring, N * sizeof(uint16_t)));
        TRY(grow(c, c->seedc, N));
        TRY(grow(c, c->igsmall, 4 * sizeof(int)));
        IgRelax R;
        R.X = X;
        R.Y = Y;
        R.adjacency = p->adjacency;
        R.per = p->per;
        R.sweeps = K;
        R.olabel = d_olab;
        R.seeds = d_seeds;
        R.nseeds = nseeds;
        R.m0 = (float *)c->memb.p;
        R.m1 = R.m0 + N;
        R.ring = (uint16_t *)c->igring.p;
        R.seedf = (uint8_t *)c->seedc.p;
        R.small = (int *)c->igsmall.p;
        R.label = out->label;
        R.mask = out->mask;
        R.membership = out->membership;
        R.ev_begin = c->ev[6];
        R.ev_end = c->ev[7];
        TRY(ig_relax_run<T>(R, d_img, s, c->sms, &ig_kernels));
        rr.nclasses = 1;
    } else if (tile_relax) {
        // the early readback landed long ago: the OIFT is still running when the sweeps
        // are queued behind it
        TRY(need_range());
        RelaxPlan pl;
        TRY(relax_plan_finish(c, p, hmm, &pl));
        TRY(relax_reserve(c, N, pl.nclasses, pl.maxl, X, Y, Z, K));
        CU(cudaMemcpyAsync(c->l2c.p, pl.l2c.data(), (pl.maxl + 1) * sizeof(int),
                           cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(c->classes.p, pl.classes.data(), pl.nclasses * sizeof(int),
                           cudaMemcpyHostToDevice, s));
        TRY(relax_launch<T>(c, p, d_img, d_seeds, nseeds, d_olab, pl, (const int *)c->l2c.p,
                            (const int *)c->classes.p, out, true));
        rr.nclasses = pl.nclasses;
        rr.dilations = 3;
    }
    const int relax_dilations = rr.dilations;
    cudaEventRecord(c->ev[3], s);
    CU(cudaStreamSynchronize(s));
    CU(cudaGetLastError());
    int levels = 0;
    long long steps = 0;
    TRY(oift_result(c->hm->g, c->hm->flag[0], &levels, &steps, c->oift_cycles));
    if (!fulln && c->hm->flag[3]) return OIFT_E_CUDA;  // a builder tile whose image box did not land
    if (tile_relax) TRY(relax_tma_status(c));
    const unsigned long long hclamp = c->hm->clamp;
    if (exact && hclamp) return OIFT_E_RANGE;
    const int nclasses = rr.nclasses;
    const long long relax_active = tile_relax ? relax_active_sweeps(c, K) : 0;
    if (st) {
        st->levels = levels;
        st->tile_steps = steps;
        st->clamped = (long long)hclamp;
        st->nclasses = nclasses;
        cudaEventElapsedTime(&st->ms_weights, c->ev[0], c->ev[1]);
        cudaEventElapsedTime(&st->ms_oift, c->ev[1], c->ev[2]);
        cudaEventElapsedTime(&st->ms_relax, c->ev[2], c->ev[3]);
        cudaEventElapsedTime(&st->ms_total, c->ev[0], c->ev[3]);
        // minmax, build, seeds, persistent OIFT, finalize (+ presence, init, seed map,
        // K sweeps, argmax when relaxing)
        // minmax, build, seeds, persistent OIFT, finalize; relaxing adds presence, 2 inits,
        // seed map, boundary tiles, dilations, histogram, K sweeps, argmax
        st->kernels = 5 + (want_relax ? (ig ? ig_kernels : 7 + relax_dilations + K) : 0);
        st->relax_active_voxel_sweeps = relax_active;
        cudaEventElapsedTime(&st->ms_oift_kernel, c->ev[4], c->ev[5]);
        st->ms_sweeps = 0.0f;
        for (int i = 0; i < 24; i++) st->oift_cycles[i] = (long long)c->oift_cycles[i];
        if (want_relax) cudaEventElapsedTime(&st->ms_sweeps, c->ev[6], c->ev[7]);
    }
    return OIFT_OK;
}

extern "C" {

int oift_b200_run_device_i16(oift_b200_ctx *c, const oift_b200_params *p, const int16_t *image,
                             const int32_t *seeds, const int32_t *seed_labels, int nseeds,
                             const oift_b200_outputs *out, oift_b200_stats *stats) {
    if (!c || !image || (nseeds > 0 && (!seeds || !seed_labels))) return OIFT_E_BAD_ARG;
    TRY(check_params(p));
    if (nseeds <= 0) return OIFT_E_NO_SEEDS;
    cudaSetDevice(c->device);
    return run_pipeline<int16_t>(c, p, image, seeds, seed_labels, nseeds, out, stats);
}

int oift_b200_run_host(oift_b200_ctx *c, const oift_b200_params *p, const int32_t *image,
                       int32_t *label, const int32_t *seeds, int nseeds, int32_t *cost,
                       float *membership, int membership_cap_classes, uint8_t *mask,
                       oift_b200_stats *stats) {
    TraceRange trace_("oift_b200_run_host");
    if (!c || !image || !label || (nseeds > 0 && !seeds)) return OIFT_E_BAD_ARG;
    TRY(check_params(p));
    if (nseeds <= 0) return OIFT_E_NO_SEEDS;
    cudaSetDevice(c->device);
    const size_t N = (size_t)p->xsize * p->ysize * p->zsize;
    cudaStream_t s = c->stream;
    // the seed labels are staged in pinned memory owned by the context, so their copy is
    // asynchronous; wait for an earlier call's copy from it (and nothing else on the stream)
    if (cudaEventSynchronize(c->ev[11]) != cudaSuccess) return OIFT_E_CUDA;
    if (c->hslab_n < (size_t)nseeds) {
        if (c->hslab) cudaFreeHost(c->hslab);
        c->hslab = nullptr;
        c->hslab_n = 0;
        if (cudaHostAlloc(&c->hslab, (size_t)nseeds * sizeof(int32_t), cudaHostAllocDefault) !=
            cudaSuccess) {
            cudaGetLastError();
            c->hslab = nullptr;
            return OIFT_E_OOM;
        }
        c->hslab_n = (size_t)nseeds;
    }
    TRY(grow(c, c->img32, N * sizeof(int32_t)));
    TRY(grow(c, c->seeds, (size_t)nseeds * sizeof(int32_t)));
    TRY(grow(c, c->slabels, (size_t)nseeds * sizeof(int32_t)));
    TRY(grow(c, c->flabel, N * sizeof(int32_t)));
    if (cost) TRY(grow(c, c->cost, N * sizeof(int32_t)));
    if (mask) TRY(grow(c, c->mask8, N));
    // the image copy is queued first: from pinned memory it runs while the host gathers the
    // seed labels (a bad seed then returns with the copy still queued into a context buffer)
    CU(cudaMemcpyAsync(c->img32.p, image, N * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    // the seed labels, gathered from the label map (a read scattered over the whole map, so
    // large seed lists are split over a few host threads); the first bad seed in list order
    // decides the error, as a single pass would
    int32_t *slab = c->hslab;
    auto gather = [&](int i0, int i1) -> int {
        for (int i = i0; i < i1; i++) {
            if (seeds[i] < 0 || (size_t)seeds[i] >= N) return OIFT_E_SEED_RANGE;
            const int lb = label[seeds[i]];
            slab[i] = lb < 0 ? 0 : lb;
            if (slab[i] > OIFT_MAX_LABEL) return OIFT_E_BAD_ARG;
        }
        return OIFT_OK;
    };
    const int nthreads = nseeds < (1 << 16) ? 1
        : (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    if (nthreads == 1) {
        TRY(gather(0, nseeds));
    } else {
        std::vector<int> rcs(nthreads, OIFT_OK);
        std::vector<std::thread> pool;
        const int chunk = (nseeds + nthreads - 1) / nthreads;
        auto run_chunk = [&](int k) {
            rcs[k] = gather(std::min(nseeds, k * chunk), std::min(nseeds, (k + 1) * chunk));
        };
        int spawned = 1;  // chunk 0 runs on the calling thread
        try {
            for (int k = 1; k < nthreads; k++, spawned++) pool.emplace_back(run_chunk, k);
        } catch (...) {
            // no exception leaves the C ABI: chunks that got no thread run here
        }
        for (int k = spawned; k < nthreads; k++) run_chunk(k);
        run_chunk(0);
        for (auto &th : pool) th.join();
        for (int k = 0; k < nthreads; k++) TRY(rcs[k]);
    }
    CU(cudaMemcpyAsync(c->seeds.p, seeds, (size_t)nseeds * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c->slabels.p, slab, (size_t)nseeds * sizeof(int32_t),
                       cudaMemcpyHostToDevice, s));
    CU(cudaEventRecord(c->ev[11], s));
    oift_b200_outputs o{};
    o.cost = cost ? (int32_t *)c->cost.p : nullptr;
    const bool relax = p->relax_sweeps > 0 || membership || mask;
    // without sweeps the labels are the OIFT labels (argmax of the one-hot start)
    if (relax)
        o.label = (int32_t *)c->flabel.p;
    else
        o.oift_label = (int32_t *)c->flabel.p;
    o.mask = mask ? (uint8_t *)c->mask8.p : nullptr;
    oift_b200_stats lst{};
    oift_b200_stats *sp = stats ? stats : &lst;
    int rc;
    if (membership) {
        // the relaxation's classes are 0 and the labels among the seeds (gft_ift.cpp:
        // 8684-8712): the membership holds one plane per class, checked against the cap
        // first; the image-graph relaxation keeps a single channel (gft_ift.cpp:7683-7847)
        std::vector<int32_t> present(slab, slab + nseeds);
        present.push_back(0);
        std::sort(present.begin(), present.end());
        const long long nclasses = p->weight_mode == OIFT_W_IMAGEGRAPH
            ? 1 : std::unique(present.begin(), present.end()) - present.begin();
        if (nclasses > membership_cap_classes) return OIFT_E_BAD_ARG;
        TRY(grow(c, c->hmemb, (size_t)nclasses * N * sizeof(float)));
        o.membership = (float *)c->hmemb.p;
    }
    rc = run_pipeline<int32_t>(c, p, (const int32_t *)c->img32.p, (const int32_t *)c->seeds.p,
                               (const int32_t *)c->slabels.p, nseeds, &o, sp);
    if (rc == OIFT_OK) {
        cudaMemcpyAsync(label, c->flabel.p, N * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        if (cost) cudaMemcpyAsync(cost, o.cost, N * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        if (mask) cudaMemcpyAsync(mask, o.mask, N, cudaMemcpyDeviceToHost, s);
        if (membership)
            cudaMemcpyAsync(membership, o.membership, (size_t)sp->nclasses * N * sizeof(float),
                            cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) rc = OIFT_E_CUDA;
    }
    return rc;
}

int oift_b200_relax_host(oift_b200_ctx *c, const oift_b200_params *p, const int32_t *image,
                         int32_t *label, const int32_t *seeds, int nseeds, float *membership,
                         int membership_cap_classes, uint8_t *mask) {
    TraceRange trace_("oift_b200_relax_host");
    if (!c || !image || !label || (nseeds > 0 && !seeds)) return OIFT_E_BAD_ARG;
    TRY(check_params(p));
    if (p->weight_mode == OIFT_W_IMAGEGRAPH) return OIFT_E_UNSUPPORTED;
    if (nseeds <= 0) return OIFT_E_NO_SEEDS;
    cudaSetDevice(c->device);
    const int X = p->xsize, Y = p->ysize, Z = p->zsize;
    const size_t N = (size_t)X * Y * Z;
    cudaStream_t s = c->stream;
    if (cudaEventSynchronize(c->ev[11]) != cudaSuccess) return OIFT_E_CUDA;
    if (c->hslab_n < (size_t)nseeds) {
        if (c->hslab) cudaFreeHost(c->hslab);
        c->hslab = nullptr;
        c->hslab_n = 0;
        if (cudaHostAlloc(&c->hslab, (size_t)nseeds * sizeof(int32_t), cudaHostAllocDefault) !=
            cudaSuccess) {
            cudaGetLastError();
            c->hslab = nullptr;
            return OIFT_E_OOM;
        }
        c->hslab_n = (size_t)nseeds;
    }
    int32_t *slab = c->hslab;
    for (int i = 0; i < nseeds; i++) {
        if (seeds[i] < 0 || (size_t)seeds[i] >= N) return OIFT_E_SEED_RANGE;
        const int lb = label[seeds[i]];
        slab[i] = lb < 0 ? 0 : lb;
        if (slab[i] > OIFT_MAX_LABEL) return OIFT_E_BAD_ARG;
    }
    TRY(grow(c, c->img32, N * sizeof(int32_t)));
    TRY(grow(c, c->seeds, (size_t)nseeds * sizeof(int32_t)));
    TRY(grow(c, c->slabels, (size_t)nseeds * sizeof(int32_t)));
    TRY(grow(c, c->flabel, N * sizeof(int32_t)));
    TRY(grow(c, c->minmax, 2 * sizeof(unsigned long long) + 2 * sizeof(int)));
    if (mask) TRY(grow(c, c->mask8, N));
    CU(cudaMemcpyAsync(c->img32.p, image, N * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c->flabel.p, label, N * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c->seeds.p, seeds, (size_t)nseeds * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c->slabels.p, slab, (size_t)nseeds * sizeof(int32_t),
                       cudaMemcpyHostToDevice, s));
    CU(cudaEventRecord(c->ev[11], s));
    // intensity range (Wmax, gft_ift.cpp:8733-8734) and the classes among the seeds
    int *d_mm = (int *)c->minmax.p;
    c->hm->mm_init[0] = 0x7fffffff;
    c->hm->mm_init[1] = (int)0x80000000;
    CU(cudaMemcpyAsync(d_mm, c->hm->mm_init, 2 * sizeof(int), cudaMemcpyHostToDevice, s));
    CU(launch_minmax<int32_t>((const int32_t *)c->img32.p, N, d_mm, c->sms, s));
    CU(cudaMemcpyAsync(c->hm->mm, d_mm, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    RelaxPlan pl;
    TRY(relax_plan(c, p, (const int32_t *)c->slabels.p, nseeds, c->hm->mm, &pl));
    if (membership && pl.nclasses > membership_cap_classes) return OIFT_E_BAD_ARG;
    if (membership) TRY(grow(c, c->hmemb, (size_t)pl.nclasses * N * sizeof(float)));
    TRY(relax_reserve(c, N, pl.nclasses, pl.maxl, X, Y, Z, p->relax_sweeps));
    CU(cudaMemcpyAsync(c->l2c.p, pl.l2c.data(), (pl.maxl + 1) * sizeof(int),
                       cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c->classes.p, pl.classes.data(), pl.nclasses * sizeof(int),
                       cudaMemcpyHostToDevice, s));
    oift_b200_outputs o{};
    o.label = (int32_t *)c->flabel.p;  // the one-hot start is read before the argmax writes
    o.mask = mask ? (uint8_t *)c->mask8.p : nullptr;
    o.membership = membership ? (float *)c->hmemb.p : nullptr;
    TRY(relax_launch<int32_t>(c, p, (const int32_t *)c->img32.p, (const int32_t *)c->seeds.p,
                              nseeds, (const int32_t *)c->flabel.p, pl, (const int *)c->l2c.p,
                              (const int *)c->classes.p, &o, false));
    CU(cudaMemcpyAsync(label, c->flabel.p, N * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    if (mask) CU(cudaMemcpyAsync(mask, c->mask8.p, N, cudaMemcpyDeviceToHost, s));
    if (membership)
        CU(cudaMemcpyAsync(membership, c->hmemb.p, (size_t)pl.nclasses * N * sizeof(float),
                           cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    CU(cudaGetLastError());
    return relax_tma_status(c);
}

int oift_b200_bottleneck_arcs(oift_b200_ctx *c, const oift_b200_params *p, const int16_t *image,
                              const int32_t *cost, const int32_t *label, const int32_t *seeds,
                              int nseeds, int64_t *arcs) {
    if (!c || !image || !cost || !label || !arcs || (nseeds > 0 && !seeds)) return OIFT_E_BAD_ARG;
    TRY(check_params(p));
    if (p->weight_mode != OIFT_W_GRAD && p->weight_mode != OIFT_W_GRAD_Q) return OIFT_E_UNSUPPORTED;
    if (p->per_class) return OIFT_E_UNSUPPORTED;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    const size_t N = (size_t)p->xsize * p->ysize * p->zsize;
    TRY(grow(c, c->bseed, N));
    TRY(grow(c, c->barcs, N * sizeof(long long)));
    TRY(grow(c, c->flag, 4 * sizeof(int)));
    CU(cudaMemsetAsync(c->bseed.p, 0, N, s));
    if (nseeds > 0)
        seed_flag_kernel<<<(nseeds + 255) / 256, 256, 0, s>>>(seeds, nseeds, N,
                                                              (uint8_t *)c->bseed.p);
    BottleneckSetup S{};
    S.X = p->xsize;
    S.Y = p->ysize;
    S.Z = p->zsize;
    S.adjacency = p->adjacency;
    S.img = image;
    S.cost = cost;
    S.label = label;
    S.seed = (const uint8_t *)c->bseed.p;
    S.wmode = p->weight_mode;
    S.wq = p->wq;
    S.per = p->per;
    return bottleneck_run(S, s, c->sms, (long long *)arcs, (long long *)c->barcs.p,
                          (int *)c->flag.p + 2, &c->hm->flag[2], nullptr);
}

int oift_b200_cost_adjoint(oift_b200_ctx *c, const oift_b200_adjoint_params *ap,
                           const int16_t *image, const float *grad_map, const int32_t *label,
                           const int64_t *arcs, const uint8_t *truth, double *loss,
                           double *grad) {
    if (!c || !ap || !image || !label || !arcs || !truth || !loss) return OIFT_E_BAD_ARG;
    if (ap->xsize <= 0 || ap->ysize <= 0 || ap->zsize <= 0 || !(ap->sigma > 0.0f) ||
        !(std::fabs(ap->alpha) <= 1.0f) || !(ap->beta >= 0.0f && ap->beta <= 1.0f) ||
        !(ap->eps >= 0.0f))
        return OIFT_E_BAD_ARG;
    if (ap->adjacency == 4 || ap->adjacency == 8) {
        if (ap->zsize != 1) return OIFT_E_BAD_ARG;
    } else if (ap->adjacency != 6 && ap->adjacency != 26) {
        return OIFT_E_BAD_ARG;
    }
    cudaSetDevice(c->device);
    const int max_blocks = c->sms * 8;
    TRY(grow(c, c->csums, (size_t)max_blocks * 9 * sizeof(double)));
    CostLossSetup S{};
    S.X = ap->xsize;
    S.Y = ap->ysize;
    S.Z = ap->zsize;
    S.adjacency = ap->adjacency;
    S.img = image;
    S.g = grad_map;
    S.label = label;
    S.arcs = (const long long *)arcs;
    S.truth = truth;
    S.sigma = ap->sigma;
    S.alpha = ap->alpha;
    S.beta = ap->beta;
    S.eps = ap->eps;
    return cost_loss_run(S, c->stream, c->sms, (double *)c->csums.p, max_blocks, loss, grad);
}

int oift_b200_build_weights_i16(oift_b200_ctx *c, const oift_b200_params *p,
                                const int16_t *image, uint16_t *weights, long long *clamped) {
    if (!c || !image || !weights) return OIFT_E_BAD_ARG;
    int chk = check_params(p);
    if (chk != OIFT_OK && chk != OIFT_E_UNSUPPORTED) return chk;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    const int X = p->xsize, Y = p->ysize, Z = p->zsize;
    const size_t N = (size_t)X * Y * Z;
    Adjacency adj = make_adjacency(p->adjacency == 4 ? 6 : (p->adjacency == 8 ? 26 : p->adjacency));
    TRY(grow(c, c->minmax, 2 * sizeof(unsigned long long) + 2 * sizeof(int)));
    unsigned long long *d_clamp = (unsigned long long *)((char *)c->minmax.p + 2 * sizeof(int) + 8);
    int *d_mm = (int *)c->minmax.p;
    BuildArgs ba;
    ba.X = X;
    ba.Y = Y;
    ba.Z = Z;
    ba.planes = oift_b200_weight_planes(p->adjacency);
    ba.mode = p->weight_mode;
    ba.cap = (p->weight_mode == OIFT_W_GRAD || p->weight_mode == OIFT_W_IMAGEGRAPH) ? OIFT_MAX_BASE : p->wq;
    for (int k = 0; k < ba.planes; k++) {
        int i = adj.n / 2 + k;
        ba.dx[k] = adj.dx[i];
        ba.dy[k] = adj.dy[i];
        ba.dz[k] = adj.dz[i];
    }
    ba.lut = nullptr;
    ba.lut_len = 0;
    ba.grad = nullptr;
    ba.blend_a = p->blend_a;
    ba.clamped = d_clamp;
    if (p->weight_mode == OIFT_W_BLEND_Q) return OIFT_E_UNSUPPORTED;
    if (p->weight_mode == OIFT_W_RBF_Q) {
        int mm_init[2] = {0x7fffffff, (int)0x80000000};
        CU(cudaMemcpyAsync(d_mm, mm_init, sizeof(mm_init), cudaMemcpyHostToDevice, s));
        CU(launch_minmax<int16_t>(image, N, d_mm, c->sms, s));
        int hmm[2];
        CU(cudaMemcpyAsync(hmm, d_mm, sizeof(hmm), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        int len = hmm[1] - hmm[0] + 1;
        std::vector<uint16_t> lut(len);
        double sg = p->rbf_sigma;
        for (int d = 0; d < len; d++) {
            double a = std::exp(-((double)d * (double)d) / (2.0 * sg * sg));
            double v = std::floor((double)p->wq * (1.0 - a) + 0.5);
            lut[d] = (uint16_t)(v < 0 ? 0 : (v > p->wq ? p->wq : v));
        }
        TRY(grow(c, c->lut, len * sizeof(uint16_t)));
        c->lut_len = 0;  // the cached pipeline table is overwritten
        CU(cudaMemcpyAsync(c->lut.p, lut.data(), len * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
        ba.lut = (const uint16_t *)c->lut.p;
        ba.lut_len = len;
    }
    CU(cudaMemsetAsync(d_clamp, 0, sizeof(unsigned long long), s));
    CU(launch_build_weights<int16_t>(image, weights, ba, c->sms, s));
    unsigned long long h = 0;
    CU(cudaMemcpyAsync(&h, d_clamp, sizeof(h), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (clamped) *clamped = (long long)h;
    return OIFT_OK;
}

// ----------------------------------------------------- reference drop-in ----
static std::mutex g_dropin_mu;
static oift_b200_ctx *g_dropin_ctx = nullptr;

int oift_b200_last_status(void) { return g_last_status; }

int oift_gpu_run(int cost_mode, const int *h_image, int *h_labels, int n, int xsize, int ysize,
                 int zsize, const float *h_per_class, int max_label, const int *h_seeds,
                 int n_seeds) {
    if (cost_mode != 0) {
        g_last_status = OIFT_E_UNSUPPORTED;
        return -1;
    }
    return oift_fmax_gpu_run(h_image, h_labels, n, xsize, ysize, zsize, h_per_class, max_label,
                             h_seeds, n_seeds);
}

int oift_fmax_gpu_run(const int *h_image, int *h_labels, int n, int xsize, int ysize, int zsize,
                      const float *h_per_class, int max_label, const int *h_seeds, int n_seeds) {
    std::lock_guard<std::mutex> lk(g_dropin_mu);
    g_last_status = OIFT_E_BAD_ARG;
    if (!h_image || !h_labels || !h_per_class || n <= 0 || max_label < 0) return -1;
    if ((long long)xsize * ysize * zsize != n) return -1;
    if (!g_dropin_ctx) {
        int dev = 0;
        cudaGetDevice(&dev);
        int rc = oift_b200_create(&g_dropin_ctx, dev);
        if (rc != OIFT_OK) {
            g_last_status = rc;
            return -1;
        }
    }
    oift_b200_params p{};
    p.xsize = xsize;
    p.ysize = ysize;
    p.zsize = zsize;
    p.adjacency = zsize == 1 ? 4 : 6;
    p.weight_mode = OIFT_W_GRAD;
    p.wq = OIFT_MAX_BASE;
    p.per_class = h_per_class;
    p.max_label = max_label;
    p.relax_sweeps = 0;
    oift_b200_stats st{};
    int rc = oift_b200_run_host(g_dropin_ctx, &p, h_image, h_labels, h_seeds, n_seeds, nullptr,
                                nullptr, 0, nullptr, &st);
    g_last_status = rc;
    return rc == OIFT_OK ? st.levels : -1;
}


// --------------------------------------------------------- steps of the CLI ----
// oiftrelax.cpp main: shift to >= 0 (263-268), GaussianBlur twice (368-377), OIFT +
// relaxation (379-401), conditional dilation of a binary result (403-414).

// Kernel3::SphericalGaussian(R = 1, s = 10, f = 1) + Normalize (gft_filtering3.cpp:106-126,
// 72-83), evaluated in float exactly as the C++ source: val = s * exp(-f * (r2 / R2)) with
// the float overload of exp, wt = float sum in Spheric order, val /= wt.
static void blur_weights(float *w0, float *w1) {
    const float R = 1.0f, sg = 10.0f, f = 1.0f, R2 = R * R;
    float val[7];
    for (int i = 0; i < 7; i++) {
        const float r2 = i == 0 ? 0.0f : 1.0f;
        val[i] = sg * std::exp(-f * (r2 / R2));
    }
    float wt = 0.0f;
    for (int i = 0; i < 7; i++) wt += val[i];
    *w0 = val[0] / wt;
    *w1 = val[1] / wt;
}

// `passes` blurs of the device int32 volume `in` into `out` (in == out allowed).
static int blur_passes_i32(oift_b200_ctx *c, const int32_t *in, int32_t *out, int X, int Y,
                           int Z, int passes) {
    const size_t N = (size_t)X * Y * Z;
    float w0, w1;
    blur_weights(&w0, &w1);
    TRY(grow(c, c->cimg1, N * sizeof(int32_t)));
    const int32_t *src = in;
    for (int i = 0; i < passes; i++) {
        // the last pass lands in `out`; earlier ones alternate so that no pass reads its
        // own output
        int32_t *dst = ((passes - 1 - i) % 2 == 0) ? out : (int32_t *)c->cimg1.p;
        if (dst == src) dst = (dst == out) ? (int32_t *)c->cimg1.p : out;
        CU(launch_gaussian_blur<int32_t>(src, dst, X, Y, Z, w0, w1, c->stream));
        src = dst;
    }
    if (src != out)
        CU(cudaMemcpyAsync(out, src, N * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
    return OIFT_OK;
}

// Spheric(r) offsets (gft_adjrel3.cpp:47-85), centre included.
static std::vector<int> spheric_offsets(float r) {
    std::vector<int> off;
    const int r0 = (int)r, r2 = (int)(r * r);
    for (int dz = -r0; dz <= r0; dz++)
        for (int dy = -r0; dy <= r0; dy++)
            for (int dx = -r0; dx <= r0; dx++)
                if (dx * dx + dy * dy + dz * dz <= r2) {
                    off.push_back(dx);
                    off.push_back(dy);
                    off.push_back(dz);
                }
    return off;
}

// Conditional dilation (oiftrelax.cpp:87-169) of the device label map by the border voxels
// whose intensity in `img` is within the percentile.  *added = voxels relabelled.
static int conditional_dilation(oift_b200_ctx *c, const int32_t *img, int32_t *label, int X,
                                int Y, int Z, float radius, float percentile, long long *added) {
    cudaStream_t s = c->stream;
    const size_t N = (size_t)X * Y * Z;
    if (added) *added = 0;
    const std::vector<int> off = spheric_offsets(radius);
    const int noff = (int)off.size() / 3;
    const size_t chunk = 8192;
    const size_t nchunks = (N + chunk - 1) / chunk;
    TRY(grow(c, c->dborder, N));
    TRY(grow(c, c->dhist, (65536 + 16) * sizeof(unsigned)));
    TRY(grow(c, c->daux, std::max((size_t)noff * 3 * sizeof(int), 2 * nchunks * sizeof(unsigned))));
    unsigned *hist = (unsigned *)c->dhist.p, *d_count = hist + 65536;
    int *d_off = (int *)c->daux.p;
    CU(cudaMemcpyAsync(d_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(hist, 0, (65536 + 16) * sizeof(unsigned), s));
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((N + 255) / 256, (size_t)c->sms * 16));
    dilation_border_kernel<<<blocks, 256, 0, s>>>(label, img, (uint8_t *)c->dborder.p, X, Y, Z,
                                                  d_off, noff, hist, d_count);
    CU(cudaGetLastError());
    std::vector<unsigned> h(65537);
    CU(cudaMemcpyAsync(h.data(), hist, 65537 * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const long long n = h[65536];
    if (n == 0) return OIFT_OK;  // the reference indexes out of range here; nothing to add
    // float index_percentile = (percentil / 100.0) * (size - 1); int value_position = (int)
    const float index_percentile = (percentile / 100.0) * (double)(size_t)(n - 1);
    const double ipd = (double)index_percentile;
    const long long vp = ipd >= 2147483647.0 ? 2147483647LL
                         : ipd <= -2147483648.0 ? -2147483648LL
                                                : (long long)static_cast<int>(index_percentile);
    const long long keep = std::min<long long>(std::max<long long>(vp + 1, 0), n);
    if (keep == 0) return OIFT_OK;
    const long long k = keep - 1;  // rank of the last voxel kept
    long long cum = 0;
    uint32_t hi = 0;
    for (; hi < 65536; hi++) {
        if (cum + h[hi] > (unsigned long long)k) break;
        cum += h[hi];
    }
    CU(cudaMemsetAsync(hist, 0, 65536 * sizeof(unsigned), s));
    dilation_hist_lo_kernel<<<blocks, 256, 0, s>>>((const uint8_t *)c->dborder.p, img, N, hi, hist);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(h.data(), hist, 65536 * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    uint32_t lo = 0;
    for (; lo < 65536; lo++) {
        if (cum + h[lo] > (unsigned long long)k) break;
        cum += h[lo];
    }
    const uint32_t pivot = (hi << 16) | lo;
    const unsigned take = (unsigned)(keep - cum);  // pivot-valued voxels kept, in address order
    unsigned *d_counts = (unsigned *)c->daux.p, *d_base = d_counts + nchunks;
    dilation_tie_count_kernel<<<(unsigned)nchunks, 256, 0, s>>>((const uint8_t *)c->dborder.p,
                                                                img, N, chunk, pivot, d_counts);
    CU(cudaGetLastError());
    std::vector<unsigned> cnt(nchunks);
    CU(cudaMemcpyAsync(cnt.data(), d_counts, nchunks * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    unsigned run = 0;
    for (size_t i = 0; i < nchunks; i++) {
        const unsigned v = cnt[i];
        cnt[i] = run;
        run += v;
    }
    CU(cudaMemcpyAsync(d_base, cnt.data(), nchunks * sizeof(unsigned), cudaMemcpyHostToDevice, s));
    dilation_apply_kernel<<<(unsigned)nchunks, 256, 0, s>>>((const uint8_t *)c->dborder.p, img,
                                                            label, N, chunk, pivot, d_base, take);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(s));
    if (added) *added = keep;
    return OIFT_OK;
}

extern "C++" {

// Every labelled voxel (!= NIL) of the device map `lab` as a seed, in address order.
static int seeds_from_labels(oift_b200_ctx *c, const int32_t *lab, size_t N, DevBuf &seeds,
                             DevBuf &slabels, int *nout) {
    cudaStream_t s = c->stream;
    const size_t chunk = 8192, nch = (N + chunk - 1) / chunk;
    TRY(grow(c, c->yaux, 2 * nch * sizeof(unsigned)));
    unsigned *d_cnt = (unsigned *)c->yaux.p, *d_base = d_cnt + nch;
    seeds_count_kernel<<<(unsigned)nch, 256, 0, s>>>(lab, N, chunk, d_cnt);
    CU(cudaGetLastError());
    std::vector<unsigned> h(nch);
    CU(cudaMemcpyAsync(h.data(), d_cnt, nch * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    unsigned long long run = 0;
    for (size_t i = 0; i < nch; i++) {
        const unsigned v = h[i];
        h[i] = (unsigned)run;
        run += v;
    }
    if (run > 0x7fffffffULL) return OIFT_E_RANGE;
    TRY(grow(c, seeds, std::max<size_t>(run, 1) * sizeof(int32_t)));
    TRY(grow(c, slabels, std::max<size_t>(run, 1) * sizeof(int32_t)));
    CU(cudaMemcpyAsync(d_base, h.data(), nch * sizeof(unsigned), cudaMemcpyHostToDevice, s));
    seeds_scatter_kernel<<<(unsigned)nch, 256, 0, s>>>(lab, N, chunk, d_base, (int32_t *)seeds.p,
                                                       (int32_t *)slabels.p);
    CU(cudaGetLastError());
    *nout = (int)run;
    return OIFT_OK;
}

// ScaleLabel(.., none) index of fine coordinate u along an axis of n fine / nc coarse
// voxels (gft_scene32.cpp:1108-1116, 1240-1262): x = (u - n/2.) * (1/2.f) + nc/2. in
// double, stored as float; (int)(x + 0.5); clamped to [0, nc - 1].
static int nn_index(int u, int n, int nc) {
    const float ratio = 1.0f / 2.0f;  // ref->dx / scn->dx, fine spacing over coarse
    const float x = (float)(((double)u - n / 2.) * (double)ratio + nc / 2.);
    int v = (int)((double)x + 0.5);
    if (v > nc - 1)
        v = nc - 1;
    else if (v < 0)
        v = 0;
    return v;
}

static int coarse_extent(int n) {  // Subsampling (gft_filtering3.cpp:449-455)
    const int c = n / 2 + n % 2;
    return c % 2 == 0 ? c + 1 : c;
}

// The two-level cascade (exp_coarse_to_fine.cpp:327-414) on the device: d_fscn is the
// blurred volume shifted to >= 0; d_label_in holds the seed labels (NIL elsewhere) of the
// nseeds device seeds.  The result goes to d_label_out.
static int run_pyramid(oift_b200_ctx *c, const oift_b200_params *p, const int32_t *d_fscn,
                       const int32_t *d_label_in, const int32_t *d_seeds, int nseeds,
                       float percentile, int32_t *d_label_out, oift_b200_stats *st) {
    TraceRange trace_("oift_b200 cascade");
    cudaStream_t s = c->stream;
    const int X = p->xsize, Y = p->ysize, Z = p->zsize;
    const size_t N = (size_t)X * Y * Z;
    const int cx = coarse_extent(X), cy = coarse_extent(Y), cz = coarse_extent(Z);
    const size_t cn = (size_t)cx * cy * cz;
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((N + 255) / 256, (size_t)c->sms * 16));
    const int cblocks = (int)std::max<size_t>(1, std::min<size_t>((cn + 255) / 256, (size_t)c->sms * 16));
    cudaEventRecord(c->ev[8], s);
    // ---- coarse pass ----
    TRY(grow(c, c->yimg, cn * sizeof(int32_t)));
    TRY(grow(c, c->ylab, cn * sizeof(int32_t)));
    TRY(grow(c, c->yfirst, cn * sizeof(unsigned)));
    pyr_subsample_kernel<<<cblocks, 256, 0, s>>>(d_fscn, (int32_t *)c->yimg.p, X, Y, Z, cx, cy, cz);
    CU(cudaMemsetAsync(c->yfirst.p, 0xFF, cn * sizeof(unsigned), s));
    if (nseeds > 0)
        pyr_coarse_first_kernel<<<std::min((nseeds + 255) / 256, c->sms * 16), 256, 0, s>>>(
            d_seeds, nseeds, X, Y, Z, cx, cy, cz, (unsigned *)c->yfirst.p);
    pyr_coarse_labels_kernel<<<cblocks, 256, 0, s>>>((const unsigned *)c->yfirst.p, d_seeds,
                                                     d_label_in, cn, (int32_t *)c->ylab.p);
    CU(cudaGetLastError());
    int ncs = 0;
    TRY(seeds_from_labels(c, (const int32_t *)c->ylab.p, cn, c->yseeds, c->yslab, &ncs));
    if (ncs == 0) return OIFT_E_NO_SEEDS;
    oift_b200_params pc = *p;
    pc.xsize = cx;
    pc.ysize = cy;
    pc.zsize = cz;
    oift_b200_outputs oc{};
    oc.label = (int32_t *)c->ylab.p;  // the coarse seed map is no longer needed
    oift_b200_stats stc{};
    TRY(run_pipeline<int32_t>(c, &pc, (const int32_t *)c->yimg.p, (const int32_t *)c->yseeds.p,
                              (const int32_t *)c->yslab.p, ncs, &oc, &stc));
    // ---- upscale, band around the coarse boundaries to NIL, merge ----
    TRY(grow(c, c->yup, N * sizeof(int32_t)));
    TRY(grow(c, c->ymerge, N * sizeof(int32_t)));
    {
        std::vector<int> tab((size_t)X + Y + Z);
        for (int u = 0; u < X; u++) tab[u] = nn_index(u, X, cx);
        for (int u = 0; u < Y; u++) tab[X + u] = nn_index(u, Y, cy);
        for (int u = 0; u < Z; u++) tab[X + Y + u] = nn_index(u, Z, cz);
        const Adjacency adj =
            make_adjacency(p->adjacency == 4 ? 6 : (p->adjacency == 8 ? 26 : p->adjacency));
        std::vector<int> off;
        for (int i = 0; i < adj.n; i++) {
            off.push_back(adj.dx[i]);
            off.push_back(adj.dy[i]);
            off.push_back(adj.dz[i]);
        }
        TRY(grow(c, c->dhist, (tab.size() + off.size()) * sizeof(int)));
        int *d_tab = (int *)c->dhist.p, *d_off = d_tab + tab.size();
        CU(cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        CU(cudaMemcpyAsync(d_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, s));
        pyr_upscale_kernel<<<blocks, 256, 0, s>>>((const int32_t *)c->ylab.p, (int32_t *)c->ymerge.p,
                                                  X, Y, Z, cx, cy, d_tab, d_tab + X, d_tab + X + Y);
        pyr_boundary_nil_kernel<<<blocks, 256, 0, s>>>((const int32_t *)c->ymerge.p,
                                                       (int32_t *)c->yup.p, X, Y, Z, d_off, adj.n);
        pyr_merge_kernel<<<blocks, 256, 0, s>>>(d_label_in, (const int32_t *)c->yup.p,
                                                (int32_t *)c->ymerge.p, N);
        CU(cudaGetLastError());
        // the tables must stay valid until the kernels above have read them
        CU(cudaStreamSynchronize(s));
    }
    // ---- fine pass: every labelled voxel is a seed ----
    int nfs = 0;
    TRY(seeds_from_labels(c, (const int32_t *)c->ymerge.p, N, c->yfseeds, c->yfslab, &nfs));
    oift_b200_outputs of{};
    of.label = d_label_out;
    TRY(run_pipeline<int32_t>(c, p, d_fscn, (const int32_t *)c->yfseeds.p,
                              (const int32_t *)c->yfslab.p, nfs, &of, st));
    if (percentile >= 0.0f) {
        int *d_mm = (int *)c->minmax.p;
        const int mm_init[2] = {0x7fffffff, (int)0x80000000};
        CU(cudaMemcpyAsync(d_mm, mm_init, sizeof(mm_init), cudaMemcpyHostToDevice, s));
        CU(launch_minmax<int32_t>(d_label_out, N, d_mm, c->sms, s));
        int hmm[2];
        CU(cudaMemcpyAsync(hmm, d_mm, sizeof(hmm), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (hmm[1] <= 1)
            TRY(conditional_dilation(c, d_fscn, d_label_out, X, Y, Z, 1.0f, percentile, nullptr));
    }
    cudaEventRecord(c->ev[9], s);
    CU(cudaStreamSynchronize(s));
    if (st) {
        // stage figures of the fine pass; the total covers both passes and the glue
        cudaEventElapsedTime(&st->ms_total, c->ev[8], c->ev[9]);
        st->levels += stc.levels;
        st->tile_steps += stc.tile_steps;
        st->kernels += stc.kernels + 9;
    }
    return OIFT_OK;
}

// Shift to >= 0 and blur: the device int32 volume the cascade and the CLI chain work on.
template <typename T>
static int shift_and_blur(oift_b200_ctx *c, const T *d_img, size_t N, int X, int Y, int Z,
                          int blur_passes, int32_t *d_out) {
    cudaStream_t s = c->stream;
    TRY(grow(c, c->minmax, 2 * sizeof(unsigned long long) + 2 * sizeof(int)));
    int *d_mm = (int *)c->minmax.p;
    const int mm_init[2] = {0x7fffffff, (int)0x80000000};
    CU(cudaMemcpyAsync(d_mm, mm_init, sizeof(mm_init), cudaMemcpyHostToDevice, s));
    CU(launch_minmax<T>(d_img, N, d_mm, c->sms, s));
    CU(launch_shift_to_i32<T>(d_img, d_out, N, d_mm, c->sms, s));
    if (blur_passes > 0) TRY(blur_passes_i32(c, d_out, d_out, X, Y, Z, blur_passes));
    return OIFT_OK;
}

}  // extern "C++"

extern "C" {

int oift_b200_gaussian_blur_i32(oift_b200_ctx *c, const int32_t *in, int32_t *out, int xsize,
                                int ysize, int zsize, int passes) {
    if (!c || !in || !out || xsize <= 0 || ysize <= 0 || zsize <= 0 || passes < 0)
        return OIFT_E_BAD_ARG;
    if (ysize > 65535 || zsize > 65535) return OIFT_E_RANGE;
    cudaSetDevice(c->device);
    const size_t N = (size_t)xsize * ysize * zsize;
    if (passes == 0) {
        if (in != out)
            CU(cudaMemcpyAsync(out, in, N * sizeof(int32_t), cudaMemcpyDeviceToDevice, c->stream));
    } else {
        TRY(blur_passes_i32(c, in, out, xsize, ysize, zsize, passes));
    }
    CU(cudaStreamSynchronize(c->stream));
    return OIFT_OK;
}

int oift_b200_conditional_dilation(oift_b200_ctx *c, const int32_t *image, int32_t *label,
                                   int xsize, int ysize, int zsize, float radius,
                                   float percentile, long long *added) {
    if (!c || !image || !label || xsize <= 0 || ysize <= 0 || zsize <= 0) return OIFT_E_BAD_ARG;
    if (!(radius >= 0.0f && radius < 6.0f) || !(std::fabs(percentile) < 1e9f)) return OIFT_E_BAD_ARG;
    cudaSetDevice(c->device);
    return conditional_dilation(c, image, label, xsize, ysize, zsize, radius, percentile, added);
}

int oift_b200_inject_boundary_seeds(int32_t *label, int xsize, int ysize, int zsize, int stride,
                                    int32_t *seeds_out, int cap) {
    // oiftrelax.cpp:175-224: voxels on the six faces, visited in z, y, x order with the
    // stride on every axis, that carry no label yet become background seeds.  With
    // seeds_out == NULL the count is returned and nothing is changed.
    if (!label || xsize <= 0 || ysize <= 0 || zsize <= 0 || stride <= 0) return OIFT_E_BAD_ARG;
    int n = 0;
    for (int z = 0; z < zsize; z += stride)
        for (int y = 0; y < ysize; y += stride)
            for (int x = 0; x < xsize; x += stride) {
                const bool face = x == 0 || x == xsize - 1 || y == 0 || y == ysize - 1 ||
                                  z == 0 || z == zsize - 1;
                if (!face) continue;
                const size_t p = (size_t)x + (size_t)y * xsize + (size_t)z * xsize * ysize;
                if (label[p] != -1) continue;
                if (seeds_out) {
                    if (n >= cap) return OIFT_E_RANGE;
                    label[p] = 0;
                    seeds_out[n] = (int32_t)p;
                }
                n++;
            }
    return n;
}

int oift_b200_read_seeds(const char *path, int xsize, int ysize, int zsize, int32_t *label,
                         int32_t *seeds_out, int cap) {
    // oiftrelax.cpp:322-352: a count, then "x y z id label" per seed; negative labels
    // become 0 (background); seeds outside the volume are dropped; the label map takes the
    // seed's label at its voxel.  With seeds_out == NULL only the in-volume count is
    // returned and the label map is left alone.  A file with fewer entries than its count
    // ends at the last complete entry.
    if (!path || xsize <= 0 || ysize <= 0 || zsize <= 0 || (seeds_out && !label)) return OIFT_E_BAD_ARG;
    FILE *fp = std::fopen(path, "r");
    if (!fp) return OIFT_E_BAD_ARG;
    int n = 0;
    if (std::fscanf(fp, " %d", &n) != 1 || n < 0) {
        std::fclose(fp);
        return OIFT_E_BAD_ARG;
    }
    int count = 0;
    for (int i = 0; i < n; i++) {
        int x, y, z, id, lb;
        if (std::fscanf(fp, " %d %d %d %d %d", &x, &y, &z, &id, &lb) != 5) break;
        if (lb < 0) lb = 0;
        if (x < 0 || y < 0 || z < 0 || x >= xsize || y >= ysize || z >= zsize) continue;
        if (lb > OIFT_MAX_LABEL) {
            std::fclose(fp);
            return OIFT_E_BAD_ARG;
        }
        if (seeds_out) {
            if (count >= cap) {
                std::fclose(fp);
                return OIFT_E_RANGE;
            }
            const size_t p = (size_t)x + (size_t)y * xsize + (size_t)z * xsize * ysize;
            seeds_out[count] = (int32_t)p;
            label[p] = lb;
        }
        count++;
    }
    std::fclose(fp);
    return count;
}

int oift_b200_read_polarity(const char *path, float *per_class, int cap) {
    // oiftrelax.cpp:280-300: a count n, then n polarities in [-1, 1]; each becomes x100 in
    // float.  Returns n; OIFT_E_BAD_ARG when the file is unreadable or short.
    if (!path) return OIFT_E_BAD_ARG;
    FILE *fp = std::fopen(path, "r");
    if (!fp) return OIFT_E_BAD_ARG;
    int n = 0;
    if (std::fscanf(fp, " %d", &n) != 1 || n <= 0) {
        std::fclose(fp);
        return OIFT_E_BAD_ARG;
    }
    if (per_class && n > cap) {
        std::fclose(fp);
        return OIFT_E_RANGE;
    }
    for (int i = 0; i < n; i++) {
        float v;
        if (std::fscanf(fp, " %f", &v) != 1) {
            std::fclose(fp);
            return OIFT_E_BAD_ARG;
        }
        if (per_class) per_class[i] = v * 100.0f;
    }
    std::fclose(fp);
    return n;
}

int oift_b200_run_cli_host(oift_b200_ctx *c, const oift_b200_params *p, const int32_t *image,
                           int32_t *label, const int32_t *seeds, int nseeds, int blur_passes,
                           float percentile, oift_b200_stats *stats) {
    TraceRange trace_("oift_b200_run_cli_host");
    if (!c || !image || !label || (nseeds > 0 && !seeds) || blur_passes < 0) return OIFT_E_BAD_ARG;
    TRY(check_params(p));
    // the cascade and the CLI chain run OIFT_Multi / ORelax_1_Multi, not the 2D image graph
    if (p->weight_mode == OIFT_W_IMAGEGRAPH) return OIFT_E_UNSUPPORTED;
    if (nseeds <= 0) return OIFT_E_NO_SEEDS;
    cudaSetDevice(c->device);
    const int X = p->xsize, Y = p->ysize, Z = p->zsize;
    if (Y > 65535 || Z > 65535) return OIFT_E_RANGE;
    const size_t N = (size_t)X * Y * Z;
    cudaStream_t s = c->stream;
    std::vector<int32_t> slab(nseeds);
    for (int i = 0; i < nseeds; i++) {
        if (seeds[i] < 0 || (size_t)seeds[i] >= N) return OIFT_E_SEED_RANGE;
        const int lb = label[seeds[i]];
        slab[i] = lb < 0 ? 0 : lb;
        if (slab[i] > OIFT_MAX_LABEL) return OIFT_E_BAD_ARG;
    }
    TRY(grow(c, c->img32, N * sizeof(int32_t)));
    TRY(grow(c, c->cimg0, N * sizeof(int32_t)));
    TRY(grow(c, c->seeds, (size_t)nseeds * sizeof(int32_t)));
    TRY(grow(c, c->slabels, (size_t)nseeds * sizeof(int32_t)));
    TRY(grow(c, c->dlabel, N * sizeof(int32_t)));
    TRY(grow(c, c->minmax, 2 * sizeof(unsigned long long) + 2 * sizeof(int)));
    CU(cudaMemcpyAsync(c->img32.p, image, N * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c->seeds.p, seeds, (size_t)nseeds * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c->slabels.p, slab.data(), (size_t)nseeds * sizeof(int32_t),
                       cudaMemcpyHostToDevice, s));
    // ---- shift to >= 0, blur ----
    int *d_mm = (int *)c->minmax.p;
    const int mm_init[2] = {0x7fffffff, (int)0x80000000};
    CU(cudaMemcpyAsync(d_mm, mm_init, sizeof(mm_init), cudaMemcpyHostToDevice, s));
    CU(launch_minmax<int32_t>((const int32_t *)c->img32.p, N, d_mm, c->sms, s));
    CU(launch_shift_to_i32<int32_t>((const int32_t *)c->img32.p, (int32_t *)c->cimg0.p, N, d_mm,
                                    c->sms, s));
    if (blur_passes > 0)
        TRY(blur_passes_i32(c, (const int32_t *)c->cimg0.p, (int32_t *)c->cimg0.p, X, Y, Z, blur_passes));
    // ---- OIFT + relaxation on the blurred image ----
    oift_b200_outputs o{};
    const bool relax = p->relax_sweeps > 0;
    if (relax)
        o.label = (int32_t *)c->dlabel.p;
    else
        o.oift_label = (int32_t *)c->dlabel.p;
    oift_b200_stats lst{};
    TRY(run_pipeline<int32_t>(c, p, (const int32_t *)c->cimg0.p, (const int32_t *)c->seeds.p,
                              (const int32_t *)c->slabels.p, nseeds, &o, stats ? stats : &lst));
    // ---- conditional dilation of a binary result ----
    if (percentile >= 0.0f) {
        CU(cudaMemcpyAsync(d_mm, mm_init, sizeof(mm_init), cudaMemcpyHostToDevice, s));
        CU(launch_minmax<int32_t>((const int32_t *)c->dlabel.p, N, d_mm, c->sms, s));
        int hmm[2];
        CU(cudaMemcpyAsync(hmm, d_mm, sizeof(hmm), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        if (hmm[1] <= 1)
            TRY(conditional_dilation(c, (const int32_t *)c->cimg0.p, (int32_t *)c->dlabel.p, X, Y,
                                     Z, 1.0f, percentile, nullptr));
    }
    CU(cudaMemcpyAsync(label, c->dlabel.p, N * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    return OIFT_OK;
}

int oift_b200_adjoint(oift_b200_ctx *c, const oift_b200_adjoint_params *ap, const int16_t *image,
                      const float *grad_map, const int32_t *labels0, const int32_t *seeds,
                      const int32_t *seed_labels, int nseeds, const uint8_t *truth,
                      float *membership_out, double *loss, double *grad) {
    if (!c || !ap || !image || !labels0 || !truth || !loss || (nseeds > 0 && (!seeds || !seed_labels)))
        return OIFT_E_BAD_ARG;
    const int X = ap->xsize, Y = ap->ysize, Z = ap->zsize;
    if (X <= 0 || Y <= 0 || Z <= 0 || ap->sweeps < 1 || ap->sweeps > 60000 || ap->checkpoint < 0)
        return OIFT_E_BAD_ARG;
    if (ap->adjacency == 4 || ap->adjacency == 8) {
        if (Z != 1) return OIFT_E_BAD_ARG;
    } else if (ap->adjacency != 6 && ap->adjacency != 26) {
        return OIFT_E_BAD_ARG;
    }
    if (ap->kernel != OIFT_ADJ_RBF && ap->kernel != OIFT_ADJ_POW8) return OIFT_E_BAD_ARG;
    if (ap->kernel == OIFT_ADJ_RBF && !(ap->sigma > 0.0f)) return OIFT_E_BAD_ARG;
    if (!(std::fabs(ap->alpha) <= 1.0f) || !(ap->beta >= 0.0f && ap->beta <= 1.0f) || !(ap->eps >= 0.0f))
        return OIFT_E_BAD_ARG;
    if (nseeds <= 0) return OIFT_E_NO_SEEDS;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    const size_t N = (size_t)X * Y * Z;
    const int K = ap->sweeps;
    int cp = ap->checkpoint;
    if (cp == 0) cp = (int)std::ceil(std::sqrt((double)K));
    if (cp > K) cp = K;
    // ---- classes: 0 and the seed labels (gft_ift.cpp:8684-8712) ----
    TRY(grow(c, c->presence, 1024 * sizeof(uint32_t)));
    CU(cudaMemsetAsync(c->presence.p, 0, 1024 * sizeof(uint32_t), s));
    seed_presence_kernel<<<std::min((nseeds + 255) / 256, c->sms * 4), 256, 0, s>>>(
        seed_labels, nseeds, (uint32_t *)c->presence.p);
    std::vector<uint32_t> bits(1024);
    CU(cudaMemcpyAsync(bits.data(), c->presence.p, 1024 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    TRY(grow(c, c->minmax, 2 * sizeof(unsigned long long) + 2 * sizeof(int)));
    int *d_mm = (int *)c->minmax.p;
    const int mm_init[2] = {0x7fffffff, (int)0x80000000};
    CU(cudaMemcpyAsync(d_mm, mm_init, sizeof(mm_init), cudaMemcpyHostToDevice, s));
    CU(launch_minmax<int16_t>(image, N, d_mm, c->sms, s));
    int hmm[2];
    CU(cudaMemcpyAsync(hmm, d_mm, sizeof(hmm), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    bits[0] |= 1u;
    std::vector<int> classes;
    for (int l = 0; l <= OIFT_MAX_LABEL; l++)
        if ((bits[l >> 5] >> (l & 31)) & 1u) classes.push_back(l);
    const int C = (int)classes.size();
    if (C > 8) return OIFT_E_UNSUPPORTED;
    const int maxl = classes.back();
    std::vector<int> l2c(maxl + 1, -1);
    for (int k = 0; k < C; k++) l2c[classes[k]] = k;
    const int bg = l2c[0];
    TRY(grow(c, c->al2c, (maxl + 1) * sizeof(int)));
    TRY(grow(c, c->aseedc, N));
    TRY(grow(c, c->adist, N * sizeof(uint16_t)));
    TRY(grow(c, c->asmall, 8 * sizeof(double)));
    const size_t wf = adjoint_work_floats(N, C, K, cp);
    TRY(grow(c, c->awork, wf * sizeof(float)));
    CU(cudaMemcpyAsync(c->al2c.p, l2c.data(), (maxl + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(c->aseedc.p, 0xFF, N, s));
    relax_seed_kernel<<<(nseeds + 255) / 256, 256, 0, s>>>(seeds, nseeds, labels0, N,
                                                           (const int *)c->al2c.p, maxl, bg,
                                                           (uint8_t *)c->aseedc.p);
    CU(cudaGetLastError());
    AdjointJob J{};
    J.X = X;
    J.Y = Y;
    J.Z = Z;
    J.adjacency = ap->adjacency;
    J.sweeps = K;
    J.checkpoint = cp;
    J.C = C;
    J.bg = bg;
    J.kernel = ap->kernel;
    J.sigma = ap->sigma;
    J.alpha = ap->alpha;
    J.beta = ap->beta;
    J.eps = ap->eps;
    J.imax = hmm[1];
    J.img = image;
    J.g = grad_map;
    J.dist = (uint16_t *)c->adist.p;
    J.seedc = (const uint8_t *)c->aseedc.p;
    J.labels0 = labels0;
    J.l2c = (const int *)c->al2c.p;
    J.maxl = maxl;
    J.truth = truth;
    J.membership_out = membership_out;
    return adjoint_run(J, s, c->sms, (float *)c->awork.p, wf, c->asmall.p, loss, grad);
}

int oift_b200_run_pyramid_host(oift_b200_ctx *c, const oift_b200_params *p, const int32_t *image,
                               int32_t *label, const int32_t *seeds, int nseeds, int blur_passes,
                               float percentile, oift_b200_stats *stats) {
    if (!c || !image || !label || (nseeds > 0 && !seeds) || blur_passes < 0) return OIFT_E_BAD_ARG;
    TRY(check_params(p));
    // the cascade and the CLI chain run OIFT_Multi / ORelax_1_Multi, not the 2D image graph
    if (p->weight_mode == OIFT_W_IMAGEGRAPH) return OIFT_E_UNSUPPORTED;
    if (nseeds <= 0) return OIFT_E_NO_SEEDS;
    cudaSetDevice(c->device);
    const int X = p->xsize, Y = p->ysize, Z = p->zsize;
    if (Y > 65535 || Z > 65535) return OIFT_E_RANGE;
    const size_t N = (size_t)X * Y * Z;
    cudaStream_t s = c->stream;
    for (int i = 0; i < nseeds; i++) {
        if (seeds[i] < 0 || (size_t)seeds[i] >= N) return OIFT_E_SEED_RANGE;
        if (label[seeds[i]] > OIFT_MAX_LABEL) return OIFT_E_BAD_ARG;
    }
    TRY(grow(c, c->img32, N * sizeof(int32_t)));
    TRY(grow(c, c->cimg0, N * sizeof(int32_t)));
    TRY(grow(c, c->seeds, (size_t)nseeds * sizeof(int32_t)));
    TRY(grow(c, c->dlabel, N * sizeof(int32_t)));
    TRY(grow(c, c->flabel, N * sizeof(int32_t)));
    CU(cudaMemcpyAsync(c->img32.p, image, N * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c->seeds.p, seeds, (size_t)nseeds * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(c->flabel.p, label, N * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    TRY(shift_and_blur<int32_t>(c, (const int32_t *)c->img32.p, N, X, Y, Z, blur_passes,
                                (int32_t *)c->cimg0.p));
    oift_b200_stats lst{};
    TRY(run_pyramid(c, p, (const int32_t *)c->cimg0.p, (const int32_t *)c->flabel.p,
                    (const int32_t *)c->seeds.p, nseeds, percentile, (int32_t *)c->dlabel.p,
                    stats ? stats : &lst));
    CU(cudaMemcpyAsync(label, c->dlabel.p, N * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    return OIFT_OK;
}

int oift_b200_run_pyramid_device_i16(oift_b200_ctx *c, const oift_b200_params *p,
                                     const int16_t *image, const int32_t *label_in,
                                     const int32_t *seeds, int nseeds, int blur_passes,
                                     float percentile, int32_t *label_out,
                                     oift_b200_stats *stats) {
    if (!c || !image || !label_in || !label_out || (nseeds > 0 && !seeds) || blur_passes < 0)
        return OIFT_E_BAD_ARG;
    TRY(check_params(p));
    // the cascade and the CLI chain run OIFT_Multi / ORelax_1_Multi, not the 2D image graph
    if (p->weight_mode == OIFT_W_IMAGEGRAPH) return OIFT_E_UNSUPPORTED;
    if (nseeds <= 0) return OIFT_E_NO_SEEDS;
    cudaSetDevice(c->device);
    const int X = p->xsize, Y = p->ysize, Z = p->zsize;
    if (Y > 65535 || Z > 65535) return OIFT_E_RANGE;
    const size_t N = (size_t)X * Y * Z;
    TRY(grow(c, c->cimg0, N * sizeof(int32_t)));
    TRY(shift_and_blur<int16_t>(c, image, N, X, Y, Z, blur_passes, (int32_t *)c->cimg0.p));
    oift_b200_stats lst{};
    return run_pyramid(c, p, (const int32_t *)c->cimg0.p, label_in, seeds, nseeds, percentile,
                       label_out, stats ? stats : &lst);
}


}  // extern "C"

// ----------------------------------------------------------------- batched driver ----
// The OIFT of one volume is bound by the latency of its level loop (grid reduction, team
// barrier, a few tile steps per level), not by the SM count: halving its CTAs slows one job
// by only a few percent.  So the driver runs the OIFT of all jobs of a call in ONE
// cooperative launch of `teams` teams of sms/teams CTAs (oift_team_run), each team pulling
// jobs from a device counter, largest volume first.  Edge codes and intensity ranges are
// computed once per distinct image before that launch; the relaxation of the jobs follows
// on RELAX_LANES sub-context streams, one host thread each (its host reads of the class set
// and the sweep histogram would otherwise serialise the jobs).
static constexpr int RELAX_LANES = 4;

static int ensure_lanes(oift_b200_ctx *c, int lanes) {
    while ((int)c->lanes.size() < lanes) {
        oift_b200_ctx *l = nullptr;
        int rc = oift_b200_create(&l, c->device);
        if (rc != OIFT_OK) return rc;
        c->lanes.push_back(l);
    }
    return OIFT_OK;
}

static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct BatchTimes {
    double wall_ms = 0, oift_ms = 0, relax_ms = 0;
};

struct BatchImg {
    const int16_t *p;
    int X, Y, Z;
    size_t woff;  // element offset of its edge codes in c->W
};

// Everything of a batched call that needs the host: per-job checks, distinct images and
// their intensity ranges, the RBF table, the weight builds to launch, job descriptors
// (uploaded), per-team scratch.  Jobs that fail a check get their status here.
struct BatchPrep {
    std::vector<BatchImg> imgs;
    std::vector<int> job_img;  // per job (from `first`): its image, -1 if the job failed a check
    std::vector<int> hmm;      // intensity min / max per image
    std::vector<BuildArgs> builds;
    std::vector<int> order;    // launch slot -> job index
    std::vector<int32_t *> olab;
    std::vector<OiftTeamJob> dj;
    int nj = 0, n3d = 0, nimg = 0;
    OiftTeamScratch S;
    OiftTeamJob *d_jobs = nullptr;
    unsigned long long *d_clamp = nullptr;
    int tile_ty = 8;  // 3D warp tile of the team kernel (oift_plan)
};

// Most teams the batch can be split into: every team must hold enough CTAs to own the tiles
// of the largest job (a CTA's tile sets live in shared memory).
static int batch_max_teams(const oift_b200_ctx *c, const oift_b200_job *jobs, int first,
                           int count, int tile_ty) {
    int need = 1;
    for (int j = first; j < first + count; j++) {
        const oift_b200_job &jb = jobs[j];
        if (jb.xsize <= 0 || jb.ysize <= 0 || jb.zsize <= 0) continue;
        const OiftPlan P = oift_plan(jb.xsize, jb.ysize, jb.zsize, tile_ty);
        need = std::max(need, oift_min_ctas(P));
    }
    return std::max(1, c->sms / need);
}

static int batch_prepare(oift_b200_ctx *c, const oift_b200_params *common, oift_b200_job *jobs,
                         int first, int count, int teams, int tile_ty, BatchPrep *bp) {
    cudaStream_t s = c->stream;
    bp->tile_ty = tile_ty == 4 ? 4 : 8;
    const int end = first + count;
    if (teams < 1 || teams > c->sms) return OIFT_E_BAD_ARG;
    // the team kernel is the 6 / 4-neighbourhood tile step on prebuilt edge codes
    if (common->adjacency != 6 && common->adjacency != 4) return OIFT_E_UNSUPPORTED;
    if (common->weight_mode == OIFT_W_BLEND_Q || common->weight_mode == OIFT_W_IMAGEGRAPH)
        return OIFT_E_UNSUPPORTED;
    const int ctas_lo = c->sms / teams, ctas_hi = (c->sms + teams - 1) / teams;

    // ---- per-job checks; distinct images (pointer + extents) ----
    std::vector<BatchImg> &imgs = bp->imgs;
    std::vector<int> &job_img = bp->job_img;
    job_img.assign(count, -1);
    size_t wtotal = 0;
    for (int j = first; j < end; j++) {
        oift_b200_job &jb = jobs[j];
        oift_b200_params p = *common;
        p.xsize = jb.xsize;
        p.ysize = jb.ysize;
        p.zsize = jb.zsize;
        p.per = jb.per;
        p.per_class = nullptr;
        p.max_label = 0;
        int st = check_params(&p);
        if (st == OIFT_OK && (!jb.image || !jb.seeds || !jb.seed_labels)) st = OIFT_E_BAD_ARG;
        if (st == OIFT_OK && jb.nseeds <= 0) st = OIFT_E_NO_SEEDS;
        jb.status = st;
        if (st != OIFT_OK) continue;
        int k = -1;
        for (size_t i = 0; i < imgs.size(); i++)
            if (imgs[i].p == jb.image && imgs[i].X == jb.xsize && imgs[i].Y == jb.ysize &&
                imgs[i].Z == jb.zsize) {
                k = (int)i;
                break;
            }
        if (k < 0) {
            k = (int)imgs.size();
            imgs.push_back({jb.image, jb.xsize, jb.ysize, jb.zsize, wtotal});
            const size_t n = (size_t)jb.xsize * jb.ysize * jb.zsize;
            wtotal += align_up(3 * n, 128);  // 256-byte aligned planes blocks
        }
        job_img[j - first] = k;
    }
    const int nimg = (int)imgs.size();
    bp->nimg = nimg;
    if (nimg == 0) return OIFT_OK;

    // ---- intensity range and edge codes, once per image ----
    TRY(grow(c, c->W, wtotal * sizeof(uint16_t)));
    TRY(grow(c, c->bmm, (size_t)nimg * (2 * sizeof(int) + sizeof(unsigned long long))));
    int *d_mm = (int *)c->bmm.p;
    unsigned long long *d_clamp = (unsigned long long *)((char *)c->bmm.p + (size_t)nimg * 2 * sizeof(int));
    {
        std::vector<int> mm_init(2 * (size_t)nimg);
        for (int i = 0; i < nimg; i++) {
            mm_init[2 * i] = 0x7fffffff;
            mm_init[2 * i + 1] = (int)0x80000000;
        }
        CU(cudaMemcpyAsync(d_mm, mm_init.data(), mm_init.size() * sizeof(int),
                           cudaMemcpyHostToDevice, s));
        CU(cudaMemsetAsync(d_clamp, 0, (size_t)nimg * sizeof(unsigned long long), s));
    }
    for (int i = 0; i < nimg; i++) {
        const size_t n = (size_t)imgs[i].X * imgs[i].Y * imgs[i].Z;
        CU(launch_minmax<int16_t>(imgs[i].p, n, d_mm + 2 * i, c->sms, s));
    }
    std::vector<int> &hmm = bp->hmm;
    hmm.assign(2 * (size_t)nimg, 0);
    CU(cudaMemcpyAsync(hmm.data(), d_mm, hmm.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const uint16_t *lut = nullptr;
    int lut_len = 0;
    if (common->weight_mode == OIFT_W_RBF_Q) {
        // the table depends on |I_p - I_q| only: one table for the widest range serves all
        long long range = 0;
        for (int i = 0; i < nimg; i++)
            range = std::max(range, (long long)hmm[2 * i + 1] - (long long)hmm[2 * i]);
        lut_len = (int)(range + 1);
        std::vector<uint16_t> t(lut_len);
        const double sg = common->rbf_sigma;
        for (int d = 0; d < lut_len; d++) {
            double a = std::exp(-((double)d * (double)d) / (2.0 * sg * sg));
            double v = std::floor((double)common->wq * (1.0 - a) + 0.5);
            t[d] = (uint16_t)(v < 0 ? 0 : (v > common->wq ? common->wq : v));
        }
        TRY(grow(c, c->lut, lut_len * sizeof(uint16_t)));
        c->lut_len = 0;  // the cached pipeline table is overwritten
        CU(cudaMemcpyAsync(c->lut.p, t.data(), lut_len * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
        lut = (const uint16_t *)c->lut.p;
    }
    const Adjacency adj = make_adjacency(6);
    for (int i = 0; i < nimg; i++) {
        BuildArgs ba;
        ba.X = imgs[i].X;
        ba.Y = imgs[i].Y;
        ba.Z = imgs[i].Z;
        ba.planes = 3;
        ba.mode = common->weight_mode;
        ba.cap = (common->weight_mode == OIFT_W_GRAD) ? OIFT_MAX_BASE : common->wq;
        for (int k = 0; k < 3; k++) {
            ba.dx[k] = adj.dx[adj.n / 2 + k];
            ba.dy[k] = adj.dy[adj.n / 2 + k];
            ba.dz[k] = adj.dz[adj.n / 2 + k];
        }
        ba.lut = lut;
        ba.lut_len = lut_len;
        ba.grad = nullptr;
        ba.blend_a = common->blend_a;
        ba.clamped = d_clamp + i;
        bp->builds.push_back(ba);
    }
    bp->d_clamp = d_clamp;

    // ---- job descriptors: 3D jobs then 2D jobs, each group largest volume first ----
    std::vector<int> &order = bp->order;
    order.clear();
    for (int j = first; j < end; j++)
        if (jobs[j].status == OIFT_OK) order.push_back(j);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const bool pa = jobs[a].zsize == 1, pb = jobs[b].zsize == 1;
        if (pa != pb) return pb;  // 3D first
        return (size_t)jobs[a].xsize * jobs[a].ysize * jobs[a].zsize >
               (size_t)jobs[b].xsize * jobs[b].ysize * jobs[b].zsize;
    });
    const int nj = (int)order.size();
    bp->nj = nj;
    std::vector<OiftTeamJob> &dj = bp->dj;
    dj.assign(nj, OiftTeamJob{});
    size_t max_n = 0, max_tiles = 0, max_mbox = 0, olab_total = 0;
    std::vector<size_t> olab_off(nj, (size_t)-1);
    for (int i = 0; i < nj; i++) {
        // a job with a label output relaxes in place; one with only a mask needs room for
        // its OIFT labels
        const oift_b200_job &jb = jobs[order[i]];
        const size_t n = (size_t)jb.xsize * jb.ysize * jb.zsize;
        if (!jb.label && jb.mask) {
            olab_off[i] = olab_total;
            olab_total += align_up(n, 64);
        }
    }
    if (olab_total) TRY(grow(c, c->bolab, olab_total * sizeof(int32_t)));
    std::vector<int32_t *> &olab = bp->olab;
    olab.assign(nj, nullptr);
    int n3d = 0;
    for (int i = 0; i < nj; i++) {
        const oift_b200_job &jb = jobs[order[i]];
        const OiftPlan P = oift_plan(jb.xsize, jb.ysize, jb.zsize, bp->tile_ty);
        const size_t n = (size_t)jb.xsize * jb.ysize * jb.zsize;
        OiftTeamJob &d = dj[i];
        d.W = (const uint16_t *)c->W.p + imgs[job_img[order[i] - first]].woff;
        d.seeds = jb.seeds;
        d.seed_labels = jb.seed_labels;
        d.cost = jb.cost;
        olab[i] = jb.label ? jb.label
                           : (olab_off[i] != (size_t)-1 ? (int32_t *)c->bolab.p + olab_off[i] : nullptr);
        d.label = olab[i];
        d.X = jb.xsize;
        d.Y = jb.ysize;
        d.Z = jb.zsize;
        d.nseeds = jb.nseeds;
        d.ntx = P.ntx;
        d.nty = P.nty;
        d.ntz = P.ntz;
        d.ntiles = P.ntiles;
        d.pol0 = -jb.per;  // label 0 takes -per (gft_ift.cpp:968)
        d.pol_default = jb.per;
        d.status = OIFT_TEAM_NOT_RUN;
        d.levels = 0;
        d.steps = 0;
        max_n = std::max(max_n, n);
        max_tiles = std::max(max_tiles, (size_t)P.ntiles);
        max_mbox = std::max(max_mbox, std::max(oift_mbox_bytes(P, ctas_lo), oift_mbox_bytes(P, ctas_hi)) /
                                          sizeof(unsigned long long));
        if (jb.zsize > 1) n3d++;
    }
    bp->n3d = n3d;
    OiftTeamScratch &S = bp->S;
    S.key_stride = align_up(max_n, 64);
    S.tpend_stride = align_up(max_tiles, 64);
    S.mbox_stride = align_up(max_mbox, 32);
    TRY(grow(c, c->bjobs, (size_t)nj * sizeof(OiftTeamJob)));
    TRY(grow(c, c->bkey, (size_t)teams * S.key_stride * sizeof(uint32_t)));
    TRY(grow(c, c->btpend, (size_t)teams * S.tpend_stride * sizeof(uint32_t)));
    TRY(grow(c, c->bmbox, (size_t)teams * S.mbox_stride * sizeof(unsigned long long)));
    TRY(grow(c, c->bglob, (size_t)teams * sizeof(OiftGlobals)));
    TRY(grow(c, c->bctl, 2 * sizeof(unsigned int)));
    S.key = (uint32_t *)c->bkey.p;
    S.tpend = (uint32_t *)c->btpend.p;
    S.mbox = (unsigned long long *)c->bmbox.p;
    S.g = (OiftGlobals *)c->bglob.p;
    S.next_job = (unsigned int *)c->bctl.p;
    S.abort = (int *)c->bctl.p + 1;
    S.spin_limit = c->spin_limit;
    S.max_levels = c->max_levels;
    OiftTeamJob *d_jobs = (OiftTeamJob *)c->bjobs.p;
    bp->d_jobs = d_jobs;
    CU(cudaMemcpyAsync(d_jobs, dj.data(), (size_t)nj * sizeof(OiftTeamJob), cudaMemcpyHostToDevice, s));
    return OIFT_OK;
}

// The device work of the batched OIFT: weight builds, optionally the descriptors restored
// from a pristine copy, one team launch per group.  Launches and device-side copies only,
// so a stream capture can record it.
static int batch_enqueue_oift(oift_b200_ctx *c, const BatchPrep &bp, int teams,
                              const OiftTeamJob *d_pristine) {
    cudaStream_t s = c->stream;
    CU(cudaMemsetAsync(bp.d_clamp, 0, (size_t)bp.nimg * sizeof(unsigned long long), s));
    for (int i = 0; i < bp.nimg; i++)
        CU(launch_build_weights<int16_t>(bp.imgs[i].p, (uint16_t *)c->W.p + bp.imgs[i].woff,
                                         bp.builds[i], c->sms, s));
    if (d_pristine)
        CU(cudaMemcpyAsync(bp.d_jobs, d_pristine, (size_t)bp.nj * sizeof(OiftTeamJob),
                           cudaMemcpyDeviceToDevice, s));
    if (bp.n3d > 0) TRY(oift_team_run(bp.d_jobs, bp.n3d, false, teams, c->sms, bp.S, s, bp.tile_ty));
    if (bp.nj - bp.n3d > 0)
        TRY(oift_team_run(bp.d_jobs + bp.n3d, bp.nj - bp.n3d, true, teams, c->sms, bp.S, s));
    return OIFT_OK;
}

static int run_batch_teams(oift_b200_ctx *c, const oift_b200_params *common,
                           oift_b200_job *jobs, int first, int count, int teams, int tile_ty,
                           BatchTimes *bt) {
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    cudaStream_t s = c->stream;
    const int end = first + count;

    BatchPrep bp;
    teams = std::min(teams, batch_max_teams(c, jobs, first, count, tile_ty));
    TRY(batch_prepare(c, common, jobs, first, count, teams, tile_ty, &bp));
    const int nimg = bp.nimg, nj = bp.nj;
    if (nimg == 0) {
        for (int j = first; j < end; j++)
            if (jobs[j].status != OIFT_OK) return jobs[j].status;
        return OIFT_OK;
    }
    const std::vector<int> &order = bp.order, &job_img = bp.job_img, &hmm = bp.hmm;
    const std::vector<int32_t *> &olab = bp.olab;
    std::vector<OiftTeamJob> &dj = bp.dj;
    OiftTeamJob *d_jobs = bp.d_jobs;
    unsigned long long *d_clamp = bp.d_clamp;
    cudaEventRecord(c->ev[0], s);
    // ---- the OIFT of every job: weight builds, one team launch per group ----
    TRY(batch_enqueue_oift(c, bp, teams, nullptr));
    cudaEventRecord(c->ev[1], s);
    std::vector<unsigned long long> hclamp(nimg);
    CU(cudaMemcpyAsync(dj.data(), d_jobs, (size_t)nj * sizeof(OiftTeamJob), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(hclamp.data(), d_clamp, nimg * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    float oift_ms = 0;
    cudaEventElapsedTime(&oift_ms, c->ev[0], c->ev[1]);
    for (int i = 0; i < nj; i++) {
        oift_b200_job &jb = jobs[order[i]];
        int st = dj[i].status;
        if (st == OIFT_TEAM_NOT_RUN) st = OIFT_E_NOT_CONVERGED;
        if (st == OIFT_OK && common->weight_mode == OIFT_W_GRAD && hclamp[job_img[order[i] - first]])
            st = OIFT_E_RANGE;
        jb.status = st;
    }
    const auto t1 = clk::now();

    // ---- relaxation of the jobs that want labels or a mask ----
    std::vector<int> rjobs;
    for (int i = 0; i < nj; i++) {
        const oift_b200_job &jb = jobs[order[i]];
        if (jb.status == OIFT_OK && (jb.label || jb.mask)) rjobs.push_back(i);
    }
    const int nl = std::min<int>(RELAX_LANES, (int)rjobs.size());
    if (nl > 0) {
        TRY(ensure_lanes(c, nl));
        std::atomic<int> next(0);
        auto worker = [&](int lane) {
            cudaSetDevice(c->device);
            oift_b200_ctx *l = c->lanes[lane];
            for (;;) {
                const int r = next.fetch_add(1);
                if (r >= (int)rjobs.size()) break;
                const int i = rjobs[r];
                oift_b200_job &jb = jobs[order[i]];
                oift_b200_params p = *common;
                p.xsize = jb.xsize;
                p.ysize = jb.ysize;
                p.zsize = jb.zsize;
                p.per = jb.per;
                p.per_class = nullptr;
                p.max_label = 0;
                oift_b200_outputs o{};
                o.label = jb.label;
                o.mask = jb.mask;
                RelaxResult rr;
                const int k = job_img[order[i] - first];
                int st = relax_stage<int16_t>(l, &p, jb.image, jb.seeds, jb.seed_labels,
                                              jb.nseeds, olab[i], &hmm[2 * k], &o, &rr);
                if (st == OIFT_OK && cudaStreamSynchronize(l->stream) != cudaSuccess) st = OIFT_E_CUDA;
                jb.status = st;
            }
        };
        std::vector<std::thread> ths;
        for (int i = 0; i < nl; i++) ths.emplace_back(worker, i);
        for (auto &t : ths) t.join();
    }
    const auto t2 = clk::now();
    if (bt) {
        bt->oift_ms = oift_ms;
        bt->relax_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
        bt->wall_ms = std::chrono::duration<double, std::milli>(t2 - t0).count();
    }
    for (int j = first; j < end; j++)
        if (jobs[j].status != OIFT_OK) return jobs[j].status;
    return OIFT_OK;
}

// ------------------------------------------------------------ batch as a CUDA graph ----
// A batch recorded once and replayed: the weight builds, the descriptor reset, the team
// launches and every job's relaxation sweeps are captured from a private context (its
// scratch cannot be reallocated by other calls), so a replay is one graph launch.  What the
// host had to read to plan the batch -- job checks, intensity ranges (relaxation Wmax, RBF
// table), each job's class set -- is fixed at recording: a replay is valid while the jobs'
// buffers stay where they are, the images keep their intensity range and the seeds their
// label set.
struct oift_b200_batch_graph {
    oift_b200_ctx *c = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    BatchPrep bp;
    int njobs = 0, weight_mode = 0, teams = 0;
    void *pristine = nullptr;  // descriptors as uploaded
    void *plans = nullptr;     // packed label -> class maps and class lists of the jobs
};

static void batch_graph_free(oift_b200_batch_graph *g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->pristine) cudaFree(g->pristine);
    if (g->plans) cudaFree(g->plans);
    if (g->c) oift_b200_destroy(g->c);
    delete g;
}

int oift_b200_batch_graph_create(oift_b200_ctx *ctx, const oift_b200_params *common,
                                 oift_b200_job *jobs, int njobs, int teams,
                                 oift_b200_batch_graph **out) {
    if (!ctx || !common || !jobs || !out || njobs <= 0 || teams < 0 || teams > ctx->sms)
        return OIFT_E_BAD_ARG;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    int tile_ty = ctx->batch_tile_ty;
    if (teams == 0) {
        // the context's autotuned choice when it has one, else half the SMs
        double best = -1.0;
        teams = ctx->sms / 2;
        for (auto &tc : ctx->tune_cands)
            if (tc.rate > best) {
                best = tc.rate;
                teams = tc.teams;
                tile_ty = tc.tile_ty;
            }
    }
    teams = std::max(1, std::min(std::min(teams, njobs), batch_max_teams(ctx, jobs, 0, njobs, tile_ty)));
    oift_b200_batch_graph *g = new oift_b200_batch_graph();
    g->njobs = njobs;
    g->weight_mode = common->weight_mode;
    g->teams = teams;
    int rc = oift_b200_create(&g->c, ctx->device);
    if (rc != OIFT_OK) {
        batch_graph_free(g);
        return rc;
    }
    oift_b200_ctx *c = g->c;
    cudaStream_t s = c->stream;
    BatchPrep &bp = g->bp;
    rc = batch_prepare(c, common, jobs, 0, njobs, teams, tile_ty, &bp);
    for (int j = 0; rc == OIFT_OK && j < njobs; j++)
        if (jobs[j].status != OIFT_OK) rc = jobs[j].status;
    if (rc == OIFT_OK && bp.nj == 0) rc = OIFT_E_BAD_ARG;
    const size_t dbytes = (size_t)bp.nj * sizeof(OiftTeamJob);
    if (rc == OIFT_OK && (cudaMalloc(&g->pristine, dbytes) != cudaSuccess ||
                          cudaMemcpyAsync(g->pristine, bp.d_jobs, dbytes, cudaMemcpyDeviceToDevice,
                                          s) != cudaSuccess)) {
        cudaGetLastError();
        rc = OIFT_E_CUDA;
    }
    // ---- relaxation plans (host reads) and the largest scratch any job needs ----
    std::vector<RelaxPlan> plans(bp.nj);
    std::vector<oift_b200_params> prm(bp.nj);
    std::vector<size_t> off(bp.nj, 0);
    std::vector<int> packed;
    for (int i = 0; rc == OIFT_OK && i < bp.nj; i++) {
        const oift_b200_job &jb = jobs[bp.order[i]];
        if (!jb.label && !jb.mask) continue;
        oift_b200_params &p = prm[i];
        p = *common;
        p.xsize = jb.xsize;
        p.ysize = jb.ysize;
        p.zsize = jb.zsize;
        p.per = jb.per;
        p.per_class = nullptr;
        p.max_label = 0;
        rc = relax_plan(c, &p, jb.seed_labels, jb.nseeds, &bp.hmm[2 * bp.job_img[bp.order[i]]],
                        &plans[i]);
        if (rc != OIFT_OK) break;
        rc = relax_reserve(c, (size_t)jb.xsize * jb.ysize * jb.zsize, plans[i].nclasses,
                           plans[i].maxl, jb.xsize, jb.ysize, jb.zsize, p.relax_sweeps);
        off[i] = packed.size();
        packed.insert(packed.end(), plans[i].l2c.begin(), plans[i].l2c.end());
        packed.insert(packed.end(), plans[i].classes.begin(), plans[i].classes.end());
    }
    if (rc == OIFT_OK && !packed.empty() &&
        (cudaMalloc(&g->plans, packed.size() * sizeof(int)) != cudaSuccess ||
         cudaMemcpyAsync(g->plans, packed.data(), packed.size() * sizeof(int),
                         cudaMemcpyHostToDevice, s) != cudaSuccess)) {
        cudaGetLastError();
        rc = OIFT_E_CUDA;
    }
    if (rc == OIFT_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = OIFT_E_CUDA;
    if (rc != OIFT_OK) {
        batch_graph_free(g);
        return rc;
    }
    // ---- record ----
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        cudaGetLastError();
        batch_graph_free(g);
        return OIFT_E_CUDA;
    }
    rc = batch_enqueue_oift(c, bp, teams, (const OiftTeamJob *)g->pristine);
    for (int i = 0; rc == OIFT_OK && i < bp.nj; i++) {
        const oift_b200_job &jb = jobs[bp.order[i]];
        if (!jb.label && !jb.mask) continue;
        oift_b200_outputs o{};
        o.label = jb.label;
        o.mask = jb.mask;
        const int *d_l2c = (const int *)g->plans + off[i];
        rc = relax_launch<int16_t>(c, &prm[i], jb.image, jb.seeds, jb.nseeds, bp.olab[i], plans[i],
                                   d_l2c, d_l2c + plans[i].l2c.size(), &o, false, false);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &graph);
    g->graph = graph;
    if (rc == OIFT_OK && (ce != cudaSuccess || !graph)) rc = OIFT_E_CUDA;
    if (rc == OIFT_OK && cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess) rc = OIFT_E_CUDA;
    if (rc != OIFT_OK) {
        cudaGetLastError();
        batch_graph_free(g);
        return rc;
    }
    *out = g;
    return OIFT_OK;
}

int oift_b200_batch_graph_launch(oift_b200_batch_graph *g, oift_b200_job *jobs, float *ms) {
    if (!g || !g->exec) return OIFT_E_BAD_ARG;
    oift_b200_ctx *c = g->c;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    BatchPrep &bp = g->bp;
    std::vector<unsigned long long> hclamp(bp.nimg);
    cudaEventRecord(c->ev[8], s);
    CU(cudaGraphLaunch(g->exec, s));
    cudaEventRecord(c->ev[9], s);
    CU(cudaMemcpyAsync(bp.dj.data(), bp.d_jobs, (size_t)bp.nj * sizeof(OiftTeamJob),
                       cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(hclamp.data(), bp.d_clamp, bp.nimg * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (ms) cudaEventElapsedTime(ms, c->ev[8], c->ev[9]);
    int rc = OIFT_OK;
    for (int i = 0; i < bp.nj; i++) {
        int st = bp.dj[i].status;
        if (st == OIFT_TEAM_NOT_RUN) st = OIFT_E_NOT_CONVERGED;
        if (st == OIFT_OK && g->weight_mode == OIFT_W_GRAD && hclamp[bp.job_img[bp.order[i]]])
            st = OIFT_E_RANGE;
        if (jobs) jobs[bp.order[i]].status = st;
        if (st != OIFT_OK && rc == OIFT_OK) rc = st;
    }
    return rc;
}

int oift_b200_batch_graph_destroy(oift_b200_batch_graph *g) {
    if (!g) return OIFT_E_BAD_ARG;
    cudaSetDevice(g->c ? g->c->device : 0);
    batch_graph_free(g);
    return OIFT_OK;
}

int oift_b200_run_batch(oift_b200_ctx *c, const oift_b200_params *common, oift_b200_job *jobs,
                        int njobs, int teams, oift_b200_batch_stats *stats) {
    TraceRange trace_("oift_b200_run_batch");
    if (!c || !common || !jobs || njobs < 0 || teams < 0 || teams > c->sms) return OIFT_E_BAD_ARG;
    if (njobs == 0) return OIFT_OK;
    cudaSetDevice(c->device);
    // teams = 0: the context's autotuner.  While exploring, each call runs with the next
    // untried candidate and records its rate (voxels per wall millisecond of the call);
    // once every candidate has a rate, calls use the fastest.
    int cand = -1;
    int tile_ty = c->batch_tile_ty;
    if (teams == 0) {
        // candidates: team counts x the two 3D warp tiles of 32 rows that keep the OIFT's
        // chains short (32 x 8 x 4 and 32 x 4 x 8; flatter tiles need more tile crossings)
        if (c->tune_cands.empty()) {
            const int G = c->sms;
            for (int ty : {8, 4})
                for (int t : {G / 2, G / 4, G, G / 8})
                    if (t >= 1) c->tune_cands.push_back({t, ty, -1.0});
        }
        for (size_t i = 0; i < c->tune_cands.size(); i++)
            if (c->tune_cands[i].rate < 0) {
                cand = (int)i;
                break;
            }
        if (cand >= 0) {
            teams = c->tune_cands[cand].teams;
            tile_ty = c->tune_cands[cand].tile_ty;
        } else {
            double best = -1.0;
            for (auto &tc : c->tune_cands)
                if (tc.rate > best) {
                    best = tc.rate;
                    teams = tc.teams;
                    tile_ty = tc.tile_ty;
                }
        }
    }
    const int used = std::min(teams, njobs);  // more teams than jobs would idle
    BatchTimes bt;
    const int rc = run_batch_teams(c, common, jobs, 0, njobs, used, tile_ty, &bt);
    if (cand >= 0 && rc == OIFT_OK) {
        double vox = 0;
        for (int j = 0; j < njobs; j++) vox += (double)jobs[j].xsize * jobs[j].ysize * jobs[j].zsize;
        c->tune_cands[cand].rate = vox / std::max(bt.wall_ms, 1e-3);
    }
    if (stats) {
        stats->tile_ty = tile_ty;
        stats->teams = used;
        stats->jobs = njobs;
        stats->tuning = cand >= 0 ? 1 : 0;
        stats->ms_wall = (float)bt.wall_ms;
        stats->ms_oift = (float)bt.oift_ms;
        stats->ms_relax = (float)bt.relax_ms;
    }
    return rc;
}

}  // extern "C"
