// kernels.cuh -- host-visible launch interfaces of the kernel translation units.
#pragma once
#include <cuda.h>

#include "common.cuh"

namespace oiftb {

struct BuildArgs {
    int X, Y, Z;
    int planes;
    int mode, cap;
    int dx[13], dy[13], dz[13];
    const uint16_t *lut;
    int lut_len;
    const int32_t *grad;
    float blend_a;
    unsigned long long *clamped;
    // optional tile-major copy of the 3 code planes of the 6 / 4 OIFT tiles (32 x tty x ttz):
    // tile t holds [plane][row][32] as the tile step stages it; null = not written
    uint16_t *Wt = nullptr;
    int tty = 0, ttz = 0, tntx = 0, tnty = 0;
    bool planes_out = true;  // false: only the tile-major copy (every OIFT tile is full)
    // set by the TMA-staged builder when a tile's image box did not land (null: that builder
    // is not used)
    int *tma_err = nullptr;
};

struct RelaxArgs {
    int X, Y, Z;
    size_t N;
    int nadj;
    int dx[26], dy[26], dz[26];
    float dpq[26];
    float Wmax;
    float per;
    int bg;
    float pcm[8];
    // gradient blend (ORelax_1_Multi_GradWeight): normalised Sobel map and mix weight
    int blend;
    float alpha;
    const int32_t *gmap;
};

// Hot scheduling counters of the persistent OIFT kernel, one 128-byte line each so
// that polling one does not serialise atomics on another.
struct OiftGlobals {
    unsigned int first;          // smallest pending key before the first level
    unsigned int runmin[3];      // level e: smallest key left pending above it (slot e % 3)
    unsigned long long first64;      // the same two for the 64-bit keys of a wide-range run
    unsigned long long runmin64[3];
    unsigned int pad0[20];
    int outstanding[3];          // level e: tiles wanted, running or announced (slot e % 3)
    unsigned int pad1[29];
    unsigned int bar_count;
    unsigned int pad2[31];
    unsigned int bar_gen;
    unsigned int pad3[31];
    int error;
    int levels;
    unsigned long long tile_steps;
    unsigned long long pushes;
    unsigned long long cycles[24];  // summed warp cycles: level sync, owner phase, queued
                                    // tiles, drain; key staging, sparse tiles, dense tiles,
                                    // #stale, #sparse, #dense; dense: masks, flood, flood
                                    // iterations, expansion, faces, pending; sparse:
                                    // worklist, flood rounds, face pushes, publication,
                                    // pending, #rounds, #voxels, #publications
    int job;       // job of the batched kernel this team works on
    int bad_seed;  // OIFT_E_* of an invalid seed of the team's current job, else 0
    unsigned int pad4[8];
};


// Default bounds of the persistent OIFT kernels' waits: about 1-2 s of polling at ~64 ns
// per poll, and far more levels than any input has (at most 32767 costs x 32768 labels
// would be reachable only by a runaway loop).
constexpr long long OIFT_DEFAULT_SPIN_LIMIT = 20000000LL;
// Tiles one CTA of the persistent OIFT kernels can own: its wanted / running sets live in
// shared memory as 64-bit words (16384 tiles = 16.7 M voxels of 32 x 8 x 4 tiles per CTA).
constexpr int OIFT_CTA_TILE_WORDS = 256;
constexpr int OIFT_DEFAULT_MAX_LEVELS = 4000000;

struct OiftPlan {
    int TY, TZ, ntx, nty, ntz, ntiles;
    unsigned int qcap;
};

// Scratch layout for one OIFT run (device pointers supplied by the caller).
struct OiftScratch {
    uint32_t *key;                // [N] (a wide-range run: [N] 64-bit keys at this address)
    uint32_t *tpend;              // [ntiles] (a wide-range run: 64-bit)
    unsigned long long *mbox;     // [3][ctas][words] re-activation bitmasks, per level slot
    OiftGlobals *g;
    unsigned int *lprof = nullptr;  // optional per-level profile [cap][2]
    int lprof_cap = 0;
    // bounded waits: polls of one wait before it gives up, and levels before the run is
    // declared runaway; either ends the launch with OIFT_E_NOT_CONVERGED
    long long spin_limit = OIFT_DEFAULT_SPIN_LIMIT;
    int max_levels = OIFT_DEFAULT_MAX_LEVELS;
};

template <typename T>
cudaError_t launch_build_weights(const T *img, uint16_t *W, const BuildArgs &a, int sms,
                                 cudaStream_t s);
template <typename T>
cudaError_t launch_minmax(const T *img, size_t n, int *mm, int sms, cudaStream_t s);

// Tensor maps of one relaxation's TMA-staged sweeps: the two ping-pong membership buffers
// as [C][Z][Y][X] floats and the image as [Z][Y][X], encoded on the host over this GPU's
// own buffers; err is a device flag a tile sets when its loads do not land.
struct RelaxTma {
    CUtensorMap memb[2];
    CUtensorMap img;
    const float *base[2];
    int *err;
};
// Encodes the maps; false when the extents do not allow TMA boxes (rows of the planes must
// start 16-byte aligned: X % 4 == 0 for int32 images, X % 8 == 0 for int16) or the driver
// entry point is missing -- the sweeps then stage with per-element copies.
bool relax_tma_encode(RelaxTma *t, const float *m0, const float *m1, const void *img,
                      bool img32, int X, int Y, int Z, int C);
// A 3D tensor map over an int16 / int32 image [Z][Y][X] with the given box (innermost
// first); false when the driver cannot encode it.
bool image_tma_encode(CUtensorMap *m, const void *img, bool img32, int X, int Y, int Z, int bx,
                      int by, int bz);

template <typename T>
cudaError_t launch_relax_tiles(int C, const float *in, float *out, const T *img,
                               const uint8_t *seedc, const uint16_t *tdist, int sweep,
                               const RelaxArgs &a, bool perclass, int ntiles, int ntx, int nty,
                               cudaStream_t s, const RelaxTma *tma = nullptr);
__global__ void relax_boundary_tiles_kernel(const int32_t *label, int X, int Y, int Z, int nadj,
                                            RelaxArgs a, uint16_t *tdist, int ntx, int nty);
__global__ void relax_tile_gap_pass_kernel(const uint16_t *din, uint16_t *dout, int ntx, int nty,
                                           int ntz, int ax, int dim, int cheb);
__global__ void relax_tile_hist_kernel(const uint16_t *tdist, int nt, int K, unsigned int *hist);
__global__ void relax_init_kernel(const int32_t *label, size_t N, int C, const int *l2c,
                                  int maxl, int bg, float *m);
__global__ void relax_seed_kernel(const int32_t *seeds, int nseeds, const int32_t *label,
                                  size_t N, const int *l2c, int maxl, int bg, uint8_t *seedc);
__global__ void seed_presence_kernel(const int32_t *seed_labels, int nseeds, uint32_t *bits);
__global__ void relax_argmax_kernel(const float *m, size_t N, int C, const int *classes,
                                    int32_t *label, uint8_t *mask);

// Warp tiling of the 6 / 4 OIFT: 32 x 32 in 2D; 32 x 8 x 4 in 3D, or 32 x 4 x 8 with tile_ty 4
// (the batched driver's second tile shape).
OiftPlan oift_plan(int X, int Y, int Z, int tile_ty = 8);
size_t oift_globals_bytes();
int oift_mbox_words(const OiftPlan &P, int ctas);
size_t oift_mbox_bytes(const OiftPlan &P, int ctas);
// Fewest CTAs that can own `ntiles` tiles (each CTA's tile sets live in shared memory).
int oift_min_ctas(const OiftPlan &P);
// One job (volume + seed set) of the batched OIFT kernel; the device copy is read by
// the team that draws it and receives the job's status.
struct OiftTeamJob {
    const uint16_t *W;  // edge codes of the job's volume, built before the launch
    const int32_t *seeds, *seed_labels;
    int32_t *cost, *label;  // device outputs, each may be null
    int X, Y, Z, nseeds;
    int ntx, nty, ntz, ntiles;
    float pol0;          // polarity (x100) of label 0
    float pol_default;   // polarity (x100) of every other label
    int status;          // out: OIFT_OK or OIFT_E_*; OIFT_TEAM_NOT_RUN until a team ends it
    int levels;          // out
    unsigned long long steps;  // out
};
#define OIFT_TEAM_NOT_RUN 1

// Per-team state of the batched kernel: team t uses key + t * key_stride and so on.
struct OiftTeamScratch {
    uint32_t *key;
    size_t key_stride;
    uint32_t *tpend;
    size_t tpend_stride;
    unsigned long long *mbox;
    size_t mbox_stride;
    OiftGlobals *g;           // [teams]
    unsigned int *next_job;   // job counter shared by the teams
    int *abort;               // set when a team stops on an error; others take no new job
    long long spin_limit = OIFT_DEFAULT_SPIN_LIMIT;  // as OiftScratch
    int max_levels = OIFT_DEFAULT_MAX_LEVELS;
};

// Batched OIFT: one cooperative launch of `ctas` CTAs split into `teams` teams of
// ctas/teams or ctas/teams + 1 CTAs; each team repeatedly draws the next job from d_jobs
// (in array order), clears its state, seeds, runs the level loop with a team barrier and
// writes cost / label.  All jobs of one call must be 2D (Z == 1) when planar, else 3D.
// The mailbox stride must hold oift_mbox_bytes for both team sizes.  Returns OIFT_OK once
// the launch is queued; per-job results are in d_jobs[].status.
// tile_ty selects the 3D warp tile: 8 (32 x 8 x 4, the default) or 4 (32 x 4 x 8).
int oift_team_run(OiftTeamJob *d_jobs, int njobs, bool planar, int teams, int ctas,
                  const OiftTeamScratch &S, cudaStream_t st, int tile_ty = 8);

// ---- steps around the path (prepost.cu) ----
template <typename T>
cudaError_t launch_shift_to_i32(const T *in, int32_t *out, size_t n, const int *d_mm, int sms,
                                cudaStream_t s);
template <typename T>
cudaError_t launch_gaussian_blur(const T *in, int32_t *out, int X, int Y, int Z, float w0,
                                 float w1, cudaStream_t s);
// Sobel gradient normalised to the image maximum (d_mm_img: image min / max on the device;
// d_mm_g: 2 ints of scratch).
template <typename T>
cudaError_t launch_sobel_normalized(const T *img, int32_t *g, int X, int Y, int Z,
                                    const int *d_mm_img, int *d_mm_g, int sms, cudaStream_t s);
__global__ void dilation_border_kernel(const int32_t *label, const int32_t *img, uint8_t *border,
                                       int X, int Y, int Z, const int *off, int noff,
                                       unsigned *hist_hi, unsigned *count);
__global__ void dilation_hist_lo_kernel(const uint8_t *border, const int32_t *img, size_t N,
                                        uint32_t hi, unsigned *hist_lo);
__global__ void dilation_tie_count_kernel(const uint8_t *border, const int32_t *img, size_t N,
                                          size_t chunk, uint32_t pivot, unsigned *counts);
__global__ void dilation_apply_kernel(const uint8_t *border, const int32_t *img, int32_t *label,
                                      size_t N, size_t chunk, uint32_t pivot,
                                      const unsigned *tie_base, unsigned take);

// Full 3x3(x3) neighbourhood OIFT (26 / 8): arc weights from the image on the fly.
struct OiftFullN {
    const void *img;
    bool img_i16;
    int wmode, wcap;
    const uint16_t *lut;
    int lut_len;
    // gradient blend: 6 / 4 face neighbourhood, weights from image + normalised Sobel map
    bool blend;
    const int32_t *gmap;
    float alpha;
    // exact weights wider than 14 bits: 64-bit keys (the scratch keys and pending keys are
    // twice as wide), base weights up to OIFT_WIDE_MAX_BASE; faces: only the 6 / 4 face
    // neighbours of the 3x3(x3) neighbourhood are arcs
    bool wide = false;
    bool faces = false;
};
// Tiling of the full-neighbourhood kernel: 32 x 4 x 4 (3D) or 32 x 16 (2D).
OiftPlan oift_plan_full(int X, int Y, int Z);

__global__ void pyr_subsample_kernel(const int32_t *fine, int32_t *coarse, int X, int Y, int Z,
                                     int cx, int cy, int cz);
__global__ void pyr_coarse_first_kernel(const int32_t *seeds, int nseeds, int X, int Y, int Z,
                                        int cx, int cy, int cz, unsigned *first);
__global__ void pyr_coarse_labels_kernel(const unsigned *first, const int32_t *seeds,
                                         const int32_t *fine_label, size_t cn, int32_t *clab);
__global__ void pyr_upscale_kernel(const int32_t *clab, int32_t *up, int X, int Y, int Z, int cx,
                                   int cy, const int *ix, const int *iy, const int *iz);
__global__ void pyr_boundary_nil_kernel(const int32_t *lab, int32_t *out, int X, int Y, int Z,
                                        const int *off, int noff);
__global__ void pyr_merge_kernel(const int32_t *label, const int32_t *up, int32_t *merged,
                                 size_t N);
__global__ void seeds_count_kernel(const int32_t *lab, size_t N, size_t chunk, unsigned *counts);
__global__ void seeds_scatter_kernel(const int32_t *lab, size_t N, size_t chunk,
                                     const unsigned *base_of, int32_t *seeds,
                                     int32_t *seed_labels);

// ---- relaxation of the oriented 2D image graph (imagegraph.cu) ----
struct IgRelax {
    int X, Y, adjacency;       // zsize == 1; 4 or 8
    float per;                 // global polarity x100
    int sweeps;
    const int32_t *olabel;     // OIFT labels
    const int32_t *seeds;
    int nseeds;
    float *m0, *m1;            // [N] each
    uint16_t *ring;            // [N]
    uint8_t *seedf;            // [N]
    int *small;                // 2 ints of scratch
    int32_t *label;            // out: binary labels, may be null
    uint8_t *mask;             // out, may be null
    float *membership;         // out: [N], may be null
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;  // around the sweeps
};
// sg->Wmax of Orient2Digraph from the largest |dI| over the in-image arcs (-1: none).
double ig_wmax(int dmax, float per);
template <typename T>
int ig_relax_run(const IgRelax &R, const T *img, cudaStream_t s, int sms, int *kernels);

// ---- adjoint of the relaxation (adjoint.cu) ----
struct AdjointJob {
    int X, Y, Z, adjacency;
    int sweeps, checkpoint;   // K, sweeps between stored states (>= 1)
    int C, bg;                // classes, background class
    int kernel;               // 0 RBF, 1 POW8
    float sigma, alpha, beta;
    double eps;               // soft-Dice smoothing
    int imax;                 // max of the image (POW8 Wmax)
    const int16_t *img;
    const float *g;           // gradient map for the blend (may be null)
    uint16_t *dist;           // [N] scratch: sweep at which a voxel joins the mask
    const uint8_t *seedc;     // [N] seed class or 0xFF
    const int32_t *labels0;   // [N] OIFT labels
    const int *l2c;           // label -> class (-1 if none), labels 0..maxl
    int maxl;
    const uint8_t *truth;     // [N] 0 / 1
    float *membership_out;    // [C][N] final membership, may be null
};
size_t adjoint_work_floats(size_t N, int C, int K, int c);

// ---- arc-weight-map adjoint (costgrad.cu) ----
// Bottleneck arcs of the fixed OIFT forest read from an integer OIFT result; arcs[p] =
// tail * 32 + direction (gft Spheric order, tail -> tail + d), -2 at seeds, -3 unreached.
struct BottleneckSetup {
    int X, Y, Z, adjacency;
    const int16_t *img;
    const int32_t *cost, *label;
    const uint8_t *seed;
    int wmode, wq;
    float per;  // global polarity x100 of the OIFT
};
__global__ void seed_flag_kernel(const int32_t *seeds, int nseeds, size_t N, uint8_t *flag);
int bottleneck_run(const BottleneckSetup &S, cudaStream_t s, int sms, long long *arcs,
                   long long *tmp, int *d_changed, int *h_changed, int *rounds_out);
// Soft-Dice loss of the cost-derived object confidence and its gradient w.r.t. (sigma,
// alpha, beta); d_sums holds max_blocks * 9 doubles.
struct CostLossSetup {
    int X, Y, Z, adjacency;
    const int16_t *img;
    const float *g;
    const int32_t *label;
    const long long *arcs;
    const uint8_t *truth;
    double sigma, alpha, beta, eps;
};
int cost_loss_run(const CostLossSetup &S, cudaStream_t s, int sms, double *d_sums,
                  int max_blocks, double *loss, double *grad);
int adjoint_run(const AdjointJob &J, cudaStream_t s, int sms, float *work, size_t work_floats,
                void *small, double *loss_out, double *grad_out);

// Queues one OIFT (seeds, persistent kernel, optional finalize) without host
// synchronisation; copy S.g and d_flag to the host after it and pass them to oift_result.
int oift_enqueue(const OiftPlan &P, const OiftScratch &S, const uint16_t *W, int X, int Y,
                 int Z, const int32_t *d_seeds, const int32_t *d_seed_labels, int nseeds,
                 const float *d_pol_table, int npol, float pol_default, int32_t *cost,
                 int32_t *label, int *d_flag, int sms, cudaStream_t st, cudaEvent_t ev_begin,
                 cudaEvent_t ev_end, const OiftFullN *fn, bool round_orient,
                 const uint16_t *Wt);
int oift_result(const OiftGlobals &g, int seed_flag, int *levels_out, long long *steps_out,
                unsigned long long *cycles_out);
int oift_run(const OiftPlan &P, const OiftScratch &S, const uint16_t *W, int X, int Y, int Z,
             const int32_t *d_seeds, const int32_t *d_seed_labels, int nseeds,
             const float *d_pol_table, int npol, float pol_default, int32_t *cost,
             int32_t *label, int *d_flag, int sms, cudaStream_t st, int *levels_out,
             long long *steps_out, cudaEvent_t ev_begin = nullptr, cudaEvent_t ev_end = nullptr,
             unsigned long long *cycles_out = nullptr, const OiftFullN *fn = nullptr,
             bool round_orient = false, const uint16_t *Wt = nullptr);

}  // namespace oiftb
