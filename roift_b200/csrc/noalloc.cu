// noalloc.cu -- OIFT on one volume without any device allocation.
//
// Who needs this: programs that cannot let a library call cudaMalloc while they run.
// Typical cases are applications whose own memory pool already holds (almost) all of the
// GPU's memory, so a private allocation fails or fragments the pool; pipelines that must
// not allocate after start-up because cudaMalloc / cudaFree synchronise the device and
// stall every other stream; and hosts that forbid plug-ins from allocating device memory
// on their own.  For them, oift_b200_oift_noalloc runs the arc-weight builder and the
// f_max OIFT with all intermediate state in one statically sized device array that the
// CUDA module owns: the caller passes only its inputs and outputs.
//
// The array is a file-scope __device__ variable.  Host code cannot use its name as a
// device address, so the first call on each device (with that device current) asks the
// runtime for the address with cudaGetSymbolAddress and keeps it; later calls reuse it.
// That first call should therefore happen before any stream capture.  Every call on a
// device shares the one array and leaves the last call's contents in it; the state that
// must start at zero is cleared by each call.  Calls that overlap on the GPU (two streams,
// two host threads) race on the array and corrupt each other's results.
#include <mutex>
#include <vector>

#include "kernels.cuh"

using namespace oiftb;

namespace {

constexpr size_t kMaxVoxels = OIFT_NOALLOC_MAX_VOXELS;
constexpr size_t kMaxTiles = 65536;        // warp tiles of 32x8x4 (3D) or 32x32 (2D)
constexpr size_t kMaxMailboxWords = 8192;  // re-activation bitmask words (8 bytes each)
constexpr size_t kMaxPolarity = 256;       // labels with their own polarity entry

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kOffW = 0;  // 3 planes of uint16 edge codes
constexpr size_t kOffKey = align256(kOffW + 3 * kMaxVoxels * sizeof(uint16_t));
constexpr size_t kOffTpend = align256(kOffKey + kMaxVoxels * sizeof(uint32_t));
constexpr size_t kOffMbox = align256(kOffTpend + kMaxTiles * sizeof(uint32_t));
constexpr size_t kOffGlob = align256(kOffMbox + kMaxMailboxWords * sizeof(unsigned long long));
constexpr size_t kOffPol = align256(kOffGlob + sizeof(OiftGlobals));
constexpr size_t kOffFlag = align256(kOffPol + kMaxPolarity * sizeof(float));
constexpr size_t kOffClamp = kOffFlag + 16;
constexpr size_t kScratchBytes = align256(kOffClamp + sizeof(unsigned long long));

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch_addr[kMaxDevices] = {};

}  // namespace

// About 10.3 MB; held by every device that loads this library, until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch on the current device (looked up once per device).
static int noalloc_scratch(unsigned char **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return OIFT_E_CUDA;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return OIFT_E_CUDA;
        }
        g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_addr[dev];
    return OIFT_OK;
}

extern "C" size_t oift_b200_noalloc_scratch_bytes(void) { return kScratchBytes; }

extern "C" int oift_b200_oift_noalloc(const int16_t *image, int xsize, int ysize, int zsize,
                                      int adjacency, int weight_mode, int wq, float per,
                                      const float *per_class, int max_label,
                                      const int32_t *seeds, const int32_t *seed_labels,
                                      int nseeds, int32_t *cost, int32_t *label, void *stream) {
    // ---- argument and size checks: nothing touches the device before they pass ----
    if (!image || !seeds || !seed_labels || (!cost && !label)) return OIFT_E_BAD_ARG;
    if (xsize <= 0 || ysize <= 0 || zsize <= 0) return OIFT_E_BAD_ARG;
    if (adjacency == 4) {
        if (zsize != 1) return OIFT_E_BAD_ARG;
    } else if (adjacency != 6) {
        return OIFT_E_UNSUPPORTED;
    }
    if (weight_mode != OIFT_W_GRAD && weight_mode != OIFT_W_GRAD_Q) return OIFT_E_UNSUPPORTED;
    if (weight_mode == OIFT_W_GRAD_Q && (wq <= 0 || wq > OIFT_MAX_BASE)) return OIFT_E_BAD_ARG;
    if (nseeds <= 0) return OIFT_E_NO_SEEDS;
    const unsigned long long N = (unsigned long long)xsize * ysize * zsize;
    if (N > kMaxVoxels) return OIFT_E_RANGE;  // larger than the static scratch
    std::vector<float> pol;
    float pol_default;
    if (per_class) {
        if (max_label < 0 || (size_t)max_label + 1 > kMaxPolarity) return OIFT_E_RANGE;
        for (int i = 0; i <= max_label; i++)
            if (!(per_class[i] >= -100.0f && per_class[i] <= 100.0f)) return OIFT_E_BAD_ARG;
        pol.assign(per_class, per_class + max_label + 1);
        pol_default = 0.0f;
    } else {
        if (!(per >= -100.0f && per <= 100.0f)) return OIFT_E_BAD_ARG;
        pol.push_back(-per);  // label 0 takes -per (gft_ift.cpp:968)
        pol_default = per;
    }
    const OiftPlan plan = oift_plan(xsize, ysize, zsize);
    if ((size_t)plan.ntiles > kMaxTiles) return OIFT_E_RANGE;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return OIFT_E_CUDA;
    }
    if (oift_mbox_bytes(plan, sms) > kMaxMailboxWords * sizeof(unsigned long long))
        return OIFT_E_RANGE;

    unsigned char *base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc != OIFT_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint16_t *W = reinterpret_cast<uint16_t *>(base + kOffW);
    float *d_pol = reinterpret_cast<float *>(base + kOffPol);
    int *d_flag = reinterpret_cast<int *>(base + kOffFlag);
    unsigned long long *d_clamp = reinterpret_cast<unsigned long long *>(base + kOffClamp);

    // ---- arc weights into the static scratch ----
    const Adjacency adj = make_adjacency(6);
    BuildArgs ba{};
    ba.X = xsize;
    ba.Y = ysize;
    ba.Z = zsize;
    ba.planes = 3;
    ba.mode = weight_mode;
    ba.cap = (weight_mode == OIFT_W_GRAD) ? OIFT_MAX_BASE : wq;
    for (int k = 0; k < 3; k++) {
        ba.dx[k] = adj.dx[adj.n / 2 + k];
        ba.dy[k] = adj.dy[adj.n / 2 + k];
        ba.dz[k] = adj.dz[adj.n / 2 + k];
    }
    ba.clamped = d_clamp;
    if (cudaMemsetAsync(d_clamp, 0, sizeof(unsigned long long), s) != cudaSuccess ||
        cudaMemcpyAsync(d_pol, pol.data(), pol.size() * sizeof(float), cudaMemcpyHostToDevice,
                        s) != cudaSuccess ||
        launch_build_weights<int16_t>(image, W, ba, sms, s) != cudaSuccess) {
        cudaGetLastError();
        return OIFT_E_CUDA;
    }

    // ---- OIFT with every piece of state inside the static scratch ----
    OiftScratch S;
    S.key = reinterpret_cast<uint32_t *>(base + kOffKey);
    S.tpend = reinterpret_cast<uint32_t *>(base + kOffTpend);
    S.mbox = reinterpret_cast<unsigned long long *>(base + kOffMbox);
    S.g = reinterpret_cast<OiftGlobals *>(base + kOffGlob);
    int levels = 0;
    long long steps = 0;
    rc = oift_run(plan, S, W, xsize, ysize, zsize, seeds, seed_labels, nseeds, d_pol,
                  (int)pol.size(), pol_default, cost, label, d_flag, sms, s, &levels, &steps);
    if (rc != OIFT_OK) return rc;
    unsigned long long clamped = 0;
    if (cudaMemcpyAsync(&clamped, d_clamp, sizeof(clamped), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return OIFT_E_CUDA;
    }
    if (weight_mode == OIFT_W_GRAD && clamped) return OIFT_E_RANGE;
    return OIFT_OK;
}
