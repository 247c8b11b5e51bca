// gft_shims.cpp -- the gft routines of the OIFT + relaxation path, defined over the C ABI
// of liboift_b200 with their exact gft signatures (gft/include/gft_ift.h:108-122, 451-465):
//
//   gft::ift::OIFT_Multi / OIFT_Multi_PerClass         -> oift_b200_run_host (no sweeps)
//   gft::ift::ORelax_1_Multi / ORelax_1_Multi_PerClass -> oift_b200_relax_host
//
// Built into libgft_oift_b200.so.  A program written against the gft library (the
// reference's oiftrelax.cpp CLI, unchanged) runs these four steps on the GPU when it links
// libgft_oift_b200.so ahead of a shared gft library: the dynamic linker binds the program's
// calls to the first definition in load order.
//
// The argument structs are the gft library's own, declared here with the same names and
// layout (gft/include/gft_scene32.h:20-27, gft/include/gft_adjrel3.h:9-23) so the symbols
// match; only data, xsize, ysize, zsize, n and the displacements are read.  S is the gft seed
// list (S[0] = count, S[1..S[0]] voxel addresses); as in OIFT_Multi, a NULL list means every
// labelled voxel is a seed.  The adjacency relation must be the 6- or 26-neighbourhood
// (Spheric(1.0) / Spheric(1.75), gft/src/gft_adjrel3.cpp:47-85; 4 / 8 on a volume one voxel
// deep).  Anything else, or a failed call, prints the status and ends the process, as the
// gft routines end it on an error.  The image is used as given (the CLI shifts and blurs it
// first); arc weights are |I_p - I_q| as in gft_ift.cpp:965-973.
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "../../include/oift_b200.h"

namespace gft {
namespace AdjRel3 {
struct v4si_layout {
    int d[4];
};
union sDisplacement3 {
    v4si_layout v;
    int data[4];
    struct {
        int x, y, z;
    } axis;
};
struct sAdjRel3 {
    sDisplacement3 *d;
    int n;
};
}  // namespace AdjRel3
namespace Scene32 {
struct sScene32 {
    int *data;
    int ***array;
    int xsize, ysize, zsize;
    float dx, dy, dz;
    int maxval, minval, n;
    void *nii_hdr;
};
}  // namespace Scene32
using AdjRel3::sAdjRel3;
using Scene32::sScene32;

namespace ift {
void OIFT_Multi(sAdjRel3 *A, sScene32 *scn, float per, int *S, sScene32 *label);
void OIFT_Multi_PerClass(sAdjRel3 *A, sScene32 *scn, const float *per_class, int max_label,
                         int *S, sScene32 *label);
void ORelax_1_Multi(sAdjRel3 *A, sScene32 *scn, float per, int *S, sScene32 *label,
                    int ntimes);
void ORelax_1_Multi_PerClass(sAdjRel3 *A, sScene32 *scn, const float *per_class, int max_label,
                             int *S, sScene32 *label, int ntimes);
}  // namespace ift
}  // namespace gft

namespace {

std::mutex g_mu;
oift_b200_ctx *g_ctx = nullptr;

[[noreturn]] void fail(const char *what, const char *why) {
    std::fprintf(stderr, "gft::ift::%s (liboift_b200): %s\n", what, why);
    std::exit(1);
}

oift_b200_ctx *context(const char *what) {
    if (!g_ctx) {
        const int rc = oift_b200_create(&g_ctx, 0);
        if (rc != OIFT_OK) fail(what, oift_b200_status_string(rc));
    }
    return g_ctx;
}

// 6 / 26 (4 / 8 on one plane) from a Spheric relation: the centre plus every offset in
// {-1,0,1}^3 with squared length <= 1 (n = 7) or <= 3 (n = 27).
int adjacency_of(const gft::sAdjRel3 *A, const gft::sScene32 *scn, const char *what) {
    if (!A || !A->d || (A->n != 7 && A->n != 27)) fail(what, "adjacency relation is not Spheric(1.0) / Spheric(1.75)");
    const int r2 = A->n == 7 ? 1 : 3;
    bool seen[27] = {false};
    for (int i = 0; i < A->n; i++) {
        const int x = A->d[i].axis.x, y = A->d[i].axis.y, z = A->d[i].axis.z;
        if (x < -1 || x > 1 || y < -1 || y > 1 || z < -1 || z > 1 || x * x + y * y + z * z > r2)
            fail(what, "adjacency relation is not Spheric(1.0) / Spheric(1.75)");
        seen[(z + 1) * 9 + (y + 1) * 3 + (x + 1)] = true;
    }
    int distinct = 0;
    for (bool b : seen) distinct += b;
    if (distinct != A->n) fail(what, "adjacency relation repeats an offset");
    if (scn->zsize == 1) return A->n == 7 ? 4 : 8;
    return A->n == 7 ? 6 : 26;
}

oift_b200_params params_of(const gft::sAdjRel3 *A, const gft::sScene32 *scn, float per,
                           const float *per_class, int max_label, int sweeps, const char *what) {
    if (!scn || !scn->data || scn->xsize <= 0 || scn->ysize <= 0 || scn->zsize <= 0)
        fail(what, "empty scene");
    oift_b200_params p{};
    p.xsize = scn->xsize;
    p.ysize = scn->ysize;
    p.zsize = scn->zsize;
    p.adjacency = adjacency_of(A, scn, what);
    p.weight_mode = OIFT_W_GRAD;
    p.wq = 4095;
    p.rbf_sigma = 150.0f;
    p.blend_a = 1.0f;
    p.per = per_class ? 0.0f : per;
    p.per_class = per_class;
    p.max_label = per_class ? max_label : 0;
    p.relax_sweeps = sweeps;
    return p;
}

// The gft seed list as 0-based addresses; NULL = every labelled voxel (gft_ift.cpp:941-948).
std::vector<int32_t> seeds_of(const int *S, const gft::sScene32 *label, const char *what) {
    std::vector<int32_t> out;
    const size_t n = (size_t)label->xsize * label->ysize * label->zsize;
    if (S) {
        for (int i = 1; i <= S[0]; i++) out.push_back(S[i]);
    } else {
        for (size_t p = 0; p < n; p++)
            if (label->data[p] != -1) out.push_back((int32_t)p);
    }
    if (out.empty()) fail(what, "no seeds");
    return out;
}

void oift(gft::sAdjRel3 *A, gft::sScene32 *scn, float per, const float *per_class, int max_label,
          int *S, gft::sScene32 *label, const char *what) {
    std::lock_guard<std::mutex> lock(g_mu);
    const oift_b200_params p = params_of(A, scn, per, per_class, max_label, 0, what);
    const std::vector<int32_t> seeds = seeds_of(S, label, what);
    const int rc = oift_b200_run_host(context(what), &p, scn->data, label->data, seeds.data(),
                                      (int)seeds.size(), nullptr, nullptr, 0, nullptr, nullptr);
    if (rc != OIFT_OK) fail(what, oift_b200_status_string(rc));
}

void relax(gft::sAdjRel3 *A, gft::sScene32 *scn, float per, const float *per_class, int max_label,
           int *S, gft::sScene32 *label, int ntimes, const char *what) {
    std::lock_guard<std::mutex> lock(g_mu);
    // without a seed list the reference runs its binary ORelax_1 instead (gft_ift.cpp:8678-8682)
    if (!S || S[0] <= 0) fail(what, "a seed list is required");
    if (ntimes < 0) fail(what, "negative sweep count");
    const oift_b200_params p = params_of(A, scn, per, per_class, max_label, ntimes, what);
    const std::vector<int32_t> seeds = seeds_of(S, label, what);
    const int rc = oift_b200_relax_host(context(what), &p, scn->data, label->data, seeds.data(),
                                        (int)seeds.size(), nullptr, 0, nullptr);
    if (rc != OIFT_OK) fail(what, oift_b200_status_string(rc));
}

}  // namespace

namespace gft {
namespace ift {

void OIFT_Multi(sAdjRel3 *A, sScene32 *scn, float per, int *S, sScene32 *label) {
    oift(A, scn, per, nullptr, 0, S, label, "OIFT_Multi");
}

void OIFT_Multi_PerClass(sAdjRel3 *A, sScene32 *scn, const float *per_class, int max_label,
                         int *S, sScene32 *label) {
    oift(A, scn, 0.0f, per_class, max_label, S, label, "OIFT_Multi_PerClass");
}

void ORelax_1_Multi(sAdjRel3 *A, sScene32 *scn, float per, int *S, sScene32 *label,
                    int ntimes) {
    relax(A, scn, per, nullptr, 0, S, label, ntimes, "ORelax_1_Multi");
}

void ORelax_1_Multi_PerClass(sAdjRel3 *A, sScene32 *scn, const float *per_class, int max_label,
                             int *S, sScene32 *label, int ntimes) {
    relax(A, scn, 0.0f, per_class, max_label, S, label, ntimes, "ORelax_1_Multi_PerClass");
}

}  // namespace ift
}  // namespace gft
