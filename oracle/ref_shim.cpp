// Test infrastructure only: a flat C entry layer over the reference gft library
// (jung0221/roift, gft/src), compiled together with the reference's own sources
// into oracle/_ref/libgft_ref.so by oracle/Makefile.  Nothing in the product links
// this file; tests, the golden-fixture generator and the CPU baseline of bench.py
// call it through ctypes as the checker and as the timed reference arm.
//
// Each function wraps one reference routine on plain arrays:
//   ref_oift_multi            -> gft::ift::OIFT_Multi            (gft/src/gft_ift.cpp:911-989)
//   ref_oift_multi_perclass   -> gft::ift::OIFT_Multi_PerClass   (gft/src/gft_ift.cpp:991-1083)
//   ref_orelax_multi          -> gft::ift::ORelax_1_Multi        (gft/src/gft_ift.cpp:8655-8911)
//   ref_orelax_multi_perclass -> gft::ift::ORelax_1_Multi_PerClass (gft/src/gft_ift.cpp:8913-9187)
//   ref_ift_fmax_graph        -> gft::ift::IFT_fmax(sGraph*) on Graph::ByEuclideanDistance
//                                (gft/src/gft_ift.cpp:4753-4809, gft/src/gft_graph.cpp:126-155)
//   ref_gaussian_blur         -> gft::Scene32::GaussianBlur      (gft/src/gft_filtering3.cpp:385-397)
//   ref_energy_min_graph      -> gft::ift::GetEnergy_Min(sGraph*) (gft/src/gft_ift.cpp:4xx)
//   ref_dilation_conditional  -> dilation_conditional             (oiftrelax.cpp:149-165)
//   ref_inject_boundary_seeds -> inject_boundary_seeds            (oiftrelax.cpp:175-224)
//   ref_imagegraph            -> ImageGraph::ByEuclideanDistance + Orient2Digraph
//                                (gft/src/gft_imagegraph.cpp:13-47, 981-1016), then
//                                ift::OIFT(sImageGraph*) with S = NULL and, for ntimes > 0,
//                                ift::ORelax_1(sImageGraph*) (gft/src/gft_ift.cpp:1358-1439,
//                                7683-7847): the 2D pipeline of gft_ift.cpp:9575-9682, 9785-9790
//   ref_imagegraph_energy     -> ift::GetEnergy_Min(sImageGraph*) (gft/src/gft_ift.cpp:287-319)
//   ref_read_volume           -> gft::Scene32::Read  (gft/src/gft_scene32.cpp:334-420, 525-580)
//   ref_write_volume          -> gft::Scene32::Write (gft/src/gft_scene32.cpp:600-660, 748-800)
//   ref_oiftrelax_chain       -> the processing chain of the CLI main (oiftrelax.cpp:
//                                263-268, 368-414): shift, GaussianBlur x2, OIFT_Multi,
//                                ORelax_1_Multi, conditional dilation when binary
// The two CLI helpers come from oiftrelax.cpp itself, compiled with its main renamed.
//
// Seeds are passed 0-based without a count; the 1-based S[0]=count list the
// reference expects is built here.  Adjacency radius: 6-adj = Spheric(1.0),
// 26-adj = Spheric(1.75) (gft/src/gft_adjrel3.cpp:47-85); with zsize == 1 they
// reduce to 4-adj and 8-adj.
#include "gft.h"
#include <cstring>
#include <cstdlib>
#include <vector>

using namespace gft;

static sScene32 *make_scene(const int *data, int X, int Y, int Z) {
    sScene32 *s = Scene32::Create(X, Y, Z);
    if (data) std::memcpy(s->data, data, sizeof(int) * (size_t)X * Y * Z);
    return s;
}

static int *make_S(const int *seeds, int nseeds) {
    int *S = (int *)calloc((size_t)nseeds + 1, sizeof(int));
    S[0] = nseeds;
    for (int i = 0; i < nseeds; i++) S[i + 1] = seeds[i];
    return S;
}

static sAdjRel3 *make_adj(int adj) {
    return (adj == 26 || adj == 8) ? AdjRel3::Spheric(1.75f) : AdjRel3::Spheric(1.0f);
}

#define REF_API __attribute__((visibility("default")))

// defined in oiftrelax.cpp (compiled into the same library with main renamed)
void dilation_conditional(gft::sScene32 *scn, gft::sScene32 *label, float radius_sphere,
                          float percentile);
int inject_boundary_seeds(gft::sScene32 *label, int *&S, int current_count, int stride);

extern "C" {

REF_API void ref_oift_multi(const int *img, int X, int Y, int Z, int adj, float per,
                    const int *seeds, int nseeds, int *label) {
    sScene32 *scn = make_scene(img, X, Y, Z);
    sScene32 *lab = make_scene(label, X, Y, Z);
    sAdjRel3 *A = make_adj(adj);
    int *S = make_S(seeds, nseeds);
    ift::OIFT_Multi(A, scn, per, S, lab);
    std::memcpy(label, lab->data, sizeof(int) * (size_t)X * Y * Z);
    free(S);
    AdjRel3::Destroy(&A);
    Scene32::Destroy(&lab);
    Scene32::Destroy(&scn);
}

REF_API void ref_oift_multi_perclass(const int *img, int X, int Y, int Z, int adj,
                             const float *per_class, int max_label,
                             const int *seeds, int nseeds, int *label) {
    sScene32 *scn = make_scene(img, X, Y, Z);
    sScene32 *lab = make_scene(label, X, Y, Z);
    sAdjRel3 *A = make_adj(adj);
    int *S = make_S(seeds, nseeds);
    ift::OIFT_Multi_PerClass(A, scn, per_class, max_label, S, lab);
    std::memcpy(label, lab->data, sizeof(int) * (size_t)X * Y * Z);
    free(S);
    AdjRel3::Destroy(&A);
    Scene32::Destroy(&lab);
    Scene32::Destroy(&scn);
}

REF_API void ref_orelax_multi(const int *img, int X, int Y, int Z, int adj, float per,
                      const int *seeds, int nseeds, int *label, int ntimes) {
    sScene32 *scn = make_scene(img, X, Y, Z);
    sScene32 *lab = make_scene(label, X, Y, Z);
    sAdjRel3 *A = make_adj(adj);
    int *S = make_S(seeds, nseeds);
    ift::ORelax_1_Multi(A, scn, per, S, lab, ntimes);
    std::memcpy(label, lab->data, sizeof(int) * (size_t)X * Y * Z);
    free(S);
    AdjRel3::Destroy(&A);
    Scene32::Destroy(&lab);
    Scene32::Destroy(&scn);
}

REF_API void ref_orelax_multi_perclass(const int *img, int X, int Y, int Z, int adj,
                               const float *per_class, int max_label,
                               const int *seeds, int nseeds, int *label, int ntimes) {
    sScene32 *scn = make_scene(img, X, Y, Z);
    sScene32 *lab = make_scene(label, X, Y, Z);
    sAdjRel3 *A = make_adj(adj);
    int *S = make_S(seeds, nseeds);
    ift::ORelax_1_Multi_PerClass(A, scn, per_class, max_label, S, lab, ntimes);
    std::memcpy(label, lab->data, sizeof(int) * (size_t)X * Y * Z);
    free(S);
    AdjRel3::Destroy(&A);
    Scene32::Destroy(&lab);
    Scene32::Destroy(&scn);
}

// Un-oriented f_max IFT with exported cost.  Arc weights are |I_p - I_q| + 1
// (ByEuclideanDistance), so cost(q) = our f_max cost + 1 on non-seed voxels.
REF_API void ref_ift_fmax_graph(const int *img, int X, int Y, int Z, int adj,
                        const int *seeds, int nseeds, int *label, int *cost) {
    sScene32 *scn = make_scene(img, X, Y, Z);
    float r = (adj == 26 || adj == 8) ? 1.75f : 1.0f;
    sGraph *g = Graph::ByEuclideanDistance(scn, r);
    int *S = make_S(seeds, nseeds);
    ift::IFT_fmax(g, S, label, cost);
    free(S);
    Graph::Destroy(&g);
    Scene32::Destroy(&scn);
}

// Un-oriented minimum cut energy on the ByEuclideanDistance graph (weights |dI|+1).
REF_API int ref_energy_min_graph(const int *img, int X, int Y, int Z, int adj,
                         const int *label, int lb) {
    sScene32 *scn = make_scene(img, X, Y, Z);
    float r = (adj == 26 || adj == 8) ? 1.75f : 1.0f;
    sGraph *g = Graph::ByEuclideanDistance(scn, r);
    int e = ift::GetEnergy_Min(g, const_cast<int *>(label), lb);
    Graph::Destroy(&g);
    Scene32::Destroy(&scn);
    return e;
}

REF_API void ref_gaussian_blur(const int *img, int X, int Y, int Z, int *out) {
    sScene32 *scn = make_scene(img, X, Y, Z);
    sScene32 *b = Scene32::GaussianBlur(scn);
    std::memcpy(out, b->data, sizeof(int) * (size_t)X * Y * Z);
    Scene32::Destroy(&b);
    Scene32::Destroy(&scn);
}


REF_API void ref_dilation_conditional(const int *img, int *label, int X, int Y, int Z,
                                      float radius, float percentile) {
    sScene32 *scn = make_scene(img, X, Y, Z);
    sScene32 *lab = make_scene(label, X, Y, Z);
    dilation_conditional(scn, lab, radius, percentile);
    std::memcpy(label, lab->data, sizeof(int) * (size_t)X * Y * Z);
    Scene32::Destroy(&lab);
    Scene32::Destroy(&scn);
}

// Appends the boundary seeds to `seeds` (nseeds entries) into out[0, cap); returns the new
// total count.
REF_API int ref_inject_boundary_seeds(int *label, int X, int Y, int Z, int stride,
                                      const int *seeds, int nseeds, int *out, int cap) {
    sScene32 *lab = make_scene(label, X, Y, Z);
    int *S = make_S(seeds, nseeds);
    inject_boundary_seeds(lab, S, nseeds, stride);
    const int total = S[0];
    for (int i = 0; i < total && i < cap; i++) out[i] = S[i + 1];
    std::memcpy(label, lab->data, sizeof(int) * (size_t)X * Y * Z);
    free(S);
    Scene32::Destroy(&lab);
    return total;
}

// The CLI chain on an unshifted image; label holds the seed labels (NIL elsewhere) and
// receives the result.  pol in [-1, 1] as on the command line.
REF_API void ref_oiftrelax_chain(const int *img, int X, int Y, int Z, double pol, int niter,
                                 float percentile, const int *seeds, int nseeds, int *label) {
    sScene32 *scn = make_scene(img, X, Y, Z);
    sScene32 *lab = make_scene(label, X, Y, Z);
    sAdjRel3 *A = AdjRel3::Spheric(1.0);
    int *S = make_S(seeds, nseeds);
    const int Imin = Scene32::GetMinimumValue(scn);
    if (Imin < 0)
        for (int p = 0; p < scn->n; p++) scn->data[p] += (-Imin);
    sScene32 *fscn = Scene32::GaussianBlur(scn);
    Scene32::Destroy(&scn);
    scn = fscn;
    fscn = Scene32::GaussianBlur(scn);
    Scene32::Destroy(&scn);
    ift::OIFT_Multi(A, fscn, pol * 100.0, S, lab);
    ift::ORelax_1_Multi(A, fscn, pol * 100.0, S, lab, niter);
    if (Scene32::GetMaximumValue(lab) <= 1) dilation_conditional(fscn, lab, 1, percentile);
    std::memcpy(label, lab->data, sizeof(int) * (size_t)X * Y * Z);
    free(S);
    AdjRel3::Destroy(&A);
    Scene32::Destroy(&lab);
    Scene32::Destroy(&fscn);
}
static sImageGraph *make_imagegraph(const int *img, int X, int Y, int adj, float per,
                                    sImage32 **im_out) {
    sImage32 *im = Image32::Create(X, Y);
    std::memcpy(im->data, img, sizeof(int) * (size_t)X * Y);
    sImageGraph *sg = ImageGraph::ByEuclideanDistance(im, adj == 8 ? 1.5f : 1.0f);
    ImageGraph::Orient2Digraph(sg, im, per);
    *im_out = im;
    return sg;
}

// label: in, NIL (-1) except at the seeds; out, the OIFT labels, or the binary relaxed
// labels when ntimes > 0.  Returns sg->Wmax.
REF_API int ref_imagegraph(const int *img, int X, int Y, int adj, float per, const int *seeds,
                           int nseeds, int *label, int ntimes) {
    sImage32 *im = nullptr;
    sImageGraph *sg = make_imagegraph(img, X, Y, adj, per, &im);
    sImage32 *lab = Image32::Create(X, Y);
    std::memcpy(lab->data, label, sizeof(int) * (size_t)X * Y);
    ift::OIFT(sg, nullptr, lab);
    if (ntimes > 0) {
        int *S = make_S(seeds, nseeds);
        ift::ORelax_1(sg, S, lab, ntimes);
        free(S);
    }
    std::memcpy(label, lab->data, sizeof(int) * (size_t)X * Y);
    const int wmax = sg->Wmax;
    Image32::Destroy(&lab);
    ImageGraph::Destroy(&sg);
    Image32::Destroy(&im);
    return wmax;
}

REF_API int ref_imagegraph_energy(const int *img, int X, int Y, int adj, float per,
                                  const int *label, int lb) {
    sImage32 *im = nullptr;
    sImageGraph *sg = make_imagegraph(img, X, Y, adj, per, &im);
    sImage32 *lab = Image32::Create(X, Y);
    std::memcpy(lab->data, label, sizeof(int) * (size_t)X * Y);
    const int e = ift::GetEnergy_Min(sg, lab, lb);
    Image32::Destroy(&lab);
    ImageGraph::Destroy(&sg);
    Image32::Destroy(&im);
    return e;
}

// Reads a volume file; data may be null (dims and spacing only).  Returns the voxel count.
REF_API int ref_read_volume(const char *path, int *data, int cap, int *dims, float *spacing) {
    sScene32 *scn = Scene32::Read(const_cast<char *>(path));
    if (!scn) return -1;
    dims[0] = scn->xsize;
    dims[1] = scn->ysize;
    dims[2] = scn->zsize;
    spacing[0] = scn->dx;
    spacing[1] = scn->dy;
    spacing[2] = scn->dz;
    const int n = scn->n;
    if (data && cap >= n) std::memcpy(data, scn->data, sizeof(int) * (size_t)n);
    Scene32::Destroy(&scn);
    return n;
}

REF_API void ref_write_volume(const char *path, const int *data, const int *dims,
                              const float *spacing) {
    sScene32 *scn = make_scene(data, dims[0], dims[1], dims[2]);
    scn->dx = spacing[0];
    scn->dy = spacing[1];
    scn->dz = spacing[2];
    Scene32::Write(scn, const_cast<char *>(path));
    Scene32::Destroy(&scn);
}

}  // extern "C"
