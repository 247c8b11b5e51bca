// Test infrastructure only: the reference's gradient-blend experiment
// (experiments/exp_gradient_weight.cpp) as library calls for the checker.  The experiment
// source is compiled here as it lies, inside a namespace and with its main renamed, so its
// own OIFT_Multi_GradWeight and ORelax_1_Multi_GradWeight are the ones called; the Sobel
// gradient is the library's Scene32::SobelFilter, normalised as the experiment's main does
// (exp_gradient_weight.cpp:596-608).  Adjacency Spheric(1.0), as in the experiment.
#include "gft.h"
#include "gft_gradient3.h"
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

namespace blend {
#define main exp_gradient_weight_main
#include "exp_gradient_weight.cpp"
#undef main
}  // namespace blend

#define REF_API __attribute__((visibility("default")))

using namespace gft;

static sScene32 *scene_of(const int *data, int X, int Y, int Z) {
    sScene32 *s = Scene32::Create(X, Y, Z);
    if (data) std::memcpy(s->data, data, sizeof(int) * (size_t)X * Y * Z);
    return s;
}

static int *s_list(const int *seeds, int nseeds) {
    int *S = (int *)calloc((size_t)nseeds + 1, sizeof(int));
    S[0] = nseeds;
    for (int i = 0; i < nseeds; i++) S[i + 1] = seeds[i];
    return S;
}

extern "C" {

REF_API void ref_sobel_normalized(const int *img, int X, int Y, int Z, int *out) {
    sScene32 *fscn = scene_of(img, X, Y, Z);
    sScene32 *g = Scene32::SobelFilter(fscn);
    const int Gmax = Scene32::GetMaximumValue(g);
    const int Wmax = Scene32::GetMaximumValue(fscn);
    if (Gmax > 0 && Wmax > 0)
        for (int p = 0; p < g->n; p++) g->data[p] = (int)((long long)g->data[p] * Wmax / Gmax);
    std::memcpy(out, g->data, sizeof(int) * (size_t)X * Y * Z);
    Scene32::Destroy(&g);
    Scene32::Destroy(&fscn);
}

// OIFT_Multi_GradWeight followed by ORelax_1_Multi_GradWeight (ntimes sweeps; 0 = OIFT
// labels only).  label: seed labels in, result out.
REF_API void ref_gradweight(const int *img, const int *grad, int X, int Y, int Z, float per,
                            float alpha, const int *seeds, int nseeds, int *label, int ntimes) {
    sScene32 *scn = scene_of(img, X, Y, Z);
    sScene32 *g = scene_of(grad, X, Y, Z);
    sScene32 *lab = scene_of(label, X, Y, Z);
    sAdjRel3 *A = AdjRel3::Spheric(1.0f);
    int *S = s_list(seeds, nseeds);
    blend::OIFT_Multi_GradWeight(A, scn, g, per, alpha, S, lab);
    if (ntimes > 0) blend::ORelax_1_Multi_GradWeight(A, scn, g, per, alpha, S, lab, ntimes);
    std::memcpy(label, lab->data, sizeof(int) * (size_t)X * Y * Z);
    free(S);
    AdjRel3::Destroy(&A);
    Scene32::Destroy(&lab);
    Scene32::Destroy(&g);
    Scene32::Destroy(&scn);
}

}  // extern "C"
