// Test infrastructure only: the reference's coarse-to-fine cascade
// (experiments/exp_coarse_to_fine.cpp) as a library call for the checker.  The experiment
// source is compiled here as it lies, inside a namespace and with its main renamed, so its
// own helpers (mark_boundary_voxels_nil, build_seeds_from_label, dilation_conditional) are
// the ones called; the steps of its main (lines 327-414) are sequenced on plain arrays:
// Subsampling, seeds mapped to (x/2, y/2, z/2) first-come, coarse OIFT_Multi +
// ORelax_1_Multi, ScaleLabel (nearest), boundary voxels to NIL, merge into the fine labels,
// every labelled voxel a seed, fine OIFT_Multi + ORelax_1_Multi, conditional dilation when
// binary.
#include "gft.h"
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <queue>
#include <string>
#include <vector>

namespace c2f {
#define main exp_coarse_to_fine_main
#include "exp_coarse_to_fine.cpp"
#undef main
}  // namespace c2f

#define REF_API __attribute__((visibility("default")))

extern "C" {

// img: the blurred, shifted volume (fscn); label: seed labels (NIL elsewhere), receives the
// result; seeds: the S list without its count.  adj: 6 or 26 (Spheric(1.0) / (1.75)).
// The polarity handed to OIFT_Multi / ORelax_1_Multi is (float)(pol * 100.0), the value the
// library's callers pass as `per`.
REF_API void ref_coarse_to_fine(const int *img, int X, int Y, int Z, int adj, double pol,
                                int niter, float percentile, const int *seeds, int nseeds,
                                int *label_io) {
    using namespace gft;
    const float per = (float)(pol * 100.0);
    sScene32 *fscn = Scene32::Create(X, Y, Z);
    std::memcpy(fscn->data, img, sizeof(int) * (size_t)X * Y * Z);
    sScene32 *label = Scene32::Create(X, Y, Z);
    std::memcpy(label->data, label_io, sizeof(int) * (size_t)X * Y * Z);
    sAdjRel3 *A = adj == 26 ? AdjRel3::Spheric(1.75f) : AdjRel3::Spheric(1.0f);
    int *S = (int *)calloc((size_t)nseeds + 1, sizeof(int));
    S[0] = nseeds;
    for (int i = 0; i < nseeds; i++) S[i + 1] = seeds[i];

    sScene32 *scn_coarse = Scene32::Subsampling(fscn);
    sScene32 *label_coarse = Scene32::Create(scn_coarse);
    Scene32::Fill(label_coarse, NIL);
    int *S_coarse = (int *)calloc((size_t)S[0] + 1, sizeof(int));
    S_coarse[0] = 0;
    for (int si = 1; si <= S[0]; si++) {
        const int pp = S[si];
        if (pp < 0 || pp >= label->n) continue;
        const int cx = Scene32::GetAddressX(label, pp) / 2;
        const int cy = Scene32::GetAddressY(label, pp) / 2;
        const int cz = Scene32::GetAddressZ(label, pp) / 2;
        if (Scene32::IsValidVoxel(scn_coarse, cx, cy, cz)) {
            const int cq = Scene32::GetVoxelAddress(scn_coarse, cx, cy, cz);
            if (label_coarse->data[cq] == NIL) {
                label_coarse->data[cq] = label->data[pp];
                S_coarse[0]++;
                S_coarse[S_coarse[0]] = cq;
            }
        }
    }
    ift::OIFT_Multi(A, scn_coarse, per, S_coarse, label_coarse);
    ift::ORelax_1_Multi(A, scn_coarse, per, S_coarse, label_coarse, niter);
    sScene32 *label_up = Scene32::ScaleLabel(label_coarse, fscn, none);
    Scene32::Destroy(&scn_coarse);
    Scene32::Destroy(&label_coarse);
    free(S_coarse);

    c2f::mark_boundary_voxels_nil(label_up, A);
    for (int pp = 0; pp < label->n; pp++)
        if (label_up->data[pp] != NIL && label->data[pp] == NIL) label->data[pp] = label_up->data[pp];
    Scene32::Destroy(&label_up);
    int n_fine = 0;
    int *S_fine = c2f::build_seeds_from_label(label, &n_fine);
    ift::OIFT_Multi(A, fscn, per, S_fine, label);
    ift::ORelax_1_Multi(A, fscn, per, S_fine, label, niter);
    free(S_fine);
    if (Scene32::GetMaximumValue(label) <= 1) c2f::dilation_conditional(fscn, label, 1.0f, percentile);
    std::memcpy(label_io, label->data, sizeof(int) * (size_t)X * Y * Z);
    free(S);
    AdjRel3::Destroy(&A);
    Scene32::Destroy(&label);
    Scene32::Destroy(&fscn);
}

}  // extern "C"
