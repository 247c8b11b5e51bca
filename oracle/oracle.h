/*
 * oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference (jung0221/roift, gft library) algorithms on
 * the OIFT + relaxation path.  It is the checker for the CUDA product: only tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py may load it.  The
 * product never links or calls it.
 *
 * Parity of this restatement is pinned against the reference itself: the reference
 * sources are compiled into oracle/_ref/libgft_ref.so (oracle/Makefile) and the tests
 * compare R1 labels, R2 costs at alpha = 0, R3 FP32 labels and the energies with it;
 * tests/golden/ holds fixtures generated from that build (tests/golden/make_golden.py).
 *
 * Conventions shared with the CUDA library (include/oift_b200.h):
 *   - voxel address p = x + y*X + z*X*Y (gft/include/gft_scene32.h:164-179);
 *   - neighbours in gft Spheric order (gft/src/gft_adjrel3.cpp:47-85), centre removed:
 *     6-adj [-z,-y,-x,+x,+y,+z], 26-adj the 3x3x3 cube in (dz,dy,dx) order; entry i
 *     and entry n-1-i (0-based, n = 6 or 26) are opposite;
 *   - weight map: one uint16 plane per "positive" direction (the second half of the
 *     list), plane k holding the edge p <-> p + d_k at address p.  Bits 0..13 = base
 *     weight, bit 14 = (I_p < I_q), bit 15 = (I_p > I_q);
 *   - labels: NIL = -1, 0 = background, >= 1 objects.
 */
#ifndef ROIFT_ORACLE_H
#define ROIFT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_NIL (-1)
#define OR_WMAX_BASE 16383

enum { OR_W_GRAD = 0, OR_W_GRAD_Q = 1, OR_W_RBF_Q = 2, OR_W_BLEND_Q = 3 };

/* Neighbour offsets (centre excluded) in Spheric order; returns 6 or 26. */
int or_adjacency(int adj, int *dx, int *dy, int *dz);

/* Builder restatement.  mode GRAD: |dI|; GRAD_Q: min(|dI|, wq);
 * RBF_Q: lut[|dI|] with lut built by or_rbf_lut; BLEND_Q: (int)(a*|dI| + (1-a)*(g_p+g_q)*0.5f)
 * clamped to wq.  Returns the number of edges whose base weight was clamped. */
long long or_build_weights(const int *img, int X, int Y, int Z, int adj, int mode, int wq,
                           const uint16_t *lut, int lut_len, const int *grad, float blend_a,
                           uint16_t *W);

/* Gaussian-RBF quantisation table: lut[d] = floor(wq*(1-exp(-d^2/(2 sigma^2))) + 0.5). */
void or_rbf_lut(double sigma, int wq, int len, uint16_t *lut);

/* Polarity of a label: table[l] for 0 <= l < ntable, else dflt (x100 units). */
typedef struct {
    const float *table;
    int ntable;
    float dflt;
} or_polarity;

/* Oriented arc weight for an arc tail -> head whose edge code is w with
 * gt/lt bits read relative to the tail; pol = polarity of the tail's label.
 * Follows gft/src/gft_ift.cpp:965-973 (int *= double, truncation). */
int or_oriented(uint16_t base, int tail_gt, int tail_lt, float pol);

/* R2: lexicographic (cost, label) Dijkstra with f_max and tail-label oriented
 * weights.  seeds[i] get key (0, max(label_in[seeds[i]], 0)); other voxels start
 * unlabelled.  Outputs cost (INT32_MAX if unreached), label (NIL if unreached) and
 * pred (-1 for seeds).  Returns the number of distinct (cost,label) levels popped. */
int or_oift_fmax(const uint16_t *W, int X, int Y, int Z, int adj, or_polarity pol,
                 const int *seeds, int nseeds, const int *label_in,
                 int *cost, int *label, int *pred);

/* R1: restatement of gft::ift::OIFT_Multi / OIFT_Multi_PerClass (Prim order, Dial
 * bucket queue with FIFO ties and a backwards-moving minimum, gft_pqueue32.cpp:300-451).
 * Works on the weight map (GRAD mode reproduces |I_p - I_q|).  label is in/out as in
 * the reference.  value = conquering arc weight, pred = predecessor, fmax = f_max
 * derived along the forest.  Any of value/pred/fmax may be NULL. */
void or_oift_prim(const uint16_t *W, int X, int Y, int Z, int adj, or_polarity pol,
                  int wmax_buckets, const int *seeds, int nseeds, int *label,
                  int *value, int *pred, int *fmax);

/* R4: oriented minimum cut energy.  For every arc p->q with label[p] != label[q],
 * weight = oriented weight with the tail's polarity; energy_all = min over all such
 * arcs; energy_lb[l] (l < nl) = min over arcs whose tail has label l.  INT32_MAX when
 * there is no such arc. */
int or_energy(const uint16_t *W, int X, int Y, int Z, int adj, or_polarity pol,
              const int *label, int nl, int *energy_lb);

/* Equal-cost tie accounting between labelling A (the lexicographic restatement R2 or the
 * CUDA result) and labelling B (the reference's Prim forest) over one cost map.  out[4]:
 * tie voxels of A (offered their cost by two labels), label differences, differences
 * where both labels are offered the voxel's cost, and unexplained differences.  flags
 * (optional) per voxel: bit 0 tie in A, bit 1 differs, bit 2 difference explained. */
void or_tie_stats(const uint16_t *W, int X, int Y, int Z, int adj, or_polarity pol,
                  const int *cost, const int *labA, const int *labB,
                  const unsigned char *is_seed, long long *out, unsigned char *flags);

/* Relaxation classes (gft_ift.cpp:8684-8720): classes = sorted labels present among
 * the seeds plus 0.  Returns nclasses, fills class_labels[<=cap]. */
int or_relax_classes(const int *seeds, int nseeds, const int *label, int n,
                     int *class_labels, int cap);

/* R3: ORelax_1_Multi (per_class == NULL, global polarity per) or
 * ORelax_1_Multi_PerClass (per_class != NULL, max_label) restated in FP32 with the
 * reference's exact operation order (gft_ift.cpp:8655-8911 / 8913-9187), masked
 * active set included.  membership out is planar [nclasses][N].  label is in/out. */
int or_relax_f32(const int *img, int X, int Y, int Z, int adj, float per,
                 const float *per_class, int max_label,
                 const int *seeds, int nseeds, int *label, int ntimes, float *membership);

/* The same sweeps in FP64 (the FP64 oracle for the FP32 kernels). */
int or_relax_f64(const int *img, int X, int Y, int Z, int adj, float per,
                 const float *per_class, int max_label,
                 const int *seeds, int nseeds, int *label, int ntimes, double *membership);

/* GaussianBlur restatement (gft_filtering3.cpp:106-126,321-346,385-397). */
void or_gaussian_blur(const int *img, int X, int Y, int Z, int *out);

/* Blend weights (experiments/exp_gradient_weight.cpp): Sobel gradient normalised to the
 * image maximum; R2 and R1 with blend arc weights; the blend relaxation (FP32). */
void or_sobel_normalized(const int *img, int X, int Y, int Z, int *out);
int or_oift_fmax_blend(const int *img, const int *g, float alpha, int X, int Y, int Z, int adj,
                       or_polarity pol, const int *seeds, int nseeds, const int *label_in,
                       int *cost, int *label);
void or_oift_prim_blend(const int *img, const int *g, float alpha, int X, int Y, int Z, int adj,
                        or_polarity pol, int wmax_buckets, const int *seeds, int nseeds,
                        int *label);
int or_relax_blend_f32(const int *img, const int *g, float alpha, int X, int Y, int Z, int adj,
                       float per, const int *seeds, int nseeds, int *label, int ntimes,
                       float *membership);

/* The oriented 2D image graph (gft_imagegraph.cpp:13-47, 981-1016): R2 and R1 with its
 * arc weights, its Wmax, and ORelax_1(sImageGraph) in FP32 (gft_ift.cpp:7683-7847). */
int or_oift_fmax_imagegraph(const int *img, int X, int Y, int adj, or_polarity pol,
                            const int *seeds, int nseeds, const int *label_in, int *cost,
                            int *label, int *pred);
void or_oift_prim_imagegraph(const int *img, int X, int Y, int adj, or_polarity pol,
                             int wmax, const int *seeds, int nseeds, int *label, int *value_out,
                             int *pred_out, int *fmax_out);
int or_imagegraph_wmax(const int *img, int X, int Y, int adj, float per);
int or_energy_imagegraph(const int *img, int X, int Y, int adj, float per, const int *label,
                         int lb);
void or_relax_imagegraph_f32(const int *img, int X, int Y, int adj, float per,
                             const int *seeds, int nseeds, int *label, int ntimes,
                             float *m_out);

/* oiftrelax.cpp:87-169 conditional dilation (label in/out); returns voxels relabelled. */
long long or_conditional_dilation(const int *img, int *label, int X, int Y, int Z,
                                  float radius, float percentile);
/* oiftrelax.cpp:175-224 boundary seeds; returns the count (out holds up to cap). */
int or_inject_boundary_seeds(int *label, int X, int Y, int Z, int stride, int *out, int cap);

#ifdef __cplusplus
}
#endif
#endif
