"""Generate the golden fixtures of tests/golden/ from the reference gft library itself.

The reference sources are compiled into oracle/_ref/libgft_ref.so (oracle/Makefile,
target `ref`); this script runs the reference routines on small seeded inputs and stores
inputs and outputs as .npz files.  The CPU test-suite checks the C restatement (the
oracle) against these files, so parity stays pinned even where the reference tree is
absent.  Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402
from roift_b200 import synth  # noqa: E402

CASES = [
    # name, shape (Z,Y,X), pol, adjacency, nlabels, per_class
    ("g3d_a", (12, 14, 16), -0.3, 6, 1, None),
    ("g3d_b", (10, 16, 20), 0.5, 6, 2, None),
    ("g3d_alpha0", (12, 12, 18), 0.0, 6, 1, None),
    ("g3d_26", (8, 10, 12), -0.5, 26, 2, None),
    ("g2d_4", (1, 24, 32), 0.5, 4, 1, None),
    ("g2d_8", (1, 20, 28), -0.2, 8, 2, None),
    ("g3d_perclass", (10, 14, 18), 0.0, 6, 3, [-30.0, 20.0, 45.0, -10.0]),
]
SWEEPS = 6


def make(name, shape, pol, adj, nl, per_class, seed):
    c = synth.small_case(seed=seed, shape=shape, pol=pol, adjacency=adj, nlabels=nl,
                         noise=120, contrast=400)
    img = c.image.astype(np.int32)
    img -= min(0, int(img.min()))
    pc = None if per_class is None else np.array(per_class, np.float32)
    lab_oift = O.ref_oift_multi(img, adj, c.seeds, c.seed_labels,
                                pol=None if pc is not None else pol, per_class=pc)
    lab_relax = O.ref_orelax_multi(img, adj, c.seeds, lab_oift, SWEEPS,
                                   pol=None if pc is not None else pol, per_class=pc)
    out = dict(image=img.reshape(shape), seeds=c.seeds, seed_labels=c.seed_labels,
               adjacency=np.int32(adj), pol=np.float32(pol), sweeps=np.int32(SWEEPS),
               per_class=pc if pc is not None else np.zeros(0, np.float32),
               ref_oift_label=lab_oift, ref_relax_label=lab_relax,
               ref_blur=O.ref_gaussian_blur(img))
    # the CLI steps: conditional dilation of the binary relaxed labels on the blurred image,
    # boundary seeds (stride 2), and the whole CLI chain on an image shifted below zero
    if nl == 1 and pc is None:
        out["ref_dilated_p50"] = O.ref_dilation_conditional(out["ref_blur"].reshape(img.shape),
                                                            lab_relax, 1.0, 50.0)
        chain_img = (img - 500).astype(np.int32)
        chain_lab = np.full(img.size, -1, np.int32)
        chain_lab[c.seeds] = c.seed_labels
        bl, bs = O.ref_inject_boundary_seeds(chain_lab, shape, 2, c.seeds)
        out["ref_boundary_label"], out["ref_boundary_seeds"] = bl, bs
        out["chain_image"] = chain_img.reshape(shape)
        out["ref_chain_label"] = O.ref_oiftrelax_chain(chain_img.reshape(shape), pol, SWEEPS,
                                                       50.0, c.seeds, chain_lab)
    # the gradient-blend experiment on the twice-blurred volume (6 / 4-adj, global polarity)
    if pc is None and adj in (6, 4):
        f = O.ref_gaussian_blur(O.ref_gaussian_blur(img).reshape(shape)).reshape(shape)
        g = O.ref_sobel_normalized(f)
        out["blend_image"] = f
        out["ref_sobel"] = g
        out["ref_blend_oift_label"] = O.ref_gradweight(f, g, 0.6, c.seeds, c.seed_labels, pol, 0)
        out["ref_blend_relax_label"] = O.ref_gradweight(f, g, 0.6, c.seeds, c.seed_labels, pol,
                                                        SWEEPS)
    # the 2D image-graph pipeline (gft_ift.cpp:9575-9682, 9785-9790): OIFT(sImageGraph) with
    # every labelled pixel as a seed, then ORelax_1(sImageGraph)
    if pc is None and adj in (4, 8):
        img2 = img.reshape(shape[1:])
        lab_ig, wmax = O.ref_imagegraph(img2, adj, c.seeds, c.seed_labels, pol, 0)
        out["ref_ig_oift_label"] = lab_ig
        out["ref_ig_wmax"] = np.int32(wmax)
        out["ref_ig_energy"] = np.int32(O.ref_imagegraph_energy(img2, adj, lab_ig, pol, 1))
        out["ref_ig_relax_label"] = O.ref_imagegraph(img2, adj, c.seeds, c.seed_labels, pol,
                                                     SWEEPS)[0]
    # the coarse-to-fine cascade on the twice-blurred volume (global polarity cases)
    if pc is None and adj in (6, 26):
        f = O.ref_gaussian_blur(O.ref_gaussian_blur(img).reshape(shape)).reshape(shape)
        lab0 = np.full(img.size, -1, np.int32)
        lab0[c.seeds] = c.seed_labels
        out["c2f_image"] = f
        out["ref_c2f_label"] = O.ref_coarse_to_fine(f, adj, pol, SWEEPS, 50.0, c.seeds, lab0)
    if pol == 0.0 and pc is None:
        cost, lab = O.ref_ift_fmax(img, adj, c.seeds, c.seed_labels)
        out["ref_ift_fmax_cost"] = cost
        out["ref_ift_fmax_label"] = lab
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def main():
    O.build(with_ref=True)
    for i, (name, shape, pol, adj, nl, pc) in enumerate(CASES):
        make(name, shape, pol, adj, nl, pc, seed=100 + i)
        print("wrote", name)


if __name__ == "__main__":
    main()
