"""TEST INFRASTRUCTURE ONLY: ctypes access to the C restatement (liboracle.so) and to
the reference gft library compiled from its own sources (_ref/libgft_ref.so).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference
legs may import this package, and only as the checker or the timed reference arm.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgft_ref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "liboift_fmax_ref.so")
# the reference source tree (jung0221/roift), where a build of the checker libraries may read
# it; unset where only the prebuilt libraries in oracle/_ref are present
REF_SRC = os.environ.get("ROIFT_REFERENCE")

NIL = -1
W_MODES = {"grad": 0, "grad_q": 1, "rbf_q": 2, "blend_q": 3}

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def ref_tree_present() -> bool:
    return bool(REF_SRC) and os.path.isdir(REF_SRC)


def build(with_ref: bool | None = None) -> None:
    """Compile liboracle.so and, when the reference tree is present (ROIFT_REFERENCE),
    libgft_ref.so, the reference's plain-GPU library and the drop-in CLI programs."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if with_ref is None:
        with_ref = ref_tree_present()
    if with_ref and ref_tree_present():
        ref = [f"REF={REF_SRC}"]
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", *ref], check=True)
        if os.path.exists("/usr/local/cuda/bin/nvcc"):
            subprocess.run(["make", "-s", "-C", HERE, "refgpu", *ref], check=True)
        pkg = os.path.join(HERE, "..", "roift_b200")
        if os.path.exists(os.path.join(pkg, "libgft_oift_b200.so")):
            subprocess.run(["make", "-s", "-j8", "-C", HERE, "dropin", *ref], check=True)


def dropin_programs():
    """The reference's CLIs built against the product (oracle/Makefile `dropin`), or None."""
    a = os.path.join(HERE, "_ref", "oiftrelax_gft_dropin")
    b = os.path.join(HERE, "_ref", "oiftrelax_fmax_gpu_dropin")
    return (a, b) if os.path.exists(a) and os.path.exists(b) else None


class _Polarity(C.Structure):
    _fields_ = [("table", C.POINTER(C.c_float)), ("ntable", C.c_int), ("dflt", C.c_float)]


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        L = C.CDLL(ORACLE_SO)
        L.or_build_weights.restype = C.c_longlong
        L.or_build_weights.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_float,
                                       _u16p]
        L.or_rbf_lut.argtypes = [C.c_double, C.c_int, C.c_int, _u16p]
        L.or_oift_fmax.restype = C.c_int
        L.or_oift_fmax.argtypes = [_u16p, C.c_int, C.c_int, C.c_int, C.c_int, _Polarity,
                                   _i32p, C.c_int, _i32p, _i32p, _i32p, C.c_void_p]
        L.or_oift_prim.argtypes = [_u16p, C.c_int, C.c_int, C.c_int, C.c_int, _Polarity,
                                   C.c_int, _i32p, C.c_int, _i32p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
        L.or_energy.restype = C.c_int
        L.or_energy.argtypes = [_u16p, C.c_int, C.c_int, C.c_int, C.c_int, _Polarity, _i32p,
                                C.c_int, _i32p]
        L.or_tie_stats.restype = None
        L.or_tie_stats.argtypes = [_u16p, C.c_int, C.c_int, C.c_int, C.c_int, _Polarity, _i32p,
                                   _i32p, _i32p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.or_relax_f32.restype = C.c_int
        L.or_relax_f32.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                   C.c_void_p, C.c_int, _i32p, C.c_int, _i32p, C.c_int,
                                   C.c_void_p]
        L.or_relax_f64.restype = C.c_int
        L.or_relax_f64.argtypes = L.or_relax_f32.argtypes
        L.or_gaussian_blur.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, _i32p]
        L.or_sobel_normalized.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, _i32p]
        L.or_oift_fmax_blend.restype = C.c_int
        L.or_oift_fmax_blend.argtypes = [_i32p, _i32p, C.c_float, C.c_int, C.c_int, C.c_int,
                                         C.c_int, _Polarity, _i32p, C.c_int, _i32p, _i32p, _i32p]
        L.or_oift_prim_blend.argtypes = [_i32p, _i32p, C.c_float, C.c_int, C.c_int, C.c_int,
                                         C.c_int, _Polarity, C.c_int, _i32p, C.c_int, _i32p]
        L.or_relax_blend_f32.restype = C.c_int
        L.or_relax_blend_f32.argtypes = [_i32p, _i32p, C.c_float, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_float, _i32p, C.c_int, _i32p, C.c_int,
                                         C.c_void_p]
        L.or_oift_fmax_imagegraph.restype = C.c_int
        L.or_oift_fmax_imagegraph.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, _Polarity,
                                              _i32p, C.c_int, _i32p, _i32p, _i32p, C.c_void_p]
        L.or_oift_prim_imagegraph.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, _Polarity,
                                              C.c_int, _i32p, C.c_int, _i32p, C.c_void_p,
                                              C.c_void_p, C.c_void_p]
        L.or_imagegraph_wmax.restype = C.c_int
        L.or_imagegraph_wmax.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_float]
        L.or_energy_imagegraph.restype = C.c_int
        L.or_energy_imagegraph.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_float, _i32p,
                                           C.c_int]
        L.or_relax_imagegraph_f32.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_float,
                                              _i32p, C.c_int, _i32p, C.c_int, C.c_void_p]
        L.or_adjacency.restype = C.c_int
        L.or_adjacency.argtypes = [C.c_int, _i32p, _i32p, _i32p]
        L.or_conditional_dilation.restype = C.c_longlong
        L.or_conditional_dilation.argtypes = [_i32p, _i32p, C.c_int, C.c_int, C.c_int,
                                              C.c_float, C.c_float]
        L.or_inject_boundary_seeds.restype = C.c_int
        L.or_inject_boundary_seeds.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                               _i32p, C.c_int]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(REF_SO)
        R.ref_oift_multi.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                     _i32p, C.c_int, _i32p]
        R.ref_oift_multi_perclass.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                              _f32p, C.c_int, _i32p, C.c_int, _i32p]
        R.ref_orelax_multi.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                       _i32p, C.c_int, _i32p, C.c_int]
        R.ref_orelax_multi_perclass.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                _f32p, C.c_int, _i32p, C.c_int, _i32p, C.c_int]
        R.ref_ift_fmax_graph.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int, _i32p,
                                         C.c_int, _i32p, _i32p]
        R.ref_energy_min_graph.restype = C.c_int
        R.ref_energy_min_graph.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int, _i32p,
                                           C.c_int]
        R.ref_gaussian_blur.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, _i32p]
        R.ref_dilation_conditional.argtypes = [_i32p, _i32p, C.c_int, C.c_int, C.c_int,
                                               C.c_float, C.c_float]
        R.ref_inject_boundary_seeds.restype = C.c_int
        R.ref_inject_boundary_seeds.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                _i32p, C.c_int, _i32p, C.c_int]
        R.ref_sobel_normalized.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, _i32p]
        R.ref_gradweight.argtypes = [_i32p, _i32p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                     _i32p, C.c_int, _i32p, C.c_int]
        R.ref_imagegraph.restype = C.c_int
        R.ref_imagegraph.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_float, _i32p, C.c_int,
                                     _i32p, C.c_int]
        R.ref_imagegraph_energy.restype = C.c_int
        R.ref_imagegraph_energy.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_float, _i32p,
                                            C.c_int]
        R.ref_read_volume.restype = C.c_int
        R.ref_read_volume.argtypes = [C.c_char_p, C.c_void_p, C.c_int, _i32p, _f32p]
        R.ref_write_volume.argtypes = [C.c_char_p, _i32p, _i32p, _f32p]
        R.ref_coarse_to_fine.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                         C.c_int, C.c_float, _i32p, C.c_int, _i32p]
        R.ref_oiftrelax_chain.argtypes = [_i32p, C.c_int, C.c_int, C.c_int, C.c_double,
                                          C.c_int, C.c_float, _i32p, C.c_int, _i32p]
        _ref = R
    return _ref


# ------------------------------------------------------------------ helpers ----
def _dims(img):
    if img.ndim == 2:
        return img.shape[1], img.shape[0], 1
    Z, Y, X = img.shape
    return X, Y, Z


def as_i32(img) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(img).reshape(-1), dtype=np.int32)


def polarity(pol: float | None = None, per_class=None):
    """Global mode: label 0 -> -per, others +per (gft_ift.cpp:968).  Per-class mode:
    per_class[l] for l <= max_label, else 0 (gft_ift.cpp:1055-1060).  Values x100."""
    if per_class is None:
        per = np.float32(pol * 100.0) if not isinstance(pol, np.float32) else pol
        table = np.array([-per], np.float32)
        keep = table
        return _Polarity(table.ctypes.data_as(C.POINTER(C.c_float)), 1, C.c_float(per)), keep
    table = np.ascontiguousarray(per_class, np.float32)
    return _Polarity(table.ctypes.data_as(C.POINTER(C.c_float)), len(table), 0.0), table


def n_planes(adj: int) -> int:
    return 13 if adj in (8, 26) else 3


def build_weights(img, adj, mode="grad", wq=4095, rbf_sigma=150.0, grad=None, blend_a=0.5):
    X, Y, Z = _dims(img)
    flat = as_i32(img)
    N = flat.size
    W = np.zeros(n_planes(adj) * N, np.uint16)
    lut = None
    lut_len = 0
    if mode == "rbf_q":
        lut_len = int(np.abs(np.diff(np.sort(flat)[[0, -1]]))[0]) + 1 if N > 1 else 1
        lut = np.zeros(lut_len, np.uint16)
        lib().or_rbf_lut(float(rbf_sigma), int(wq), lut_len, lut)
    g = as_i32(grad) if grad is not None else None
    ncl = lib().or_build_weights(flat, X, Y, Z, adj, W_MODES[mode], int(wq),
                                 lut.ctypes.data if lut is not None else None, lut_len,
                                 g.ctypes.data if g is not None else None, float(blend_a), W)
    return W, int(ncl)


def oift_fmax(W, shape_xyz, adj, seeds, seed_labels, pol=None, per_class=None, want_pred=False):
    """R2.  Returns (cost, label, levels[, pred])."""
    X, Y, Z = shape_xyz
    N = X * Y * Z
    lab_in = np.full(N, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab_in[seeds] = seed_labels
    cost = np.empty(N, np.int32)
    label = np.empty(N, np.int32)
    pred = np.empty(N, np.int32) if want_pred else None
    P, keep = polarity(pol, per_class)
    levels = lib().or_oift_fmax(W, X, Y, Z, adj, P, seeds, len(seeds), lab_in, cost, label,
                                pred.ctypes.data if pred is not None else None)
    return (cost, label, levels, pred) if want_pred else (cost, label, levels)


def _offsets(adj):
    """Neighbour offsets of Spheric(1.0) (4 / 6) or Spheric(1.75) (8 / 26) without the
    centre (gft_adjrel3.cpp:47-85); z offsets only in 3D."""
    r2 = 3 if adj in (8, 26) else 1
    out = []
    for dz in ((0,) if adj in (4, 8) else (-1, 0, 1)):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if (dx, dy, dz) != (0, 0, 0) and dx * dx + dy * dy + dz * dz <= r2:
                    out.append((dx, dy, dz))
    return out


def oift_fmax_wide(img, adj, seeds, seed_labels, pol=None, per_class=None):
    """R2 for exact weights of any width: the lexicographic (cost, label) Dijkstra of the
    f_max path cost in which a seed keeps its label (its key lies below every offer) and
    the arc p -> q weighs |I_p - I_q| oriented by the tail's label,
    (int)(w * (1 +/- per/100.0)) in double as gft/src/gft_ift.cpp:965-973 evaluates it, with
    no 14-bit edge code in between.  A pure-Python heap loop: small volumes only.
    Returns (cost, label) with cost 0 at the seeds."""
    import heapq
    X, Y, Z = _dims(img)
    I = [int(v) for v in as_i32(img)]
    N = X * Y * Z
    if per_class is None:
        per = float(np.float32(pol * 100.0))
        table, dflt = [-per], per
    else:
        table, dflt = [float(v) for v in np.asarray(per_class, np.float32)], 0.0
    pol_of = lambda l: table[l] if l < len(table) else dflt
    offs = _offsets(adj)
    INF = (1 << 62, 1 << 62)
    key = [INF] * N
    for s, l in zip(np.asarray(seeds).tolist(), np.asarray(seed_labels).tolist()):
        k = (0, max(int(l), 0))
        if k < key[s]:
            key[s] = k
    heap = [(key[p][0], key[p][1], p) for p in set(np.asarray(seeds).tolist())]
    heapq.heapify(heap)
    done = [False] * N
    while heap:
        f, l, p = heapq.heappop(heap)
        if done[p] or (f, l) != key[p]:
            continue
        done[p] = True
        c = f - 1 if f > 0 else 0
        fgt, flt = 1.0 + pol_of(l) / 100.0, 1.0 - pol_of(l) / 100.0
        x, y, z = p % X, (p // X) % Y, p // (X * Y)
        for dx, dy, dz in offs:
            qx, qy, qz = x + dx, y + dy, z + dz
            if not (0 <= qx < X and 0 <= qy < Y and 0 <= qz < Z):
                continue
            q = qx + qy * X + qz * X * Y
            if done[q]:
                continue
            d = I[p] - I[q]
            b = abs(d)
            w = int(b * fgt) if d > 0 else (int(b * flt) if d < 0 else b)
            k = (max(c, w) + 1, l)
            if k < key[q]:
                key[q] = k
                heapq.heappush(heap, (k[0], k[1], q))
    cost = np.array([k[0] - 1 if 0 < k[0] < (1 << 62) else 0 for k in key], np.int64)
    label = np.array([k[1] if k[0] < (1 << 62) else NIL for k in key], np.int32)
    return cost, label


def energy_wide(img, adj, label, pol=None, per_class=None):
    """Oriented cut energy (gft_ift.cpp:287-319, as or_energy): the smallest weight of an
    arc p -> q with label[q] != label[p], oriented by the polarity of label[p], with exact
    weights of any width."""
    X, Y, Z = _dims(img)
    I = as_i32(img).astype(np.int64).reshape(Z, Y, X)
    lab = np.asarray(label).reshape(Z, Y, X)
    if per_class is None:
        per = float(np.float32(pol * 100.0))
        table, dflt = np.array([-per]), per
    else:
        table, dflt = np.asarray(per_class, np.float64), 0.0
    pl = np.where((lab >= 0) & (lab < len(table)), table[np.clip(lab, 0, len(table) - 1)], dflt)
    e = None
    for dx, dy, dz in _offsets(adj):
        sl_p = tuple(slice(max(0, -o), n - max(0, o)) for o, n in ((dz, Z), (dy, Y), (dx, X)))
        sl_q = tuple(slice(max(0, o), n - max(0, -o)) for o, n in ((dz, Z), (dy, Y), (dx, X)))
        d = I[sl_p] - I[sl_q]
        b = np.abs(d).astype(np.float64)
        f = pl[sl_p] / 100.0
        w = np.where(d > 0, np.trunc(b * (1.0 + f)), np.where(d < 0, np.trunc(b * (1.0 - f)), b))
        m = lab[sl_p] != lab[sl_q]
        if m.any():
            v = int(w[m].min())
            e = v if e is None else min(e, v)
    return e


def oift_prim(W, shape_xyz, adj, seeds, seed_labels, pol=None, per_class=None):
    """R1 (restated OIFT_Multi).  Returns (label, value, pred, fmax)."""
    X, Y, Z = shape_xyz
    N = X * Y * Z
    lab = np.full(N, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab[seeds] = seed_labels
    val = np.empty(N, np.int32)
    pred = np.empty(N, np.int32)
    fmax = np.empty(N, np.int32)
    P, keep = polarity(pol, per_class)
    maxw = int((W & 0x3FFF).max()) if W.size else 0
    maxp = 100.0 if per_class is None else float(np.abs(per_class).max())
    buckets = int(maxw * (1.0 + max(abs(pol or 0) * 100, maxp) / 100.0)) + 2
    lib().or_oift_prim(W, X, Y, Z, adj, P, buckets, seeds, len(seeds), lab,
                       val.ctypes.data, pred.ctypes.data, fmax.ctypes.data)
    return lab, val, pred, fmax


def energy(W, shape_xyz, adj, label, nl, pol=None, per_class=None):
    X, Y, Z = shape_xyz
    e_lb = np.empty(max(nl, 1), np.int32)
    P, keep = polarity(pol, per_class)
    e = lib().or_energy(W, X, Y, Z, adj, P, np.ascontiguousarray(label, np.int32), nl, e_lb)
    return e, e_lb[:nl]


def tie_stats(W, shape_xyz, adj, cost, lab_a, lab_b, seeds, pol=None, per_class=None,
              want_flags=False):
    """Equal-cost tie accounting of labelling A (R2 / the CUDA result) against labelling B
    (the reference Prim forest) over the cost map `cost`.  Returns a dict with
    ties (voxels offered their cost by two labels in A), diffs, explained (differences
    where both labels reach the voxel at its cost) and unexplained; flags per voxel when
    asked (bit 0 tie, bit 1 differs, bit 2 explained)."""
    X, Y, Z = shape_xyz
    N = X * Y * Z
    is_seed = np.zeros(N, np.uint8)
    is_seed[np.asarray(seeds, np.int64)] = 1
    out = np.zeros(4, np.int64)
    flags = np.zeros(N, np.uint8) if want_flags else None
    P, keep = polarity(pol, per_class)
    lib().or_tie_stats(W, X, Y, Z, adj, P, np.ascontiguousarray(cost, np.int32).reshape(-1),
                       np.ascontiguousarray(lab_a, np.int32).reshape(-1),
                       np.ascontiguousarray(lab_b, np.int32).reshape(-1),
                       is_seed.ctypes.data, out.ctypes.data,
                       flags.ctypes.data if flags is not None else None)
    d = {"ties": int(out[0]), "diffs": int(out[1]), "explained": int(out[2]),
         "unexplained": int(out[3])}
    if want_flags:
        d["flags"] = flags
    return d


def relax(img, adj, seeds, label, ntimes, pol=None, per_class=None, fp64=False):
    """R3.  Returns (label_out, membership [C, N], nclasses)."""
    X, Y, Z = _dims(img)
    flat = as_i32(img)
    N = flat.size
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab = np.ascontiguousarray(label, np.int32).copy()
    # class count first (membership size)
    present = {0} | {int(l) for l in lab[seeds] if l >= 0}
    nc = len(present)
    mem = np.empty(nc * N, np.float64 if fp64 else np.float32)
    pc = None
    ml = 0
    if per_class is not None:
        pc = np.ascontiguousarray(per_class, np.float32)
        ml = len(pc) - 1
    fn = lib().or_relax_f64 if fp64 else lib().or_relax_f32
    got = fn(flat, X, Y, Z, adj, float(np.float32((pol or 0.0) * 100.0)),
             pc.ctypes.data if pc is not None else None, ml, seeds, len(seeds), lab, int(ntimes),
             mem.ctypes.data)
    assert got == nc, (got, nc)
    return lab, mem.reshape(nc, N), nc


def conditional_dilation(img, label, radius=1.0, percentile=50.0):
    """R-restatement of oiftrelax.cpp:87-169 on copies: (label after, voxels added)."""
    X, Y, Z = _dims(img)
    lab = np.ascontiguousarray(label, np.int32).reshape(-1).copy()
    n = lib().or_conditional_dilation(as_i32(img), lab, X, Y, Z, radius, percentile)
    return lab, n


def inject_boundary_seeds(label, shape_zyx, stride):
    """Restatement of oiftrelax.cpp:175-224: (label after, new seeds)."""
    Z, Y, X = shape_zyx
    lab = np.ascontiguousarray(label, np.int32).reshape(-1).copy()
    out = np.empty(X * Y * Z, np.int32)
    n = lib().or_inject_boundary_seeds(lab, X, Y, Z, stride, out, len(out))
    return lab, out[:n].copy()


def oiftrelax_chain(img, pol, niter, percentile, seeds, seed_labels, oift="r2", blur=2):
    """The CLI chain restated (oiftrelax.cpp main 263-268, 368-414): shift to >= 0, `blur`
    Gaussian blurs, exact-gradient OIFT (R2, or R1 = OIFT_Multi's Prim order), R3-FP32
    relaxation with niter sweeps, conditional dilation (Spheric(1)) when binary.
    Returns (label, blurred image)."""
    shape = img.shape
    X, Y, Z = _dims(img)
    b = np.asarray(img, np.int64)
    b = (b - min(0, int(b.min()))).astype(np.int32)
    for _ in range(blur):
        b = gaussian_blur(b.reshape(shape)).reshape(shape)
    W, _ = build_weights(b, 6 if Z > 1 else 4, "grad")
    adj = 6 if Z > 1 else 4
    if oift == "r2":
        _, lab, _ = oift_fmax(W, (X, Y, Z), adj, seeds, seed_labels, pol=pol)
    else:
        lab = oift_prim(W, (X, Y, Z), adj, seeds, seed_labels, pol=pol)[0]
    out, _, _ = relax(b, adj, seeds, lab, niter, pol=pol)
    if out.max() <= 1:
        out, _ = conditional_dilation(b, out, 1.0, percentile)
    return out, b


def coarse_size(n):
    """Scene32::Subsampling extent (gft_filtering3.cpp:449-455): n/2 + n%2, made odd."""
    c = n // 2 + n % 2
    return c + 1 if c % 2 == 0 else c


def subsample(fscn):
    """Scene32::Subsampling (gft_filtering3.cpp:445-476): coarse voxel v takes the fine
    voxel (v - c/2) * 2 + n/2 (integer halves) when inside, else 0."""
    Z, Y, X = fscn.shape
    cz, cy, cx = coarse_size(Z), coarse_size(Y), coarse_size(X)
    out = np.zeros((cz, cy, cx), np.int32)
    ux = (np.arange(cx) - cx // 2) * 2 + X // 2
    uy = (np.arange(cy) - cy // 2) * 2 + Y // 2
    uz = (np.arange(cz) - cz // 2) * 2 + Z // 2
    vx, vy, vz = (ux >= 0) & (ux < X), (uy >= 0) & (uy < Y), (uz >= 0) & (uz < Z)
    out[np.ix_(vz, vy, vx)] = fscn[np.ix_(uz[vz], uy[vy], ux[vx])]
    return out


def scale_label_nn(lab_c, coarse_shape, fine_shape):
    """Scene32::ScaleLabel(..., none) = Scale nearest (gft_scene32.cpp:1091-1120,
    1240-1262): x = (u - n/2.) * 0.5 + c/2. in double stored as float, index
    (int)(x + 0.5) truncated toward zero, clamped to the coarse extent."""
    def axis(n, c):
        u = np.arange(n, dtype=np.float64)
        x = ((u - n / 2.0) * np.float64(np.float32(0.5)) + c / 2.0).astype(np.float32)
        i = np.trunc(x.astype(np.float64) + 0.5).astype(np.int64)
        return np.clip(i, 0, c - 1)
    (Z, Y, X), (cz, cy, cx) = fine_shape, coarse_shape
    lc = lab_c.reshape(coarse_shape)
    return lc[np.ix_(axis(Z, cz), axis(Y, cy), axis(X, cx))].reshape(-1)


def mark_boundary_nil(label, shape, adj):
    """Labelled voxels with a neighbour (adjacency without the centre) of another value,
    NIL included, become NIL (exp_coarse_to_fine.cpp:216-249)."""
    Z, Y, X = shape
    lab = label.reshape(shape)
    dx, dy, dz = (np.zeros(26, np.int32) for _ in range(3))
    n = lib().or_adjacency(adj, dx, dy, dz)
    pad = np.pad(lab, 1, constant_values=-2)  # -2: outside the volume
    bnd = np.zeros(shape, bool)
    for i in range(n):
        sz, sy, sx = int(dz[i]), int(dy[i]), int(dx[i])
        nb = pad[1 + sz:1 + sz + Z, 1 + sy:1 + sy + Y, 1 + sx:1 + sx + X]
        bnd |= (nb != -2) & (nb != lab)
    out = lab.copy()
    out[bnd & (lab != NIL)] = NIL
    return out.reshape(-1)


def coarse_to_fine(fscn, adj, pol, niter, percentile, seeds, label, mode="grad", wq=4095,
                   rbf_sigma=150.0, oift="r2"):
    """The two-level cascade (exp_coarse_to_fine.cpp:327-414) restated on the blurred,
    shifted volume with the oracle's OIFT (R2, or R1 = OIFT_Multi's order) and R3-FP32
    relaxation.  label: seed labels (NIL elsewhere).  Returns the label map."""
    shape = fscn.shape
    Z, Y, X = shape
    lab = np.ascontiguousarray(label, np.int32).reshape(-1).copy()
    coarse = subsample(fscn)
    cshape = coarse.shape
    cz, cy, cx = cshape
    lab_c = np.full(coarse.size, NIL, np.int32)
    cs = []
    for pp in np.asarray(seeds, np.int64):
        x, y, z = int(pp % X), int((pp // X) % Y), int(pp // (X * Y))
        q = x // 2 + (y // 2) * cx + (z // 2) * cx * cy
        if x // 2 < cx and y // 2 < cy and z // 2 < cz and lab_c[q] == NIL:
            lab_c[q] = lab[pp]
            cs.append(q)
    cs = np.array(cs, np.int32)

    def solve(img, sd, lab_in):
        X_, Y_, Z_ = img.shape[2], img.shape[1], img.shape[0]
        W, _ = build_weights(img, adj, mode, wq=wq, rbf_sigma=rbf_sigma)
        sl = lab_in[sd]
        if oift == "r2":
            _, lo, _ = oift_fmax(W, (X_, Y_, Z_), adj, sd, sl, pol=pol)
        else:
            lo = oift_prim(W, (X_, Y_, Z_), adj, sd, sl, pol=pol)[0]
        out, _, _ = relax(img, adj, sd, lo, niter, pol=pol)
        return out

    lab_c = solve(coarse, cs, lab_c)
    up = mark_boundary_nil(scale_label_nn(lab_c, cshape, shape), shape, adj)
    merged = np.where((up != NIL) & (lab == NIL), up, lab).astype(np.int32)
    fs = np.nonzero(merged != NIL)[0].astype(np.int32)
    out = solve(fscn, fs, merged)
    if out.max() <= 1:
        out, _ = conditional_dilation(fscn, out, 1.0, percentile)
    return out


def sobel_normalized(img):
    """Scene32::SobelFilter normalised to the image maximum (exp_gradient_weight.cpp)."""
    X, Y, Z = _dims(img)
    out = np.empty(X * Y * Z, np.int32)
    lib().or_sobel_normalized(as_i32(img), X, Y, Z, out)
    return out


def oift_fmax_blend(img, g, alpha, adj, seeds, seed_labels, pol=None):
    """R2 with the blend weights of OIFT_Multi_GradWeight: (cost, label, levels)."""
    X, Y, Z = _dims(img)
    N = X * Y * Z
    lab_in = np.full(N, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab_in[seeds] = seed_labels
    cost = np.empty(N, np.int32)
    label = np.empty(N, np.int32)
    P, keep = polarity(pol)
    levels = lib().or_oift_fmax_blend(as_i32(img), as_i32(g), float(alpha), X, Y, Z, adj, P,
                                      seeds, len(seeds), lab_in, cost, label)
    return cost, label, levels


def oift_prim_blend(img, g, alpha, adj, seeds, seed_labels, pol=None):
    """R1 with the blend weights (OIFT_Multi_GradWeight's Prim / FIFO order): labels."""
    X, Y, Z = _dims(img)
    N = X * Y * Z
    lab = np.full(N, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab[seeds] = seed_labels
    P, keep = polarity(pol)
    gi = as_i32(g)
    wmax = int(max(as_i32(img).max(), gi.max()) * 2) + 2
    lib().or_oift_prim_blend(as_i32(img), gi, float(alpha), X, Y, Z, adj, P, wmax, seeds,
                             len(seeds), lab)
    return lab


def relax_blend(img, g, alpha, adj, seeds, label, ntimes, pol):
    """ORelax_1_Multi_GradWeight restated in FP32: (labels, membership [C, N])."""
    X, Y, Z = _dims(img)
    flat = as_i32(img)
    N = flat.size
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab = np.ascontiguousarray(label, np.int32).copy()
    nc = len({0} | {int(l) for l in lab[seeds] if l >= 0})
    mem = np.empty(nc * N, np.float32)
    got = lib().or_relax_blend_f32(flat, as_i32(g), float(alpha), X, Y, Z, adj,
                                   float(np.float32((pol or 0.0) * 100.0)), seeds, len(seeds),
                                   lab, int(ntimes), mem.ctypes.data)
    assert got == nc
    return lab, mem.reshape(nc, N)


def _ig_dims(img):
    X, Y, Z = _dims(img)
    assert Z == 1, "the image graph is 2D"
    return X, Y


def imagegraph_wmax(img, adj, pol):
    """sg->Wmax of Orient2Digraph on ByEuclideanDistance(img, r) (4: r = 1, 8: r = 1.5)."""
    X, Y = _ig_dims(img)
    return int(lib().or_imagegraph_wmax(as_i32(img), X, Y, adj, float(np.float32(pol * 100.0))))


def oift_fmax_imagegraph(img, adj, seeds, seed_labels, pol, want_pred=False):
    """R2 with the oriented image-graph weights: (cost, label, levels[, pred])."""
    X, Y = _ig_dims(img)
    N = X * Y
    lab_in = np.full(N, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab_in[seeds] = seed_labels
    cost = np.empty(N, np.int32)
    label = np.empty(N, np.int32)
    pred = np.empty(N, np.int32) if want_pred else None
    P, keep = polarity(pol)
    levels = lib().or_oift_fmax_imagegraph(as_i32(img), X, Y, adj, P, seeds, len(seeds), lab_in,
                                           cost, label,
                                           pred.ctypes.data if pred is not None else None)
    return (cost, label, levels, pred) if want_pred else (cost, label, levels)


def oift_prim_imagegraph(img, adj, seeds, seed_labels, pol):
    """R1 on the oriented image graph (OIFT(sImageGraph), seeds queued in the given order):
    (label, value, pred, fmax)."""
    X, Y = _ig_dims(img)
    N = X * Y
    lab = np.full(N, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab[seeds] = seed_labels
    val, pred, fmax = (np.empty(N, np.int32) for _ in range(3))
    P, keep = polarity(pol)
    lib().or_oift_prim_imagegraph(as_i32(img), X, Y, adj, P, imagegraph_wmax(img, adj, pol),
                                  seeds, len(seeds), lab, val.ctypes.data, pred.ctypes.data,
                                  fmax.ctypes.data)
    return lab, val, pred, fmax


def energy_imagegraph(img, adj, label, pol, lb=1):
    """GetEnergy_Min(sImageGraph) restated: the cut energy of label lb."""
    X, Y = _ig_dims(img)
    return int(lib().or_energy_imagegraph(as_i32(img), X, Y, adj, float(np.float32(pol * 100.0)),
                                          np.ascontiguousarray(label, np.int32).reshape(-1), lb))


def relax_imagegraph(img, adj, seeds, label, ntimes, pol):
    """ORelax_1(sImageGraph) restated in FP32: (binary labels, memberships [N])."""
    X, Y = _ig_dims(img)
    lab = np.ascontiguousarray(label, np.int32).reshape(-1).copy()
    seeds = np.ascontiguousarray(seeds, np.int32)
    m = np.empty(X * Y, np.float32)
    lib().or_relax_imagegraph_f32(as_i32(img), X, Y, adj, float(np.float32(pol * 100.0)), seeds,
                                  len(seeds), lab, int(ntimes), m.ctypes.data)
    return lab, m


def gaussian_blur(img):
    X, Y, Z = _dims(img)
    out = np.empty(X * Y * Z, np.int32)
    lib().or_gaussian_blur(as_i32(img), X, Y, Z, out)
    return out


# ------------------------------------------------------- reference wrappers ----
def ref_oift_multi(img, adj, seeds, seed_labels, pol=None, per_class=None):
    X, Y, Z = _dims(img)
    N = X * Y * Z
    lab = np.full(N, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab[seeds] = seed_labels
    if per_class is None:
        ref().ref_oift_multi(as_i32(img), X, Y, Z, adj, np.float32(pol * 100.0), seeds,
                             len(seeds), lab)
    else:
        pc = np.ascontiguousarray(per_class, np.float32)
        ref().ref_oift_multi_perclass(as_i32(img), X, Y, Z, adj, pc, len(pc) - 1, seeds,
                                      len(seeds), lab)
    return lab


def ref_orelax_multi(img, adj, seeds, label, ntimes, pol=None, per_class=None):
    X, Y, Z = _dims(img)
    lab = np.ascontiguousarray(label, np.int32).copy()
    seeds = np.ascontiguousarray(seeds, np.int32)
    if per_class is None:
        ref().ref_orelax_multi(as_i32(img), X, Y, Z, adj, np.float32(pol * 100.0), seeds,
                               len(seeds), lab, int(ntimes))
    else:
        pc = np.ascontiguousarray(per_class, np.float32)
        ref().ref_orelax_multi_perclass(as_i32(img), X, Y, Z, adj, pc, len(pc) - 1, seeds,
                                        len(seeds), lab, int(ntimes))
    return lab


def ref_ift_fmax(img, adj, seeds, seed_labels):
    X, Y, Z = _dims(img)
    N = X * Y * Z
    lab = np.full(N, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab[seeds] = seed_labels
    cost = np.empty(N, np.int32)
    ref().ref_ift_fmax_graph(as_i32(img), X, Y, Z, adj, seeds, len(seeds), lab, cost)
    return cost, lab


def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_SO)


def ref_oift_fmax_gpu_run(img, seeds, seed_labels, per_class):
    """The reference's own plain-GPU f_max OIFT (gpu/oift_fmax_gpu.cu:139-259) compiled for
    sm_100a.  Returns (labels, waves).  Its labels depend on arrival order."""
    L = C.CDLL(REF_GPU_SO)
    L.oift_fmax_gpu_run.argtypes = [_i32p, _i32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p,
                                    C.c_int, _i32p, C.c_int]
    X, Y, Z = _dims(img)
    N = X * Y * Z
    lab = np.full(N, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab[seeds] = seed_labels
    pc = np.ascontiguousarray(per_class, np.float32)
    im = as_i32(img)
    # the reference prints its wave progress on stdout; keep it off the caller's stdout
    import sys
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    try:
        os.dup2(devnull, 1)
        waves = L.oift_fmax_gpu_run(im, lab, N, X, Y, Z, pc, len(pc) - 1, seeds, len(seeds))
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    return lab, waves


def ref_dilation_conditional(img, label, radius=1.0, percentile=50.0):
    """Reference dilation_conditional (oiftrelax.cpp:149-165) on copies; returns the label."""
    X, Y, Z = _dims(img)
    lab = np.ascontiguousarray(label, np.int32).reshape(-1).copy()
    ref().ref_dilation_conditional(as_i32(img), lab, X, Y, Z, radius, percentile)
    return lab


def ref_inject_boundary_seeds(label, shape_zyx, stride, seeds):
    """Reference inject_boundary_seeds: (label after, seeds after)."""
    Z, Y, X = shape_zyx
    lab = np.ascontiguousarray(label, np.int32).reshape(-1).copy()
    sd = np.ascontiguousarray(seeds, np.int32)
    out = np.empty(len(sd) + X * Y * Z, np.int32)
    n = ref().ref_inject_boundary_seeds(lab, X, Y, Z, stride, sd, len(sd), out, len(out))
    return lab, out[:n].copy()


def ref_oiftrelax_chain(img, pol, niter, percentile, seeds, label):
    """The reference CLI chain (shift, blur x2, OIFT_Multi, ORelax_1_Multi, dilation)."""
    X, Y, Z = _dims(img)
    lab = np.ascontiguousarray(label, np.int32).reshape(-1).copy()
    ref().ref_oiftrelax_chain(as_i32(img), X, Y, Z, float(pol), int(niter), float(percentile),
                              np.ascontiguousarray(seeds, np.int32), len(seeds), lab)
    return lab


def ref_coarse_to_fine(fscn, adj, pol, niter, percentile, seeds, label):
    """The reference coarse-to-fine cascade (experiments/exp_coarse_to_fine.cpp:327-414) on
    the blurred, shifted volume; label holds the seed labels.  Returns the label map."""
    X, Y, Z = _dims(fscn)
    lab = np.ascontiguousarray(label, np.int32).reshape(-1).copy()
    ref().ref_coarse_to_fine(as_i32(fscn), X, Y, Z, adj, float(pol), int(niter),
                             float(percentile), np.ascontiguousarray(seeds, np.int32),
                             len(seeds), lab)
    return lab


def ref_sobel_normalized(img):
    X, Y, Z = _dims(img)
    out = np.empty(X * Y * Z, np.int32)
    ref().ref_sobel_normalized(as_i32(img), X, Y, Z, out)
    return out


def ref_gradweight(img, g, alpha, seeds, seed_labels, pol, ntimes):
    """Reference OIFT_Multi_GradWeight (+ ORelax_1_Multi_GradWeight when ntimes > 0)."""
    X, Y, Z = _dims(img)
    lab = np.full(X * Y * Z, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab[seeds] = seed_labels
    ref().ref_gradweight(as_i32(img), as_i32(g), X, Y, Z, float(np.float32(pol * 100.0)),
                         float(alpha), seeds, len(seeds), lab, int(ntimes))
    return lab


def ref_imagegraph(img, adj, seeds, seed_labels, pol, ntimes=0):
    """The reference 2D pipeline: ByEuclideanDistance + Orient2Digraph, OIFT(sImageGraph)
    with every labelled pixel as a seed, ORelax_1(sImageGraph) when ntimes > 0:
    (labels, Wmax)."""
    X, Y = _ig_dims(img)
    lab = np.full(X * Y, NIL, np.int32)
    seeds = np.ascontiguousarray(seeds, np.int32)
    lab[seeds] = seed_labels
    wmax = ref().ref_imagegraph(as_i32(img), X, Y, adj, float(np.float32(pol * 100.0)), seeds,
                                len(seeds), lab, int(ntimes))
    return lab, int(wmax)


def ref_imagegraph_energy(img, adj, label, pol, lb=1):
    """GetEnergy_Min(sImageGraph) of a label map on the reference's oriented image graph."""
    X, Y = _ig_dims(img)
    return int(ref().ref_imagegraph_energy(as_i32(img), X, Y, adj, float(np.float32(pol * 100.0)),
                                           np.ascontiguousarray(label, np.int32).reshape(-1), lb))


def ref_read_volume(path):
    """Scene32::Read: (int32 array (Z, Y, X), spacing (dx, dy, dz))."""
    dims = np.zeros(3, np.int32)
    sp = np.zeros(3, np.float32)
    n = ref().ref_read_volume(os.fsencode(path), None, 0, dims, sp)
    assert n >= 0
    out = np.empty(n, np.int32)
    ref().ref_read_volume(os.fsencode(path), out.ctypes.data, n, dims, sp)
    X, Y, Z = (int(v) for v in dims)
    return out.reshape(Z, Y, X), tuple(float(v) for v in sp)


def ref_write_volume(path, vol, spacing):
    """Scene32::Write of an int32 volume (Z, Y, X)."""
    v = np.ascontiguousarray(vol, np.int32)
    Z, Y, X = v.shape
    ref().ref_write_volume(os.fsencode(path), v.reshape(-1), np.array([X, Y, Z], np.int32),
                           np.array(spacing, np.float32))


def ref_gaussian_blur(img):
    X, Y, Z = _dims(img)
    out = np.empty(X * Y * Z, np.int32)
    ref().ref_gaussian_blur(as_i32(img), X, Y, Z, out)
    return out
