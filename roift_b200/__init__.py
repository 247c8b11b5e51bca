"""roift_b200 -- B200-native (sm_100a) OIFT + relaxation, Python host mirror.

The compute path is liboift_b200.so (CUDA kernels behind the C ABI declared in
include/oift_b200.h).  This module binds that ABI with ctypes and mirrors the
reference call surface of the path:

  * oift_fmax_gpu_run / oift_gpu_run   -- gpu/oift_fmax_gpu.cu:139-149, gpu/oift_gpu.cu:149-158
  * OIFT_Multi / OIFT_Multi_PerClass   -- gft/include/gft_ift.h:108-122 (labels in place)
  * ORelax_1_Multi / ORelax_1_Multi_PerClass -- gft/include/gft_ift.h:451-465

There is no CPU fallback: importing works without a GPU (so the ABI can be inspected),
but every compute call raises if the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboift_b200.so")
HEADER = os.path.join(HERE, "..", "include", "oift_b200.h")

NIL = -1
OK = 0
STATUS = {0: "OK", -1: "BAD_ARG", -2: "NO_SEEDS", -3: "OOM", -4: "NOT_CONVERGED",
          -5: "QUEUE_OVERFLOW", -6: "CUDA", -7: "RANGE", -8: "UNSUPPORTED", -9: "SEED_RANGE"}
E_BAD_ARG, E_NO_SEEDS, E_OOM, E_NOT_CONVERGED, E_QUEUE_OVERFLOW = -1, -2, -3, -4, -5
E_CUDA, E_RANGE, E_UNSUPPORTED, E_SEED_RANGE = -6, -7, -8, -9
W_MODES = {"grad": 0, "grad_q": 1, "rbf_q": 2, "blend_q": 3, "imagegraph": 4}


class OiftError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status})")


class Params(C.Structure):
    _fields_ = [("xsize", C.c_int), ("ysize", C.c_int), ("zsize", C.c_int),
                ("adjacency", C.c_int), ("weight_mode", C.c_int), ("wq", C.c_int),
                ("rbf_sigma", C.c_float), ("blend_a", C.c_float), ("per", C.c_float),
                ("per_class", C.POINTER(C.c_float)), ("max_label", C.c_int),
                ("relax_sweeps", C.c_int)]


class Outputs(C.Structure):
    _fields_ = [("cost", C.c_void_p), ("oift_label", C.c_void_p), ("label", C.c_void_p),
                ("mask", C.c_void_p), ("membership", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("levels", C.c_int), ("tile_steps", C.c_longlong), ("clamped", C.c_longlong),
                ("nclasses", C.c_int), ("ms_weights", C.c_float), ("ms_oift", C.c_float),
                ("ms_relax", C.c_float), ("ms_total", C.c_float), ("kernels", C.c_int),
                ("ms_oift_kernel", C.c_float), ("ms_sweeps", C.c_float),
                ("oift_cycles", C.c_longlong * 24),
                ("relax_active_voxel_sweeps", C.c_longlong)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["oift_cycles"] = list(self.oift_cycles)
        return d


class Job(C.Structure):
    """oift_b200_job: one (volume, seed set) of the batched driver (device pointers)."""
    _fields_ = [("image", C.c_void_p), ("xsize", C.c_int), ("ysize", C.c_int),
                ("zsize", C.c_int), ("seeds", C.c_void_p), ("seed_labels", C.c_void_p),
                ("nseeds", C.c_int), ("per", C.c_float), ("cost", C.c_void_p),
                ("label", C.c_void_p), ("mask", C.c_void_p), ("status", C.c_int)]


class AdjointParams(C.Structure):
    """oift_b200_adjoint_params."""
    _fields_ = [("xsize", C.c_int), ("ysize", C.c_int), ("zsize", C.c_int),
                ("adjacency", C.c_int), ("sweeps", C.c_int), ("checkpoint", C.c_int),
                ("kernel", C.c_int), ("sigma", C.c_float), ("alpha", C.c_float),
                ("beta", C.c_float), ("eps", C.c_float)]


ADJ_KERNELS = {"rbf": 0, "pow8": 1}


class BatchStats(C.Structure):
    _fields_ = [("teams", C.c_int), ("jobs", C.c_int), ("tuning", C.c_int),
                ("ms_wall", C.c_float), ("ms_oift", C.c_float), ("ms_relax", C.c_float),
                ("tile_ty", C.c_int)]


EXPORTS = ["oift_b200_create", "oift_b200_destroy", "oift_b200_scratch_bytes",
           "oift_b200_set_stream", "oift_b200_status_string", "oift_b200_run_device_i16",
           "oift_b200_run_host", "oift_b200_relax_host", "oift_b200_build_weights_i16",
           "oift_b200_weight_planes",
           "oift_fmax_gpu_run", "oift_gpu_run", "oift_b200_last_status",
           "oift_b200_level_profile", "oift_b200_selftest_div100",
           "oift_b200_oift_noalloc", "oift_b200_noalloc_scratch_bytes",
           "oift_b200_run_batch", "oift_b200_set_oift_grid", "oift_b200_set_limits",
           "oift_b200_set_batch_tile",
           "oift_b200_gaussian_blur_i32",
           "oift_b200_conditional_dilation", "oift_b200_inject_boundary_seeds",
           "oift_b200_run_cli_host", "oift_b200_run_pyramid_host",
           "oift_b200_run_pyramid_device_i16", "oift_b200_adjoint",
           "oift_b200_bottleneck_arcs", "oift_b200_cost_adjoint",
           "oift_b200_batch_graph_create", "oift_b200_batch_graph_launch",
           "oift_b200_batch_graph_destroy", "oift_b200_read_seeds", "oift_b200_read_polarity",
           "oift_b200_read_volume", "oift_b200_write_volume"]

_lib = None


def lib():
    """Load liboift_b200.so (build it first with roift_b200.build.build())."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: the CUDA extension is not built "
                          "(python -m roift_b200.build); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        vp, i32p = C.c_void_p, np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        L.oift_b200_create.argtypes = [C.POINTER(vp), C.c_int]
        L.oift_b200_destroy.argtypes = [vp]
        L.oift_b200_scratch_bytes.restype = C.c_size_t
        L.oift_b200_scratch_bytes.argtypes = [vp]
        L.oift_b200_set_stream.argtypes = [vp, vp]
        L.oift_b200_status_string.restype = C.c_char_p
        L.oift_b200_run_device_i16.argtypes = [vp, C.POINTER(Params), vp, vp, vp, C.c_int,
                                               C.POINTER(Outputs), C.POINTER(Stats)]
        L.oift_b200_run_host.argtypes = [vp, C.POINTER(Params), i32p, i32p, i32p, C.c_int,
                                         vp, vp, C.c_int, vp, C.POINTER(Stats)]
        L.oift_b200_level_profile.argtypes = [vp, vp, C.c_int]
        L.oift_b200_run_batch.argtypes = [vp, C.POINTER(Params), C.POINTER(Job), C.c_int, C.c_int,
                                          C.POINTER(BatchStats)]
        L.oift_b200_set_oift_grid.argtypes = [vp, C.c_int]
        L.oift_b200_set_limits.argtypes = [vp, C.c_longlong, C.c_int]
        L.oift_b200_set_batch_tile.argtypes = [vp, C.c_int]
        L.oift_b200_relax_host.argtypes = [vp, C.POINTER(Params), i32p, i32p, i32p, C.c_int,
                                           vp, C.c_int, vp]
        L.oift_b200_batch_graph_create.argtypes = [vp, C.POINTER(Params), C.POINTER(Job), C.c_int,
                                                   C.c_int, C.POINTER(vp)]
        L.oift_b200_batch_graph_launch.argtypes = [vp, C.POINTER(Job), C.POINTER(C.c_float)]
        L.oift_b200_batch_graph_destroy.argtypes = [vp]
        L.oift_b200_read_seeds.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, vp, vp, C.c_int]
        L.oift_b200_read_polarity.argtypes = [C.c_char_p, vp, C.c_int]
        L.oift_b200_read_volume.argtypes = [C.c_char_p, vp, C.c_size_t, C.POINTER(C.c_int),
                                            C.POINTER(C.c_float)]
        L.oift_b200_write_volume.argtypes = [C.c_char_p, vp, C.POINTER(C.c_int),
                                             C.POINTER(C.c_float)]
        L.oift_b200_selftest_div100.argtypes = [C.POINTER(C.c_ulonglong), C.POINTER(C.c_uint)]
        L.oift_b200_oift_noalloc.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.c_int, C.c_float, vp, C.c_int, vp, vp, C.c_int,
                                             vp, vp, vp]
        L.oift_b200_noalloc_scratch_bytes.restype = C.c_size_t
        L.oift_b200_build_weights_i16.argtypes = [vp, C.POINTER(Params), vp, vp,
                                                  C.POINTER(C.c_longlong)]
        L.oift_fmax_gpu_run.argtypes = [i32p, i32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                        np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"),
                                        C.c_int, i32p, C.c_int]
        L.oift_gpu_run.argtypes = [C.c_int] + L.oift_fmax_gpu_run.argtypes
        L.oift_b200_gaussian_blur_i32.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int,
                                                  C.c_int]
        L.oift_b200_conditional_dilation.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int,
                                                     C.c_float, C.c_float,
                                                     C.POINTER(C.c_longlong)]
        L.oift_b200_inject_boundary_seeds.argtypes = [i32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                      vp, C.c_int]
        L.oift_b200_run_cli_host.argtypes = [vp, C.POINTER(Params), i32p, i32p, i32p, C.c_int,
                                             C.c_int, C.c_float, C.POINTER(Stats)]
        L.oift_b200_run_pyramid_host.argtypes = L.oift_b200_run_cli_host.argtypes
        L.oift_b200_adjoint.argtypes = [vp, C.POINTER(AdjointParams), vp, vp, vp, vp, vp, C.c_int,
                                        vp, vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.oift_b200_bottleneck_arcs.argtypes = [vp, C.POINTER(Params), vp, vp, vp, vp, C.c_int,
                                                vp]
        L.oift_b200_cost_adjoint.argtypes = [vp, C.POINTER(AdjointParams), vp, vp, vp, vp, vp,
                                             C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.oift_b200_run_pyramid_device_i16.argtypes = [vp, C.POINTER(Params), vp, vp, vp, C.c_int,
                                                       C.c_int, C.c_float, vp,
                                                       C.POINTER(Stats)]
        _lib = L
    return _lib


def make_params(shape_zyx, adjacency=6, weight_mode="grad", wq=4095, rbf_sigma=150.0,
                blend_a=0.5, pol=None, per_class=None, sweeps=0):
    """Parameters; pol in [-1,1] becomes per = (float)(pol*100.0) as the CLI passes it
    (oiftrelax.cpp:387), per_class values are already x100."""
    if len(shape_zyx) == 2:
        Z, (Y, X) = 1, shape_zyx
    else:
        Z, Y, X = shape_zyx
    p = Params()
    p.xsize, p.ysize, p.zsize = X, Y, Z
    p.adjacency = adjacency
    p.weight_mode = W_MODES[weight_mode]
    p.wq = wq
    p.rbf_sigma = rbf_sigma
    p.blend_a = blend_a
    keep = None
    if per_class is not None:
        keep = np.ascontiguousarray(per_class, np.float32)
        p.per_class = keep.ctypes.data_as(C.POINTER(C.c_float))
        p.max_label = len(keep) - 1
        p.per = 0.0
    else:
        p.per = float(np.float32((pol or 0.0) * 100.0))
        p.per_class = None
        p.max_label = 0
    p.relax_sweeps = sweeps
    p._keep = keep
    return p


class Context:
    """Device scratch + stream owner (oift_b200_create / oift_b200_destroy)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        rc = lib().oift_b200_create(C.byref(self._h), device)
        if rc != OK:
            raise OiftError(rc, "oift_b200_create")
        self.device = device

    def close(self):
        if self._h:
            lib().oift_b200_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        rc = lib().oift_b200_set_stream(self._h, C.c_void_p(stream_ptr or 0))
        if rc != OK:
            raise OiftError(rc, "oift_b200_set_stream")

    def scratch_bytes(self) -> int:
        return int(lib().oift_b200_scratch_bytes(self._h))

    def run_device(self, params, image_ptr, seeds_ptr, labels_ptr, nseeds, cost=None,
                   oift_label=None, label=None, mask=None, membership=None) -> Stats:
        """Full pipeline on device pointers (ints).  Output pointers may be None."""
        out = Outputs(cost or 0, oift_label or 0, label or 0, mask or 0, membership or 0)
        st = Stats()
        rc = lib().oift_b200_run_device_i16(self._h, C.byref(params), C.c_void_p(image_ptr),
                                            C.c_void_p(seeds_ptr), C.c_void_p(labels_ptr),
                                            int(nseeds), C.byref(out), C.byref(st))
        if rc != OK:
            raise OiftError(rc, "oift_b200_run_device_i16")
        return st

    def run_host(self, params, image, label, seeds, want_cost=False, want_membership=0,
                 want_mask=False):
        """Full pipeline on host arrays (reference-style int32 image, labels in/out)."""
        img = np.ascontiguousarray(np.asarray(image).reshape(-1), np.int32)
        lab = np.ascontiguousarray(label, np.int32)
        sd = np.ascontiguousarray(seeds, np.int32)
        N = img.size
        cost = np.empty(N, np.int32) if want_cost else None
        memb = np.empty(want_membership * N, np.float32) if want_membership else None
        mask = np.empty(N, np.uint8) if want_mask else None
        st = Stats()
        rc = lib().oift_b200_run_host(self._h, C.byref(params), img, lab, sd, len(sd),
                                      cost.ctypes.data if cost is not None else None,
                                      memb.ctypes.data if memb is not None else None,
                                      int(want_membership),
                                      mask.ctypes.data if mask is not None else None,
                                      C.byref(st))
        if rc != OK:
            raise OiftError(rc, "oift_b200_run_host")
        if memb is not None:
            memb = memb[: st.nclasses * N].reshape(st.nclasses, N)
        return lab, cost, memb, mask, st

    def relax_host(self, params, image, label, seeds, want_membership=0, want_mask=False):
        """The relaxation alone (ORelax_1_Multi): relaxes the labels `label` (e.g. an OIFT's)
        with params.relax_sweeps sweeps; returns (labels, membership or None, mask or None)."""
        img = np.ascontiguousarray(np.asarray(image).reshape(-1), np.int32)
        lab = np.ascontiguousarray(label, np.int32).reshape(-1).copy()
        sd = np.ascontiguousarray(seeds, np.int32)
        N = img.size
        memb = np.empty(want_membership * N, np.float32) if want_membership else None
        mask = np.empty(N, np.uint8) if want_mask else None
        rc = lib().oift_b200_relax_host(self._h, C.byref(params), img, lab, sd, len(sd),
                                        memb.ctypes.data if memb is not None else None,
                                        int(want_membership),
                                        mask.ctypes.data if mask is not None else None)
        if rc != OK:
            raise OiftError(rc, "oift_b200_relax_host")
        return lab, memb, mask

    def run_batch(self, params, jobs, teams=0) -> BatchStats:
        """Batched driver: `jobs` is a ctypes array of Job (device pointers); teams = 0
        autotunes the number of OIFT teams the GPU is split into (the first calls of a
        context measure one candidate each; stats.tuning is 1 for those calls)."""
        st = BatchStats()
        rc = lib().oift_b200_run_batch(self._h, C.byref(params), jobs, len(jobs), int(teams),
                                       C.byref(st))
        if rc != OK:
            raise OiftError(rc, "oift_b200_run_batch")
        return st

    def batch_graph(self, params, jobs, teams=0) -> "BatchGraph":
        """Record the batch once into a CUDA graph (see oift_b200_batch_graph_create)."""
        h = C.c_void_p()
        rc = lib().oift_b200_batch_graph_create(self._h, C.byref(params), jobs, len(jobs),
                                                int(teams), C.byref(h))
        if rc != OK:
            raise OiftError(rc, "oift_b200_batch_graph_create")
        return BatchGraph(h, jobs)

    def set_limits(self, spin_limit: int = 0, max_levels: int = 0):
        """Bounds of the OIFT kernels' device waits (polls of one wait, levels of a run);
        0 restores the defaults.  Reaching one ends the call with E_NOT_CONVERGED."""
        rc = lib().oift_b200_set_limits(self._h, C.c_longlong(int(spin_limit)), int(max_levels))
        if rc != OK:
            raise OiftError(rc, "oift_b200_set_limits")

    def set_batch_tile(self, tile_ty: int):
        """Warp tile of the batched OIFT for explicit team counts: 8 (32x8x4) or 4 (32x4x8)."""
        rc = lib().oift_b200_set_batch_tile(self._h, int(tile_ty))
        if rc != OK:
            raise OiftError(rc, "oift_b200_set_batch_tile")

    def set_oift_grid(self, ctas: int):
        rc = lib().oift_b200_set_oift_grid(self._h, int(ctas))
        if rc != OK:
            raise OiftError(rc, "oift_b200_set_oift_grid")

    def gaussian_blur(self, in_ptr, out_ptr, shape_zyx, passes=1):
        """`passes` Gaussian blurs of a device int32 volume (in == out allowed)."""
        Z, Y, X = shape_zyx
        rc = lib().oift_b200_gaussian_blur_i32(self._h, C.c_void_p(in_ptr), C.c_void_p(out_ptr),
                                               X, Y, Z, int(passes))
        if rc != OK:
            raise OiftError(rc, "oift_b200_gaussian_blur_i32")

    def conditional_dilation(self, image_ptr, label_ptr, shape_zyx, radius=1.0,
                             percentile=50.0) -> int:
        """Conditional dilation of a device int32 label map; returns the voxels added."""
        Z, Y, X = shape_zyx
        added = C.c_longlong(0)
        rc = lib().oift_b200_conditional_dilation(self._h, C.c_void_p(image_ptr),
                                                  C.c_void_p(label_ptr), X, Y, Z, float(radius),
                                                  float(percentile), C.byref(added))
        if rc != OK:
            raise OiftError(rc, "oift_b200_conditional_dilation")
        return added.value

    def run_cli_host(self, params, image, label, seeds, blur_passes=2, percentile=50.0):
        """The CLI chain (shift, blur, OIFT, relaxation, conditional dilation) on host
        arrays; `label` (seed labels in) receives the result."""
        img = np.ascontiguousarray(np.asarray(image).reshape(-1), np.int32)
        lab = np.ascontiguousarray(label, np.int32)
        sd = np.ascontiguousarray(seeds, np.int32)
        st = Stats()
        rc = lib().oift_b200_run_cli_host(self._h, C.byref(params), img, lab, sd, len(sd),
                                          int(blur_passes), float(percentile), C.byref(st))
        if rc != OK:
            raise OiftError(rc, "oift_b200_run_cli_host")
        return lab, st

    def run_pyramid_host(self, params, image, label, seeds, blur_passes=2, percentile=50.0):
        """Two-level coarse-to-fine cascade on host arrays (unshifted int32 image; `label`
        holds the seed labels, NIL elsewhere, and receives the result)."""
        img = np.ascontiguousarray(np.asarray(image).reshape(-1), np.int32)
        lab = np.ascontiguousarray(label, np.int32)
        sd = np.ascontiguousarray(seeds, np.int32)
        st = Stats()
        rc = lib().oift_b200_run_pyramid_host(self._h, C.byref(params), img, lab, sd, len(sd),
                                              int(blur_passes), float(percentile), C.byref(st))
        if rc != OK:
            raise OiftError(rc, "oift_b200_run_pyramid_host")
        return lab, st

    def run_pyramid_device(self, params, image_ptr, label_in_ptr, seeds_ptr, nseeds,
                           label_out_ptr, blur_passes=2, percentile=50.0) -> Stats:
        """The cascade on device arrays (int16 image, int32 labels and seeds)."""
        st = Stats()
        rc = lib().oift_b200_run_pyramid_device_i16(
            self._h, C.byref(params), C.c_void_p(image_ptr), C.c_void_p(label_in_ptr),
            C.c_void_p(seeds_ptr), int(nseeds), int(blur_passes), float(percentile),
            C.c_void_p(label_out_ptr), C.byref(st))
        if rc != OK:
            raise OiftError(rc, "oift_b200_run_pyramid_device_i16")
        return st

    def adjoint(self, shape_zyx, image_ptr, labels0_ptr, seeds_ptr, seed_labels_ptr, nseeds,
                truth_ptr, sigma=150.0, alpha=0.0, beta=1.0, sweeps=10, checkpoint=0,
                kernel="rbf", adjacency=6, eps=1.0, grad_map_ptr=None, membership_ptr=None,
                want_grad=True):
        """Soft-Dice loss after `sweeps` relaxation sweeps and its gradient with respect to
        (sigma, alpha, beta).  Returns (loss, np.array([dL/dsigma, dL/dalpha, dL/dbeta]))."""
        Z, Y, X = shape_zyx
        ap = AdjointParams(X, Y, Z, adjacency, int(sweeps), int(checkpoint), ADJ_KERNELS[kernel],
                           float(sigma), float(alpha), float(beta), float(eps))
        loss = C.c_double(0.0)
        g = (C.c_double * 3)()
        rc = lib().oift_b200_adjoint(self._h, C.byref(ap), C.c_void_p(image_ptr),
                                     C.c_void_p(grad_map_ptr) if grad_map_ptr else None,
                                     C.c_void_p(labels0_ptr), C.c_void_p(seeds_ptr),
                                     C.c_void_p(seed_labels_ptr), int(nseeds),
                                     C.c_void_p(truth_ptr),
                                     C.c_void_p(membership_ptr) if membership_ptr else None,
                                     C.byref(loss), g if want_grad else None)
        if rc != OK:
            raise OiftError(rc, "oift_b200_adjoint")
        return loss.value, np.array(list(g))

    def bottleneck_arcs(self, params, image_ptr, cost_ptr, label_ptr, seeds_ptr, nseeds,
                        arcs_ptr):
        """Per-voxel bottleneck arc of the fixed OIFT forest (int64 [N] device output:
        tail * 32 + direction, -2 at seeds, -3 unreached) from an integer OIFT result."""
        rc = lib().oift_b200_bottleneck_arcs(self._h, C.byref(params), C.c_void_p(image_ptr),
                                             C.c_void_p(cost_ptr), C.c_void_p(label_ptr),
                                             C.c_void_p(seeds_ptr), int(nseeds),
                                             C.c_void_p(arcs_ptr))
        if rc != OK:
            raise OiftError(rc, "oift_b200_bottleneck_arcs")

    def cost_adjoint(self, shape_zyx, image_ptr, label_ptr, arcs_ptr, truth_ptr, sigma=150.0,
                     alpha=0.0, beta=1.0, eps=1.0, adjacency=6, grad_map_ptr=None,
                     want_grad=True):
        """Soft-Dice loss of the object confidence of the cost map (continuous RBF weights
        of the bottleneck arcs) and its gradient w.r.t. (sigma, alpha, beta)."""
        Z, Y, X = shape_zyx
        ap = AdjointParams(X, Y, Z, adjacency, 1, 0, ADJ_KERNELS["rbf"], float(sigma),
                           float(alpha), float(beta), float(eps))
        loss = C.c_double(0.0)
        g = (C.c_double * 3)()
        rc = lib().oift_b200_cost_adjoint(self._h, C.byref(ap), C.c_void_p(image_ptr),
                                          C.c_void_p(grad_map_ptr) if grad_map_ptr else None,
                                          C.c_void_p(label_ptr), C.c_void_p(arcs_ptr),
                                          C.c_void_p(truth_ptr), C.byref(loss),
                                          g if want_grad else None)
        if rc != OK:
            raise OiftError(rc, "oift_b200_cost_adjoint")
        return loss.value, np.array(list(g))

    def level_profile(self, cap=8192):
        """(cycles, tile activations) per OIFT level of the last run."""
        buf = np.zeros(2 * cap, np.uint32)
        n = lib().oift_b200_level_profile(self._h, buf.ctypes.data_as(C.c_void_p), cap)
        if n < 0:
            raise OiftError(n, "oift_b200_level_profile")
        return buf[: 2 * n].reshape(n, 2)

    def build_weights(self, params, image_ptr, weights_ptr) -> int:
        cl = C.c_longlong(0)
        rc = lib().oift_b200_build_weights_i16(self._h, C.byref(params), C.c_void_p(image_ptr),
                                               C.c_void_p(weights_ptr), C.byref(cl))
        if rc != OK:
            raise OiftError(rc, "oift_b200_build_weights_i16")
        return cl.value


class BatchGraph:
    """A recorded batch: launch() replays it and returns the device milliseconds."""

    def __init__(self, handle, jobs):
        self._h = handle
        self.jobs = jobs

    def launch(self) -> float:
        ms = C.c_float(0.0)
        rc = lib().oift_b200_batch_graph_launch(self._h, self.jobs, C.byref(ms))
        if rc != OK:
            raise OiftError(rc, "oift_b200_batch_graph_launch")
        return ms.value

    def close(self):
        if self._h:
            lib().oift_b200_batch_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_seeds(path, shape_zyx, label):
    """Seeds file of the CLI (host-only): returns the seed addresses; `label` (int32, NIL
    elsewhere) receives the seed labels."""
    Z, Y, X = shape_zyx
    n = lib().oift_b200_read_seeds(os.fsencode(path), X, Y, Z, None, None, 0)
    if n < 0:
        raise OiftError(n, "oift_b200_read_seeds")
    out = np.empty(max(n, 1), np.int32)
    n = lib().oift_b200_read_seeds(os.fsencode(path), X, Y, Z, label.ctypes.data,
                                   out.ctypes.data, n)
    if n < 0:
        raise OiftError(n, "oift_b200_read_seeds")
    return out[:n].copy()


def read_polarity(path):
    """Per-class polarity file of the CLI: the values x100 (float32)."""
    n = lib().oift_b200_read_polarity(os.fsencode(path), None, 0)
    if n < 0:
        raise OiftError(n, "oift_b200_read_polarity")
    out = np.empty(n, np.float32)
    n = lib().oift_b200_read_polarity(os.fsencode(path), out.ctypes.data, n)
    if n < 0:
        raise OiftError(n, "oift_b200_read_polarity")
    return out


def read_volume(path):
    """Volume file of the CLI (.scn, NIfTI-1 .nii / .nii.gz / .hdr+.img), host only:
    (int32 array shaped (Z, Y, X), spacing (dx, dy, dz))."""
    dims, sp = (C.c_int * 3)(), (C.c_float * 3)()
    st = lib().oift_b200_read_volume(os.fsencode(path), None, 0, dims, sp)
    if st != 0:
        raise OiftError(st, "oift_b200_read_volume")
    X, Y, Z = dims
    out = np.empty((Z, Y, X), np.int32)
    st = lib().oift_b200_read_volume(os.fsencode(path), out.ctypes.data, out.size, dims, sp)
    if st != 0:
        raise OiftError(st, "oift_b200_read_volume")
    return out, tuple(float(v) for v in sp)


def write_volume(path, vol, spacing=(1.0, 1.0, 1.0)):
    """Writes an int32 volume shaped (Z, Y, X) (or (Y, X)) as Scene32::Write does."""
    v = np.ascontiguousarray(vol, np.int32)
    Z, Y, X = (1,) + v.shape if v.ndim == 2 else v.shape
    dims = (C.c_int * 3)(X, Y, Z)
    sp = (C.c_float * 3)(*spacing)
    st = lib().oift_b200_write_volume(os.fsencode(path), v.ctypes.data, dims, sp)
    if st != 0:
        raise OiftError(st, "oift_b200_write_volume")


def inject_boundary_seeds(label, shape_zyx, stride):
    """Boundary seeds of the CLI (host-only): returns the new seeds; `label` (int32, NIL =
    -1) is updated in place."""
    Z, Y, X = shape_zyx
    n = lib().oift_b200_inject_boundary_seeds(label, X, Y, Z, int(stride), None, 0)
    if n < 0:
        raise OiftError(n, "oift_b200_inject_boundary_seeds")
    out = np.empty(max(n, 1), np.int32)
    n = lib().oift_b200_inject_boundary_seeds(label, X, Y, Z, int(stride), out.ctypes.data, n)
    if n < 0:
        raise OiftError(n, "oift_b200_inject_boundary_seeds")
    return out[:n].copy()


def oift_noalloc(image_ptr, shape_zyx, seeds_ptr, labels_ptr, nseeds, cost_ptr=None,
                 label_ptr=None, adjacency=6, weight_mode="grad_q", wq=4095, pol=None,
                 per_class=None, stream_ptr=None) -> None:
    """OIFT on device buffers with no device allocation (oift_b200_oift_noalloc).

    For callers that cannot allow a library to call cudaMalloc while they run: the
    weights and the OIFT state live in a static device array of the library (limit
    OIFT_NOALLOC_MAX_VOXELS = 2^20 voxels).  Calls that overlap on the GPU race."""
    Z, Y, X = shape_zyx if len(shape_zyx) == 3 else (1,) + tuple(shape_zyx)
    keep = None
    if per_class is not None:
        keep = np.ascontiguousarray(per_class, np.float32)
        pc, ml, per = keep.ctypes.data, len(keep) - 1, 0.0
    else:
        pc, ml, per = None, 0, float(np.float32((pol or 0.0) * 100.0))
    rc = lib().oift_b200_oift_noalloc(C.c_void_p(image_ptr), X, Y, Z, adjacency,
                                      W_MODES[weight_mode], wq, per, pc, ml,
                                      C.c_void_p(seeds_ptr), C.c_void_p(labels_ptr), int(nseeds),
                                      C.c_void_p(cost_ptr or 0), C.c_void_p(label_ptr or 0),
                                      C.c_void_p(stream_ptr or 0))
    del keep
    if rc != OK:
        raise OiftError(rc, "oift_b200_oift_noalloc")


def selftest_div100():
    """(mismatches, first bad bit pattern) of the sweep's x/100 against IEEE division."""
    bad, first = C.c_ulonglong(0), C.c_uint(0)
    rc = lib().oift_b200_selftest_div100(C.byref(bad), C.byref(first))
    if rc != OK:
        raise OiftError(rc, "oift_b200_selftest_div100")
    return bad.value, first.value


def weight_planes(adjacency: int) -> int:
    return int(lib().oift_b200_weight_planes(adjacency))


# ------------------------------------------------ reference call surface ----
def oift_fmax_gpu_run(image, labels, xsize, ysize, zsize, per_class, seeds) -> int:
    """gpu/oift_fmax_gpu.cu:139-149: labels (int32, NIL except seeds) updated in place;
    returns the number of levels, raises on error."""
    img = np.ascontiguousarray(np.asarray(image).reshape(-1), np.int32)
    pc = np.ascontiguousarray(per_class, np.float32)
    sd = np.ascontiguousarray(seeds, np.int32)
    assert labels.dtype == np.int32 and labels.flags.c_contiguous
    r = lib().oift_fmax_gpu_run(img, labels, img.size, xsize, ysize, zsize, pc, len(pc) - 1,
                                sd, len(sd))
    if r < 0:
        raise OiftError(lib().oift_b200_last_status(), "oift_fmax_gpu_run")
    return r


_default_ctx = None


def _ctx():
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _shape_of(scn):
    a = np.asarray(scn)
    return a.shape if a.ndim == 3 else (1,) + a.shape


def OIFT_Multi(adjacency, scn, per, S, label, per_class=None):
    """gft::ift::OIFT_Multi(A, scn, per, S, label) on the GPU: label (flat int32, NIL
    except seeds) is overwritten with the OIFT labels.  per is x100 as in the reference.
    Returns the f_max cost map."""
    shp = _shape_of(scn)
    if per_class is None:
        p = make_params(shp, adjacency=adjacency, weight_mode="grad", pol=None)
        p.per = float(np.float32(per))
    else:
        p = make_params(shp, adjacency=adjacency, weight_mode="grad", per_class=per_class)
    lab, cost, _, _, _ = _ctx().run_host(p, scn, label, S, want_cost=True)
    return cost


def ORelax_1_Multi(adjacency, scn, per, S, label, ntimes, per_class=None):
    """OIFT + gft::ift::ORelax_1_Multi on the GPU (label in = seeds, out = relaxed labels).
    Returns the relaxed membership [classes, N]."""
    shp = _shape_of(scn)
    if per_class is None:
        p = make_params(shp, adjacency=adjacency, weight_mode="grad", sweeps=ntimes)
        p.per = float(np.float32(per))
    else:
        p = make_params(shp, adjacency=adjacency, weight_mode="grad", per_class=per_class,
                        sweeps=ntimes)
    _, _, memb, _, _ = _ctx().run_host(p, scn, label, S, want_membership=8)
    return memb
