"""patchtable_b200: B200-native PatchTable build and nearest-neighbour-field query.

Python binding of the C ABI in include/patchtable_b200.h (ctypes over the in-tree
libpatchtable_b200.so).  Names follow the reference's C++ API (patchtable/patchtable.h:4359-4491,
patchtable/patchtable_params.h):

    p = PatchTableParams("-speed 3 -coherence_spatial 4")   # PatchTableParams(argc, argv)
    table = PatchTable(p, b)                                # PatchTable<>(&p, b, allowed)
    ann = table.lookup(a)                                   # table.lookup(a, ann)

``ann`` is a (h-7) x (w-7) x 3 float64 array [NNF_X, NNF_Y, NNF_DIST] like the reference's.
Errors raise PatchTableError with the library's message; there is no CPU fallback: if the
library or a GPU is missing, construction fails.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = ["PatchTableParams", "PatchTable", "PatchTableError", "QueryBatch", "NNF_X", "NNF_Y", "NNF_DIST", "lib",
           "descriptor", "launch_count", "reset_launch_count"]

NNF_X, NNF_Y, NNF_DIST = 0, 1, 2
PT_MAX_DIMS = 16
PT_PATH_MAX = 256
HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpatchtable_b200.so")

STATUS = {0: "PT_OK", 1: "PT_BAD_ARG", 2: "PT_OOM", 3: "PT_CUDA_ERR", 4: "PT_TIMEOUT", 5: "PT_UNSUPPORTED", 6: "PT_IO"}


class PatchTableError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__("%s: %s" % (STATUS.get(status, status), message))
        self.status = status


class _Params(C.Structure):
    """Mirror of pt_params (include/patchtable_b200.h)."""
    _fields_ = [
        ("limit", C.c_double),
        ("ndims", C.c_int), ("nchroma", C.c_int), ("grid_ndims", C.c_int),
        ("nslices", C.c_int * PT_MAX_DIMS), ("n_nslices", C.c_int),
        ("partition_step", C.c_int),
        ("populate_random", C.c_int), ("populate_nearest", C.c_int),
        ("run_dt", C.c_int), ("dt_algo", C.c_int), ("dt_iters", C.c_int),
        ("kcoherence", C.c_int), ("kcoherence_min_dist", C.c_int), ("kcoherence_step", C.c_int),
        ("kcoherence_iter", C.c_int),
        ("flann_reset_step", C.c_int), ("flann_build_step", C.c_int),
        ("triangle_factor", C.c_double),
        ("prop_iters", C.c_int), ("query_step", C.c_int), ("do_prop", C.c_int), ("prop_dist", C.c_int),
        ("coherence_spatial", C.c_double), ("coherence_temporal", C.c_double),
        ("do_table_lookup", C.c_int), ("do_rs", C.c_int), ("spatial", C.c_int),
        ("allowed_index", C.c_int),
        ("recalc_dist_temporal", C.c_int), ("sanitize_input", C.c_int), ("init_random", C.c_int),
        ("convert_colorspace", C.c_int), ("colorspace", C.c_int),
        ("is_descriptor", C.c_int), ("descriptor_padded", C.c_int),
        ("patch_w", C.c_int),
        ("threads", C.c_int), ("verbose", C.c_int), ("query_iters", C.c_int), ("ntables", C.c_int),
        ("table_ratio", C.c_double),
        ("lookup_algo", C.c_int), ("kcoherence_algo", C.c_int), ("dim_algo", C.c_int),
        ("incoherence", C.c_int), ("randomize_dt", C.c_int), ("parallel_dt", C.c_int),
        ("populate_exptime", C.c_int), ("dt_mode", C.c_int),
        ("load_filename", C.c_char * PT_PATH_MAX),
        ("save_filename", C.c_char * PT_PATH_MAX),
        ("gpu_prop_passes", C.c_int),
        ("gpu_jump", C.c_int),
        ("gpu_pull_max", C.c_int),
        ("gpu_tile", C.c_int),
        ("pca_samples", C.c_int), ("pca_subtract_mean", C.c_int), ("pca_mean", C.c_int),
        ("gpu_bands", C.c_int),
        ("gpu_kc_max", C.c_int),
    ]


_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")

_lib = None


def lib() -> C.CDLL:
    """Loads the native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise PatchTableError(1, "native library %s is missing; run python -m patchtable_b200.build" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    P = C.POINTER(_Params)
    vp = C.c_void_p
    L.pt_params_default.argtypes = [P]
    L.pt_params_default.restype = None
    L.pt_params_set_speed.argtypes = [P, C.c_int]
    L.pt_params_from_switches.argtypes = [P, C.c_char_p]
    L.pt_table_create.argtypes = [P, _f32p, C.c_int, C.c_int, C.c_int, vp, C.POINTER(vp)]
    L.pt_table_create_with_descriptor.argtypes = [P, _f32p, C.c_int, C.c_int, _f32p, vp, C.POINTER(vp)]
    L.pt_table_free.argtypes = [vp]
    L.pt_table_subtable.argtypes = [vp, C.c_int, C.POINTER(vp)]
    L.pt_table_save.argtypes = [vp, C.c_char_p]
    L.pt_table_load.argtypes = [P, C.c_char_p, C.POINTER(vp)]
    L.pt_table_image_shape.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.pt_table_free.restype = None
    L.pt_table_set_params.argtypes = [vp, P]
    L.pt_table_lookup.argtypes = [vp, _f32p, C.c_int, C.c_int, _f64p, vp, vp, C.POINTER(C.c_double)]
    L.pt_table_lookup_device.argtypes = [vp, vp, C.c_int, C.c_int, vp, vp]
    L.pt_table_shape.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int64)]
    L.pt_table_shape.restype = C.c_int
    L.pt_table_get_cells.argtypes = [vp, _i32p]
    L.pt_table_get_descriptor.argtypes = [vp, _f32p]
    L.pt_table_get_partition.argtypes = [vp, C.c_int, _f32p, _f32p, _f32p, _i32p, _f32p]
    L.pt_table_get_kcoherence.argtypes = [vp, _i32p, _f32p]
    L.pt_table_add_count.argtypes = [vp]
    L.pt_table_add_count.restype = C.c_int64
    L.pt_table_dt_levels.argtypes = [vp]
    L.pt_table_build_profile.argtypes = [vp, C.POINTER(C.c_double), C.c_int]
    L.pt_table_lookup_profile.argtypes = [vp, vp, C.c_int, C.c_int, vp, vp, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
    L.pt_descriptor.argtypes = [P, _f32p, C.c_int, C.c_int, _f32p]
    L.pt_tc_gemm_f32.argtypes = [vp, C.c_int, vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp]
    fp = C.POINTER(C.c_float)
    L.pt_proposal_create.argtypes = [C.c_uint32, C.POINTER(vp)]
    L.pt_proposal_free.argtypes = [vp]
    L.pt_proposal_free.restype = None
    L.pt_proposal_num_params.restype = C.c_int
    L.pt_proposal_get_params.argtypes = [vp, _f32p]
    L.pt_proposal_set_params.argtypes = [vp, _f32p]
    L.pt_proposal_configure.argtypes = [vp, C.c_float, C.c_int]
    L.pt_proposal_train_step.argtypes = [vp, vp, vp, C.c_int, C.c_float, C.c_float, fp, vp]
    L.pt_proposal_gradient.argtypes = [vp, vp, vp, C.c_int, fp, vp, vp]
    L.pt_proposal_forward.argtypes = [vp, vp, C.c_int, vp, vp]
    L.pt_proposal_sync.argtypes = [vp, vp]
    L.pt_table_proposal_samples.argtypes = [vp, vp, C.c_int, C.c_int, vp, vp, vp, vp]
    L.pt_table_proposal_infer.argtypes = [vp, vp, vp, C.c_int, C.c_int, vp, vp, vp, vp]
    L.pt_table_lookup_batch.argtypes = [vp, C.c_int, vp, vp, vp, vp]
    L.pt_batch_create.argtypes = [vp, C.c_int, vp, vp, C.POINTER(vp)]
    L.pt_batch_free.argtypes = [vp]
    L.pt_batch_free.restype = None
    L.pt_batch_layout.argtypes = [vp, vp, vp, vp]
    L.pt_batch_set_tile.argtypes = [vp, C.c_int]
    L.pt_batch_tile.argtypes = [vp]
    L.pt_batch_tile.restype = C.c_int
    L.pt_batch_lookup.argtypes = [vp, vp, vp, vp]
    L.pt_batch_autotune.argtypes = [vp, vp, vp, vp, C.POINTER(C.c_int), vp]
    L.pt_batch_capture.argtypes = [vp, vp, vp, vp]
    L.pt_batch_replay.argtypes = [vp, vp]
    L.pt_table_lookup_learned.argtypes = [vp, vp, _f32p, C.c_int, C.c_int, _f64p, C.POINTER(C.c_double)]
    L.pt_table_lookup_learned_device.argtypes = [vp, vp, vp, C.c_int, C.c_int, vp, vp]
    L.pt_table_lookup_proposed_profile.argtypes = [vp, vp, C.c_int, C.c_int, vp, vp, C.c_float, C.c_int, vp, vp,
                                                   C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
    L.pt_table_lookup_learned_profile.argtypes = [vp, vp, vp, C.c_int, C.c_int, vp, vp, C.POINTER(C.c_double),
                                                  C.POINTER(C.c_uint64)]
    L.pt_last_error.restype = C.c_char_p
    L.pt_version.restype = C.c_char_p
    L.pt_set_host_threads.argtypes = [C.c_int]
    L.pt_set_lean_kernels.argtypes = [C.c_int]
    L.pt_set_lean_kernels.restype = C.c_int
    L.pt_table_last_transfer.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.pt_set_spin_limit.argtypes = [C.c_int64]
    L.pt_set_spin_limit.restype = C.c_int64
    L.pt_set_device_alloc_limit.argtypes = [C.c_int64]
    L.pt_set_device_alloc_limit.restype = C.c_int64
    L.pt_device_bytes_in_use.restype = C.c_int64
    L.pt_kernel_launch_count.restype = C.c_int64
    L.pt_kernel_launch_count_reset.restype = None
    _lib = L
    return L


def _check(status: int) -> None:
    if status != 0:
        raise PatchTableError(status, lib().pt_last_error().decode(errors="replace"))


class PatchTableParams:
    """PatchTableParams (patchtable/patchtable_params.h:23-161): reference defaults (speed 3),
    then command-line switches, as PatchTableParams(argc, argv) parses them."""

    def __init__(self, switches: str = ""):
        object.__setattr__(self, "_p", _Params())
        lib().pt_params_default(C.byref(self._p))
        if switches:
            self.set_from_switches(switches)

    def set_from_switches(self, switches: str) -> None:
        """Applies command-line switches ("-speed 3 -coherence_spatial 4"); every switch counts,
        as with PatchTableParams(argc, argv) whose argv[0] is the program name."""
        _check(lib().pt_params_from_switches(C.byref(self._p), ("patchtable " + switches).encode()))

    def set_speed(self, i: int) -> None:
        _check(lib().pt_params_set_speed(C.byref(self._p), int(i)))

    def set_schedule(self, sched) -> None:
        """GPU query schedule (passes, first jump, pull candidates[, k-coherence neighbours]):
        gpu_prop_passes, gpu_jump, gpu_pull_max and gpu_kc_max (0 when not given)."""
        self.gpu_prop_passes, self.gpu_jump, self.gpu_pull_max = (int(v) for v in sched[:3])
        self.gpu_kc_max = int(sched[3]) if len(sched) > 3 else 0

    @property
    def nslices(self):
        return [self._p.nslices[i] for i in range(self._p.n_nslices)]

    def __getattr__(self, name):
        p = object.__getattribute__(self, "_p")
        v = getattr(p, name)
        return v.decode() if isinstance(v, bytes) else v

    def __setattr__(self, name, value):
        if name == "nslices":
            self._p.n_nslices = len(value)
            for i, v in enumerate(value):
                self._p.nslices[i] = int(v)
            return
        if not hasattr(self._p, name):
            raise AttributeError(name)
        setattr(self._p, name, value.encode() if isinstance(value, str) else value)

    def as_dict(self) -> dict:
        d = {f: getattr(self, f) for f, _ in _Params._fields_ if f not in ("nslices", "n_nslices")}
        d["nslices"] = self.nslices
        return d


def schedule_name(sched) -> str:
    """passes/jump/pull candidates, plus /k-coherence neighbours when set (-1 = none)."""
    return "/".join(str(int(v)) for v in (sched if len(sched) > 3 and sched[3] else sched[:3]))


def _img(x, channels=3):
    x = np.ascontiguousarray(x, np.float32)
    if x.ndim != 3 or x.shape[2] != channels:
        raise PatchTableError(1, "expected an H x W x %d float image, got shape %s" % (channels, x.shape))
    return x


def _virtual(params, shape):
    """The image whose (h-7) x (w-7) patches an input covers: the image itself, or in descriptor
    mode the virtual image around its pixels (patchtable.h:2489-2507)."""
    if params.is_descriptor:
        d = -7 if params.descriptor_padded else 7
        return shape[0] + d, shape[1] + d
    return shape[0], shape[1]


class PatchTable:
    """PatchTable<float, float, int32_t> (patchtable/patchtable.h:4359-4491) on the GPU.

    With params.is_descriptor, b and the queries are H x W x C descriptor images (3 <= C <= 16;
    the table takes ndims = C) and the NNF has one record per pixel (per interior pixel with
    params.descriptor_padded: (H-14) x (W-14))."""

    def __init__(self, params: PatchTableParams, b, allowed_patches=None, wh0=None):
        b = np.asarray(b)
        b = _img(b, b.shape[2] if (params.is_descriptor and b.ndim == 3) else 3)
        self.params = params
        self.shape_b = b.shape
        h = C.c_void_p()
        al = None
        vh, vw = _virtual(params, b.shape)
        if allowed_patches is not None:
            allowed_patches = np.ascontiguousarray(allowed_patches, np.int32)
            if allowed_patches.shape != (vh - 7, vw - 7):
                raise PatchTableError(1, "allowed_patches must be %d x %d (one entry per patch)" % (vh - 7, vw - 7))
            al = allowed_patches.ctypes.data_as(C.c_void_p)
        if wh0 is None:
            _check(lib().pt_table_create(C.byref(params._p), b, b.shape[0], b.shape[1], b.shape[2], al, C.byref(h)))
        else:
            wh0 = np.ascontiguousarray(wh0, np.float32)
            _check(lib().pt_table_create_with_descriptor(C.byref(params._p), b, b.shape[0], b.shape[1], wh0, al, C.byref(h)))
        self._h = h
        self.last_seconds = 0.0
        self._set_shape()

    def _set_shape(self):
        hh, ww = C.c_int(), C.c_int()
        _check(lib().pt_table_image_shape(self._h, C.byref(hh), C.byref(ww)))
        self.shape_b = (hh.value, ww.value, 3)

    def save(self, filename: str) -> None:
        """PatchTable<>::save (patchtable.h:4470-4490), in the reference's file format."""
        _check(lib().pt_table_save(self._h, str(filename).encode()))

    @classmethod
    def load(cls, params: PatchTableParams, filename: str) -> "PatchTable":
        """PatchTableFixedN(p, filename): a table read from a file in the reference's format."""
        obj = cls.__new__(cls)
        obj.params = params
        h = C.c_void_p()
        _check(lib().pt_table_load(C.byref(params._p), str(filename).encode(), C.byref(h)))
        obj._h = h
        obj.last_seconds = 0.0
        obj._set_shape()
        return obj

    def sub_table(self, i: int) -> "PatchTable":
        """Further table i of a multi-table (ntables > 1) build, owned by this table."""
        h = C.c_void_p()
        _check(lib().pt_table_subtable(self._h, i, C.byref(h)))
        obj = PatchTable.__new__(PatchTable)
        obj.params = PatchTableParams()
        C.memmove(C.byref(obj.params._p), C.byref(self.params._p), C.sizeof(obj.params._p))
        obj.params.kcoherence = 0
        obj._h = h
        obj._owner = self
        obj.last_seconds = 0.0
        obj._set_shape()
        return obj

    def close(self) -> None:
        if getattr(self, "_owner", None) is not None:      # a further table belongs to its owner
            self._h = C.c_void_p()
            return
        if getattr(self, "_h", None) and self._h.value:
            lib().pt_table_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def lookup(self, a, ann_prev=None, coherence_temporal_sv=None, out=None):
        """PatchTable::lookup (patchtable.h:4448): returns the NNF (written into `out` when given,
        e.g. a pinned buffer); the wall time of the call (including a's descriptor, like the
        reference's return value) is in self.last_seconds."""
        a = np.asarray(a)
        a = _img(a, a.shape[2] if (self.params.is_descriptor and a.ndim == 3) else 3)
        vh, vw = _virtual(self.params, a.shape)
        shape = (vh - 7, vw - 7, 3)
        if out is not None:
            if out.shape != shape or out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]:
                raise PatchTableError(1, "out must be a C-contiguous float64 array of shape %s" % (shape,))
            ann = out
        else:
            ann = np.empty(shape, np.float64)
        secs = C.c_double()
        self._sync_params()
        prev_arr = sv_arr = None
        if ann_prev is not None:
            prev_arr = np.ascontiguousarray(ann_prev, np.float64)
            if prev_arr.shape != shape:
                raise PatchTableError(1, "ann_prev must have shape %s" % (shape,))
        if coherence_temporal_sv is not None:
            sv_arr = np.ascontiguousarray(coherence_temporal_sv, np.float32)
            if sv_arr.shape != shape[:2]:
                raise PatchTableError(1, "coherence_temporal_sv must have shape %s" % (shape[:2],))
        prev = None if prev_arr is None else prev_arr.ctypes.data_as(C.c_void_p)
        sv = None if sv_arr is None else sv_arr.ctypes.data_as(C.c_void_p)
        _check(lib().pt_table_lookup(self._h, a, a.shape[0], a.shape[1], ann, prev, sv, C.byref(secs)))
        self.last_seconds = secs.value
        return ann

    def _sync_params(self) -> None:
        # the reference's table reads the query fields of the caller's params on every lookup
        _check(lib().pt_table_set_params(self._h, C.byref(self.params._p)))

    def lookup_device(self, a_ptr: int, h: int, w: int, ann_ptr: int, stream: int = 0) -> None:
        """Device-resident lookup: a_ptr / ann_ptr are device addresses (e.g. torch data_ptr())."""
        self._sync_params()
        _check(lib().pt_table_lookup_device(self._h, C.c_void_p(a_ptr), h, w, C.c_void_p(ann_ptr), C.c_void_p(stream)))

    STAGES = ("descriptor", "cells", "init", "choose", "pull", "output")

    def lookup_profile(self, a_ptr: int, h: int, w: int, ann_ptr: int, stream: int = 0):
        """Device lookup with per-stage device times (ms) and SSD work counters."""
        ms = (C.c_double * 6)()
        ctr = (C.c_uint64 * 4)()
        self._sync_params()
        _check(lib().pt_table_lookup_profile(self._h, C.c_void_p(a_ptr), h, w, C.c_void_p(ann_ptr),
                                             C.c_void_p(stream), ms, ctr))
        return dict(zip(self.STAGES, list(ms))), dict(choose_cand=ctr[0], choose_rows=ctr[1],
                                                     pull_cand=ctr[2], pull_rows=ctr[3])

    # -- batches ---------------------------------------------------------------------------------
    def lookup_batch(self, images):
        """pt_table_lookup_batch: NNFs of several host images (any sizes) in one batched query."""
        imgs = [_img(x, np.shape(x)[2] if (self.params.is_descriptor and np.ndim(x) == 3) else 3) for x in images]
        n = len(imgs)
        if n == 0:
            return []
        outs = [np.empty((x.shape[0] - 7, x.shape[1] - 7, 3), np.float64) for x in imgs]
        A = (C.c_void_p * n)(*[x.ctypes.data for x in imgs])
        O = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        H = (C.c_int * n)(*[x.shape[0] for x in imgs])
        W = (C.c_int * n)(*[x.shape[1] for x in imgs])
        self._sync_params()
        _check(lib().pt_table_lookup_batch(self._h, n, A, H, W, O))
        return outs

    def batch(self, sizes):
        """A reusable device batch for images of the given (h, w) sizes (QueryBatch)."""
        return QueryBatch(self, sizes)

    # -- learned proposals (patchtable_b200.proposal.ProposalNet) -----------------------------
    def lookup_learned(self, a, net, out=None):
        """lookup() with the proposal network's candidates for confident patches."""
        a = _img(a)
        shape = (a.shape[0] - 7, a.shape[1] - 7, 3)
        if out is not None:
            if out.shape != shape or out.dtype != np.float64 or not out.flags["C_CONTIGUOUS"]:
                raise PatchTableError(1, "out must be a C-contiguous float64 array of shape %s" % (shape,))
            ann = out
        else:
            ann = np.empty(shape, np.float64)
        secs = C.c_double()
        self._sync_params()
        _check(lib().pt_table_lookup_learned(self._h, net.handle, a, a.shape[0], a.shape[1], ann, C.byref(secs)))
        self.last_seconds = secs.value
        return ann

    def lookup_learned_device(self, net, a_ptr: int, h: int, w: int, ann_ptr: int, stream: int = 0) -> None:
        self._sync_params()
        _check(lib().pt_table_lookup_learned_device(self._h, net.handle, C.c_void_p(a_ptr), h, w, C.c_void_p(ann_ptr),
                                                    C.c_void_p(stream)))

    LEARNED_STAGES = STAGES + ("proposal",)

    def lookup_learned_profile(self, net, a_ptr: int, h: int, w: int, ann_ptr: int, stream: int = 0):
        ms = (C.c_double * 7)()
        ctr = (C.c_uint64 * 6)()
        self._sync_params()
        _check(lib().pt_table_lookup_learned_profile(self._h, net.handle, C.c_void_p(a_ptr), h, w, C.c_void_p(ann_ptr),
                                                     C.c_void_p(stream), ms, ctr))
        return dict(zip(self.LEARNED_STAGES, list(ms))), dict(choose_cand=ctr[0], choose_rows=ctr[1], pull_cand=ctr[2],
                                                             pull_rows=ctr[3], confident=ctr[4], proposals=ctr[5])

    def lookup_proposed_profile(self, a_ptr: int, h: int, w: int, cand_ptr: int, conf_ptr: int, threshold: float,
                                ann_ptr: int, stream: int = 0, kcoh_confident: bool = False):
        """The learned query with caller-supplied proposals (device P x 8 table entries, P confidences)."""
        ms = (C.c_double * 7)()
        ctr = (C.c_uint64 * 6)()
        self._sync_params()
        _check(lib().pt_table_lookup_proposed_profile(self._h, C.c_void_p(a_ptr), h, w, C.c_void_p(cand_ptr),
                                                      C.c_void_p(conf_ptr), C.c_float(threshold), int(kcoh_confident),
                                                      C.c_void_p(ann_ptr), C.c_void_p(stream), ms, ctr))
        return dict(zip(self.LEARNED_STAGES, list(ms))), dict(choose_cand=ctr[0], choose_rows=ctr[1], pull_cand=ctr[2],
                                                             pull_rows=ctr[3], confident=ctr[4], proposals=ctr[5])

    def proposal_samples(self, a_ptr: int, h: int, w: int, ann_ptr: int, x_ptr: int, lab_ptr: int, stream: int = 0):
        """Training features (BF16 [P x 16]) and label bytes ([P x 8]) of a query image and its NNF."""
        _check(lib().pt_table_proposal_samples(self._h, C.c_void_p(a_ptr), h, w, C.c_void_p(ann_ptr), C.c_void_p(x_ptr),
                                               C.c_void_p(lab_ptr), C.c_void_p(stream)))

    def proposal_infer(self, net, a_ptr: int, h: int, w: int, cand_ptr: int, conf_ptr: int, logits_ptr: int = 0,
                       stream: int = 0):
        _check(lib().pt_table_proposal_infer(self._h, net.handle, C.c_void_p(a_ptr), h, w, C.c_void_p(cand_ptr),
                                             C.c_void_p(conf_ptr), C.c_void_p(logits_ptr or None), C.c_void_p(stream)))

    # -- introspection for parity tests --------------------------------------------------------
    def shape(self):
        ns = (C.c_int * PT_MAX_DIMS)()
        nc = C.c_int64()
        g = lib().pt_table_shape(self._h, ns, C.byref(nc))
        return [ns[i] for i in range(g)], nc.value

    def table(self):
        _, nc = self.shape()
        out = np.empty(nc, np.int32)
        _check(lib().pt_table_get_cells(self._h, out))
        return out

    def descriptor(self):
        H, W, _ = self.shape_b
        out = np.empty((H - 7, W - 7, self.params.ndims), np.float32)
        _check(lib().pt_table_get_descriptor(self._h, out))
        return out

    def partition(self, dim):
        ns, _ = self.shape()
        n = ns[dim]
        c, l, r = (np.empty(n, np.float32) for _ in range(3))
        tb = np.empty(16384, np.int32)
        mmr = np.empty(3, np.float32)
        _check(lib().pt_table_get_partition(self._h, dim, c, l, r, tb, mmr))
        return dict(centers=c, lsizes=l, rsizes=r, to_bin=tb, min=mmr[0], max=mmr[1], range=mmr[2])

    def kcoherence(self):
        H, W, _ = self.shape_b
        k = self.params.kcoherence
        pos = np.empty((H - 7) * (W - 7) * k, np.int32)
        dist = np.empty((H - 7) * (W - 7) * k, np.float32)
        _check(lib().pt_table_get_kcoherence(self._h, pos, dist))
        return pos.reshape(H - 7, W - 7, k), dist.reshape(H - 7, W - 7, k)

    def add_count(self) -> int:
        return int(lib().pt_table_add_count(self._h))

    def dt_levels(self) -> int:
        return int(lib().pt_table_dt_levels(self._h))

    def last_transfer(self):
        """(host->device bytes, device->host bytes) of the last host lookup."""
        h2d, d2h = C.c_int64(), C.c_int64()
        _check(lib().pt_table_last_transfer(self._h, C.byref(h2d), C.byref(d2h)))
        return int(h2d.value), int(d2h.value)

    BUILD_STAGES = ("descriptor", "kcoherence", "partition", "shuffle", "populate_dt", "total")

    def build_profile(self):
        """Wall-clock milliseconds of the build's stages (each ended with the stream drained)."""
        ms = (C.c_double * len(self.BUILD_STAGES))()
        _check(lib().pt_table_build_profile(self._h, ms, len(self.BUILD_STAGES)))
        return dict(zip(self.BUILD_STAGES, list(ms)))


class QueryBatch:
    """pt_batch: concatenated device buffers for a fixed list of query sizes against one table.

    Inputs and outputs are device addresses of the concatenated images (pixel_offset[i] RGB
    triples into the input) and NNFs (patch_offset[i] records into the output)."""

    def __init__(self, table: PatchTable, sizes):
        self.table = table
        self.sizes = [(int(h), int(w)) for h, w in sizes]
        n = len(self.sizes)
        H = (C.c_int * n)(*[h for h, _ in self.sizes])
        W = (C.c_int * n)(*[w for _, w in self.sizes])
        hb = C.c_void_p()
        _check(lib().pt_batch_create(table._h, n, H, W, C.byref(hb)))
        self._h = hb
        po = np.empty(n, np.int64)
        qo = np.empty(n, np.int64)
        tot = np.empty(2, np.int64)
        _check(lib().pt_batch_layout(hb, po.ctypes.data_as(C.c_void_p), qo.ctypes.data_as(C.c_void_p),
                                     tot.ctypes.data_as(C.c_void_p)))
        self.pixel_offset, self.patch_offset = po, qo
        self.pixels, self.patches = int(tot[0]), int(tot[1])

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().pt_batch_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def lookup(self, d_rgb: int, d_ann: int, stream: int = 0) -> None:
        self.table._sync_params()
        _check(lib().pt_batch_lookup(self._h, C.c_void_p(d_rgb), C.c_void_p(d_ann), C.c_void_p(stream)))

    def set_tile(self, patches_per_cta: int) -> None:
        _check(lib().pt_batch_set_tile(self._h, int(patches_per_cta)))

    @property
    def tile(self) -> int:
        return int(lib().pt_batch_tile(self._h))

    def autotune(self, d_rgb: int, d_ann: int, stream: int = 0):
        """(best patches per CTA, {patches per CTA: best ms of 3})."""
        self.table._sync_params()
        best = C.c_int()
        ms = (C.c_float * 4)()
        _check(lib().pt_batch_autotune(self._h, C.c_void_p(d_rgb), C.c_void_p(d_ann), C.c_void_p(stream), C.byref(best), ms))
        return best.value, dict(zip((32, 64, 128, 256), list(ms)))

    def capture(self, d_rgb: int, d_ann: int, stream: int = 0) -> None:
        self.table._sync_params()
        _check(lib().pt_batch_capture(self._h, C.c_void_p(d_rgb), C.c_void_p(d_ann), C.c_void_p(stream)))

    def replay(self, stream: int = 0) -> None:
        _check(lib().pt_batch_replay(self._h, C.c_void_p(stream)))


def descriptor(params: PatchTableParams, img):
    """Descriptor of every 8x8 patch of an RGB image, (h-7) x (w-7) x ndims."""
    img = _img(img)
    out = np.empty((img.shape[0] - 7, img.shape[1] - 7, params.ndims), np.float32)
    _check(lib().pt_descriptor(C.byref(params._p), img, img.shape[0], img.shape[1], out))
    return out


def set_host_threads(n: int) -> int:
    """Host threads that widen downloaded NNFs to float64 (n <= 0: default).  Returns the previous count."""
    return int(lib().pt_set_host_threads(int(n)))


def set_lean_kernels(on: bool) -> bool:
    """Specialised choose / pull variants (bit-identical to the general kernels); False runs the
    general kernels.  Returns the previous setting."""
    return bool(lib().pt_set_lean_kernels(1 if on else 0))


def set_spin_limit(polls: int) -> int:
    """Polls after which a device-side wait of the library gives up (PT_TIMEOUT); negative restores
    the default.  Returns the previous value."""
    return int(lib().pt_set_spin_limit(int(polls)))


def set_device_alloc_limit(nbytes: int) -> int:
    """Cap on the device memory the library holds (PT_OOM beyond it); negative removes the cap.
    Returns the previous cap."""
    return int(lib().pt_set_device_alloc_limit(int(nbytes)))


def device_bytes_in_use() -> int:
    return int(lib().pt_device_bytes_in_use())


def launch_count() -> int:
    return int(lib().pt_kernel_launch_count())


def reset_launch_count() -> None:
    lib().pt_kernel_launch_count_reset()
