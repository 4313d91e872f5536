"""ctypes front-ends of the CPU oracles (test infrastructure only).

``Oracle``     -- this repository's restatement (oracle/pt_oracle.cpp -> _build/libptoracle.so).
``Reference``  -- the reference's own sources compiled in place (oracle/_ref/libptref.so).

Both take numpy float32 H x W x 3 images in [0, 1] and return numpy arrays.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libptoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libptref.so")
REF_CLI = os.path.join(HERE, "_ref", "patchtable")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def _opt(arr, dtype):
    if arr is None:
        return None
    return np.ascontiguousarray(arr, dtype=dtype).ctypes.data_as(C.c_void_p)


class OrcParams(C.Structure):
    """Mirror of orc_params in pt_oracle.cpp."""
    _fields_ = [
        ("ndims", C.c_int), ("nchroma", C.c_int), ("grid_ndims", C.c_int),
        ("limit", C.c_double),
        ("nslices", C.c_int * 16), ("n_nslices", C.c_int),
        ("partition_step", C.c_int),
        ("populate_random", C.c_int),
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
        ("convert_colorspace", C.c_int),
        ("is_descriptor", C.c_int), ("descriptor_padded", C.c_int),
        ("ntables", C.c_int), ("table_ratio", C.c_double),
        ("dim_algo", C.c_int), ("pca_samples", C.c_int), ("pca_subtract_mean", C.c_int), ("pca_mean", C.c_int),
        ("colorspace", C.c_int),
    ]


#: Scalar fields of orc_params that carry the reference parameter of the same name.
PARAM_FIELDS = [f for f, _ in OrcParams._fields_ if f not in ("nslices", "n_nslices")]


def params_from_dict(d: dict) -> OrcParams:
    p = OrcParams()
    for f in PARAM_FIELDS:
        setattr(p, f, type(getattr(p, f))(d[f]))
    ns = d.get("nslices") or []
    p.n_nslices = len(ns)
    for i, v in enumerate(ns):
        p.nslices[i] = int(v)
    return p


class Oracle:
    """The restatement (oracle/pt_oracle.cpp)."""

    def __init__(self, path: str = ORACLE_SO):
        L = self.lib = C.CDLL(path)
        L.orc_build.restype = C.c_void_p
        L.orc_build.argtypes = [C.POINTER(OrcParams), _f32p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_table_shape.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
        L.orc_table_add_count.argtypes = [C.c_void_p]
        L.orc_kc_max_knn.argtypes = [C.c_void_p]
        L.orc_get_table.argtypes = [C.c_void_p, _i32p]
        L.orc_get_wh0.argtypes = [C.c_void_p, _f32p]
        L.orc_get_partition.argtypes = [C.c_void_p, C.c_int, _f32p, _f32p, _f32p, _i32p, _f32p]
        L.orc_get_kcoherence.argtypes = [C.c_void_p, _i32p, _f32p]
        L.orc_lookup.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, _f64p, C.c_void_p, C.c_void_p]
        L.orc_rgb2yuv.argtypes = [_f32p, C.c_int, C.c_int, _f32p]
        L.orc_rgb2lab.argtypes = [_f32p, C.c_int, C.c_int, _f32p]
        L.orc_gck.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        L.orc_descriptor.argtypes = [C.POINTER(OrcParams), _f32p, C.c_int, C.c_int, _f32p]
        L.orc_patch_dist.restype = C.c_float
        L.orc_patch_dist.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p, C.c_int, C.c_int, C.c_int]
        L.orc_subtable.restype = C.c_void_p
        L.orc_subtable.argtypes = [C.c_void_p, C.c_int]
        L.orc_patch_dist_approx.restype = C.c_float
        L.orc_patch_dist_approx.argtypes = [_f32p, _f32p, C.c_int]
        L.orc_scale_slices.argtypes = [_i32p, C.c_int, C.c_double, _i32p]
        L.orc_srand.argtypes = [C.c_uint]

    def srand(self, s: int = 1) -> None:
        self.lib.orc_srand(s)

    def rgb2yuv(self, img):
        img = np.ascontiguousarray(img, np.float32)
        out = np.empty_like(img)
        self.lib.orc_rgb2yuv(img, img.shape[0], img.shape[1], out)
        return out

    def rgb2lab(self, img):
        img = np.ascontiguousarray(img, np.float32)
        out = np.empty_like(img)
        self.lib.orc_rgb2lab(img, img.shape[0], img.shape[1], out)
        return out

    def gck(self, yuv, n: int, nchroma: int):
        yuv = np.ascontiguousarray(yuv, np.float32)
        h, w, _ = yuv.shape
        out = np.zeros((h + 7, w + 7, n + 2 * nchroma), np.float32)
        self.lib.orc_gck(yuv, h, w, n, nchroma, out)
        return out

    def descriptor(self, params: dict, img):
        img = np.ascontiguousarray(img, np.float32)
        h, w, _ = img.shape
        out = np.zeros((h + 7, w + 7, params["ndims"]), np.float32)
        p = params_from_dict(params)
        self.lib.orc_descriptor(C.byref(p), img, h, w, out)
        return out

    def patch_dist(self, a, ax, ay, b, bx, by) -> float:
        return self.lib.orc_patch_dist(a, a.shape[1], ax, ay, b, b.shape[1], bx, by)

    def patch_dist_approx(self, av, bv, nd: int) -> float:
        """Descriptor-mode distance of two vectors (each at least max(nd, 4) floats: with 3
        dimensions the fourth float takes part, as in the reference)."""
        return self.lib.orc_patch_dist_approx(np.ascontiguousarray(av, np.float32), np.ascontiguousarray(bv, np.float32), nd)

    def scale_slices(self, ns, limit):
        ns = np.ascontiguousarray(ns, np.int32)
        out = np.empty_like(ns)
        self.lib.orc_scale_slices(ns, len(ns), float(limit), out)
        return out

    def build(self, params: dict, b, allowed=None, wh0=None) -> "OracleTable":
        b = np.ascontiguousarray(b, np.float32)
        if params.get("is_descriptor"):
            # the reference's constructor takes ndims from the input and drops chroma (patchtable.h:4398-4401)
            params = dict(params, ndims=b.shape[2], nchroma=0)
        p = params_from_dict(params)
        h = self.lib.orc_build(C.byref(p), b, b.shape[0], b.shape[1], _opt(allowed, np.int32), _opt(wh0, np.float32))
        return OracleTable(self, h, params, b.shape)


def virtual_shape(params: dict, shape):
    """Image whose (h-7) x (w-7) patches the table or query covers: the image itself, or in
    descriptor mode the virtual image around the descriptors (patchtable.h:2489-2507)."""
    H, W = shape[0], shape[1]
    if params.get("is_descriptor"):
        return (H - 7, W - 7) if params.get("descriptor_padded") else (H + 7, W + 7)
    return (H, W)


class OracleTable:
    def __init__(self, orc: Oracle, handle, params, bshape):
        self.orc, self.h, self.params = orc, handle, params
        self.bshape = virtual_shape(params, bshape) + (3,)
        self.owner = None

    def sub_table(self, i: int) -> "OracleTable":
        """Further table i of an ntables > 1 build (owned by this table)."""
        h = self.orc.lib.orc_subtable(self.h, i)
        if not h:
            raise IndexError(i)
        sub = OracleTable.__new__(OracleTable)
        sub.orc, sub.h, sub.params, sub.bshape = self.orc, h, dict(self.params, kcoherence=0), self.bshape
        sub.owner = self
        return sub

    def __del__(self):
        if getattr(self, "owner", None) is not None:
            return
        if getattr(self, "h", None):
            self.orc.lib.orc_free(self.h)
            self.h = None

    def shape(self):
        ns = (C.c_int * 16)()
        nc = C.c_longlong()
        g = self.orc.lib.orc_table_shape(self.h, ns, C.byref(nc))
        return [ns[i] for i in range(g)], nc.value

    def add_count(self) -> int:
        return self.orc.lib.orc_table_add_count(self.h)

    def kc_max_knn(self) -> int:
        """Longest neighbour list (knn) the k-coherence search asked for."""
        return self.orc.lib.orc_kc_max_knn(self.h)

    def table(self):
        ns, nc = self.shape()
        out = np.empty(nc, np.int32)
        self.orc.lib.orc_get_table(self.h, out)
        return out

    def wh0(self):
        H, W, _ = self.bshape
        out = np.empty((H + 7, W + 7, self.params["ndims"]), np.float32)
        self.orc.lib.orc_get_wh0(self.h, out)
        return out

    def partition(self, dim):
        ns, _ = self.shape()
        n = ns[dim]
        c, l, r = (np.empty(n, np.float32) for _ in range(3))
        tb = np.empty(16384, np.int32)
        mmr = np.empty(3, np.float32)
        self.orc.lib.orc_get_partition(self.h, dim, c, l, r, tb, mmr)
        return dict(centers=c, lsizes=l, rsizes=r, to_bin=tb, min=mmr[0], max=mmr[1], range=mmr[2])

    def kcoherence(self):
        H, W, _ = self.bshape
        k = self.params["kcoherence"]
        pos = np.empty((H - 7) * (W - 7) * k, np.int32)
        dist = np.empty((H - 7) * (W - 7) * k, np.float32)
        self.orc.lib.orc_get_kcoherence(self.h, pos, dist)
        return pos.reshape(H - 7, W - 7, k), dist.reshape(H - 7, W - 7, k)

    def lookup(self, a, ann_prev=None, coh_sv=None):
        a = np.ascontiguousarray(a, np.float32)
        vh, vw = virtual_shape(self.params, a.shape)
        ann = np.zeros((vh - 7, vw - 7, 3), np.float64)
        self.orc.lib.orc_lookup(self.h, a, a.shape[0], a.shape[1], ann, _opt(ann_prev, np.float64), _opt(coh_sv, np.float32))
        return ann


class Reference:
    """The reference's own implementation (oracle/_ref/libptref.so)."""

    def __init__(self, path: str = REF_SO):
        L = self.lib = C.CDLL(path)
        L.ptref_create.restype = C.c_void_p
        L.ptref_create.argtypes = [C.c_char_p, _f32p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        L.ptref_free.argtypes = [C.c_void_p]
        L.ptref_lookup.restype = C.c_double
        L.ptref_lookup.argtypes = [C.c_void_p, _f32p, C.c_int, C.c_int, C.c_int, _f64p, C.c_void_p]
        L.ptref_table_shape.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int]
        L.ptref_table_add_count.argtypes = [C.c_void_p]
        L.ptref_get_table.argtypes = [C.c_void_p, _i32p]
        L.ptref_get_wh0.argtypes = [C.c_void_p, _f32p]
        L.ptref_get_partition.argtypes = [C.c_void_p, C.c_int, _f32p, _f32p, _f32p, _i32p, _f32p]
        L.ptref_get_kcoherence.argtypes = [C.c_void_p, _i32p, _f32p]
        L.ptref_gck.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        L.ptref_rgb2yuv.argtypes = [_f32p, C.c_int, C.c_int, _f32p]
        L.ptref_scale_slices.argtypes = [_i32p, C.c_int, C.c_double, _i32p]
        L.ptref_params_new.restype = C.c_void_p
        L.ptref_params_new.argtypes = [C.c_char_p]
        L.ptref_params_free.argtypes = [C.c_void_p]
        L.ptref_params_get.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double)]
        L.ptref_params_nslices.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int]
        L.ptref_srand.argtypes = [C.c_uint]
        L.ptref_set_threads.argtypes = [C.c_int]
        L.ptref_ndims.argtypes = [C.c_void_p]

    def srand(self, s: int = 1) -> None:
        self.lib.ptref_srand(s)

    def set_threads(self, n: int) -> None:
        self.lib.ptref_set_threads(n)

    def params(self, switches: str = "") -> dict:
        """Parameters as parsed by the reference (PatchTableParams(argc, argv))."""
        h = self.lib.ptref_params_new(switches.encode())
        out = {}
        v = C.c_double()
        for f in PARAM_FIELDS:
            if self.lib.ptref_params_get(h, f.encode(), C.byref(v)) == 0:
                is_int = dict(OrcParams._fields_)[f] is C.c_int
                out[f] = int(v.value) if is_int else v.value
        ns = (C.c_int * 16)()
        n = self.lib.ptref_params_nslices(h, ns, 16)
        out["nslices"] = [ns[i] for i in range(n)]
        self.lib.ptref_params_free(h)
        for f in PARAM_FIELDS:
            if f not in out:
                raise KeyError(f)
        return out

    def gck(self, yuv, n, nchroma):
        yuv = np.ascontiguousarray(yuv, np.float32)
        h, w, _ = yuv.shape
        out = np.zeros((h + 7, w + 7, n + 2 * nchroma), np.float32)
        self.lib.ptref_gck(yuv, h, w, n, nchroma, out)
        return out

    def rgb2yuv(self, img):
        img = np.ascontiguousarray(img, np.float32)
        out = np.empty_like(img)
        self.lib.ptref_rgb2yuv(img, img.shape[0], img.shape[1], out)
        return out

    def scale_slices(self, ns, limit):
        ns = np.ascontiguousarray(ns, np.int32)
        out = np.empty_like(ns)
        self.lib.ptref_scale_slices(ns, len(ns), float(limit), out)
        return out

    def build(self, switches: str, b, allowed=None, verbose: int = 0) -> "RefTable":
        b = np.ascontiguousarray(b, np.float32)
        secs = C.c_double()
        h = self.lib.ptref_create(switches.encode(), b, b.shape[0], b.shape[1], b.shape[2],
                                  _opt(allowed, np.int32), verbose, C.byref(secs))
        params = self.params(switches)
        t = RefTable(self, h, virtual_shape(params, b.shape) + (3,), params)
        t.build_seconds = secs.value
        return t


class RefTable:
    def __init__(self, ref: Reference, handle, bshape, params):
        self.ref, self.h, self.bshape, self.params = ref, handle, bshape, params
        self.ndims = ref.lib.ptref_ndims(handle)

    def __del__(self):
        if getattr(self, "h", None):
            self.ref.lib.ptref_free(self.h)
            self.h = None

    def shape(self):
        ns = (C.c_int * 16)()
        g = self.ref.lib.ptref_table_shape(self.h, ns, 16)
        ns = [ns[i] for i in range(g)]
        return ns, int(np.prod(ns, dtype=np.int64))

    def add_count(self) -> int:
        return self.ref.lib.ptref_table_add_count(self.h)

    def table(self):
        _, nc = self.shape()
        out = np.empty(nc, np.int32)
        self.ref.lib.ptref_get_table(self.h, out)
        return out

    def wh0(self):
        H, W, _ = self.bshape
        out = np.empty((H + 7, W + 7, self.ndims), np.float32)
        self.ref.lib.ptref_get_wh0(self.h, out)
        return out

    def partition(self, dim):
        ns, _ = self.shape()
        n = ns[dim]
        c, l, r = (np.empty(n, np.float32) for _ in range(3))
        tb = np.empty(16384, np.int32)
        mmr = np.empty(3, np.float32)
        self.ref.lib.ptref_get_partition(self.h, dim, c, l, r, tb, mmr)
        return dict(centers=c, lsizes=l, rsizes=r, to_bin=tb, min=mmr[0], max=mmr[1], range=mmr[2])

    def kcoherence(self):
        H, W, _ = self.bshape
        k = int(self.params["kcoherence"])
        pos = np.empty((H - 7) * (W - 7) * k, np.int32)
        dist = np.empty((H - 7) * (W - 7) * k, np.float32)
        self.ref.lib.ptref_get_kcoherence(self.h, pos, dist)
        return pos.reshape(H - 7, W - 7, k), dist.reshape(H - 7, W - 7, k)

    def lookup(self, a, ann_prev=None):
        a = np.ascontiguousarray(a, np.float32)
        vh, vw = virtual_shape(self.params, a.shape)
        ann = np.zeros((vh - 7, vw - 7, 3), np.float64)
        secs = self.ref.lib.ptref_lookup(self.h, a, a.shape[0], a.shape[1], a.shape[2], ann, _opt(ann_prev, np.float64))
        return ann, secs


def mean_dist(ann) -> float:
    """get_mean_dist, patchtable_main.cpp:90-101: mean of sqrt(max(d, 0))."""
    d = np.maximum(np.asarray(ann)[..., 2], 0.0)
    return float(np.sqrt(d).mean())


def recompute_dists(a, b, ann) -> np.ndarray:
    """Per-patch double-precision SSD of the NNF (recompute_mean_dist, patchtable_main.cpp:103-172,
    without clamping: callers check bounds first)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    bx = np.asarray(ann[..., 0]).astype(np.int64)
    by = np.asarray(ann[..., 1]).astype(np.int64)
    eh, ew = bx.shape
    ys, xs = np.mgrid[0:eh, 0:ew]
    d = np.zeros((eh, ew))
    for dy in range(8):
        for dx in range(8):
            diff = a[ys + dy, xs + dx] - b[by + dy, bx + dx]
            d += (diff * diff).sum(-1)
    return d


def recompute_mean_dist(a, b, ann) -> float:
    return float(np.sqrt(recompute_dists(a, b, ann)).mean())
