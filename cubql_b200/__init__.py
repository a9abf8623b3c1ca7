"""cubql_b200 -- B200-native BVH build-and-query (host side).

Python mirror of the cuBQL entry points for the BinaryBVH<float,3> path,
calling the CUDA library libbq.so through its C ABI (include/bq.h):

    cuBQL::gpuBuilder            -> gpuBuilder(boxes, BuildConfig)
    cuBQL::cuda::radixBuilder    -> cuda.radixBuilder(boxes, BuildConfig)
    cuBQL::cuda::rebinRadixBuilder -> cuda.rebinRadixBuilder(boxes, BuildConfig)
    cuBQL::cuda::free            -> cuda.free(bvh)
    gpuBuilder_impl::refit       -> refit(bvh, boxes)
    points::findClosest          -> points.findClosest(bvh, points, queries)
    points::findKNN              -> points.findKNN(bvh, points, queries, k)
    triangles::findClosest       -> triangles.findClosest(bvh, tris, verts, queries)
    (no reference counterpart)   -> triangles.distanceBackward(...)

Device memory, streams and tensors come from PyTorch; the work is done by
the sm_100a kernels of libbq.so.  There is no CPU fallback: importing
this package fails if libbq.so is missing.
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbq.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `python cubql_b200/build.py` "
                      "(there is no fallback implementation)")
_lib = ctypes.CDLL(LIB_PATH)

# ---------------------------------------------------------------------------
# constants (include/bq.h)
# ---------------------------------------------------------------------------
BQ_OK = 0
BQ_ERR_INVALID_ARGUMENT = 1
BQ_ERR_CUDA = 2
BQ_ERR_ALLOC = 3
BQ_ERR_STACK_OVERFLOW = 4
BQ_ERR_TIMEOUT = 5
BQ_ERR_UNSUPPORTED = 6
TIES_LOWEST_ID = 0
TIES_REFERENCE = 1


class BQError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libbq error {code}: {msg}")
        self.code = code


class bq_bvh3f(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_void_p), ("numNodes", ctypes.c_uint32),
                ("primIDs", ctypes.c_void_p), ("numPrims", ctypes.c_uint32)]


class bq_wide_bvh3f(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_void_p), ("numNodes", ctypes.c_uint32), ("primIDs", ctypes.c_void_p),
                ("numPrims", ctypes.c_uint32)]


class bq_build_config(ctypes.Structure):
    _fields_ = [("maxAllowedLeafSize", ctypes.c_int), ("makeLeafThreshold", ctypes.c_int),
                ("buildMethod", ctypes.c_int)]


MALLOC_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t,
                             ctypes.c_void_p)
FREE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)


class bq_allocator(ctypes.Structure):
    _fields_ = [("ctx", ctypes.c_void_p), ("malloc", MALLOC_FN), ("free", FREE_FN), ("scratchFromPool", ctypes.c_int)]


class bq_tuning(ctypes.Structure):
    _fields_ = [("makeLeafThreshold", ctypes.c_int), ("stackDepth", ctypes.c_int), ("blockSize", ctypes.c_int),
                ("queriesPerWarp", ctypes.c_int), ("buildMs", ctypes.c_float), ("queryMs", ctypes.c_float)]


class bq_query_config(ctypes.Structure):
    _fields_ = [("tieMode", ctypes.c_int), ("stackDepth", ctypes.c_int), ("blockSize", ctypes.c_int),
                ("reorder", ctypes.c_int), ("queriesPerWarp", ctypes.c_int), ("lanesPerQuery", ctypes.c_int)]


_P = ctypes.c_void_p
_U = ctypes.c_uint32
_I = ctypes.c_int
_F = ctypes.c_float
_SIGS = {
    "bq_build_morton63_f3": [ctypes.POINTER(bq_bvh3f), _P, _U, ctypes.POINTER(bq_build_config),
                             ctypes.POINTER(bq_allocator), _P],
    "bq_build_rebin_morton30_f3": [ctypes.POINTER(bq_bvh3f), _P, _U, ctypes.POINTER(bq_build_config),
                                   ctypes.POINTER(bq_allocator), _P],
    "bq_build_spatial_median_f3": [ctypes.POINTER(bq_bvh3f), _P, _U, ctypes.POINTER(bq_build_config),
                                   ctypes.POINTER(bq_allocator), _P],
    "bq_build_sah_f3": [ctypes.POINTER(bq_bvh3f), _P, _U, ctypes.POINTER(bq_build_config), ctypes.POINTER(bq_allocator),
                        _P],
    "bq_refit_f3": [ctypes.POINTER(bq_bvh3f), _P, ctypes.POINTER(bq_allocator), _P],
    "bq_refit_noalloc_f3": [ctypes.POINTER(bq_bvh3f), _P, _P],
    "bq_free_f3": [ctypes.POINTER(bq_bvh3f), ctypes.POINTER(bq_allocator), _P],
    "bq_closest_point_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _U, _F, ctypes.POINTER(bq_query_config), _P, _P,
                            ctypes.POINTER(bq_allocator), _P],
    "bq_closest_point_exclude_id_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _U, _P, _F, ctypes.POINTER(bq_query_config),
                                       _P, _P, ctypes.POINTER(bq_allocator), _P],
    "bq_closest_point_exclude_self_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _U, _F, ctypes.POINTER(bq_query_config),
                                         _P, _P, ctypes.POINTER(bq_allocator), _P],
    "bq_box_query_count_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _U, _P, ctypes.POINTER(bq_allocator), _P],
    "bq_box_query_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _U, _P, ctypes.c_uint64, _P, ctypes.POINTER(bq_allocator),
                        _P],
    "bq_box_query_slab_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _U, _U, _P, _P, _P, ctypes.POINTER(bq_allocator),
                             _P],
    "bq_box_query_gather_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _U, _U, _P, _P, _P, _P, ctypes.c_uint64, _P,
                               ctypes.POINTER(bq_allocator), _P],
    "bq_build_wide_f3": [ctypes.POINTER(bq_wide_bvh3f), _I, _P, _U, ctypes.POINTER(bq_build_config),
                         ctypes.POINTER(bq_allocator), _P],
    "bq_collapse_wide_f3": [ctypes.POINTER(bq_wide_bvh3f), _I, ctypes.POINTER(bq_bvh3f), ctypes.POINTER(bq_allocator),
                            _P],
    "bq_wide_free_f3": [ctypes.POINTER(bq_wide_bvh3f), ctypes.POINTER(bq_allocator), _P],
    "bq_wide_closest_point_f3": [ctypes.POINTER(bq_wide_bvh3f), _I, _P, _P, _U, _F, ctypes.POINTER(bq_query_config),
                                 _P, _P, ctypes.POINTER(bq_allocator), _P],
    "bq_wide_box_query_count_f3": [ctypes.POINTER(bq_wide_bvh3f), _I, _P, _P, _U, _P, ctypes.POINTER(bq_allocator),
                                   _P],
    "bq_wide_box_query_f3": [ctypes.POINTER(bq_wide_bvh3f), _I, _P, _P, _U, _P, ctypes.c_uint64, _P,
                             ctypes.POINTER(bq_allocator), _P],
    "bq_wide_box_query_slab_f3": [ctypes.POINTER(bq_wide_bvh3f), _I, _P, _P, _U, _U, _P, _P, _P,
                                  ctypes.POINTER(bq_allocator), _P],
    "bq_wide_box_query_gather_f3": [ctypes.POINTER(bq_wide_bvh3f), _I, _P, _P, _U, _U, _P, _P, _P, _P,
                                    ctypes.c_uint64, _P, ctypes.POINTER(bq_allocator), _P],
    "bq_knn_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _U, _I, _F, ctypes.POINTER(bq_query_config), _P, _P, _P,
                  ctypes.POINTER(bq_allocator), _P],
    "bq_tri_closest_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _P, _U, _F, ctypes.POINTER(bq_query_config), _P, _P, _P,
                          ctypes.POINTER(bq_allocator), _P],
    "bq_tri_distance_bwd_f3": [_P, _P, _U, _P, _U, _P, _P, _P, _P, ctypes.POINTER(bq_allocator), _P],
    "bq_query_visit_counts_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _U, _I, _F, ctypes.POINTER(bq_query_config),
                                 ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(bq_allocator), _P],
    "bq_tri_visit_counts_f3": [ctypes.POINTER(bq_bvh3f), _P, _P, _P, _U, _F, ctypes.POINTER(bq_query_config),
                               ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(bq_allocator), _P],
    "bq_batched_build_morton63_f3": [_P, _P, _U, _U, ctypes.POINTER(bq_build_config), _P, _P, _P, _P,
                                     ctypes.POINTER(bq_allocator), _P],
    "bq_batched_knn_f3": [_P, _P, _P, _P, _P, _U, _U, _I, _F, ctypes.POINTER(bq_query_config), _P, _P, _P, _P,
                          ctypes.POINTER(bq_allocator), _P],
    "bq_batched_refit_f3": [_P, _P, _U, _U, _P, _P, _P, ctypes.POINTER(bq_allocator), _P],
    "bq_batched_tri_closest_f3": [_P, _P, _P, _P, _P, _P, _U, _U, _F, ctypes.POINTER(bq_query_config), _P, _P, _P,
                                  _P, ctypes.POINTER(bq_allocator), _P],
    "bq_autotune_batched_knn_f3": [_P, _P, _P, _U, _U, _P, _P, _U, _I, _P, ctypes.POINTER(bq_allocator), _P],
    "bq_autotune_query_f3": [_P, _P, _U, _P, _U, _I, _P, ctypes.POINTER(bq_allocator), _P],
    "bq_tri_boxes_f3": [_P, _P, _U, _P, _P],
    "bq_points_to_boxes_f3": [_P, _U, _P, _P],
    "bq_load_binary": [ctypes.c_char_p, ctypes.c_size_t, _P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)],
    "bq_save_binary": [ctypes.c_char_p, _P, ctypes.c_uint64, ctypes.c_size_t],
    "bq_load_points_f64_as_f32": [ctypes.c_char_p, _I, _P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)],
    "bq_debug_inject_sort_timeout": [_I],
    "bq_last_error_string": [],
    "bq_version": [],
    "bq_profile_enable": [_I],
    "bq_profile_reset": [],
    "bq_profile_count": [],
    "bq_profile_entry": [_I, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_uint64),
                         ctypes.POINTER(ctypes.c_double)],
}
for _name, _args in _SIGS.items():
    _fn = getattr(_lib, _name)
    _fn.argtypes = _args
    _fn.restype = ctypes.c_char_p if _name == "bq_last_error_string" else ctypes.c_int


def exported_symbols():
    """Names of the C entry points this package binds."""
    return list(_SIGS)


def _check(code):
    if code != BQ_OK:
        raise BQError(code, _lib.bq_last_error_string().decode())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


# ---------------------------------------------------------------------------
# torch-backed allocator: every buffer libbq allocates is a torch tensor
# ---------------------------------------------------------------------------
class TorchAllocator:
    """bq_allocator whose blocks come from PyTorch's caching allocator.

    Blocks are uint8 CUDA tensors kept alive in `live` until libbq frees
    them; `view(ptr)` returns the tensor behind a pointer libbq handed out.
    Replaces cuBQL::GpuMemoryResource (cuBQL/builder/cuda.h:31-78)."""

    def __init__(self, device=None):
        self.device = torch.device(device or "cuda")
        self.live = {}
        self._m = MALLOC_FN(self._malloc)
        self._f = FREE_FN(self._free)
        # temporaries from libbq's stream-ordered pool; trees from torch
        self.c = bq_allocator(None, self._m, self._f, 1)

    def _malloc(self, ctx, out, size, stream):
        try:
            t = torch.empty(max(int(size), 1), dtype=torch.uint8, device=self.device)
        except Exception:  # out of memory: report through the status code
            return 1
        self.live[t.data_ptr()] = t
        out[0] = t.data_ptr()
        return 0

    def _free(self, ctx, ptr, stream):
        self.live.pop(ptr, None)
        return 0

    def view(self, ptr, dtype, count):
        base = self.live[ptr]
        return base[: count * torch.empty((), dtype=dtype).element_size()].view(dtype)


_default_alloc = {}


def default_allocator():
    dev = torch.cuda.current_device()
    if dev not in _default_alloc:
        _default_alloc[dev] = TorchAllocator(torch.device("cuda", dev))
    return _default_alloc[dev]


# ---------------------------------------------------------------------------
# BVH container (cuBQL/bvh.h:71-111)
# ---------------------------------------------------------------------------
class BuildConfig:
    """cuBQL::BuildConfig (cuBQL/bvh.h:31-64)."""
    SPATIAL_MEDIAN = 0
    SAH = 1
    ELH = 2

    def __init__(self, makeLeafThreshold=0, maxAllowedLeafSize=1 << 15, buildMethod=0):
        self.makeLeafThreshold = makeLeafThreshold
        self.maxAllowedLeafSize = maxAllowedLeafSize
        self.buildMethod = buildMethod

    def enableSAH(self):
        """BuildConfig::enableSAH (cuBQL/bvh.h:32)."""
        self.buildMethod = BuildConfig.SAH
        return self

    def enableELH(self):
        """BuildConfig::enableELH (cuBQL/bvh.h:33)."""
        self.buildMethod = BuildConfig.ELH
        return self

    def c(self):
        return bq_build_config(self.maxAllowedLeafSize, self.makeLeafThreshold, self.buildMethod)


NODE_DTYPE = None  # numpy structured dtype, set lazily


def node_dtype():
    import numpy as np
    global NODE_DTYPE
    if NODE_DTYPE is None:
        NODE_DTYPE = np.dtype([("lower", "<f4", 3), ("upper", "<f4", 3), ("admin", "<u8")])
        assert NODE_DTYPE.itemsize == 32
    return NODE_DTYPE


class BinaryBVH:
    """BinaryBVH<float,3>: nodes (32 B each) and primIDs in device memory."""

    def __init__(self, c, allocator):
        self.c = c
        self.allocator = allocator

    @property
    def numNodes(self):
        return self.c.numNodes

    @property
    def numPrims(self):
        return self.c.numPrims

    def nodes_tensor(self):
        """(numNodes, 8) float32 view: lower xyz, upper xyz, admin as 2 words."""
        if self.c.numNodes == 0:
            return torch.empty((0, 8), dtype=torch.float32, device="cuda")
        return self.allocator.view(self.c.nodes, torch.float32, 8 * self.c.numNodes).view(-1, 8)

    def primids_tensor(self):
        if self.c.numPrims == 0:
            return torch.empty((0,), dtype=torch.int32, device="cuda")
        return self.allocator.view(self.c.primIDs, torch.int32, self.c.numPrims)

    def to_host(self):
        """(nodes as a numpy structured array, primIDs as uint32)."""
        import numpy as np
        torch.cuda.synchronize()
        if self.c.numNodes == 0:
            return np.zeros(0, dtype=node_dtype()), np.zeros(0, dtype=np.uint32)
        nodes = self.nodes_tensor().cpu().numpy().view(node_dtype()).reshape(-1)
        prims = self.primids_tensor().cpu().numpy().view(np.uint32)
        return nodes, prims

    def free(self):
        if self.c.nodes or self.c.primIDs:
            _check(_lib.bq_free_f3(ctypes.byref(self.c), ctypes.byref(self.allocator.c), _stream()))


class WideBVH:
    """WideBVH<float,3,width>: numNodes wide nodes of `width` 32-byte slots
    (box + valid/offset/count word) and primIDs in device memory."""

    def __init__(self, c, width, allocator):
        self.c = c
        self.width = width
        self.allocator = allocator

    @property
    def numNodes(self):
        return self.c.numNodes

    @property
    def numPrims(self):
        return self.c.numPrims

    def to_host(self):
        """(slots as a numpy structured array of numNodes*width records whose
        `admin` field is the slot word, primIDs as uint32)."""
        import numpy as np
        torch.cuda.synchronize()
        if self.c.numNodes == 0:
            return np.zeros(0, dtype=node_dtype()), np.zeros(0, dtype=np.uint32)
        slots = self.allocator.view(self.c.nodes, torch.float32, 8 * self.width * self.c.numNodes)
        slots = slots.cpu().numpy().view(node_dtype()).reshape(-1)
        prims = self.allocator.view(self.c.primIDs, torch.int32, self.c.numPrims).cpu().numpy().view(np.uint32)
        return slots, prims

    def free(self):
        if self.c.nodes or self.c.primIDs:
            _check(_lib.bq_wide_free_f3(ctypes.byref(self.c), ctypes.byref(self.allocator.c), _stream()))


def _as_boxes(boxes):
    if boxes.dtype != torch.float32 or not boxes.is_cuda:
        raise TypeError("boxes must be a float32 CUDA tensor of shape (N, 6)")
    return boxes.contiguous().view(-1, 6)


def _build(fn, boxes, config, allocator):
    boxes = _as_boxes(boxes)
    allocator = allocator or default_allocator()
    cfg = (config or BuildConfig()).c()
    c = bq_bvh3f()
    _check(fn(ctypes.byref(c), _ptr(boxes), boxes.shape[0], ctypes.byref(cfg), ctypes.byref(allocator.c), _stream()))
    bvh = BinaryBVH(c, allocator)
    bvh._boxes = boxes  # keep the input alive for refits
    return bvh


def gpuBuilder(boxes, config=None, allocator=None):
    """cuBQL::gpuBuilder (cuBQL/builder/cuda.h:91-99): spatial-median build."""
    return _build(_lib.bq_build_spatial_median_f3, boxes, config, allocator)


def gpuBuilderWide(boxes, width=4, config=None, allocator=None):
    """cuBQL::gpuBuilder(WideBVH<float,3,width>&, ...) (cuBQL/builder/cuda.h:100-116,
    cuBQL/builder/cuda/wide_gpu_builder.h:162-213): spatial-median build
    collapsed to `width` (2, 4 or 8) children per node."""
    boxes = _as_boxes(boxes)
    allocator = allocator or default_allocator()
    cfg = (config or BuildConfig()).c()
    c = bq_wide_bvh3f()
    _check(_lib.bq_build_wide_f3(ctypes.byref(c), width, _ptr(boxes), boxes.shape[0], ctypes.byref(cfg),
                                 ctypes.byref(allocator.c), _stream()))
    return WideBVH(c, width, allocator)


def collapse(bvh, width=4):
    """bq_collapse_wide_f3: a WideBVH from any BinaryBVH (own primIDs copy)."""
    c = bq_wide_bvh3f()
    _check(_lib.bq_collapse_wide_f3(ctypes.byref(c), width, ctypes.byref(bvh.c), ctypes.byref(bvh.allocator.c),
                                    _stream()))
    return WideBVH(c, width, bvh.allocator)


def refit(bvh, boxes):
    """gpuBuilder_impl::refit (cuBQL/builder/cuda/sm_builder.h:677-693)."""
    boxes = _as_boxes(boxes)
    _check(_lib.bq_refit_f3(ctypes.byref(bvh.c), _ptr(boxes), ctypes.byref(bvh.allocator.c), _stream()))


class cuda:
    """cuBQL::cuda:: entry points."""

    @staticmethod
    def radixBuilder(boxes, config=None, allocator=None):
        """cuBQL::cuda::radixBuilder (cuBQL/builder/cuda.h:134-140), 63-bit keys."""
        return _build(_lib.bq_build_morton63_f3, boxes, config, allocator)

    @staticmethod
    def sahBuilder(boxes, config=None, allocator=None):
        """cuBQL::cuda::sahBuilder (cuBQL/builder/cuda.h:118-129): binned SAH."""
        return _build(_lib.bq_build_sah_f3, boxes, config, allocator)

    @staticmethod
    def rebinRadixBuilder(boxes, config=None, allocator=None):
        """cuBQL::cuda::rebinRadixBuilder (cuBQL/builder/cuda.h:143-154), 30-bit
        keys with rebinning of equal-key runs."""
        return _build(_lib.bq_build_rebin_morton30_f3, boxes, config, allocator)

    @staticmethod
    def free(bvh):
        """cuBQL::cuda::free (cuBQL/builder/cuda.h:158-161)."""
        bvh.free()


def query_config(tieMode=TIES_LOWEST_ID, stackDepth=64, blockSize=128, reorder=1, queriesPerWarp=32, lanesPerQuery=1):
    return bq_query_config(tieMode, stackDepth, blockSize, reorder, queriesPerWarp, lanesPerQuery)


def _vec3(t, name):
    if t.dtype != torch.float32 or not t.is_cuda:
        raise TypeError(f"{name} must be a float32 CUDA tensor of shape (N, 3)")
    return t.contiguous().view(-1, 3)


class points:
    @staticmethod
    def findClosest(bvh, data, queries, maxSqrDist=float("inf"), qcfg=None):
        """points::findClosest (cuBQL/queries/points/findClosest.h:336-360), batched.
        Returns (ids int32, sqrDist float32); -1 / inf where nothing is closer
        than maxSqrDist."""
        data, queries = _vec3(data, "points"), _vec3(queries, "queries")
        nq = queries.shape[0]
        ids = torch.empty(nq, dtype=torch.int32, device=queries.device)
        d = torch.empty(nq, dtype=torch.float32, device=queries.device)
        q = qcfg or query_config()
        if isinstance(bvh, WideBVH):  # findClosest(WideBVH) (findClosest.h:363-386)
            _check(_lib.bq_wide_closest_point_f3(ctypes.byref(bvh.c), bvh.width, _ptr(data), _ptr(queries), nq,
                                                 maxSqrDist, ctypes.byref(q), _ptr(ids), _ptr(d),
                                                 ctypes.byref(bvh.allocator.c), _stream()))
            return ids, d
        _check(_lib.bq_closest_point_f3(ctypes.byref(bvh.c), _ptr(data), _ptr(queries), nq, maxSqrDist,
                                        ctypes.byref(q), _ptr(ids), _ptr(d), ctypes.byref(bvh.allocator.c),
                                        _stream()))
        return ids, d

    @staticmethod
    def findClosest_exludeID(bvh, data, queries, excludeIds, maxSqrDist=float("inf"), qcfg=None):
        """points::findClosest_exludeID (cuBQL/queries/points/findClosest.h:278-305),
        batched: query q never returns prim excludeIds[q] (-1: no exclusion)."""
        data, queries = _vec3(data, "points"), _vec3(queries, "queries")
        nq = queries.shape[0]
        ex = excludeIds.to(device=queries.device, dtype=torch.int32).contiguous()
        if ex.numel() != nq:
            raise ValueError("excludeIds needs one entry per query")
        ids = torch.empty(nq, dtype=torch.int32, device=queries.device)
        d = torch.empty(nq, dtype=torch.float32, device=queries.device)
        q = qcfg or query_config()
        _check(_lib.bq_closest_point_exclude_id_f3(ctypes.byref(bvh.c), _ptr(data), _ptr(queries), nq, _ptr(ex),
                                                   maxSqrDist, ctypes.byref(q), _ptr(ids), _ptr(d),
                                                   ctypes.byref(bvh.allocator.c), _stream()))
        return ids, d

    @staticmethod
    def findClosest_exludeSelf(bvh, data, queries, maxSqrDist=float("inf"), qcfg=None):
        """points::findClosest_exludeSelf (cuBQL/queries/points/findClosest.h:307-334),
        batched: data points equal to the query are skipped."""
        data, queries = _vec3(data, "points"), _vec3(queries, "queries")
        nq = queries.shape[0]
        ids = torch.empty(nq, dtype=torch.int32, device=queries.device)
        d = torch.empty(nq, dtype=torch.float32, device=queries.device)
        q = qcfg or query_config()
        _check(_lib.bq_closest_point_exclude_self_f3(ctypes.byref(bvh.c), _ptr(data), _ptr(queries), nq, maxSqrDist,
                                                     ctypes.byref(q), _ptr(ids), _ptr(d),
                                                     ctypes.byref(bvh.allocator.c), _stream()))
        return ids, d

    @staticmethod
    def findKNN(bvh, data, queries, k, maxSqrDist=float("inf"), qcfg=None):
        """points::findKNN (cuBQL/queries/points/knn.h:75-116), batched.
        Returns (ids (nq,k) int32, sqrDist (nq,k) float32, numFound (nq,) int32)."""
        data, queries = _vec3(data, "points"), _vec3(queries, "queries")
        nq = queries.shape[0]
        ids = torch.empty((nq, k), dtype=torch.int32, device=queries.device)
        d = torch.empty((nq, k), dtype=torch.float32, device=queries.device)
        nf = torch.empty(nq, dtype=torch.int32, device=queries.device)
        q = qcfg or query_config()
        _check(_lib.bq_knn_f3(ctypes.byref(bvh.c), _ptr(data), _ptr(queries), nq, k, maxSqrDist, ctypes.byref(q),
                              _ptr(ids), _ptr(d), _ptr(nf), ctypes.byref(bvh.allocator.c), _stream()))
        return ids, d, nf

    @staticmethod
    def visitCounts(bvh, data, queries, k=0, maxSqrDist=float("inf"), qcfg=None):
        """Traversal visit counts of findClosest (k == 0) or findKNN (k > 0)
        over the queries, as the reference's buildQual / checkBuilders
        traversal-step counters: dict with the inner nodes expanded (two
        32-byte children loaded each), the node admin words loaded (16 B) and
        the prims tested."""
        data, queries = _vec3(data, "points"), _vec3(queries, "queries")
        out = (ctypes.c_uint64 * 3)()
        q = qcfg or query_config()
        _check(_lib.bq_query_visit_counts_f3(ctypes.byref(bvh.c), _ptr(data), _ptr(queries), queries.shape[0], k,
                                             maxSqrDist, ctypes.byref(q), out, ctypes.byref(bvh.allocator.c),
                                             _stream()))
        return {"inner_nodes": out[0], "admin_loads": out[1], "prims": out[2]}


class fixedBoxQuery:
    """cuBQL::fixedBoxQuery::forEachPrim (cuBQL/traversal/fixedBoxQuery.h:143-156)
    with a per-prim box test, batched over query boxes: the prims whose box
    overlaps each query box (closed intervals, cuBQL/math/box.h:208-212)."""

    @staticmethod
    def count(bvh, boxes, queryBoxes):
        """bq_box_query_count_f3: uint32 (nq,) number of overlapping prims."""
        boxes, queryBoxes = _as_boxes(boxes), _as_boxes(queryBoxes)
        nq = queryBoxes.shape[0]
        counts = torch.empty(nq, dtype=torch.int32, device=queryBoxes.device)
        if isinstance(bvh, WideBVH):
            _check(_lib.bq_wide_box_query_count_f3(ctypes.byref(bvh.c), bvh.width, _ptr(boxes), _ptr(queryBoxes), nq,
                                                   _ptr(counts), ctypes.byref(bvh.allocator.c), _stream()))
            return counts
        _check(_lib.bq_box_query_count_f3(ctypes.byref(bvh.c), _ptr(boxes), _ptr(queryBoxes), nq, _ptr(counts),
                                          ctypes.byref(bvh.allocator.c), _stream()))
        return counts

    @staticmethod
    def findPrims(bvh, boxes, queryBoxes, slabCap=None):
        """Returns (offsets int64 (nq+1,), ids int32); the prims of query q are
        ids[offsets[q]:offsets[q+1]] in the reference's visiting order
        (forEachLeaf: depth first, first child first).

        One traversal (bq_box_query_slab_f3, then bq_box_query_gather_f3): the
        first slabCap ids of every query are kept in a slab during it
        (default: up to 64 per query within 256 MB) and only queries with
        more are traversed again.  slabCap=0 runs the two-pass form
        (bq_box_query_count_f3, then bq_box_query_f3).  Same result."""
        boxes, queryBoxes = _as_boxes(boxes), _as_boxes(queryBoxes)
        nq = queryBoxes.shape[0]
        dev = queryBoxes.device
        wide = isinstance(bvh, WideBVH)
        if slabCap is None:
            slabCap = max(4, min(64, (1 << 26) // max(nq, 1)))
        if slabCap < 0:
            raise BQError(1, "slabCap must be >= 0")
        if slabCap == 0:
            counts = fixedBoxQuery.count(bvh, boxes, queryBoxes)
        else:
            slab = torch.empty(max(nq * slabCap, 1), dtype=torch.int32, device=dev)
            counts = torch.empty(max(nq, 1), dtype=torch.int32, device=dev)
            ovf = torch.empty(nq + 1, dtype=torch.int32, device=dev)
            if wide:
                _check(_lib.bq_wide_box_query_slab_f3(ctypes.byref(bvh.c), bvh.width, _ptr(boxes), _ptr(queryBoxes),
                                                      nq, slabCap, _ptr(slab), _ptr(counts), _ptr(ovf),
                                                      ctypes.byref(bvh.allocator.c), _stream()))
            else:
                _check(_lib.bq_box_query_slab_f3(ctypes.byref(bvh.c), _ptr(boxes), _ptr(queryBoxes), nq, slabCap,
                                                 _ptr(slab), _ptr(counts), _ptr(ovf), ctypes.byref(bvh.allocator.c),
                                                 _stream()))
            counts = counts[:nq]
        offsets = torch.zeros(nq + 1, dtype=torch.int64, device=dev)
        torch.cumsum(counts.to(torch.int64), 0, out=offsets[1:])
        total = int(offsets[-1].item())
        if total >= 1 << 32:
            raise BQError(1, "box query results exceed 2^32 entries")
        ids = torch.empty(max(total, 1), dtype=torch.int32, device=dev)
        off32 = offsets[:-1].to(torch.int32).contiguous()
        if slabCap == 0:
            if wide:
                _check(_lib.bq_wide_box_query_f3(ctypes.byref(bvh.c), bvh.width, _ptr(boxes), _ptr(queryBoxes), nq,
                                                 _ptr(off32), total, _ptr(ids), ctypes.byref(bvh.allocator.c),
                                                 _stream()))
            else:
                _check(_lib.bq_box_query_f3(ctypes.byref(bvh.c), _ptr(boxes), _ptr(queryBoxes), nq, _ptr(off32),
                                            total, _ptr(ids), ctypes.byref(bvh.allocator.c), _stream()))
        elif wide:
            _check(_lib.bq_wide_box_query_gather_f3(ctypes.byref(bvh.c), bvh.width, _ptr(boxes), _ptr(queryBoxes), nq,
                                                    slabCap, _ptr(slab), _ptr(counts), _ptr(ovf), _ptr(off32), total,
                                                    _ptr(ids), ctypes.byref(bvh.allocator.c), _stream()))
        else:
            _check(_lib.bq_box_query_gather_f3(ctypes.byref(bvh.c), _ptr(boxes), _ptr(queryBoxes), nq, slabCap,
                                               _ptr(slab), _ptr(counts), _ptr(ovf), _ptr(off32), total, _ptr(ids),
                                               ctypes.byref(bvh.allocator.c), _stream()))
        return offsets, ids[:total]


class triangles:
    @staticmethod
    def boxes(tris, verts):
        """Triangle::bounds() for every triangle (cuBQL/queries/triangles/Triangle.h:40-41)."""
        nt = tris.shape[0]
        out = torch.empty((nt, 6), dtype=torch.float32, device=verts.device)
        _check(_lib.bq_tri_boxes_f3(_ptr(tris.contiguous()), _ptr(verts.contiguous()), nt, _ptr(out), _stream()))
        return out

    @staticmethod
    def findClosest(bvh, tris, verts, queries, maxSqrDist=float("inf"), qcfg=None):
        """triangles::findClosest (cuBQL/queries/triangles/findClosest.h:132-152), batched.
        Returns (ids, sqrDist, P)."""
        queries = _vec3(queries, "queries")
        nq = queries.shape[0]
        ids = torch.empty(nq, dtype=torch.int32, device=queries.device)
        d = torch.empty(nq, dtype=torch.float32, device=queries.device)
        P = torch.empty((nq, 3), dtype=torch.float32, device=queries.device)
        q = qcfg or query_config()
        _check(_lib.bq_tri_closest_f3(ctypes.byref(bvh.c), _ptr(tris.contiguous()), _ptr(verts.contiguous()),
                                      _ptr(queries), nq, maxSqrDist, ctypes.byref(q), _ptr(ids), _ptr(d), _ptr(P),
                                      ctypes.byref(bvh.allocator.c), _stream()))
        return ids, d, P

    @staticmethod
    def visitCounts(bvh, tris, verts, queries, maxSqrDist=float("inf"), qcfg=None):
        """Traversal visit counts of findClosest over the queries (see
        points.visitCounts); 'prims' counts triangles tested."""
        queries = _vec3(queries, "queries")
        out = (ctypes.c_uint64 * 3)()
        q = qcfg or query_config()
        _check(_lib.bq_tri_visit_counts_f3(ctypes.byref(bvh.c), _ptr(tris.contiguous()), _ptr(verts.contiguous()),
                                           _ptr(queries), queries.shape[0], maxSqrDist, ctypes.byref(q), out,
                                           ctypes.byref(bvh.allocator.c), _stream()))
        return {"inner_nodes": out[0], "admin_loads": out[1], "prims": out[2]}

    @staticmethod
    def distanceBackward(tris, verts, queries, ids, gradSqr, allocator=None):
        """Adjoint of findClosest's squared distance (no reference counterpart).
        Returns (gradQueries (nq,3), gradVerts (nv,3))."""
        allocator = allocator or default_allocator()
        nq = queries.shape[0]
        nv = verts.shape[0]
        gq = torch.empty((nq, 3), dtype=torch.float32, device=queries.device)
        gv = torch.empty((nv, 3), dtype=torch.float32, device=queries.device)
        _check(_lib.bq_tri_distance_bwd_f3(_ptr(tris.contiguous()), _ptr(verts.contiguous()), nv,
                                           _ptr(queries.contiguous()), nq, _ptr(ids.contiguous()),
                                           _ptr(gradSqr.contiguous()), _ptr(gq), _ptr(gv), ctypes.byref(allocator.c),
                                           _stream()))
        return gq, gv


class Batch:
    """Many clouds built in one pass (bq_batched_build_morton63_f3).

    `boxes` (N,6) holds the clouds back to back; `offsets` (numSegs+1,)
    int32/uint32 gives each cloud's first box.  Every cloud's tree equals
    cuda.radixBuilder on that cloud alone; `tree(s)` views it as a
    BinaryBVH-like object.  Buffers are torch tensors owned by the batch."""

    def __init__(self, boxes, offsets, config=None, allocator=None, stream_alloc_null=False):
        boxes = _as_boxes(boxes)
        self.boxes = boxes
        self.offsets = offsets.to(device=boxes.device, dtype=torch.int32).contiguous()
        self.numSegs = self.offsets.numel() - 1
        n = boxes.shape[0]
        self.nodes = torch.empty((2 * max(n, 1), 8), dtype=torch.float32, device=boxes.device)
        self.primIDs = torch.empty(max(n, 1), dtype=torch.int32, device=boxes.device)
        self.bvhs = torch.empty((max(self.numSegs, 1), 4), dtype=torch.int64, device=boxes.device)
        self.err = torch.zeros(1, dtype=torch.int32, device=boxes.device)
        cfg = (config or BuildConfig()).c()
        alloc = None if stream_alloc_null else ctypes.byref((allocator or default_allocator()).c)
        _check(_lib.bq_batched_build_morton63_f3(_ptr(boxes), _ptr(self.offsets), self.numSegs, n, ctypes.byref(cfg),
                                                 _ptr(self.nodes), _ptr(self.primIDs), _ptr(self.bvhs),
                                                 _ptr(self.err), alloc, _stream()))

    def descriptors(self):
        """(numNodes, numPrims, nodeOffset, primOffset) per cloud, on the host."""
        torch.cuda.synchronize()
        d = self.bvhs.cpu().numpy()
        nodes_base = self.nodes.data_ptr()
        prim_base = self.primIDs.data_ptr()
        out = []
        for s in range(self.numSegs):
            p_nodes, nn_np = int(d[s, 0]), int(d[s, 1]) & 0xFFFFFFFF
            p_prims, npr = int(d[s, 2]), int(d[s, 3]) & 0xFFFFFFFF
            out.append((nn_np, npr, (p_nodes - nodes_base) // 32 if nn_np else 0,
                        (p_prims - prim_base) // 4 if npr else 0))
        return out

    def tree_host(self, s):
        """(nodes numpy structured array, primIDs uint32) of cloud s."""
        import numpy as np
        nn, npr, no, po = self.descriptors()[s]
        nodes = self.nodes[no: no + nn].cpu().numpy().view(node_dtype()).reshape(-1)
        prims = self.primIDs[po: po + npr].cpu().numpy().view(np.uint32)
        return nodes, prims


def batched_refit(batch, boxes, allocator=None, stream_alloc_null=False):
    """bq_batched_refit_f3: refit every tree of `batch` to new boxes."""
    boxes = _as_boxes(boxes)
    alloc = None if stream_alloc_null else ctypes.byref((allocator or default_allocator()).c)
    _check(_lib.bq_batched_refit_f3(_ptr(batch.bvhs), _ptr(batch.offsets), batch.numSegs, boxes.shape[0],
                                    _ptr(batch.nodes), _ptr(batch.primIDs), _ptr(boxes), alloc, _stream()))


def batched_tri_closest(batch, tris, verts, queries, queryOffsets, maxSqrDist=float("inf"), qcfg=None,
                        allocator=None, stream_alloc_null=False):
    """bq_batched_tri_closest_f3 over a Batch built on triangle boxes; returns
    (global triangle ids, sqrDist, P)."""
    queries = _vec3(queries, "queries")
    nq = queries.shape[0]
    ids = torch.empty(nq, dtype=torch.int32, device=queries.device)
    d = torch.empty(nq, dtype=torch.float32, device=queries.device)
    P = torch.empty((nq, 3), dtype=torch.float32, device=queries.device)
    qoff = queryOffsets.to(device=queries.device, dtype=torch.int32).contiguous()
    q = qcfg or query_config()
    alloc = None if stream_alloc_null else ctypes.byref((allocator or default_allocator()).c)
    _check(_lib.bq_batched_tri_closest_f3(_ptr(batch.bvhs), _ptr(batch.offsets), _ptr(tris.contiguous()),
                                          _ptr(verts.contiguous()), _ptr(queries), _ptr(qoff), batch.numSegs, nq,
                                          maxSqrDist, ctypes.byref(q), _ptr(ids), _ptr(d), _ptr(P), _ptr(batch.err),
                                          alloc, _stream()))
    return ids, d, P


def batched_knn(batch, points, pointOffsets, queries, queryOffsets, k, maxSqrDist=float("inf"), qcfg=None,
                allocator=None, stream_alloc_null=False):
    """bq_batched_knn_f3: ids are cloud-local.  Returns (ids, sqrDist, numFound)."""
    points, queries = _vec3(points, "points"), _vec3(queries, "queries")
    nq = queries.shape[0]
    ids = torch.empty((nq, k), dtype=torch.int32, device=queries.device)
    d = torch.empty((nq, k), dtype=torch.float32, device=queries.device)
    nf = torch.empty(nq, dtype=torch.int32, device=queries.device)
    poff = pointOffsets.to(device=queries.device, dtype=torch.int32).contiguous()
    qoff = queryOffsets.to(device=queries.device, dtype=torch.int32).contiguous()
    q = qcfg or query_config()
    alloc = None if stream_alloc_null else ctypes.byref((allocator or default_allocator()).c)
    _check(_lib.bq_batched_knn_f3(_ptr(batch.bvhs), _ptr(poff), _ptr(points), _ptr(queries), _ptr(qoff),
                                  batch.numSegs, nq, k, maxSqrDist, ctypes.byref(q), _ptr(ids), _ptr(d), _ptr(nf),
                                  _ptr(batch.err), alloc, _stream()))
    return ids, d, nf


def autotune_batched_knn(boxes, points, offsets, queries, queryOffsets, k):
    """bq_autotune_batched_knn_f3: the fastest (leaf, stack, block,
    queriesPerWarp) for this batch; returns a dict."""
    boxes = _as_boxes(boxes)
    points, queries = _vec3(points, "points"), _vec3(queries, "queries")
    off = offsets.to(device=boxes.device, dtype=torch.int32).contiguous()
    qoff = queryOffsets.to(device=boxes.device, dtype=torch.int32).contiguous()
    best = bq_tuning()
    _check(_lib.bq_autotune_batched_knn_f3(_ptr(boxes), _ptr(points), _ptr(off), off.numel() - 1, boxes.shape[0],
                                           _ptr(queries), _ptr(qoff), queries.shape[0], k, ctypes.byref(best), None,
                                           _stream()))
    return {f: getattr(best, f) for f, _ in bq_tuning._fields_}


def points_to_boxes(pts):
    """box3f().including(p) per point (testing/points/closestPoint.cu:22-29)."""
    pts = _vec3(pts, "points")
    out = torch.empty((pts.shape[0], 6), dtype=torch.float32, device=pts.device)
    _check(_lib.bq_points_to_boxes_f3(_ptr(pts), pts.shape[0], _ptr(out), _stream()))
    return out


class io:
    """The reference samples' binary-dump format (samples/common/IO.h:27-70):
    an 8-byte count, then the raw elements."""

    @staticmethod
    def loadBinary(path, dtype):
        """loadBinary<T>: a numpy array of `dtype` elements (a structured or
        sub-array dtype for vector types, e.g. ('<f8', 3) for vec3d)."""
        import numpy as np
        dt = np.dtype(dtype)
        n = ctypes.c_uint64()
        _check(_lib.bq_load_binary(os.fsencode(path), dt.itemsize, None, 0, ctypes.byref(n)))
        out = np.empty(n.value, dtype=dt)
        _check(_lib.bq_load_binary(os.fsencode(path), dt.itemsize, out.ctypes.data_as(ctypes.c_void_p), n.value,
                                   ctypes.byref(n)))
        return out

    @staticmethod
    def saveBinary(path, data):
        """saveBinary<T>: writes len(data) elements of data's dtype."""
        import numpy as np
        a = np.ascontiguousarray(data)
        item = a.dtype.itemsize * int(np.prod(a.shape[1:], dtype=np.int64))  # one row per element
        _check(_lib.bq_save_binary(os.fsencode(path), a.ctypes.data_as(ctypes.c_void_p), a.shape[0], item))

    @staticmethod
    def loadPoints(path, dims=3):
        """A vec_t<double,dims> point file as float32 (N, dims):
        loadBinary + convert<float,dims>."""
        import numpy as np
        n = ctypes.c_uint64()
        _check(_lib.bq_load_points_f64_as_f32(os.fsencode(path), dims, None, 0, ctypes.byref(n)))
        out = np.empty((n.value, dims), dtype=np.float32)
        _check(_lib.bq_load_points_f64_as_f32(os.fsencode(path), dims, out.ctypes.data_as(ctypes.c_void_p), n.value,
                                              ctypes.byref(n)))
        return out


def version():
    return _lib.bq_version()


class profile:
    """Phase profiler (CUDA events around every kernel phase of libbq calls
    made by this thread).  Usage:  with profile() as prof: ...;  prof.table
    maps phase name -> (launches, milliseconds)."""

    def __enter__(self):
        _check(_lib.bq_profile_reset())
        _check(_lib.bq_profile_enable(1))
        self.table = {}
        return self

    def __exit__(self, *exc):
        torch.cuda.synchronize()
        _check(_lib.bq_profile_enable(0))
        for i in range(_lib.bq_profile_count()):
            name, launches, ms = ctypes.c_char_p(), ctypes.c_uint64(), ctypes.c_double()
            _check(_lib.bq_profile_entry(i, ctypes.byref(name), ctypes.byref(launches), ctypes.byref(ms)))
            self.table[name.value.decode()] = (launches.value, ms.value)
        _check(_lib.bq_profile_reset())
        return False
