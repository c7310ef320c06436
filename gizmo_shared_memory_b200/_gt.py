"""ctypes binding of libgt.so (include/gt.h), the B200 tree-gravity library.

The binding is thin on purpose: every call goes straight to the C ABI that C/C++ callers use.
Host numpy arrays go through ``GT_MEM_HOST`` (the library copies in and out); torch CUDA tensors go
through ``GT_MEM_DEVICE`` with the context bound to torch's current stream, so library kernels and
torch work are ordered on one stream.  There is no CPU fallback: importing this module on a
machine where ``lib/libgt.so`` was not built raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgt.so")

GT_OK = 0
GT_MEM_HOST, GT_MEM_DEVICE = 0, 1
GT_KEY_PEANO, GT_KEY_MORTON = 0, 1
GT_GROUP_LEAF, GT_GROUP_BATCH, GT_GROUP_NODE, GT_GROUP_SINGLE = 0, 1, 2, 3
GT_MAC_PLAIN, GT_MAC_LEARNED, GT_MAC_NODE = 0, 1, 2
GT_MAC_NODE_FEATURES = (1 << 1) | (1 << 2) | (1 << 5)
GT_DIRECT_FP64, GT_DIRECT_FP32 = 0, 1
GT_OUT_TARGETS, GT_OUT_ORIGINAL = 0, 1
GT_NGB_GATHER, GT_NGB_REVERSE, GT_NGB_PAIRS = 0, 1, 2
GT_EVENT_HMAX = 6

STATUS = {0: "GT_OK", 1: "GT_ERR_INVALID", 2: "GT_ERR_CUDA", 3: "GT_ERR_NOMEM",
          4: "GT_ERR_UNSUPPORTED", 5: "GT_ERR_OVERFLOW", 6: "GT_ERR_TIMEOUT",
          7: "GT_ERR_NONFINITE", 8: "GT_ERR_DEVICE"}

# exported symbols declared in include/gt.h
EXPORTS = [
    "gt_version", "gt_status_string", "gt_build_options_default", "gt_walk_options_default",
    "gt_context_create", "gt_context_destroy", "gt_last_error", "gt_context_get_stream",
    "gt_context_set_stream", "gt_synchronize", "gt_launch_count", "gt_build", "gt_tree_free",
    "gt_tree_info_get", "gt_tree_download", "gt_tree_keys", "gt_accel_grouped", "gt_accel",
    "gt_potential", "gt_walk_stats_get", "gt_form_aold", "gt_direct", "gt_peano_keys",
    "gt_measure_peaks", "gt_direct_noalloc", "gt_mac_train_options_default", "gt_mac_sample",
    "gt_mac_train", "gt_mac_predict", "gt_mac_gradient", "gt_build_systems", "gt_tree_systems",
    "gt_plan_create", "gt_plan_launch", "gt_plan_destroy", "gt_tune_options_default", "gt_autotune",
    "gt_accel_grouped_ext", "gt_tree_velocities", "gt_tree_velocity_moments", "gt_tree_events",
    "gt_tree_refresh", "gt_tree_node_state", "gt_tree_particles", "gt_tree_gas",
    "gt_ngb_options_default", "gt_tree_hmax", "gt_ngb_search", "gt_density_options_default", "gt_density",
    "gt_direct_gas", "gt_mac_ceiling", "gt_tree_audit", "gt_ngb_count", "gt_ngb_counters_get",
]

GT_NGB_COUNTERS = 13


class GTError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class BuildOptions(C.Structure):
    _fields_ = [("key_mode", C.c_int), ("leaf_max", C.c_int), ("max_level", C.c_int),
                ("randomize_seed", C.c_longlong), ("nodelta", C.c_int), ("validate", C.c_int),
                ("shift", C.c_double * 3)]


class WalkOptions(C.Structure):
    _fields_ = [("group_mode", C.c_int), ("group_max", C.c_int), ("mac", C.c_int),
                ("out_order", C.c_int), ("async_", C.c_int), ("count", C.c_int),
                ("block_warps", C.c_int), ("list_capacity", C.c_int),
                ("stack_capacity", C.c_int), ("dtype_out_f32", C.c_int),
                ("mac_model", C.c_void_p), ("mac_kappa", C.c_double), ("mac_band", C.c_double * 2),
                ("sink_direct_radius", C.c_double), ("no_window_pairs", C.c_int)]


class TuneEntry(C.Structure):
    _fields_ = [("group_mode", C.c_int), ("group_size", C.c_int), ("block_warps", C.c_int),
                ("list_capacity", C.c_int), ("mac", C.c_int), ("mac_kappa", C.c_double),
                ("ms", C.c_double), ("p99", C.c_double), ("median", C.c_double), ("accepted", C.c_int)]


class TuneOptions(C.Structure):
    _fields_ = [("reps", C.c_int), ("p99_max", C.c_double), ("n_sample", C.c_int64),
                ("sample", C.c_void_p), ("ref_ax", C.c_void_p), ("ref_ay", C.c_void_p),
                ("ref_az", C.c_void_p), ("mac_model", C.c_void_p), ("n_kappa", C.c_int),
                ("kappa", C.c_void_p), ("mac_band", C.c_double * 2), ("mac_mode", C.c_int)]


class NgbOptions(C.Structure):
    _fields_ = [("mode", C.c_int), ("box", C.c_double), ("elapsed", C.c_double), ("n_gas", C.c_int64),
                ("h", C.c_void_p), ("systems", C.c_void_p)]


class DensityOptions(C.Structure):
    _fields_ = [("des_ngb", C.c_double), ("ngb_tol", C.c_double), ("box", C.c_double), ("elapsed", C.c_double),
                ("n_dims", C.c_int), ("face_correction", C.c_int), ("h_start", C.c_void_p),
                ("cond_prev", C.c_void_p)]


class MacTrainOptions(C.Structure):
    _fields_ = [("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_double), ("tau", C.c_double),
                ("seed", C.c_uint64), ("feature_mask", C.c_uint32)]


MAC_MODEL_FLOATS = 2 * 8 + 32 * 8 + 32 + 32 * 32 + 32 + 32 + 1
MAC_PARAM_FLOATS = MAC_MODEL_FLOATS - 16


class TreeInfo(C.Structure):
    _fields_ = [("n", C.c_int64), ("n_live", C.c_int64), ("n_nodes", C.c_int64),
                ("n_levels", C.c_int32), ("root", C.c_int32), ("center", C.c_double * 3),
                ("side", C.c_double), ("build_ms", C.c_double * 7), ("n_systems", C.c_int64)]


class WalkStats(C.Structure):
    _fields_ = [("groups", C.c_int64), ("nodes_visited", C.c_int64), ("multipole", C.c_int64),
                ("pairs", C.c_int64), ("targets", C.c_int64), ("max_stack", C.c_int64),
                ("list_flushes", C.c_int64), ("traversal_steps", C.c_int64), ("walk_ms", C.c_double)]


class NodeArrays(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("cx", "cy", "cz", "mass", "size", "delta", "soft", "gcx",
                                          "gcy", "gcz", "first", "next", "plo", "phi", "parent",
                                          "level", "w_s", "w_len", "w_soft")]


_LIB = None


def load_library(path: str = LIB_PATH):
    """Load libgt.so, declaring every entry point; raises if it was not built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with __graft_entry__.build() "
                           "(there is no CPU fallback)")
    L = C.CDLL(path)
    vp, i64, d = C.c_void_p, C.c_int64, C.c_double
    L.gt_version.restype = C.c_int
    L.gt_status_string.restype = C.c_char_p
    L.gt_status_string.argtypes = [C.c_int]
    L.gt_build_options_default.argtypes = [C.POINTER(BuildOptions)]
    L.gt_walk_options_default.argtypes = [C.POINTER(WalkOptions)]
    L.gt_context_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.gt_context_destroy.argtypes = [vp]
    L.gt_last_error.restype = C.c_char_p
    L.gt_last_error.argtypes = [vp]
    L.gt_context_get_stream.argtypes = [vp, C.POINTER(vp)]
    L.gt_context_set_stream.argtypes = [vp, vp]
    L.gt_synchronize.argtypes = [vp]
    L.gt_launch_count.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.gt_build.argtypes = [vp, i64, vp, vp, vp, vp, vp, C.c_int, C.POINTER(BuildOptions), C.POINTER(vp)]
    L.gt_build_systems.argtypes = [vp, i64, C.c_int32, vp, vp, vp, vp, vp, vp, C.c_int,
                                   C.POINTER(BuildOptions), C.POINTER(vp)]
    L.gt_tree_systems.argtypes = [vp, vp, vp]
    L.gt_tree_free.argtypes = [vp]
    L.gt_tree_info_get.argtypes = [vp, C.POINTER(TreeInfo)]
    L.gt_tree_download.argtypes = [vp, vp, vp, vp, vp, C.POINTER(NodeArrays)]
    L.gt_tree_keys.argtypes = [vp, vp, vp]
    L.gt_accel_grouped.argtypes = [vp, vp, i64, vp, vp, d, d, C.c_int, C.POINTER(WalkOptions),
                                   C.c_int, vp, vp, vp, vp]
    L.gt_accel.argtypes = [vp, vp, i64, vp, d, d, vp, C.c_int, vp, vp, vp]
    L.gt_accel_grouped_ext.argtypes = [vp, vp, i64, vp, vp, d, d, C.c_int, C.POINTER(WalkOptions),
                                       C.c_int, vp, vp, vp, vp, vp, vp]
    L.gt_tree_velocities.argtypes = [vp, vp, vp, vp, vp, C.c_int, C.c_int]
    L.gt_tree_velocity_moments.argtypes = [vp, vp, vp, vp, vp, vp]
    L.gt_tree_events.argtypes = [vp, vp, C.c_int, i64, vp, vp, vp, vp, vp, d, d, C.c_int]
    L.gt_tree_refresh.argtypes = [vp, vp, d]
    L.gt_tree_node_state.argtypes = [vp, vp, d, vp, vp, vp, vp, vp]
    L.gt_tree_particles.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.c_int]
    L.gt_tree_gas.argtypes = [vp, vp, vp, vp, C.c_int]
    L.gt_direct_gas.argtypes = [vp, i64, vp, vp, vp, vp, vp, vp, vp, i64, vp, d, C.c_int, vp, vp, vp]
    L.gt_ngb_options_default.restype = None
    L.gt_ngb_options_default.argtypes = [vp]
    L.gt_tree_hmax.argtypes = [vp, vp, vp, C.c_int64, C.c_int]
    L.gt_ngb_search.argtypes = [vp, vp, C.c_int64, vp, vp, vp, vp, vp, C.c_int, vp, vp, C.c_int64, vp]
    L.gt_density_options_default.restype = None
    L.gt_density_options_default.argtypes = [vp]
    L.gt_density.argtypes = [vp, vp, C.c_int64, vp, vp, C.c_int, vp, vp, vp, vp]
    L.gt_potential.argtypes = [vp, vp, i64, vp, d, d, vp, C.c_int, vp]
    L.gt_walk_stats_get.argtypes = [vp, C.POINTER(WalkStats)]
    L.gt_form_aold.argtypes = [vp, i64, vp, vp, vp, d, d, C.c_int, vp]
    L.gt_direct.argtypes = [vp, i64, vp, vp, vp, vp, vp, i64, vp, d, C.c_int, C.c_int, vp, vp, vp, vp]
    L.gt_peano_keys.argtypes = [vp, i64, vp, vp, vp, vp, d, C.c_int, C.c_int, vp, vp, vp, vp]
    L.gt_measure_peaks.argtypes = [vp, C.POINTER(d), C.POINTER(d)]
    L.gt_direct_noalloc.argtypes = [i64, vp, vp, vp, vp, vp, i64, vp, d, C.c_int, vp, vp, vp, vp, vp]
    L.gt_mac_train_options_default.argtypes = [C.POINTER(MacTrainOptions)]
    L.gt_mac_sample.argtypes = [vp, vp, vp, d, C.c_int, i64, d, d, i64, C.c_int, vp, vp, vp,
                                C.POINTER(i64)]
    L.gt_tree_audit.argtypes = [vp, vp, C.POINTER(i64), C.c_char_p, C.c_size_t]
    L.gt_ngb_count.argtypes = [vp, C.c_int]
    L.gt_ngb_counters_get.argtypes = [vp, vp, C.c_int]
    L.gt_mac_ceiling.argtypes = [vp, vp, vp, d, C.c_int, i64, vp, C.c_int, d, d, d, d, C.c_int, vp, vp, vp, vp]
    L.gt_mac_train.argtypes = [vp, i64, vp, vp, C.POINTER(MacTrainOptions), C.c_int, vp, C.POINTER(d)]
    L.gt_mac_predict.argtypes = [vp, vp, i64, vp, C.c_int, vp]
    L.gt_mac_gradient.argtypes = [vp, vp, i64, vp, vp, d, C.c_int, vp, C.POINTER(d)]
    L.gt_plan_create.argtypes = [vp, vp, vp, d, d, C.c_int, C.POINTER(WalkOptions), vp, vp, vp, vp,
                                 C.POINTER(vp)]
    L.gt_plan_launch.argtypes = [vp]
    L.gt_plan_destroy.argtypes = [vp]
    L.gt_tune_options_default.argtypes = [C.POINTER(TuneOptions)]
    L.gt_autotune.argtypes = [vp, vp, vp, C.c_int, d, d, C.POINTER(TuneOptions), C.POINTER(WalkOptions),
                              C.POINTER(C.c_int), vp, C.c_int, C.POINTER(C.c_int)]
    void_fns = ("gt_build_options_default", "gt_walk_options_default", "gt_mac_train_options_default",
                "gt_tune_options_default")
    for name in EXPORTS:
        getattr(L, name).restype = None if name in void_fns else C.c_int
    L.gt_last_error.restype = C.c_char_p
    L.gt_status_string.restype = C.c_char_p
    _LIB = L
    return L


def _ptr(a):
    """Address of a numpy array or torch tensor (or None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


def _is_dev(a):
    return a is not None and not isinstance(a, np.ndarray) and getattr(a, "is_cuda", False)


class Tree:
    def __init__(self, ctx: "Context", handle):
        self.ctx = ctx
        self.h = handle

    def free(self):
        if self.h:
            load_library().gt_tree_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def systems(self):
        """(live tree-position offsets [n_systems + 1], root cells [n_systems, 4]: centre, side)."""
        S = self.info()["n_systems"]
        off = np.zeros(S + 1, np.int64)
        roots = np.zeros((S, 4), np.float64)
        self.ctx._check(load_library().gt_tree_systems(self.h, off.ctypes.data, roots.ctypes.data))
        return off, roots

    def info(self) -> dict:
        inf = TreeInfo()
        self.ctx._check(load_library().gt_tree_info_get(self.h, C.byref(inf)))
        return {"n": inf.n, "n_live": inf.n_live, "n_nodes": inf.n_nodes, "n_levels": inf.n_levels,
                "center": tuple(inf.center), "side": inf.side, "n_systems": inf.n_systems,
                "build_ms": dict(zip(("bbox", "keys", "sort", "structure", "moments", "pack", "total"),
                                     list(inf.build_ms)))}

    @property
    def n_live(self):
        return self.info()["n_live"]

    def download(self, nodes=True):
        inf = self.info()
        n, nl, nn = inf["n"], inf["n_live"], inf["n_nodes"]
        ob = np.empty(nl, np.uint32)
        rank = np.empty(n, np.uint32)
        leaf = np.empty(n, np.int32)
        out = {"orderbuf": ob, "rank": rank, "leaf_of": leaf}
        na = None
        if nodes:
            arr = {}
            for k in ("cx", "cy", "cz", "mass", "size", "delta", "soft", "gcx", "gcy", "gcz", "w_s"):
                arr[k] = np.empty(nn)
            for k in ("first", "next", "plo", "phi", "parent", "level"):
                arr[k] = np.empty(nn, np.int32)
            arr["w_len"] = np.empty(nn, np.float32)
            arr["w_soft"] = np.empty(nn, np.float32)
            na = NodeArrays(**{k: v.ctypes.data for k, v in arr.items()})
            out.update(arr)
        L = load_library()
        self.ctx._check(L.gt_tree_download(self.ctx.h, self.h, ob.ctypes.data, rank.ctypes.data,
                                           leaf.ctypes.data, C.byref(na) if na else None))
        return out

    def keys(self):
        nl = self.info()["n_live"]
        k = np.empty(max(nl, 1), np.uint64)
        self.ctx._check(load_library().gt_tree_keys(self.ctx.h, self.h, k.ctypes.data))
        return k[:nl]


class Plan:
    """A captured all-active walk (gt_plan_create); launch() replays it asynchronously."""

    def __init__(self, ctx: "Context", handle, keep):
        self.ctx = ctx
        self.h = handle
        self._keep = keep  # the device arrays the graph points at

    def launch(self):
        self.ctx._check(load_library().gt_plan_launch(self.h))

    def free(self):
        if self.h:
            load_library().gt_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Context:
    """One gt_context (device, stream, workspace)."""

    def __init__(self, device: int = 0, torch_stream: bool = False):
        L = load_library()
        h = C.c_void_p()
        st = L.gt_context_create(device, C.byref(h))
        if st != GT_OK:
            raise GTError(st, f"gt_context_create(device={device})")
        self.h = h
        self.device = device
        if torch_stream:
            self.bind_torch_stream()

    def close(self):
        if getattr(self, "h", None):
            load_library().gt_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != GT_OK:
            msg = load_library().gt_last_error(self.h)
            raise GTError(st, msg.decode() if msg else "")

    def bind_torch_stream(self):
        import torch

        s = torch.cuda.current_stream(self.device)
        self._check(load_library().gt_context_set_stream(self.h, C.c_void_p(s.cuda_stream)))

    def synchronize(self):
        self._check(load_library().gt_synchronize(self.h))

    def launches(self) -> int:
        c = C.c_uint64()
        self._check(load_library().gt_launch_count(self.h, C.byref(c)))
        return int(c.value)

    def stats(self) -> dict:
        s = WalkStats()
        self._check(load_library().gt_walk_stats_get(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in WalkStats._fields_}

    # ---- build -----------------------------------------------------------------------------
    def build(self, P, key_mode=GT_KEY_PEANO, randomize_seed=-1, nodelta=False, leaf_max=16,
              max_level=20, validate=True, shift=(0.0, 0.0, 0.0), offsets=None) -> Tree:
        """Build a tree; with `offsets` (n_systems + 1 input offsets) a forest of independent
        systems in one pass (gt_build_systems)."""
        o = BuildOptions()
        load_library().gt_build_options_default(C.byref(o))
        o.key_mode = key_mode
        o.randomize_seed = randomize_seed
        o.nodelta = int(nodelta)
        o.leaf_max = leaf_max
        o.max_level = max_level
        o.validate = int(validate)
        for k in range(3):
            o.shift[k] = shift[k]
        x, y, z, m = P["x"], P["y"], P["z"], P["m"]
        soft = P.get("soft")
        dev = _is_dev(x)
        if not dev:
            x, y, z, m = (np.ascontiguousarray(a, np.float64) for a in (x, y, z, m))
            soft = None if soft is None else np.ascontiguousarray(soft, np.float64)
        h = C.c_void_p()
        mem = GT_MEM_DEVICE if dev else GT_MEM_HOST
        if offsets is None:
            self._check(load_library().gt_build(self.h, len(m), _ptr(x), _ptr(y), _ptr(z), _ptr(m),
                                                 _ptr(soft), mem, C.byref(o), C.byref(h)))
        else:
            off = np.ascontiguousarray(offsets, np.int64)
            self._check(load_library().gt_build_systems(self.h, len(m), len(off) - 1, off.ctypes.data,
                                                         _ptr(x), _ptr(y), _ptr(z), _ptr(m), _ptr(soft),
                                                         mem, C.byref(o), C.byref(h)))
        return Tree(self, h)

    # ---- walks -----------------------------------------------------------------------------
    def _walk_opts(self, group_mode=GT_GROUP_LEAF, group_max=32, out_order=GT_OUT_TARGETS,
                   count=False, block_warps=0, async_=False, mac=GT_MAC_PLAIN, mac_model=None, list_capacity=0,
                   mac_kappa=1.0, mac_band=(0.0, 0.0), sink_direct_radius=0.0, window_pairs=True):
        o = WalkOptions()
        load_library().gt_walk_options_default(C.byref(o))
        o.sink_direct_radius = sink_direct_radius
        o.no_window_pairs = 0 if window_pairs else 1
        o.group_mode = group_mode
        o.group_max = group_max
        o.out_order = out_order
        o.count = int(count)
        o.block_warps = block_warps
        o.list_capacity = list_capacity
        o.async_ = int(async_)
        o.mac = mac
        if mac_model is not None:
            self._mac_keep = np.ascontiguousarray(mac_model, np.float32)
            o.mac = mac if mac != GT_MAC_PLAIN else GT_MAC_LEARNED
            o.mac_model = self._mac_keep.ctypes.data
            o.mac_kappa = mac_kappa
            o.mac_band[0], o.mac_band[1] = mac_band
        return o

    # ---- plans and the autotuner ----------------------------------------------------------------
    def plan(self, tree: Tree, aold, outs, theta=0.0, G=1.0, batch=0, phi=None, **opts) -> Plan:
        """Capture the all-active walk into a graph; aold and outs = (ax, ay, az) are device
        tensors (n_live, tree order) whose contents may change between launches."""
        o = self._walk_opts(**opts)
        h = C.c_void_p()
        self._check(load_library().gt_plan_create(self.h, tree.h, _ptr(aold), theta, G, batch, C.byref(o),
                                                  _ptr(outs[0]), _ptr(outs[1]), _ptr(outs[2]), _ptr(phi),
                                                  C.byref(h)))
        return Plan(self, h, (tree, aold, outs, phi, o))

    def autotune(self, tree: Tree, aold, theta=0.0, G=1.0, sample=None, ref=None, p99_max=5e-3, reps=3,
                 mac_model=None, kappas=(), mac_band=(0.0, 0.0), mac=GT_MAC_LEARNED, max_entries=64):
        """Measure candidate launch configurations (gt_autotune).  Returns (walk options for
        accel_grouped as a dict, entries as a list of dicts)."""
        o = TuneOptions()
        L = load_library()
        L.gt_tune_options_default(C.byref(o))
        o.reps = reps
        o.p99_max = p99_max
        keep = []
        if sample is not None:
            smp = np.ascontiguousarray(sample, np.uint32)
            rx, ry, rz = (np.ascontiguousarray(r, np.float64) for r in ref)
            keep += [smp, rx, ry, rz]
            o.n_sample = len(smp)
            o.sample, o.ref_ax, o.ref_ay, o.ref_az = smp.ctypes.data, rx.ctypes.data, ry.ctypes.data, rz.ctypes.data
        if mac_model is not None:
            mm = np.ascontiguousarray(mac_model, np.float32)
            kp = np.ascontiguousarray(kappas, np.float64)
            keep += [mm, kp]
            o.mac_model = mm.ctypes.data
            o.n_kappa = len(kp)
            o.kappa = kp.ctypes.data
            o.mac_band[0], o.mac_band[1] = mac_band
            o.mac_mode = mac
        dev = _is_dev(aold)
        if not dev:
            aold = np.ascontiguousarray(aold, np.float64)
        best = WalkOptions()
        bb = C.c_int()
        ents = (TuneEntry * max_entries)()
        ne = C.c_int()
        self._check(L.gt_autotune(self.h, tree.h, _ptr(aold), GT_MEM_DEVICE if dev else GT_MEM_HOST, theta, G,
                                  C.byref(o), C.byref(best), C.byref(bb), ents, max_entries, C.byref(ne)))
        entries = [{k: getattr(e, k) for k, _ in TuneEntry._fields_} for e in ents[:ne.value]]
        opts = {"group_mode": best.group_mode, "group_max": best.group_max, "block_warps": best.block_warps,
                "list_capacity": best.list_capacity, "batch": bb.value}
        if best.mac != GT_MAC_PLAIN:
            opts.update(mac=best.mac, mac_model=mac_model, mac_kappa=best.mac_kappa, mac_band=tuple(mac_band))
        return opts, entries

    # ---- learned criterion ---------------------------------------------------------------------
    def mac_sample(self, tree: "Tree", amag, alpha, window=32, stride=1, rho_lo=0.02, rho_hi=50.0,
                   capacity=1 << 20):
        """Training samples from a plain walk; amag = |a| per live particle in tree order."""
        amag = np.ascontiguousarray(amag.cpu().numpy() if _is_dev(amag) else amag, np.float64)
        f = np.empty((capacity, 8), np.float32)
        lab = np.empty(capacity, np.float32)
        rho = np.empty(capacity, np.float32)
        ns = C.c_int64()
        self._check(load_library().gt_mac_sample(self.h, tree.h, _ptr(amag), alpha, window, stride,
                                                 rho_lo, rho_hi, capacity, GT_MEM_HOST, _ptr(f),
                                                 _ptr(lab), _ptr(rho), C.byref(ns)))
        k = min(ns.value, capacity)
        return f[:k], lab[:k], rho[:k], ns.value

    def mac_ceiling(self, tree: "Tree", amag, alpha, windows, window=32, mode=0, eps=0.0, band=(0.0, 0.0),
                    cost_exp=0.0):
        """The exact-label walk (gt_mac_ceiling) over the given window indices; amag = |a| per live
        particle in tree order.  Returns ((ax, ay, az), counts) with counts [n_windows, 5]: node
        visits, monopole and pair interactions, labelled nodes, particles summed for labels."""
        amag = np.ascontiguousarray(amag.cpu().numpy() if _is_dev(amag) else amag, np.float64)
        w = np.ascontiguousarray(windows, np.int64)
        ns = max(len(w) * window, 1)
        ax, ay, az = np.empty(ns), np.empty(ns), np.empty(ns)
        cnt = np.empty((max(len(w), 1), 5), np.int64)
        self._check(load_library().gt_mac_ceiling(self.h, tree.h, _ptr(amag), alpha, window, len(w), _ptr(w),
                                                  mode, eps, cost_exp, band[0], band[1], GT_MEM_HOST, _ptr(ax), _ptr(ay),
                                                  _ptr(az), _ptr(cnt)))
        k = len(w) * window
        return (ax[:k], ay[:k], az[:k]), cnt[:len(w)]

    def mac_train(self, features, labels, epochs=30, batch=4096, lr=2e-3, tau=0.9, seed=1, feature_mask=0xFF):
        o = MacTrainOptions(epochs=epochs, batch=batch, lr=lr, tau=tau, seed=seed, feature_mask=feature_mask)
        X = np.ascontiguousarray(features, np.float32)
        Y = np.ascontiguousarray(labels, np.float32)
        model = np.empty(MAC_MODEL_FLOATS, np.float32)
        loss = C.c_double()
        self._check(load_library().gt_mac_train(self.h, len(Y), _ptr(X), _ptr(Y), C.byref(o),
                                                GT_MEM_HOST, _ptr(model), C.byref(loss)))
        return model, loss.value

    def mac_predict(self, model, features):
        X = np.ascontiguousarray(features, np.float32)
        m = np.ascontiguousarray(model, np.float32)
        out = np.empty(max(len(X), 1), np.float32)
        self._check(load_library().gt_mac_predict(self.h, _ptr(m), len(X), _ptr(X), GT_MEM_HOST, _ptr(out)))
        return out[:len(X)]

    def mac_gradient(self, model, features, labels, tau=0.9):
        X = np.ascontiguousarray(features, np.float32)
        Y = np.ascontiguousarray(labels, np.float32)
        m = np.ascontiguousarray(model, np.float32)
        g = np.empty(MAC_PARAM_FLOATS, np.float32)
        loss = C.c_double()
        self._check(load_library().gt_mac_gradient(self.h, _ptr(m), len(Y), _ptr(X), _ptr(Y), tau,
                                                   GT_MEM_HOST, _ptr(g), C.byref(loss)))
        return g, loss.value

    @staticmethod
    def _targets(targets):
        if targets is None:
            return None, 0
        if _is_dev(targets):
            return targets, int(targets.numel())
        t = np.ascontiguousarray(targets, np.uint32)
        return t, len(t)

    def _outs(self, nout, dev, want_acc=True, want_phi=False, like=None):
        if dev:
            import torch

            mk = lambda: torch.empty(nout, dtype=torch.float64, device=like.device if like is not None
                                     else f"cuda:{self.device}")
        else:
            mk = lambda: np.empty(max(nout, 1), np.float64)
        ax = ay = az = phi = None
        if want_acc:
            ax, ay, az = mk(), mk(), mk()
        if want_phi:
            phi = mk()
        return ax, ay, az, phi

    def accel_grouped(self, tree: Tree, targets=None, aold=None, theta=0.0, G=1.0, batch=0,
                      want_phi=False, device_out=False, outs=None, **opts):
        t, nt = self._targets(targets)
        dev = _is_dev(t) or _is_dev(aold) or device_out or (outs is not None and _is_dev(outs[0]))
        if t is None:
            nt = tree.info()["n_live"] if opts.get("out_order", 0) == GT_OUT_TARGETS else tree.info()["n"]
        o = self._walk_opts(**opts)
        if outs is None:
            ax, ay, az, phi = self._outs(nt, dev, True, want_phi)
        else:
            ax, ay, az, phi = outs
        if not dev and aold is not None:
            aold = np.ascontiguousarray(aold, np.float64)
        self._check(load_library().gt_accel_grouped(
            self.h, tree.h, nt if targets is not None else 0, _ptr(t), _ptr(aold), theta, G, batch,
            C.byref(o), GT_MEM_DEVICE if dev else GT_MEM_HOST, _ptr(ax), _ptr(ay), _ptr(az), _ptr(phi)))
        if not dev:
            ax, ay, az = ax[:nt], ay[:nt], az[:nt]
            phi = phi[:nt] if phi is not None else None
        return (ax, ay, az, phi) if want_phi else (ax, ay, az)

    def accel_grouped_ext(self, tree: Tree, targets=None, aold=None, theta=0.0, G=1.0, batch=0, tidal=True,
                          jerk=False, want_phi=False, outs=None, **opts):
        """Grouped walk with the tidal tensor ([nt, 6]: xx yy zz xy yz xz, not times G) and the
        jerk ([nt, 3]); host arrays.  Returns (ax, ay, az, phi, tidal, jerk).  With outs =
        (ax, ay, az, phi, tidal, jerk) device tensors (any may be None) the walk writes them on the
        device; targets and aold are then device tensors or None."""
        if outs is not None:
            o = self._walk_opts(**opts)
            t, nt = self._targets(targets)
            if t is None:
                nt = tree.info()["n_live"]
            self._check(load_library().gt_accel_grouped_ext(
                self.h, tree.h, nt if targets is not None else 0, _ptr(t), _ptr(aold), theta, G, batch, C.byref(o),
                GT_MEM_DEVICE, *[_ptr(x) for x in outs]))
            return outs
        t, nt = self._targets(targets)
        if t is None:
            nt = tree.info()["n_live"] if opts.get("out_order", 0) == GT_OUT_TARGETS else tree.info()["n"]
        o = self._walk_opts(**opts)
        ax, ay, az, phi = self._outs(nt, False, True, want_phi)
        tt = np.empty((max(nt, 1), 6)) if tidal else None
        jj = np.empty((max(nt, 1), 3)) if jerk else None
        ao = np.ascontiguousarray(aold, np.float64) if aold is not None else None
        self._check(load_library().gt_accel_grouped_ext(
            self.h, tree.h, nt if targets is not None else 0, _ptr(t), _ptr(ao), theta, G, batch, C.byref(o),
            GT_MEM_HOST, _ptr(ax), _ptr(ay), _ptr(az), _ptr(phi), _ptr(tt), _ptr(jj)))
        cut = lambda a: None if a is None else a[:nt]
        return cut(ax), cut(ay), cut(az), cut(phi), cut(tt), cut(jj)

    def tree_audit(self, tree: Tree):
        """gt_tree_audit: (number of violations, the first one's message)."""
        nb = C.c_int64()
        buf = C.create_string_buffer(512)
        self._check(load_library().gt_tree_audit(self.h, tree.h, C.byref(nb), buf, 512))
        return nb.value, buf.value.decode()

    def tree_velocities(self, tree: Tree, vx, vy, vz, particles_only=False):
        """Attach velocities (indexed like the build input): node vcom and vmax, for the jerk."""
        dev = _is_dev(vx)
        if not dev:
            vx, vy, vz = (np.ascontiguousarray(a, np.float64) for a in (vx, vy, vz))
        self._check(load_library().gt_tree_velocities(self.h, tree.h, _ptr(vx), _ptr(vy), _ptr(vz),
                                                      int(particles_only), GT_MEM_DEVICE if dev else GT_MEM_HOST))

    # ---- tree reuse ---------------------------------------------------------------------------
    def tree_events(self, tree: Tree, kind, leaf, a=None, x=None, v=None, f=None, tau=0.0, box=0.0):
        """Events of one kind (GT_EVENT_*: 0 kick, 1 shift, 2 vmax, 3 soft, 4 mass, 5 pad, 6 hmax) on
        leaf nodes of this tree: host arrays, or device tensors (int32 leaves, float64 a, x, v,
        float32 f)."""
        if _is_dev(leaf):
            self._check(load_library().gt_tree_events(self.h, tree.h, kind, int(leaf.numel()), _ptr(leaf), _ptr(a),
                                                      _ptr(x), _ptr(v), _ptr(f), tau, box, GT_MEM_DEVICE))
            return
        lf = np.ascontiguousarray(leaf, np.int32)
        cv = lambda q, dt: None if q is None else np.ascontiguousarray(q, dt)
        a, x, v, f = cv(a, np.float64), cv(x, np.float64), cv(v, np.float64), cv(f, np.float32)
        self._check(load_library().gt_tree_events(self.h, tree.h, kind, len(lf), _ptr(lf), _ptr(a), _ptr(x),
                                                  _ptr(v), _ptr(f), tau, box, GT_MEM_HOST))

    def tree_refresh(self, tree: Tree, tau):
        self._check(load_library().gt_tree_refresh(self.h, tree.h, tau))

    def tree_node_state(self, tree: Tree, tau):
        nn = max(tree.info()["n_nodes"], 1)
        out = {"com": np.empty((nn, 3)), "vel": np.empty((nn, 3)), "mass": np.empty(nn),
               "vmax": np.empty(nn, np.float32), "xpad": np.empty(nn, np.float32)}
        self._check(load_library().gt_tree_node_state(self.h, tree.h, tau, _ptr(out["com"]), _ptr(out["vel"]),
                                                      _ptr(out["mass"]), _ptr(out["vmax"]), _ptr(out["xpad"])))
        return out

    def tree_particles(self, tree: Tree, x=None, y=None, z=None, m=None, soft=None):
        """The particles' current state (indexed like the build input; None keeps a field): host
        arrays or device tensors."""
        if any(_is_dev(q) for q in (x, y, z, m, soft)):
            self._check(load_library().gt_tree_particles(self.h, tree.h, _ptr(x), _ptr(y), _ptr(z), _ptr(m),
                                                         _ptr(soft), GT_MEM_DEVICE))
            return
        cv = lambda q: None if q is None else np.ascontiguousarray(q, np.float64)
        x, y, z, m, soft = (cv(q) for q in (x, y, z, m, soft))
        self._check(load_library().gt_tree_particles(self.h, tree.h, _ptr(x), _ptr(y), _ptr(z), _ptr(m),
                                                     _ptr(soft), GT_MEM_HOST))

    def tree_gas(self, tree: Tree, type=None, zeta=None):
        """Attach particle types (uint8, GIZMO numbering: 0 gas, 5 sink; None = all gas) and the
        adaptive-softening zeta (None = none), indexed like the build input: walks returning
        accelerations then apply the zeta terms of gas-gas pairs, and sink_direct_radius > 0 in
        the walk options turns on sink-direct opening.  Host arrays or device tensors."""
        dev = _is_dev(type) or _is_dev(zeta)
        if not dev:
            type = None if type is None else np.ascontiguousarray(type, np.uint8)
            zeta = None if zeta is None else np.ascontiguousarray(zeta, np.float64)
        self._check(load_library().gt_tree_gas(self.h, tree.h, _ptr(type), _ptr(zeta),
                                               GT_MEM_DEVICE if dev else GT_MEM_HOST))

    # ---- neighbour search and the density solve ------------------------------------------------
    def tree_hmax(self, tree: Tree, h, n_gas):
        """Tree::init_hmax: per-node largest support radius of the gas particles [0, n_gas)."""
        dev = _is_dev(h)
        if not dev:
            h = np.ascontiguousarray(h, np.float64)
        self._check(load_library().gt_tree_hmax(self.h, tree.h, _ptr(h), int(n_gas),
                                                GT_MEM_DEVICE if dev else GT_MEM_HOST))

    def ngb_search(self, tree: Tree, cx, cy, cz, radius, mode=GT_NGB_GATHER, h=None, n_gas=0, box=0.0,
                   elapsed=0.0, systems=None):
        """Neighbour lists as CSR (start [n+1] int64, found uint32 particle indices), host arrays.
        On a forest, systems (per centre) names the one system each centre searches; None: all."""
        cx, cy, cz, radius = (np.ascontiguousarray(a, np.float64) for a in (cx, cy, cz, radius))
        o = NgbOptions()
        L = load_library()
        L.gt_ngb_options_default(C.byref(o))
        o.mode, o.box, o.elapsed, o.n_gas = mode, box, elapsed, int(n_gas)
        hh = None if h is None else np.ascontiguousarray(h, np.float64)
        o.h = _ptr(hh)
        ss = None if systems is None else np.ascontiguousarray(systems, np.int32)
        o.systems = _ptr(ss)
        n = len(cx)
        start = np.zeros(n + 1, np.int64)
        tot = C.c_int64(0)
        # one call with room for 48 neighbours per centre; a second, sized, call if that overflows
        found = np.empty(max(48 * n, 1024), np.uint32)
        st = L.gt_ngb_search(self.h, tree.h, n, _ptr(cx), _ptr(cy), _ptr(cz), _ptr(radius), C.byref(o),
                             GT_MEM_HOST, _ptr(start), _ptr(found), len(found), C.byref(tot))
        if st == 5:  # GT_ERR_OVERFLOW: start and the total are filled
            found = np.empty(max(tot.value, 1), np.uint32)
            st = L.gt_ngb_search(self.h, tree.h, n, _ptr(cx), _ptr(cy), _ptr(cz), _ptr(radius), C.byref(o),
                                 GT_MEM_HOST, _ptr(start), _ptr(found), len(found), C.byref(tot))
        self._check(st)
        return start, found[: tot.value]

    def density(self, tree: Tree, targets, des_ngb=32.0, ngb_tol=0.05, h_start=None, box=0.0, n_dims=3,
                cond_prev=None, face_correction=True, elapsed=0.0):
        """shmem::density on the GPU: dict of h, rho, nngb, iters per target.  Host arrays, or,
        when targets is a CUDA tensor, device tensors throughout (h_start and cond_prev too)."""
        dev = _is_dev(targets)
        o = DensityOptions()
        L = load_library()
        L.gt_density_options_default(C.byref(o))
        o.des_ngb, o.ngb_tol, o.box, o.n_dims = des_ngb, ngb_tol, box, n_dims
        o.face_correction, o.elapsed = int(face_correction), elapsed
        if dev:
            import torch

            t, hs, cp = targets, h_start, cond_prev
            nt = int(t.numel())
            h = torch.empty(nt, dtype=torch.float64, device=t.device)
            rho = torch.empty_like(h)
            nngb = torch.empty(nt, dtype=torch.int32, device=t.device)
            iters = torch.empty_like(nngb)
        else:
            t = np.ascontiguousarray(targets, np.uint32)
            nt = len(t)
            hs = None if h_start is None else np.ascontiguousarray(h_start, np.float64)
            cp = None if cond_prev is None else np.ascontiguousarray(cond_prev, np.float64)
            h, rho = np.zeros(nt), np.zeros(nt)
            nngb, iters = np.zeros(nt, np.int32), np.zeros(nt, np.int32)
        o.h_start, o.cond_prev = _ptr(hs), _ptr(cp)
        self._check(L.gt_density(self.h, tree.h, nt, _ptr(t), C.byref(o), GT_MEM_DEVICE if dev else GT_MEM_HOST,
                                 _ptr(h), _ptr(rho), _ptr(nngb), _ptr(iters)))
        return {"h": h, "rho": rho, "nngb": nngb, "iters": iters}

    def ngb_count(self, enable=True):
        """SHMEM_NGB_COUNT on this context: tally the gather searches and density solves."""
        self._check(load_library().gt_ngb_count(self.h, int(bool(enable))))

    def ngb_counters(self, reset=False):
        """The tallies: dict of calls, nodes, examined, kept, pad_nodes and the iteration histogram
        hiter[8] (slot i: targets that took i + 1 iterations; the last, 8 or more)."""
        v = np.zeros(GT_NGB_COUNTERS, np.int64)
        self._check(load_library().gt_ngb_counters_get(self.h, _ptr(v), int(bool(reset))))
        names = ("calls", "nodes", "examined", "kept", "pad_nodes")
        out = {k: int(v[i]) for i, k in enumerate(names)}
        out["hiter"] = v[5:].copy()
        return out

    def velocity_moments(self, tree: Tree):
        nn = tree.info()["n_nodes"]
        v = [np.empty(max(nn, 1)) for _ in range(3)]
        vmax = np.empty(max(nn, 1), np.float32)
        self._check(load_library().gt_tree_velocity_moments(self.h, tree.h, _ptr(v[0]), _ptr(v[1]), _ptr(v[2]),
                                                            _ptr(vmax)))
        return [a[:nn] for a in v], vmax[:nn]

    def accel(self, tree: Tree, targets=None, theta=0.0, G=1.0, aold=None):
        t, nt = self._targets(targets)
        if t is None:
            nt = tree.info()["n_live"]
        dev = _is_dev(t)
        ax, ay, az, _ = self._outs(nt, dev)
        if not dev and aold is not None:
            aold = np.ascontiguousarray(aold, np.float64)
        self._check(load_library().gt_accel(self.h, tree.h, nt if targets is not None else 0, _ptr(t),
                                            theta, G, _ptr(aold), GT_MEM_DEVICE if dev else GT_MEM_HOST,
                                            _ptr(ax), _ptr(ay), _ptr(az)))
        return (ax[:nt], ay[:nt], az[:nt]) if not dev else (ax, ay, az)

    def potential(self, tree: Tree, targets=None, theta=0.0, G=1.0, aold=None):
        t, nt = self._targets(targets)
        if t is None:
            nt = tree.info()["n_live"]
        dev = _is_dev(t)
        _, _, _, phi = self._outs(nt, dev, False, True)
        if not dev and aold is not None:
            aold = np.ascontiguousarray(aold, np.float64)
        self._check(load_library().gt_potential(self.h, tree.h, nt if targets is not None else 0,
                                                _ptr(t), theta, G, _ptr(aold),
                                                GT_MEM_DEVICE if dev else GT_MEM_HOST, _ptr(phi)))
        return phi[:nt] if not dev else phi

    def form_aold(self, ax, ay, az, alpha, G=1.0):
        dev = _is_dev(ax)
        n = int(ax.numel()) if dev else len(ax)
        if dev:
            import torch

            out = torch.empty(n, dtype=torch.float64, device=ax.device)
        else:
            ax, ay, az = (np.ascontiguousarray(a, np.float64) for a in (ax, ay, az))
            out = np.empty(max(n, 1))
        self._check(load_library().gt_form_aold(self.h, n, _ptr(ax), _ptr(ay), _ptr(az), alpha, G,
                                                GT_MEM_DEVICE if dev else GT_MEM_HOST, _ptr(out)))
        return out if dev else out[:n]

    def direct_gas(self, P, targets, type=None, zeta=None, G=1.0):
        """FP64 direct sum with the zeta terms of gas-gas pairs (accel_brute on particles with
        types and zeta); host arrays.  Returns (ax, ay, az)."""
        x, y, z, m = (np.ascontiguousarray(P[k], np.float64) for k in ("x", "y", "z", "m"))
        soft = P.get("soft")
        soft = None if soft is None else np.ascontiguousarray(soft, np.float64)
        ty = None if type is None else np.ascontiguousarray(type, np.uint8)
        ze = None if zeta is None else np.ascontiguousarray(zeta, np.float64)
        t = np.ascontiguousarray(targets, np.uint32)
        ax, ay, az = np.empty(max(len(t), 1)), np.empty(max(len(t), 1)), np.empty(max(len(t), 1))
        self._check(load_library().gt_direct_gas(self.h, len(m), _ptr(x), _ptr(y), _ptr(z), _ptr(m), _ptr(soft),
                                                 _ptr(ty), _ptr(ze), len(t), _ptr(t), G, GT_MEM_HOST, _ptr(ax),
                                                 _ptr(ay), _ptr(az)))
        return ax[:len(t)], ay[:len(t)], az[:len(t)]

    def direct(self, P, targets, G=1.0, precision=GT_DIRECT_FP64, want_phi=True):
        x, y, z, m = P["x"], P["y"], P["z"], P["m"]
        soft = P.get("soft")
        dev = _is_dev(x)
        if not dev:
            x, y, z, m = (np.ascontiguousarray(a, np.float64) for a in (x, y, z, m))
            soft = None if soft is None else np.ascontiguousarray(soft, np.float64)
        t, nt = self._targets(targets)
        if dev and not _is_dev(t):
            import torch

            t = torch.as_tensor(np.asarray(t, np.uint32).view(np.int32), device=x.device)
        ax, ay, az, phi = self._outs(nt, dev, True, want_phi)
        n = int(m.numel()) if dev else len(m)
        self._check(load_library().gt_direct(self.h, n, _ptr(x), _ptr(y), _ptr(z), _ptr(m),
                                             _ptr(soft), nt, _ptr(t), G, precision,
                                             GT_MEM_DEVICE if dev else GT_MEM_HOST, _ptr(ax),
                                             _ptr(ay), _ptr(az), _ptr(phi)))
        if not dev:
            ax, ay, az = ax[:nt], ay[:nt], az[:nt]
            phi = phi[:nt] if phi is not None else None
        return (ax, ay, az, phi) if want_phi else (ax, ay, az)

    def measure_peaks(self):
        a, b = C.c_double(), C.c_double()
        self._check(load_library().gt_measure_peaks(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def peano_keys(self, x, y, z, corner, length, bits=42):
        x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
        n = len(x)
        outs = [np.empty(max(n, 1), np.uint64) for _ in range(4)]
        c = (C.c_double * 3)(*corner)
        self._check(load_library().gt_peano_keys(self.h, n, _ptr(x), _ptr(y), _ptr(z), c, length,
                                                 bits, GT_MEM_HOST, *[_ptr(o) for o in outs]))
        return [o[:n] for o in outs]
