"""Python binding of libgkway.so (the B200 multilevel k-way partitioner).

A thin ctypes layer over the C ABI in ``include/gkway.h``.  The library is the
product; this module exists for scripts, tests and the benchmark.  It never
falls back to a CPU implementation: if the shared library is missing or fails
to load, every call raises.

The package directory name contains a hyphen, so import it with
``load_package()`` from the repository root (``__graft_entry__`` and the tests
do) or add the repository to ``sys.path`` and use ``importlib``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgkway.so")
CLI_PATH = os.path.join(HERE, "bin", "g-kway")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "gkway.h")

MAX_LEVELS = 64
GKW_OK = 0
GKW_E_INVALID = 1
GKW_E_CUDA = 2
GKW_E_NOMEM = 3
GKW_E_UNSUPPORTED = 4
GKW_E_INIT = 5
GKW_E_INTERNAL = 6
GKW_E_PENDING = 7
INIT_DEVICE = 0
INIT_CALLBACK = 1

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)

INIT_FN = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, _i32p, _i32p, _i32p, _i32p,
                           ctypes.c_int32, _i32p)


class GkwError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"gkw status {status}: {msg}")
        self.status = status


class Csr(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("nnz", ctypes.c_int64),
        ("xadj", ctypes.c_void_p),
        ("adjncy", ctypes.c_void_p),
        ("adjwgt", ctypes.c_void_p),
        ("vwgt", ctypes.c_void_p),
    ]


class Options(ctypes.Structure):
    _fields_ = [
        ("eps", ctypes.c_double),
        ("group_cap", ctypes.c_int32),
        ("threshold_factor", ctypes.c_int32),
        ("move_cap", ctypes.c_int32),
        ("init_method", ctypes.c_int32),
        ("init_fn", INIT_FN),
        ("init_user", ctypes.c_void_p),
        ("seed", ctypes.c_uint64),
        ("init_trials", ctypes.c_int32),
        ("enforce_balance", ctypes.c_int32),
        ("balance_skip_levels", ctypes.c_int32),
        ("reserved1", ctypes.c_int32),
        ("coarse_vertex_frac", ctypes.c_double),
        ("reserved", ctypes.c_int32 * 2),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("n_levels", ctypes.c_int32),
        ("level_n", ctypes.c_int64 * MAX_LEVELS),
        ("level_m", ctypes.c_int64 * MAX_LEVELS),
        ("uf_rounds", ctypes.c_int32 * MAX_LEVELS),
        ("refine_rounds", ctypes.c_int32 * MAX_LEVELS),
        ("refine_moves", ctypes.c_int64 * MAX_LEVELS),
        ("balance_rounds", ctypes.c_int32 * MAX_LEVELS),
        ("balance_moves", ctypes.c_int64 * MAX_LEVELS),
        ("init_cut", ctypes.c_int64),
        ("cut", ctypes.c_int64),
        ("max_part_weight", ctypes.c_int64),
        ("maxw", ctypes.c_float),
        ("ms_coarsen", ctypes.c_double),
        ("ms_init", ctypes.c_double),
        ("ms_refine", ctypes.c_double),
        ("ms_total", ctypes.c_double),
        ("ms_level", ctypes.c_double * MAX_LEVELS),
        ("round_entries", ctypes.c_int64 * MAX_LEVELS),
    ]

    def as_dict(self) -> dict:
        nl = self.n_levels
        return dict(
            n_levels=nl,
            level_n=list(self.level_n[:nl]),
            level_m=list(self.level_m[:nl]),
            uf_rounds=list(self.uf_rounds[: max(nl - 1, 0)]),
            refine_rounds=list(self.refine_rounds[: max(nl - 1, 0)]),
            refine_moves=list(self.refine_moves[: max(nl - 1, 0)]),
            balance_rounds=list(self.balance_rounds[:nl]),
            balance_moves=list(self.balance_moves[:nl]),
            init_cut=int(self.init_cut), cut=int(self.cut), max_part_weight=int(self.max_part_weight),
            maxw=float(self.maxw), ms_coarsen=self.ms_coarsen, ms_init=self.ms_init,
            ms_refine=self.ms_refine, ms_total=self.ms_total,
            ms_level=list(self.ms_level[:nl]), round_entries=list(self.round_entries[:nl]),
        )


class Tuning(ctypes.Structure):
    _fields_ = [("match_lanes", ctypes.c_int32 * 4), ("level_verts_per_cta", ctypes.c_int32),
                ("level_min_ctas", ctypes.c_int32), ("coarsen_fused_max_n", ctypes.c_int32),
                ("coarsen_verts_per_cta", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {"match_lanes": list(self.match_lanes), "level_verts_per_cta": int(self.level_verts_per_cta),
                "level_min_ctas": int(self.level_min_ctas), "coarsen_fused_max_n": int(self.coarsen_fused_max_n),
                "coarsen_verts_per_cta": int(self.coarsen_verts_per_cta)}


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("slots", ctypes.c_int32),
        ("narrow_max_n", ctypes.c_int32),
        ("pool_bytes", ctypes.c_int64),
        ("slot_keep_bytes", ctypes.c_int64),
        ("max_bypass", ctypes.c_int32),
        ("batch_union", ctypes.c_int32),
        ("batch_max_n", ctypes.c_int32),
        ("batch_graph_max_n", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 4),
    ]


class RequestInfo(ctypes.Structure):
    _fields_ = [
        ("queue_ms", ctypes.c_double),
        ("run_ms", ctypes.c_double),
        ("latency_ms", ctypes.c_double),
        ("predicted_bytes", ctypes.c_int64),
        ("slot", ctypes.c_int32),
        ("n_levels", ctypes.c_int32),
        ("batch_graphs", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_int64),
        ("completed", ctypes.c_int64),
        ("failed", ctypes.c_int64),
        ("p50_ms", ctypes.c_double),
        ("p99_ms", ctypes.c_double),
        ("max_ms", ctypes.c_double),
        ("mean_queue_ms", ctypes.c_double),
        ("graphs_per_s", ctypes.c_double),
        ("peak_reserved_bytes", ctypes.c_int64),
        ("peak_running", ctypes.c_int32),
        ("slots", ctypes.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class CsrBatch(ctypes.Structure):
    _fields_ = [
        ("graph", Csr),
        ("n_graphs", ctypes.c_int32),
        ("graph_ptr", ctypes.c_void_p),
        ("k", ctypes.c_void_p),
        ("eps", ctypes.c_void_p),
    ]


# (name, restype, argtypes) of every C-ABI entry point
_VP = ctypes.c_void_p
_SIGS = [
    ("gkw_create", ctypes.c_int, [ctypes.POINTER(_VP), ctypes.c_int32]),
    ("gkw_destroy", ctypes.c_int, [_VP]),
    ("gkw_set_stream", ctypes.c_int, [_VP, _VP]),
    ("gkw_get_stream", _VP, [_VP]),
    ("gkw_last_error", ctypes.c_char_p, []),
    ("gkw_default_options", None, [ctypes.POINTER(Options)]),
    ("gkw_version", ctypes.c_char_p, []),
    ("gkw_kernel_launches", ctypes.c_uint64, []),
    ("gkw_partition", ctypes.c_int, [_VP, ctypes.POINTER(Csr), ctypes.c_int32, ctypes.POINTER(Options), _VP,
                                     _i64p, ctypes.POINTER(Stats)]),
    ("gkw_partition_device", ctypes.c_int, [_VP, ctypes.POINTER(Csr), ctypes.c_int32, ctypes.POINTER(Options),
                                            _VP, _i64p, ctypes.POINTER(Stats)]),
    ("gkw_partition_multi_k", ctypes.c_int, [_VP, ctypes.POINTER(Csr), ctypes.c_int32, _VP, ctypes.POINTER(Options),
                                             _VP, _VP]),
    ("gkw_match", ctypes.c_int, [_VP, ctypes.POINTER(Csr), _VP]),
    ("gkw_union_find", ctypes.c_int, [_VP, ctypes.c_int32, _VP, _VP, _VP, _i32p]),
    ("gkw_group_map", ctypes.c_int, [_VP, ctypes.c_int32, _VP, _VP, ctypes.c_int32, _VP, _i32p]),
    ("gkw_contract", ctypes.c_int, [_VP, ctypes.POINTER(Csr), _VP, ctypes.c_int32, _VP, _VP, _VP, _VP, _i64p]),
    ("gkw_update_vertex_info", ctypes.c_int, [_VP, ctypes.POINTER(Csr), ctypes.c_int32, _VP, _VP, _VP, _VP, _VP]),
    ("gkw_refine", ctypes.c_int, [_VP, ctypes.POINTER(Csr), ctypes.c_int32, ctypes.c_float, ctypes.c_int32, _VP,
                                  _VP, _VP, _VP, _VP, _VP, ctypes.c_int32, _i32p, _i64p]),
    ("gkw_init_partition", ctypes.c_int, [_VP, ctypes.POINTER(Csr), ctypes.c_int32, ctypes.c_double,
                                          ctypes.c_uint64, ctypes.c_int32, _VP]),
    ("gkw_cut", ctypes.c_int, [_VP, ctypes.POINTER(Csr), _VP, ctypes.c_int32, _i64p, _i64p]),
    ("gkw_cut_noalloc", ctypes.c_int, [ctypes.POINTER(Csr), _VP, ctypes.c_int32, _VP, _i64p, _i64p]),
    ("gkw_read_metis", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, _i32p, _i64p, ctypes.POINTER(_i32p),
                                      ctypes.POINTER(_i32p), ctypes.POINTER(_i32p), ctypes.POINTER(_i32p)]),
    ("gkw_write_partition", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, _i32p]),
    ("gkw_free", None, [_VP]),
    ("gkw_get_tuning", ctypes.c_int, [_VP, ctypes.POINTER(Tuning)]),
    ("gkw_set_tuning", ctypes.c_int, [_VP, ctypes.POINTER(Tuning)]),
    ("gkw_autotune", ctypes.c_int, [_VP, ctypes.POINTER(Csr), ctypes.c_int32, ctypes.POINTER(Options),
                                    ctypes.POINTER(Tuning)]),
    ("gkw_read_metis_device", ctypes.c_int, [_VP, ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(Csr)]),
    ("gkw_free_device_graph", None, [ctypes.POINTER(Csr)]),
    ("gkw_write_partition_device", ctypes.c_int, [_VP, ctypes.c_char_p, ctypes.c_int32, _VP]),
    ("gkw_max_part_weight", ctypes.c_float, [ctypes.c_int64, ctypes.c_int32, ctypes.c_double]),
    ("gkw_balance_cap", ctypes.c_float, [ctypes.c_int64, ctypes.c_int32, ctypes.c_double]),
    ("gkw_balance", ctypes.c_int, [_VP, ctypes.POINTER(Csr), ctypes.c_int32, ctypes.c_float, ctypes.c_int32, _VP,
                                   _VP, _VP, _VP, _VP, _i32p, _i64p]),
    ("gkw_server_default_config", None, [ctypes.POINTER(ServerConfig)]),
    ("gkw_server_create", ctypes.c_int, [ctypes.POINTER(_VP), ctypes.c_int32, ctypes.POINTER(ServerConfig)]),
    ("gkw_server_destroy", ctypes.c_int, [_VP]),
    ("gkw_predict_footprint", ctypes.c_int64, [ctypes.c_int32, ctypes.c_int64, ctypes.c_int32]),
    ("gkw_server_submit", ctypes.c_int, [_VP, ctypes.POINTER(Csr), ctypes.c_int32, ctypes.POINTER(Options),
                                         _i64p]),
    ("gkw_server_poll", ctypes.c_int, [_VP, ctypes.c_int64, ctypes.c_int32, _VP, _i64p,
                                       ctypes.POINTER(RequestInfo)]),
    ("gkw_server_stats_get", ctypes.c_int, [_VP, ctypes.POINTER(ServerStats), ctypes.c_int32]),
    ("gkw_partition_batch", ctypes.c_int, [_VP, ctypes.POINTER(CsrBatch), ctypes.POINTER(Options), _VP, _i64p,
                                           _i32p]),
]

_lib = None


def build() -> None:
    """Compile libgkway.so and the CLI in place (nvcc, sm_100a)."""
    subprocess.run(["make", "-s", "-C", HERE, f"-j{os.cpu_count() or 4}"], check=True)


def lib():
    """The loaded shared library; raises if it is missing (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GkwError(GKW_E_INTERNAL, f"{LIB_PATH} is missing: run build() first")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def launch_count() -> int:
    """Kernels launched by the library in this process so far."""
    return int(lib().gkw_kernel_launches())


def last_error() -> str:
    s = lib().gkw_last_error()
    return s.decode() if s else ""


def check(status: int) -> None:
    if status != GKW_OK:
        raise GkwError(status, last_error())


def default_options(**kw) -> Options:
    o = Options()
    lib().gkw_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def max_part_weight(total_vwgt: int, k: int, eps: float = 0.03) -> float:
    return float(lib().gkw_max_part_weight(int(total_vwgt), int(k), float(eps)))


def balance_cap(total_vwgt: int, k: int, eps: float = 0.03) -> float:
    return float(lib().gkw_balance_cap(int(total_vwgt), int(k), float(eps)))


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def read_metis(path: str, reference_quirks: bool = False):
    """Parse a METIS .graph file with the library's parser -> (xadj, adjncy, adjwgt, vwgt) 0-based."""
    n = ctypes.c_int32()
    nnz = ctypes.c_int64()
    ptrs = [_i32p() for _ in range(4)]
    check(lib().gkw_read_metis(path.encode(), int(reference_quirks), ctypes.byref(n), ctypes.byref(nnz),
                               *[ctypes.byref(p) for p in ptrs]))
    try:
        sizes = [n.value + 1, nnz.value, nnz.value, n.value]
        out = [np.ctypeslib.as_array(p, (max(s, 1),))[:s].copy() for p, s in zip(ptrs, sizes)]
    finally:
        for p in ptrs:
            lib().gkw_free(ctypes.cast(p, _VP))
    return tuple(out)


def write_partition(path: str, part) -> None:
    part = _i32(part)
    check(lib().gkw_write_partition(path.encode(), int(part.shape[0]), part.ctypes.data_as(_i32p)))


def _csr_host(xadj, adjncy, adjwgt=None, vwgt=None):
    keep = [_i32(xadj), _i32(adjncy)]
    keep.append(None if adjwgt is None else _i32(adjwgt))
    keep.append(None if vwgt is None else _i32(vwgt))
    c = Csr()
    c.n = keep[0].shape[0] - 1
    c.nnz = keep[1].shape[0]
    c.xadj = keep[0].ctypes.data
    c.adjncy = keep[1].ctypes.data if keep[1].shape[0] else None
    c.adjwgt = None if keep[2] is None or not keep[2].shape[0] else keep[2].ctypes.data
    c.vwgt = None if keep[3] is None or not keep[3].shape[0] else keep[3].ctypes.data
    return c, keep


def _csr_dev(xadj, adjncy, adjwgt, vwgt):
    """Csr over torch CUDA int32 tensors (no copy)."""
    c = Csr()
    c.n = int(xadj.shape[0]) - 1
    c.nnz = int(adjncy.shape[0])
    c.xadj = xadj.data_ptr()
    c.adjncy = adjncy.data_ptr() if adjncy.numel() else None
    c.adjwgt = adjwgt.data_ptr() if adjwgt is not None and adjwgt.numel() else None
    c.vwgt = vwgt.data_ptr() if vwgt is not None and vwgt.numel() else None
    return c


class Handle:
    """One library handle (CUDA stream + device memory pools) on one device."""

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        check(lib().gkw_create(ctypes.byref(self._h), int(device)))
        self.device = device

    def close(self):
        if self._h:
            lib().gkw_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return int(lib().gkw_get_stream(self._h) or 0)

    def set_stream(self, stream_ptr: int) -> None:
        check(lib().gkw_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    # ---- whole partitioner ----
    def partition(self, xadj, adjncy, adjwgt, vwgt, k: int, opts: Options | None = None,
                  init=None, part_out: np.ndarray | None = None):
        """Host arrays in, host part out. ``init``: optional callable for the coarsest
        level, ``init(xadj, adjncy, adjwgt, vwgt, k) -> part`` (numpy)."""
        c, keep = _csr_host(xadj, adjncy, adjwgt, vwgt)
        o = opts if opts is not None else default_options()
        cb_keep = None
        if init is not None:
            cb_keep = _make_init_cb(init)
            o.init_method = INIT_CALLBACK
            o.init_fn = cb_keep
        part = part_out if part_out is not None else np.empty(c.n, np.int32)
        cut = ctypes.c_int64()
        st = Stats()
        rc = lib().gkw_partition(self._h, ctypes.byref(c), int(k), ctypes.byref(o),
                                 part.ctypes.data if c.n else None, ctypes.byref(cut), ctypes.byref(st))
        del keep, cb_keep
        check(rc)
        return part, int(cut.value), st.as_dict()

    def partition_multi_k(self, xadj, adjncy, adjwgt, vwgt, ks, opts: Options | None = None):
        """One graph for several k, coarsened once -> (parts [len(ks), n], cuts [len(ks)]);
        row q equals ``partition(..., ks[q])``."""
        c, keep = _csr_host(xadj, adjncy, adjwgt, vwgt)
        kk = np.ascontiguousarray(ks, dtype=np.int32)
        o = opts if opts is not None else default_options()
        parts = np.empty((kk.shape[0], c.n), np.int32)
        cuts = np.zeros(max(kk.shape[0], 1), np.int64)
        rc = lib().gkw_partition_multi_k(self._h, ctypes.byref(c), int(kk.shape[0]),
                                         kk.ctypes.data if kk.shape[0] else None, ctypes.byref(o),
                                         parts.ctypes.data if parts.size else None, cuts.ctypes.data)
        del keep
        check(rc)
        return parts, cuts[:kk.shape[0]]

    def partition_device(self, xadj, adjncy, adjwgt, vwgt, k: int, part_out, opts: Options | None = None,
                         stats: bool = True):
        """torch CUDA int32 tensors in, part written into ``part_out`` (torch CUDA int32)."""
        c = _csr_dev(xadj, adjncy, adjwgt, vwgt)
        o = opts if opts is not None else default_options()
        cut = ctypes.c_int64()
        st = Stats()
        check(lib().gkw_partition_device(self._h, ctypes.byref(c), int(k), ctypes.byref(o),
                                         part_out.data_ptr() if c.n else None, ctypes.byref(cut),
                                         ctypes.byref(st) if stats else None))
        return int(cut.value), (st.as_dict() if stats else None)

    # ---- per-phase entry points (torch CUDA tensors) ----
    def match(self, g) -> "torch.Tensor":
        import torch
        cand = torch.empty(g[0].shape[0] - 1, dtype=torch.int32, device=g[0].device)
        c = _csr_dev(*g)
        check(lib().gkw_match(self._h, ctypes.byref(c), cand.data_ptr() if cand.numel() else None))
        return cand

    def union_find(self, cand):
        import torch
        n = int(cand.shape[0])
        root = torch.empty(n, dtype=torch.int32, device=cand.device)
        dist = torch.empty(n, dtype=torch.int32, device=cand.device)
        r = ctypes.c_int32()
        check(lib().gkw_union_find(self._h, n, cand.data_ptr() if n else None, root.data_ptr() if n else None,
                                   dist.data_ptr() if n else None, ctypes.byref(r)))
        return root, dist, int(r.value)

    def group_map(self, root, dist, group_cap: int = 6):
        import torch
        n = int(root.shape[0])
        cmap = torch.empty(n, dtype=torch.int32, device=root.device)
        nc = ctypes.c_int32()
        check(lib().gkw_group_map(self._h, n, root.data_ptr() if n else None, dist.data_ptr() if n else None,
                                  int(group_cap), cmap.data_ptr() if n else None, ctypes.byref(nc)))
        return cmap, int(nc.value)

    def contract(self, g, cmap, nc: int):
        import torch
        dev = g[0].device
        m = int(g[1].shape[0])
        cx = torch.empty(nc + 1, dtype=torch.int32, device=dev)
        ca = torch.empty(max(m, 1), dtype=torch.int32, device=dev)
        cw = torch.empty(max(m, 1), dtype=torch.int32, device=dev)
        cv = torch.empty(max(nc, 1), dtype=torch.int32, device=dev)
        mc = ctypes.c_int64()
        c = _csr_dev(*g)
        check(lib().gkw_contract(self._h, ctypes.byref(c), cmap.data_ptr() if cmap.numel() else None, int(nc),
                                 cx.data_ptr(), ca.data_ptr(), cw.data_ptr(), cv.data_ptr(), ctypes.byref(mc)))
        return cx, ca[: mc.value], cw[: mc.value], cv[:nc]

    def update_vertex_info(self, g, k, part, updated, boundary, gain, target):
        c = _csr_dev(*g)
        check(lib().gkw_update_vertex_info(self._h, ctypes.byref(c), int(k), part.data_ptr(), updated.data_ptr(),
                                           boundary.data_ptr(), gain.data_ptr(), target.data_ptr()))

    def refine(self, g, k, maxw, move_cap, part, boundary, gain, target, updated, pw, initial_update=True):
        c = _csr_dev(*g)
        r = ctypes.c_int32()
        mv = ctypes.c_int64()
        check(lib().gkw_refine(self._h, ctypes.byref(c), int(k), float(maxw), int(move_cap), part.data_ptr(),
                               boundary.data_ptr(), gain.data_ptr(), target.data_ptr(),
                               updated.data_ptr() if updated is not None else None, pw.data_ptr(),
                               int(initial_update), ctypes.byref(r), ctypes.byref(mv)))
        return int(r.value), int(mv.value)

    def balance(self, g, k, cap, move_cap, part, boundary, gain, target, pw):
        c = _csr_dev(*g)
        r = ctypes.c_int32()
        mv = ctypes.c_int64()
        check(lib().gkw_balance(self._h, ctypes.byref(c), int(k), float(cap), int(move_cap), part.data_ptr(),
                                boundary.data_ptr(), gain.data_ptr(), target.data_ptr(), pw.data_ptr(),
                                ctypes.byref(r), ctypes.byref(mv)))
        return int(r.value), int(mv.value)

    def init_partition(self, g, k, eps=0.03, seed=1, trials=8):
        import torch
        part = torch.empty(max(int(g[0].shape[0]) - 1, 1), dtype=torch.int32, device=g[0].device)
        c = _csr_dev(*g)
        check(lib().gkw_init_partition(self._h, ctypes.byref(c), int(k), float(eps), int(seed), int(trials),
                                       part.data_ptr()))
        return part[: int(g[0].shape[0]) - 1]

    # ---- launch shapes ----
    def tuning(self) -> dict:
        t = Tuning()
        check(lib().gkw_get_tuning(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, match_lanes=(4, 8, 16, 32), level_verts_per_cta=512, level_min_ctas=32,
                   coarsen_fused_max_n=0, coarsen_verts_per_cta=256) -> None:
        t = Tuning((ctypes.c_int32 * 4)(*match_lanes), int(level_verts_per_cta), int(level_min_ctas),
                   int(coarsen_fused_max_n), int(coarsen_verts_per_cta))
        check(lib().gkw_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self, xadj, adjncy, adjwgt, vwgt, k: int, opts: Options | None = None) -> dict:
        """gkw_autotune on torch CUDA int32 tensors; returns the chosen shapes."""
        c = _csr_dev(xadj, adjncy, adjwgt, vwgt)
        o = opts if opts is not None else default_options()
        t = Tuning()
        check(lib().gkw_autotune(self._h, ctypes.byref(c), int(k), ctypes.byref(o), ctypes.byref(t)))
        return t.as_dict()

    # ---- METIS files parsed and written on the device ----
    def read_metis_device(self, path: str, reference_quirks: bool = False):
        """Parse a METIS .graph file on the device -> (xadj, adjncy, adjwgt, vwgt) as
        torch CUDA int32 tensors (copies; the library's arrays are released)."""
        import torch
        c = Csr()
        check(lib().gkw_read_metis_device(self._h, path.encode(), int(reference_quirks), ctypes.byref(c)))
        try:
            dev = torch.device("cuda", self.device)
            out = []
            for ptr, cnt in ((c.xadj, c.n + 1), (c.adjncy, c.nnz), (c.adjwgt, c.nnz), (c.vwgt, c.n)):
                addr = ctypes.cast(ptr, ctypes.c_void_p).value
                if cnt > 0 and addr:
                    out.append(torch.as_tensor(_DeviceArray(addr, int(cnt)), device=dev).clone())
                else:
                    out.append(torch.empty(0, dtype=torch.int32, device=dev))
            torch.cuda.synchronize(dev)
        finally:
            lib().gkw_free_device_graph(ctypes.byref(c))
        return tuple(out)

    def write_partition_device(self, path: str, part) -> None:
        """Write part ids (a torch CUDA int32 tensor) one per line, formatted on the device."""
        n = int(part.numel())
        check(lib().gkw_write_partition_device(self._h, path.encode(), n, part.data_ptr() if n else None))

    def cut(self, g, part, k):
        c = _csr_dev(*g)
        cut = ctypes.c_int64()
        pw = np.zeros(k, np.int64)
        check(lib().gkw_cut(self._h, ctypes.byref(c), part.data_ptr(), int(k), ctypes.byref(cut),
                            pw.ctypes.data_as(_i64p)))
        return int(cut.value), pw


class _DeviceArray:
    """A view of device int32 memory for torch.as_tensor (CUDA array interface)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<i4", "data": (ptr, False),
                                         "version": 2, "strides": None}


def predict_footprint(n: int, nnz: int, k: int) -> int:
    """Predicted device bytes of one partition (the server's admission measure)."""
    return int(lib().gkw_predict_footprint(int(n), int(nnz), int(k)))


def server_config(**kw) -> ServerConfig:
    c = ServerConfig()
    lib().gkw_server_default_config(ctypes.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def concat_graphs(graphs):
    """Disjoint union of CSR graphs (objects with xadj/adjncy/adjwgt/vwgt) ->
    (xadj, adjncy, adjwgt, vwgt, graph_ptr) with global 0-based ids."""
    ns = [int(g.xadj.shape[0]) - 1 for g in graphs]
    ms = [int(g.adjncy.shape[0]) for g in graphs]
    vptr = np.zeros(len(graphs) + 1, np.int64)
    eptr = np.zeros(len(graphs) + 1, np.int64)
    vptr[1:] = np.cumsum(ns)
    eptr[1:] = np.cumsum(ms)
    if vptr[-1] >= 2 ** 31 or eptr[-1] >= 2 ** 31:
        raise GkwError(GKW_E_UNSUPPORTED, "batch too large for int32 offsets")
    xadj = np.zeros(int(vptr[-1]) + 1, np.int32)
    adjncy = np.empty(int(eptr[-1]), np.int32)
    adjwgt = np.empty(int(eptr[-1]), np.int32)
    vwgt = np.empty(int(vptr[-1]), np.int32)
    for i, g in enumerate(graphs):
        v0, v1, e0, e1 = int(vptr[i]), int(vptr[i + 1]), int(eptr[i]), int(eptr[i + 1])
        xadj[v0 + 1:v1 + 1] = g.xadj[1:].astype(np.int64) + e0
        adjncy[e0:e1] = g.adjncy.astype(np.int64) + v0
        adjwgt[e0:e1] = g.adjwgt
        vwgt[v0:v1] = g.vwgt
    return xadj, adjncy, adjwgt, vwgt, vptr.astype(np.int32)


class Server:
    """Batched and served partitioning on one device: ``slots`` concurrent
    partitions fed from one queue, admitted by predicted device footprint."""

    def __init__(self, device: int = 0, **cfg):
        self._s = ctypes.c_void_p()
        c = server_config(**cfg)
        check(lib().gkw_server_create(ctypes.byref(self._s), int(device), ctypes.byref(c)))

    def close(self):
        if self._s:
            lib().gkw_server_destroy(self._s)
            self._s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, xadj, adjncy, adjwgt, vwgt, k: int, opts: Options | None = None) -> int:
        c, keep = _csr_host(xadj, adjncy, adjwgt, vwgt)
        o = opts if opts is not None else default_options()
        t = ctypes.c_int64()
        rc = lib().gkw_server_submit(self._s, ctypes.byref(c), int(k), ctypes.byref(o), ctypes.byref(t))
        del keep
        check(rc)
        return int(t.value)

    def poll(self, ticket: int, n: int, wait_ms: int = -1):
        """(part, cut, info) when the request is done, None while it is pending."""
        part = np.empty(max(n, 1), np.int32)
        cut = ctypes.c_int64()
        info = RequestInfo()
        rc = lib().gkw_server_poll(self._s, int(ticket), int(wait_ms), part.ctypes.data, ctypes.byref(cut),
                                   ctypes.byref(info))
        if rc == GKW_E_PENDING:
            return None
        check(rc)
        return part[:n], int(cut.value), {name: getattr(info, name) for name, _ in info._fields_}

    def stats(self, reset: bool = False) -> dict:
        st = ServerStats()
        check(lib().gkw_server_stats_get(self._s, ctypes.byref(st), int(reset)))
        return st.as_dict()

    def partition_batch(self, xadj, adjncy, adjwgt, vwgt, graph_ptr, ks, eps=None, opts: Options | None = None,
                        raise_on_error: bool = True):
        """Concatenated CSR (global ids) + graph_ptr -> (part with per-graph ids, cuts, statuses)."""
        c, keep = _csr_host(xadj, adjncy, adjwgt, vwgt)
        gp = _i32(graph_ptr)
        kk = _i32(ks)
        ee = None if eps is None else np.ascontiguousarray(eps, dtype=np.float64)
        b = CsrBatch()
        b.graph = c
        b.n_graphs = int(kk.shape[0])
        b.graph_ptr = gp.ctypes.data
        b.k = kk.ctypes.data if kk.shape[0] else None
        b.eps = None if ee is None else ee.ctypes.data
        o = opts if opts is not None else default_options()
        part = np.empty(max(c.n, 1), np.int32)
        cuts = np.zeros(max(b.n_graphs, 1), np.int64)
        sts = np.zeros(max(b.n_graphs, 1), np.int32)
        rc = lib().gkw_partition_batch(self._s, ctypes.byref(b), ctypes.byref(o), part.ctypes.data,
                                       cuts.ctypes.data_as(_i64p), sts.ctypes.data_as(_i32p))
        del keep
        if raise_on_error:
            check(rc)
        return part[:c.n], cuts[:b.n_graphs], sts[:b.n_graphs]


def _make_init_cb(init):
    def cb(user, n, xadj, adjncy, adjwgt, vwgt, k, part):
        try:
            x = np.ctypeslib.as_array(xadj, (n + 1,)).copy()
            m = int(x[-1])
            if m:
                a = np.ctypeslib.as_array(adjncy, (m,)).copy()
                w = np.ctypeslib.as_array(adjwgt, (m,)).copy()
            else:
                a = np.zeros(0, np.int32)
                w = np.zeros(0, np.int32)
            vw = np.ctypeslib.as_array(vwgt, (n,)).copy() if n else np.zeros(0, np.int32)
            p = np.asarray(init(x, a, w, vw, k), dtype=np.int32)
            if n:
                np.ctypeslib.as_array(part, (n,))[:] = p
            return 0
        except Exception:
            return -1
    return INIT_FN(cb)


def cut_noalloc(g, part, k: int, stream: int = 0):
    """gkw_cut_noalloc over torch CUDA tensors: (cut, part weights).  Allocates
    no device memory and needs no handle; runs on `stream` (a cudaStream_t as
    an int, 0 = the default stream) of the current device."""
    if int(k) < 1:
        raise GkwError(GKW_E_UNSUPPORTED, "gkw_cut_noalloc: k must be in [1, 8190]")
    c = _csr_dev(*g)
    cut = ctypes.c_int64()
    pw = np.zeros(k, np.int64)
    check(lib().gkw_cut_noalloc(ctypes.byref(c), part.data_ptr() if part.numel() else None, int(k),
                                ctypes.c_void_p(stream), ctypes.byref(cut), pw.ctypes.data_as(_i64p)))
    return int(cut.value), pw


def exported_symbols() -> list[str]:
    """Names of the C-ABI functions declared in include/gkway.h."""
    import re
    src = open(HEADER_PATH).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gkw_[a-z_0-9]+)\s*\(", src)) - {"gkw_init_fn"})
