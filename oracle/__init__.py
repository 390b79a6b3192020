"""ctypes binding of the oracle (test infrastructure only).

The oracle is a CPU restatement of the reference partitioner (see
``gkway_oracle.cpp``).  Only the tests, the smoke check and the CPU-baseline leg
of ``bench.py`` use it, as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
METIS_PATH = os.path.join(HERE, "_ref", "libmetis.so")
N11_PATH = os.path.join(HERE, "_ref", "delaunay_n11.graph")

MAX_LEVELS = 64

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)

INIT_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int32, _i32p, _i32p, _i32p, _i32p,
                           ctypes.c_int32, _i32p)


class Opts(ctypes.Structure):
    _fields_ = [
        ("group_cap", ctypes.c_int32),
        ("threshold_factor", ctypes.c_int32),
        ("move_cap", ctypes.c_int32),
        ("eps", ctypes.c_double),
        ("init_method", ctypes.c_int32),
        ("init_fn", INIT_FN),
        ("init_user", ctypes.c_void_p),
        ("enforce_balance", ctypes.c_int32),
        ("balance_skip_levels", ctypes.c_int32),
        ("coarse_vertex_frac", ctypes.c_double),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("n_levels", ctypes.c_int32),
        ("level_n", ctypes.c_int64 * MAX_LEVELS),
        ("level_m", ctypes.c_int64 * MAX_LEVELS),
        ("uf_launches", ctypes.c_int32 * MAX_LEVELS),
        ("refine_rounds", ctypes.c_int32 * MAX_LEVELS),
        ("refine_moves", ctypes.c_int64 * MAX_LEVELS),
        ("balance_rounds", ctypes.c_int32 * MAX_LEVELS),
        ("balance_moves", ctypes.c_int64 * MAX_LEVELS),
        ("init_cut", ctypes.c_int64),
        ("cut", ctypes.c_int64),
        ("max_part_weight", ctypes.c_int64),
        ("maxw", ctypes.c_float),
        ("status", ctypes.c_int32),
    ]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_match.restype = None
        L.orc_union_find.restype = ctypes.c_int32
        L.orc_group_map.restype = ctypes.c_int32
        L.orc_coarse_vwgt.restype = None
        L.orc_contract.restype = ctypes.c_int64
        L.orc_set_metis.restype = ctypes.c_int
        L.orc_set_metis.argtypes = [ctypes.c_char_p]
        L.orc_has_metis.restype = ctypes.c_int
        L.orc_metis_kway.restype = ctypes.c_int
        L.orc_metis_recursive.restype = ctypes.c_int
        L.orc_cut.restype = ctypes.c_int64
        L.orc_max_part_weight.restype = ctypes.c_float
        L.orc_max_part_weight.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_double]
        L.orc_partition.restype = ctypes.c_int
        L.orc_refine.restype = ctypes.c_int32
        L.orc_refine.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, _i32p, ctypes.c_int32,
                                 ctypes.c_float, ctypes.c_int32, _i32p, _i32p, _i32p, _i32p, _i32p,
                                 _i64p, _i64p, _i64p, ctypes.c_int32]
        if os.path.exists(METIS_PATH):
            L.orc_set_metis(METIS_PATH.encode())
        _lib = L
    return _lib


def has_metis() -> bool:
    return bool(lib().orc_has_metis())


def _p(a: np.ndarray):
    if a.dtype == np.int32:
        return a.ctypes.data_as(_i32p)
    if a.dtype == np.int64:
        return a.ctypes.data_as(_i64p)
    raise TypeError(a.dtype)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def match(g) -> np.ndarray:
    cand = np.empty(g.n, np.int32)
    lib().orc_match(ctypes.c_int32(g.n), _p(g.xadj), _p(g.adjncy), _p(g.adjwgt), _p(cand))
    return cand


def union_find(cand: np.ndarray):
    cand = _c(cand)
    n = cand.shape[0]
    root = np.empty(n, np.int32)
    dist = np.empty(n, np.int32)
    launches = lib().orc_union_find(ctypes.c_int32(n), _p(cand), _p(root), _p(dist))
    return root, dist, int(launches)


def group_map(root, dist, group_cap: int = 6):
    root, dist = _c(root), _c(dist)
    n = root.shape[0]
    cmap = np.empty(n, np.int32)
    order = np.empty(n, np.int32)
    nc = lib().orc_group_map(ctypes.c_int32(n), _p(root), _p(dist), ctypes.c_int32(group_cap),
                             _p(cmap), _p(order))
    return cmap, int(nc), order


def coarse_vwgt(vwgt, cmap, nc: int) -> np.ndarray:
    vwgt, cmap = _c(vwgt), _c(cmap)
    out = np.empty(nc, np.int32)
    lib().orc_coarse_vwgt(ctypes.c_int32(vwgt.shape[0]), _p(vwgt), _p(cmap), ctypes.c_int32(nc), _p(out))
    return out


def contract(g, cmap, nc: int):
    cmap = _c(cmap)
    cx = np.empty(nc + 1, np.int32)
    ca = np.empty(max(g.m, 1), np.int32)
    cw = np.empty(max(g.m, 1), np.int32)
    mc = lib().orc_contract(ctypes.c_int32(g.n), _p(g.xadj), _p(g.adjncy), _p(g.adjwgt), _p(cmap),
                            ctypes.c_int32(nc), _p(cx), _p(ca), _p(cw))
    return cx, ca[:mc].copy(), cw[:mc].copy()


def metis_kway(g, k: int):
    part = np.empty(g.n, np.int32)
    obj = ctypes.c_int64(0)
    rc = lib().orc_metis_kway(ctypes.c_int32(g.n), _p(g.xadj), _p(g.adjncy), _p(g.adjwgt), _p(g.vwgt),
                              ctypes.c_int32(k), _p(part), ctypes.byref(obj))
    if rc != 1:
        raise RuntimeError(f"METIS failed: {rc}")
    return part, int(obj.value)


def metis_recursive(g, k: int):
    """METIS_PartGraphRecursive (the recursive-bisection alternative to the
    k-way call of metis_partition.hpp:46-47, metis.h:185) -> (part, cut)."""
    part = np.empty(g.n, np.int32)
    obj = ctypes.c_int64(0)
    rc = lib().orc_metis_recursive(ctypes.c_int32(g.n), _p(g.xadj), _p(g.adjncy), _p(g.adjwgt), _p(g.vwgt),
                                   ctypes.c_int32(k), _p(part), ctypes.byref(obj))
    if rc != 1:
        raise RuntimeError(f"METIS failed: {rc}")
    return part, int(obj.value)


def cut(g, part) -> int:
    part = _c(part)
    return int(lib().orc_cut(ctypes.c_int32(g.n), _p(g.xadj), _p(g.adjncy), _p(g.adjwgt), _p(part)))


def part_weights(g, part, k: int) -> np.ndarray:
    part = _c(part)
    pw = np.empty(k, np.int64)
    lib().orc_part_weights(ctypes.c_int32(g.n), _p(g.vwgt), _p(part), ctypes.c_int32(k), _p(pw))
    return pw


def max_part_weight(total_vwgt: int, k: int, eps: float = 0.03) -> float:
    return float(lib().orc_max_part_weight(total_vwgt, k, eps))


def balance_cap(total_vwgt: int, k: int, eps: float = 0.03) -> float:
    L = lib()
    L.orc_balance_cap.restype = ctypes.c_float
    L.orc_balance_cap.argtypes = [ctypes.c_int64, ctypes.c_int32, ctypes.c_double]
    return float(L.orc_balance_cap(total_vwgt, k, eps))


def update_vertex_info(g, k, part, updated, boundary, gain, target):
    part, updated = _c(part), _c(updated)
    boundary, gain, target = _c(boundary).copy(), _c(gain).copy(), _c(target).copy()
    lib().orc_update_vertex_info(ctypes.c_int32(g.n), _p(g.xadj), _p(g.adjncy), _p(g.adjwgt),
                                 ctypes.c_int32(k), _p(part), _p(updated), _p(boundary), _p(gain),
                                 _p(target))
    return boundary, gain, target


def refine(g, k, maxw, part, boundary, gain, target, updated, pw, move_cap=1024, initial_update=True):
    part, boundary, gain, target, updated = (_c(a).copy() for a in (part, boundary, gain, target, updated))
    pw = np.ascontiguousarray(pw, dtype=np.int64).copy()
    moves = ctypes.c_int64(0)
    gsum = ctypes.c_int64(0)
    rounds = lib().orc_refine(g.n, _p(g.xadj), _p(g.adjncy), _p(g.adjwgt), _p(g.vwgt), k, maxw, move_cap,
                              _p(part), _p(boundary), _p(gain), _p(target), _p(updated), _p(pw),
                              ctypes.byref(moves), ctypes.byref(gsum), int(initial_update))
    return dict(part=part, boundary=boundary, gain=gain, target=target, updated=updated, pw=pw,
                rounds=int(rounds), moves=int(moves.value), gain_sum=int(gsum.value))


def partition(g, k: int, *, init=None, group_cap=6, threshold_factor=20, move_cap=1024, eps=0.03,
              enforce_balance=False, balance_skip_levels=1, coarse_vertex_frac=0.5):
    """Run the whole reference algorithm.

    ``init``: None -> the bundled METIS (the reference's initial partitioner);
    otherwise a callable ``init(coarse_csr_arrays..., k) -> part`` used for the
    coarsest level.  ``balance_skip_levels`` and ``coarse_vertex_frac`` act in
    default mode (``enforce_balance``) only, with the library's defaults.
    """
    opts = Opts()
    opts.group_cap = group_cap
    opts.threshold_factor = threshold_factor
    opts.move_cap = move_cap
    opts.eps = eps
    opts.enforce_balance = int(enforce_balance)
    opts.balance_skip_levels = int(balance_skip_levels)
    opts.coarse_vertex_frac = float(coarse_vertex_frac)
    keep = None
    if init is None:
        if not has_metis():
            raise RuntimeError("METIS library not available")
        opts.init_method = 0
        opts.init_fn = INIT_FN()
    else:
        def cb(user, n, xadj, adjncy, adjwgt, vwgt, kk, part):
            x = np.ctypeslib.as_array(xadj, (n + 1,)).copy()
            m = int(x[-1])
            if m:
                a = np.ctypeslib.as_array(adjncy, (m,)).copy()
                w = np.ctypeslib.as_array(adjwgt, (m,)).copy()
            else:
                a = np.zeros(0, np.int32)
                w = np.zeros(0, np.int32)
            vw = np.ctypeslib.as_array(vwgt, (n,)).copy() if n else np.zeros(0, np.int32)
            p = np.asarray(init(x, a, w, vw, kk), dtype=np.int32)
            if n:
                np.ctypeslib.as_array(part, (n,))[:] = p
            return 0
        keep = INIT_FN(cb)
        opts.init_method = 1
        opts.init_fn = keep
    res = Result()
    part = np.empty(g.n, np.int32)
    rc = lib().orc_partition(ctypes.c_int32(g.n), _p(g.xadj), _p(g.adjncy), _p(g.adjwgt), _p(g.vwgt),
                             ctypes.c_int32(k), ctypes.byref(opts), _p(part), ctypes.byref(res))
    del keep
    if rc != 0:
        raise RuntimeError(f"oracle partition failed: {rc}")
    nl = res.n_levels
    info = dict(
        n_levels=nl,
        level_n=list(res.level_n[:nl]),
        level_m=list(res.level_m[:nl]),
        uf_launches=list(res.uf_launches[: max(nl - 1, 0)]),
        refine_rounds=list(res.refine_rounds[: max(nl - 1, 0)]),
        refine_moves=list(res.refine_moves[: max(nl - 1, 0)]),
        balance_rounds=list(res.balance_rounds[:nl]),
        balance_moves=list(res.balance_moves[:nl]),
        init_cut=int(res.init_cut), cut=int(res.cut), max_part_weight=int(res.max_part_weight),
        maxw=float(res.maxw),
    )
    return part, info


def read_metis_graph(path: str):
    """Minimal METIS .graph reader for the checker (fmt 0/1/10/11, ncon 1)."""
    from importlib import util as _u
    gen = _load_generators()
    with open(path) as f:
        lines = [ln for ln in f if not ln.lstrip().startswith("%")]
    head = lines[0].split()
    n, me = int(head[0]), int(head[1])
    fmt = head[2] if len(head) > 2 else "0"
    fmt = fmt.zfill(3)
    has_vw, has_ew = fmt[1] == "1", fmt[2] == "1"
    xadj = [0]
    adj, wgt, vw = [], [], []
    for i in range(n):
        tok = [int(t) for t in lines[1 + i].split()] if 1 + i < len(lines) else []
        j = 0
        if has_vw:
            vw.append(tok[0]); j = 1
        else:
            vw.append(1)
        while j < len(tok):
            adj.append(tok[j] - 1)
            if has_ew:
                wgt.append(tok[j + 1]); j += 2
            else:
                wgt.append(1); j += 1
        xadj.append(len(adj))
    return gen.Csr(np.array(xadj, np.int32), np.array(adj, np.int32), np.array(wgt, np.int32),
                   np.array(vw, np.int32))


def _load_generators():
    import importlib.util
    import sys
    name = "dac_g_kway_b200_generators"
    if name in sys.modules:
        return sys.modules[name]
    path = os.path.join(os.path.dirname(HERE), "dac_g-kway_b200", "generators.py")
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def init_partition(g, k: int, eps: float = 0.03, seed: int = 1, trials: int = 8) -> np.ndarray:
    """The device initial partitioner's algorithm, restated on the CPU."""
    part = np.empty(g.n, np.int32)
    L = lib()
    L.orc_init_partition.restype = None
    L.orc_init_partition.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, _i32p, ctypes.c_int32, ctypes.c_double,
                                     ctypes.c_uint64, ctypes.c_int32, _i32p]
    L.orc_init_partition(g.n, _p(g.xadj), _p(g.adjncy), _p(g.adjwgt), _p(g.vwgt), int(k), float(eps),
                         int(seed), int(trials), _p(part))
    return part


def balance(g, k, cap, part, boundary, gain, target, pw, move_cap=1024):
    """Balance rounds alone (default mode), in the oracle."""
    part, boundary, gain, target = (_c(a).copy() for a in (part, boundary, gain, target))
    pw = np.ascontiguousarray(pw, dtype=np.int64).copy()
    moves = ctypes.c_int64(0)
    L = lib()
    L.orc_balance.restype = ctypes.c_int32
    L.orc_balance.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, _i32p, ctypes.c_int32, ctypes.c_float,
                              ctypes.c_int32, _i32p, _i32p, _i32p, _i32p, _i64p, _i64p]
    rounds = L.orc_balance(g.n, _p(g.xadj), _p(g.adjncy), _p(g.adjwgt), _p(g.vwgt), int(k), float(cap),
                           int(move_cap), _p(part), _p(boundary), _p(gain), _p(target), _p(pw), ctypes.byref(moves))
    return dict(part=part, boundary=boundary, gain=gain, target=target, pw=pw, rounds=int(rounds),
                moves=int(moves.value))
