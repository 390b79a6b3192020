"""ctypes binding of the reference-kernel checker ``_ref/librefkern.so``
(test infrastructure only).

The library runs the reference's own CUDA kernels (copied unchanged out of the
reference's gkway/coarsen.hpp and gkway/uncoarsen.hpp when the oracle is built
from a reference tree; see refkern.cu for what runs on the host instead).  The
tests compare its results with the oracle's restatement of the same rules.
Arrays in and out are 0-based int32, as in the oracle.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "librefkern.so")

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u64p = ctypes.POINTER(ctypes.c_uint64)
INIT_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int32, _i32p, _i32p, _i32p, _i32p,
                           ctypes.c_int32, _i32p)
UF_FN = ctypes.CFUNCTYPE(ctypes.c_int32, ctypes.c_int32, _i32p, _i32p, _i32p)

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _c(a, dtype=np.int32) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a: np.ndarray, t=_i32p):
    return a.ctypes.data_as(t)


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what}: reference-kernel checker returned {rc}")


def match(g) -> np.ndarray:
    cand = np.empty(g.n, np.int32)
    x, a, w, vw = (_c(t) for t in (g.xadj, g.adjncy, g.adjwgt, g.vwgt))
    _check(lib().rk_match(g.n, _p(x), _p(a), _p(w), _p(vw), _p(cand)), "matching_with_score")
    return cand


def union_find(cand):
    """HEC_union_find to its fixed point -> (keys u64: (1-based label << 32) | iteration, launches)."""
    cand = _c(cand)
    keys = np.empty(cand.shape[0], np.uint64)
    launches = ctypes.c_int32(0)
    _check(lib().rk_union_find(cand.shape[0], _p(cand), _p(keys, _u64p), ctypes.byref(launches)),
           "HEC_union_find")
    return keys, launches.value


def group_map(root, dist, group_cap: int = 6):
    """Coarse ids from 0-based labels and low bits -> (cmap, nc)."""
    root, dist = _c(root), _c(dist)
    keys = ((root.astype(np.uint64) + 1) << np.uint64(32)) | dist.astype(np.uint64)
    cmap = np.empty(root.shape[0], np.int32)
    nc = ctypes.c_int32(0)
    _check(lib().rk_group_map(root.shape[0], _p(keys, _u64p), group_cap, _p(cmap), ctypes.byref(nc)),
           "group kernels")
    return cmap, nc.value


def coarse_vwgt(vwgt, cmap, nc: int) -> np.ndarray:
    vwgt, cmap = _c(vwgt), _c(cmap)
    out = np.empty(nc, np.int32)
    _check(lib().rk_coarse_vwgt(vwgt.shape[0], _p(vwgt), _p(cmap), nc, _p(out)), "cal_coarsen_vwgt")
    return out


def contract(g, cmap, nc: int):
    x, a, w, cmap = _c(g.xadj), _c(g.adjncy), _c(g.adjwgt), _c(cmap)
    cx = np.empty(nc + 1, np.int32)
    ca = np.empty(max(a.shape[0], 1), np.int32)
    cw = np.empty(max(a.shape[0], 1), np.int32)
    mc = ctypes.c_int64(0)
    _check(lib().rk_contract(g.n, _p(x), _p(a), _p(w), _p(cmap), nc, _p(cx), _p(ca), _p(cw), ctypes.byref(mc)),
           "contraction kernels")
    return cx, ca[:mc.value].copy(), cw[:mc.value].copy()


def expand(cmap, part_c, bnd_c):
    """expand_partition -> (part, boundary, gain, target, updated) of the finer level."""
    cmap, part_c, bnd_c = _c(cmap), _c(part_c), _c(bnd_c)
    n = cmap.shape[0]
    outs = [np.empty(n, np.int32) for _ in range(5)]
    _check(lib().rk_expand(n, _p(cmap), _p(part_c), _p(bnd_c), part_c.shape[0], *(_p(o) for o in outs)),
           "expand_partition")
    return tuple(outs)


def update_vertex_info(g, k: int, part, updated, boundary, gain, target):
    """update_vertex_info on the flagged vertices -> (boundary, gain, target)."""
    x, a, w = _c(g.xadj), _c(g.adjncy), _c(g.adjwgt)
    part, updated = _c(part), _c(updated)
    b, gn, t = _c(boundary).copy(), _c(gain).copy(), _c(target).copy()
    _check(lib().rk_update_vertex_info(g.n, _p(x), _p(a), _p(w), k, _p(part), _p(updated), _p(b), _p(gn), _p(t)),
           "update_vertex_info")
    return b, gn, t


def refine(g, k, maxw, part, boundary, gain, target, updated, pw, move_cap=1024, initial_update=True):
    """One level's refinement loop, with the calling convention of oracle.refine."""
    x, a, w, vw = (_c(t) for t in (g.xadj, g.adjncy, g.adjwgt, g.vwgt))
    part, boundary, gain, target, updated = (_c(t).copy() for t in (part, boundary, gain, target, updated))
    pw = _c(pw, np.int64).copy()
    moves, gsum, rounds = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int32(0)
    _check(lib().rk_refine(g.n, _p(x), _p(a), _p(w), _p(vw), k, ctypes.c_float(maxw), move_cap, _p(part),
                           _p(boundary), _p(gain), _p(target), _p(updated), _p(pw, _i64p), ctypes.byref(moves),
                           ctypes.byref(gsum), int(bool(initial_update)), ctypes.byref(rounds)),
           "refinement kernels")
    return dict(part=part, boundary=boundary, gain=gain, target=target, updated=updated, pw=pw,
                rounds=rounds.value, moves=moves.value, gain_sum=gsum.value)


def cutsize(g, part) -> int:
    x, a, w, part = _c(g.xadj), _c(g.adjncy), _c(g.adjwgt), _c(part)
    cut = ctypes.c_int64(0)
    _check(lib().rk_cutsize(g.n, _p(x), _p(a), _p(w), _p(part), ctypes.byref(cut)), "calculate_cutsize")
    return cut.value


def partition(g, k: int, init, union_find_fn):
    """The reference's whole partitioner on its kernels.

    init(xadj, adjncy, adjwgt, vwgt, k) -> part of the coarsest level (METIS in
    the reference); union_find_fn(cand) -> (root, dist), the labels and low
    bits of the union-find (the oracle's canonical schedule).
    Returns (part, info) with cut, level sizes and refinement rounds."""
    x, a, w, vw = (_c(t) for t in (g.xadj, g.adjncy, g.adjwgt, g.vwgt))
    err = []

    def cb(_user, n, px, pa, pw_, pv, kk, out):
        try:
            m = px[n]
            arrs = [np.ctypeslib.as_array(px, (n + 1,)).copy()]
            for ptr, cnt in ((pa, m), (pw_, m), (pv, n)):
                arrs.append(np.ctypeslib.as_array(ptr, (cnt,)).copy() if cnt else np.zeros(0, np.int32))
            p = np.asarray(init(*arrs, kk), dtype=np.int32)
            ctypes.memmove(out, p.ctypes.data, 4 * n)
            return 0
        except Exception as e:   # reported after the call
            err.append(e)
            return 1

    def ufcb(n, pc, proot, pdist):
        c = np.ctypeslib.as_array(pc, (n,)).copy()
        root, dist = union_find_fn(c)
        ctypes.memmove(proot, _c(root).ctypes.data, 4 * n)
        ctypes.memmove(pdist, _c(dist).ctypes.data, 4 * n)
        return 0

    icb, ucb = INIT_FN(cb), UF_FN(ufcb)
    part = np.empty(g.n, np.int32)
    cut, nlev = ctypes.c_int64(0), ctypes.c_int32(0)
    ln, lm = (ctypes.c_int64 * 64)(), (ctypes.c_int64 * 64)()
    rr = (ctypes.c_int32 * 64)()
    rc = lib().rk_partition(g.n, _p(x), _p(a), _p(w), _p(vw), k, ucb, icb, None, _p(part), ctypes.byref(cut),
                            ctypes.byref(nlev), ln, lm, rr)
    if err:
        raise err[0]
    _check(rc, "reference partitioner")
    L = nlev.value
    return part, dict(cut=cut.value, level_n=list(ln[:L]), level_m=list(lm[:L]),
                      refine_rounds=list(rr[:max(L - 1, 0)]))
