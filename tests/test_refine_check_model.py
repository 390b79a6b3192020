"""A model of the level kernel's sort-free balance check (refine_check_risk in
dac_g-kway_b200/csrc/refine.cu) against the reference's definition of the
balanced prefix, on random rounds on the CPU.

Reference rule (uncoarsen.hpp:239-288, 471-488): sort the round's candidate
moves by (gain desc, vertex asc); index j is balanced when every part p whose
running weight change D[p][j] after moves 0..j is positive keeps
(float)(pw[p] + D[p][j]) <= MAXW; moves 0..pos apply, pos = the LARGEST
balanced index (Q11), index 0 counting as balanced.

The check instead (i) flags the parts whose inflow bound passes MAXW, (ii)
lets every move apply when no flagged part ends over MAXW at the last index,
and otherwise (iii) turns the moves into or out of flagged parts into events,
marks for each event with D > 0 and (float)(pw + D) > MAXW the key range up to
its part's next event, and applies the moves whose keys are at most the
largest unmarked key (the smallest key when every key is marked)."""
import numpy as np

INT_MAX = (1 << 31) - 1


def f32(x: int) -> np.float32:
    return np.float32(np.uint32(x & 0xFFFFFFFF))


def reference_applied(moves, pw, maxw):
    """moves: list of (key, src, dst, w). Returns the number of moves applied."""
    order = sorted(moves)
    D = {}
    pos = 0
    for j, (_, s, d, w) in enumerate(order):
        D[d] = D.get(d, 0) + w
        D[s] = D.get(s, 0) - w
        if all(not (v > 0 and f32(pw[p] + v) > maxw) for p, v in D.items()):
            pos = j
    return pos + 1


def check_applied(moves, pw, maxw):
    inflow, net = {}, {}
    for _, s, d, w in moves:
        inflow[d] = inflow.get(d, 0) + w
        net[d] = net.get(d, 0) + w
        net[s] = net.get(s, 0) - w
    # (i) the inflow bound grows with every candidate; one add past MAXW flags the part
    flagged = {p for p, v in inflow.items() if pw[p] + v >= (1 << 32) or f32(pw[p] + v) > maxw}
    # (ii) the last index
    if not any(net.get(p, 0) > 0 and f32(pw[p] + net[p]) > maxw for p in flagged):
        return len(moves)
    # (iii) events of flagged parts, marked key ranges, the largest unmarked key
    events = {}
    for key, s, d, w in moves:
        if s in flagged:
            events.setdefault(s, []).append((key, -w))
        if d in flagged:
            events.setdefault(d, []).append((key, w))
    ranges = []
    for p, ev in events.items():
        for key, _ in ev:
            D = sum(dw for k2, dw in ev if k2 <= key)
            nxt = min((k2 for k2, _ in ev if k2 > key), default=None)
            if D > 0 and f32(pw[p] + D) > maxw:
                ranges.append((key, nxt))
    keys = [m[0] for m in moves]
    unmarked = [k for k in keys if not any(lo <= k and (hi is None or k < hi) for lo, hi in ranges)]
    kstar = max(unmarked) if unmarked else min(keys)
    return sum(1 for k in keys if k <= kstar)


def random_round(rng):
    k = int(rng.integers(2, 12))
    cnt = int(rng.integers(1, 40))
    base = int(rng.integers(0, 200))
    pw = [base + int(rng.integers(0, 60)) for _ in range(k)]
    maxw = np.float32(base + rng.integers(20, 90))
    verts = rng.choice(10 * cnt, size=cnt, replace=False)
    moves = []
    for v in verts:
        s = int(rng.integers(0, k))
        d = int((s + rng.integers(1, k)) % k)
        gain = int(rng.integers(1, 6))                  # ties in gain: the vertex id decides
        w = int(rng.integers(0, 25)) if rng.random() < 0.9 else 0
        moves.append((((INT_MAX - gain) << 32) | int(v), s, d, w))
    return moves, pw, maxw


def test_sort_free_check_equals_the_largest_balanced_index():
    rng = np.random.default_rng(20261204)
    for _ in range(3000):
        moves, pw, maxw = random_round(rng)
        assert check_applied(moves, pw, maxw) == reference_applied(moves, pw, maxw), (moves, pw, maxw)


def test_float_rounding_of_large_part_weights():
    # above 2^24 a float step is larger than 1: the reference compares in float
    rng = np.random.default_rng(7)
    for _ in range(500):
        moves, pw, maxw = random_round(rng)
        pw = [p + (1 << 25) for p in pw]
        maxw = np.float32(float(maxw) + (1 << 25))
        assert check_applied(moves, pw, maxw) == reference_applied(moves, pw, maxw)
