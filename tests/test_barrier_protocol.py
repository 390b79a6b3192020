"""A model of the counting grid barrier (grid_barrier_count in
dac_g-kway_b200/csrc/device_util.cuh), run under random schedules on the CPU.

Each CTA adds (count << 32 | arrival) to word k % 3 at barrier k -- CTA 0 adds
2^31 - (G - 1) to the arrival half, the others 1, so bit 31 sets exactly when
the last CTA arrives -- and polls until it sees bit 31; the last arriver
clears word (k + 2) % 3 before its next arrival.  The model interleaves every
atomic add, poll and clear of G CTAs at random and checks that every CTA reads
each barrier's exact sum, that no CTA passes a barrier early, and that no
schedule deadlocks.  Memory ordering is taken as sequentially consistent:
this checks the protocol's logic (the rotation of three words), not the
release/acquire fences that carry it on the device."""
import random

import pytest

FLIP = 1 << 31
MASK64 = (1 << 64) - 1


def run_schedule(G: int, nbar: int, seed: int):
    rng = random.Random(seed)
    words = [0, 0, 0]                       # cleared before the first counting barrier
    contrib = [[rng.randrange(0, 5000) for _ in range(nbar)] for _ in range(G)]
    want = [sum(contrib[c][k] for c in range(G)) for k in range(nbar)]
    k = [0] * G                             # next barrier of each CTA
    state = ["arrive"] * G                  # arrive | poll | clear | done
    arrived = [0] * nbar                    # CTAs that have added to barrier k
    got = [[None] * nbar for _ in range(G)]
    steps = 0
    while any(s != "done" for s in state):
        steps += 1
        assert steps < 200 * G * nbar, "no progress: a schedule deadlocked"
        c = rng.choice([i for i in range(G) if state[i] != "done"])
        b = k[c]
        w = b % 3
        if state[c] == "arrive":
            add = (contrib[c][b] << 32) | ((FLIP - (G - 1)) if c == 0 else 1)
            old = words[w]
            words[w] = (old + add) & MASK64
            arrived[b] += 1
            cur = words[w]
            if cur & FLIP:                  # the last arrival
                assert arrived[b] == G
                got[c][b] = cur >> 32
                state[c] = "clear"
            else:
                state[c] = "poll"
        elif state[c] == "poll":
            cur = words[w]
            if cur & FLIP:
                assert arrived[b] == G, "a CTA passed a barrier before every CTA arrived"
                got[c][b] = cur >> 32
                k[c] += 1
                state[c] = "arrive" if k[c] < nbar else "done"
        elif state[c] == "clear":
            words[(b + 2) % 3] = 0
            k[c] += 1
            state[c] = "arrive" if k[c] < nbar else "done"
    for c in range(G):
        assert got[c] == want, (G, seed, c)


@pytest.mark.parametrize("G", [2, 3, 7, 32])
def test_counting_barrier_sums_under_random_schedules(G):
    for seed in range(40):
        run_schedule(G, nbar=30, seed=seed * 7919 + G)


def test_counting_barrier_words_never_carry():
    """The arrival half of a cleared word sums to exactly 2^31, so it never
    carries into the count half, for any grid size up to 2^31 CTAs."""
    for G in (2, 148, 296, 1 << 20):
        assert (FLIP - (G - 1)) + (G - 1) == FLIP < (1 << 32)
