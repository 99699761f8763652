"""The pair walk's leaf rule on the CPU: a node's leaf triangles tested together, each accepted pair
entering its owner's slot as the minimum of (distance bits << 32 | pair index), give the result of
Photon's sequential leaf walk (traverse.h:93-104: a triangle is accepted when its distance is below the
current tmax, which it then lowers), for closest hits, and the first accepted pair for any-hit walks.
The cases draw exact distance ties, rejected (alpha-masked) candidates, distances at and beyond tmax,
NaN and pairs split across two rounds of 32, on which the owner's tmax drops between rounds."""
import numpy as np

ROUND = 32


def sequential(ts, ok, tmax, any_hit):
    """Photon's order: one triangle at a time; returns (index, distance) of the hit, or (-1, tmax)."""
    best = -1
    for j, (t, a) in enumerate(zip(ts, ok)):
        if a and t > 0.0 and t < tmax:  # NaN compares false, as in the intersection test
            tmax, best = t, j
            if any_hit:
                break
    return best, tmax


def pair_rule(ts, ok, tmax, any_hit):
    """The pair pass: rounds of 32 pairs; within a round every pair is tested against the owner's tmax
    at the round's start and enters a 64-bit minimum; between rounds the owner takes its minimum."""
    best, answered = -1, False
    for base in range(0, len(ts), ROUND):
        slot = None
        for p in range(base, min(base + ROUND, len(ts))):
            t, a = ts[p], ok[p]
            round_tmax = 0.0 if answered else tmax
            if a and t > 0.0 and t < round_tmax:
                bits = int(np.float32(t).view(np.uint32))
                key = p if any_hit else (bits << 32) | p
                slot = key if slot is None else min(slot, key)
        if slot is not None:
            best = slot & 0xFFFFFFFF
            if any_hit:
                answered = True
            else:
                tmax = float(np.uint32(slot >> 32).view(np.float32))
    return best, tmax


def test_pair_rule_equals_the_sequential_leaf_walk():
    rng = np.random.default_rng(11)
    cases = 0
    for trial in range(4000):
        n = int(rng.integers(1, 70))  # up to three rounds of 32
        pool = rng.random(max(1, n // 3)).astype(np.float32) * 10  # shared values: exact ties
        ts = np.where(rng.random(n) < 0.5, rng.choice(pool, n), rng.random(n).astype(np.float32) * 10).astype(np.float32)
        ts[rng.random(n) < 0.05] = np.float32(np.nan)
        ts[rng.random(n) < 0.05] = np.float32(-1.0)
        ok = rng.random(n) < 0.8  # the rest: alpha-masked candidates that let the ray through
        tmax = np.float32(np.inf) if trial % 3 == 0 else np.float32(rng.random() * 12)
        if trial % 7 == 0 and n:
            ts[int(rng.integers(0, n))] = tmax  # a distance equal to tmax is not accepted
        for any_hit in (False, True):
            want = sequential(ts.tolist(), ok.tolist(), float(tmax), any_hit)
            got = pair_rule(ts.tolist(), ok.tolist(), float(tmax), any_hit)
            assert got[0] == want[0], (trial, any_hit, got, want)
            if not any_hit:
                assert np.float32(got[1]) == np.float32(want[1]) or (want[0] < 0 and got[0] < 0)
            cases += 1
    assert cases == 8000
