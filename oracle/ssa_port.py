"""ORACLE TEST INFRASTRUCTURE — not part of the product; only tests/ import it.

A CPU restatement of MarkovKit's gillespie (markovkit/ssa.hpp:42-74) over a reaction network
with tabulated propensities, drawing its random numbers from the same stream the device uses, so
that device paths can be checked sample by sample:

- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011): key = the seed's two 32-bit halves,
  counter = (draw counter low, high, path low, high); pinned by the authors' known-answer
  vectors in tests/test_ssa_oracle.py;
- a uniform double in [0, 1) from the top 53 bits of each 64-bit half of a block, the first
  half first;
- per jump: wait -log(1 - u) / total, then the first reaction whose cumulative listed rate
  exceeds u * total (rates summed in reaction order, unlisted ones skipped).

The reference itself draws from a host generator (num::rng, whose source is absent with the
numerics library), so this pins the algorithm and the stream, not the reference's samples.
Pure-Python loops: a few paths only.
"""

from __future__ import annotations

import math

_MASK = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    """one Philox4x32-10 block: ctr four 32-bit words, key two"""
    x0, x1, x2, x3 = ctr
    a, b = key
    for _ in range(10):
        p0 = 0xD2511F53 * x0
        p1 = 0xCD9E8D57 * x2
        x0, x1, x2, x3 = ((p1 >> 32) ^ x1 ^ a) & _MASK, p1 & _MASK, ((p0 >> 32) ^ x3 ^ b) & _MASK, p0 & _MASK
        a = (a + 0x9E3779B9) & _MASK
        b = (b + 0xBB67AE85) & _MASK
    return x0, x1, x2, x3


class Stream:
    """the uniforms of one path"""

    def __init__(self, seed: int, path: int):
        self.key = (seed & _MASK, (seed >> 32) & _MASK)
        self.path = path
        self.draw = 0
        self.spare = None

    def uniform(self) -> float:
        if self.spare is not None:
            u, self.spare = self.spare, None
            return u
        o = philox4x32_10((self.draw & _MASK, (self.draw >> 32) & _MASK, self.path & _MASK, (self.path >> 32) & _MASK),
                          self.key)
        self.draw += 1
        m0 = ((o[0] << 32) | o[1]) >> 11
        m1 = ((o[2] << 32) | o[3]) >> 11
        self.spare = m1 * 2.0 ** -53
        return m0 * 2.0 ** -53


def gillespie(change, rates, bounds, initial, final_time, seed, path, max_jumps=None):
    """(times, states) of path `path`, as ssa.hpp:42-74 builds them; rates[r][box index] with
    species 0 most significant; raises when the path would leave the box"""
    S = len(initial)
    stride = [1] * S
    for s in range(S - 2, -1, -1):
        stride[s] = stride[s + 1] * (bounds[s + 1] + 1)
    rng = Stream(seed, path)
    x = list(initial)
    times, states = [0.0], [tuple(x)]
    t = 0.0
    jumps = 0
    cap = max_jumps if max_jumps is not None else 1 << 62
    while jumps < cap:
        idx = sum(x[s] * stride[s] for s in range(S))
        a = []
        total = 0.0
        for r, ch in enumerate(change):
            rate = rates[r][idx]
            ok = all(x[s] + ch[s] >= 0 for s in range(S)) and rate > 0.0
            a.append(rate if ok else 0.0)
            if ok:
                total += rate
        if not total > 0.0:
            break
        t += -math.log(1.0 - rng.uniform()) / total
        if t > final_time:
            break
        target = rng.uniform() * total
        acc, chosen = 0.0, -1
        for r, ar in enumerate(a):
            if ar > 0.0:
                acc += ar
                if chosen < 0 and target < acc:
                    chosen = r
        if chosen < 0:
            chosen = max(r for r, ar in enumerate(a) if ar > 0.0)
        y = [x[s] + change[chosen][s] for s in range(S)]
        if any(y[s] > bounds[s] for s in range(S)):
            raise OverflowError("the path leaves the box")
        x = y
        jumps += 1
        times.append(t)
        states.append(tuple(x))
    if jumps < cap:
        times.append(final_time)
        states.append(tuple(x))
    return times, states
