"""Host emulation of the fused kernel's Jacobi schedule (update2q.cu).

Replays, with the kernel's own index arithmetic, which column pairs each
sweep rotates -- intra-duo round, duo round robin inside each slot, cross
rounds between the two slots, and the alternating slot exchanges between the
two CTAs -- and checks that every pair of the C_pad columns is visited exactly
once per sweep and that no round gives a column to two warps.
"""
import itertools

import pytest

K_WARPS = 16


def rr_elem(k, r, nd2):
    return 0 if k == 0 else 1 + (k - 1 + r) % (nd2 - 1)


def step_pairs(slots, w, internal):
    """Column pairs (by global id) one CTA rotates in one block-step; also checks per-round disjointness."""
    nd = w // 2
    col = lambda s, j: slots[s][j]
    out = []

    def round_(tasks):
        seen = set()
        for cols in tasks:
            for c in cols:
                assert c not in seen, "column used twice in one round"
                seen.add(c)

    if internal:
        tasks = []
        for t in range(2 * nd):
            slot, d = divmod(t, nd)
            tasks.append((col(slot, 2 * d), col(slot, 2 * d + 1)))
            out.append((col(slot, 2 * d), col(slot, 2 * d + 1)))
        round_(tasks)
        nd2 = nd + (nd & 1)
        half = nd2 // 2
        for r in range(nd2 - 1):
            tasks = []
            for t in range(2 * half):
                slot, k = divmod(t, half)
                u, v = rr_elem(k, r, nd2), rr_elem(nd2 - 1 - k, r, nd2)
                if u < nd and v < nd:
                    cs = [col(slot, 2 * u), col(slot, 2 * u + 1), col(slot, 2 * v), col(slot, 2 * v + 1)]
                    tasks.append(cs)
                    out += [(cs[0], cs[2]), (cs[1], cs[3]), (cs[0], cs[3]), (cs[1], cs[2])]
            round_(tasks)
    for r in range(nd):
        tasks = []
        for t in range(nd):
            v = (t + r) % nd
            cs = [col(0, 2 * t), col(0, 2 * t + 1), col(1, 2 * v), col(1, 2 * v + 1)]
            tasks.append(cs)
            out += [(cs[0], cs[2]), (cs[1], cs[3]), (cs[0], cs[3]), (cs[1], cs[2])]
        round_(tasks)
    return out


def exchange(cta_slots, parity):
    my0 = 1                      # CTA0 always sends slot 1
    my1 = parity                 # CTA1 sends slot 0 (A) or slot 1 (B)
    cta_slots[0][my0], cta_slots[1][my1] = cta_slots[1][my1], cta_slots[0][my0]


@pytest.mark.parametrize("c", [2, 4, 6, 8, 10, 16, 18, 32, 34, 62, 64, 96, 128])
def test_every_pair_once_per_sweep(c):
    cpad = (c + 7) // 8 * 8
    w = cpad // 4
    # CTA c, local column j -> global id c*2w + j; slot s holds local columns [s*w, s*w+w)
    cta_slots = [[[cr * 2 * w + s * w + j for j in range(w)] for s in range(2)] for cr in range(2)]
    parity = 0
    for sweep in range(4):
        seen = []
        for step in range(3):
            for cr in range(2):
                seen += step_pairs(cta_slots[cr], w, step == 0)
            exchange(cta_slots, parity)
            parity ^= 1
        norm = sorted(tuple(sorted(p)) for p in seen)
        assert len(norm) == len(set(norm)), "a pair was rotated twice in one sweep"
        assert set(norm) == set(itertools.combinations(range(cpad), 2))
        assert len(norm) <= K_WARPS * 10 ** 6
