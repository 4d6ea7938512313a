"""Host emulation of the fused kernel's Jacobi schedule (update2q.cu).

Replays, with the kernel's own index arithmetic, which column pairs each
sweep rotates -- inner pairs of every column quad, the quad round robin inside
each slot, the cross rounds between the two slots, and the alternating slot
exchanges between the two CTAs -- and checks that every pair of the C_pad
columns is visited exactly once per sweep, that no round gives a column to two
warps, and that the four rotations of each rotate4 phase are disjoint.
"""
import itertools

import pytest

K_WARPS = 16


def rr_elem(k, r, nd2):
    return 0 if k == 0 else 1 + (k - 1 + r) % (nd2 - 1)


N_WARPS = 8


def quad_cross(P, Q):
    """Pairs of quad_cross(): phase k pairs P_i with Q_{(i+k) mod 4}."""
    out = []
    for k in range(4):
        ph = [(P[i], Q[(i + k) % 4]) for i in range(4)]
        flat = [c for pr in ph for c in pr]
        assert len(set(flat)) == 8, "a phase reuses a column"
        out += ph
    return out


def quad_inner2(A, B):
    """Pairs of quad_inner2(): phases (01|23), (02|13), (03|12) of both quads."""
    out = []
    for (i, j), (k, l) in (((0, 1), (2, 3)), ((0, 2), (1, 3)), ((0, 3), (1, 2))):
        ph = [(A[i], A[j]), (A[k], A[l]), (B[i], B[j]), (B[k], B[l])]
        flat = [c for pr in ph for c in pr]
        assert len(set(flat)) == 8, "a phase reuses a column"
        out += ph
    return out


def step_pairs(slots, w, internal):
    """Column pairs (by global id) one CTA rotates in one block-step, following
    internal_rounds() and cross_rounds() in update2q.cu, with per-round column
    disjointness across warps."""
    nq = w // 4
    quad = lambda s, q: [slots[s][4 * q + k] for k in range(4)]
    out = []

    def round_(tasks):
        flat = [c for cols in tasks for c in cols]
        assert len(set(flat)) == len(flat), "column used twice in one round"

    if internal:
        tasks = []
        for warp in range(N_WARPS):
            for t in range(2 * warp, 2 * nq, 2 * N_WARPS):
                A, B = quad(*divmod(t, nq)), quad(*divmod(t + 1, nq))
                tasks.append(A + B)
                out += quad_inner2(A, B)
        round_(tasks)
        nq2 = nq + (nq & 1)
        half = nq2 // 2
        for r in range(nq2 - 1):
            tasks = []
            for warp in range(N_WARPS):
                for t in range(warp, 2 * half, N_WARPS):
                    slot, k = divmod(t, half)
                    u, v = rr_elem(k, r, nq2), rr_elem(nq2 - 1 - k, r, nq2)
                    if u < nq and v < nq:
                        P, Q = quad(slot, u), quad(slot, v)
                        tasks.append(P + Q)
                        out += quad_cross(P, Q)
            round_(tasks)
    for r in range(nq):
        tasks = []
        for t in range(min(nq, N_WARPS)):
            P, Q = quad(0, t), quad(1, (t + r) % nq)
            tasks.append(P + Q)
            out += quad_cross(P, Q)
        round_(tasks)
    return out


def exchange(cta_slots, parity):
    my0 = 1                      # CTA0 always sends slot 1
    my1 = parity                 # CTA1 sends slot 0 (A) or slot 1 (B)
    cta_slots[0][my0], cta_slots[1][my1] = cta_slots[1][my1], cta_slots[0][my0]


@pytest.mark.parametrize("c", [2, 4, 6, 8, 10, 16, 18, 32, 34, 62, 64, 96, 128])
def test_every_pair_once_per_sweep(c):
    cpad = (c + 15) // 16 * 16
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
