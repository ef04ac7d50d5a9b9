"""The prime-factor + Rader transform plans of the pressure solve, on the host.

The device engine (wildfires_b200/csrc/fft_pr.cuh) and its host tables (plan_pr
in wildfires_b200/csrc/solver.cu) split a length n = N1 P into an N1-point DFT
and N1 Rader transforms of the prime P, whose cyclic convolutions of length
P - 1 = F1 F2 F3 are Good-Thomas transforms over the factors.  This test
restates the same index maps and the same passes in numpy, slot by slot in the
engine's shared-memory layout, and holds the result to numpy's FFT for every
compiled plan, forward and inverse, in the plain run and in the slotted run the
x transform uses (its copies place the line in the slot table's order); so the
plan arithmetic is pinned without a GPU (the GPU tests hold the engine itself
to the oracle).
"""
import os
import re

import numpy as np
import pytest


def compiled_plans():
    """(N1, P, F1, F2, F3) of every plan the library compiles (the PrPlans list
    of wildfires_b200/csrc/poisson.cu)."""
    src = open(os.path.join(os.path.dirname(__file__), "..", "wildfires_b200", "csrc", "poisson.cu")).read()
    block = src[src.index("using PrPlans = PlanList<"):]
    block = block[:block.index(";")]
    plans = [tuple(int(v) for v in m.groups(default="1"))
             for m in re.finditer(r"PrPlan<(\d+), (\d+), (\d+), (\d+)(?:, (\d+))?>", block)]
    assert plans, "no plan found in poisson.cu"
    return plans


PLANS = compiled_plans()


def primitive_root(P):
    fac, x, r = [], P - 1, 2
    while x > 1:
        if x % r == 0:
            fac.append(r)
            while x % r == 0:
                x //= r
        r += 1
    return next(g for g in range(2, P) if all(pow(g, (P - 1) // q, P) != 1 for q in fac))


def inv_mod(a, m):
    return next((t for t in range(m) if a * t % m == 1 % m), 0)


def tables(N1, P, F1, F2, F3):
    """The host tables: slot map, output map, B' in (j1, jM, jL) order, e1."""
    n, Q = N1 * P, P - 1
    M, L = (F2, F3) if F3 > 1 else (1, F2)
    g = primitive_root(P)
    gi = pow(g, P - 2, P)
    e2 = N1 * inv_mod(N1 % P, P) % n
    e1 = P * inv_mod(P % N1, N1) % n if N1 > 1 else 0
    pmap = [0] * (P + Q)
    for q1 in range(F1):
        for qm in range(M):
            for ql in range(L):
                q = ((Q // F1) * q1 + (Q // M) * qm + (Q // L) * ql) % Q
                slot = (q1 * M + qm) * L + ql
                pmap[1 + slot] = pow(g, q, P)
                pmap[P + slot] = e2 * pow(gi, q, P) % n
    b = np.exp(-2j * np.pi * np.array([pow(gi, t, P) for t in range(Q)]) / P)
    B = np.fft.fft(b) / Q

    def weight(F):
        return (Q // F) * inv_mod((Q // F) % F, F) if F > 1 else 0

    c1, cm, cl = weight(F1), weight(M), weight(L)
    rb = np.zeros(Q, complex)
    for j1 in range(F1):
        for jm in range(M):
            for jl in range(L):
                rb[(j1 * M + jm) * L + jl] = B[(j1 * c1 + jm * cm + jl * cl) % Q]
    return pmap, rb, e1, M, L


def engine(x, N1, P, F1, F2, F3, inverse=False, slotted=False):
    """The engine's passes on a line buffer laid out as in shared memory.
    slotted: the line arrives in the slot table's order (input x[j] at its
    slot) and leaves in it (X[k] at its slot), as the x kernel stages it;
    pass A then reads slot n1 SS + u and B3 writes slot m1 UB + u."""
    n = N1 * P
    pmap, rb, e1, M, L = tables(N1, P, F1, F2, F3)
    SS = P + ((M * L - P) % 8 + 8) % 8
    UB = N1 * M * L
    buf = np.zeros(max(n, N1 * SS) + 8, complex)
    xin = np.conj(x) if inverse else x.copy()
    if slotted:
        ins, outs, _, _ = slot_tables(N1, P, F1, F2, F3)
        buf[ins] = xin
    D = np.fft.fft

    def ID(v):
        return np.conj(D(np.conj(v)))

    def pos(k1, a, bm, cl):
        return k1 * SS + 1 + (a * M + bm) * L + cl

    for u in range(P):                                         # pass A: DFT_N1
        if slotted:                                            # one round at a time, own slots
            v = D(np.array([buf[n1 * SS + u] for n1 in range(N1)]))
        else:
            v = D(np.array([xin[(N1 * pmap[u] + P * n1) % n] for n1 in range(N1)]))
        for k1 in range(N1):
            buf[k1 * SS + u] = v[k1]
    for k1 in range(N1):
        for qm in range(M):                                    # B1: DFT_F1 over q1
            for ql in range(L):
                idx = [pos(k1, q1, qm, ql) for q1 in range(F1)]
                buf[idx] = D(buf[idx])
        for j1 in range(F1):                                   # B2a: DFT_M over qM
            for ql in range(L):
                idx = [pos(k1, j1, qm, ql) for qm in range(M)]
                buf[idx] = D(buf[idx])
        for j1 in range(F1):                                   # B2: DFT_L, * B', IDFT_L
            for jm in range(M):
                idx = [pos(k1, j1, jm, ql) for ql in range(L)]
                v = D(buf[idx])
                a0 = 0.0
                if j1 == 0 and jm == 0:
                    a0 = buf[k1 * SS]
                    buf[k1 * SS] = a0 + v[0]
                v = v * rb[(j1 * M + jm) * L:(j1 * M + jm) * L + L]
                v[0] += a0
                buf[idx] = ID(v)
        for j1 in range(F1):                                   # B2b: IDFT_M over jM
            for ml in range(L):
                idx = [pos(k1, j1, jm, ml) for jm in range(M)]
                buf[idx] = ID(buf[idx])
    out = np.zeros(n, complex)
    slots = np.zeros(n, complex)
    for k1 in range(N1):                                       # B3: IDFT_F1, outputs
        kb = k1 * e1 % n
        for mm in range(M):
            for ml in range(L):
                y = ID(buf[[pos(k1, j1, mm, ml) for j1 in range(F1)]])
                for m1 in range(F1):
                    k = (kb + pmap[P + (m1 * M + mm) * L + ml]) % n
                    out[k] = np.conj(y[m1]) if inverse else y[m1]
                    slots[m1 * UB + k1 * M * L + mm * L + ml] = out[k]
        out[kb] = np.conj(buf[k1 * SS]) if inverse else buf[k1 * SS]
        slots[F1 * UB + k1] = out[kb]
    return slots[outs] if slotted else out


@pytest.mark.parametrize("slotted", [False, True], ids=["plain", "slotted"])
@pytest.mark.parametrize("plan", PLANS, ids=lambda p: "n%d" % (p[0] * p[1]))
def test_rader_plan_matches_numpy_fft(plan, slotted):
    n = plan[0] * plan[1]
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    fwd = engine(x, *plan, slotted=slotted)
    inv = engine(x, *plan, inverse=True, slotted=slotted)
    assert np.max(np.abs(fwd - np.fft.fft(x))) <= 1e-13 * np.max(np.abs(fwd))
    assert np.max(np.abs(inv - n * np.fft.ifft(x))) <= 1e-13 * np.max(np.abs(inv))


@pytest.mark.parametrize("plan", PLANS, ids=lambda p: "n%d" % (p[0] * p[1]))
def test_rader_plan_slots_are_a_permutation(plan):
    """The slot map covers every input index once and the output map every
    output index once (apart from the DC term of each sub-line)."""
    N1, P = plan[0], plan[1]
    pmap, _, e1, _, _ = tables(*plan)
    assert sorted(pmap[:P]) == list(range(P))
    outs = sorted(((k1 * e1) + pmap[P + s]) % (N1 * P) for k1 in range(N1) for s in range(P - 1))
    outs += [k1 * e1 % (N1 * P) for k1 in range(N1)]
    assert sorted(outs) == list(range(N1 * P))


def slot_tables(N1, P, F1, F2, F3):
    """The slot table of the slotted run (plan_pr in wildfires_b200/csrc/solver.cu):
    input x[j] at n1 SS + u for j = N1 map[u] + P n1 (mod n); output X[k] at
    m1 UB + u (u = k1 M L + w) or, for the DC term of k1, at F1 UB + k1."""
    n = N1 * P
    pmap, _, e1, M, L = tables(N1, P, F1, F2, F3)
    SS = P + ((M * L - P) % 8 + 8) % 8
    UB = N1 * M * L
    ins, outs = [-1] * n, [-1] * n
    for u in range(P):
        for n1 in range(N1):
            ins[(N1 * pmap[u] + P * n1) % n] = n1 * SS + u
    for k1 in range(N1):
        kb = k1 * e1 % n
        for w in range(M * L):
            for m1 in range(F1):
                outs[(kb + pmap[P + w + M * L * m1]) % n] = m1 * UB + k1 * M * L + w
        outs[kb] = F1 * UB + k1
    return ins, outs, SS, UB


@pytest.mark.parametrize("plan", PLANS, ids=lambda p: "n%d" % (p[0] * p[1]))
def test_slot_tables_are_the_passes_permutations(plan):
    """Every input lands on the slot pass A reads for it (distinct slots inside
    the N1 sub-lines), and every output slot is the one pass B3 posts that
    output to (each of the n slots exactly once)."""
    N1, P, F1 = plan[0], plan[1], plan[2]
    n = N1 * P
    ins, outs, SS, UB = slot_tables(*plan)
    assert min(ins) >= 0 and len(set(ins)) == n and max(ins) < N1 * SS
    assert sorted(outs) == list(range(n))
    pmap, _, e1, M, L = tables(*plan)
    # pass A's gather: slot n1 SS + u holds x[N1 map[u] + P n1]
    for j in range(n):
        n1, u = divmod(ins[j], SS)
        assert (N1 * pmap[u] + P * n1) % n == j
    # pass B3's scatter: slot m1 UB + u is the output the unit (k1, w) =
    # divmod(u, M L) posts for m1, slot F1 UB + k1 the DC term of k1
    for k in range(n):
        s = outs[k]
        if s < F1 * UB:
            m1, u = divmod(s, UB)
            k1, w = divmod(u, M * L)
            assert (k1 * e1 + pmap[P + w + M * L * m1]) % n == k
        else:
            assert (s - F1 * UB) * e1 % n == k
