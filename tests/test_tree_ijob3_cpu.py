"""The tree form of dlaebz IJOB=3, restated on the CPU.

Range I needs the intervals that hold eigenvalues il-1 and iu
(SRC/mrrr_val.c:295-319 on the whole matrix, the dlarrd set-up on each
block, SRC/LAPACK/odrrd.f): a bisection from a given first point whose every
step is a Sturm count over all n rows.  On the device (`dv_ijob3_tree`) a
group of L lanes runs it: after the first count, the midpoints of the next
log2(L) steps form a binary tree that follows from the current interval,
each lane counts at one node, and the group walks the tree with the loop's
updates and tests.  The claim is that the walk ends on the sequential
loop's interval and counts bit for bit, iteration cap included.  This test
restates both in plain Python (IEEE double arithmetic, the same operations)
and compares them.
"""
import numpy as np
import pytest


def sturm(d, e2, pivmin, c):
    """Sturm count with the IJOB=2/3 rule (odebz.f loop 90); e2[j-1] is the
    squared off-diagonal entry above row j."""
    t = d[0] - c
    cnt = 0
    if t <= pivmin:
        cnt = 1
        t = min(t, -pivmin)
    for j in range(1, len(d)):
        t = d[j] - e2[j - 1] / t - c
        if t <= pivmin:
            cnt += 1
            t = min(t, -pivmin)
    return cnt


def ijob3(d, e2, piv, abstol, reltol, nitmax, nval, c, a, b, na, nb):
    """The sequential loop (dv_ijob3, odebz.f IJOB=3)."""
    for _ in range(1, nitmax + 1):
        k = sturm(d, e2, piv, c)
        if k <= nval:
            a, na = c, k
        if k >= nval:
            b, nb = c, k
        w = abs(b - a)
        t = max(abs(b), abs(a))
        if w < max(max(abstol, piv), reltol * t) or na >= nb:
            break
        c = 0.5 * (a + b)
    return a, b, na, nb


def ijob3_tree(L, d, e2, piv, abstol, reltol, nitmax, nval, c, a, b, na, nb):
    """The group walk of dv_ijob3_tree with L lanes."""
    depth = L.bit_length() - 1
    tol0 = max(abstol, piv)
    it = 0
    done = nitmax < 1
    if not done:
        k = sturm(d, e2, piv, c)
        if k <= nval:
            a, na = c, k
        if k >= nval:
            b, nb = c, k
        it = 1
        done = (abs(b - a) < max(tol0, reltol * max(abs(b), abs(a))) or na >= nb
                or it >= nitmax)
    while not done:
        raw = []
        for lane in range(L):   # lane t counts at heap node max(t, 1)
            node = max(lane, 1)
            lo, hi = a, b
            for bit in range(node.bit_length() - 2, -1, -1):
                m = 0.5 * (lo + hi)
                if (node >> bit) & 1:
                    lo = m
                else:
                    hi = m
            raw.append(sturm(d, e2, piv, 0.5 * (lo + hi)))
        node = 1
        for _ in range(depth):
            cv = raw[node]
            if not done:
                cm = 0.5 * (a + b)
                if cv <= nval:
                    a, na = cm, cv
                if cv >= nval:
                    b, nb = cm, cv
                node = 2 * node + 1 if cv < nval else 2 * node
                it += 1
                done = (abs(b - a) < max(tol0, reltol * max(abs(b), abs(a))) or na >= nb
                        or it >= nitmax)
    return a, b, na, nb


def _matrices():
    rng = np.random.default_rng(7)
    for k in range(24):
        n = int(rng.integers(4, 48))
        if k % 4 == 0:       # 1-2-1: equally spaced, well separated
            d, e = np.full(n, 2.0), np.ones(n - 1)
        elif k % 4 == 1:     # glued Wilkinson-like: near-degenerate pairs
            h = n // 2
            d = np.abs(np.arange(n) - h).astype(float)
            e = np.ones(n - 1)
            e[h - 1] = 1e-12
        else:
            d, e = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n - 1)
        yield k, d, e * e, e


@pytest.mark.parametrize("L", [2, 4, 16, 32])
def test_tree_ijob3_equals_sequential_loop(L):
    eps = np.finfo(float).eps
    checked = 0
    for k, d, e2, e in _matrices():
        n = len(d)
        piv = np.finfo(float).tiny * max(1.0, float(e2.max()))
        r = np.r_[0.0, np.abs(e)] + np.r_[np.abs(e), 0.0]
        gl, gu = float((d - r).min()) - 1e-9, float((d + r).max()) + 1e-9
        for nval, c in ((k % n, gl), (n - k % n, gu), (n // 2, gl)):
            for nitmax in (1, 3, 7, 80):
                args = (d, e2, piv, 1e-300, 4 * eps, nitmax, nval, c, gl, gu, -1, n + 1)
                assert ijob3_tree(L, *args) == ijob3(*args), (k, nval, nitmax)
                checked += 1
    assert checked == 24 * 3 * 4
