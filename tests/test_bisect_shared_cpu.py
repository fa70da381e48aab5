"""The shared-interval bisection of stage A, restated on the CPU.

The device runs dlarrd's per-eigenvalue bisection (dlaebz IJOB=2 loop,
SRC/LAPACK/odebz.f loops 90-120) breadth-first: the intervals that several
eigenvalues of a block share are counted once (k_bis_count), and each
eigenvalue continues alone once a count separates it (k_bisect_cont).  The
claim is that every eigenvalue then sees exactly the operations of its own
sequential loop.  This test restates both orders in plain Python (IEEE
double arithmetic, the same operations) and checks that they give the same
intervals bit for bit, including the depth limit after which the tree's
remaining nodes are split into single states.
"""
import numpy as np
import pytest


def sturm(d, e2, pivmin, c):
    """Sturm count with the IJOB=2/3 rule (odebz.f loop 90)."""
    t = d[0] - c
    cnt = 0
    if t <= pivmin:
        cnt = 1
        t = min(t, -pivmin)
    for j in range(1, len(d)):
        t = d[j] - e2[j] / t - c
        if t <= pivmin:
            cnt += 1
            t = min(t, -pivmin)
    return cnt


def converged(a, b, abstol, pivmin, reltol):
    return abs(b - a) < max(max(abstol, pivmin), reltol * max(abs(b), abs(a)))


def bisect_one(d, e2, pivmin, abstol, reltol, itmax, j, a, b, na, nb, it0=0):
    """One eigenvalue's loop (dv_bisect_one), optionally continued after it0 steps."""
    c = 0.5 * (a + b)
    for it in range(it0 + 1, itmax + 1):
        cnt = min(nb, max(na, sturm(d, e2, pivmin, c)))
        if j <= cnt:
            b, nb = c, cnt
        else:
            a, na = c, cnt
        if converged(a, b, abstol, pivmin, reltol) or na >= nb:
            break
        c = 0.5 * (a + b)
    return a, b


def bisect_shared(d, e2, pivmin, abstol, reltol, itmax, gl, gu, nab1, nab2, depth_cap):
    """Breadth-first over the shared intervals (k_bis_roots/count/scatter),
    then the single eigenvalues continued alone (k_bisect_cont)."""
    out = {}
    singles = []
    if nab2 - nab1 == 1:
        singles.append((gl, gu, nab1, nab2, 0))
        level = []
    else:
        level = [(gl, gu, nab1, nab2, 0)]
    depth = 0
    while level:
        split = depth + 1 >= depth_cap
        nxt = []
        for a, b, na, nb, it in level:
            c = 0.5 * (a + b)
            cnt = min(nb, max(na, sturm(d, e2, pivmin, c)))
            for side in (0, 1):
                ca, cb = (c, b) if side else (a, c)
                cna, cnb = (cnt, nb) if side else (na, cnt)
                if cnb <= cna:
                    continue
                cit = it + 1
                if converged(ca, cb, abstol, pivmin, reltol) or cit >= itmax:
                    for j in range(cna + 1, cnb + 1):
                        out[j] = (ca, cb)
                elif cnb - cna == 1 or split:
                    for j in range(cna + 1, cnb + 1):
                        singles.append((ca, cb, cna, cnb, cit, j))
                else:
                    nxt.append((ca, cb, cna, cnb, cit))
        level = nxt
        depth += 1
        if split:
            break
    for s in singles:
        if len(s) == 5:   # a root with one eigenvalue
            a, b, na, nb, it = s
            j = nb
        else:
            a, b, na, nb, it, j = s
        out[j] = bisect_one(d, e2, pivmin, abstol, reltol, itmax, j, a, b, na, nb, it)
    return out


def _cases():
    rng = np.random.default_rng(12)
    for n in (1, 2, 7, 40):
        D = rng.uniform(-1, 1, n)
        E = rng.uniform(-1, 1, n)
        yield f"random{n}", D, E
    yield "one-two-one", np.full(30, 2.0), np.ones(30)
    # a glued Wilkinson matrix: pairs of nearly equal eigenvalues keep
    # multi-eigenvalue nodes alive to the depth limit
    w = np.abs(np.arange(21) - 10.0)
    D = np.concatenate([w, w])
    E = np.concatenate([np.ones(20), [1e-12], np.ones(20), [0.0]])
    yield "glued-wilkinson", D, E


@pytest.mark.parametrize("depth_cap", [1, 3, 16])
@pytest.mark.parametrize("name,D,E", list(_cases()), ids=lambda v: v if isinstance(v, str) else "")
def test_shared_equals_per_eigenvalue(name, D, E, depth_cap):
    n = len(D)
    d = [float(x) for x in D]
    e2 = [0.0] + [float(x) * float(x) for x in E[: n - 1]]
    tnorm = max(abs(x) for x in d) + (2 * max(abs(x) for x in E[: n - 1]) if n > 1 else 0.0)
    gl, gu = -tnorm - 1e-3, tnorm + 1e-3
    pivmin = np.finfo(float).tiny * max(1.0, max(e2))
    abstol, reltol = 2 * pivmin, 1.5e-8
    itmax = int((np.log(gu - gl + pivmin) - np.log(pivmin)) / np.log(2.0)) + 2
    nab1, nab2 = sturm(d, e2, pivmin, gl), sturm(d, e2, pivmin, gu)
    shared = bisect_shared(d, e2, pivmin, abstol, reltol, itmax, gl, gu, nab1, nab2, depth_cap)
    assert sorted(shared) == list(range(nab1 + 1, nab2 + 1))
    for j in range(nab1 + 1, nab2 + 1):
        one = bisect_one(d, e2, pivmin, abstol, reltol, itmax, j, gl, gu, nab1, nab2)
        assert shared[j] == one, (name, j, shared[j], one)
