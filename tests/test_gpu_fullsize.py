"""Parity at the sizes the benchmark runs.

* The 4096-problem mixed batch (n log-uniform in [32, 4096], 25 % 1-2-1,
  D, E ~ U(-1, 1), seed 3, jobz V, range A) solved in ONE device pass, the
  pass bench.py times: every problem's count, ordering and scaled residual
  (<= 10) checked on the device, its orthogonality <= 10 but for at most
  0.1 % of the problems, which stay <= 20 and equal the oracle bit for bit;
  every 1-2-1 problem against its closed form lambda_k = 2 - 2 cos(k
  pi/(n+1)) within 10 n eps ||T||; a 64-problem sample stratified by n equal
  to the oracle bit for bit (W, Z, Zsupp and the overwritten D, E).
* The 20010-row glued Wilkinson matrix (range I, il = 1, iu = 10005) and the
  40000-row half-random, half-glued matrix (range A): eigenvalue count and
  index range exact, eigenvalues within 10 n eps ||T|| of the reference's own
  mrrr() (oracle/_ref, eigenvalues only, all host cores).  A range-V call on
  the 20010-row matrix checks the count in (vl, vu] against the reference's
  jobz = "C" count.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import mr3smp_b200 as M
import oracle
from conftest import EPS, tnorm
from mr3smp_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _stratified(ns, count):
    order = np.argsort(np.asarray(ns), kind="stable")
    pick = np.linspace(0, len(order) - 1, count).round().astype(int)
    return sorted({int(order[i]) for i in pick})


def _resid_orth_dev(d, e, w, Z, n):
    """Scaled residual and orthogonality of one problem, all on the device."""
    import torch
    tn = max(float(d.abs().max()), float(e[: n - 1].abs().max()) if n > 1 else 0.0) or 1.0
    TZ = d[:, None] * Z
    if n > 1:
        TZ[:-1] += e[: n - 1, None] * Z[1:]
        TZ[1:] += e[: n - 1, None] * Z[:-1]
    res = float((TZ - Z * w[None, :]).abs().max()) / (n * EPS * tn)
    G = Z.T @ Z
    G.diagonal().sub_(1.0)
    orth = float(G.abs().max()) / (n * EPS)
    return res, orth


def test_mixed_batch_4096_one_pass():
    import torch
    batch = wl.mixed_batch(4096, seed=3)
    problems = [(D, E) for D, E, _ in batch]
    kinds = [k for _, _, k in batch]
    ns = [len(D) for D, E in problems]
    S = M.Solver(0)
    recs, T = M.device_batch(problems)
    S.solve(recs, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    offs, zoffs = T["offs"], T["zoffs"]
    bad = []
    worst = 0.0
    n121 = 0
    for k, n in enumerate(ns):
        q = recs[k]
        assert q.info == 0 and q.m == n, (k, q.info, q.m, n)
        d = T["D0"][offs[k]:offs[k] + n]
        e = T["E0"][offs[k]:offs[k] + n]
        w = T["W"][offs[k]:offs[k] + n]
        Z = T["Z"][zoffs[k]:zoffs[k] + n * n].view(n, n).T   # column-major n x n
        assert bool((w[1:] >= w[:-1]).all()), f"problem {k}: W not ascending"
        res, orth = _resid_orth_dev(d, e, w, Z, n)
        worst = max(worst, res, orth)
        if res > 10.0 or orth > 10.0:
            bad.append((k, n, res, orth))
        if kinds[k] == "121":
            n121 += 1
            exact = wl.one_two_one_eigs(n)
            err = np.abs(w.cpu().numpy() - exact).max()
            assert err <= 10 * n * EPS * 2.0, (k, n, err)
    print(f"4096 problems, {sum(ns)} eigenpairs: worst resid/orth {worst:.3g}, "
          f"{n121} 1-2-1 problems on their closed form; above 10: {bad}")
    # MRRR bounds the orthogonality by a modest multiple of n eps, not by 10
    # itself: a few problems of this batch land just above 10 (the reference
    # shows the same on its own runs).  Every residual must be within 10; at
    # most 0.1 % of the problems may have their orthogonality in (10, 20],
    # and those must be the oracle's results bit for bit (the reference's
    # algorithm, not a device error).
    assert all(res <= 10.0 for _, _, res, _ in bad), bad
    assert len(bad) <= 4 and all(orth <= 20.0 for _, _, _, orth in bad), bad

    # a stratified sample, and the problems above 10, bit for bit against the oracle
    sample = sorted(set(_stratified(ns, 64)) | {k for k, _, _, _ in bad})
    Wh, Dh, Eh = T["W"].cpu().numpy(), T["D"].cpu().numpy(), T["E"].cpu().numpy()
    Zsh = T["Zsupp"].cpu().numpy()

    def check(k):
        n = ns[k]
        D, E = problems[k]
        o = oracle.mrrr("V", "A", D, E)
        assert o["info"] == 0 and o["m"] == n
        Zk = T["Z"][zoffs[k]:zoffs[k] + n * n].cpu().numpy().reshape(n, n).T
        sl = slice(offs[k], offs[k] + n)
        same = (np.array_equal(Wh[sl], o["W"]) and np.array_equal(Dh[sl], o["D"])
                and np.array_equal(Eh[sl], o["E"]) and np.array_equal(Zk, o["Z"])
                and np.array_equal(Zsh[2 * offs[k]:2 * offs[k] + 2 * n], o["Zsupp"]))
        return k, n, same

    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        out = list(ex.map(check, sample))
    diff = [(k, n) for k, n, same in out if not same]
    assert not diff, f"{len(diff)} of {len(out)} sampled problems differ from the oracle: {diff[:8]}"


def _ref_eigs(jobz, rng, D, E, **kw):
    if oracle.ref_lib() is None:
        pytest.skip("the reference library (oracle/_ref) is not built")
    threads = os.cpu_count() or 1
    return oracle.ref_mrrr(jobz, rng, D, E, threads=threads, **kw)


def test_glued_wilkinson_20010_counts_and_eigenvalues_vs_reference():
    D, E = wl.glued_wilkinson(30, 667, 1e-12)
    n = len(D)
    tn = tnorm(D, E)
    g = M.mrrr("V", "I", D, E, il=1, iu=n // 2)
    ref = _ref_eigs("N", "I", D, E, il=1, iu=n // 2)
    assert g["info"] == 0 and ref["info"] == 0
    assert g["m"] == ref["m"] == n // 2
    assert (g["il"], g["iu"]) == (ref["il"], ref["iu"]) == (1, n // 2)
    err = np.abs(g["W"] - ref["W"]).max()
    print(f"C2: m={g['m']}, max |W - W_ref| = {err:.3g} ({err / (n * EPS * tn):.3g} n eps ||T||)")
    assert err <= 10 * n * EPS * tn
    # eigenvalues only on the GPU: the same count and index range
    gn = M.mrrr("N", "I", D, E, il=1, iu=n // 2)
    assert gn["m"] == n // 2 and np.abs(gn["W"] - ref["W"]).max() <= 10 * n * EPS * tn
    # range V inside the clustered spectrum, its ends in the widest gaps near
    # eigenvalues 4000 and 7000: the count in (vl, vu] is the reference's
    Wr = ref["W"]
    i0 = 3900 + int(np.argmax(np.diff(Wr[3900:4100])))
    i1 = 6900 + int(np.argmax(np.diff(Wr[6900:7100])))
    vl, vu = 0.5 * (Wr[i0] + Wr[i0 + 1]), 0.5 * (Wr[i1] + Wr[i1 + 1])
    gc = M.mrrr("C", "V", D, E, vl=vl, vu=vu)
    rc = _ref_eigs("C", "V", D, E, vl=vl, vu=vu)
    assert gc["info"] == 0 and gc["m"] == rc["m"] == i1 - i0, (gc["m"], rc["m"], i1 - i0)
    gv = M.mrrr("N", "V", D, E, vl=vl, vu=vu)
    assert gv["m"] == rc["m"]
    assert np.abs(gv["W"] - Wr[i0 + 1:i1 + 1]).max() <= 10 * n * EPS * tn


def test_large_mixed_40000_counts_and_eigenvalues_vs_reference():
    D, E = wl.large_mixed(40000)
    n = len(D)
    tn = tnorm(D, E)
    g = M.mrrr("N", "A", D, E)
    ref = _ref_eigs("N", "A", D, E)
    assert g["info"] == 0 and ref["info"] == 0
    assert g["m"] == ref["m"] == n
    err = np.abs(g["W"] - ref["W"]).max()
    print(f"C5: max |W - W_ref| = {err:.3g} ({err / (n * EPS * tn):.3g} n eps ||T||)")
    assert err <= 10 * n * EPS * tn
