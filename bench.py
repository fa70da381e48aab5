#!/usr/bin/env python
"""Benchmark of the B200 MRRR solver on the 4096-problem mixed batch.

Workload (per GPU): 4096 independent symmetric tridiagonals, n log-uniform in
[32, 4096] from a seed, 25 % of them the 1-2-1 matrix, the rest D, E i.i.d.
uniform(-1, 1); jobz = V, range = A.  One step solves the whole batch.

  value  eigenpairs/s of the batched device pass, inputs already in HBM
  e2e    the same through the C ABI (mr3_batched) with pinned host buffers:
         host-to-device copies of D, E and device-to-host copies of W, Z,
         Zsupp, D, E inside the timed region
  percall  eigenpairs/s of one mrrr()-style device call per problem (a
         stratified sample of the batch), and the batched/per-call ratio
  roofline  the dominant kernel against the measured FP64 division
         throughput (every Sturm-count step is one IEEE division)
  cpu_baseline  the reference's own mrrr() (oracle/_ref) on the host cores,
         PMR_NUM_THREADS = all cores, on a stratified sample of the batch

``--impl reference`` times only the reference CPU implementation, with the
same metric.  Under torchrun each rank solves its own batch (weak scaling,
no collective on the data path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "eigenpairs/s, 4096-problem mixed batch (jobz=V, range=A)"


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def rank_batch(wl, count: int, seed: int, nmax: int, rank: int):
    """This rank's share of the job: an independent batch seeded seed + rank
    (problems are independent; ranks exchange nothing)."""
    return wl.mixed_batch(count, seed=seed + rank, nmax=nmax)


def job_throughput(dist, device, ms_total: float, steps: int, pairs_per_step: int):
    """Whole-job eigenpairs/s: the eigenpairs of all ranks over the slowest
    rank's time.  Returns (value, ms_per_step)."""
    import torch
    ms, pairs = float(ms_total), float(pairs_per_step)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        p = torch.tensor([pairs], dtype=torch.float64, device=device)
        dist.all_reduce(p, op=dist.ReduceOp.SUM)
        ms, pairs = float(t.item()), float(p.item())
    ms_per_step = ms / steps
    return pairs / (ms_per_step * 1e-3), ms_per_step


def _stratified(ns, count):
    """Indices of `count` problems spread evenly over the batch sorted by n."""
    order = np.argsort(np.asarray(ns), kind="stable")
    if count >= len(order):
        return [int(i) for i in order]
    pick = np.linspace(0, len(order) - 1, count).round().astype(int)
    return [int(order[i]) for i in pick]


def _clocks_start(device_index):
    path = tempfile.mktemp(suffix=".csv")
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        proc = subprocess.Popen(["nvidia-smi", "-i", str(device_index), f"--query-gpu={q}",
                                 "--format=csv,noheader,nounits", "-lms", "200"],
                                stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None, path
    return proc, path


def _clocks_stop(proc, path):
    if proc is None:
        return None
    proc.terminate()
    try:
        proc.wait(timeout=5)
    except Exception:
        proc.kill()
    sm, mx, reasons = [], 0.0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(path):
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            mx = max(mx, float(f[2]))
        except ValueError:
            continue
        for nm, v in zip(names, f[5:9]):
            if v.lower().startswith("active"):
                reasons.add(nm)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


# --------------------------------------------------------------------------
# CPU baseline: the reference's own mrrr() on a bounded sample
# --------------------------------------------------------------------------
def host_cores():
    """(physical cores, logical CPUs) of this host."""
    logical = os.cpu_count() or 1
    try:
        import psutil
        phys = psutil.cpu_count(logical=False) or logical
    except Exception:
        phys = logical
    return int(phys), int(logical)


def check_host_result(D, E, r, rng):
    """Scaled residual and orthogonality of one host result (numpy): the
    residual over every column; the orthogonality of every column pair for
    n <= 1024, else of 64 random columns against all columns."""
    n = len(D)
    eps = np.finfo(np.float64).eps
    W, Z = r["W"], r["Z"]
    m = Z.shape[1]
    if m == 0:
        return 0.0, 0.0
    e = np.asarray(E[: n - 1], dtype=np.float64)
    tn = max(np.abs(D).max(), np.abs(e).max() if n > 1 else 0.0) or 1.0
    TZ = D[:, None] * Z
    TZ[:-1] += e[:, None] * Z[1:]
    TZ[1:] += e[:, None] * Z[:-1]
    res = np.abs(TZ - Z * W[None, :]).max() / (n * eps * tn)
    cols = np.arange(m) if n <= 1024 else np.sort(rng.choice(m, size=min(64, m), replace=False))
    G = Z.T @ Z[:, cols]
    G[cols, np.arange(len(cols))] -= 1.0
    return float(res), float(np.abs(G).max() / (n * eps))


def cpu_reference(problems, budget_s: float):
    """Time the reference mrrr() (oracle/_ref) problem by problem on a
    stratified sample whose predicted cost is about budget_s seconds, with
    PMR_NUM_THREADS = every host thread.  Every result is checked outside
    the timed calls (the reference's asserts are compiled out): a problem
    with info != 0, a wrong count, or residual or orthogonality above 10
    (units n eps ||T||, n eps) is a failure and its eigenpairs do not count.
    Returns (eigenpairs/s, dict)."""
    import oracle
    if oracle.ref_lib() is None:
        return None, {"unavailable": "reference library oracle/_ref not built"}
    phys, cores = host_cores()   # all the host threads the reference can use
    os.environ["PMR_NUM_THREADS"] = str(cores)
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    ns = [len(D) for D, E in problems]
    # calibrate on one mid-size problem
    mid = _stratified(ns, 9)[6]
    t0 = time.perf_counter()
    oracle.ref_mrrr("V", "A", problems[mid][0], problems[mid][1], threads=cores)
    dt = max(time.perf_counter() - t0, 1e-4)
    rate = ns[mid] ** 2 / dt                      # n^2 units per second
    want = budget_s * rate
    total = float(sum(n * n for n in ns))
    count = int(max(8, min(len(ns), round(len(ns) * want / total))))
    sample = _stratified(ns, count)
    rng = np.random.default_rng(0)
    el, pairs, bad, worst = 0.0, 0, 0, 0.0
    for i in sample:
        D, E = problems[i]
        t0 = time.perf_counter()
        r = oracle.ref_mrrr("V", "A", D, E, threads=cores)
        el += time.perf_counter() - t0
        ok = r["info"] == 0 and r["m"] == len(D)
        if ok:
            res, orth = check_host_result(D, E, r, rng)
            worst = max(worst, res, orth)
            ok = res <= 10.0 and orth <= 10.0
        if ok:
            pairs += r["m"]
        else:
            bad += 1
    info = {"value": pairs / el, "unit": "eigenpairs/s", "cores": cores, "physical_cores": phys,
            "kind": "reference",
            "sample": f"{len(sample)} of {len(ns)} problems stratified by n "
                      f"({pairs} checked eigenpairs, {el:.1f} s in mrrr()), "
                      f"PMR_NUM_THREADS={cores} (every host thread; {phys} physical cores), "
                      "OPENBLAS_NUM_THREADS=1",
            "mrrr_seconds": el, "checked": True, "checked_problems": len(sample), "checked_bad": bad,
            "checked_worst_resid_orth": worst,
            "check": "every sampled result: info, count, residual; orthogonality of all "
                     "columns (n <= 1024) or 64 random columns (larger n); failures excluded"}
    return pairs / el, info


def check_batch(recs, T, ns):
    """Checks every problem of a device batch in place on the device: info,
    count, ascending W, scaled residual max|T z - lambda z|/(n eps ||T||) and
    orthogonality max|Z^T Z - I|/(n eps), both <= 10.  Returns a summary with
    the eigenpairs of the problems that passed (pairs_ok)."""
    import torch
    eps = float(np.finfo(np.float64).eps)
    offs, zoffs = T["offs"], T["zoffs"]
    bad, worst, pairs_ok = 0, 0.0, 0
    for k, n in enumerate(ns):
        q = recs[k]
        ok = q.info == 0 and q.m == n
        if ok:
            d = T["D0"][offs[k]:offs[k] + n]
            e = T["E0"][offs[k]:offs[k] + n - 1]
            w = T["W"][offs[k]:offs[k] + n]
            Z = T["Z"][zoffs[k]:zoffs[k] + n * n].view(n, n).T
            tn = max(float(d.abs().max()), float(e.abs().max()) if n > 1 else 0.0) or 1.0
            TZ = d[:, None] * Z
            if n > 1:
                TZ[:-1] += e[:, None] * Z[1:]
                TZ[1:] += e[:, None] * Z[:-1]
            res = float((TZ - Z * w[None, :]).abs().max()) / (n * eps * tn)
            G = Z.T @ Z
            G.diagonal().sub_(1.0)
            orth = float(G.abs().max()) / (n * eps)
            asc = bool((w[1:] >= w[:-1]).all()) if n > 1 else True
            worst = max(worst, res, orth)
            ok = asc and res <= 10.0 and orth <= 10.0
        if ok:
            pairs_ok += n
        else:
            bad += 1
    return {"checked": True, "checked_problems": len(ns), "checked_bad": bad,
            "checked_worst_resid_orth": worst, "pairs_ok": pairs_ok,
            "how": "every problem on the device: info, m = n, ascending W, residual and "
                   "orthogonality <= 10 (units n eps ||T||, n eps); failures count no eigenpairs"}


SERVE_SIZES = (64, 256, 1024, 4096, 16384)
SERVE_PROBS = (0.4, 0.3, 0.2, 0.08, 0.02)


class _ZPool:
    """Device buffers for the eigenvectors of in-flight serving requests,
    recycled by size, with the bytes held (in flight or idle) kept within
    the device budget: a request whose Z does not fit waits until finished
    requests give theirs back (admission by device memory)."""

    def __init__(self, budget):
        import threading
        self.budget, self.held, self.out = budget, 0, 0
        self.free = {}
        self.cv = threading.Condition()

    def _drop_idle(self, need):
        for k, v in self.free.items():
            while v and (need is None or self.held + need > self.budget):
                v.pop()
                self.held -= 8 * k

    def get(self, size):
        import torch
        while True:
            with self.cv:
                while True:
                    lst = self.free.get(size)
                    if lst:
                        self.out += 1
                        return lst.pop()
                    if self.held + 8 * size <= self.budget:
                        self.held += 8 * size
                        break
                    self._drop_idle(8 * size)   # idle buffers of other sizes first
                    if self.held + 8 * size <= self.budget:
                        self.held += 8 * size
                        break
                    self.cv.wait()
            try:
                buf = torch.empty(max(size, 1), dtype=torch.float64, device="cuda")
                with self.cv:
                    self.out += 1
                return buf
            except torch.OutOfMemoryError:
                # the device holds less than the budget: give the bytes back,
                # drop idle buffers, and wait for a request in flight to finish
                with self.cv:
                    self.held -= 8 * size
                    self._drop_idle(None)
                    torch.cuda.empty_cache()
                    if self.out == 0:
                        raise
                    self.cv.wait(timeout=1.0)

    def put(self, size, buf):
        with self.cv:
            self.out -= 1
            self.free.setdefault(size, []).append(buf)
            self.cv.notify_all()


def run_serving(M, wl, rates, count: int, seed: int, budget: int):
    """The serving configuration: Poisson streams of independent requests
    through the serving API with continuous batching, one stream per rate.

    Sizes n in SERVE_SIZES with SERVE_PROBS, D, E ~ U(-1,1), range
    alternating A and I (il = 1, iu = ceil(n/10)), jobz V.  Requests are
    device requests: D, E staged in device memory beforehand (as they would
    arrive from an earlier device step), W, Z, Zsupp written in device
    memory and kept there -- the eigenvectors held by requests in flight stay
    within the device budget, a request waiting for admission until they
    fit.  Latency = scheduled arrival to result ready (client queueing and
    admission waits included).  Returns one record per rate."""
    import threading
    import torch
    rng = np.random.default_rng(seed)
    ns = rng.choice(SERVE_SIZES, size=count, p=SERVE_PROBS).astype(int)
    rng_i = np.arange(count) % 2 == 1
    cols = np.where(rng_i, -(-ns // 10), ns)
    offs = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    D0 = np.empty(int(offs[-1]))
    E0 = np.empty(int(offs[-1]))
    for k, n in enumerate(ns):
        d, e = wl.uniform(int(n), seed=seed * 100003 + k)
        D0[offs[k]:offs[k + 1]] = d
        E0[offs[k]:offs[k + 1]] = e
    D0t = torch.from_numpy(D0).cuda()
    E0t = torch.from_numpy(E0).cuda()
    Dt, Et = torch.empty_like(D0t), torch.empty_like(E0t)
    Wt = torch.empty_like(D0t)
    St = torch.empty(2 * int(offs[-1]), dtype=torch.int32, device="cuda")
    pool = _ZPool(budget)
    pairs = (cols).astype(np.int64)
    out = []
    S = M.Server(budget_bytes=budget)
    try:
        # warm-up: every lane's workspaces at the largest sizes
        for n in SERVE_SIZES:
            D, E = wl.uniform(int(n), seed=1)
            for rg in ("A", "I"):
                c = n if rg == "A" else -(-n // 10)
                z = pool.get(n * c)
                d = dict(jobz="V", range=rg, il=1, iu=c,
                         D=torch.tensor(D, device="cuda"), E=torch.tensor(E, device="cuda"),
                         W=torch.empty(n, dtype=torch.float64, device="cuda"), Z=z,
                         Zsupp=torch.empty(2 * n, dtype=torch.int32, device="cuda"))
                ts = [S.submit_device(d) for _ in range(4)]
                for t in ts:
                    S.poll(t, wait=True)
                pool.put(n * c, z)
        def stream(arrivals, count):
            """Requests 0..count-1 of the mix, submitted at the given arrival
            times (seconds from the start); one record."""
            Dt.copy_(D0t)
            Et.copy_(E0t)
            torch.cuda.synchronize()
            reqs = []
            for k in range(count):
                n, o = int(ns[k]), int(offs[k])
                q = M.CudaProb()
                q.n, q.jobz, q.range = n, 1, (3 if rng_i[k] else 1)
                q.il, q.iu, q.tryrac, q.ldz = 1, int(cols[k]), 0, n
                q.D = Dt.data_ptr() + 8 * o
                q.E = Et.data_ptr() + 8 * o
                q.W = Wt.data_ptr() + 8 * o
                q.Zsupp = St.data_ptr() + 8 * o
                reqs.append(q)
            b0 = S.stats()
            sub = [None] * count
            zbuf = [None] * count
            lat = np.zeros(count)
            qwait = np.zeros(count)
            done_t = np.zeros(count)
            bad = [0]
            okm = np.zeros(count, dtype=np.int64)
            ready = threading.Semaphore(0)

            stop = [False, count]   # a failed submission ends the stream at stop[1]

            def poller():
                for k in range(count):
                    ready.acquire()
                    if stop[0] and k >= stop[1]:
                        break
                    t, t_arr, t_sub = sub[k]
                    (info, m, _), l = S.poll(t, wait=True, raw=True)
                    done_t[k] = time.perf_counter()
                    lat[k] = (t_sub - t_arr) * 1e3 + l
                    tq = S.timing(t)
                    qwait[k] = (t_sub - t_arr) * 1e3 + (tq[0] if tq else 0.0)
                    if info != 0 or m != cols[k]:
                        bad[0] += 1
                    else:
                        okm[k] = 1
                    pool.put(int(ns[k] * cols[k]), zbuf[k])
                    zbuf[k] = None

            th = threading.Thread(target=poller, daemon=True)
            th.start()
            t0 = time.perf_counter()
            error = None
            try:
                for k in range(count):
                    ta = t0 + arrivals[k]
                    d = ta - time.perf_counter()
                    if d > 0:
                        time.sleep(d)
                    z = pool.get(int(ns[k] * cols[k]))   # waits while the budget is full
                    zbuf[k] = z
                    reqs[k].Z = z.data_ptr()
                    ts = time.perf_counter()
                    sub[k] = (S.submit_device(None, req=reqs[k]), ta, ts)
                    ready.release()
            except Exception as ex:   # record it; the requests already in flight finish
                error = f"{type(ex).__name__}: {ex}"[:300]
                stop[0], stop[1] = True, k
                ready.release()
            th.join()
            done_n = count if error is None else stop[1]
            if done_n == 0:
                return {"error": error}
            lat, qwait, done_t = lat[:done_n], qwait[:done_n], done_t[:done_n]
            el = float(done_t.max() - t0)
            b1 = S.stats()
            by_n = {}
            nsd = ns[:done_n]
            for n in SERVE_SIZES:
                sel = lat[nsd == n]
                if len(sel):
                    by_n[str(n)] = {"count": int(len(sel)),
                                    "p50_ms": round(float(np.percentile(sel, 50)), 3),
                                    "p99_ms": round(float(np.percentile(sel, 99)), 3)}
            nb = b1["batches"] - b0["batches"]
            rec = {"requests": done_n,
                   "p50_ms": round(float(np.percentile(lat, 50)), 3),
                   "p99_ms": round(float(np.percentile(lat, 99)), 3),
                   "queue_p50_ms": round(float(np.percentile(qwait, 50)), 3),
                   "eigenpairs_per_s": float((pairs[:done_n] * okm[:done_n]).sum() / el),
                   "requests_per_s": done_n / el, "failed": bad[0],
                   "batches": nb, "requests_per_batch": round(done_n / max(nb, 1), 2),
                   "batches_overlapping_others": b1["batches_overlapping_others"]
                   - b0["batches_overlapping_others"],
                   "by_n": by_n}
            if error:
                rec["error"] = error
            return rec

        # a burst of the mix before the timed streams: every lane meets its
        # largest batches (work arrays at their steady-state sizes) before
        # the budget for eigenvectors is fixed and the streams are timed
        nburst = min(count, 2000)
        stream(np.zeros(nburst), nburst)
        # the lanes' workspaces now hold their largest sizes: the eigenvector
        # budget is what the device has left beside them (at most the
        # configured budget), with 6 GB of headroom for growing work arrays
        with pool.cv:
            pool._drop_idle(None)
        torch.cuda.empty_cache()
        free_b = int(torch.cuda.mem_get_info()[0])
        pool.budget = max(1 << 30, min(budget, free_b - (6 << 30)))
        for rate in rates:
            arrivals = np.cumsum(np.random.default_rng(seed + int(rate)).exponential(1.0 / rate,
                                                                                   size=count))
            rec = stream(arrivals, count)
            out.append({"rate_per_s": rate, **rec})
        lanes = S.stats()["lanes"]
    finally:
        S.close()
    return {"streams": out, "lanes": lanes, "budget_gb_configured": budget / 2**30,
            "budget_gb": round(pool.budget / 2**30, 1),
            "mix": "n in {64,256,1024,4096,16384} w.p. {.4,.3,.2,.08,.02}; range A/I alternating "
                   "(I: il=1, iu=ceil(n/10)); D,E U(-1,1); jobz V",
            "api": "mr3_server_submit_device/poll (C ABI): D, E staged in HBM, W, Z, Zsupp "
                   "resident in HBM (Z within the budget)"}


def _workload(args):
    return (f"mixed batch: {args.count} tridiagonals, n log-uniform [32,{args.nmax}], "
            "25% 1-2-1, D,E uniform(-1,1), jobz=V range=A")


def run_reference(args):
    ws, rank, local = _dist()
    if rank != 0:
        return 0
    from mr3smp_b200 import workloads as wl
    probs = [(D, E) for D, E, _ in wl.mixed_batch(args.count, seed=args.seed, nmax=args.nmax)]
    budget = args.ref_step_seconds
    for _ in range(args.warmup):
        v, info = cpu_reference(probs, budget / 4)
        if v is None:
            print(json.dumps({"impl": "reference", "unavailable": info["unavailable"]}))
            return 0
    vals, secs, bad, checked, worst = [], [], 0, 0, 0.0
    info = None
    for _ in range(args.steps):
        v, info = cpu_reference(probs, budget)
        vals.append(v)
        secs.append(info["mrrr_seconds"])
        bad += info["checked_bad"]
        checked += info["checked_problems"]
        worst = max(worst, info["checked_worst_resid_orth"])
    value = float(np.mean(vals))
    info = {**info, "value": value, "checked_problems": checked, "checked_bad": bad,
            "checked_worst_resid_orth": worst}
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "eigenpairs/s",
           "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": 1e3 * float(np.mean(secs)),
           "higher_is_better": True, "dtype": "f64", "data": "synthetic",
           "config": {"workload": _workload(args), "problems_per_gpu": args.count,
                      "seed": args.seed,
                      "step": f"a stratified sample of about {budget:.0f} s of reference "
                              "mrrr() calls (results checked outside the calls)"},
           "cpu_baseline": info,
           "e2e": {"value": value, "unit": "eigenpairs/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
_DENSE_REF = r"""
import json, os, sys, time
import numpy as np
sys.path.insert(0, sys.argv[1])
import oracle
n, seed, threads = int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4])
rng = np.random.default_rng(seed)
B = rng.uniform(-1.0, 1.0, (n, n))
A = (B + B.T) * 0.5
t0 = time.perf_counter()
r = oracle.ref_dsyeig("V", "A", "L", A, threads=threads)
print(json.dumps({"seconds": time.perf_counter() - t0, "info": r["info"], "m": r["m"]}))
"""


def run_single(M, wl, which: str, hbm_gbs):
    """One large solve on the device (arrays resident in HBM, CUDA events on
    the solve's stream, after one warm-up solve): the 20010-row glued
    Wilkinson matrix (30 blocks of W+ of size 667, glue 1e-12; jobz V,
    range I, il = 1, iu = 10005) or the 40000-row matrix, half uniform
    (-1, 1), half glued W+ blocks of size 401 with glue 1e-10 (jobz V, range
    A; 12.8 GB of Z).  Reports seconds, eigenpairs/s, the residual and
    orthogonality of the result, and the Z write against the HBM copy
    bandwidth."""
    import torch
    if which == "c2":
        D, E = wl.glued_wilkinson(30, 667, 1e-12)
        n = len(D)
        rng, il, iu = 3, 1, n // 2
    else:
        D, E = wl.large_mixed(40000)
        n = len(D)
        rng, il, iu = 1, 1, n
    m = iu - il + 1
    dev = "cuda"
    D0 = torch.tensor(D, device=dev)
    E0 = torch.tensor(E, device=dev)
    Dd, Ed = D0.clone(), E0.clone()
    W = torch.zeros(n, dtype=torch.float64, device=dev)
    Z = torch.empty(n * m, dtype=torch.float64, device=dev)
    Zs = torch.zeros(2 * n, dtype=torch.int32, device=dev)
    rec = (M.CudaProb * 1)()
    q = rec[0]
    q.n, q.jobz, q.range, q.il, q.iu, q.tryrac, q.ldz = n, 1, rng, il, iu, 0, n
    q.D, q.E, q.W, q.Z, q.Zsupp = (Dd.data_ptr(), Ed.data_ptr(), W.data_ptr(), Z.data_ptr(),
                                   Zs.data_ptr())
    S = M.Solver(torch.cuda.current_device())
    st = torch.cuda.current_stream()
    times = []
    for _ in range(2):   # warm-up, then the timed solve
        Dd.copy_(D0)
        Ed.copy_(E0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        S.solve(rec, st.cuda_stream)
        e1.record(st)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
    sec = times[-1]
    # one more solve with per-kernel events, streams serialised (for the
    # detail file: where a single large solve spends its time)
    Dd.copy_(D0)
    Ed.copy_(E0)
    torch.cuda.synchronize()
    S.profile(2)
    S.solve(rec, st.cuda_stream)
    torch.cuda.synchronize()
    kern, ctr = S.profile_read()
    S.profile(False)
    prof = {"kernels_ms": {k: round(v[0], 2) for k, v in
                           sorted(kern.items(), key=lambda kv: -kv[1][0])},
            "launches": {k: v[1] for k, v in kern.items()},
            "work_counters": dict(zip(M.Solver.KERNEL_GROUPS, ctr))}
    from mr3smp_b200.workloads import residual_orth_torch
    ok = rec[0].info == 0 and rec[0].m == m
    res, orth = residual_orth_torch(D, E, W[:m].cpu().numpy(), Z.view(m, n).T)
    zb = 8.0 * n * m
    out = {"workload": ("glued W+ 30x667 (glue 1e-12), n=20010, jobz=V range=I 1..10005"
                        if which == "c2" else
                        "n=40000: half U(-1,1), half glued W+ 401 (glue 1e-10), jobz=V range=A"),
           "seconds": sec, "eigenpairs_per_s": m / sec, "ok": bool(ok),
           "resid": res, "orth": orth, "z_bytes": zb,
           "z_write_gbs": zb / sec * 1e-9,
           "z_write_frac_of_hbm": (zb / sec * 1e-9 / hbm_gbs) if hbm_gbs else None,
           "api": "mr3_cuda_solve, arrays resident in HBM, CUDA events",
           "_profile": prof}
    S.close()
    del Z, W
    torch.cuda.empty_cache()
    return out


def run_dense(M, n, seed, with_ref):
    """The dense driver dsyeig (SRC/dense.c:151-232) on a seeded n x n
    symmetric matrix, entries U(-1, 1): wall time through the C ABI from host
    memory (reduction, tridiagonal solve, back-transformation and the copies
    included), checked by residual and orthogonality; beside it the
    reference's dsyeig on the host cores (a separate process, so that its
    LAPACK runs with all cores)."""
    rng = np.random.default_rng(seed)
    B = rng.uniform(-1.0, 1.0, (n, n))
    A = (B + B.T) * 0.5
    M.dsyeig("V", "A", "L", A[:64, :64])   # loads the device LAPACK
    t0 = time.perf_counter()
    r = M.dsyeig("V", "A", "L", A)
    sec = time.perf_counter() - t0
    if r["info"] != 0:
        return {"n": n, "info": r["info"]}
    Z, W = r["Z"], r["W"]
    eps = np.finfo(np.float64).eps
    nrm = np.abs(W).max()
    out = {"n": n, "seconds": sec, "eigenpairs_per_s": n / sec, "api": "dsyeig (C ABI), host arrays",
           "resid": float(np.abs(A @ Z - Z * W).max() / (n * eps * nrm)),
           "orth": float(np.abs(Z.T @ Z - np.eye(n)).max() / (n * eps)),
           "steps": "dsytrd and dormtr: cuSOLVER; tridiagonal: this solver"}
    if with_ref and os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libmrrr_ref.so")):
        cores = os.cpu_count() or 1
        env = dict(os.environ, OPENBLAS_NUM_THREADS=str(cores))
        p = subprocess.run([sys.executable, "-c", _DENSE_REF, ROOT, str(n), str(seed), str(cores)],
                           env=env, capture_output=True, text=True, timeout=1800)
        try:
            ref = json.loads(p.stdout.strip().splitlines()[-1])
            out["reference"] = {"seconds": ref["seconds"], "eigenpairs_per_s": n / ref["seconds"],
                                "cores": cores, "kind": "reference",
                                "setup": "reference dsyeig, OpenBLAS and PMR_NUM_THREADS = cores"}
        except Exception:
            out["reference"] = {"error": (p.stderr or "")[-300:]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--count", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--nmax", type=int, default=4096,
                    help="largest n of the batch (smaller values make small profiling cases)")
    ap.add_argument("--percall-sample", type=int, default=128)
    ap.add_argument("--detail-out", default="",
                    help="file for the per-kernel times and work counters (default: a file "
                         "in the temporary directory)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--ref-step-seconds", type=float, default=4.0)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve-rates", default="1000,5000,20000",
                    help="request rates (per second) of the serving streams, comma-separated")
    ap.add_argument("--serve-count", type=int, default=10000,
                    help="requests per serving stream")
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the single 20010-row and 40000-row solves")
    ap.add_argument("--dense", type=int, default=0,
                    help="also time the dense driver dsyeig on an n x n symmetric matrix "
                         "(and the reference's on the host cores); 0 = off")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import mr3smp_b200 as M
    from mr3smp_b200 import workloads as wl

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}

    # workload: this rank's batch
    batch = rank_batch(wl, args.count, args.seed, args.nmax, rank)
    problems = [(D, E) for D, E, _ in batch]
    ns = [len(D) for D, E in problems]
    pairs_per_step = int(sum(ns))
    zbytes = 8 * sum(n * n for n in ns)

    S = M.Solver(local)
    recs, T = M.device_batch(problems)
    l2_flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB
    stream = torch.cuda.current_stream()

    def step():
        T["D"].copy_(T["D0"])
        T["E"].copy_(T["E0"])
        S.solve(recs, stream.cuda_stream)
        l2_flush.fill_(1.0)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # every problem of the batch is checked (outside the timed region) on the
    # result of the last warm-up step; a failure does not count as eigenpairs
    check = check_batch(recs, T, ns)
    pairs_per_step = check.pop("pairs_ok")

    # timed region (no per-kernel events inside it)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    cproc, cpath = _clocks_start(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    ev0.record(stream)
    for _ in range(args.steps):
        step()
        launches += S.last_launches() + 2   # solver kernels + the two input copies' kernels
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    clocks = _clocks_stop(cproc, cpath)
    value, ms_per_step = job_throughput(dist, "cuda", ms, args.steps, pairs_per_step)
    # one more step, outside the timed region, with every launch bracketed by
    # CUDA events and the streams serialised (the rounds do not share the GPU
    # with the next level's cluster kernels), so that each kernel's time is
    # its own: the per-kernel times and work counters of one step
    S.profile(2)
    step()
    torch.cuda.synchronize()
    kern, ctr = S.profile_read()
    S.profile(False)

    # roofline: the dominant kernel, algorithmic divisions per second
    div_gops = fma_tflops = None
    L = M.lib()
    L.mr3_cuda_fp64_peaks.restype = __import__("ctypes").c_int
    import ctypes
    a, b = ctypes.c_double(), ctypes.c_double()
    if L.mr3_cuda_fp64_peaks(local, ctypes.byref(a), ctypes.byref(b)) == 0:
        fma_tflops, div_gops = a.value, b.value
    groups = M.Solver.KERNEL_GROUPS
    # kernel family -> (counter group, divisions per counted unit)
    fam = {}
    for k, (kms, kc) in kern.items():
        f = k.split("<")[0]   # the instantiations of one template are one family
        if f == "k_sng_finish":   # its dlar1v rows are counted with the rounds'
            f = "k_sng_round"
        a_, b_ = fam.get(f, (0.0, 0))
        fam[f] = (a_ + kms, b_ + kc)
    kmap = {"k_bisect": (0, [1, 0, 0, 0]), "k_refine_root": (1, [0, 1, 0, 0]),
            "k_cl_ext": (2, [0, 1, 0, 0]), "k_cl_rrf": (2, [0, 0, 0, 1]),
            "k_refine_cl": (3, [0, 1, 0, 0]), "k_sng_round": (4, [0, 0, 2, 0]),
            "k_sng_bisect": (4, [0, 1, 0, 0])}
    # the dominant kernel family among those with an algorithmic count
    tname, (tms, tcnt) = max(((f, v) for f, v in fam.items() if f in kmap),
                             key=lambda kv: kv[1][0])
    roof = None
    if tname in kmap:
        g, w = kmap[tname]
        divs = sum(ctr[g][k] * w[k] for k in range(4))
        if tname == "k_cl_ext":
            divs = ctr[2][1]
        if tname == "k_cl_rrf":
            divs = ctr[2][3]
        avg_ms = tms / max(tcnt, 1)
        per_launch = divs / max(tcnt, 1)
        achieved = per_launch / (avg_ms * 1e-3) * 1e-9
        traffic = None
        if tname == "k_sng_round":
            # DRAM bytes per dlar1v row of the singleton kernels, measured with
            # ncu (dram__bytes_read.sum + dram__bytes_write.sum) on a
            # 256-problem mixed batch (n <= 4096), scaled by this run's rows
            traffic = {"bytes_per_launch": 48.4 * ctr[4][2] / max(tcnt, 1),
                       "algorithmic_bytes_per_launch": zbytes / max(tcnt, 1),   # the Z write
                       "source": "ncu on a 256-problem mixed batch (n <= 4096): 48.4 B per "
                                 "dlar1v row (checkpoints and child representations; the "
                                 "Z write is about 3 B per row), scaled by the live "
                                 "dlar1v-row counter"}
        roof = {"bound": "fp64-div", "kernel": tname, "achieved": achieved,
                "peak": div_gops, "unit": "Gdiv/s",
                "frac": (achieved / div_gops) if div_gops else None,
                "peak_source": "measured in-run (independent IEEE double divisions)",
                "traffic": traffic, "avg_launch_ms": avg_ms, "launches": tcnt,
                "algorithmic_divisions_per_launch": per_launch}
    hbm = peaks.get("hbm_gbs")
    roof_hbm = {"bound": "hbm", "what": "Z written per step / step time", "achieved":
                zbytes / (ms_per_step * 1e-3) * 1e-9, "peak": hbm, "unit": "GB/s",
                "frac": (zbytes / (ms_per_step * 1e-3) * 1e-9 / hbm) if hbm else None,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if hbm else None}

    # per-call comparator on a stratified sample (same device, one call each)
    percall = None
    if rank == 0 and args.percall_sample > 0:
        idx = _stratified(ns, args.percall_sample)
        sub = [problems[i] for i in idx]
        precs, PT = M.device_batch(sub)
        single = []
        for k in range(len(sub)):
            one = (M.CudaProb * 1)()
            one[0] = precs[k]
            single.append(one)
        for one in single[:4]:
            S.solve(one, stream.cuda_stream)
        PT["D"].copy_(PT["D0"])
        PT["E"].copy_(PT["E0"])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for one in single:
            S.solve(one, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        pms = e0.elapsed_time(e1)
        spairs = sum(len(D) for D, E in sub)
        # the same sample as one batched pass
        PT["D"].copy_(PT["D0"])
        PT["E"].copy_(PT["E0"])
        torch.cuda.synchronize()
        e0.record(stream)
        S.solve(precs, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        bms = e0.elapsed_time(e1)
        percall = {"value": spairs / (pms * 1e-3), "unit": "eigenpairs/s",
                   "sample": f"{len(sub)} problems stratified by n ({spairs} eigenpairs)",
                   "sample_batched_value": spairs / (bms * 1e-3),
                   "batched_over_percall": value / ws / (spairs / (pms * 1e-3))}
        del PT, precs, single

    # end to end through the C ABI with pinned host buffers
    # the batch's device arrays (56 GB of Z) and the timed solver's
    # workspaces are no longer needed
    del T, recs
    S.close()
    torch.cuda.empty_cache()

    large = None
    if rank == 0 and not args.no_large:
        hbm = peaks.get("hbm_gbs")
        large = {"c2": run_single(M, wl, "c2", hbm), "c5": run_single(M, wl, "c5", hbm)}

    serving = None
    if rank == 0 and not args.no_serve:
        rates = [float(x) for x in args.serve_rates.split(",") if x]
        serving = run_serving(M, wl, rates, args.serve_count, args.seed,
                              int(args.serve_budget_gb * 2**30))
        torch.cuda.empty_cache()

    e2e = None
    if rank == 0 and not args.no_e2e:
        hp = (M.HostProb * len(problems))()
        keep = []
        h2d = d2h = 0
        for k, (D, E) in enumerate(problems):
            n = len(D)
            Dh = torch.empty(n, dtype=torch.float64, pin_memory=True)
            Eh = torch.empty(n, dtype=torch.float64, pin_memory=True)
            Wh = torch.empty(n, dtype=torch.float64, pin_memory=True)
            Zh = torch.empty(n * n, dtype=torch.float64, pin_memory=True)
            Sh = torch.empty(2 * n, dtype=torch.int32, pin_memory=True)
            keep.append((Dh, Eh, Wh, Zh, Sh, D, E))
            h = hp[k]
            h.jobz, h.range, h.n, h.il, h.iu, h.tryrac, h.ldz = b"V", b"A", n, 1, 1, 0, n
            h.D = ctypes.cast(Dh.data_ptr(), ctypes.POINTER(ctypes.c_double))
            h.E = ctypes.cast(Eh.data_ptr(), ctypes.POINTER(ctypes.c_double))
            h.W = ctypes.cast(Wh.data_ptr(), ctypes.POINTER(ctypes.c_double))
            h.Z = ctypes.cast(Zh.data_ptr(), ctypes.POINTER(ctypes.c_double))
            h.Zsupp = ctypes.cast(Sh.data_ptr(), ctypes.POINTER(ctypes.c_int))
            h2d += 16 * n
            d2h += 8 * n + 8 * n * n + 8 * n + 16 * n
        def e2e_step():
            for Dh, Eh, Wh, Zh, Sh, D, E in keep:
                Dh.numpy()[:] = D
                Eh.numpy()[:] = E
            rc = L.mr3_batched(len(problems), hp)
            if rc != 0:
                raise SystemExit(f"mr3_batched failed rc={rc}: {M.last_error()}")
        e2e_step()   # warm-up (allocates the device workspace)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        el = (time.perf_counter() - t0) / args.e2e_steps
        # measured on rank 0 (its page-locked copy of the batch); with N ranks the
        # job figure is N times rank 0's, the ranks' batches being alike
        e2e = {"value": ws * pairs_per_step / el, "unit": "eigenpairs/s",
               "measured_on": "rank 0" if ws > 1 else "the only rank",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": el * 1e3, "api": "mr3_batched (C ABI), pinned host buffers",
               "steps": args.e2e_steps}
        del keep, hp

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        _, cpu = cpu_reference(problems, args.cpu_seconds)

    dense = None
    if rank == 0 and args.dense > 0:
        dense = run_dense(M, args.dense, args.seed, not args.no_cpu)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    # one profiled step (streams serialised) after the timed region
    detail = {"kernels_ms_per_step": {k: v[0] for k, v in
                                      sorted(kern.items(), key=lambda kv: -kv[1][0])},
              "kernel_launches_per_step": {k: v[1] for k, v in kern.items()},
              "work_counters": dict(zip(groups, ctr)),
              "how": "one step after the timed region, every launch bracketed by CUDA events, "
                     "the singleton rounds on the solve's stream (no overlap with the next "
                     "level's cluster kernels)"}
    if large:   # the large solves' per-kernel profiles go to the file only
        detail["large_profiles"] = {k: v.pop("_profile", None) for k, v in large.items()}
    detail_path = args.detail_out or os.path.join(tempfile.gettempdir(), "mr3_bench_detail.json")
    with open(detail_path, "w") as f:
        json.dump(detail, f, indent=1)
    top = sorted(detail["kernels_ms_per_step"].items(), key=lambda kv: -kv[1])[:6]
    out = {
        "metric": METRIC, "value": value, "unit": "eigenpairs/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded numpy)",
        "config": {"workload": _workload(args),
                   "problems_per_gpu": args.count, "seed": args.seed,
                   "eigenpairs_per_step_per_gpu": pairs_per_step,
                   "z_bytes_per_step_per_gpu": zbytes,
                   "l2": "flushed between steps by a 256 MB write; each step also writes "
                         f"{zbytes / 1e9:.1f} GB of Z"},
        "e2e": e2e, "gpu_launches": launches, "clocks": clocks, "roofline": roof,
        "check": check, "cpu_baseline": cpu, "dense": dense,
        "fp64_peaks": {"fma_tflops": fma_tflops, "div_gops": div_gops},
        "top_kernels_ms_per_step": {k: round(v, 2) for k, v in top},
        "detail_file": detail_path,
        "roofline_hbm": roof_hbm, "large": large, "percall": percall, "serving": serving,
    }
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
