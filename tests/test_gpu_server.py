"""The serving front end (mr3_server_*): requests of mixed sizes and ranges
submitted as a stream, from several host threads, with host or
device-resident arrays, are solved with continuous batching on several
lanes, and each result is identical to the one the same request gets
alone."""
import threading

import numpy as np
import pytest

import mr3smp_b200 as M
import oracle
from conftest import assert_same
from mr3smp_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _requests(count=40, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.choice([8, 40, 150, 600, 2500]))
        D, E = wl.uniform(n, seed=1000 + k)
        if k % 2 == 0:
            out.append(dict(jobz="V", range="A", D=D, E=E))
        else:
            out.append(dict(jobz="V", range="I", D=D, E=E, il=1, iu=max(1, -(-n // 10))))
    return out


def _kw(p):
    return {x: p[x] for x in ("vl", "vu", "il", "iu", "tryrac") if x in p}


def test_server_stream_equals_single_calls_and_oracle():
    reqs = _requests()
    S = M.Server()
    try:
        tickets = [S.submit(p) for p in reqs]
        res = [S.poll(t, wait=True) for t in tickets]
        st = S.stats()
    finally:
        S.close()
    assert st["solved"] == len(reqs) and st["batches"] >= 1
    for k, (p, (r, lat)) in enumerate(zip(reqs, res)):
        assert lat is not None and lat > 0.0
        alone = M.mrrr(p["jobz"], p["range"], p["D"], p["E"], **_kw(p))
        assert_same(r, alone, f"request {k} vs alone")
        if len(p["D"]) <= 600:
            o = oracle.mrrr(p["jobz"], p["range"], p["D"], p["E"], **_kw(p))
            assert_same(r, o, f"request {k} vs oracle")


def test_server_alone_and_mixed_identical_from_threads():
    reqs = _requests(count=24, seed=9)
    S = M.Server()
    try:
        alone = []
        for p in reqs:   # one at a time: every batch holds one request
            alone.append(S.poll(S.submit(p), wait=True)[0])
        mixed = [None] * len(reqs)

        def client(idx):
            ts = [(i, S.submit(reqs[i])) for i in idx]
            for i, t in ts:
                mixed[i] = S.poll(t, wait=True)[0]

        th = [threading.Thread(target=client, args=(list(range(j, len(reqs), 3)),)) for j in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    finally:
        S.close()
    for k in range(len(reqs)):
        assert_same(mixed[k], alone[k], f"request {k} mixed vs alone")


def test_server_rejects_bad_and_oversized_requests():
    S = M.Server(budget_bytes=64 << 20)
    try:
        D, E = wl.uniform(3000, seed=1)
        with pytest.raises(M.MR3Error):
            S.submit(dict(jobz="V", range="A", D=D, E=E))   # 72 MB of Z > 64 MB
        D, E = wl.uniform(50, seed=2)
        with pytest.raises(M.MR3Error):
            S.submit(dict(jobz="V", range="I", D=D, E=E, il=5, iu=4))
        t = S.submit(dict(jobz="V", range="A", D=D, E=E))
        r, _ = S.poll(t, wait=True)
        assert r["info"] == 0 and r["m"] == 50
    finally:
        S.close()


def _c4_requests(count, seed):
    """The serving mix at sizes up to 4096: n in {64, 256, 1024, 4096},
    range A and I (il = 1, iu = ceil(n/10)) alternating, D, E ~ U(-1, 1)."""
    rng = np.random.default_rng(seed)
    ns = rng.choice([64, 256, 1024, 4096], size=count, p=[0.4, 0.3, 0.2, 0.1])
    out = []
    for k, n in enumerate(ns):
        n = int(n)
        D, E = wl.uniform(n, seed=seed * 1000 + k)
        if k % 2 == 0:
            out.append(dict(jobz="V", range="A", D=D, E=E))
        else:
            out.append(dict(jobz="V", range="I", D=D, E=E, il=1, iu=-(-n // 10)))
    return out


def _device_arrays(p):
    import torch
    n = len(p["D"])
    cols = n if p["range"] == "A" else p["iu"] - p["il"] + 1
    return dict(p, D=torch.tensor(p["D"], device="cuda"), E=torch.tensor(p["E"], device="cuda"),
                W=torch.zeros(n, dtype=torch.float64, device="cuda"),
                Z=torch.zeros(n * cols, dtype=torch.float64, device="cuda"),
                Zsupp=torch.zeros(2 * n, dtype=torch.int32, device="cuda"))


def test_server_device_requests_c4_sizes_alone_and_mixed():
    """Device-resident requests of the serving mix (n up to 4096), submitted
    all at once so that lanes admit them while others are in flight: every
    result (W, Z, Zsupp, the overwritten D, E) equals the request's result
    alone, bit for bit."""
    import torch
    reqs = _c4_requests(48, seed=17)
    dev = [_device_arrays(p) for p in reqs]
    S = M.Server()
    try:
        tickets = [S.submit_device(d) for d in dev]
        res = [S.poll(t, wait=True)[0] for t in tickets]
        st = S.stats()
    finally:
        S.close()
    torch.cuda.synchronize()
    assert st["solved"] == len(reqs) and st["lanes"] >= 2
    print("batches", st["batches"], "overlapping others", st["batches_overlapping_others"])
    for k, (p, d, r) in enumerate(zip(reqs, dev, res)):
        n = len(p["D"])
        alone = M.mrrr(p["jobz"], p["range"], p["D"], p["E"], **_kw(p))
        assert r["info"] == 0 and r["m"] == alone["m"], k
        m = r["m"]
        assert np.array_equal(d["W"].cpu().numpy()[:m], alone["W"]), k
        Z = d["Z"].cpu().numpy()[: n * m].reshape(m, n).T
        assert np.array_equal(Z, alone["Z"]), k
        assert np.array_equal(d["Zsupp"].cpu().numpy()[: 2 * m], alone["Zsupp"]), k
        assert np.array_equal(d["D"].cpu().numpy(), alone["D"]), k
        assert np.array_equal(d["E"].cpu().numpy(), alone["E"]), k


def test_server_budget_admits_in_turn():
    """A budget that holds one large request at a time: requests wait for
    admission until the bytes in flight allow them, and all finish with
    their results alone."""
    reqs = _c4_requests(12, seed=23)
    big = max(8 * len(p["D"]) * (len(p["D"]) if p["range"] == "A" else p["iu"])
              + 560 * len(p["D"]) for p in reqs)
    S = M.Server(budget_bytes=big + (1 << 20))
    try:
        tickets = [S.submit(p) for p in reqs]
        res = [S.poll(t, wait=True)[0] for t in tickets]
    finally:
        S.close()
    for k, (p, r) in enumerate(zip(reqs, res)):
        alone = M.mrrr(p["jobz"], p["range"], p["D"], p["E"], **_kw(p))
        assert_same(r, alone, f"request {k}")


def test_server_bad_request_does_not_poison_its_batch():
    """A request with a NaN in D, submitted among good ones, gets info 2; the
    others, batched with it, equal their results alone."""
    reqs = _c4_requests(10, seed=29)
    bad = dict(reqs[4], D=reqs[4]["D"].copy())
    bad["D"][3] = np.nan
    reqs[4] = bad
    S = M.Server()
    try:
        tickets = [S.submit(p) for p in reqs]
        res = [S.poll(t, wait=True)[0] for t in tickets]
    finally:
        S.close()
    for k, (p, r) in enumerate(zip(reqs, res)):
        if k == 4:
            assert r["info"] == 2 and r["m"] == 0
            continue
        alone = M.mrrr(p["jobz"], p["range"], p["D"], p["E"], **_kw(p))
        assert_same(r, alone, f"request {k}")
