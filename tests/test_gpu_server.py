"""The serving front end (mr3_server_*): requests of mixed sizes and ranges
submitted as a stream, from several host threads, are solved in batches,
and each result is identical to the one the same request gets alone."""
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
    S = M.Server(budget_bytes=64 << 20)   # 8 MB for the small class, 56 MB large
    try:
        D, E = wl.uniform(3000, seed=1)
        with pytest.raises(M.MR3Error):
            S.submit(dict(jobz="V", range="A", D=D, E=E))   # 72 MB of Z > 56 MB
        D, E = wl.uniform(50, seed=2)
        with pytest.raises(M.MR3Error):
            S.submit(dict(jobz="V", range="I", D=D, E=E, il=5, iu=4))
        t = S.submit(dict(jobz="V", range="A", D=D, E=E))
        r, _ = S.poll(t, wait=True)
        assert r["info"] == 0 and r["m"] == 50
    finally:
        S.close()
