"""Batched solves: every problem's result is identical alone and in the
batch, and identical to the oracle's."""
import numpy as np
import pytest

import mr3smp_b200 as M
import oracle
from conftest import assert_same
from mr3smp_b200 import workloads as wl
from zoo import small_zoo

pytestmark = pytest.mark.gpu


def _problems():
    probs = []
    for D, E, kind in wl.mixed_batch(24, seed=21, nmin=8, nmax=600):
        probs.append(dict(jobz="V", range="A", D=D, E=E))
    for name, D, E, jz, rg, kw in small_zoo()[:20]:
        p = dict(jobz=jz, range=rg, D=D, E=E)
        p.update(kw)
        probs.append(p)
    return probs


def test_batched_equals_single_and_oracle():
    probs = _problems()
    res = M.mrrr_batched(probs)
    for k, (p, r) in enumerate(zip(probs, res)):
        kw = {x: p[x] for x in ("vl", "vu", "il", "iu", "tryrac") if x in p}
        single = M.mrrr(p["jobz"], p["range"], p["D"], p["E"], **kw)
        assert_same(r, single, f"batch[{k}] vs single")
        o = oracle.mrrr(p["jobz"], p["range"], p["D"], p["E"], **kw)
        assert_same(r, o, f"batch[{k}] vs oracle")


def test_batch_order_does_not_matter():
    probs = _problems()
    res = M.mrrr_batched(probs)
    rev = M.mrrr_batched(probs[::-1])[::-1]
    for k, (a, b) in enumerate(zip(res, rev)):
        assert_same(a, b, f"order {k}")


def test_pipelined_chunks_identical(monkeypatch):
    """A batch solved in many chunks (Z copies of one chunk overlapping the
    next chunk's solve) returns exactly what the one-pass batch returns."""
    probs = _problems()
    whole = M.mrrr_batched(probs)
    monkeypatch.setenv("MR3_PIPE_BYTES", str(64 * 1024))
    chunked = M.mrrr_batched(probs)
    for k, (a, b) in enumerate(zip(whole, chunked)):
        assert_same(a, b, f"chunked {k}")
