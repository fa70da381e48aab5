"""The dqds route on the GPU (MR3_NTHREADS at or below 12 m / n selects it,
as the reference's thread count does, SRC/mrrr_val.c:279-285, 409-412):
the device path equals the oracle's dqds route bit for bit (W, Z, Zsupp,
the overwritten D/E, counts and bounds), one problem at a time and in a
batch, and agrees with the reference's own mrrr() run with 8 threads within
the tolerances of the other parity tests."""
import numpy as np
import pytest

import mr3smp_b200 as M
import oracle
from conftest import EPS, assert_same, tnorm
from mr3smp_b200 import workloads as wl
from zoo import small_zoo

pytestmark = pytest.mark.gpu


def _cases():
    out = [c for c in small_zoo() if len(c[1]) >= 2 and c[3] != "C"]
    for n in (600, 1500):
        D, E = wl.uniform(n, seed=n)
        out.append((f"uniform{n}_V_A", D, E, "V", "A", {}))
    D, E = wl.one_two_one(800)
    out.append(("121_800_V_A", D, E, "V", "A", {}))
    D, E = wl.glued_wilkinson(4, 201, 1e-12)
    out.append(("glued4x201_V_A", D, E, "V", "A", {}))
    D, E = wl.uniform(1000, seed=3)
    out.append(("uniform1000_V_I", D, E, "V", "I", dict(il=1, iu=700)))
    out.append(("uniform1000_N_A", D, E, "N", "A", {}))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_gpu_dqds_route_equals_oracle(case, monkeypatch):
    name, D, E, jz, rg, kw = case
    monkeypatch.setenv("MR3_NTHREADS", "8")
    g = M.mrrr(jz, rg, D, E, **kw)
    o = oracle.mrrr(jz, rg, D, E, **kw)
    assert_same(g, o, name)
    n = len(D)
    if n >= 500 and oracle.ref_lib() is not None:
        r = oracle.ref_mrrr(jz, rg, D, E, threads=8, **kw)
        assert r["m"] == g["m"]
        assert np.abs(g["W"] - r["W"]).max() <= 10 * n * EPS * tnorm(D, E)


def test_gpu_dqds_route_batched(monkeypatch):
    monkeypatch.setenv("MR3_NTHREADS", "8")
    probs = [dict(jobz="V", range="A", D=D, E=E)
             for D, E, _ in wl.mixed_batch(16, seed=31, nmin=16, nmax=700)]
    res = M.mrrr_batched(probs)
    for k, (p, r) in enumerate(zip(probs, res)):
        assert_same(r, oracle.mrrr("V", "A", p["D"], p["E"]), f"batch[{k}]")
