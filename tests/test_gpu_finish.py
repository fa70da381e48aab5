"""The finish of a level's short singleton list.  With MR3_FINISH_MAX large
every singleton left after the first round is finished by k_sng_finish, a
warp each, in both forms -- lane 0's checkpointed dlar1v, and the split form
(MR3_FINISH_SPLIT=1: the two sweeps on two lanes at once, the twist index
chosen by the warp).  With MR3_FINISH_MAX=0 and MR3_ITER_MAX large the
round kernel's iterating form (a lane per singleton, every remaining call
in one launch, bisections by the whole warp) does it.  With both 0 the
rounds alone do the work.  The results equal the oracle's bit for bit in
every form."""
import pytest

import mr3smp_b200 as M
import oracle
from conftest import assert_same
from mr3smp_b200 import workloads as wl
from zoo import medium_zoo, small_zoo

pytestmark = pytest.mark.gpu


def _cases():
    keep = ("uniform100_V_A", "uniform257_V_I", "uniform257_tryrac", "121_150", "w21_V_A",
            "glued6x41_V_A", "glued6x41_V_I", "split300_V_A", "huge_scale", "tight_cluster",
            "graded_tryrac")
    out = [c for c in small_zoo() if c[0] in keep]
    out += [c for c in medium_zoo() if c[0] in ("config1_uniform1000", "glued10x201_I",
                                                 "large_mixed3000")]
    return out


def _form(form, monkeypatch):
    if form in ("rounds", "iter"):
        monkeypatch.setenv("MR3_FINISH_MAX", "0")
        monkeypatch.setenv("MR3_ITER_MAX", "0" if form == "rounds" else "100000000")
    else:
        monkeypatch.setenv("MR3_FINISH_MAX", "100000000")
        monkeypatch.setenv("MR3_FINISH_SPLIT", "1" if form == "split" else "0")


@pytest.mark.parametrize("form", ["split", "lane0", "iter", "rounds"])
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_finish_forms_equal_oracle(case, form, monkeypatch):
    name, D, E, jz, rg, kw = case
    _form(form, monkeypatch)
    g = M.mrrr(jz, rg, D, E, **kw)
    o = oracle.mrrr(jz, rg, D, E, **kw)
    assert_same(g, o, f"{name} ({form})")


@pytest.mark.parametrize("form", ["split", "lane0", "iter"])
def test_finish_forms_batched(form, monkeypatch):
    _form(form, monkeypatch)
    probs = [dict(jobz="V", range="A", D=D, E=E)
             for D, E, _ in wl.mixed_batch(20, seed=41, nmin=8, nmax=900)]
    res = M.mrrr_batched(probs)
    for k, (p, r) in enumerate(zip(probs, res)):
        assert_same(r, oracle.mrrr("V", "A", p["D"], p["E"]), f"batch[{k}] ({form})")
