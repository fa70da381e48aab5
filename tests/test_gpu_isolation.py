"""Per-problem isolation: a problem with a non-finite entry in a batch is
refused with info 2 and the others' results are bit for bit what they are
alone, through the host-array path (mr3_batched, screened on the host) and
the device-array path (mr3_batched_device, screened on the device)."""
import numpy as np
import pytest

import mr3smp_b200 as M
from conftest import assert_same
from mr3smp_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _batch():
    probs = [dict(jobz="V", range="A", D=D, E=E)
             for D, E, _ in wl.mixed_batch(12, seed=77, nmin=16, nmax=400)]
    bad_d = probs[3]["D"].copy()
    bad_d[5] = np.nan
    bad_e = probs[7]["E"].copy()
    bad_e[0] = np.inf
    probs[3] = dict(probs[3], D=bad_d)
    probs[7] = dict(probs[7], E=bad_e)
    return probs, {3, 7}


def test_nonfinite_problem_isolated_host_path():
    probs, bad = _batch()
    res = M.mrrr_batched(probs)
    for k, (p, r) in enumerate(zip(probs, res)):
        if k in bad:
            assert r["info"] == 2 and r["m"] == 0
            continue
        alone = M.mrrr(p["jobz"], p["range"], p["D"], p["E"])
        assert_same(r, alone, f"problem {k}")


def test_nonfinite_problem_isolated_device_path():
    import torch
    probs, bad = _batch()
    dev = []
    for p in probs:
        n = len(p["D"])
        dev.append(dict(jobz="V", range="A",
                        D=torch.tensor(p["D"], device="cuda"), E=torch.tensor(p["E"], device="cuda"),
                        W=torch.zeros(n, dtype=torch.float64, device="cuda"),
                        Z=torch.zeros(n * n, dtype=torch.float64, device="cuda"),
                        Zsupp=torch.zeros(2 * n, dtype=torch.int32, device="cuda")))
    rc, out = M.mrrr_batched_device(dev)
    torch.cuda.synchronize()
    assert rc == 2
    for k, (p, q) in enumerate(zip(probs, out)):
        if k in bad:
            assert q.info == 2 and q.m == 0
            continue
        n = len(p["D"])
        alone = M.mrrr("V", "A", p["D"], p["E"])
        assert q.info == 0 and q.m == n
        assert np.array_equal(dev[k]["W"].cpu().numpy(), alone["W"])
        Z = dev[k]["Z"].cpu().numpy().reshape(n, n).T
        assert np.array_equal(Z, alone["Z"])
