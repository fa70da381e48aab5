"""The serving admission rule (server.c mr3__srv_admit) on the CPU: queued
requests are taken in arrival order, all of one kind, within the device
budget left (a request that does not fit is passed over and those behind
it can still be taken) and the batch's work cap (the first request always
fits the cap), and lanes for small requests take only n <= 2048."""
import ctypes as C

import mr3smp_b200 as M


class View(C.Structure):
    _fields_ = [("kind", C.c_int), ("n", C.c_int), ("bytes", C.c_size_t), ("work", C.c_double)]


def _admit(reqs, small_only=0, budget=1 << 40, used=0, work_cap=1e30, maxk=4096):
    L = M.lib()
    f = L.mr3__srv_admit
    f.restype = C.c_int
    f.argtypes = [C.POINTER(View), C.c_int, C.c_int, C.c_size_t, C.c_size_t, C.c_double, C.c_int,
                  C.POINTER(C.c_int)]
    arr = (View * max(len(reqs), 1))(*[View(*r) for r in reqs])
    out = (C.c_int * max(len(reqs), 1))()
    k = f(arr, len(reqs), small_only, budget, used, work_cap, maxk, out)
    return [out[i] for i in range(k)]


def test_fifo_one_kind():
    reqs = [(1, 64, 10, 1.0), (0, 64, 10, 1.0), (1, 256, 10, 1.0), (1, 64, 10, 1.0)]
    assert _admit(reqs) == [0, 2, 3]
    assert _admit(reqs[1:]) == [0]          # a host request first: host requests only


def test_budget_passes_over_what_does_not_fit():
    reqs = [(1, 64, 50, 1.0), (1, 4096, 500, 1.0), (1, 256, 40, 1.0), (1, 64, 20, 1.0)]
    assert _admit(reqs, budget=100) == [0, 2]
    assert _admit(reqs, budget=100, used=60) == [2]
    assert _admit(reqs, budget=100, used=95) == []


def test_work_cap_and_first_request():
    reqs = [(1, 16384, 10, 1e9), (1, 64, 10, 5.0), (1, 64, 10, 5.0)]
    assert _admit(reqs, work_cap=100.0) == [0]          # the first always goes
    assert _admit(reqs[1:], work_cap=7.0) == [0]
    assert _admit(reqs[1:], work_cap=10.0) == [0, 1]


def test_small_lanes_and_batch_limit():
    reqs = [(1, 16384, 1, 1.0), (1, 1024, 1, 1.0), (1, 2048, 1, 1.0), (1, 4096, 1, 1.0)]
    assert _admit(reqs, small_only=1) == [1, 2]
    assert _admit(reqs, maxk=2) == [0, 1]
