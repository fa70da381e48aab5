"""CPU tests of the native library: it builds, loads without a GPU, exports
every entry point its headers declare, and rejects bad arguments exactly as
the reference does (SRC/mrrr.c:119-138) without touching a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import mr3smp_b200 as M
from mr3smp_b200 import build as B

INC = os.path.join(os.path.dirname(B.HERE), "include")


def declared_functions():
    names = set()
    for f in os.listdir(INC):
        if not f.endswith(".h"):
            continue
        txt = open(os.path.join(INC, f)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = re.sub(r"^\s*typedef[^;]*;", "", txt, flags=re.M | re.S)   # function-pointer types
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w ]*?[\s\*]+(\w+)\s*\(", txt, re.M):
            if m.group(1) not in ("if", "for", "while", "sizeof", "return"):
                names.add(m.group(1))
    return sorted(names)


def test_library_builds_and_exports_all_declared_symbols():
    path = B.build()
    L = C.CDLL(path)
    names = declared_functions()
    assert "mrrr" in names and "mr3_cuda_solve" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_bad_arguments_return_1_without_gpu():
    D = np.linspace(-1, 1, 10)
    E = np.full(10, 0.5)
    assert M.mrrr("X", "A", D, E)["info"] == 1
    assert M.mrrr("V", "Q", D, E)["info"] == 1
    assert M.mrrr("V", "V", D, E, vl=1.0, vu=0.5)["info"] == 1
    assert M.mrrr("V", "V", D, E, vl=1.0, vu=1.0)["info"] == 1
    assert M.mrrr("V", "I", D, E, il=0, iu=3)["info"] == 1
    assert M.mrrr("V", "I", D, E, il=4, iu=3)["info"] == 1
    assert M.mrrr("V", "I", D, E, il=1, iu=11)["info"] == 1
    assert M.mrrr("V", "A", D[:0], E[:0])["info"] == 1
    assert M.mrrr("V", "A", D, E, ldz=5)["info"] == 1


def test_count_only_all_and_index_without_gpu():
    D = np.linspace(-1, 1, 10)
    E = np.full(10, 0.5)
    r = M.mrrr("C", "A", D, E)
    assert r["info"] == 0 and r["m"] == 10
    r = M.mrrr("c", "i", D, E, il=3, iu=7)
    assert r["info"] == 0 and r["m"] == 5


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(M, "LIB_PATH", str(tmp_path / "nope.so"))
    monkeypatch.setattr(M, "_lib", None)
    with pytest.raises(M.MR3Error):
        M.lib()


def test_server_create_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(M.MR3Error):
        M.Server()


@pytest.mark.parametrize("where", ["D0", "Dlast", "E0", "Einf"])
def test_non_finite_input_refused_without_gpu(where):
    """A NaN or infinity among the entries the solve reads (D[0..n-1],
    E[0..n-2]) is refused with info 2 before any device work; E[n-1] is not
    read (the reference overwrites it), so a NaN there is accepted."""
    D = np.linspace(-1, 1, 10)
    E = np.full(10, 0.5)
    if where == "D0":
        D[0] = np.nan
    elif where == "Dlast":
        D[-1] = np.inf
    elif where == "E0":
        E[0] = np.nan
    else:
        E[8] = -np.inf
    assert M.mrrr("V", "A", D, E)["info"] == 2
    assert M.mrrr("N", "V", D, E, vl=-1.0, vu=1.0)["info"] == 2
    # counting with range A or I never reads the matrix (SRC/mrrr.c:130-138)
    assert M.mrrr("C", "A", D, E)["info"] == 0
