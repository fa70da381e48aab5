"""Matrix zoo for parity tests: (name, D, E, jobz, range, kwargs)."""
import numpy as np

from mr3smp_b200 import workloads as wl


def small_zoo():
    cases = []
    for n in (2, 3, 4, 7, 10, 33, 100):
        D, E = wl.uniform(n, seed=100 + n)
        cases.append((f"uniform{n}_V_A", D, E, "V", "A", {}))
    D, E = wl.uniform(1, seed=1)
    cases.append(("n1_V_A", D, E, "V", "A", {}))
    cases.append(("n1_N_V_out", D, E, "N", "V", dict(vl=5.0, vu=6.0)))
    D, E = wl.uniform(257, seed=7)
    cases.append(("uniform257_N_A", D, E, "N", "A", {}))
    cases.append(("uniform257_V_I", D, E, "V", "I", dict(il=20, iu=200)))
    cases.append(("uniform257_V_V", D, E, "V", "V", dict(vl=-0.5, vu=0.25)))
    cases.append(("uniform257_C_V", D, E, "C", "V", dict(vl=-0.5, vu=0.25)))
    cases.append(("uniform257_N_I", D, E, "N", "I", dict(il=1, iu=1)))
    cases.append(("uniform257_V_Iall", D, E, "V", "I", dict(il=1, iu=257)))
    cases.append(("uniform257_V_Vall", D, E, "V", "V", dict(vl=-10.0, vu=10.0)))
    cases.append(("uniform257_V_Vempty", D, E, "V", "V", dict(vl=5.0, vu=6.0)))
    cases.append(("uniform257_tryrac", D, E, "V", "A", dict(tryrac=1)))
    D, E = wl.one_two_one(150)
    cases.append(("121_150", D, E, "V", "A", {}))
    D = wl.wilkinson_plus(21)
    E = np.ones(21)
    E[-1] = 0
    cases.append(("w21_V_A", D, E, "V", "A", {}))
    cases.append(("w21_V_I", D, E, "V", "I", dict(il=3, iu=18)))
    cases.append(("w21_V_V", D, E, "V", "V", dict(vl=-1.22, vu=5.93)))
    D, E = wl.glued_wilkinson(6, 41, 1e-12)
    cases.append(("glued6x41_V_A", D, E, "V", "A", {}))
    cases.append(("glued6x41_V_I", D, E, "V", "I", dict(il=1, iu=123)))
    D, E = wl.uniform(300, seed=9)
    E[[0, 57, 58, 200, 298]] = 0.0
    cases.append(("split300_V_A", D, E, "V", "A", {}))
    cases.append(("split300_V_I", D, E, "V", "I", dict(il=40, iu=260)))
    D, E = wl.uniform(200, seed=10)
    cases.append(("tiny_scale", D * 1e-160, E * 1e-160, "V", "A", {}))
    cases.append(("huge_scale", D * 1e160, E * 1e160, "V", "A", {}))
    cases.append(("huge_scale_V", D * 1e160, E * 1e160, "V", "V", dict(vl=-1e159, vu=2e159)))
    g = 10.0 ** -np.arange(40)
    cases.append(("graded_tryrac", 3 * g, np.r_[np.sqrt(g[:-1] * g[1:]), 0.0], "V", "A", dict(tryrac=1)))
    cases.append(("graded_tryrac_N", 3 * g, np.r_[np.sqrt(g[:-1] * g[1:]), 0.0], "N", "A", dict(tryrac=1)))
    Dz = np.zeros(50)
    Ez = np.zeros(50)
    Dz[::7] = 1.0
    cases.append(("diag_zero_offdiag", Dz, Ez, "V", "A", {}))
    D = np.ones(64)
    E = np.full(64, 1e-3)
    E[-1] = 0
    cases.append(("tight_cluster", D, E, "V", "A", {}))
    return cases


def medium_zoo():
    cases = []
    D, E = wl.uniform(1000, seed=1)
    cases.append(("config1_uniform1000", D, E, "V", "A", dict(tryrac=1)))
    D, E = wl.glued_wilkinson(10, 201, 1e-12)
    cases.append(("glued10x201_I", D, E, "V", "I", dict(il=1, iu=1005)))
    D, E = wl.one_two_one(2000)
    cases.append(("121_2000", D, E, "V", "A", {}))
    D, E = wl.large_mixed(3000, seed=5, bs=101)
    cases.append(("large_mixed3000", D, E, "V", "A", {}))
    # high relative accuracy at scale: a matrix graded over 280 decades whose
    # relative off-diagonals (1/3 each) pass dlarrr, so tryrac survives and
    # dlarrj refines every eigenvalue (SRC/mrrr.c:452-520)
    g = 10.0 ** (-np.arange(2000) * (280.0 / 2000))
    Dg, Eg = 3.0 * g, np.r_[np.sqrt(g[:-1] * g[1:]), 0.0]
    cases.append(("graded2000_tryrac_V_A", Dg, Eg, "V", "A", dict(tryrac=1)))
    cases.append(("graded2000_tryrac_N_I", Dg, Eg, "N", "I", dict(il=100, iu=1900, tryrac=1)))
    # range V and its count at scale
    D, E = wl.uniform(3000, seed=12)
    cases.append(("uniform3000_V_V", D, E, "V", "V", dict(vl=-0.7, vu=1.3)))
    cases.append(("uniform3000_C_V", D, E, "C", "V", dict(vl=-0.7, vu=1.3)))
    return cases
