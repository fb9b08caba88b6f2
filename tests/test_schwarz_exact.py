"""The host Schwarz bounds (igpu_schwarz_bounds, the values every plan
screens with) are the reference's Basis::schwarz_bounds bit for bit
(src/integrals.rs:842-862 under the Auto engine policy): compared with the
oracle's restatement on the bench systems, the reference's test fixtures and
a spherical f cut, as 64-bit patterns.  Runs on the CPU: the entry needs no
device."""
import ctypes

import numpy as np
import pytest

import oracle_py as O
from integral_b200 import _lib
from integral_b200 import systems as S


def host_bounds(shells):
    arr = (_lib.IgpuShell * max(1, len(shells)))()
    keep = []
    for k, s in enumerate(shells):
        ex = np.ascontiguousarray(s["exps"], dtype=np.float64)
        co = np.ascontiguousarray(s["coefs"], dtype=np.float64)
        keep += [ex, co]
        arr[k].l = s["l"]
        arr[k].spherical = 1 if s.get("spherical") else 0
        for c in range(3):
            arr[k].center[c] = s["center"][c]
        arr[k].nprim = len(ex)
        arr[k].exps = ex.ctypes.data_as(_lib.c_double_p)
        arr[k].coefs = co.ctypes.data_as(_lib.c_double_p)
    q = np.empty(len(shells) ** 2)
    n_rys = ctypes.c_size_t()
    rc = _lib.lib().igpu_schwarz_bounds(arr, len(shells), q.ctypes.data_as(_lib.c_double_p), ctypes.byref(n_rys))
    assert rc == 0, _lib.lib().igpu_last_error_string()
    return q.reshape(len(shells), len(shells)), n_rys.value


def rys_pairs(shells):
    """Ordered shell pairs whose diagonal quartet the reference's Auto policy
    evaluates with the Rys engine."""
    out = np.zeros((len(shells), len(shells)), dtype=bool)
    for i, a in enumerate(shells):
        for j, b in enumerate(shells):
            ne = a["l"] + b["l"]
            out[i, j] = O.select_engine(ne, ne, (len(a["exps"]) * len(b["exps"])) ** 2) == "rys"
    return out


def assert_bitwise(shells):
    q, n_rys = host_bounds(shells)
    rys = rys_pairs(shells)
    assert n_rys == int(rys.sum()) and np.array_equal(np.isnan(q), rys)
    ref = O.OracleBasis(shells).schwarz("auto")
    exact = ~rys
    assert exact.any()
    assert q[exact].view(np.uint64).tolist() == ref[exact].view(np.uint64).tolist(), \
        float(np.max(np.abs(q[exact] - ref[exact])))
    return int(rys.sum())


def g_molecule(natom, seed=5):
    """The molecule-batch recipe (spherical s,s,p,p,d,f,g, 3 primitives)."""
    rng = np.random.default_rng(seed)
    centers = S.place_atoms(rng, natom, 2.5 * natom ** (1.0 / 3.0), 1.6)
    return S.build_shells(rng, centers, "ssppdfg", 3, 0.1, 2.4, 0.2, 1.0, spherical=True)


CASES = {
    "dense-6atom": lambda: S.dense_eri_system()["shells"],
    "jk-fixture-cart": lambda: S.direct_contractor_fixture(False),
    "jk-fixture-sph": lambda: S.direct_contractor_fixture(True),
    "grad-fixture-cart": lambda: S.direct_grad_fixture(False),
    "grad-fixture-sph": lambda: S.direct_grad_fixture(True),
    "sph-f-6atom": lambda: S.jk_spherical_system(natom=6, side=9.0)["shells"],
    "g-3atom": lambda: g_molecule(3),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_host_schwarz_is_the_reference_bit_for_bit(case):
    assert_bitwise(CASES[case]())


@pytest.mark.parametrize("system", ["jk-64atom", "grad-100atom"])
def test_host_schwarz_bit_for_bit_at_full_size(system):
    shells = S.jk_system()["shells"] if system == "jk-64atom" else S.grad_system()["shells"]
    # contracted shells only: the Auto policy picks OS/HGP for every pair
    assert assert_bitwise(shells) == 0


def test_pairs_the_auto_policy_sends_to_rys_are_reported():
    # one primitive per shell at l_i + l_j = 4: Auto picks the Rys engine
    shells = [{"l": 2, "spherical": False, "center": [0.0, 0.0, 0.0], "exps": [0.7], "coefs": [1.0]},
              {"l": 0, "spherical": False, "center": [0.0, 0.0, 1.2], "exps": [0.4, 1.3], "coefs": [1.0, 0.5]}]
    assert O.select_engine(4, 4, 1) == "rys"
    assert assert_bitwise(shells) == 1
    # the reference's extended gradient fixture has such pairs (single
    # primitive shells up to d)
    assert assert_bitwise(S.grad_extended_fixture()) > 0
