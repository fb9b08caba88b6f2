"""GPU parity of the CUDA path against the oracle (run on a B200).

Every call goes through the C ABI of libintegral_b200.so (via the Python
mirror of the reference API).  Tolerances follow the reference's contract:
FP64 ERIs element-wise within 1e-12 relative / 1e-14 absolute of the oracle
on significant elements (|x| >= 1e-3 * peak, the convention of
tests/two_electron.rs:109-123) and within 1e-13 * peak absolutely
everywhere; J/K within 1e-12 of max |J|, |K|; the screened quartet list
identical (count and order-independent fingerprint); mixed precision within
1e-6 Eh of the FP64 energy.
"""
import os

import numpy as np
import pytest

import integral_b200 as ib
import oracle_py as O
from integral_b200 import systems as S

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def loaded_libs():
    return open("/proc/self/maps").read()


def check_eri(gpu, ref):
    peak = float(np.max(np.abs(ref)))
    d = np.abs(gpu - ref)
    sig = np.abs(ref) >= 1e-3 * peak
    assert float(np.max(d[sig] / np.abs(ref[sig]))) < 1e-12
    assert float(np.max(d[sig] - 1e-12 * np.abs(ref[sig]))) <= 1e-14
    assert float(np.max(d)) < 1e-13 * max(peak, 1.0)


def energy(D, J, K):
    return sum(0.5 * float(np.sum(D[d] * (J[d] - 0.5 * K[d]))) for d in range(len(D)))


def test_oracle_checks_with_the_reference_rys_tables():
    """The oracle that checks the GPU here carries the reference's literal
    Rys coefficients (extracted at its build), not its own regeneration."""
    assert O.lib().orc_rys_tables_are_reference_literals()


def test_product_library_is_the_one_loaded():
    s = S.dense_eri_system()
    ib.Basis(s["shells"]).plan()
    assert os.path.join(ROOT, "integral_b200", "libintegral_b200.so") in loaded_libs()


def test_dense_eri_matches_oracle():
    s = S.dense_eri_system()
    gpu = ib.Basis(s["shells"]).eri()
    ref = O.OracleBasis(s["shells"]).eri()
    check_eri(gpu, ref)
    n = 54
    T = gpu.reshape(n, n, n, n)
    # every slot written once from its canonical quartet: exact 8-fold symmetry
    # for slots related by a shell-level permutation
    assert np.array_equal(T, T.transpose(2, 3, 0, 1)) or float(np.max(np.abs(T - T.transpose(2, 3, 0, 1)))) < 1e-14


def test_eri_builder_matches_dense():
    s = S.dense_eri_system()
    B = ib.Basis(s["shells"])
    ref = O.OracleBasis(s["shells"]).eri()
    check_eri(ib.EriBuilder(B).build(), ref)
    # partition + fill of a subset writes exactly the subset's rows
    eb = ib.EriBuilder(B)
    out = np.zeros(eb.output_len())
    tasks = eb.partition(out)
    eb.fill_many(tasks[::7])
    n = B.nao()
    offs = B.offsets()
    nf = [sh.n_func() for sh in B.shells()]
    rows = np.zeros((n, n), dtype=bool)
    for t in tasks[::7]:
        i, j = t.bra
        rows[offs[i]:offs[i] + nf[i], offs[j]:offs[j] + nf[j]] = True
        rows[offs[j]:offs[j] + nf[j], offs[i]:offs[i] + nf[i]] = True
    O4 = out.reshape(n, n, n * n)
    R4 = ref.reshape(n, n, n * n)
    assert float(np.max(np.abs(O4[~rows]))) == 0.0
    assert float(np.max(np.abs(O4[rows] - R4[rows]))) < 1e-13 * float(np.max(np.abs(ref)))


def g_molecule(natom, seed=5):
    """The molecule-batch recipe (spherical s,s,p,p,d,f,g, 3 primitives)."""
    rng = np.random.default_rng(seed)
    centers = S.place_atoms(rng, natom, 2.5 * natom ** (1.0 / 3.0), 1.6)
    return S.build_shells(rng, centers, "ssppdfg", 3, 0.1, 2.4, 0.2, 1.0, spherical=True)


@pytest.mark.parametrize("system", ["jk-8atom", "jk-64atom", "grad-100atom", "sph-f-6atom", "g-3atom"])
def test_schwarz_bounds_are_the_reference_bit_for_bit(system):
    """The plan screens with the reference's own Schwarz bounds, bit for bit
    (every pair of these contracted bases is an OS/HGP diagonal under the
    Auto policy), so the screened quartet lists match by construction.  The
    f and g cases run the warp-per-pair evaluation of the larger classes."""
    shells = {"jk-8atom": lambda: S.jk_system(natom=8, side=8.0)["shells"],
              "jk-64atom": lambda: S.jk_system()["shells"],
              "grad-100atom": lambda: S.grad_system()["shells"],
              "sph-f-6atom": lambda: S.jk_spherical_system(natom=6, side=9.0)["shells"],
              "g-3atom": lambda: g_molecule(3)}[system]()
    q = ib.Basis(shells).schwarz_bounds().reshape(len(shells), -1)
    qo = O.OracleBasis(shells).schwarz()
    assert q.view(np.uint64).tolist() == qo.view(np.uint64).tolist()


def test_schwarz_bounds_of_rys_pairs_within_the_eri_contract():
    """Pairs the Auto policy evaluates with Rys (single primitives, the
    reference's extended gradient fixture) keep the device evaluation."""
    shells = S.grad_extended_fixture()
    q = ib.Basis(shells).schwarz_bounds().reshape(len(shells), -1)
    qo = O.OracleBasis(shells).schwarz()
    assert float(np.max(np.abs(q - qo) / np.maximum(qo, 1e-300))) < 1e-12


@pytest.mark.parametrize("spherical", [False, True], ids=["cart", "sph"])
def test_reference_direct_contractor_fixture(spherical):
    """tests/direct_contractor.rs: 4 shells s,p,d,f, two densities, threshold 0."""
    shells = S.direct_contractor_fixture(spherical)
    B = ib.Basis(shells)
    n = B.nao()
    D = S.direct_contractor_densities(n)
    J, K = B.direct_contractor().jk(D, 0.0)
    OB = O.OracleBasis(shells)
    Jo, Ko, cnt, hsh = OB.direct_jk(D, 0.0)
    assert float(np.max(np.abs(J - Jo))) < 1e-12 * float(np.max(np.abs(Jo)))
    assert float(np.max(np.abs(K - Ko))) < 1e-12 * float(np.max(np.abs(Ko)))
    E = OB.eri().reshape(n, n, n, n)
    for d in range(2):
        assert float(np.max(np.abs(J[d] - np.einsum("abcd,cd->ab", E, D[d])))) < 1e-9
        assert float(np.max(np.abs(K[d] - np.einsum("abcd,bd->ac", E, D[d])))) < 1e-9


def test_jk_small_system_matches_oracle_with_exact_quartet_list():
    s = S.jk_system(natom=8, side=8.0)
    B = ib.Basis(s["shells"])
    dc = B.direct_contractor()
    J, K = dc.jk(s["dens"], s["threshold"])
    st = dc.last_stats()
    Jo, Ko, cnt, hsh = O.OracleBasis(s["shells"]).direct_jk(s["dens"], s["threshold"], nthreads=8)
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    assert float(np.max(np.abs(J - Jo))) < 1e-12 * float(np.max(np.abs(Jo)))
    assert float(np.max(np.abs(K - Ko))) < 1e-12 * float(np.max(np.abs(Ko)))


def test_jk_nonsymmetric_density_matches_oracle():
    s = S.jk_system(natom=5, side=6.0, ndens=2)
    rng = np.random.default_rng(7)
    D = s["dens"] + 0.01 * rng.normal(size=s["dens"].shape)
    B = ib.Basis(s["shells"])
    J, K = B.direct_contractor().jk(D, 1e-12)
    Jo, Ko, _, _ = O.OracleBasis(s["shells"]).direct_jk(D, 1e-12)
    assert float(np.max(np.abs(J - Jo))) < 1e-12 * float(np.max(np.abs(Jo)))
    assert float(np.max(np.abs(K - Ko))) < 1e-12 * float(np.max(np.abs(Ko)))


def test_jk_bra_subset_matches_oracle():
    s = S.jk_system(natom=8, side=8.0)
    B = ib.Basis(s["shells"])
    dc = B.direct_contractor()
    nbra = len(dc.bra_pairs())
    bras = np.random.default_rng(3).choice(nbra, 60, replace=False)
    J, K = dc.jk(s["dens"], 1e-12, bras=bras)
    st = dc.last_stats()
    Jo, Ko, cnt, hsh = O.OracleBasis(s["shells"]).direct_jk(s["dens"], 1e-12, bras=bras)
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    assert float(np.max(np.abs(J - Jo))) < 1e-12 * float(np.max(np.abs(Jo)))


def test_jk_full_size_quartet_list_and_sampled_parity():
    """64-atom, nao 960 system at threshold 1e-12: the complete screened
    quartet list equals the oracle's; J/K of a seeded sample of bra pairs
    match the oracle's on the same sample."""
    s = S.jk_system()
    B = ib.Basis(s["shells"])
    dc = B.direct_contractor()
    OB = O.OracleBasis(s["shells"])
    dc.jk(s["dens"], s["threshold"])
    st = dc.last_stats()
    _, _, cnt, hsh = OB.direct_jk(s["dens"], s["threshold"], nthreads=os.cpu_count() or 8, count_only=True)
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    nbra = len(dc.bra_pairs())
    bras = np.random.default_rng(11).choice(nbra, 16, replace=False)
    J, K = dc.jk(s["dens"], s["threshold"], bras=bras)
    Jo, Ko, c2, h2 = OB.direct_jk(s["dens"], s["threshold"], bras=bras, nthreads=os.cpu_count() or 8)
    st = dc.last_stats()
    assert st["quartets"] == c2 and st["quartet_hash"] == h2
    assert float(np.max(np.abs(J - Jo))) < 1e-12 * float(np.max(np.abs(Jo)))
    assert float(np.max(np.abs(K - Ko))) < 1e-12 * float(np.max(np.abs(Ko)))


def test_jk_spherical_f_shells_matches_oracle():
    """The 200-atom spherical recipe (s,s,s,p,p,d,d,f; 4 primitives
    0.08*2.2^k; tau 1e-11) on 4 atoms: every class up to (ff|ff) in real
    solid harmonics, exact quartet list and J/K within 1e-12."""
    s = S.jk_spherical_system(natom=4, side=6.0, ndens=2, nocc=40)
    dc = ib.Basis(s["shells"]).direct_contractor()
    J, K = dc.jk(s["dens"], s["threshold"])
    st = dc.last_stats()
    Jo, Ko, cnt, hsh = O.OracleBasis(s["shells"]).direct_jk(s["dens"], s["threshold"], nthreads=os.cpu_count() or 8)
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    assert float(np.max(np.abs(J - Jo))) < 1e-12 * float(np.max(np.abs(Jo)))
    assert float(np.max(np.abs(K - Ko))) < 1e-12 * float(np.max(np.abs(Ko)))


def test_mixed_precision_energy_error_full_size():
    s = S.jk_system()
    dc = ib.Basis(s["shells"]).direct_contractor()
    J64, K64 = dc.jk(s["dens"], s["threshold"], precision=0)
    J32, K32 = dc.jk(s["dens"], s["threshold"], precision=1)
    st = dc.last_stats()
    assert st["quartets_fp32"] > 0.5 * st["quartets"]
    assert abs(energy(s["dens"], J32, K32) - energy(s["dens"], J64, K64)) <= 1e-6


def test_error_codes_on_device():
    s = S.jk_system(natom=3, side=5.0, ndens=1)
    dc = ib.Basis(s["shells"]).direct_contractor()
    with pytest.raises(ib.IntegralError) as e:
        dc.jk(s["dens"], 1e-12, bras=[10 ** 6])
    assert e.value.code == -8
    with pytest.raises(ib.IntegralError) as e:
        dc.jk(np.zeros((65, dc.nao(), dc.nao())), 1e-12)
    assert e.value.code == -6
