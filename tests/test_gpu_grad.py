"""GPU parity of the density-direct ERI gradient (DirectGradContractor).

Calls go through igpu_grad in libintegral_b200.so via the Python mirror of
the reference API.  Checks follow tests/direct_grad_contractor.rs: the
gradient against the oracle's restatement of src/direct_grad.rs (1e-12 of
max |g| in FP64), the screened quartet list (count and fingerprint) equal to
the oracle's, zero net force, central finite differences of the GPU energy
E = 1/2 tr(D J) - 1/4 tr(D K) at h = 1e-4 bohr (tolerance 1e-6), bra
subsets, and the FP32-mixed gradient against the FP64 one.
"""
import os

import numpy as np
import pytest

import integral_b200 as ib
import oracle_py as O
from integral_b200 import systems as S

pytestmark = pytest.mark.gpu

NTHR = os.cpu_count() or 8


def terms(coul, exch):
    c = [ib.GradDensityTerm(f, l, r) for f, l, r in coul]
    x = [ib.GradDensityTerm(f, l, r) for f, l, r in exch]
    return c, x


def gpu_grad(shells, coul, exch, threshold, precision=0, bras=None):
    B = ib.Basis(shells)
    gc = B.direct_grad_contractor()
    c, x = terms(coul, exch)
    dens = gc.density(c, x)
    out = np.zeros((gc.natom(), 3))
    gc.accumulate_bra_pairs(ib.DirectGradWorkspace(), bras, dens, threshold, out, precision)
    return out, gc.last_stats()


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("spherical", [False, True], ids=["cart", "sph"])
def test_reference_direct_grad_fixture(spherical):
    """tests/direct_grad_contractor.rs:32-113: 6 shells up to f on three
    centres, two Coulomb-type and two exchange-type terms, threshold 0."""
    shells = S.direct_grad_fixture(spherical)
    n = O.OracleBasis(shells).nao
    coul, exch = S.grad_fixture_terms(n)
    g, st = gpu_grad(shells, coul, exch, 0.0)
    go, cnt, hsh = O.OracleBasis(shells).direct_grad(coul, exch, 0.0)
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    assert rel(g, go) < 1e-12
    assert float(np.max(np.abs(g.sum(axis=0)))) < 1e-10 * float(np.max(np.abs(g)))


def test_grad_small_system_exact_list_and_values():
    s = S.grad_system(natom=8, side=9.6)
    coul, exch = s["coulomb"], s["exchange"]
    g, st = gpu_grad(s["shells"], coul, exch, s["threshold"])
    go, cnt, hsh = O.OracleBasis(s["shells"]).direct_grad(coul, exch, s["threshold"], nthreads=NTHR)
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    assert rel(g, go) < 1e-12
    assert float(np.max(np.abs(g.sum(axis=0)))) < 1e-10 * float(np.max(np.abs(g)))


def test_grad_bra_subset_matches_oracle():
    s = S.grad_system(natom=8, side=9.6)
    coul, exch = s["coulomb"], s["exchange"]
    nbra = len(ib.Basis(s["shells"]).direct_grad_contractor().bra_pairs())
    bras = np.random.default_rng(5).choice(nbra, 50, replace=False)
    g, st = gpu_grad(s["shells"], coul, exch, 1e-12, bras=bras)
    go, cnt, hsh = O.OracleBasis(s["shells"]).direct_grad(coul, exch, 1e-12, bras=bras)
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    assert rel(g, go) < 1e-12


def test_grad_matches_finite_difference_of_gpu_energy():
    """Central differences of E(R) = 1/2 tr(D J[D]) - 1/4 tr(D K[D]) from the
    GPU J/K path, D fixed in the AO basis, h = 1e-4 bohr."""
    s = S.grad_system(seed=9, natom=4, side=6.0)
    D = s["dens"]
    g, _ = gpu_grad(s["shells"], s["coulomb"], s["exchange"], 0.0)
    atoms = ib.Basis(s["shells"]).atoms()
    h = 1e-4
    rng = np.random.default_rng(12)
    picks = [(int(rng.integers(len(atoms))), int(rng.integers(3))) for _ in range(6)]

    def energy(shells):
        J, K = ib.Basis(shells).direct_contractor().jk(D[None], 0.0)
        return 0.5 * float(np.sum(D * J[0])) - 0.25 * float(np.sum(D * K[0]))

    for a, x in picks:
        c0 = np.array(atoms[a])

        def moved(delta):
            out = []
            for sh in s["shells"]:
                sh2 = dict(sh)
                if np.array_equal(np.array(sh["center"]), c0):
                    cc = list(sh["center"])
                    cc[x] += delta
                    sh2["center"] = cc
                out.append(sh2)
            return out

        fd = (energy(moved(h)) - energy(moved(-h))) / (2 * h)
        assert abs(fd - g[a, x]) < 1e-6, (a, x, fd, g[a, x])


def test_grad_mixed_precision_close_to_fp64():
    s = S.grad_system(natom=16, side=12.0)
    g64, _ = gpu_grad(s["shells"], s["coulomb"], s["exchange"], s["threshold"], precision=0)
    g32, st = gpu_grad(s["shells"], s["coulomb"], s["exchange"], s["threshold"], precision=1)
    assert st["quartets_fp32"] > 0
    assert float(np.max(np.abs(g32 - g64))) < 1e-6


def test_grad_full_size_quartet_list_and_sampled_parity():
    """100 atoms, nao 1400 (s,s,p,p,d Cartesian) at threshold 1e-12: the whole
    screened list equals the oracle's; values on a seeded bra sample."""
    s = S.grad_system()
    coul, exch = s["coulomb"], s["exchange"]
    OB = O.OracleBasis(s["shells"])
    g, st = gpu_grad(s["shells"], coul, exch, s["threshold"])
    _, cnt, hsh = OB.direct_grad(coul, exch, s["threshold"], nthreads=NTHR, count_only=True)
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    assert float(np.max(np.abs(g.sum(axis=0)))) < 1e-10 * float(np.max(np.abs(g)))
    nbra = len(ib.Basis(s["shells"]).direct_grad_contractor().bra_pairs())
    bras = np.random.default_rng(13).choice(nbra, 12, replace=False)
    gs, st2 = gpu_grad(s["shells"], coul, exch, s["threshold"], bras=bras)
    go, c2, h2 = OB.direct_grad(coul, exch, s["threshold"], bras=bras, nthreads=NTHR)
    assert st2["quartets"] == c2 and st2["quartet_hash"] == h2
    assert rel(gs, go) < 1e-12


def test_grad_error_codes():
    s = S.grad_system(natom=3, side=5.0)
    gc = ib.Basis(s["shells"]).direct_grad_contractor()
    c, x = terms(s["coulomb"], s["exchange"])
    dens = gc.density(c, x)
    out = np.zeros((gc.natom(), 3))
    with pytest.raises(ib.IntegralError) as e:
        gc.accumulate_bra_pairs(ib.DirectGradWorkspace(), [10 ** 7], dens, 1e-12, out)
    assert e.value.code == -8
    with pytest.raises(ib.IntegralError) as e:
        gc.accumulate_bra_pairs(ib.DirectGradWorkspace(), None, dens, 1e-12, out, precision=7)
    assert e.value.code == -1


def test_grad_finite_difference_full_size_12_coordinates():
    """The 100-atom, nao 1400 gradient system at tau 1e-12: the FP64 GPU
    gradient against central differences (h = 1e-4 bohr) of the GPU energy
    E = 1/2 tr(D J) - 1/4 tr(D K) on 12 seeded (atom, axis) coordinates.

    Only quartets with a shell on the moved atom A depend on R_A.  With A's
    shells placed last (the energy and gradient do not depend on the shell
    order; D is permuted with the AOs), a canonical quartet (ij|kl) contains
    a shell of A exactly when its largest index i does, so the bra pairs
    (i, j) with i on A give both E_A(R_A +- h), whose difference is that of
    the full energies, and the complete gradient row of A."""
    s = S.grad_system()
    shells, D = s["shells"], s["dens"]
    nf = [S.n_func(sh["l"], False) for sh in shells]
    offs = np.concatenate([[0], np.cumsum(nf)])
    centers = [tuple(sh["center"]) for sh in shells]
    atoms = list(dict.fromkeys(centers))
    rng = np.random.default_rng(2024)
    picks = [(int(rng.integers(len(atoms))), int(rng.integers(3))) for _ in range(12)]
    h = 1e-4
    for a, x in picks:
        on_a = [k for k, c in enumerate(centers) if c == atoms[a]]
        order = [k for k in range(len(shells)) if k not in on_a] + on_a
        ao = np.concatenate([np.arange(offs[k], offs[k + 1]) for k in order])
        Dp = np.ascontiguousarray(D[np.ix_(ao, ao)])
        first = len(shells) - len(on_a)
        bras = np.array([i * (i + 1) // 2 + j for i in range(first, len(shells)) for j in range(i + 1)])

        def placed(delta):
            out = []
            for k in order:
                sh = dict(shells[k])
                if k in on_a:
                    c = list(sh["center"])
                    c[x] += delta
                    sh["center"] = c
                out.append(sh)
            return out

        def energy(delta):
            J, K = ib.Basis(placed(delta)).direct_contractor().jk(Dp[None], s["threshold"], bras=bras)
            return 0.5 * float(np.sum(Dp * J[0])) - 0.25 * float(np.sum(Dp * K[0]))

        fd = (energy(h) - energy(-h)) / (2 * h)
        g, _ = gpu_grad(placed(0.0), [(0.5, Dp, Dp)], [(-0.25, Dp, Dp)], s["threshold"], bras=bras)
        moved_row = len(atoms) - 1  # A's centre appears last in the reordered basis
        assert abs(fd - g[moved_row, x]) < 1e-6, (a, x, fd, g[moved_row, x])
