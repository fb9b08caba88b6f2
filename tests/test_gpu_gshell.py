"""GPU parity of the g-shell classes (l = 4, the highest shell of the
molecule-batch workload) against the oracle: the dense tensor and single
(gg|gg) blocks, Cartesian and spherical, within the reference's contract
between its own engines, direct J/K with the exact screened quartet list,
and the gradient (raised tables to l = 5)."""
import numpy as np
import pytest

import integral_b200 as ib
import oracle_py as O
from integral_b200 import systems as S

pytestmark = pytest.mark.gpu


def check_eri(gpu, ref):
    """The reference's own contract between its two engines,
    |os - rys| <= 1e-11 + 1e-10 |x| element-wise (tests/cross_engine.rs:40-56):
    the GPU's quadrature against the Auto (OS/HGP) evaluation.  On g blocks of
    two-primitive shells the reference's own OS and Rys engines differ by up
    to 7e-9 relative on significant elements (3e-11 of the peak)."""
    d = np.abs(gpu - ref)
    assert np.all(d <= 1e-11 + 1e-10 * np.abs(ref)), float(np.max(d - 1e-10 * np.abs(ref)))


def two_centre_g(spherical):
    """s, d, g on one centre and p, g on another (2 primitives each)."""
    rng = np.random.default_rng(41)
    out = []
    for centre, letters in (([0.0, 0.0, 0.0], "sdg"), ([0.7, -0.4, 1.1], "pg")):
        for k, letter in enumerate(letters):
            exps = [0.9 * 2.5 ** j * (1.0 + 0.1 * k) for j in range(2)]
            out.append(dict(l=S.L_OF[letter], spherical=spherical, center=centre, exps=exps,
                            coefs=[float(x) for x in rng.uniform(0.3, 1.0, 2)]))
    return out


@pytest.mark.parametrize("spherical", [False, True], ids=["cart", "sph"])
def test_dense_eri_with_g_shells(spherical):
    shells = two_centre_g(spherical)
    check_eri(ib.Basis(shells).eri(), O.OracleBasis(shells).eri())


@pytest.mark.parametrize("spherical", [False, True], ids=["cart", "sph"])
def test_gggg_block(spherical):
    shells = two_centre_g(spherical)
    B, OB = ib.Basis(shells), O.OracleBasis(shells)
    for q in [(2, 4, 2, 4), (4, 4, 4, 4), (2, 2, 4, 2), (4, 0, 2, 3)]:
        check_eri(B.eri_block(*q), OB.eri_block(*q).reshape(-1))


def molecule(natom, seed):
    """One molecule of the batch recipe: spherical s,s,p,p,d,f,g of 3
    primitives 0.1*2.4^k in a cube of side 2.5 n^(1/3)."""
    rng = np.random.default_rng(seed)
    centers = S.place_atoms(rng, natom, 2.5 * natom ** (1.0 / 3.0), 1.6)
    shells = S.build_shells(rng, centers, "ssppdfg", 3, 0.1, 2.4, 0.2, 1.0, spherical=True)
    D = S.densities(rng, S.nao_of(shells), max(1, S.nao_of(shells) // 4), 1)
    return shells, D


def test_jk_with_g_shells_exact_list():
    shells, D = molecule(3, 7)
    dc = ib.Basis(shells).direct_contractor()
    J, K = dc.jk(D, 1e-11)
    st = dc.last_stats()
    Jo, Ko, cnt, hsh = O.OracleBasis(shells).direct_jk(D, 1e-11, nthreads=16)
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    assert float(np.max(np.abs(J - Jo))) < 1e-12 * float(np.max(np.abs(Jo)))
    assert float(np.max(np.abs(K - Ko))) < 1e-12 * float(np.max(np.abs(Ko)))
    Jm, Km = dc.jk(D, 1e-11, precision=1)
    e = lambda Jx, Kx: 0.5 * float(np.sum(D[0] * (Jx[0] - 0.5 * Kx[0])))
    assert abs(e(Jm, Km) - e(J, K)) < 1e-7


def test_gradient_with_g_shells():
    """The gradient classes of g shells (raised tables to l = 5): the exact
    screened list, and the gradient within 1e-10 of its maximum against the
    oracle (whose shifted classes the Auto policy also sends to OS/HGP)."""
    shells, D = molecule(3, 8)
    gc = ib.Basis(shells).direct_grad_contractor()
    coul, exch = [(0.5, D[0], D[0])], [(-0.25, D[0], D[0])]
    dens = gc.density([ib.GradDensityTerm(*t) for t in coul], [ib.GradDensityTerm(*t) for t in exch])
    out = np.zeros((gc.natom(), 3))
    gc.accumulate_bra_pairs(ib.DirectGradWorkspace(), None, dens, 1e-11, out)
    st = gc.last_stats()
    ref, cnt, hsh = O.OracleBasis(shells).direct_grad(coul, exch, 1e-11, nthreads=16)
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    assert float(np.max(np.abs(out - ref))) < 1e-10 * float(np.max(np.abs(ref)))
    assert float(np.max(np.abs(out.sum(axis=0)))) < 1e-9 * float(np.max(np.abs(out)))


def spread_molecule(natom, letters, seed=9):
    """Atoms over a 12-bohr cube with exponents 0.3*2.4^k: the shell pairs
    span up to 10 bohr, where FP32 rounding in the recurrences of high-l
    classes is amplified most."""
    rng = np.random.default_rng(seed)
    centers = S.place_atoms(rng, natom, 12.0, 1.8)
    shells = S.build_shells(rng, centers, letters, 3, 0.3, 2.4, 0.2, 1.0, spherical=True)
    nao = S.nao_of(shells)
    return shells, S.densities(rng, nao, max(1, nao // 4), 1)


@pytest.mark.parametrize("letters", ["ssppdf", "ssppdfg"], ids=["f", "g"])
def test_mixed_precision_error_with_high_l(letters):
    """MIXED precision at the default cutoffs keeps the energy error of f and
    g systems within 1e-7 Eh: classes with f or g shells take quartets into
    FP32 only below 1/100 or 1/10^4 of the cutoff (at one cutoff for all
    classes this 9-atom g system was off by 2.8e-4 Eh at 1e-3)."""
    shells, D = spread_molecule(9, letters)
    dc = ib.Basis(shells).direct_contractor()
    J64, K64 = dc.jk(D, 1e-11, precision=0)
    J32, K32 = dc.jk(D, 1e-11, precision=1)
    st = dc.last_stats()
    assert st["quartets_fp32"] > 0.3 * st["quartets"]
    e = lambda Jx, Kx: 0.5 * float(np.sum(D[0] * (Jx[0] - 0.5 * Kx[0])))
    assert abs(e(J32, K32) - e(J64, K64)) < 1e-7

