"""Seeded synthetic systems for the two-electron benchmarks and parity tests.

The reference quotes its benchmarks on synthetic molecules (no public data
set): atoms placed uniformly at random in a cube with a minimum pair
separation, even-tempered primitive exponents and uniform random contraction
coefficients, and densities ``D = C Cᵀ`` with ``C`` normal of standard
deviation ``1/sqrt(nao)``.  Every generator here is deterministic for its seed.

Shells are returned as dicts ``{l, spherical, center, exps, coefs}`` which
both :class:`integral_b200.Basis` and the test oracle accept.  AO counts are
derived from the shell lists exactly as the reference derives them
(``Basis::nao`` = Σ n_func), never padded to a quoted figure.
"""
from __future__ import annotations

import numpy as np

L_OF = {"s": 0, "p": 1, "d": 2, "f": 3, "g": 4, "h": 5}


def n_cart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


def n_func(l: int, spherical: bool) -> int:
    return 2 * l + 1 if spherical else n_cart(l)


def place_atoms(rng, natom: int, side: float, min_sep: float, max_tries: int = 200000):
    """Uniform positions in [0, side)^3 by rejection sampling on the minimum
    pair separation."""
    pts = []
    tries = 0
    while len(pts) < natom:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place %d atoms in a %.2f cube at separation %.2f" % (natom, side, min_sep))
        p = rng.uniform(0.0, side, size=3)
        if all(np.sum((p - q) ** 2) >= min_sep * min_sep for q in pts):
            pts.append(p)
    return np.array(pts)


def build_shells(rng, centers, shell_letters, nprim, exp_base, exp_ratio, coef_lo, coef_hi,
                 spherical=False, scale_lo=None, scale_hi=None):
    shells = []
    for c in centers:
        for letter in shell_letters:
            l = L_OF[letter]
            scale = rng.uniform(scale_lo, scale_hi) if scale_lo is not None else 1.0
            exps = [exp_base * exp_ratio ** k * scale for k in range(nprim)]
            coefs = list(rng.uniform(coef_lo, coef_hi, size=nprim))
            shells.append(dict(l=l, spherical=spherical, center=[float(x) for x in c],
                               exps=[float(e) for e in exps], coefs=[float(x) for x in coefs]))
    return shells


def nao_of(shells) -> int:
    return sum(n_func(s["l"], s.get("spherical", False)) for s in shells)


def densities(rng, nao: int, nocc: int, count: int):
    """``count`` symmetric densities D = C Cᵀ, C ~ N(0, 1/sqrt(nao)), nao x nocc."""
    out = []
    for _ in range(count):
        C = rng.normal(0.0, 1.0 / np.sqrt(nao), size=(nao, nocc))
        D = C @ C.T
        out.append(0.5 * (D + D.T))
    return np.array(out)


# ----------------------------------------------------------------- configs

def dense_eri_system(seed: int = 1):
    """6 atoms in an 8-bohr cube (min separation 1.5), s,s,s,p,p Cartesian shells
    of 3 primitives with exponents 0.15*3^k scaled per shell by U(0.8,1.2),
    coefficients U(0.2,1.0): nao = 54, dense 54^4 tensor, no screening."""
    rng = np.random.default_rng(seed)
    centers = place_atoms(rng, 6, 8.0, 1.5)
    shells = build_shells(rng, centers, "ssspp", 3, 0.15, 3.0, 0.2, 1.0,
                          scale_lo=0.8, scale_hi=1.2)
    return dict(name="dense_eri_6atom_sp", shells=shells, seed=seed)


def jk_system(seed: int = 2, natom: int = 64, side: float = 20.0, ndens: int = 4, nocc: int = 80):
    """64 atoms in a 20-bohr cube (min separation 1.8), Cartesian s,s,s,p,p,d,
    3 primitives 0.1*2.5^k, coefficients U(0.2,1.0): nao = 960; four densities
    D = C Cᵀ with C 960 x 80; Schwarz threshold 1e-12."""
    rng = np.random.default_rng(seed)
    centers = place_atoms(rng, natom, side, 1.8)
    shells = build_shells(rng, centers, "sssppd", 3, 0.1, 2.5, 0.2, 1.0)
    nao = nao_of(shells)
    D = densities(rng, nao, nocc, ndens)
    return dict(name="jk_64atom_spd_cart", shells=shells, dens=D, threshold=1e-12, seed=seed)


def jk_spherical_system(seed: int = 3, natom: int = 200, side: float = 32.0, ndens: int = 2, nocc: int = 400):
    """200 atoms in a 32-bohr cube (min separation 1.8), spherical
    s,s,s,p,p,d,d,f, 4 primitives 0.08*2.2^k, coefficients U(0.1,1.0):
    nao = 5200 (26 spherical functions per atom); two densities with nocc 400;
    Schwarz threshold 1e-11."""
    rng = np.random.default_rng(seed)
    centers = place_atoms(rng, natom, side, 1.8)
    shells = build_shells(rng, centers, "sssppddf", 4, 0.08, 2.2, 0.1, 1.0, spherical=True)
    nao = nao_of(shells)
    D = densities(rng, nao, min(nocc, nao), ndens)
    return dict(name="jk_200atom_spdf_sph", shells=shells, dens=D, threshold=1e-11, seed=seed)


def grad_system(seed: int = 4, natom: int = 100, side: float = 24.0, nocc: int = 120):
    """100 atoms in a 24-bohr cube (min separation 1.8), Cartesian s,s,p,p,d,
    3 primitives 0.12*2.5^k, coefficients U(0.2,1.0): nao = 1400.  Two-particle
    density: Coulomb term (1/2, D, D) and exchange term (-1/4, D, D)."""
    rng = np.random.default_rng(seed)
    centers = place_atoms(rng, natom, side, 1.8)
    shells = build_shells(rng, centers, "ssppd", 3, 0.12, 2.5, 0.2, 1.0)
    nao = nao_of(shells)
    D = densities(rng, nao, min(nocc, nao), 1)[0]
    return dict(name="grad_100atom_spd_cart", shells=shells, dens=D, threshold=1e-12, seed=seed,
                coulomb=[(0.5, D, D)], exchange=[(-0.25, D, D)])


def molecule_batch(seed: int = 5, nmol: int = 256, lo: int = 4, hi: int = 40):
    """256 molecules with atom counts U{4..40}, each in a cube of side
    2.5*n^(1/3) (min separation 1.6), spherical s,s,p,p,d,f,g, 3 primitives
    0.1*2.4^k, coefficients U(0.2,1.0); densities with nocc = nao/4."""
    rng = np.random.default_rng(seed)
    mols = []
    for m in range(nmol):
        n = int(rng.integers(lo, hi + 1))
        centers = place_atoms(rng, n, 2.5 * n ** (1.0 / 3.0), 1.6)
        shells = build_shells(rng, centers, "ssppdfg", 3, 0.1, 2.4, 0.2, 1.0, spherical=True)
        nao = nao_of(shells)
        D = densities(rng, nao, max(1, nao // 4), 1)[0]
        mols.append(dict(shells=shells, dens=D))
    return dict(name="batch_256mol_spdfg_sph", molecules=mols, seed=seed)


# ------------------------------------------------- reference test fixtures

def direct_contractor_fixture(spherical: bool):
    """The 4-shell basis of the reference's tests/direct_contractor.rs:3-10."""
    return [
        dict(l=0, spherical=spherical, center=[0.0, 0.0, 0.0], exps=[1.2, 0.35], coefs=[0.7, 0.4]),
        dict(l=1, spherical=spherical, center=[0.2, -0.1, 0.5], exps=[0.8], coefs=[1.0]),
        dict(l=2, spherical=spherical, center=[-0.3, 0.4, -0.2], exps=[0.6], coefs=[1.0]),
        dict(l=3, spherical=spherical, center=[0.1, 0.3, 0.7], exps=[0.5], coefs=[1.0]),
    ]


def direct_contractor_densities(nao: int):
    """tests/direct_contractor.rs:33-39: two densities ((p+3s)%17-8)*0.013."""
    return np.array([[((p + 3 * shift) % 17 - 8.0) * 0.013 for p in range(nao * nao)]
                     for shift in range(2)]).reshape(2, nao, nao)


def direct_grad_fixture(spherical: bool):
    """The 6-shell, 3-centre basis of tests/direct_grad_contractor.rs:32-45."""
    a = [0.0, 0.0, 0.0]
    b = [0.9, -0.4, 0.6]
    c = [-0.7, 1.1, -0.3]
    return [
        dict(l=0, spherical=spherical, center=a, exps=[1.9, 0.45], coefs=[0.6, 0.5]),
        dict(l=1, spherical=spherical, center=a, exps=[0.8, 0.3], coefs=[0.7, 0.4]),
        dict(l=2, spherical=spherical, center=b, exps=[0.7], coefs=[1.0]),
        dict(l=0, spherical=spherical, center=b, exps=[0.5], coefs=[1.0]),
        dict(l=3, spherical=spherical, center=c, exps=[0.6], coefs=[1.0]),
        dict(l=1, spherical=spherical, center=c, exps=[1.1, 0.4], coefs=[0.3, 0.8]),
    ]


def grad_symmetric(n: int, seed: int):
    """tests/direct_grad_contractor.rs:47-58."""
    m = np.zeros((n, n))
    for p in range(n):
        for q in range(p + 1):
            v = (((p * 7 + q * 13 + seed * 5) % 23) - 11.0) * 0.017
            m[p, q] = v
            m[q, p] = v
    return m


def grad_fixture_terms(n: int):
    """tests/direct_grad_contractor.rs:60-104: two Coulomb-type and two
    exchange-type product terms over three symmetric matrices."""
    p, da, db = grad_symmetric(n, 1), grad_symmetric(n, 2), grad_symmetric(n, 3)
    return [(0.5, p, p), (0.3, da, db)], [(-0.5, da, da), (-0.2, db, p)]


# --------------------------------------------------------- density fitting

def df_fixture():
    """The main and auxiliary bases of the reference's tests/df.rs:31-51:
    main = contracted s, two p on one centre, spherical d; aux = s, p,
    spherical d, contracted s on or near the same centres."""
    main = [
        dict(l=0, spherical=False, center=[0.0, 0.0, 0.0], exps=[1.4, 0.5], coefs=[0.6, 0.5]),
        dict(l=1, spherical=False, center=[0.6, -0.3, 0.2], exps=[0.9], coefs=[1.0]),
        dict(l=1, spherical=False, center=[0.6, -0.3, 0.2], exps=[0.4], coefs=[1.0]),
        dict(l=2, spherical=True, center=[-0.4, 0.7, -0.1], exps=[1.1], coefs=[1.0]),
    ]
    aux = [
        dict(l=0, spherical=False, center=[0.0, 0.0, 0.0], exps=[2.1], coefs=[1.0]),
        dict(l=1, spherical=False, center=[0.6, -0.3, 0.2], exps=[1.3], coefs=[1.0]),
        dict(l=2, spherical=True, center=[-0.4, 0.7, -0.1], exps=[0.8], coefs=[1.0]),
        dict(l=0, spherical=False, center=[0.3, 0.1, -0.2], exps=[1.9, 0.7], coefs=[0.4, 0.8]),
    ]
    return main, aux


def df_system(seed: int = 6, natom: int = 5, side: float = 7.0, spherical: bool = True):
    """Density-fitting parity case: ``natom`` atoms in a ``side``-bohr cube
    (min separation 1.5); main s,s,p,p,d,f of 3 primitives 0.12*2.5^k
    (coefficients U(0.2,1.0)); aux s,p,d,f,s,p,d of single primitives
    0.2*1.8^k scaled per shell by U(0.8,1.2), one kind for both bases."""
    rng = np.random.default_rng(seed)
    centers = place_atoms(rng, natom, side, 1.5)
    main = build_shells(rng, centers, "ssppdf", 3, 0.12, 2.5, 0.2, 1.0, spherical=spherical)
    aux = []
    for c in centers:
        for k, letter in enumerate("spdfspd"):
            e = 0.2 * 1.8 ** k * rng.uniform(0.8, 1.2)
            aux.append(dict(l=L_OF[letter], spherical=spherical, center=[float(x) for x in c],
                            exps=[float(e)], coefs=[1.0]))
    return dict(name="df_%datom" % natom, main=main, aux=aux, seed=seed)


def grad_extended_fixture():
    """tests/direct_grad_contractor.rs:636-660: four atoms 8.5 to 19.3 bohr
    apart with diffuse valence shells (s of 2 primitives, p, and a spherical
    d on every other atom), so shell-pair overlaps span many orders."""
    atoms = [[0.0, 0.0, 0.0], [8.5, 0.0, 0.5], [8.0, 9.0, -0.4], [19.0, 3.0, 1.0]]
    shells = []
    for a, at in enumerate(atoms):
        shells.append(dict(l=0, spherical=False, center=at, exps=[1.2, 0.25], coefs=[0.5, 0.6]))
        shells.append(dict(l=1, spherical=False, center=at, exps=[0.3], coefs=[1.0]))
        if a % 2 == 0:
            shells.append(dict(l=2, spherical=True, center=at, exps=[0.28], coefs=[1.0]))
    return shells
