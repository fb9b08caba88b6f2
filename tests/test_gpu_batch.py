"""Molecule batches (igpu_batch_*): many independent molecules of uneven
size, every class in one persistent launch and the step captured in a CUDA
graph.  Each molecule's J, K and gradient must equal those of a plan of that
molecule alone (within the J/K contract, 1e-12 of the maxima; the quartet
counts add up exactly), the oracle directly on two molecules, and a replay
of the captured graph must reproduce the first step."""
import numpy as np
import pytest

import integral_b200 as ib
import oracle_py as O
from integral_b200 import systems as S

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def molecules(letters, counts, seed=5, spherical=True):
    """The batch recipe (3 primitives 0.1*2.4^k, cube side 2.5 n^(1/3), min
    separation 1.6) with the given shell letters and atom counts."""
    rng = np.random.default_rng(seed)
    out = []
    for n in counts:
        centers = S.place_atoms(rng, n, 2.5 * n ** (1.0 / 3.0), 1.6)
        shells = S.build_shells(rng, centers, letters, 3, 0.1, 2.4, 0.2, 1.0, spherical=spherical)
        nao = S.nao_of(shells)
        out.append((shells, S.densities(rng, nao, max(1, nao // 4), 1)[0]))
    return out


def per_molecule(shells, D, thr, gradient):
    dc = ib.Basis(shells).direct_contractor()
    J, K = dc.jk(D[None], thr)
    q = dc.last_stats()["quartets"]
    g = None
    if gradient:
        gc = ib.Basis(shells).direct_grad_contractor()
        dens = gc.density([ib.GradDensityTerm(0.5, D, D)], [ib.GradDensityTerm(-0.25, D, D)])
        g = gc.contract(dens, threshold=thr)
    return J[0], K[0], g, q


@pytest.mark.parametrize("letters", ["ssppdf", "ssppdfg"], ids=["spdf", "spdfg"])
def test_batch_equals_per_molecule_plans(letters):
    gradient = True
    g = "g" in letters
    mols = molecules(letters, [3, 6, 2, 5] if g else [3, 6, 2, 5, 4, 7])
    thr = 1e-11
    batch = ib.MoleculeBatch([m[0] for m in mols])
    J, K, G = batch.jk_grad([m[1] for m in mols], thr, gradient=gradient)
    # a second step replays the captured graph and reproduces the first
    J2, K2, G2 = batch.jk_grad([m[1] for m in mols], thr, gradient=gradient)
    for a, b in zip(J + K + G, J2 + K2 + G2):
        assert rel(a, b) < 1e-13
    total = 0
    for (shells, D), Jb, Kb, Gb in zip(mols, J, K, G):
        Jm, Km, Gm, q = per_molecule(shells, D, thr, gradient)
        total += q
        assert rel(Jb, Jm) < 1e-12 and rel(Kb, Km) < 1e-12
        if gradient:
            assert rel(Gb, Gm) < 1e-12
    # every quartet of every molecule, and no other: the batch screens with
    # the same bit-exact Schwarz bounds as the single plans
    batch.jk_grad([m[1] for m in mols], thr, gradient=False)
    assert batch.last_stats()["quartets"] == total
    # molecules against the oracle; with g shells the oracle's Auto policy
    # evaluates many quartets with OS/HGP, which agrees with Rys only to the
    # reference's own cross-engine contract (1e-11 + 1e-10 |x| per element,
    # tests/cross_engine.rs:40-56), so J/K are held to 1e-11 of their maxima
    bar = 1e-11 if g else 1e-12
    for k in ((1,) if g else (1, 4)):
        shells, D = mols[k]
        Jo, Ko, _, _ = O.OracleBasis(shells).direct_jk(D[None], thr, nthreads=16)
        assert rel(J[k], Jo[0]) < bar and rel(K[k], Ko[0]) < bar


def spread_molecules(counts, seed=9):
    """Molecules spread over a 12-bohr cube with tighter exponents
    (0.3*2.4^k): unlike the compact batch recipe, whose every quartet has a
    Schwarz product above the mixed cutoff, these have FP32 quartets."""
    rng = np.random.default_rng(seed)
    out = []
    for n in counts:
        centers = S.place_atoms(rng, n, 12.0, 1.8)
        shells = S.build_shells(rng, centers, "ssppdfg", 3, 0.3, 2.4, 0.2, 1.0, spherical=True)
        nao = S.nao_of(shells)
        out.append((shells, S.densities(rng, nao, max(1, nao // 4), 1)[0]))
    return out


def test_batch_mixed_precision_energy():
    mols = spread_molecules([6, 9, 5])
    batch = ib.MoleculeBatch([m[0] for m in mols])
    D = [m[1] for m in mols]
    J64, K64, _ = batch.jk_grad(D, 1e-11, precision=0, gradient=False)
    J32, K32, _ = batch.jk_grad(D, 1e-11, precision=1, gradient=False)
    st = batch.last_stats()
    assert 0 < st["quartets_fp32"] < st["quartets"]
    for d, a, b, c, e in zip(D, J64, K64, J32, K32):
        dE = 0.5 * float(np.sum(d * ((c - a) - 0.5 * (e - b))))
        assert abs(dE) < 1e-7
    # the same molecules in single mixed plans (whose FP32/FP64 split keys
    # on each molecule's own max |D|, not the batch's): within the FP32
    # rounding of the small quartets
    for (shells, Dm), Jb, Kb in zip(mols, J32, K32):
        Jm, Km = ib.Basis(shells).direct_contractor().jk(Dm[None], 1e-11, precision=1)
        assert rel(Jb, Jm[0]) < 1e-8 and rel(Kb, Km[0]) < 1e-8


def test_batch_argument_errors():
    mols = molecules("sspp", [2, 3])
    batch = ib.MoleculeBatch([m[0] for m in mols])
    with pytest.raises(ib.IntegralError) as e:
        batch.jk_grad([mols[0][1]], 1e-11)
    assert e.value.code == -7
    with pytest.raises(ib.IntegralError) as e:
        batch.jk_grad([m[1] for m in mols], 1e-11, precision=5)
    assert e.value.code == -1
