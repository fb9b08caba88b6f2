"""Properties of the GPU gradient that the reference's
tests/direct_grad_contractor.rs:556-690 checks: Coulomb-only plus
exchange-only equals both terms (1e-12), no terms is exactly zero, bra-pair
tasks summed in any order give the full contraction (1e-12), and on the
extended four-atom system the screened error stays below 100 tau for tau in
{1e-12, 1e-9, 1e-6} while tau = inf drops every quartet."""
import numpy as np
import pytest

import integral_b200 as ib
import oracle_py as O
from integral_b200 import systems as S

pytestmark = pytest.mark.gpu


def contractor(shells):
    return ib.Basis(shells).direct_grad_contractor()


def contract(gc, coul, exch, threshold=0.0, bras=None):
    dens = gc.density([ib.GradDensityTerm(*t) for t in coul], [ib.GradDensityTerm(*t) for t in exch])
    out = np.zeros((gc.natom(), 3))
    gc.accumulate_bra_pairs(ib.DirectGradWorkspace(), bras, dens, threshold, out)
    return out, gc.last_stats()


def test_term_lists_are_additive_and_empty_terms_give_zero():
    shells = S.direct_grad_fixture(True)
    gc = contractor(shells)
    coul, exch = S.grad_fixture_terms(O.OracleBasis(shells).nao)
    both, _ = contract(gc, coul, exch)
    c_only, _ = contract(gc, coul, [])
    x_only, _ = contract(gc, [], exch)
    assert float(np.max(np.abs(c_only))) > 1e-3 and float(np.max(np.abs(x_only))) > 1e-3
    assert float(np.max(np.abs(c_only + x_only - both))) < 1e-12
    nothing, _ = contract(gc, [], [])
    assert np.all(nothing == 0.0)


def test_bra_tasks_sum_in_any_order():
    shells = S.direct_grad_fixture(True)
    gc = contractor(shells)
    p = S.grad_symmetric(O.OracleBasis(shells).nao, 4)
    terms = [(1.0, p, p)]
    serial, _ = contract(gc, terms, terms)
    rev = np.arange(len(gc.bra_pairs()))[::-1]
    parts = [contract(gc, terms, terms, bras=rev[t::2])[0] for t in range(2)]
    assert float(np.max(np.abs(parts[0] + parts[1] - serial))) < 1e-12


def test_screening_error_is_bounded_on_extended_system():
    shells = S.grad_extended_fixture()
    gc = contractor(shells)
    OB = O.OracleBasis(shells)
    coul, exch = S.grad_fixture_terms(OB.nao)
    exact, _ = contract(gc, coul, exch)
    ref, _, _ = OB.direct_grad(coul, exch, 0.0)
    assert float(np.max(np.abs(exact - ref))) < 1e-12 * float(np.max(np.abs(ref)))
    for thr in (1e-12, 1e-9, 1e-6):
        screened, st = contract(gc, coul, exch, thr)
        _, cnt, hsh = OB.direct_grad(coul, exch, thr)
        assert st["quartets"] == cnt and st["quartet_hash"] == hsh
        assert float(np.max(np.abs(screened - exact))) < 100.0 * thr
    nothing, st = contract(gc, coul, exch, float("inf"))
    assert st["quartets"] == 0 and np.all(nothing == 0.0)


def test_repeated_bra_pair_is_rejected():
    shells = S.direct_grad_fixture(False)
    gc = contractor(shells)
    coul, exch = S.grad_fixture_terms(O.OracleBasis(shells).nao)
    with pytest.raises(ib.IntegralError) as e:
        contract(gc, coul, exch, bras=[3, 5, 3])
    assert e.value.code == -1
    dc = ib.Basis(shells).direct_contractor()
    D = S.grad_symmetric(O.OracleBasis(shells).nao, 2)[None]
    with pytest.raises(ib.IntegralError):
        dc.jk(D, 0.0, bras=[1, 1])
