"""The chunk autotuners (igpu_autotune_jk, igpu_autotune_grad): after
tuning, every launch runs with a chunk from the candidate set, and J, K and
the gradient equal the untuned builds within 1e-12 of their maxima (only
the order of the atomic additions changes)."""
import numpy as np
import pytest

import integral_b200 as ib
from integral_b200 import systems as S

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results_and_sets_candidate_chunks():
    import torch
    s = S.jk_system(natom=8, side=8.0, ndens=2)
    dc = ib.Basis(s["shells"]).direct_contractor()
    D = torch.from_numpy(s["dens"]).cuda()
    J0, K0 = torch.zeros_like(D), torch.zeros_like(D)
    dc.jk_device(D.data_ptr(), 2, J0.data_ptr(), K0.data_ptr(), s["threshold"], True, 1)
    before = [r["chunk"] for r in dc.plan.profile()]
    dc.autotune_device(D.data_ptr(), 2, s["threshold"], 1)
    J1, K1 = torch.zeros_like(D), torch.zeros_like(D)
    dc.jk_device(D.data_ptr(), 2, J1.data_ptr(), K1.data_ptr(), s["threshold"], True, 1)
    prof = dc.plan.profile()
    for r in prof:
        teams_per_warp = 32 // r["team"]
        assert r["chunk"] % teams_per_warp == 0 and r["chunk"] // teams_per_warp in (4, 8, 16, 32, 64)
    # untuned: 16 grabs per warp-team set, fewer for launches too small to
    # give every warp of the grid four grabs
    assert all(1 <= c // (32 // r["team"]) <= 16 for c, r in zip(before, prof))
    for a, b in ((J0, J1), (K0, K1)):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert float(np.max(np.abs(a - b))) < 1e-12 * float(np.max(np.abs(a)))


def test_gradient_autotune_keeps_results():
    shells = S.direct_grad_fixture(True)
    gc = ib.Basis(shells).direct_grad_contractor()
    n = gc.nao()
    coul, exch = S.grad_fixture_terms(n)
    dens = gc.density([ib.GradDensityTerm(*t) for t in coul], [ib.GradDensityTerm(*t) for t in exch])
    g0 = gc.contract(dens, threshold=0.0, precision=1)
    gc.autotune(dens, 0.0, 1)
    g1 = gc.contract(dens, threshold=0.0, precision=1)
    for r in gc._plan.profile():
        assert r["chunk"] // (32 // r["team"]) in (4, 8, 16, 32, 64)
    assert float(np.max(np.abs(g0 - g1))) < 1e-12 * float(np.max(np.abs(g0)))
