"""The J/K chunk autotuner (igpu_autotune_jk): after tuning, every J/K
launch runs with a chunk from the candidate set, and J and K equal the
untuned build within 1e-12 of their maxima (only the order of the atomic
additions changes)."""
import numpy as np
import pytest

import integral_b200 as ib
from integral_b200 import systems as S

pytestmark = [pytest.mark.gpu, pytest.mark.skip(reason="pending its first run on a B200")]


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
    assert all(c // (32 // r["team"]) == 16 for c, r in zip(before, prof))
    for a, b in ((J0, J1), (K0, K1)):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert float(np.max(np.abs(a - b))) < 1e-12 * float(np.max(np.abs(a)))
