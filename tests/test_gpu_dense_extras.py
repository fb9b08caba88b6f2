"""GPU parity of Basis::eri_block (src/integrals.rs:600-640) and
Basis::eri_screened (src/integrals.rs:864-981) against the oracle: blocks
in canonical and permuted shell orders, Cartesian and spherical, within the
dense-ERI tolerances; the screened tensor element-wise, with the
ScreeningStats counts equal to the oracle's."""
import numpy as np
import pytest

import integral_b200 as ib
import oracle_py as O
from integral_b200 import systems as S

pytestmark = pytest.mark.gpu


def check(gpu, ref):
    peak = float(np.max(np.abs(ref)))
    d = np.abs(gpu - ref)
    sig = np.abs(ref) >= 1e-3 * peak
    assert float(np.max(d[sig] / np.abs(ref[sig]))) < 1e-12
    assert float(np.max(d)) < 1e-13 * max(peak, 1.0)


@pytest.mark.parametrize("spherical", [False, True], ids=["cart", "sph"])
def test_eri_block_in_any_shell_order(spherical):
    shells = S.direct_contractor_fixture(spherical)
    B, OB = ib.Basis(shells), O.OracleBasis(shells)
    for q in [(0, 0, 0, 0), (3, 2, 1, 0), (0, 1, 2, 3), (1, 3, 0, 2), (2, 2, 3, 1), (3, 3, 3, 3), (1, 0, 1, 0)]:
        check(B.eri_block(*q), OB.eri_block(*q).reshape(-1))


def test_eri_screened_matches_oracle():
    s = S.dense_eri_system()
    B, OB = ib.Basis(s["shells"]), O.OracleBasis(s["shells"])
    for tau in (0.0, 1e-8, 1e-4):
        gpu, st = B.eri_screened(tau)
        ref, total, skipped = OB.eri_screened(tau)
        assert st.shell_quartets_total == total and st.shell_quartets_skipped == skipped and st.tau == tau
        check(gpu, ref)
        skipped = ~OB.screened_mask(tau).reshape(-1)
        assert np.all(gpu[skipped] == 0.0)
