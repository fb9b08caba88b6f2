"""GPU parity of the long-range operator erf(omega r12)/r12 (EriKernel::Erf,
src/integrals.rs:304-321) against the oracle's Rys restatement of the
attenuated quadrature (src/engine/rys.rs:163-175): the dense tensor
(Basis::eri_kernel) and EriBuilder::kernel under the dense-ERI tolerances,
and the density-direct gradient (DirectGradContractor with an Erf kernel)
within 1e-12 of the oracle's with the identical quartet list.  The Coulomb
default is restored after every attenuated call."""
import numpy as np
import pytest

import integral_b200 as ib
import oracle_py as O
from integral_b200 import systems as S
from test_gpu_parity import check_eri

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("omega", [0.3, 1.0])
def test_erf_dense_eri_matches_oracle(omega):
    s = S.dense_eri_system()
    B = ib.Basis(s["shells"])
    gpu = B.eri_kernel(ib.EriKernel.Erf(omega))
    ref = O.OracleBasis(s["shells"]).eri_erf(omega)
    check_eri(gpu, ref)
    # the builder evaluates the same operator; Coulomb again afterwards
    check_eri(ib.EriBuilder(B).kernel(ib.EriKernel.Erf(omega)).build(), ref)
    check_eri(B.eri(), O.OracleBasis(s["shells"]).eri())


def test_erf_spherical_f_shells_match_oracle():
    shells = S.direct_contractor_fixture(True)
    gpu = ib.Basis(shells).eri_kernel(ib.EriKernel.Erf(0.5))
    check_eri(gpu, O.OracleBasis(shells).eri_erf(0.5))


@pytest.mark.parametrize("spherical", [False, True], ids=["cart", "sph"])
def test_erf_gradient_matches_oracle(spherical):
    shells = S.direct_grad_fixture(spherical)
    n = O.OracleBasis(shells).nao
    coul, exch = S.grad_fixture_terms(n)
    B = ib.Basis(shells)
    gc = B.direct_grad_contractor()
    dens = gc.density([ib.GradDensityTerm(*t) for t in coul], [ib.GradDensityTerm(*t) for t in exch])
    g = gc.contract(dens, kernel=ib.EriKernel.Erf(0.5), threshold=0.0)
    st = gc.last_stats()
    with O.erf(0.5):
        go, cnt, hsh = O.OracleBasis(shells).direct_grad(coul, exch, 0.0, engine="rys")
    assert st["quartets"] == cnt and st["quartet_hash"] == hsh
    assert float(np.max(np.abs(g - go))) < 1e-12 * float(np.max(np.abs(go)))
    assert float(np.max(np.abs(g.sum(axis=0)))) < 1e-10 * float(np.max(np.abs(g)))
    # Coulomb is the default again
    g0 = gc.contract(dens, threshold=0.0)
    go0, _, _ = O.OracleBasis(shells).direct_grad(coul, exch, 0.0)
    assert float(np.max(np.abs(g0 - go0))) < 1e-12 * float(np.max(np.abs(go0)))


def test_erf_omega_is_validated_by_the_library():
    """igpu_set_erf_omega rejects what check_erf_omega (src/integrals.rs:
    316-321) rejects, whatever the host side let through."""
    s = S.dense_eri_system()
    B = ib.Basis(s["shells"])
    for bad in (-0.5, float("nan"), float("inf")):
        with pytest.raises(ib.IntegralError):
            B.eri_kernel(ib.EriKernel(bad))
