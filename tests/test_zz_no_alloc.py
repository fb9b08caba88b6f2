"""The J/K entry point that allocates no device memory
(igpu_jk_device_static, for callers whose device memory is owned by their
own pool allocator) against the allocating one (igpu_jk_device) on the same
device-resident densities, within the J/K tolerance of the other GPU tests.

Collected last on purpose (file name): it must pass after every other GPU
test has run in the same process, and alone.
"""
import numpy as np
import pytest

import integral_b200 as ib
from integral_b200 import systems as S

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


def test_static_entry_matches_allocating_entry_on_two_calls_in_a_row():
    import torch

    s = S.jk_system(natom=8, side=8.0, ndens=2)
    dc = ib.Basis(s["shells"]).direct_contractor()
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(21)
    # one symmetric and one non-symmetric density
    Dh = s["dens"].copy()
    Dh[1] += 0.01 * rng.normal(size=Dh[1].shape)
    D = torch.tensor(Dh, dtype=torch.float64, device=dev).contiguous()
    thr = s["threshold"]
    J0 = torch.zeros_like(D)
    K0 = torch.zeros_like(D)
    dc.jk_device(D.data_ptr(), 2, J0.data_ptr(), K0.data_ptr(), thr)
    torch.cuda.synchronize()
    outs = [(torch.zeros_like(D), torch.zeros_like(D)) for _ in range(2)]
    # the first static call does the per-device set-up; the ones after it
    # must leave the device's free memory exactly where it was
    free_before = None
    for J, K in outs:
        dc.jk_device_static(D.data_ptr(), 2, J.data_ptr(), K.data_ptr(), thr)
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if free_before is not None:
            assert free_after == free_before
        free_before = free_after
        assert rel(J, J0) < 1e-12
        assert rel(K, K0) < 1e-12
    J, K = outs[-1]
    # outputs accumulate
    dc.jk_device_static(D.data_ptr(), 2, J.data_ptr(), K.data_ptr(), thr)
    torch.cuda.synchronize()
    assert rel(J, 2 * J0) < 1e-12
    assert rel(K, 2 * K0) < 1e-12


def test_static_entry_requires_a_prepared_task_list():
    import torch

    s = S.jk_system(natom=4, side=6.0, ndens=1)
    dc = ib.Basis(s["shells"]).direct_contractor()
    D = torch.tensor(s["dens"], dtype=torch.float64, device="cuda").contiguous()
    J = torch.zeros_like(D)
    K = torch.zeros_like(D)
    with pytest.raises(ib.IntegralError) as e:
        dc.jk_device_static(D.data_ptr(), 1, J.data_ptr(), K.data_ptr(), 3.7e-13)
    assert e.value.code == -1
