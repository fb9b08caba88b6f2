"""CPU-side checks of the product: the C-ABI library loads and exports every
symbol declared in include/integral_gpu.h, argument validation and error
codes that need no device, the synthetic systems, and the multi-rank
sharding (world size 2 over gloo)."""
import ctypes
import os
import re

import numpy as np
import pytest

import integral_b200 as ib
from integral_b200 import _lib, sharding
from integral_b200 import systems as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "integral_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|uint32_t|const char\*)\s+(igpu_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.EXPORTED)


def test_abi_version():
    assert ib.abi_version() == 1


def _shell(l=0, nprim=1, exps=(1.0,), coefs=(1.0,)):
    s = _lib.IgpuShell()
    s.l = l
    s.spherical = 0
    ex = (ctypes.c_double * max(1, len(exps)))(*exps)
    co = (ctypes.c_double * max(1, len(coefs)))(*coefs)
    s.nprim = nprim
    s.exps = ctypes.cast(ex, _lib.c_double_p)
    s.coefs = ctypes.cast(co, _lib.c_double_p)
    return s, (ex, co)


def test_plan_create_validation_codes():
    L = _lib.lib()
    h = ctypes.c_void_p()
    s, keep = _shell(nprim=0)
    assert L.igpu_plan_create(ctypes.byref(s), 1, 0, ctypes.byref(h)) == -2  # EmptyContraction
    s, keep = _shell(l=7)
    assert L.igpu_plan_create(ctypes.byref(s), 1, 0, ctypes.byref(h)) == -4  # AngularMomentumTooHigh
    s, keep = _shell()
    assert L.igpu_plan_create(ctypes.byref(s), 1, 5, ctypes.byref(h)) == -1  # unknown engine
    assert L.igpu_plan_create(ctypes.byref(s), 1, 0, None) == -1
    assert b"NULL" in L.igpu_last_error_string()


def test_batch_create_validation_codes():
    L = _lib.lib()
    h = ctypes.c_void_p()
    s, keep = _shell()
    counts = (ctypes.c_size_t * 2)(1, 0)
    assert L.igpu_batch_create(ctypes.byref(s), counts, 0, ctypes.byref(h)) == -1   # no molecules
    assert L.igpu_batch_create(ctypes.byref(s), counts, 2, ctypes.byref(h)) == -1   # molecule without shells
    one = (ctypes.c_size_t * 1)(1)
    bad, keep2 = _shell(nprim=0)
    assert L.igpu_batch_create(ctypes.byref(bad), one, 1, ctypes.byref(h)) == -2    # EmptyContraction
    bad, keep3 = _shell(l=7)
    assert L.igpu_batch_create(ctypes.byref(bad), one, 1, ctypes.byref(h)) == -4    # AngularMomentumTooHigh
    assert L.igpu_batch_create(ctypes.byref(s), one, 1, None) == -1
    assert L.igpu_batch_destroy(None) == 0


def test_ctypes_structs_match_the_header_layout(tmp_path):
    """Every struct of include/integral_gpu.h, compiled by the host C
    compiler, has the size and field offsets of its ctypes mirror."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    mirrors = {"igpu_shell": _lib.IgpuShell, "igpu_term": _lib.IgpuTerm, "igpu_stats": _lib.IgpuStats,
               "igpu_launch_record": _lib.IgpuLaunchRecord}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "integral_gpu.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append('printf("%%s %%zu\\n", "%s", sizeof(%s));' % (cname, cname))
        for f, _ in py._fields_:
            lines.append('printf("%%s.%%s %%zu\\n", "%s", "%s", offsetof(%s, %s));' % (cname, f, cname, f))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                        text=True).stdout.splitlines())
    for cname, py in mirrors.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got["%s.%s" % (cname, f)]) == getattr(py, f).offset, (cname, f)
    L = _lib.lib()
    assert L.igpu_autotune_jk(None, None, 1, 0.0, 0, None) == -1


def test_density_fitting_entries_reject_null_arguments():
    L = _lib.lib()
    assert L.igpu_plan_attach_aux(None, None, 0) == -1
    assert L.igpu_aux_query(None, None, None) == -1
    assert L.igpu_schwarz_aux(None, None) == -1
    assert L.igpu_eri_2c(None, None) == -1
    assert L.igpu_eri_3c(None, None, 0, None, None) == -1
    assert b"NULL" in L.igpu_last_error_string()


def test_python_shell_validation_mirrors_reference():
    with pytest.raises(ib.IntegralError) as e:
        ib.Shell(0, [0, 0, 0], [], [])
    assert e.value.code == -2
    with pytest.raises(ib.IntegralError) as e:
        ib.Shell(0, [0, 0, 0], [1.0, 2.0], [1.0])
    assert e.value.code == -3
    with pytest.raises(ib.IntegralError) as e:
        ib.Shell(7, [0, 0, 0], [1.0], [1.0])
    assert e.value.code == -4
    s = ib.Shell.new_spherical(3, [0, 0, 0], [1.0], [1.0])
    assert s.n_func() == 7 and s.n_cart() == 10
    s = ib.Shell.with_kind(2, [0, 0, 0], [1.0], [1.0], ib.ShellKind.Spherical)
    assert s.n_func() == 5 and s.kind() == ib.ShellKind.Spherical


def test_erf_kernel_requires_finite_positive_omega():
    # tests/erf_kernel.rs:512-524: omega <= 0 (or not finite) is rejected
    for bad in (0.0, -0.5, float("nan"), float("inf")):
        with pytest.raises(ib.IntegralError):
            ib.EriKernel.Erf(bad)
    assert ib.EriKernel.Erf(0.4).omega == 0.4
    assert ib.EriKernel.Coulomb.omega == 0.0


def test_basis_metadata_without_device():
    shells = [ib.Shell.from_dict(d) for d in S.direct_grad_fixture(False)]
    B = ib.Basis(shells)
    assert B.nao() == 1 + 3 + 6 + 1 + 10 + 3
    assert B.offsets() == [0, 1, 4, 10, 11, 21]
    assert len(B.atoms()) == 3


def test_synthetic_system_sizes():
    # AO counts follow the shell lists (Basis::nao), never a quoted figure
    assert S.nao_of(S.dense_eri_system()["shells"]) == 54
    assert S.nao_of(S.jk_system()["shells"]) == 960
    assert S.nao_of(S.jk_spherical_system()["shells"]) == 5200
    assert S.nao_of(S.grad_system()["shells"]) == 1400
    a = S.jk_system()
    b = S.jk_system()
    assert np.array_equal(a["dens"], b["dens"])


def test_bra_shards_partition_the_pairs():
    nbra = 1000
    parts = [sharding.bra_shard(nbra, r, 3) for r in range(3)]
    allp = np.sort(np.concatenate(parts))
    assert np.array_equal(allp, np.arange(nbra))


def _rank_main(rank, world, port, result_path):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    import oracle_py as O
    from integral_b200 import sharding as sh
    from integral_b200 import systems as syst
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    s = syst.jk_system(natom=5, side=6.0, ndens=2)
    B = O.OracleBasis(s["shells"])
    nbra = len(s["shells"]) * (len(s["shells"]) + 1) // 2
    J, K, cnt, _ = B.direct_jk(s["dens"], 1e-12, bras=sh.bra_shard(nbra, rank, world))
    counts = np.array([float(cnt)])
    sh.all_reduce_sum([J, K, counts])
    if rank == 0:
        np.savez(result_path, J=J, K=K, count=counts)
    dist.destroy_process_group()


def test_two_rank_sharded_jk_equals_single_rank(tmp_path):
    """World size 2 over gloo: each rank builds the J/K of its bra shard and
    one all-reduce sums them; the result equals the unsharded build."""
    import socket

    import torch.multiprocessing as mp
    sock = socket.socket()
    sock.bind(("127.0.0.1", 0))
    port = sock.getsockname()[1]
    sock.close()
    out = str(tmp_path / "r.npz")
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    import oracle_py as O
    s = S.jk_system(natom=5, side=6.0, ndens=2)
    B = O.OracleBasis(s["shells"])
    J, K, cnt, _ = B.direct_jk(s["dens"], 1e-12)
    r = np.load(out)
    assert int(r["count"][0]) == cnt
    assert float(np.max(np.abs(r["J"] - J))) < 1e-12 * float(np.max(np.abs(J)))
    assert float(np.max(np.abs(r["K"] - K))) < 1e-12 * float(np.max(np.abs(K)))


def _grad_rank_main(rank, world, port, result_path):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    import oracle_py as O
    from integral_b200 import sharding as sh
    from integral_b200 import systems as syst
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    shells = syst.direct_grad_fixture(False)
    B = O.OracleBasis(shells)
    coul, exch = syst.grad_fixture_terms(B.nao)
    nbra = len(shells) * (len(shells) + 1) // 2
    g, cnt, _ = B.direct_grad(coul, exch, 1e-10, bras=sh.bra_shard(nbra, rank, world))
    counts = np.array([float(cnt)])
    sh.all_reduce_sum([g, counts])
    if rank == 0:
        np.savez(result_path, g=g, count=counts)
    dist.destroy_process_group()


def test_two_rank_sharded_gradient_equals_single_rank(tmp_path):
    """World size 2 over gloo: each rank contracts the gradient of its bra
    shard (DirectGradContractor::accumulate_bra_pair over its pairs); one
    all-reduce of the natom x 3 forces gives the unsharded contraction."""
    import socket

    import torch.multiprocessing as mp
    sock = socket.socket()
    sock.bind(("127.0.0.1", 0))
    port = sock.getsockname()[1]
    sock.close()
    out = str(tmp_path / "g.npz")
    mp.start_processes(_grad_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    import oracle_py as O
    shells = S.direct_grad_fixture(False)
    B = O.OracleBasis(shells)
    coul, exch = S.grad_fixture_terms(B.nao)
    g, cnt, _ = B.direct_grad(coul, exch, 1e-10)
    r = np.load(out)
    assert int(r["count"][0]) == cnt
    assert float(np.max(np.abs(r["g"] - g))) < 1e-12 * float(np.max(np.abs(g)))


def test_bench_reference_arm_prints_the_contract_line():
    """bench.py --impl reference (the reference algorithm on the host cores,
    via the C++ restatement) prints one JSON line with the contract's keys."""
    import json
    import subprocess
    import sys

    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--cpu-sample-bras", "12"], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_integration_guide_binds_every_entry_point():
    """The Rust extern block of the integration guide declares every entry
    point of the header, and nothing else."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    header = open(os.path.join(root, "include", "integral_gpu.h")).read()
    guide = open(os.path.join(root, "INTEGRATION.md")).read()
    declared = set(re.findall(r"\b(igpu_[a-z0-9_]+)\s*\(", header))
    bound = set(re.findall(r"pub fn (igpu_[a-z0-9_]+)", guide))
    assert declared == bound, (sorted(declared - bound), sorted(bound - declared))

