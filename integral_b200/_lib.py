"""ctypes binding of libintegral_b200.so (the C ABI of include/integral_gpu.h).

The shared library is built in-tree (``make -C integral_b200/csrc``); there is
no fallback: if it is missing or the device is absent, calls fail loudly.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libintegral_b200.so")

c_double_p = ctypes.POINTER(ctypes.c_double)
c_u32_p = ctypes.POINTER(ctypes.c_uint32)
c_size_p = ctypes.POINTER(ctypes.c_size_t)


class IgpuShell(ctypes.Structure):
    _fields_ = [("l", ctypes.c_int), ("spherical", ctypes.c_int), ("center", ctypes.c_double * 3),
                ("nprim", ctypes.c_int), ("exps", c_double_p), ("coefs", c_double_p)]


class IgpuTerm(ctypes.Structure):
    _fields_ = [("factor", ctypes.c_double), ("left", c_double_p), ("right", c_double_p)]


class IgpuStats(ctypes.Structure):
    _fields_ = [("quartets", ctypes.c_uint64), ("quartet_hash", ctypes.c_uint64),
                ("quartets_fp32", ctypes.c_uint64), ("prim_quartets", ctypes.c_uint64),
                ("model_flops", ctypes.c_double), ("kernel_ms", ctypes.c_double),
                ("launches", ctypes.c_uint32)]


class IgpuLaunchRecord(ctypes.Structure):
    _fields_ = [("la", ctypes.c_int), ("lb", ctypes.c_int), ("lc", ctypes.c_int), ("ld", ctypes.c_int),
                ("fp32", ctypes.c_int), ("team", ctypes.c_int), ("grid", ctypes.c_uint32),
                ("tasks", ctypes.c_uint64), ("quartets", ctypes.c_uint64), ("prim_quartets", ctypes.c_uint64),
                ("ms", ctypes.c_double), ("model_flops", ctypes.c_double), ("chunk", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


STATUS = {
    0: "ok", -1: "invalid argument", -2: "empty contraction", -3: "mismatched contraction",
    -4: "angular momentum too high", -5: "angular momentum too high for gradient",
    -6: "density count", -7: "length mismatch", -8: "non-canonical bra pair", -9: "CUDA error",
    -10: "out of device memory", -11: "unsupported", -12: "no CUDA device",
}

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libintegral_b200.so is not built: run `make -C integral_b200/csrc` "
                           "(or __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.igpu_abi_version.restype = ctypes.c_uint32
    L.igpu_last_error_string.restype = ctypes.c_char_p
    L.igpu_plan_create.argtypes = [ctypes.POINTER(IgpuShell), ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(vp)]
    L.igpu_plan_destroy.argtypes = [vp]
    L.igpu_plan_query.argtypes = [vp, c_size_p, c_size_p, c_size_p, c_size_p]
    L.igpu_bra_pairs.argtypes = [vp, c_u32_p]
    L.igpu_atoms.argtypes = [vp, c_double_p]
    L.igpu_schwarz.argtypes = [vp, c_double_p]
    L.igpu_schwarz_bounds.argtypes = [ctypes.POINTER(IgpuShell), ctypes.c_size_t, c_double_p, c_size_p]
    L.igpu_set_mixed_cutoff.argtypes = [vp, ctypes.c_double]
    L.igpu_set_mixed_prim_cutoff.argtypes = [vp, ctypes.c_double]
    L.igpu_get_mixed_cutoffs.argtypes = [vp, c_double_p, c_double_p]
    L.igpu_set_erf_omega.argtypes = [vp, ctypes.c_double]
    L.igpu_eri_dense.argtypes = [vp, c_double_p]
    L.igpu_eri_builder_fill.argtypes = [vp, c_u32_p, ctypes.c_size_t, c_double_p]
    L.igpu_eri_packed.argtypes = [vp, ctypes.c_double, c_u32_p, ctypes.c_size_t, c_double_p]
    L.igpu_eri_screened.argtypes = [vp, ctypes.c_double, c_double_p, ctypes.POINTER(ctypes.c_uint64),
                                    ctypes.POINTER(ctypes.c_uint64)]
    L.igpu_eri_block.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_double_p]
    L.igpu_plan_attach_aux.argtypes = [vp, ctypes.POINTER(IgpuShell), ctypes.c_size_t]
    L.igpu_aux_query.argtypes = [vp, c_size_p, c_size_p]
    L.igpu_schwarz_aux.argtypes = [vp, c_double_p]
    L.igpu_eri_2c.argtypes = [vp, c_double_p]
    L.igpu_eri_3c.argtypes = [vp, c_u32_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint8), c_double_p]
    L.igpu_density_shell_bounds.argtypes = [vp, c_double_p, ctypes.c_int, c_double_p]
    L.igpu_jk.argtypes = [vp, c_double_p, ctypes.c_int, c_u32_p, ctypes.c_size_t, ctypes.c_double,
                          ctypes.c_int, ctypes.c_int, c_double_p, c_double_p]
    L.igpu_jk_device.argtypes = [vp, vp, ctypes.c_int, c_u32_p, ctypes.c_size_t, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int, vp, vp, vp]
    L.igpu_jk_device_static.argtypes = [vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, vp, vp, vp]
    L.igpu_grad.argtypes = [vp, ctypes.POINTER(IgpuTerm), ctypes.c_int, ctypes.POINTER(IgpuTerm), ctypes.c_int,
                            c_u32_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_int, c_double_p]
    L.igpu_grad_device.argtypes = [vp, ctypes.POINTER(IgpuTerm), ctypes.c_int, ctypes.POINTER(IgpuTerm),
                                   ctypes.c_int, c_u32_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_int, vp, vp]
    L.igpu_last_stats.argtypes = [vp, ctypes.POINTER(IgpuStats)]
    L.igpu_last_profile.argtypes = [vp, ctypes.POINTER(IgpuLaunchRecord), ctypes.c_size_t, c_size_p]
    L.igpu_autotune_jk.argtypes = [vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, vp]
    L.igpu_autotune_grad.argtypes = [vp, ctypes.POINTER(IgpuTerm), ctypes.c_int, ctypes.POINTER(IgpuTerm),
                                     ctypes.c_int, ctypes.c_double, ctypes.c_int]
    L.igpu_batch_create.argtypes = [ctypes.POINTER(IgpuShell), c_size_p, ctypes.c_size_t, ctypes.POINTER(vp)]
    L.igpu_batch_destroy.argtypes = [vp]
    L.igpu_batch_query.argtypes = [vp, ctypes.c_size_t, c_size_p, c_size_p, c_size_p]
    L.igpu_batch_jk_grad.argtypes = [vp, c_double_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_double, c_double_p, c_double_p, c_double_p,
                                     ctypes.POINTER(IgpuStats)]
    L.igpu_batch_set_mixed_cutoff.argtypes = [vp, ctypes.c_double]
    _lib = L
    return L


EXPORTED = [
    "igpu_abi_version", "igpu_last_error_string", "igpu_plan_create", "igpu_plan_destroy", "igpu_plan_query",
    "igpu_bra_pairs", "igpu_atoms", "igpu_schwarz", "igpu_schwarz_bounds", "igpu_set_mixed_cutoff", "igpu_set_mixed_prim_cutoff", "igpu_get_mixed_cutoffs", "igpu_set_erf_omega",
    "igpu_eri_dense",
    "igpu_eri_builder_fill", "igpu_eri_screened", "igpu_eri_block", "igpu_eri_packed", "igpu_plan_attach_aux", "igpu_aux_query", "igpu_schwarz_aux",
    "igpu_eri_2c", "igpu_eri_3c", "igpu_density_shell_bounds", "igpu_jk", "igpu_jk_device", "igpu_jk_device_static",
    "igpu_grad",
    "igpu_grad_device", "igpu_last_stats", "igpu_last_profile", "igpu_autotune_jk", "igpu_autotune_grad",
    "igpu_batch_create", "igpu_batch_destroy", "igpu_batch_query", "igpu_batch_jk_grad", "igpu_batch_set_mixed_cutoff",
]


def check(rc: int):
    if rc != 0:
        msg = lib().igpu_last_error_string().decode(errors="replace")
        from . import IntegralError
        raise IntegralError(rc, STATUS.get(rc, "error"), msg)
