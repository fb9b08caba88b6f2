"""integral_b200 — B200-native two-electron integrals behind the API of the
Rust crate ``integral`` (nmrtist/integral 0.4.3).

The host-side classes mirror the reference's public types so callers (and the
parity tests) read like the reference's own code:

=========================  ==================================================
reference (Rust)           here
=========================  ==================================================
``Shell`` / ``ShellKind``  :class:`Shell`, :class:`ShellKind` (src/shell.rs)
``Basis``                  :class:`Basis` (``nao``, ``atoms``, ``eri``,
                           ``schwarz_bounds``, ``direct_contractor``, ...)
``Engine``                 :class:`Engine` (src/integrals.rs:329-338)
``EriBuilder``             :class:`EriBuilder` (src/eri_builder.rs)
``PackedEriBuilder``       :class:`PackedEriBuilder`, :class:`PackedBraFill`,
                           :class:`PackedEriWorkspace` (src/packed_eri.rs)
``Eri3cBuilder``           :class:`Eri3cBuilder`, :class:`Bra3cFill`;
                           ``Basis.eri_2c``, ``Basis.schwarz_aux_bounds``
                           (src/df.rs)
``EriKernel``              :class:`EriKernel` (``Coulomb``, ``Erf(omega)``;
                           src/integrals.rs:304-321)
``ScreeningStats``         :class:`ScreeningStats` (src/integrals.rs:983-1005)
``select_engine``          :func:`select_engine` (src/integrals.rs:374-388)
``DirectContractor``       :class:`DirectContractor`, :class:`DirectWorkspace`,
                           :class:`DirectBuffers` (src/direct.rs)
``DirectGradContractor``   :class:`DirectGradContractor`,
                           :class:`GradDensityTerm`, :class:`GradDensity`,
                           :class:`DirectGradWorkspace` (src/direct_grad.rs)
``IntegralError``          :class:`IntegralError` (src/lib.rs:83-162)
=========================  ==================================================

Every quartet is evaluated by the CUDA kernels of ``libintegral_b200.so``
(sm_100a) through the C ABI declared in ``include/integral_gpu.h``; there is
no CPU evaluation path.  Besides the reference's per-bra-pair methods, the
contractors accept a whole bra-pair list in one call (one launch sequence),
which is how a GPU caller should drive them.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import IgpuShell, IgpuStats, IgpuTerm, c_double_p, c_u32_p

MAX_L = 6
MAX_GRAD_L = MAX_L - 1


class IntegralError(Exception):
    """A failed call; ``code`` is the C-ABI status (include/integral_gpu.h)."""

    def __init__(self, code: int, kind: str, message: str = ""):
        super().__init__("%s (%d): %s" % (kind, code, message))
        self.code = code
        self.kind = kind


class ShellKind(enum.Enum):
    Cartesian = 0
    Spherical = 1


class Engine(enum.IntEnum):
    Auto = 0
    OsHgp = 1
    Rys = 2


class EriKernel:
    """Two-electron operator (src/integrals.rs:304-312): EriKernel.Coulomb
    (1/r12) or EriKernel.Erf(omega) (the long-range erf(omega r12)/r12,
    omega finite and > 0)."""

    Coulomb = None  # set below

    def __init__(self, omega: float = 0.0):
        self.omega = float(omega)

    @classmethod
    def Erf(cls, omega: float) -> "EriKernel":
        if not (omega > 0.0 and np.isfinite(omega)):
            raise IntegralError(-1, "invalid argument", "EriKernel::Erf requires a finite omega > 0")
        return cls(omega)

    def __repr__(self):
        return "EriKernel.Coulomb" if self.omega == 0.0 else "EriKernel.Erf(omega=%r)" % self.omega


EriKernel.Coulomb = EriKernel(0.0)


def select_engine(ne: int, nf: int, contraction_degree: int) -> Engine:
    """select_engine (src/integrals.rs:374-388): the reference's CPU engine
    policy for a quartet of bra / ket angular sums ne, nf and primitive
    product contraction_degree: OS/HGP from degree 1 up to l_total 5, from
    degree 3 up to l_total 16 when max(ne, nf) <= 6, from degree 16 above
    that, Rys for l_total >= 17.  Kept for API parity: the GPU evaluates
    every class with its Rys kernels whatever this returns."""
    l_total = ne + nf
    if l_total >= 17:
        return Engine.Rys
    if l_total <= 5:
        threshold = 1
    elif max(ne, nf) <= 6:
        threshold = 3
    else:
        threshold = 16
    return Engine.OsHgp if contraction_degree >= threshold else Engine.Rys


def _omega_of(kernel) -> float:
    return 0.0 if kernel is None else float(kernel.omega)


@dataclass
class ScreeningStats:
    """Outcome of a Schwarz-screened dense build (src/integrals.rs:983-1005):
    canonical shell quartets considered and skipped, and tau."""
    shell_quartets_total: int
    shell_quartets_skipped: int
    tau: float

    def skipped_fraction(self) -> float:
        if self.shell_quartets_total == 0:
            return 0.0
        return self.shell_quartets_skipped / self.shell_quartets_total


def n_cart(l: int) -> int:
    return (l + 1) * (l + 2) // 2


class Shell:
    """A contracted shell (src/shell.rs:49-188).  Coefficients are raw; the
    per-primitive normalisation is applied by the plan."""

    def __init__(self, l: int, center, exponents, coefficients, kind: ShellKind = ShellKind.Cartesian):
        exps = [float(x) for x in exponents]
        coefs = [float(x) for x in coefficients]
        if len(exps) == 0:
            raise IntegralError(-2, "empty contraction", "shell has no primitives")
        if len(exps) != len(coefs):
            raise IntegralError(-3, "mismatched contraction",
                                "%d exponents but %d coefficients" % (len(exps), len(coefs)))
        if l > MAX_L:
            raise IntegralError(-4, "angular momentum too high", "l=%d exceeds %d" % (l, MAX_L))
        self._l = int(l)
        self._center = tuple(float(c) for c in center)
        self._exps = exps
        self._coefs = coefs
        self._kind = kind

    @classmethod
    def new(cls, l, center, exponents, coefficients):
        return cls(l, center, exponents, coefficients, ShellKind.Cartesian)

    @classmethod
    def new_spherical(cls, l, center, exponents, coefficients):
        return cls(l, center, exponents, coefficients, ShellKind.Spherical)

    @classmethod
    def with_kind(cls, l, center, exponents, coefficients, kind: ShellKind):
        """Shell::with_kind (src/shell.rs:92-118)."""
        return cls(l, center, exponents, coefficients, kind)

    @classmethod
    def from_dict(cls, d):
        return cls(d["l"], d["center"], d["exps"], d["coefs"],
                   ShellKind.Spherical if d.get("spherical") else ShellKind.Cartesian)

    def l(self) -> int:
        return self._l

    def center(self):
        return self._center

    def exponents(self):
        return list(self._exps)

    def coefficients(self):
        return list(self._coefs)

    def kind(self) -> ShellKind:
        return self._kind

    def n_cart(self) -> int:
        return n_cart(self._l)

    def n_func(self) -> int:
        return 2 * self._l + 1 if self._kind == ShellKind.Spherical else n_cart(self._l)

    def n_prim(self) -> int:
        return len(self._exps)


class _Plan:
    """Owner of one igpu_plan (device-resident precompute)."""

    def set_erf_omega(self, omega: float):
        """Operator of later calls: 0 Coulomb, > 0 erf(omega r)/r."""
        _lib.check(_lib.lib().igpu_set_erf_omega(self.h, float(omega)))

    @staticmethod
    def _shell_array(shells: Sequence[Shell], keep: list):
        arr = (IgpuShell * max(1, len(shells)))()
        for k, s in enumerate(shells):
            ex = np.ascontiguousarray(s._exps, dtype=np.float64)
            co = np.ascontiguousarray(s._coefs, dtype=np.float64)
            keep += [ex, co]
            arr[k].l = s._l
            arr[k].spherical = 1 if s._kind == ShellKind.Spherical else 0
            for c in range(3):
                arr[k].center[c] = s._center[c]
            arr[k].nprim = len(s._exps)
            arr[k].exps = ex.ctypes.data_as(c_double_p)
            arr[k].coefs = co.ctypes.data_as(c_double_p)
        return arr

    def attach_aux(self, aux: "Basis"):
        """Attach `aux` as the density-fitting basis (once per aux object)."""
        if getattr(self, "_aux", None) is aux:
            return
        keep = []
        arr = self._shell_array(aux._shells, keep)
        self._aux = None
        _lib.check(_lib.lib().igpu_plan_attach_aux(self.h, arr, len(aux._shells)))
        naux, nsh = ctypes.c_size_t(), ctypes.c_size_t()
        _lib.check(_lib.lib().igpu_aux_query(self.h, ctypes.byref(naux), ctypes.byref(nsh)))
        self._aux, self.naux, self.naux_sh = aux, naux.value, nsh.value

    def __init__(self, shells: Sequence[Shell], engine: Engine):
        L = _lib.lib()
        self._keep = []
        arr = self._shell_array(shells, self._keep)
        h = ctypes.c_void_p()
        _lib.check(L.igpu_plan_create(arr, len(shells), int(engine), ctypes.byref(h)))
        self.h = h
        nao, natom, nbra, nsh = (ctypes.c_size_t() for _ in range(4))
        _lib.check(L.igpu_plan_query(h, ctypes.byref(nao), ctypes.byref(natom), ctypes.byref(nbra),
                                     ctypes.byref(nsh)))
        self.nao, self.natom, self.nbra, self.nsh = nao.value, natom.value, nbra.value, nsh.value

    def __del__(self):
        try:
            if getattr(self, "h", None):
                _lib.lib().igpu_plan_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def bra_pairs(self):
        out = np.zeros(2 * self.nbra, dtype=np.uint32)
        _lib.check(_lib.lib().igpu_bra_pairs(self.h, out.ctypes.data_as(c_u32_p)))
        return [(int(out[2 * p]), int(out[2 * p + 1])) for p in range(self.nbra)]

    def stats(self) -> dict:
        st = IgpuStats()
        _lib.check(_lib.lib().igpu_last_stats(self.h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in IgpuStats._fields_}

    def profile(self) -> list:
        """Per-launch records (class, precision, time, counters) of the last call."""
        n = ctypes.c_size_t()
        _lib.check(_lib.lib().igpu_last_profile(self.h, None, 0, ctypes.byref(n)))
        arr = (_lib.IgpuLaunchRecord * max(1, n.value))()
        _lib.check(_lib.lib().igpu_last_profile(self.h, arr, n.value, ctypes.byref(n)))
        return [{f: getattr(arr[k], f) for f, _ in _lib.IgpuLaunchRecord._fields_} for k in range(n.value)]


class Basis:
    """An ordered list of shells (src/shell.rs:193-276)."""

    def __init__(self, shells: Sequence[Shell]):
        self._shells = [s if isinstance(s, Shell) else Shell.from_dict(s) for s in shells]
        self._plans = {}

    @classmethod
    def new(cls, shells: Sequence[Shell]) -> "Basis":
        """Basis::new (src/shell.rs)."""
        return cls(shells)

    def shells(self):
        return list(self._shells)

    def nao(self) -> int:
        return sum(s.n_func() for s in self._shells)

    def nao_cart(self) -> int:
        return sum(s.n_cart() for s in self._shells)

    def offsets(self):
        out, acc = [], 0
        for s in self._shells:
            out.append(acc)
            acc += s.n_func()
        return out

    def atoms(self):
        atoms = []
        for s in self._shells:
            if s._center not in atoms:
                atoms.append(s._center)
        return atoms

    def plan(self, engine: Engine = Engine.Auto) -> _Plan:
        if engine not in self._plans:
            self._plans[engine] = _Plan(self._shells, engine)
        return self._plans[engine]

    # --- dense ERIs (src/integrals.rs:664-754)
    def eri(self) -> np.ndarray:
        return self.eri_with(Engine.Auto)

    def eri_kernel(self, kernel: "EriKernel") -> np.ndarray:
        """Basis::eri_kernel (src/integrals.rs:773-820): the dense tensor of
        the given operator (Coulomb or long-range erf)."""
        p = self.plan(Engine.Auto)
        p.set_erf_omega(_omega_of(kernel))
        try:
            n = p.nao
            out = np.empty(n ** 4)
            _lib.check(_lib.lib().igpu_eri_dense(p.h, out.ctypes.data_as(c_double_p)))
        finally:
            p.set_erf_omega(0.0)
        return out

    def eri_block(self, i: int, j: int, k: int, l: int) -> np.ndarray:
        """Basis::eri_block (src/integrals.rs:600-619): the (ij|kl) block,
        row-major [n_i][n_j][n_k][n_l] over the shells' functions."""
        return self.eri_block_with(Engine.Auto, i, j, k, l)

    def eri_block_with(self, engine: Engine, i: int, j: int, k: int, l: int) -> np.ndarray:
        nsh = len(self._shells)
        if not all(0 <= x < nsh for x in (i, j, k, l)):
            raise IntegralError(-1, "invalid argument", "shell index out of range")
        p = self.plan(engine)
        out = np.empty(int(np.prod([self._shells[x].n_func() for x in (i, j, k, l)])))
        _lib.check(_lib.lib().igpu_eri_block(p.h, i, j, k, l, out.ctypes.data_as(c_double_p)))
        return out

    def eri_screened(self, tau: float):
        """Basis::eri_screened (src/integrals.rs:864-981): the dense tensor
        with canonical quartets of Q_ij*Q_kl < tau left zero, and its
        ScreeningStats."""
        return self.eri_screened_with(Engine.Auto, tau)

    def eri_screened_with(self, engine: Engine, tau: float):
        p = self.plan(engine)
        out = np.empty(p.nao ** 4)
        total, skipped = ctypes.c_uint64(), ctypes.c_uint64()
        _lib.check(_lib.lib().igpu_eri_screened(p.h, float(tau), out.ctypes.data_as(c_double_p),
                                                ctypes.byref(total), ctypes.byref(skipped)))
        return out, ScreeningStats(total.value, skipped.value, float(tau))

    def eri_with(self, engine: Engine) -> np.ndarray:
        p = self.plan(engine)
        n = p.nao
        out = np.empty(n ** 4)
        _lib.check(_lib.lib().igpu_eri_dense(p.h, out.ctypes.data_as(c_double_p)))
        return out

    def schwarz_bounds(self) -> np.ndarray:
        """Basis::schwarz_bounds (src/integrals.rs:835-862): nsh x nsh,
        row-major, evaluated on the device at plan creation."""
        return self.schwarz_bounds_with(Engine.Auto)

    def schwarz_bounds_with(self, engine: Engine) -> np.ndarray:
        p = self.plan(engine)
        q = np.empty(p.nsh * p.nsh)
        _lib.check(_lib.lib().igpu_schwarz(p.h, q.ctypes.data_as(c_double_p)))
        return q

    def eri_builder(self) -> "EriBuilder":
        """Basis::eri_builder (src/eri_builder.rs:575-577): EriBuilder::new(self)."""
        return EriBuilder(self)

    def direct_contractor(self) -> "DirectContractor":
        return DirectContractor(self)

    def direct_grad_contractor(self) -> "DirectGradContractor":
        return DirectGradContractor(self)

    def packed_eri_builder(self) -> "PackedEriBuilder":
        return PackedEriBuilder(self)

    # --- density fitting over this basis as the auxiliary basis (src/df.rs)
    def _aux_plan(self, engine: Engine) -> _Plan:
        p = self.plan(engine)
        p.attach_aux(self)
        return p

    def eri_2c(self) -> np.ndarray:
        """Basis::eri_2c (src/df.rs:49-51): the metric (P|Q), row-major
        naux x naux, exactly symmetric."""
        return self.eri_2c_with(Engine.Auto)

    def eri_2c_with(self, engine: Engine) -> np.ndarray:
        p = self._aux_plan(engine)
        out = np.empty(p.naux * p.naux)
        _lib.check(_lib.lib().igpu_eri_2c(p.h, out.ctypes.data_as(c_double_p)))
        return out

    def eri_2c_kernel(self, kernel: "EriKernel") -> np.ndarray:
        """Basis::eri_2c_kernel (src/df.rs:100-145)."""
        p = self._aux_plan(Engine.Auto)
        p.set_erf_omega(_omega_of(kernel))
        try:
            out = np.empty(p.naux * p.naux)
            _lib.check(_lib.lib().igpu_eri_2c(p.h, out.ctypes.data_as(c_double_p)))
        finally:
            p.set_erf_omega(0.0)
        return out

    def schwarz_aux_bounds(self) -> np.ndarray:
        """Basis::schwarz_aux_bounds (src/df.rs:250-286): one factor per shell."""
        return self.schwarz_aux_bounds_with(Engine.Auto)

    def schwarz_aux_bounds_with(self, engine: Engine) -> np.ndarray:
        p = self._aux_plan(engine)
        out = np.empty(p.naux_sh)
        _lib.check(_lib.lib().igpu_schwarz_aux(p.h, out.ctypes.data_as(c_double_p)))
        return out

    def eri_3c_block(self, aux: "Basis", ish: int, jsh: int, psh: int) -> np.ndarray:
        """Basis::eri_3c_block (src/df.rs:148-150): (ij|P) row-major
        [n_i, n_j, n_p], P fastest."""
        return self.eri_3c_block_with(Engine.Auto, aux, ish, jsh, psh)

    def eri_3c_block_with(self, engine: Engine, aux: "Basis", ish: int, jsh: int, psh: int,
                          kernel: "EriKernel" = None) -> np.ndarray:
        nsh, nash = len(self._shells), len(aux._shells)
        if not (0 <= ish < nsh and 0 <= jsh < nsh and 0 <= psh < nash):
            raise IntegralError(-1, "invalid argument", "shell index out of range")
        b = Eri3cBuilder(self, aux, engine)
        i, j = max(ish, jsh), min(ish, jsh)
        out = np.zeros(b.output_len())
        keep = np.zeros(nash, dtype=np.uint8)
        keep[psh] = 1
        b._run(np.array([i * (i + 1) // 2 + j], dtype=np.uint32), keep, out, kernel)
        n, naux = self.nao(), aux.nao()
        oi, oj, op = self.offsets()[ish], self.offsets()[jsh], aux.offsets()[psh]
        ni, nj, np_ = self._shells[ish].n_func(), self._shells[jsh].n_func(), aux._shells[psh].n_func()
        T = out.reshape(n, n, naux)
        return np.ascontiguousarray(T[oi:oi + ni, oj:oj + nj, op:op + np_]).reshape(-1)

    def eri_3c_block_kernel(self, aux: "Basis", ish: int, jsh: int, psh: int, kernel: "EriKernel") -> np.ndarray:
        """Basis::eri_3c_block_kernel (src/df.rs:201-246)."""
        return self.eri_3c_block_with(Engine.Auto, aux, ish, jsh, psh, kernel)

    def eri_3c_builder(self, aux: "Basis") -> "Eri3cBuilder":
        """Basis::eri_3c_builder (src/df.rs:288-290)."""
        return Eri3cBuilder(self, aux)


# ------------------------------------------------------------ EriBuilder

@dataclass
class BraPairFill:
    """One task of EriBuilder.partition: the canonical bra pair and the
    caller's output tensor it fills (rows owned by the pair)."""
    bra: tuple
    index: int
    out: np.ndarray


class EriBuilder:
    """Dense ERI assembly over canonical bra pairs (src/eri_builder.rs)."""

    def __init__(self, basis: Basis, engine: Engine = Engine.Auto):
        self._basis = basis
        self._plan = basis.plan(engine)
        self._pairs = self._plan.bra_pairs()
        self._omega = 0.0

    @classmethod
    def new(cls, basis):
        return cls(basis)

    @classmethod
    def with_engine(cls, basis, engine):
        return cls(basis, engine)

    def kernel(self, k: "EriKernel") -> "EriBuilder":
        """EriBuilder::kernel (src/eri_builder.rs:280-304): the operator the
        later fills evaluate; builder-style, returns self."""
        self._omega = _omega_of(k)
        return self

    def bra_pairs(self):
        return list(self._pairs)

    def output_len(self) -> int:
        return self._plan.nao ** 4

    def _run(self, idx, n, out):
        self._plan.set_erf_omega(self._omega)
        try:
            _lib.check(_lib.lib().igpu_eri_builder_fill(self._plan.h, idx, n, out.ctypes.data_as(c_double_p)))
        finally:
            self._plan.set_erf_omega(0.0)

    def partition(self, out: np.ndarray):
        if out.size != self.output_len():
            raise IntegralError(-7, "length mismatch", "ERI output buffer must be nao^4")
        return [BraPairFill(bra, k, out) for k, bra in enumerate(self._pairs)]

    def fill(self, task: BraPairFill):
        self.fill_many([task])

    def fill_many(self, tasks: Sequence[BraPairFill]):
        """Fill several tasks sharing one output buffer in one launch sequence."""
        if not tasks:
            return
        out = tasks[0].out
        if not out.flags["C_CONTIGUOUS"] or out.dtype != np.float64:
            raise IntegralError(-1, "invalid argument", "output must be contiguous float64")
        idx = np.ascontiguousarray([t.index for t in tasks], dtype=np.uint32)
        self._run(idx.ctypes.data_as(c_u32_p), len(idx), out)

    def build(self) -> np.ndarray:
        out = np.zeros(self.output_len())
        self._run(None, 0, out)
        return out


# ------------------------------------------------------ density fitting

@dataclass
class Bra3cFill:
    """One task of Eri3cBuilder.partition (src/df.rs:531-547): the canonical
    main bra pair (i, j) and the output buffer whose (i, j) and (j, i) row
    bands it fills."""
    bra: tuple
    index: int
    out: np.ndarray


class Eri3cBuilder:
    """The dense 3-centre tensor (mu nu|P), row-major [nao, nao, naux] with P
    fastest, over canonical main bra pairs (src/df.rs:325-520).  Each aux
    shell is evaluated with the unit s dummy (df.rs:33-38)."""

    def __init__(self, main: Basis, aux: Basis, engine: Engine = Engine.Auto):
        self._main, self._aux = main, aux
        self._plan = main.plan(engine)
        self._pairs = self._plan.bra_pairs()
        self._naux = aux.nao()

    @classmethod
    def new(cls, main: Basis, aux: Basis) -> "Eri3cBuilder":
        return cls(main, aux)

    @classmethod
    def with_engine(cls, main: Basis, aux: Basis, engine: Engine) -> "Eri3cBuilder":
        return cls(main, aux, engine)

    def bra_pairs(self):
        return list(self._pairs)

    def output_len(self) -> int:
        return self._plan.nao * self._plan.nao * self._naux

    def partition(self, out: np.ndarray):
        if out.size != self.output_len():
            raise IntegralError(-7, "length mismatch", "3c output buffer must be nao^2*naux = %d elements"
                                % self.output_len())
        return [Bra3cFill(bra, k, out) for k, bra in enumerate(self._pairs)]

    def _run(self, idx, keep, out, kernel=None):
        if not out.flags["C_CONTIGUOUS"] or out.dtype != np.float64 or out.size != self.output_len():
            raise IntegralError(-7, "length mismatch", "output must be contiguous float64 of nao^2*naux")
        p = self._plan
        p.attach_aux(self._aux)
        p.set_erf_omega(_omega_of(kernel))
        try:
            _lib.check(_lib.lib().igpu_eri_3c(
                p.h, idx.ctypes.data_as(c_u32_p) if idx is not None else None, 0 if idx is None else len(idx),
                keep.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if keep is not None else None,
                out.ctypes.data_as(c_double_p)))
        finally:
            p.set_erf_omega(0.0)

    def fill(self, task: Bra3cFill):
        """Eri3cBuilder::fill (src/df.rs:463-465)."""
        self.fill_many([task])

    def fill_filtered(self, task: Bra3cFill, keep):
        """Eri3cBuilder::fill_filtered (src/df.rs:475-513): only the aux
        shells p with keep(p) true; the others' slots are left untouched."""
        mask = np.array([1 if keep(p) else 0 for p in range(len(self._aux._shells))], dtype=np.uint8)
        self._run(np.array([task.index], dtype=np.uint32), mask, task.out)

    def fill_many(self, tasks: Sequence[Bra3cFill]):
        """Fill several tasks sharing one output buffer in one launch sequence."""
        if not tasks:
            return
        idx = np.ascontiguousarray([t.index for t in tasks], dtype=np.uint32)
        self._run(idx, None, tasks[0].out)

    def build(self) -> np.ndarray:
        """Eri3cBuilder::build (src/df.rs:516-522)."""
        out = np.zeros(self.output_len())
        self._run(None, None, out)
        return out


class PackedEriWorkspace:
    """Worker-local scratch of the reference (src/packed_eri.rs:36-50); the
    device plan keeps its own, kept for API parity."""


@dataclass
class PackedBraFill:
    """One task of PackedEriBuilder.partition: the canonical bra pair and its
    contiguous row range of the packed tensor (`rows`, a view of `out`)."""
    bra: int
    rows: np.ndarray
    out: np.ndarray


class PackedEriBuilder:
    """The symmetry-unique ERI tensor (src/packed_eri.rs): each canonical
    shell quartet evaluated once, stored as the lower triangle over AO-pair
    indices numbered shell-pair blocked (canonical shell pair (i >= j), then
    (a, b) row-major with b <= a when i == j); (t|u), u <= t, at
    t(t+1)/2 + u."""

    def __init__(self, basis: Basis, engine: Engine = Engine.Auto):
        self._plan = basis.plan(engine)
        sh = basis.shells()
        offs = basis.offsets()
        nsh = len(sh)
        self._pairs = [(i, j) for i in range(nsh) for j in range(i + 1)]
        self._ao_pairs = []
        self._start = []
        for i, j in self._pairs:
            self._start.append(len(self._ao_pairs))
            for a in range(sh[i].n_func()):
                for b in range(a + 1 if i == j else sh[j].n_func()):
                    self._ao_pairs.append((offs[i] + a, offs[j] + b))
        self._start.append(len(self._ao_pairs))

    @classmethod
    def new(cls, basis):
        return cls(basis)

    @classmethod
    def with_engine(cls, basis, engine):
        return cls(basis, engine)

    def bra_pairs(self):
        return list(self._pairs)

    def ao_pairs(self):
        return list(self._ao_pairs)

    def output_len(self) -> int:
        m = len(self._ao_pairs)
        return m * (m + 1) // 2

    def partition(self, out: np.ndarray):
        if out.size != self.output_len():
            raise IntegralError(-7, "length mismatch",
                                "packed ERI output buffer must hold %d elements" % self.output_len())
        tasks = []
        for bra in range(len(self._pairs)):
            lo, hi = self._start[bra], self._start[bra + 1]
            tasks.append(PackedBraFill(bra, out[lo * (lo + 1) // 2: hi * (hi + 1) // 2], out))
        return tasks

    def fill(self, workspace, task: PackedBraFill, threshold: float):
        self.fill_many([task], threshold)

    def fill_many(self, tasks: Sequence[PackedBraFill], threshold: float):
        """Fill several tasks of one output buffer in one launch sequence."""
        if not tasks:
            return
        out = tasks[0].out
        if not out.flags["C_CONTIGUOUS"] or out.dtype != np.float64:
            raise IntegralError(-1, "invalid argument", "output must be contiguous float64")
        idx = np.ascontiguousarray([t.bra for t in tasks], dtype=np.uint32)
        _lib.check(_lib.lib().igpu_eri_packed(self._plan.h, float(threshold), idx.ctypes.data_as(c_u32_p),
                                              len(idx), out.ctypes.data_as(c_double_p)))

    def build(self, threshold: float) -> np.ndarray:
        out = np.zeros(self.output_len())
        _lib.check(_lib.lib().igpu_eri_packed(self._plan.h, float(threshold), None, 0,
                                              out.ctypes.data_as(c_double_p)))
        return out


# ------------------------------------------------------------- direct J/K

class DirectWorkspace:
    """Worker-local state (src/direct.rs:19-33).  The device plan keeps its
    own scratch, so the workspace carries nothing; it exists for API parity."""


@dataclass
class DirectBuffers:
    coulomb: np.ndarray
    exchange: Optional[np.ndarray] = None


class DirectContractor:
    """Integral-direct J/K (src/direct.rs)."""

    def __init__(self, basis: Basis, engine: Engine = Engine.Auto):
        self._plan = basis.plan(engine)
        self._pairs = self._plan.bra_pairs()
        self._nsh = self._plan.nsh

    @classmethod
    def new(cls, basis):
        return cls(basis)

    @classmethod
    def with_engine(cls, basis, engine):
        return cls(basis, engine)

    def nao(self) -> int:
        return self._plan.nao

    def bra_pairs(self):
        return list(self._pairs)

    @property
    def plan(self) -> _Plan:
        return self._plan

    def density_shell_bounds(self, densities):
        D = _dens_array(densities, self._plan.nao)
        out = np.empty((D.shape[0], self._nsh * self._nsh))
        _lib.check(_lib.lib().igpu_density_shell_bounds(self._plan.h, D.ctypes.data_as(c_double_p),
                                                         D.shape[0], out.ctypes.data_as(c_double_p)))
        return [out[d] for d in range(D.shape[0])]

    def accumulate_bra_pair(self, workspace, bra, densities, density_bounds, threshold, want_exchange, outputs):
        """One canonical bra pair, as the reference (direct.rs:131-218)."""
        i, j = bra
        if j > i:
            raise IntegralError(-8, "non-canonical bra pair", "bra must satisfy i >= j")
        p = i * (i + 1) // 2 + j
        self.accumulate_bra_pairs(workspace, [p], densities, density_bounds, threshold, want_exchange, outputs)

    def accumulate_bra_pairs(self, workspace, bra_indices, densities, density_bounds, threshold, want_exchange,
                             outputs, precision: int = 0):
        """Many canonical bra pairs (indices into bra_pairs(), None = all) in
        one launch sequence.  outputs: list of DirectBuffers (accumulated)."""
        D = _dens_array(densities, self._plan.nao)
        nd = D.shape[0]
        if not (1 <= nd <= 64):
            raise IntegralError(-6, "density count", "1..64 densities")
        if len(outputs) != nd or (density_bounds is not None and len(density_bounds) != nd):
            raise IntegralError(-7, "length mismatch", "one output (and bound) per density")
        n2 = self._plan.nao ** 2
        J = np.zeros((nd, n2))
        K = np.zeros((nd, n2)) if want_exchange else None
        sub = None if bra_indices is None else np.ascontiguousarray(bra_indices, dtype=np.uint32)
        _lib.check(_lib.lib().igpu_jk(
            self._plan.h, D.ctypes.data_as(c_double_p), nd,
            sub.ctypes.data_as(c_u32_p) if sub is not None else None, 0 if sub is None else len(sub),
            float(threshold), int(bool(want_exchange)), int(precision), J.ctypes.data_as(c_double_p),
            K.ctypes.data_as(c_double_p) if K is not None else None))
        for d, o in enumerate(outputs):
            if o.coulomb.size != n2:
                raise IntegralError(-7, "length mismatch", "coulomb buffer must be nao^2")
            o.coulomb.reshape(-1)[:] += J[d]
            if want_exchange:
                if o.exchange is None or o.exchange.size != n2:
                    raise IntegralError(-7, "length mismatch", "exchange buffer required")
                o.exchange.reshape(-1)[:] += K[d]

    def jk(self, densities, threshold, want_exchange=True, precision: int = 0, bras=None):
        """Convenience: full J (and K) for the densities, host arrays."""
        D = _dens_array(densities, self._plan.nao)
        nd, n = D.shape[0], self._plan.nao
        outs = [DirectBuffers(np.zeros((n, n)), np.zeros((n, n)) if want_exchange else None) for _ in range(nd)]
        self.accumulate_bra_pairs(DirectWorkspace(), bras, D, None, threshold, want_exchange, outs, precision)
        J = np.array([o.coulomb for o in outs])
        K = np.array([o.exchange for o in outs]) if want_exchange else None
        return J, K

    def jk_device(self, d_dens, ndens, d_J, d_K, threshold, want_exchange=True, precision: int = 0,
                  bras=None, stream=None):
        """Device-resident D/J/K (raw device pointers, e.g. tensor.data_ptr())."""
        sub = None if bras is None else np.ascontiguousarray(bras, dtype=np.uint32)
        _lib.check(_lib.lib().igpu_jk_device(
            self._plan.h, ctypes.c_void_p(d_dens), ndens,
            sub.ctypes.data_as(c_u32_p) if sub is not None else None, 0 if sub is None else len(sub),
            float(threshold), int(bool(want_exchange)), int(precision), ctypes.c_void_p(d_J),
            ctypes.c_void_p(d_K if want_exchange else 0), ctypes.c_void_p(stream or 0)))

    def autotune_device(self, d_dens, ndens, threshold, precision: int = 1, stream=None):
        """Chunk autotuner (igpu_autotune_jk; no reference counterpart): times
        the J/K build of the device densities at candidate chunk sizes and
        keeps the fastest per angular class and precision for later calls."""
        _lib.check(_lib.lib().igpu_autotune_jk(self._plan.h, ctypes.c_void_p(d_dens), int(ndens), float(threshold),
                                               int(precision), ctypes.c_void_p(stream or 0)))

    def set_mixed_cutoff(self, cutoff: float):
        """MIXED precision: quartets with Q_bra*Q_ket*max|D| below `cutoff`
        (default 1e-3) run in FP32 (igpu_set_mixed_cutoff)."""
        _lib.check(_lib.lib().igpu_set_mixed_cutoff(self._plan.h, float(cutoff)))

    def mixed_cutoffs(self):
        """(cutoff, primitive eps) of MIXED precision (igpu_get_mixed_cutoffs)."""
        c, e = ctypes.c_double(), ctypes.c_double()
        _lib.check(_lib.lib().igpu_get_mixed_cutoffs(self._plan.h, ctypes.byref(c), ctypes.byref(e)))
        return c.value, e.value

    def set_mixed_prim_cutoff(self, eps: float):
        """MIXED precision: inside the FP32 quartets, skip primitive quartets
        whose magnitude bound times max|D| is below `eps`
        (igpu_set_mixed_prim_cutoff; 0 evaluates all of them)."""
        _lib.check(_lib.lib().igpu_set_mixed_prim_cutoff(self._plan.h, float(eps)))

    def jk_device_static(self, d_dens, ndens, d_J, d_K, threshold, want_exchange=True, stream=None):
        """FP64 J/K on device pointers that allocates no device memory
        (igpu_jk_device_static), for callers whose device memory belongs to
        their own pool allocator or that cannot afford cudaFree's implicit
        synchronisation.  Needs one earlier jk/jk_device call with the same
        threshold; adds into J and K; calls sharing a GPU must not overlap."""
        _lib.check(_lib.lib().igpu_jk_device_static(
            self._plan.h, ctypes.c_void_p(d_dens), ndens, float(threshold), int(bool(want_exchange)),
            ctypes.c_void_p(d_J), ctypes.c_void_p(d_K if want_exchange else 0), ctypes.c_void_p(stream or 0)))

    def last_stats(self) -> dict:
        return self._plan.stats()


def _dens_array(densities, nao):
    if isinstance(densities, np.ndarray):
        D = densities
    else:
        D = np.array([np.asarray(d, dtype=np.float64).reshape(-1) for d in densities])
    D = np.ascontiguousarray(D, dtype=np.float64).reshape(-1, nao * nao)
    return D


# ------------------------------------------------------------- gradient

@dataclass
class GradDensityTerm:
    factor: float
    left: np.ndarray
    right: np.ndarray


@dataclass
class GradDensity:
    coulomb: list
    exchange: list
    nao: int


class DirectGradWorkspace:
    """Worker-local state (src/direct_grad.rs:50-68); nothing to hold on the
    device side, kept for API parity."""


class DirectGradContractor:
    """Density-direct ERI nuclear gradient dE/dR (src/direct_grad.rs)."""

    def __init__(self, basis: Basis, engine: Engine = Engine.Auto):
        for s in basis.shells():
            if s.l() > MAX_GRAD_L:
                raise IntegralError(-5, "angular momentum too high for gradient",
                                    "l=%d exceeds %d" % (s.l(), MAX_GRAD_L))
        self._plan = basis.plan(engine)
        self._pairs = self._plan.bra_pairs()

    @classmethod
    def new(cls, basis):
        return cls(basis)

    @classmethod
    def with_engine(cls, basis, engine):
        return cls(basis, engine)

    def nao(self) -> int:
        return self._plan.nao

    def natom(self) -> int:
        return self._plan.natom

    def bra_pairs(self):
        return list(self._pairs)

    def set_mixed_cutoff(self, cutoff: float):
        """MIXED precision: quartets whose Schwarz product times the term
        matrices' maximum is below `cutoff` run in FP32 (igpu_set_mixed_cutoff)."""
        _lib.check(_lib.lib().igpu_set_mixed_cutoff(self._plan.h, float(cutoff)))

    def density(self, coulomb: Sequence[GradDensityTerm], exchange: Sequence[GradDensityTerm]) -> GradDensity:
        n2 = self._plan.nao ** 2
        for t in list(coulomb) + list(exchange):
            if np.asarray(t.left).size != n2 or np.asarray(t.right).size != n2:
                raise IntegralError(-7, "length mismatch", "density matrices must be nao x nao")
        return GradDensity(list(coulomb), list(exchange), self._plan.nao)

    def _terms(self, terms):
        arr = (IgpuTerm * max(1, len(terms)))()
        keep = []
        for k, t in enumerate(terms):
            l = np.ascontiguousarray(t.left, dtype=np.float64).reshape(-1)
            r = np.ascontiguousarray(t.right, dtype=np.float64).reshape(-1)
            keep += [l, r]
            arr[k].factor = float(t.factor)
            arr[k].left = l.ctypes.data_as(c_double_p)
            arr[k].right = r.ctypes.data_as(c_double_p)
        return arr, keep

    def autotune(self, density: GradDensity, threshold: float, precision: int = 1):
        """Chunk autotuner of the gradient launches (igpu_autotune_grad; no
        reference counterpart): ten gradient builds of `density`; later
        calls use the per-class chunks measured fastest."""
        ca, k1 = self._terms(density.coulomb)
        xa, k2 = self._terms(density.exchange)
        _lib.check(_lib.lib().igpu_autotune_grad(self._plan.h, ca, len(density.coulomb), xa, len(density.exchange),
                                                 float(threshold), int(precision)))

    def accumulate_bra_pairs(self, workspace, bra_indices, density: GradDensity, threshold: float, out: np.ndarray,
                             precision: int = 0, kernel: "EriKernel" = None):
        if density.nao != self._plan.nao:
            raise IntegralError(-1, "invalid argument", "density prepared for a different plan")
        if out.shape != (self._plan.natom, 3):
            raise IntegralError(-7, "length mismatch", "out must be natom x 3")
        ca, k1 = self._terms(density.coulomb)
        xa, k2 = self._terms(density.exchange)
        res = np.zeros(self._plan.natom * 3)
        sub = None if bra_indices is None else np.ascontiguousarray(bra_indices, dtype=np.uint32)
        self._plan.set_erf_omega(_omega_of(kernel))
        try:
            _lib.check(_lib.lib().igpu_grad(
                self._plan.h, ca, len(density.coulomb), xa, len(density.exchange),
                sub.ctypes.data_as(c_u32_p) if sub is not None else None, 0 if sub is None else len(sub),
                float(threshold), int(precision), res.ctypes.data_as(c_double_p)))
        finally:
            self._plan.set_erf_omega(0.0)
        out += res.reshape(-1, 3)

    def accumulate_bra_pair(self, workspace, bra, density, kernel, threshold, out):
        i, j = bra
        if j > i:
            raise IntegralError(-8, "non-canonical bra pair", "bra must satisfy i >= j")
        self.accumulate_bra_pairs(workspace, [i * (i + 1) // 2 + j], density, threshold, out, kernel=kernel)

    def contract(self, density: GradDensity, kernel=None, threshold: float = 0.0, precision: int = 0) -> np.ndarray:
        out = np.zeros((self._plan.natom, 3))
        self.accumulate_bra_pairs(DirectGradWorkspace(), None, density, threshold, out, precision, kernel=kernel)
        return out

    def last_stats(self) -> dict:
        return self._plan.stats()


def abi_version() -> int:
    return int(_lib.lib().igpu_abi_version())


class MoleculeBatch:
    """Many independent molecules of uneven size in one batch
    (igpu_batch_*).  No reference counterpart: the reference's callers loop
    over one DirectContractor / DirectGradContractor per molecule
    (src/direct.rs:19-21, src/direct_grad.rs:140-142).  One step runs, for
    every molecule, the J/K build of its density and (optionally) the
    density-direct gradient of the Coulomb term (coulomb_factor, D, D) and
    the exchange term (exchange_factor, D, D), each molecule screened and
    evaluated exactly as its own plan would; every angular class of every
    molecule runs in one persistent launch, and the step is a CUDA graph
    captured on first use and replayed afterwards."""

    def __init__(self, molecules: Sequence[Sequence[Shell]]):
        L = _lib.lib()
        mols = [[s if isinstance(s, Shell) else Shell.from_dict(s) for s in m] for m in molecules]
        flat = [s for m in mols for s in m]
        self._keep = []
        arr = _Plan._shell_array(flat, self._keep)
        counts = np.array([len(m) for m in mols], dtype=np.uintp)
        self._keep.append(counts)
        h = ctypes.c_void_p()
        _lib.check(L.igpu_batch_create(arr, counts.ctypes.data_as(_lib.c_size_p), len(mols), ctypes.byref(h)))
        self.h = h
        self._nao, self._natom = [], []
        for m in range(len(mols)):
            nao, natom, nsh = (ctypes.c_size_t() for _ in range(3))
            _lib.check(L.igpu_batch_query(h, m, ctypes.byref(nao), ctypes.byref(natom), ctypes.byref(nsh)))
            self._nao.append(nao.value)
            self._natom.append(natom.value)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                _lib.lib().igpu_batch_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def __len__(self) -> int:
        return len(self._nao)

    def nao(self, m: int) -> int:
        return self._nao[m]

    def natom(self, m: int) -> int:
        return self._natom[m]

    def set_mixed_cutoff(self, cutoff: float):
        _lib.check(_lib.lib().igpu_batch_set_mixed_cutoff(self.h, float(cutoff)))

    def jk_grad(self, densities, threshold: float, precision: int = 0, want_exchange: bool = True,
                gradient: bool = True, coulomb_factor: float = 0.5, exchange_factor: float = -0.25):
        """densities: one nao_m x nao_m matrix per molecule.  Returns lists of
        J, K (None without exchange) and gradients (natom_m x 3, None without
        gradient) per molecule."""
        if len(densities) != len(self._nao):
            raise IntegralError(-7, "length mismatch", "one density per molecule")
        for D, n in zip(densities, self._nao):
            if np.shape(D) != (n, n):
                raise IntegralError(-7, "length mismatch", "density of shape (%d, %d) expected" % (n, n))
        dens = np.ascontiguousarray(np.concatenate([np.asarray(D, dtype=np.float64).reshape(-1)
                                                    for D in densities]))
        J = np.zeros_like(dens)
        K = np.zeros_like(dens) if want_exchange else None
        G = np.zeros(3 * sum(self._natom)) if gradient else None
        st = IgpuStats()
        _lib.check(_lib.lib().igpu_batch_jk_grad(
            self.h, dens.ctypes.data_as(c_double_p), float(threshold), int(precision), int(bool(want_exchange)),
            int(bool(gradient)), float(coulomb_factor), float(exchange_factor), J.ctypes.data_as(c_double_p),
            K.ctypes.data_as(c_double_p) if K is not None else None,
            G.ctypes.data_as(c_double_p) if G is not None else None, ctypes.byref(st)))
        self._stats = {f: getattr(st, f) for f, _ in IgpuStats._fields_}
        out_j, out_k, out_g = [], [], []
        o = og = 0
        for n, na in zip(self._nao, self._natom):
            out_j.append(J[o:o + n * n].reshape(n, n))
            out_k.append(K[o:o + n * n].reshape(n, n) if K is not None else None)
            out_g.append(G[og:og + 3 * na].reshape(na, 3) if G is not None else None)
            o += n * n
            og += 3 * na
        return out_j, out_k, out_g

    def last_stats(self) -> dict:
        return dict(getattr(self, "_stats", {}))
