"""ctypes access to the CPU oracle (oracle/liboracle.so) — test infrastructure.

The oracle is the C++ restatement of the reference's two-electron path.  Only
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
use it, always as the checker, never as the thing measured or shipped.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int_p = ctypes.POINTER(ctypes.c_int)
c_u64_p = ctypes.POINTER(ctypes.c_uint64)


def _dp(a):
    return a.ctypes.data_as(c_double_p)


def _ip(a):
    return a.ctypes.data_as(c_int_p)


def build():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_basis_new.restype = ctypes.c_void_p
        L.orc_basis_new.argtypes = [ctypes.c_int, c_int_p, c_int_p, c_double_p, c_int_p, c_double_p, c_double_p]
        L.orc_basis_free.argtypes = [ctypes.c_void_p]
        L.orc_nao.argtypes = [ctypes.c_void_p]
        L.orc_natom.argtypes = [ctypes.c_void_p]
        L.orc_eri.argtypes = [ctypes.c_void_p, ctypes.c_int, c_double_p]
        L.orc_set_erf_omega.argtypes = [ctypes.c_double]
        L.orc_eri_block.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_int] * 4 + [c_double_p]
        L.orc_schwarz.argtypes = [ctypes.c_void_p, ctypes.c_int, c_double_p]
        L.orc_direct_new.restype = ctypes.c_void_p
        L.orc_direct_new.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_direct_free.argtypes = [ctypes.c_void_p]
        L.orc_direct_schwarz.argtypes = [ctypes.c_void_p, c_double_p]
        L.orc_density_bounds.argtypes = [ctypes.c_void_p, c_double_p, c_double_p]
        L.orc_direct_jk.argtypes = [ctypes.c_void_p, ctypes.c_int, c_double_p, ctypes.c_double, ctypes.c_int,
                                    c_int_p, ctypes.c_int, ctypes.c_int, c_double_p, c_double_p,
                                    c_u64_p, c_u64_p, ctypes.c_int]
        L.orc_jk_quartets.restype = ctypes.c_long
        L.orc_jk_quartets.argtypes = [ctypes.c_void_p, ctypes.c_int, c_double_p, ctypes.c_double, c_int_p,
                                      ctypes.c_int, c_int_p, c_u64_p, ctypes.c_long]
        L.orc_grad_new.restype = ctypes.c_void_p
        L.orc_grad_new.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_grad_free.argtypes = [ctypes.c_void_p]
        L.orc_direct_grad.argtypes = [ctypes.c_void_p, ctypes.c_int, c_double_p, c_double_p, c_double_p,
                                      ctypes.c_int, c_double_p, c_double_p, c_double_p, ctypes.c_double,
                                      c_int_p, ctypes.c_int, ctypes.c_int, c_double_p, c_u64_p, c_u64_p,
                                      ctypes.c_int]
        L.orc_eri_grad_contract.argtypes = [ctypes.c_void_p, c_double_p, c_double_p]
        L.orc_boys.argtypes = [ctypes.c_int, ctypes.c_double, c_double_p]
        L.orc_boys_reference.argtypes = [ctypes.c_int, ctypes.c_double, c_double_p]
        L.orc_rys.argtypes = [ctypes.c_int, ctypes.c_double, c_double_p, c_double_p]
        L.orc_rys_finite_reference.argtypes = [ctypes.c_int, ctypes.c_double, c_double_p, c_double_p]
        L.orc_rys_table_nsub.argtypes = [ctypes.c_int, c_double_p]
        L.orc_rys_table_copy.argtypes = [ctypes.c_int, ctypes.c_int, c_double_p, c_double_p]
        L.orc_c2s.argtypes = [ctypes.c_int, c_double_p]
        L.orc_cart_norm.restype = ctypes.c_double
        L.orc_cart_norm.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_select_engine.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_int_p]
        L.orc_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


ENGINES = {"auto": 0, "os": 1, "rys": 2}


class OracleBasis:
    """A basis held by the oracle.  ``shells`` is a list of dicts with keys
    l, spherical, center, exps, coefs (the integral_b200.systems layout)."""

    def __init__(self, shells):
        L = lib()
        self.shells = shells
        self.nsh = len(shells)
        ls = np.array([s["l"] for s in shells], dtype=np.int32)
        sph = np.array([1 if s.get("spherical") else 0 for s in shells], dtype=np.int32)
        cen = np.array([s["center"] for s in shells], dtype=np.float64).reshape(-1)
        npr = np.array([len(s["exps"]) for s in shells], dtype=np.int32)
        ex = np.concatenate([np.asarray(s["exps"], dtype=np.float64) for s in shells])
        co = np.concatenate([np.asarray(s["coefs"], dtype=np.float64) for s in shells])
        self._keep = (ls, sph, cen, npr, ex, co)
        self.h = L.orc_basis_new(self.nsh, _ip(ls), _ip(sph), _dp(cen), _ip(npr), _dp(ex), _dp(co))
        if not self.h:
            raise ValueError(L.orc_last_error().decode())
        self.nao = L.orc_nao(self.h)
        self.natom = L.orc_natom(self.h)
        self._direct = {}
        self._grad = {}

    def __del__(self):
        try:
            L = lib()
            for p in self._direct.values():
                L.orc_direct_free(p)
            for g in self._grad.values():
                L.orc_grad_free(g)
            if self.h:
                L.orc_basis_free(self.h)
        except Exception:
            pass

    def eri_erf(self, omega):
        """Dense tensor of erf(omega r)/r (Basis::eri_kernel,
        src/integrals.rs:773-820): Rys for every quartet."""
        with erf(omega):
            return self.eri("rys")

    def eri(self, engine="auto"):
        n = self.nao
        out = np.zeros(n ** 4)
        lib().orc_eri(self.h, ENGINES[engine], _dp(out))
        return out

    def eri_screened(self, tau, engine="auto"):
        """Basis::eri_screened_with (src/integrals.rs:880-981): the dense
        tensor with every canonical quartet of Q_ij*Q_kl < tau left zero in
        all its permutation slots; returns (tensor, total, skipped) over the
        canonical quartets.  The bound is permutation-invariant, so the mask
        is taken over all ordered shell quartets."""
        E = self.eri(engine)
        Q = self.schwarz(engine)
        n = self.nsh
        K = self.screened_mask(tau, engine)
        pairs = [(i, j) for i in range(n) for j in range(i + 1)]
        total = skipped = 0
        for p, (i, j) in enumerate(pairs):
            for (k, l) in pairs[:p + 1]:
                total += 1
                if Q[i, j] * Q[k, l] < tau:
                    skipped += 1
        return np.where(K.reshape(-1), E, 0.0), total, skipped

    def screened_mask(self, tau, engine="auto"):
        """nao^4 boolean mask of the elements whose shell quartet passes
        Q_ij*Q_kl >= tau (src/integrals.rs:905-909)."""
        Q = self.schwarz(engine)
        keep = np.multiply.outer(Q, Q) >= tau  # [i, j, k, l]
        nf = [(2 * s["l"] + 1) if s.get("spherical") else (s["l"] + 1) * (s["l"] + 2) // 2 for s in self.shells]
        owner = np.repeat(np.arange(self.nsh), nf)
        return keep[np.ix_(owner, owner, owner, owner)]

    def eri_block(self, i, j, k, l, engine="auto"):
        nf = [(2 * s["l"] + 1) if s.get("spherical") else (s["l"] + 1) * (s["l"] + 2) // 2
              for s in (self.shells[i], self.shells[j], self.shells[k], self.shells[l])]
        out = np.zeros(int(np.prod(nf)))
        lib().orc_eri_block(self.h, ENGINES[engine], i, j, k, l, _dp(out))
        return out.reshape(nf)

    def schwarz(self, engine="auto"):
        q = np.zeros(self.nsh * self.nsh)
        lib().orc_schwarz(self.h, ENGINES[engine], _dp(q))
        return q.reshape(self.nsh, self.nsh)

    def _dplan(self, engine):
        if engine not in self._direct:
            self._direct[engine] = lib().orc_direct_new(self.h, ENGINES[engine])
        return self._direct[engine]

    def _gplan(self, engine):
        if engine not in self._grad:
            g = lib().orc_grad_new(self.h, ENGINES[engine])
            if not g:
                raise ValueError(lib().orc_last_error().decode())
            self._grad[engine] = g
        return self._grad[engine]

    def direct_jk(self, dens, threshold, want_k=True, bras=None, nthreads=1, engine="auto",
                  count_only=False):
        """J/K (ndens, nao, nao) over canonical bra-pair indices ``bras``
        (None = all), plus the screened-quartet count and fingerprint."""
        D = np.ascontiguousarray(np.asarray(dens, dtype=np.float64).reshape(-1, self.nao, self.nao))
        nd = D.shape[0]
        J = np.zeros_like(D)
        K = np.zeros_like(D)
        cnt = ctypes.c_uint64()
        hsh = ctypes.c_uint64()
        b = None if bras is None else np.ascontiguousarray(bras, dtype=np.int32)
        rc = lib().orc_direct_jk(self._dplan(engine), nd, _dp(D), threshold, int(want_k),
                                 _ip(b) if b is not None else None, -1 if b is None else len(b),
                                 nthreads, _dp(J), _dp(K), ctypes.byref(cnt), ctypes.byref(hsh),
                                 int(count_only))
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return J, K, cnt.value, hsh.value

    def jk_quartets(self, dens, threshold, bras=None, cap=10_000_000):
        D = np.ascontiguousarray(np.asarray(dens, dtype=np.float64).reshape(-1, self.nao, self.nao))
        b = None if bras is None else np.ascontiguousarray(bras, dtype=np.int32)
        out = np.zeros((cap, 4), dtype=np.int32)
        masks = np.zeros(cap, dtype=np.uint64)
        n = lib().orc_jk_quartets(self._dplan("auto"), D.shape[0], _dp(D), threshold,
                                  _ip(b) if b is not None else None, -1 if b is None else len(b),
                                  _ip(out), masks.ctypes.data_as(c_u64_p), cap)
        n = min(n, cap)
        return out[:n], masks[:n]

    def direct_schwarz(self):
        q = np.zeros(self.nsh * self.nsh)
        lib().orc_direct_schwarz(self._dplan("auto"), _dp(q))
        return q.reshape(self.nsh, self.nsh)

    def direct_grad(self, coulomb, exchange, threshold, bras=None, nthreads=1, engine="auto",
                    count_only=False):
        """coulomb / exchange: lists of (factor, left, right)."""
        n2 = self.nao * self.nao

        def pack(terms):
            f = np.array([t[0] for t in terms], dtype=np.float64)
            lft = np.ascontiguousarray(np.array([np.asarray(t[1]).reshape(n2) for t in terms]).reshape(-1)) \
                if terms else np.zeros(1)
            rgt = np.ascontiguousarray(np.array([np.asarray(t[2]).reshape(n2) for t in terms]).reshape(-1)) \
                if terms else np.zeros(1)
            return f if len(f) else np.zeros(1), lft, rgt

        cf, cl, cr = pack(coulomb)
        xf, xl, xr = pack(exchange)
        out = np.zeros(self.natom * 3)
        cnt = ctypes.c_uint64()
        hsh = ctypes.c_uint64()
        b = None if bras is None else np.ascontiguousarray(bras, dtype=np.int32)
        rc = lib().orc_direct_grad(self._gplan(engine), len(coulomb), _dp(cf), _dp(cl), _dp(cr),
                                   len(exchange), _dp(xf), _dp(xl), _dp(xr), threshold,
                                   _ip(b) if b is not None else None, -1 if b is None else len(b),
                                   nthreads, _dp(out), ctypes.byref(cnt), ctypes.byref(hsh),
                                   int(count_only))
        if rc != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return out.reshape(self.natom, 3), cnt.value, hsh.value

    def eri_grad_contract(self, gamma, engine="auto"):
        """Basis::eri_grad_contract_with (src/grad.rs:427-470): the gradient of
        sum gamma[p,q,r,s] (pq|rs) over all ordered quartets; gamma nao^4."""
        g = np.ascontiguousarray(gamma, dtype=np.float64).reshape(-1)
        if g.size != self.nao ** 4:
            raise ValueError("gamma must have nao^4 elements")
        out = np.zeros(self.natom * 3)
        if lib().orc_eri_grad_contract(self._gplan(engine), _dp(g), _dp(out)) != 0:
            raise RuntimeError(lib().orc_last_error().decode())
        return out.reshape(self.natom, 3)


class erf:
    """Context: the oracle's Rys evaluations use erf(omega r)/r inside."""

    def __init__(self, omega):
        self.omega = float(omega)

    def __enter__(self):
        lib().orc_set_erf_omega(self.omega)
        return self

    def __exit__(self, *exc):
        lib().orc_set_erf_omega(0.0)
        return False


def boys(m, t, reference=False):
    out = np.zeros(m + 1)
    (lib().orc_boys_reference if reference else lib().orc_boys)(m, t, _dp(out))
    return out


def rys(n, t, finite_reference=False):
    r = np.zeros(n)
    w = np.zeros(n)
    (lib().orc_rys_finite_reference if finite_reference else lib().orc_rys)(n, t, _dp(r), _dp(w))
    return r, w


def rys_table(n, regenerated=True):
    worst = ctypes.c_double()
    nsub = lib().orc_rys_table_nsub(n, ctypes.byref(worst))
    if not regenerated and lib().orc_rys_tables_are_reference_literals():
        nsub = None
    r = np.zeros(16 * 15 * 17 * 2)
    w = np.zeros(16 * 15 * 17 * 2)
    lib().orc_rys_table_copy(n, int(regenerated), _dp(r), _dp(w))
    if nsub is None:
        nz = np.nonzero(r)[0]
        nsub = (nz[-1] // 17 + 1) // n if len(nz) else 0
    m = nsub * n * 17
    return nsub, worst.value, r[:m].reshape(nsub * n, 17), w[:m].reshape(nsub * n, 17)


def c2s(l):
    out = np.zeros((2 * l + 1) * (l + 1) * (l + 2) // 2)
    lib().orc_c2s(l, _dp(out))
    return out.reshape(2 * l + 1, (l + 1) * (l + 2) // 2)


def cart_norm(a, lx, ly, lz):
    return lib().orc_cart_norm(a, lx, ly, lz)


def select_engine(ne, nf, deg):
    o = ctypes.c_int()
    lib().orc_select_engine(ne, nf, deg, ctypes.byref(o))
    return ["auto", "os", "rys"][o.value]


# ------------------------------------------------------- density fitting

def _nf(s):
    return (2 * s["l"] + 1) if s.get("spherical") else (s["l"] + 1) * (s["l"] + 2) // 2


def _offsets(shells):
    out, acc = [], 0
    for s in shells:
        out.append(acc)
        acc += _nf(s)
    return out, acc


def unit_s(center):
    """The unit s dummy of src/df.rs:33-38: one zero-exponent primitive of
    coefficient 1 (exempt from normalisation, src/shell.rs:182-187), the
    constant function 1."""
    return dict(l=0, spherical=False, center=list(center), exps=[0.0], coefs=[1.0])


def df_eri_3c(main, aux, engine="auto", keep=None):
    """Eri3cBuilder::build / fill_filtered (src/df.rs:463-522): for every
    canonical main pair (i >= j) and aux shell p (with keep[p]), the block
    (ij|p 1s) into the (i, j) band and, for i != j, the (j, i) band of the
    row-major [nao, nao, naux] tensor, P fastest."""
    nm, na = len(main), len(aux)
    B = OracleBasis(list(main) + list(aux) + [unit_s(s["center"]) for s in aux])
    mo, nao = _offsets(main)
    ao, naux = _offsets(aux)
    out = np.zeros((nao, nao, naux))
    for i in range(nm):
        for j in range(i + 1):
            ni, nj = _nf(main[i]), _nf(main[j])
            for p in range(na):
                if keep is not None and not keep[p]:
                    continue
                blk = B.eri_block(i, j, nm + p, nm + na + p, engine)[..., 0]
                sl = slice(ao[p], ao[p] + _nf(aux[p]))
                out[mo[i]:mo[i] + ni, mo[j]:mo[j] + nj, sl] = blk
                if i != j:
                    out[mo[j]:mo[j] + nj, mo[i]:mo[i] + ni, sl] = blk.transpose(1, 0, 2)
    return out.reshape(-1)


def df_eri_3c_block(main, aux, ish, jsh, psh, engine="auto"):
    """Basis::eri_3c_block_with (src/df.rs:155-185): (ij|p 1s), [n_i, n_j, n_p]."""
    nm = len(main)
    B = OracleBasis(list(main) + [aux[psh], unit_s(aux[psh]["center"])])
    return B.eri_block(ish, jsh, nm, nm + 1, engine)[..., 0].reshape(-1)


def df_eri_2c(aux, engine="auto"):
    """Basis::eri_2c_with (src/df.rs:56-93): (p 1s|q 1s) for q <= p, written
    to both orientations in the reference's element order, so a diagonal
    shell block takes its lower-triangle values on both sides."""
    na = len(aux)
    B = OracleBasis(list(aux) + [unit_s(s["center"]) for s in aux])
    ao, naux = _offsets(aux)
    out = np.zeros((naux, naux))
    for p in range(na):
        for q in range(p + 1):
            blk = B.eri_block(p, na + p, q, na + q, engine)[:, 0, :, 0]
            for a in range(blk.shape[0]):
                for b in range(blk.shape[1]):
                    out[ao[p] + a, ao[q] + b] = blk[a, b]
                    out[ao[q] + b, ao[p] + a] = blk[a, b]
    return out.reshape(-1)


def df_schwarz_aux(aux, engine="auto"):
    """Basis::schwarz_aux_bounds_with (src/df.rs:257-286): sqrt of the
    largest diagonal element of the (p 1s|p 1s) block, per aux shell."""
    na = len(aux)
    B = OracleBasis(list(aux) + [unit_s(s["center"]) for s in aux])
    out = np.zeros(na)
    for p in range(na):
        blk = B.eri_block(p, na + p, p, na + p, engine)[:, 0, :, 0]
        out[p] = np.sqrt(np.max(np.abs(np.diag(blk))))
    return out
