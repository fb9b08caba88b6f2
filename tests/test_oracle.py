"""CPU checks of the oracle (the C++ restatement of the reference path)
against the reference's own known answers and golden fixtures.

Mirrors the reference's unit tests: src/math/boys.rs:432-684,
src/math/rys.rs:574-781, tests/c2s_independent_reference.rs,
src/math/norm.rs:95-145, tests/two_electron.rs, tests/screening.rs,
tests/direct_contractor.rs and tests/direct_grad_contractor.rs.
"""
import json
import math
import os

import numpy as np
import pytest

import oracle_py as O
from integral_b200 import systems as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# ---------------------------------------------------------------- Boys

def test_boys_known_value():
    # boys.rs:517-520
    assert abs(O.boys(0, 1.0)[0] - 0.7468241328124271) < 1e-14


def test_boys_at_zero_is_inverse_odd():
    # boys.rs:468-483
    f = O.boys(24, 0.0)
    for m in range(25):
        assert abs(f[m] - 1.0 / (2 * m + 1)) < 1e-15


def test_boys_table_matches_reference_path():
    # boys.rs:485-514: the Taylor table reproduces the series/asymptotic path
    worst = 0.0
    for t in np.arange(0.0, 95.0, 0.037):
        for m in (0, 1, 4, 8, 12, 16, 20, 24):
            a = O.boys(m, float(t))
            b = O.boys(m, float(t), reference=True)
            worst = max(worst, float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))))
    assert worst < 1e-12, worst


def test_boys_downward_recurrence():
    for t in (0.3, 2.5, 17.0, 60.0):
        f = O.boys(10, t)
        for m in range(1, 11):
            assert abs(f[m - 1] - (2 * t * f[m] + math.exp(-t)) / (2 * m - 1)) <= 1e-13 * f[m - 1]


# ------------------------------------------------------------------ Rys

@pytest.mark.parametrize("n", list(range(1, 14)))
def test_rys_moments_and_shape(n):
    # rys.rs:578-626: sum w x^k = F_k(T), roots in (0,1) ascending, w > 0
    for t in (0.0, 1e-4, 0.5, 2.0, 7.0, 20.0, 45.0, 80.0, 150.0, 1000.0):
        r, w = O.rys(n, t)
        fm = O.boys(2 * n - 1, t, reference=True)
        for k in range(2 * n):
            q = float(np.sum(w * r ** k))
            assert abs(q - fm[k]) <= 1e-9 * abs(fm[k]) + 1e-300, (n, t, k)
        assert np.all(r > 0) and np.all(r < 1) and np.all(w > 0)
        assert np.all(np.diff(r) > 0)


def test_one_point_quadrature_is_mean_and_mass():
    # rys.rs:648-660
    for t in (0.0, 0.7, 5.0, 30.0):
        r, w = O.rys(1, t)
        f = O.boys(1, t, reference=True)
        assert abs(r[0] - f[1] / f[0]) < 1e-14 and abs(w[0] - f[0]) < 1e-14


def test_rys_table_generator_reproduces_reference_tables():
    """The restated generator (xtask/src/gen_rys_tables.rs) picks the same
    subdivision as the reference's committed tables and agrees with their
    coefficients to the f64 rounding of the generating eigen-solve."""
    gold = json.load(open(os.path.join(GOLDEN, "rys_tables.json")))["tables"]
    worst = 0.0
    for n in range(1, 14):
        nsub, _, rc, wc = O.rys_table(n, regenerated=True)
        g = gold[str(n)]
        assert nsub == g["n_sub"]
        for mine, ref in ((rc[0], g["root_first"]), (rc[-1], g["root_last"]),
                          (wc[0], g["weight_first"]), (wc[-1], g["weight_last"])):
            worst = max(worst, float(np.max(np.abs(np.asarray(mine) - np.asarray(ref)))))
    assert worst < 5e-15, worst


def test_runtime_tables_are_reference_literals_when_built_with_them():
    import hashlib
    import struct
    if not O.lib().orc_rys_tables_are_reference_literals():
        pytest.skip("oracle built without the extracted reference tables")
    gold = json.load(open(os.path.join(GOLDEN, "rys_tables.json")))["tables"]
    for n in range(1, 14):
        nsub, _, rc, wc = O.rys_table(n, regenerated=False)
        for arr, key in ((rc, "root_sha256"), (wc, "weight_sha256")):
            flat = [float(v) for v in np.asarray(arr).reshape(-1)]
            assert hashlib.sha256(struct.pack("<%dd" % len(flat), *flat)).hexdigest() == gold[str(n)][key]


# --------------------------------------------------------- c2s, norms, AM

def test_c2s_matches_signed_mpmath_reference():
    rows = json.load(open(os.path.join(GOLDEN, "c2s_signed.json")))["rows"]
    for l in range(5):
        m = O.c2s(l)
        ref = np.array(rows[str(l)])
        assert m.shape == ref.shape
        assert float(np.max(np.abs(m - ref))) < 1e-12


def test_normalized_primitive_has_unit_self_overlap():
    # norm.rs:95-145
    def df(n):
        a = 1.0
        while n > 1:
            a *= n
            n -= 2
        return a
    for alpha in (0.1, 0.8, 3.3, 25.0, 1e5):
        for lx, ly, lz in ((0, 0, 0), (1, 0, 0), (0, 1, 1), (2, 0, 0), (1, 1, 1), (3, 2, 1)):
            n = O.cart_norm(alpha, lx, ly, lz)
            L = lx + ly + lz
            raw = df(2 * lx - 1) * df(2 * ly - 1) * df(2 * lz - 1) / (4 * alpha) ** L * (math.pi / (2 * alpha)) ** 1.5
            assert abs(n * n * raw - 1.0) < 1e-12


def test_select_engine_bands():
    # integrals.rs:374-388 and tests/dispatch.rs
    assert O.select_engine(2, 3, 1) == "os"
    assert O.select_engine(3, 3, 2) == "rys"
    assert O.select_engine(3, 3, 3) == "os"
    assert O.select_engine(8, 2, 15) == "rys"
    assert O.select_engine(8, 2, 16) == "os"
    assert O.select_engine(9, 8, 10000) == "rys"


# ------------------------------------------------------------------ ERIs

@pytest.fixture(scope="module", params=[False, True], ids=["cart", "sph"])
def fixture_basis(request):
    shells = S.direct_contractor_fixture(request.param)
    return O.OracleBasis(shells)


def test_os_and_rys_agree(fixture_basis):
    # tests/cross_engine.rs: the two engines agree to 1e-11
    a = fixture_basis.eri("os")
    b = fixture_basis.eri("rys")
    peak = float(np.max(np.abs(a)))
    assert float(np.max(np.abs(a - b))) < 1e-11 * max(peak, 1.0)


def test_eightfold_symmetry(fixture_basis):
    n = fixture_basis.nao
    T = fixture_basis.eri().reshape(n, n, n, n)
    for perm in ((1, 0, 2, 3), (0, 1, 3, 2), (2, 3, 0, 1), (3, 2, 1, 0)):
        assert float(np.max(np.abs(T - T.transpose(perm)))) < 1e-13


def test_schwarz_bounds_every_element(fixture_basis):
    # tests/screening.rs: |(mu nu|la si)| <= Q_ij Q_kl
    shells = fixture_basis.shells
    q = fixture_basis.schwarz()
    n = len(shells)
    for i in range(n):
        for j in range(n):
            for k in range(n):
                for l in range(n):
                    blk = fixture_basis.eri_block(i, j, k, l)
                    assert float(np.max(np.abs(blk))) <= q[i, j] * q[k, l] * (1 + 1e-12) + 1e-300


def test_direct_jk_matches_dense_contraction(fixture_basis):
    # tests/direct_contractor.rs: threshold 0, two densities, max |dJK| < 1e-9
    n = fixture_basis.nao
    D = S.direct_contractor_densities(n)
    for engine in ("os", "rys"):
        J, K, _, _ = fixture_basis.direct_jk(D, 0.0, engine=engine)
        E = fixture_basis.eri(engine).reshape(n, n, n, n)
        for d in range(2):
            Jr = np.einsum("abcd,cd->ab", E, D[d])
            Kr = np.einsum("abcd,bd->ac", E, D[d])
            assert float(np.max(np.abs(J[d] - Jr))) < 1e-9
            assert float(np.max(np.abs(K[d] - Kr))) < 1e-9


def test_direct_jk_threads_match_serial():
    sh = S.jk_system(natom=6, side=7.0)
    B = O.OracleBasis(sh["shells"])
    J1, K1, c1, h1 = B.direct_jk(sh["dens"], 1e-12, nthreads=1)
    J4, K4, c4, h4 = B.direct_jk(sh["dens"], 1e-12, nthreads=4)
    assert (c1, h1) == (c4, h4)
    # only the summation order of the per-worker buffers differs
    assert float(np.max(np.abs(J1 - J4))) < 1e-13 * float(np.max(np.abs(J1)))
    assert float(np.max(np.abs(K1 - K4))) < 1e-13 * float(np.max(np.abs(K1)))


# -------------------------------------------------------------- gradient

def _dense_energy(basis, coulomb, exchange):
    n = basis.nao
    E = basis.eri().reshape(n, n, n, n)
    e = 0.0
    for f, L, R in coulomb:
        e += f * np.einsum("pq,pqrs,rs->", L, E, R)
    for f, L, R in exchange:
        e += f * np.einsum("pr,pqrs,qs->", L, E, R)
    return e


@pytest.mark.parametrize("spherical", [False, True])
def test_direct_gradient_matches_finite_difference(spherical):
    # tests/direct_grad_contractor.rs: central FD at h = 2e-4, tolerance 1e-6
    shells = S.direct_grad_fixture(spherical)
    B = O.OracleBasis(shells)
    n = B.nao
    coul, exch = S.grad_fixture_terms(n)
    g, _, _ = B.direct_grad(coul, exch, 0.0)
    # zero net force
    assert float(np.max(np.abs(g.sum(axis=0)))) < 1e-10
    h = 2e-4
    atoms = []
    for s in shells:
        if s["center"] not in atoms:
            atoms.append(s["center"])
    for a in range(len(atoms)):
        for x in range(3):
            vals = []
            for sgn in (+1, -1):
                moved = []
                for s in shells:
                    c = list(s["center"])
                    if s["center"] == atoms[a]:
                        c[x] += sgn * h
                    moved.append(dict(s, center=c))
                vals.append(_dense_energy(O.OracleBasis(moved), coul, exch))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(fd - g[a, x]) < 1e-6, (a, x, fd, g[a, x])


def test_gradient_single_atom_is_zero():
    shells = [dict(s, center=[0.1, -0.2, 0.3]) for s in S.direct_grad_fixture(False)]
    B = O.OracleBasis(shells)
    coul, exch = S.grad_fixture_terms(B.nao)
    g, cnt, _ = B.direct_grad(coul, exch, 0.0)
    assert cnt == 0 and float(np.max(np.abs(g))) == 0.0


# ------------------------------------------------------ erf attenuation

def test_erf_ss_quartet_is_the_attenuated_boys_formula():
    """(ss|ss) of erf(omega r)/r for single primitives equals
    2 pi^(5/2)/(p q sqrt(p+q)) K_ab K_cd sqrt(s) F_0(s T), s = omega^2/(rho+omega^2)
    (the root/weight transform of crates/integral/src/engine/rys.rs:163-175)."""
    A, Bc, C, D = [0.0, 0.0, 0.0], [0.3, -0.2, 0.5], [1.1, 0.4, -0.6], [0.9, 1.2, 0.1]
    ex = [1.3, 0.7, 0.9, 0.45]
    shells = [dict(l=0, spherical=False, center=c, exps=[e], coefs=[1.0]) for c, e in zip((A, Bc, C, D), ex)]
    OB = O.OracleBasis(shells)
    omega = 0.4
    with O.erf(omega):
        got = OB.eri_block(0, 1, 2, 3, "rys").reshape(-1)[0]
    a, b, c, d = ex
    p, q = a + b, c + d
    P = (a * np.array(A) + b * np.array(Bc)) / p
    Q = (c * np.array(C) + d * np.array(D)) / q
    kab = np.exp(-a * b / p * np.sum((np.array(A) - np.array(Bc)) ** 2))
    kcd = np.exp(-c * d / q * np.sum((np.array(C) - np.array(D)) ** 2))
    rho = p * q / (p + q)
    T = rho * np.sum((P - Q) ** 2)
    s = omega ** 2 / (rho + omega ** 2)
    norm = np.prod([(2 * e / np.pi) ** 0.75 for e in ex])
    want = 2 * np.pi ** 2.5 / (p * q * np.sqrt(p + q)) * kab * kcd * np.sqrt(s) * O.boys(0, s * T)[0] * norm
    assert abs(got - want) < 1e-13 * abs(want)


def test_erf_at_large_omega_is_coulomb():
    shells = S.direct_contractor_fixture(False)
    OB = O.OracleBasis(shells)
    coul = OB.eri("rys")
    att = OB.eri_erf(1e9)
    assert float(np.max(np.abs(att - coul))) < 1e-12 * float(np.max(np.abs(coul)))
    # and smaller omega attenuates: |erf| < |Coulomb| on the diagonal
    att2 = OB.eri_erf(0.3)
    n = OB.nao
    dc, da = coul.reshape(n, n, n, n), att2.reshape(n, n, n, n)
    diag_c = np.array([dc[i, j, i, j] for i in range(n) for j in range(n)])
    diag_a = np.array([da[i, j, i, j] for i in range(n) for j in range(n)])
    assert np.all(diag_a < diag_c)


def test_erf_gradient_matches_finite_difference():
    # tests/erf_gradients.rs:132-146: the attenuated gradient against central
    # differences of the attenuated energy, omega in {0.3, 1.0}
    shells = S.direct_grad_fixture(False)
    B = O.OracleBasis(shells)
    n = B.nao
    coul, exch = S.grad_fixture_terms(n)
    atoms = []
    for s in shells:
        if s["center"] not in atoms:
            atoms.append(s["center"])
    h = 2e-4
    for omega in (0.3, 1.0):
        with O.erf(omega):
            g, _, _ = B.direct_grad(coul, exch, 0.0, engine="rys")
        g0, _, _ = B.direct_grad(coul, exch, 0.0, engine="rys")
        assert float(np.max(np.abs(g - g0))) > 1e-3 * float(np.max(np.abs(g0)))
        assert float(np.max(np.abs(g.sum(axis=0)))) < 1e-10
        for a, x in ((0, 0), (1, 2), (2, 1)):
            vals = []
            for sgn in (+1, -1):
                moved = [dict(s, center=[c + (sgn * h if (s["center"] == atoms[a] and k == x) else 0.0)
                                         for k, c in enumerate(s["center"])]) for s in shells]
                E = O.OracleBasis(moved).eri_erf(omega).reshape(n, n, n, n)
                e = sum(f * np.einsum("pq,pqrs,rs->", L, E, R) for f, L, R in coul)
                e += sum(f * np.einsum("pr,pqrs,qs->", L, E, R) for f, L, R in exch)
                vals.append(e)
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(fd - g[a, x]) < 1e-6, (omega, a, x, fd, g[a, x])


# ------------------------------------------------------ density fitting
# The oracle's restatement of src/df.rs pinned by the reference's own
# tests/df.rs: closed forms, the zero-exponent limit, cross-engine agreement,
# positive definiteness and the aux Schwarz bound.

def _s_norm(a):
    return (2.0 * a / np.pi) ** 0.75


def _close(a, b, tol):
    assert abs(a - b) / max(abs(b), 1.0) < tol, (a, b)


def test_df_2c_concentric_s_closed_form():
    # tests/df.rs:53-68
    a, b = 0.9, 1.7
    aux = [dict(l=0, spherical=False, center=[0.0] * 3, exps=[a], coefs=[1.0]),
           dict(l=0, spherical=False, center=[0.0] * 3, exps=[b], coefs=[1.0])]
    m = O.df_eri_2c(aux)
    pref = lambda x, y: 2.0 * np.pi ** 2.5 / (x * y * np.sqrt(x + y))
    _close(m[1], _s_norm(a) * _s_norm(b) * pref(a, b), 1e-12)
    _close(m[0], _s_norm(a) ** 2 * pref(a, a), 1e-12)
    _close(m[3], _s_norm(b) ** 2 * pref(b, b), 1e-12)
    assert m[1] == m[2]


def test_df_3c_concentric_s_closed_form():
    # tests/df.rs:70-91
    a, b, c = 0.8, 1.1, 0.6
    main = [dict(l=0, spherical=False, center=[0.0] * 3, exps=[a], coefs=[1.0]),
            dict(l=0, spherical=False, center=[0.0] * 3, exps=[b], coefs=[1.0])]
    aux = [dict(l=0, spherical=False, center=[0.0] * 3, exps=[c], coefs=[1.0])]
    blk = O.df_eri_3c_block(main, aux, 0, 1, 0)
    p = a + b
    want = _s_norm(a) * _s_norm(b) * _s_norm(c) * 2.0 * np.pi ** 2.5 / (p * c * np.sqrt(p + c))
    assert blk.size == 1
    _close(blk[0], want, 1e-12)


def test_df_3c_matches_tiny_exponent_four_centre_limit():
    # tests/df.rs:93-123: the dummy against an explicit s shell of exponent
    # 1e-12 with effective coefficient 1
    main, aux = S.df_fixture()
    eps = 1e-12
    nm = len(main)
    for psh, sp in enumerate(aux):
        tiny = dict(l=0, spherical=False, center=list(sp["center"]), exps=[eps], coefs=[1.0 / _s_norm(eps)])
        four = O.OracleBasis(list(main) + [sp, tiny])
        for ish in range(nm):
            for jsh in range(nm):
                got = O.df_eri_3c_block(main, aux, ish, jsh, psh)
                want = four.eri_block(ish, jsh, nm, nm + 1).reshape(-1)
                peak = float(np.max(np.abs(want)))
                assert float(np.max(np.abs(got - want))) <= 1e-8 * peak + 1e-12


def test_df_cross_engine_symmetry_and_definiteness():
    # tests/df.rs:125-195
    main, aux = S.df_fixture()
    os_, rys = O.df_eri_2c(aux, "os"), O.df_eri_2c(aux, "rys")
    peak = float(np.max(np.abs(os_)))
    assert float(np.max(np.abs(os_ - rys))) <= 1e-11 * max(peak, 1.0)
    m = O.df_eri_2c(aux)
    n = int(round(np.sqrt(m.size)))
    M = m.reshape(n, n)
    assert np.array_equal(M, M.T) and np.all(np.diag(M) > 0.0)
    np.linalg.cholesky(M)
    for ish in range(len(main)):
        for jsh in range(len(main)):
            for psh in range(len(aux)):
                a = O.df_eri_3c_block(main, aux, ish, jsh, psh, "os")
                b = O.df_eri_3c_block(main, aux, ish, jsh, psh, "rys")
                assert float(np.max(np.abs(a - b))) <= 1e-11 * max(float(np.max(np.abs(a))), 1.0)


def test_df_schwarz_aux_bound_holds_for_all_3c_blocks():
    # tests/df.rs:197-222
    main, aux = S.df_fixture()
    q = O.OracleBasis(main).schwarz()
    qp = O.df_schwarz_aux(aux)
    assert qp.shape == (len(aux),)
    for ish in range(len(main)):
        for jsh in range(len(main)):
            for psh in range(len(aux)):
                bound = q[ish, jsh] * qp[psh]
                blk = O.df_eri_3c_block(main, aux, ish, jsh, psh)
                assert float(np.max(np.abs(blk))) <= bound * (1.0 + 1e-10) + 1e-14


def test_df_builder_equals_blockwise_assembly_and_erf_limit():
    # tests/df.rs:224-266: the assembled tensor is the blocks in both bands;
    # tests/erf_kernel.rs:428-481: erf at large omega is Coulomb
    main, aux = S.df_fixture()
    T = O.df_eri_3c(main, aux)
    mo, nao = O._offsets(main)
    ao, naux = O._offsets(aux)
    T = T.reshape(nao, nao, naux)
    for ish in range(len(main)):
        for jsh in range(len(main)):
            for psh in range(len(aux)):
                ni, nj, npp = O._nf(main[ish]), O._nf(main[jsh]), O._nf(aux[psh])
                blk = O.df_eri_3c_block(main, aux, ish, jsh, psh).reshape(ni, nj, npp)
                got = T[mo[ish]:mo[ish] + ni, mo[jsh]:mo[jsh] + nj, ao[psh]:ao[psh] + npp]
                assert float(np.max(np.abs(got - blk))) <= 1e-13 * max(float(np.max(np.abs(blk))), 1.0)
    with O.erf(1e9):
        T2 = O.df_eri_3c(main, aux, "rys").reshape(nao, nao, naux)
        M2 = O.df_eri_2c(aux, "rys")
    assert float(np.max(np.abs(T2 - T))) < 1e-12 * float(np.max(np.abs(T)))
    M = O.df_eri_2c(aux)
    assert float(np.max(np.abs(M2 - M))) < 1e-12 * float(np.max(np.abs(M)))



# ------------------------------------------------- dense-gamma gradient

def _dense_gamma(n, coulomb, exchange):
    """tests/direct_grad_contractor.rs:106-129."""
    G = np.zeros((n, n, n, n))
    for f, L, R in coulomb:
        G += f * np.einsum("pq,rs->pqrs", L, R)
    for f, L, R in exchange:
        G += f * np.einsum("pr,qs->pqrs", L, R)
    return G


@pytest.mark.parametrize("spherical,engine,omega", [(False, "os", 0.0), (True, "os", 0.0), (False, "rys", 0.0),
                                                    (True, "auto", 0.0), (True, "rys", 0.3), (False, "rys", 1.7)])
def test_direct_gradient_matches_dense_gamma_contraction(spherical, engine, omega):
    # tests/direct_grad_contractor.rs:157-225: the density-direct contraction
    # equals eri_grad_contract of the dense gamma within 1e-10, zero net force
    shells = S.direct_grad_fixture(spherical)
    B = O.OracleBasis(shells)
    n = B.nao
    coul, exch = S.grad_fixture_terms(n)
    gamma = _dense_gamma(n, coul, exch)
    with O.erf(omega):
        ref = B.eri_grad_contract(gamma, engine)
        g, _, _ = B.direct_grad(coul, exch, 0.0, engine=engine)
    assert float(np.max(np.abs(g - ref))) < 1e-10
    assert float(np.max(np.abs(g.sum(axis=0)))) < 1e-10
    assert float(np.max(np.abs(g))) > 1e-3


def test_gradient_term_lists_are_additive_and_bra_order_free():
    # tests/direct_grad_contractor.rs:556-612: coulomb-only + exchange-only
    # = both; no terms = exact zero; bra tasks summed in reverse order over
    # two partial outputs = the serial contraction
    shells = S.direct_grad_fixture(True)
    B = O.OracleBasis(shells)
    coul, exch = S.grad_fixture_terms(B.nao)
    both, _, _ = B.direct_grad(coul, exch, 0.0)
    c_only, _, _ = B.direct_grad(coul, [], 0.0)
    x_only, _, _ = B.direct_grad([], exch, 0.0)
    assert float(np.max(np.abs(c_only))) > 1e-3 and float(np.max(np.abs(x_only))) > 1e-3
    assert float(np.max(np.abs(c_only + x_only - both))) < 1e-12
    nothing, _, _ = B.direct_grad([], [], 0.0)
    assert np.all(nothing == 0.0)
    p = S.grad_symmetric(B.nao, 4)
    terms = [(1.0, p, p)]
    serial, _, _ = B.direct_grad(terms, terms, 0.0)
    nbra = len(shells) * (len(shells) + 1) // 2
    rev = np.arange(nbra)[::-1]
    parts = [B.direct_grad(terms, terms, 0.0, bras=rev[t::2])[0] for t in range(2)]
    assert float(np.max(np.abs(parts[0] + parts[1] - serial))) < 1e-12


def test_gradient_screening_error_is_bounded_on_extended_system():
    # tests/direct_grad_contractor.rs:662-690: tau = 0 equals the dense
    # contraction; the screened error stays below 100 tau; tau = inf drops
    # every quartet
    shells = S.grad_extended_fixture()
    B = O.OracleBasis(shells)
    n = B.nao
    coul, exch = S.grad_fixture_terms(n)
    ref = B.eri_grad_contract(_dense_gamma(n, coul, exch))
    exact, _, _ = B.direct_grad(coul, exch, 0.0)
    assert float(np.max(np.abs(exact))) > 1e-3
    assert float(np.max(np.abs(exact - ref))) < 1e-10
    for thr in (1e-12, 1e-9, 1e-6):
        screened, _, _ = B.direct_grad(coul, exch, thr)
        assert float(np.max(np.abs(screened - exact))) < 100.0 * thr
    nothing, cnt, _ = B.direct_grad(coul, exch, float("inf"))
    assert cnt == 0 and np.all(nothing == 0.0)



# ------------------------------------------------- screened dense tensor

def test_screened_tensor_keeps_retained_elements_and_bounds_the_rest():
    # tests/screening.rs: |(mu nu|la si)| <= Q_ij Q_kl element-wise, the
    # screened tensor equals the unscreened one on retained elements, and
    # tau = 0 is the unscreened tensor
    s = S.dense_eri_system()
    B = O.OracleBasis(s["shells"])
    E = B.eri()
    Q = B.schwarz()
    n = B.nsh
    nf = [3 if sh["l"] == 1 else 1 for sh in s["shells"]]
    owner = np.repeat(np.arange(n), nf)
    bound = np.multiply.outer(Q, Q)[np.ix_(owner, owner, owner, owner)].reshape(-1)
    assert np.all(np.abs(E) <= bound * (1 + 1e-12) + 1e-15)
    E0, total, skipped = B.eri_screened(0.0)
    assert np.array_equal(E0, E) and skipped == 0
    npairs = n * (n + 1) // 2
    assert total == npairs * (npairs + 1) // 2 == 108345
    tau = 1e-4
    Es, total, skipped = B.eri_screened(tau)
    assert 0 < skipped < total
    kept = Es != 0.0
    assert np.array_equal(Es[kept], E[kept])
    assert float(np.max(np.abs(E[~kept]))) < tau



def test_select_engine_policy_matches_the_oracle():
    # src/integrals.rs:374-388 (tests/dispatch.rs: every threshold boundary)
    import integral_b200 as ib
    for ne in range(0, 13):
        for nf in range(0, 13):
            for deg in (1, 2, 3, 4, 15, 16, 17, 81, 256):
                want = {"os": ib.Engine.OsHgp, "rys": ib.Engine.Rys}[O.select_engine(ne, nf, deg)]
                assert ib.select_engine(ne, nf, deg) == want, (ne, nf, deg)


def test_df_erf_metric_concentric_s_closed_form():
    # tests/erf_kernel.rs:428-481 (2c/3c through the unit-s dummy under
    # erf): two concentric s functions have T = 0, so
    # (P|Q)_erf = N_a N_b 2 pi^(5/2) / (a b sqrt(a+b)) * sqrt(s),
    # s = omega^2 / (rho + omega^2), rho = a b / (a + b)
    a, b, omega = 0.9, 1.7, 0.6
    aux = [dict(l=0, spherical=False, center=[0.0] * 3, exps=[a], coefs=[1.0]),
           dict(l=0, spherical=False, center=[0.0] * 3, exps=[b], coefs=[1.0])]
    with O.erf(omega):
        m = O.df_eri_2c(aux, "rys")
    rho = a * b / (a + b)
    sc = omega ** 2 / (rho + omega ** 2)
    want = _s_norm(a) * _s_norm(b) * 2.0 * np.pi ** 2.5 / (a * b * np.sqrt(a + b)) * np.sqrt(sc)
    _close(m[1], want, 1e-12)
    assert m[1] == m[2]
