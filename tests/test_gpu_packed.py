"""GPU parity of the packed symmetry-unique ERI tensor (PackedEriBuilder,
src/packed_eri.rs) against the oracle's dense tensor, on the 6-atom, nao 54
Cartesian s,s,s,p,p system: every packed element (t|u), u <= t, is
eri[p,q,r,s] of its AO pairs (t = (p,q), u = (r,s)); tolerances of the dense
ERI test (1e-12 relative on significant elements, 1e-13 of the peak
everywhere); Schwarz-screened blocks are zero; a fill of a bra subset writes
exactly those bras' rows."""
import numpy as np
import pytest

import integral_b200 as ib
import oracle_py as O
from integral_b200 import systems as S

pytestmark = pytest.mark.gpu


def expected_packed(E, ao_pairs):
    P = np.asarray(ao_pairs)
    m = len(P)
    out = np.zeros(m * (m + 1) // 2)
    for t in range(m):
        p, q = P[t]
        out[t * (t + 1) // 2: t * (t + 1) // 2 + t + 1] = E[p, q, P[: t + 1, 0], P[: t + 1, 1]]
    return out


def pair_starts(basis):
    """First AO-pair index of every canonical shell pair (i >= j, row-major):
    n_i(n_i+1)/2 pairs on a diagonal shell pair, n_i*n_j otherwise."""
    nf = [sh.n_func() for sh in basis.shells()]
    starts = [0]
    for i in range(len(nf)):
        for j in range(i + 1):
            starts.append(starts[-1] + (nf[i] * (nf[i] + 1) // 2 if i == j else nf[i] * nf[j]))
    return starts


def owners(starts):
    own = np.zeros(starts[-1], dtype=np.int64)
    for k in range(len(starts) - 1):
        own[starts[k]:starts[k + 1]] = k
    return own


def check(gpu, ref):
    peak = float(np.max(np.abs(ref)))
    d = np.abs(gpu - ref)
    sig = np.abs(ref) >= 1e-3 * peak
    assert float(np.max(d[sig] / np.abs(ref[sig]))) < 1e-12
    assert float(np.max(d)) < 1e-13 * max(peak, 1.0)


def test_packed_layout_follows_the_reference():
    s = S.dense_eri_system()
    B = ib.Basis(s["shells"])
    pb = B.packed_eri_builder()
    nao = B.nao()
    aop = pb.ao_pairs()
    assert len(aop) == nao * (nao + 1) // 2
    assert all(p >= q for p, q in aop)
    assert len(set(aop)) == len(aop)
    assert pb.output_len() == len(aop) * (len(aop) + 1) // 2


def test_packed_build_matches_dense_oracle():
    s = S.dense_eri_system()
    B = ib.Basis(s["shells"])
    pb = B.packed_eri_builder()
    n = B.nao()
    E = O.OracleBasis(s["shells"]).eri().reshape(n, n, n, n)
    check(pb.build(0.0), expected_packed(E, pb.ao_pairs()))


def test_packed_screened_build_zeroes_exactly_the_screened_blocks():
    s = S.dense_eri_system()
    B = ib.Basis(s["shells"])
    pb = B.packed_eri_builder()
    n = B.nao()
    OB = O.OracleBasis(s["shells"])
    E = OB.eri().reshape(n, n, n, n)
    Q = OB.schwarz()
    qp = np.array([Q[i, j] for i, j in pb.bra_pairs()])
    # a threshold in the widest gap of the sorted Q_bra*Q_ket products, so
    # the device's and the oracle's bounds cannot disagree on any quartet
    prods = np.unique(np.outer(qp, qp)[np.tril_indices(len(qp))])
    prods = prods[prods > 0]
    lo, hi = int(0.2 * len(prods)), int(0.8 * len(prods))
    ratios = prods[lo + 1:hi] / prods[lo:hi - 1]
    k = lo + int(np.argmax(ratios))
    thr = float(np.sqrt(prods[k] * prods[k + 1]))
    assert prods[k + 1] / prods[k] > 1 + 1e-9
    gpu = pb.build(thr)
    ref = expected_packed(E, pb.ao_pairs())
    own = owners(pair_starts(B))
    m = len(own)
    screened = np.zeros(ref.size, dtype=bool)
    for t in range(m):
        row = slice(t * (t + 1) // 2, t * (t + 1) // 2 + t + 1)
        screened[row] = qp[own[t]] * qp[own[: t + 1]] < thr  # packed_eri.rs:184-187
    assert 0 < np.count_nonzero(screened) < screened.size
    ref[screened] = 0.0
    check(gpu, ref)
    assert float(np.max(np.abs(gpu[screened]))) == 0.0


def test_packed_fill_of_a_bra_subset_writes_its_rows():
    s = S.dense_eri_system()
    B = ib.Basis(s["shells"])
    pb = B.packed_eri_builder()
    starts = pair_starts(B)
    full = pb.build(0.0)
    out = np.zeros(pb.output_len())
    tasks = pb.partition(out)
    chosen = tasks[::5]
    pb.fill_many(chosen, 0.0)

    def rows_of(bra):
        lo, hi = starts[bra], starts[bra + 1]
        return slice(lo * (lo + 1) // 2, hi * (hi + 1) // 2)

    mask = np.zeros(out.size, dtype=bool)
    for t in chosen:
        mask[rows_of(t.bra)] = True
        assert t.rows.size == rows_of(t.bra).stop - rows_of(t.bra).start
    assert float(np.max(np.abs(out[~mask]))) == 0.0
    assert np.array_equal(out[mask], full[mask])
    # one more task through the single-task entry, into the same buffer
    pb.fill(ib.PackedEriWorkspace(), tasks[1], 0.0)
    assert np.array_equal(out[rows_of(1)], full[rows_of(1)])
