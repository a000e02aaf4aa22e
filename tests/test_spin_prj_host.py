"""Spin projection of an ME list onto its singlet part (spin_prj_list /
spin_prj_blk, contract/spin_prj_list.f, contract/spin_prj_blk.f): the
oracle's restatement checked against Fock space, independently of the
reference's coupling-coefficient machinery.

Every list element is the operator a+(c_1)..a+(c_n) a(a_n)..a(a_1) of its
creator and annihilator spin orbitals (the dense convention of melist).  After
the projection the operator of the list commutes with S+ and S-; the
projection is idempotent; its rank equals the dimension of the singlet
operators spanned by the class (the null space of X -> ([S+,X], [S-,X])); a
one-body class ends with alpha and beta elements equal to their mean."""
import numpy as np
import pytest
import scipy.sparse as sps

from binding import Oracle, OracleError
from gccu import H, P, V, occ8
from melist import ListView

SPACE = (1, [[2], [2], [1], [0]])
SPACE_C2 = (2, [[1, 1], [2, 1], [0, 0], [0, 0]])
CLASSES = {
    "t1": occ8({P: 1}, {H: 1}),
    "t2": occ8({P: 2}, {H: 2}),
    "t3": occ8({P: 3}, {H: 3}),
    "pv_hh": occ8({P: 1, V: 1}, {H: 2}),
    "ph_ph": occ8({P: 1, H: 1}, {P: 1, H: 1}),
    "pp_vh": occ8({P: 2}, {V: 1, H: 1}),
    "pv_hv": occ8({P: 1, V: 1}, {H: 1, V: 1}),
    "hh_hh": occ8({H: 2}, {H: 2}),
}


class Fock:
    """Jordan-Wigner operators of the spin orbitals of an orbital space"""

    def __init__(self, norb_type):
        self.mode = {}
        for t in range(4):
            for so in range(2 * norb_type[t]):
                self.mode[(t, so)] = len(self.mode)
        n = len(self.mode)
        self.dim = 1 << n
        states = np.arange(self.dim)
        self.a = []
        for j in range(n):
            occ = (states >> j) & 1 == 1
            src = states[occ]
            below = np.array([bin(int(s) & ((1 << j) - 1)).count("1") for s in src])
            sign = np.where(below % 2 == 1, -1.0, 1.0)
            self.a.append(sps.csr_matrix((sign, (src ^ (1 << j), src)),
                                         shape=(self.dim, self.dim)))
        self.splus = sps.csr_matrix((self.dim, self.dim))
        for (t, so), j in self.mode.items():
            if so % 2 == 0:
                self.splus = self.splus + self.a[j].T @ self.a[self.mode[(t, so + 1)]]
        self.sminus = self.splus.T.tocsr()

    def op(self, cre, ann):
        """a+(cre[0])..a+(cre[-1]) a(ann[-1])..a(ann[0]) on (type, so) modes"""
        m = sps.identity(self.dim, format="csr")
        for t in cre:
            m = m @ self.a[self.mode[t]].T
        for t in reversed(ann):
            m = m @ self.a[self.mode[t]]
        return m


def _class_elements(o, lid, occ, nsym):
    """per list element of the class: (index, creator modes, annihilator modes)"""
    view = ListView(o, lid, [occ], nsym)
    out = []
    for off, comps, strs, ld in view.blocks(1):
        grids = np.meshgrid(*[np.arange(s.shape[0]) for s in strs], indexing="ij")
        idx = off + sum(g * d for g, d in zip(grids, ld))
        for pos in np.ndindex(*[s.shape[0] for s in strs]):
            modes = []
            for j, (t, _) in enumerate(comps):
                modes.append([(t, int(so)) for so in strs[j][pos[j]]])
            out.append((int(idx[pos]), modes))
    return out


def _setup(space, occ, gamt=1):
    nsym, norb = space
    o = Oracle(nsym, norb)
    lid, n = o.define_list(o.define_op([occ]), gamt=gamt)
    return o, lid, n


def _operators(space, occ, o, lid):
    nsym, norb = space
    fock = Fock([sum(r) for r in norb])
    ncomp_c = sum(1 for t in (3, 1, 2, 0) if occ[t] > 0)
    ops = {}
    for idx, modes in _class_elements(o, lid, occ, nsym):
        cre = [m for c in modes[:ncomp_c] for m in c]
        ann = [m for c in modes[ncomp_c:] for m in c]
        ops[idx] = fock.op(cre, ann)
    return fock, ops


def _commutator_norm(fock, ops, x):
    X = sum(x[i] * m for i, m in ops.items())
    cp = fock.splus @ X - X @ fock.splus
    cm = fock.sminus @ X - X @ fock.sminus
    return np.sqrt(sps.linalg.norm(cp) ** 2 + sps.linalg.norm(cm) ** 2), sps.linalg.norm(X)


@pytest.mark.parametrize("name", list(CLASSES))
@pytest.mark.parametrize("space", [SPACE, SPACE_C2], ids=["c1", "c2"])
def test_projected_list_commutes_with_spin_ladders(built, name, space):
    occ = CLASSES[name]
    if space is SPACE_C2 and occ[V] + occ[4 + V] > 0:
        pytest.skip("no valence orbitals in this space")
    o, lid, n = _setup(space, occ)
    if n == 0:
        pytest.skip("empty class")
    fock, ops = _operators(space, occ, o, lid)
    assert sorted(ops) == list(range(n))
    x = np.random.default_rng(7).standard_normal(n)
    c0, x0 = _commutator_norm(fock, ops, x)
    assert c0 > 1e-3 * x0  # a random operator is no singlet
    y = x.copy()
    xn = o.spin_prj(lid, y, 1)
    assert np.isclose(xn[0], y @ y, rtol=1e-13)
    c1, x1 = _commutator_norm(fock, ops, y)
    assert x1 > 1e-3 * x0
    assert c1 <= 1e-12 * x1, (name, c1, x1)
    z = y.copy()
    o.spin_prj(lid, z, 1)
    assert np.max(np.abs(z - y)) <= 1e-13 * np.abs(y).max()


@pytest.mark.parametrize("name", ["t1", "t2", "t3", "pv_hh", "ph_ph", "pv_hv"])
def test_projection_rank_is_the_singlet_dimension(built, name):
    occ = CLASSES[name]
    o, lid, n = _setup(SPACE, occ)
    fock, ops = _operators(SPACE, occ, o, lid)
    # projection matrix column by column
    Pm = np.zeros((n, n))
    for e in range(n):
        u = np.zeros(n)
        u[e] = 1.0
        o.spin_prj(lid, u, 1)
        Pm[:, e] = u
    assert np.allclose(Pm @ Pm, Pm, atol=1e-13)
    # Gram matrix of the commutator map over the elements
    cs = [None] * n
    for i, m in ops.items():
        cs[i] = (fock.splus @ m - m @ fock.splus, fock.sminus @ m - m @ fock.sminus)
    G = np.zeros((n, n))
    for i in range(n):
        for j in range(i, n):
            g = sum((cs[i][k].multiply(cs[j][k])).sum() for k in range(2))
            G[i, j] = G[j, i] = g
    w = np.linalg.eigvalsh(G)
    singlet_dim = int(np.sum(w < 1e-9 * max(1.0, w.max())))
    rank = int(np.linalg.matrix_rank(Pm, tol=1e-10))
    assert rank == singlet_dim, (name, rank, singlet_dim)
    assert np.abs(Pm.T @ G @ Pm).max() <= 1e-10 * max(1.0, np.abs(G).max())


@pytest.mark.parametrize("name", ["p4_h4", "pphh_pphh"])
def test_four_body_projection_commutes_with_spin_ladders(built, name):
    # four creators and four annihilators: 70 spin cases, 14 coupling paths
    space = (1, [[3], [2], [0], [0]])
    occ = {"p4_h4": occ8({P: 4}, {H: 4}), "pphh_pphh": occ8({P: 2, H: 2}, {P: 2, H: 2})}[name]
    o, lid, n = _setup(space, occ)
    fock, ops = _operators(space, occ, o, lid)
    x = np.random.default_rng(9).standard_normal(n)
    c0, x0 = _commutator_norm(fock, ops, x)
    assert c0 > 1e-3 * x0
    o.spin_prj(lid, x, 1)
    c1, x1 = _commutator_norm(fock, ops, x)
    assert x1 > 1e-3 * x0 and c1 <= 1e-12 * x1, (c1, x1)


def test_one_body_class_averages_alpha_and_beta(built):
    occ = CLASSES["t1"]
    o, lid, n = _setup(SPACE, occ)
    view = ListView(o, lid, [occ], SPACE[0])
    x = np.random.default_rng(3).standard_normal(n)
    y = x.copy()
    o.spin_prj(lid, y, 1)
    by = {}
    for off, comps, strs, ld in view.blocks(1):
        for ic in range(strs[0].shape[0]):
            for ia in range(strs[1].shape[0]):
                so_c, so_a = int(strs[0][ic][0]), int(strs[1][ia][0])
                key = (so_c // 2, so_a // 2)
                by.setdefault(key, {})[(so_c % 2, so_a % 2)] = off + ic * ld[0] + ia * ld[1]
    assert len(by) == n // 2
    for key, e in by.items():
        aa, bb = e[(0, 0)], e[(1, 1)]
        mean = 0.5 * (x[aa] + x[bb])
        assert abs(y[aa] - mean) < 1e-14 and abs(y[bb] - mean) < 1e-14
    # spin-changing elements (alpha -> beta) have Ms(C) != Ms(A): not in an Ms = 0 list
    assert all(set(e) == {(0, 0), (1, 1)} for e in by.values())


def test_projection_rejects_what_the_reference_rejects(built):
    o, lid, n = _setup(SPACE, occ8({P: 1}, {H: 2}))
    with pytest.raises(OracleError, match="particle-conserving"):
        o.spin_prj(lid, np.zeros(n), 1)
    o, lid, n = _setup(SPACE, CLASSES["t2"])
    with pytest.raises(OracleError, match="singlet"):
        o.spin_prj(lid, np.zeros(n), 1, s2=2)
    nsym, norb = SPACE
    lid2, n2 = o.define_list(o.define_op([CLASSES["ph_ph"]]), mst=2)
    with pytest.raises(OracleError, match="ms"):
        o.spin_prj(lid2, np.zeros(n2), 1)


def test_scalar_class_is_unchanged(built):
    o, lid, n = _setup(SPACE, occ8())
    x = np.array([1.25])
    xn = o.spin_prj(lid, x, 1)
    assert x[0] == 1.25 and xn[0] == 1.5625
