"""Coupled-cluster residuals by brute force in the full Fock space of a few
spin orbitals (test helper, not product code): R_mu = <mu| e^-T H e^T |0>
with H = sum h_pq p+ q + 1/4 sum <pq||rs> p+ q+ s r, h = F - sum_i <pi||qi>,
|0> the determinant of the holes, and the excitation operator of the element
(a1 < a2 < ...; i1 < i2 < ...) of an excitation list taken as
a+_a1 a+_a2 ... a_i2 a_i1, the order the engine's lists use.  Spin orbitals
as in dense_cc.spin_orbital: holes first, then particles."""
import itertools

import numpy as np
import scipy.sparse as sps


def _annihilators(n):
    """a_p on the 2^n determinants (bit p = spin orbital p), Jordan-Wigner signs"""
    dim = 1 << n
    states = np.arange(dim)
    ops = []
    for p in range(n):
        occ = (states >> p) & 1 == 1
        src = states[occ]
        below = np.array([bin(s & ((1 << p) - 1)).count("1") for s in src])
        sign = np.where(below % 2, -1.0, 1.0)
        ops.append(sps.csr_matrix((sign, (src ^ (1 << p), src)), shape=(dim, dim)))
    return ops


def perm_sign(p):
    inv = sum(1 for i in range(len(p)) for j in range(i + 1, len(p)) if p[i] > p[j])
    return -1.0 if inv % 2 else 1.0


class FockSpace:
    def __init__(self, F, W, no):
        n = F.shape[0]
        self.n, self.no, self.nv = n, no, n - no
        self.a = _annihilators(n)
        self.c = [x.T.tocsr() for x in self.a]
        h = F - sum(W[:, i, :, i] for i in range(no))
        dim = 1 << n
        Hm = sps.csr_matrix((dim, dim))
        for p, q in zip(*np.nonzero(h)):
            Hm = Hm + h[p, q] * (self.c[p] @ self.a[q])
        cc = {}
        aa = {}
        for p, q, r, s in zip(*np.nonzero(W)):
            if (p, q) not in cc:
                cc[p, q] = self.c[p] @ self.c[q]
            if (s, r) not in aa:
                aa[s, r] = self.a[s] @ self.a[r]
            Hm = Hm + 0.25 * W[p, q, r, s] * (cc[p, q] @ aa[s, r])
        self.H = Hm.tocsr()
        self.ref = (1 << no) - 1

    def excitation(self, parts, holes):
        """a+_a1 .. a+_an a_in .. a_i1 (global spin-orbital indices)"""
        M = sps.identity(1 << self.n, format="csr")
        for a in parts:
            M = M @ self.c[a]
        for i in reversed(holes):
            M = M @ self.a[i]
        return M

    def _strings(self, rank):
        return itertools.product(itertools.combinations(range(self.nv), rank),
                                 itertools.combinations(range(self.no), rank))

    def t_operator(self, amps):
        """amps: {rank: dense antisymmetric t[a1..an, i1..in]} (type-local indices)"""
        dim = 1 << self.n
        T = sps.csr_matrix((dim, dim))
        for rank, t in amps.items():
            for pa, hi in self._strings(rank):
                v = t[pa + hi]
                if v != 0:
                    T = T + v * self.excitation([self.no + a for a in pa], list(hi))
        return T.tocsr()

    def residuals(self, amps, maxexc):
        """{0: correlation energy, rank: dense antisymmetric R[a.., i..]}"""
        T = self.t_operator(amps)
        v = np.zeros(1 << self.n)
        v[self.ref] = 1.0
        et = v.copy()
        term = v.copy()
        for k in range(1, self.no + 1):
            term = T @ term / k
            et = et + term
        w = self.H @ et
        out = w.copy()
        term = w.copy()
        for k in range(1, self.no + 1):
            term = -(T @ term) / k
            out = out + term
        res = {0: out[self.ref] - self.H[self.ref, self.ref]}
        for rank in range(1, maxexc + 1):
            R = np.zeros((self.nv,) * rank + (self.no,) * rank)
            for pa, hi in self._strings(rank):
                E = self.excitation([self.no + a for a in pa], list(hi))
                val = E[:, [self.ref]].toarray().ravel() @ out
                for pp in itertools.permutations(range(rank)):
                    for hp in itertools.permutations(range(rank)):
                        R[tuple(pa[x] for x in pp) + tuple(hi[x] for x in hp)] = \
                            perm_sign(pp) * perm_sign(hp) * val
            res[rank] = R
        return res


def random_amplitudes(rank, nv, no, rng, scale=0.1):
    """dense antisymmetric amplitudes of total Ms 0 (what an excitation list
    with mst = 0 stores; spin orbital 2k+1 is beta)"""
    t = np.zeros((nv,) * rank + (no,) * rank)
    for pa in itertools.combinations(range(nv), rank):
        for hi in itertools.combinations(range(no), rank):
            if sum(x % 2 for x in pa) != sum(x % 2 for x in hi):
                continue
            val = scale * rng.standard_normal()
            for pp in itertools.permutations(range(rank)):
                for hp in itertools.permutations(range(rank)):
                    t[tuple(pa[x] for x in pp) + tuple(hi[x] for x in hp)] = \
                        perm_sign(pp) * perm_sign(hp) * val
    return t


def non_canonical_fock(F, no, rng, scale=0.05):
    """F plus random symmetric spin-conserving hole-particle elements"""
    n = F.shape[0]
    X = scale * rng.standard_normal((n, n))
    X = (X + X.T) * (np.arange(n)[:, None] % 2 == np.arange(n)[None, :] % 2)
    X[:no, :no] = 0
    X[no:, no:] = 0
    return F + X
