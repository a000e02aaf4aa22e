"""Host-side access to ME lists: element addressing and dense <-> list
conversion.

An ME list stores, per occupation class, the (Ms, IRREP, distribution)
blocks of set_op_dim2 (operators/set_op_dim2.f); inside a block the element
of component strings (s_1..s_n) sits at sum_j s_j*ldim_j with the leading
dimensions of set_op_ldim_c (contract/set_op_ldim_c.f: X,P,V,H major,
creators before annihilators).

Dense convention used by the host (and the tests): the tensor of one class
has one axis per electron, creator components first, then annihilator
components, each side in X,P,V,H order; an axis runs over the type-local
spin orbitals 2*orb+spin (alpha 0, beta 1).  The stored element of sorted
strings equals the dense tensor at those spin orbitals.

`src` is any object with .strings(type, nel, idxms, gam) and .dists(list)
(the engine binding; the test oracle has the same methods).
"""
import numpy as np

HPVX_SEQ = (3, 1, 2, 0)  # X, P, V, H


def condensed(occ):
    """components (type, occupation) of creators and annihilators"""
    occ = np.asarray(occ)
    c = [(t, int(occ[t])) for t in HPVX_SEQ if occ[t] > 0]
    a = [(t, int(occ[4 + t])) for t in HPVX_SEQ if occ[4 + t] > 0]
    return c, a


def decode_did(did, comps, nsym):
    """per component (idxms, irrep) from a distribution id (msgmdid2)"""
    out = []
    for _, n in comps:
        r = did % ((n + 1) * nsym)
        did //= (n + 1) * nsym
        out.append((r // nsym + 1, r % nsym + 1))
    return out


def ldims(c, a, lens):
    """leading dimensions per component (creators then annihilators)"""
    ld = [0] * (len(c) + len(a))
    cur = 1
    for t in HPVX_SEQ:
        for i, (tc, _) in enumerate(c):
            if tc == t:
                ld[i] = cur
                cur *= lens[i]
        for i, (ta, _) in enumerate(a):
            if ta == t:
                ld[len(c) + i] = cur
                cur *= lens[len(c) + i]
    return ld


def spin_orbitals(orb, spn):
    """type-local spin-orbital indices of strings (n, nel): pairs give alpha, beta"""
    so = 2 * (orb - 1) + (spn == -1)
    pair = spn == 2
    if pair.any():
        # second member of a pair is the beta spin orbital
        second = np.zeros_like(pair)
        second[:, 1:] = pair[:, 1:] & pair[:, :-1] & (orb[:, 1:] == orb[:, :-1])
        so = so + second
    return so


class ListView:
    """Element addressing of one ME list for host code."""

    def __init__(self, src, list_id, occs, nsym):
        self.src = src
        self.id = list_id
        self.occs = [np.asarray(o) for o in occs]
        self.nsym = nsym
        self.rows = src.dists(list_id)
        self._strings = {}

    def strings(self, typ, nel, idxms, gam):
        k = (typ, nel, idxms, gam)
        if k not in self._strings:
            orb, spn = self.src.strings(typ, nel, idxms, gam)
            self._strings[k] = spin_orbitals(orb, spn)
        return self._strings[k]

    def blocks(self, iblk):
        """yield (offset, comps, per-component spin-orbital strings, ldims)"""
        c, a = condensed(self.occs[iblk - 1])
        comps = c + a
        for r in self.rows[self.rows[:, 0] == iblk]:
            off, did = int(r[4]), int(r[7])
            dist = decode_did(did, comps, self.nsym)
            strs = [self.strings(t, n, ix, g) for (t, n), (ix, g) in zip(comps, dist)]
            lens = [s.shape[0] for s in strs]
            yield off, comps, strs, ldims(c, a, lens)

    def fill(self, x, iblk, value):
        """x[elements of class iblk] = value(list of index arrays, one per
        electron axis, broadcast over the component grid)"""
        for off, comps, strs, ld in self.blocks(iblk):
            ncomp = len(strs)
            axes = []
            for j, s in enumerate(strs):
                shape = [1] * ncomp
                shape[j] = s.shape[0]
                for e in range(s.shape[1]):
                    axes.append(s[:, e].reshape(shape))
            vals = np.broadcast_to(value(axes), [s.shape[0] for s in strs])
            pos = np.zeros([1] * ncomp, dtype=np.int64)
            for j, s in enumerate(strs):
                shape = [1] * ncomp
                shape[j] = s.shape[0]
                pos = pos + np.arange(s.shape[0]).reshape(shape) * ld[j]
            pos = np.broadcast_to(pos, vals.shape)
            x[off + pos.reshape(-1)] = vals.reshape(-1)

    def from_dense(self, dense, n):
        """list vector from {iblk: dense tensor}"""
        x = np.zeros(n)
        for iblk, D in dense.items():
            self.fill(x, iblk, lambda axes, D=D: D[tuple(axes)])
        return x

    def to_dense(self, x, iblk, shape):
        """dense antisymmetric tensor of class iblk from the list vector"""
        D = np.zeros(shape)
        c, a = condensed(self.occs[iblk - 1])
        comps = c + a
        for off, comps_, strs, ld in self.blocks(iblk):
            ncomp = len(strs)
            idx = np.zeros([s.shape[0] for s in strs], dtype=np.int64)
            for j, s in enumerate(strs):
                shape = [1] * ncomp
                shape[j] = s.shape[0]
                idx = idx + np.arange(s.shape[0]).reshape(shape) * ld[j]
            vals = x[off + idx.reshape(-1)]
            grid = np.stack(np.meshgrid(*[np.arange(s.shape[0]) for s in strs], indexing="ij"),
                            -1).reshape(-1, ncomp)
            # all permutations inside each component with their parity
            import itertools
            perms = []
            for (t, ne) in comps:
                ps = []
                for p in itertools.permutations(range(ne)):
                    inv = sum(1 for i in range(ne) for j in range(i + 1, ne) if p[i] > p[j])
                    ps.append((p, -1 if inv % 2 else 1))
                perms.append(ps)
            for combo in itertools.product(*perms):
                sign = np.prod([s for _, s in combo])
                index = []
                for j, (p, _) in enumerate(combo):
                    s = strs[j][grid[:, j]]
                    index.extend(s[:, list(p)].T)
                D[tuple(index)] = sign * vals
        return D
