"""Hamiltonians for the contraction engine: the MOLPRO FCIDUMP import path
(input/read_env_molpro_dump.f, input/import_hamint_molpro_dump.f) and the
seeded synthetic Hamiltonians of the benchmark configurations.

Orbitals are split per irrep into frozen / active occupied (hole type H) /
virtual (particle type P) / deleted, and ordered inside a type by irrep, then
by their position in the input -- the orbital sequence of the reference's
string graphs (mostnd ranges per irrep and GAS, include/def_orbinf.h).

The Fock matrix is built from the one-electron integrals plus the core
contributions of all occupied orbitals, f_pq = h_pq + sum_k [2(pq|kk) -
(pk|kq)] (input/import_fock_molpro_dump.f:114-126).
"""
import os

import numpy as np


class OrbitalSpace:
    def __init__(self, orbsym, nocc, nfrozen=None, ndeleted=None):
        orbsym = np.asarray(orbsym)
        nsym = int(orbsym.max())
        nsym = 1 if nsym == 1 else (2 if nsym == 2 else (4 if nsym <= 4 else 8))
        self.nsym = nsym
        nfrozen = list(nfrozen or [0] * nsym) + [0] * 8
        ndeleted = list(ndeleted or [0] * nsym) + [0] * 8
        nocc = list(nocc) + [0] * 8
        self.frozen, self.hole, self.part, self.occ_all = [], [], [], []
        self.norb = np.zeros((4, 8), dtype=np.int64)
        for g in range(1, nsym + 1):
            idx = [i for i, s in enumerate(orbsym) if s == g]
            nf, no, nd = nfrozen[g - 1], nocc[g - 1], ndeleted[g - 1]
            self.frozen += idx[:nf]
            self.occ_all += idx[:no]
            self.hole += idx[nf:no]
            virt = idx[no:len(idx) - nd]
            self.part += virt
            self.norb[0, g - 1] = no - nf
            self.norb[1, g - 1] = len(virt)
        self.orbsym = orbsym
        self.hole = np.array(self.hole, dtype=np.int64)
        self.part = np.array(self.part, dtype=np.int64)
        self.occ_all = np.array(self.occ_all, dtype=np.int64)

    def type_orbitals(self, t):
        return self.hole if t == 0 else self.part

    @property
    def nh(self):
        return len(self.hole)

    @property
    def np_(self):
        return len(self.part)


def fcidump_records(path):
    """header and records of an FCIDUMP: text (&FCI NORB,NELEC,MS2,ORBSYM,ISYM
    namelist, then value p q r s records, input/read_env_molpro_dump.f:39-57)
    or the fixture .npz form; returns norb, orbsym, vals, idx (1-based
    orbital indices, 0 for the absent ones)"""
    if path.endswith(".npz"):
        d = np.load(path)
        return dict(norb=int(d["norb"]), orbsym=d["orbsym"], vals=d["vals"], idx=d["idx"])
    import re
    text = open(path).read()
    head, body = text.split("/", 1)
    norb = int(re.search(r"NORB\s*=\s*(\d+)", head).group(1))
    orbsym = np.array([int(x) for x in re.search(r"ORBSYM\s*=\s*([\d,\s]+?),\s*ISYM", head)
                       .group(1).replace(",", " ").split()])
    rec = np.array([l.split() for l in body.splitlines() if len(l.split()) == 5])
    return dict(norb=norb, orbsym=orbsym, vals=rec[:, 0].astype(float),
                idx=rec[:, 1:].astype(int))


# the eight index orders of a real (pq|rs)
ERI_PERMS = ((0, 1, 2, 3), (1, 0, 2, 3), (0, 1, 3, 2), (1, 0, 3, 2),
             (2, 3, 0, 1), (3, 2, 0, 1), (2, 3, 1, 0), (3, 2, 1, 0))


def read_fcidump(path):
    """one-electron matrix h, (pq|rs) with its eight-fold symmetry and the
    core energy from an FCIDUMP (records with r = s = 0 are h_pq, all-zero
    indices the core energy)"""
    r = fcidump_records(path)
    norb, vals, idx = r["norb"], np.asarray(r["vals"], float), np.asarray(r["idx"], int)
    core = (idx == 0).all(axis=1)
    one = (idx[:, 2] == 0) & (idx[:, 3] == 0) & ~core
    two = ~(core | one)
    h = np.zeros((norb, norb))
    p, q = idx[one, 0] - 1, idx[one, 1] - 1
    h[p, q] = vals[one]
    h[q, p] = vals[one]
    eri = np.zeros((norb,) * 4)
    ix = (idx[two] - 1).T
    for perm in ERI_PERMS:
        eri[ix[perm[0]], ix[perm[1]], ix[perm[2]], ix[perm[3]]] = vals[two]
    ecore = float(vals[core][-1]) if core.any() else 0.0
    return dict(norb=norb, orbsym=r["orbsym"], h=h, eri=eri, ecore=ecore)


def fock(h, eri, occ):
    J = np.einsum("pqkk->pq", eri[:, :, occ][:, :, :, occ])
    K = np.einsum("pkkq->pq", eri[:, occ][:, :, occ])
    return h + 2 * J - K


class DenseIntegrals:
    """spatial Fock matrix and (pq|rs) in memory (small systems)"""

    def __init__(self, space, f, eri):
        self.space, self.f, self.eri = space, f, eri

    def fock(self, p, q):
        return self.f[p, q]

    def eri_elems(self, p, q, r, s):
        return self.eri[p, q, r, s]


def synthetic(nocc, nvir, naux, seed, nsym=1, occ_range=(-1.5, -0.3), vir_range=(0.1, 4.0),
              gap=None, dtype=np.float64, sigma=0.05):
    """seeded synthetic closed-shell Hamiltonian: canonical diagonal Fock with
    occupied energies U[occ_range], virtual energies U[vir_range] (or a
    HOMO-LUMO gap), (pq|rs) = sum_P B_pq^P B_rs^P with B symmetric in pq:
    the entries with p <= q are drawn from N(0, sigma^2) (sigma = 0.05 by
    default) and mirrored to q > p, so every entry has that distribution.
    The exchange-type integrals (pq|pq) = sum_P (B_pq^P)^2 are then about
    naux * sigma^2 Eh.  With nsym > 1 irreps are assigned round-robin to
    orbitals and auxiliary functions and B_pq^P vanishes unless
    irrep(p) x irrep(q) = irrep(P), so every integral is totally symmetric.
    Returns (space, eps, B) with B of shape (norb, norb, naux)."""
    rng = np.random.default_rng(seed)
    n = nocc + nvir
    eo = np.sort(rng.uniform(*occ_range, size=nocc))
    if gap is not None:
        ev = np.sort(eo.max() + gap + rng.uniform(0.0, vir_range[1] - vir_range[0], size=nvir))
        ev[0] = eo.max() + gap
    else:
        ev = np.sort(rng.uniform(*vir_range, size=nvir))
    eps = np.concatenate([eo, ev])
    sym = np.arange(n) % nsym + 1
    B = rng.normal(0.0, sigma, size=(n, n, naux)).astype(dtype)
    upper = np.arange(n)[:, None] <= np.arange(n)[None, :]
    B = np.where(upper[:, :, None], B, B.transpose(1, 0, 2))
    if nsym > 1:
        psym = np.arange(naux) % nsym
        mask = ((sym[:, None] - 1) ^ (sym[None, :] - 1))[:, :, None] == psym[None, None, :]
        B *= mask
    # reorder orbitals by irrep (stable), occupied ones first within each irrep
    occ_flag = np.arange(n) < nocc
    order = np.lexsort((np.arange(n), ~occ_flag, sym))
    eps, sym = eps[order], sym[order]
    B = B[order][:, order]
    nocc_irrep = [int(np.sum(occ_flag[order][sym == g])) for g in range(1, nsym + 1)]
    space = OrbitalSpace(sym, nocc_irrep)
    return space, eps, B


class FactorizedIntegrals:
    """diagonal Fock eps and (pq|rs) = sum_P B_pq^P B_rs^P"""

    def __init__(self, space, eps, B):
        self.space, self.eps, self.B = space, eps, B

    def fock(self, p, q):
        return np.where(p == q, self.eps[p], 0.0)

    def eri_elems(self, p, q, r, s):
        return np.einsum("...P,...P->...", self.B[p, q], self.B[r, s])

    def dense_eri(self):
        return np.einsum("pqP,rsP->pqrs", self.B, self.B)
