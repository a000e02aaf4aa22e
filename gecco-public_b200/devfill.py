"""Filling ME lists on the device (set-up of the Hamiltonian).

The reference sorts integrals into its ME lists on the host during import
(input/import_h2_molpro_dump.f, "no batch algorithm").  Here the lists are
generated on the GPU and written in place into the engine's device memory:
per (class, Ms, IRREP, distribution) block the component strings are turned
into spin orbitals, the Fock elements and the antisymmetrised <c1c2||a1a2>
are gathered from spatial integrals on the device and scattered to the
block's element positions.  The spatial integrals are either factorised,
(pq|rs) = sum_P B_pq^P B_rs^P (TorchIntegrals), or dense (pq|rs) with the
Fock matrix (TorchDenseIntegrals; from_fcidump scatters an FCIDUMP's records
into them on the device).  torch is used as device-memory plumbing for this
set-up step only.
"""
import numpy as np
import torch

from melist import condensed, decode_did, ldims, spin_orbitals


class _CudaArray:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


def list_tensor(engine, lid, n):
    """torch view (no copy) of an engine list in device memory"""
    return torch.as_tensor(_CudaArray(engine.device_ptr(lid), n), device="cuda")


class DeviceListView:
    def __init__(self, engine, lid, occs, nsym, chunk=1 << 26, device="cuda"):
        self.e, self.id, self.nsym, self.chunk = engine, lid, nsym, chunk
        self.device = device
        self.occs = [np.asarray(o) for o in occs]
        self.rows = engine.dists(lid)
        self._str = {}

    def strings(self, t, n, ix, g):
        k = (t, n, ix, g)
        if k not in self._str:
            orb, spn = self.e.strings(t, n, ix, g)
            self._str[k] = torch.as_tensor(spin_orbitals(orb, spn), device=self.device)
        return self._str[k]

    def fill(self, x, iblk, value):
        c, a = condensed(self.occs[iblk - 1])
        comps = c + a
        for r in self.rows[self.rows[:, 0] == iblk]:
            off, did = int(r[4]), int(r[7])
            dist = decode_did(did, comps, self.nsym)
            strs = [self.strings(t, n, ix, g) for (t, n), (ix, g) in zip(comps, dist)]
            lens = [s.shape[0] for s in strs]
            ld = ldims(c, a, lens)
            rest = int(np.prod(lens[1:])) if len(lens) > 1 else 1
            step = max(1, self.chunk // max(rest, 1))
            for r0 in range(0, lens[0], step):
                r1 = min(lens[0], r0 + step)
                sub = [strs[0][r0:r1]] + strs[1:]
                nc = len(sub)
                axes = []
                for j, s in enumerate(sub):
                    shape = [1] * nc
                    shape[j] = s.shape[0]
                    for el in range(s.shape[1]):
                        axes.append(s[:, el].reshape(shape))
                grid = [s.shape[0] for s in sub]
                vals = value(axes).expand(grid)
                pos = torch.zeros([1] * nc, dtype=torch.int64, device=self.device)
                for j, s in enumerate(sub):
                    shape = [1] * nc
                    shape[j] = s.shape[0]
                    base = torch.arange(s.shape[0], device=self.device, dtype=torch.int64)
                    if j == 0:
                        base = base + r0
                    pos = pos + base.reshape(shape) * ld[j]
                pos = pos.expand(grid)
                x[off + pos.reshape(-1)] = vals.reshape(-1)


class TorchDenseIntegrals:
    """device form of DenseIntegrals: the spatial Fock matrix f and (pq|rs);
    the denominators use the Fock matrix's diagonal"""

    def __init__(self, space, f, eri, device="cuda"):
        self.space = space
        self.device = device
        self.f = torch.as_tensor(f, device=device, dtype=torch.float64)
        self.eri_pqrs = torch.as_tensor(eri, device=device, dtype=torch.float64)
        self.eps = torch.diagonal(self.f).clone()
        self.orbs = [torch.as_tensor(space.type_orbitals(t), device=device) for t in (0, 1)]
        self.ecore = 0.0

    @classmethod
    def from_fcidump(cls, path, nocc, nfrozen=None, ndeleted=None, device="cuda"):
        """the FCIDUMP's records (parsed on the host) scattered into h and
        (pq|rs) with its eight-fold symmetry on the device, the closed-shell
        Fock matrix f = h + 2J - K of the nocc (per irrep) lowest orbitals
        formed there"""
        import hamiltonian as hm
        r = hm.fcidump_records(path)
        n = int(r["norb"])
        space = hm.OrbitalSpace(r["orbsym"], nocc, nfrozen, ndeleted)
        vals = torch.as_tensor(np.asarray(r["vals"], dtype=np.float64), device=device)
        idx = torch.as_tensor(np.asarray(r["idx"], dtype=np.int64), device=device)
        core = (idx == 0).all(dim=1)
        one = (idx[:, 2] == 0) & (idx[:, 3] == 0) & ~core
        two = ~(core | one)
        h = torch.zeros((n, n), dtype=torch.float64, device=device)
        p, q = idx[one, 0] - 1, idx[one, 1] - 1
        h[p, q] = vals[one]
        h[q, p] = vals[one]
        eri = torch.zeros((n,) * 4, dtype=torch.float64, device=device)
        ix = (idx[two] - 1).t()
        for perm in hm.ERI_PERMS:
            eri[ix[perm[0]], ix[perm[1]], ix[perm[2]], ix[perm[3]]] = vals[two]
        occ = torch.as_tensor(space.occ_all, device=device)
        J = torch.einsum("pqkk->pq", eri[:, :, occ][:, :, :, occ])
        K = torch.einsum("pkkq->pq", eri[:, occ][:, :, occ])
        out = cls(space, h + 2 * J - K, eri, device)
        out.ecore = float(vals[core][-1]) if bool(core.any()) else 0.0
        return out

    def glob(self, t, so):
        return self.orbs[t][so // 2], so % 2

    def fock(self, t1, so1, t2, so2):
        (p, s1), (q, s2) = self.glob(t1, so1), self.glob(t2, so2)
        return torch.where(s1 == s2, self.f[p, q],
                           torch.zeros((), device=self.device, dtype=torch.float64))

    def eri(self, t, so):
        """<c1 c2 || a1 a2> = (c1 a1|c2 a2) - (c1 a2|c2 a1) with spin deltas"""
        (c1, s1), (c2, s2) = self.glob(t[0], so[0]), self.glob(t[1], so[1])
        (a1, r1), (a2, r2) = self.glob(t[2], so[2]), self.glob(t[3], so[3])
        direct = self.eri_pqrs[c1, a1, c2, a2] * ((s1 == r1) & (s2 == r2))
        exch = self.eri_pqrs[c1, a2, c2, a1] * ((s1 == r2) & (s2 == r1))
        return direct - exch

    def release(self):
        if self.device != "cpu":
            torch.cuda.empty_cache()


class TorchIntegrals:
    """device form of FactorizedIntegrals (diagonal Fock eps, factors B)"""

    def __init__(self, space, eps, B, device="cuda"):
        self.space = space
        self.device = device
        self.eps = torch.as_tensor(eps, device=device, dtype=torch.float64)
        self.B = torch.as_tensor(B, device=device, dtype=torch.float64)
        self.orbs = [torch.as_tensor(space.type_orbitals(t), device=device) for t in (0, 1)]
        self._mats = {}

    def glob(self, t, so):
        return self.orbs[t][so // 2], so % 2

    def fock(self, t1, so1, t2, so2):
        (p, s1), (q, s2) = self.glob(t1, so1), self.glob(t2, so2)
        return torch.where((p == q) & (s1 == s2), self.eps[p],
                           torch.zeros((), device=self.device, dtype=torch.float64))

    def mat(self, t1, t2, t3, t4):
        """spatial (pq|rs), p in t1, q in t2, r in t3, s in t4, as a matrix
        [(p,q), (r,s)]"""
        k = (t1, t2, t3, t4)
        if k in self._mats:
            return self._mats[k]
        kt = (t3, t4, t1, t2)
        if kt in self._mats:
            return self._mats[kt].t()
        o = self.orbs
        b1 = self.B[o[t1]][:, o[t2]].reshape(-1, self.B.shape[2])
        b2 = self.B[o[t3]][:, o[t4]].reshape(-1, self.B.shape[2])
        self._mats[k] = b1 @ b2.t()
        return self._mats[k]

    def eri(self, t, so):
        """<c1 c2 || a1 a2> for axis types t[0..3] and spin-orbital index tensors"""
        (c1, s1), (c2, s2) = self.glob(t[0], so[0]), self.glob(t[1], so[1])
        (a1, r1), (a2, r2) = self.glob(t[2], so[2]), self.glob(t[3], so[3])
        n = [len(self.orbs[x]) for x in range(2)]

        def gather(tp, tq, tr, ts, p, q, r, s):
            M = self.mat(tp, tq, tr, ts)
            row = (p * n[tq] + q)
            col = (r * n[ts] + s)
            return M[row, col]

        direct = gather(t[0], t[2], t[1], t[3], so[0] // 2, so[2] // 2, so[1] // 2, so[3] // 2)
        direct = direct * ((s1 == r1) & (s2 == r2))
        exch = gather(t[0], t[3], t[1], t[2], so[0] // 2, so[3] // 2, so[1] // 2, so[2] // 2)
        exch = exch * ((s1 == r2) & (s2 == r1))
        return direct - exch

    def release(self):
        self._mats.clear()
        if self.device != "cpu":
            torch.cuda.empty_cache()
