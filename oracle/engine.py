"""The oracle behind the engine's Python interface.

TEST INFRASTRUCTURE / CPU BASELINE: exposes the subset of gccu.Engine that
the CC driver uses (lists, [CONTR], [ADD], diavc, dot products) on top of the
CPU restatement in oracle.cpp, with host arrays as ME lists.  Used by the
tests as the checker and by bench.py's cpu_baseline / --impl reference legs.
"""
import numpy as np

from binding import Oracle, add_opblk, diavc


class OracleEngine:
    def __init__(self, route=3, str_block=200, cnt_block=-1):
        self.route = route
        self.str_block = str_block
        self.cnt_block = cnt_block
        self.o = None
        self.data = {}
        self.occs = {}
        self.absym = {}
        self.nblk = {}
        self.stats = np.zeros(8)

    def close(self):
        pass

    def register_orbinfo(self, nsym, norb):
        self.o = Oracle(nsym, norb)

    def strings(self, typ, nel, idxms, gam):
        return self.o.strings(typ, nel, idxms, gam)

    def define_operator(self, occs):
        oid = self.o.define_op(occs)
        self.occs[oid] = [np.asarray(x) for x in occs]
        return oid

    def register_list(self, op, gamt=1, mst=0, absym=0):
        lid, n = self.o.define_list(op, gamt, mst, absym)
        self.data[lid] = np.zeros(max(n, 1))[:n] if n else np.zeros(0)
        self.absym[lid] = absym
        self.nblk[lid] = len(self.occs[op])
        return lid, n

    def dists(self, lid):
        return self.o.dists(lid)

    def block(self, lid, iblk):
        return self.o.block(lid, iblk)

    def upload(self, lid, x):
        self.data[lid][:] = x

    def download(self, lid, n):
        return self.data[lid][:n].copy()

    def zero(self, lid):
        self.data[lid][:] = 0.0

    def set_shard(self, rank=0, nranks=1):
        from binding import set_shard
        set_shard(rank, nranks)

    def freeze(self, lid, frozen=True):
        pass  # host arrays: nothing is derived from a list

    def set_precision(self, mode):
        pass  # the oracle computes in FP64 only

    def contract(self, op1, op2, res, ex1, ex2, cnt, fact=1.0, update=True, use_tr=False,
                 xret=0, desc=None):
        (l1, b1), (l2, b2), (l12, b12) = op1, op2, res
        self.o.contract(self.route, l1, b1, self.data[l1], l2, b2, self.data[l2], l12, b12,
                        self.data[l12], ex1, ex2, cnt, fact, update=update, use_tr=use_tr,
                        str_block=self.str_block, cnt_block=self.cnt_block, stats=self.stats)
        if xret == 1:
            off, ln = self.o.block(l12, b12)
            x = self.data[l12][off:off + ln]
            return float(x @ x)
        return 0.0

    def add_block(self, fac, lin, iblk_in, lout, iblk_out, reset=False, typ=0):
        oi, ni = self.o.block(lin, iblk_in)
        oo, no = self.o.block(lout, iblk_out)
        assert ni == no
        out = self.data[lout][oo:oo + no].copy()
        xn = add_opblk(out, np.ascontiguousarray(self.data[lin][oi:oi + ni]), fac, reset, typ or 1)
        self.data[lout][oo:oo + no] = out
        return xn

    def scale(self, lid, fac):
        self.data[lid] *= fac

    def dot(self, a, b):
        return float(self.data[a] @ self.data[b])

    def precondition(self, out, inp, diag, fac=1.0, shift=0.0):
        self.data[out][:] = diavc(self.data[inp], self.data[diag], fac, shift)

    def sym_ab(self, lid, iblk, prefac=0.5, relfac=1.0):
        self.o.sym_ab(lid, iblk, self.data[lid], prefac, relfac)

    def spin_prj(self, lid, nblk=0, s2=0):
        xn = self.o.spin_prj(lid, self.data[lid], self.nblk[lid], s2)
        return xn[:nblk] if nblk else None

    def graph_begin(self):
        raise NotImplementedError("no graphs on the CPU oracle")

    def sync(self):
        pass
