"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline legs import this module, and only as the checker / timed CPU
baseline.  The product library never loads the oracle.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

I64 = ctypes.c_int64
P64 = ctypes.POINTER(ctypes.c_int64)
PD = ctypes.POINTER(ctypes.c_double)


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.ora_create.restype = ctypes.c_void_p
        L.ora_create.argtypes = [I64, P64]
        L.ora_destroy.argtypes = [ctypes.c_void_p]
        L.ora_last_error.restype = ctypes.c_char_p
        L.ora_graph_nstr.restype = I64
        L.ora_graph_nstr.argtypes = [ctypes.c_void_p, I64, I64, I64, I64]
        L.ora_graph_strings.restype = I64
        L.ora_graph_strings.argtypes = [ctypes.c_void_p, I64, I64, I64, I64, P64, P64]
        L.ora_strmap_block.restype = I64
        L.ora_strmap_block.argtypes = [ctypes.c_void_p] + [I64] * 7 + [P64]
        L.ora_define_op.restype = I64
        L.ora_define_op.argtypes = [ctypes.c_void_p, P64, I64]
        L.ora_trace.argtypes = [ctypes.c_void_p, I64, I64, PD, I64, I64, PD, P64,
                                ctypes.c_double, I64]
        L.ora_define_op_joined.restype = I64
        L.ora_define_op_joined.argtypes = [ctypes.c_void_p, P64, I64, I64]
        L.ora_reorder.argtypes = [ctypes.c_void_p, I64, I64, PD, I64, I64, PD, I64, P64, P64,
                                  P64, ctypes.c_double, I64, I64]
        L.ora_define_list.restype = I64
        L.ora_define_list.argtypes = [ctypes.c_void_p, I64, I64, I64, I64, P64]
        L.ora_list_block.restype = ctypes.c_int
        L.ora_list_block.argtypes = [ctypes.c_void_p, I64, I64, P64, P64]
        L.ora_list_dists.restype = I64
        L.ora_list_dists.argtypes = [ctypes.c_void_p, I64, P64, I64]
        L.ora_contract.restype = ctypes.c_int
        L.ora_contract.argtypes = ([ctypes.c_void_p, I64, I64, I64, PD, I64, I64, PD, I64, I64,
                                    PD, P64, P64, P64, ctypes.c_double, I64, I64, I64, I64, PD,
                                    PD])
        L.ora_contract_t.restype = ctypes.c_int
        L.ora_contract_t.argtypes = ([ctypes.c_void_p, I64, I64, I64, PD, I64, I64, PD, I64, I64,
                                      PD, P64, P64, P64, ctypes.c_double, I64, I64, I64, I64, I64,
                                      PD])
        L.ora_sym_ab_blk.restype = ctypes.c_int
        L.ora_sym_ab_blk.argtypes = [ctypes.c_void_p, I64, I64, PD, ctypes.c_double,
                                     ctypes.c_double]
        L.ora_spin_prj_list.restype = ctypes.c_int
        L.ora_spin_prj_list.argtypes = [ctypes.c_void_p, I64, I64, PD, PD]
        L.ora_add_opblk.restype = ctypes.c_int
        L.ora_add_opblk.argtypes = [PD, I64, ctypes.c_double, PD, PD, I64, I64]
        L.ora_diavc.restype = None
        L.ora_diavc.argtypes = [PD, PD, ctypes.c_double, PD, ctypes.c_double, I64]
        _lib = L
    return _lib


def _p64(a):
    return a.ctypes.data_as(P64)


def _pd(a):
    return a.ctypes.data_as(PD)


class OracleError(RuntimeError):
    pass


def _chk(rc):
    if rc is None or (isinstance(rc, int) and rc < 0):
        raise OracleError(lib().ora_last_error().decode())
    return rc


class Oracle:
    """CPU restatement of the reference path for one orbital space."""

    def __init__(self, nsym, norb):
        L = lib()
        a = np.zeros(32, dtype=np.int64)
        norb = np.asarray(norb, dtype=np.int64)
        a.reshape(4, 8)[:, : norb.shape[1]] = norb
        self._keep = a
        self.ctx = L.ora_create(nsym, _p64(a))
        if not self.ctx:
            raise OracleError(L.ora_last_error().decode())
        self.nsym = nsym

    def __del__(self):
        if getattr(self, "ctx", None) and _lib is not None:
            _lib.ora_destroy(self.ctx)
            self.ctx = None

    def nstr(self, typ, nel, idxms, gam):
        return _chk(lib().ora_graph_nstr(self.ctx, typ, nel, idxms, gam))

    def strings(self, typ, nel, idxms, gam):
        n = self.nstr(typ, nel, idxms, gam)
        orb = np.zeros(max(n * nel, 1), dtype=np.int64)
        spn = np.zeros(max(n * nel, 1), dtype=np.int64)
        _chk(lib().ora_graph_strings(self.ctx, typ, nel, idxms, gam, _p64(orb), _p64(spn)))
        return orb[: n * nel].reshape(n, nel), spn[: n * nel].reshape(n, nel)

    def strmap(self, typ, nel1, nel2, idxms1, idxms2, gam1, gam2):
        n1 = self.nstr(typ, nel1, idxms1, gam1)
        n2 = self.nstr(typ, nel2, idxms2, gam2)
        m = np.zeros(max(n1 * n2, 1), dtype=np.int64)
        _chk(lib().ora_strmap_block(self.ctx, typ, nel1, nel2, idxms1, idxms2, gam1, gam2,
                                    _p64(m)))
        return m[: n1 * n2].reshape(n2, n1)

    def define_op(self, occ):
        occ = np.ascontiguousarray(np.asarray(occ, dtype=np.int64).reshape(-1, 8))
        return _chk(lib().ora_define_op(self.ctx, _p64(occ), occ.shape[0]))

    def define_op_joined(self, occ, nj):
        occ = np.ascontiguousarray(np.asarray(occ, dtype=np.int64).reshape(-1, 8))
        assert occ.shape[0] % nj == 0
        return _chk(lib().ora_define_op_joined(self.ctx, _p64(occ), nj, occ.shape[0] // nj))

    def reorder(self, lori, bori, xori, lreo, breo, xreo, shifts, fac=1.0, sign_reo=1,
                update=True):
        """reo_op_wmaps_c: shifts = [(occ8, from_vtx, to_vtx), ...] (1-based);
        xreo (the whole reordered list) is updated in place"""
        n = len(shifts)
        occ = np.zeros((max(n, 1), 8), dtype=np.int64)
        fr = np.zeros(max(n, 1), dtype=np.int64)
        to = np.zeros(max(n, 1), dtype=np.int64)
        for s, (o, f, t) in enumerate(shifts):
            occ[s] = np.asarray(o).reshape(8)
            fr[s], to[s] = f, t
        _chk(lib().ora_reorder(self.ctx, lori, bori, _pd(xori), lreo, breo, _pd(xreo), n,
                               _p64(occ), _p64(fr), _p64(to), fac, sign_reo, int(update)))

    def trace(self, lop, bop, xop, lres, bres, xres, cnt, fac=1.0, update=True):
        """trace_op: xres (whole result list) += fac * sum_J xop(IC*J, IA*J)"""
        c = np.ascontiguousarray(np.asarray(cnt, dtype=np.int64).reshape(8))
        _chk(lib().ora_trace(self.ctx, lop, bop, _pd(xop), lres, bres, _pd(xres), _p64(c), fac,
                             int(update)))

    def define_list(self, op, gamt=1, mst=0, absym=0):
        ln = np.zeros(1, dtype=np.int64)
        lid = _chk(lib().ora_define_list(self.ctx, op, gamt, mst, absym, _p64(ln)))
        return lid, int(ln[0])

    def block(self, lst, iblk):
        off = np.zeros(1, dtype=np.int64)
        ln = np.zeros(1, dtype=np.int64)
        _chk(lib().ora_list_block(self.ctx, lst, iblk, _p64(off), _p64(ln)))
        return int(off[0]), int(ln[0])

    def dists(self, lst):
        n = _chk(lib().ora_list_dists(self.ctx, lst, _p64(np.zeros(8, np.int64)), 0))
        rows = np.zeros((max(n, 1), 8), dtype=np.int64)
        _chk(lib().ora_list_dists(self.ctx, lst, _p64(rows), n))
        return rows[:n]

    def contract(self, route, l1, b1, x1, l2, b2, x2, l12, b12, x12, ex1, ex2, cnt, fact,
                 update=True, use_tr=False, str_block=200, cnt_block=-1, stats=None,
                 tra=(0, 0, 0)):
        """x12 is updated in place (whole list buffer).  Returns xret.
        tra = (tra_op1, tra_op2, tra_res): classes used as their adjoints."""
        xret = np.zeros(1)
        if b12 == 0:
            xret[0] = 0.0 if not update else (x12[0] if x12 is not None and x12.size else 0.0)
        e1 = np.ascontiguousarray(np.asarray(ex1, dtype=np.int64).reshape(8))
        e2 = np.ascontiguousarray(np.asarray(ex2, dtype=np.int64).reshape(8))
        cn = np.ascontiguousarray(np.asarray(cnt, dtype=np.int64).reshape(8))
        st = stats if stats is not None else np.zeros(8)
        dummy = np.zeros(1)
        if any(tra):
            rc = lib().ora_contract_t(self.ctx, route, l1, b1, _pd(x1), l2, b2, _pd(x2), l12,
                                      b12, _pd(x12 if x12 is not None else dummy), _p64(e1),
                                      _p64(e2), _p64(cn), fact, int(update), int(use_tr),
                                      int(tra[0]), int(tra[1]), int(tra[2]), _pd(xret))
        else:
            rc = lib().ora_contract(self.ctx, route, l1, b1, _pd(x1), l2, b2, _pd(x2), l12, b12,
                                    _pd(x12 if x12 is not None else dummy), _p64(e1), _p64(e2),
                                    _p64(cn), fact, int(update), int(use_tr), str_block,
                                    cnt_block, _pd(xret), _pd(st))
        _chk(rc)
        return float(xret[0])

    def add_transp(self, fac, lin, bin_, xin, lout, bout, xout, tra_in, tra_out, reset=False,
                   typ=1):
        """add_opblk_transp: out(IC,IA) += fac * in(IA,IC) (xout updated in place)"""
        L = lib()
        L.ora_add_opblk_transp.restype = ctypes.c_int
        L.ora_add_opblk_transp.argtypes = [ctypes.c_void_p, PD, I64, ctypes.c_double, I64, I64,
                                           PD, I64, I64, PD, I64, I64, I64]
        xn = np.zeros(1)
        _chk(L.ora_add_opblk_transp(self.ctx, _pd(xn), typ, fac, lin, bin_,
                                    _pd(np.ascontiguousarray(xin)), lout, bout, _pd(xout),
                                    int(tra_in), int(tra_out), int(reset)))
        return float(xn[0])

    def spin_prj(self, lst, x, nblk, s2=0):
        """spin_prj_list: x (the whole list) projected onto its singlet part in
        place; returns the squared norm of every occupation class"""
        xn = np.zeros(max(nblk, 1))
        _chk(lib().ora_spin_prj_list(self.ctx, lst, s2, _pd(x), _pd(xn)))
        return xn[:nblk]

    def sym_ab(self, lst, iblk, x, prefac=0.5, relfac=1.0):
        _chk(lib().ora_sym_ab_blk(self.ctx, lst, iblk, _pd(x), prefac, relfac))


def openblas_path():
    import glob

    import numpy
    libs = glob.glob(os.path.join(os.path.dirname(numpy.__file__) + ".libs",
                                  "libscipy_openblas64_*.so"))
    return libs[0] if libs else None


def set_blas(nthreads=0, path=None):
    """route-3 dgemm through the ILP64 OpenBLAS bundled with numpy"""
    L = lib()
    L.ora_set_blas.restype = ctypes.c_int
    L.ora_set_blas.argtypes = [ctypes.c_char_p, I64]
    path = path or openblas_path()
    if path is None:
        raise OracleError("no ILP64 OpenBLAS found")
    _chk(L.ora_set_blas(path.encode(), nthreads))
    return path


def set_shard(rank, nranks):
    """each contraction computes only the block contractions dealt to this rank"""
    L = lib()
    L.ora_set_shard.argtypes = [I64, I64]
    L.ora_set_shard.restype = None
    L.ora_set_shard(rank, nranks)


def sampling(stride):
    L = lib()
    L.ora_sampling.argtypes = [I64]
    L.ora_sampling.restype = None
    L.ora_sampling(stride)


def sampling_report():
    L = lib()
    L.ora_sampling_report.argtypes = [PD]
    L.ora_sampling_report.restype = None
    out = np.zeros(6)
    L.ora_sampling_report(_pd(out))
    return dict(t_short=out[0], t_sampled=out[1], batches=int(out[2]), done=int(out[3]),
                shorts=int(out[4]), shorts_done=int(out[5]))


def scaled_time(wall, rep):
    """wall time of a sampled evaluation scaled to the full work: the
    executed long-operand batches scaled by their count (every short-operand
    gather and everything outside route 3 runs in full)"""
    return wall + rep["t_sampled"] * (rep["batches"] / max(rep["done"], 1) - 1.0)


def add_opblk(xout, xin, fac, reset=False, typ=1):
    xn = np.zeros(1)
    lib().ora_add_opblk(_pd(xn), typ, fac, _pd(xin), _pd(xout), xout.size, int(reset))
    return float(xn[0])


def diavc(vin, diag, fac=1.0, shift=0.0):
    out = np.zeros_like(vin)
    lib().ora_diavc(_pd(out), _pd(np.ascontiguousarray(vin)), fac,
                    _pd(np.ascontiguousarray(diag)), shift, vin.size)
    return out
