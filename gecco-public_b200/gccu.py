"""Python binding of the engine's C ABI (include/gccu.h) over ctypes.

The reference drives this path from Fortran (frm_sched2 -> fs_contr_drv ->
contr_op1op2, contract/frm_sched2.f:288-306); here the same calls are made
from Python for the tests, the solver driver and the benchmark.  The library
is the in-tree build ``gecco-public_b200/libgccu.so``; nothing falls back to a
CPU implementation: a missing library is an error.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgccu.so")

I64 = ctypes.c_int64
P64 = ctypes.POINTER(ctypes.c_int64)
PD = ctypes.POINTER(ctypes.c_double)

H, P, V, X = 0, 1, 2, 3  # hpvx types
LP_NWEIGHTS = 1217  # weights of the learned preconditioner (GCCU_LP_NWEIGHTS)


class BcDesc(ctypes.Structure):
    _fields_ = [("list_op1", I64), ("iblk_op1", I64), ("list_op2", I64), ("iblk_op2", I64),
                ("list_res", I64), ("iblk_res", I64), ("tra_op1", I64), ("tra_op2", I64),
                ("tra_res", I64), ("occ_ex1", I64 * 8), ("occ_ex2", I64 * 8),
                ("occ_cnt", I64 * 8)]


class ReoDesc(ctypes.Structure):
    _fields_ = [("list_ori", I64), ("iblk_ori", I64), ("list_reo", I64), ("iblk_reo", I64),
                ("nshift", I64), ("occ_shift", (I64 * 8) * 4), ("from_vtx", I64 * 4),
                ("to_vtx", I64 * 4)]


# commands of a formula item (include/gccu.h)
CMD_TARGET, CMD_NEW, CMD_DEL, CMD_ADD, CMD_CONTR, CMD_REORDER = 1, 2, 3, 4, 5, 6


class FormulaItem(ctypes.Structure):
    _fields_ = [("command", I64), ("list", I64), ("init", I64), ("mult", I64), ("list_in", I64),
                ("iblk_in", I64), ("iblk_out", I64), ("reset", I64), ("tra_in", I64),
                ("tra_out", I64), ("update", I64), ("use_tr", I64), ("sign_reo", I64),
                ("fac", ctypes.c_double), ("bc", BcDesc), ("reo", ReoDesc)]


class GccuError(RuntimeError):
    pass


_lib = None

_SIGS = {
    "gccu_init": [I64, I64],
    "gccu_finalize": [],
    "gccu_last_error": [ctypes.c_char_p, I64],
    "gccu_register_orbinfo": [I64, P64],
    "gccu_graph_nstr": [I64, I64, I64, I64, P64],
    "gccu_graph_index": [I64, I64, P64, P64, P64],
    "gccu_graph_strings": [I64, I64, I64, I64, P64, P64, I64, P64],
    "gccu_strmap_block": [I64, I64, I64, I64, I64, I64, I64, P64, I64],
    "gccu_define_operator": [P64, I64, P64],
    "gccu_define_operator_joined": [P64, I64, I64, P64],
    "gccu_reorder": [ctypes.POINTER(ReoDesc), ctypes.c_double, I64, I64, I64, PD],
    "gccu_reorder_info": [ctypes.POINTER(ReoDesc), P64, P64],
    "gccu_trace": [I64, I64, I64, I64, P64, ctypes.c_double, I64, I64, PD],
    "gccu_set_precision": [I64],
    "gccu_set_wait_limit": [I64],
    "gccu_set_shard": [I64, I64],
    "gccu_set_tuning": [I64, I64],
    "gccu_tuning_report": [PD, I64, P64],
    "gccu_plan_stats": [PD],
    "gccu_lp_set_weights": [PD, I64],
    "gccu_lp_get_weights": [PD, I64],
    "gccu_lp_precondition": [I64, I64, I64, I64, ctypes.c_double, ctypes.c_double],
    "gccu_lp_rows": [I64, I64, I64, I64, ctypes.c_double, ctypes.c_double, P64, I64, PD],
    "gccu_lp_load_samples": [PD, PD, I64],
    "gccu_lp_gradient": [PD, PD],
    "gccu_lp_train": [I64, I64, ctypes.c_double, I64, PD],
    "gccu_mem_info": [P64, P64],
    "gccu_device_info": [P64],
    "gccu_trace_info": [I64, I64, I64, I64, P64, P64, P64],
    "gccu_register_list": [I64, I64, I64, I64, P64, P64],
    "gccu_list_block": [I64, I64, P64, P64],
    "gccu_list_dists": [I64, P64, I64, P64],
    "gccu_upload_list": [I64, PD, I64],
    "gccu_download_list": [I64, PD, I64],
    "gccu_zero_list": [I64],
    "gccu_list_device_ptr": [I64, ctypes.POINTER(ctypes.c_void_p)],
    "gccu_freeze_list": [I64, I64],
    "gccu_contract": [ctypes.POINTER(BcDesc), ctypes.c_double, I64, I64, I64, PD],
    "gccu_plan_info": [ctypes.POINTER(BcDesc), I64, P64, PD],
    "gccu_plan_items": [ctypes.POINTER(BcDesc), I64, P64, I64, P64],
    "gccu_contract_noalloc": [ctypes.POINTER(BcDesc), ctypes.c_double, I64, I64],
    "gccu_add_block": [ctypes.c_double, I64, I64, I64, I64, I64, I64, PD],
    "gccu_scale_list": [I64, ctypes.c_double],
    "gccu_add_block_transp": [ctypes.c_double, I64, I64, I64, I64, I64, I64, I64, I64, PD],
    "gccu_dot_lists": [I64, I64, PD],
    "gccu_sym_ab": [I64, I64, ctypes.c_double, ctypes.c_double],
    "gccu_spin_prj_list": [I64, I64, PD],
    "gccu_register_intermediate": [I64, I64, I64, I64, P64, P64],
    "gccu_formula_define": [ctypes.c_void_p, I64, P64],
    "gccu_formula_run": [I64, PD, I64],
    "gccu_formula_info": [I64, P64],
    "gccu_intermediate_offset": [I64, P64],
    "gccu_precondition": [I64, I64, I64, ctypes.c_double, ctypes.c_double],
    "gccu_graph_begin": [],
    "gccu_graph_end": [P64],
    "gccu_graph_launch": [I64],
    "gccu_sync": [],
    "gccu_stats": [PD, P64],
    "gccu_reset_stats": [],
    "gccu_put_vec": [I64, I64, ctypes.c_void_p, I64],
    "gccu_get_vec": [I64, I64, ctypes.c_void_p, I64],
    "gccu_event_record": [I64],
    "gccu_event_elapsed": [I64, I64, PD],
    "gccu_profile": [I64],
    "gccu_profile_report": [PD, I64, P64],
}


def build(verbose=False):
    """Compile libgccu.so in-tree for sm_100a (nvcc cross-compiles, no GPU needed)."""
    cmd = ["make", "-C", HERE, "-j8"]
    if verbose:
        subprocess.check_call(cmd)
    else:
        subprocess.check_call(cmd, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GccuError(f"engine library {LIB_PATH} is missing: build it with "
                            "`make -C gecco-public_b200` (or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def exported_symbols():
    return sorted(_SIGS)


def _err():
    buf = ctypes.create_string_buffer(1024)
    lib().gccu_last_error(buf, 1024)
    return buf.value.decode()


def _call(name, *args):
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise GccuError(f"{name}: {_err()}")


def _p64(a):
    return a.ctypes.data_as(P64)


def _pd(a):
    return a.ctypes.data_as(PD)


def occ8(c=None, a=None):
    """occupation [C(H,P,V,X), A(H,P,V,X)] from dicts {type: count}"""
    v = np.zeros(8, dtype=np.int64)
    for t, n in (c or {}).items():
        v[t] = n
    for t, n in (a or {}).items():
        v[4 + t] = n
    return v


class Engine:
    """One engine instance (the library keeps one global engine per process)."""

    def __init__(self, device=0, memmax=0):
        _call("gccu_init", device, memmax)
        self.device = device
        self._alive = True

    def close(self):
        if self._alive:
            _call("gccu_finalize")
            self._alive = False

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- orbital space / graphs
    def register_orbinfo(self, nsym, norb):
        a = np.zeros((4, 8), dtype=np.int64)
        norb = np.asarray(norb, dtype=np.int64)
        a[:, : norb.shape[1]] = norb
        self._norb = a.copy()
        _call("gccu_register_orbinfo", nsym, _p64(a.reshape(-1)))

    def nstr(self, typ, nel, idxms, gam):
        r = np.zeros(1, np.int64)
        _call("gccu_graph_nstr", typ, nel, idxms, gam, _p64(r))
        return int(r[0])

    def string_index(self, typ, orb, spn):
        orb = np.ascontiguousarray(orb, dtype=np.int64)
        spn = np.ascontiguousarray(spn, dtype=np.int64)
        r = np.zeros(1, np.int64)
        _call("gccu_graph_index", typ, orb.size, _p64(orb), _p64(spn), _p64(r))
        return int(r[0])

    def strings(self, typ, nel, idxms, gam):
        """strings of one graph block in address order: (orb[n,nel] 1-based, spn[n,nel])"""
        n = np.zeros(1, np.int64)
        e = np.zeros(1, np.int64)
        _call("gccu_graph_strings", typ, nel, idxms, gam, _p64(e), _p64(e), 0, _p64(n))
        ns = int(n[0])
        orb = np.zeros(max(ns * nel, 1), np.int64)
        spn = np.zeros(max(ns * nel, 1), np.int64)
        _call("gccu_graph_strings", typ, nel, idxms, gam, _p64(orb), _p64(spn), ns, _p64(n))
        return orb[: ns * nel].reshape(ns, nel), spn[: ns * nel].reshape(ns, nel)

    def strmap(self, typ, nel1, nel2, idxms1, idxms2, gam1, gam2):
        n1 = self.nstr(typ, nel1, idxms1, gam1)
        n2 = self.nstr(typ, nel2, idxms2, gam2)
        m = np.zeros(max(n1 * n2, 1), np.int64)
        _call("gccu_strmap_block", typ, nel1, nel2, idxms1, idxms2, gam1, gam2, _p64(m), m.size)
        return m[: n1 * n2].reshape(n2, n1)

    # ---- operators / lists
    def define_operator(self, occs):
        o = np.ascontiguousarray(np.asarray(occs, dtype=np.int64).reshape(-1, 8))
        r = np.zeros(1, np.int64)
        _call("gccu_define_operator", _p64(o), o.shape[0], _p64(r))
        return int(r[0])

    def define_operator_joined(self, occs, njoined):
        """joined operator: occs has nblk*njoined occupations, the vertices of
        a class consecutive"""
        o = np.ascontiguousarray(np.asarray(occs, dtype=np.int64).reshape(-1, 8))
        assert o.shape[0] % njoined == 0
        r = np.zeros(1, np.int64)
        _call("gccu_define_operator_joined", _p64(o), njoined, o.shape[0] // njoined, _p64(r))
        return int(r[0])

    @staticmethod
    def reo_desc(ori, reo, shifts):
        """ori/reo = (list, iblk); shifts = [(occ8, from_vtx, to_vtx), ...] (1-based)"""
        d = ReoDesc()
        d.list_ori, d.iblk_ori = ori
        d.list_reo, d.iblk_reo = reo
        d.nshift = len(shifts)
        for s, (occ, fr, to) in enumerate(shifts):
            for k, v in enumerate(np.asarray(occ).reshape(8)):
                d.occ_shift[s][k] = int(v)
            d.from_vtx[s] = fr
            d.to_vtx[s] = to
        return d

    def reorder(self, ori, reo, shifts, fac=1.0, sign_reo=1, update=True, xret=0):
        d = self.reo_desc(ori, reo, shifts)
        r = np.zeros(1)
        _call("gccu_reorder", ctypes.byref(d), fac, sign_reo, int(update), xret, _pd(r))
        return float(r[0])

    def reorder_info(self, ori, reo, shifts):
        d = self.reo_desc(ori, reo, shifts)
        n = np.zeros(1, np.int64)
        m = np.zeros(1, np.int64)
        _call("gccu_reorder_info", ctypes.byref(d), _p64(n), _p64(m))
        return int(n[0]), int(m[0])

    def set_precision(self, mode):
        """0 = FP64 (default), 1 = split TF32 on the tcgen05 tensor cores,
        2 = FP64 emulated with five int8 slices on the tcgen05 tensor
        cores, 3 = the same with four slices"""
        _call("gccu_set_precision", int(mode))

    # ---- learned correction of the diagonal step
    def lp_set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        _call("gccu_lp_set_weights", _pd(w), w.size)

    def lp_get_weights(self):
        w = np.zeros(LP_NWEIGHTS)
        _call("gccu_lp_get_weights", _pd(w), w.size)
        return w

    def lp_precondition(self, out, inp, diag, prev=0, fac=1.0, shift=0.0):
        _call("gccu_lp_precondition", out, inp, diag, prev, fac, shift)

    def lp_rows(self, inp, diag, prev, amp, idx, fac=1.0, shift=0.0):
        """(x0, x1, x2, plain step, amplitude) of the elements idx"""
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        rows = np.zeros((max(idx.size, 1), 5))
        _call("gccu_lp_rows", inp, diag, prev, amp, fac, shift, _p64(idx), idx.size, _pd(rows))
        return rows[: idx.size]

    def lp_load_samples(self, rows, target):
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        target = np.ascontiguousarray(target, dtype=np.float64)
        assert rows.shape == (target.size, 5)
        _call("gccu_lp_load_samples", _pd(rows), _pd(target), target.size)

    def lp_gradient(self):
        g = np.zeros(LP_NWEIGHTS)
        l = np.zeros(1)
        _call("gccu_lp_gradient", _pd(g), _pd(l))
        return g, float(l[0])

    def lp_train(self, steps, batch, lr, seed=0):
        l = np.zeros(1)
        _call("gccu_lp_train", steps, batch, lr, seed, _pd(l))
        return float(l[0])

    def set_tuning(self, mode, candidate=0):
        """0 fixed tile rule, 1 autotune at first call, 2 force a candidate"""
        _call("gccu_set_tuning", int(mode), int(candidate))

    def tuning_report(self):
        """rows (block contractions, chosen candidate, ms per candidate...)"""
        n = np.zeros(1, np.int64)
        rows = np.zeros((256, 8))
        _call("gccu_tuning_report", _pd(rows), 256, _p64(n))
        return rows[: min(int(n[0]), 256)]

    def plan_stats(self):
        """{"plans", "host_s", "maps_s", "tune_s", "build_s"}: time spent
        making contraction plans, by stage"""
        out = np.zeros(10)
        _call("gccu_plan_stats", _pd(out))
        keys = ("plans", "host_s", "maps_s", "tune_s", "build_s", "tables_s", "upload_s",
                "const_s", "desc_s", "alloc_s")
        return {k: (int(v) if k == "plans" else float(v)) for k, v in zip(keys, out)}

    def set_shard(self, rank=0, nranks=1):
        """run only this rank's share of every contraction's output tiles"""
        _call("gccu_set_shard", int(rank), int(nranks))

    def set_wait_limit(self, polls=-1):
        """mbarrier polls per tensor-core pipeline wait (negative: default)"""
        _call("gccu_set_wait_limit", int(polls))

    def mem_info(self):
        """(bytes of device memory the engine holds, its cap or 0)"""
        u = np.zeros(1, np.int64)
        c = np.zeros(1, np.int64)
        _call("gccu_mem_info", _p64(u), _p64(c))
        return int(u[0]), int(c[0])

    def device_info(self):
        """(compute capability, SMs, binary version and PTX version of the
        tensor-core kernel)"""
        r = np.zeros(4, np.int64)
        _call("gccu_device_info", _p64(r))
        return tuple(int(x) for x in r)

    def trace(self, op, res, cnt, fact=1.0, update=True, xret=0):
        """partial trace res(IC,IA) += fact * sum_J op(IC*J, IA*J); op/res =
        (list, iblk), cnt = occupation of J (creators = annihilators)"""
        c = np.ascontiguousarray(np.asarray(cnt, dtype=np.int64).reshape(8))
        r = np.zeros(1)
        _call("gccu_trace", op[0], op[1], res[0], res[1], _p64(c), fact, int(update), xret,
              _pd(r))
        return float(r[0])

    def trace_info(self, op, res, cnt):
        c = np.ascontiguousarray(np.asarray(cnt, dtype=np.int64).reshape(8))
        n = np.zeros(1, np.int64)
        m = np.zeros(1, np.int64)
        _call("gccu_trace_info", op[0], op[1], res[0], res[1], _p64(c), _p64(n), _p64(m))
        return int(n[0]), int(m[0])

    def register_list(self, op, gamt=1, mst=0, absym=0):
        lid = np.zeros(1, np.int64)
        ln = np.zeros(1, np.int64)
        _call("gccu_register_list", op, gamt, mst, absym, _p64(lid), _p64(ln))
        return int(lid[0]), int(ln[0])

    def register_intermediate(self, op, gamt=1, mst=0, absym=0):
        """a list without memory of its own, placed in the arena of the
        formula whose [NEW] names it"""
        lid = np.zeros(1, np.int64)
        ln = np.zeros(1, np.int64)
        _call("gccu_register_intermediate", op, gamt, mst, absym, _p64(lid), _p64(ln))
        return int(lid[0]), int(ln[0])

    def formula_define(self, items):
        """items: FormulaItem sequence; returns the formula id"""
        arr = (FormulaItem * max(len(items), 1))(*items)
        fid = np.zeros(1, np.int64)
        _call("gccu_formula_define", ctypes.cast(arr, ctypes.c_void_p), len(items), _p64(fid))
        return int(fid[0])

    def formula_run(self, fid, ntargets=0):
        """run a formula; with ntargets > 0 return the targets' values"""
        if ntargets:
            r = np.zeros(ntargets)
            _call("gccu_formula_run", fid, _pd(r), ntargets)
            return r
        _call("gccu_formula_run", fid, PD(), 0)
        return None

    def formula_info(self, fid):
        r = np.zeros(4, np.int64)
        _call("gccu_formula_info", fid, _p64(r))
        return dict(arena_bytes=int(r[0]), sum_bytes=int(r[1]), targets=int(r[2]),
                    items=int(r[3]))

    def intermediate_offset(self, lst):
        r = np.zeros(1, np.int64)
        _call("gccu_intermediate_offset", lst, _p64(r))
        return int(r[0])

    def block(self, lst, iblk):
        off = np.zeros(1, np.int64)
        ln = np.zeros(1, np.int64)
        _call("gccu_list_block", lst, iblk, _p64(off), _p64(ln))
        return int(off[0]), int(ln[0])

    def dists(self, lst):
        n = np.zeros(1, np.int64)
        _call("gccu_list_dists", lst, _p64(np.zeros(8, np.int64)), 0, _p64(n))
        rows = np.zeros((max(int(n[0]), 1), 8), np.int64)
        _call("gccu_list_dists", lst, _p64(rows), int(n[0]), _p64(n))
        return rows[: int(n[0])]

    def upload(self, lst, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        _call("gccu_upload_list", lst, _pd(x), x.size)

    def download(self, lst, n):
        x = np.zeros(n)
        _call("gccu_download_list", lst, _pd(x), n)
        return x

    def zero(self, lst):
        _call("gccu_zero_list", lst)

    def freeze(self, lst, frozen=True):
        """declare a list constant (contractions then cache the panels they
        derive from it) or release it"""
        _call("gccu_freeze_list", lst, int(frozen))

    def device_ptr(self, lst):
        p = ctypes.c_void_p()
        _call("gccu_list_device_ptr", lst, ctypes.byref(p))
        return p.value

    # ---- contraction / vector operations
    @staticmethod
    def desc(op1, op2, res, ex1, ex2, cnt, tra=(0, 0, 0)):
        """tra = (tra_op1, tra_op2, tra_res): classes used as their adjoints"""
        d = BcDesc()
        d.list_op1, d.iblk_op1 = op1
        d.list_op2, d.iblk_op2 = op2
        d.list_res, d.iblk_res = res
        d.tra_op1, d.tra_op2, d.tra_res = (int(t) for t in tra)
        for k in range(8):
            d.occ_ex1[k] = int(ex1[k])
            d.occ_ex2[k] = int(ex2[k])
            d.occ_cnt[k] = int(cnt[k])
        return d

    def contract(self, op1, op2, res, ex1, ex2, cnt, fact=1.0, update=True, use_tr=False,
                 xret=0, desc=None, tra=(0, 0, 0)):
        d = desc if desc is not None else self.desc(op1, op2, res, ex1, ex2, cnt, tra)
        r = np.zeros(1)
        _call("gccu_contract", ctypes.byref(d), fact, int(update), int(use_tr), xret, _pd(r))
        return float(r[0])

    def contract_noalloc(self, op1, op2, res, ex1, ex2, cnt, fact=1.0, update=True,
                         use_tr=False, desc=None):
        """gccu_contract_noalloc: a contraction already run once through
        contract(), with its operand panels in the library's fixed device
        array; allocates nothing"""
        d = desc if desc is not None else self.desc(op1, op2, res, ex1, ex2, cnt)
        _call("gccu_contract_noalloc", ctypes.byref(d), fact, int(update), int(use_tr))

    def plan_info(self, op1, op2, res, ex1, ex2, cnt, use_tr=False, tra=(0, 0, 0)):
        d = self.desc(op1, op2, res, ex1, ex2, cnt, tra)
        n = np.zeros(1, np.int64)
        st = np.zeros(8)
        _call("gccu_plan_info", ctypes.byref(d), int(use_tr), _p64(n), _pd(st))
        return int(n[0]), st

    def plan_items(self, op1, op2, res, ex1, ex2, cnt, use_tr=False, tra=(0, 0, 0)):
        """rows (M, N, K, maps op1, maps op2, maps result, kfast1, kfast2) of
        the planned block contractions"""
        d = self.desc(op1, op2, res, ex1, ex2, cnt, tra)
        n = np.zeros(1, np.int64)
        _call("gccu_plan_items", ctypes.byref(d), int(use_tr), _p64(np.zeros(8, np.int64)), 0,
              _p64(n))
        rows = np.zeros((max(int(n[0]), 1), 8), np.int64)
        _call("gccu_plan_items", ctypes.byref(d), int(use_tr), _p64(rows), int(n[0]), _p64(n))
        return rows[: int(n[0])]

    def add_block(self, fac, lin, iblk_in, lout, iblk_out, reset=False, typ=0):
        r = np.zeros(1)
        _call("gccu_add_block", fac, lin, iblk_in, lout, iblk_out, int(reset), typ, _pd(r))
        return float(r[0])

    def add_block_transp(self, fac, lin, iblk_in, lout, iblk_out, tra_in=True, tra_out=False,
                         reset=False, typ=0):
        """out(IC,IA) = (reset ? 0 : out) + fac*in(IA,IC) (add_opblk_transp)"""
        r = np.zeros(1)
        _call("gccu_add_block_transp", fac, lin, iblk_in, lout, iblk_out, int(tra_in),
              int(tra_out), int(reset), typ, _pd(r))
        return float(r[0])

    def scale(self, lst, fac):
        _call("gccu_scale_list", lst, fac)

    def dot(self, a, b):
        r = np.zeros(1)
        _call("gccu_dot_lists", a, b, _pd(r))
        return float(r[0])

    def sym_ab(self, lst, iblk, prefac=0.5, relfac=1.0):
        _call("gccu_sym_ab", lst, iblk, prefac, relfac)

    def spin_prj(self, lst, nblk=0, s2=0):
        """project the list onto its singlet part in place (spin_prj_list);
        with nblk > 0 return the squared norm of each of its nblk classes"""
        if nblk:
            r = np.zeros(nblk)
            _call("gccu_spin_prj_list", lst, s2, _pd(r))
            return r
        _call("gccu_spin_prj_list", lst, s2, PD())
        return None

    def precondition(self, out, inp, diag, fac=1.0, shift=0.0):
        _call("gccu_precondition", out, inp, diag, fac, shift)

    # ---- graphs / sync / stats
    def graph_begin(self):
        _call("gccu_graph_begin")

    def graph_end(self):
        r = np.zeros(1, np.int64)
        _call("gccu_graph_end", _p64(r))
        return int(r[0])

    def graph_launch(self, gid):
        _call("gccu_graph_launch", gid)

    def sync(self):
        _call("gccu_sync")

    def stats(self):
        st = np.zeros(8)
        n = np.zeros(1, np.int64)
        _call("gccu_stats", _pd(st), _p64(n))
        return st, int(n[0])

    def reset_stats(self):
        _call("gccu_reset_stats")

    # ---- ranged transfers (host or device pointers)
    def put_vec(self, lst, offset, ptr, n):
        _call("gccu_put_vec", lst, offset, ctypes.c_void_p(ptr), n)

    def get_vec(self, lst, offset, ptr, n):
        _call("gccu_get_vec", lst, offset, ctypes.c_void_p(ptr), n)

    # ---- timing
    def event_record(self, slot):
        _call("gccu_event_record", slot)

    def event_elapsed(self, a, b):
        r = np.zeros(1)
        _call("gccu_event_elapsed", a, b, _pd(r))
        return float(r[0])

    def profile(self, enable=True):
        _call("gccu_profile", int(enable))

    def profile_report(self):
        """rows (flops per call, calls, kernel ms, items, tiles, gather ms)"""
        n = np.zeros(1, np.int64)
        rows = np.zeros((4096, 6))
        _call("gccu_profile_report", _pd(rows), 4096, _p64(n))
        return rows[: min(int(n[0]), 4096)]
