"""Coupled-cluster drivers on top of the contraction engine.

The reference generates its CC equations as formula files (lists of [ADD] /
[CONTR] items over operator blocks, include/def_formula_item.h) and evaluates
them with frm_sched2 (contract/frm_sched2.f:117-365) inside solve_nleq
(solve/solve_nleq.f:377-787).  Formula generation is outside the engine's
scope; the formulas below are closed-shell spin-orbital CCSD (the
Stanton-Gauss intermediates, J. Chem. Phys. 94, 4334 (1991)), MP2, and CCSDT
(the connected expansion of e^-T H e^T term by term) written directly as
binary contractions in the reference's occupation language.
Each [CONTR] factor is the product of the topological sign and the
combinatorial factor of that contraction (what the reference stores as
binary_contr%fact); tests/test_cc_formula.py checks every item against its
dense spin-orbital tensor expression.

Evaluation goes through the engine's C ABI only (gccu_contract,
gccu_add_block, gccu_precondition, ...); the first evaluation plans every
contraction, later ones can be replayed from a CUDA graph.
"""
import numpy as np

from gccu import H, P, occ8
from melist import ListView, condensed

# ---- operator blocks ---------------------------------------------------------
HH, HP, PH, PP = occ8({H: 1}, {H: 1}), occ8({H: 1}, {P: 1}), occ8({P: 1}, {H: 1}), occ8(
    {P: 1}, {P: 1})
HHHH, HHPH, HHPP = occ8({H: 2}, {H: 2}), occ8({H: 2}, {H: 1, P: 1}), occ8({H: 2}, {P: 2})
PHHH, PHPH, PHPP = (occ8({H: 1, P: 1}, {H: 2}), occ8({H: 1, P: 1}, {H: 1, P: 1}),
                    occ8({H: 1, P: 1}, {P: 2}))
PPHH, PPPH, PPPP = occ8({P: 2}, {H: 2}), occ8({P: 2}, {H: 1, P: 1}), occ8({P: 2}, {P: 2})
SCAL = occ8()

FOCK_BLOCKS = [HH, HP, PH, PP]
V_BLOCKS = [HHHH, HHPH, HHPP, PHHH, PHPH, PHPP, PPHH, PPPH, PPPP]


def cnt(c=None, a=None):
    return occ8(c, a)


# ---- formulas: ("ADD", res, src, fac, reset) / ("CONTR", res, op1, op2, cnt, fac, update)
# res/src/op1/op2 = (operator name, block occupation)

def _A(res, src, fac=1.0, reset=True, name=""):
    return dict(kind="ADD", res=res, src=src, fac=fac, reset=reset, name=name)


def _C(res, op1, op2, c, fac, update=True, name=""):
    return dict(kind="CONTR", res=res, op1=op1, op2=op2, cnt=c, fac=fac, update=update, name=name)


MP2_OPERATORS = {"F": FOCK_BLOCKS, "V": V_BLOCKS, "T2": [PPHH], "R2": [PPHH], "E": [SCAL]}

MP2_FORMULA = [
    _C(("E", SCAL), ("V", HHPP), ("T2", PPHH), cnt({H: 2}, {P: 2}), 1.0, False, "e_mp2"),
    _A(("R2", PPHH), ("V", PPHH), 1.0, True, "r2_v"),
    _C(("R2", PPHH), ("F", PP), ("T2", PPHH), cnt(None, {P: 1}), 1.0, True, "r2_fpp"),
    _C(("R2", PPHH), ("F", HH), ("T2", PPHH), cnt({H: 1}), 1.0, True, "r2_fhh"),
]

CCSD_OPERATORS = {
    "F": FOCK_BLOCKS, "V": V_BLOCKS, "T1": [PH], "T2": [PPHH], "R1": [PH], "R2": [PPHH],
    "TAU": [PPHH], "TAUT": [PPHH], "E": [SCAL], "XFPP": [PP], "XFHH": [HH], "XFHP": [HP],
    "F2PP": [PP], "F2HH": [HH], "XW": [HHHH], "XWT": [PHPH], "Y": [PHPP], "Z": [PHHH],
    "HJB": [PH],
}

CCSD_FORMULA = [
    # tau = t2 + P(ab) t1 t1 ; tau~ = t2 + 1/2 P(ab) t1 t1
    _A(("TAU", PPHH), ("T2", PPHH), 1.0, True, "tau_t2"),
    _C(("TAU", PPHH), ("T1", PH), ("T1", PH), cnt(), -0.5, True, "tau_t1t1"),
    _A(("TAUT", PPHH), ("T2", PPHH), 1.0, True, "taut_t2"),
    _C(("TAUT", PPHH), ("T1", PH), ("T1", PH), cnt(), -0.25, True, "taut_t1t1"),
    # energy: f_ia t_i^a + 1/4 <ij||ab> tau_ij^ab
    _C(("E", SCAL), ("F", HP), ("T1", PH), cnt({H: 1}, {P: 1}), 1.0, False, "e_ft1"),
    _C(("E", SCAL), ("V", HHPP), ("TAU", PPHH), cnt({H: 2}, {P: 2}), 1.0, True, "e_vtau"),
    # F_ae
    _A(("XFPP", PP), ("F", PP), 1.0, True, "fae_f"),
    _C(("XFPP", PP), ("F", HP), ("T1", PH), cnt({H: 1}), -0.5, True, "fae_ft1"),
    _C(("XFPP", PP), ("V", PHPP), ("T1", PH), cnt({H: 1}, {P: 1}), -1.0, True, "fae_vt1"),
    _C(("XFPP", PP), ("TAUT", PPHH), ("V", HHPP), cnt({P: 1}, {H: 2}), -1.0, True, "fae_tautv"),
    # F_mi
    _A(("XFHH", HH), ("F", HH), 1.0, True, "fmi_f"),
    _C(("XFHH", HH), ("F", HP), ("T1", PH), cnt(None, {P: 1}), 0.5, True, "fmi_ft1"),
    _C(("XFHH", HH), ("V", HHPH), ("T1", PH), cnt({H: 1}, {P: 1}), 1.0, True, "fmi_vt1"),
    _C(("XFHH", HH), ("V", HHPP), ("TAUT", PPHH), cnt({H: 1}, {P: 2}), 1.0, True, "fmi_vtaut"),
    # F_me
    _A(("XFHP", HP), ("F", HP), 1.0, True, "fme_f"),
    _C(("XFHP", HP), ("V", HHPP), ("T1", PH), cnt({H: 1}, {P: 1}), 1.0, True, "fme_vt1"),
    # W_mnij (with 1/2 tau <mn||ef>, which absorbs the tau-tau part of W_abef)
    _A(("XW", HHHH), ("V", HHHH), 1.0, True, "wmnij_v"),
    _C(("XW", HHHH), ("V", HHPH), ("T1", PH), cnt(None, {P: 1}), 1.0, True, "wmnij_vt1"),
    _C(("XW", HHHH), ("V", HHPP), ("TAU", PPHH), cnt(None, {P: 2}), 1.0, True, "wmnij_vtau"),
    # W~_mbej (W_mbej without the bare integral), stored as [b m; e j]
    _C(("XWT", PHPH), ("V", PHPP), ("T1", PH), cnt(None, {P: 1}), 1.0, False, "wmbej_vt1a"),
    _C(("XWT", PHPH), ("V", HHPH), ("T1", PH), cnt({H: 1}), 1.0, True, "wmbej_vt1b"),
    _C(("XWT", PHPH), ("V", HHPP), ("T2", PPHH), cnt({H: 1}, {P: 1}), 0.5, True, "wmbej_vt2"),
    _C(("Y", PHPP), ("V", HHPP), ("T1", PH), cnt({H: 1}), -1.0, False, "y_vt1"),
    _C(("XWT", PHPH), ("Y", PHPP), ("T1", PH), cnt(None, {P: 1}), 1.0, True, "wmbej_yt1"),
    # T1 residual
    _A(("R1", PH), ("F", PH), 1.0, True, "r1_f"),
    _C(("R1", PH), ("XFPP", PP), ("T1", PH), cnt(None, {P: 1}), 1.0, True, "r1_fae"),
    _C(("R1", PH), ("T1", PH), ("XFHH", HH), cnt(None, {H: 1}), -1.0, True, "r1_fmi"),
    _C(("R1", PH), ("T2", PPHH), ("XFHP", HP), cnt({P: 1}, {H: 1}), 1.0, True, "r1_fme"),
    _C(("R1", PH), ("V", PHPH), ("T1", PH), cnt({H: 1}, {P: 1}), -1.0, True, "r1_vt1"),
    _C(("R1", PH), ("V", PHPP), ("T2", PPHH), cnt({H: 1}, {P: 2}), -1.0, True, "r1_vt2a"),
    _C(("R1", PH), ("T2", PPHH), ("V", HHPH), cnt({P: 1}, {H: 2}), -1.0, True, "r1_vt2b"),
    # T2 residual
    _A(("F2PP", PP), ("XFPP", PP), 1.0, True, "f2pp"),
    _C(("F2PP", PP), ("XFHP", HP), ("T1", PH), cnt({H: 1}), -0.5, True, "f2pp_t1"),
    _A(("F2HH", HH), ("XFHH", HH), 1.0, True, "f2hh"),
    _C(("F2HH", HH), ("XFHP", HP), ("T1", PH), cnt(None, {P: 1}), 0.5, True, "f2hh_t1"),
    _A(("R2", PPHH), ("V", PPHH), 1.0, True, "r2_v"),
    _C(("R2", PPHH), ("F2PP", PP), ("T2", PPHH), cnt(None, {P: 1}), 1.0, True, "r2_fae"),
    _C(("R2", PPHH), ("F2HH", HH), ("T2", PPHH), cnt({H: 1}), 1.0, True, "r2_fmi"),
    _C(("R2", PPHH), ("TAU", PPHH), ("XW", HHHH), cnt(None, {H: 2}), 1.0, True, "r2_wmnij"),
    _C(("R2", PPHH), ("V", PPPP), ("TAU", PPHH), cnt(None, {P: 2}), 1.0, True, "r2_ladder"),
    _C(("Z", PHHH), ("V", PHPP), ("TAU", PPHH), cnt(None, {P: 2}), 1.0, False, "z_vtau"),
    _C(("R2", PPHH), ("Z", PHHH), ("T1", PH), cnt({H: 1}), -1.0, True, "r2_zt1"),
    _C(("R2", PPHH), ("TAU", PPHH), ("V", PHPH), cnt({P: 1}, {H: 1}), 1.0, True, "r2_ring_v"),
    _C(("R2", PPHH), ("T2", PPHH), ("XWT", PHPH), cnt({P: 1}, {H: 1}), -1.0, True, "r2_ring_w"),
    _C(("HJB", PH), ("V", PHPH), ("T1", PH), cnt({H: 1}, {P: 1}), -1.0, False, "h_vt1"),
    _C(("R2", PPHH), ("T1", PH), ("HJB", PH), cnt(), 1.0, True, "r2_t1h"),
    _C(("R2", PPHH), ("V", PPPH), ("T1", PH), cnt(None, {P: 1}), 1.0, True, "r2_vt1a"),
    _C(("R2", PPHH), ("T1", PH), ("V", PHHH), cnt(None, {H: 1}), 1.0, True, "r2_vt1b"),
]


# ---- CC of any excitation level (CCSDT = maxexc 3) -------------------------------
# The residuals R_mu = <mu| (H e^T)_c |0> for mu up to maxexc-fold excitations
# and the energy E = <0| (H e^T)_c |0>, T = T1 + ... + T_maxexc, written term
# by term as chains of binary contractions: a class of F or V, then T_n1,
# T_n2, ... attached one [CONTR] at a time, attachment (n, h, p) contracting h
# hole creators and p particle annihilators of the Hamiltonian class with T_n
# (T's lines can only meet the Hamiltonian's).  The T's commute, so each term
# is listed once, with its attachments in non-decreasing (n, h, p) order.  A
# term's factor is the product of the Wick signs of its attachments
# (contraction_sign) over the product of m! for every group of m identical
# attachments; the intermediates of a chain are formed with factor 1 and its
# last contraction carries the factor.  Unfactorised: no dressed
# intermediates are shared between terms beyond common chain prefixes.
# tests/test_ccsdt_formula.py checks the residuals and the energy of CCSDT
# and CCSDTQ against <mu| e^-T H e^T |0> evaluated in the full Fock space of
# a few spin orbitals, with a non-canonical Fock matrix.

FOCK_CLASSES = {"HH": HH, "HP": HP, "PH": PH, "PP": PP}
V_CLASSES = {"HHHH": HHHH, "HHPH": HHPH, "HHPP": HHPP, "PHHH": PHHH, "PHPH": PHPH,
             "PHPP": PHPP, "PPHH": PPHH, "PPPH": PPPH, "PPPP": PPPP}
T_CLASSES = {n: occ8({P: n}, {H: n}) for n in range(1, 5)}


def attach(x, n, h, p):
    """(ex1, ex2, cnt, result) of contracting h hole creators and p particle
    annihilators of class x with T_n"""
    c = np.asarray(cnt({H: h} if h else None, {P: p} if p else None))
    ex1 = np.asarray(x) - c
    ex2 = np.asarray(T_CLASSES[n]) - np.concatenate([c[4:], c[:4]])
    return ex1, ex2, c, ex1 + ex2


def excitation_terms(maxexc):
    """every connected term of <mu| (H e^T)_c |0>, rank(mu) <= maxexc (0 =
    the energy), T up to T_maxexc: [(list, class, attachments, rank)]"""
    terms = []

    def rec(name, key, x, steps):
        if x[0] == 0 and x[5] == 0:  # no hole creator, no particle annihilator left
            if x[1] == x[4] <= maxexc:
                terms.append((name, key, tuple(steps), int(x[1])))
            return
        last = steps[-1] if steps else (0, 0, 0)
        for n in range(1, maxexc + 1):
            for h in range(min(x[0], n) + 1):
                for p in range(min(x[5], n) + 1):
                    if h + p == 0 or (n, h, p) < last:
                        continue
                    y = attach(x, n, h, p)[3]
                    if y[1] <= maxexc and y[4] <= maxexc:
                        rec(name, key, y, steps + [(n, h, p)])

    for key, occ in FOCK_CLASSES.items():
        rec("F", key, np.asarray(occ), [])
    for key, occ in V_CLASSES.items():
        rec("V", key, np.asarray(occ), [])
    return terms


def contraction_sign(x, n, h, p):
    """Wick sign of attaching T_n to class x over h hole and p particle lines.
    An element's operator is a+(C string) a(A string reversed); each string
    is the concatenation over the types, in the condensed order (particles
    before holes), of that type's piece, and a merged piece lists its
    sources in the order the string maps merge them: op1 (cnt, ex1), op2
    (cnt+, ex2), result creators (ex1, ex2), result annihilators (ex2, ex1).
    The sign is the parity of the permutation that brings every contracted
    pair together (op1's operator on the left) and the rest into the
    result's order."""
    ex1, ex2, c, _ = attach(x, n, h, p)
    order = (P, H)
    lab = iter(range(1 << 20))
    pieces = {}
    for t in order:
        for key, k in (("cC", c[t]), ("cA", c[4 + t]), ("1C", ex1[t]), ("1A", ex1[4 + t]),
                       ("2C", ex2[t]), ("2A", ex2[4 + t])):
            pieces[key, t] = [next(lab) for _ in range(int(k))]

    def operator(tag, cre, ann):
        cs = sum((pieces[k, t] for t in order for k in cre), [])
        an = sum((pieces[k, t] for t in order for k in ann), [])
        return [(tag, "c", i) for i in cs] + [(tag, "a", i) for i in reversed(an)]

    seq = operator(1, ("cC", "1C"), ("cA", "1A")) + operator(2, ("cA", "2C"), ("cC", "2A"))
    target = []
    for t in order:
        target += sum(([(1, "c", i), (2, "a", i)] for i in pieces["cC", t]), [])
        target += sum(([(1, "a", i), (2, "c", i)] for i in pieces["cA", t]), [])
    owner = {(k, i): tag for tag, k, i in seq}
    target += [(owner[k, i], k, i) for _, k, i in operator(0, ("1C", "2C"), ("2A", "1A"))]
    pos = {o: i for i, o in enumerate(seq)}
    perm = [pos[o] for o in target]
    inv = sum(1 for a in range(len(perm)) for b in range(a + 1, len(perm)) if perm[a] > perm[b])
    return -1.0 if inv % 2 else 1.0


def term_factor(name, key, steps):
    """product of the attachments' Wick signs over the product of m! of
    identical attachments"""
    from math import factorial
    x = np.asarray((FOCK_CLASSES if name == "F" else V_CLASSES)[key])
    f = 1.0
    for n, h, p in steps:
        f *= contraction_sign(x, n, h, p)
        x = attach(x, n, h, p)[3]
    for st in set(steps):
        f /= factorial(steps.count(st))
    return f


def excitation_formula(maxexc):
    """operators and [ADD]/[CONTR] items of the residuals and the energy;
    the first item writing a result list overwrites it"""
    ops = {"F": FOCK_BLOCKS, "V": V_BLOCKS, "E": [SCAL]}
    for n in range(1, maxexc + 1):
        ops[f"T{n}"] = [T_CLASSES[n]]
        ops[f"R{n}"] = [T_CLASSES[n]]
    items, inter, written = [], {}, set()
    for name, key, steps, rank in excitation_terms(maxexc):
        fac = term_factor(name, key, steps)
        x = np.asarray((FOCK_CLASSES if name == "F" else V_CLASSES)[key])
        res = "E" if rank == 0 else f"R{rank}"
        rocc = SCAL if rank == 0 else T_CLASSES[rank]
        label = name + key + "".join(f"_{n}{h}{p}" for n, h, p in steps)
        if not steps:
            items.append(_A((res, rocc), (name, x), fac, res not in written, label))
            written.add(res)
            continue
        src = (name, x)
        for k, (n, h, p) in enumerate(steps):
            c, y = attach(x, n, h, p)[2:]
            if k == len(steps) - 1:
                items.append(_C((res, rocc), src, (f"T{n}", T_CLASSES[n]), c, fac,
                                res in written, label))
                written.add(res)
            else:
                prefix = (name, key, steps[:k + 1])
                if prefix not in inter:
                    inter[prefix] = f"X{len(inter) + 1}"
                    ops[inter[prefix]] = [y]
                    items.append(_C((inter[prefix], y), src, (f"T{n}", T_CLASSES[n]), c, 1.0,
                                    False, label[:len(name + key)] + "".join(
                                        f"_{a}{b}{d}" for a, b, d in steps[:k + 1])))
                src = (inter[prefix], y)
            x = y
    return ops, items




# ---- filling the Hamiltonian lists -------------------------------------------

def _axis_types(occ):
    c, a = condensed(occ)
    return [t for t, n in c for _ in range(n)] + [t for t, n in a for _ in range(n)]


def fill_hamiltonian(view_f, view_v, nf, nv, ints):
    """host vectors of the Fock list (blocks HH,HP,PH,PP) and the
    antisymmetrised two-electron list <c1c2||a1a2> (9 blocks)"""
    sp = ints.space

    def glob(t, so):
        return sp.type_orbitals(t)[so // 2], so % 2

    xf = np.zeros(nf)
    for ib, occ in enumerate(FOCK_BLOCKS, 1):
        tc, ta = _axis_types(occ)

        def val(ax, tc=tc, ta=ta):
            (p, sp_), (q, sq) = glob(tc, ax[0]), glob(ta, ax[1])
            return ints.fock(p, q) * (sp_ == sq)

        view_f.fill(xf, ib, val)
    xv = np.zeros(nv)
    for ib, occ in enumerate(V_BLOCKS, 1):
        t = _axis_types(occ)

        def val(ax, t=t):
            (c1, s1), (c2, s2) = glob(t[0], ax[0]), glob(t[1], ax[1])
            (a1, r1), (a2, r2) = glob(t[2], ax[2]), glob(t[3], ax[3])
            direct = ints.eri_elems(c1, a1, c2, a2) * ((s1 == r1) & (s2 == r2))
            exch = ints.eri_elems(c1, a2, c2, a1) * ((s1 == r2) & (s2 == r1))
            return direct - exch

        view_v.fill(xv, ib, val)
    return xf, xv


def fill_denominators(view, n, occ, ints):
    """orbital-energy differences sum eps(particles) - sum eps(holes) with the
    shape of an excitation list (dia4op, contract/dia4op.f)"""
    sp = ints.space
    types = _axis_types(occ)
    c, _ = condensed(occ)
    ncre = sum(k for _, k in c)
    x = np.zeros(n)

    def val(ax):
        d = 0.0
        for k, (t, so) in enumerate(zip(types, ax)):
            p = sp.type_orbitals(t)[so // 2]
            e = ints.fock(p, p)
            d = d + (e if k < ncre else -e)
        return d

    view.fill(x, 1, val)
    return x


# ---- solver -------------------------------------------------------------------

class Shard:
    """owner-computes evaluation over the ranks of a process group: the
    contractions into the residual and energy lists run only this rank's
    share of their output tiles (gccu_set_shard), [ADD]s into them count on
    rank 0 only, the intermediates are computed in full on every rank, and
    after each evaluation the residual and energy lists are summed over the
    ranks; amplitudes, DIIS and the step stay replicated.  `dist` is
    torch.distributed with an initialised group (NCCL for device lists, gloo
    for host lists)."""

    LISTS = ("R1", "R2", "E")

    def __init__(self, dist):
        self.dist = dist
        self.rank = dist.get_rank()
        self.n = dist.get_world_size()

    def reduce(self, solver):
        import torch
        e = solver.e
        e.sync()
        for name in self.LISTS:
            if name not in solver.lists:
                continue
            lid, n, _ = solver.lists[name]
            if hasattr(e, "data"):  # host lists (the CPU oracle)
                t = torch.from_numpy(e.data[lid])
            else:
                from devfill import list_tensor
                t = list_tensor(e, lid, n)
            self.dist.all_reduce(t)
        if not hasattr(e, "data"):
            torch.cuda.synchronize()


class CCSolver:
    """Jacobi/DIIS solution of the CC amplitude equations with device-resident
    lists (solve_nleq with method=diis, solve/solve_nleq.f; diagonal step
    diavc, baserout/diavc.f; DIIS subspace, solve/optc_diis_extr.f)."""

    # lists that hold the Hamiltonian, amplitudes, residuals and the energy;
    # the others of a formula are its intermediates
    PERSISTENT = ("F", "V", "T1", "T2", "T3", "T4", "R1", "R2", "R3", "R4", "E")

    def __init__(self, engine, ints, method="ccsd", use_tr=False, maxsub=8, shift=0.0,
                 learned=None, shard=None, spin_project=False, native_formula=False):
        self.e = engine
        # native_formula: the formula runs as one item list in the engine
        # (gccu_formula_run), its intermediates created and deleted by
        # [NEW] / [DEL] items in one arena (not with a sharded solve)
        self.native = native_formula and shard is None
        self.fid = None
        # project the residuals onto their singlet part after each evaluation
        # (result lists with a spin, frm_sched2's end-of-target step)
        self.spin_project = spin_project
        self.shard = shard  # Shard: residual contractions split over ranks
        self.ints = ints
        self.method = method
        self.use_tr = use_tr
        self.maxsub = maxsub
        self.shift = shift  # level shift of the diagonal preconditioner (diavc)
        # learned correction of the diagonal step (weights loaded into the
        # engine), used for a step only if the last step reduced the residual
        # norm; plain diavc otherwise (counted in self.fallbacks)
        self.learned = learned is not None
        self.fallbacks = 0
        self.recorder = None  # called with the solver before each step (sampling)
        sp = ints.space
        self.nsym = sp.nsym
        engine.register_orbinfo(sp.nsym, sp.norb)
        if method in ("ccsdt", "ccsdtq"):
            ops, self.formula = excitation_formula(3 if method == "ccsdt" else 4)
        else:
            ops = MP2_OPERATORS if method == "mp2" else CCSD_OPERATORS
            self.formula = MP2_FORMULA if method == "mp2" else CCSD_FORMULA
        self.lists = {}
        for name, blocks in ops.items():
            opid = engine.define_operator(blocks)
            absym = 1 if use_tr and name not in ("F", "V", "E") else 0
            if use_tr and name in ("F", "V"):
                absym = 1
            if self.native and name not in self.PERSISTENT:
                lid, n = engine.register_intermediate(opid, absym=absym)
            else:
                lid, n = engine.register_list(opid, absym=absym)
            self.lists[name] = (lid, n, blocks)
        self.amps = {"mp2": ["T2"], "ccsdt": ["T1", "T2", "T3"],
                     "ccsdtq": ["T1", "T2", "T3", "T4"]}.get(method, ["T1", "T2"])
        self.res = {f"T{n}": f"R{n}" for n in range(1, 5)}
        # denominators, steps (the last one kept for the learned step's
        # inputs) and DIIS subspace
        for a in self.amps:
            blocks = self.lists[a][2]
            for extra in ("D" + a, "S" + a, "P" + a):
                opid = engine.define_operator(blocks)
                lid, n = engine.register_list(opid)
                self.lists[extra] = (lid, n, blocks)
        self.graph = None
        self.history = []
        if self.learned:
            engine.lp_set_weights(learned)
        if self.native:
            self.fid = engine.formula_define(self.formula_items())

    def formula_items(self):
        """the formula as engine items (frm_sched2's commands): [INIT
        TARGET] wherever the result list changes (the residuals' last ones
        project onto the singlet with spin_project), [NEW] before an
        intermediate's first item and [DEL] after its last"""
        import gccu
        inter = {n for n in self.lists if n not in self.PERSISTENT and n in
                 {x for it in self.formula for x in self._names(it)}}
        first, last = {}, {}
        for i, it in enumerate(self.formula):
            for n in self._names(it):
                if n in inter:
                    first.setdefault(n, i)
                    last[n] = i
        last_seg = {}
        for i, it in enumerate(self.formula):
            if i == 0 or self.formula[i - 1]["res"][0] != it["res"][0]:
                last_seg[it["res"][0]] = i
        items = []
        for i, it in enumerate(self.formula):
            for n in sorted(n for n, f in first.items() if f == i):
                items.append(gccu.FormulaItem(command=gccu.CMD_NEW, list=self.lid(n)))
            res = it["res"][0]
            if i == 0 or self.formula[i - 1]["res"][0] != res:
                proj = self.spin_project and res in self.res.values() and last_seg[res] == i
                items.append(gccu.FormulaItem(command=gccu.CMD_TARGET, list=self.lid(res),
                                              mult=1 if proj else 0))
            if it["kind"] == "ADD":
                (lo, bo), (li, bi) = self.blk(it["res"]), self.blk(it["src"])
                items.append(gccu.FormulaItem(command=gccu.CMD_ADD, list=lo, iblk_out=bo,
                                              list_in=li, iblk_in=bi, fac=it["fac"],
                                              reset=int(it["reset"])))
            else:
                bc, use_tr = self._bc(it)
                items.append(gccu.FormulaItem(command=gccu.CMD_CONTR, bc=bc, fac=it["fac"],
                                              update=int(it["update"]), use_tr=int(use_tr)))
            for n in sorted(n for n, l in last.items() if l == i):
                items.append(gccu.FormulaItem(command=gccu.CMD_DEL, list=self.lid(n)))
        return items

    @staticmethod
    def _names(it):
        ops = [it["src"]] if it["kind"] == "ADD" else [it["op1"], it["op2"]]
        return [it["res"][0]] + [o[0] for o in ops]

    def _bc(self, it):
        """engine descriptor of a [CONTR] item and whether it runs under use_tr"""
        o1, o2, r = self.blk(it["op1"]), self.blk(it["op2"]), self.blk(it["res"])
        c = np.asarray(it["cnt"])
        ex1 = np.asarray(it["op1"][1]) - c
        ex2 = np.asarray(it["op2"][1]) - np.concatenate([c[4:], c[:4]])
        use_tr = self.use_tr and it["res"][0] not in ("E",)
        return self.e.desc(o1, o2, r, ex1, ex2, c), use_tr

    def lid(self, name):
        return self.lists[name][0]

    def blk(self, ref):
        name, occ = ref
        blocks = self.lists[name][2]
        for i, b in enumerate(blocks, 1):
            if np.array_equal(b, occ):
                return (self.lists[name][0], i)
        raise KeyError(ref)

    def view(self, name):
        lid, n, blocks = self.lists[name]
        return ListView(self.e, lid, blocks, self.nsym)

    def load_hamiltonian(self):
        xf, xv = fill_hamiltonian(self.view("F"), self.view("V"), self.lists["F"][1],
                                  self.lists["V"][1], self.ints)
        self.e.upload(self.lid("F"), xf)
        self.e.upload(self.lid("V"), xv)
        for a in self.amps:
            n = self.lists[a][1]
            d = fill_denominators(self.view("D" + a), n, self.lists[a][2][0], self.ints)
            self.e.upload(self.lid("D" + a), d)
            self.e.zero(self.lid(a))
        self.freeze_hamiltonian()

    def freeze_hamiltonian(self, frozen=True):
        """the Fock and two-electron lists are constant during the solve: the
        engine may keep the operand panels it derives from them"""
        for name in ("F", "V"):
            self.e.freeze(self.lid(name), frozen)

    def load_hamiltonian_device(self, tints):
        """generate the Hamiltonian and denominator lists on the device
        (devfill.TorchIntegrals) directly in the engine's list memory"""
        import torch

        from devfill import DeviceListView, list_tensor
        dev = tints.device
        if dev == "cpu":
            def tensor(lid, n):
                return torch.from_numpy(self.e.data[lid])
        else:
            def tensor(lid, n):
                return list_tensor(self.e, lid, n)
        self.e.sync()
        for name in ("F", "V"):
            lid, n, blocks = self.lists[name]
            x = tensor(lid, n)
            view = DeviceListView(self.e, lid, blocks, self.nsym, device=dev)
            for ib, occ in enumerate(blocks, 1):
                t = _axis_types(occ)
                if name == "F":
                    view.fill(x, ib, lambda ax, t=t: tints.fock(t[0], ax[0], t[1], ax[1]))
                else:
                    view.fill(x, ib, lambda ax, t=t: tints.eri(t, ax))
        tints.release()
        for a in self.amps:
            lid, n, blocks = self.lists["D" + a]
            x = tensor(lid, n)
            types = _axis_types(blocks[0])
            ncre = sum(k for _, k in condensed(blocks[0])[0])

            def den(ax, types=types, ncre=ncre):
                d = 0.0
                for k, (t, so) in enumerate(zip(types, ax)):
                    e = tints.eps[tints.orbs[t][so // 2]]
                    d = d + (e if k < ncre else -e)
                return d

            DeviceListView(self.e, lid, blocks, self.nsym, device=dev).fill(x, 1, den)
        if dev != "cpu":
            torch.cuda.synchronize()
        for a in self.amps:
            self.e.zero(self.lid(a))
        self.freeze_hamiltonian()

    def evaluate(self):
        """one formula evaluation (frm_sched2 over the item list)"""
        if self.fid is not None:
            self.e.formula_run(self.fid)
            return
        for it in self.formula:
            self.run_item(it)

    def run_item(self, it):
        """one [ADD] or [CONTR] item of the formula"""
        sharded = self.shard is not None and it["res"][0] in Shard.LISTS
        if it["kind"] == "ADD":
            (lo, bo), (li, bi) = self.blk(it["res"]), self.blk(it["src"])
            fac = it["fac"] if not sharded or self.shard.rank == 0 else 0.0
            self.e.add_block(fac, li, bi, lo, bo, reset=it["reset"])
        elif sharded:
            self.e.set_shard(self.shard.rank, self.shard.n)
            try:
                self._contract(it)
            finally:
                self.e.set_shard(0, 1)
        else:
            self._contract(it)

    def _contract(self, it):
        o1, o2, r = self.blk(it["op1"]), self.blk(it["op2"]), self.blk(it["res"])
        c = np.asarray(it["cnt"])
        occ1 = np.asarray(it["op1"][1])
        occ2 = np.asarray(it["op2"][1])
        ex1 = occ1 - c
        ex2 = occ2 - np.concatenate([c[4:], c[:4]])
        use_tr = self.use_tr and it["res"][0] not in ("E",)
        self.e.contract(o1, o2, r, ex1, ex2, c, fact=it["fac"], update=it["update"],
                        use_tr=use_tr)

    def energy(self):
        return float(self.e.download(self.lid("E"), 1)[0])

    def residual_norm(self):
        return float(np.sqrt(sum(self.e.dot(self.lid(self.res[a]), self.lid(self.res[a]))
                                 for a in self.amps)))

    def use_learned_step(self):
        """the learned step is taken while the residual norm decreases"""
        if not self.learned:
            return False
        h = self.history
        ok = len(h) < 2 or h[-1][2] < h[-2][2]
        if not ok:
            self.fallbacks += 1
        return ok

    def precondition(self, out, a, learned):
        """out = -R/D (diavc) or its learned correction; the step is kept as
        the previous step of the next call"""
        if learned:
            self.e.lp_precondition(out, self.lid(self.res[a]), self.lid("D" + a),
                                   self.lid("P" + a), fac=-1.0, shift=self.shift)
        else:
            self.e.precondition(out, self.lid(self.res[a]), self.lid("D" + a), fac=-1.0,
                                shift=self.shift)
        if self.learned or self.recorder is not None:
            self.e.add_block(1.0, out, 1, self.lid("P" + a), 1, reset=True)

    def step(self):
        """t <- t - R/D (diagonal preconditioner)"""
        if self.recorder is not None:
            self.recorder(self)
        learned = self.use_learned_step()
        for a in self.amps:
            self.precondition(self.lid("S" + a), a, learned)
            self.e.add_block(1.0, self.lid("S" + a), 1, self.lid(a), 1)

    def _diis_lists(self):
        if hasattr(self, "_diis"):
            return self._diis
        slots = []
        for k in range(self.maxsub):
            slot = {}
            for a in self.amps:
                blocks = self.lists[a][2]
                for kind in ("t", "e"):
                    lid, n = self.e.register_list(self.e.define_operator(blocks))
                    slot[(kind, a)] = lid
            slots.append(slot)
        self._diis = dict(slots=slots, used=[], B=np.zeros((self.maxsub, self.maxsub)))
        return self._diis

    def diis_step(self):
        """preconditioned step, then DIIS extrapolation over the last maxsub
        (amplitude, step) pairs (optc_diis_sbsp_add / optc_diis_extr,
        solve/optc_diis_sbsp_add.f:125-145, solve/optc_diis_extr.f:67,82)"""
        d = self._diis_lists()
        used = d["used"]
        # slot to overwrite: the oldest one when the subspace is full
        k = len(used) if len(used) < self.maxsub else used.pop(0)
        used.append(k)
        slot = d["slots"][k]
        if self.recorder is not None:
            self.recorder(self)
        learned = self.use_learned_step()
        for a in self.amps:
            self.precondition(slot[("e", a)], a, learned)
            self.e.add_block(1.0, self.lid(a), 1, slot[("t", a)], 1, reset=True)
            self.e.add_block(1.0, slot[("e", a)], 1, slot[("t", a)], 1)
        B = d["B"]
        for j in used:
            v = sum(self.e.dot(slot[("e", a)], d["slots"][j][("e", a)]) for a in self.amps)
            B[k, j] = B[j, k] = v
        m = len(used)
        A = np.zeros((m + 1, m + 1))
        A[:m, :m] = B[np.ix_(used, used)]
        scale = np.max(np.abs(np.diag(A[:m, :m]))) or 1.0
        A[:m, :m] /= scale
        A[m, :m] = A[:m, m] = -1.0
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        try:
            c = np.linalg.solve(A, rhs)[:m]
        except np.linalg.LinAlgError:
            c = np.zeros(m)
            c[-1] = 1.0
        for a in self.amps:
            for i, j in enumerate(used):
                self.e.add_block(float(c[i]), d["slots"][j][("t", a)], 1, self.lid(a), 1,
                                 reset=(i == 0))
        return c

    def iterate(self, diis=True):
        """one CC iteration: formula evaluation (summed over the ranks when
        sharded), energy and residual norm"""
        if self.graph is not None:
            self.e.graph_launch(self.graph)
        else:
            self.evaluate()
        if self.shard is not None:
            self.shard.reduce(self)
        if self.spin_project and self.fid is None:
            self.project_residuals()
        en = self.energy()
        rn = self.residual_norm()
        return en, rn

    def project_residuals(self):
        """singlet projection of the residual lists (spin_prj_list at the end
        of each target, contract/frm_sched2.f:146-149)"""
        for a in self.amps:
            self.e.spin_prj(self.lid(self.res[a]))

    def capture(self):
        """record one formula evaluation as a CUDA graph (plans must exist)"""
        self.e.graph_begin()
        self.evaluate()
        self.graph = self.e.graph_end()

    def solve_mixed(self, maxiter=60, conv=1e-8, switch=1e-5, callback=None, stop=None,
                    stall=None, reset_diis=False, final=0, schedule=None):
        """Mixed-precision solve: the contractions run in split TF32 on the
        tensor cores (engine precision 1) while the residual norm is above
        `switch`, and in precision `final` (0 = FP64, 2 = FP64 emulated with
        int8 slices) after that; `schedule`, a list of (precision, residual
        norm below which the next entry takes over; None for the last), sets
        any sequence of precisions instead.  The CC fixed-point iteration
        corrects the errors of the cheaper iterations; the DIIS subspace,
        residuals, energies and amplitude updates stay FP64 throughout.  With
        `stall`, the solve also moves on once a residual norm is above `stall`
        times the previous one (the residual has reached the precision's error
        floor); `reset_diis` empties the DIIS subspace at each switch.  Each
        precision's evaluation runs once eagerly (planning) and is then
        replayed from its own CUDA graph.  stop(it, energy, residual) may end
        the solve early.  Returns the last energy; switched_at lists the
        iterations after which the precision changed."""
        if schedule is None:
            schedule = [(1, switch), (final, None)]
        stage = 0
        mode = schedule[0][0]
        self.e.set_precision(mode)
        graphs, planned = {}, set()
        en = None
        self.switched_at = None
        switches = []
        prev = None
        for it in range(1, maxiter + 1):
            if mode not in graphs and mode in planned:
                self.capture()
                graphs[mode] = self.graph
            self.graph = graphs.get(mode)
            en, rn = self.iterate()
            planned.add(mode)
            self.history.append((it, en, rn))
            if callback:
                callback(it, en, rn)
            if rn < conv or (stop is not None and stop(it, en, rn)):
                break
            limit = schedule[stage][1]
            if limit is not None and (rn < limit or (stall is not None and prev is not None and
                                                     rn > stall * prev)):
                stage += 1
                mode = schedule[stage][0]
                self.e.set_precision(mode)
                switches.append(it)
                if reset_diis and hasattr(self, "_diis"):
                    self._diis["used"].clear()
            prev = rn
            self.diis_step()
        self.switched_at = switches[0] if len(switches) == 1 else (switches or None)
        self.e.set_precision(0)
        self.graph = None
        return en

    def solve(self, maxiter=50, conv=1e-8, use_graph=False, diis=True, callback=None,
              econv=None):
        e_old = None
        for it in range(1, maxiter + 1):
            if use_graph and self.graph is None and it > 1:
                self.capture()
            en, rn = self.iterate()
            self.history.append((it, en, rn))
            if callback:
                callback(it, en, rn)
            if rn < conv or (econv is not None and e_old is not None and abs(en - e_old) < econv):
                return en
            if diis:
                self.diis_step()
            else:
                self.step()
            e_old = en
        return en
