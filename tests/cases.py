"""Shared test cases: orbital spaces and binary contractions in the
reference's occupation language (test helper, not product code)."""
import numpy as np

from gccu import H, P, V, occ8

# (nsym, norb[type][irrep]) orbital spaces
SPACES = {
    "c1_small": (1, [[3], [5], [0], [0]]),
    "c2v": (4, [[2, 1, 1, 0], [3, 2, 2, 1], [0] * 4, [0] * 4]),
    "d2h": (8, [[1, 1, 0, 1, 0, 1, 0, 0], [2, 1, 1, 1, 1, 1, 1, 1], [0] * 8, [0] * 8]),
    "c1_val": (1, [[2], [4], [2], [0]]),
}


def cnt_dag(c):
    c = np.asarray(c)
    return np.concatenate([c[4:], c[:4]])


# binary contractions: (name, op1 occ, op2 occ, res occ, ex1, ex2, cnt)
def _bc(name, ex1, ex2, cnt):
    ex1, ex2, cnt = np.asarray(ex1), np.asarray(ex2), np.asarray(cnt)
    op1 = ex1 + cnt
    op2 = ex2 + cnt_dag(cnt)
    res = ex1 + ex2
    return (name, op1, op2, res, ex1, ex2, cnt)


CONTRACTIONS = [
    # Fock particle block on doubles: F(P;P) T2, one particle contracted
    _bc("fpp_t2", occ8({P: 1}), occ8({P: 1}, {H: 2}), occ8(None, {P: 1})),
    # Fock hole block on doubles: F(H;H) T2, one hole contracted
    _bc("fhh_t2", occ8(None, {H: 1}), occ8({P: 2}, {H: 1}), occ8({H: 1})),
    # particle ladder: H(PP;PP) T2
    _bc("pp_ladder", occ8({P: 2}), occ8(None, {H: 2}), occ8(None, {P: 2})),
    # hole ladder: W(HH;HH) T2 (contracts the holes of T2 with W's creators)
    _bc("hh_ladder", occ8(None, {H: 2}), occ8({P: 2}), occ8({H: 2})),
    # ring: W(PH;PH) T2, one hole and one particle contracted
    _bc("ring", occ8({P: 1}, {H: 1}), occ8({P: 1}, {H: 1}), occ8({H: 1}, {P: 1})),
    # energy-like full contraction: H(HH;PP) T2 -> scalar
    _bc("energy", occ8(), occ8(), occ8({H: 2}, {P: 2})),
    # singles into doubles: T1 x H(PH;HH) -> (PP;HH)
    _bc("t1_vphhh", occ8({P: 1}), occ8({P: 1}, {H: 2}), occ8(None, {H: 1})),
    # outer product: T1 T1 -> T2-like, nothing contracted
    _bc("t1t1", occ8({P: 1}, {H: 1}), occ8({P: 1}, {H: 1}), occ8()),
    # three-body: T3-like (PPP;HHH) x F(H;H)
    _bc("t3_fhh", occ8({P: 3}, {H: 2}), occ8(None, {H: 1}), occ8(None, {H: 1})),
]


def contractions_for(space):
    if space == "c1_val":
        return CONTRACTIONS + [
            _bc("val_mix", occ8({V: 1}, {H: 1}), occ8({P: 1}, {V: 1}), occ8({V: 1}, {P: 1}))]
    return CONTRACTIONS


# reorders of joined operators: (name, njoined, vertices of the original
# class, vertices of the reordered class, shifts [(occ, from_vtx, to_vtx)]);
# every operator has as many creators as annihilators (total Ms 0 lists)
def _reo(name, ori, shifts):
    nj = len(ori)
    ori = [np.asarray(o) for o in ori]
    reo = [o.copy() for o in ori]
    for occ, fr, to in shifts:
        reo[fr - 1] = reo[fr - 1] - np.asarray(occ)
        reo[to - 1] = reo[to - 1] + np.asarray(occ)
        assert (reo[fr - 1] >= 0).all()
    return (name, nj, ori, reo, shifts)


REORDERS = [
    # a creator moves to a vertex that holds only an annihilator: same
    # condensed components, a pure change of vertex
    _reo("move_p", [occ8({P: 1}), occ8(None, {H: 1})], [(occ8({P: 1}), 1, 2)]),
    # two T1-like vertices: a particle creator joins the other vertex (merge)
    _reo("merge_p", [occ8({P: 1}, {H: 1}), occ8({P: 1}, {H: 1})], [(occ8({P: 1}), 1, 2)]),
    # a hole annihilator joins the other vertex
    _reo("merge_h", [occ8({P: 1}, {H: 1}), occ8({P: 1}, {H: 1})], [(occ8(None, {H: 1}), 2, 1)]),
    # two shifts in opposite directions
    _reo("swap_ph", [occ8({P: 1}, {H: 1}), occ8({P: 1}, {H: 1})],
         [(occ8({P: 1}), 1, 2), (occ8(None, {H: 1}), 2, 1)]),
    # a one-body vertex hands its creator to a doubles-like vertex
    _reo("merge_pp", [occ8({P: 2}, {H: 2}), occ8({P: 1}, {H: 1})], [(occ8({P: 1}), 2, 1)]),
    # nothing moves
    _reo("none", [occ8({P: 1}, {H: 1}), occ8({P: 1}, {H: 1})], []),
]


def reorders_for(space):
    if space == "c1_val":
        return REORDERS + [_reo("val_move", [occ8({V: 1}, {H: 1}), occ8({P: 1}, {V: 1})],
                                [(occ8({V: 1}), 1, 2)])]
    return REORDERS


# partial traces (self-contractions): (name, operator, result, contracted J);
# operator = result + J on both sides, J the same on creators and annihilators
def _tr(name, res, cnt):
    res, cnt = np.asarray(res), np.asarray(cnt)
    return (name, res + cnt, res, cnt)


TRACES = [
    _tr("full_p", occ8(), occ8({P: 1}, {P: 1})),
    _tr("w_over_h", occ8({P: 1}, {P: 1}), occ8({H: 1}, {H: 1})),
    _tr("pp_over_p", occ8({P: 1}, {P: 1}), occ8({P: 1}, {P: 1})),
    _tr("full_hh", occ8(), occ8({H: 2}, {H: 2})),
    _tr("t2like_over_ph", occ8({P: 1}, {H: 1}), occ8({P: 1, H: 1}, {P: 1, H: 1})),
]


def traces_for(space):
    if space == "c1_val":
        return TRACES + [_tr("v_over_v", occ8({P: 1}, {P: 1}), occ8({V: 1}, {V: 1}))]
    return TRACES


def random_list(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n)


# operands used transposed: (tra_op1, tra_op2, tra_res) patterns
TRANSPOSES = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 1, 1)]


def _encode_did(comps, dist, nsym):
    did, base = 0, 1
    for (_, n), (ix, g) in zip(comps, dist):
        did += ((ix - 1) * nsym + g - 1) * base
        base *= (n + 1) * nsym
    return did


def transpose_list(src, lid_s, occ_s, x, lid_t, n_t, nsym):
    """List vector of the adjoint class (occupation cnt_dag(occ_s), total
    Ms negated) of the one-class list lid_s: its element with creator
    strings J and annihilator strings I is the element of x with creator
    strings I and annihilator strings J.  src: engine or oracle binding."""
    from melist import condensed, decode_did, ldims

    cs, as_ = condensed(occ_s)
    ct, at = condensed(cnt_dag(occ_s))
    where = {int(r[7]): int(r[4]) for r in src.dists(lid_t) if r[0] == 1}
    y = np.full(n_t, np.nan)
    for r in src.dists(lid_s):
        if r[0] != 1:
            continue
        off, did = int(r[4]), int(r[7])
        dist = decode_did(did, cs + as_, nsym)
        lens = [src.strings(t, n, ix, g)[0].shape[0] for (t, n), (ix, g) in zip(cs + as_, dist)]
        nc = len(cs)
        dist_t, lens_t = dist[nc:] + dist[:nc], lens[nc:] + lens[:nc]
        off_t = where[_encode_did(ct + at, dist_t, nsym)]
        grids = np.meshgrid(*[np.arange(n) for n in lens], indexing="ij")
        pos_s = np.asarray(sum(g * d for g, d in zip(grids, ldims(cs, as_, lens))))
        pos_t = np.asarray(sum(g * d for g, d in zip(grids[nc:] + grids[:nc],
                                                     ldims(ct, at, lens_t))))
        y[off_t + pos_t.ravel()] = x[off + pos_s.ravel()]
    assert not np.isnan(y).any()
    return y


def transpose_variants(space):
    """(case, (gamt, mst) of op1, op2, result): symmetric lists, then a
    non-totally-symmetric op1 and a spin-changing op2 where the space allows"""
    nsym = SPACES[space][0]
    for case in contractions_for(space):
        yield case, ((1, 0), (1, 0), (1, 0))
        if nsym > 1:
            yield case, ((2, 0), (1, 0), (2, 0))
        if case[2][:4].sum() > 0 and case[2][4:].sum() > 0:
            yield case, ((1, 0), (1, 2), (1, 2))


def _define_list(src, occ, gamt, mst, oracle):
    op = src.define_op([occ]) if oracle else src.define_operator([occ])
    return src.define_list(op, gamt, mst) if oracle else src.register_list(op, gamt, mst)


def transpose_operands(src, case, sym, tra, oracle):
    """per operand: (stored list, its length, explicit list, its length,
    stored occupation); the stored list holds the adjoint class when the
    operand is used transposed"""
    out = []
    for occ, (g, m), t in zip(case[1:4], sym, tra):
        le, ne = _define_list(src, occ, g, m, oracle)
        if t:
            ls, ns = _define_list(src, cnt_dag(occ), g, -m, oracle)
            out.append((ls, ns, le, ne, cnt_dag(occ)))
        else:
            out.append((le, ne, le, ne, occ))
    return out
