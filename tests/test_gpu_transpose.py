"""GPU parity of contractions with operands used transposed (tra_op1 /
tra_op2 / tra_op1op2): every case matches the oracle's route-2 kernel to
1e-12 relative on the FP64 path, and to split-TF32 accuracy on a space whose
blocks take the tensor-core path.  The transposed [ADD]
(gccu_add_block_transp, add_opblk_transp) matches the oracle's restatement
for input and output transposed in turn."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import (SPACES, TRANSPOSES, contractions_for, random_list, transpose_operands,
                   transpose_variants)

pytestmark = pytest.mark.gpu

RTOL = 1e-12


@pytest.fixture
def engine(built):
    e = gccu.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("space", list(SPACES))
def test_transposed_contractions_match_oracle(engine, space):
    nsym, norb = SPACES[space]
    engine.register_orbinfo(nsym, norb)
    nrun = 0
    for i, (case, sym) in enumerate(transpose_variants(space)):
        for j, tra in enumerate(TRANSPOSES):
            o = Oracle(nsym, norb)
            ops_o = transpose_operands(o, case, sym, tra, True)
            ops_e = transpose_operands(engine, case, sym, tra, False)
            if min(op[1] for op in ops_o) == 0:
                continue
            assert [op[1] for op in ops_o] == [op[1] for op in ops_e]
            xs = [random_list(op[1], 31 * i + 7 * j + k) for k, op in enumerate(ops_o)]
            for op, x in zip(ops_e, xs):
                engine.upload(op[0], x)
            ex1, ex2, cnt = case[4:7]
            update = (i + j) % 2 == 0
            ref = xs[2].copy()
            o.contract(2, ops_o[0][0], 1, xs[0], ops_o[1][0], 1, xs[1], ops_o[2][0], 1, ref,
                       ex1, ex2, cnt, -0.5, update=update, tra=tra)
            engine.contract(*[(op[0], 1) for op in ops_e], ex1, ex2, cnt, fact=-0.5,
                            update=update, tra=tra)
            got = engine.download(ops_e[2][0], ops_e[2][1])
            assert np.max(np.abs(got - ref)) <= RTOL * max(1.0, np.abs(ref).max()), \
                (case[0], sym, tra)
            nrun += 1
    assert nrun > 0


RTOL_TC = 2e-5  # split TF32, FP32 accumulation over <= 4096 terms


def test_transposed_contractions_tensor_cores(engine):
    # 6 holes, 24 particles: the ladder- and ring-like blocks have hundreds of
    # rows, columns and contraction indices and run on the tensor cores
    nsym, norb = 1, [[6], [24], [0], [0]]
    engine.register_orbinfo(nsym, norb)
    diffs = []
    for i, case in enumerate(contractions_for("c1_small")):
        for j, tra in enumerate(TRANSPOSES):
            sym = ((1, 0), (1, 0), (1, 0))
            o = Oracle(nsym, norb)
            ops_o = transpose_operands(o, case, sym, tra, True)
            ops_e = transpose_operands(engine, case, sym, tra, False)
            xs = [random_list(op[1], 41 * i + 5 * j + k) for k, op in enumerate(ops_o)]
            for op, x in zip(ops_e, xs):
                engine.upload(op[0], x)
            ex1, ex2, cnt = case[4:7]
            ref = np.zeros(ops_o[2][1])
            o.contract(2, ops_o[0][0], 1, xs[0], ops_o[1][0], 1, xs[1], ops_o[2][0], 1, ref,
                       ex1, ex2, cnt, 0.5, update=False, tra=tra)
            scale = max(1.0, np.abs(ref).max())
            got = {}
            for mode in (1, 0):
                engine.set_precision(mode)
                engine.contract(*[(op[0], 1) for op in ops_e], ex1, ex2, cnt, fact=0.5,
                                update=False, tra=tra)
                got[mode] = engine.download(ops_e[2][0], ops_e[2][1])
            engine.set_precision(0)
            assert np.max(np.abs(got[1] - ref)) <= RTOL_TC * scale, (case[0], tra)
            assert np.max(np.abs(got[0] - ref)) <= RTOL * scale, (case[0], tra)
            diffs.append(np.max(np.abs(got[1] - got[0])) / scale)
    assert max(diffs) > 1e-10, "no transposed contraction took the tensor-core path"


@pytest.mark.parametrize("space", list(SPACES))
def test_add_block_transp_matches_oracle(engine, space):
    # gccu_add_block_transp (add_opblk_transp) against the oracle's
    # restatement, both sides transposed in turn, with reset, update and the
    # returned squared norm
    from cases import cnt_dag
    from test_transpose_host import add_transp_variants
    nsym, norb = SPACES[space]
    engine.register_orbinfo(nsym, norb)
    nrun = 0
    for i, (occ, (g, m)) in enumerate(add_transp_variants(space)):
        o = Oracle(nsym, norb)
        lo, no = engine.register_list(engine.define_operator([occ]), g, m)
        li, ni = engine.register_list(engine.define_operator([cnt_dag(occ)]), g, -m)
        olo, _ = o.define_list(o.define_op([occ]), g, m)
        oli, _ = o.define_list(o.define_op([cnt_dag(occ)]), g, -m)
        if no == 0:
            continue
        for tra_in, tra_out in ((1, 0), (0, 1)):
            for reset in (False, True):
                xin, xout = random_list(ni, 5 * i + reset), random_list(no, 5 * i + 2)
                engine.upload(li, xin)
                engine.upload(lo, xout)
                xn = engine.add_block_transp(-0.4, li, 1, lo, 1, tra_in, tra_out, reset, typ=1)
                got = engine.download(lo, no)
                ref = xout.copy()
                xr = o.add_transp(-0.4, oli, 1, xin, olo, 1, ref, tra_in, tra_out, reset=reset)
                assert np.max(np.abs(got - ref)) <= 1e-14 * max(1.0, np.abs(ref).max())
                assert xn == pytest.approx(xr, rel=1e-12)
                nrun += 1
    assert nrun > 0
