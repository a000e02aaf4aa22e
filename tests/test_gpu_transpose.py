"""GPU parity of contractions with operands used transposed (tra_op1 /
tra_op2 / tra_op1op2): every case matches the oracle's route-2 kernel to
1e-12 relative (FP64 path)."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import SPACES, TRANSPOSES, random_list, transpose_operands, transpose_variants

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
