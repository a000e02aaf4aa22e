"""gccu_contract_noalloc (operand panels and launch descriptors in the
library's fixed device array, no allocation) gives the same results as
gccu_contract, on two calls in a row with different inputs, leaves the
engine's device memory and the device's free memory unchanged, and rejects a
contraction whose panels do not fit the fixed array."""
import numpy as np
import pytest

import gccu
from cases import SPACES, contractions_for, random_list

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # same FP64 kernels; only the panel and descriptor memory differs


@pytest.fixture
def engine(built):
    e = gccu.Engine(0)
    yield e
    e.close()


def _lists(e, case):
    _, op1, op2, res = case[:4]
    out = []
    for occ in (op1, op2, res):
        lid, n = e.register_list(e.define_operator([occ]))
        out.append((lid, n))
    return out


def _close(got, ref):
    return np.max(np.abs(got - ref), initial=0.0) <= RTOL * max(1.0, np.abs(ref).max(initial=0.0))


@pytest.mark.parametrize("space", list(SPACES))
def test_noalloc_matches_contract(engine, space):
    import torch

    nsym, norb = SPACES[space]
    engine.register_orbinfo(nsym, norb)
    for i, case in enumerate(contractions_for(space)):
        (l1, n1), (l2, n2), (l12, n12) = _lists(engine, case)
        ex1, ex2, cnt = case[4], case[5], case[6]
        args = ((l1, 1), (l2, 1), (l12, 1), ex1, ex2, cnt)
        for call, update in enumerate((True, False)):
            seed = 100 * i + 10 * call
            engine.upload(l1, random_list(n1, seed))
            engine.upload(l2, random_list(n2, seed + 1))
            x12 = random_list(n12, seed + 2)
            engine.upload(l12, x12)
            engine.contract(*args, fact=-0.75, update=update)  # plans on first use
            ref = engine.download(l12, n12)
            engine.upload(l12, x12)
            engine.sync()
            used = engine.mem_info()[0]
            free = torch.cuda.mem_get_info(0)[0]
            engine.contract_noalloc(*args, fact=-0.75, update=update)
            got = engine.download(l12, n12)
            assert _close(got, ref), (case[0], call)
            assert engine.mem_info()[0] == used, case[0]
            if i > 0:  # after the first call, which may load the module
                assert torch.cuda.mem_get_info(0)[0] == free, case[0]


def test_noalloc_rejects_panels_beyond_the_fixed_array(engine):
    # a three-body operator gathered for one contracted hole: 159 MiB of
    # operand panels, more than the 64 MiB the fixed array holds
    nsym, norb = 1, [[6], [40], [0], [0]]
    engine.register_orbinfo(nsym, norb)
    case = [c for c in contractions_for("c1_small") if c[0] == "t3_fhh"][0]
    (l1, n1), (l2, n2), (l12, _) = _lists(engine, case)
    engine.upload(l1, random_list(n1, 3))
    engine.upload(l2, random_list(n2, 4))
    args = ((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6])
    engine.contract(*args, update=False)
    with pytest.raises(gccu.GccuError, match="MiB"):
        engine.contract_noalloc(*args, update=False)


def test_noalloc_needs_a_plan(engine):
    nsym, norb = SPACES["c2v"]
    engine.register_orbinfo(nsym, norb)
    case = contractions_for("c2v")[0]
    (l1, _), (l2, _), (l12, _) = _lists(engine, case)
    with pytest.raises(gccu.GccuError, match="has not been planned"):
        engine.contract_noalloc((l1, 1), (l2, 1), (l12, 1), case[4], case[5], case[6])


def test_noalloc_split_tf32(engine):
    # precision mode 1: the tensor-core items' split panels live in the
    # engine's workspace, which the first gccu_contract of the descriptor
    # sized; the allocation-free call reuses it
    nsym, norb = 1, [[6], [24], [0], [0]]
    engine.register_orbinfo(nsym, norb)
    engine.set_precision(1)
    try:
        for i, case in enumerate(contractions_for("c1_small")):
            (l1, n1), (l2, n2), (l12, n12) = _lists(engine, case)
            ex1, ex2, cnt = case[4], case[5], case[6]
            args = ((l1, 1), (l2, 1), (l12, 1), ex1, ex2, cnt)
            engine.upload(l1, random_list(n1, 7 * i))
            engine.upload(l2, random_list(n2, 7 * i + 1))
            engine.zero(l12)
            engine.contract(*args, fact=0.5, update=False)
            ref = engine.download(l12, n12)
            engine.upload(l12, random_list(n12, 7 * i + 2))
            engine.contract_noalloc(*args, fact=0.5, update=False)
            got = engine.download(l12, n12)
            assert _close(got, ref), case[0]
    finally:
        engine.set_precision(0)
