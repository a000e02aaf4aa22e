"""Joined (multi-vertex) operators and reorders on the host: the engine's
ME-list layout of joined operators equals the oracle's set_op_dim2
restatement, reorder plans build, and the oracle's reorder
(reo_op_wmaps_c) is a plain signed copy when the shift changes no
condensed component."""
import numpy as np
import pytest

import gccu
from binding import Oracle
from cases import SPACES, random_list, reorders_for


@pytest.fixture
def host(built):
    e = gccu.Engine(-1)
    yield e
    e.close()


def _define(e, o, nj, vertices):
    occ = np.stack(vertices)
    le, n = e.register_list(e.define_operator_joined(occ, nj))
    lo, no = o.define_list(o.define_op_joined(occ, nj))
    assert n == no
    return le, lo, n


@pytest.mark.parametrize("space", list(SPACES))
def test_joined_layout_matches_oracle(host, space):
    nsym, norb = SPACES[space]
    host.register_orbinfo(nsym, norb)
    o = Oracle(nsym, norb)
    for name, nj, ori, reo, shifts in reorders_for(space):
        for vertices in (ori, reo):
            le, lo, n = _define(host, o, nj, vertices)
            assert np.array_equal(host.dists(le), o.dists(lo)), name


@pytest.mark.parametrize("space", list(SPACES))
def test_reorder_plans(host, space):
    nsym, norb = SPACES[space]
    host.register_orbinfo(nsym, norb)
    o = Oracle(nsym, norb)
    for name, nj, ori, reo, shifts in reorders_for(space):
        lo_e, _, _ = _define(host, o, nj, ori)
        lr_e, _, _ = _define(host, o, nj, reo)
        ncases, nel = host.reorder_info((lo_e, 1), (lr_e, 1), shifts)
        assert ncases > 0 and nel > 0, name


@pytest.mark.parametrize("space", list(SPACES))
def test_oracle_pure_move_is_a_copy(space):
    nsym, norb = SPACES[space]
    o = Oracle(nsym, norb)
    for name, nj, ori, reo, shifts in reorders_for(space):
        if name not in ("move_p", "none", "val_move"):
            continue
        occ_o, occ_r = np.stack(ori), np.stack(reo)
        lo, n = o.define_list(o.define_op_joined(occ_o, nj))
        lr, nr = o.define_list(o.define_op_joined(occ_r, nj))
        assert n == nr
        x = random_list(n, 7)
        y = np.zeros(nr)
        o.reorder(lo, 1, x, lr, 1, y, shifts, fac=0.5, sign_reo=-1, update=False)
        assert np.allclose(y, -0.5 * x, rtol=0, atol=1e-15), name
