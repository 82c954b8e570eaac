"""Cell fields across the host/device boundary (anb_set_state / anb_get_state): the staged,
chunked copies and the device-side permutation between input and layout numbering return every
value bit for bit, on a mesh of one chunk per field and on one of several chunks per field; a
null pressure array leaves the caller's array alone; set_state zeroes the face fluxes."""
import ctypes as ct

import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, random_state

pytestmark = pytest.mark.gpu
PRM = dict(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3)


@pytest.mark.parametrize("shape", [(12, 6, 6), (140, 66, 66)])
def test_state_round_trip_is_exact(shape):
    m, bc, _ = channel(*shape, jitter=0.1, seed=3, obstacle=True)
    s = anb.Solver(m, anb.default_params(**PRM))
    s.set_bc(bc)
    st = random_state(m, seed=7)
    s.set_state(*st)
    g = s.get_state(with_phi=True)
    for k, a in zip("uvwp", st):
        assert np.array_equal(g[k], a), k
    assert not np.any(g["phi"])
    # refilled arrays, and a second set_state after a step overwrites every value
    s.iterate(1)
    st2 = random_state(m, seed=8)
    s.set_state(*st2)
    s.get_state(with_phi=False, out=g)
    for k, a in zip("uvwp", st2):
        assert np.array_equal(g[k], a), k


def test_get_state_without_pressure_leaves_it_alone():
    m, bc, _ = channel(20, 8, 8, jitter=0.1, seed=4)
    s = anb.Solver(m, anb.default_params(**PRM))
    s.set_bc(bc)
    st = random_state(m, seed=9)
    s.set_state(*st)
    C = m.n_cells
    u, v, w = np.zeros(C), np.zeros(C), np.zeros(C)
    p = np.full(C, -5.0)
    dp = ct.POINTER(ct.c_double)
    rc = anb.lib().anb_get_state(s._h, u.ctypes.data_as(dp), v.ctypes.data_as(dp), w.ctypes.data_as(dp), None, None)
    assert rc == anb.ANB_OK
    assert np.array_equal(u, st[0]) and np.array_equal(v, st[1]) and np.array_equal(w, st[2])
    assert np.all(p == -5.0)
