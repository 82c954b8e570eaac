"""Solver loops as one graph launch: a while node over pairs of AMG-PCG iterations (pressure) or
of Jacobi-BiCGSTAB iterations (momentum), its condition set on the device.

The loop graphs replay the same kernels with the same arguments as the host-driven loops (the
reference's HYPRE PCG and BiCGSTAB solves, apps/generic_simple_v1/src/main.cu:2584-2641 and 2570), so the fields and the
iteration counts of a few SIMPLE steps must equal those of a run with ANB_NO_LOOP_GRAPH=1 bit for bit,
in FP64 and in the mixed-precision inner solves, also when every solve is done at its start.
"""
import os

import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, initial_state

pytestmark = pytest.mark.gpu

PRM = dict(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3)


def _run(m, bc, steps, no_loop, **kw):
    if no_loop:
        os.environ["ANB_NO_LOOP_GRAPH"] = "1"
    try:
        s = anb.Solver(m, anb.default_params(**PRM, **kw))
        s.set_bc(bc)
        s.set_state(*initial_state(m, bc))
        _, st = s.iterate(steps)
        g = s.get_state()
        s.close()
    finally:
        os.environ.pop("ANB_NO_LOOP_GRAPH", None)
    return g, st


@pytest.mark.parametrize("kw", [dict(), dict(precision=1), dict(n_nonorth_corr=2, n_pressure_corr=1)])
def test_loop_graph_matches_host_loop(kw):
    m, bc, _ = channel(nx=24, ny=10, nz=10, jitter=0.15, seed=2, obstacle=True)
    g0, st0 = _run(m, bc, 6, True, **kw)
    g1, st1 = _run(m, bc, 6, False, **kw)
    for k in ("u", "v", "w", "p", "phi"):
        assert np.array_equal(g0[k], g1[k]), k
    for key in ("its_p_total", "its_u", "its_v", "its_w"):
        assert [x[key] for x in st0] == [x[key] for x in st1], key


def test_solve_done_at_init():
    # every pressure solve starts below its (huge) tolerance: no iteration, the same fields
    m, bc, _ = channel(nx=12, ny=6, nz=6)
    g0, st0 = _run(m, bc, 3, True, p_tol=1e30)
    g1, st1 = _run(m, bc, 3, False, p_tol=1e30)
    assert all(x["its_p_total"] == 0 for x in st1), st1
    for k in ("u", "v", "w", "p", "phi"):
        assert np.array_equal(g0[k], g1[k]), k
