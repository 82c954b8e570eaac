"""PCG SpMV with the matrix slots staged in shared memory by bulk copies (k_pcg_pq_staged) against
the register kernel (k_pcg_pq, ANB_SELL_STAGED=0).  Each row's arithmetic is the same, in the same
order; the p.q partial sums follow the grid, and the two kernels get different full-wave grids
where their occupancies differ (rows of at most four slots: 8 staged blocks per SM against 6).
With the grid fixed (ANB_GRID=fixed, both kernels on the same number of blocks) a few SIMPLE steps
give bit-identical fields and iteration counts, in FP64 and in the mixed-precision inner solves,
on meshes whose rows fill one partial chunk, several chunks per block, and hex (6-slot) and tet
(4-slot) rows; with the default grids the fields agree to the solver tolerance."""
import os

import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, initial_state

pytestmark = pytest.mark.gpu

PRM = dict(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3, n_nonorth_corr=2)
SHAPES = [(24, 10, 10, False), (120, 50, 50, False), (90, 40, 40, True)]


def _run(m, bc, steps, staged, fixed_grid, **kw):
    env = {"ANB_SELL_STAGED": "1" if staged else "0"}
    if fixed_grid:
        env["ANB_GRID"] = "fixed"
    os.environ.update(env)
    try:
        s = anb.Solver(m, anb.default_params(**PRM, **kw))
        s.set_bc(bc)
        s.set_state(*initial_state(m, bc))
        _, st = s.iterate(steps)
        g = s.get_state()
        s.close()
    finally:
        for k in env:
            os.environ.pop(k, None)
    return g, st


def _case(shape):
    nx, ny, nz, tets = shape
    return channel(nx=nx, ny=ny, nz=nz, jitter=0.15, seed=2, obstacle=not tets, tets=tets)


@pytest.mark.parametrize("kw", [dict(), dict(precision=1)])
@pytest.mark.parametrize("shape", SHAPES)
def test_staged_spmv_matches_register_kernel(kw, shape):
    m, bc, _ = _case(shape)
    g0, st0 = _run(m, bc, 4, False, True, **kw)
    g1, st1 = _run(m, bc, 4, True, True, **kw)
    assert [x["its_p_total"] for x in st0] == [x["its_p_total"] for x in st1]
    for k in ("u", "v", "w", "p", "phi"):
        assert np.array_equal(g0[k], g1[k]), k


def test_staged_spmv_default_grid_within_solver_tolerance():
    m, bc, _ = _case(SHAPES[2])
    g0, _ = _run(m, bc, 4, False, False)
    g1, _ = _run(m, bc, 4, True, False)
    for k in ("u", "v", "w", "p"):
        scale = max(np.max(np.abs(g0[k])), 1e-30)
        assert np.max(np.abs(g0[k] - g1[k])) <= 1e-6 * scale, k
