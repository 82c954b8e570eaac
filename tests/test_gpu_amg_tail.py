"""The coarse tail of the AMG V-cycle (the small CSR levels and the dense level run as one
thread-block-cluster kernel) does the per-level kernels' arithmetic in the same order, so the
SIMPLE fields must be bit-identical with the tail off, on and covering every CSR level, in FP64 and
in the mixed-precision method."""
import os

import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, initial_state

pytestmark = pytest.mark.gpu

PRM = dict(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3, n_nonorth_corr=1)


def _run(m, bc, init, tail_rows, precision):
    old = os.environ.get("ANB_AMG_TAIL_ROWS")
    os.environ["ANB_AMG_TAIL_ROWS"] = str(tail_rows)
    try:
        s = anb.Solver(m, anb.default_params(precision=precision, **PRM))
        s.set_bc(bc)
        s.set_state(*init)
        _, st = s.iterate(6)
        return s.get_state(), st
    finally:
        if old is None:
            os.environ.pop("ANB_AMG_TAIL_ROWS")
        else:
            os.environ["ANB_AMG_TAIL_ROWS"] = old


@pytest.mark.parametrize("precision", [0, 1])
def test_tail_is_bit_identical(precision):
    # 36k cells: five or six levels, so 3000 rows splits the CSR levels between launches and tail
    m, bc, _ = channel(nx=60, ny=25, nz=24, jitter=0.15, seed=3, obstacle=True)
    init = initial_state(m, bc)
    ref, st0 = _run(m, bc, init, 0, precision)
    for rows in (3000, 1 << 30):
        got, st = _run(m, bc, init, rows, precision)
        assert [x["its_p_total"] for x in st] == [x["its_p_total"] for x in st0], rows
        for k in ("u", "v", "w", "p", "phi"):
            assert np.array_equal(got[k], ref[k]), (rows, k)
