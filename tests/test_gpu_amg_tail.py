"""Two launch-saving forms of the AMG V-cycle do the per-level kernels' arithmetic in the same order,
so the SIMPLE fields must be bit-identical with them on or off, in FP64 and in the mixed-precision
method:

* the coarse tail: the small CSR levels and the dense level run as one thread-block-cluster kernel
  (ANB_AMG_TAIL_ROWS: 0 = off, a huge value = every CSR level in the tail);
* the fused down sweep: down sweep and restriction of a CSR level as one warp-per-aggregate
  kernel (ANB_AMG_FUSED_DOWN_ROWS: 0 = off, a huge value = every CSR level above the tail)."""
import os

import numpy as np
import pytest

import anabasis_b200 as anb
from tests.cases import channel, initial_state

pytestmark = pytest.mark.gpu

PRM = dict(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3, n_nonorth_corr=1)
KNOBS = ("ANB_AMG_TAIL_ROWS", "ANB_AMG_FUSED_DOWN_ROWS")


def _run(m, bc, init, precision, tail_rows, fused_rows):
    old = {k: os.environ.get(k) for k in KNOBS}
    os.environ["ANB_AMG_TAIL_ROWS"] = str(tail_rows)
    os.environ["ANB_AMG_FUSED_DOWN_ROWS"] = str(fused_rows)
    try:
        s = anb.Solver(m, anb.default_params(precision=precision, **PRM))
        s.set_bc(bc)
        s.set_state(*init)
        _, st = s.iterate(6)
        return s.get_state(), st
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.mark.parametrize("precision", [0, 1])
def test_launch_saving_forms_are_bit_identical(precision):
    # 36k cells: five or six levels, so 3000 rows splits the CSR levels between launches and tail
    m, bc, _ = channel(nx=60, ny=25, nz=24, jitter=0.15, seed=3, obstacle=True)
    init = initial_state(m, bc)
    ref, st0 = _run(m, bc, init, precision, 0, 0)
    for tail, fused in ((3000, 0), (1 << 30, 0), (0, 1 << 30), (3000, 1 << 30), (1024, 65536)):
        got, st = _run(m, bc, init, precision, tail, fused)
        assert [x["its_p_total"] for x in st] == [x["its_p_total"] for x in st0], (tail, fused)
        for k in ("u", "v", "w", "p", "phi"):
            assert np.array_equal(got[k], ref[k]), (tail, fused, k)


def _run_sell(m, bc, init, precision, sell_min_rows):
    old = os.environ.get("ANB_AMG_SELL_MIN_ROWS")
    os.environ["ANB_AMG_SELL_MIN_ROWS"] = str(sell_min_rows)
    try:
        return _run(m, bc, init, precision, 1024, 65536)
    finally:
        if old is None:
            os.environ.pop("ANB_AMG_SELL_MIN_ROWS", None)
        else:
            os.environ["ANB_AMG_SELL_MIN_ROWS"] = old


@pytest.mark.parametrize("precision", [0, 1])
def test_sell_coarse_levels_match_csr(precision):
    """Large coarse levels stored SELL-32 (run by the level-0 kernels) hold the same operator as the
    CSR form; only the summation order of a row differs, so the preconditioner is the same to
    rounding and every pressure solve still reaches its 1e-10 tolerance."""
    m, bc, _ = channel(nx=60, ny=25, nz=24, jitter=0.15, seed=3, obstacle=True)
    init = initial_state(m, bc)
    ref, st0 = _run_sell(m, bc, init, precision, 1 << 30)   # every coarse level CSR
    got, st = _run_sell(m, bc, init, precision, 1000)       # levels above 1000 rows SELL-32
    for a, b in zip(st, st0):
        assert abs(a["its_p_total"] - b["its_p_total"]) <= 2
    scale = max(np.abs(ref[k]).max() for k in ("u", "v", "w"))
    tol = 1e-7 if precision == 0 else 1e-5  # the mixed method's FP32 inner solves round differently
    for k in ("u", "v", "w"):
        assert np.abs(got[k] - ref[k]).max() <= tol * scale, k
