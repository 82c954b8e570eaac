"""The oracle's own channel case (oracle/channel.cpp) against the library's and the reference's.

The benchmark's reference arm builds its mesh and boundary values through the oracle alone (no
product library in that process), so the oracle generator must reproduce the library's channel
mesh exactly (points bit for bit, the same face order) and its boundary evaluation must reproduce
both the library's and the reference's own apply_bc_specs_to_legacy_face_arrays
(velocity_bc_eval.cu:197-290, compiled from the reference tree into oracle/_ref when present).
"""
import numpy as np
import pytest

import oracle
from tests import refshim
from tests.cases import channel

CASES = [dict(nx=6, ny=4, nz=4), dict(nx=12, ny=6, nz=6, jitter=0.15, seed=3),
         dict(nx=24, ny=10, nz=10, jitter=0.15, seed=2, obstacle=True),
         dict(nx=40, ny=14, nz=9, jitter=0.15, seed=0, obstacle=True)]


@pytest.mark.parametrize("kw", CASES)
def test_channel_mesh_matches_library(kw):
    m, bc, d = channel(**kw)
    a = m.topology()
    o, obc, state = oracle.channel_case(**kw)
    b = o.topology()
    for k in ("points", "face_offsets", "face_points", "owner", "neighbour", "patch_start", "patch_size"):
        assert np.array_equal(np.asarray(a[k]), b[k]), k
    for k in ("type_u", "type_v", "type_w", "type_p", "u", "v", "w", "p"):
        assert np.array_equal(np.asarray(bc[k]), obc[k]), k


@pytest.mark.skipif(not refshim.available(), reason="reference shim not built")
@pytest.mark.parametrize("kw", CASES[1:3])
def test_channel_bc_matches_reference(kw):
    m, bc, d = channel(**kw)
    m.write(d / "polyMesh")
    ref = refshim.RefMesh(d / "polyMesh")
    rbc = ref.bc_eval(d / "case.bc")
    o, obc, _ = oracle.channel_case(**kw)
    for k in ("type_u", "type_v", "type_w", "type_p", "u", "v", "w", "p"):
        assert np.array_equal(np.asarray(rbc[k]), obc[k]), k


def test_channel_case_runs_without_library():
    o, bc, state = oracle.channel_case(8, 4, 4, jitter=0.1, seed=1, obstacle=False)
    s, st = o.run(oracle.params(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3), 2, *state)
    assert len(st) == 2 and np.isfinite(s["u"]).all()


def test_amg_pcg_matches_jacobi_pcg():
    """The oracle's aggregation-AMG PCG (the timed CPU baseline's pressure solver, standing in for the
    reference's BoomerAMG-PCG) reaches the same SIMPLE fields as its Jacobi PCG at near round-off
    inner tolerances, with far fewer iterations."""
    from tests.cases import initial_state

    m, bc, _ = channel(nx=24, ny=10, nz=10, jitter=0.15, seed=2, obstacle=True)
    init = initial_state(m, bc)
    out = {}
    for amg in (0, 1):
        o = oracle.Oracle(m.topology())
        o.set_bc(bc)
        prm = oracle.params(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3, vel_tol=1e-15, p_tol=1e-15, vel_maxit=5000,
                            p_maxit=20000, tol_mass=0.0, tol_vel=0.0, p_use_amg=amg)
        out[amg] = o.run(prm, 5, *init)
    (r0, s0), (r1, s1) = out[0], out[1]
    for k in ("u", "v", "w", "p"):
        assert np.abs(r1[k] - r0[k]).max() <= 1e-10 * np.abs(r0[k]).max(), k
    assert sum(x["its_p_total"] for x in s1) * 3 < sum(x["its_p_total"] for x in s0)
