"""Parity on the benchmark configurations themselves (FP64 plain method).

* Config 1: the 40 x 20 x 20 channel (16,000 hexes), parabolic box inlet H = 0.41, Umax = 0.45,
  fixed-p outlet, no-slip walls, rho 1, mu 1e-3, relaxation 0.7 / 0.3, 2 non-orthogonal
  correctors, 300 outer iterations.  The drop-in program runs against the reference program
  compiled from its own sources (oracle/_ref/gsv1_ref, HYPRE replaced by a host Jacobi-CG /
  BiCGSTAB stand-in) on the same polyMesh and case file, and the library runs against the CPU
  oracle, both with inner tolerances near round-off so the result does not depend on the linear
  solver (the fixed-iteration protocol of the reference's SIMPLE loop, main.cu:3388-3634).
* Config 2: the 200 x 70 x 70 obstacle channel (970,480 jittered hexes, seed 0), the benchmark's
  own workload, for a few outer iterations against the oracle.  At this size the pressure AMG has
  its full depth: SELL-32 coarse levels above 65,536 rows, the fused coarse down sweep and the
  cluster tail all run on their real shapes.

Bar: 1e-8 relative to each field's largest magnitude for u, v, w, p and the face flux, and to the
largest force component for the nine patch-force components.
"""
import subprocess

import numpy as np
import pytest

import anabasis_b200 as anb
import oracle
from tests.cases import channel, initial_state, rel_err
from tests.test_gpu_reference_run import CASE, REF_BIN, read_summary, read_vtu_fields

pytestmark = pytest.mark.gpu

PRM = dict(rho=1.0, mu=1e-3, u_relax=0.7, p_relax=0.3, n_nonorth_corr=2)
FKEYS = [f"{f}Force_{x}" for f in ("pressure", "viscous", "total") for x in "xyz"]


@pytest.mark.skipif(not REF_BIN.exists(), reason="reference program not built (oracle/build_ref.sh)")
def test_config1_against_reference_program(tmp_path):
    m, bc, _ = channel(40, 20, 20)
    assert m.n_cells == 16000
    mesh_dir = tmp_path / "constant" / "polyMesh"
    m.write(mesh_dir)
    steps = 300
    runs = {}
    for tag, exe in (("ref", REF_BIN), ("anb", anb.APP_PATH)):
        case = tmp_path / f"{tag}.case"
        case.write_text(CASE.format(mesh=mesh_dir, out=tmp_path / tag, nsteps=steps, force="patch_0_0", extra=""))
        r = subprocess.run([str(exe), "-case-config", str(case)], capture_output=True, text=True, timeout=1500)
        assert r.returncode == 0, (tag, r.stdout[-2000:], r.stderr[-2000:])
        runs[tag] = dict(vtu=read_vtu_fields(tmp_path / f"{tag}_final.vtu"),
                         summary=read_summary(tmp_path / f"{tag}_summary.txt"))
    a, b = runs["anb"], runs["ref"]
    assert a["summary"]["steps"] == b["summary"]["steps"] == steps
    assert rel_err(a["vtu"]["U"], b["vtu"]["U"]) < 1e-8
    assert rel_err(a["vtu"]["p"], b["vtu"]["p"]) < 1e-8
    fscale = max(abs(b["summary"][k]) for k in FKEYS)
    for k in FKEYS:
        assert abs(a["summary"][k] - b["summary"][k]) <= 1e-8 * fscale, k
    for k in ("maxAbsU", "maxAbsV", "maxAbsW", "maxAbsP", "patchForceArea"):
        assert abs(a["summary"][k] - b["summary"][k]) <= 1e-8 * abs(b["summary"][k]), k


def _library_vs_oracle(m, bc, steps, tight, force_patch):
    params = anb.default_params(**PRM, **tight)
    s = anb.Solver(m, params)
    s.set_bc(bc)
    u0, v0, w0, p0 = initial_state(m, bc)
    s.set_state(u0, v0, w0, p0)
    rc, st = s.iterate(steps)
    assert len(st) == steps
    g = s.get_state()
    o = oracle.Oracle(m.topology())
    o.set_bc(bc)
    # no early stop in the oracle either (config 1 meets 1e-10 after 95 steps): both run `steps` steps
    ref, rst = o.run(oracle.params(**PRM, **tight, n_threads=0, tol_mass=0.0, tol_vel=0.0), steps, u0, v0, w0,
                     p0)
    assert len(rst) == steps
    for k in ("u", "v", "w", "p", "phi"):
        assert rel_err(g[k], ref[k]) < 1e-8, (k, rel_err(g[k], ref[k]))
    k = m.topology()["patch_names"].index(force_patch)
    f = s.patch_force(k, -1)
    fo = o.patch_force(k, -1, PRM["mu"], ref["u"], ref["v"], ref["w"], ref["p"])
    got = np.array(f["Fp"] + f["Fv"] + f["F"])
    assert np.abs(got - fo[:9]).max() <= 1e-8 * np.abs(fo[:9]).max()
    # the monitors of every step
    for a, b in zip(st, rst):  # (a converged run's du sits at the round-off level, ~1e-11)
        assert abs(a["du_rel"] - b["du"]) <= 1e-6 * b["du"] + 1e-12
    return st, rst


def test_config1_against_oracle():
    m, bc, _ = channel(40, 20, 20)
    tight = dict(vel_tol=1e-15, p_tol=1e-15, vel_maxit=5000, p_maxit=20000)
    _library_vs_oracle(m, bc, 300, tight, "patch_0_0")


def test_config2_against_oracle():
    m, bc, _ = channel(200, 70, 70, jitter=0.15, seed=0, obstacle=True)
    assert (m.n_cells, m.n_internal) == (970480, 2876926)
    # momentum to 1e-13 absolute (about 1e-15 of |b| here; tighter sits on the round-off floor of a
    # 970k-row BiCGSTAB), pressure to 1e-15 absolute (1e-13 of |b|)
    tight = dict(vel_tol=1e-13, p_tol=1e-15, vel_maxit=5000, p_maxit=20000)
    _library_vs_oracle(m, bc, 4, tight, "patch_3_0")
