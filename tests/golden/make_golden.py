"""Generates tests/golden/*.npz from the reference's own host code.

Runs only where the reference tree is mounted (it uses oracle/_ref/libgsv1ref.so, compiled from
the reference sources by oracle/build_ref.sh).  Every array in the fixture comes from the
reference's functions: read_openfoam_polymesh geometry (main.cu:582-599), the BC system
(bc_runtime_config.cu / velocity_bc_eval.cu), compute_lsq_gradient (main.cu:601-618),
build_rhiechow_predicted_flux_stokes_3d (644-716), continuity_residual (718-728) and
compute_patch_forces_wall_shear (2828-2933), on a 6x4x4 jittered channel mesh.

    python tests/golden/make_golden.py
"""
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import anabasis_b200 as anb  # noqa: E402  (mesh generator only)
from tests import refshim  # noqa: E402
from tests.cases import BC_TEXT  # noqa: E402


def main():
    d = Path(tempfile.mkdtemp())
    m = anb.HostMesh.channel(6, 4, 4, jitter=0.15, seed=21)
    m.write(d)
    (d / "c.bc").write_text(BC_TEXT.format(pout=0.25))
    ref = refshim.RefMesh(d)
    g = ref.geometry()
    bc = ref.bc_eval(d / "c.bc")
    C = ref.n_cells
    rng = np.random.default_rng(2024)
    phi = np.sin(2.0 * g["cc"][0::3]) + 3.0 * g["cc"][1::3] ** 2 + 0.1 * rng.standard_normal(C)
    u = 0.3 + 0.05 * rng.standard_normal(C)
    v = 0.05 * rng.standard_normal(C)
    w = 0.05 * rng.standard_normal(C)
    p = 0.01 * rng.standard_normal(C)
    rau = 1e-3 * (1 + 0.2 * rng.random(C))
    out = {k: g[k] for k in ("cc", "vol", "xf", "nf", "sf", "af")}
    out.update({"bc_" + k: bc[k] for k in bc})
    out.update(phi=phi, u=u, v=v, w=w, p=p, rau=rau)
    for key in "uvwp":
        out["grad_" + key] = ref.gradient(bc["type_" + key], bc[key], phi)
    gp = ref.gradient(bc["type_p"], bc["p"], p)
    out["phi_star"] = ref.rhie_chow(u, v, w, p, gp, rau, bc, 1.0)
    out["div_star"] = ref.continuity(out["phi_star"])
    out["force_patch0"] = ref.patch_force(0, u, v, w, p, 1.0, 1e-3, -1)
    np.savez_compressed(Path(__file__).resolve().parent / "channel_6x4x4_j15.npz", **out)
    print("wrote", len(out), "arrays,", C, "cells")


if __name__ == "__main__":
    main()
