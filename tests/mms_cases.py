"""Manufactured-solution problems of the reference's scalar-library apps, on unit-cube meshes.

  poisson_dirichlet  apps/poisson_mms_lib/main.cu with libpoisson/include/mms.h: phi = sin sin sin,
                     -lap phi = 3 pi^2 phi, Dirichlet everywhere, nNonOrthCorr 10 (app default)
  poisson_neumann    apps/poisson_mms_neumann_lib/main.cu: phi = cos cos cos, pure Neumann with the
                     volume-mean source removed, reference cell 0 fixed to the exact value
  poisson_mixed      apps/poisson_mms_mixed_lib/main.cu: cos cos cos, Dirichlet on the x = 0 patch,
                     Neumann elsewhere
  transport_central  apps/scalar_mms_lib/main.cu defaults: sin sin sin convected by
                     u = (1 + y, 0.5 - x, 0.25), gamma 0.1, central convection, orthogonal diffusion
  transport_upwind_mixed  same field, upwind convection, non-orthogonal diffusion (2 correctors),
                     Dirichlet on x = 0 and the side walls, prescribed normal gradient on x = 1

Each problem is evaluated from the geometry the reference computes (cell centres and volumes, face
centres, unit normals and area vectors) exactly as the apps do.
"""
from __future__ import annotations

import numpy as np

import anabasis_b200 as anb

PI = 3.141592653589793238462643383279502884
PROBLEMS = ["poisson_dirichlet", "poisson_neumann", "poisson_mixed", "transport_central", "transport_upwind_mixed"]
# patch names of the channel generator: walls (y, z), x = 0, x = 1
WALLS, INLET, OUTLET = "patch_0_0", "patch_1_0", "patch_2_0"


def unit_cube(n: int, jitter: float = 0.0, seed: int = 0, tets: bool = False) -> anb.HostMesh:
    return anb.HostMesh.channel(n, n, n, lx=1.0, ly=1.0, lz=1.0, jitter=jitter, seed=seed, tets=tets)


def sin3(x):
    return np.sin(PI * x[:, 0]) * np.sin(PI * x[:, 1]) * np.sin(PI * x[:, 2])


def grad_sin3(x):
    s, c = np.sin(PI * x), np.cos(PI * x)
    return PI * np.stack([c[:, 0] * s[:, 1] * s[:, 2], s[:, 0] * c[:, 1] * s[:, 2], s[:, 0] * s[:, 1] * c[:, 2]], 1)


def cos3(x):
    return np.cos(PI * x[:, 0]) * np.cos(PI * x[:, 1]) * np.cos(PI * x[:, 2])


def grad_cos3(x):
    s, c = np.sin(PI * x), np.cos(PI * x)
    return -PI * np.stack([s[:, 0] * c[:, 1] * c[:, 2], c[:, 0] * s[:, 1] * c[:, 2], c[:, 0] * c[:, 1] * s[:, 2]], 1)


def velocity(x):
    return np.stack([1.0 + x[:, 1], 0.5 - x[:, 0], np.full(len(x), 0.25)], 1)


def geometry(mesh: anb.HostMesh) -> dict:
    t = mesh.topology()
    g = mesh.geometry()
    return dict(cc=g["cc"].reshape(-1, 3), vol=g["vol"], xf=g["xf"].reshape(-1, 3), nf=g["nf"].reshape(-1, 3),
                sf=g["sf"].reshape(-1, 3), names=t["patch_names"], start=t["patch_start"], size=t["patch_size"],
                n_internal=mesh.n_internal, n_faces=mesh.n_faces, owner=t["owner"], neighbour=t["neighbour"])


def _bc(geo, dirichlet_patches, value_fn, grad_fn, neumann_type=1):
    F = geo["n_faces"]
    bt = np.zeros(F, np.int32)
    bv = np.zeros(F)
    for k, name in enumerate(geo["names"]):
        s, n = int(geo["start"][k]), int(geo["size"][k])
        x, nrm = geo["xf"][s:s + n], geo["nf"][s:s + n]
        if dirichlet_patches is None or name in dirichlet_patches:
            bt[s:s + n] = 0
            bv[s:s + n] = value_fn(x)
        else:
            bt[s:s + n] = neumann_type
            bv[s:s + n] = (grad_fn(x) * nrm).sum(1)
    return bt, bv


def problem(name: str, geo: dict) -> dict:
    """Inputs of one MMS problem: src/su, sp, flux, gamma, bc arrays, options, exact cell values."""
    C, F = len(geo["vol"]), geo["n_faces"]
    cc = geo["cc"]
    if name == "poisson_dirichlet":
        bt, bv = _bc(geo, None, sin3, grad_sin3)
        return dict(transport=False, src=3.0 * PI * PI * sin3(cc), gamma=np.ones(F), bt=bt, bv=bv, nonorth=True,
                    n_corr=10, ref_cell=-1, ref_value=0.0, exact=sin3(cc))
    if name == "poisson_neumann":
        bt, bv = _bc(geo, set(), cos3, grad_cos3)
        src = 3.0 * PI * PI * cos3(cc)
        src = src - (src * geo["vol"]).sum() / geo["vol"].sum()
        return dict(transport=False, src=src, gamma=np.ones(F), bt=bt, bv=bv, nonorth=True, n_corr=10, ref_cell=0,
                    ref_value=float(cos3(cc[:1])[0]), exact=cos3(cc))
    if name == "poisson_mixed":
        bt, bv = _bc(geo, {INLET}, cos3, grad_cos3)
        return dict(transport=False, src=3.0 * PI * PI * cos3(cc), gamma=np.ones(F), bt=bt, bv=bv, nonorth=True,
                    n_corr=10, ref_cell=-1, ref_value=0.0, exact=cos3(cc))
    gamma = 0.1
    flux = (velocity(geo["xf"]) * geo["sf"]).sum(1)
    su = (velocity(cc) * grad_sin3(cc)).sum(1) + 3.0 * gamma * PI * PI * sin3(cc)
    if name == "transport_central":
        bt, bv = _bc(geo, None, sin3, grad_sin3)
        return dict(transport=True, src=su, sp=np.zeros(C), flux=flux, gamma=np.full(F, gamma), bt=bt, bv=bv,
                    upwind=False, nonorth=False, n_corr=0, exact=sin3(cc))
    if name == "transport_upwind_mixed":
        bt, bv = _bc(geo, {INLET, WALLS}, sin3, grad_sin3)
        return dict(transport=True, src=su, sp=np.zeros(C), flux=flux, gamma=np.full(F, gamma), bt=bt, bv=bv,
                    upwind=True, nonorth=True, n_corr=2, exact=sin3(cc))
    raise KeyError(name)


# mesh sequences of the order study: (label, sizes, jitter, tets)
SEQUENCES = [("hex", (8, 16, 32), 0.0, False), ("hex_jitter", (8, 16, 32), 0.15, False),
             ("tet", (4, 8, 16), 0.0, True)]


def oracle_solve(asm, p: dict) -> np.ndarray:
    from oracle import mms

    if p["transport"]:
        return mms.solve_transport(asm, p["gamma"], p["src"], p["sp"], p["flux"], p["bt"], p["bv"],
                                   upwind=p["upwind"], nonorth=p["nonorth"], n_corr=p["n_corr"])
    return mms.solve_elliptic(asm, p["gamma"], p["src"], p["bt"], p["bv"], nonorth=p["nonorth"], n_corr=p["n_corr"],
                              ref_cell=p["ref_cell"], ref_value=p["ref_value"])


def gpu_solve(solver: anb.Solver, p: dict) -> tuple[np.ndarray, dict]:
    if p["transport"]:
        return solver.scalar_transport_solve(p["gamma"], p["src"], p["bt"], p["bv"], face_flux=p["flux"], sp=p["sp"],
                                             upwind=p["upwind"], diffusion_nonorth=p["nonorth"],
                                             nonorth_corr=p["n_corr"], abs_tol=1e-13, max_iter=20000)
    return solver.scalar_elliptic_solve(p["src"], p["bt"], p["bv"], gamma_face=p["gamma"],
                                        laplacian_nonorth=p["nonorth"], nonorth_corr=p["n_corr"],
                                        use_reference_cell=p["ref_cell"] >= 0, reference_cell=max(p["ref_cell"], 0),
                                        reference_value=p["ref_value"], abs_tol=1e-13, max_iter=4000)


def orders(errs: list[float]) -> list[float]:
    return [float(np.log(errs[i] / errs[i + 1]) / np.log(2.0)) for i in range(len(errs) - 1)]
