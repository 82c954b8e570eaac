"""Host-side mirror of the reference's scalar libraries over libanb.so.

libpoisson (libpoisson/include/{bc,poisson_library}.h, src/poisson_library.cu:3-47) and libscalar
(libscalar/include/scalar_transport_library.h, src/scalar_transport_library.cu:475-514): the same
names, option fields, argument meaning and error messages; the solves run on the GPU through
anb_scalar_elliptic_solve / anb_scalar_transport_solve.  Boundary evaluators are vectorised: they
receive one patch's face centres and unit outward normals as (n, 3) arrays and return n values
(the reference calls them once per face with the same arguments).
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field
from typing import Callable

import numpy as np

from . import HostMesh, Solver

ScalarBCFunc = Callable[[np.ndarray, np.ndarray], np.ndarray]


class ScalarBCType(enum.IntEnum):
    """Boundary kinds; values are the ANB_SCALAR_* codes of include/anb.h."""
    Dirichlet = 0
    Neumann = 1            # libpoisson Neumann / libscalar NeumannGradient: prescribed d(phi)/dn
    ZeroGradient = 2       # libscalar only


NeumannGradient = ScalarBCType.Neumann


@dataclass
class ScalarPatchBC:
    patchName: str
    type: ScalarBCType = ScalarBCType.Dirichlet
    evaluator: ScalarBCFunc | None = None


@dataclass
class ScalarBCSet:
    patches: list[ScalarPatchBC] = field(default_factory=list)


def make_dirichlet_patch_bc(patch_name: str, fn: ScalarBCFunc) -> ScalarPatchBC:
    return ScalarPatchBC(patch_name, ScalarBCType.Dirichlet, fn)


def make_neumann_patch_bc(patch_name: str, fn: ScalarBCFunc) -> ScalarPatchBC:
    return ScalarPatchBC(patch_name, ScalarBCType.Neumann, fn)


def make_neumann_gradient_patch_bc(patch_name: str, fn: ScalarBCFunc) -> ScalarPatchBC:
    return ScalarPatchBC(patch_name, ScalarBCType.Neumann, fn)


def make_zero_gradient_patch_bc(patch_name: str) -> ScalarPatchBC:
    return ScalarPatchBC(patch_name, ScalarBCType.ZeroGradient, lambda x, n: np.zeros(len(x)))


def make_dirichlet_constant_bc(patch_name: str, value: float) -> ScalarPatchBC:
    return make_dirichlet_patch_bc(patch_name, lambda x, n: np.full(len(x), float(value)))


def make_neumann_constant_bc(patch_name: str, value: float) -> ScalarPatchBC:
    return make_neumann_patch_bc(patch_name, lambda x, n: np.full(len(x), float(value)))


make_neumann_gradient_constant_bc = make_neumann_constant_bc


class ScalarMesh:
    """A mesh with its geometry and one libanb.so context for the scalar solves."""

    def __init__(self, mesh: HostMesh, device: int = 0):
        self.mesh = mesh
        self.solver = Solver(mesh, device=device)
        t = mesh.topology()
        g = mesh.geometry()
        self.patch_names = t["patch_names"]
        self.patch_start = t["patch_start"]
        self.patch_size = t["patch_size"]
        self.n_cells, self.n_faces, self.n_internal = mesh.n_cells, mesh.n_faces, mesh.n_internal
        self.cc = g["cc"].reshape(-1, 3)
        self.vol = g["vol"]
        self.xf = g["xf"].reshape(-1, 3)
        self.nf = g["nf"].reshape(-1, 3)
        self.sf = g["sf"].reshape(-1, 3)
        self.af = g["af"]
        self.max_nonorth = g["max_nonorth"]


def build_boundary_face_data(m: ScalarMesh, bc_set: ScalarBCSet, library: str = "libpoisson"):
    """Per-face BC type and value (boundary entries filled), libpoisson/src/bc.cu:3-35 or
    libscalar/src/scalar_transport_library.cu:62-118 (the latter's message for a missing patch)."""
    by_name = {}
    for bc in bc_set.patches:
        by_name[bc.patchName] = bc
    types = np.zeros(m.n_faces, np.int32)
    values = np.zeros(m.n_faces)
    for k, name in enumerate(m.patch_names):
        s, n = int(m.patch_start[k]), int(m.patch_size[k])
        if n == 0:
            continue
        bc = by_name.get(name)
        if bc is None:
            if library == "libscalar":
                raise RuntimeError(f"No scalar BC provided for patch '{name}'")
            raise RuntimeError(f"No BC supplied for patch '{name}'")
        if bc.evaluator is None:
            raise RuntimeError(f"BC evaluator missing for patch '{name}'")
        if library == "libpoisson" and bc.type == ScalarBCType.ZeroGradient:
            raise RuntimeError(f"ZeroGradient is a libscalar boundary type (patch '{name}')")
        types[s:s + n] = int(bc.type)
        values[s:s + n] = np.asarray(bc.evaluator(m.xf[s:s + n], m.nf[s:s + n]), np.float64).reshape(n)
    return types, values


@dataclass
class HypreOptions:
    """The solver controls the reference passes to HYPRE (libpoisson/include/hypre_backend.h); here
    maxIter, relTol and absTol (tol when absTol < 0) drive the library's AMG-PCG, the AMG fields
    are accepted for interface compatibility."""
    maxIter: int = 4000
    relTol: float = 0.0
    absTol: float = -1.0
    tol: float = -1.0
    monitor: int = 1
    amgMaxIter: int = 1
    amgRelaxType: int = 18
    amgCoarsenType: int = 8
    amgInterpType: int = 6
    amgAggLevels: int = 1
    amgAggInterpType: int = 4
    amgNumSweeps: int = 1
    amgRAP2: int = 0
    amgPmax: int = 4
    amgKeepTranspose: int = 1
    amgTruncFactor: float = 0.0
    amgStrongThreshold: float = -1.0


@dataclass
class EllipticOptions:
    nNonOrthCorr: int = 2
    gradScheme: str = "lsq"
    laplacianScheme: str = "nonorth"
    useReferenceCell: bool = False
    referenceCell: int = 0
    referenceValue: float = 0.0
    hypre: HypreOptions = field(default_factory=HypreOptions)


@dataclass
class EllipticResult:
    phi: np.ndarray
    iterations: int
    finalRelResNorm: float
    info: dict


def solve_scalar_elliptic(m: ScalarMesh, gamma_face, cell_source, bc_set: ScalarBCSet,
                          opts: EllipticOptions) -> EllipticResult:
    """-div(gamma grad phi) = source (libpoisson/src/poisson_library.cu:3-47)."""
    if opts.gradScheme != "lsq":
        raise RuntimeError("Only gradScheme=lsq is implemented in this build.")
    if opts.laplacianScheme not in ("orth", "nonorth"):
        raise RuntimeError("Use laplacianScheme=orth or laplacianScheme=nonorth.")
    types, values = build_boundary_face_data(m, bc_set, "libpoisson")
    h = opts.hypre
    abs_tol = h.absTol if h.absTol >= 0.0 else (h.tol if h.tol >= 0.0 else 0.0)
    phi, info = m.solver.scalar_elliptic_solve(
        cell_source, types, values, gamma_face=gamma_face, laplacian_nonorth=opts.laplacianScheme == "nonorth",
        nonorth_corr=opts.nNonOrthCorr, use_reference_cell=opts.useReferenceCell,
        reference_cell=opts.referenceCell, reference_value=opts.referenceValue, abs_tol=abs_tol,
        rel_tol=max(h.relTol, 0.0), max_iter=h.maxIter)
    return EllipticResult(phi, info["iterations"], info["final_rel_res"], info)


def solve_poisson(m: ScalarMesh, cell_source, bc_set: ScalarBCSet, opts: EllipticOptions) -> EllipticResult:
    return solve_scalar_elliptic(m, None, cell_source, bc_set, opts)


class ConvectionScheme(enum.IntEnum):
    Central = 0
    Upwind = 1


class DiffusionScheme(enum.IntEnum):
    Orth = 0
    NonOrth = 1


@dataclass
class ScalarTransportInputs:
    faceFlux: np.ndarray   # nFaces, owner -> neighbour / outward
    gammaFace: np.ndarray  # nFaces
    Su: np.ndarray         # nCells
    Sp: np.ndarray         # nCells, implicit linearised source


@dataclass
class ScalarTransportOptions:
    convectionScheme: ConvectionScheme = ConvectionScheme.Central
    diffusionScheme: DiffusionScheme = DiffusionScheme.NonOrth
    nNonOrthCorr: int = 2
    linearSolver: str = "BiCGSTAB"
    preconditioner: str = "Jacobi"
    maxIter: int = 4000
    relTol: float = 0.0
    absTol: float = 1.0e-10
    monitor: int = 0


@dataclass
class ScalarTransportResult:
    phi: np.ndarray
    iterations: int
    finalRelRes: float
    info: dict


def solve_steady_scalar_transport(m: ScalarMesh, inp: ScalarTransportInputs, bc_set: ScalarBCSet,
                                  opt: ScalarTransportOptions, x0=None) -> ScalarTransportResult:
    """div(F phi) - div(gamma grad phi) = Su + Sp phi (scalar_transport_library.cu:475-514)."""
    for name, arr, n in (("faceFlux", inp.faceFlux, m.n_faces), ("gammaFace", inp.gammaFace, m.n_faces),
                         ("Su", inp.Su, m.n_cells), ("Sp", inp.Sp, m.n_cells)):
        if len(arr) != n:
            size = "mesh.nFaces" if n == m.n_faces else "mesh.nCells"
            raise RuntimeError(f"{name} must have size {size}")
    if opt.linearSolver != "BiCGSTAB":
        raise RuntimeError("Only BiCGSTAB is implemented in this libscalar build.")
    if opt.preconditioner != "Jacobi":
        raise RuntimeError("Only Jacobi/DiagScale is implemented in this libscalar build.")
    if x0 is not None and len(x0) != m.n_cells:
        raise RuntimeError("x0 must have size mesh.nCells")
    types, values = build_boundary_face_data(m, bc_set, "libscalar")
    phi, info = m.solver.scalar_transport_solve(
        inp.gammaFace, inp.Su, types, values, face_flux=inp.faceFlux, sp=inp.Sp,
        upwind=opt.convectionScheme == ConvectionScheme.Upwind,
        diffusion_nonorth=opt.diffusionScheme == DiffusionScheme.NonOrth, nonorth_corr=opt.nNonOrthCorr,
        abs_tol=opt.absTol, rel_tol=opt.relTol, max_iter=opt.maxIter, x0=x0)
    return ScalarTransportResult(phi, info["iterations"], info["final_rel_res"], info)
