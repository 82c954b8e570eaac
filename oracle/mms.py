"""Oracle solve loops of the reference's scalar libraries (TEST INFRASTRUCTURE ONLY).

The outer loops restate solve_scalar_elliptic (libpoisson/src/poisson_library.cu:3-47) and
solve_steady_scalar_transport (libscalar/src/scalar_transport_library.cu:475-514): per pass, the
LSQ gradient of the current phi, assembly, one linear solve.  The assemblies are the oracle's C++
restatements (orc_scalar_gradient / orc_scalar_assemble) or, through `ref`, the reference's own
host functions; the linear solves are SuperLU (scipy), exact to rounding, standing in for
HYPRE's PCG+BoomerAMG and BiCGSTAB+DiagScale (HYPRE is not vendored).  Only tests/ may use it.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sps
import scipy.sparse.linalg as spla


def face_form_csr(n_cells, owner, neigh, sys) -> sps.csr_matrix:
    """diag / a_pn / a_np face-coefficient form -> CSR."""
    I = len(neigh)
    rows = np.concatenate([np.arange(n_cells), owner[:I], neigh])
    cols = np.concatenate([np.arange(n_cells), neigh, owner[:I]])
    vals = np.concatenate([sys["diag"], sys["a_pn"], sys["a_np"]])
    return sps.csr_matrix((vals, (rows, cols)), shape=(n_cells, n_cells))


class OracleAssembler:
    """Gradient + assembly from the oracle restatement."""

    def __init__(self, oracle, topo):
        self.o = oracle
        self.n = oracle.n_cells
        self.owner = np.asarray(topo["owner"])
        self.neigh = np.asarray(topo["neighbour"])

    def gradient(self, transport, bt, bv, phi):
        return self.o.scalar_gradient(bt, bv, phi)

    def system(self, transport, upwind, nonorth, gamma, src, sp, flux, bt, bv, grad, ref_cell, ref_value):
        s = self.o.scalar_assemble(transport, upwind, nonorth, gamma, src, bt, bv, grad, flux=flux, sp=sp,
                                   ref_cell=ref_cell, ref_value=ref_value)
        return face_form_csr(self.n, self.owner, self.neigh, s), s["rhs"]


def linear_solve(A: sps.csr_matrix, b: np.ndarray, x0=None, rtol: float = 1e-14) -> np.ndarray:
    """Jacobi-preconditioned CG (symmetric A) or BiCGSTAB to ||r|| <= rtol ||b||; SuperLU for small
    systems or when the iteration stalls."""
    n = A.shape[0]
    if n <= 4000:
        return spla.spsolve(A.tocsc(), b)
    dinv = 1.0 / A.diagonal()
    M = spla.LinearOperator((n, n), matvec=lambda v: dinv * v)
    sym = abs(A - A.T).max() <= 1e-14 * abs(A).max()
    fn = spla.cg if sym else spla.bicgstab
    x, info = fn(A, b, x0=x0, rtol=rtol, atol=0.0, maxiter=50 * n, M=M)
    if info != 0 or np.linalg.norm(b - A @ x) > 10 * rtol * np.linalg.norm(b):
        x = spla.spsolve(A.tocsc(), b)
    return x


def solve_elliptic(asm, gamma, src, bt, bv, nonorth=True, n_corr=2, ref_cell=-1, ref_value=0.0):
    n_outer = n_corr + 1 if nonorth else 1
    phi = np.zeros(asm.n)
    for _ in range(n_outer):
        grad = asm.gradient(False, bt, bv, phi)
        A, b = asm.system(False, False, nonorth, gamma, src, None, None, bt, bv, grad, ref_cell, ref_value)
        phi = linear_solve(A, b, x0=phi)
    return phi


def solve_transport(asm, gamma, su, sp, flux, bt, bv, upwind=False, nonorth=False, n_corr=0, x0=None):
    n_outer = n_corr + 1 if nonorth else 1
    phi = np.zeros(asm.n) if x0 is None else np.array(x0, np.float64)
    for _ in range(n_outer):
        grad = asm.gradient(True, bt, bv, phi)
        A, b = asm.system(True, upwind, nonorth, gamma, su, sp, flux, bt, bv, grad, -1, 0.0)
        phi = linear_solve(A, b, x0=phi)
    return phi


def error_norms(phi, exact, vol) -> dict:
    """Volume-weighted L1 / L2 and max errors (apps/poisson_mms_lib/main.cu:182-200)."""
    err = np.abs(phi - exact)
    V = vol.sum()
    return dict(l1=float((vol * err).sum() / V), l2=float(np.sqrt((vol * err * err).sum() / V)),
                linf=float(err.max()))
