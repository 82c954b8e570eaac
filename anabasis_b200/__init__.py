"""anabasis_b200 - B200 implementation of the steady SIMPLE outer iteration of the reference's
generic_simple_v1 (OpenFOAM polyMesh, runtime .case/.bc boundary conditions).

The product is the C ABI library ``_lib/libanb.so`` (include/anb.h, include/anb_host.h) and the
drop-in executable ``_lib/anabasis_simple``.  This module is a thin ctypes mirror used by tests
and the benchmark; it never computes anything itself and raises if the library is missing.
"""
from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "_lib" / "libanb.so"
APP_PATH = _PKG / "_lib" / "anabasis_simple"

ANB_OK = 0
ANB_NOT_CONVERGED = 1
ANB_ERR_INVALID = 2
ANB_ERR_CUDA = 3
ANB_ERR_MESH = 4
ANB_ERR_IO = 5
ANB_ERR_UNSUPPORTED = 6
ANB_ERR_DIVERGED = 7

_lib = None

_dp = ct.POINTER(ct.c_double)
_ip = ct.POINTER(ct.c_int)


class MeshDesc(ct.Structure):
    _fields_ = [("n_points", ct.c_int), ("points", _dp), ("n_faces", ct.c_int), ("face_offsets", _ip),
                ("face_points", _ip), ("n_internal_faces", ct.c_int), ("owner", _ip), ("neighbour", _ip),
                ("n_patches", ct.c_int), ("patch_start", _ip), ("patch_size", _ip)]


class Params(ct.Structure):
    _fields_ = [("rho", ct.c_double), ("mu", ct.c_double), ("u_relax", ct.c_double), ("p_relax", ct.c_double),
                ("n_nonorth_corr", ct.c_int), ("n_vel_nonorth_corr", ct.c_int), ("n_pressure_corr", ct.c_int),
                ("vel_maxit", ct.c_int), ("vel_tol", ct.c_double), ("vel_rel_tol", ct.c_double),
                ("p_maxit", ct.c_int), ("p_tol", ct.c_double), ("p_rel_tol", ct.c_double),
                ("corr_tol", ct.c_double), ("p_amg_rebuild_every", ct.c_int), ("p_use_amg", ct.c_int),
                ("precision", ct.c_int), ("device", ct.c_int), ("p_amg_setup_scope", ct.c_int),
                ("mom_amg", ct.c_int), ("mixed_refine", ct.c_int), ("mixed_inner_rtol", ct.c_double)]


class IterStats(ct.Structure):
    _fields_ = [("step", ct.c_int), ("status", ct.c_int), ("mass_res", ct.c_double), ("du_rel", ct.c_double),
                ("dv_rel", ct.c_double), ("dw_rel", ct.c_double), ("dp_rel", ct.c_double), ("its_u", ct.c_int),
                ("its_v", ct.c_int), ("its_w", ct.c_int), ("its_p_last", ct.c_int), ("its_p_total", ct.c_int),
                ("iter_seconds", ct.c_double)]


class ForceReport(ct.Structure):
    _fields_ = [("valid", ct.c_int), ("n_faces", ct.c_int), ("area", ct.c_double), ("Fp", ct.c_double * 3),
                ("Fv", ct.c_double * 3), ("F", ct.c_double * 3), ("min_wall_distance", ct.c_double),
                ("max_wall_distance", ct.c_double), ("max_ut", ct.c_double), ("max_shear_mag", ct.c_double)]


class AdjointInfo(ct.Structure):
    _fields_ = [("iterations", ct.c_int), ("converged", ct.c_int), ("res_norm", ct.c_double),
                ("rhs_norm", ct.c_double), ("seconds", ct.c_double), ("prec_mom_its", ct.c_int),
                ("prec_p_its", ct.c_int)]


class SolveInfo(ct.Structure):
    _fields_ = [("iterations", ct.c_int), ("converged", ct.c_int), ("outer", ct.c_int),
                ("final_res_norm", ct.c_double), ("final_rel_res", ct.c_double)]


# exported symbols and their signatures (restype, argtypes); checked against include/*.h by tests
SIGNATURES = {
    "anb_default_params": (None, [ct.POINTER(Params)]),
    "anb_create": (ct.c_int, [ct.POINTER(MeshDesc), ct.POINTER(Params), ct.POINTER(ct.c_void_p)]),
    "anb_destroy": (None, [ct.c_void_p]),
    "anb_last_error": (ct.c_char_p, [ct.c_void_p]),
    "anb_setup_times": (ct.c_int, [ct.c_void_p, _dp]),
    "anb_get_geometry": (ct.c_int, [ct.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp]),
    "anb_get_sizes": (ct.c_int, [ct.c_void_p, _ip, _ip, _ip, _ip]),
    "anb_set_bc": (ct.c_int, [ct.c_void_p, _ip, _ip, _ip, _ip, _dp, _dp, _dp, _dp]),
    "anb_set_state": (ct.c_int, [ct.c_void_p, _dp, _dp, _dp, _dp]),
    "anb_get_state": (ct.c_int, [ct.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    "anb_simple_iterate": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_double, ct.c_double, ct.POINTER(IterStats), _ip]),
    "anb_patch_force": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.POINTER(ForceReport)]),
    "anb_patch_force_nalloc": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, ct.POINTER(ForceReport)]),
    "anb_set_viscosity": (ct.c_int, [ct.c_void_p, ct.c_double]),
    "anb_steady_residual": (ct.c_int, [ct.c_void_p, _dp, _dp]),
    "anb_force_objective": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, _dp, _dp, _dp]),
    "anb_newton_solve": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_double, ct.c_int, _ip, _dp,
                                    ct.POINTER(AdjointInfo)]),
    "anb_tangent_linear": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, _dp, _dp, ct.c_double, _dp,
                                      ct.POINTER(AdjointInfo)]),
    "anb_adjoint_force_grad": (ct.c_int, [ct.c_void_p, ct.c_int, ct.c_int, _dp, _dp, _dp, _dp,
                                          ct.POINTER(AdjointInfo)]),
    "anb_debug_jvp": (ct.c_int, [ct.c_void_p, _dp, _dp, ct.c_double, _dp]),
    "anb_debug_vjp": (ct.c_int, [ct.c_void_p, _dp, _dp, _dp, _dp]),
    "anb_scalar_elliptic_solve": (ct.c_int, [ct.c_void_p, _dp, _dp, _ip, _dp, ct.c_int, ct.c_int, ct.c_int, ct.c_int,
                                             ct.c_double, ct.c_double, ct.c_double, ct.c_int, _dp,
                                             ct.POINTER(SolveInfo)]),
    "anb_scalar_transport_solve": (ct.c_int, [ct.c_void_p, _dp, _dp, _dp, _dp, _ip, _dp, ct.c_int, ct.c_int, ct.c_int,
                                              ct.c_double, ct.c_double, ct.c_int, _dp, _dp, ct.POINTER(SolveInfo)]),
    "anb_profile_select": (ct.c_int, [ct.c_void_p, ct.c_int]),
    "anb_profile_read": (ct.c_int, [ct.c_void_p, ct.POINTER(ct.c_longlong), _dp, _dp]),
    "anb_launch_count": (ct.c_longlong, []),
    "anb_debug_gradient": (ct.c_int, [ct.c_void_p, ct.c_int, _dp, _dp, _dp, _dp]),
    "anb_debug_momentum": (ct.c_int, [ct.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "anb_debug_pressure": (ct.c_int, [ct.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "anb_debug_pressure_solve": (ct.c_int, [ct.c_void_p, _dp, _dp, _ip, _dp]),
    "anb_debug_nonorth": (ct.c_int, [ct.c_void_p, _dp, _dp, _dp, _dp, _dp]),
    "anb_mesh_read_polymesh": (ct.c_int, [ct.c_char_p, ct.POINTER(ct.c_void_p), ct.c_char_p, ct.c_int]),
    "anb_mesh_make_channel": (ct.c_int, [ct.c_int, ct.c_int, ct.c_int, ct.c_double, ct.c_double, ct.c_double,
                                          ct.c_double, ct.c_ulonglong, ct.c_int, ct.c_int,
                                          ct.POINTER(ct.c_void_p), ct.c_char_p, ct.c_int]),
    "anb_mesh_write_polymesh": (ct.c_int, [ct.c_void_p, ct.c_char_p, ct.c_char_p, ct.c_int]),
    "anb_mesh_free": (None, [ct.c_void_p]),
    "anb_mesh_sizes": (None, [ct.c_void_p, _ip]),
    "anb_mesh_topology": (None, [ct.c_void_p, _dp, _ip, _ip, _ip, _ip, _ip, _ip]),
    "anb_mesh_patch_name": (ct.c_char_p, [ct.c_void_p, ct.c_int]),
    "anb_mesh_geometry": (ct.c_int, [ct.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp, ct.c_char_p, ct.c_int]),
    "anb_bc_evaluate": (ct.c_int, [ct.c_void_p, ct.c_char_p, _ip, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp,
                                    ct.c_char_p, ct.c_int]),
    "anb_expand_case_args": (ct.c_int, [ct.c_int, ct.POINTER(ct.c_char_p), ct.c_char_p, ct.c_int, ct.c_char_p,
                                         ct.c_int]),
    "anb_write_vtu": (ct.c_int, [ct.c_void_p, ct.c_char_p, _dp, _dp, _dp, _dp, _dp, ct.c_char_p, ct.c_int]),
    "anb_write_vtu_binary": (ct.c_int, [ct.c_void_p, ct.c_char_p, _dp, _dp, _dp, _dp, _dp, ct.c_char_p, ct.c_int]),
}


def lib() -> ct.CDLL:
    """Loads libanb.so (raises FileNotFoundError when it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is missing: run `python -m anabasis_b200.build`")
        L = ct.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _i(a):
    return None if a is None else a.ctypes.data_as(_ip)


class AnbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class HostMesh:
    """polyMesh topology + geometry held by libanb.so (anb_hmesh)."""

    def __init__(self, handle: ct.c_void_p):
        self._h = handle
        s = np.zeros(6, np.int32)
        lib().anb_mesh_sizes(self._h, _i(s))
        self.n_points, self.n_faces, self.n_face_points, self.n_internal, self.n_cells, self.n_patches = map(int, s)

    @classmethod
    def read(cls, polymesh_dir: str | os.PathLike) -> "HostMesh":
        h = ct.c_void_p()
        err = ct.create_string_buffer(1024)
        if lib().anb_mesh_read_polymesh(str(polymesh_dir).encode(), ct.byref(h), err, 1024) != 0:
            raise AnbError(ANB_ERR_IO, err.value.decode())
        return cls(h)

    @classmethod
    def channel(cls, nx: int, ny: int, nz: int, lx=2.5, ly=0.41, lz=0.41, jitter=0.0, seed=0, obstacle=False,
                tets=False) -> "HostMesh":
        h = ct.c_void_p()
        err = ct.create_string_buffer(1024)
        if lib().anb_mesh_make_channel(nx, ny, nz, lx, ly, lz, jitter, seed, int(obstacle), int(tets), ct.byref(h),
                                       err, 1024) != 0:
            raise AnbError(ANB_ERR_MESH, err.value.decode())
        return cls(h)

    def write(self, polymesh_dir: str | os.PathLike) -> None:
        err = ct.create_string_buffer(1024)
        if lib().anb_mesh_write_polymesh(self._h, str(polymesh_dir).encode(), err, 1024) != 0:
            raise AnbError(ANB_ERR_IO, err.value.decode())

    def topology(self) -> dict:
        pts = np.zeros(3 * self.n_points)
        fo = np.zeros(self.n_faces + 1, np.int32)
        fp = np.zeros(self.n_face_points, np.int32)
        own = np.zeros(self.n_faces, np.int32)
        nei = np.zeros(max(self.n_internal, 1), np.int32)
        ps = np.zeros(self.n_patches, np.int32)
        pn = np.zeros(self.n_patches, np.int32)
        lib().anb_mesh_topology(self._h, _d(pts), _i(fo), _i(fp), _i(own), _i(nei), _i(ps), _i(pn))
        names = [lib().anb_mesh_patch_name(self._h, k).decode() for k in range(self.n_patches)]
        return dict(points=pts, face_offsets=fo, face_points=fp, owner=own, neighbour=nei[: self.n_internal],
                    patch_start=ps, patch_size=pn, patch_names=names)

    def geometry(self) -> dict:
        C, F = self.n_cells, self.n_faces
        g = dict(cc=np.zeros(3 * C), vol=np.zeros(C), xf=np.zeros(3 * F), nf=np.zeros(3 * F), sf=np.zeros(3 * F),
                 af=np.zeros(F))
        mx = np.zeros(1)
        err = ct.create_string_buffer(1024)
        if lib().anb_mesh_geometry(self._h, _d(g["cc"]), _d(g["vol"]), _d(g["xf"]), _d(g["nf"]), _d(g["sf"]),
                                   _d(g["af"]), _d(mx), err, 1024) != 0:
            raise AnbError(ANB_ERR_MESH, err.value.decode())
        g["max_nonorth"] = float(mx[0])
        return g

    def evaluate_bc(self, bc_path: str | os.PathLike) -> dict:
        P, F = self.n_patches, self.n_faces
        out = {k: np.zeros(P, np.int32) for k in ("type_u", "type_v", "type_w", "type_p")}
        out.update({k: np.zeros(F) for k in ("u", "v", "w", "p")})
        out["patch_table"] = np.zeros(10 * P)
        err = ct.create_string_buffer(2048)
        if lib().anb_bc_evaluate(self._h, str(bc_path).encode(), _i(out["type_u"]), _i(out["type_v"]),
                                 _i(out["type_w"]), _i(out["type_p"]), _d(out["u"]), _d(out["v"]), _d(out["w"]),
                                 _d(out["p"]), _d(out["patch_table"]), err, 2048) != 0:
            raise AnbError(ANB_ERR_INVALID, err.value.decode())
        return out

    def write_vtu(self, filename, u, v, w, p, div_corr=None, binary=False) -> None:
        """ASCII VTU as the reference writes it, or (binary=True) the appended raw-binary VTU."""
        err = ct.create_string_buffer(1024)
        dc = np.zeros(self.n_cells) if div_corr is None else np.ascontiguousarray(div_corr, np.float64)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (u, v, w, p)]
        fn = lib().anb_write_vtu_binary if binary else lib().anb_write_vtu
        if fn(self._h, str(filename).encode(), *map(_d, arrs), _d(dc), err, 1024) != 0:
            raise AnbError(ANB_ERR_IO, err.value.decode())

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            _lib.anb_mesh_free(self._h)
            self._h = None


def default_params(**kw) -> Params:
    p = Params()
    lib().anb_default_params(ct.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Solver:
    """One libanb.so context (anb_ctx) on one GPU."""

    def __init__(self, mesh: HostMesh, params: Params | None = None, **kw):
        self.mesh = mesh
        self.params = params if params is not None else default_params(**kw)
        t = mesh.topology()
        self._keep = t
        md = MeshDesc(mesh.n_points, _d(t["points"]), mesh.n_faces, _i(t["face_offsets"]), _i(t["face_points"]),
                      mesh.n_internal, _i(t["owner"]), _i(t["neighbour"]), mesh.n_patches, _i(t["patch_start"]),
                      _i(t["patch_size"]))
        h = ct.c_void_p()
        rc = lib().anb_create(ct.byref(md), ct.byref(self.params), ct.byref(h))
        if rc != ANB_OK:
            raise AnbError(rc, lib().anb_last_error(None).decode())
        self._h = h
        self.n_cells = mesh.n_cells
        self.n_faces = mesh.n_faces
        self.n_internal = mesh.n_internal

    def _check(self, rc: int, ok=(ANB_OK,)) -> int:
        if rc not in ok:
            raise AnbError(rc, lib().anb_last_error(self._h).decode())
        return rc

    def set_bc(self, bc: dict) -> None:
        self._check(lib().anb_set_bc(self._h, _i(bc["type_u"]), _i(bc["type_v"]), _i(bc["type_w"]),
                                     _i(bc["type_p"]), _d(bc["u"]), _d(bc["v"]), _d(bc["w"]), _d(bc["p"])))

    def set_state(self, u, v, w, p) -> None:
        arrs = [np.ascontiguousarray(a, np.float64) for a in (u, v, w, p)]
        self._check(lib().anb_set_state(self._h, *map(_d, arrs)))

    def get_state(self, with_phi: bool = True, out: dict | None = None) -> dict:
        """Fields in input numbering.  `out` (a dict returned by an earlier call) is filled in place,
        which spares a caller that reads the state every step the allocation and first-touch page
        faults of fresh arrays."""
        C, F = self.n_cells, self.n_faces
        o = out if out is not None else dict(u=np.zeros(C), v=np.zeros(C), w=np.zeros(C), p=np.zeros(C))
        if with_phi and o.get("phi") is None:
            o["phi"] = np.zeros(F)
        elif not with_phi:
            o["phi"] = None
        for k, n in (("u", C), ("v", C), ("w", C), ("p", C)) + ((("phi", F),) if with_phi else ()):
            a = o[k]
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and a.size == n):
                raise ValueError(f"out[{k!r}] must be a contiguous float64 array of {n} values")
        self._check(lib().anb_get_state(self._h, _d(o["u"]), _d(o["v"]), _d(o["w"]), _d(o["p"]), _d(o["phi"])))
        return o

    def scalar_elliptic_solve(self, cell_source, bc_type, bc_value, gamma_face=None, laplacian_nonorth=True,
                              nonorth_corr=2, use_reference_cell=False, reference_cell=0, reference_value=0.0,
                              abs_tol=1e-12, rel_tol=0.0, max_iter=4000) -> tuple[np.ndarray, dict]:
        """anb_scalar_elliptic_solve: face arrays nFaces long (input order), cell arrays nCells."""
        phi = np.zeros(self.n_cells)
        info = SolveInfo()
        g = None if gamma_face is None else np.ascontiguousarray(gamma_face, np.float64)
        src = np.ascontiguousarray(cell_source, np.float64)
        bt = np.ascontiguousarray(bc_type, np.int32)
        bv = np.ascontiguousarray(bc_value, np.float64)
        self._check(lib().anb_scalar_elliptic_solve(self._h, _d(g), _d(src), _i(bt), _d(bv), int(laplacian_nonorth),
                                                    nonorth_corr, int(use_reference_cell), reference_cell,
                                                    reference_value, abs_tol, rel_tol, max_iter, _d(phi),
                                                    ct.byref(info)), ok=(ANB_OK, ANB_NOT_CONVERGED))
        return phi, dict((f, getattr(info, f)) for f, _ in SolveInfo._fields_)

    def scalar_transport_solve(self, gamma_face, su, bc_type, bc_value, face_flux=None, sp=None, upwind=False,
                               diffusion_nonorth=True, nonorth_corr=2, abs_tol=1e-10, rel_tol=0.0, max_iter=4000,
                               x0=None) -> tuple[np.ndarray, dict]:
        """anb_scalar_transport_solve: face arrays nFaces long (input order), cell arrays nCells."""
        phi = np.zeros(self.n_cells)
        info = SolveInfo()
        arr = lambda a, t=np.float64: None if a is None else np.ascontiguousarray(a, t)  # noqa: E731
        g, s_u, s_p, fl, x = arr(gamma_face), arr(su), arr(sp), arr(face_flux), arr(x0)
        bt, bv = arr(bc_type, np.int32), arr(bc_value)
        self._check(lib().anb_scalar_transport_solve(self._h, _d(fl), _d(g), _d(s_u), _d(s_p), _i(bt), _d(bv),
                                                     int(upwind), int(diffusion_nonorth), nonorth_corr, abs_tol,
                                                     rel_tol, max_iter, _d(x), _d(phi), ct.byref(info)),
                    ok=(ANB_OK, ANB_NOT_CONVERGED))
        return phi, dict((f, getattr(info, f)) for f, _ in SolveInfo._fields_)

    # ---- steady sensitivities (include/anb.h) ----
    def set_viscosity(self, mu: float) -> None:
        self._check(lib().anb_set_viscosity(self._h, float(mu)))
        self.params.mu = float(mu)

    def steady_residual(self) -> tuple[np.ndarray, np.ndarray]:
        r = np.zeros(4 * self.n_cells)
        n = np.zeros(2)
        self._check(lib().anb_steady_residual(self._h, _d(r), _d(n)))
        return r, n

    def force_objective(self, patch: int, direction=(1.0, 0.0, 0.0), normal_sign: int = -1) -> tuple[float, float]:
        d = np.ascontiguousarray(direction, np.float64)
        J, jm = ct.c_double(0), ct.c_double(0)
        self._check(lib().anb_force_objective(self._h, patch, normal_sign, _d(d), ct.byref(J), ct.byref(jm)))
        return J.value, jm.value

    def newton_solve(self, max_newton=8, tol=1e-12, lin_max_iter=400) -> dict:
        info = AdjointInfo()
        steps, rn = ct.c_int(0), ct.c_double(0)
        rc = lib().anb_newton_solve(self._h, max_newton, tol, lin_max_iter, ct.byref(steps), ct.byref(rn),
                                    ct.byref(info))
        self._check(rc, ok=(ANB_OK, ANB_NOT_CONVERGED))
        return dict(steps=steps.value, res_norm=rn.value, converged=rc == ANB_OK, iterations=info.iterations,
                    seconds=info.seconds, prec_mom_its=info.prec_mom_its, prec_p_its=info.prec_p_its)

    def tangent_linear(self, patch, direction, dbc, dmu, normal_sign=-1) -> tuple[float, dict]:
        d = np.ascontiguousarray(direction, np.float64)
        b = np.ascontiguousarray(dbc, np.float64)
        info = AdjointInfo()
        dJ = ct.c_double(0)
        self._check(lib().anb_tangent_linear(self._h, patch, normal_sign, _d(d), _d(b), float(dmu), ct.byref(dJ),
                                             ct.byref(info)), ok=(ANB_OK, ANB_NOT_CONVERGED))
        return dJ.value, dict((f, getattr(info, f)) for f, _ in AdjointInfo._fields_)

    def adjoint_force_grad(self, patch, direction=(1.0, 0.0, 0.0), normal_sign=-1) -> tuple[np.ndarray, float, float, dict]:
        d = np.ascontiguousarray(direction, np.float64)
        g = np.zeros(3 * self.n_faces)
        gm, J = ct.c_double(0), ct.c_double(0)
        info = AdjointInfo()
        self._check(lib().anb_adjoint_force_grad(self._h, patch, normal_sign, _d(d), _d(g), ct.byref(gm), ct.byref(J),
                                                 ct.byref(info)), ok=(ANB_OK, ANB_NOT_CONVERGED))
        return g, gm.value, J.value, dict((f, getattr(info, f)) for f, _ in AdjointInfo._fields_)

    def debug_jvp(self, dX, dbc=None, dmu=0.0) -> np.ndarray:
        out = np.zeros(4 * self.n_cells)
        x = np.ascontiguousarray(dX, np.float64)
        b = None if dbc is None else np.ascontiguousarray(dbc, np.float64)
        self._check(lib().anb_debug_jvp(self._h, _d(x), _d(b), float(dmu), _d(out)))
        return out

    def debug_vjp(self, w) -> tuple[np.ndarray, np.ndarray, float]:
        out = np.zeros(4 * self.n_cells)
        g = np.zeros(3 * self.n_faces)
        gm = np.zeros(1)
        self._check(lib().anb_debug_vjp(self._h, _d(np.ascontiguousarray(w, np.float64)), _d(out), _d(g), _d(gm)))
        return out, g, float(gm[0])

    def iterate(self, nsteps: int, tol_mass=-1.0, tol_vel=-1.0) -> tuple[int, list]:
        st = (IterStats * max(nsteps, 1))()
        done = ct.c_int(0)
        rc = lib().anb_simple_iterate(self._h, nsteps, tol_mass, tol_vel, st, ct.byref(done))
        self._check(rc, ok=(ANB_OK, ANB_NOT_CONVERGED, ANB_ERR_DIVERGED))
        stats = [dict((f, getattr(st[i], f)) for f, _ in IterStats._fields_) for i in range(done.value)]
        return rc, stats

    def patch_force(self, patch: int, normal_sign: int = -1) -> dict:
        r = ForceReport()
        self._check(lib().anb_patch_force(self._h, patch, normal_sign, ct.byref(r)))
        return dict(valid=r.valid, n_faces=r.n_faces, area=r.area, Fp=list(r.Fp), Fv=list(r.Fv), F=list(r.F))

    def debug_gradient(self, field: int, phi) -> np.ndarray:
        C = self.n_cells
        g = np.zeros((3, C))
        phi = np.ascontiguousarray(phi, np.float64)
        self._check(lib().anb_debug_gradient(self._h, field, _d(phi), _d(g[0]), _d(g[1]), _d(g[2])))
        return g

    def debug_momentum(self, u, v, w, p) -> dict:
        C, I = self.n_cells, self.n_internal
        o = dict(diag=np.zeros(C), a_pn=np.zeros(I), a_np=np.zeros(I), rhs=np.zeros(3 * C), rau=np.zeros(C))
        arrs = [np.ascontiguousarray(a, np.float64) for a in (u, v, w, p)]
        self._check(lib().anb_debug_momentum(self._h, *map(_d, arrs), _d(o["diag"]), _d(o["a_pn"]), _d(o["a_np"]),
                                             _d(o["rhs"]), _d(o["rau"])))
        return o

    def debug_pressure(self, u, v, w, p, rau) -> dict:
        C, I, F = self.n_cells, self.n_internal, self.n_faces
        o = dict(diag=np.zeros(C), a_pn=np.zeros(I), phi_star=np.zeros(F), div_star=np.zeros(C))
        arrs = [np.ascontiguousarray(a, np.float64) for a in (u, v, w, p, rau)]
        self._check(lib().anb_debug_pressure(self._h, *map(_d, arrs), _d(o["diag"]), _d(o["a_pn"]),
                                             _d(o["phi_star"]), _d(o["div_star"])))
        return o

    def debug_nonorth(self, rau, grad) -> np.ndarray:
        """Divergence of the non-orthogonal correction flux for rAU and grad p' (3 x nCells)."""
        g = np.ascontiguousarray(np.asarray(grad, np.float64).reshape(3, -1))
        rau = np.ascontiguousarray(rau, np.float64)
        div = np.zeros(self.n_cells)
        self._check(lib().anb_debug_nonorth(self._h, _d(rau), _d(g[0]), _d(g[1]), _d(g[2]), _d(div)))
        return div

    def debug_pressure_solve(self, b, x0) -> tuple[np.ndarray, int, float]:
        b = np.ascontiguousarray(b, np.float64)
        x = np.array(x0, np.float64)
        its = ct.c_int(0)
        res = ct.c_double(0)
        self._check(lib().anb_debug_pressure_solve(self._h, _d(b), _d(x), ct.byref(its), ct.byref(res)),
                    ok=(ANB_OK, ANB_NOT_CONVERGED))
        return x, its.value, res.value

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            lib().anb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def expand_case_args(argv: list[str]) -> list[str]:
    """`-case-config` expansion of the front end (raises AnbError with the reference's message)."""
    arr = (ct.c_char_p * len(argv))(*[a.encode() for a in argv])
    out = ct.create_string_buffer(1 << 16)
    err = ct.create_string_buffer(4096)
    n = lib().anb_expand_case_args(len(argv), arr, out, 1 << 16, err, 4096)
    if n < 0:
        raise AnbError(ANB_ERR_INVALID, err.value.decode())
    return [s.decode() for s in out.raw.split(b"\0")[:n]]


def build(force: bool = False) -> Path:
    from .build import build as _build
    return _build(force=force)
