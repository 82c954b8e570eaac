"""CPU oracle of the SIMPLE outer iteration (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline/reference legs may import this
package.  It wraps liboracle.so (oracle.cpp, a restatement of the reference's
apps/generic_simple_v1/src/main.cu with file:line citations) and, when built, the reference's
own host code compiled from the reference tree into oracle/_ref/ (see build.py).
"""
from __future__ import annotations

import ctypes as ct
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_dp = ct.POINTER(ct.c_double)
_ip = ct.POINTER(ct.c_int)
_lib = None


class OrcParams(ct.Structure):
    _fields_ = [("rho", ct.c_double), ("mu", ct.c_double), ("u_relax", ct.c_double), ("p_relax", ct.c_double),
                ("n_nonorth_corr", ct.c_int), ("n_vel_nonorth_corr", ct.c_int), ("n_pressure_corr", ct.c_int),
                ("vel_maxit", ct.c_int), ("vel_tol", ct.c_double), ("vel_rel_tol", ct.c_double),
                ("p_maxit", ct.c_int), ("p_tol", ct.c_double), ("p_rel_tol", ct.c_double),
                ("corr_tol", ct.c_double), ("tol_mass", ct.c_double), ("tol_vel", ct.c_double),
                ("n_threads", ct.c_int), ("p_use_amg", ct.c_int)]


class OrcStats(ct.Structure):
    _fields_ = [("mass_res", ct.c_double), ("du", ct.c_double), ("dv", ct.c_double), ("dw", ct.c_double),
                ("dp", ct.c_double), ("its_u", ct.c_int), ("its_v", ct.c_int), ("its_w", ct.c_int),
                ("its_p_last", ct.c_int), ("its_p_total", ct.c_int)]


def lib() -> ct.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            from .build import build_oracle
            build_oracle()
        L = ct.CDLL(str(LIB))
        L.orc_mesh_create.restype = ct.c_void_p
        L.orc_mesh_create.argtypes = [ct.c_int, _dp, ct.c_int, _ip, _ip, ct.c_int, _ip, _ip, ct.c_int, _ip, _ip,
                                      ct.c_char_p, ct.c_int]
        L.orc_mesh_free.argtypes = [ct.c_void_p]
        L.orc_mesh_ncells.restype = ct.c_int
        L.orc_mesh_ncells.argtypes = [ct.c_void_p]
        L.orc_mesh_sizes.argtypes = [ct.c_void_p, _ip]
        L.orc_mesh_patches.argtypes = [ct.c_void_p, _ip, _ip]
        L.orc_mesh_topology.argtypes = [ct.c_void_p, _dp, _ip, _ip, _ip, _ip]
        L.orc_channel_create.restype = ct.c_void_p
        L.orc_channel_create.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_double, ct.c_double, ct.c_double,
                                         ct.c_double, ct.c_ulonglong, ct.c_int, _dp, ct.c_char_p, ct.c_int]
        L.orc_eval_bc.restype = ct.c_int
        L.orc_eval_bc.argtypes = [ct.c_void_p, _ip, _dp, _ip, _dp] + [_ip] * 4 + [_dp] * 4 + [ct.c_char_p, ct.c_int]
        L.orc_mesh_geometry.argtypes = [ct.c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_set_bc.argtypes = [ct.c_void_p, _ip, _ip, _ip, _ip, _dp, _dp, _dp, _dp]
        L.orc_lsq_gradient.argtypes = [ct.c_void_p, ct.c_int, _dp, _dp, _dp, _dp]
        L.orc_momentum.argtypes = [ct.c_void_p, ct.c_double, ct.c_double, ct.c_double, _dp, _dp, _dp, _dp, _dp, _dp,
                                   _dp, _dp, _dp]
        L.orc_pressure.argtypes = [ct.c_void_p, ct.c_double, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_nonorth.argtypes = [ct.c_void_p, _dp, _dp, _dp, _dp]
        L.orc_flux_correct.argtypes = [ct.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.orc_simple_run.restype = ct.c_int
        L.orc_simple_run.argtypes = [ct.c_void_p, ct.POINTER(OrcParams), ct.c_int, _dp, _dp, _dp, _dp, _dp,
                                     ct.POINTER(OrcStats)]
        L.orc_patch_force.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_double, _dp, _dp, _dp, _dp, _dp]
        L.orc_scalar_gradient.argtypes = [ct.c_void_p, _ip, _dp, _dp, _dp, _dp, _dp]
        L.orc_scalar_assemble.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, _dp, _dp, _dp, _dp, _ip, _dp,
                                          _dp, ct.c_int, ct.c_double, _dp, _dp, _dp, _dp]
        _lib = L
    return _lib


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _i(a):
    return None if a is None else a.ctypes.data_as(_ip)


class Oracle:
    """Oracle mesh + boundary conditions; topology dict as returned by HostMesh.topology()."""

    def __init__(self, topo: dict | None = None, _handle=None):
        if _handle is None:
            nf = len(topo["face_offsets"]) - 1
            err = ct.create_string_buffer(1024)
            h = lib().orc_mesh_create(len(topo["points"]) // 3, _d(topo["points"]), nf, _i(topo["face_offsets"]),
                                      _i(topo["face_points"]), len(topo["neighbour"]), _i(topo["owner"]),
                                      _i(topo["neighbour"]), len(topo["patch_start"]), _i(topo["patch_start"]),
                                      _i(topo["patch_size"]), err, 1024)
            if not h:
                raise RuntimeError(err.value.decode())
            _handle = h
        self._h = ct.c_void_p(_handle)
        s = np.zeros(6, np.int32)
        lib().orc_mesh_sizes(self._h, _i(s))
        self.n_points, self.n_faces, self.n_internal, self.n_cells, self.n_patches, self._nfp = map(int, s)
        self.t = topo

    @classmethod
    def channel(cls, nx, ny, nz, lx=2.5, ly=0.41, lz=0.41, jitter=0.0, seed=0, obstacle=False) -> "Oracle":
        """The synthetic channel mesh built by the oracle itself (channel.cpp), hexes only."""
        err = ct.create_string_buffer(1024)
        h = lib().orc_channel_create(nx, ny, nz, lx, ly, lz, jitter, seed, int(obstacle), None, err, 1024)
        if not h:
            raise RuntimeError(err.value.decode())
        return cls(_handle=h)

    def topology(self) -> dict:
        t = dict(points=np.zeros(3 * self.n_points), face_offsets=np.zeros(self.n_faces + 1, np.int32),
                 face_points=np.zeros(self._nfp, np.int32), owner=np.zeros(self.n_faces, np.int32),
                 neighbour=np.zeros(self.n_internal, np.int32), patch_start=np.zeros(self.n_patches, np.int32),
                 patch_size=np.zeros(self.n_patches, np.int32))
        lib().orc_mesh_topology(self._h, _d(t["points"]), _i(t["face_offsets"]), _i(t["face_points"]),
                                _i(t["owner"]), _i(t["neighbour"]))
        lib().orc_mesh_patches(self._h, _i(t["patch_start"]), _i(t["patch_size"]))
        return t

    def eval_bc(self, velocity: list, pressure: list) -> dict:
        """Boundary values per patch (orc_eval_bc): velocity[k] = (ORC_VEL_* kind, params...),
        pressure[k] = (ORC_P_* kind, value).  Returns the dict that set_bc takes."""
        P, F = self.n_patches, self.n_faces
        vk = np.array([v[0] for v in velocity], np.int32)
        vp = np.zeros((P, 4))
        for k, v in enumerate(velocity):
            vp[k, :len(v) - 1] = v[1:]
        pk = np.array([p[0] for p in pressure], np.int32)
        pv = np.array([p[1] if len(p) > 1 else 0.0 for p in pressure], np.float64)
        bc = {f"type_{q}": np.zeros(P, np.int32) for q in "uvwp"}
        bc.update({q: np.zeros(F) for q in "uvwp"})
        err = ct.create_string_buffer(1024)
        vp = np.ascontiguousarray(vp.reshape(-1))
        rc = lib().orc_eval_bc(self._h, _i(vk), _d(vp), _i(pk), _d(pv), _i(bc["type_u"]), _i(bc["type_v"]),
                               _i(bc["type_w"]), _i(bc["type_p"]), _d(bc["u"]), _d(bc["v"]), _d(bc["w"]),
                               _d(bc["p"]), err, 1024)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return bc

    def geometry(self) -> dict:
        C, F = self.n_cells, self.n_faces
        g = dict(cc=np.zeros(3 * C), vol=np.zeros(C), xf=np.zeros(3 * F), nf=np.zeros(3 * F), sf=np.zeros(3 * F),
                 af=np.zeros(F))
        mx = np.zeros(1)
        lib().orc_mesh_geometry(self._h, _d(g["cc"]), _d(g["vol"]), _d(g["xf"]), _d(g["nf"]), _d(g["sf"]),
                                _d(g["af"]), _d(mx))
        g["max_nonorth"] = float(mx[0])
        return g

    def set_bc(self, bc: dict) -> None:
        self._bc = bc
        lib().orc_set_bc(self._h, _i(bc["type_u"]), _i(bc["type_v"]), _i(bc["type_w"]), _i(bc["type_p"]),
                         _d(bc["u"]), _d(bc["v"]), _d(bc["w"]), _d(bc["p"]))

    def gradient(self, field: int, phi) -> np.ndarray:
        g = np.zeros((3, self.n_cells))
        phi = np.ascontiguousarray(phi, np.float64)
        lib().orc_lsq_gradient(self._h, field, _d(phi), _d(g[0]), _d(g[1]), _d(g[2]))
        return g

    def momentum(self, rho, mu, u_relax, u, v, w, p) -> dict:
        C, I = self.n_cells, self.n_internal
        o = dict(diag=np.zeros(C), a_pn=np.zeros(I), a_np=np.zeros(I), rhs=np.zeros(3 * C), rau=np.zeros(C))
        arrs = [np.ascontiguousarray(a, np.float64) for a in (u, v, w, p)]
        lib().orc_momentum(self._h, rho, mu, u_relax, *map(_d, arrs), _d(o["diag"]), _d(o["a_pn"]), _d(o["a_np"]),
                           _d(o["rhs"]), _d(o["rau"]))
        return o

    def pressure(self, rho, u, v, w, p, rau) -> dict:
        C, I, F = self.n_cells, self.n_internal, self.n_faces
        o = dict(diag=np.zeros(C), a_pn=np.zeros(I), phi_star=np.zeros(F), div_star=np.zeros(C))
        arrs = [np.ascontiguousarray(a, np.float64) for a in (u, v, w, p, rau)]
        lib().orc_pressure(self._h, rho, *map(_d, arrs), _d(o["diag"]), _d(o["a_pn"]), _d(o["phi_star"]),
                           _d(o["div_star"]))
        return o

    def nonorth(self, rau, grad) -> tuple[np.ndarray, np.ndarray]:
        phi = np.zeros(self.n_faces)
        div = np.zeros(self.n_cells)
        g = np.ascontiguousarray(np.asarray(grad, np.float64).reshape(-1))
        lib().orc_nonorth(self._h, _d(np.ascontiguousarray(rau, np.float64)), _d(g), _d(phi), _d(div))
        return phi, div

    def flux_correct(self, rau, phi_star, pcorr, grad) -> np.ndarray:
        out = np.zeros(self.n_faces)
        g = np.ascontiguousarray(np.asarray(grad, np.float64).reshape(-1))
        a = [np.ascontiguousarray(x, np.float64) for x in (rau, phi_star, pcorr)]
        lib().orc_flux_correct(self._h, *map(_d, a), _d(g), _d(out))
        return out

    def run(self, params: OrcParams, nsteps: int, u, v, w, p) -> tuple[dict, list]:
        st = (OrcStats * max(nsteps, 1))()
        s = dict(u=np.array(u, np.float64), v=np.array(v, np.float64), w=np.array(w, np.float64),
                 p=np.array(p, np.float64), phi=np.zeros(self.n_faces))
        done = lib().orc_simple_run(self._h, ct.byref(params), nsteps, _d(s["u"]), _d(s["v"]), _d(s["w"]),
                                    _d(s["p"]), _d(s["phi"]), st)
        stats = [dict((f, getattr(st[i], f)) for f, _ in OrcStats._fields_) for i in range(done)]
        return s, stats

    def patch_force(self, patch, sign, mu, u, v, w, p) -> np.ndarray:
        o = np.zeros(11)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (u, v, w, p)]
        lib().orc_patch_force(self._h, patch, sign, mu, *map(_d, arrs), _d(o))
        return o

    def scalar_gradient(self, bc_type, bc_value, phi) -> np.ndarray:
        """libpoisson/libscalar LSQ gradient (3 x nCells)."""
        g = np.zeros((3, self.n_cells))
        bt = np.ascontiguousarray(bc_type, np.int32)
        bv = np.ascontiguousarray(bc_value, np.float64)
        ph = np.ascontiguousarray(phi, np.float64)
        lib().orc_scalar_gradient(self._h, _i(bt), _d(bv), _d(ph), _d(g[0]), _d(g[1]), _d(g[2]))
        return g

    def scalar_assemble(self, transport, upwind, nonorth, gamma, src, bc_type, bc_value, grad, flux=None, sp=None,
                        ref_cell=-1, ref_value=0.0) -> dict:
        """Elliptic (transport=False) or transport system in face-coefficient form."""
        C, I = self.n_cells, self.n_internal
        o = dict(diag=np.zeros(C), a_pn=np.zeros(I), a_np=np.zeros(I), rhs=np.zeros(C))
        f64 = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)  # noqa: E731
        gm, fl, sr, spp, bv = f64(gamma), f64(flux), f64(src), f64(sp), f64(bc_value)
        g = np.ascontiguousarray(np.asarray(grad, np.float64).reshape(-1))
        bt = np.ascontiguousarray(bc_type, np.int32)
        lib().orc_scalar_assemble(self._h, int(transport), int(upwind), int(nonorth), _d(gm), _d(fl), _d(sr), _d(spp),
                                  _i(bt), _d(bv), _d(g), int(ref_cell), float(ref_value), _d(o["diag"]),
                                  _d(o["a_pn"]), _d(o["a_np"]), _d(o["rhs"]))
        return o

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            _lib.orc_mesh_free(self._h)
            self._h = None


VEL_WALL_NOSLIP, VEL_ZERO_GRADIENT, VEL_UNIFORM, VEL_PARABOLIC_BOX = 0, 1, 2, 3
P_ZERO_GRADIENT, P_FIXED_VALUE = 0, 1


def channel_case(nx, ny, nz, jitter=0.0, seed=0, obstacle=False, pout=0.0):
    """The benchmark channel case built without the product library: the oracle's mesh, the
    boundary values of the channel boundary file (patch_0_0 wall_noslip / zero_gradient p,
    patch_1_0 parabolic_box_inlet 0.41 0.45 y z average_patch_normal / zero_gradient p, patch_2_0
    zero_gradient / fixed_value pout, patch_3_0 wall_noslip / zero_gradient p) and the initial state
    of main.cu:3302-3322 (mean inlet velocity everywhere, p = 0).  Returns (oracle, bc, state)."""
    o = Oracle.channel(nx, ny, nz, jitter=jitter, seed=seed, obstacle=obstacle)
    vel = [(VEL_WALL_NOSLIP,), (VEL_PARABOLIC_BOX, 0.41, 0.45, 1, 2), (VEL_ZERO_GRADIENT,)]
    pre = [(P_ZERO_GRADIENT,), (P_ZERO_GRADIENT,), (P_FIXED_VALUE, pout)]
    if obstacle:
        vel.append((VEL_WALL_NOSLIP,))
        pre.append((P_ZERO_GRADIENT,))
    bc = o.eval_bc(vel, pre)
    o.set_bc(bc)
    t = o.topology()
    sl = slice(int(t["patch_start"][1]), int(t["patch_start"][1] + t["patch_size"][1]))
    C = o.n_cells
    state = (np.full(C, bc["u"][sl].mean()), np.full(C, bc["v"][sl].mean()), np.full(C, bc["w"][sl].mean()),
             np.zeros(C))
    return o, bc, state


def params(**kw) -> OrcParams:
    """Oracle controls with the reference defaults (main.cu:73-103)."""
    p = OrcParams(rho=1.0, mu=0.05, u_relax=0.7, p_relax=1.0, n_nonorth_corr=2, n_vel_nonorth_corr=0,
                  n_pressure_corr=0, vel_maxit=100, vel_tol=1e-10, vel_rel_tol=0.0, p_maxit=4000, p_tol=1e-10,
                  p_rel_tol=0.0, corr_tol=1e-12, tol_mass=1e-10, tol_vel=1e-10, n_threads=0, p_use_amg=0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p
