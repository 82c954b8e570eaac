"""ctypes access to the reference's own host code (oracle/_ref/libgsv1ref.so, built by
oracle/build_ref.sh from the reference tree).  Test infrastructure only."""
from __future__ import annotations

import ctypes as ct
from pathlib import Path

import numpy as np

LIB = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libgsv1ref.so"
_dp = ct.POINTER(ct.c_double)
_ip = ct.POINTER(ct.c_int)
_lib = None


def available() -> bool:
    return LIB.exists()


def lib() -> ct.CDLL:
    global _lib
    if _lib is None:
        L = ct.CDLL(str(LIB))
        L.ref_read_mesh.restype = ct.c_void_p
        L.ref_read_mesh.argtypes = [ct.c_char_p, ct.c_char_p, ct.c_int]
        L.ref_free_mesh.argtypes = [ct.c_void_p]
        L.ref_mesh_sizes.argtypes = [ct.c_void_p, _ip]
        L.ref_mesh_geometry.argtypes = [ct.c_void_p] + [_dp] * 7
        L.ref_lsq_gradient.argtypes = [ct.c_void_p, _ip, _dp, _dp, _dp]
        L.ref_rhie_chow.argtypes = [ct.c_void_p] + [_dp] * 6 + [_ip, _dp] * 3 + [ct.c_double, _dp]
        L.ref_continuity.argtypes = [ct.c_void_p, _dp, _dp]
        L.ref_nonorth.argtypes = [ct.c_void_p, _dp, _ip, _dp, _dp, _dp]
        L.ref_flux_correct.argtypes = [ct.c_void_p, _dp, _ip, _dp, _dp, _dp, _dp, _dp]
        L.ref_patch_force.argtypes = [ct.c_void_p, ct.c_int] + [_dp] * 4 + [ct.c_double, ct.c_double, ct.c_int, _dp]
        L.ref_write_vtu.restype = ct.c_int
        L.ref_write_vtu.argtypes = [ct.c_void_p, ct.c_char_p] + [_dp] * 4
        L.ref_expand_case.restype = ct.c_int
        L.ref_expand_case.argtypes = [ct.c_int, ct.POINTER(ct.c_char_p), ct.c_char_p, ct.c_int, ct.c_char_p, ct.c_int]
        L.ref_bc_eval.restype = ct.c_int
        L.ref_bc_eval.argtypes = [ct.c_void_p, ct.c_char_p] + [_ip] * 4 + [_dp] * 4 + [ct.c_char_p, ct.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class RefMesh:
    def __init__(self, polymesh_dir):
        err = ct.create_string_buffer(1024)
        h = lib().ref_read_mesh(str(polymesh_dir).encode(), err, 1024)
        if not h:
            raise RuntimeError(err.value.decode())
        self._h = ct.c_void_p(h)
        s = np.zeros(5, np.int32)
        lib().ref_mesh_sizes(self._h, _i(s))
        self.n_points, self.n_faces, self.n_internal, self.n_cells, self.n_patches = map(int, s)

    def geometry(self) -> dict:
        C, F = self.n_cells, self.n_faces
        g = dict(cc=np.zeros(3 * C), vol=np.zeros(C), xf=np.zeros(3 * F), nf=np.zeros(3 * F), sf=np.zeros(3 * F),
                 af=np.zeros(F))
        mx = np.zeros(1)
        lib().ref_mesh_geometry(self._h, _d(g["cc"]), _d(g["vol"]), _d(g["xf"]), _d(g["nf"]), _d(g["sf"]),
                                _d(g["af"]), _d(mx))
        g["max_nonorth"] = float(mx[0])
        return g

    def gradient(self, types, face_vals, phi) -> np.ndarray:
        g = np.zeros(3 * self.n_cells)
        lib().ref_lsq_gradient(self._h, _i(np.ascontiguousarray(types, np.int32)),
                               _d(np.ascontiguousarray(face_vals, np.float64)),
                               _d(np.ascontiguousarray(phi, np.float64)), _d(g))
        return g.reshape(-1, 3).T

    def rhie_chow(self, u, v, w, p, gradp, rau, bc, rho) -> np.ndarray:
        out = np.zeros(self.n_faces)
        ga = np.ascontiguousarray(np.asarray(gradp).T.reshape(-1))
        a = [np.ascontiguousarray(x, np.float64) for x in (u, v, w, p, ga, rau)]
        lib().ref_rhie_chow(self._h, *map(_d, a), _i(bc["type_u"]), _d(bc["u"]), _i(bc["type_v"]), _d(bc["v"]),
                            _i(bc["type_w"]), _d(bc["w"]), rho, _d(out))
        return out

    def continuity(self, phi) -> np.ndarray:
        out = np.zeros(self.n_cells)
        lib().ref_continuity(self._h, _d(np.ascontiguousarray(phi, np.float64)), _d(out))
        return out

    def nonorth(self, rau, types_p, grad) -> tuple[np.ndarray, np.ndarray]:
        phi = np.zeros(self.n_faces)
        div = np.zeros(self.n_cells)
        ga = np.ascontiguousarray(np.asarray(grad).T.reshape(-1))
        lib().ref_nonorth(self._h, _d(np.ascontiguousarray(rau, np.float64)), _i(types_p), _d(ga), _d(phi), _d(div))
        return phi, div

    def flux_correct(self, rau, types_p, p_face, phi_star, pcorr, grad) -> np.ndarray:
        out = np.zeros(self.n_faces)
        ga = np.ascontiguousarray(np.asarray(grad).T.reshape(-1))
        a = [np.ascontiguousarray(x, np.float64) for x in (rau,)]
        lib().ref_flux_correct(self._h, _d(a[0]), _i(types_p), _d(p_face), _d(np.ascontiguousarray(phi_star)),
                               _d(np.ascontiguousarray(pcorr, np.float64)), _d(ga), _d(out))
        return out

    def patch_force(self, patch, u, v, w, p, rho, mu, sign) -> np.ndarray:
        out = np.zeros(11)
        a = [np.ascontiguousarray(x, np.float64) for x in (u, v, w, p)]
        lib().ref_patch_force(self._h, patch, *map(_d, a), rho, mu, sign, _d(out))
        return out

    def write_vtu(self, fn, u, v, w, p) -> None:
        a = [np.ascontiguousarray(x, np.float64) for x in (u, v, w, p)]
        assert lib().ref_write_vtu(self._h, str(fn).encode(), *map(_d, a)) == 0

    def bc_eval(self, path) -> dict:
        P, F = self.n_patches, self.n_faces
        out = {k: np.zeros(P, np.int32) for k in ("type_u", "type_v", "type_w", "type_p")}
        out.update({k: np.zeros(F) for k in ("u", "v", "w", "p")})
        err = ct.create_string_buffer(2048)
        rc = lib().ref_bc_eval(self._h, str(path).encode(), _i(out["type_u"]), _i(out["type_v"]), _i(out["type_w"]),
                               _i(out["type_p"]), _d(out["u"]), _d(out["v"]), _d(out["w"]), _d(out["p"]), err, 2048)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return out

    def __del__(self):
        if getattr(self, "_h", None) is not None and _lib is not None:
            _lib.ref_free_mesh(self._h)


def expand_case(argv: list[str]) -> list[str]:
    """Reference expand_case_config_args; raises RuntimeError with its message."""
    arr = (ct.c_char_p * len(argv))(*[a.encode() for a in argv])
    out = ct.create_string_buffer(1 << 16)
    err = ct.create_string_buffer(4096)
    n = lib().ref_expand_case(len(argv), arr, out, 1 << 16, err, 4096)
    if n < 0:
        raise RuntimeError(err.value.decode())
    return out.raw.split(b"\0")[:n] and [s.decode() for s in out.raw.split(b"\0")[:n]]


# ---- the reference's scalar libraries (oracle/_ref/libscalarref.so) ---------------------------
SCALAR_LIB = LIB.parent / "libscalarref.so"
_slib = None


def scalar_available() -> bool:
    return SCALAR_LIB.exists()


def slib() -> ct.CDLL:
    global _slib
    if _slib is None:
        L = ct.CDLL(str(SCALAR_LIB))
        L.rsm_open.restype = ct.c_void_p
        L.rsm_open.argtypes = [ct.c_char_p, ct.c_char_p, ct.c_int]
        L.rsm_close.argtypes = [ct.c_void_p]
        L.rsm_sizes.argtypes = [ct.c_void_p, _ip]
        L.rsm_geometry.argtypes = [ct.c_void_p, _dp, _dp]
        L.rsm_pattern.argtypes = [ct.c_void_p, _ip, _ip]
        L.rst_pattern.argtypes = [ct.c_void_p, _ip, _ip]
        L.rsm_poisson_gradient.argtypes = [ct.c_void_p, _ip, _dp, _dp, _dp]
        L.rsm_poisson_assemble.restype = ct.c_int
        L.rsm_poisson_assemble.argtypes = [ct.c_void_p, _dp, _dp, _ip, _dp, _dp, ct.c_int, ct.c_int, ct.c_int,
                                           ct.c_double, _dp, _dp, ct.c_char_p, ct.c_int]
        L.rst_gradient.argtypes = [ct.c_void_p, _ip, _dp, _dp, _dp]
        L.rst_assemble.restype = ct.c_int
        L.rst_assemble.argtypes = [ct.c_void_p, _dp, _dp, _dp, _dp, _ip, _dp, _dp, ct.c_int, ct.c_int, _dp, _dp,
                                   ct.c_char_p, ct.c_int]
        _slib = L
    return _slib


class RefScalar:
    """libpoisson / libscalar host functions on a polyMesh read by libpoisson's reader; same
    gradient/system interface as oracle.mms.OracleAssembler."""

    def __init__(self, polymesh_dir):
        err = ct.create_string_buffer(1024)
        h = slib().rsm_open(str(polymesh_dir).encode(), err, 1024)
        if not h:
            raise RuntimeError(err.value.decode())
        self._h = ct.c_void_p(h)
        s = np.zeros(4, np.int32)
        slib().rsm_sizes(self._h, _i(s))
        self.n, self.n_faces, self.n_internal, self.nnz = map(int, s)
        self.row_off = np.zeros(self.n + 1, np.int32)
        self.cols = np.zeros(self.nnz, np.int32)
        slib().rsm_pattern(self._h, _i(self.row_off), _i(self.cols))
        self.cc = np.zeros(3 * self.n)
        self.vol = np.zeros(self.n)
        slib().rsm_geometry(self._h, _d(self.cc), _d(self.vol))

    def transport_pattern(self):
        ro = np.zeros(self.n + 1, np.int32)
        co = np.zeros(self.nnz, np.int32)
        slib().rst_pattern(self._h, _i(ro), _i(co))
        return ro, co

    def gradient(self, transport, bt, bv, phi):
        g = np.zeros(3 * self.n)
        bt = np.ascontiguousarray(bt, np.int32)
        bv = np.ascontiguousarray(bv, np.float64)
        ph = np.ascontiguousarray(phi, np.float64)
        fn = slib().rst_gradient if transport else slib().rsm_poisson_gradient
        fn(self._h, _i(bt), _d(bv), _d(ph), _d(g))
        return g.reshape(3, self.n)

    def system(self, transport, upwind, nonorth, gamma, src, sp, flux, bt, bv, grad, ref_cell, ref_value):
        import scipy.sparse as sps

        vals = np.zeros(self.nnz)
        rhs = np.zeros(self.n)
        err = ct.create_string_buffer(1024)
        f64 = lambda a, n: np.zeros(n) if a is None else np.ascontiguousarray(a, np.float64)  # noqa: E731
        g = np.ascontiguousarray(np.asarray(grad, np.float64).reshape(-1))
        bt = np.ascontiguousarray(bt, np.int32)
        bv = np.ascontiguousarray(bv, np.float64)
        gm = f64(gamma, self.n_faces)
        if transport:
            rc = slib().rst_assemble(self._h, _d(f64(flux, self.n_faces)), _d(gm), _d(f64(src, self.n)),
                                     _d(f64(sp, self.n)), _i(bt), _d(bv), _d(g), int(upwind), int(nonorth),
                                     _d(vals), _d(rhs), err, 1024)
        else:
            rc = slib().rsm_poisson_assemble(self._h, _d(gm), _d(f64(src, self.n)), _i(bt), _d(bv), _d(g),
                                             int(nonorth), int(ref_cell >= 0), max(ref_cell, 0), float(ref_value),
                                             _d(vals), _d(rhs), err, 1024)
        if rc:
            raise RuntimeError(err.value.decode())
        return sps.csr_matrix((vals, self.cols, self.row_off), shape=(self.n, self.n)), rhs

    def __del__(self):
        if getattr(self, "_h", None) is not None and _slib is not None:
            _slib.rsm_close(self._h)
            self._h = None
