"""ctypes bindings to the parity checkers.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()``
and by the cpu_baseline leg of ``bench.py``; the product (``wasl_b200``) never
imports this module.

* ``Oracle`` wraps ``oracle/liboracle.so``: the C restatement of the reference
  hot path (``wasl_oracle.c``).
* ``Reference`` wraps ``oracle/_ref/libwaslref.so``: the reference's own C++
  numerical core compiled from its sources, through ``ref_shim.cpp``.  It is
  optional: ``Reference.available()`` is False where it was not built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libwaslref.so")

_d = C.POINTER(C.c_double)
_i32 = C.POINTER(C.c_int32)
_i64 = C.POINTER(C.c_int64)
_u8 = C.POINTER(C.c_uint8)


def build(reference_root: str | None = None) -> None:
    """Compile liboracle.so, and the reference checker when the reference
    checkout is given (argument or REF environment variable) and present."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    root = reference_root or os.environ.get("REF")
    if root and os.path.isdir(os.path.join(root, "cpp", "src")):
        subprocess.check_call(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={root}"])
        if os.path.exists(os.path.join(os.path.dirname(HERE), "wasl_b200", "libwasl_b200.so")):
            subprocess.check_call(["make", "-s", "-C", HERE, "gpu-case", f"REF={root}"])


def _p(a, t=_d):
    return a.ctypes.data_as(t)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class WoTriMesh(C.Structure):
    _fields_ = [
        ("element_count", C.c_int64), ("face_count", C.c_int64),
        ("vertices", _d), ("nodes", _i64),
        ("face_left", _i32), ("face_right", _i32),
        ("face_left_edge", _i32), ("face_right_edge", _i32),
        ("face_left_v0", _i64), ("face_right_v0", _i64),
        ("face_normal_x", _d), ("face_normal_y", _d),
    ]


class WoLineMesh(C.Structure):
    _fields_ = [
        ("element_count", C.c_int64), ("face_count", C.c_int64),
        ("x_left", _d), ("x_right", _d),
        ("face_left", _i32), ("face_right", _i32),
        ("face_x", _d), ("face_normal", _d),
    ]


class WoStencil(C.Structure):
    _fields_ = [
        ("element_count", C.c_int64), ("mode_count", C.c_int),
        ("polynomial_order", C.c_int), ("maximum_neighbors", C.c_int),
        ("highest_degree_begin", C.c_int), ("check_point_count", C.c_int),
        ("neighbors", _i32), ("transforms", _d),
        ("normal_x", _d), ("normal_y", _d), ("check_basis", _d),
    ]


class WoEulerTriSetup(C.Structure):
    _fields_ = [
        ("boundary_kind", C.c_int), ("donors", _i32), ("donor_basis", _d),
        ("stencil", C.POINTER(WoStencil)),
        ("threshold", C.c_double), ("density_floor", C.c_double),
        ("pressure_floor", C.c_double),
    ]


def tri_modes(p):
    return (p + 1) * (p + 2) // 2


class Oracle:
    """The C restatement of the reference algorithms (liboracle.so)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        self.lib = L = C.CDLL(path)
        L.wo_tri_mesh_build.argtypes = [C.c_int64, _i64, _d, C.c_int64, _i64, C.POINTER(WoTriMesh)]
        L.wo_tri_mesh_free.argtypes = [C.POINTER(WoTriMesh)]
        L.wo_line_mesh_build.argtypes = [C.c_int64, _i64, _d, C.c_int64, _i64, C.POINTER(WoLineMesh)]
        L.wo_line_mesh_free.argtypes = [C.POINTER(WoLineMesh)]
        L.wo_dubiner_basis.argtypes = [C.c_double, C.c_double, C.c_int, _d]
        L.wo_dubiner_basis_gradient.argtypes = [C.c_double, C.c_double, C.c_int, _d, _d]
        L.wo_legendre_basis.argtypes = [C.c_double, C.c_int, _d]
        L.wo_legendre_basis_gradient.argtypes = [C.c_double, C.c_int, _d]
        L.wo_gauss_legendre.argtypes = [C.c_int, _d, _d]
        L.wo_tri_volume_rule.argtypes = [C.c_int, _d, _d, _d]
        L.wo_tri_edge_rules.argtypes = [C.c_int, _d, _d, _d, _d, _d]
        L.wo_hllc_flux.argtypes = [C.c_double, _d, _d, C.c_double, C.c_double, _d]
        tm = C.POINTER(WoTriMesh)
        lm = C.POINTER(WoLineMesh)
        L.wo_euler_tri_residual.argtypes = [tm, C.c_double, C.c_int, _d, _d, _d]
        L.wo_euler_line_residual.argtypes = [lm, C.c_double, C.c_int, _d, _d, _d]
        L.wo_scalar_line_residual.argtypes = [lm, C.c_double, C.c_int, _d, _d, _d]
        L.wo_scalar_tri_residual.argtypes = [tm, C.c_double, C.c_double, C.c_int, _d, _d, _d]
        L.wo_periodic_tri_trace.argtypes = [tm, C.c_int, _i32, _d]
        L.wo_periodic_tri_euler_exterior.argtypes = [tm, C.c_int, _i32, _d, _d, _d]
        L.wo_periodic_tri_scalar_exterior.argtypes = [tm, C.c_int, _i32, _d, _d, _d]
        L.wo_transmissive_tri_euler_exterior.argtypes = [tm, C.c_int, _d, _d]
        L.wo_line_euler_exterior.argtypes = [lm, C.c_int, C.c_int, C.c_int, _d, _d]
        L.wo_line_scalar_exterior.argtypes = [lm, C.c_int, C.c_int, C.c_double, C.c_int,
                                              C.c_double, _d, _d]
        st = C.POINTER(WoStencil)
        L.wo_tri_stencil.argtypes = [tm, C.c_int, _i32, C.c_int, st]
        L.wo_line_stencil.argtypes = [lm, C.c_int, C.c_int, st]
        L.wo_stencil_free.argtypes = [st]
        L.wo_limit_euler.argtypes = [st, C.c_double, C.c_double, C.c_double, C.c_double, _d, _u8,
                                     _i64]
        L.wo_troubled_flags.argtypes = [st, C.c_double, _d, _u8]
        L.wo_positivity.argtypes = [C.c_double, _d, C.c_int, _d, C.c_int, C.c_double, C.c_double,
                                    _d]
        L.wo_characteristic_weno.argtypes = [C.c_double, _d, C.c_double, C.c_double, _d, _d,
                                             C.c_int, C.c_int, _d]
        L.wo_euler_tri_cfl.argtypes = [tm, C.c_double, _d, C.c_int, C.c_double, _d]
        L.wo_euler_line_cfl.argtypes = [lm, C.c_double, _d, C.c_int, C.c_double, _d]
        L.wo_tri_minimum_altitude.argtypes = [tm]
        L.wo_tri_minimum_altitude.restype = C.c_double
        L.wo_line_advection_cfl.argtypes = [lm, C.c_double, C.c_int, C.c_double]
        L.wo_line_advection_cfl.restype = C.c_double
        L.wo_tri_scalar_cfl.argtypes = [tm, C.c_double, C.c_double, C.c_int, C.c_double]
        L.wo_tri_scalar_cfl.restype = C.c_double
        L.wo_euler_tri_step.argtypes = [tm, C.POINTER(WoEulerTriSetup), C.c_double, C.c_int,
                                        C.c_double, _d, _u8]
        L.wo_euler_line_step.argtypes = [lm, C.c_int, C.c_int, st, C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.c_int, C.c_double, _d, _u8]
        L.wo_scalar_line_step.argtypes = [lm, C.c_int, C.c_double, C.c_int, C.c_double,
                                          C.c_double, C.c_int, C.c_double, _d]
        L.wo_scalar_tri_step.argtypes = [tm, _i32, _d, C.c_double, C.c_double, C.c_int,
                                         C.c_double, _d]
        L.wo_tri_rule_points.argtypes = [tm, C.c_int, _d, _d]
        L.wo_tri_project.argtypes = [tm, C.c_int, C.c_int, C.c_int, _d, _d]
        L.wo_line_rule_points.argtypes = [lm, C.c_int, _d]
        L.wo_line_project.argtypes = [lm, C.c_int, C.c_int, C.c_int, _d, _d]
        L.wo_tri_mass.argtypes = [tm, _d, C.c_int64]
        L.wo_tri_mass.restype = C.c_double
        L.wo_line_mass.argtypes = [lm, _d, C.c_int64]
        L.wo_line_mass.restype = C.c_double

    # ---- basis / quadrature -------------------------------------------------
    def dubiner(self, xi, eta, p):
        out = np.zeros(tri_modes(p))
        self.lib.wo_dubiner_basis(xi, eta, p, _p(out))
        return out

    def dubiner_gradient(self, xi, eta, p):
        gx, ge = np.zeros(tri_modes(p)), np.zeros(tri_modes(p))
        self.lib.wo_dubiner_basis_gradient(xi, eta, p, _p(gx), _p(ge))
        return gx, ge

    def legendre(self, xi, p):
        out = np.zeros(p + 1)
        self.lib.wo_legendre_basis(xi, p, _p(out))
        return out

    def gauss_legendre(self, n):
        pts, wts = np.zeros(8), np.zeros(8)
        k = self.lib.wo_gauss_legendre(n, _p(pts), _p(wts))
        return pts[:k].copy(), wts[:k].copy()

    def tri_volume_rule(self, p):
        n = (p + 1) ** 2
        xi, eta, w = np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib.wo_tri_volume_rule(p, _p(xi), _p(eta), _p(w))
        return xi, eta, w

    def tri_edge_rules(self, p):
        n = 3 * (p + 1)
        xi, eta, w, nx, ny = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(3), np.zeros(3)
        self.lib.wo_tri_edge_rules(p, _p(xi), _p(eta), _p(w), _p(nx), _p(ny))
        return xi, eta, w, nx, ny

    def hllc(self, gamma, left, right, nx, ny):
        out = np.zeros(4)
        self.lib.wo_hllc_flux(gamma, _p(f64(left)), _p(f64(right)), nx, ny, _p(out))
        return out

    def characteristic_weno(self, gamma, average, nx, ny, target, candidates, count, M):
        out = np.zeros(4 * M)
        self.lib.wo_characteristic_weno(gamma, _p(f64(average)), nx, ny, _p(f64(target)),
                                        _p(f64(candidates)), count, M, _p(out))
        return out

    def positivity(self, gamma, coefficients, M, basis, npts, rf, pf):
        c = f64(coefficients).copy()
        scale = np.zeros(1)
        rc = self.lib.wo_positivity(gamma, _p(c), M, _p(f64(basis)), npts, rf, pf, _p(scale))
        return rc, c, scale[0]

    # ---- meshes ---------------------------------------------------------------
    def tri_mesh(self, tags, xy, tris):
        return OracleTriMesh(self, tags, xy, tris)

    def line_mesh(self, tags, x, segs):
        return OracleLineMesh(self, tags, x, segs)


def _view(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


class OracleTriMesh:
    def __init__(self, oracle: Oracle, tags, xy, tris):
        self.o, self.lib = oracle, oracle.lib
        self.s = WoTriMesh()
        tags = np.ascontiguousarray(tags, dtype=np.int64)
        xy = f64(xy)
        tris = np.ascontiguousarray(tris, dtype=np.int64)
        rc = self.lib.wo_tri_mesh_build(len(tags), _p(tags, _i64), _p(xy), len(tris),
                                        _p(tris, _i64), C.byref(self.s))
        if rc != 0:
            raise ValueError(f"oracle triangle mesh build failed ({rc})")
        ne, nf = self.s.element_count, self.s.face_count
        self.ne, self.nf = ne, nf
        self.vertices = _view(self.s.vertices, 6 * ne, np.float64).reshape(ne, 6)
        self.nodes = _view(self.s.nodes, 3 * ne, np.int64).reshape(ne, 3)
        self.face_left = _view(self.s.face_left, nf, np.int32)
        self.face_right = _view(self.s.face_right, nf, np.int32)
        self.face_left_edge = _view(self.s.face_left_edge, nf, np.int32)
        self.face_right_edge = _view(self.s.face_right_edge, nf, np.int32)
        self.face_left_v0 = _view(self.s.face_left_v0, nf, np.int64)
        self.face_right_v0 = _view(self.s.face_right_v0, nf, np.int64)
        self.face_normal_x = _view(self.s.face_normal_x, nf, np.float64)
        self.face_normal_y = _view(self.s.face_normal_y, nf, np.float64)

    def __del__(self):
        try:
            self.lib.wo_tri_mesh_free(C.byref(self.s))
        except Exception:
            pass

    @property
    def ptr(self):
        return C.byref(self.s)

    def euler_residual(self, gamma, p, c, ext):
        rhs = np.zeros_like(f64(c))
        self.lib.wo_euler_tri_residual(self.ptr, gamma, p, _p(f64(c)), _p(f64(ext)), _p(rhs))
        return rhs

    def scalar_residual(self, vx, vy, p, c, ext):
        rhs = np.zeros_like(f64(c))
        self.lib.wo_scalar_tri_residual(self.ptr, vx, vy, p, _p(f64(c)), _p(f64(ext)), _p(rhs))
        return rhs

    def periodic_trace(self, p):
        Q, M = p + 1, tri_modes(p)
        donors = np.zeros(self.nf * Q, dtype=np.int32)
        basis = np.zeros(self.nf * Q * M)
        rc = self.lib.wo_periodic_tri_trace(self.ptr, p, _p(donors, _i32), _p(basis))
        if rc != 0:
            raise ValueError(f"periodic trace failed ({rc})")
        return donors, basis

    def periodic_exterior(self, p, donors, basis, c):
        ext = np.zeros(4 * self.nf * (p + 1))
        self.lib.wo_periodic_tri_euler_exterior(self.ptr, p, _p(donors, _i32), _p(basis),
                                                _p(f64(c)), _p(ext))
        return ext

    def periodic_scalar_exterior(self, p, donors, basis, c):
        ext = np.zeros(self.nf * (p + 1))
        self.lib.wo_periodic_tri_scalar_exterior(self.ptr, p, _p(donors, _i32), _p(basis),
                                                 _p(f64(c)), _p(ext))
        return ext

    def transmissive_exterior(self, p, c):
        ext = np.zeros(4 * self.nf * (p + 1))
        self.lib.wo_transmissive_tri_euler_exterior(self.ptr, p, _p(f64(c)), _p(ext))
        return ext

    def stencil(self, p, donors=None):
        return OracleStencil(self, p, donors)

    def cfl(self, gamma, c, p, cfl):
        dt = np.zeros(1)
        rc = self.lib.wo_euler_tri_cfl(self.ptr, gamma, _p(f64(c)), p, cfl, _p(dt))
        if rc != 0:
            raise ValueError("simulation: Euler cell average is not physical")
        return dt[0]

    def minimum_altitude(self):
        return self.lib.wo_tri_minimum_altitude(self.ptr)

    def scalar_cfl(self, vx, vy, p, cfl):
        return self.lib.wo_tri_scalar_cfl(self.ptr, vx, vy, p, cfl)

    def euler_step(self, gamma, p, dt, c, boundary="periodic", donors=None, basis=None,
                   stencil=None, threshold=1e-3, density_floor=1e-10, pressure_floor=1e-10,
                   return_flags=False):
        """One SSP-RK3 step in place on c; returns the per-stage flags if asked."""
        setup = WoEulerTriSetup()
        setup.boundary_kind = 3 if boundary == "transmissive" else 0
        if setup.boundary_kind == 0:
            setup.donors = _p(donors, _i32)
            setup.donor_basis = _p(basis)
        if stencil is not None:
            setup.stencil = C.pointer(stencil.s)
        setup.threshold, setup.density_floor, setup.pressure_floor = (
            threshold, density_floor, pressure_floor)
        flags = np.zeros(3 * self.ne, dtype=np.uint8)
        assert c.dtype == np.float64 and c.flags.c_contiguous
        rc = self.lib.wo_euler_tri_step(self.ptr, C.byref(setup), gamma, p, dt, _p(c),
                                        _p(flags, _u8))
        if rc != 0:
            raise ValueError("Euler positivity limiter: cell average is below a floor")
        return flags.reshape(3, self.ne) if return_flags else None

    def scalar_step(self, vx, vy, p, dt, c, donors, basis):
        self.lib.wo_scalar_tri_step(self.ptr, _p(donors, _i32), _p(basis), vx, vy, p, dt, _p(c))

    def rule_points(self, rule_order):
        Q = (rule_order + 1) ** 2
        x, y = np.zeros(self.ne * Q), np.zeros(self.ne * Q)
        self.lib.wo_tri_rule_points(self.ptr, rule_order, _p(x), _p(y))
        return x.reshape(self.ne, Q), y.reshape(self.ne, Q)

    def project(self, p, rule_order, values):
        """values [element][point][variable] -> U[variable][mode][element]"""
        values = f64(values)
        nv = values.shape[-1]
        c = np.zeros(nv * tri_modes(p) * self.ne)
        self.lib.wo_tri_project(self.ptr, p, rule_order, nv, _p(values), _p(c))
        return c

    def mass(self, mode0, stride):
        return self.lib.wo_tri_mass(self.ptr, _p(f64(mode0)), stride)


class OracleLineMesh:
    def __init__(self, oracle: Oracle, tags, x, segs):
        self.o, self.lib = oracle, oracle.lib
        self.s = WoLineMesh()
        tags = np.ascontiguousarray(tags, dtype=np.int64)
        x = f64(x)
        segs = np.ascontiguousarray(segs, dtype=np.int64)
        rc = self.lib.wo_line_mesh_build(len(tags), _p(tags, _i64), _p(x), len(segs),
                                         _p(segs, _i64), C.byref(self.s))
        if rc != 0:
            raise ValueError(f"oracle line mesh build failed ({rc})")
        self.ne, self.nf = self.s.element_count, self.s.face_count
        self.x_left = _view(self.s.x_left, self.ne, np.float64)
        self.x_right = _view(self.s.x_right, self.ne, np.float64)

    def __del__(self):
        try:
            self.lib.wo_line_mesh_free(C.byref(self.s))
        except Exception:
            pass

    @property
    def ptr(self):
        return C.byref(self.s)

    def euler_residual(self, gamma, p, c, ext):
        rhs = np.zeros_like(f64(c))
        self.lib.wo_euler_line_residual(self.ptr, gamma, p, _p(f64(c)), _p(f64(ext)), _p(rhs))
        return rhs

    def scalar_residual(self, a, p, c, ext):
        rhs = np.zeros_like(f64(c))
        self.lib.wo_scalar_line_residual(self.ptr, a, p, _p(f64(c)), _p(f64(ext)), _p(rhs))
        return rhs

    def euler_exterior(self, p, left_kind, right_kind, c):
        ext = np.zeros(4 * self.nf)
        rc = self.lib.wo_line_euler_exterior(self.ptr, p, left_kind, right_kind, _p(f64(c)),
                                             _p(ext))
        if rc != 0:
            raise ValueError("line Euler exterior: inflow is not implemented")
        return ext

    def scalar_exterior(self, p, lk, lv, rk, rv, c):
        ext = np.zeros(self.nf)
        self.lib.wo_line_scalar_exterior(self.ptr, p, lk, lv, rk, rv, _p(f64(c)), _p(ext))
        return ext

    def stencil(self, p, periodic=True):
        return OracleStencil(self, p, None, periodic=periodic)

    def cfl(self, gamma, c, p, cfl):
        dt = np.zeros(1)
        rc = self.lib.wo_euler_line_cfl(self.ptr, gamma, _p(f64(c)), p, cfl, _p(dt))
        if rc != 0:
            raise ValueError("simulation: Euler cell average is not physical")
        return dt[0]

    def advection_cfl(self, a, p, cfl):
        return self.lib.wo_line_advection_cfl(self.ptr, a, p, cfl)

    def euler_step(self, gamma, p, dt, c, left_kind=0, right_kind=0, stencil=None,
                   threshold=1e-3, density_floor=1e-10, pressure_floor=1e-10,
                   return_flags=False):
        """In place on c; with return_flags the troubled sets [stage][element]."""
        st = C.pointer(stencil.s) if stencil is not None else None
        flags = np.zeros(3 * self.ne, dtype=np.uint8)
        rc = self.lib.wo_euler_line_step(self.ptr, left_kind, right_kind, st, threshold,
                                         density_floor, pressure_floor, gamma, p, dt, _p(c),
                                         _p(flags, _u8))
        if rc != 0:
            raise ValueError("Euler line step failed")
        if return_flags:
            return flags.reshape(3, self.ne)

    def scalar_step(self, a, p, dt, c, lk=0, lv=0.0, rk=0, rv=0.0):
        self.lib.wo_scalar_line_step(self.ptr, lk, lv, rk, rv, a, p, dt, _p(c))

    def rule_points(self, n):
        x = np.zeros(self.ne * n)
        self.lib.wo_line_rule_points(self.ptr, n, _p(x))
        return x.reshape(self.ne, n)

    def project(self, p, n, values):
        values = f64(values)
        nv = values.shape[-1]
        c = np.zeros(nv * (p + 1) * self.ne)
        self.lib.wo_line_project(self.ptr, p, n, nv, _p(values), _p(c))
        return c

    def mass(self, mode0, stride):
        return self.lib.wo_line_mass(self.ptr, _p(f64(mode0)), stride)


class OracleStencil:
    def __init__(self, mesh, p, donors=None, periodic=True):
        self.mesh, self.lib = mesh, mesh.lib
        self.s = WoStencil()
        if isinstance(mesh, OracleTriMesh):
            d = _p(donors, _i32) if donors is not None else None
            self.lib.wo_tri_stencil(mesh.ptr, p, d, p + 1, C.byref(self.s))
        else:
            self.lib.wo_line_stencil(mesh.ptr, p, 1 if periodic else 0, C.byref(self.s))
        s = self.s
        ne, nb, M = s.element_count, s.maximum_neighbors, s.mode_count
        self.M, self.nb = M, nb
        self.neighbors = _view(s.neighbors, ne * nb, np.int32).reshape(ne, nb)
        self.transforms = _view(s.transforms, ne * nb * M * M, np.float64).reshape(ne, nb, M, M)
        self.normal_x = _view(s.normal_x, ne, np.float64)
        self.normal_y = _view(s.normal_y, ne, np.float64)
        self.check_basis = _view(s.check_basis, s.check_point_count * M, np.float64).reshape(
            s.check_point_count, M)
        self.highest_degree_begin = s.highest_degree_begin

    def __del__(self):
        try:
            self.lib.wo_stencil_free(C.byref(self.s))
        except Exception:
            pass

    def limit(self, gamma, threshold, rf, pf, c):
        """In place on c; returns the troubled flags."""
        flags = np.zeros(self.s.element_count, dtype=np.uint8)
        bad = np.zeros(1, dtype=np.int64)
        rc = self.lib.wo_limit_euler(C.byref(self.s), gamma, threshold, rf, pf, _p(c),
                                     _p(flags, _u8), _p(bad, _i64))
        if rc != 0:
            raise ValueError(f"Euler positivity limiter: element {bad[0]}")
        return flags

    def flags(self, threshold, c):
        flags = np.zeros(self.s.element_count, dtype=np.uint8)
        self.lib.wo_troubled_flags(C.byref(self.s), threshold, _p(f64(c)), _p(flags, _u8))
        return flags


class Reference:
    """The reference's own numerical core (oracle/_ref/libwaslref.so)."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def __init__(self, path: str = REF_SO):
        self.lib = L = C.CDLL(path)
        vp = C.c_void_p
        L.wr_last_error.restype = C.c_char_p
        L.wr_tri_mesh_new.restype = vp
        L.wr_tri_mesh_new.argtypes = [C.c_int64, _i64, _d, C.c_int64, _i64]
        L.wr_tri_mesh_free.argtypes = [vp]
        L.wr_tri_mesh_face_count.argtypes = [vp]
        L.wr_tri_mesh_face_count.restype = C.c_int64
        L.wr_tri_mesh_export.argtypes = [vp, _d, _i64, _i32, _i32, _i32, _i32, _i64, _i64, _d, _d]
        L.wr_line_mesh_new.restype = vp
        L.wr_line_mesh_new.argtypes = [C.c_int64, _i64, _d, C.c_int64, _i64]
        L.wr_line_mesh_free.argtypes = [vp]
        L.wr_line_mesh_export.argtypes = [vp, _d, _d]
        L.wr_euler_tri_residual.argtypes = [vp, C.c_double, C.c_int, _d, _d, _d]
        L.wr_euler_line_residual.argtypes = [vp, C.c_double, C.c_int, _d, _d, _d]
        L.wr_scalar_line_residual.argtypes = [vp, C.c_double, C.c_int, _d, _d, _d]
        L.wr_scalar_tri_residual.argtypes = [vp, C.c_double, C.c_double, C.c_int, _d, _d, _d]
        L.wr_hllc_flux.argtypes = [C.c_double, _d, _d, C.c_double, C.c_double, _d]
        L.wr_periodic_tri_trace.argtypes = [vp, C.c_int, _i32, _d]
        L.wr_periodic_tri_euler_exterior.argtypes = [vp, C.c_int, _i32, _d, _d, _d]
        L.wr_line_euler_exterior.argtypes = [vp, C.c_int, C.c_int, C.c_int, _d, _d]
        L.wr_tri_stencil_new.restype = vp
        L.wr_tri_stencil_new.argtypes = [vp, C.c_int, _i32]
        L.wr_line_stencil_new.restype = vp
        L.wr_line_stencil_new.argtypes = [vp, C.c_int, C.c_int]
        L.wr_stencil_free.argtypes = [vp]
        L.wr_stencil_export.argtypes = [vp, _i32, _d, _d, _d, _d, C.POINTER(C.c_int)]
        L.wr_limit_euler.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, _d]
        L.wr_euler_tri_cfl.argtypes = [vp, C.c_double, _d, C.c_int, C.c_double, _d]
        L.wr_euler_line_cfl.argtypes = [vp, C.c_double, _d, C.c_int, C.c_double, _d]
        L.wr_euler_tri_step.argtypes = [vp, _i32, _d, vp, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_int, C.c_double, _d]
        L.wr_euler_tri_step_ex.argtypes = [vp, C.c_int, _i32, _d, vp, C.c_double, C.c_double,
                                           C.c_double, C.c_double, C.c_int, C.c_double, _d, _u8]
        L.wr_euler_line_step.argtypes = [vp, C.c_int, C.c_int, vp, C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.c_int, C.c_double, _d]
        L.wr_scalar_line_run.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_uint64, _d, C.POINTER(C.c_uint64), _d]
        L.wr_scalar_line_step.argtypes = [vp, C.c_int, C.c_double, C.c_int, C.c_double,
                                          C.c_double, C.c_int, C.c_double, _d]

    def err(self):
        return self.lib.wr_last_error().decode()

    def tri_mesh(self, tags, xy, tris):
        return RefTriMesh(self, tags, xy, tris)

    def line_mesh(self, tags, x, segs):
        return RefLineMesh(self, tags, x, segs)

    def hllc(self, gamma, left, right, nx, ny):
        out = np.zeros(4)
        self.lib.wr_hllc_flux(gamma, _p(f64(left)), _p(f64(right)), nx, ny, _p(out))
        return out


class RefTriMesh:
    def __init__(self, ref: Reference, tags, xy, tris):
        self.r, self.lib = ref, ref.lib
        tags = np.ascontiguousarray(tags, dtype=np.int64)
        xy = f64(xy)
        tris = np.ascontiguousarray(tris, dtype=np.int64)
        self.h = self.lib.wr_tri_mesh_new(len(tags), _p(tags, _i64), _p(xy), len(tris),
                                          _p(tris, _i64))
        if not self.h:
            raise ValueError(ref.err())
        self.ne = len(tris)
        self.nf = self.lib.wr_tri_mesh_face_count(self.h)

    def __del__(self):
        try:
            self.lib.wr_tri_mesh_free(self.h)
        except Exception:
            pass

    def export(self):
        ne, nf = self.ne, self.nf
        out = dict(vertices=np.zeros((ne, 6)), nodes=np.zeros((ne, 3), np.int64),
                   face_left=np.zeros(nf, np.int32), face_right=np.zeros(nf, np.int32),
                   face_left_edge=np.zeros(nf, np.int32), face_right_edge=np.zeros(nf, np.int32),
                   face_left_v0=np.zeros(nf, np.int64), face_right_v0=np.zeros(nf, np.int64),
                   face_normal_x=np.zeros(nf), face_normal_y=np.zeros(nf))
        self.lib.wr_tri_mesh_export(
            self.h, _p(out["vertices"]), _p(out["nodes"], _i64), _p(out["face_left"], _i32),
            _p(out["face_right"], _i32), _p(out["face_left_edge"], _i32),
            _p(out["face_right_edge"], _i32), _p(out["face_left_v0"], _i64),
            _p(out["face_right_v0"], _i64), _p(out["face_normal_x"]), _p(out["face_normal_y"]))
        return out

    def euler_residual(self, gamma, p, c, ext):
        rhs = np.zeros_like(f64(c))
        self.lib.wr_euler_tri_residual(self.h, gamma, p, _p(f64(c)), _p(f64(ext)), _p(rhs))
        return rhs

    def scalar_residual(self, vx, vy, p, c, ext):
        rhs = np.zeros_like(f64(c))
        self.lib.wr_scalar_tri_residual(self.h, vx, vy, p, _p(f64(c)), _p(f64(ext)), _p(rhs))
        return rhs

    def periodic_trace(self, p):
        Q, M = p + 1, tri_modes(p)
        donors = np.zeros(self.nf * Q, dtype=np.int32)
        basis = np.zeros(self.nf * Q * M)
        if self.lib.wr_periodic_tri_trace(self.h, p, _p(donors, _i32), _p(basis)) != 0:
            raise ValueError(self.r.err())
        return donors, basis

    def periodic_exterior(self, p, donors, basis, c):
        ext = np.zeros(4 * self.nf * (p + 1))
        self.lib.wr_periodic_tri_euler_exterior(self.h, p, _p(donors, _i32), _p(basis),
                                                _p(f64(c)), _p(ext))
        return ext

    def stencil(self, p, donors=None):
        return RefStencil(self, p, donors)

    def cfl(self, gamma, c, p, cfl):
        dt = np.zeros(1)
        if self.lib.wr_euler_tri_cfl(self.h, gamma, _p(f64(c)), p, cfl, _p(dt)) != 0:
            raise ValueError(self.r.err())
        return dt[0]

    def euler_step(self, gamma, p, dt, c, donors, basis, stencil=None, threshold=1e-3,
                   density_floor=1e-10, pressure_floor=1e-10):
        st = stencil.h if stencil is not None else None
        rc = self.lib.wr_euler_tri_step(self.h, _p(donors, _i32), _p(basis), st, threshold,
                                        density_floor, pressure_floor, gamma, p, dt, _p(c))
        if rc != 0:
            raise ValueError(self.r.err())


    def euler_step_ex(self, gamma, p, dt, c, boundary="periodic", donors=None, basis=None,
                      stencil=None, threshold=1e-3, density_floor=1e-10, pressure_floor=1e-10):
        """One SSP-RK3 step in place with the periodic (donors, basis) or the
        transmissive exterior; returns the per-stage troubled-cell flags
        [3][ne] when a stencil is given."""
        kind = {"periodic": 0, "transmissive": 3}[boundary]
        flags = np.zeros((3, self.ne), np.uint8)
        st = stencil.h if stencil is not None else None
        d = _p(donors, _i32) if donors is not None else None
        b = _p(basis) if basis is not None else None
        rc = self.lib.wr_euler_tri_step_ex(self.h, kind, d, b, st, threshold, density_floor,
                                           pressure_floor, gamma, p, dt, _p(c), _p(flags, _u8))
        if rc != 0:
            raise ValueError(self.r.err())
        return flags


class RefLineMesh:
    def __init__(self, ref: Reference, tags, x, segs):
        self.r, self.lib = ref, ref.lib
        tags = np.ascontiguousarray(tags, dtype=np.int64)
        x = f64(x)
        segs = np.ascontiguousarray(segs, dtype=np.int64)
        self.h = self.lib.wr_line_mesh_new(len(tags), _p(tags, _i64), _p(x), len(segs),
                                           _p(segs, _i64))
        if not self.h:
            raise ValueError(ref.err())
        self.ne = len(segs)
        self.nf = self.ne + 1

    def __del__(self):
        try:
            self.lib.wr_line_mesh_free(self.h)
        except Exception:
            pass

    def export(self):
        xl, xr = np.zeros(self.ne), np.zeros(self.ne)
        self.lib.wr_line_mesh_export(self.h, _p(xl), _p(xr))
        return xl, xr

    def euler_residual(self, gamma, p, c, ext):
        rhs = np.zeros_like(f64(c))
        self.lib.wr_euler_line_residual(self.h, gamma, p, _p(f64(c)), _p(f64(ext)), _p(rhs))
        return rhs

    def scalar_residual(self, a, p, c, ext):
        rhs = np.zeros_like(f64(c))
        self.lib.wr_scalar_line_residual(self.h, a, p, _p(f64(c)), _p(f64(ext)), _p(rhs))
        return rhs

    def euler_exterior(self, p, lk, rk, c):
        ext = np.zeros(4 * self.nf)
        if self.lib.wr_line_euler_exterior(self.h, p, lk, rk, _p(f64(c)), _p(ext)) != 0:
            raise ValueError(self.r.err())
        return ext

    def stencil(self, p, periodic=True):
        return RefStencil(self, p, None, periodic=periodic)

    def cfl(self, gamma, c, p, cfl):
        dt = np.zeros(1)
        if self.lib.wr_euler_line_cfl(self.h, gamma, _p(f64(c)), p, cfl, _p(dt)) != 0:
            raise ValueError(self.r.err())
        return dt[0]

    def euler_step(self, gamma, p, dt, c, left_kind=0, right_kind=0, stencil=None,
                   threshold=1e-3, density_floor=1e-10, pressure_floor=1e-10):
        st = stencil.h if stencil is not None else None
        rc = self.lib.wr_euler_line_step(self.h, left_kind, right_kind, st, threshold,
                                         density_floor, pressure_floor, gamma, p, dt, _p(c))
        if rc != 0:
            raise ValueError(self.r.err())

    def scalar_step(self, a, p, dt, c, lk=0, lv=0.0, rk=0, rv=0.0):
        self.lib.wr_scalar_line_step(self.h, lk, lv, rk, rv, a, p, dt, _p(c))

    def scalar_run(self, a, p, cfl, start_time, end_time, c, max_steps=2**62):
        """The reference's periodic advection run in place (c: U[element][mode]);
        returns (steps, time)."""
        steps, t = C.c_uint64(), np.zeros(1)
        if self.lib.wr_scalar_line_run(self.h, p, a, cfl, start_time, end_time, max_steps,
                                       _p(c), C.byref(steps), _p(t)) != 0:
            raise ValueError(self.r.err())
        return steps.value, float(t[0])


class RefStencil:
    def __init__(self, mesh, p, donors=None, periodic=True):
        self.mesh, self.lib = mesh, mesh.lib
        if isinstance(mesh, RefTriMesh):
            d = _p(donors, _i32) if donors is not None else None
            self.h = self.lib.wr_tri_stencil_new(mesh.h, p, d)
            self.M, self.nb = tri_modes(p), 3
            nchk = (p + 1) ** 2 + 3 * (p + 1)
        else:
            self.h = self.lib.wr_line_stencil_new(mesh.h, p, 1 if periodic else 0)
            self.M, self.nb = p + 1, 2
            nchk = max(1, p + 1) + 2
        ne, nb, M = mesh.ne, self.nb, self.M
        self.neighbors = np.zeros((ne, nb), np.int32)
        self.transforms = np.zeros((ne, nb, M, M))
        self.normal_x, self.normal_y = np.zeros(ne), np.zeros(ne)
        self.check_basis = np.zeros((nchk, M))
        cnt = C.c_int(0)
        self.lib.wr_stencil_export(self.h, _p(self.neighbors, _i32), _p(self.transforms),
                                   _p(self.normal_x), _p(self.normal_y), _p(self.check_basis),
                                   C.byref(cnt))

    def __del__(self):
        try:
            self.lib.wr_stencil_free(self.h)
        except Exception:
            pass

    def limit(self, gamma, threshold, rf, pf, c):
        if self.lib.wr_limit_euler(self.h, gamma, threshold, rf, pf, _p(c)) != 0:
            raise ValueError(self.mesh.r.err())
