"""Drop-in Python surface of ``gw_fopt.bubble_gw.many_bubbles`` for the bulk-flow path.

Mirrors the PyO3 classes of the reference
(rust/py-bubble-gw/src/py_many_bubbles/*.rs, stubs in
src/gw_fopt/bubble_gw/many_bubbles.pyi:16-231): same class and method names,
keyword-only arguments, return dtypes/shapes and exception classes
(IndexError for an out-of-range bubble index, ValueError otherwise,
py_generalized_bulk_flow.rs:117-126).  Geometry and validation run in the
C++ host library and the spectrum on the GPU, both through the C ABI
(include/bubble_gw.h, include/bubble_gw_b200.h).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Sequence

import numpy as np

from . import _lib as L

__all__ = [
    "Isometry3", "ParallelepipedLattice", "CartesianLattice", "SphericalLattice", "EmptyLattice",
    "LatticeBubbles", "ExponentialTimeCutoff", "GeneralizedBulkFlow", "NewGeneralizedBulkFlow",
]


def _raise(err: L.BgwError):
    msg = err.message
    if msg.startswith("Index ") and " out of bounds for max " in msg:
        idx, mx = msg[len("Index "):].split(" out of bounds for max ")
        raise IndexError(f"Index {idx} out of bounds (max: {mx})") from None
    raise ValueError(msg) from None


def _call(status):
    try:
        L.check(status)
    except L.BgwError as e:
        _raise(e)


# ----------------------------------------------------------------------------
# Isometry3 (rust/py-bubble-gw/src/py_many_bubbles/py_isometry.rs)
# ----------------------------------------------------------------------------
def _euler(roll, pitch, yaw):
    # nalgebra Rotation3::from_euler_angles: R = Rz(yaw) Ry(pitch) Rx(roll)
    sr, cr = math.sin(roll), math.cos(roll)
    sp, cp = math.sin(pitch), math.cos(pitch)
    sy, cy = math.sin(yaw), math.cos(yaw)
    return np.array([[cy * cp, cy * sp * sr - sy * cr, cy * sp * cr + sy * sr],
                     [sy * cp, sy * sp * sr + cy * cr, sy * sp * cr - cy * sr],
                     [-sp, cp * sr, cp * cr]])


def _nearest_rotation(m):
    u, _, vt = np.linalg.svd(np.asarray(m, dtype=np.float64))
    r = u @ vt
    if np.linalg.det(r) < 0:
        u[:, -1] = -u[:, -1]
        r = u @ vt
    return r


def _rotation_from_input(euler_angles, rotation_matrix):
    if euler_angles is not None and rotation_matrix is not None:
        raise ValueError("Specify either euler_angles or rotation_matrix, not both.")
    if euler_angles is not None:
        return _euler(*[float(v) for v in euler_angles])
    if rotation_matrix is not None:
        return _nearest_rotation(rotation_matrix)
    return np.eye(3)


class Isometry3:
    """Rigid motion p -> R p + t."""

    def __init__(self, translation=(0.0, 0.0, 0.0), *, euler_angles=None, rotation_matrix=None):
        self._t = np.asarray(translation, dtype=np.float64).reshape(3).copy()
        self._r = _rotation_from_input(euler_angles, rotation_matrix)

    @classmethod
    def _from(cls, r, t):
        obj = cls.__new__(cls)
        obj._r = np.asarray(r, dtype=np.float64)
        obj._t = np.asarray(t, dtype=np.float64).reshape(3)
        return obj

    @staticmethod
    def identity():
        return Isometry3._from(np.eye(3), np.zeros(3))

    @staticmethod
    def from_translation(translation):
        return Isometry3._from(np.eye(3), translation)

    @staticmethod
    def from_rotation(*, euler_angles=None, rotation_matrix=None):
        return Isometry3._from(_rotation_from_input(euler_angles, rotation_matrix), np.zeros(3))

    @staticmethod
    def from_euler_angles(roll, pitch, yaw):
        return Isometry3._from(_euler(roll, pitch, yaw), np.zeros(3))

    @staticmethod
    def from_axis_angle(axis, angle):
        a = np.asarray(axis, dtype=np.float64).reshape(3)
        n = float(np.linalg.norm(a))
        if n < np.finfo(np.float64).eps:
            raise ValueError("Axis must be a non-zero vector.")
        u = a / n
        K = np.array([[0, -u[2], u[1]], [u[2], 0, -u[0]], [-u[1], u[0], 0]])
        r = np.eye(3) + math.sin(angle) * K + (1.0 - math.cos(angle)) * (K @ K)
        return Isometry3._from(r, np.zeros(3))

    def transform(self, other: "Isometry3") -> "Isometry3":
        return Isometry3._from(self._r @ other._r, self._r @ other._t + self._t)

    def rotate(self, *, euler_angles=None, rotation_matrix=None):
        return Isometry3._from(_rotation_from_input(euler_angles, rotation_matrix) @ self._r, self._t)

    def translate(self, translation):
        return Isometry3._from(self._r, self._t + np.asarray(translation, dtype=np.float64))

    @property
    def translation(self):
        return tuple(float(v) for v in self._t)

    @property
    def rotation_matrix(self):
        return tuple(tuple(float(v) for v in row) for row in self._r)

    def apply_points(self, pts):
        pts = np.asarray(pts, dtype=np.float64).reshape(-1, 3)
        return pts @ self._r.T + self._t

    def __repr__(self):
        t = self._t
        return f"Isometry3(translation=[{t[0]:.3f}, {t[1]:.3f}, {t[2]:.3f}], rotation=...)"


# ----------------------------------------------------------------------------
# Lattices (rust/py-bubble-gw/src/py_many_bubbles/py_lattice.rs)
# ----------------------------------------------------------------------------
_EPS = np.finfo(np.float64).eps


class _Lattice:
    _kind = L.LATTICE_EMPTY

    def _params(self) -> np.ndarray:
        return np.zeros(0)

    def parameters(self):
        return [float(v) for v in self._params()]


class ParallelepipedLattice(_Lattice):
    _kind = L.LATTICE_PARALLELEPIPED

    def __init__(self, origin, basis):
        self._origin = np.asarray(origin, dtype=np.float64).reshape(3).copy()
        self._basis = np.asarray(basis, dtype=np.float64).reshape(3, 3).copy()  # rows = e1, e2, e3
        if abs(np.linalg.det(self._basis.T)) <= _EPS:
            raise ValueError("Basis vectors are linearly dependent (zero volume)")

    def name(self):
        return "ParallelepipedLattice"

    @staticmethod
    def axis_aligned(origin, lx, ly, lz):
        return ParallelepipedLattice(origin, np.diag([lx, ly, lz]))

    @staticmethod
    def cube_centered(center, side):
        h = side / 2.0
        return ParallelepipedLattice(np.asarray(center, dtype=np.float64) - h, np.eye(3) * side)

    def _params(self):
        return np.concatenate([self._origin, self._basis.ravel()])

    def transform(self, iso: Isometry3):
        obj = self.__class__.__new__(self.__class__)
        obj._origin = iso.apply_points(self._origin)[0]
        obj._basis = self._basis @ iso._r.T
        return obj

    @property
    def origin(self):
        return tuple(float(v) for v in self._origin)

    @property
    def basis(self):
        return tuple(tuple(float(v) for v in row) for row in self._basis)

    @property
    def normalized_basis(self):
        out = []
        for e in self._basis:
            n2 = float(e @ e)
            out.append(tuple(float(v) for v in (e / math.sqrt(n2) if n2 > _EPS else np.zeros(3))))
        return tuple(out)

    @property
    def volume(self):
        return float(abs(np.linalg.det(self._basis.T)))


class CartesianLattice(ParallelepipedLattice):
    _kind = L.LATTICE_CARTESIAN

    def __init__(self, origin, basis):
        super().__init__(origin, basis)
        e1, e2, e3 = self._basis
        eps = 1e-10
        if abs(e1 @ e2) > eps or abs(e1 @ e3) > eps or abs(e2 @ e3) > eps:
            raise ValueError("Basis vectors are not pairwise orthogonal")

    def name(self):
        return "CartesianLattice"

    @staticmethod
    def with_origin_and_sizes(origin, sizes):
        return CartesianLattice(origin, np.diag(np.asarray(sizes, dtype=np.float64)))

    @property
    def side_lengths(self):
        return tuple(float(np.linalg.norm(e)) for e in self._basis)


class SphericalLattice(_Lattice):
    _kind = L.LATTICE_SPHERICAL

    def __init__(self, center, radius):
        self._center = np.asarray(center, dtype=np.float64).reshape(3).copy()
        self._radius = float(radius)

    def name(self):
        return "SphericalLattice"

    def _params(self):
        return np.concatenate([self._center, [self._radius]])

    def transform(self, iso: Isometry3):
        return SphericalLattice(iso.apply_points(self._center)[0], self._radius)

    @property
    def center(self):
        return tuple(float(v) for v in self._center)

    @property
    def radius(self):
        return self._radius

    @property
    def volume(self):
        return (4.0 / 3.0) * math.pi * self._radius ** 3


class EmptyLattice(_Lattice):
    _kind = L.LATTICE_EMPTY

    def name(self):
        return "EmptyLattice"

    def transform(self, iso):
        return EmptyLattice()

    @property
    def volume(self):
        return 0.0

    def __repr__(self):
        return "EmptyLattice()"


def _contains(lattice: _Lattice, points) -> list:
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
    out = np.zeros(pts.shape[0], dtype=np.uint8)
    n_out = C.c_size_t(0)
    par = np.ascontiguousarray(lattice._params())
    _call(L.lib().bgwx_lattice_contains(lattice._kind, L.ptr(par), L.ptr(pts), pts.shape[0],
                                        out.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(n_out)))
    return [bool(v) for v in out[: n_out.value]]


_LATTICE_TYPE = {L.LATTICE_PARALLELEPIPED: "Parallelepiped", L.LATTICE_CARTESIAN: "Cartesian",
                 L.LATTICE_SPHERICAL: "Spherical", L.LATTICE_EMPTY: "Empty"}


# ----------------------------------------------------------------------------
# LatticeBubbles (rust/py-bubble-gw/src/py_many_bubbles/py_lattice_bubbles.rs,
# rust/bubble-gw/src/many_bubbles/lattice_bubbles.rs)
# ----------------------------------------------------------------------------
def _as_bubbles(a) -> np.ndarray:
    arr = np.asarray(a, dtype=np.float64)
    if arr.ndim != 2:
        raise TypeError("bubble arrays must be 2-D (n, 4) float64 arrays")
    return np.ascontiguousarray(arr)


class LatticeBubbles:
    def __init__(self, lattice, bubbles_interior, bubbles_exterior=None):
        if not isinstance(lattice, _Lattice):
            raise ValueError("Expected a lattice instance: ParallelepipedLattice, CartesianLattice, "
                             "SphericalLattice, or EmptyLattice")
        interior = _as_bubbles(bubbles_interior)
        exterior = np.zeros((0, 4)) if bubbles_exterior is None else _as_bubbles(bubbles_exterior)
        # lattice_bubbles.rs:216-263
        if interior.shape[1] != 4 or exterior.shape[1] != 4:
            raise ValueError(f"Array shape mismatch: Expected 4 columns, got {interior.shape[1]} for interior, "
                             f"{exterior.shape[1]} for exterior")
        inside_int = _contains(lattice, interior[:, 1:4])
        inside_ext = _contains(lattice, exterior[:, 1:4])
        out_int = [i for i, v in enumerate(inside_int) if not v]
        in_ext = [i for i, v in enumerate(inside_ext) if v]
        if out_int:
            raise ValueError("Interior bubbles formed outside lattice: [" +
                             ", ".join(f"Interior({i})" for i in out_int) + "]")
        if in_ext:
            raise ValueError("Exterior bubbles formed inside lattice: [" +
                             ", ".join(f"Exterior({i})" for i in in_ext) + "]")
        _call(L.lib().bgwx_check_causality(L.ptr(interior), interior.shape[0], L.ptr(exterior), exterior.shape[0]))
        self._lattice = lattice
        self._interior = interior.copy()
        self._exterior = exterior.copy()

    @classmethod
    def _raw(cls, lattice, interior, exterior):
        obj = cls.__new__(cls)
        obj._lattice = lattice
        obj._interior = np.ascontiguousarray(interior, dtype=np.float64)
        obj._exterior = np.ascontiguousarray(exterior, dtype=np.float64)
        return obj

    def __repr__(self):
        return (f"LatticeBubbles(lattice_type={_LATTICE_TYPE[self._lattice._kind]}, "
                f"n_interior={self._interior.shape[0]}, n_exterior={self._exterior.shape[0]})")

    def parameters(self):
        return self._lattice.parameters()

    def contains(self, points):
        return _contains(self._lattice, points)

    def transform(self, iso: Isometry3) -> "LatticeBubbles":
        def tr(b):
            out = b.copy()
            if b.shape[0]:
                out[:, 1:4] = iso.apply_points(b[:, 1:4])
            return out
        return LatticeBubbles._raw(self._lattice.transform(iso), tr(self._interior), tr(self._exterior))

    def with_boundary_condition(self, boundary_condition: str = "periodic") -> None:
        bc = {"periodic": L.BC_PERIODIC, "reflection": L.BC_REFLECTION, "none": L.BC_NONE}.get(
            str(boundary_condition).lower())
        if bc is None:
            raise ValueError("Invalid boundary condition. Expected 'periodic' or 'reflection'.")
        n = self._interior.shape[0]
        cap = 6 * n
        out = np.zeros((max(cap, 1), 4))
        n_out = C.c_size_t(0)
        par = np.ascontiguousarray(self._lattice._params())
        _call(L.lib().bgwx_lattice_exterior(self._lattice._kind, L.ptr(par), bc, L.ptr(self._interior), n,
                                            L.ptr(out), cap, C.byref(n_out)))
        self._exterior = np.ascontiguousarray(out[: n_out.value])

    def translate_time_mut(self, t_shift: float) -> None:
        self._interior[:, 0] += t_shift
        self._exterior[:, 0] += t_shift

    def translate_time(self, t_shift: float) -> "LatticeBubbles":
        obj = LatticeBubbles._raw(self._lattice, self._interior.copy(), self._exterior.copy())
        obj.translate_time_mut(t_shift)
        return obj

    def normalize_time_mut(self) -> None:
        times = np.concatenate([self._interior[:, 0], self._exterior[:, 0]])
        if times.size and np.isfinite(times.min()):
            self.translate_time_mut(-float(times.min()))

    def normalize_time(self) -> "LatticeBubbles":
        obj = LatticeBubbles._raw(self._lattice, self._interior.copy(), self._exterior.copy())
        obj.normalize_time_mut()
        return obj

    @property
    def lattice(self):
        return self._lattice

    @property
    def bubbles_interior(self):
        return self._interior.copy()

    @property
    def bubbles_exterior(self):
        return self._exterior.copy()

    @property
    def lattice_type(self):
        return _LATTICE_TYPE[self._lattice._kind]

    @property
    def volume(self):
        return float(self._lattice.volume)

    @property
    def reference_point(self):
        lat = self._lattice
        if isinstance(lat, ParallelepipedLattice):
            return lat.origin
        if isinstance(lat, SphericalLattice):
            return lat.center
        return (0.0, 0.0, 0.0)


# ----------------------------------------------------------------------------
# ExponentialTimeCutoff (rust/bubble-gw/src/time_cutoff.rs:15-43)
# ----------------------------------------------------------------------------
class ExponentialTimeCutoff:
    def __init__(self, smax: float, ratio_t_cut: Optional[float] = None, ratio_t_0: Optional[float] = None):
        self.smax = float(smax)
        self.ratio_t_cut = ratio_t_cut
        self.ratio_t_0 = ratio_t_0
        rc = 0.999999999 if ratio_t_cut is None else float(ratio_t_cut)
        r0 = 0.25 if ratio_t_0 is None else float(ratio_t_0)
        self._t_cut = rc * self.smax
        self._t_0 = r0 * (self.smax - self._t_cut)

    @property
    def t_cut(self):
        return self._t_cut

    @property
    def t_0(self):
        return self._t_0

    def _config(self):
        return L.BgwTimeCutoffConfig(1, self.smax, math.nan if self.ratio_t_cut is None else self.ratio_t_cut,
                                     math.nan if self.ratio_t_0 is None else self.ratio_t_0)


_UNIT_CUTOFF = L.BgwTimeCutoffConfig(0, 0.0, math.nan, math.nan)


def _cutoff_config(time_cutoff):
    if time_cutoff is None:
        return _UNIT_CUTOFF
    if not isinstance(time_cutoff, ExponentialTimeCutoff):
        raise TypeError("time_cutoff must be an ExponentialTimeCutoff or None")
    return time_cutoff._config()


def _linspace(a, b, n):
    step = (b - a) / (n - 1) if n > 1 else 0.0
    return [a + step * i for i in range(n)]


# ----------------------------------------------------------------------------
# GeneralizedBulkFlow (rust/py-bubble-gw/src/py_many_bubbles/py_generalized_bulk_flow.rs:156-441)
# ----------------------------------------------------------------------------
class GeneralizedBulkFlow:
    def __init__(self, lattice_bubbles: LatticeBubbles):
        if not isinstance(lattice_bubbles, LatticeBubbles):
            raise TypeError("lattice_bubbles must be a LatticeBubbles")
        self._interior = lattice_bubbles._interior.copy()
        self._exterior = lattice_bubbles._exterior.copy()
        h = C.c_void_p()
        _call(L.lib().bgwx_generalized_bulk_flow_new_unchecked(
            C.byref(h), L.ptr(self._interior), self._interior.shape[0], L.ptr(self._exterior),
            self._exterior.shape[0]))
        self._h = h
        self._coefficients = np.array([[1.0]])
        self._powers = np.array([[3.0]])
        self._damping = None
        self._n_cos = None
        self._n_phi = None
        self._pushed = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                L.lib().bgw_generalized_bulk_flow_free(h)
            except Exception:
                pass
            self._h = None

    # --- configuration -------------------------------------------------------
    def set_num_threads(self, num_threads: int) -> None:
        if int(num_threads) < 0:
            raise OverflowError("can't convert negative int to unsigned")
        _call(L.lib().bgw_generalized_bulk_flow_set_num_threads(self._h, int(num_threads)))

    def set_coefficients_sets(self, coefficients_sets) -> None:
        self._coefficients = np.array(coefficients_sets, dtype=np.float64, ndmin=2)

    def set_powers_sets(self, powers_sets) -> None:
        self._powers = np.array(powers_sets, dtype=np.float64, ndmin=2)

    def set_gradient_scaling_params(self, coefficients_sets, powers_sets, damping_factor=None) -> None:
        # generalized_bulk_flow.rs:315-363
        cs = [list(map(float, v)) for v in coefficients_sets]
        ps = [list(map(float, v)) for v in powers_sets]
        nc = len(cs[0]) if cs else 0
        if any(len(v) != nc for v in cs):
            raise ValueError("Array shape mismatch: All coefficient sets must have the same length")
        npw = len(ps[0]) if ps else 0
        if any(len(v) != npw for v in ps):
            raise ValueError("Array shape mismatch: All power sets must have the same length")
        if len(cs) != len(ps):
            raise ValueError("Array shape mismatch: Number of coefficient sets and power sets must be equal")
        self._coefficients = np.array(cs, dtype=np.float64).reshape(len(cs), nc)
        self._powers = np.array(ps, dtype=np.float64).reshape(len(ps), npw)
        self._damping = None if damping_factor is None else float(damping_factor)

    def set_resolution(self, n_cos_thetax: int, n_phix: int, precompute_first_bubbles: bool = True) -> None:
        _call(L.lib().bgw_generalized_bulk_flow_set_resolution(self._h, int(n_cos_thetax), int(n_phix),
                                                               bool(precompute_first_bubbles)))
        self._n_cos, self._n_phi = int(n_cos_thetax), int(n_phix)

    def _push_params(self):
        co, po = self._coefficients, self._powers
        if co.shape != po.shape:
            raise ValueError(f"Array shape mismatch: coefficients_sets {co.shape} and powers_sets {po.shape} "
                             "must have the same shape")
        key = (co.tobytes(), po.tobytes(), co.shape, self._damping)
        if key == self._pushed:
            return
        S, M = co.shape
        if M == 0:
            raise ValueError("Array shape mismatch: coefficient sets must not be empty")
        co = np.ascontiguousarray(co)
        po = np.ascontiguousarray(po)
        _call(L.lib().bgw_generalized_bulk_flow_set_gradient_scaling_params(
            self._h, L.ptr(co), L.ptr(po), S, M, math.nan if self._damping is None else self._damping))
        self._pushed = key

    def set_kernel(self, kernel: str) -> None:
        """Selects the spectrum kernel: 'fp64_direct', 'fp64_factored' or 'mixed' (B200 extension)."""
        k = {"fp64_direct": L.KERNEL_FP64_DIRECT, "fp64_factored": L.KERNEL_FP64_FACTORED,
             "mixed": L.KERNEL_MIXED, "mixed_simt": L.KERNEL_MIXED_SIMT}[kernel]
        _call(L.lib().bgwx_generalized_bulk_flow_set_kernel(self._h, k))

    def set_launch_shape(self, frames_per_launch: int = 0, row_parts: int = 0) -> None:
        """Fixes how spectrum calls are cut into launches (B200 extension): at most
        ``frames_per_launch`` k-hat frames per launch and ``row_parts`` cos-theta row
        parts per tensor-core GEMM tile; 0 keeps the automatic choice of either."""
        if frames_per_launch < 0 or row_parts < 0:
            raise ValueError("frames_per_launch and row_parts must be >= 0")
        _call(L.lib().bgwx_generalized_bulk_flow_set_launch_shape(self._h, int(frames_per_launch), int(row_parts)))

    def set_autotune(self, enabled: bool = True) -> None:
        """Measured launch shapes (B200 extension): the first spectrum call of each problem
        shape on a factored kernel times candidate shapes on its own first frames and keeps
        the fastest; ``BGWX_AUTOTUNE_CACHE`` may name a file that keeps the choices."""
        _call(L.lib().bgwx_generalized_bulk_flow_set_autotune(self._h, bool(enabled)))

    def last_launch_shape(self) -> tuple[int, int]:
        """(frames per launch, GEMM row parts) of the last spectrum call; (0, 0) before one."""
        f, r = C.c_size_t(0), C.c_size_t(0)
        _call(L.lib().bgwx_generalized_bulk_flow_last_launch_shape(self._h, C.byref(f), C.byref(r)))
        return int(f.value), int(r.value)

    def set_gemm_stages(self, stages: int = 0) -> None:
        """Pipeline stages of the mixed kernel's tensor-core GEMM (B200 extension): 3, 4 or 5,
        or 0 for the automatic (or autotuned) choice.  The result does not depend on it."""
        _call(L.lib().bgwx_generalized_bulk_flow_set_gemm_stages(self._h, int(stages)))

    def last_gemm_stages(self) -> int:
        """GEMM stages of the last spectrum call (0 when it did not run the tensor-core GEMM)."""
        n = C.c_size_t(0)
        _call(L.lib().bgwx_generalized_bulk_flow_last_gemm_stages(self._h, C.byref(n)))
        return int(n.value)

    def set_mask_chunking(self, chunking: int = 0) -> None:
        """Blocks of the first-collider search per (bubble, k-hat frame): 1, 2 or 4 times the
        automatic number; 0 keeps the automatic (or measured) choice (B200 extension).  The masks
        are the same for every choice."""
        _call(L.lib().bgwx_generalized_bulk_flow_set_mask_chunking(self._h, int(chunking)))

    def last_mask_chunking(self) -> int:
        """Mask-search chunking of the last spectrum call."""
        n = C.c_size_t(0)
        _call(L.lib().bgwx_generalized_bulk_flow_last_mask_chunking(self._h, C.byref(n)))
        return int(n.value)

    # --- geometry -------------------------------------------------------------
    def _require_res(self, name="n_cos_thetax"):
        if self._n_cos is None:
            raise ValueError(f"Field '{name}' is not initialized")

    def _check_a(self, a_idx):
        n = self._interior.shape[0]
        if a_idx < 0 or a_idx >= n:
            raise IndexError(f"Index {a_idx} out of bounds (max: {n})")

    def compute_first_colliding_bubble(self, a_idx: int) -> np.ndarray:
        """(n_cos, n_phi) int32: -1 None, i Interior(i), -(i+2) Exterior(i) (PYGBF:235-247), on the GPU."""
        self._require_res()
        self._check_a(int(a_idx))
        out = np.empty((self._n_cos, self._n_phi), dtype=np.int32)
        _call(L.lib().bgwx_generalized_bulk_flow_first_colliding(
            self._h, int(a_idx), int(a_idx) + 1, out.ctypes.data_as(C.POINTER(C.c_int32)), None))
        return out

    def _directions(self):
        cos_t = _linspace(-1.0, 1.0, self._n_cos)
        phi = _linspace(0.0, 2.0 * math.pi, self._n_phi)
        d = np.empty((self._n_cos, self._n_phi, 4))
        for i, c in enumerate(cos_t):
            s = abs(math.sqrt(1.0 - c * c))
            for j, p in enumerate(phi):
                d[i, j] = (1.0, s * math.cos(p), s * math.sin(p), c)
        return d

    def compute_delta_tab(self, a_idx: int, first_bubble) -> np.ndarray:
        """Collision delays for given first-collider codes (generalized_bulk_flow.rs:421-471)."""
        self._require_res()
        self._check_a(int(a_idx))
        fb = np.asarray(first_bubble, dtype=np.int32)
        if fb.shape != (self._n_cos, self._n_phi):
            raise ValueError(f"Array shape mismatch: First bubble array must match resolution: expected "
                             f"[{self._n_cos}, {self._n_phi}], got {list(fb.shape)}")
        n_int = self._interior.shape[0]
        allb = np.concatenate([self._interior, self._exterior])
        xa = self._interior[int(a_idx)]
        dirs = self._directions()
        out = np.zeros(fb.shape)
        for (i, j), code in np.ndenumerate(fb):
            if code == -1:
                continue
            b = int(code) if code >= 0 else n_int + (-int(code) - 2)
            d = [float(allb[b, q]) - float(xa[q]) for q in range(4)]
            x = dirs[i, j]
            dsq = (((-d[0]) * d[0] + d[1] * d[1]) + d[2] * d[2]) + d[3] * d[3]
            dot = (((-d[0]) * x[0] + d[1] * x[1]) + d[2] * x[2]) + d[3] * x[3]
            out[i, j] = 0.0 if abs(dot) < 1e-10 else dsq / (2.0 * dot)
        return out

    def compute_collision_status(self, a_idx: int, t: float, first_bubble, delta_tab_grid) -> np.ndarray:
        """0 NeverCollided, 1 AlreadyCollided, 2 NotYetCollided (generalized_bulk_flow.rs:369-414)."""
        self._require_res()
        self._check_a(int(a_idx))
        fb = np.asarray(first_bubble, dtype=np.int32)
        dt = np.asarray(delta_tab_grid, dtype=np.float64)
        shape = (self._n_cos, self._n_phi)
        if fb.shape != shape or dt.shape != shape:
            raise ValueError(f"Array shape mismatch: Input arrays must match resolution: expected "
                             f"[{shape[0]}, {shape[1]}], got first_bubble: {list(fb.shape)}, "
                             f"delta_tab_grid: {list(dt.shape)}")
        delta_ta = float(t) - float(self._interior[int(a_idx), 0])
        status = np.where((dt > 0.0) & (delta_ta >= dt), 1, 2).astype(np.int32)
        status[fb == -1] = 0
        return status

    # --- spectrum ---------------------------------------------------------------
    def _compute(self, w_arr, t_begin, t_end, n_t, selected, time_cutoff):
        self._push_params()
        w = np.ascontiguousarray(np.asarray(w_arr, dtype=np.float64).ravel())
        S = self._coefficients.shape[0]
        out = np.zeros((2, S, w.size), dtype=np.complex128)
        if selected is not None:
            sel = np.ascontiguousarray(selected, dtype=np.uint64)
            psel = sel.ctypes.data_as(C.POINTER(C.c_size_t))
            nsel = sel.size
        else:
            psel, nsel = None, 0
        _call(L.lib().bgw_generalized_bulk_flow_compute_c_integral(
            self._h, L.ptr(w), w.size, t_begin is not None, 0.0 if t_begin is None else float(t_begin),
            float(t_end), int(n_t), psel, nsel, _cutoff_config(time_cutoff),
            out.ctypes.data_as(C.POINTER(L.BgwComplex64)), out.size))
        return out

    @staticmethod
    def _selected(selected_bubbles):
        if selected_bubbles is None:
            return None
        arr = np.asarray(selected_bubbles)
        if arr.ndim != 1:
            raise ValueError("selected_bubbles must be a contiguous 1-D array in C order")
        if arr.size and (not np.issubdtype(arr.dtype, np.integer) or arr.min() < 0):
            raise TypeError("selected_bubbles must hold non-negative integers")
        # a non-null pointer marks "Some(slice)" even when empty
        return np.ascontiguousarray(arr.astype(np.uint64)) if arr.size else np.zeros(1, dtype=np.uint64)[:0]

    def compute_c_integral(self, w_arr, *, t_begin=None, t_end, n_t, selected_bubbles=None, time_cutoff=None):
        """(2, n_sets, n_w) complex128 = [C_+, C_x] (PYGBF:381-428), computed on the GPU."""
        sel = self._selected(selected_bubbles)
        if sel is not None and sel.size == 0:
            # Some(empty) -> zeros after the n_t check (generalized_bulk_flow.rs:946-957)
            if int(n_t) < 2:
                raise ValueError("Invalid resolution: n_t must be >= 2 for integration")
            return np.zeros((2, self._coefficients.shape[0], np.asarray(w_arr).size), dtype=np.complex128)
        return self._compute(w_arr, t_begin, t_end, n_t, sel, time_cutoff)

    def compute_c_integral_fixed_bubble(self, a_idx, w_arr, t_begin, t_end, n_t, time_cutoff=None):
        """One bubble's (2, n_sets, n_w) contribution (generalized_bulk_flow.rs:775-873)."""
        self._check_a(int(a_idx))
        tb = 0.0 if t_begin is None else float(t_begin)
        if tb > float(t_end):
            raise ValueError(f"Invalid time range: t_begin={_rust_f64(tb)} > t_end={_rust_f64(float(t_end))}")
        if int(n_t) < 2:
            return np.zeros((2, self._coefficients.shape[0], np.asarray(w_arr).size), dtype=np.complex128)
        return self._compute(w_arr, t_begin, t_end, n_t, np.array([int(a_idx)], dtype=np.uint64), time_cutoff)

    def compute_c_integral_khat(self, w_arr, khat, *, t_begin=None, t_end, n_t, selected_bubbles=None,
                                time_cutoff=None):
        """(K, 2, n_sets, n_w) complex128: the spectrum along each unit k-hat row (B200 extension).

        Each k-hat block equals compute_c_integral on the configuration rotated
        by R(k) (the Rodrigues rotation taking k-hat to z about k x z)."""
        self._push_params()
        w = np.ascontiguousarray(np.asarray(w_arr, dtype=np.float64).ravel())
        kh = np.ascontiguousarray(np.asarray(khat, dtype=np.float64).reshape(-1, 3))
        S = self._coefficients.shape[0]
        out = np.zeros((kh.shape[0], 2, S, w.size), dtype=np.complex128)
        sel = self._selected(selected_bubbles)
        if sel is not None and sel.size == 0:
            return out
        psel = sel.ctypes.data_as(C.POINTER(C.c_size_t)) if sel is not None else None
        _call(L.lib().bgwx_generalized_bulk_flow_compute_c_integral_khat(
            self._h, L.ptr(w), w.size, t_begin is not None, 0.0 if t_begin is None else float(t_begin),
            float(t_end), int(n_t), L.ptr(kh), kh.shape[0], psel, 0 if sel is None else sel.size,
            _cutoff_config(time_cutoff), out.ctypes.data_as(C.POINTER(L.BgwComplex64)), out.size))
        return out

    def compute_c_integrand_fixed_bubble(self, a_idx, w_arr, t_begin, t_end, n_t):
        """(2, n_sets, n_w, n_t) complex128: bubble a_idx's time-resolved integrand
        (generalized_bulk_flow.rs:776-866), computed on the GPU."""
        self._check_a(int(a_idx))
        n_t = int(n_t)
        S = self._coefficients.shape[0]
        w = np.ascontiguousarray(np.asarray(w_arr, dtype=np.float64).ravel())
        if float(self._interior[int(a_idx), 0]) >= float(t_end) or n_t < 2:
            # a bubble nucleating at or after t_end gives zeros (:786-789); with fewer
            # than two steps dt is 0 and every value vanishes (:798-799)
            tb = 0.0 if t_begin is None else float(t_begin)
            if float(self._interior[int(a_idx), 0]) < float(t_end) and tb > float(t_end):
                raise ValueError(f"Invalid time range: t_begin={_rust_f64(tb)} > t_end={_rust_f64(float(t_end))}")
            return np.zeros((2, S, w.size, max(n_t, 0)), dtype=np.complex128)
        return self.compute_c_integrand(w, t_begin=t_begin, t_end=t_end, n_t=n_t,
                                        selected_bubbles=np.array([int(a_idx)]))

    def compute_c_integrand(self, w_arr, *, t_begin=None, t_end, n_t, selected_bubbles=None):
        """(2, n_sets, n_w, n_t) complex128: the time-resolved integrand summed over
        the selected bubbles (generalized_bulk_flow.rs:875-920), computed on the GPU."""
        self._push_params()
        w = np.ascontiguousarray(np.asarray(w_arr, dtype=np.float64).ravel())
        S = self._coefficients.shape[0]
        if int(n_t) < 0:
            raise OverflowError("can't convert negative int to unsigned")
        out = np.zeros((2, S, w.size, int(n_t)), dtype=np.complex128)
        sel = self._selected(selected_bubbles)
        psel = sel.ctypes.data_as(C.POINTER(C.c_size_t)) if sel is not None else None
        _call(L.lib().bgwx_generalized_bulk_flow_compute_c_integrand(
            self._h, L.ptr(w), w.size, t_begin is not None, 0.0 if t_begin is None else float(t_begin),
            float(t_end), int(n_t), psel, 0 if sel is None else sel.size,
            out.ctypes.data_as(C.POINTER(L.BgwComplex64)), out.size))
        return out

    # --- properties -------------------------------------------------------------
    @property
    def bubbles_interior(self):
        return self._interior.copy()

    @property
    def bubbles_exterior(self):
        return self._exterior.copy()

    @property
    def coefficients_sets(self):
        return self._coefficients.copy()

    @property
    def get_powers_sets(self):
        return self._powers.copy()

    @property
    def cos_thetax(self):
        self._require_res("cos_thetax")
        return np.array(_linspace(-1.0, 1.0, self._n_cos))

    @property
    def phix(self):
        self._require_res("phix")
        return np.array(_linspace(0.0, 2.0 * math.pi, self._n_phi))

    def last_timings(self) -> dict:
        """Device timings of the last compute call (B200 extension)."""
        t = L.BgwxTimings()
        _call(L.lib().bgwx_generalized_bulk_flow_last_timings(self._h, C.byref(t)))
        return {f: getattr(t, f) for f, _ in L.BgwxTimings._fields_}


class NewGeneralizedBulkFlow(GeneralizedBulkFlow):
    """The tensor form (the reference's NewGeneralizedBulkFlow,
    rust/py-bubble-gw/src/py_many_bubbles/py_new_generalized_bulk_flow.rs and
    rust/bubble-gw/src/many_bubbles/new_generalized_bulk_flow.rs): C_ij(w) in six
    components xx, xy, xz, yy, yz, zz, from the phi integral of x_i x_j (t - t_n)^3 f
    instead of the cos 2phi / sin 2phi projections.  Configuration and geometry
    methods are those of GeneralizedBulkFlow; the spectrum runs in plain FP64 on
    the GPU (the direct kernel), with no time cutoff (the tensor form has none)."""

    def _compute_tensor(self, w_arr, t_begin, t_end, n_t, selected, khat=None):
        self._push_params()
        w = np.ascontiguousarray(np.asarray(w_arr, dtype=np.float64).ravel())
        S = self._coefficients.shape[0]
        kh = None if khat is None else np.ascontiguousarray(np.asarray(khat, dtype=np.float64).reshape(-1, 3))
        K = 1 if kh is None else kh.shape[0]
        out = np.zeros((K, 6, S, w.size), dtype=np.complex128)
        if selected is not None:
            sel = np.ascontiguousarray(selected, dtype=np.uint64)
            psel, nsel = sel.ctypes.data_as(C.POINTER(C.c_size_t)), sel.size
        else:
            psel, nsel = None, 0
        _call(L.lib().bgwx_generalized_bulk_flow_compute_c_tensor_khat(
            self._h, L.ptr(w), w.size, t_begin is not None, 0.0 if t_begin is None else float(t_begin),
            float(t_end), int(n_t), L.ptr(kh) if kh is not None else None, 0 if kh is None else K, psel, nsel,
            out.ctypes.data_as(C.POINTER(L.BgwComplex64)), out.size))
        return out if khat is not None else out[0]

    def compute_c_tensor(self, w_arr, *, t_begin=None, t_end, n_t, selected_bubbles=None):
        """(6, n_sets, n_w) complex128, summed over the selected bubbles (new_generalized_bulk_flow.rs:1205-1275)."""
        if int(n_t) < 2:
            raise ValueError("Invalid resolution: n_t must be >= 2 for integration")
        sel = self._selected(selected_bubbles)
        if sel is not None and sel.size == 0:
            return np.zeros((6, self._coefficients.shape[0], np.asarray(w_arr).size), dtype=np.complex128)
        return self._compute_tensor(w_arr, t_begin, t_end, n_t, sel)

    def compute_c_tensor_fixed_bubble(self, a_idx, w_arr, t_begin, t_end, n_t):
        """One bubble's (6, n_sets, n_w) contribution (new_generalized_bulk_flow.rs:1067-1203)."""
        self._check_a(int(a_idx))
        tb = 0.0 if t_begin is None else float(t_begin)
        if tb > float(t_end):
            raise ValueError(f"Invalid time range: t_begin={_rust_f64(tb)} > t_end={_rust_f64(float(t_end))}")
        if int(n_t) < 2:
            return np.zeros((6, self._coefficients.shape[0], np.asarray(w_arr).size), dtype=np.complex128)
        return self._compute_tensor(w_arr, t_begin, t_end, n_t, np.array([int(a_idx)], dtype=np.uint64))

    def compute_c_tensor_khat(self, w_arr, khat, *, t_begin=None, t_end, n_t, selected_bubbles=None):
        """(K, 6, n_sets, n_w): the tensor of each k-hat row's rotated configuration (B200 extension)."""
        if int(n_t) < 2:
            raise ValueError("Invalid resolution: n_t must be >= 2 for integration")
        sel = self._selected(selected_bubbles)
        kh = np.asarray(khat, dtype=np.float64).reshape(-1, 3)
        if sel is not None and sel.size == 0:
            return np.zeros((kh.shape[0], 6, self._coefficients.shape[0], np.asarray(w_arr).size),
                            dtype=np.complex128)
        return self._compute_tensor(w_arr, t_begin, t_end, n_t, sel, khat=kh)


    def compute_c_tensor_integrand(self, w_arr, *, t_begin=None, t_end, n_t, selected_bubbles=None):
        """(6, n_sets, n_w, n_t): the time-resolved tensor integrand summed over the selected
        bubbles (new_generalized_bulk_flow.rs:993-1065), computed on the GPU."""
        self._push_params()
        w = np.ascontiguousarray(np.asarray(w_arr, dtype=np.float64).ravel())
        S = self._coefficients.shape[0]
        if int(n_t) < 0:
            raise OverflowError("can't convert negative int to unsigned")
        out = np.zeros((6, S, w.size, int(n_t)), dtype=np.complex128)
        sel = self._selected(selected_bubbles)
        psel = sel.ctypes.data_as(C.POINTER(C.c_size_t)) if sel is not None else None
        _call(L.lib().bgwx_generalized_bulk_flow_compute_c_tensor_integrand(
            self._h, L.ptr(w), w.size, t_begin is not None, 0.0 if t_begin is None else float(t_begin),
            float(t_end), int(n_t), psel, 0 if sel is None else sel.size,
            out.ctypes.data_as(C.POINTER(L.BgwComplex64)), out.size))
        return out

    def compute_c_tensor_integrand_fixed_bubble(self, a_idx, w_arr, t_begin, t_end, n_t):
        """(6, n_sets, n_w, n_t): bubble a_idx's time-resolved tensor integrand
        (new_generalized_bulk_flow.rs:832-991)."""
        self._check_a(int(a_idx))
        n_t = int(n_t)
        S = self._coefficients.shape[0]
        w = np.ascontiguousarray(np.asarray(w_arr, dtype=np.float64).ravel())
        if float(self._interior[int(a_idx), 0]) >= float(t_end) or n_t < 2:
            tb = 0.0 if t_begin is None else float(t_begin)
            if float(self._interior[int(a_idx), 0]) < float(t_end) and tb > float(t_end):
                raise ValueError(f"Invalid time range: t_begin={_rust_f64(tb)} > t_end={_rust_f64(float(t_end))}")
            return np.zeros((6, S, w.size, max(n_t, 0)), dtype=np.complex128)
        return self.compute_c_tensor_integrand(w, t_begin=t_begin, t_end=t_end, n_t=n_t,
                                               selected_bubbles=np.array([int(a_idx)]))


def tt_energy(c_tensor, khat=(0.0, 0.0, 1.0)):
    """Lambda_ij,lm(k) C*_ij C_lm = Tr[P C* P C] - |Tr[P C]|^2 / 2, P = 1 - k k^T
    (docs/generalized_bulkflow.md:8-17), for c_tensor (6, ...) in the order
    xx, xy, xz, yy, yz, zz; the energy per ln w and solid angle is 2 G w^3 times
    this (with T = kappa rho v^3 C).  For k = z it is 2 (|C_+|^2 + |C_x|^2) with
    C_+ = (C_xx - C_yy) / 2, C_x = C_xy."""
    c = np.asarray(c_tensor)
    k = np.asarray(khat, dtype=np.float64)
    k = k / np.linalg.norm(k)
    idx = [[0, 1, 2], [1, 3, 4], [2, 4, 5]]
    T = np.stack([np.stack([c[idx[i][j]] for j in range(3)]) for i in range(3)])  # (3, 3, ...)
    P = np.eye(3) - np.outer(k, k)
    PT = np.einsum("ij,jl...->il...", P, T)
    tr_pc = np.einsum("ii...->...", PT)
    tr_pcpc = np.einsum("ij...,ji...->...", np.conj(PT), PT)
    return np.real(tr_pcpc) - 0.5 * np.abs(tr_pc) ** 2


def _rust_f64(x: float) -> str:
    """Rust's Display of f64 (shortest round-trip, positional)."""
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    if x == 0.0:
        return "-0" if math.copysign(1.0, x) < 0 else "0"
    r = repr(x)
    neg = r.startswith("-")
    r = r.lstrip("-")
    if "e" in r:
        mant, exp = r.split("e")
        exp = int(exp)
        digits = mant.replace(".", "")
        point = (mant.index(".") if "." in mant else len(mant)) + exp
    else:
        digits = r.replace(".", "")
        point = r.index(".") if "." in r else len(r)
        # strip leading zeros of "0.00x"
        stripped = digits.lstrip("0")
        point -= len(digits) - len(stripped)
        digits = stripped
    digits = digits.rstrip("0") or "0"
    if point <= 0:
        s = "0." + "0" * (-point) + digits
    elif point >= len(digits):
        s = digits + "0" * (point - len(digits))
    else:
        s = digits[:point] + "." + digits[point:]
    return ("-" if neg else "") + s
