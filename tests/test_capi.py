"""C ABI checks that need no GPU: the library loads, exports every symbol the
headers declare, and reproduces the reference's argument validation and
error reporting (rust/c-bubble-gw/src/lib.rs:104-574,
rust/c-bubble-gw/tests/c_api.rs)."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

from gw_fopt_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("bubble_gw.h", "bubble_gw_b200.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(bgwx?_[a-z0-9_]+)\s*\(", src))
    return names


def test_every_declared_symbol_is_exported():
    lib = L.lib()
    names = declared_symbols()
    assert "bgw_generalized_bulk_flow_compute_c_integral" in names
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert names <= set(L.SIGNATURES), sorted(names - set(L.SIGNATURES))


def test_header_compiles_as_c_and_cxx(tmp_path):
    import shutil
    import subprocess
    for cc, std, ext in (("gcc", "-std=c11", "c"), ("g++", "-std=c++17", "cpp")):
        if not shutil.which(cc):
            pytest.skip(f"{cc} missing")
        src = tmp_path / f"t.{ext}"
        src.write_text('#include "bubble_gw_b200.h"\nint main(void){return (int)BGW_STATUS_OK;}\n')
        subprocess.run([cc, std, "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                        str(tmp_path / f"t_{ext}")], check=True)


def last_error():
    return L.lib().bgw_last_error_message().decode()


def new_handle(interior, exterior=None):
    interior = np.ascontiguousarray(interior, dtype=np.float64)
    exterior = np.zeros((0, 4)) if exterior is None else np.ascontiguousarray(exterior, dtype=np.float64)
    h = C.c_void_p()
    st = L.lib().bgw_generalized_bulk_flow_empty_lattice_new(C.byref(h), L.ptr(interior), interior.shape[0],
                                                              L.ptr(exterior), exterior.shape[0])
    return st, h


def test_version_and_error_roundtrip():
    lib = L.lib()
    assert lib.bgw_version().decode().startswith("0.1.0")
    st = lib.bgw_generalized_bulk_flow_set_num_threads(None, 1)
    assert st == L.CALCULATION_ERROR
    assert last_error() == "bulk_flow must not be null"
    st, h = new_handle([[0.0, 0, 0, 0]])
    assert st == L.OK and last_error() == ""
    assert lib.bgw_generalized_bulk_flow_set_num_threads(h, 0) == L.CALCULATION_ERROR
    assert last_error() == "num_threads must be > 0"
    assert lib.bgw_generalized_bulk_flow_set_num_threads(h, 4) == L.OK
    lib.bgw_generalized_bulk_flow_free(h)
    lib.bgw_generalized_bulk_flow_free(None)


def test_new_null_out_and_null_arrays():
    lib = L.lib()
    st = lib.bgw_generalized_bulk_flow_empty_lattice_new(None, None, 0, None, 0)
    assert st == L.NULL_POINTER and last_error() == "out must not be null"
    h = C.c_void_p(1234)
    st = lib.bgw_generalized_bulk_flow_empty_lattice_new(C.byref(h), None, 2, None, 0)
    assert st == L.CALCULATION_ERROR and h.value is None
    assert last_error() == "bubbles_interior must not be null"
    # zero-length arrays may be NULL
    st = lib.bgw_generalized_bulk_flow_empty_lattice_new(C.byref(h), None, 0, None, 0)
    assert st == L.OK
    lib.bgw_generalized_bulk_flow_free(h)


def test_causality_error_message():
    st, h = new_handle([[0.0, 0, 0, 0], [1.0, 0.5, 0, 0]])
    assert st == L.CALCULATION_ERROR and not h.value
    assert last_error() == ("Bubble Interior(0) is formed inside bubble Interior(1) at initial time "
                            "(overlapping light cones)")
    st, h = new_handle([[0.0, 0, 0, 0]], [[1.0, 0.25, 0, 0]])
    assert "Interior(0) is formed inside bubble Exterior(0)" in last_error()


def test_resolution_and_params_validation():
    lib = L.lib()
    st, h = new_handle([[0.0, 0, 0, 0]])
    assert lib.bgw_generalized_bulk_flow_set_resolution(h, 1, 5, True) == L.CALCULATION_ERROR
    assert last_error() == "Invalid resolution: Angular resolutions must be greater than one"
    assert lib.bgw_generalized_bulk_flow_set_resolution(h, 4, 5, True) == L.OK
    c = np.array([0.0, 1.0])
    p = np.array([3.0, 3.0])
    assert lib.bgw_generalized_bulk_flow_set_gradient_scaling_params(h, L.ptr(c), L.ptr(p), 2, 1,
                                                                       math.nan) == L.OK
    assert lib.bgw_generalized_bulk_flow_set_gradient_scaling_params(h, None, L.ptr(p), 2, 1,
                                                                       math.nan) == L.CALCULATION_ERROR
    assert last_error() == "coefficients must not be null"
    # chunks(0) panics in the reference's C ABI
    assert lib.bgw_generalized_bulk_flow_set_gradient_scaling_params(h, L.ptr(c), L.ptr(p), 2, 0,
                                                                       math.nan) == L.PANIC
    lib.bgw_generalized_bulk_flow_free(h)


def compute(h, w, n_t=10, t_begin=None, t_end=1.0, selected=None, out_len=None, n_sets=1):
    w = np.ascontiguousarray(w, dtype=np.float64)
    n = 2 * n_sets * w.size if out_len is None else out_len
    out = (L.BgwComplex64 * max(n, 1))()
    cut = L.BgwTimeCutoffConfig(0, 0.0, math.nan, math.nan)
    if selected is not None:
        sel = np.ascontiguousarray(selected, dtype=np.uint64)
        psel = sel.ctypes.data_as(C.POINTER(C.c_size_t))
        nsel = sel.size
    else:
        psel, nsel = None, 0
    return L.lib().bgw_generalized_bulk_flow_compute_c_integral(
        h, L.ptr(w), w.size, t_begin is not None, t_begin or 0.0, t_end, n_t, psel, nsel, cut, out, n), out


def test_compute_validation_order_without_gpu():
    st, h = new_handle([[0.0, 0, 0, 0], [0.0, 3.0, 0, 0]])
    # n_t < 2 is checked first
    st, _ = compute(h, [1.0], n_t=1)
    assert st == L.CALCULATION_ERROR and last_error() == "Invalid resolution: n_t must be >= 2 for integration"
    # invalid bubble index
    st, _ = compute(h, [1.0], selected=[0, 7])
    assert st == L.CALCULATION_ERROR and last_error() == "Index 7 out of bounds for max 2"
    # empty selection -> zeros, no device needed
    sel = np.zeros(1, dtype=np.uint64)
    out = (L.BgwComplex64 * 2)()
    cut = L.BgwTimeCutoffConfig(0, 0.0, math.nan, math.nan)
    w = np.array([1.0])
    st = L.lib().bgw_generalized_bulk_flow_compute_c_integral(h, L.ptr(w), 1, False, 0.0, 1.0, 10,
                                                              sel.ctypes.data_as(C.POINTER(C.c_size_t)), 0,
                                                              cut, out, 2)
    assert st == L.OK
    # out_len mismatch is reported after the work
    st, _ = compute(h, [1.0], selected=np.zeros(0), out_len=3)
    # (a NULL selection pointer with n=0 means "all bubbles")
    # bad time range precedes the resolution check
    st, _ = compute(h, [1.0], t_begin=2.0, t_end=1.0)
    assert st == L.CALCULATION_ERROR and last_error() == "Invalid time range: t_begin=2 > t_end=1"
    # no resolution set
    st, _ = compute(h, [1.0])
    assert st == L.CALCULATION_ERROR and last_error() == "Field 'n_cos_thetax' is not initialized"
    L.lib().bgw_generalized_bulk_flow_free(h)


def test_compute_without_gpu_fails_loudly():
    if L.lib().bgwx_device_count() > 0:
        pytest.skip("a GPU is visible")
    st, h = new_handle([[0.0, 0, 0, 0], [0.0, 3.0, 0, 0]])
    assert L.lib().bgw_generalized_bulk_flow_set_resolution(h, 4, 5, True) == L.OK
    st, _ = compute(h, [1.0])
    assert st == L.CALCULATION_ERROR
    assert "no CUDA device" in last_error()
    L.lib().bgw_generalized_bulk_flow_free(h)


def test_rotation_for_khat_matches_oracle():
    from oracle import oracle as O
    from gw_fopt_b200 import workloads as W
    R = np.zeros(9)
    for k in W.fibonacci_khat(9):
        L.lib().bgwx_rotation_for_khat(k[0], k[1], k[2], L.ptr(R))
        assert np.array_equal(R.reshape(3, 3), O.rotation_for_khat(k))


def test_lattice_images_and_containment():
    from gw_fopt_b200 import many_bubbles as mb
    from gw_fopt_b200 import workloads as W
    b, _ = W.uniform_config(5, 2.0, 0.1, seed=7)
    lat = mb.CartesianLattice([0, 0, 0], [[2, 0, 0], [0, 2, 0], [0, 0, 2]])
    lb = mb.LatticeBubbles(lat, b)
    lb.with_boundary_condition("periodic")
    assert np.array_equal(lb.bubbles_exterior, W.periodic_images(b, 2.0))
    lb.with_boundary_condition("reflection")
    ext = lb.bubbles_exterior
    assert ext.shape == (30, 4)
    np.testing.assert_allclose(ext[0, 1], -b[0, 1])            # mirror across x = 0
    np.testing.assert_allclose(ext[1, 1], 4.0 - b[0, 1])       # mirror across x = 2
    lb.with_boundary_condition("none")
    assert lb.bubbles_exterior.shape == (0, 4)
    with pytest.raises(ValueError, match="Invalid boundary condition"):
        lb.with_boundary_condition("twisted")
    assert lb.contains([[1.0, 1.0, 1.0], [3.0, 0, 0]]) == [True, False]
    sph = mb.SphericalLattice([0, 0, 0], 1.0)
    assert mb.LatticeBubbles(sph, [[0.0, 0.1, 0.2, 0.3]]).contains([[0.0, 0.0, 1.5]]) == [False]
    assert mb.LatticeBubbles(mb.EmptyLattice(), [[0.0, 5, 5, 5]]).contains([[0.0, 0, 0]]) == []
    with pytest.raises(ValueError, match=r"Interior bubbles formed outside lattice: \[Interior\(1\)\]"):
        mb.LatticeBubbles(lat, [[0.0, 1, 1, 1], [0.0, 3, 1, 1]])
    with pytest.raises(ValueError, match=r"Exterior bubbles formed inside lattice: \[Exterior\(0\)\]"):
        mb.LatticeBubbles(lat, [[0.0, 1, 1, 1]], [[0.0, 0.5, 0.5, 0.5]])
    with pytest.raises(ValueError, match="Expected 4 columns"):
        mb.LatticeBubbles(lat, np.zeros((2, 3)))
    with pytest.raises(ValueError, match="not pairwise orthogonal"):
        mb.CartesianLattice([0, 0, 0], [[1, 0, 0], [1, 1, 0], [0, 0, 1]])


def test_python_surface_errors_without_gpu():
    from gw_fopt_b200 import many_bubbles as mb
    lb = mb.LatticeBubbles(mb.EmptyLattice(), np.array([[0.0, 0, 10, 0], [0.0, 0, 0, 0]]))
    g = mb.GeneralizedBulkFlow(lb)
    with pytest.raises(ValueError, match="Field 'cos_thetax' is not initialized"):
        g.cos_thetax
    g.set_resolution(4, 5)
    np.testing.assert_array_equal(g.cos_thetax, [-1.0 + (2.0 / 3.0) * i for i in range(4)])
    with pytest.raises(IndexError, match=r"Index 5 out of bounds \(max: 2\)"):
        g.compute_c_integral([1.0], t_end=8.0, n_t=40, selected_bubbles=np.array([5]))
    with pytest.raises(ValueError, match="n_t must be >= 2"):
        g.compute_c_integral([1.0], t_end=8.0, n_t=1)
    with pytest.raises(ValueError, match="All coefficient sets must have the same length"):
        g.set_gradient_scaling_params([[1.0], [1.0, 2.0]], [[3.0], [3.0]])
    with pytest.raises(ValueError, match="Number of coefficient sets and power sets must be equal"):
        g.set_gradient_scaling_params([[1.0]], [[3.0], [3.0]])
    out = g.compute_c_integral([1.0, 2.0], t_end=8.0, n_t=40, selected_bubbles=np.array([], dtype=np.int64))
    assert out.shape == (2, 1, 2) and not out.any()
    # delta_tab / collision status are host utilities (generalized_bulk_flow.rs:369-471)
    fb = np.full((4, 5), -1, dtype=np.int32)
    fb[1, 3] = 1
    fb[2, 3] = 1
    dt = g.compute_delta_tab(0, fb)
    assert dt[1, 3] == pytest.approx(5.0 / math.sqrt(1 - 1 / 9.0), rel=1e-15)
    st = g.compute_collision_status(0, 6.0, fb, dt)
    assert st[0, 0] == 0 and st[1, 3] == 1
    st = g.compute_collision_status(0, 1.0, fb, dt)
    assert st[1, 3] == 2
    cut = mb.ExponentialTimeCutoff(2.0, 0.5)
    assert cut.t_cut == 1.0 and cut.t_0 == 0.25


def test_launch_shape_settings_without_gpu():
    from gw_fopt_b200 import many_bubbles as mb
    lb = mb.LatticeBubbles(mb.EmptyLattice(), np.array([[0.0, 0, 10, 0], [0.0, 0, 0, 0]]))
    g = mb.GeneralizedBulkFlow(lb)
    assert g.last_launch_shape() == (0, 0)
    g.set_launch_shape(2, 3)
    g.set_launch_shape()
    g.set_autotune(True)
    g.set_autotune(False)
    with pytest.raises(ValueError, match="row_parts must be at most 16"):
        g.set_launch_shape(1, 17)
    with pytest.raises(ValueError, match=">= 0"):
        g.set_launch_shape(-1, 0)
    f, r = C.c_size_t(7), C.c_size_t(7)
    assert L.lib().bgwx_generalized_bulk_flow_last_launch_shape(None, C.byref(f), C.byref(r)) != 0
