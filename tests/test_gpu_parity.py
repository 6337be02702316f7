"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Masks (first-collider codes and collision delays) must be bitwise equal to
the oracle's; spectra must agree to 1e-12 relative (norm over (+/x, sets) at
each w, max over w) for the FP64 kernels.  Cases follow the reference's own
tests and examples: the two-bubble C-ABI test (rust/c-bubble-gw/tests/c_api.rs:137-141),
the five-bubble bench geometry (rust/benches/bulk_flow_bench.rs:9-15), confY
with periodic images (docs/examples/generalized_bulkflow.py:743-757) and the
synthetic benchmark configurations.
"""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from gw_fopt_b200 import many_bubbles as mb
from gw_fopt_b200 import workloads as W

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FACTORED_PER_W_TOL = 1e-10
MIXED_TOL = 1e-6
SIMT_PER_W_BOUND = 1e-4
KERNELS = ["fp64_direct", "fp64_factored", "mixed", "mixed_simt"]
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_small.npz")


def err_per_w(got, ref):
    """max over w of ||got - ref||_2 / ||ref||_2 over all leading axes (k-hat, +/x, sets)."""
    g = got.reshape(-1, got.shape[-1])
    r = ref.reshape(-1, ref.shape[-1])
    num = np.linalg.norm(g - r, axis=0)
    den = np.linalg.norm(r, axis=0)
    scale = np.linalg.norm(r)
    return float(np.max(num / np.maximum(den, 1e-300 + 1e-13 * scale)))


def global_err(got, ref):
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))


def check(kernel, got, ref, label):
    """Per-kernel tolerances, all asserted per w (norm over k-hat, +/x and sets at each w):
    fp64_direct   follows the reference's arithmetic term by term: <= 1e-12 per w;
    fp64_factored forms the phase as w t (1 - c) + w (t_a c - z_a), whose rounding differs
                  from the reference's per-term rounding: <= 1e-12 globally and <= 1e-10 per w
                  (the difference grows at spectral dips, where |C(w)| is small);
    mixed         the int8 digit-slice tensor-core GEMM: <= 1e-6 per w;
    mixed_simt    FP32 operands on CUDA cores: <= 1e-6 globally; per w only a regression
                  bound (its absolute error floor, ~6e-8 of the terms, exceeds 1e-6 of |C(w)|
                  at deep dips)."""
    pw, glob = err_per_w(got, ref), global_err(got, ref)
    print(f"{label} {kernel}: per-w max {pw:.3e} global {glob:.3e}")
    if kernel == "fp64_direct":
        assert pw < FP64_TOL
    elif kernel == "fp64_factored":
        assert glob < FP64_TOL and pw < FACTORED_PER_W_TOL
    elif kernel == "mixed":
        assert pw < MIXED_TOL
    else:
        assert glob < MIXED_TOL and pw < SIMT_PER_W_BOUND


def golden_cases():
    g = np.load(GOLDEN)
    names = sorted({k.split("__")[0] for k in g.files})
    out = {}
    for n in names:
        out[n] = {k.split("__", 1)[1]: g[k] for k in g.files if k.startswith(n + "__")}
    return out


def make_flow(interior, exterior, n_cos, n_phi, coeffs=((1.0,),), powers=((3.0,),), damping=None,
              kernel="fp64_direct"):
    lb = mb.LatticeBubbles(mb.EmptyLattice(), np.asarray(interior, dtype=np.float64),
                           np.asarray(exterior, dtype=np.float64))
    g = mb.GeneralizedBulkFlow(lb)
    g.set_resolution(n_cos, n_phi)
    g.set_gradient_scaling_params([list(r) for r in coeffs], [list(r) for r in powers],
                                  None if damping is None or np.isnan(damping) else float(damping))
    g.set_kernel(kernel)
    return g


@pytest.mark.parametrize("name", ["capi2", "bench5", "confY", "cfg1_damped"])
def test_masks_bitwise_vs_golden(gpu_available, name):
    p = golden_cases()[name]
    g = make_flow(p["interior"], p["exterior"], int(p["n_cos"]), int(p["n_phi"]))
    for a in range(p["interior"].shape[0]):
        assert np.array_equal(g.compute_first_colliding_bubble(a), p["codes"][a]), (name, a)


def test_delta_tab_bitwise(gpu_available):
    import ctypes as C
    from gw_fopt_b200 import _lib as L
    c = W.config(2)
    n_cos = n_phi = 48
    lb = mb.LatticeBubbles(mb.EmptyLattice(), c.interior, c.exterior)
    g = mb.GeneralizedBulkFlow(lb)
    g.set_resolution(n_cos, n_phi)
    a0, a1 = 10, 26
    codes = np.empty((a1 - a0, n_cos, n_phi), dtype=np.int32)
    tau = np.empty((a1 - a0, n_cos, n_phi))
    L.check(L.lib().bgwx_generalized_bulk_flow_first_colliding(
        g._h, a0, a1, codes.ctypes.data_as(C.POINTER(C.c_int32)), tau.ctypes.data_as(C.POINTER(C.c_double))))
    rc, rt = O.first_colliding(c.interior, c.exterior, n_cos, n_phi, a0, a1, with_delta_tab=True)
    assert np.array_equal(codes, rc)
    assert np.array_equal(tau, rt)


def crowded_hemisphere(seed=11, n_near=700, n_far=300):
    """Radiating bubble 0 at the origin; n_near colliders within 0.05-0.1 of it on the +z side
    (more than one candidate list holds) and n_far colliders at 0.6-0.8 on the -z side, all
    nucleating at t = 0.  Directions into -z find their first collider only past the list,
    so the search takes its exhaustive path there."""
    rng = np.random.default_rng(seed)

    def shell(n, r0, r1, sign):
        v = rng.normal(size=(n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        v[:, 2] = sign * np.abs(v[:, 2])
        return v * rng.uniform(r0, r1, size=(n, 1))

    pts = np.concatenate([np.zeros((1, 3)), shell(n_near, 0.05, 0.1, 1.0), shell(n_far, 0.6, 0.8, -1.0)])
    return np.concatenate([np.zeros((pts.shape[0], 1)), pts], axis=1)


def test_masks_exhaustive_path_bitwise(gpu_available):
    import ctypes as C
    from gw_fopt_b200 import _lib as L
    interior = crowded_hemisphere()
    n_cos = n_phi = 24
    g = mb.GeneralizedBulkFlow(mb.LatticeBubbles(mb.EmptyLattice(), interior, np.zeros((0, 4))))
    g.set_resolution(n_cos, n_phi)
    codes = np.empty((2, n_cos, n_phi), dtype=np.int32)
    tau = np.empty((2, n_cos, n_phi))
    L.check(L.lib().bgwx_generalized_bulk_flow_first_colliding(
        g._h, 0, 2, codes.ctypes.data_as(C.POINTER(C.c_int32)), tau.ctypes.data_as(C.POINTER(C.c_double))))
    assert g.last_timings()["fallbacks"] > 0  # the exhaustive path ran
    rc, rt = O.first_colliding(interior, None, n_cos, n_phi, 0, 2, with_delta_tab=True)
    assert np.array_equal(codes, rc)
    assert np.array_equal(tau, rt)


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("name", ["capi2", "bench5", "confY", "cfg1_damped"])
def test_spectrum_vs_golden(gpu_available, name, kernel):
    p = golden_cases()[name]
    g = make_flow(p["interior"], p["exterior"], int(p["n_cos"]), int(p["n_phi"]), p["coeffs"], p["powers"],
                  float(p["damping"]), kernel=kernel)
    out = g.compute_c_integral(p["w"], t_begin=float(p["t_begin"]), t_end=float(p["t_end"]), n_t=int(p["n_t"]))
    assert out.shape == p["out"].shape and out.dtype == np.complex128
    check(kernel, out, p["out"], name)


def test_capi_case_matches_reference_test_shape(gpu_available):
    # rust/c-bubble-gw/tests/c_api.rs:135-218 through the reference-named C ABI
    p = golden_cases()["capi2"]
    g = make_flow(p["interior"], p["exterior"], 4, 5, [[0.0], [1.0]], [[3.0], [3.0]])
    out = g.compute_c_integral([0.5, 1.0], t_begin=0.0, t_end=8.0, n_t=40)
    np.testing.assert_allclose(out, p["out"], rtol=1e-10, atol=1e-10)


def test_selected_duplicates_and_late_bubbles(gpu_available):
    c = W.config(1)
    interior, ext = c.interior, c.exterior
    t_end = float(np.median(interior[:, 0]))  # half of the bubbles nucleate after t_end
    late = np.flatnonzero(interior[:, 0] > t_end)
    early = np.flatnonzero(interior[:, 0] < t_end)
    g = make_flow(interior, ext, 12, 14, [[1.0]], [[5.0]])
    sel = np.array([early[0], late[0], early[0], early[1]])
    out = g.compute_c_integral(c.w, t_begin=0.0, t_end=t_end, n_t=64, selected_bubbles=sel)
    ref = O.compute_c_integral(interior, ext, 12, 14, c.w, t_end, 64, t_begin=0.0, coefficients=[[1.0]],
                               powers=[[5.0]], selected=sel)
    only_late = g.compute_c_integral(c.w, t_begin=0.0, t_end=t_end, n_t=64, selected_bubbles=late)
    assert not only_late.any()
    assert err_per_w(out, ref) < FP64_TOL


@pytest.mark.parametrize("kernel", KERNELS)
def test_exponential_cutoff_and_t_begin(gpu_available, kernel):
    c = W.config(1)
    g = make_flow(c.interior, c.exterior, 16, 16, [[1.0], [0.5]], [[5.0], [2.5]], kernel=kernel)
    cut = mb.ExponentialTimeCutoff(1.5, 0.6, 0.3)
    out = g.compute_c_integral(c.w, t_begin=0.05, t_end=1.5, n_t=96, time_cutoff=cut)
    ref = O.compute_c_integral(c.interior, c.exterior, 16, 16, c.w, 1.5, 96, t_begin=0.05,
                               coefficients=[[1.0], [0.5]], powers=[[5.0], [2.5]], cutoff=(1.5, 0.6, 0.3))
    check(kernel, out, ref, "cutoff")


@pytest.mark.parametrize("kernel", KERNELS)
def test_config1_all_khat(gpu_available, kernel):
    c = W.config(1)
    g = make_flow(c.interior, c.exterior, c.n_cos, c.n_phi, c.coefficients, c.powers, kernel=kernel)
    out = g.compute_c_integral_khat(c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=c.n_t)
    ref = O.compute_c_integral_khat(c.interior, c.exterior, c.khat, c.n_cos, c.n_phi, c.w, c.t_begin, c.t_end,
                                    c.n_t, coefficients=c.coefficients, powers=c.powers)
    assert out.shape == (16, 2, 1, 32)
    check(kernel, out, ref, "config1")


@pytest.mark.parametrize("kernel", KERNELS)
def test_config2_subset(gpu_available, kernel):
    """Config 2 geometry (512 bubbles, 3584 with images, 128x128 patches, T=512, W=128),
    a slice of radiating bubbles: with all colliders present, any subset of
    radiators is an exact partial sum (generalized_bulk_flow.rs:953-981)."""
    c = W.config(2)
    sel = np.arange(0, 512, 97)
    g = make_flow(c.interior, c.exterior, c.n_cos, c.n_phi, c.coefficients, c.powers, kernel=kernel)
    kh = c.khat[[0, 17]]
    out = g.compute_c_integral_khat(c.w, kh, t_begin=0.0, t_end=c.t_end, n_t=c.n_t, selected_bubbles=sel)
    ref = np.zeros_like(out)
    for q, k in enumerate(kh):
        R = O.rotation_for_khat(k)
        ri, re = O.rotate(R, c.interior), O.rotate(R, c.exterior)
        ref[q] = O.compute_c_integral(ri, re, c.n_cos, c.n_phi, c.w, c.t_end, c.n_t, t_begin=0.0,
                                      coefficients=c.coefficients, powers=c.powers, selected=sel)
    check(kernel, out, ref, "config2 subset")


@pytest.mark.parametrize("kernel", ["fp64_factored", "mixed"])
def test_dense_collision_blocks(gpu_available, kernel):
    """Config 2 geometry with 192 phi patches and 1056 steps (33 blocks of 32): a row's
    collisions crowd into a few step blocks with more than 32 events each, the case
    in which k_beta sums each step's events by match groups."""
    c = W.config(2)
    sel = np.array([5, 300])
    n_cos, n_phi, n_t, w = 16, 192, 1056, c.w[::16]
    g = make_flow(c.interior, c.exterior, n_cos, n_phi, c.coefficients, c.powers, kernel=kernel)
    out = g.compute_c_integral(w, t_begin=0.0, t_end=c.t_end, n_t=n_t, selected_bubbles=sel)
    ref = O.compute_c_integral(c.interior, c.exterior, n_cos, n_phi, w, c.t_end, n_t, t_begin=0.0,
                               coefficients=c.coefficients, powers=c.powers, selected=sel)
    # the case under test occurs: some row has a 32-step block holding more than 32 collisions
    codes, tau = O.first_colliding(c.interior, c.exterior, n_cos, n_phi, 5, 6, with_delta_tab=True)
    t_arr = np.linspace(0.0, c.t_end, n_t)
    ta = c.interior[5, 0]
    k = np.searchsorted(t_arr - ta, tau[0], side="left")
    busiest = max(np.bincount(k[i][(tau[0][i] > 0) & (k[i] < n_t)] // 32, minlength=33).max() for i in range(n_cos))
    assert busiest > 32
    check(kernel, out, ref, "dense collision blocks")


def test_python_fixed_bubble_and_masks(gpu_available):
    p = golden_cases()["bench5"]
    g = make_flow(p["interior"], p["exterior"], int(p["n_cos"]), int(p["n_phi"]), p["coeffs"], p["powers"])
    one = g.compute_c_integral_fixed_bubble(2, p["w"], 0.0, 15.0, 200)
    ref = O.compute_c_integral(p["interior"], p["exterior"], int(p["n_cos"]), int(p["n_phi"]), p["w"], 15.0, 200,
                               t_begin=0.0, coefficients=p["coeffs"], powers=p["powers"], selected=[2])
    assert err_per_w(one, ref) < FP64_TOL
    with pytest.raises(IndexError):
        g.compute_c_integral_fixed_bubble(9, p["w"], 0.0, 15.0, 200)


def test_config3_slice_per_w(gpu_available):
    """Config 3 geometry (4096 bubbles, 28672 colliders with images, 192x192 patches, T = 1024,
    256 w): 64 radiating bubbles spread over nucleation order with every collider present (an
    exact partial sum, generalized_bulk_flow.rs:953-981), 2 k-hat, every w.
    mixed vs fp64_factored <= 1e-6 per w; fp64_factored vs fp64_direct <= 1e-10 per w;
    fp64_direct vs the oracle on one radiating bubble <= 1e-12 per w."""
    c = W.config(3, k_subset=2)
    sel = np.arange(0, c.n, 64)
    out = {}
    for kernel in ("fp64_direct", "fp64_factored", "mixed"):
        g = make_flow(c.interior, c.exterior, c.n_cos, c.n_phi, c.coefficients, c.powers, kernel=kernel)
        out[kernel] = g.compute_c_integral_khat(c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=c.n_t,
                                                selected_bubbles=sel)
    e_mixed = err_per_w(out["mixed"], out["fp64_factored"])
    e_fact = err_per_w(out["fp64_factored"], out["fp64_direct"])
    print(f"config3 slice: mixed vs fp64_factored per-w {e_mixed:.3e}; fp64_factored vs fp64_direct {e_fact:.3e}")
    assert e_mixed < MIXED_TOL
    assert e_fact < FACTORED_PER_W_TOL
    # one radiating bubble, first k-hat, against the oracle
    a = int(sel[3])
    g = make_flow(c.interior, c.exterior, c.n_cos, c.n_phi, c.coefficients, c.powers, kernel="fp64_direct")
    one = g.compute_c_integral_khat(c.w, c.khat[:1], t_begin=c.t_begin, t_end=c.t_end, n_t=c.n_t,
                                    selected_bubbles=[a])
    R = O.rotation_for_khat(c.khat[0])
    ref = O.compute_c_integral(O.rotate(R, c.interior), O.rotate(R, c.exterior), c.n_cos, c.n_phi, c.w, c.t_end,
                               c.n_t, t_begin=c.t_begin, coefficients=c.coefficients, powers=c.powers, selected=[a])
    check("fp64_direct", one[0], ref, "config3 one bubble")
