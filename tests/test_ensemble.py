"""Batched ensemble (BulkFlowEnsemble / bgwx_generalized_bulk_flow_compute_ensemble_khat).

Each realization's block must be bit-identical to the single-configuration
k-hat call on that realization alone, and agree with the oracle (per
realization, per k-hat: compute_c_integral on the rotated configuration) to
the kernel's tolerance.  Host-side argument checks run without a GPU.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from gw_fopt_b200 import _lib as L
from gw_fopt_b200 import many_bubbles as mb
from gw_fopt_b200 import workloads as W
from gw_fopt_b200.ensemble import BulkFlowEnsemble, ensemble_mean_power

from test_gpu_parity import KERNELS, check, err_per_w, make_flow


def small_ensemble(n_real=4, seed=11):
    return W.ensemble(n_real=n_real, seed=seed, n_min=4, n_max=14, beta_lo=5.0, beta_hi=15.0)


def test_rejects_acausal_realization():
    reals = small_ensemble(2)
    bad_i = np.array([[0.0, 0.5, 0.5, 0.5], [0.5, 0.6, 0.5, 0.5]])  # second bubble nucleates inside the first
    ens = BulkFlowEnsemble(reals + [(bad_i, np.zeros((0, 4)))])
    ens.set_resolution(8, 8)
    with pytest.raises(ValueError):
        ens.compute_c_integral_khat([1.0, 2.0], [[0.0, 0.0, 1.0]], t_end=1.0, n_t=8)


def test_offsets_and_length_checks():
    h = C.c_void_p()
    L.check(L.lib().bgwx_generalized_bulk_flow_new_unchecked(C.byref(h), None, 0, None, 0))
    try:
        L.check(L.lib().bgw_generalized_bulk_flow_set_resolution(h, 4, 4, False))
        inter = np.zeros((3, 4))
        ext = np.zeros((0, 4))
        szp = C.POINTER(C.c_size_t)
        w = np.array([1.0])
        kh = np.array([0.0, 0.0, 1.0])
        out = (L.BgwComplex64 * 4)()
        cut = L.BgwTimeCutoffConfig(0, 0.0, float("nan"), float("nan"))

        def call(io, eo, n_real, out_len):
            io = np.asarray(io, dtype=np.uintp)
            eo = np.asarray(eo, dtype=np.uintp)
            return L.lib().bgwx_generalized_bulk_flow_compute_ensemble_khat(
                h, L.ptr(inter), io.ctypes.data_as(szp), L.ptr(ext), eo.ctypes.data_as(szp), n_real, False,
                L.ptr(w), 1, False, 0.0, 1.0, 8, L.ptr(kh), 1, cut, out, out_len)

        assert call([0, 2, 1], [0, 0, 0], 2, 4) == 3
        assert b"non-decreasing" in L.lib().bgw_last_error_message()
        assert call([1, 2, 3], [0, 0, 0], 2, 4) == 3
        assert b"start at 0" in L.lib().bgw_last_error_message()
        assert call([0, 1, 3], [0, 0, 0], 2, 3) == 3
        assert b"out_len=3" in L.lib().bgw_last_error_message()
    finally:
        L.lib().bgw_generalized_bulk_flow_free(h)


def test_mean_power():
    c = np.array([[[1 + 1j]], [[3 + 0j]]])
    assert np.allclose(ensemble_mean_power(c), [[5.5]])


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", KERNELS)
def test_ensemble_matches_single_and_oracle(gpu_available, kernel):
    reals = small_ensemble(4)
    reals.append((np.zeros((0, 4)), np.zeros((0, 4))))  # an empty realization yields zeros
    n_cos, n_phi, n_t = 12, 10, 48
    w = np.geomspace(1.0, 300.0, 12)
    kh = W.fibonacci_khat(3)
    co, po = [[1.0], [0.5]], [[5.0], [3.5]]
    ens = BulkFlowEnsemble(reals)
    ens.set_resolution(n_cos, n_phi)
    ens.set_gradient_scaling_params(co, po)
    ens.set_kernel(kernel)
    out = ens.compute_c_integral_khat(w, kh, t_end=1.5, n_t=n_t)
    assert out.shape == (5, 3, 2, 2, 12)
    assert not out[4].any()
    for r, (inter, ext) in enumerate(reals[:4]):
        g = make_flow(inter, ext, n_cos, n_phi, co, po, kernel=kernel)
        single = g.compute_c_integral_khat(w, kh, t_end=1.5, n_t=n_t)
        assert np.array_equal(out[r], single), r
        ref = O.compute_c_integral_khat(inter, ext, kh, n_cos, n_phi, w, 0.0, 1.5, n_t, coefficients=co,
                                        powers=po)
        check(kernel, out[r], ref, f"ensemble r={r}")
    t = ens.last_timings()
    assert t["total_ms"] > 0 and t["launches"] > 0


@pytest.mark.gpu
def test_config4_realizations_per_w(gpu_available):
    """Config 4 (the batched-ensemble workload: N_r ~ U{50..800}, beta_r L ~ U[5, 15], 96x96 patches,
    T = 384, 128 w): its largest and smallest realizations and two others in one ensemble call on
    2 k-hat, mixed against fp64_factored per realization, <= 1e-6 per w."""
    c = W.ensemble_config(k_subset=2)
    sizes = [inter.shape[0] for inter, _ in c.realizations]
    pick = sorted({int(np.argmax(sizes)), int(np.argmin(sizes)), 0, 100})
    reals = [c.realizations[r] for r in pick]
    out = {}
    for kernel in ("mixed", "fp64_factored"):
        ens = BulkFlowEnsemble(reals, validate=False)
        ens.set_resolution(c.n_cos, c.n_phi)
        ens.set_gradient_scaling_params(c.coefficients.tolist(), c.powers.tolist())
        ens.set_kernel(kernel)
        out[kernel] = ens.compute_c_integral_khat(c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=c.n_t)
    for q, r in enumerate(pick):
        e = err_per_w(out["mixed"][q], out["fp64_factored"][q])
        print(f"config4 realization {r} ({sizes[r]} bubbles): mixed vs fp64_factored per-w {e:.3e}")
        assert e < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["mixed", "fp64_factored"])
def test_batched_multi_tile_realizations_bitwise(gpu_available, kernel):
    """Realizations of more than one GEMM column tile (70 and 150 radiating bubbles, the column
    tiles padded per realization) next to a 3-bubble one, in one batched call: every realization's
    block equals its own single-configuration call bit for bit when both use the same cos-theta row
    split, and the masks of each realization see only its own colliders."""
    reals = [W.exponential_nucleation(70, 9.0, seed=5), W.exponential_nucleation(3, 6.0, seed=6),
             W.exponential_nucleation(150, 12.0, seed=7)]
    n_cos, n_phi, n_t = 24, 16, 96
    w = np.geomspace(1.0, 500.0, 10)
    kh = W.fibonacci_khat(2)
    co, po = [[1.0]], [[5.0]]
    ens = BulkFlowEnsemble(reals, validate=False)
    ens.set_resolution(n_cos, n_phi)
    ens.set_gradient_scaling_params(co, po)
    ens.set_kernel(kernel)
    L.check(L.lib().bgwx_generalized_bulk_flow_set_launch_shape(ens._h, 1, 2))
    out = ens.compute_c_integral_khat(w, kh, t_end=1.5, n_t=n_t)
    for r, (inter, ext) in enumerate(reals):
        g = make_flow(inter, ext, n_cos, n_phi, co, po, kernel=kernel)
        g.set_launch_shape(2, 2)
        single = g.compute_c_integral_khat(w, kh, t_end=1.5, n_t=n_t)
        assert np.array_equal(out[r], single), r


@pytest.mark.gpu
def test_batched_graph_capture_and_replay(gpu_available):
    """The batched launch sequence runs eagerly on the first call of a problem shape, is captured
    into a CUDA graph by the second and replayed by later calls: all three give the same bits, and a
    replay with other realizations of the same sizes (uploaded before the graph is launched) equals
    their own eager calls."""
    def reals_for(seed):
        return [W.exponential_nucleation(n, 8.0, seed=seed + q) for q, n in enumerate((40, 9, 70))]

    n_cos, n_phi, n_t = 16, 12, 64
    w = np.geomspace(1.0, 300.0, 8)
    kh = W.fibonacci_khat(2)

    def make(reals):
        e = BulkFlowEnsemble(reals, validate=False)
        e.set_resolution(n_cos, n_phi)
        e.set_gradient_scaling_params([[1.0]], [[5.0]])
        e.set_kernel("mixed")
        return e

    first = reals_for(20)
    ens = make(first)
    outs, replays = [], []
    for _ in range(3):
        outs.append(ens.compute_c_integral_khat(w, kh, t_end=1.5, n_t=n_t))
        replays.append(ens.last_timings()["graph_replays"])
    assert replays == [0, 0, 1]
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    # same sizes, other bubbles (the ensemble's arrays rewritten in place): the handle's graph is
    # replayed on the new inputs
    second = reals_for(40)
    assert all(a.shape == a0.shape and b.shape == b0.shape for (a, b), (a0, b0) in zip(second, first))
    ref = make(second).compute_c_integral_khat(w, kh, t_end=1.5, n_t=n_t)
    ens._interior[...] = np.concatenate([a for a, _ in second])
    ens._exterior[...] = np.concatenate([b for _, b in second])
    got = ens.compute_c_integral_khat(w, kh, t_end=1.5, n_t=n_t)
    assert ens.last_timings()["graph_replays"] == 1
    assert np.array_equal(got, ref)
