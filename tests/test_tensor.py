"""The tensor form (the reference's NewGeneralizedBulkFlow, new_generalized_bulk_flow.rs):
C_ij in six components, plain FP64 on the GPU against the oracle's restatement
(oracle/bgw_oracle.cpp: b_tensor, c_tensor_increment) to 1e-12 relative per w,
and against the scalar form: C_+ = (C_xx - C_yy)/2 and C_x = C_xy hold exactly in
exact arithmetic (the tensor's phi basis cos^2, sin^2 against the scalar's cos 2phi).
"""
import numpy as np
import pytest

from oracle import oracle as O
from gw_fopt_b200 import many_bubbles as mb
from gw_fopt_b200 import workloads as W

TOL = 1e-12


def err_per_w(got, ref):
    g = got.reshape(-1, got.shape[-1])
    r = ref.reshape(-1, ref.shape[-1])
    num = np.linalg.norm(g - r, axis=0)
    den = np.linalg.norm(r, axis=0)
    return float(np.max(num / np.maximum(den, 1e-300 + 1e-13 * np.linalg.norm(r))))


def test_oracle_tensor_reduces_to_scalar_form():
    c = W.config(1)
    coeffs, powers = [[1.0], [0.5]], [[5.0], [2.5]]
    T = O.compute_c_tensor(c.interior, c.exterior, 12, 10, c.w, 1.5, 40, coefficients=coeffs, powers=powers,
                           damping=0.7)
    S = O.compute_c_integral(c.interior, c.exterior, 12, 10, c.w, 1.5, 40, coefficients=coeffs, powers=powers,
                             damping=0.7)
    assert err_per_w(0.5 * (T[0] - T[3]), S[0]) < 1e-12
    assert err_per_w(T[1], S[1]) < 1e-12


def test_tt_energy_along_z_is_twice_the_polarisation_power():
    rng = np.random.default_rng(3)
    c = rng.normal(size=(6, 2, 7)) + 1j * rng.normal(size=(6, 2, 7))
    e = mb.tt_energy(c)
    assert np.allclose(e, 2 * (np.abs(0.5 * (c[0] - c[3])) ** 2 + np.abs(c[1]) ** 2), rtol=1e-14, atol=0)
    # rotational covariance: the energy along k of C equals that along z of R C R^T with R k = z
    k = np.array([0.3, -0.5, 0.81])
    k /= np.linalg.norm(k)
    R = O.rotation_for_khat(k)
    idx = [[0, 1, 2], [1, 3, 4], [2, 4, 5]]
    T = np.array([[c[idx[i][j]] for j in range(3)] for i in range(3)])
    Tr = np.einsum("ai,bj,ij...->ab...", R, R, T)
    cr = np.stack([Tr[0, 0], Tr[0, 1], Tr[0, 2], Tr[1, 1], Tr[1, 2], Tr[2, 2]])
    assert np.allclose(mb.tt_energy(c, k), mb.tt_energy(cr), rtol=1e-12, atol=0)


def make(c, coeffs, powers, damping=None, n_cos=16, n_phi=16):
    g = mb.NewGeneralizedBulkFlow(mb.LatticeBubbles(mb.EmptyLattice(), c.interior, c.exterior))
    g.set_resolution(n_cos, n_phi)
    g.set_gradient_scaling_params(coeffs, powers, damping)
    return g


@pytest.mark.gpu
def test_gpu_tensor_matches_oracle(gpu_available):
    c = W.config(1)
    for coeffs, powers, damping in (([[1.0]], [[5.0]], None), ([[1.0], [0.5]], [[5.0], [2.5]], 0.7)):
        g = make(c, coeffs, powers, damping)
        got = g.compute_c_tensor(c.w, t_end=1.5, n_t=64)
        ref = O.compute_c_tensor(c.interior, c.exterior, 16, 16, c.w, 1.5, 64, coefficients=coeffs, powers=powers,
                                 damping=damping)
        assert got.shape == ref.shape == (6, len(coeffs), c.w.size)
        assert err_per_w(got, ref) < TOL
        one = g.compute_c_tensor_fixed_bubble(3, c.w, 0.05, 1.5, 64)
        ref1 = O.compute_c_tensor(c.interior, c.exterior, 16, 16, c.w, 1.5, 64, t_begin=0.05, coefficients=coeffs,
                                  powers=powers, damping=damping, selected=[3])
        assert err_per_w(one, ref1) < TOL


@pytest.mark.gpu
def test_gpu_tensor_khat_and_scalar_consistency(gpu_available):
    c = W.config(1)
    g = make(c, [[1.0]], [[5.0]])
    kh = c.khat[:3]
    got = g.compute_c_tensor_khat(c.w, kh, t_end=1.5, n_t=48)
    ref = O.compute_c_tensor_khat(c.interior, c.exterior, kh, 16, 16, c.w, 1.5, 48, coefficients=[[1.0]],
                                  powers=[[5.0]])
    assert err_per_w(got, ref) < TOL
    s = mb.GeneralizedBulkFlow(mb.LatticeBubbles(mb.EmptyLattice(), c.interior, c.exterior))
    s.set_resolution(16, 16)
    s.set_gradient_scaling_params([[1.0]], [[5.0]])
    sc = s.compute_c_integral_khat(c.w, kh, t_begin=0.0, t_end=1.5, n_t=48)
    assert err_per_w(0.5 * (got[:, 0] - got[:, 3]), sc[:, 0]) < TOL
    assert err_per_w(got[:, 1], sc[:, 1]) < TOL
    assert np.array_equal(g.compute_c_tensor(c.w, t_end=1.5, n_t=48, selected_bubbles=np.array([], dtype=int)),
                          np.zeros((6, 1, c.w.size), dtype=complex))


@pytest.mark.gpu
def test_gpu_tensor_integrand_sums_to_the_tensor(gpu_available):
    c = W.config(1)
    g = make(c, [[1.0], [0.5]], [[5.0], [2.5]], 0.7)
    tot = g.compute_c_tensor(c.w, t_end=1.5, n_t=40)
    integ = g.compute_c_tensor_integrand(c.w, t_end=1.5, n_t=40)
    assert integ.shape == (6, 2, c.w.size, 40)
    assert err_per_w(integ.sum(axis=-1), tot) < TOL
    one = g.compute_c_tensor_integrand_fixed_bubble(2, c.w, None, 1.5, 40)
    ref1 = O.compute_c_tensor(c.interior, c.exterior, 16, 16, c.w, 1.5, 40, coefficients=[[1.0], [0.5]],
                              powers=[[5.0], [2.5]], damping=0.7, selected=[2])
    assert err_per_w(one.sum(axis=-1), ref1) < TOL
