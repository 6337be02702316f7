"""Pins the oracle (CPU f64 restatement of the reference) with known answers.

No reference-produced numbers exist for this path (the Rust crate cannot be
built here and rust/bubble-gw/tests/envelope_2bubbles_scan=n_phix.csv is not
in the snapshot), so the oracle is pinned by:
  * closed-form masks/delays of the reference's two-bubble test geometry
    (rust/c-bubble-gw/tests/c_api.rs:137-141);
  * invariances of the discretised spectrum that hold exactly or to rounding
    (isolated bubble, azimuthal grid rotation, time and z translation,
    power-of-two scaling, linearity in the coefficient sets);
  * an independent vectorised numpy evaluation of the same discretised sums.
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from gw_fopt_b200 import workloads as W

CAPI2 = np.array([[0.0, 0.0, 10.0, 0.0], [0.0, 0.0, 0.0, 0.0]])
BENCH5 = np.array([[0.0, 0.0, 10.0, 0.0], [0.0, 0.0, 0.0, 0.0], [0.0, 4.0, 0.0, 4.0], [0.0, 4.0, 2.0, 4.0],
                   [0.0, 0.0, 2.0, 1.0]])


def rel_err(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def test_two_bubble_masks_closed_form():
    # bubble 0 at y=10, bubble 1 at the origin, both t=0: bubble 1 is first along
    # directions with sin(theta) sin(phi) < 0 and tau = 5 / (sin(theta) |sin(phi)|)
    n_cos, n_phi = 9, 13
    codes, tau = O.first_colliding(CAPI2, None, n_cos, n_phi, with_delta_tab=True)
    dirs = O.directions(n_cos, n_phi)
    sy = dirs[..., 1]
    exp0 = np.where(-10.0 * sy > 1e-10, 1, -1)
    exp1 = np.where(10.0 * sy > 1e-10, 0, -1)
    assert np.array_equal(codes[0], exp0)
    assert np.array_equal(codes[1], exp1)
    m0 = codes[0] == 1
    np.testing.assert_allclose(tau[0][m0], 5.0 / np.abs(sy[m0]), rtol=1e-14)
    assert np.all(tau[0][~m0] == 0.0)


def test_isolated_bubble_is_zero():
    out = O.compute_c_integral(np.array([[0.1, 0.2, 0.3, 0.4]]), None, 16, 17, [1.0, 10.0, 100.0], 3.0, 50)
    assert np.abs(out).max() < 1e-14


def test_power_of_two_scaling_is_exact():
    w = np.geomspace(0.1, 10.0, 5)
    a = O.compute_c_integral(BENCH5, None, 8, 11, w, 15.0, 40, t_begin=0.0, coefficients=[[0.0], [1.0]],
                             powers=[[3.0], [3.0]])
    b2 = BENCH5 * 2.0
    b = O.compute_c_integral(b2, None, 8, 11, w / 2.0, 30.0, 40, t_begin=0.0, coefficients=[[0.0], [1.0]],
                             powers=[[3.0], [3.0]])
    assert np.array_equal(b, 16.0 * a)


def test_time_translation_phase():
    w = np.geomspace(0.1, 5.0, 6)
    s = 0.375
    a = O.compute_c_integral(BENCH5, None, 8, 11, w, 15.0, 60, t_begin=0.0)
    shifted = BENCH5.copy()
    shifted[:, 0] += s
    b = O.compute_c_integral(shifted, None, 8, 11, w, 15.0 + s, 60, t_begin=s)
    assert rel_err(b, a * np.exp(1j * w * s)[None, None, :]) < 1e-12


def test_z_and_xy_translation():
    w = np.geomspace(0.1, 5.0, 6)
    a = O.compute_c_integral(BENCH5, None, 8, 11, w, 15.0, 60, t_begin=0.0)
    dz = BENCH5.copy()
    dz[:, 3] += 0.75
    b = O.compute_c_integral(dz, None, 8, 11, w, 15.0, 60, t_begin=0.0)
    assert rel_err(b, a * np.exp(-1j * w * 0.75)[None, None, :]) < 1e-12
    dxy = BENCH5.copy()
    dxy[:, 1] += 0.5
    dxy[:, 2] -= 0.25
    c = O.compute_c_integral(dxy, None, 8, 11, w, 15.0, 60, t_begin=0.0)
    assert rel_err(c, a) < 1e-12


def test_azimuthal_grid_rotation():
    n_phi = 13
    m = 3
    alpha = 2.0 * math.pi * m / (n_phi - 1)
    w = np.geomspace(0.1, 5.0, 5)
    a = O.compute_c_integral(BENCH5, None, 9, n_phi, w, 15.0, 50, t_begin=0.0)
    ca, sa = math.cos(alpha), math.sin(alpha)
    rot = BENCH5.copy()
    rot[:, 1] = ca * BENCH5[:, 1] - sa * BENCH5[:, 2]
    rot[:, 2] = sa * BENCH5[:, 1] + ca * BENCH5[:, 2]
    b = O.compute_c_integral(rot, None, 9, n_phi, w, 15.0, 50, t_begin=0.0)
    c2, s2 = math.cos(2 * alpha), math.sin(2 * alpha)
    exp_plus = c2 * a[0] - s2 * a[1]
    exp_cross = s2 * a[0] + c2 * a[1]
    assert rel_err(b[0], exp_plus) < 1e-10
    assert rel_err(b[1], exp_cross) < 1e-10


def test_linearity_in_coefficients():
    w = np.geomspace(0.1, 5.0, 5)
    out = O.compute_c_integral(BENCH5, None, 8, 11, w, 15.0, 40, t_begin=0.0,
                               coefficients=[[0.3], [0.7], [1.0]], powers=[[4.0], [4.0], [4.0]])
    env = O.compute_c_integral(BENCH5, None, 8, 11, w, 15.0, 40, t_begin=0.0, coefficients=[[0.0]],
                               powers=[[4.0]])
    # C(a) = C(0) + a * (C(1) - C(0)) since f is affine in a for collided patches
    lin = env[:, 0] + 0.3 * (out[:, 2] - env[:, 0])
    assert rel_err(out[:, 0], lin) < 1e-12
    assert rel_err(out[:, 0] + out[:, 1] - env[:, 0], out[:, 2]) < 1e-12


def _numpy_spectrum(interior, exterior, n_cos, n_phi, w, t_begin, t_end, n_t, coeffs, powers):
    """Vectorised evaluation of the discretised sums of generalized_bulk_flow.rs:481-984."""
    allb = np.concatenate([interior, exterior])
    n_int = interior.shape[0]
    cos_t = np.array([-1.0 + (2.0 / (n_cos - 1)) * i for i in range(n_cos)])
    phi = np.array([0.0 + (2.0 * math.pi / (n_phi - 1)) * j for j in range(n_phi)])
    codes, tau = O.first_colliding(interior, exterior, n_cos, n_phi, with_delta_tab=True)
    t = np.array([t_begin + ((t_end - t_begin) / (n_t - 1)) * k for k in range(n_t)])
    dt = t[1] - t[0]
    wphi = np.ones(n_phi)
    wphi[[0, -1]] = 0.5
    wcos = np.ones(n_cos)
    wcos[[0, -1]] = 0.5
    wt = np.ones(n_t)
    wt[[0, -1]] = 0.5
    dphi = 2.0 * math.pi / n_phi
    dcos = 2.0 / (n_cos - 1)
    S = len(coeffs)
    out = np.zeros((2, S, len(w)), dtype=complex)
    for a in range(n_int):
        ta, za = interior[a, 0], interior[a, 3]
        for k in range(n_t):
            if not (ta <= t[k]):
                continue
            d = t[k] - ta
            if d <= 0:
                continue
            coll = (tau[a] > 0) & (d >= tau[a])
            for s in range(S):
                r = np.where(coll, tau[a] / d, 0.0)
                f = np.where(coll, sum(c * r ** p for c, p in zip(coeffs[s], powers[s])), 1.0)
                bp = 0.5 * (1 - cos_t ** 2) * (f * np.cos(2 * phi) * wphi).sum(1) * dphi * d ** 3
                bm = 0.5 * (1 - cos_t ** 2) * (f * np.sin(2 * phi) * wphi).sum(1) * dphi * d ** 3
                ph = np.exp(-1j * np.outer(w, d * cos_t)) * dcos * wcos
                A_p = ph @ bp
                A_m = ph @ bm
                fac = np.exp(1j * w * (t[k] - za)) * wt[k] * dt / (6 * math.pi)
                out[0, s] += A_p * fac
                out[1, s] += A_m * fac
    return out


@pytest.mark.parametrize("case", ["bench5", "config1"])
def test_oracle_matches_numpy_restatement(case):
    if case == "bench5":
        interior, exterior = BENCH5, np.zeros((0, 4))
        args = dict(n_cos=7, n_phi=10, w=np.geomspace(1e-2, 1e2, 7), t_begin=0.0, t_end=15.0, n_t=30)
        co, po = [[0.0], [1.0]], [[3.0], [3.0]]
    else:
        c = W.config(1)
        interior, exterior = c.interior, c.exterior
        args = dict(n_cos=8, n_phi=9, w=c.w[::4], t_begin=0.0, t_end=1.5, n_t=24)
        co, po = [[1.0]], [[5.0]]
    ref = _numpy_spectrum(interior, exterior, coeffs=co, powers=po, **args)
    got = O.compute_c_integral(interior, exterior, args["n_cos"], args["n_phi"], args["w"], args["t_end"],
                               args["n_t"], t_begin=args["t_begin"], coefficients=co, powers=po)
    assert rel_err(got, ref) < 1e-11


def test_rotation_convention():
    R = O.rotation_for_khat([0.0, 0.0, 1.0])
    assert np.array_equal(R, np.eye(3))
    R = O.rotation_for_khat([0.0, 0.0, -1.0])
    assert np.array_equal(R, np.diag([1.0, -1.0, -1.0]))
    for k in W.fibonacci_khat(7):
        R = O.rotation_for_khat(k)
        np.testing.assert_allclose(R @ k, [0, 0, 1], atol=1e-14)
        np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-14)
        assert np.linalg.det(R) > 0


def test_exponential_cutoff():
    t = np.linspace(0.0, 2.0, 9)
    out = O.time_cutoff(t, 1.5, 0.5, 0.25)
    t_cut, t_0 = 0.75, 0.25 * (1.5 - 0.75)
    exp = np.where(t < t_cut, 1.0, np.exp(-((t - t_cut) ** 2) / t_0 ** 2))
    np.testing.assert_allclose(out, exp, rtol=1e-15)


def test_validation():
    O.validate(BENCH5)
    with pytest.raises(O.OracleError, match="formed inside bubble"):
        O.validate(np.array([[0.0, 0, 0, 0], [1.0, 0.5, 0, 0]]))


def test_golden_fixtures_reproduce():
    """The committed golden fixtures were produced by this oracle (tests/golden/make_golden.py)."""
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "golden_small.npz")
    g = np.load(path, allow_pickle=False)
    names = [k[:-len("__out")] for k in g.files if k.endswith("__out")]
    assert names
    for name in names:
        p = {k.split("__", 1)[1]: g[k] for k in g.files if k.startswith(name + "__")}
        out = O.compute_c_integral(p["interior"], p["exterior"], int(p["n_cos"]), int(p["n_phi"]), p["w"],
                                   float(p["t_end"]), int(p["n_t"]), t_begin=float(p["t_begin"]),
                                   coefficients=p["coeffs"], powers=p["powers"],
                                   damping=None if np.isnan(p["damping"]) else float(p["damping"]))
        assert np.array_equal(out, p["out"]), name
        codes = O.first_colliding(p["interior"], p["exterior"], int(p["n_cos"]), int(p["n_phi"]))
        assert np.array_equal(codes, p["codes"]), name


def test_integrand_sums_to_integral():
    """compute_c_integrand summed over t equals compute_c_integral without a time cutoff
    (generalized_bulk_flow.rs:776-866 against :775-873)."""
    c = W.config(1)
    kw = dict(t_begin=0.0, coefficients=[[1.0], [0.5]], powers=[[5.0], [3.0]], damping=0.7)
    it = O.compute_c_integrand(c.interior, c.exterior, 10, 12, c.w[:5], 1.5, 33, **kw)
    ci = O.compute_c_integral(c.interior, c.exterior, 10, 12, c.w[:5], 1.5, 33, **kw)
    assert it.shape == (2, 2, 5, 33)
    assert np.abs(it.sum(-1) - ci).max() <= 1e-13 * np.abs(ci).max()
    tn = c.interior[:, 0]
    t = np.linspace(0.0, 1.5, 33)
    one = O.compute_c_integrand(c.interior, c.exterior, 10, 12, c.w[:5], 1.5, 33, selected=[2], **kw)
    assert not one[..., t <= tn[2]].any()
