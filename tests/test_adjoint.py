"""Adjoint of the spectrum (config-5 path): gradients with respect to the scaling
coefficients, their powers and the bubbles' nucleation events.

CPU: the oracle's FP64 adjoint (oracle/adjoint.py) against central finite
differences (h = 1e-6) of the oracle's forward spectrum, and the fit
parametrisation.  GPU: the library's adjoint kernels against the oracle's
adjoint, and the torch.autograd path against central finite differences of
the library's FP64 forward (agreement 1e-5).
"""
import numpy as np
import pytest
import torch

from oracle import adjoint as OA
from oracle import oracle as O
from gw_fopt_b200 import workloads as W

H = 1e-6
FD_TOL = 1e-5


def central_fd(fun, h=H):
    """Central difference at h, and whether it is free of a kink within 2h.

    The spectrum is piecewise smooth: a patch's collision status flips where
    dt_k crosses its delay tau, and the first collider changes where two
    bubbles' walls arrive together.  Across such a point the derivative jumps;
    a central difference that straddles one measures an average slope.  A
    difference at h that disagrees with the one at 2h marks such a point."""
    d1 = (fun(h) - fun(-h)) / (2 * h)
    d2 = (fun(2 * h) - fun(-2 * h)) / (4 * h)
    return d1, abs(d1 - d2) <= 1e-6 * max(abs(d1), abs(d2), 1e-300)


def small_case(seed=3, n=4):
    inter, ext = W.uniform_config(n, 1.0, 0.2, seed=seed)
    return dict(inter=inter, ext=ext, n_cos=8, n_phi=9, n_t=24, w=np.geomspace(1, 60, 5), kh=W.fibonacci_khat(2))


def oracle_loss(c, inter, co, po, G, damping):
    ext = W.periodic_images(inter, 1.0)
    C = O.compute_c_integral_khat(inter, ext, c["kh"], c["n_cos"], c["n_phi"], c["w"], 0.0, 1.5, c["n_t"],
                                  coefficients=co, powers=po, damping=damping)
    return float(np.real(np.sum(np.conj(G) * C)))


@pytest.mark.parametrize("damping", [None, 0.8])
def test_oracle_adjoint_vs_finite_differences(damping):
    c = small_case()
    rng = np.random.default_rng(0)
    co = np.array([[0.7, 0.3]])
    po = np.array([[5.0, 3.5]])
    G = rng.normal(size=(2, 2, 1, 5)) + 1j * rng.normal(size=(2, 2, 1, 5))
    gc, gp, gb = OA.spectrum_vjp(c["inter"], c["ext"], c["kh"], c["n_cos"], c["n_phi"], c["w"], 0.0, 1.5,
                                 c["n_t"], G, co, po, damping=damping)
    n = c["inter"].shape[0]
    gi = gb[:n] + gb[n:].reshape(n, 6, 4).sum(1)
    for name, arr, an in [("co", co, gc), ("po", po, gp)]:
        for idx in [(0, 0), (0, 1)]:
            p, m = arr.copy(), arr.copy()
            p[idx] += H
            m[idx] -= H
            args_p = (p, po) if name == "co" else (co, p)
            args_m = (m, po) if name == "co" else (co, m)
            fd = (oracle_loss(c, c["inter"], *args_p, G, damping) - oracle_loss(c, c["inter"], *args_m, G, damping)) / (2 * H)
            assert abs(fd - an[idx]) <= FD_TOL * abs(fd), (name, idx, fd, an[idx])
    checked = 0
    for a in range(n):
        for q in range(4):
            def fun(h, a=a, q=q):
                x = c["inter"].copy()
                x[a, q] += h
                return oracle_loss(c, x, co, po, G, damping)
            fd, smooth = central_fd(fun)
            if not smooth:
                continue
            checked += 1
            assert abs(fd - gi[a, q]) <= FD_TOL * max(abs(fd), 1e-3 * np.abs(gi).max()), (a, q, fd, gi[a, q])
    assert checked >= 12


def test_fit_parametrisation_and_loss():
    from gw_fopt_b200.autograd import SurfaceTensionFit, log_power_residual
    fit = SurfaceTensionFit(xi=1.5, alpha=0.8, gamma=0.5, delta=0.2)
    co, po = fit()
    assert torch.allclose(co, torch.tensor([[0.8, 0.2]], dtype=torch.float64))
    assert torch.allclose(po, torch.tensor([[5.0, 4.5]], dtype=torch.float64))
    c = torch.randn(2, 2, 1, 3, 2, dtype=torch.float64, requires_grad=True)
    tgt = torch.rand(2, 1, 3, dtype=torch.float64) + 0.5
    loss = log_power_residual(c, tgt)
    loss.backward()
    assert c.grad is not None and torch.isfinite(c.grad).all()


def _library_model(c, kernel="fp64_factored", damping=None):
    from gw_fopt_b200.autograd import BulkFlowSpectrum
    return BulkFlowSpectrum(n_cos=c["n_cos"], n_phi=c["n_phi"], w=c["w"], khat=c["kh"], t_end=1.5, n_t=c["n_t"],
                            box=1.0, damping=damping, kernel=kernel)


@pytest.mark.gpu
@pytest.mark.parametrize("sets", [((0.7, 0.3), (5.0, 3.5)), ((1.0,), (5.0,))])
@pytest.mark.parametrize("damping", [None, 0.8])
def test_library_adjoint_vs_oracle(gpu_available, sets, damping):
    c = small_case(seed=5, n=6)
    c["n_cos"], c["n_phi"], c["n_t"] = 10, 12, 40
    co = np.array([sets[0]])
    po = np.array([sets[1]])
    if len(sets[0]) == 1:  # two coefficient sets of one term each
        co = np.array([[1.0], [0.4]])
        po = np.array([[5.0], [2.5]])
    S = co.shape[0]
    rng = np.random.default_rng(1)
    G = rng.normal(size=(2, 2, S, 5)) + 1j * rng.normal(size=(2, 2, S, 5))
    m = _library_model(c, damping=damping)
    gc, gp, gx = m.vjp(co, po, c["inter"], G)
    oc, op, ob = OA.spectrum_vjp(c["inter"], c["ext"], c["kh"], c["n_cos"], c["n_phi"], c["w"], 0.0, 1.5,
                                 c["n_t"], G, co, po, damping=damping)
    n = c["inter"].shape[0]
    ox = ob[:n] + ob[n:].reshape(n, 6, 4).sum(1)
    for got, ref in [(gc, oc), (gp, op), (gx, ox)]:
        assert np.allclose(got, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max()), (got, ref)


@pytest.mark.gpu
def test_autograd_vs_finite_differences(gpu_available):
    from gw_fopt_b200.autograd import SurfaceTensionFit, log_power_residual
    c = small_case(seed=7, n=8)
    c["n_cos"], c["n_phi"], c["n_t"] = 16, 16, 64
    c["w"] = np.geomspace(1.0, 200.0, 12)
    c["kh"] = W.fibonacci_khat(3)
    m = _library_model(c)
    fit = SurfaceTensionFit(xi=1.5, alpha=0.9, gamma=0.3, delta=0.1)
    x = torch.tensor(c["inter"], dtype=torch.float64, requires_grad=True)
    with torch.no_grad():
        co_t, po_t = SurfaceTensionFit(xi=2.0, alpha=1.0, gamma=0.0, delta=0.0)()
        target = (m(co_t, po_t, x) ** 2).sum(-1).sum(1) * 1.1
    co, po = fit()
    loss = log_power_residual(m(co, po, x), target)
    loss.backward()

    def f(xi=1.5, alpha=0.9, gamma=0.3, delta=0.1, xx=None):
        with torch.no_grad():
            cc, pp = SurfaceTensionFit(xi, alpha, gamma, delta)()
            return float(log_power_residual(m(cc, pp, x if xx is None else xx), target))

    base = dict(xi=1.5, alpha=0.9, gamma=0.3, delta=0.1)
    for name in base:
        p, q = dict(base), dict(base)
        p[name] += H
        q[name] -= H
        fd = (f(**p) - f(**q)) / (2 * H)
        an = float(getattr(fit, name).grad)
        assert abs(fd - an) <= FD_TOL * abs(fd), (name, fd, an)
    gx = x.grad.numpy()
    scale = np.abs(gx).max()
    checked = 0
    for a, q in [(0, 0), (1, 1), (2, 2), (3, 3), (4, 1), (5, 0), (6, 2), (7, 3)]:
        def fun(h, a=a, q=q):
            xx = x.detach().clone()
            xx[a, q] += h
            return f(xx=xx)
        fd, smooth = central_fd(fun)
        if not smooth:
            continue
        checked += 1
        assert abs(fd - gx[a, q]) <= FD_TOL * max(abs(fd), 1e-2 * scale), (a, q, fd, gx[a, q])
    assert checked >= 5


@pytest.mark.gpu
def test_config5_adjoint_vs_numpy_and_fd(gpu_available):
    """Config 5 (256 bubbles at beta L = 6 with periodic images, 64x64 patches, T = 256, 64 w) on its
    first k-hat: the library's FP64 adjoint against the numpy FP64 adjoint for the coefficients, the
    powers and every bubble row (1e-9), and the autograd path of the fit loss against central
    differences (h = 1e-6) of the library's FP64 forward for (xi, alpha, gamma, delta) and a sample of
    nucleation coordinates (1e-5)."""
    from gw_fopt_b200.autograd import BulkFlowSpectrum, SurfaceTensionFit, log_power_residual
    c = W.config(5, k_subset=1)
    n = c.interior.shape[0]
    model = BulkFlowSpectrum(n_cos=c.n_cos, n_phi=c.n_phi, w=c.w, khat=c.khat, t_end=c.t_end, n_t=c.n_t,
                             t_begin=c.t_begin, box=1.0, kernel="fp64_factored")
    rng = np.random.default_rng(5)
    G = rng.normal(size=(1, 2, 1, c.w.size)) + 1j * rng.normal(size=(1, 2, 1, c.w.size))
    gc, gp, gx = model.vjp(c.coefficients, c.powers, c.interior, G)
    oc, op, ob = OA.spectrum_vjp(c.interior, c.exterior, c.khat, c.n_cos, c.n_phi, c.w, c.t_begin, c.t_end,
                                 c.n_t, G, c.coefficients, c.powers)
    ox = ob[:n] + ob[n:].reshape(n, 6, 4).sum(1)
    for got, ref in [(gc, oc), (gp, op), (gx, ox)]:
        assert np.allclose(got, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())

    fit = SurfaceTensionFit(xi=1.5, alpha=1.0, gamma=0.0, delta=0.0)
    x = torch.tensor(c.interior, dtype=torch.float64, requires_grad=True)
    with torch.no_grad():
        co_t, po_t = SurfaceTensionFit(xi=2.0, alpha=1.1, gamma=0.4, delta=-0.1)()
        target = (model(co_t, po_t, x) ** 2).sum(-1).sum(1)
    co, po = fit()
    loss = log_power_residual(model(co, po, x), target)
    loss.backward()

    def f(xi=1.5, alpha=1.0, gamma=0.0, delta=0.0, xx=None):
        with torch.no_grad():
            cc, pp = SurfaceTensionFit(xi, alpha, gamma, delta)()
            return float(log_power_residual(model(cc, pp, x if xx is None else xx), target))

    base = dict(xi=1.5, alpha=1.0, gamma=0.0, delta=0.0)
    for name in base:
        p, q = dict(base), dict(base)
        p[name] += H
        q[name] -= H
        fd = (f(**p) - f(**q)) / (2 * H)
        an = float(getattr(fit, name).grad)
        assert abs(fd - an) <= FD_TOL * max(abs(fd), 1e-12), (name, fd, an)
    gxa = x.grad.numpy()
    scale = np.abs(gxa).max()
    checked = 0
    for a in range(3, n, 8):
        for q in range(4):
            def fun(h, a=a, q=q):
                xx = x.detach().clone()
                xx[a, q] += h
                return f(xx=xx)
            fd, smooth = central_fd(fun)
            if not smooth:
                continue
            checked += 1
            assert abs(fd - gxa[a, q]) <= FD_TOL * max(abs(fd), 1e-2 * scale), (a, q, fd, gxa[a, q])
    # 256 bubbles put kinks (collision-status flips) near most coordinates; enough stay smooth
    assert checked >= 8


@pytest.mark.gpu
def test_adjoint_bitwise_repeatable(gpu_available):
    """The bubble gradients are sums of many contributions accumulated by concurrent blocks; they
    are formed as fixed-point integer sums, so repeated calls give the same bits."""
    c = small_case(seed=9, n=8)
    c["n_cos"], c["n_phi"], c["n_t"] = 16, 16, 48
    c["kh"] = W.fibonacci_khat(4)
    m = _library_model(c)
    rng = np.random.default_rng(3)
    G = rng.normal(size=(4, 2, 1, 5)) + 1j * rng.normal(size=(4, 2, 1, 5))
    co, po = np.array([[0.7, 0.3]]), np.array([[5.0, 3.5]])
    first = m.vjp(co, po, c["inter"], G)
    for _ in range(3):
        again = m.vjp(co, po, c["inter"], G)
        for x, y in zip(first, again):
            assert np.array_equal(x, y)


@pytest.mark.gpu
def test_mixed_adjoint_vs_fp64_adjoint_and_fd(gpu_available):
    """With a mixed kernel the backward's products P and Q run in FP32 (folded into FP64 every 16
    frequencies): its gradients match the FP64 adjoint to 1e-5 (measured ~1e-7) for coefficients,
    powers and bubble rows, and the mixed autograd gradient of the fit loss matches central
    differences of the FP64 forward to 1e-5."""
    from gw_fopt_b200.autograd import SurfaceTensionFit, log_power_residual
    c = small_case(seed=7, n=8)
    c["n_cos"], c["n_phi"], c["n_t"] = 16, 16, 64
    c["w"] = np.geomspace(1.0, 200.0, 40)
    c["kh"] = W.fibonacci_khat(3)
    co = np.array([[1.0, 0.3]])
    po = np.array([[5.0, 3.5]])
    rng = np.random.default_rng(3)
    G = rng.normal(size=(3, 2, 1, 40)) + 1j * rng.normal(size=(3, 2, 1, 40))
    got = _library_model(c, kernel="mixed").vjp(co, po, c["inter"], G)
    ref = _library_model(c, kernel="fp64_factored").vjp(co, po, c["inter"], G)
    for g_, r_ in zip(got, ref):
        err = np.abs(g_ - r_).max() / np.abs(r_).max()
        print(f"mixed vs FP64 adjoint: {err:.2e}")
        assert err < 1e-5
    m = _library_model(c, kernel="mixed")
    m64 = _library_model(c, kernel="fp64_factored")
    x = torch.tensor(c["inter"], dtype=torch.float64, requires_grad=True)
    with torch.no_grad():
        co_t, po_t = SurfaceTensionFit(xi=2.0, alpha=1.0, gamma=0.0, delta=0.0)()
        target = (m64(co_t, po_t, x) ** 2).sum(-1).sum(1) * 1.1
    fit = SurfaceTensionFit(xi=1.5, alpha=0.9, gamma=0.3, delta=0.1)
    cc, pp = fit()
    log_power_residual(m(cc, pp, x), target).backward()
    base = dict(xi=1.5, alpha=0.9, gamma=0.3, delta=0.1)

    def f(**kw):
        with torch.no_grad():
            a, b = SurfaceTensionFit(**kw)()
            return float(log_power_residual(m64(a, b, x), target))

    for name in base:
        p, q = dict(base), dict(base)
        p[name] += H
        q[name] -= H
        fd = (f(**p) - f(**q)) / (2 * H)
        an = float(getattr(fit, name).grad)
        assert abs(fd - an) <= FD_TOL * abs(fd), (name, fd, an)


@pytest.mark.gpu
def test_kept_masks_give_the_same_gradients(gpu_available):
    """A backward after a forward on the same bubbles reads the forward's masks (keep_masks): the
    gradients are the same bits as with the masks searched again, and after the bubbles move the
    kept masks no longer match and are not used."""
    c = small_case(seed=9, n=8)
    c["n_cos"], c["n_phi"], c["n_t"] = 16, 16, 64
    c["w"] = np.geomspace(1.0, 200.0, 12)
    c["kh"] = W.fibonacci_khat(3)
    co = np.array([[1.0, 0.3]])
    po = np.array([[5.0, 3.5]])
    rng = np.random.default_rng(4)
    G = rng.normal(size=(3, 2, 1, 12)) + 1j * rng.normal(size=(3, 2, 1, 12))
    for kernel in ("fp64_factored", "mixed"):
        fresh = _library_model(c, kernel=kernel)
        ref = fresh.vjp(co, po, c["inter"], G)
        kept = _library_model(c, kernel=kernel)
        kept._forward(co, po, c["inter"])
        got = kept.vjp(co, po, c["inter"], G)
        for g_, r_ in zip(got, ref):
            np.testing.assert_array_equal(g_, r_)
        moved = c["inter"].copy()
        moved[:, 1] += 1e-3
        kept._forward(co, po, c["inter"])
        got2 = kept.vjp(co, po, moved, G)
        ref2 = _library_model(c, kernel=kernel).vjp(co, po, moved, G)
        for g_, r_ in zip(got2, ref2):
            np.testing.assert_array_equal(g_, r_)
