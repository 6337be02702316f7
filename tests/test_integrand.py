"""Time-resolved integrand (compute_c_integrand / compute_c_integrand_fixed_bubble,
rust/bubble-gw/src/many_bubbles/generalized_bulk_flow.rs:776-920).

CPU: argument checks through the C ABI.  GPU: against the oracle to 1e-12 (max
error over all entries, relative to the largest entry), the fixed-bubble form,
empty and late selections, and the sum over t against compute_c_integral.
"""
import numpy as np
import pytest

from oracle import oracle as O
from gw_fopt_b200 import many_bubbles as mb
from gw_fopt_b200 import workloads as W

from test_gpu_parity import make_flow

TOL = 1e-12


def rel(got, ref):
    return float(np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300))


def test_argument_checks_without_gpu():
    c = W.config(1)
    g = make_flow(c.interior, c.exterior, 8, 8)
    with pytest.raises(ValueError):
        g.compute_c_integrand(c.w[:3], t_end=1.5, n_t=1)
    with pytest.raises(IndexError):
        g.compute_c_integrand(c.w[:3], t_end=1.5, n_t=8, selected_bubbles=np.array([99]))
    with pytest.raises(IndexError):
        g.compute_c_integrand_fixed_bubble(99, c.w[:3], 0.0, 1.5, 8)
    z = g.compute_c_integrand(c.w[:3], t_end=1.5, n_t=8, selected_bubbles=np.array([], dtype=np.int64))
    assert z.shape == (2, 1, 3, 8) and not z.any()
    assert not g.compute_c_integrand_fixed_bubble(0, c.w[:3], 0.0, 1.5, 1).any()


@pytest.mark.gpu
@pytest.mark.parametrize("damping", [None, 0.6])
def test_integrand_vs_oracle(gpu_available, damping):
    c = W.config(1)
    co, po = [[1.0], [0.4]], [[5.0], [3.5]]
    g = make_flow(c.interior, c.exterior, 12, 14, co, po, damping=damping)
    got = g.compute_c_integrand(c.w[:10], t_begin=0.05, t_end=1.5, n_t=48)
    ref = O.compute_c_integrand(c.interior, c.exterior, 12, 14, c.w[:10], 1.5, 48, t_begin=0.05,
                                coefficients=co, powers=po, damping=damping)
    assert got.shape == ref.shape == (2, 2, 10, 48)
    assert rel(got, ref) < TOL
    one = g.compute_c_integrand_fixed_bubble(3, c.w[:10], 0.05, 1.5, 48)
    ref1 = O.compute_c_integrand(c.interior, c.exterior, 12, 14, c.w[:10], 1.5, 48, t_begin=0.05,
                                 coefficients=co, powers=po, damping=damping, selected=[3])
    assert rel(one, ref1) < TOL
    # the sum over t is the integral without a time cutoff
    integral = g.compute_c_integral(c.w[:10], t_begin=0.05, t_end=1.5, n_t=48)
    assert rel(got.sum(-1), integral) < 1e-11


@pytest.mark.gpu
def test_integrand_selection_and_late_bubbles(gpu_available):
    c = W.config(1)
    t_end = float(np.median(c.interior[:, 0]))
    late = np.flatnonzero(c.interior[:, 0] >= t_end)
    g = make_flow(c.interior, c.exterior, 10, 10, [[1.0]], [[5.0]])
    z = g.compute_c_integrand(c.w[:4], t_begin=0.0, t_end=t_end, n_t=16, selected_bubbles=late)
    assert not z.any()
    sel = np.array([0, 2, 0, 5])
    got = g.compute_c_integrand(c.w[:4], t_begin=0.0, t_end=1.2, n_t=20, selected_bubbles=sel)
    ref = O.compute_c_integrand(c.interior, c.exterior, 10, 10, c.w[:4], 1.2, 20, t_begin=0.0,
                                coefficients=[[1.0]], powers=[[5.0]], selected=sel)
    assert rel(got, ref) < TOL
