"""Spectrum post-processing (the reference's DataGwBulkFlow, data_gw_bulkflow.py:26-190)
and bubble CSV I/O (lattice_bubbles.rs:480-572).

CPU: the oracle against golden vectors made by running the reference's own
DataGwBulkFlow (tests/golden/make_postprocess_golden.py), the host-side weight
mapping and its errors, and CSV round trips.  GPU: the C ABI kernel against the
oracle, host and device-pointer forms, on the golden inputs and on a spectrum
computed by the library.  Tolerance 1e-12 relative (FP64 arithmetic in a
different summation order).
"""
import os

import numpy as np
import pytest

from oracle import postprocess as OP
from gw_fopt_b200 import bubble_io as IO
from gw_fopt_b200 import many_bubbles as mb
from gw_fopt_b200 import postprocess as PP
from gw_fopt_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(__file__), "golden", "postprocess_golden.npz")
TOL = 1e-12


def gold():
    g = np.load(GOLD)
    return {k: g[k] for k in g.files}


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_oracle_matches_reference_golden():
    g = gold()
    spec = OP.de_dlogw_dcosthetak(g["c"], g["w"], g["xi_powers"].tolist(), g["xi_coefficients"].tolist(),
                                  g["powers_sets"].tolist())
    assert np.array_equal(spec, g["spectra"])  # the same numpy operations in the same order
    de = OP.de_dlogw(g["c"], g["w"], g["cos_thetak"], g["xi_powers"].tolist(), g["xi_coefficients"].tolist(),
                     g["powers_sets"].tolist())
    assert np.array_equal(de, g["de_dlogw"])
    f = OP.de_dlogw_interp(g["w"], de, float(g["interp_d"]), 1.0, float(g["interp_rho"]))
    assert np.allclose(f(g["w_eval"]), g["interp"], rtol=1e-14, atol=0)


def test_set_weights_mapping_and_errors():
    w = PP.set_weights([2.0, 0.5, 1.0, 2.0], [0.25, 0.2, 0.3, 0.25], [5.0, 3.5, 4.0])
    assert np.array_equal(w, [0.5, 0.2, 0.3])
    with pytest.raises(ValueError, match="same length"):
        PP.set_weights([2.0], [0.5, 0.5], [5.0])
    with pytest.raises(ValueError, match="sum to 1"):
        PP.set_weights([2.0], [0.5], [5.0])
    PP.set_weights([2.0], [0.5], [5.0], check_sum=False)
    with pytest.raises(ValueError, match="not in powers_sets_sample"):
        PP.set_weights([7.0], [1.0], [5.0])
    with pytest.raises(ValueError, match="envelope"):
        PP.set_weights([None], [1.0], [5.0])
    with pytest.raises(ValueError, match="numbers or None"):
        PP.set_weights(["2"], [1.0], [5.0])
    with pytest.raises(ValueError, match="lists or numpy arrays"):
        PP.set_weights(2.0, [1.0], [5.0])


def test_csv_round_trip(tmp_path):
    c = W.config(1)
    for headers in (False, True):
        pi, pe = tmp_path / f"i{headers}.csv", tmp_path / f"e{headers}.csv"
        lb = mb.LatticeBubbles(mb.EmptyLattice(), c.interior, c.exterior)
        IO.save_to_csv_files(lb, pi, pe, has_headers=headers)
        back = IO.from_csv_files(pi, pe, mb.EmptyLattice(), has_headers=headers)
        assert np.array_equal(back.bubbles_interior, c.interior)
        assert np.array_equal(back.bubbles_exterior, c.exterior)
        if headers:
            assert open(pi).readline().strip() == "t,x,y,z"
    bad = tmp_path / "bad.csv"
    bad.write_text("0,1,2\n0,1,2\n")
    with pytest.raises(ValueError, match="columns"):
        IO.load_bubbles_from_csv(bad)
    ragged = tmp_path / "ragged.csv"
    ragged.write_text("0,1,2,3\n0,1,2\n")
    with pytest.raises(ValueError, match="different lengths"):
        IO.load_bubbles_from_csv(ragged)


def two_bubble_flow():
    return mb.GeneralizedBulkFlow(mb.LatticeBubbles(mb.EmptyLattice(), np.array([[0.0, 0.0, 0.0, 0.0],
                                                                                  [0.0, 0.0, 0.0, 1.0]])))


@pytest.mark.gpu
def test_gpu_power_spectrum_golden(gpu_available):
    g = gold()
    flow = two_bubble_flow()
    a = PP.set_weights(g["xi_powers"].tolist(), g["xi_coefficients"].tolist(), g["powers_sets"])
    spec, de = PP.power_spectrum(flow, g["c"], g["w"], a, g["cos_thetak"])
    assert rel(spec, g["spectra"]) < TOL
    assert rel(de, g["de_dlogw"]) < TOL
    de2 = PP.de_dlogw(flow, g["c"], g["w"], g["cos_thetak"], g["xi_powers"].tolist(),
                      g["xi_coefficients"].tolist(), g["powers_sets"])
    assert np.array_equal(de2, de)
    # one direction: the integral over cos(theta_k) is zero
    s1, d1 = PP.power_spectrum(flow, g["c"][:1], g["w"], a, g["cos_thetak"][:1])
    assert rel(s1, g["spectra"][:1]) < TOL and np.all(d1 == 0.0)


@pytest.mark.gpu
def test_gpu_power_spectrum_of_computed_spectrum_device_form(gpu_available):
    import torch
    c = W.config(1)
    flow = mb.GeneralizedBulkFlow(mb.LatticeBubbles(mb.EmptyLattice(), c.interior, c.exterior))
    flow.set_resolution(c.n_cos, c.n_phi)
    flow.set_gradient_scaling_params([[1.0], [0.5]], [[5.0], [3.5]])
    out = flow.compute_c_integral_khat(c.w, c.khat, t_begin=c.t_begin, t_end=c.t_end, n_t=c.n_t)
    K, _, S, Wn = out.shape
    ck = c.khat[:, 2]
    xi_p, xi_c, ps = [2.0, 0.5], [0.6, 0.4], [5.0, 3.5]
    ref_spec = OP.de_dlogw_dcosthetak(out, c.w, xi_p, xi_c, ps)
    ref_de = OP.de_dlogw(out, c.w, ck, xi_p, xi_c, ps)
    a = PP.set_weights(xi_p, xi_c, ps)
    spec, de = PP.power_spectrum(flow, out, c.w, a, ck)
    assert rel(spec, ref_spec) < TOL and rel(de, ref_de) < TOL
    dev = torch.device("cuda:0")
    cd = torch.from_numpy(out.view(np.float64).copy()).to(dev)
    sd = torch.empty((K, Wn), dtype=torch.float64, device=dev)
    dd = torch.empty((Wn,), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    PP.power_spectrum_device(flow, cd.data_ptr(), K, S, c.w, a, ck, sd.data_ptr(), dd.data_ptr())
    assert np.array_equal(sd.cpu().numpy(), spec) and np.array_equal(dd.cpu().numpy(), de)
