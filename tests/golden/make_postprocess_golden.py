"""Generates postprocess_golden.npz by running the reference's own post-processing
(src/gw_fopt/bubble_dynamics/utils/data_gw_bulkflow.py, DataGwBulkFlow) on seeded
synthetic bulk-flow output.

Run in a container that has the reference source tree; its root directory is
the required argument:

    python tests/golden/make_postprocess_golden.py <reference-root>
  The reference module imports the compiled
extension gw_fopt.bubble_gw only for utils.sample; a stand-in that returns its
first argument as an array is installed, and the rows carry their w and power
lists directly.  filter_dataframe.py and data_gw_bulkflow.py are loaded from
the reference tree unchanged.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

import numpy as np
import pandas as pd


def load_reference(root):
    udir = os.path.join(root, "src", "gw_fopt", "bubble_dynamics", "utils")
    utils = types.ModuleType("gw_fopt.bubble_gw.utils")
    utils.sample = lambda values, *rest: np.asarray(values, dtype=np.float64)
    bg = types.ModuleType("gw_fopt.bubble_gw")
    bg.utils = utils
    top = types.ModuleType("gw_fopt")
    top.bubble_gw = bg
    sys.modules.update({"gw_fopt": top, "gw_fopt.bubble_gw": bg, "gw_fopt.bubble_gw.utils": utils})
    pkg = types.ModuleType("refpost")
    pkg.__path__ = [udir]
    sys.modules["refpost"] = pkg
    for name in ("filter_dataframe", "data_gw_bulkflow"):
        spec = importlib.util.spec_from_file_location(f"refpost.{name}", os.path.join(udir, f"{name}.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[f"refpost.{name}"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["refpost.data_gw_bulkflow"].DataGwBulkFlow


def main(root):
    DataGwBulkFlow = load_reference(root)
    rng = np.random.default_rng(20261204)
    K, S, W = 9, 3, 40
    powers_sets = [5.0, 3.5, 4.0]                      # xi + 3
    w = np.geomspace(1.0, 3.0e3, W)
    c = (rng.normal(size=(K, 2, S, W)) + 1j * rng.normal(size=(K, 2, S, W))) * 1e-3 / (1.0 + w / 100.0)
    cos_thetak = rng.uniform(-1.0, 1.0, size=K)         # deliberately unsorted rows
    xi_powers, xi_coefficients = [2.0, 0.5, 1.0], [0.5, 0.2, 0.3]
    df = pd.DataFrame({
        "d": [1.0] * K,
        "_pset_id": list(range(K)),
        "cos_theta_k": cos_thetak,
        "w_sample": [(w.tolist(),)] * K,
        "powers_sets_sample": [(powers_sets,)] * K,
        "c_bulkflow": [c[k] for k in range(K)],
        "c_envelope": [np.zeros((2, W), dtype=complex)] * K,
    })
    data = DataGwBulkFlow(df, d0=1.0)
    spec = data.de_dlogw_dcosthetak(xi_powers, xi_coefficients)
    de = data.de_dlogw(xi_powers, xi_coefficients)
    w_eval = np.geomspace(2.0, 2.5e3, 17) / 1.7
    interp = data.de_dlogw_interp(xi_powers, xi_coefficients, d=1.7, rho_vacuum=0.8)(w_eval)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "postprocess_golden.npz")
    np.savez(out, c=c, w=w, cos_thetak=cos_thetak, powers_sets=np.array(powers_sets),
             xi_powers=np.array(xi_powers), xi_coefficients=np.array(xi_coefficients), spectra=spec, de_dlogw=de,
             interp_d=1.7, interp_rho=0.8, w_eval=w_eval, interp=interp)
    print("wrote", out, spec.shape, de.shape)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_postprocess_golden.py <reference-root>")
    main(sys.argv[1])
