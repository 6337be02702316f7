"""Generates tests/golden/golden_small.npz from the oracle.

The reference crate cannot be run here, so the golden vectors are the
oracle's (the CPU f64 restatement in oracle/), pinned by the known-answer
tests of tests/test_oracle_kat.py.  They freeze small parity cases so that GPU
tests and future oracle edits are checked against the same numbers.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from gw_fopt_b200 import workloads as W  # noqa: E402

CAPI2 = np.array([[0.0, 0.0, 10.0, 0.0], [0.0, 0.0, 0.0, 0.0]])
BENCH5 = np.array([[0.0, 0.0, 10.0, 0.0], [0.0, 0.0, 0.0, 0.0], [0.0, 4.0, 0.0, 4.0], [0.0, 4.0, 2.0, 4.0],
                   [0.0, 0.0, 2.0, 1.0]])


def cases():
    c1 = W.config(1)
    conf_y = np.loadtxt(os.path.join(os.path.dirname(__file__), "confY.txt"))
    return {
        # rust/c-bubble-gw/tests/c_api.rs:137-141 (4x5 patches, n_t=40, w=[0.5,1.0])
        "capi2": dict(interior=CAPI2, exterior=np.zeros((0, 4)), n_cos=4, n_phi=5, w=np.array([0.5, 1.0]),
                      t_begin=0.0, t_end=8.0, n_t=40, coeffs=np.array([[0.0], [1.0]]),
                      powers=np.array([[3.0], [3.0]]), damping=np.nan),
        # rust/benches/bulk_flow_bench.rs:9-15 at reduced resolution
        "bench5": dict(interior=BENCH5, exterior=np.zeros((0, 4)), n_cos=20, n_phi=40,
                       w=np.geomspace(1e-2, 1e2, 12), t_begin=0.0, t_end=15.0, n_t=200,
                       coeffs=np.array([[0.0], [1.0]]), powers=np.array([[3.0], [3.0]]), damping=np.nan),
        # docs/examples/generalized_bulkflow.py:743-757 (confY, L=2, periodic) at low resolution
        "confY": dict(interior=conf_y, exterior=W.periodic_images(conf_y, 2.0), n_cos=16, n_phi=17,
                      w=np.geomspace(0.5, 50.0, 8), t_begin=0.0, t_end=3.0, n_t=64,
                      coeffs=np.array([[1.0]]), powers=np.array([[5.0]]), damping=np.nan),
        # config 1 geometry, k = z, with two terms and damping
        "cfg1_damped": dict(interior=c1.interior, exterior=c1.exterior, n_cos=32, n_phi=32, w=c1.w,
                            t_begin=0.0, t_end=1.5, n_t=128, coeffs=np.array([[0.6, 0.4], [1.0, 0.0]]),
                            powers=np.array([[5.0, 3.0], [4.0, 2.0]]), damping=0.3),
    }


def main():
    out = {}
    for name, p in cases().items():
        res = O.compute_c_integral(p["interior"], p["exterior"], p["n_cos"], p["n_phi"], p["w"], p["t_end"],
                                   p["n_t"], t_begin=p["t_begin"], coefficients=p["coeffs"], powers=p["powers"],
                                   damping=None if np.isnan(p["damping"]) else p["damping"])
        codes = O.first_colliding(p["interior"], p["exterior"], p["n_cos"], p["n_phi"])
        for k, v in p.items():
            out[f"{name}__{k}"] = np.asarray(v)
        out[f"{name}__out"] = res
        out[f"{name}__codes"] = codes
    np.savez_compressed(os.path.join(os.path.dirname(__file__), "golden_small.npz"), **out)


if __name__ == "__main__":
    main()
