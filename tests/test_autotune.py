"""Launch shapes of the spectrum calls: fixed (set_launch_shape) and measured
(set_autotune).  Frames are independent and the GEMM row parts only regroup
FP64 partial sums, so every shape must give the automatic shape's spectrum to
FP64 rounding; with the same row parts, frames per launch change nothing."""
import os

import numpy as np
import pytest

from gw_fopt_b200 import many_bubbles as mb
from gw_fopt_b200 import workloads as W

pytestmark = pytest.mark.gpu


def flow(kernel):
    c = W.config(2)
    lb = mb.LatticeBubbles(mb.EmptyLattice(), c.interior, c.exterior)
    g = mb.GeneralizedBulkFlow(lb)
    g.set_resolution(c.n_cos, c.n_phi)
    g.set_gradient_scaling_params(c.coefficients.tolist(), c.powers.tolist())
    g.set_kernel(kernel)
    return c, g


def spectrum(c, g):
    sel = np.arange(0, 512, 41)
    return g.compute_c_integral_khat(c.w, c.khat[:6], t_begin=0.0, t_end=c.t_end, n_t=c.n_t, selected_bubbles=sel)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("kernel", ["mixed", "fp64_factored"])
def test_fixed_shapes_match_automatic(gpu_available, kernel):
    c, g = flow(kernel)
    ref = spectrum(c, g)
    f0, r0 = g.last_launch_shape()
    assert f0 >= 1 and r0 >= 1
    shapes = [(4, 1), (1, 3), (2, 2), (5, 0)] if kernel == "mixed" else [(4, 0), (1, 0)]
    for f, r in shapes:
        g.set_launch_shape(f, r)
        out = spectrum(c, g)
        fu, ru = g.last_launch_shape()
        assert fu == min(f, f0)
        assert ru == (r if kernel == "mixed" and r else ru) and (kernel == "mixed" or ru == 1)
        e = rel(out, ref)
        print(kernel, (f, r), "->", (fu, ru), f"rel {e:.2e}")
        assert e < 1e-13
    # with the row parts fixed, the frames per launch change nothing
    outs = []
    for f in (6, 4, 1):
        g.set_launch_shape(f, 2)
        outs.append(spectrum(c, g))
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])


def test_autotune_choice_is_kept_and_exact(gpu_available, tmp_path, monkeypatch):
    cache = tmp_path / "shapes.txt"
    monkeypatch.setenv("BGWX_AUTOTUNE_CACHE", str(cache))
    c, g = flow("mixed")
    ref = spectrum(c, g)
    g.set_autotune(True)
    out = spectrum(c, g)
    f, r = g.last_launch_shape()
    assert f >= 1 and 1 <= r <= 16
    assert rel(out, ref) < 1e-13
    st = g.last_gemm_stages()
    assert st in (3, 4, 5)
    lines = cache.read_text().splitlines()
    assert len(lines) == 1
    key, fs, rs, ss, ms = lines[0].split()
    assert "k2:" in key and (int(fs), int(rs), int(ss), int(ms)) == (f, r, st, g.last_mask_chunking())
    assert int(ms) in (1, 2, 4)
    # the second call of the same shape reuses the choice (nothing new is written)
    out2 = spectrum(c, g)
    np.testing.assert_array_equal(out2, out)
    assert g.last_launch_shape() == (f, r)
    assert len(cache.read_text().splitlines()) == 1
    assert g.last_gemm_stages() == st
    # a fixed shape takes precedence; the GEMM's stage count does not change the result
    g.set_launch_shape(1, 1)
    spectrum(c, g)
    assert g.last_launch_shape() == (1, 1)
    outs = {}
    for stages in (3, 5):
        g.set_gemm_stages(stages)
        outs[stages] = spectrum(c, g)
        assert g.last_gemm_stages() == stages
    np.testing.assert_array_equal(outs[3], outs[5])


@pytest.mark.parametrize("kernel", ["mixed", "fp64_factored"])
def test_mask_chunking_gives_the_same_spectrum(gpu_available, kernel):
    """The first-collider search cut into 1, 2 or 4 times the automatic number of blocks per
    (bubble, frame): every direction is decided exactly whatever seeds its block's rows give, so
    the masks and the spectrum are the same bits."""
    c, g = flow(kernel)
    g.set_launch_shape(2, 2 if kernel == "mixed" else 0)
    outs = []
    for mc in (1, 2, 4):
        g.set_mask_chunking(mc)
        outs.append(spectrum(c, g))
        assert g.last_mask_chunking() == mc
    for o in outs[1:]:
        np.testing.assert_array_equal(o, outs[0])
    with pytest.raises(ValueError):
        g.set_mask_chunking(3)
