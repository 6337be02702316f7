"""GPU test of bgwx_first_colliding_noalloc, the first-collider search for
callers that cannot allocate device memory (frameworks that serve all device
memory from their own pool, services that must not allocate after start-up).

Every input and output lives in caller-owned device memory (allocated here by
torch, as such a caller's pool would); the entry point itself uses only its
fixed static work array.  Its codes and collision delays must equal, bit for
bit, those of the allocating entry point bgwx_generalized_bulk_flow_first_colliding,
on two calls in a row that reuse the shared work array.  The file name sorts
last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C
import math

import numpy as np
import pytest

from gw_fopt_b200 import _lib as L
from gw_fopt_b200 import many_bubbles as mb
from gw_fopt_b200 import workloads as W

pytestmark = pytest.mark.gpu


def direction_table(n_cos, n_phi):
    """(n_cos*n_phi, 4) rows (1, s cos phi, s sin phi, c), the reference's grid (libm sin/cos)."""
    cos_t = [-1.0 + (2.0 / (n_cos - 1)) * i for i in range(n_cos)]
    phi = [0.0 + (2.0 * math.pi / (n_phi - 1)) * j for j in range(n_phi)]
    out = np.empty((n_cos * n_phi, 4))
    for i, c in enumerate(cos_t):
        s = abs(math.sqrt(1.0 - c * c))
        for j, p in enumerate(phi):
            out[i * n_phi + j] = (1.0, s * math.cos(p), s * math.sin(p), c)
    return out


def test_noalloc_matches_allocating_entry_point(gpu_available):
    import torch
    lib = L.lib()
    cfg = W.config(2)  # 512 bubbles, 3072 periodic images
    n_cos, n_phi = 40, 48
    nd = n_cos * n_phi
    n_int = cfg.interior.shape[0]
    n_tot = n_int + cfg.exterior.shape[0]

    # the allocating entry point, over every interior bubble
    g = mb.GeneralizedBulkFlow(mb.LatticeBubbles(mb.EmptyLattice(), cfg.interior, cfg.exterior))
    g.set_resolution(n_cos, n_phi)
    ref_codes = np.empty((n_int, n_cos, n_phi), dtype=np.int32)
    ref_tau = np.empty((n_int, n_cos, n_phi))
    L.check(lib.bgwx_generalized_bulk_flow_first_colliding(
        g._h, 0, n_int, ref_codes.ctypes.data_as(C.POINTER(C.c_int32)),
        ref_tau.ctypes.data_as(C.POINTER(C.c_double))))

    dev = torch.device("cuda", 0)
    bubbles = torch.tensor(np.concatenate([cfg.interior, cfg.exterior]), dtype=torch.float64, device=dev)
    dirs = torch.tensor(direction_table(n_cos, n_phi), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    # two calls in a row sharing the library's static work array
    for sel in (np.arange(7, 307), np.arange(0, 512)[::-1].copy()):
        d_sel = torch.tensor(sel.astype(np.int32), device=dev)  # uint32 bit patterns, all < 2^31
        codes = torch.full((sel.size, nd), 12345, dtype=torch.int32, device=dev)
        tau = torch.full((sel.size, nd), -1.0, dtype=torch.float64, device=dev)
        st = lib.bgwx_first_colliding_noalloc(
            C.c_void_p(bubbles.data_ptr()), n_int, n_tot, C.c_void_p(d_sel.data_ptr()), sel.size,
            C.c_void_p(dirs.data_ptr()), nd, C.c_void_p(codes.data_ptr()), C.c_void_p(tau.data_ptr()),
            C.c_void_p(stream.cuda_stream))
        assert st == L.OK, lib.bgw_last_error_message().decode()
        torch.cuda.synchronize()
        got_codes = codes.cpu().numpy().reshape(sel.size, n_cos, n_phi)
        got_tau = tau.cpu().numpy().reshape(sel.size, n_cos, n_phi)
        assert np.array_equal(got_codes, ref_codes[sel])
        assert np.array_equal(got_tau, ref_tau[sel])

    # an index past the interior bubbles cannot be checked on the host (it lives in device
    # memory): its row reads INT32_MIN codes and NaN delays, the other rows are unaffected
    sel = np.array([3, n_int, 200], dtype=np.int64)
    d_sel = torch.tensor(sel.astype(np.int32), device=dev)
    codes = torch.full((sel.size, nd), 12345, dtype=torch.int32, device=dev)
    tau = torch.full((sel.size, nd), -1.0, dtype=torch.float64, device=dev)
    st = lib.bgwx_first_colliding_noalloc(
        C.c_void_p(bubbles.data_ptr()), n_int, n_tot, C.c_void_p(d_sel.data_ptr()), sel.size,
        C.c_void_p(dirs.data_ptr()), nd, C.c_void_p(codes.data_ptr()), C.c_void_p(tau.data_ptr()),
        C.c_void_p(stream.cuda_stream))
    assert st == L.OK, lib.bgw_last_error_message().decode()
    torch.cuda.synchronize()
    got_codes = codes.cpu().numpy().reshape(sel.size, n_cos, n_phi)
    got_tau = tau.cpu().numpy().reshape(sel.size, n_cos, n_phi)
    assert np.all(got_codes[1] == np.iinfo(np.int32).min)
    assert np.all(np.isnan(got_tau[1]))
    for row, a in ((0, 3), (2, 200)):
        assert np.array_equal(got_codes[row], ref_codes[a])
        assert np.array_equal(got_tau[row], ref_tau[a])

    # more radiating bubbles than the static work array holds: a clear error, nothing launched
    big = torch.zeros(513, dtype=torch.int32, device=dev)
    st = lib.bgwx_first_colliding_noalloc(
        C.c_void_p(bubbles.data_ptr()), n_int, n_tot, C.c_void_p(big.data_ptr()), 513, C.c_void_p(dirs.data_ptr()),
        nd, C.c_void_p(codes.data_ptr()), C.c_void_p(tau.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert st == L.CALCULATION_ERROR
    assert "exceeds the no-allocation limit of 512" in lib.bgw_last_error_message().decode()
