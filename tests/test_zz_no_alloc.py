"""The allocation-free residual entry point against the regular one.

frg_residual2d_noalloc serves callers that cannot call cudaMalloc when they
need a residual (their device memory belongs to their own pool or budget):
they pass device buffers they already own and the library uses a fixed
device scratch array instead of allocating.  This test calls it through the
C ABI with torch-owned device buffers and checks it twice in a row, on
different states, against frg_residual within the residual tolerance (1e-12
relative L-infinity) and against the oracle within the production-path
tolerance (1e-11: library-built tables and exact affine metrics, as in
test_gpu_parity.test_residual_2d_affine_path).  It sits in its own file
collected last.
"""
import ctypes as C

import numpy as np
import pytest

from pairs import four_quadrant_state, pair_2d, rel_linf, smooth_state_2d

pytestmark = pytest.mark.gpu


def _noalloc(solve, u_host, t=0.0):
    import torch

    from frforge_b200 import _lib as L

    u_dev = torch.from_numpy(np.ascontiguousarray(u_host.ravel(order="F"))).to("cuda")
    du_dev = torch.full_like(u_dev, float("nan"))
    stream = torch.cuda.current_stream()
    rc = L.load().frg_residual2d_noalloc(C.byref(solve.desc), C.c_void_p(u_dev.data_ptr()),
                                         C.c_void_p(du_dev.data_ptr()), float(t),
                                         C.c_void_p(stream.cuda_stream))
    assert rc == 0, rc
    torch.cuda.synchronize()
    return du_dev.cpu().numpy().reshape(u_host.shape, order="F")


@pytest.mark.parametrize("cfg", [
    dict(p=3, nx=24, ny=20, flux="hllc", method="persson", bcs=("transmissive",) * 4),
    dict(p=2, nx=16, ny=16, flux="rusanov", method="persson", av_form="element_local_DD"),
    dict(p=4, nx=9, ny=7, flux="hllc", method="null",
         bcs=("reflecting", "transmissive", "periodic", "periodic")),
])
def test_noalloc_matches_frg_residual(cfg):
    orc, state, solve = pair_2d(**cfg)
    states = [four_quadrant_state(orc), smooth_state_2d(orc)]
    for u in states:  # two calls in a row share the scratch array
        solve.upload(u, 0.0)
        ref = solve.residual()
        got = _noalloc(solve, u)
        assert np.all(np.isfinite(got))
        assert rel_linf(got, ref) <= 1e-12, rel_linf(got, ref)
        orc.set_state(u)
        orc.t = 0.0
        assert rel_linf(got, orc.residual()) <= 1e-11


def test_noalloc_rejects_oversized_mesh():
    from frforge_b200 import _lib as L

    orc, state, solve = pair_2d(p=1, nx=4, ny=4)
    d = L.frg_solve_desc.from_buffer_copy(solve.desc)
    d.nx, d.ny = 1024, 1024  # 1M elements > FRG_NOALLOC_MAX_ELEMENTS
    rc = L.load().frg_residual2d_noalloc(C.byref(d), C.c_void_p(1), C.c_void_p(1), 0.0, None)
    assert rc == L.FRG_ERR_INVALID_ARG
