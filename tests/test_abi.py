"""CPU-side checks of the C-ABI library: it loads, exports every symbol that
include/frforge_cuda.h declares, and its host-side set-up (operator tables,
error mapping) behaves; no kernel is launched."""
import os
import re

import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "frforge_cuda.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_]+\**\s+\**(frg_[a-z0-9_]+)\(", hdr, re.M)))


def test_library_exports_every_declared_symbol():
    lib = L.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for name in syms:
        assert hasattr(lib, name), name
        assert name in L.SIGNATURES, f"{name} lacks a ctypes signature"


def test_abi_version_and_status_strings():
    lib = L.load()
    assert lib.frg_abi_version() == 1
    assert b"sm_100a" in lib.frg_version()
    assert lib.frg_status_string(L.FRG_DIVERGED) == b"diverged"


@pytest.mark.parametrize("points", ["gl", "gll"])
@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_host_operators_match_oracle(p, points):
    import oracle as O

    o = F.build_operators(p, points)
    r = O.build_operators(p, points)
    for k in ("xi", "w", "l_L", "l_R", "gL_xi", "gR_xi", "gL", "gR"):
        assert np.allclose(getattr(o, k), r[k], rtol=0, atol=5e-14), k
    assert np.allclose(o.D, r["D"], rtol=0, atol=5e-13)
    assert np.allclose(o.V_legendre, r["V"], rtol=0, atol=5e-15)


def test_invalid_operator_request():
    with pytest.raises(ValueError):
        F.build_operators(6)
    with pytest.raises(ValueError):
        F.build_operators(3, "gauss")


def test_mesh_vertices_match_julia_range():
    import oracle as O

    s = O.OracleSolver.one_d(p=1, nel=100, xl=0.0, xr=10.0)
    x = s.coords().ravel(order="F")
    m = F.Mesh1D(0.0, 10.0, 100)
    xm = m.physical_coords(F.build_operators(1)).ravel(order="F")
    assert np.allclose(x, xm, rtol=0, atol=1e-15)
    assert F.julia_range(0.0, 0.4, 5)[2] == 0.2
    assert F.julia_range(0.0, 10.0, 101)[3] == 0.3


def test_scheme_and_registry():
    assert F.DEFAULT_SCHEME == F.SchemeConfig("gl", "rusanov", "ssp_rk3")
    s = F.parse_scheme(points="GLL", flux="hllc", time="ssp-rk2")
    assert (s.points, s.flux, s.time) == ("gll", "hllc", "ssp_rk2")
    with pytest.raises(ValueError):
        F.SchemeConfig(points="xyz")
    assert F.scheme_dict(F.DEFAULT_SCHEME)["time"] == "SSP-RK3"
    assert set(["null", "persson_av", "scaled_persson"]) <= set(F.list_methods())
    m = F.get_capturing_method("scaled_persson")
    assert m.gpu_spec()["c_av"] == 0.5
    assert F.get_capturing_method("persson_av").gpu_spec()["c_av"] == 0.1
    assert F.method_params(F.get_capturing_method("persson_av"))["av_form"] == "conservative_br0"


def test_unsupported_hook_detected_on_host():
    class Probe(F.AbstractCapturingMethod):
        pass

    class Override(F.PerssonAVMethod):
        def post_step_(self, state, eq):
            return None

    with pytest.raises(F.UnsupportedHookError):
        Probe().gpu_spec()
    with pytest.raises(F.UnsupportedHookError):
        Override().gpu_spec()
    assert F.NullCapturing().gpu_spec()["method"] == "null"
