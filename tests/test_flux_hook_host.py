"""The numerical_flux_method slot's host side (no GPU): the registry resolves
the plugin's device implementations to that slot, the plugin's descriptor
names them, and its host restatement of the scaled Rusanov flux equals the
oracle's Rusanov flux at alpha = 1 and scales its dissipation otherwise."""
import ctypes as C

import numpy as np
import pytest

import frforge_b200 as F
import oracle as O
from frforge_b200 import _lib as L


@pytest.mark.parametrize("name", ["flux_rusanov", "flux_hllc"])
def test_registry_resolves_to_the_flux_slot(name):
    sl, hid = C.c_int(), C.c_int()
    assert L.load().frg_hook_lookup(name.encode(), C.byref(sl), C.byref(hid)) == 0
    assert sl.value == L.HOOK_SLOT["numerical_flux_method"] and hid.value > 0


def test_plugin_descriptor_names_the_device_hook():
    spec = F.FluxOverridePersson("rusanov", 0.6, c_av=0.2).gpu_spec()
    assert spec["method"] == "persson" and spec["c_av"] == 0.2
    assert spec["hooks"] == {"numerical_flux_method": ("flux_rusanov", (0.6,))}
    assert F.get_capturing_method("persson_av_flux_override", flux="hllc").gpu_spec()["hooks"] == {
        "numerical_flux_method": ("flux_hllc", ())}


def test_an_override_without_a_device_name_is_refused():
    class HostOnlyFlux(F.PerssonAVMethod):
        def numerical_flux_method(self, eq, uL, uR):
            return None

    with pytest.raises(L.UnsupportedHookError):
        HostOnlyFlux().gpu_spec()


def test_host_restatement_against_the_oracle_flux():
    eq = F.Euler1D(1.4)
    g = np.random.default_rng(3)
    for _ in range(50):
        rL, rR = g.uniform(0.1, 2.0, 2)
        uL = eq.primitives_to_conserved(rL, g.uniform(-1, 1), g.uniform(0.1, 2.0))
        uR = eq.primitives_to_conserved(rR, g.uniform(-1, 1), g.uniform(0.1, 2.0))
        ref = O.flux_1d("rusanov", 1.4, uL, uR)
        one = F.FluxOverridePersson("rusanov", 1.0).numerical_flux_method(eq, uL, uR)
        assert np.allclose(one, ref, rtol=1e-14, atol=1e-14)
        half = F.FluxOverridePersson("rusanov", 0.5).numerical_flux_method(eq, uL, uR)
        central = F.FluxOverridePersson("rusanov", 0.0).numerical_flux_method(eq, uL, uR)
        assert np.allclose(half, 0.5 * (one + central), rtol=1e-13, atol=1e-13)
