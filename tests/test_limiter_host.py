"""Host restatement of the Zhang-Shu post-step hook (frforge_b200.limiters)
on the CPU: it restores positive density and pressure at every solution
point, keeps every element integral, leaves admissible elements untouched,
and a method that overrides post_step! is accepted by the GPU descriptor
only because it names a device implementation."""
import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200.limiters import zhang_shu_limit_
from frforge_b200.methods import UnsupportedHookError


def _state_2d(seed=3):
    rng = np.random.default_rng(seed)
    eq = F.Euler2D(1.4)
    ops = F.build_operators(3)
    mesh = F.Mesh2D(0.0, 1.0, 0.0, 2.0, 4, 3, *[F.PeriodicBC() for _ in range(4)])
    st = F.allocate_state(mesh, ops, 4)
    X, Y = mesh.physical_coords(ops)
    st.u[...] = eq.primitives_to_conserved(1.0 + 0.3 * np.sin(3 * X) * np.cos(2 * Y), 0.2 * np.cos(X),
                                           -0.1 + 0 * X, 0.8 + 0.2 * np.sin(Y))
    return eq, st, rng


def _element_integrals(st):
    w = st.ops.w
    m = st.mesh
    e = np.arange(m.n_elements)
    J = (m.Jx[e % m.nx] * m.Jy[e // m.nx])[None, None, :, None]
    return np.sum(w[:, None, None, None] * w[None, :, None, None] * J * st.u, axis=(0, 1))


def test_restores_positivity_and_keeps_integrals():
    eq, st, rng = _state_2d()
    # spoil a few points: negative density in element 2, negative pressure in element 7
    st.u[1, 2, 2, 0] = -0.05
    st.u[0, 3, 7, 3] = 0.01
    before = _element_integrals(st)
    untouched = st.u[:, :, 5, :].copy()
    zhang_shu_limit_(st, eq, 1e-13, 1e-13)
    assert np.all(st.u[..., 0] >= 1e-13 * (1 - 1e-12))
    assert np.all(eq.pressure(st.u) >= 1e-13 * (1 - 1e-9) - 1e-15)
    assert np.allclose(_element_integrals(st), before, rtol=1e-13, atol=1e-15)
    assert np.array_equal(st.u[:, :, 5, :], untouched)


def test_1d_limiter():
    eq = F.Euler1D(1.4)
    ops = F.build_operators(2)
    mesh = F.Mesh1D(0.0, 1.0, 6, F.TransmissiveBC(), F.TransmissiveBC())
    st = F.allocate_state(mesh, ops, 3)
    x = mesh.physical_coords(ops)
    st.u[...] = eq.primitives_to_conserved(1.0 + 0.2 * x, 0.1 + 0 * x, 1.0 + 0 * x)
    st.u[0, 4, 2] = 0.2  # tiny energy: negative pressure at one point
    w, J = ops.w, mesh.J
    before = np.sum(w[:, None, None] * J[None, :, None] * st.u, axis=0)
    zhang_shu_limit_(st, eq)
    assert np.all(eq.pressure(st.u) > 0)
    assert np.allclose(np.sum(w[:, None, None] * J[None, :, None] * st.u, axis=0), before, rtol=1e-13)


def test_method_needs_a_device_hook_name():
    m = F.PositivityPreservingPersson()
    spec = m.gpu_spec()
    assert spec["hooks"] == {"post_step": ("positivity_zhang_shu", (1e-13, 1e-13))}
    assert spec["method"] == "persson"

    class HostOnly(F.PerssonAVMethod):
        def post_step_(self, state, eq):
            return None

    with pytest.raises(UnsupportedHookError):
        HostOnly().gpu_spec()
    assert "persson_av_positive" in F.list_methods()


def test_registry_lists_the_device_hook():
    from frforge_b200 import _lib as L

    hooks = L.device_hooks()
    assert hooks["positivity_zhang_shu"] == (L.HOOK_SLOT["post_step"], 1, 2)


def test_method_hooks_resolve_through_the_registry():
    # what Batch.add and Server.submit attach to an instance: slot and id from
    # the registry, the method's parameters as given
    from frforge_b200 import _lib as L
    from frforge_b200.gpu import method_hooks

    (sl, hid, par), = method_hooks(F.PositivityPreservingPersson(eps_rho=2e-3, eps_p=5e-4))
    assert (sl, hid) == (L.HOOK_SLOT["post_step"], 1)
    assert par.dtype == np.float64 and list(par) == [2e-3, 5e-4]
    assert method_hooks(F.PerssonAVMethod()) == []
    assert method_hooks(None) == []
