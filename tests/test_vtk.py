"""High-order VTU writer (frforge_b200.vtk) against the reference's own VTU
tests (test/test_vtk.jl, test/test_2d.jl:176-190): VTK Lagrange node
orders, point counts, GL -> equispaced interpolation of polynomials, cell
types and connectivity, discontinuous duplicated nodes, field names; plus a
polynomial state whose written values must equal the polynomial at the
written node coordinates."""
import numpy as np
import pytest

import frforge_b200 as F
from frforge_b200 import vtk as V


def test_line_node_order():
    assert np.allclose(V.vtk_lagrange_line_nodes(1), [-1.0, 1.0])
    n2 = V.vtk_lagrange_line_nodes(2)
    assert n2[0] == -1 and n2[1] == 1 and n2[2] == 0
    n3 = V.vtk_lagrange_line_nodes(3)
    assert len(n3) == 4 and np.allclose(n3, [-1, 1, -1 + 2 / 3, -1 + 4 / 3])


def test_quad_node_order():
    assert V.vtk_lagrange_quad_nodes(1) == [(-1, -1), (1, -1), (1, 1), (-1, 1)]
    n2 = V.vtk_lagrange_quad_nodes(2)
    assert n2[4:] == [(0.0, -1.0), (1.0, 0.0), (0.0, 1.0), (-1.0, 0.0), (0.0, 0.0)]
    assert len(V.vtk_lagrange_quad_nodes(4)) == 25
    with pytest.raises(ValueError):
        V.vtk_lagrange_quad_nodes(0)


def test_point_counts():
    assert V.vtk_point_counts_1d(5, 3) == (20, 5, 4)
    assert V.vtk_point_counts_2d(6, 2) == (54, 6, 9)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_gl_to_equi_reproduces_polynomials(p):
    ops = F.build_operators(p)
    I = V.gl_to_equi_interp(ops)
    xe = V.vtk_lagrange_line_nodes(p)
    for k in range(p + 1):
        assert np.allclose(I @ (ops.xi ** k), xe ** k, atol=1e-12)


def test_write_1d_euler_density_wave(tmp_path):
    eq = F.Euler1D(1.4)
    ops = F.build_operators(2)
    mesh = F.Mesh1D(0.0, 1.0, 3, F.PeriodicBC(), F.PeriodicBC())
    st = F.allocate_state(mesh, ops, 3)
    F.set_initial_condition_(st, lambda x: eq.primitives_to_conserved(1 + 0.2 * np.sin(2 * np.pi * x), 1.0, 1.0))
    path = V.write_vtu_high_order(str(tmp_path / "euler.vtu"), st, eq)
    info = V.parse_vtu_basic(path)
    assert info["n_points"] == 9 and info["n_cells"] == 3
    assert info["types"] == [V.VTK_LAGRANGE_LINE] * 3
    assert info["connectivity"][:3] == [0, 1, 2] and len(info["connectivity"]) == 9
    for name in ("rho", "u", "p", "rho_u", "E"):
        assert f'Name="{name}"' in info["text"]


def test_discontinuous_points_keep_jumps(tmp_path):
    eq = F.Euler1D(1.4)
    ops = F.build_operators(1)
    mesh = F.Mesh1D(0.0, 1.0, 2, F.TransmissiveBC(), F.TransmissiveBC())
    st = F.allocate_state(mesh, ops, 3)
    F.set_initial_condition_(st, lambda x: eq.primitives_to_conserved(np.where(x < 0.5, 1.0, 0.125), 0.0,
                                                                       np.where(x < 0.5, 1.0, 0.1)))
    path = V.write_vtu_high_order(str(tmp_path / "jump.vtu"), st, eq)
    info = V.parse_vtu_basic(path)
    assert info["n_points"] == 4 and info["n_cells"] == 2
    rho = V.read_point_field(path, "rho")
    assert np.allclose(rho, [1.0, 1.0, 0.125, 0.125])  # duplicated interface nodes, one per side


@pytest.mark.parametrize("wavy", [None, 0.05])
def test_write_2d_polynomial_values(tmp_path, wavy):
    # rho is a polynomial of degree <= p in (xi, eta) on every element of an
    # affine mesh, so the values at the VTK nodes are exact; on the wavy mesh
    # the node coordinates follow the wavy map
    p = 3
    eq = F.Euler2D(1.4)
    ops = F.build_operators(p)
    bcs = [F.PeriodicBC() for _ in range(4)]
    mesh = F.make_wavy_mesh2d(4, 3, amp=wavy, left_bc=bcs[0], right_bc=bcs[1], bottom_bc=bcs[2],
                              top_bc=bcs[3]) if wavy else F.Mesh2D(0.0, 1.0, 0.0, 1.0, 4, 3, *bcs)
    st = F.allocate_state(mesh, ops, 4)
    X, Y = mesh.physical_coords(ops)
    Xa, Ya = F.Mesh2D(0.0, 1.0, 0.0, 1.0, 4, 3, *bcs).physical_coords(ops)  # reference-element coordinates
    poly = lambda x, y: 1.0 + 0.1 * x + 0.2 * y ** 2 + 0.05 * x * y ** 3  # noqa: E731
    st.u[...] = eq.primitives_to_conserved(poly(Xa, Ya), 0.3, -0.2, 1.0)
    path = V.write_vtu_high_order(str(tmp_path / "q.vtu"), st, eq)
    info = V.parse_vtu_basic(path)
    n_pts, n_cells, n_per = V.vtk_point_counts_2d(12, p)
    assert info["n_points"] == n_pts and info["types"] == [V.VTK_LAGRANGE_QUAD] * n_cells
    assert len(info["connectivity"]) == n_pts
    rho = V.read_point_field(path, "rho")
    u = V.read_point_field(path, "u")
    # affine node coordinates of every element, in VTK order
    nodes = V.vtk_lagrange_quad_nodes(p)
    xi = np.array([a for a, _ in nodes])
    eta = np.array([b for _, b in nodes])
    e = np.arange(12)
    xc = (np.arange(4) + 0.5) / 4
    yc = (np.arange(3) + 0.5) / 3
    xa = (xc[e % 4][None, :] + 0.125 * xi[:, None]).T.ravel()
    ya = (yc[e // 4][None, :] + (1.0 / 6.0) * eta[:, None]).T.ravel()
    assert np.allclose(rho, poly(xa, ya), atol=1e-12)
    assert np.allclose(u, 0.3, atol=1e-12)
    for name in ("rho", "u", "v", "p", "rho_u", "rho_v", "E"):
        assert f'Name="{name}"' in info["text"]
    assert "CellData" not in info["text"]


def test_cell_and_point_fields(tmp_path):
    eq = F.Euler2D(1.4)
    ops = F.build_operators(1)
    mesh = F.Mesh2D(0.0, 1.0, 0.0, 1.0, 2, 2, *[F.PeriodicBC() for _ in range(4)])
    st = F.allocate_state(mesh, ops, 4)
    st.u[...] = eq.primitives_to_conserved(1.0, 0.0, 0.0, 1.0)
    path = V.write_vtu_high_order(str(tmp_path / "c.vtu"), st, eq, cell_fields={"sensor": [0.0, 0.1, 0.2, 0.3]},
                                  point_fields={"extra": np.arange(16.0)})
    txt = open(path).read()
    assert "<CellData>" in txt and 'Name="sensor"' in txt and 'Name="extra"' in txt
    assert np.allclose(V.read_point_field(path, "sensor"), np.repeat([0.0, 0.1, 0.2, 0.3], 4))
    with pytest.raises(ValueError):
        V.write_vtu_high_order(str(tmp_path / "bad.vtu"), st, eq, cell_fields={"x": [1.0]})


@pytest.mark.gpu
def test_write_with_capturing_fields(tmp_path):
    from frforge_b200.workloads import four_quadrant_ic, four_quadrant_states

    eq = F.Euler2D(1.4)
    ops = F.build_operators(2)
    mesh = F.Mesh2D(0.0, 1.0, 0.0, 1.0, 6, 6, *[F.TransmissiveBC() for _ in range(4)])
    st = F.allocate_state(mesh, ops, 4)
    X, Y = mesh.physical_coords(ops)
    st.u[...] = four_quadrant_ic(X, Y, four_quadrant_states(3, 0.25))
    m = F.PerssonAVMethod(c_av=0.1)
    path = V.write_vtu_high_order_with_capturing(str(tmp_path / "cap.vtu"), st, eq, m)
    txt = open(path).read()
    assert 'Name="sensor"' in txt and 'Name="av"' in txt and 'Name="rho"' in txt
    sigma = np.zeros(36)
    F.sense_(sigma, m, st, eq)
    assert np.array_equal(V.read_point_field(path, "sensor")[::9], sigma)
    assert np.all(sigma >= 0)


def _points(text):
    import re

    m = re.search(r"<Points>\s*<DataArray[^>]*>(.*?)</DataArray>", text, re.S)
    return np.array([float(v) for v in m.group(1).split()])


def _field_close(a, b, tol=1e-14):
    scale = max(float(np.max(np.abs(b))), 1.0)
    return float(np.max(np.abs(a - b))) / scale <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("wavy", [None, 0.05])
def test_device_point_data_matches_host_2d(tmp_path, p, wavy):
    # the node coordinates, GL -> VTK-node interpolation and Euler point fields
    # evaluated on the device from the solve's state equal the host writer's
    from frforge_b200.workloads import four_quadrant_ic, four_quadrant_states

    eq = F.Euler2D(1.4)
    ops = F.build_operators(p)
    bcs = [F.PeriodicBC() for _ in range(4)]
    mesh = F.make_wavy_mesh2d(7, 5, amp=wavy, left_bc=bcs[0], right_bc=bcs[1], bottom_bc=bcs[2],
                              top_bc=bcs[3]) if wavy else F.Mesh2D(0.0, 1.0, 0.0, 1.0, 7, 5, *bcs)
    st = F.allocate_state(mesh, ops, 4)
    X, Y = mesh.physical_coords(ops)
    st.u[...] = four_quadrant_ic(X, Y, four_quadrant_states(5, 0.25))
    st.u[..., 0] *= 1.0 + 0.1 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    solve = F.GpuSolve(st, eq, F.NullCapturing())
    solve.upload(st.u, 0.0)
    host = V.write_vtu_high_order(str(tmp_path / "host.vtu"), st, eq)
    dev = V.write_vtu_high_order(str(tmp_path / "dev.vtu"), st, eq, solve=solve)
    hi, di = V.parse_vtu_basic(host), V.parse_vtu_basic(dev)
    assert hi["n_points"] == di["n_points"] and hi["types"] == di["types"]
    assert hi["connectivity"] == di["connectivity"]
    coords_h, _ = V.device_point_data(solve, st)  # also directly
    for name in ("rho", "u", "v", "p", "rho_u", "rho_v", "E"):
        assert _field_close(V.read_point_field(dev, name), V.read_point_field(host, name)), name
    assert _field_close(_points(di["text"]), _points(hi["text"]))
    assert coords_h.shape == (di["n_points"], 3)
    solve.close()


@pytest.mark.gpu
def test_device_point_data_matches_host_1d(tmp_path):
    eq = F.Euler1D(1.4)
    p = 3
    ops = F.build_operators(p)
    mesh = F.Mesh1D(0.0, 1.0, 40, F.TransmissiveBC(), F.TransmissiveBC())
    st = F.allocate_state(mesh, ops, 3)
    x = mesh.physical_coords(ops)
    st.u[...] = eq.primitives_to_conserved(1.0 + 0.3 * np.sin(2 * np.pi * x), 0.2 + 0 * x, 1.0 + 0.1 * x)
    solve = F.GpuSolve(st, eq, F.NullCapturing())
    solve.upload(st.u, 0.0)
    host = V.write_vtu_high_order(str(tmp_path / "h.vtu"), st, eq)
    dev = V.write_vtu_high_order(str(tmp_path / "d.vtu"), st, eq, solve=solve)
    for name in ("rho", "u", "p", "rho_u", "E"):
        assert _field_close(V.read_point_field(dev, name), V.read_point_field(host, name)), name
    assert V.parse_vtu_basic(dev)["connectivity"] == V.parse_vtu_basic(host)["connectivity"]
    solve.close()
