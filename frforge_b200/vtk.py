"""High-order VTU output of a solution state (src/io/VTKHighOrder.jl).

Discontinuous VTK XML UnstructuredGrid files with Lagrange cells, as the
reference writes them:

* 1D: VTK_LAGRANGE_LINE (68) cells of p+1 equispaced nodes in VTK order
  (vertices, then interiors), values interpolated from the GL solution points
  (``gl_to_equi_interp``, VTKHighOrder.jl:8-41); point fields rho, u, p,
  rho_u, E (VTKHighOrder.jl:55-213).
* 2D: VTK_LAGRANGE_QUAD (70) cells of (p+1)^2 nodes in VTK order (corners,
  edge interiors bottom / right / top / left, then the face interior),
  coordinates from physical_xy including the wavy map, point fields rho, u,
  v, p, rho_u, rho_v, E and optional point / cell fields
  (VTKHighOrder.jl:265-488); ``write_vtu_high_order_with_capturing`` adds the
  element sensor and artificial viscosity (VTKHighOrder.jl:492-574), with the
  sensor evaluated on the GPU.

Every element owns its nodes (face nodes duplicated), so jumps between
elements are kept.  Values are written in the shortest decimal form that
reads back to the same double.

With ``solve=`` (a GpuSolve of the state), the node coordinates, the
interpolation and the Euler point fields are evaluated on the device from
the solve's current state (frg_vtk_point_data); only the node data is
downloaded.
"""
from __future__ import annotations

import os
import re
from typing import Dict, Optional

import numpy as np

from .equations import EPS, Euler1D, Euler2D

VTK_LAGRANGE_LINE = 68
VTK_LAGRANGE_QUAD = 70


def vtk_lagrange_line_nodes(p: int) -> np.ndarray:
    """Equispaced nodes on [-1, 1] in VTK Lagrange line order: the two
    vertices, then the interior nodes left to right (VTKHighOrder.jl:8-27)."""
    if p < 0:
        raise ValueError("p must be >= 0")
    if p == 0:
        return np.zeros(1)
    nodes = [-1.0, 1.0] + [-1.0 + 2.0 * k / p for k in range(1, p)]
    return np.array(nodes)


def vtk_lagrange_quad_nodes(p: int):
    """(xi, eta) nodes on [-1, 1]^2 in VTK Lagrange quad order: corners SW,
    SE, NE, NW; edge interiors bottom (xi up), right (eta up), top (xi down),
    left (eta down); face interior with xi fastest (VTKHighOrder.jl:239-286)."""
    if p < 1:
        raise ValueError("p >= 1 for quads")
    nodes = [(-1.0, -1.0), (1.0, -1.0), (1.0, 1.0), (-1.0, 1.0)]
    if p >= 2:
        inner = [-1.0 + 2.0 * k / p for k in range(1, p)]
        nodes += [(x, -1.0) for x in inner]
        nodes += [(1.0, y) for y in inner]
        nodes += [(1.0 - 2.0 * k / p, 1.0) for k in range(1, p)]
        nodes += [(-1.0, 1.0 - 2.0 * k / p) for k in range(1, p)]
        nodes += [(-1.0 + 2.0 * ii / p, -1.0 + 2.0 * jj / p) for jj in range(1, p) for ii in range(1, p)]
    return nodes


def vtk_point_counts_1d(n_elements: int, p: int):
    return n_elements * (p + 1), n_elements, p + 1


def vtk_point_counts_2d(n_elements: int, p: int):
    n_per = (p + 1) ** 2
    return n_elements * n_per, n_elements, n_per


def lagrange_at(xi: np.ndarray, x: float) -> np.ndarray:
    """Values of the Lagrange basis on the nodes xi at the point x."""
    xi = np.asarray(xi, dtype=np.float64)
    out = np.ones(len(xi))
    for j in range(len(xi)):
        for m in range(len(xi)):
            if m != j:
                out[j] *= (x - xi[m]) / (xi[j] - xi[m])
    return out


def gl_to_equi_interp(ops) -> np.ndarray:
    """I with u_equi = I u_GL at the VTK line nodes (VTKHighOrder.jl:29-41)."""
    return np.stack([lagrange_at(ops.xi, x) for x in vtk_lagrange_line_nodes(ops.p)])


def _fmt(values) -> str:
    return " ".join(repr(float(v)) for v in np.asarray(values, dtype=np.float64).ravel())


def _write(path, coords, n_cells, n_per, cell_type, fields, names, cell_data=None):
    n_points = coords.shape[0]
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    conn = np.arange(n_points, dtype=np.int64).reshape(n_cells, n_per)
    with open(path, "w") as f:
        w = f.write
        w('<?xml version="1.0"?>\n')
        w('<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">\n')
        w("  <UnstructuredGrid>\n")
        w(f'    <Piece NumberOfPoints="{n_points}" NumberOfCells="{n_cells}">\n')
        w("      <Points>\n")
        w('        <DataArray type="Float64" NumberOfComponents="3" format="ascii">\n')
        for row in coords:
            w("          " + _fmt(row) + "\n")
        w("        </DataArray>\n")
        w("      </Points>\n")
        w("      <Cells>\n")
        w('        <DataArray type="Int32" Name="connectivity" format="ascii">\n')
        for row in conn:
            w("          " + " ".join(str(int(v)) for v in row) + "\n")
        w("        </DataArray>\n")
        w('        <DataArray type="Int32" Name="offsets" format="ascii">\n')
        w("          " + " ".join(str(n_per * (e + 1)) for e in range(n_cells)) + "\n")
        w("        </DataArray>\n")
        w('        <DataArray type="UInt8" Name="types" format="ascii">\n')
        w("          " + " ".join([str(cell_type)] * n_cells) + "\n")
        w("        </DataArray>\n")
        w("      </Cells>\n")
        w(f'      <PointData Scalars="{names[0]}">\n')
        for name in names:
            w(f'        <DataArray type="Float64" Name="{name}" format="ascii">\n')
            w("          " + _fmt(fields[name]) + "\n")
            w("        </DataArray>\n")
        w("      </PointData>\n")
        if cell_data:
            w("      <CellData>\n")
            for name in sorted(cell_data):
                w(f'        <DataArray type="Float64" Name="{name}" format="ascii">\n')
                w("          " + _fmt(cell_data[name]) + "\n")
                w("        </DataArray>\n")
            w("      </CellData>\n")
        w("    </Piece>\n")
        w("  </UnstructuredGrid>\n")
        w("</VTKFile>\n")
    return path


def _physical_xy(mesh, xi: np.ndarray, eta: np.ndarray):
    """physical_xy (MeshMetrics2D.jl:49-74) of reference points (xi, eta) in
    every element: arrays [n_nodes, Nel]."""
    xc = (mesh.x_vertices[:-1] + mesh.x_vertices[1:]) / 2.0
    yc = (mesh.y_vertices[:-1] + mesh.y_vertices[1:]) / 2.0
    e = np.arange(mesh.n_elements)
    jx, jy = e % mesh.nx, e // mesh.nx
    X = xc[jx][None, :] + mesh.Jx[jx][None, :] * xi[:, None]
    Y = yc[jy][None, :] + mesh.Jy[jy][None, :] * eta[:, None]
    if getattr(mesh, "wavy_amp", None) is not None:
        a = mesh.wavy_amp
        return X + a * np.sin(2 * np.pi * Y) * np.sin(np.pi * X), Y + a * np.sin(2 * np.pi * X) * np.sin(np.pi * Y)
    return X, Y


def device_point_data(solve, state):
    """(coords [n_points, 3], {field: values}) of the VTU nodes, evaluated on
    the device from the solve's current state (frg_vtk_point_data)."""
    import ctypes as C

    from . import _lib as L

    p = state.ops.p
    if state.dim == 1:
        xi = vtk_lagrange_line_nodes(p)
        eta = None
        names = ["rho", "u", "p", "rho_u", "E"]
    else:
        nodes = vtk_lagrange_quad_nodes(p)
        xi = np.array([a for a, _ in nodes])
        eta = np.ascontiguousarray([b for _, b in nodes], dtype=np.float64)
        names = ["rho", "u", "v", "p", "rho_u", "rho_v", "E"]
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    n_per = xi.size
    n_pts = state.mesh.n_elements * n_per
    nc = 1 if state.dim == 1 else 2
    xy = np.empty(nc * n_pts)
    f = np.empty(len(names) * n_pts)
    L.check(L.load().frg_vtk_point_data(solve.handle, n_per, L.dptr(xi), L.dptr(eta) if eta is not None else None,
                                        L.dptr(xy), L.dptr(f), n_pts), solve.ctx.handle, "frg_vtk_point_data")
    coords = np.zeros((n_pts, 3))
    coords[:, 0] = xy[:n_pts]
    if nc == 2:
        coords[:, 1] = xy[n_pts:]
    return coords, {n: f[k * n_pts:(k + 1) * n_pts] for k, n in enumerate(names)}


def write_vtu_high_order(path: str, state, eq, cell_fields: Optional[Dict[str, np.ndarray]] = None,
                         point_fields: Optional[Dict[str, np.ndarray]] = None, solve=None) -> str:
    """write_vtu_high_order(path, state, eq; cell_fields, point_fields); with
    solve= the point data comes from the device state of that GpuSolve."""
    ops, mesh = state.ops, state.mesh
    p = ops.p
    if solve is not None and isinstance(eq, (Euler1D, Euler2D)):
        coords, fields = device_point_data(solve, state)
        names = list(fields)
        n_per = p + 1 if state.dim == 1 else (p + 1) ** 2
        Nel = mesh.n_elements
        n_pts = Nel * n_per
        for name, vec in (point_fields or {}).items():
            vec = np.asarray(vec, dtype=np.float64).ravel()
            if vec.size != n_pts:
                raise ValueError(f"point field {name} length {vec.size} != n_pts {n_pts}")
            fields[name] = vec
        cell_data = {}
        for name, vec in (cell_fields or {}).items():
            vec = np.asarray(vec, dtype=np.float64).ravel()
            if vec.size != Nel:
                raise ValueError(f"cell field {name} length {vec.size} != Nel {Nel}")
            cell_data[name] = vec
            fields[name] = np.repeat(vec, n_per)
        names = names + sorted(n for n in fields if n not in names)
        ctype = VTK_LAGRANGE_LINE if state.dim == 1 else VTK_LAGRANGE_QUAD
        return _write(path, coords, Nel, n_per, ctype, fields, names, cell_data or None)
    if state.dim == 1:
        Nel = mesh.n_elements
        I = gl_to_equi_interp(ops)
        xe = vtk_lagrange_line_nodes(p)
        mid = (mesh.x_vertices[:-1] + mesh.x_vertices[1:]) / 2.0
        x = (mid[None, :] + mesh.J[None, :] * xe[:, None]).T.ravel()  # [Nel*(p+1)], element-major
        U = np.einsum("ak,kec->eac", I, state.u).reshape(-1, state.u.shape[-1])
        coords = np.stack([x, np.zeros_like(x), np.zeros_like(x)], axis=1)
        fields = {}
        names = ["u"]
        if isinstance(eq, Euler1D):
            rho, ru, E = U[:, 0], U[:, 1], U[:, 2]
            fields = {"rho": rho, "u": ru / np.maximum(rho, EPS), "p": eq.pressure(U), "rho_u": ru, "E": E}
            names = ["rho", "u", "p", "rho_u", "E"]
        else:
            fields = {"u": U[:, 0]}
        return _write(path, coords, Nel, p + 1, VTK_LAGRANGE_LINE, fields, names)

    nodes = vtk_lagrange_quad_nodes(p)
    n_per = len(nodes)
    Nel = mesh.n_elements
    xi = np.array([a for a, _ in nodes])
    eta = np.array([b for _, b in nodes])
    Lx = np.stack([lagrange_at(ops.xi, a) for a in xi])   # [n_per, Np]
    Ly = np.stack([lagrange_at(ops.xi, b) for b in eta])  # [n_per, Np]
    X, Y = _physical_xy(mesh, xi, eta)
    # U[a, e, c] = sum_ij u[i, j, e, c] l_i(xi_a) l_j(eta_a)
    U = np.einsum("ai,aj,ijec->eac", Lx, Ly, state.u).reshape(-1, state.u.shape[-1])
    coords = np.stack([X.T.ravel(), Y.T.ravel(), np.zeros(Nel * n_per)], axis=1)
    n_pts = Nel * n_per
    if isinstance(eq, Euler2D):
        rho = U[:, 0]
        r = np.maximum(rho, EPS)
        fields = {"rho": rho, "u": U[:, 1] / r, "v": U[:, 2] / r, "p": eq.pressure(U), "rho_u": U[:, 1],
                  "rho_v": U[:, 2], "E": U[:, 3]}
        names = ["rho", "u", "v", "p", "rho_u", "rho_v", "E"]
    else:
        fields = {"u": U[:, 0]}
        names = ["u"]
    for name, vec in (point_fields or {}).items():
        vec = np.asarray(vec, dtype=np.float64).ravel()
        if vec.size != n_pts:
            raise ValueError(f"point field {name} length {vec.size} != n_pts {n_pts}")
        fields[name] = vec
    cell_data = {}
    for name, vec in (cell_fields or {}).items():
        vec = np.asarray(vec, dtype=np.float64).ravel()
        if vec.size != Nel:
            raise ValueError(f"cell field {name} length {vec.size} != Nel {Nel}")
        cell_data[name] = vec
        fields[name] = np.repeat(vec, n_per)  # also on the points, for coloring
    names = names + sorted(n for n in fields if n not in names)
    return _write(path, coords, Nel, n_per, VTK_LAGRANGE_QUAD, fields, names, cell_data)


def element_viscosities_2d(state, eq, sigma: np.ndarray, c_av: float) -> np.ndarray:
    """eps_e = c_av sigma_e (h_e / max(p, 1)) lambda_e with lambda_e the
    largest max(|u| + c, |v| + c) of the element (PerssonAV2D.jl:89-109)."""
    U = state.u
    r = np.maximum(U[..., 0], EPS)
    u, v = U[..., 1] / r, U[..., 2] / r
    pr = np.maximum(eq.pressure(U), EPS)
    c = np.sqrt(eq.gamma * pr / r)
    lam = np.maximum(np.max(np.maximum(np.abs(u) + c, np.abs(v) + c), axis=(0, 1)), EPS)
    if state.metrics is not None and "h_char" in state.metrics:
        h = np.asarray(state.metrics["h_char"], dtype=np.float64).ravel()
    else:
        m = state.mesh
        e = np.arange(m.n_elements)
        h = np.minimum(m.dx[e % m.nx], m.dy[e // m.nx])
    eps = c_av * sigma * (h / max(state.ops.p, 1)) * lam
    return np.where(sigma > 0.0, eps, 0.0)


def write_vtu_high_order_with_capturing(path: str, state, eq, method) -> str:
    """2D VTU with the element sensor and artificial viscosity as cell fields
    (VTKHighOrder.jl:540-574); the sensor runs on the GPU."""
    from .gpu import sense_

    sigma = np.zeros(state.mesh.n_elements)
    sense_(sigma, method, state, eq)
    spec = method.gpu_spec()
    eps = element_viscosities_2d(state, eq, sigma, spec["c_av"]) if spec["method"] == "persson" else \
        np.zeros_like(sigma)
    return write_vtu_high_order(path, state, eq, cell_fields={"sensor": sigma, "av": eps})


def parse_vtu_basic(path: str) -> dict:
    """Point / cell counts, cell types and connectivity of a VTU written here
    (parse_vtu_basic, VTKHighOrder.jl:215-237)."""
    txt = open(path).read()
    m_pts = re.search(r'NumberOfPoints="(\d+)"', txt)
    m_cells = re.search(r'NumberOfCells="(\d+)"', txt)
    tm = re.search(r'Name="types"[^>]*>(.*?)</DataArray>', txt, re.S)
    cm = re.search(r'Name="connectivity"[^>]*>(.*?)</DataArray>', txt, re.S)
    return {"n_points": int(m_pts.group(1)) if m_pts else -1, "n_cells": int(m_cells.group(1)) if m_cells else -1,
            "types": [int(t) for t in tm.group(1).split()] if tm else [],
            "connectivity": [int(t) for t in cm.group(1).split()] if cm else [], "text": txt}


def read_point_field(path: str, name: str) -> np.ndarray:
    txt = open(path).read()
    m = re.search(rf'Name="{name}" format="ascii">(.*?)</DataArray>', txt, re.S)
    return np.array([float(t) for t in m.group(1).split()])
