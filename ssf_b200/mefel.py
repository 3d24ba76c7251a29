"""Host-side mirror of the MEFEL / TRFEL assembly entry points on the GPU.

* ``stiffness_matrix(mesh)`` -- MEFEL/SRC/globmat.cpp:41: element loop +
  localisation, here one call of ``sgpu_assemble`` (pattern, colouring,
  batched integration and scatter on the device);
* ``conductivity_matrix`` / ``capacity_matrix`` -- TRFEL/SRC/globmatt.cpp:19/92;
* ``mefel_right_hand_side(mesh, lc)`` -- globmat.cpp:2369 for nodal loads
  (loadcase::assemble, MEFEL/SRC/loadcase.cpp:400);
* ``solve_linear_statics(mesh, ...)`` -- MEFEL/SRC/lssolver.cpp:31-80:
  assemble once, solve every load case.

Meshes are :class:`ssf_b200.decks.Mesh` objects (nodes, elements, constraint
flags, materials and loads as a SIFEL deck describes them).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .gefel import DeviceMatrix, Result

KIND = {"hex8": L.ELEM_HEX8, "quad4": L.ELEM_QUAD4, "hex8t_k": L.ELEM_HEX8T_K, "hex8t_c": L.ELEM_HEX8T_C}


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _assemble(mesh, kind: str, rho=None):
    coords = _c(mesh.coords, np.float64)
    elems = _c(mesh.elems, np.int64)
    cn = _c(mesh.code_numbers(), np.int64)
    emat = _c(mesh.mats[mesh.emat], np.float64)
    thick = _c(mesh.thick, np.float64) if mesh.thick is not None else None
    rr = _c(rho, np.float64) if rho is not None else None
    keep = (coords, elems, cn, emat, thick, rr)
    m = L.Mesh(KIND[kind], cn.shape[1], coords.shape[0], coords.ctypes.data, elems.shape[0], elems.ctypes.data,
               cn.ctypes.data, emat.ctypes.data, thick.ctypes.data if thick is not None else None,
               rr.ctypes.data if rr is not None else None)
    h = C.c_void_p()
    info = L.AssemblyInfo()
    L.check(L.lib().sgpu_assemble(C.byref(m), C.byref(h), C.byref(info)))
    del keep
    dm = DeviceMatrix.from_handle(h, info.n, 1)
    dm.assembly = info.as_dict()
    return dm


def stiffness_matrix(mesh) -> DeviceMatrix:
    """Global stiffness matrix of a hex8 / quad4 mesh, assembled on the GPU."""
    return _assemble(mesh, mesh.kind)


def conductivity_matrix(mesh) -> DeviceMatrix:
    return _assemble(mesh, "hex8t_k")


def capacity_matrix(mesh, rho=None) -> DeviceMatrix:
    return _assemble(mesh, "hex8t_c", rho)


def mefel_right_hand_side(mesh, lc: int = 0) -> np.ndarray:
    """Nodal forces of load case ``lc`` in equation order."""
    cn = mesh.code_numbers().reshape(-1)
    f = np.zeros(mesh.ndof)
    vals = mesh.loads[lc].reshape(-1)
    m = cn > 0
    np.add.at(f, cn[m] - 1, vals[m])
    return f


def solve_linear_statics(mesh, ni=100000, res=1e-20, mode="fp64"):
    """Assemble K once, then solve every load case (lssolver.cpp:78-80)."""
    K = stiffness_matrix(mesh)
    out, results = [], []
    try:
        for lc in range(mesh.loads.shape[0]):
            f = mefel_right_hand_side(mesh, lc)
            x, r = K.pcg(f, ni=ni, res=res, crit="scr", prec=1, mode=mode)
            out.append(x)
            results.append(r)
    finally:
        K.close()
    return np.stack(out), results
