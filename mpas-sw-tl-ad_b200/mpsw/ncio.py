"""MPAS grid files and state trajectories in netCDF, for the drivers of the model.

The reference drivers read an MPAS grid / initial-condition file with netCDF4
(src/mpas_sw_driver.py:33-119: dimensions nCells, nEdges, nVertices, maxEdges, maxEdges2,
vertexDegree, optional nVertLevels; the connectivity and geometry variables assigned to the
module transposed), write the forward trajectory for the adjoint run (demo/run-fwd.py:51-64:
latCell, lonCell, latEdge, lonEdge in degrees; ux, uy, h on (nTime, nCell), u on (nTime, nEdge))
and read it back step by step (demo/run-adj.py:17-18, 44-45).  netCDF4 is not available here, so
this module uses ``scipy.io.netcdf_file``: netCDF classic and 64-bit-offset files (what MPAS
grid tools write by default); netCDF-4/HDF5 files are refused with a clear error.

* ``read_grid(path)``: the mesh as a dict in the layout of ``mpsw.mesh.icosahedral_mesh``
  (arrays as in the file, index arrays 1-based).
* ``load_grid(module, path_or_mesh)``: what ``read_dims`` + ``read_vars`` do to the module
  object (dimensions, ``var_allocation``, every mesh array, ``on_a_sphere``, ``sphere_radius``).
* ``write_grid(path, mesh)``: an MPAS grid file from a mesh dict (for example a generated
  icosahedral mesh), readable by MPAS tools and by ``read_grid``.
* ``TrajectoryWriter`` / ``read_trajectory``: the forward demo's output file.
"""
from __future__ import annotations

import os

import numpy as np

# dims of every mesh variable, as MPAS grid files declare them
GRID_VARS = {
    'latCell': ('nCells',), 'lonCell': ('nCells',), 'xCell': ('nCells',), 'yCell': ('nCells',),
    'zCell': ('nCells',), 'latEdge': ('nEdges',), 'lonEdge': ('nEdges',), 'xEdge': ('nEdges',),
    'yEdge': ('nEdges',), 'zEdge': ('nEdges',), 'latVertex': ('nVertices',),
    'lonVertex': ('nVertices',), 'xVertex': ('nVertices',), 'yVertex': ('nVertices',),
    'zVertex': ('nVertices',), 'cellsOnEdge': ('nEdges', 'TWO'), 'nEdgesOnCell': ('nCells',),
    'nEdgesOnEdge': ('nEdges',), 'edgesOnCell': ('nCells', 'maxEdges'),
    'edgesOnEdge': ('nEdges', 'maxEdges2'), 'weightsOnEdge': ('nEdges', 'maxEdges2'),
    'dvEdge': ('nEdges',), 'dcEdge': ('nEdges',), 'angleEdge': ('nEdges',),
    'areaCell': ('nCells',), 'areaTriangle': ('nVertices',), 'cellsOnCell': ('nCells', 'maxEdges'),
    'verticesOnCell': ('nCells', 'maxEdges'), 'verticesOnEdge': ('nEdges', 'TWO'),
    'edgesOnVertex': ('nVertices', 'vertexDegree'), 'cellsOnVertex': ('nVertices', 'vertexDegree'),
    'kiteAreasOnVertex': ('nVertices', 'vertexDegree'), 'meshDensity': ('nCells',),
}
INT_VARS = {'cellsOnEdge', 'nEdgesOnCell', 'nEdgesOnEdge', 'edgesOnCell', 'edgesOnEdge',
            'cellsOnCell', 'verticesOnCell', 'verticesOnEdge', 'edgesOnVertex', 'cellsOnVertex'}
DIMS = ('nCells', 'nEdges', 'nVertices', 'maxEdges', 'maxEdges2', 'vertexDegree')


def _open(path, mode='r'):
    from scipy.io import netcdf_file
    if mode == 'r':
        with open(path, 'rb') as f:
            magic = f.read(4)
        if magic[:3] != b'CDF':
            raise ValueError('%s is not a netCDF classic / 64-bit-offset file (netCDF-4/HDF5 files '
                             'need netCDF4, which is not installed)' % path)
        return netcdf_file(path, 'r', mmap=False)
    return netcdf_file(path, mode, version=2)


def _attr(f, name, default=None):
    v = f._attributes.get(name, default)
    return v.decode() if isinstance(v, bytes) else v


def read_grid(path: str) -> dict:
    """The mesh of an MPAS grid file (variables as stored, index arrays 1-based)."""
    with _open(path) as f:
        mesh = {d: int(f.dimensions[d]) for d in DIMS}
        mesh['nVertLevels'] = int(f.dimensions['nVertLevels']) if 'nVertLevels' in f.dimensions else 1
        for name in GRID_VARS:
            if name not in f.variables:
                if name == 'meshDensity':
                    mesh[name] = np.ones(mesh['nCells'])
                    continue
                raise KeyError('%s: variable %s missing' % (path, name))
            a = np.array(f.variables[name][:])
            mesh[name] = a.astype(np.int32) if name in INT_VARS else a.astype(np.float64)
        sphere = _attr(f, 'on_a_sphere', 'YES')
        mesh['on_a_sphere'] = str(sphere).strip().upper() == 'YES'
        mesh['sphere_radius'] = float(_attr(f, 'sphere_radius', 1.0))
    return mesh


def write_grid(path: str, mesh: dict, sphere_radius: float = 1.0) -> None:
    """Write ``mesh`` (a dict with the MPAS names) as an MPAS grid file."""
    with _open(path, 'w') as f:
        for d in DIMS:
            f.createDimension(d, int(mesh[d]))
        f.createDimension('TWO', 2)
        f.createDimension('nVertLevels', int(mesh.get('nVertLevels', 1)))
        f.on_a_sphere = b'YES'
        f.sphere_radius = float(sphere_radius)
        for name, dims in GRID_VARS.items():
            a = np.asarray(mesh[name])
            v = f.createVariable(name, 'i' if name in INT_VARS else 'd', dims)
            v[:] = a.astype(np.int32 if name in INT_VARS else np.float64)


def load_grid(module, grid, n_tracers: int = 1) -> dict:
    """Dimensions and mesh of an MPAS grid (a path or a ``read_grid`` dict) into the module
    object, as the reference driver's read_dims and read_vars do (src/mpas_sw_driver.py:33-119),
    including ``var_allocation``.  Returns the mesh dict."""
    mesh = read_grid(grid) if isinstance(grid, (str, os.PathLike)) else grid
    module.nvertlevels = int(mesh.get('nVertLevels', 1))
    module.ncells, module.nedges, module.nvertices = mesh['nCells'], mesh['nEdges'], mesh['nVertices']
    module.maxedges, module.maxedges2 = mesh['maxEdges'], mesh['maxEdges2']
    module.vertexdegree = mesh['vertexDegree']
    module.r3 = 3
    module.ntracers = n_tracers
    nC, nE, nV = mesh['nCells'], mesh['nEdges'], mesh['nVertices']
    for k, v in (('ncellssolve', nC), ('nedgessolve', nE), ('nverticessolve', nV), ('cellstart', 1),
                 ('cellend', nC), ('vertexstart', 1), ('vertexend', nV), ('edgestart', 1), ('edgeend', nE),
                 ('cellsolvestart', 1), ('cellsolveend', nC), ('vertexsolvestart', 1),
                 ('vertexsolveend', nV), ('edgesolvestart', 1), ('edgesolveend', nE)):
        setattr(module, k, v)
    module.var_allocation()
    module.on_a_sphere = True
    module.is_periodic = False
    module.sphere_radius = float(mesh.get('sphere_radius', 1.0))
    for name in GRID_VARS:
        setattr(module, name.lower(), np.asarray(mesh[name]).T)
    return mesh


class TrajectoryWriter:
    """Collects states at output times and writes the forward demo's file (demo/run-fwd.py:51-64):
    ``append(module)`` records uReconstructZonal, uReconstructMeridional, h and u of time level 1."""

    def __init__(self, path: str):
        self.path = path
        self.ux, self.uy, self.h, self.u = [], [], [], []
        self.lat = None

    def append(self, module) -> None:
        if self.lat is None:
            self.lat = (np.asarray(module.latcell).ravel().copy(), np.asarray(module.loncell).ravel().copy(),
                        np.asarray(module.latedge).ravel().copy(), np.asarray(module.lonedge).ravel().copy())
        self.ux.append(np.asarray(module.ureconstructzonal)[0].copy())
        self.uy.append(np.asarray(module.ureconstructmeridional)[0].copy())
        self.h.append(np.asarray(module.h)[0, 0].copy())
        self.u.append(np.asarray(module.u)[0, 0].copy())

    def write(self) -> None:
        if self.lat is None:
            raise ValueError('no states recorded')
        r2d = 180.0 / np.pi
        latc, lonc, late, lone = self.lat
        with _open(self.path, 'w') as f:
            f.createDimension('nCell', latc.size)
            f.createDimension('nTime', len(self.h))
            f.createDimension('nEdge', late.size)
            f.createVariable('latCell', 'f', ('nCell',))[:] = (latc * r2d).astype(np.float32)
            f.createVariable('lonCell', 'f', ('nCell',))[:] = (lonc * r2d).astype(np.float32)
            f.createVariable('ux', 'd', ('nTime', 'nCell'))[:] = np.array(self.ux)
            f.createVariable('uy', 'd', ('nTime', 'nCell'))[:] = np.array(self.uy)
            f.createVariable('h', 'd', ('nTime', 'nCell'))[:] = np.array(self.h)
            f.createVariable('latEdge', 'f', ('nEdge',))[:] = (late * r2d).astype(np.float32)
            f.createVariable('lonEdge', 'f', ('nEdge',))[:] = (lone * r2d).astype(np.float32)
            f.createVariable('u', 'd', ('nTime', 'nEdge'))[:] = np.array(self.u)


def read_trajectory(path: str) -> dict:
    """The variables of a trajectory file as arrays: ``u`` (nTime, nEdge), ``h`` (nTime, nCell),
    ``ux``, ``uy``, and the coordinates (degrees)."""
    with _open(path) as f:
        return {k: np.array(v[:]) for k, v in f.variables.items()}
