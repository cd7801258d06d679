"""Generate the golden vectors in this folder: ``golden_L{0,1,2,3}.npz``.

The reference ships no tests, fixtures or data, and its Fortran cannot be built without a
Fortran compiler, so its outputs cannot be recorded.  These fixtures are the oracle's outputs
(oracle/sw_oracle.c, a restatement of src/mpas_sw_dyncore*.f90 and the sw_rk4* drivers of
src/mpas_sw_module.f90) on the bisected-icosahedron meshes of levels 0-3, kept so that every
later change of the oracle, the mesh generator or the engine is checked against the same
numbers:

* ``mesh_sha256``: hash of the mesh arrays the drivers assign (connectivity and geometry);
* ``tc5_*``: Williamson test case 5 (src/mpas_sw_testcases.f90), dt = 600 s, no viscosity:
  the initial state, the state after 1 and after 12 calls of sw_rk4;
* ``seeded_*``: seeded balanced flow over seeded mountains with del2 + del4 viscosity and
  bottom drag, dt = 300 s: initial state and topography, one sw_rk4 step, one sw_rk4_tlm step
  of a seeded perturbation, one sw_rk4_adj step of a seeded adjoint, and the two inner
  products of link_tlm_adj (for the perturbation 1e-3 * state that it assumes).

Run from the repository root: ``python tests/golden/make_golden.py`` (rewrites the files).
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, 'mpas-sw-tl-ad_b200'), os.path.join(ROOT, 'oracle'),
          os.path.join(ROOT, 'tests')):
    if p not in sys.path:
        sys.path.insert(0, p)

LEVELS = (0, 1, 2, 3)
SEEDED_CFG = dict(dt=300.0, visc2=1.0e5, visc4=5.0e14, drag=True)
MESH_KEYS = ('cellsOnEdge', 'verticesOnEdge', 'edgesOnEdge', 'nEdgesOnEdge', 'weightsOnEdge',
             'edgesOnCell', 'nEdgesOnCell', 'cellsOnCell', 'verticesOnCell', 'cellsOnVertex',
             'edgesOnVertex', 'kiteAreasOnVertex', 'dcEdge', 'dvEdge', 'areaCell',
             'areaTriangle', 'angleEdge', 'xCell', 'yCell', 'zCell', 'latCell', 'lonCell')


def path(level: int) -> str:
    return os.path.join(HERE, 'golden_L%d.npz' % level)


def mesh_hash(mesh: dict) -> str:
    h = hashlib.sha256()
    for k in MESH_KEYS:
        a = np.ascontiguousarray(mesh[k])
        h.update(k.encode())
        h.update(str(a.dtype).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def perturbation(level: int, m, seed: int):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(int(m.nedges)) * 0.1, rng.standard_normal(int(m.ncells)))


def compute(make_module, level: int, inputs: dict | None = None) -> dict:
    """Run the golden cases on a fresh module from `make_module()` (oracle or engine shim).
    With `inputs` (a loaded golden file) the initial states are taken from it instead of being
    regenerated, so the dynamics are checked on exactly the recorded inputs."""
    from helpers import mesh, setup
    out = {'mesh_sha256': np.array(mesh_hash(mesh(level)))}

    m = setup(make_module(), level, 'tc5', dt=600.0)
    if inputs is not None:
        m.u[0, 0] = inputs['tc5_u0']
        m.h[0, 0] = inputs['tc5_h0']
    out['tc5_u0'], out['tc5_h0'] = m.u[0, 0].copy(), m.h[0, 0].copy()
    m.sw_rk4()
    out['tc5_u1'], out['tc5_h1'] = m.u[0, 0].copy(), m.h[0, 0].copy()
    for _ in range(11):
        m.sw_rk4()
    out['tc5_u12'], out['tc5_h12'] = m.u[0, 0].copy(), m.h[0, 0].copy()

    m = setup(make_module(), level, 'seeded', tl=True, ad=True, **SEEDED_CFG)
    if inputs is not None:
        m.h_s = inputs['seeded_hs'][None, :]
        m.u[0, 0] = inputs['seeded_u0']
        m.h[0, 0] = inputs['seeded_h0']
    u0, h0 = m.u[0, 0].copy(), m.h[0, 0].copy()
    out['seeded_u0'], out['seeded_h0'] = u0, h0
    out['seeded_hs'] = np.asarray(m.h_s).reshape(-1).copy()
    m.sw_rk4()
    out['seeded_u1'], out['seeded_h1'] = m.u[0, 0].copy(), m.h[0, 0].copy()

    du, dh = perturbation(level, m, 11) if inputs is None else (inputs['seeded_du'], inputs['seeded_dh'])
    out['seeded_du'], out['seeded_dh'] = du, dh
    m.u[0, 0], m.h[0, 0] = u0, h0
    m.u_tl[0, 0], m.h_tl[0, 0] = du, dh
    m.sw_rk4_tlm()
    out['seeded_utl1'], out['seeded_htl1'] = m.u_tl[0, 0].copy(), m.h_tl[0, 0].copy()

    au, ah = perturbation(level, m, 12) if inputs is None else (inputs['seeded_au'], inputs['seeded_ah'])
    out['seeded_au'], out['seeded_ah'] = au, ah
    m.u[0, 0], m.h[0, 0] = u0, h0
    m.u_ad[0, 0], m.h_ad[0, 0] = au, ah
    m.sw_rk4_adj()
    out['seeded_uad0'], out['seeded_had0'] = m.u_ad[0, 0].copy(), m.h_ad[0, 0].copy()

    # link_tlm_adj forms its RHS with the perturbation 1e-3 * state (src/mpas_sw_module.f90:1210)
    # and accumulates into u_ad(1), h_ad(1), which must start at zero
    m.u[0, 0], m.h[0, 0] = u0, h0
    m.u_tl[0, 0], m.h_tl[0, 0] = u0 * 1.0e-3, h0 * 1.0e-3
    m.u_ad[...] = 0.0
    m.h_ad[...] = 0.0
    lhs, rhs = m.link_tlm_adj()
    out['seeded_link'] = np.array([lhs, rhs])
    return out


def main():
    import oracle as O
    O.build()
    for level in LEVELS:
        res = compute(O.OracleModule, level)
        np.savez_compressed(path(level), **res)
        print('wrote', os.path.relpath(path(level), ROOT), '(%d arrays)' % len(res))


if __name__ == '__main__':
    main()
