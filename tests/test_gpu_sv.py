"""Singular vectors of the window's tangent-linear propagator (mpsw/sv.py) against a dense SVD
of the propagator built column by column with one batched tangent-linear sweep of every unit
vector (level-2 mesh, 642 unknowns)."""
import numpy as np
import pytest

from helpers import setup
from module_sw_mpas import MpasSwModule

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


def test_leading_singular_vectors_match_dense_svd():
    from mpsw.sv import leading_singular_vectors
    from mpsw.torch_api import Engine
    m = setup(MpasSwModule(), 2, 'seeded', tl=True, ad=True, dt=600.0)
    e = Engine(m)
    w = e.window(6, ckpt_every=3)
    n = e.nE + e.nC
    eye = torch.eye(n, dtype=torch.float64, device='cuda')
    du, dh = eye[:e.nE].contiguous(), eye[e.nE:].contiguous()
    w.tl_internal(du, dh)
    M = torch.cat([du, dh]).cpu().numpy()            # column j = M e_j
    s_dense = np.linalg.svd(M, compute_uv=False)
    sigma, vecs = leading_singular_vectors(w, k=4, block=8, steps=40)
    sigma = sigma.cpu().numpy()
    assert np.allclose(sigma, s_dense[:4], rtol=1e-8), (sigma, s_dense[:4])
    V = vecs.cpu().numpy()
    assert np.allclose(V.T @ V, np.eye(4), atol=1e-10)
    assert np.allclose(np.linalg.norm(M @ V, axis=0), sigma, rtol=1e-8)
