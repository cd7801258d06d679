"""Leading singular vectors of the window's tangent-linear propagator (the use the reference's
papers make of the TL and AD models: optimal perturbations over a forecast window).

For the window's propagator M (initial perturbation -> final perturbation, both in the engine's
internal order: nEdges u values then nCells h values) and a diagonal norm D^2 (weights w > 0 on
both ends, identity by default), the leading singular values and right singular vectors of
D M D^-1 are found by block Lanczos on A = D^-1 M^T D^2 M D^-1: each Krylov block costs one
batched tangent-linear sweep and one batched adjoint sweep over its B members (B on the
trailing dimension); the basis is kept orthonormal by full reorthogonalisation, and a
Rayleigh-Ritz step over the whole basis gives the singular values.  New: the reference has no
such driver.
"""
from __future__ import annotations

import torch

from .torch_api import FP64


def _apply(window, x, precision, d):
    """A x for a block x of shape [n, b] (float64, CUDA): D^-1 M^T D^2 M D^-1 x."""
    e = window.e
    nE = e.nE
    z = x / d[:, None]
    du = z[:nE].contiguous()
    dh = z[nE:].contiguous()
    window.tl_internal(du, dh, precision)
    y = torch.cat([du, dh]) * (d * d)[:, None]
    au = y[:nE].contiguous()
    ah = y[nE:].contiguous()
    window.ad_internal(au, ah, precision)
    return torch.cat([au, ah]) / d[:, None]


def leading_singular_vectors(window, k: int = 4, block: int = 8, steps: int = 10,
                             precision: int = FP64, weights=None, seed: int = 0):
    """The k leading singular values (descending) and right singular vectors ([n, k], internal
    order, orthonormal in the coordinates D x) of the window's tangent-linear propagator, from a
    block Krylov space of ``steps`` blocks of ``block`` members.  ``weights``: optional [n]
    tensor of the diagonal norm."""
    e = window.e
    n = e.nE + e.nC
    dev = torch.device('cuda')
    d = torch.ones(n, dtype=torch.float64, device=dev) if weights is None else \
        torch.as_tensor(weights, dtype=torch.float64, device=dev).sqrt()
    if torch.any(d <= 0):
        raise ValueError('weights must be positive')
    g = torch.Generator(device='cpu').manual_seed(seed)
    q = torch.linalg.qr(torch.randn(n, block, generator=g, dtype=torch.float64).to(dev))[0]
    basis, images = [], []
    for _ in range(steps):
        z = _apply(window, q, precision, d)
        basis.append(q)
        images.append(z)
        if sum(b.shape[1] for b in basis) >= n:
            break
        kb = torch.cat(basis, dim=1)
        w = z - kb @ (kb.T @ z)
        w = w - kb @ (kb.T @ w)  # second pass keeps the basis orthonormal to rounding
        q = torch.linalg.qr(w)[0]
    kb, ak = torch.cat(basis, dim=1), torch.cat(images, dim=1)
    h = kb.T @ ak
    lam, v = torch.linalg.eigh(0.5 * (h + h.T))
    order = torch.argsort(lam, descending=True)[:k]
    sigma = torch.sqrt(torch.clamp(lam[order], min=0.0))
    return sigma, kb @ v[:, order]
