"""PyTorch front end of the engine: device-resident batched windows and the RK4 step as a
``torch.autograd.Function`` whose backward is the engine's adjoint step.

All tensors are CUDA float64 in the reference numbering: edges ``[nEdges, B]`` for u and
cells ``[nCells, B]`` for h (members on the trailing dimension).  PyTorch provides device
memory and the stream; the arithmetic runs in libmpsw.so's kernels.
"""
from __future__ import annotations

import ctypes

import torch

from ._lib import Handle

FP64, FP32 = 0, 1
_CELL, _EDGE = 0, 1


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check_member(t: torch.Tensor, n: int, what: str) -> torch.Tensor:
    if not (t.is_cuda and t.dtype == torch.float64):
        raise TypeError(f'{what} must be a CUDA float64 tensor')
    if t.dim() == 1:
        t = t.unsqueeze(1)
    if t.shape[0] != n:
        raise ValueError(f'{what}: expected {n} rows, got {tuple(t.shape)}')
    return t.contiguous()


class Engine:
    """Device-side access to one module instance (an ``mpas_sw_module`` after
    ``sw_mpas_init_block``)."""

    def __init__(self, module):
        module.sync()
        self.module = module
        self.h: Handle = module.handle
        self.nC = int(module.ncells)
        self.nE = int(module.nedges)

    # ---- layout -------------------------------------------------------------------------
    def to_internal(self, x: torch.Tensor, kind: int, out: torch.Tensor | None = None) -> torch.Tensor:
        """x in the reference numbering -> internal order (into `out` when given: a contiguous
        CUDA float64 tensor of x's shape, so a repeated call allocates nothing)."""
        return self._permute('mpsw_to_internal', x, kind, out)

    def to_reference(self, x: torch.Tensor, kind: int, out: torch.Tensor | None = None) -> torch.Tensor:
        return self._permute('mpsw_to_reference', x, kind, out)

    def _permute(self, fn, x, kind, out):
        n = self.nE if kind == _EDGE else self.nC
        x = _check_member(x, n, 'input')
        if out is None:
            out = torch.empty_like(x)
        elif out.shape != x.shape or out.dtype != torch.float64 or not out.is_cuda or not out.is_contiguous():
            raise ValueError(f'out must be a contiguous CUDA float64 tensor of shape {tuple(x.shape)}')
        self.h.call(fn, kind, x.shape[1], _ptr(x), _ptr(out), _stream())
        return out

    # ---- state ---------------------------------------------------------------------------
    def set_state(self, u: torch.Tensor, h: torch.Tensor) -> None:
        u = _check_member(u, self.nE, 'u')
        h = _check_member(h, self.nC, 'h')
        self.h.call('mpsw_state_from_device', _ptr(u), _ptr(h), _stream())
        self.module.__dict__['_stale'].update({'u', 'h'})

    def get_state(self):
        u = torch.empty(self.nE, dtype=torch.float64, device='cuda')
        h = torch.empty(self.nC, dtype=torch.float64, device='cuda')
        self.h.call('mpsw_state_to_device', _ptr(u), _ptr(h), _stream())
        return u, h

    # ---- windows -------------------------------------------------------------------------
    def window(self, nsteps: int, ckpt_every: int = 16, storage: int = -1,
               max_bytes: float = 0.0, snapshots: int = 0) -> 'Window':
        return Window(self, nsteps, ckpt_every, storage, max_bytes, snapshots)


class Window:
    """``nsteps`` RK4 steps from the engine's current state, checkpointed every
    ``ckpt_every`` steps; batched tangent-linear and adjoint sweeps over it.

    ``storage`` selects whether every RK stage's linearisation point is also kept in device
    memory (``mpsw_window_storage``): -1 automatic (within ``max_bytes``, 0 = 40% of free
    memory), 0 checkpoints only, 1 FP64, 2 FP32, 3 both.  ``snapshots`` > 0 reverses a window
    whose stages are not stored by binomial checkpointing with that many snapshot states
    (``mpsw_window_snapshots``) instead of checkpoints every ``ckpt_every`` steps.  Results do
    not depend on either."""

    def __init__(self, engine: Engine, nsteps: int, ckpt_every: int = 16, storage: int = -1,
                 max_bytes: float = 0.0, snapshots: int = 0):
        self.e = engine
        self.nsteps = nsteps
        engine.module.sync()  # pending host-side edits of the module's state first
        engine.h.call('mpsw_window_storage', int(storage), float(max_bytes))
        engine.h.call('mpsw_window_snapshots', int(snapshots))
        engine.h.call('mpsw_window_init', int(nsteps), int(ckpt_every), _stream())

    def forward_steps(self) -> int:
        """Nonlinear steps the last adjoint sweep recomputed to re-form states."""
        import ctypes
        n = ctypes.c_longlong()
        self.e.h.call('mpsw_window_forward_steps', ctypes.byref(n))
        return n.value

    def final_state(self):
        u = torch.empty(self.e.nE, 1, dtype=torch.float64, device='cuda')
        h = torch.empty(self.e.nC, 1, dtype=torch.float64, device='cuda')
        self.e.h.call('mpsw_window_final_state', _ptr(u), _ptr(h), _stream())
        return self.e.to_reference(u, _EDGE)[:, 0], self.e.to_reference(h, _CELL)[:, 0]

    def tl_internal(self, du: torch.Tensor, dh: torch.Tensor, precision: int = FP64) -> None:
        """In place on internal-order members ([nEdges, B], [nCells, B], contiguous)."""
        B = du.shape[1]
        self.e.h.call('mpsw_window_tl', int(precision), B, _ptr(du), _ptr(dh), _stream())

    def ad_internal(self, au: torch.Tensor, ah: torch.Tensor, precision: int = FP64) -> None:
        B = au.shape[1]
        self.e.h.call('mpsw_window_ad', int(precision), B, _ptr(au), _ptr(ah), _stream())

    def tl(self, du: torch.Tensor, dh: torch.Tensor, precision: int = FP64, work=None, out=None):
        """Tangent linear of the window for B members (reference order in and out).

        work: optional (u, h) internal-order scratch and out: optional (u, h) results, each
        contiguous CUDA float64 of the members' shapes, so repeated sweeps allocate nothing."""
        return self._sweep(self.tl_internal, du, dh, precision, work, out)

    def ad(self, au: torch.Tensor, ah: torch.Tensor, precision: int = FP64, work=None, out=None):
        """Adjoint of the window for B members: final-state adjoints in, initial-state out
        (work, out as for tl)."""
        return self._sweep(self.ad_internal, au, ah, precision, work, out)

    def _sweep(self, fn, xu, xh, precision, work, out):
        wu, wh = work if work is not None else (None, None)
        ou, oh = out if out is not None else (None, None)
        xu_i = self.e.to_internal(xu, _EDGE, wu)
        xh_i = self.e.to_internal(xh, _CELL, wh)
        fn(xu_i, xh_i, precision)
        return self.e.to_reference(xu_i, _EDGE, ou), self.e.to_reference(xh_i, _CELL, oh)


class RK4Step(torch.autograd.Function):
    """One sw_rk4 step (src/mpas_sw_module.f90:528-635) of the state (u, h) as an autograd
    function; backward runs the engine's adjoint step (:783-1002) linearised at the step's
    input state.  u, h: CUDA float64 vectors in the reference numbering."""

    @staticmethod
    def forward(ctx, u, h, engine: Engine):
        engine.set_state(u, h)
        w = Window(engine, 1, 1)
        u1, h1 = w.final_state()
        ctx.engine = engine
        ctx.save_for_backward(u, h)
        return u1, h1

    @staticmethod
    def backward(ctx, gu, gh):
        u, h = ctx.saved_tensors
        e = ctx.engine
        e.set_state(u, h)
        w = Window(e, 1, 1)
        au, ah = w.ad(gu.to(torch.float64).contiguous(), gh.to(torch.float64).contiguous())
        return au[:, 0], ah[:, 0], None


def rk4_step(u, h, engine: Engine):
    return RK4Step.apply(u, h, engine)
