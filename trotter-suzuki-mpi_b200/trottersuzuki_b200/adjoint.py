"""Differentiable real-time evolution: the hand-written adjoint behind torch.autograd.

    engine = AdjointEngine(make_desc(grid, hamiltonian, dt), dt, steps, checkpoint_every)
    psi_T = evolve(V, psi0, engine)          # V: float64 [H, W], psi0: complex128 [H, W], CUDA
    loss(psi_T).backward()                   # V.grad, psi0.grad from the adjoint kernel

The forward pass is the fused B200 Trotter step (the Solver's kernel, table
exp(-i V dt) built on the device from V); the backward pass is the fused
adjoint step of include/ts_b200.h (ts_b200_adjoint_*): by inverse steps for
linear evolution (checkpoint_every = 0), by checkpointed recomputation for
the nonlinear GPE.  Gradients use PyTorch's convention for complex tensors
(dL/dre + i dL/dim for a real loss L).  torch provides device memory and
streams only; no torch operator computes any part of the evolution.
"""
import ctypes as C

from . import _capi
from ._capi import check, lib


class AdjointEngine:
    """Device state of one differentiable evolution (one backward per forward)."""

    def __init__(self, desc, delta_t, steps, checkpoint_every=0):
        self.desc = desc
        self.shape = (desc.dim_y, desc.dim_x)
        self.delta_t = float(delta_t)
        self.steps = int(steps)
        self.checkpoint_every = int(checkpoint_every)
        self._a = C.c_void_p()
        check(lib().ts_b200_adjoint_create(C.byref(desc), self.delta_t, self.steps,
                                           self.checkpoint_every, C.byref(self._a)))

    def _check(self, status):
        check(status, adjoint=self._a)

    def close(self):
        if self._a:
            lib().ts_b200_adjoint_destroy(self._a)
            self._a = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        self._check(lib().ts_b200_adjoint_set_stream(self._a, C.c_void_p(stream_ptr)))

    def set_segments(self, adjoint_rows=0, forward_rows=0):
        """Rows per segment task of the adjoint pass and of the forward steps
        (0 keeps the current choice)."""
        self._check(lib().ts_b200_adjoint_set_segments(self._a, int(adjoint_rows),
                                                       int(forward_rows)))

    def forward_ptrs(self, v_ptr, psi0_ptr, psi_t_ptr):
        self._check(lib().ts_b200_adjoint_forward(self._a, C.c_void_p(v_ptr), C.c_void_p(psi0_ptr),
                                                  C.c_void_p(psi_t_ptr)))

    def backward_ptrs(self, grad_psi_t_ptr, grad_v_ptr, grad_psi0_ptr):
        self._check(lib().ts_b200_adjoint_backward(self._a, C.c_void_p(grad_psi_t_ptr),
                                                   C.c_void_p(grad_v_ptr),
                                                   C.c_void_p(grad_psi0_ptr)))

    def synchronize(self):
        self._check(lib().ts_b200_adjoint_synchronize(self._a))

    # -- torch tensors ------------------------------------------------------
    def _bind(self, device):
        """Queue the engine's work on torch's current stream; torch's legacy
        default stream (handle 0) cannot be shared, so then the engine uses its
        own stream and both sides synchronise around each call."""
        import torch
        s = torch.cuda.current_stream(device)
        if s.cuda_stream != 0:
            self.set_stream(s.cuda_stream)
            return False
        s.synchronize()
        self.set_stream(0)
        return True

    def forward(self, V, psi0):
        """psi(T) (complex128 CUDA tensor) for V (float64) and psi0 (complex128)."""
        import torch
        H, W = self.shape
        if tuple(V.shape) != (H, W) or tuple(psi0.shape) != (H, W):
            raise ValueError(f"V and psi0 must have shape {(H, W)}")
        if V.dtype != torch.float64 or psi0.dtype != torch.complex128:
            raise TypeError("V must be float64 and psi0 complex128")
        if not (V.is_cuda and psi0.is_cuda):
            raise ValueError("V and psi0 must be CUDA tensors")
        V = V.detach().contiguous()
        psi0 = psi0.detach().contiguous()
        psi_t = torch.empty_like(psi0)
        own = self._bind(V.device)
        self.forward_ptrs(V.data_ptr(), psi0.data_ptr(), psi_t.data_ptr())
        if own:
            self.synchronize()
        return psi_t

    def backward(self, grad_psi_t):
        """(dL/dV, dL/dpsi0) for dL/dpsi(T) (complex128, dL/dre + i dL/dim)."""
        import torch
        g = grad_psi_t.detach().contiguous()
        if g.dtype != torch.complex128:
            g = g.to(torch.complex128)
        grad_v = torch.empty(self.shape, dtype=torch.float64, device=g.device)
        grad_psi0 = torch.empty(self.shape, dtype=torch.complex128, device=g.device)
        own = self._bind(g.device)
        self.backward_ptrs(g.data_ptr(), grad_v.data_ptr(), grad_psi0.data_ptr())
        if own:
            self.synchronize()
        return grad_v, grad_psi0


def _function():
    import torch

    class TrotterEvolution(torch.autograd.Function):
        """psi(T) = S^T psi0 for the potential V; backward by the adjoint kernel."""

        @staticmethod
        def forward(ctx, V, psi0, engine):
            ctx.engine = engine
            return engine.forward(V, psi0)

        @staticmethod
        def backward(ctx, grad_psi_t):
            grad_v, grad_psi0 = ctx.engine.backward(grad_psi_t)
            return grad_v, grad_psi0, None

    return TrotterEvolution


_FN = None


def evolve(V, psi0, engine):
    """Differentiable psi(T) for potential V (float64 [H, W]) and psi0 (complex128 [H, W])."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(V, psi0, engine)


__all__ = ["AdjointEngine", "evolve", "_capi"]
