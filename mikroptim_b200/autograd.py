"""PyTorch autograd over the device path: the merit and the residuals of run points x as
differentiable functions, with the gradients from the adjoint reverse sweep.

    problem = AdjointProblem(batch, layout, variables)     # templates: 1 variant or one per run
    x = torch.tensor(x0, device="cuda", requires_grad=True)  # [runs][P], float64
    merit(x, problem).sum().backward()                     # x.grad = d merit / d x

`Merit` returns merit_i = sum_k r_ik^2 (the MERIT mode, penalty rows included) and its
gradient 2 J_i^T r_i, read from column P of the fused adjoint normal equations (J never
leaves the GPU). `Residuals` returns the residual rows and applies J^T to the incoming
gradient with the materialised adjoint Jacobian. Both evaluate x on the device
(VariableSet::apply in mkb_apply_variables_device); there is no CPU path.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _capi
from .batch import ResidualLayout, SystemBatchHost
from .engine import DeviceSystemBatch, _stream_handle


class AdjointProblem:
    """Templates, layout and variables of a family of run points, uploaded once."""

    def __init__(self, batch: SystemBatchHost, layout: ResidualLayout, variables,
                 device="cuda"):
        self.host, self.layout, self.variables = batch, layout, variables
        self.templates = DeviceSystemBatch(batch, device)
        self.device = self.templates.device
        self.P = variables.size
        self._vars = variables.c_struct()
        self._plan = layout.plan(batch)
        self._lib = _capi.lib()

    def _x(self, x: torch.Tensor) -> torch.Tensor:
        if x.dim() != 2 or x.shape[1] != self.P:
            raise ValueError(f"x must be [runs][{self.P}], got {tuple(x.shape)}")
        t = self.templates.variants
        if t != 1 and t != x.shape[0]:
            raise ValueError("templates must hold 1 variant or one per run")
        return x.detach().to(device=self.device, dtype=torch.float64).contiguous()

    def records_at(self, x: torch.Tensor) -> DeviceSystemBatch:
        """A device batch of the run points x (one variant per run)."""
        x = self._x(x)
        runs = x.shape[0]
        out = DeviceSystemBatch.__new__(DeviceSystemBatch)
        out.device, out.topology, out.variants = self.device, self.templates.topology, runs
        out.stride, out.type = self.templates.stride, self.templates.type
        out.non_coaxial = self.templates.non_coaxial
        out.ghost_plates = self.templates.ghost_plates
        out.ghost_terms = self.templates.ghost_terms
        out.glass, out.wavelength_nm = self.templates.glass, self.templates.wavelength_nm
        out.variant_surfaces = None
        out.records = torch.empty((max(runs, 1), out.stride), dtype=torch.float64,
                                  device=self.device)
        b = self.templates.c_struct()
        rc = self._lib.mkb_apply_variables_device(C.byref(b), C.byref(self._vars),
                                                  C.c_void_p(x.data_ptr()), runs,
                                                  C.c_void_p(out.records.data_ptr()),
                                                  _stream_handle(None))
        _capi.check(rc, "apply variables")
        return out

    def merit(self, x: torch.Tensor) -> torch.Tensor:
        from .engine import merit_device
        return merit_device(self.records_at(x), self.layout, self.host).merit

    def residuals(self, x: torch.Tensor) -> torch.Tensor:
        from .engine import residuals_device
        return residuals_device(self.records_at(x), self.layout, self.host).residuals

    def normal_equations(self, x: torch.Tensor) -> torch.Tensor:
        """Fused adjoint + normal equations: [runs][P+1][P+1] = [J r]^T [J r]."""
        x = self._x(x)
        runs = x.shape[0]
        b = self.templates.c_struct()
        need = int(self._lib.mkb_adjoint_jacobian_workspace_bytes(C.byref(b), runs))
        ws = torch.empty(max(need, 1), dtype=torch.uint8, device=self.device)
        gram = torch.empty((runs, self.P + 1, self.P + 1), dtype=torch.float64,
                           device=self.device)
        rc = self._lib.mkb_adjoint_normal_equations_device(
            C.byref(b), C.byref(self._plan), C.byref(self._vars), C.c_void_p(x.data_ptr()),
            runs, C.c_void_p(gram.data_ptr()), C.c_void_p(ws.data_ptr()), ws.numel(),
            _stream_handle(None))
        _capi.check(rc, "adjoint normal equations")
        return gram

    def jacobian(self, x: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """Materialised adjoint Jacobian J [runs][P][R] and the residuals r [runs][R]."""
        from .engine import adjoint_jacobian_device
        J, r0, _ = adjoint_jacobian_device(self.templates, self.layout, self.host,
                                           self.variables, self._x(x).cpu().numpy())
        return J, r0


class Merit(torch.autograd.Function):
    """merit [runs] of the run points x [runs][P]; backward: 2 J^T r per run."""

    @staticmethod
    def forward(ctx, x: torch.Tensor, problem: AdjointProblem) -> torch.Tensor:
        ctx.problem = problem
        ctx.save_for_backward(x)
        return problem.merit(x).to(x.dtype)

    @staticmethod
    def backward(ctx, grad: torch.Tensor):
        (x,) = ctx.saved_tensors
        problem = ctx.problem
        gram = problem.normal_equations(x)
        g = gram[:, :problem.P, problem.P]  # J^T r
        return (2.0 * grad.to(g.dtype)[:, None] * g).to(x.dtype), None


class Residuals(torch.autograd.Function):
    """residual rows [runs][R] of the run points x [runs][P]; backward: J^T grad per run."""

    @staticmethod
    def forward(ctx, x: torch.Tensor, problem: AdjointProblem) -> torch.Tensor:
        J, r = problem.jacobian(x)
        ctx.save_for_backward(J)
        return r.to(x.dtype)

    @staticmethod
    def backward(ctx, grad: torch.Tensor):
        (J,) = ctx.saved_tensors
        return torch.einsum("ipr,ir->ip", J, grad.to(J.dtype)), None


def merit(x: torch.Tensor, problem: AdjointProblem) -> torch.Tensor:
    return Merit.apply(x, problem)


def residuals(x: torch.Tensor, problem: AdjointProblem) -> torch.Tensor:
    return Residuals.apply(x, problem)
