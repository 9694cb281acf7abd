"""The differentiable form: the cutoff LJ(C2) + Coulomb(C1) energy as a
``torch.autograd.Function`` whose backward is the hand-written force kernel.

* forward: E(x, q, T) -- the force kernel's energy (COULOMB + LENNARDJONES);
  x are positions (n, 3), q scaled charges (n,) (charge x SQRTCOULOMBCONSTANT,
  as ProtoMol's Atom::scaledCharge), T the LJ table (ntypes, ntypes, 4) of
  {A, B, A14, B14} that the pair loop reads.
* backward: dE/dx = -F from the force kernel (mixed or FP64, the force's
  precision); dE/dq and dE/dT from the FP64 parameter-gradient kernel
  (pmb200_param_grad_device).  Per-type dE/dsigma, dE/depsilon follow by
  autograd through ``lj_table`` (Lorentz-Berthelot mixing, the rule
  ProtoMol's BuildTopology applies, protomol/src/protomol/topology/
  BuildTopology.cpp:651-657).
* double backward: the gradient dE/dx is itself a Function whose backward,
  for an incoming w, returns H w (Hessian-vector product) and the
  derivatives of w . dE/dx with respect to q and T
  (pmb200_hvp_device, FP64).  torch.autograd.grad(..., create_graph=True)
  therefore gives Hessian-vector products, and a force-matching loss
  sum |F(theta) - F_target|^2 can be differentiated with respect to the
  parameters.

Second derivatives with respect to the parameters alone (d^2E/dq^2, ...)
are not provided (their backward raises).  Every call runs on the GPU
through libpmb200; there is no CPU path.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .force import NonbondedCutoffB200SystemForce, PeriodicTopology

SQRTCOULOMBCONSTANT = 18.2226123264  # protomol/src/protomol/base/PMConstants.cpp:64


def lj_table(sigma, epsilon):
    """(ntypes, ntypes, 4) table {A, B, A14, B14} from per-type sigma and
    epsilon (torch tensors): sigma_ab = (sigma_a + sigma_b) / 2, epsilon_ab =
    sqrt(epsilon_a epsilon_b), A = 4 eps sigma^12, B = 4 eps sigma^6; pairs
    with a zero epsilon get zeros (no NaN gradient through the square
    root)."""
    s = 0.5 * (sigma[:, None] + sigma[None, :])
    prod = epsilon[:, None] * epsilon[None, :]
    pos = prod > 0
    e = torch.where(pos, torch.sqrt(torch.where(pos, prod, torch.ones_like(prod))),
                    torch.zeros_like(prod))
    s6 = s ** 6
    A = 4.0 * e * s6 * s6
    B = 4.0 * e * s6
    return torch.stack([A, B, A, B], dim=-1)


class _Handle:
    """One device force context; the autograd functions hand it their
    parameter tensors before every kernel call."""

    def __init__(self, topo: PeriodicTopology, force: NonbondedCutoffB200SystemForce):
        self.topo = topo
        self.force = force

    def sync_params(self, q, table):
        """Copies the charges and the table into the context on the device,
        queued on torch's stream ahead of the kernels that read them (no
        host round trip; a non-finite value is reported by the next sync)."""
        self.force._ensure(self.topo)
        dev = torch.device("cuda", self.force.device)
        qd = q.detach().to(device=dev, dtype=torch.float64).contiguous()
        td = table.detach().to(device=dev, dtype=torch.float64).contiguous()
        if qd.numel() != self.topo.n or td.numel() != self.topo.ntypes ** 2 * 4:
            raise ValueError("charges must hold n values and the table ntypes^2 * 4")
        # (the temporaries' memory is reused only by work queued later on
        # this stream, after the copies)
        self.force.update_params_device(self.topo, qd.data_ptr(), td.data_ptr(), self.stream())

    def stream(self):
        """torch's current stream as a CUDA stream handle.  torch's default
        stream is the legacy default stream, whose handle 0 would select the
        context's own stream in libpmb200; pass the runtime's explicit legacy
        handle (cudaStreamLegacy, 0x1) instead so the kernels stay ordered
        with torch's work."""
        h = torch.cuda.current_stream().cuda_stream
        return h if h else 0x1


def _check_pos(pos):
    if not (pos.is_cuda and pos.dtype == torch.float64 and pos.is_contiguous()):
        raise TypeError("positions must be a contiguous float64 CUDA tensor (n, 3)")


class _Gradient(torch.autograd.Function):
    """G = dE/dx (= -F); backward: H w and d(w . G)/d(q, T)."""

    @staticmethod
    def forward(ctx, pos, q, table, h):
        _check_pos(pos)
        h.sync_params(q, table)
        frc = torch.zeros_like(pos)
        h.force.evaluate_device(h.topo, pos.data_ptr(), frc.data_ptr(), None, 0, h.stream())
        ctx.save_for_backward(pos, q, table)
        ctx.h = h
        return -frc

    @staticmethod
    def backward(ctx, w):
        pos, q, table = ctx.saved_tensors
        h = ctx.h
        h.sync_params(q, table)
        w = w.detach().to(torch.float64).contiguous()
        hv = torch.empty_like(pos)
        # the parameter derivatives only when asked for (a plain Hessian-vector
        # product skips their kernel work)
        need_q, need_t = ctx.needs_input_grad[1], ctx.needs_input_grad[2]
        dq = torch.empty(q.shape, dtype=torch.float64, device=pos.device) if need_q else None
        dt = torch.empty(table.shape, dtype=torch.float64, device=pos.device) if need_t else None
        h.force.hvp_device(h.topo, pos.data_ptr(), w.data_ptr(), hv.data_ptr(),
                           dq.data_ptr() if need_q else None, dt.data_ptr() if need_t else None,
                           h.stream())
        return (hv, dq.to(q.dtype) if need_q else None, dt.to(table.dtype) if need_t else None,
                None)


class _Energy(torch.autograd.Function):
    """E(x, q, T); backward through the force kernel and the parameter
    gradient kernel."""

    @staticmethod
    def forward(ctx, pos, q, table, h):
        _check_pos(pos)
        h.sync_params(q, table)
        frc = torch.zeros_like(pos)
        out = torch.zeros(20, dtype=torch.float64, device=pos.device)
        h.force.evaluate_device(h.topo, pos.data_ptr(), frc.data_ptr(), out.data_ptr(),
                                _lib.PMB200_ENERGY, h.stream())
        ctx.save_for_backward(pos, q, table)
        ctx.h = h
        return out[0] + out[1]

    @staticmethod
    def backward(ctx, gE):
        pos, q, table = ctx.saved_tensors
        h = ctx.h
        gx = gq = gt = None
        if ctx.needs_input_grad[0]:
            # differentiable: its own backward is the Hessian-vector product
            gx = gE * _Gradient.apply(pos, q, table, h)
        if ctx.needs_input_grad[1] or ctx.needs_input_grad[2]:
            h.sync_params(q, table)
            dq = torch.empty(q.shape, dtype=torch.float64, device=pos.device)
            dt = torch.empty(table.shape, dtype=torch.float64, device=pos.device)
            h.force.param_grad_device(h.topo, pos.data_ptr(), dq.data_ptr(), dt.data_ptr(),
                                      h.stream())
            gq = _NoSecond.apply(gE * dq.to(q.dtype))
            gt = _NoSecond.apply(gE * dt.to(table.dtype))
        return gx, gq, gt, None


class _NoSecond(torch.autograd.Function):
    """Identity whose backward refuses: second derivatives with respect to
    the parameters alone are not provided."""

    @staticmethod
    def forward(ctx, x):
        return x.clone()

    @staticmethod
    def backward(ctx, g):
        raise RuntimeError("second derivatives of the energy with respect to the charges or "
                           "the LJ table are not provided")


class NonbondedEnergy:
    """Differentiable energy of one periodic system.

    ``energy(pos, q, table)`` -> E (0-d tensor); ``forces(pos, q, table)`` ->
    -dE/dx, differentiable (its gradients go through the HVP kernel).
    ``sysd`` is a system dict (protomoladdon_b200.water) or a
    PeriodicTopology plus the four cutoff parameters."""

    def __init__(self, topo, ron, rc_lj, rc_coul, rc_alg, precision="mixed", device=0):
        if isinstance(topo, dict):
            topo = PeriodicTopology.from_dict(topo)
        self.topo = topo
        self.force = NonbondedCutoffB200SystemForce(ron, rc_lj, rc_coul, rc_alg,
                                                    precision=precision, device=device)
        self._h = _Handle(topo, self.force)

    @classmethod
    def from_system(cls, sysd, **kw):
        return cls(PeriodicTopology.from_dict(sysd), sysd["ron"], sysd["rc_lj"], sysd["rc_coul"],
                   sysd["rc_alg"], **kw)

    def initial_params(self, device="cuda"):
        """(q_scaled, table) tensors holding the topology's current values."""
        q = torch.tensor(np.asarray(self.topo.qscaled), dtype=torch.float64, device=device)
        t = torch.tensor(np.asarray(self.topo.lj).reshape(self.topo.ntypes, self.topo.ntypes, 4),
                         dtype=torch.float64, device=device)
        return q, t

    def energy(self, pos, q, table):
        return _Energy.apply(pos, q, table, self._h)

    def gradient(self, pos, q, table):
        """dE/dx (= -F), differentiable."""
        return _Gradient.apply(pos, q, table, self._h)

    def forces(self, pos, q, table):
        return -self.gradient(pos, q, table)

    def close(self):
        self.force.close()
