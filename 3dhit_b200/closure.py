"""Learned subgrid-stress (SGS) closure for coarse LES.

A pointwise MLP maps the 9 filtered velocity-gradient components du_i/dx_j
at a grid point to the 6 components of the SGS stress tau_ij
(xx, yy, zz, xy, xz, yz): 9 -> 64 -> 64 -> 64 -> 6 with GELU (tanh form), bf16 weights and
activations, float32 accumulation.  Forward and backward run in the
tensor-core kernels behind ``hit_mlp_forward`` / ``hit_mlp_train_grads``
(include/hit3d.h); torch holds the float32 master weights and runs the Adam
optimiser on the gradients those kernels return.

The reference has no closure (its LES/closure work is a stated direction of
the project); this package adds it as the learned part of the solver.
"""

from __future__ import annotations

import math

import torch

from . import _native as nat

__all__ = ["ClosureMLP", "FEATURES", "OUTPUTS"]

FEATURES = 9
OUTPUTS = 6
HIDDEN = 64


class ClosureMLP:
    """float32 master weights (``W1`` [9,64], ``b1`` .. ``W4`` [64,6], ``b4``)
    and feature/target normalisation (``x_scale`` [9], ``y_scale`` [6]): the
    network sees x / x_scale and predicts tau / y_scale."""

    def __init__(self, device, seed=0):
        g = torch.Generator().manual_seed(seed)

        def lin(i, o):
            bound = 1.0 / math.sqrt(i)
            w = (torch.rand(i, o, generator=g) * 2 - 1) * bound
            b = (torch.rand(o, generator=g) * 2 - 1) * bound
            return w.to(device), b.to(device)

        self.device = torch.device(device)
        self.W1, self.b1 = lin(FEATURES, HIDDEN)
        self.W2, self.b2 = lin(HIDDEN, HIDDEN)
        self.W3, self.b3 = lin(HIDDEN, HIDDEN)
        self.W4, self.b4 = lin(HIDDEN, OUTPUTS)
        self.x_scale = torch.ones(FEATURES, device=self.device)
        self.y_scale = torch.ones(OUTPUTS, device=self.device)
        self.sgs_scale = 1.0  # calibration of the physical stress (energy-transfer matching)
        self._err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._ws = None
        self._packed = None
        self._physical = None

    @property
    def params(self):
        return [self.W1, self.b1, self.W2, self.b2, self.W3, self.b3, self.W4, self.b4]

    def state_dict(self):
        d = {k: getattr(self, k).detach().cpu() for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4")}
        d.update(x_scale=self.x_scale.cpu(), y_scale=self.y_scale.cpu(), sgs_scale=torch.tensor(float(self.sgs_scale)))
        return d

    def load_state_dict(self, d):
        for k, v in d.items():
            if k == "sgs_scale":
                self.sgs_scale = float(v)
            else:
                getattr(self, k).copy_(v.to(self.device))
        self._packed = None
        self._physical = None

    def pack(self):
        """bf16 device operands of the kernels (rebuilt after every update)."""
        bf = torch.bfloat16
        dev = self.device
        w1t = torch.zeros(64, 16, device=dev)
        w1t[:, :FEATURES] = self.W1.T
        w1t[:, 15] = self.b1
        w4t = torch.zeros(16, 64, device=dev)
        w4t[:OUTPUTS] = self.W4.T
        w4 = torch.zeros(64, 16, device=dev)
        w4[:, :OUTPUTS] = self.W4
        b4 = torch.zeros(16, device=dev)
        b4[:OUTPUTS] = self.b4
        w1 = torch.zeros(16, 64, device=dev)  # backward layer 1 (input cotangents, `vjp`)
        w1[:FEATURES] = self.W1
        keep = dict(w1=w1.to(bf).contiguous(),
            w1t=w1t.to(bf).contiguous(), w2t=self.W2.T.to(bf).contiguous(), w3t=self.W3.T.to(bf).contiguous(),
            w4t=w4t.to(bf).contiguous(), w2=self.W2.to(bf).contiguous(), w3=self.W3.to(bf).contiguous(),
            w4=w4.to(bf).contiguous(), b2=self.b2.float().contiguous(), b3=self.b3.float().contiguous(),
            b4=b4.contiguous())
        w = nat.MlpWeights(**{k: v.data_ptr() for k, v in keep.items() if k != "w1"})
        self._packed = (w, keep)
        return w

    def _weights(self):
        if self._packed is None:
            self.pack()
        return self._packed[0]

    def raw_forward(self, x):
        """Network output for normalised features x [P, 9] (float32, device)."""
        x = x.to(self.device, torch.float32).contiguous()
        y = torch.empty(x.shape[0], OUTPUTS, device=self.device)
        nat.call("hit_mlp_forward", ctypes_ref(self._weights()), nat.ptr(x), x.shape[0], nat.ptr(y), nat.ptr(self._err),
                 nat.stream_ptr(self.device))
        return y

    def __call__(self, grads):
        """SGS stress [P, 6] from velocity gradients [P, 9] (physical units)."""
        return self.raw_forward(grads / self.x_scale) * self.y_scale

    def pack_physical(self):
        """bf16 operands with the normalisation folded in (x / x_scale into W1,
        y_scale into W4 and b4): the network maps physical gradients to the
        physical stress."""
        W1, W4, b4 = self.W1, self.W4, self.b4
        ys = self.y_scale * float(self.sgs_scale)
        self.W1 = W1 / self.x_scale[:, None]
        self.W4, self.b4 = W4 * ys[None, :], b4 * ys
        try:
            w = self.pack()
        finally:
            self.W1, self.W4, self.b4 = W1, W4, b4
        self._physical = self._packed
        self._packed = None
        return w

    def forward_fields(self, grads, out, ctas_per_sm=0):
        """SGS stress fields out (6, P) from gradient fields grads (9, P)
        (component-major, physical units, float32 device tensors);
        ``ctas_per_sm`` > 0 caps the kernel's CTAs per SM (when it runs beside
        other work)."""
        if getattr(self, "_physical", None) is None:
            self.pack_physical()
        P = grads.shape[1]
        nat.call("hit_mlp_forward_strided", ctypes_ref(self._physical[0]), nat.ptr(grads), P, 1, P, nat.ptr(out), P, 1,
                 int(ctas_per_sm), nat.ptr(self._err), nat.stream_ptr(self.device))
        return out

    def loss_and_grads(self, x, tau):
        """Mean-squared loss of the network on normalised (x, tau) and the
        gradients of every parameter (stored in ``p.grad``)."""
        x = x.to(self.device, torch.float32).contiguous()
        tau = tau.to(self.device, torch.float32).contiguous()
        P = x.shape[0]
        nbytes = nat.load().hit_mlp_workspace_bytes(P)
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        dev = self.device
        dW1 = torch.empty(16, 64, device=dev)
        dW2 = torch.empty(65, 64, device=dev)
        dW3 = torch.empty(65, 64, device=dev)
        dW4 = torch.empty(65, 16, device=dev)
        loss = torch.empty(1, dtype=torch.float64, device=dev)
        nat.call("hit_mlp_train_grads", ctypes_ref(self._weights()), nat.ptr(x), nat.ptr(tau), P, nat.ptr(self._ws),
                 nat.ptr(dW1), nat.ptr(dW2), nat.ptr(dW3), nat.ptr(dW4), nat.ptr(loss), nat.ptr(self._err),
                 nat.stream_ptr(dev))
        self.W1.grad = dW1[:FEATURES].clone()
        self.b1.grad = dW1[15].clone()
        self.W2.grad, self.b2.grad = dW2[:64].clone(), dW2[64].clone()
        self.W3.grad, self.b3.grad = dW3[:64].clone(), dW3[64].clone()
        self.W4.grad, self.b4.grad = dW4[:64, :OUTPUTS].clone(), dW4[64, :OUTPUTS].clone()
        return loss

    def vjp(self, grads, ybar):
        """Reverse-mode product through `forward_fields`: for the gradient
        fields ``grads`` (9, P) and the cotangent ``ybar`` (6, P) of the
        physical stress, returns the cotangent of ``grads`` (9, P) and those
        of the master parameters (a list in the order of `params`), by the
        tensor-core backward (``hit_mlp_vjp``).  P a multiple of 16."""
        if getattr(self, "_physical", None) is None:
            self.pack_physical()
        w, keep = self._physical
        P = grads.shape[1]
        nbytes = nat.load().hit_mlp_workspace_bytes(P)
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        dev = self.device
        dW1 = torch.empty(16, 64, device=dev)
        dW2 = torch.empty(65, 64, device=dev)
        dW3 = torch.empty(65, 64, device=dev)
        dW4 = torch.empty(65, 16, device=dev)
        xbar = torch.empty(FEATURES, P, device=dev)
        grads = grads.contiguous()
        ybar = ybar.to(torch.float32).contiguous()
        nat.call("hit_mlp_vjp", ctypes_ref(w), keep["w1"].data_ptr(), nat.ptr(grads), P, 1, nat.ptr(ybar), P, 1, P,
                 nat.ptr(self._ws), nat.ptr(dW1), nat.ptr(dW2), nat.ptr(dW3), nat.ptr(dW4), nat.ptr(xbar),
                 nat.ptr(self._err), nat.stream_ptr(dev))
        # the physical operands are W1 / x_scale and (W4, b4) * y_scale * sgs_scale
        ys = self.y_scale * float(self.sgs_scale)
        g = [dW1[:FEATURES] / self.x_scale[:, None], dW1[15].clone(), dW2[:64].clone(), dW2[64].clone(),
             dW3[:64].clone(), dW3[64].clone(), dW4[:64, :OUTPUTS] * ys[None, :], dW4[64, :OUTPUTS] * ys]
        return xbar, g

    def check_errors(self):
        if int(self._err.item()) != 0:
            raise RuntimeError("a tensor-core wait of the closure MLP timed out")


def ctypes_ref(struct):
    import ctypes
    return ctypes.addressof(struct)
