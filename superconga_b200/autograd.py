"""torch.autograd face of the engine's hand-written adjoint.

``FreeEnergy.apply(delta, a, b_ext, ctx, w_omega, beta_j)`` returns
L = w_omega * Omega + sum(beta_j * j) for the complex order parameter
``delta`` [Nc][N0][N0] (complex128), the induced vector potential ``a``
[2][N0][N0] (internal units, float64) and the external field ``b_ext``
(0-d float64, B0 units), evaluated on the engine context ``ctx`` with its
incoming boundary values held fixed (one frozen-boundary pass of the
self-consistency map, ComputeFreeEnergy.h:281-414, ComputeCurrent.h:175-222).
``backward`` runs the adjoint sweep (gamma checkpointed every 16 sites) and
returns dL/dDelta, dL/dA and dL/dB_ext in PyTorch's convention for complex
inputs (dL/dRe + i dL/dIm).

``edge_current_weights`` builds beta_j for the total azimuthal current of a
ring of sites near the grain's edge.
"""
from __future__ import annotations

import numpy as np
import torch


def _planar(delta: torch.Tensor) -> np.ndarray:
    d = delta.detach().to("cpu", torch.complex128).numpy()
    return np.ascontiguousarray(np.stack([d.real, d.imag], axis=1))


class FreeEnergy(torch.autograd.Function):
    @staticmethod
    def forward(fctx, delta, a, b_ext, ctx, w_omega=1.0, beta_j=None):
        d = _planar(delta)
        av = np.ascontiguousarray(a.detach().to("cpu", torch.float64).numpy())
        b = float(b_ext.detach().cpu())
        ctx.set_state(d, av)
        ctx.set_external_field(b)
        fe = ctx.evaluate()
        loss = w_omega * fe
        if beta_j is not None:
            _, j, _ = ctx.results()
            loss += float(np.sum(np.asarray(beta_j) * j))
        fctx.engine = ctx
        fctx.args = (d, av, b, w_omega, beta_j)
        fctx.devices = (delta.device, a.device, b_ext.device)
        return torch.tensor(loss, dtype=torch.float64, device=delta.device)

    @staticmethod
    def backward(fctx, grad_out):
        ctx = fctx.engine
        d, av, b, w_omega, beta_j = fctx.args
        ctx.set_state(d, av)
        ctx.set_external_field(b)
        gd, ga, gb = ctx.adjoint(w_omega, beta_j)
        g = float(grad_out.detach().cpu())
        gdel = torch.from_numpy(gd[:, 0] + 1j * gd[:, 1]).to(fctx.devices[0]) * g
        ga_t = torch.from_numpy(ga).to(fctx.devices[1]) * g
        gb_t = torch.tensor(gb * g, dtype=torch.float64, device=fctx.devices[2])
        return gdel, ga_t, gb_t, None, None, None


def edge_current_weights(domain: np.ndarray, h: float, width: float) -> np.ndarray:
    """beta [2][N0][N0] with sum(beta * j) the azimuthal current (z x r_hat) . j
    summed over the grain sites within ``width`` (in xi0) of the grain's
    outermost radius, measured from the lattice centre."""
    n0 = domain.shape[0]
    yy, xx = np.mgrid[0:n0, 0:n0].astype(np.float64)
    c = 0.5 * (n0 - 1)
    x, y = (xx - c) * h, (yy - c) * h
    r = np.hypot(x, y)
    inside = domain > 0
    rmax = r[inside].max()
    ring = inside & (r > rmax - width)
    rs = np.where(r > 0, r, 1.0)
    beta = np.zeros((2, n0, n0))
    beta[0] = np.where(ring, -y / rs, 0.0)
    beta[1] = np.where(ring, x / rs, 0.0)
    return beta
