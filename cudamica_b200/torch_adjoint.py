"""The engine's log-likelihood and its hand-written adjoint as a
torch.autograd.Function, for checking the adjoint against autograd and finite
differences.  The forward and backward both call the C ABI
(amica_set_params + amica_loglik_adjoint); torch only carries the tensors.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import Amica


class AmicaLogLik(torch.autograd.Function):
    """L(W, mu, beta, rho) at the engine's data and its other parameters.

    W is in the engine's storage order (column-major per model).  One sweep of
    the fused E-step in gradient mode gives L and dL/dW, dL/dmu, dL/dbeta,
    dL/drho together; backward scales them by the incoming gradient."""

    @staticmethod
    def forward(ctx, W, mu, beta, rho, engine: Amica):
        A = np.linalg.inv(W.detach().cpu().double().numpy().transpose(0, 2, 1)).transpose(0, 2, 1)
        engine.set_params(A=np.ascontiguousarray(A), mu=mu.detach().cpu().double().numpy(),
                          beta=beta.detach().cpu().double().numpy(),
                          rho=rho.detach().cpu().double().numpy())
        ll, g = engine.adjoint()
        ctx.grads = {k: torch.from_numpy(v).to(W.dtype) for k, v in g.items()}
        return torch.tensor(ll, dtype=W.dtype)

    @staticmethod
    def backward(ctx, gout):
        g = ctx.grads
        return gout * g["W"], gout * g["mu"], gout * g["beta"], gout * g["rho"], None
