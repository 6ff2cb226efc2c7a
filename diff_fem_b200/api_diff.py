"""``sim_act`` / ``sim_all``: the reference's autograd wrappers (python/api_diff.py)
over the engine.  Same signatures; outputs keep the dtype of the input q
(float64 in, float64 out; the reference always returns float32)."""
from __future__ import annotations

import numpy as np
import torch

from . import pydifem as pd


def _np(t):
    return t.detach().cpu().numpy().astype(np.float64)


class SimAct(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, qd, jq, jqd, tau, env, is_act):
        ctx.save_for_backward(q, qd, jq, jqd, tau)
        ctx.env = env
        ctx.phase = env.mPhase
        ctx.levels = [o.GetActivationLevelsAggregate() for o in env.mDfobjs]
        ctx.is_act = is_act
        x, v, a, b = pd.forward_act(_np(q), _np(qd), _np(jq), _np(jqd), _np(tau), env, is_act)
        dt = q.dtype
        return (torch.tensor(x, dtype=dt), torch.tensor(v, dtype=dt), torch.tensor(a, dtype=dt), torch.tensor(b, dtype=dt))

    @staticmethod
    def backward(ctx, dldq, dldqd, dldjq, dldjqd):
        q, qd, jq, jqd, tau = ctx.saved_tensors
        env = ctx.env
        env.mPhase = ctx.phase
        for o, lv in zip(env.mDfobjs, ctx.levels):
            o.SetActivationLevelsAggregate(lv)
        dq, dqd, djq, djqd, dtau = pd.backward_act(_np(q), _np(qd), _np(jq), _np(jqd), _np(tau), _np(dldq), _np(dldqd),
                                                   _np(dldjq), _np(dldjqd), env, ctx.is_act)
        dt = q.dtype
        gjq = torch.tensor(djq, dtype=jq.dtype) if np.size(djq) == jq.numel() else torch.zeros_like(jq)
        gjqd = torch.tensor(djqd, dtype=jqd.dtype) if np.size(djqd) == jqd.numel() else torch.zeros_like(jqd)
        return (torch.tensor(dq, dtype=dt), torch.tensor(dqd, dtype=dt), gjq, gjqd,
                torch.tensor(dtau, dtype=tau.dtype), None, None)


sim_act = SimAct.apply


class SimAll(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q, qd, tau, env):
        ctx.env = env
        x, v = pd.forward_all(_np(q), _np(qd), _np(tau), env)
        ctx.save_for_backward(torch.tensor(x), torch.tensor(v), tau)
        dt = q.dtype
        return torch.tensor(x, dtype=dt), torch.tensor(v, dtype=dt)

    @staticmethod
    def backward(ctx, dldq, dldqd):
        q, qd, tau = ctx.saved_tensors
        dq, dqd, dtau = pd.backward_all(_np(q), _np(qd), _np(tau), _np(dldq), _np(dldqd), ctx.env)
        return (torch.tensor(dq, dtype=dldq.dtype), torch.tensor(dqd, dtype=dldq.dtype),
                torch.tensor(dtau, dtype=tau.dtype), None)


sim_all = SimAll.apply
