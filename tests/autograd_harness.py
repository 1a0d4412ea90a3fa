"""Test-harness wrapper of the C-ABI gradient as a torch.autograd.Function.

The library's gradient entry point (sfd_gradient) computes J^T r for the residual r = pred - obs
of its own forward.  Given the upstream gradient G of the records, backward() passes
obs = pred - G, so the residual the adjoint sees is G and the returned model gradient is J^T G:
the vector-Jacobian product autograd asks for.  Tensors live on the host; the engine copies them
to and from the device.  Only tests use this module.
"""
import numpy as np
import torch


class AcousticRecords(torch.autograd.Function):
    """records = F(vp) for an Engine of the 2-D acoustic scheme with its shots already set."""

    @staticmethod
    def forward(ctx, vp, engine, den):
        m = vp.detach().cpu().numpy().astype(np.float32)
        engine.set_model(m, den)
        rec = engine.forward()
        ctx.engine, ctx.den, ctx.model, ctx.rec = engine, den, m, rec
        return torch.from_numpy(rec.copy())

    @staticmethod
    def backward(ctx, grad_rec):
        e = ctx.engine
        e.set_model(ctx.model, ctx.den)
        obs = (ctx.rec.astype(np.float64) - grad_rec.detach().cpu().numpy()).astype(np.float32)
        _, g, _ = e.gradient(obs)
        return torch.from_numpy(g.astype(np.float32)), None, None


class ViscoacousticRecords(torch.autograd.Function):
    """records = F(vp, 1/Q) for an Engine of the viscoacoustic scheme with its shots already set."""

    @staticmethod
    def forward(ctx, vp, invq, engine, rho):
        m = vp.detach().cpu().numpy().astype(np.float32)
        q = (1.0 / invq.detach().cpu().numpy().astype(np.float64)).astype(np.float32)
        engine.set_model(m, rho, q)
        rec = engine.forward()
        ctx.engine, ctx.rho, ctx.model, ctx.q, ctx.rec = engine, rho, m, q, rec
        return torch.from_numpy(rec.copy())

    @staticmethod
    def backward(ctx, grad_rec):
        e = ctx.engine
        e.set_model(ctx.model, ctx.rho, ctx.q)
        obs = (ctx.rec.astype(np.float64) - grad_rec.detach().cpu().numpy()).astype(np.float32)
        _, gv, gq = e.gradient(obs, want_invq=True)
        return torch.from_numpy(gv.astype(np.float32)), torch.from_numpy(gq.astype(np.float32)), None, None
