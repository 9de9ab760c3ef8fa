"""Thin torch.autograd.Function over the library's discrete adjoint, for
tests only: u^n = (n channel steps from u0 with velocity wall data bc), with
the backward pass a cdns_adjoint_run of the projection objective seeded by
the incoming gradient (the vector-Jacobian product of the n-step map).

Complex tensors follow torch's convention, grad = dL/dRe + i dL/dIm, which
is the library's: the projection objective Re <g, u^n> has gradients
(du^n/du0)^T g and (du^n/dbc)^T g under the real inner product."""
import torch


class ChannelSteps(torch.autograd.Function):
    @staticmethod
    def forward(fctx, u0, bc, context, nsteps, checkpoint_interval):
        context.set_velocity(u0.detach().cpu().numpy())
        context.set_velocity_bc(bc.detach().cpu().numpy())
        context.run(1, nsteps)
        context.synchronize()
        fctx.save_for_backward(u0, bc)
        fctx.context, fctx.nsteps, fctx.kck = context, nsteps, checkpoint_interval
        return torch.from_numpy(context.get_velocity())

    @staticmethod
    def backward(fctx, grad_u):
        u0, bc = fctx.saved_tensors
        c = fctx.context
        c.set_velocity(u0.detach().cpu().numpy())
        _, gu, gb = c.adjoint_run(fctx.nsteps, fctx.kck, control=bc.detach().cpu().numpy(),
                                  weights=grad_u.detach().cpu().numpy())
        return torch.from_numpy(gu), torch.from_numpy(gb), None, None, None


def channel_steps(u0, bc, context, nsteps, checkpoint_interval):
    return ChannelSteps.apply(u0, bc, context, nsteps, checkpoint_interval)
