"""Test-harness wrapper: N fused steps as a torch.autograd.Function whose
backward is the library's discrete adjoint (hcl_adjoint_forward/backward).
Only the tests use it; the product API is the C ABI."""
import torch


class FusedSteps(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, dom, nsteps, dts, precision, checkpoint_every):
        nd = dom.ndim
        U0 = U0.contiguous()
        dom.set_state(U0[0], U0[1:1 + nd], U0[1 + nd], device=True)
        dom.adjoint_forward(nsteps, dts=dts, precision=precision, checkpoint_every=checkpoint_every)
        UN = torch.empty_like(U0)
        dom.get_state(out=(UN[0], UN[1:1 + nd], UN[1 + nd]), device=True)
        ctx.dom = dom
        return UN

    @staticmethod
    def backward(ctx, gUN):
        g = torch.empty_like(gUN)
        ctx.dom.adjoint_backward(gUN.contiguous(), g, device=True)
        torch.cuda.synchronize()
        return g, None, None, None, None, None
