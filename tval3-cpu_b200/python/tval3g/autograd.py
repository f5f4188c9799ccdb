"""torch.autograd binding of the differentiable unrolled solve.

The forward and the backward are the C ABI's tval3g_unrolled_forward /
tval3g_unrolled_backward (hand-written CUDA adjoint); this module only moves
tensors.  The decisions of a forward (step lengths, multiplier updates) live
in the handle, so a backward must use the handle of its own forward, before
that handle runs another forward.
"""
import torch

from . import capi


class UnrolledTVAL3(torch.autograd.Function):
    """U = F(b, mu, beta): b (count, m) float32 on the GPU, mu and beta (K,)
    float64; returns U (count, n) float32 = U_K / scl of every instance."""

    @staticmethod
    def forward(ctx, b, mu, beta, handle):
        if not b.is_cuda or b.dtype != torch.float32:
            raise TypeError("b must be a float32 CUDA tensor")
        b = b.contiguous()
        count = b.shape[0]
        U = torch.empty((count, handle.spec.n), device=b.device, dtype=torch.float32)
        stream = torch.cuda.current_stream(b.device).cuda_stream
        handle.forward([b[i] for i in range(count)], mu.detach().double().cpu().numpy(),
                       beta.detach().double().cpu().numpy(), [U[i] for i in range(count)], stream=stream)
        ctx.handle = handle
        ctx.mu_meta = (mu.dtype, mu.device)
        ctx.beta_meta = (beta.dtype, beta.device)
        return U

    @staticmethod
    def backward(ctx, gU):
        gU = gU.contiguous().float()
        count = gU.shape[0]
        gb = torch.empty((count, ctx.handle.spec.b_len), device=gU.device, dtype=torch.float32)
        stream = torch.cuda.current_stream(gU.device).cuda_stream
        gmu, gbeta = ctx.handle.backward([gU[i] for i in range(count)], [gb[i] for i in range(count)], stream=stream)
        (mdt, mdev), (bdt, bdev) = ctx.mu_meta, ctx.beta_meta
        return (gb, torch.as_tensor(gmu, dtype=mdt, device=mdev), torch.as_tensor(gbeta, dtype=bdt, device=bdev),
                None)


def unrolled_tval3(b, mu, beta, handle):
    return UnrolledTVAL3.apply(b, mu, beta, handle)
