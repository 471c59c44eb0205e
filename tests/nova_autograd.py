"""torch.autograd.Function over the C ABI's forward (nova_b200_render with differentiable
parameters) and replay adjoint (nova_b200_backward).  Test harness only: the library exposes the
forward/backward pair; this wrapper lets torch optimisers drive it."""
import torch


class NovaRender(torch.autograd.Function):
    """image = render(albedo (n_tris, 3), roughness (n_materials,)) for one context and frame."""

    @staticmethod
    def forward(ctx, albedo, roughness, context, frame, height, width):
        albedo = albedo.detach().contiguous()
        roughness = roughness.detach().contiguous()
        context.set_diff_params(albedo.data_ptr(), roughness.data_ptr())
        img = torch.zeros((height, width, 4), dtype=torch.float32, device=albedo.device)
        try:
            context.render(frame, film_device_ptr=img.data_ptr())
        finally:
            context.set_diff_params(None, None)
        ctx.save_for_backward(albedo, roughness)
        ctx.context, ctx.frame = context, frame
        return img

    @staticmethod
    def backward(ctx, grad_img):
        albedo, roughness = ctx.saved_tensors
        g = grad_img.detach().contiguous()
        ga = torch.zeros_like(albedo)
        gr = torch.zeros_like(roughness)
        ctx.context.set_diff_params(albedo.data_ptr(), roughness.data_ptr())
        try:
            # the forward's per-path radiance is reused when nothing rendered on the context since
            ctx.context.backward(ctx.frame, g.data_ptr(), ga.data_ptr(), gr.data_ptr(), reuse_primal=True)
        finally:
            ctx.context.set_diff_params(None, None)
        return ga, gr, None, None, None, None


def render(albedo, roughness, context, frame, height, width):
    return NovaRender.apply(albedo, roughness, context, frame, height, width)
