"""Differentiable BM3Dv2 basic estimate for PyTorch.

A thin torch extension over the library's C ABI: ``BM3DFunction`` is a
``torch.autograd.Function`` whose forward pass is
``vsfeel_bm3d_forward_saved`` (the plain denoiser that also records the match
table and the threshold keep bits of every stack, plus the per-output
denominators) and whose backward pass is ``vsfeel_bm3d_backward``, the
adjoint kernel. The gradient is that of the denoiser with its block matches,
keep masks and aggregation weights frozen at the forward pass -- with those
fixed the denoiser is linear in its input and the adjoint is exact. The
extractor's rounding (``extractor_exp != 0``) is taken as the identity.

The reference plugin has no differentiable form; the forward output equals
the plain path's (``BM3Dv2``) on the same input.

Work is enqueued on torch's current CUDA stream. A ``Denoiser`` owns one
library context, whose accumulator planes are reused by each call: calls on
one ``Denoiser`` must run in stream order (one stream, or synchronised).
"""

from __future__ import annotations

import ctypes

from . import Error, _lib, _make_args, GRAYS


class Denoiser:
    """A BM3Dv2 context for clips of one shape (N, H, W) on one device."""

    def __init__(self, shape, device=0, sigma=None, block_step=None, bm_range=None, radius=None,
                 ps_num=None, ps_range=None, extractor_exp=None):
        n, h, w = (int(v) for v in shape)
        self.shape = (n, h, w)
        self.device = int(device)
        self.lib = _lib.load()
        vi = _lib.VideoInfo(w, h, n, GRAYS.color_family, GRAYS.sample_type, 32, 0, 0)
        args, _ = _make_args(None, sigma, block_step, bm_range, radius, ps_num, ps_range, None,
                             extractor_exp)
        handle = ctypes.c_void_p()
        if self.lib.vsfeel_bm3d_create(ctypes.byref(args), ctypes.byref(vi), self.device,
                                       ctypes.byref(handle)) != _lib.OK:
            raise Error(_lib.last_error(self.lib))
        self.handle = handle
        self.layout = _lib.SavedInfo()
        self._check(self.lib.vsfeel_bm3d_saved_layout(self.handle, ctypes.byref(self.layout)))

    @property
    def info(self) -> _lib.Info:
        inf = _lib.Info()
        self._check(self.lib.vsfeel_bm3d_get_info(self.handle, ctypes.byref(inf)))
        return inf

    def _check(self, rc: int) -> None:
        if rc != _lib.OK:
            raise Error(_lib.last_error(self.lib))

    def _validate(self, t, name: str):
        import torch

        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32
                and t.dim() == 3 and t.stride(2) == 1):
            raise Error(f"BM3D: {name} must be a CUDA float32 (N, H, W) tensor with "
                        "contiguous rows")
        if tuple(t.shape) != self.shape:
            raise Error(f"BM3D: {name} has shape {tuple(t.shape)}, the context {self.shape}")
        if t.device.index != self.device:
            raise Error(f"BM3D: {name} is on {t.device}, the context on cuda:{self.device}")

    def plain(self, x, out=None):
        """The plain forward pass (no saved state) into out, on torch's
        current stream."""
        import torch

        self._validate(x, "input")
        if out is None:
            out = torch.empty(self.shape, dtype=torch.float32, device=x.device)
        self._validate(out, "output")
        stream = torch.cuda.current_stream(x.device).cuda_stream
        self._check(self.lib.vsfeel_bm3d_process_device(
            self.handle, x.data_ptr(), x.stride(0), x.stride(1), out.data_ptr(), out.stride(0),
            out.stride(1), 0, self.shape[0], stream))
        return out

    def forward_saved(self, x):
        """(output, saved) for x; saved is a uint8 CUDA tensor of the frozen state."""
        import torch

        self._validate(x, "input")
        out = torch.empty(self.shape, dtype=torch.float32, device=x.device)
        saved = torch.empty(int(self.layout.bytes), dtype=torch.uint8, device=x.device)
        stream = torch.cuda.current_stream(x.device).cuda_stream
        self._check(self.lib.vsfeel_bm3d_forward_saved(
            self.handle, x.data_ptr(), x.stride(0), x.stride(1), out.data_ptr(), out.stride(0),
            out.stride(1), saved.data_ptr(), stream))
        return out, saved

    def backward(self, saved, grad_out):
        """dLoss/dInput from dLoss/dOutput and the state of forward_saved."""
        import torch

        self._validate(grad_out, "grad_output")
        grad_in = torch.empty(self.shape, dtype=torch.float32, device=grad_out.device)
        stream = torch.cuda.current_stream(grad_out.device).cuda_stream
        self._check(self.lib.vsfeel_bm3d_backward(
            self.handle, saved.data_ptr(), grad_out.data_ptr(), grad_out.stride(0),
            grad_out.stride(1), grad_in.data_ptr(), grad_in.stride(0), grad_in.stride(1), stream))
        return grad_in

    def __call__(self, x):
        return BM3DFunction.apply(x, self)

    def close(self) -> None:
        h = getattr(self, "handle", None)
        if h:
            # kernels enqueued on the caller's streams may still use the
            # context's buffers: finish the device's work before freeing
            import sys

            torch = sys.modules.get("torch")
            if torch is not None and torch.cuda.is_initialized():
                torch.cuda.synchronize(self.device)
            self.lib.vsfeel_bm3d_free(h)
            self.handle = None

    def __del__(self):
        self.close()


def _function():
    import torch

    class BM3DFunction(torch.autograd.Function):
        """out = BM3DFunction.apply(x, denoiser)."""

        @staticmethod
        def forward(ctx, x, denoiser):
            out, saved = denoiser.forward_saved(x)
            ctx.save_for_backward(saved)
            ctx.denoiser = denoiser
            return out

        @staticmethod
        def backward(ctx, grad_out):
            (saved,) = ctx.saved_tensors
            g = grad_out
            if g.dim() != 3 or g.stride(2) != 1 or not g.is_contiguous():
                g = g.contiguous()
            return ctx.denoiser.backward(saved, g), None

    return BM3DFunction


class _Lazy:
    """Defers the torch import until the Function is first used."""

    _fn = None

    def __getattr__(self, name):
        if _Lazy._fn is None:
            _Lazy._fn = _function()
        return getattr(_Lazy._fn, name)


BM3DFunction = _Lazy()


def bm3d(x, sigma=None, block_step=None, bm_range=None, radius=None, ps_num=None, ps_range=None,
         extractor_exp=None):
    """Differentiable BM3Dv2 basic estimate of a CUDA float32 clip (N, H, W)."""
    den = Denoiser(tuple(x.shape), x.device.index or 0, sigma=sigma, block_step=block_step,
                   bm_range=bm_range, radius=radius, ps_num=ps_num, ps_range=ps_range,
                   extractor_exp=extractor_exp)
    return BM3DFunction.apply(x, den)
