"""TEST INFRASTRUCTURE: FP64 PyTorch form of the frozen-match BM3D operator.

With the match table, the threshold keep masks and so the weights of a
forward pass held fixed, the BM3Dv2 basic estimate is a linear map of its
input clip X (src/bm3d.comp:358-399 transform and threshold, :697-715
scatter; src/bm3d_agg.comp:36-52 normalisation; slice bookkeeping
src/bm3d.cpp:369-371):

    out_n = (1 / D_n) * sum over the slices (m, z) that output n reads, with
            multiplicity, of sum over the groups g of stack m of
            sum over the matches k of g with z_k = z of
            w_g * [C^T M_g C P_g]_k placed at (x_k, y_k)

P_g holds the group's 8 patches, patch k read from frame clamp(m - r + z_k)
at (x_k, y_k); C is the orthonormal 3D DCT (the reference's transform pair is
4*C per axis forward and 4*C^T inverse with a 1/4096 scale in between, so the
scales cancel); M_g is the group's keep mask and w_g = 1 / popcount(M_g);
D_n is the denominator the forward pass recorded. The extractor's rounding
is not modelled.

The saved state is the buffer that vsfeel_bm3d_forward_saved fills, in the
layout of vsfeel_bm3d_saved_info. Used only by the gradient tests, as the
FP64 reference the CUDA adjoint is checked against.
"""

from __future__ import annotations

import math

import numpy as np


def clamp_frame(f: int, nframes: int) -> int:
    return min(max(f, 0), nframes - 1)


def agg_slice(i: int, n: int, nframes: int, radius: int) -> int:
    """src/bm3d.cpp:369-371."""
    if radius == 0:
        return 0
    return min(max(2 * radius - i, n - nframes + 1 + radius), n + radius)


def slice_reads(m: int, z: int, nframes: int, radius: int) -> int:
    """Times output clamp(m - r + z) sums slice z of stack m
    (src/bm3d.cpp:628-696 sums slice agg_slice(i, n) of stack clamp(n - r + i))."""
    n = clamp_frame(m - radius + z, nframes)
    return sum(1 for i in range(2 * radius + 1)
               if clamp_frame(n - radius + i, nframes) == m
               and agg_slice(i, n, nframes, radius) == z)


def dct_matrix(dtype=np.float64) -> np.ndarray:
    """Orthonormal 8-point DCT-II, C[u, x] = s(u) cos(pi (2x + 1) u / 16)."""
    c = np.empty((8, 8), dtype=np.float64)
    for u in range(8):
        s = math.sqrt(1.0 / 8.0) if u == 0 else math.sqrt(2.0 / 8.0)
        for x in range(8):
            c[u, x] = s * math.cos(math.pi * (2 * x + 1) * u / 16.0)
    return c.astype(dtype)


class SavedState:
    """Decoded saved state of one forward pass (torch tensors on `device`)."""

    def __init__(self, saved_bytes, layout, nframes: int, height: int, width: int, radius: int,
                 device=None):
        raw = saved_bytes.detach().cpu().numpy() if hasattr(saved_bytes, "detach") else \
            np.asarray(saved_bytes)
        raw = raw.view(np.uint8)
        nb = int(layout.num_blocks)
        sb = int(layout.stack_bytes)
        tables, words = [], []
        for m in range(nframes):
            rec = raw[m * sb:(m + 1) * sb]
            xy = rec[layout.match_xy_offset:layout.match_xy_offset + nb * 32].view(np.uint32)
            xy = xy.reshape(nb, 8)
            zp = rec[layout.match_z_offset:layout.match_z_offset + nb * 4].view(np.uint32)
            table = np.empty((nb, 8, 3), dtype=np.int64)
            table[:, :, 0] = xy & 0xFFFF
            table[:, :, 1] = xy >> 16
            table[:, :, 2] = np.stack([(zp >> (4 * k)) & 15 for k in range(8)], axis=1)
            tables.append(table)
            words.append(rec[layout.mask_offset:layout.mask_offset + nb * 64].view(np.uint64)
                         .reshape(nb, 8))
        dpitch, dframe = int(layout.den_row_stride), int(layout.den_frame_stride)
        den = raw[layout.den_offset:layout.den_offset + 4 * nframes * dframe].view(np.float32)
        den = den.reshape(nframes, dframe)[:, :height * dpitch].reshape(nframes, height, dpitch)
        self._setup(tables, words, np.ascontiguousarray(den[:, :, :width]), nframes, height,
                    width, radius, device)

    @classmethod
    def from_tables(cls, tables, words, nframes: int, height: int, width: int, radius: int,
                    device=None):
        """State from per-stack match tables [nblocks, 8, 3] and keep words
        [nblocks, 8]; the denominators are recomputed from the weights."""
        st = cls.__new__(cls)
        st._setup(tables, words, None, nframes, height, width, radius, device)
        st.den = st.denominators()
        return st

    def _setup(self, tables, words, den, nframes, height, width, radius, device):
        import torch

        self.nframes, self.height, self.width, self.radius = nframes, height, width, radius
        self.nblocks = int(np.asarray(tables[0]).shape[0])
        dev = device if device is not None else "cpu"
        t = np.stack([np.asarray(a, dtype=np.int64) for a in tables])   # [N, nb, 8, 3]
        self.x = torch.from_numpy(np.ascontiguousarray(t[..., 0])).to(dev)
        self.y = torch.from_numpy(np.ascontiguousarray(t[..., 1])).to(dev)
        self.z = torch.from_numpy(np.ascontiguousarray(t[..., 2])).to(dev)
        w = np.stack([np.asarray(a, dtype=np.uint64) for a in words])    # [N, nb, 8]
        # word h, bit 8*g + v -> mask[m, b, g, v, h]
        bits = (w[..., None] >> np.arange(64, dtype=np.uint64)) & np.uint64(1)
        bits = bits.reshape(nframes, self.nblocks, 8, 8, 8).transpose(0, 1, 3, 4, 2)
        self.mask = torch.from_numpy(np.ascontiguousarray(bits, dtype=np.float64)).to(dev)
        self.den = None if den is None else torch.from_numpy(den).to(dev).double()
        reads = np.zeros((nframes, 2 * radius + 1), dtype=np.float64)
        for m in range(nframes):
            for z in range(2 * radius + 1):
                reads[m, z] = slice_reads(m, z, nframes, radius)
        self.reads = torch.from_numpy(reads).to(dev)
        self.C = torch.from_numpy(dct_matrix()).to(dev)
        self.weight = 1.0 / self.mask.sum(dim=(2, 3, 4))     # [N, nb]

    # -- building blocks -----------------------------------------------------
    def _frames_of(self, m: int, z):
        import torch

        return torch.clamp(m - self.radius + z, 0, self.nframes - 1)

    def _flat_index(self, m: int, sel=None):
        """Flat clip index of every pixel of every patch: [nb, 8, 8, 8]."""
        import torch

        x, y, z = self.x[m], self.y[m], self.z[m]
        if sel is not None:
            x, y, z = x[sel], y[sel], z[sel]
        f = self._frames_of(m, z)
        ar = torch.arange(8, device=x.device)
        rows = y[:, :, None, None] + ar[None, None, :, None]
        cols = x[:, :, None, None] + ar[None, None, None, :]
        return (f[:, :, None, None] * self.height + rows) * self.width + cols

    def _filter(self, patches, mask):
        """C^T M C applied to [nb, 8(k), 8(row), 8(col)] patches."""
        import torch

        C = self.C
        spec = torch.einsum("gk,vr,hc,bkrc->bgvh", C, C, C, patches)
        return torch.einsum("gk,vr,hc,bgvh->bkrc", C, C, C, spec * mask)

    # -- the operator ----------------------------------------------------------
    def apply(self, x):
        """The frozen operator on x (N, H, W) in FP64; differentiable in x."""
        import torch

        xf = x.reshape(-1)
        num = torch.zeros_like(xf)
        for m in range(self.nframes):
            idx = self._flat_index(m)
            q = self._filter(xf[idx], self.mask[m])
            scale = self.weight[m][:, None] * self.reads[m][self.z[m]]  # [nb, 8]
            num = num.index_add(0, idx.reshape(-1), (q * scale[:, :, None, None]).reshape(-1))
        return num.reshape(x.shape) / self.den

    def denominators(self):
        """The denominators recomputed in FP64 from the weights."""
        import torch

        den = torch.zeros(self.nframes * self.height * self.width, dtype=torch.float64,
                          device=self.weight.device)
        for m in range(self.nframes):
            idx = self._flat_index(m)
            scale = self.weight[m][:, None] * self.reads[m][self.z[m]]
            den.index_add_(0, idx.reshape(-1),
                           scale[:, :, None, None].expand(idx.shape).reshape(-1))
        return den.reshape(self.nframes, self.height, self.width)

    def central_differences(self, x, weights, pixels, h: float = 1e-6):
        """FP64 central differences of L(x) = sum(weights * apply(x)) at the
        given (frame, row, col) pixels, step h. For pixel p only the groups
        that gather p depend on x_p, so L(x +- h e_p) is evaluated on those
        groups' terms; the other terms of L cancel in the difference."""
        import torch

        xf = x.reshape(-1).double()
        wd = (weights.double() / self.den).reshape(-1)
        tw = 2 * self.radius + 1
        index = {}
        out = []
        for (f, row, col) in pixels:
            p = (int(f) * self.height + int(row)) * self.width + int(col)
            total = 0.0
            for m in range(self.nframes):
                if all(clamp_frame(m - self.radius + z, self.nframes) != int(f) for z in range(tw)):
                    continue
                if m not in index:
                    index[m] = self._flat_index(m)
                idx = index[m]                                  # [nb, 8, 8, 8]
                sel = (idx == p).flatten(1).any(dim=1)
                if not bool(sel.any()):
                    continue
                ids = idx[sel]
                scale = self.weight[m][sel][:, None] * self.reads[m][self.z[m][sel]]
                vals = []
                for sgn in (1.0, -1.0):
                    patches = xf[ids] + sgn * h * (ids == p).double()
                    q = self._filter(patches, self.mask[m][sel])
                    vals.append(((q * scale[:, :, None, None]) * wd[ids]).sum())
                total += float((vals[0] - vals[1]) / (2.0 * h))
            out.append(total)
        return torch.tensor(out, dtype=torch.float64)
