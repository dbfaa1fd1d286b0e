"""Host <-> device staging shared by the drop-in classes.

The reference's public methods take ``(N, 3)`` / ``(N,)`` float64 numpy arrays
and return fresh numpy arrays.  The same methods here also accept CUDA torch
tensors (then nothing crosses PCIe and torch tensors are returned).
"""

from __future__ import annotations

import numpy as np

from . import _native as N


class DeviceState:
    """SoA device copy of (positions, radii) for one call."""

    __slots__ = ("n", "pos", "r", "aos")

    def __init__(self, n, pos, r, aos):
        self.n, self.pos, self.r, self.aos = n, pos, r, aos


class Stager:
    """Uploads inputs and downloads results through pinned buffers."""

    def __init__(self, ctx: N.Context):
        self.ctx = ctx
        self.buf = N.Buffers(ctx.device)
        self.torch = ctx.torch

    # -- inputs ---------------------------------------------------------------
    def positions(self, positions, radii, tag="in") -> tuple[DeviceState, bool]:
        """Returns the device state and whether the inputs were CUDA tensors."""
        torch = self.torch
        if N.is_cuda_tensor(positions):
            pos = positions.to(dtype=torch.float64).reshape(-1, 3).contiguous()
            n = pos.shape[0]
            r = radii if N.is_cuda_tensor(radii) else torch.as_tensor(np.asarray(radii), device=pos.device)
            r = r.to(dtype=torch.float64).reshape(-1).contiguous()
            soa = self.buf.dev(tag + "_soa", (3, n))
            self.ctx.aos_to_soa(n, pos, soa)
            return DeviceState(n, soa, r, pos), True
        p = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        rr = np.ascontiguousarray(radii, dtype=np.float64).reshape(-1)
        n = p.shape[0]
        if rr.shape[0] != n:
            raise ValueError(f"radii has {rr.shape[0]} entries for {n} positions")
        hp = self.buf.host(tag + "_hpos", (n, 3))
        hr = self.buf.host(tag + "_hr", (n,))
        hp.numpy()[...] = p
        hr.numpy()[...] = rr
        dp = self.buf.dev(tag + "_aos", (n, 3))
        dr = self.buf.dev(tag + "_r", (n,))
        dp.copy_(hp, non_blocking=True)
        dr.copy_(hr, non_blocking=True)
        soa = self.buf.dev(tag + "_soa", (3, n))
        self.ctx.aos_to_soa(n, dp, soa)
        return DeviceState(n, soa, dr, dp), False

    def vectors(self, arr, n, tag) -> tuple:
        """(N, 3) numpy or CUDA tensor -> SoA device tensor."""
        torch = self.torch
        if N.is_cuda_tensor(arr):
            a = arr.to(dtype=torch.float64).reshape(-1, 3).contiguous()
        else:
            h = self.buf.host(tag + "_h", (n, 3))
            h.numpy()[...] = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1, 3)
            a = self.buf.dev(tag + "_aos", (n, 3))
            a.copy_(h, non_blocking=True)
        soa = self.buf.dev(tag + "_soa", (3, n))
        self.ctx.aos_to_soa(n, a, soa)
        return soa

    # -- outputs --------------------------------------------------------------
    def to_aos_tensor(self, soa, n):
        out = self.torch.empty((n, 3), dtype=self.torch.float64, device=self.ctx.device)
        self.ctx.soa_to_aos(n, soa, out)
        return out

    def download(self, soas, n):
        """SoA device arrays -> fresh (N, 3) numpy arrays (synchronises)."""
        hosts = []
        for k, soa in enumerate(soas):
            d = self.buf.dev(f"out{k}_aos", (n, 3))
            self.ctx.soa_to_aos(n, soa, d)
            h = self.buf.host(f"out{k}_h", (n, 3))
            h.copy_(d, non_blocking=True)
            hosts.append(h)
        self.torch.cuda.current_stream(self.ctx.device).synchronize()
        return [h.numpy().copy() for h in hosts]
