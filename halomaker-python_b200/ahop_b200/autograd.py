"""torch.autograd.Function wrappers over the hand-written adjoint kernels.

SPHDensity: rho(positions) with the neighbour lists held fixed (the finder's
lists, nvoisins per particle); backward runs ahop_density_adjoint, which
recomputes the kernel weights from positions instead of storing them.
HaloPotential: the direct-sum potential of every halo (FP64 form of
ahop_halo_props); backward runs ahop_epot_grad, whose per-particle gradient is
minus the direct-sum gravitational force.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from . import halo_props


class AhopAdjParams(C.Structure):
    _fields_ = [("nvoisins", C.c_int32), ("pad", C.c_int32), ("xlong", C.c_double), ("ylong", C.c_double),
                ("zlong", C.c_double)]


def _bind():
    lib = L.lib()
    lib.ahop_density_fixed.argtypes = [C.POINTER(AhopAdjParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                       C.c_void_p, C.c_void_p]
    lib.ahop_density_adjoint.argtypes = [C.POINTER(AhopAdjParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                         C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ahop_epot_grad.argtypes = [C.POINTER(halo_props.AhopHaloParams), C.c_void_p, C.c_void_p, C.c_int64,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def density_fixed(pos, mass, nei, box=1.0):
    """Density of every particle from fixed lists nei (n, nvoisins) int32 (0-based)."""
    lib = _bind()
    p = AhopAdjParams(nei.shape[1], 0, box, box, box)
    out = torch.empty(pos.shape[0], dtype=torch.float64, device=pos.device)
    L.check(lib.ahop_density_fixed(C.byref(p), pos.data_ptr(), mass.data_ptr(), nei.data_ptr(), pos.shape[0],
                                   out.data_ptr(), _stream()), "density_fixed")
    return out


class SPHDensity(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, mass, nei, box):
        pos = pos.contiguous()
        ctx.save_for_backward(pos, mass, nei)
        ctx.box = box
        return density_fixed(pos, mass, nei, box)

    @staticmethod
    def backward(ctx, gdens):
        pos, mass, nei = ctx.saved_tensors
        lib = _bind()
        p = AhopAdjParams(nei.shape[1], 0, ctx.box, ctx.box, ctx.box)
        gpos = torch.zeros_like(pos)
        g = gdens.contiguous().to(torch.float64)
        L.check(lib.ahop_density_adjoint(C.byref(p), pos.data_ptr(), mass.data_ptr(), nei.data_ptr(),
                                         pos.shape[0], g.data_ptr(), gpos.data_ptr(), _stream()), "density_adjoint")
        return gpos, None, None, None


class HaloPotential(torch.autograd.Function):
    """E_pot per halo (FP64 direct sum); off is a CPU int64 tensor of offsets."""

    @staticmethod
    def forward(ctx, pos, mass, off, Lbox, G=430.1):
        pos = pos.contiguous()
        dev = pos.device
        d_off = off.to(dev)
        nh = off.numel() - 1
        vel = torch.zeros_like(pos)
        out = torch.zeros((nh, halo_props.NF), dtype=torch.float64, device=dev)
        halo_props.compute_device(d_off, pos, vel, mass, mass, out, Lbox, 0.0, G, epot=1,
                                  stream=torch.cuda.current_stream())
        centre = out[:, halo_props.FIELDS.index("icenter")].to(torch.int32).contiguous()
        ctx.save_for_backward(pos, mass, d_off, centre)
        ctx.off = off
        ctx.Lbox, ctx.G = Lbox, G
        return out[:, halo_props.FIELDS.index("ep64")].clone()

    @staticmethod
    def backward(ctx, gh):
        pos, mass, d_off, centre = ctx.saved_tensors
        lib = _bind()
        p = halo_props.params(ctx.Lbox, 0.0, ctx.G, True, 1)
        gpos = torch.zeros_like(pos)
        h_off = np.ascontiguousarray(ctx.off.numpy(), np.int64)
        g = gh.contiguous().to(torch.float64)
        L.check(lib.ahop_epot_grad(C.byref(p), d_off.data_ptr(), h_off.ctypes.data, len(h_off) - 1, pos.data_ptr(),
                                   mass.data_ptr(), centre.data_ptr(), g.data_ptr(), gpos.data_ptr(), _stream()),
                "epot_grad")
        return gpos, None, None, None, None
