"""Python side of libpolymer_fock: the FOURINDEX_ERI call and the device context.

* :func:`fourindex_eri` is the reference-facing call: host arrays in, host
  C_C/X_C out, through ``pfe_fourindex_eri`` (the entry point a Fortran
  ISO_C_BINDING shim binds).
* :class:`DeviceFock` keeps a ``pfe_context`` and runs Fock builds on
  device-resident torch tensors (``pfe_context_fock`` on torch's current
  stream) -- the form the GPU SCF loop uses.
* :func:`onee` computes the caller-side S_P/T_P/N_P on the device.

All of it needs the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np
import torch

from . import capi
from .capi import PfeCensus, PfeOneeArgs, check, lib
from .system import System, from_fortran, to_fortran


def onee_args(sysm: System):
    """The pfe_onee_args block of a system, and the arrays it points into (keep
    them alive for as long as the block is used)."""
    b, d = sysm.basis, sysm.deck
    keep = dict(p_shell=np.asfortranarray(b.p_shell.astype(np.int32)),
                ang=np.ascontiguousarray(b.p_shell_ang.astype(np.int32)),
                atom=np.ascontiguousarray(b.pgs_atom.astype(np.int32)),
                x=np.ascontiguousarray(b.pgs[:, 0]), y=np.ascontiguousarray(b.pgs[:, 1]),
                z=np.ascontiguousarray(b.pgs[:, 2]), zt=np.ascontiguousarray(b.zt),
                iatom=np.array(d.atoms, dtype=np.int32),
                ax=np.array([c[0] for c in d.coords]), ay=np.array([c[1] for c in d.coords]),
                az=np.array([c[2] for c in d.coords]), ig=np.asfortranarray(sysm.igamma))
    a = PfeOneeArgs()
    a.npgs, a.npshell, a.natom = b.npgs, b.npshell, d.natom
    a.p_shell = capi.iptr(keep['p_shell'])
    a.p_shell_ang = capi.iptr(keep['ang'])
    a.pgs_atom = capi.iptr(keep['atom'])
    a.pgsx, a.pgsy, a.pgsz = capi.dptr(keep['x']), capi.dptr(keep['y']), capi.dptr(keep['z'])
    a.zt = capi.dptr(keep['zt'])
    a.iatom = capi.iptr(keep['iatom'])
    a.atomx, a.atomy, a.atomz = capi.dptr(keep['ax']), capi.dptr(keep['ay']), capi.dptr(keep['az'])
    for k in range(3):
        a.cel1[k], a.cel2[k], a.period[k] = d.cel1[k], d.cel2[k], d.period[k]
    a.helix = d.helix
    a.igamma = capi.dptr(keep['ig'])
    return a, keep


def onee(sysm: System):
    """(S_P, T_P, N_P) cell-major from the device kernels (OVERLAP_KINETIC / NUCLEAR_ATTRACTION)."""
    L = lib()
    b = sysm.basis
    a, keep = onee_args(sysm)
    nc = sysm.ncell1
    n = b.npgs * b.npgs * nc
    s, t, v = np.zeros(n), np.zeros(n), np.zeros(n)
    check(L, L.pfe_overlap_kinetic(ctypes.byref(a), capi.dptr(s), capi.dptr(t)))
    check(L, L.pfe_nuclear_attraction(ctypes.byref(a), capi.dptr(v)))
    return (from_fortran(s, (nc,), b.npgs).copy(), from_fortran(t, (nc,), b.npgs).copy(),
            from_fortran(v, (nc,), b.npgs).copy())


def fourindex_eri(sysm: System, p_p: np.ndarray, p_p_helix: Optional[np.ndarray] = None,
                  **kw) -> Tuple[np.ndarray, np.ndarray]:
    """FOURINDEX_ERI through the C ABI with host buffers: cell-major P_P -> (C_C, X_C)."""
    L = lib()
    a, keep = sysm.pfe_args(p_p, p_p_helix, **kw)
    nc = sysm.ncell1
    n = sysm.basis.ncgs
    c = np.zeros(n * n * nc)
    x = np.zeros_like(c)
    check(L, L.pfe_fourindex_eri(ctypes.byref(a), capi.dptr(c), capi.dptr(x)))
    return from_fortran(c, (nc,), n).copy(), from_fortran(x, (nc,), n).copy()


def fourindex_eri_gradient(sysm: System, p_p: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """The two-electron nuclear gradient for the density P_P (molecules) through
    the C ABI: (grad_J, grad_K), each (natom, 3), the derivatives of
    1/2 sum (ij|kl) P_ij P_kl and of -1/4 sum (ij|kl) P_ik P_jl at fixed P."""
    L = lib()
    a, keep = sysm.pfe_args(p_p, None)
    natom = sysm.deck.natom
    atom = np.ascontiguousarray(sysm.basis.pgs_atom.astype(np.int32))
    gj = np.zeros(3 * natom)
    gk = np.zeros(3 * natom)
    check(L, L.pfe_fourindex_eri_gradient(ctypes.byref(a), capi.iptr(atom), natom, capi.dptr(gj), capi.dptr(gk)))
    return gj.reshape(3, natom).T.copy(), gk.reshape(3, natom).T.copy()


class DeviceFock:
    """A pfe_context bound to one System; callable as the SCF's FockBuilder."""

    def __init__(self, sysm: System, device: int = 0, primitive_targets: bool = False, **kw):
        self.L = lib()
        self.sys = sysm
        self.device = device
        h = ctypes.c_void_p()
        check(self.L, self.L.pfe_context_create(device, ctypes.byref(h)))
        self.ctx = h
        if primitive_targets:
            check(self.L, self.L.pfe_context_primitive_targets(self.ctx, 1))
        a, keep = sysm.pfe_args(None, None, **kw)
        check(self.L, self.L.pfe_context_setup(self.ctx, ctypes.byref(a)))
        nc, n = sysm.ncell1, sysm.basis.ncgs
        dev = torch.device('cuda', device)
        self.out_c = torch.empty((nc, n, n), dtype=torch.float64, device=dev)
        self.out_x = torch.empty((nc, n, n), dtype=torch.float64, device=dev)

    def census(self) -> dict:
        c = PfeCensus()
        check(self.L, self.L.pfe_context_census(self.ctx, ctypes.byref(c)))
        return {'quartets': c.quartets, 'quartets_ref': c.quartets_ref, 'flops': c.flops,
                'quartets_fp32': c.quartets_fp32, 'pairs': c.pairs, 'kernel_launches': c.kernel_launches}

    def autotune(self, p_p: torch.Tensor) -> None:
        """Pick the fastest execution variant per quartet class on this density (cell-major)."""
        pp = p_p.transpose(-1, -2).contiguous()
        s = torch.cuda.current_stream(self.device).cuda_stream
        check(self.L, self.L.pfe_context_autotune(self.ctx, ctypes.c_void_p(pp.data_ptr()), None, ctypes.c_void_p(s)))

    def force_variant(self, v: int) -> None:
        check(self.L, self.L.pfe_context_force_variant(self.ctx, v))

    def set_screening(self, mixed_cutoff: float = 0.0, density_tol: float = 0.0) -> None:
        """FP32 recursion below mixed_cutoff and density screening below density_tol (0: off)."""
        mode = capi.PFE_PREC_MIXED if mixed_cutoff > 0.0 else capi.PFE_PREC_FP64
        check(self.L, self.L.pfe_context_set_screening(self.ctx, mode, float(mixed_cutoff), float(density_tol)))

    def from_pc(self, p_c: torch.Tensor):
        """Molecules: contracted device P_C (ncgs x ncgs) -> (C_C, X_C), fully asynchronous."""
        pc = p_c.reshape(p_c.shape[-2:]).transpose(-1, -2).contiguous()
        s = torch.cuda.current_stream(self.device).cuda_stream
        check(self.L, self.L.pfe_context_fock_pc(self.ctx, ctypes.c_void_p(pc.data_ptr()),
                                                 ctypes.c_void_p(self.out_c.data_ptr()),
                                                 ctypes.c_void_p(self.out_x.data_ptr()), ctypes.c_void_p(s)))
        return self.out_c.transpose(-1, -2).clone(), self.out_x.transpose(-1, -2).clone()

    def run_fortran(self, d_pp: torch.Tensor, d_pph: Optional[torch.Tensor], out_c: torch.Tensor,
                    out_x: torch.Tensor, stream=None) -> None:
        """Raw call on Fortran-layout device buffers (no layout conversion)."""
        s = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        check(self.L, self.L.pfe_context_fock(self.ctx, ctypes.c_void_p(d_pp.data_ptr()),
                                              ctypes.c_void_p(d_pph.data_ptr()) if d_pph is not None else None,
                                              ctypes.c_void_p(out_c.data_ptr()),
                                              ctypes.c_void_p(out_x.data_ptr()), ctypes.c_void_p(s)))

    def __call__(self, p_p: torch.Tensor, p_ph: Optional[torch.Tensor] = None):
        """Cell-major device P_P (and P_P_HELIX) -> cell-major device (C_C, X_C)."""
        pp = p_p.transpose(-1, -2).contiguous()
        ph = p_ph.transpose(-1, -2).contiguous() if p_ph is not None else None
        self.run_fortran(pp, ph, self.out_c, self.out_x)
        return self.out_c.transpose(-1, -2).clone(), self.out_x.transpose(-1, -2).clone()

    def close(self):
        if self.ctx is not None:
            self.L.pfe_context_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def host_fock_builder(sysm: System, **kw):
    """A FockBuilder going through the host C ABI each call (the drop-in path)."""

    def f(p_p, p_ph):
        pp = p_p.detach().cpu().numpy()
        ph = p_ph.detach().cpu().numpy() if p_ph is not None else None
        c, x = fourindex_eri(sysm, pp, ph, **kw)
        return (torch.tensor(c, dtype=torch.float64, device=p_p.device),
                torch.tensor(x, dtype=torch.float64, device=p_p.device))
    return f


class DeviceBatch:
    """Fock builds of many molecules at once (``pfe_batch``): each quartet class
    is one kernel launch over the work of every molecule.  Densities and outputs
    live packed in one device buffer each, molecule k's ncgs x ncgs matrix
    (column-major) at ``off[k]``."""

    def __init__(self, systems, device: int = 0, **kw):
        self.L = lib()
        self.systems = list(systems)
        self.device = device
        h = ctypes.c_void_p()
        check(self.L, self.L.pfe_batch_create(device, ctypes.byref(h)))
        self.handle = h
        args, self._keep = [], []
        for s in self.systems:
            if s.ncell1 != 1:
                raise ValueError('a batch holds molecules only')
            a, keep = s.pfe_args(None, None, **kw)
            args.append(a)
            self._keep.append(keep)
        arr = (capi.PfeArgs * len(args))(*args)
        check(self.L, self.L.pfe_batch_setup(self.handle, arr, len(args)))
        off = (ctypes.c_int64 * (len(args) + 1))()
        n = self.L.pfe_batch_offsets(self.handle, off)
        if n != len(args):
            raise capi.FockError('pfe_batch_offsets: %d instances, expected %d' % (n, len(args)))
        self.off = [int(v) for v in off]
        self.ncgs = [s.basis.ncgs for s in self.systems]
        dev = torch.device('cuda', device)
        self.p_c = torch.zeros(self.off[-1], dtype=torch.float64, device=dev)
        self.out_c = torch.empty_like(self.p_c)
        self.out_x = torch.empty_like(self.p_c)

    def __len__(self) -> int:
        return len(self.systems)

    def census(self) -> dict:
        c = PfeCensus()
        check(self.L, self.L.pfe_batch_census(self.handle, ctypes.byref(c)))
        return {'quartets': c.quartets, 'quartets_ref': c.quartets_ref, 'flops': c.flops,
                'quartets_fp32': c.quartets_fp32, 'pairs': c.pairs, 'kernel_launches': c.kernel_launches}

    def set_screening(self, mixed_cutoff: float = 0.0, density_tol: float = 0.0) -> None:
        mode = capi.PFE_PREC_MIXED if mixed_cutoff > 0.0 else capi.PFE_PREC_FP64
        check(self.L, self.L.pfe_batch_set_screening(self.handle, mode, float(mixed_cutoff), float(density_tol)))

    def set_instance_screening(self, k: int, mixed_cutoff: float = 0.0, density_tol: float = 0.0) -> None:
        """Screening of molecule k alone (its launch record is rebuilt at the next build)."""
        mode = capi.PFE_PREC_MIXED if mixed_cutoff > 0.0 else capi.PFE_PREC_FP64
        check(self.L, self.L.pfe_batch_set_instance_screening(self.handle, int(k), mode, float(mixed_cutoff),
                                                              float(density_tol)))

    def view(self, packed: torch.Tensor, k: int) -> torch.Tensor:
        """Molecule k's matrix of a packed buffer (a transposed view: row-major indices)."""
        n = self.ncgs[k]
        return packed[self.off[k]:self.off[k + 1]].view(n, n).t()

    def autotune(self, p_c: torch.Tensor) -> None:
        """Time every execution variant per quartet class on packed densities p_c; keep the fastest."""
        s = torch.cuda.current_stream(self.device).cuda_stream
        check(self.L, self.L.pfe_batch_autotune(self.handle, ctypes.c_void_p(p_c.data_ptr()), ctypes.c_void_p(s)))

    def schedule(self) -> list:
        """(class, variant, tuned ms per variant, quartets) of every joined quartet class."""
        st = (capi.PfeKernelStat * 64)()
        n = self.L.pfe_batch_schedule(self.handle, st, 64)
        if n < 0:
            check(self.L, n)
        return [{'cls': '%04d' % x.cls, 'variant': x.variant, 'grid_mult': x.grid_mult,
                 'tuned_ms': list(x.tuned_ms), 'quartets': x.quartets} for x in st[:n]]

    def refresh(self, p_c: torch.Tensor) -> None:
        """Rewrite the launch records for densities packed in p_c with the current
        screening (before replaying a captured build; no replay may be in flight)."""
        check(self.L, self.L.pfe_batch_refresh(self.handle, ctypes.c_void_p(p_c.data_ptr())))

    def run_packed(self, p_c: torch.Tensor, out_c: torch.Tensor, out_x: torch.Tensor, stream=None) -> None:
        """Raw call on packed device buffers (pfe_batch_fock_pc), asynchronous."""
        s = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        check(self.L, self.L.pfe_batch_fock_pc(self.handle, ctypes.c_void_p(p_c.data_ptr()),
                                               ctypes.c_void_p(out_c.data_ptr()),
                                               ctypes.c_void_p(out_x.data_ptr()), ctypes.c_void_p(s)))

    def __call__(self, p_list):
        """List of device P_C (ncgs x ncgs) -> list of (C_C, X_C)."""
        for k, p in enumerate(p_list):
            self.view(self.p_c, k).copy_(p)
        self.run_packed(self.p_c, self.out_c, self.out_x)
        return [(self.view(self.out_c, k).clone(), self.view(self.out_x, k).clone()) for k in range(len(self))]

    def close(self):
        if self.handle is not None:
            self.L.pfe_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
