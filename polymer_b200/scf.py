"""SCF loop around the Fock build: the caller of FOURINDEX_ERI.

Restates SELF_CONSISTENT_FIELD (src/pselfconsistentfield.f90:1-162) with its
helpers: ROTATE_DENSITYMATRIX (src/pdensitymatrix.f90:516-568), FOCK_BUILD
(src/pfock.f90:1-518: Fock assembly F=T+V+J-1/2*x*K, k-point Fourier sums,
Cartesian->spherical rows, canonical orthogonalisation with LINDEP, Fermi
level by bisection at TEMPHF (1e-4 K when zero), new density), STORE
(RMS density change and Pulay matrix, src/pdensitymatrix.f90:131-208), DIIS
(density extrapolation over the last min(8,ISCF) inputs, :253-339) or RELAX
(:212-249), DECONTRACT (P_P = CC^T P_C CC, :343-381) and ENERGY_CALC
(src/pselfconsistentfield.f90:487-648).  The DIIS history is kept in memory
instead of being re-read from JOBNAME.chk every iteration.

Written with torch so that the same code runs on the CPU (tests with the
oracle) and on the GPU next to the CUDA Fock build.  The EISPACK Hermitian
solver of the reference is replaced by torch.linalg.eigh; eigenvectors of
degenerate eigenvalues may differ, the density does not.
"""
from __future__ import annotations

import dataclasses
import math
import time
from typing import Callable, List, Optional, Tuple

import numpy as np
import torch

from .inputdeck import BOLTZMANN, PI
from .system import System


FockBuilder = Callable[[torch.Tensor, Optional[torch.Tensor]], Tuple[torch.Tensor, torch.Tensor]]


@dataclasses.dataclass
class SCFIteration:
    iscf: int
    idiis: int
    asymmetry: float
    density_change: float
    energy: float
    fermi: float
    seconds: float


@dataclasses.dataclass
class SCFResult:
    converged: bool
    energy: float
    components: dict
    iterations: List[SCFIteration]
    p_c: torch.Tensor
    epsilon: torch.Tensor
    fermi: float
    fock_seconds: float = 0.0
    wall_seconds: float = 0.0


class SCFError(RuntimeError):
    pass


class HostState:
    """Tensors of one SCF run (the INTEGRAL module arrays), on one device."""

    def __init__(self, sysm: System, device='cpu'):
        d = sysm.deck
        self.sys = sysm
        self.device = torch.device(device)
        f64 = dict(dtype=torch.float64, device=self.device)
        self.cc = torch.tensor(sysm.basis.cc, **f64)
        self.c2s = torch.tensor(sysm.c2s, **f64)
        self.s_c = torch.tensor(sysm.s_c, **f64)
        self.t_c = torch.tensor(sysm.t_c, **f64)
        self.n_c = torch.tensor(sysm.n_c, **f64)
        self.p2h = torch.tensor(sysm.p2h, **f64)
        self.cells = sysm.cells
        q = torch.tensor(sysm.cells, dtype=torch.float64, device=self.device)
        kv = d.kpoints
        ks = [(ix, iy, iz) for ix in range(-kv[0], max(0, kv[0] - 1) + 1)
              for iy in range(-kv[1], max(0, kv[1] - 1) + 1)
              for iz in range(-kv[2], max(0, kv[2] - 1) + 1)]
        self.kpts = ks
        ph = torch.zeros((len(ks), len(sysm.cells)), dtype=torch.float64, device=self.device)
        for n, (ix, iy, iz) in enumerate(ks):
            for ax, (ii, kk) in enumerate(zip((ix, iy, iz), kv)):
                if kk != 0:
                    ph[n] += PI * ii / kk * q[:, ax]
        self.phase = torch.polar(torch.ones_like(ph), ph)  # exp(i*phase), (nk, ncell)
        self.nk_weight = 1.0 / (max(1, 2 * kv[0]) * max(1, 2 * kv[1]) * max(1, 2 * kv[2]))


def guess_density(sysm: System) -> np.ndarray:
    """Nuclear-charge diagonal guess (GUESS_DENSITYMATRIX, src/pdensitymatrix.f90:83-127)."""
    b, d = sysm.basis, sysm.deck
    p = np.zeros((sysm.ncell1, b.ncgs, b.ncgs))
    c0 = sysm.cell_index(0, 0, 0)
    real_row = np.any(b.cc != 0.0, axis=1)
    for ia, z in enumerate(d.atoms):
        xyz = d.coords[ia]
        on = [k for k in range(b.ncgs) if real_row[k] and b.cgs[k, 0] == xyz[0]
              and b.cgs[k, 1] == xyz[1] and b.cgs[k, 2] == xyz[2]]
        if not on:
            raise SCFError('AN INTERNAL PROGRAM ERROR IS DETECTED IN GUESS_DENSITYMATRIX')
        for k in on:
            p[c0, k, k] = float(z) / len(on)
    return p


def decontract(st: HostState, p_c: torch.Tensor) -> torch.Tensor:
    """P_P(:,:,q) = CC^T P_C(:,:,q) CC."""
    return st.cc.T @ p_c @ st.cc


def rotate(st: HostState, p_p: torch.Tensor) -> Optional[torch.Tensor]:
    """P_P_HELIX(:,:,q2,q1) = P2H(q2)^T P_P(q1-q2) P2H(q1) for |q1-q2|<=CEL1 (x only)."""
    d = st.sys.deck
    if d.helix == 0.0:
        return None
    c1x, c2x = d.cel1[0], d.cel2[0]
    h3 = c1x + c2x
    n = p_p.shape[-1]
    out = torch.zeros((2 * h3 + 1, 2 * c2x + 1, n, n), dtype=p_p.dtype, device=p_p.device)
    for q2 in range(-c2x, c2x + 1):
        for q1 in range(-h3, h3 + 1):
            if -c1x <= q1 - q2 <= c1x:
                out[q1 + h3, q2 + c2x] = st.p2h[q2 + h3].T @ p_p[st.sys.cell_index(q1 - q2)] @ st.p2h[q1 + h3]
    return out


def fermi_occupations(eps: np.ndarray, nelec: int, temphf: float, nk_weight: float):
    """Fermi level by the reference's bracketing bisection (src/pfock.f90:339-424)."""
    t = temphf if temphf > 0.0 else 1.0e-4
    kt = BOLTZMANN * t

    def count(mu):
        with np.errstate(over='ignore'):
            occ = 2.0 / (np.exp((eps - mu) / kt) + 1.0)
        return occ.sum() * nk_weight - nelec

    f1, f2 = float(eps.min()), float(eps.max())
    f12 = 0.5 * (f1 + f2)
    for _ in range(100000):
        n1, n2, n12 = count(f1), count(f2), count(f12)
        if n1 > n12:
            raise SCFError('DETERMINATION OF FERMI ENERGY FAILED 2')
        if n12 > n2:
            raise SCFError('DETERMINATION OF FERMI ENERGY FAILED 3')
        if abs(n12) < 1.0e-10:
            break
        if n1 > 0.0 and n2 > 0.0:
            f2, f1 = f1, f1 - 0.1
        elif n1 < 0.0 and n2 < 0.0:
            f1, f2 = f2, f2 + 0.1
        elif n1 < 0.0 and n12 >= 0.0:
            f2 = f12
        elif n12 <= 0.0 and n2 > 0.0:
            f1 = f12
        else:
            raise SCFError('DETERMINATION OF FERMI ENERGY FAILED 4')
        f12 = 0.5 * (f1 + f2)
    else:
        raise SCFError('DETERMINATION OF FERMI ENERGY FAILED (no convergence)')
    mu = f12
    with np.errstate(over='ignore'):
        occ = 2.0 / (np.exp((eps - mu) / kt) + 1.0)
    return mu, occ


def fock_build(st: HostState, f_c: torch.Tensor):
    """New density from the real-space Fock matrices (FOCK_BUILD)."""
    sysm, d = st.sys, st.sys.deck
    ncgs = sysm.basis.ncgs
    cplx = torch.complex128
    ws_all = torch.einsum('kc,cij->kij', st.phase, st.s_c.to(cplx))
    wf_all = torch.einsum('kc,cij->kij', st.phase, f_c.to(cplx))
    asym = float((wf_all - wf_all.conj().transpose(-1, -2)).abs().max())
    wf_all = 0.5 * (wf_all + wf_all.conj().transpose(-1, -2))
    c2s = st.c2s.to(cplx)
    ws_all = c2s @ ws_all @ c2s.T
    wf_all = c2s @ wf_all @ c2s.T
    e_s, v_s = torch.linalg.eigh(ws_all)
    nk = len(st.kpts)
    eps = torch.full((nk, ncgs), 1.0e99, dtype=torch.float64, device=st.device)
    cos = []
    for k in range(nk):
        keep = e_s[k] > d.lindep
        x = v_s[k][:, keep] / torch.sqrt(e_s[k][keep]).to(cplx)
        fp = x.conj().T @ wf_all[k] @ x
        e_f, c_f = torch.linalg.eigh(fp)
        eps[k, :e_f.shape[0]] = e_f
        co = c2s.T @ (x @ c_f)           # CO(K,J) = sum_L WF(L,J) C2S(L,K)
        cos.append(co)
    eps_np = eps.cpu().numpy()
    mu, occ = fermi_occupations(eps_np, sysm.deck.nelectrons, d.temphf, st.nk_weight)
    occ_t = torch.tensor(occ, dtype=torch.float64, device=st.device)
    p_out = torch.zeros((sysm.ncell1, ncgs, ncgs), dtype=torch.float64, device=st.device)
    for k in range(nk):
        co = cos[k]
        m = co.shape[1]
        # WS(K,J) = sum_L f_L conj(CO(K,L)) CO(J,L); P_C_OUT(L,K,q) += Re WS(L,K) e^{i phase q} W
        ws = (co.conj() * occ_t[k, :m].to(cplx)) @ co.T
        p_out += (ws.unsqueeze(0) * st.phase[k].view(-1, 1, 1)).real * st.nk_weight
    return p_out, eps, mu, asym


def energy(st: HostState, p_c, c_c, x_c, hfx: float, e_nuc: float, temphf: float, eps, fermi, nelec):
    """ENERGY_CALC (src/pselfconsistentfield.f90:487-648), HF terms only."""
    comp = {'nuclear_repulsion': e_nuc,
            'kinetic': float((p_c * st.t_c).sum()),
            'nuclear_attraction': float((p_c * st.n_c).sum()),
            'coulomb': float((p_c * 0.5 * c_c).sum()),
            'exchange': float(-(p_c * 0.25 * x_c).sum() * hfx)}
    e = e_nuc + comp['kinetic'] + comp['nuclear_attraction'] + comp['coulomb'] + comp['exchange']
    if temphf > 0.0:
        comp['internal'] = e
        comp['chemical_potential'] = -2.0 * (nelec // 2) * fermi
        e += comp['chemical_potential']
        kt = BOLTZMANN * temphf
        s = 0.0
        ev = eps[0].cpu().numpy()  # Gamma point, as the reference (EPSILON(J,0,0,0))
        for ej in ev:
            with np.errstate(over='ignore'):
                fm = 1.0 / (math.exp(min((ej - fermi) / kt, 700.0)) + 1.0)
            fp = 1.0 - fm
            if fm > 0.0 and fp > 0.0:
                s += 2.0 * (fm * math.log(fm) + fp * math.log(fp)) * kt
        comp['entropy'] = s
        e += s
    comp['total'] = e
    return e, comp


def run_scf(sysm: System, fock: FockBuilder, *, device='cpu', p_c0: Optional[np.ndarray] = None,
            max_cycles: Optional[int] = None, scfconv: Optional[float] = None,
            log: Optional[Callable[[str], None]] = None, raise_on_fail: bool = True) -> SCFResult:
    """SELF_CONSISTENT_FIELD with the Fock build supplied by ``fock``.

    ``fock(P_P, P_P_HELIX)`` maps cell-major primitive densities to cell-major
    contracted (C_C, X_C): the FOURINDEX_ERI contract.
    """
    t0 = time.perf_counter()
    d = sysm.deck
    st = HostState(sysm, device)
    p_c = torch.tensor(guess_density(sysm) if p_c0 is None else p_c0, dtype=torch.float64, device=st.device)
    p_p = decontract(st, p_c)
    nelec = d.nelectrons
    if nelec % 2:
        raise SCFError('ODD NUMBER OF ELECTRONS')
    ncycles = max_cycles or d.scfcycles
    conv = d.scfconv if scfconv is None else scfconv
    hist_in: List[torch.Tensor] = []     # P_C of each iteration (chk column 1)
    hist_d: List[torch.Tensor] = []      # P_C_OUT - P_C of each iteration (chk column 2)
    pulay = np.zeros((ncycles + 1, ncycles + 1))
    iters: List[SCFIteration] = []
    fock_s = 0.0
    denom = float(sysm.ncell1 * sysm.basis.ncgs ** 2)
    e_old = 0.0
    converged = False
    c_c = x_c = None
    eps = None
    mu = 0.0
    for iscf in range(1, ncycles + 1):
        ti = time.perf_counter()
        p_ph = rotate(st, p_p)
        tf = time.perf_counter()
        c_c, x_c = fock(p_p, p_ph)
        fock_s += time.perf_counter() - tf
        f_c = st.t_c + st.n_c + c_c - 0.5 * x_c * d.hfexchange
        p_out, eps, mu, asym = fock_build(st, f_c)
        dp = p_out - p_c
        pulay[iscf, iscf] = float((dp * dp).sum())
        for i in range(1, iscf):
            pulay[i, iscf] = pulay[iscf, i] = float((hist_d[i - 1] * dp).sum())
        dchg = math.sqrt(pulay[iscf, iscf] / denom)
        hist_in.append(p_c.clone())
        hist_d.append(dp.clone())
        if d.diis != 0 and iscf >= d.diis and (iscf - d.diis) % 2 == 0:
            iterm = min(8, iscf)
            bm = np.zeros((iterm + 1, iterm + 1))
            for i in range(iterm):
                for j in range(iterm):
                    bm[j, i] = pulay[iscf - j, iscf - i]
                bm[i, iterm] = bm[iterm, i] = -1.0
            rhs = np.zeros(iterm + 1)
            rhs[iterm] = -1.0
            coef = np.linalg.solve(bm, rhs)
            p_new = torch.zeros_like(p_c)
            for k in range(iterm):            # C(k+1) pairs with iteration iscf-k
                p_new += float(coef[k]) * hist_in[iscf - 1 - k]
            p_c = p_new
            idiis = iterm
        else:
            p_c = d.scfrelax * p_out + (1.0 - d.scfrelax) * p_c
            idiis = 0
        p_p = decontract(st, p_c)
        e, comp = energy(st, p_c, c_c, x_c, d.hfexchange, sysm.e_nuc, d.temphf, eps, mu, nelec)
        it = SCFIteration(iscf, idiis, asym, dchg, e, mu, time.perf_counter() - ti)
        iters.append(it)
        if log:
            log('%3d %3d  %9.3e %15.12f %17.10f %15.10f %10.4f' % (iscf, idiis, asym, dchg, e,
                                                                   e - e_old if iscf > 1 else 0.0, it.seconds))
        if dchg < conv:
            converged = True
            break
        e_old = e
    if not converged and raise_on_fail:
        raise SCFError('SCF CONVERGENCE NOT MET')
    e, comp = energy(st, p_c, c_c, x_c, d.hfexchange, sysm.e_nuc, d.temphf, eps, mu, nelec)
    return SCFResult(converged, e, comp, iters, p_c, eps, mu, fock_s, time.perf_counter() - t0)
