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
    energy_variational: Optional[float] = None   # E[P] with J/K built from the final P itself


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
        # a molecule (one cell, the Gamma point only) runs FOCK_BUILD in real arithmetic
        self.gamma_only = len(ks) == 1 and len(self.cells) == 1
        self._xorth = None   # canonical orthogonaliser of the overlap, fixed for the geometry


def _eigh(a: torch.Tensor):
    """torch.linalg.eigh, retried on the CPU if the device solver reports a failure."""
    try:
        return torch.linalg.eigh(a)
    except RuntimeError:
        e, v = torch.linalg.eigh(a.cpu())
        return e.to(a.device), v.to(a.device)


def _nvtx_iteration(iscf: int) -> None:
    """NVTX range of one SCF iteration (closes the previous one): the phases a
    profiler timeline shows around the Fock builds."""
    if iscf > 1:
        torch.cuda.nvtx.range_pop()
    torch.cuda.nvtx.range_push('SCF iteration %d' % iscf)


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


def core_guess(st: HostState) -> torch.Tensor:
    """Density of the core Hamiltonian T + V (no counterpart in the reference, whose
    guess is the nuclear-charge diagonal): FOCK_BUILD applied to F = T + V."""
    p_out, _, _, _ = fock_build(st, st.t_c + st.n_c)
    return p_out


@dataclasses.dataclass
class FastOptions:
    """Time-to-solution options of run_scf (no counterpart in the reference).

    incremental: build J/K from the change of the density since the last build
      (J(P) = J(P_ref) + J(P - P_ref); the build is linear in P), with a full
      rebuild every ``reset_every`` builds;
    density_tol: skip quartets with Schwarz*Schwarz*max|dP| below it in the
      incremental builds;
    density_tol_rel: when positive, the incremental builds' tolerance follows
      the RMS density change d of the previous iteration:
      min(max(density_tol, density_tol_rel * d), density_tol_max) -- loose
      while the density still moves, density_tol near convergence;
    mixed_cutoff: FP32 recursion where Schwarz*Schwarz*max|P| is below it;
    guess: 'nuclear' (the reference's), 'core', or a callable(System, HostState)
      returning a cell-major P_C tensor;
    final_full: once converged, one more iteration with a full FP64 build, whose
      energy is reported (the fast path is checked against the plain method);
    fallback_error: with a callable guess, if max|FPS - SPF| of the first
      iteration exceeds it, the SCF restarts from the nuclear-charge guess.
    """
    incremental: bool = True
    density_tol: float = 1e-11
    density_tol_rel: float = 1e-4
    density_tol_max: float = 1e-8
    mixed_cutoff: float = 0.0
    reset_every: int = 8
    guess: object = 'nuclear'
    final_full: bool = True
    fallback_error: float = 0.5   # a learned guess whose first commutator error exceeds it is replaced


def incremental_tol(opts: FastOptions, last_change: float) -> float:
    """Density tolerance of an incremental build after an iteration whose RMS
    density change was `last_change` (see FastOptions.density_tol_rel)."""
    if opts.density_tol_rel <= 0.0 or not math.isfinite(last_change):
        return opts.density_tol
    return min(max(opts.density_tol, opts.density_tol_rel * last_change), max(opts.density_tol_max, opts.density_tol))


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


def _fock_build_gamma(st: HostState, f_c: torch.Tensor):
    """FOCK_BUILD of a molecule: the k-sum is the identity, so the Hermitian
    problem is real symmetric; the canonical orthogonaliser of the overlap (a
    property of the geometry) is computed once and kept."""
    sysm, d = st.sys, st.sys.deck
    ncgs = sysm.basis.ncgs
    f = f_c[0]
    asym = float((f - f.T).abs().max())
    c2s = st.c2s
    if st._xorth is None:
        e_s, v_s = _eigh(c2s @ st.s_c[0] @ c2s.T)
        keep = e_s > d.lindep
        st._xorth = v_s[:, keep] / torch.sqrt(e_s[keep])
    x = st._xorth
    wf = c2s @ (0.5 * (f + f.T)) @ c2s.T
    e_f, c_f = _eigh(x.T @ wf @ x)
    eps = torch.full((1, ncgs), 1.0e99, dtype=torch.float64, device=st.device)
    eps[0, :e_f.shape[0]] = e_f
    co = c2s.T @ (x @ c_f)
    mu, occ = fermi_occupations(eps.cpu().numpy(), sysm.deck.nelectrons, d.temphf, st.nk_weight)
    occ_t = torch.tensor(occ[0, :co.shape[1]], dtype=torch.float64, device=st.device)
    p_out = ((co * occ_t) @ co.T * st.nk_weight).unsqueeze(0)
    return p_out, eps, mu, asym


def fock_build(st: HostState, f_c: torch.Tensor):
    """New density from the real-space Fock matrices (FOCK_BUILD)."""
    if st.gamma_only:
        return _fock_build_gamma(st, f_c)
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
    e_s, v_s = _eigh(ws_all)
    nk = len(st.kpts)
    eps = torch.full((nk, ncgs), 1.0e99, dtype=torch.float64, device=st.device)
    cos = []
    for k in range(nk):
        keep = e_s[k] > d.lindep
        x = v_s[k][:, keep] / torch.sqrt(e_s[k][keep]).to(cplx)
        fp = x.conj().T @ wf_all[k] @ x
        e_f, c_f = _eigh(fp)
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
    t, v, j, k = torch.stack([(p_c * st.t_c).sum(), (p_c * st.n_c).sum(), (p_c * 0.5 * c_c).sum(),
                              -(p_c * 0.25 * x_c).sum() * hfx]).tolist()
    comp = {'nuclear_repulsion': e_nuc, 'kinetic': t, 'nuclear_attraction': v, 'coulomb': j, 'exchange': k}
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


def variational_energy(st: HostState, fock, p_c: torch.Tensor, eps, mu) -> Tuple[float, float]:
    """E[P] with J/K of P itself from a full FP64 build; returns (energy, build seconds)."""
    d = st.sys.deck
    tf = time.perf_counter()
    if hasattr(fock, 'from_pc') and st.sys.ncell1 == 1:
        fock.set_screening()
        c_v, x_v = fock.from_pc(p_c)
    else:
        p_p = decontract(st, p_c)
        c_v, x_v = fock(p_p, rotate(st, p_p))
    tb = time.perf_counter() - tf
    e, _ = energy(st, p_c, c_v, x_v, d.hfexchange, st.sys.e_nuc, d.temphf, eps, mu, d.nelectrons)
    return e, tb


def run_scf(sysm: System, fock: FockBuilder, *, device='cpu', p_c0: Optional[np.ndarray] = None,
            max_cycles: Optional[int] = None, scfconv: Optional[float] = None,
            log: Optional[Callable[[str], None]] = None, raise_on_fail: bool = True,
            fast: Optional[FastOptions] = None, variational: bool = False,
            chk: Optional[str] = None) -> SCFResult:
    """SELF_CONSISTENT_FIELD with the Fock build supplied by ``fock``.

    ``fock(P_P, P_P_HELIX)`` maps cell-major primitive densities to cell-major
    contracted (C_C, X_C): the FOURINDEX_ERI contract.  With ``fast`` (molecules,
    a DeviceFock builder) the iterations use the options of FastOptions; without
    it the loop is the reference's.  The reference reports E with the new density
    and the J/K of the previous one; ``variational`` adds E[P] of the density of
    the last diagonalisation (idempotent, so E[P] is second order in its error)
    with its own full FP64 J/K: one more build, the energy two runs are compared by.
    ``chk``: the reference's JOBNAME.chk (polymer_b200/chk.py): the initial
    density is restored from it when it holds a compatible block
    (RESTORE_DENSITYMATRIX at SINGLEPOINT; otherwise the guess), and every
    iteration's block is written to it as STORE_DENSITYMATRIX does, so the
    Fortran driver can resume from this run and this run from the driver's.
    """
    t0 = time.perf_counter()
    d = sysm.deck
    st = HostState(sysm, device)
    if fast is not None and (sysm.ncell1 != 1 or not hasattr(fock, 'from_pc')):
        raise SCFError('the fast SCF options need a molecule and a device Fock builder')
    restored = None
    if chk is not None and p_c0 is None:
        from . import chk as chk_mod
        restored, msg = chk_mod.restore(chk, sysm.basis.ncgs, d.cel1)
        if log:
            log(msg)
    if p_c0 is not None:
        p_c = torch.tensor(p_c0, dtype=torch.float64, device=st.device)
    elif restored is not None:
        p_c = torch.tensor(restored, dtype=torch.float64, device=st.device)
    elif fast is not None and fast.guess == 'core':
        p_c = core_guess(st)
    elif fast is not None and callable(fast.guess):
        p_c = fast.guess(sysm, st).to(dtype=torch.float64, device=st.device)
    else:
        p_c = torch.tensor(guess_density(sysm), dtype=torch.float64, device=st.device)
    p_p = decontract(st, p_c)
    ref = None          # (P_C, C_C, X_C) of the last build, for incremental builds
    nbuild = 0
    final_pending = False
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
        _nvtx_iteration(iscf)
        ti = time.perf_counter()
        tf = time.perf_counter()
        if fast is None:
            p_ph = rotate(st, p_p)
            c_c, x_c = fock(p_p, p_ph)
        else:
            full = final_pending or ref is None or not fast.incremental or nbuild % max(1, fast.reset_every) == 0
            if full:
                fock.set_screening(mixed_cutoff=0.0 if final_pending else fast.mixed_cutoff)
                c_c, x_c = fock.from_pc(p_c)
            else:
                fock.set_screening(mixed_cutoff=fast.mixed_cutoff, density_tol=fast.density_tol)
                dc, dx = fock.from_pc(p_c - ref[0])
                c_c, x_c = ref[1] + dc, ref[2] + dx
            fock.set_screening()
            ref = (p_c.clone(), c_c, x_c)
            nbuild += 1
        fock_s += time.perf_counter() - tf
        f_c = st.t_c + st.n_c + c_c - 0.5 * x_c * d.hfexchange
        p_out, eps, mu, asym = fock_build(st, f_c)
        p_last = p_out
        dp = p_out - p_c
        dots = torch.stack([(h * dp).sum() for h in hist_d] + [(dp * dp).sum()]).cpu().numpy()
        pulay[iscf, iscf] = dots[-1]
        for i in range(1, iscf):
            pulay[i, iscf] = pulay[iscf, i] = dots[i - 1]
        dchg = math.sqrt(pulay[iscf, iscf] / denom)
        hist_in.append(p_c.clone())
        hist_d.append(dp.clone())
        if chk is not None:
            from . import chk as chk_mod
            chk_mod.store(chk, iscf, p_c.cpu().numpy(), p_out.cpu().numpy(), d.cel1, pulay=False)
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
            if fast is not None and fast.final_full and not final_pending:
                final_pending = True      # one more iteration on a full FP64 build checks the result
                e_old = e
                continue
            converged = True
            break
        final_pending = False
        e_old = e
    torch.cuda.nvtx.range_pop()   # the last iteration's range
    if not converged and raise_on_fail:
        raise SCFError('SCF CONVERGENCE NOT MET')
    e, comp = energy(st, p_c, c_c, x_c, d.hfexchange, sysm.e_nuc, d.temphf, eps, mu, nelec)
    e_var = None
    if variational:
        e_var, t_var = variational_energy(st, fock, p_last, eps, mu)
        fock_s += t_var
    return SCFResult(converged, e, comp, iters, p_c, eps, mu, fock_s, time.perf_counter() - t0, e_var)


def run_scf_fast(sysm: System, fock, *, opts: Optional[FastOptions] = None, device='cuda',
                 max_cycles: Optional[int] = None, scfconv: Optional[float] = None, ndiis: int = 8,
                 log: Optional[Callable[[str], None]] = None, raise_on_fail: bool = True) -> SCFResult:
    """Time-to-solution RHF for molecules (no counterpart in the reference).

    Same Hamiltonian, basis, orthogonalisation (LINDEP) and convergence test
    (RMS change of P_C below SCFCONV) as SELF_CONSISTENT_FIELD, with:
    Pulay's commutator DIIS on the Fock matrix (error FPS - SPF in the
    orthonormal basis, last ``ndiis`` iterations) in place of the reference's
    density extrapolation; J/K from the DeviceFock ``fock`` with the options of
    ``opts`` (incremental density-screened builds, FP32 recursion, guess); and,
    once converged, one more iteration on a full FP64 build whose energy
    E[P] = tr P (H + J/2 - K/4) of the idempotent density P is reported.
    Zero-temperature closed shells only (aufbau occupations).
    """
    opts = opts or FastOptions()
    t0 = time.perf_counter()
    d = sysm.deck
    if sysm.ncell1 != 1 or not hasattr(fock, 'from_pc'):
        raise SCFError('the fast SCF needs a molecule and a device Fock builder')
    if d.temphf > 0.0 or d.nelectrons % 2:
        raise SCFError('the fast SCF handles zero-temperature closed shells only')
    st = HostState(sysm, device)
    if opts.guess == 'core':
        p_c = core_guess(st)
    elif callable(opts.guess):
        p_c = opts.guess(sysm, st).to(dtype=torch.float64, device=st.device)
    else:
        p_c = torch.tensor(guess_density(sysm), dtype=torch.float64, device=st.device)
    learned = callable(opts.guess)
    fallback = False
    nocc = d.nelectrons // 2
    c2s, s0 = st.c2s, st.s_c[0]
    e_s, v_s = _eigh(c2s @ s0 @ c2s.T)
    keep = e_s > d.lindep
    w = c2s.T @ (v_s[:, keep] / torch.sqrt(e_s[keep]))     # orthonormal -> contracted Cartesian
    ws = w.T @ s0                                            # P_ortho = ws P ws^T
    h = st.t_c[0] + st.n_c[0]
    ncycles = max_cycles or d.scfcycles
    conv = d.scfconv if scfconv is None else scfconv
    denom = float(sysm.basis.ncgs ** 2)
    hist_f: List[torch.Tensor] = []
    hist_e: List[torch.Tensor] = []
    iters: List[SCFIteration] = []
    ref = None
    nbuild = 0
    final_pending = False
    converged = False
    fock_s = 0.0
    e = 0.0
    eps = None
    last_change = math.inf
    for iscf in range(1, ncycles + 1):
        _nvtx_iteration(iscf)
        ti = time.perf_counter()
        full = final_pending or ref is None or not opts.incremental or nbuild % max(1, opts.reset_every) == 0
        tf = time.perf_counter()
        if full:
            fock.set_screening(mixed_cutoff=0.0 if final_pending else opts.mixed_cutoff)
            c_c, x_c = fock.from_pc(p_c)
        else:
            fock.set_screening(mixed_cutoff=opts.mixed_cutoff, density_tol=incremental_tol(opts, last_change))
            dc, dx = fock.from_pc(p_c - ref[0])
            c_c, x_c = ref[1] + dc, ref[2] + dx
        fock.set_screening()
        fock_s += time.perf_counter() - tf
        ref = (p_c.clone(), c_c, x_c)
        nbuild += 1
        f = h + c_c[0] - 0.5 * d.hfexchange * x_c[0]
        f = 0.5 * (f + f.T)
        fo = w.T @ f @ w
        po = ws @ p_c[0] @ ws.T
        err = fo @ po - po @ fo
        hist_f.append(fo)
        hist_e.append(err)
        if len(hist_f) > ndiis:
            hist_f.pop(0)
            hist_e.pop(0)
        m = len(hist_f)
        e_vals = torch.stack([(p_c[0] * (h + 0.5 * c_c[0] - 0.25 * d.hfexchange * x_c[0])).sum(),
                              err.abs().max()] + [(hist_e[i] * hist_e[j]).sum() for i in range(m) for j in range(i, m)])
        vals = e_vals.cpu().numpy()
        e = float(vals[0]) + sysm.e_nuc
        fe = float(vals[1])
        if learned and iscf == 1 and fe > opts.fallback_error:
            # the learned guess is checked against the plain one: restart from the nuclear-charge guess
            fallback = True
            p_c = torch.tensor(guess_density(sysm), dtype=torch.float64, device=st.device)
            hist_f.clear()
            hist_e.clear()
            ref = None
            nbuild = 0
            if log:
                log('  1  guess error %.3e above %.3e: nuclear-charge guess' % (fe, opts.fallback_error))
            continue
        if m >= 2:
            bm = np.zeros((m + 1, m + 1))
            k = 2
            for i in range(m):
                for j in range(i, m):
                    bm[i, j] = bm[j, i] = vals[k]
                    k += 1
            bm[:m, m] = bm[m, :m] = -1.0
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            try:
                coef = np.linalg.solve(bm, rhs)[:m]
            except np.linalg.LinAlgError:
                coef = np.zeros(m)
                coef[-1] = 1.0
            fo = sum(float(cf) * fh for cf, fh in zip(coef, hist_f))
        eo, co = _eigh(fo)
        cc = w @ co[:, :nocc]
        p_new = (2.0 * cc @ cc.T).unsqueeze(0)
        eps = torch.full((1, sysm.basis.ncgs), 1.0e99, dtype=torch.float64, device=st.device)
        eps[0, :eo.shape[0]] = eo
        dchg = math.sqrt(float(((p_new - p_c) ** 2).sum()) / denom)
        last_change = dchg
        it = SCFIteration(iscf, m if m >= 2 else 0, fe, dchg, e, float(eo[nocc - 1]), time.perf_counter() - ti)
        iters.append(it)
        if log:
            log('%3d %3d  %9.3e %15.12f %17.10f %s %10.4f' % (iscf, it.idiis, fe, dchg, e, 'full' if full else 'incr',
                                                                it.seconds))
        if final_pending and dchg < conv:
            converged = True          # e is E[P] of the idempotent p_c with its own full FP64 J/K
            break
        final_pending = dchg < conv
        p_c = p_new
    torch.cuda.nvtx.range_pop()   # the last iteration's range
    if not converged and raise_on_fail:
        raise SCFError('SCF CONVERGENCE NOT MET')
    comp = {'total': e, 'guess_fallback': fallback, 'first_error': iters[0].asymmetry if iters else None}
    res = SCFResult(converged, e, comp, iters, p_c, eps, float(iters[-1].fermi) if iters else 0.0, fock_s,
                    time.perf_counter() - t0, e)
    return res
