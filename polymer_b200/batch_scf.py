"""Batched closed-shell SCF of many molecules on one GPU (no counterpart in the
reference, whose SELF_CONSISTENT_FIELD, src/pselfconsistentfield.f90:1-162,
runs one system).

Every SCF iteration of the whole batch does:

* one batched Fock build (``pfe_batch_fock_pc``: one kernel launch per quartet
  class over every molecule's work), incremental from the change of each
  molecule's density with density screening and optional FP32 recursion, as
  the fast single-molecule SCF (``scf.run_scf_fast``) does; screening is set
  per molecule, so a converged molecule (zero difference) skips all of its
  quartets;
* per group of molecules of equal size, batched FP64 products on the GPU:
  Fock assembly F = H + J - K/2, Pulay's commutator DIIS (error FPS - SPF in
  the orthonormal LINDEP basis), and the new density as the spectral projector
  on the nocc lowest orbitals, computed by second-order spectral projection
  (SP2: Niklasson, Phys. Rev. B 66, 155115 (2002), with the trace rule of
  Niklasson, Tymczak and Challacombe) -- products only, no diagonalisation;
* one device-to-host read of a few numbers per molecule (energy, DIIS error,
  density change) to decide convergence.

Convergence and energy are those of the single-molecule path: RMS change of
P_C below SCFCONV, then one more iteration on a full FP64 build whose energy
E[P] = tr P (H + J/2 - K/4) + E_nuc of the idempotent density is reported.
"""
from __future__ import annotations

import dataclasses
import math
import time
from typing import Callable, List, Optional, Sequence

import numpy as np
import torch
from torch.cuda import nvtx

from . import fock as fock_mod
from . import scf_ops
from .scf import SCFError, guess_density, incremental_tol
from .system import System

F64 = torch.float64

# per-molecule states of one iteration
_FULL, _INCR, _FINAL, _DONE = 0, 1, 2, 3


@dataclasses.dataclass
class BatchOptions:
    """incremental / density_tol(_rel, _max) / mixed_cutoff / reset_every as in
    scf.FastOptions (per molecule, from its own density change);
    guess: 'nuclear' (the reference's GUESS_DENSITYMATRIX), 'core', or an object
    with ``raw(sysm) -> np.ndarray`` (and optionally ``raw_many(systems)``)
    giving an unpurified contracted density per molecule (the learned guess),
    purified here on the GPU and checked by
    ``fallback_error`` (first DIIS error above it: restart from 'nuclear')."""
    incremental: bool = True
    density_tol: float = 1e-11
    density_tol_rel: float = 1e-4
    density_tol_max: float = 1e-8
    mixed_cutoff: float = 0.0
    reset_every: int = 8
    guess: object = 'nuclear'
    fallback_error: float = 0.5
    ndiis: int = 8
    sp2_tol: float = 1e-12
    sp2_max: int = 200


@dataclasses.dataclass
class BatchResult:
    energy: np.ndarray          # E[P] per molecule (Eh), input order
    converged: np.ndarray       # bool per molecule
    iterations: np.ndarray      # SCF iterations per molecule (to convergence)
    builds: int                 # batched Fock builds
    seconds: float
    first_error: np.ndarray     # max|FPS - SPF| of the first iteration per molecule
    fallback: np.ndarray        # the learned guess was rejected
    p_c: List[torch.Tensor]     # converged contracted densities, input order
    sp2_steps: int              # SP2 products over the run (per group, summed)
    phases: Optional[dict] = None   # seconds per phase when profiled (see run_batch_scf)


class _Group:
    """Molecules of one size (ncgs, nocc), contiguous in the packed buffers."""

    def __init__(self, members: List[int], systems: List[System], lo: int, device):
        s0 = systems[members[0]]
        self.members = members
        self.n = s0.basis.ncgs
        self.nocc = s0.deck.nelectrons // 2
        self.B = len(members)
        self.lo, self.hi = lo, lo + self.B * self.n * self.n
        n, B = self.n, self.B
        f64 = dict(dtype=F64, device=device)
        self.h = torch.empty((B, n, n), **f64)
        self.w = torch.zeros((B, n, n), **f64)
        self.ws = torch.zeros((B, n, n), **f64)
        self.pad = torch.zeros((B, n), dtype=torch.bool, device=device)
        self.hfx = torch.empty((B, 1, 1), **f64)
        self.e_nuc = torch.empty(B, **f64)
        ns = s0.c2s.shape[0]
        c2s = torch.empty((B, ns, n), **f64)
        s = torch.empty((B, n, n), **f64)
        for i, k in enumerate(members):
            sysm = systems[k]
            if (sysm.basis.ncgs, sysm.deck.nelectrons // 2, sysm.c2s.shape[0]) != (n, self.nocc, ns):
                raise SCFError('a batch group holds molecules of one size')
            c2s[i] = torch.tensor(sysm.c2s, **f64)
            s[i] = torch.tensor(sysm.s_c[0], **f64)
            self.h[i] = torch.tensor(sysm.t_c[0] + sysm.n_c[0], **f64)
            self.hfx[i] = sysm.deck.hfexchange
            self.e_nuc[i] = sysm.e_nuc
            lindep = sysm.deck.lindep
        # canonical orthogonalisation (LINDEP), one batched solver call; dropped
        # directions become zero columns, marked in `pad`
        e_s, v_s = torch.linalg.eigh(c2s @ s @ c2s.transpose(1, 2))
        keep = e_s > lindep
        if int(keep.sum(-1).min()) < self.nocc:
            raise SCFError('fewer independent functions than occupied orbitals')
        scale = torch.where(keep, 1.0 / torch.sqrt(e_s.clamp_min(lindep)), torch.zeros_like(e_s))
        self.w[:, :, :ns] = c2s.transpose(1, 2) @ (v_s * scale[:, None, :])
        self.ws = self.w.transpose(1, 2) @ s
        self.pad[:, :ns] = ~keep
        self.pad[:, ns:] = True
        self.nd = 0   # DIIS history slots in use
        self.slot = 0

    def view(self, packed: torch.Tensor) -> torch.Tensor:
        return packed[self.lo:self.hi].view(self.B, self.n, self.n)


def sp2_projector(f: torch.Tensor, nocc: int, pad: torch.Tensor, tol: float = 1e-12, max_steps: int = 200,
                  first_check: int = 12, fixed_steps: Optional[int] = None, ops=None):
    """Projector on the `nocc` lowest eigenvectors of each symmetric f [B, n, n]
    (slots marked in `pad` [B, n] are decoupled and left empty), by SP2.

    Gershgorin bounds [lo, hi] of the spectrum map f to X0 = (hi - f)/(hi - lo)
    with eigenvalues in [0, 1], occupied ones nearest 1; each step replaces X by
    X^2 or 2X - X^2, whichever brings tr X^2 closer to nocc.  Adaptive mode runs
    until the idempotency defect tr(X - X^2) before a step is below `tol` for
    every matrix (checked after `first_check` steps, then every other step);
    with `fixed_steps` it runs exactly that many steps and reads nothing back
    (the form a CUDA graph can hold).  `ops`: scf_ops implementation (default:
    the one for f's device).  Returns (X, steps, defect per matrix)."""
    ops = ops or scf_ops.ops_for(f.device)
    x = ops.sp2_init(f, pad)
    steps = 0
    while True:
        x2 = torch.bmm(x, x)
        defect = ops.sp2_step(x, x2, nocc)
        steps += 1
        if fixed_steps is not None:
            if steps >= fixed_steps:
                return x, steps, defect
            continue
        if steps >= first_check and steps % 2 == 0 and float(defect.max()) < tol:
            return x, steps, defect
        if steps >= max_steps:
            raise SCFError('SP2 projection did not converge')


def pulay_coefficients(hist_e: torch.Tensor, valid: torch.Tensor, slot: torch.Tensor) -> torch.Tensor:
    """Pulay coefficients of the valid history slots (scf_ops.pulay_coefficients)."""
    return scf_ops.pulay_coefficients(hist_e, valid, slot)


def _check_system(sysm: System) -> None:
    d = sysm.deck
    if sysm.ncell1 != 1:
        raise SCFError('the batched SCF takes molecules only')
    if d.temphf > 0.0 or d.nelectrons % 2:
        raise SCFError('the batched SCF handles zero-temperature closed shells only')


def _key(sysm: System):
    return (sysm.basis.ncgs, sysm.deck.nelectrons // 2, sysm.c2s.shape[0])


def sorted_order(systems: Sequence[System]) -> List[int]:
    """The order the batch keeps molecules in: grouped by size (a DeviceBatch
    passed to run_batch_scf must hold the systems in this order)."""
    return sorted(range(len(systems)), key=lambda k: _key(systems[k]))


def _projector(g: _Group, f_ortho: torch.Tensor, opts: BatchOptions, ops, fixed: Optional[int] = None):
    """W D W^T with D the SP2 projector of f_ortho (P_C is twice it); adaptive steps unless `fixed`."""
    d, steps, defect = sp2_projector(f_ortho, g.nocc, g.pad, opts.sp2_tol, opts.sp2_max,
                                     first_check=max(8, g.sp2_last - 2), fixed_steps=fixed, ops=ops)
    if fixed is None:
        g.sp2_last = steps
        g.sp2_seen = max(g.sp2_seen, steps)
    return torch.bmm(torch.bmm(g.w, d), g.w.transpose(1, 2)), steps, defect


def run_batch_scf(systems: Sequence[System], opts: Optional[BatchOptions] = None, device=0,
                  max_cycles: Optional[int] = None, scfconv: Optional[float] = None,
                  batch: Optional['fock_mod.DeviceBatch'] = None,
                  log: Optional[Callable[[str], None]] = None, raise_on_fail: bool = True,
                  profile: bool = False, graph: bool = False) -> BatchResult:
    """RHF of every molecule of `systems` (zero temperature, closed shells) as one batch.

    ``device``: a CUDA device index (the batch is then built here), or any torch
    device together with a ``batch`` object offering the DeviceBatch interface
    (``off``, ``systems``, ``view``, ``run_packed``, ``set_instance_screening``).

    ``graph``: from the third iteration on, the device part of an iteration
    (outcome of the last one, density differences, the batched build, Fock
    assembly, DIIS, SP2 with a fixed step count, the statistics) is one CUDA
    graph replay; the host reads the statistics, sets the per-molecule
    screening and masks, and replays.  The SP2 step count is the largest the
    eager iterations needed plus a margin, raised (and the graph recaptured)
    whenever a replay leaves a projector defect above the tolerance."""
    opts = opts or BatchOptions()
    t0 = time.perf_counter()
    dev = torch.device('cuda', device) if isinstance(device, int) else torch.device(device)
    graph = graph and dev.type == 'cuda'
    nmol = len(systems)
    for s in systems:
        _check_system(s)
    order = sorted_order(systems)
    ssys = [systems[k] for k in order]
    learned = not isinstance(opts.guess, str)
    fb = batch if batch is not None else fock_mod.DeviceBatch(ssys, dev.index or 0)
    if len(fb) != nmol or any(a is not b for a, b in zip(fb.systems, ssys)):
        raise SCFError('the DeviceBatch must hold the systems in sorted_order')
    groups: List[_Group] = []
    k = 0
    while k < nmol:
        k1 = k
        while k1 < nmol and _key(ssys[k1]) == _key(ssys[k]):
            k1 += 1
        g = _Group(list(range(k, k1)), ssys, fb.off[k], dev)
        g.sl = slice(k, k1)
        g.sp2_last = g.sp2_seen = 0
        g.sp2_fixed = None
        groups.append(g)
        k = k1
    ops = scf_ops.ops_for(dev)
    conv = np.array([s.deck.scfconv if scfconv is None else scfconv for s in ssys])
    ncycles = max_cycles or max(s.deck.scfcycles for s in ssys)
    total = fb.off[-1]
    f64 = dict(dtype=F64, device=dev)
    p, p_ref, c_ref, x_ref = (torch.zeros(total, **f64) for _ in range(4))
    dp, dc, dx, p_new = (torch.zeros(total, **f64) for _ in range(4))
    sp2_steps = [0]
    # eager iterations: host (density update), build, update (DIIS, projector);
    # graph iterations: capture (its eager run and the capture) or replay (the
    # host's per-molecule bookkeeping, then build and update in one replay)
    phases = {'setup': 0.0, 'guess': 0.0, 'build': 0.0, 'update': 0.0, 'host': 0.0, 'capture': 0.0, 'replay': 0.0}
    tmark = [time.perf_counter()]

    def mark(name):
        # with `profile`, wall time per phase (the device is synchronised at each mark)
        if profile:
            if dev.type == 'cuda':
                if torch.cuda.is_current_stream_capturing():
                    return
                torch.cuda.synchronize(dev)
            t = time.perf_counter()
            phases[name] += t - tmark[0]
            tmark[0] = t

    mark('setup')

    def nuclear(kk: int) -> torch.Tensor:
        return torch.tensor(guess_density(ssys[kk])[0], **f64)

    # ---- initial densities
    if opts.guess == 'nuclear':
        for kk in range(nmol):
            fb.view(p, kk).copy_(nuclear(kk))
    elif opts.guess == 'core':
        for g in groups:
            q, st, _ = _projector(g, g.w.transpose(1, 2) @ g.h @ g.w, opts, ops)
            g.view(p).copy_(2.0 * q)
            sp2_steps[0] += st
    elif learned:
        # occupied natural orbitals of the predicted density: the projector on the
        # nocc lowest eigenvectors of -D, D = P/2 in the orthonormal basis
        raws = opts.guess.raw_many(ssys) if hasattr(opts.guess, 'raw_many') else [opts.guess.raw(s) for s in ssys]
        for kk in range(nmol):
            fb.view(p, kk).copy_(torch.tensor(np.asarray(raws[kk]), **f64))
        for g in groups:
            dm = 0.5 * g.ws @ g.view(p) @ g.ws.transpose(1, 2)
            q, st, _ = _projector(g, -0.5 * (dm + dm.transpose(1, 2)), opts, ops)
            g.view(p).copy_(2.0 * q)
            sp2_steps[0] += st
    else:
        raise SCFError('unknown guess %r' % (opts.guess,))
    p_nuc = None
    if learned:
        p_nuc = torch.zeros(total, **f64)
        for kk in range(nmol):
            fb.view(p_nuc, kk).copy_(nuclear(kk))
    mark('guess')

    D = max(1, opts.ndiis)
    for g in groups:
        g.hist_f = torch.zeros((g.B, D, g.n, g.n), **f64)
        g.hist_e = torch.zeros((g.B, D, g.n, g.n), **f64)
        g.valid = torch.zeros((g.B, D), dtype=torch.bool, device=dev)
        ops.prepare(g)
    # device-side inputs of an iteration (fixed addresses: a captured graph reads them)
    take_t = torch.zeros(nmol, dtype=torch.bool, device=dev)
    restart_t = torch.zeros(nmol, dtype=torch.bool, device=dev)
    incr_t = torch.zeros(nmol, **f64)
    live_t = torch.ones(nmol, **f64)
    slot_t = torch.zeros(1, dtype=torch.long, device=dev)
    stats_t = torch.zeros((nmol, 4), **f64)

    def device_step(fixed: bool):
        """The device part of one iteration (no host synchronisation when `fixed`)."""
        for g in groups:
            sl = g.sl
            ops.next_density(g, g.view(p), g.view(p_new), g.view(p_nuc) if p_nuc is not None else None, take_t[sl],
                             restart_t[sl], incr_t[sl], live_t[sl], g.view(p_ref), g.view(dp))
        mark('host')
        nvtx.range_push('batched Fock build')
        fb.run_packed(dp, dc, dx)
        nvtx.range_pop()
        mark('build')
        nvtx.range_push('Fock assembly, DIIS, SP2 projector')
        for g in groups:
            sl = g.sl
            pv = g.view(p)
            f, e = ops.fock_assemble(g, g.view(dc), g.view(dx), g.view(c_ref), g.view(x_ref), pv, g.view(p_ref),
                                     incr_t[sl])
            wt = g.w.transpose(1, 2)
            fo = torch.bmm(torch.bmm(wt, f), g.w)
            po = torch.bmm(torch.bmm(g.ws, pv), g.ws.transpose(1, 2))
            # commutator F_o P_o - P_o F_o = A - A^T with A = F_o P_o (both symmetric)
            fe = ops.commutator(g, torch.bmm(fo, po), fo, slot_t)
            fx = ops.diis(g, slot_t)
            q, st, defect = _projector(g, fx, opts, ops, g.sp2_fixed if fixed else None)
            sp2_steps[0] += st
            ops.finish(g, 2.0, q, pv, g.view(p_new), e, fe, defect, stats_t[sl])
        slot_t.add_(1).remainder_(D)
        nvtx.range_pop()

    state = np.full(nmol, _FULL)
    nbuild = np.zeros(nmol, dtype=int)
    have_ref = np.zeros(nmol, dtype=bool)
    final_pending = np.zeros(nmol, dtype=bool)
    done = np.zeros(nmol, dtype=bool)
    converged = np.zeros(nmol, dtype=bool)
    first = np.ones(nmol, dtype=bool)
    fallback = np.zeros(nmol, dtype=bool)
    first_err = np.zeros(nmol)
    energy = np.zeros(nmol)
    iters = np.zeros(nmol, dtype=int)
    last_change = np.full(nmol, np.inf)
    take = np.zeros(nmol, dtype=bool)
    restart = np.zeros(nmol, dtype=bool)
    screen = [None] * nmol
    builds = 0
    cuda_graph = None
    replays = 0
    for it in range(1, ncycles + 1):
        if it > 1:
            nvtx.range_pop()
        nvtx.range_push('batched SCF iteration %d' % it)
        # ---- per-molecule build mode and screening
        for kk in range(nmol):
            if done[kk]:
                st, sc = _DONE, (0.0, max(opts.density_tol, 1e-300))
            elif final_pending[kk]:
                st, sc = _FINAL, (0.0, 0.0)
            elif not have_ref[kk] or not opts.incremental or nbuild[kk] % max(1, opts.reset_every) == 0:
                st, sc = _FULL, (opts.mixed_cutoff, 0.0)
            else:
                st, sc = _INCR, (opts.mixed_cutoff, incremental_tol(opts, float(last_change[kk])))
            state[kk] = st
            if screen[kk] != sc:
                fb.set_instance_screening(kk, *sc)
                screen[kk] = sc
        take_t.copy_(torch.from_numpy(take))
        restart_t.copy_(torch.from_numpy(restart))
        incr_t.copy_(torch.from_numpy(((state == _INCR) | (state == _DONE)).astype(np.float64)))
        live_t.copy_(torch.from_numpy((state != _DONE).astype(np.float64)))
        if graph and it >= 3:
            if cuda_graph is None:
                for g in groups:
                    g.sp2_fixed = g.sp2_fixed or (g.sp2_seen + 6)
                fb.refresh(dp)
                side = torch.cuda.Stream(dev)
                side.wait_stream(torch.cuda.current_stream(dev))
                with torch.cuda.stream(side):
                    device_step(True)            # this iteration, run eagerly on the capture stream
                torch.cuda.current_stream(dev).wait_stream(side)
                torch.cuda.synchronize(dev)
                host_stats = stats_t.cpu().numpy()
                cuda_graph = torch.cuda.CUDAGraph()
                with torch.cuda.graph(cuda_graph, stream=side):
                    device_step(True)
                torch.cuda.synchronize(dev)
                mark('capture')
            else:
                fb.refresh(dp)
                cuda_graph.replay()
                replays += 1
                host_stats = stats_t.cpu().numpy()
                mark('replay')
        else:
            device_step(False)
            host_stats = stats_t.cpu().numpy()
        builds += 1
        nbuild[~done] += 1
        mark('update')
        host = host_stats
        if cuda_graph is not None and float(host[~done, 3].max() if (~done).any() else 0.0) > 1e3 * opts.sp2_tol:
            # a replay's projectors are not converged: more SP2 steps, capture again
            for g in groups:
                g.sp2_fixed += 8
            cuda_graph = None
        take[:] = False
        restart[:] = False
        for kk in range(nmol):
            if done[kk]:
                continue
            e_k, fe_k, dchg_k, _ = host[kk]
            iters[kk] = it
            last_change[kk] = dchg_k
            have_ref[kk] = True
            if first[kk]:
                first[kk] = False
                first_err[kk] = fe_k
                if learned and fe_k > opts.fallback_error:
                    # the learned guess is checked against the plain one: restart from the nuclear-charge guess
                    fallback[kk] = True
                    restart[kk] = True
                    have_ref[kk] = False
                    nbuild[kk] = 0
                    last_change[kk] = np.inf
                    continue
            if final_pending[kk] and dchg_k < conv[kk]:
                converged[kk] = done[kk] = True
                energy[kk] = e_k
                continue
            final_pending[kk] = dchg_k < conv[kk]
            take[kk] = True
        if log:
            nd = int(done.sum())
            log('%3d  done %4d/%d  max DIIS error %.3e  max dP %.3e%s' % (
                it, nd, nmol, float(host[~done, 1].max()) if nd < nmol else 0.0,
                float(host[~done, 2].max()) if nd < nmol else 0.0, '  (graph)' if cuda_graph is not None else ''))
        if done.all():
            break
    nvtx.range_pop()   # the last iteration's range
    # apply the last outcome (molecules that did not converge keep their newest density)
    for g in groups:
        tk = torch.from_numpy(take[g.sl]).to(dev)
        g.view(p).copy_(torch.where(tk[:, None, None], g.view(p_new), g.view(p)))
    if dev.type == 'cuda':
        torch.cuda.synchronize(dev)
    if not converged.all() and raise_on_fail:
        raise SCFError('SCF CONVERGENCE NOT MET for %d of %d molecules' % (int((~converged).sum()), nmol))
    inv = np.empty(nmol, dtype=int)
    inv[np.array(order)] = np.arange(nmol)
    p_out = [fb.view(p, int(inv[k])).t().clone() for k in range(nmol)]
    if profile:
        phases['graph_replays'] = replays
    res = BatchResult(energy[inv], converged[inv], iters[inv], builds, time.perf_counter() - t0, first_err[inv],
                      fallback[inv], p_out, sp2_steps[0], phases if profile else None)
    if batch is None:
        fb.close()
    return res
