#!/usr/bin/env python
"""Fock-build throughput of the CUDA library on the alkane workload.

One step = one direct J/K build (FOURINDEX_ERI) of all-trans C20H42 in
6-31G** (seeded jitter 0.02 A, INTTOL 1e-10, FP64) with a fixed density.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value: Fock builds/s with P_P resident in HBM (pfe_context_fock), CUDA
  events on the launch stream, L2 flushed (256 MiB write) before every step.
* e2e: the same metric through the reference-facing C ABI pfe_fourindex_eri
  with pinned host buffers (P_P upload and C_C/X_C download inside the step).
* roofline: the kernel with the largest time share, its algorithmic FP64 flops
  over its event-timed duration, against the FP64 FMA-pipe peak measured here.
* cpu_baseline: the CPU oracle (a restatement of the reference loop) on a
  bounded sample of bra shells, extrapolated to one full build, one core.
* scf: time to a converged SCF of the same molecule, the reference's loop with
  full FP64 builds against the time-to-solution path (batch_scf / scf.run_scf_fast).
* batch (--batch N, default 256; 0 skips it): N uneven water clusters in
  cc-pVDZ as one batch -- batched Fock builds/s (default schedule and after the
  batch autotuner), and the time to converged SCF of the whole set, one plain
  FP64 GPU SCF per molecule against the batched SCF (with and without the
  learned guess and the FP32 recursion).
* other_configs: C40H82 6-31G** and the helical chain at CUTOFF 5/10 (build
  rates; the chain also with its far cells in FP32).
* mixed: the C20H42 build with the FP32 recursion below Schwarz x density
  1e-6, its max|dF| and dE against the FP64 build.
* N > 1 (torchrun): every rank computes its share of the quartet chunks and the
  J/K matrices are summed with one NCCL all-reduce -- the reference's
  MPI_ALLREDUCE of J/K; total work is fixed (strong scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = 'Fock builds/s & time-to-converged SCF (1e-8 Eh) vs plain FP64 GPU, 1 B200'
N_ALKANE = 20
INTTOL = 1.0e-10


def workload_name(n=N_ALKANE):
    return 'C%dH%d 6-31G** all-trans alkane (seeded jitter 0.02 A), molecule, INTTOL %.0e' % (n, 2 * n + 2, INTTOL)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""

    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.th = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + self.FIELDS,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        mhz, mx, reasons = [], 0.0, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            p = [x.strip() for x in ln.split(',')]
            if len(p) < 9:
                continue
            try:
                mhz.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == 'active':
                    reasons.add(nm)
        return {'sm_mhz': statistics.median(mhz) if mhz else None, 'sm_max_mhz': mx or None,
                'reasons': sorted(reasons), 'samples': len(mhz)}


def build_problem(device: int):
    import numpy as np
    import torch
    from polymer_b200 import fock, geometry, scf, system
    deck = geometry.alkane_deck(N_ALKANE, inttol=INTTOL)
    sysm = system.build_system(deck, fock.onee)
    # a realistic density: one SCF iteration from the nuclear-charge guess
    st = scf.HostState(sysm, 'cuda:%d' % device)
    p_c = torch.tensor(scf.guess_density(sysm), dtype=torch.float64, device=st.device)
    p_p = scf.decontract(st, p_c)
    df0 = fock.DeviceFock(sysm, device)
    c_c, x_c = df0(p_p)
    p_out, _, _, _ = scf.fock_build(st, st.t_c + st.n_c + c_c - 0.5 * x_c)
    p_p = scf.decontract(st, p_out)
    df0.close()
    return sysm, p_p, p_out


def measure_fp64_peak(device: int) -> float:
    import ctypes
    from polymer_b200 import capi
    L = capi.lib()
    v = ctypes.c_double(0.0)
    capi.check(L, L.pfe_measure_fp64_peak(device, ctypes.byref(v)))
    return v.value


def ncu_traffic_per_launch():
    """DRAM bytes of the dominant kernel from the committed ncu summary, if present."""
    path = os.path.join(ROOT, 'profiles', 'roofline_traffic.json')
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return None


def cpu_baseline(sysm, p_p_np, budget_s: float = 15.0):
    """Oracle on bra shells I = 0 (mod stride), extrapolated to a full build, 1 thread.

    The cost per bra shell varies by orders of magnitude (s shells against d
    shells), so the stride is sized from a first sample spread over the whole
    shell list (every n/8-th shell), not from one shell."""
    import oracle
    n = sysm.basis.npshell
    t0 = time.perf_counter()
    oracle.fourindex_eri_sample(sysm, p_p_np, n + 1, n)   # no bra shell: the fixed KL/Schwarz part
    t_fixed = time.perf_counter() - t0

    def sample(stride):
        t = time.perf_counter()
        oracle.fourindex_eri_sample(sysm, p_p_np, stride, 0)
        return time.perf_counter() - t - t_fixed, len(range(0, n, stride))

    stride = max(1, n // 8)
    t_s, sampled = sample(stride)
    per = max(t_s, 1e-6) / sampled                 # mean seconds per bra shell
    want = int(max(1.0, (budget_s - t_fixed) / per))
    if want > sampled:
        stride = max(1, -(-n // want))
        t_s, sampled = sample(stride)
    t_full = t_fixed + max(t_s, 0.0) * n / sampled
    return {'value': 1.0 / t_full, 'unit': 'Fock builds/s', 'cores': 1, 'kind': 'port',
            'sample': 'oracle FOURINDEX_ERI restatement (the reference loop: no permutational symmetry) over bra '
                      'shells I = 0 mod %d (%d of %d), extrapolated to a full build: %.1f s; one core, as the '
                      'reference runs a molecule on one busy rank' % (stride, sampled, n, t_full),
            'seconds_per_build': t_full}


def _ref_system():
    """The workload's System with the oracle's S_P (T/V are not needed by the Fock build)."""
    import oracle
    from polymer_b200 import geometry, system

    def onee_s(sysm):
        s_p, t_p, _ = oracle.onee_overlap(sysm)
        return s_p, t_p, t_p * 0.0
    return system.build_system(geometry.alkane_deck(N_ALKANE, inttol=INTTOL), onee_s)


_REF_SYS = None


def _ref_worker(args):
    """Oracle FOURINDEX_ERI restricted to bra shells I = offset (mod stride)."""
    global _REF_SYS
    import numpy as np
    import oracle
    stride, offset = args
    if _REF_SYS is None:
        _REF_SYS = _ref_system()
    n = _REF_SYS.basis.npgs
    pp = np.zeros((1, n, n))
    t0 = time.perf_counter()
    oracle.fourindex_eri_sample(_REF_SYS, pp, stride, offset)
    return time.perf_counter() - t0


def run_reference(args):
    """The reference's CPU algorithm (oracle port; Fortran is not buildable here) on all host cores."""
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return 0
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    sysm = _ref_system()
    n = sysm.basis.npshell
    per_worker = 2
    stride = max(1, n // per_worker)          # I = offset (mod stride): per_worker shells each
    ctx = mp.get_context('spawn')
    walls, fixed = [], []
    with ctx.Pool(cores) as pool:
        pool.map(_ref_worker, [(n + 1, n)] * cores)          # set-up of every worker
        fixed = pool.map(_ref_worker, [(n + 1, n)] * cores)  # the per-build KL/Schwarz part alone
        t_fixed = statistics.median(fixed)
        for it in range(args.warmup + args.steps):
            # every worker takes `per_worker` bra shells; the offsets rotate over the molecule
            offs = [(stride, (it * cores + c) % stride) for c in range(cores)]
            t0 = time.perf_counter()
            ts = pool.map(_ref_worker, offs)
            wall = time.perf_counter() - t0
            if it >= args.warmup:
                shells = sum(len(range(o, n, stride)) for _, o in offs)
                walls.append((wall, max(ts), shells))
    # a full build on `cores` processes: the fixed part once, the n bra shells spread over the cores
    per_shell = statistics.mean((max(w[1] - t_fixed, 1e-6)) * cores / w[2] for w in walls)
    t_full = t_fixed + per_shell * n / cores
    value = 1.0 / t_full
    line = {'metric': METRIC, 'value': value, 'unit': 'Fock builds/s', 'n_gpus': args.gpus, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': 1e3 * statistics.mean(w[0] for w in walls),
            'higher_is_better': True, 'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'impl': 'reference',
            'config': {'workload': workload_name(), 'parallelism': 'cpu x%d processes' % cores},
            'cpu_baseline': {'value': value, 'unit': 'Fock builds/s', 'cores': cores, 'kind': 'port',
                             'sample': 'per step %d bra shells of %d on %d processes (stride %d), extrapolated '
                                       'to one full build (%.1f s); the Fortran reference cannot be compiled here '
                                       '(no gfortran/mpif90). The oracle port splits the bra shells over the '
                                       'processes, which the reference cannot do for a molecule (one (Q1,Q2) '
                                       'ticket: one busy MPI rank), so this rate is an upper bound on the '
                                       "reference's" % (walls[0][2], n, cores, stride, t_full)},
            'e2e': {'value': value, 'unit': 'Fock builds/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line))
    return 0


def build_rate(sysm, device: int, p_p, p_ph=None, steps: int = 3, warmup: int = 1, **kw):
    """Fock builds/s of one system with device-resident densities (CUDA events,
    L2 flushed before each build), with its census rates; also returns the
    last build's (C_C, X_C) in the Fortran layout."""
    import torch
    from polymer_b200 import fock
    dev = torch.device('cuda', device)
    t0 = time.perf_counter()
    df = fock.DeviceFock(sysm, device, **kw)
    torch.cuda.synchronize(dev)
    t_setup = time.perf_counter() - t0
    pp = p_p.transpose(-1, -2).contiguous()
    ph = p_ph.transpose(-1, -2).contiguous() if p_ph is not None else None
    nc, n = sysm.ncell1, sysm.basis.ncgs
    out_c = torch.empty((nc, n, n), dtype=torch.float64, device=dev)
    out_x = torch.empty_like(out_c)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(warmup):
        df.run_fortran(pp, ph, out_c, out_x)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    stream = torch.cuda.current_stream(dev)
    for k in range(steps):
        flush.fill_(float(k))
        evs[k][0].record(stream)
        df.run_fortran(pp, ph, out_c, out_x)
        evs[k][1].record(stream)
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in evs) / steps
    cen = df.census()
    df.close()
    return ({'build_ms': ms, 'builds_per_s': 1000.0 / ms, 'setup_s': t_setup, 'npgs': sysm.basis.npgs,
             'ncgs': sysm.basis.ncgs, 'quartets_per_build': cen['quartets'],
             'quartets_per_s': cen['quartets'] / (ms * 1e-3), 'tflops': cen['flops'] / (ms * 1e-3) / 1e12,
             'quartets_fp32': cen['quartets_fp32'], 'launches_per_build': int(cen['kernel_launches'])},
            (out_c, out_x))


def extra_legs(device: int, peak: float):
    """The other Fock-build configurations at their own sizes: C40H82 6-31G**
    (1936 primitives, beyond the reference's 1024-primitive cap) and the helical
    polyethylene chain in 6-31G at CUTOFF1/CUTOFF2 = 5/10 (translation-indexed
    quartets, FP64).  Densities: one SCF iteration from the nuclear-charge guess
    (C40H82), the nuclear-charge guess rotated into P_P_HELIX (the chain)."""
    import torch
    from polymer_b200 import fock, geometry, scf, system
    dev = torch.device('cuda', device)
    out = {}
    s40 = system.build_system(geometry.alkane_deck(40, inttol=INTTOL), fock.onee)
    st = scf.HostState(s40, dev)
    p_p = scf.decontract(st, torch.tensor(scf.guess_density(s40), dtype=torch.float64, device=dev))
    r, _ = build_rate(s40, device, p_p)
    r['workload'] = workload_name(40)
    r['frac_fp64_peak'] = r['tflops'] / peak if peak else None
    out['c40h82'] = r
    sh = system.build_system(geometry.polyethylene_deck('6-31G', cutoff1=5, cutoff2=10, kpoints=16), fock.onee)
    st = scf.HostState(sh, dev)
    p_p = scf.decontract(st, torch.tensor(scf.guess_density(sh), dtype=torch.float64, device=dev))
    p_ph = scf.rotate(st, p_p)
    r, (c64, x64) = build_rate(sh, device, p_p, p_ph)
    r['workload'] = ('helical polyethylene 6-31G (C2H4 cell, period 2.55 A, 180 deg screw, seeded jitter 0.01 A), '
                     'CUTOFF1/CUTOFF2 = 5/10, INTTOL 1e-10, FP64')
    r['frac_fp64_peak'] = r['tflops'] / peak if peak else None
    # far cells (ket images outside the CUTOFF1 box) in FP32, near cells in FP64
    c64, x64 = c64.clone(), x64.clone()
    rm, (cm, xm) = build_rate(sh, device, p_p, p_ph, precision=1, mixed_cutoff=1e-6)
    dj, dk = cm - c64, xm - x64
    r['mixed_far_cells_fp32'] = {'build_ms': rm['build_ms'], 'builds_per_s': rm['builds_per_s'],
                                 'quartets_fp32_fraction': rm['quartets_fp32'] / max(rm['quartets_per_build'], 1.0),
                                 'max_abs_dF': float((dj - 0.5 * dk).abs().max()),
                                 'max_abs_dJ': float(dj.abs().max()), 'max_abs_dK': float(dk.abs().max()),
                                 'against': 'the FP64 build of the same density (pinned to the oracle at this '
                                            'configuration by the full-size parity tests)'}
    out['helix_pe_631g_5_10'] = r
    return out


class _EventTimedFock:
    """A DeviceFock whose calls (Fock builds) are bracketed by CUDA events on the
    current stream, so that the device time of a whole SCF's builds can be summed."""

    def __init__(self, df, dev):
        self._df, self._dev, self._ev = df, dev, []

    def __call__(self, *a, **kw):
        import torch
        s = torch.cuda.current_stream(self._dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        r = self._df(*a, **kw)
        e1.record(s)
        self._ev.append((e0, e1))
        return r

    def __getattr__(self, name):
        return getattr(self._df, name)

    def device_s(self) -> float:
        import torch
        torch.cuda.synchronize(self._dev)
        return sum(a.elapsed_time(b) for a, b in self._ev) * 1e-3


def batch_leg(n_clusters: int, device: int, steps: int, warmup: int, autotune: bool = False, scf_runs: bool = True):
    """Uneven water clusters (cc-pVDZ, k ~ U{1..16} as geometry.water_batch_decks
    draws them) as one batch: batched full FP64 Fock builds per second, and the
    time to converged SCF of the whole set -- one plain FP64 GPU SCF per molecule
    (the reference's loop, a DeviceFock each) against the batched SCF (set-up of
    its DeviceBatch included), every molecule compared by E[P] of its final
    idempotent density with full FP64 J/K."""
    import numpy as np
    import torch
    from polymer_b200 import batch_scf, fock, geometry, guess, scf, system
    dev = torch.device('cuda', device)
    decks = geometry.water_batch_decks(n_clusters)
    t0 = time.perf_counter()
    systems = [system.build_system(d, fock.onee) for d in decks]
    t_sys = time.perf_counter() - t0
    ssys = [systems[k] for k in batch_scf.sorted_order(systems)]
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    fb = fock.DeviceBatch(ssys, device)
    torch.cuda.synchronize(dev)
    t_setup = time.perf_counter() - t0
    cen = fb.census()
    pc = torch.zeros_like(fb.p_c)
    for k, s in enumerate(ssys):
        fb.view(pc, k).copy_(torch.tensor(scf.guess_density(s)[0], device=dev))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(warmup):
        fb.run_packed(pc, fb.out_c, fb.out_x)
    torch.cuda.synchronize(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.fill_(float(k))
        evs[k][0].record()
        fb.run_packed(pc, fb.out_c, fb.out_x)
        evs[k][1].record()
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in evs) / steps
    ms_tuned, sched = None, fb.schedule()
    if True:
        # the same builds after the batch autotuner picked each class's variant on them
        t_tune = time.perf_counter()
        fb.autotune(pc)
        t_tune = time.perf_counter() - t_tune
        for k in range(steps):
            flush.fill_(float(k))
            evs[k][0].record()
            fb.run_packed(pc, fb.out_c, fb.out_x)
            evs[k][1].record()
        torch.cuda.synchronize(dev)
        ms_tuned = sum(a.elapsed_time(b) for a, b in evs) / steps
        sched = fb.schedule()
    fb.close()

    out = {'workload': '%d water clusters, cc-pVDZ, k ~ U{1..16} (seed 2000, cluster i from seed 2001+i), '
                       'INTTOL 1e-10' % n_clusters,
           'molecules': n_clusters, 'ncgs_total': int(sum(s.basis.ncgs for s in systems)),
           'systems_s': t_sys, 'batch_setup_s': t_setup,
           'build_ms': ms, 'builds_per_s': 1000.0 / ms, 'quartets_per_build': cen['quartets'],
           'quartets_per_s': cen['quartets'] / (ms * 1e-3), 'tflops': cen['flops'] / (ms * 1e-3) / 1e12,
           'launches_per_build': int(cen['kernel_launches']),
           'build_ms_autotuned': ms_tuned, 'autotune_s': t_tune,
           'variants': {x['cls']: x['variant'] for x in sched},
           'schedule': 'build_ms: default table; build_ms_autotuned: after pfe_batch_autotune on the batch',
           'l2': 'flushed before every timed build (256 MiB write)'}
    if not scf_runs:
        return out
    # plain: the reference's loop with full FP64 builds, one molecule after another
    e_plain, it_plain = [], []
    t_plain_builds = 0.0
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for s in systems:
        df = _EventTimedFock(fock.DeviceFock(s, device), dev)
        r = scf.run_scf(s, df, device=dev, variational=True)
        e_plain.append(r.energy_variational)
        it_plain.append(len(r.iterations))
        t_plain_builds += df.device_s()
        df.close()
    torch.cuda.synchronize(dev)
    t_plain = time.perf_counter() - t0
    e_plain = np.array(e_plain)
    lg = guess.LearnedGuess.load(guess.MODEL, device=dev)
    runs = {}
    # one untimed run first (allocator pools, lazily loaded kernels), then each
    # configuration twice: the better time is reported, both are listed
    batch_scf.run_batch_scf(systems, batch_scf.BatchOptions(), device=device, graph=True)
    for name, opts in (('batched', batch_scf.BatchOptions()),
                       ('batched+learned', batch_scf.BatchOptions(guess=lg)),
                       ('batched+learned+mixed', batch_scf.BatchOptions(guess=lg, mixed_cutoff=1e-6))):
        times = []
        for _ in range(2):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            res = batch_scf.run_batch_scf(systems, opts, device=device, graph=True)   # builds (and frees) its batch
            torch.cuda.synchronize(dev)
            times.append(time.perf_counter() - t0)
        t = min(times)
        runs[name] = {'s': t, 's_each': times, 'speedup_vs_plain': t_plain / t, 'builds': res.builds,
                      'iterations_mean': float(res.iterations.mean()), 'iterations_max': int(res.iterations.max()),
                      'converged': bool(res.converged.all()),
                      'max_abs_dE_vs_plain': float(np.abs(res.energy - e_plain).max()),
                      'guess_fallbacks': int(res.fallback.sum()),
                      'options': {'density_tol': opts.density_tol, 'density_tol_rel': opts.density_tol_rel,
                                  'mixed_cutoff': opts.mixed_cutoff, 'reset_every': opts.reset_every,
                                  'guess': opts.guess if isinstance(opts.guess, str) else 'learned',
                                  'cuda_graph': 'each iteration from the third on is one graph replay'}}
    out['scf'] = {'plain_fp64_s': t_plain, 'plain_iterations_mean': float(np.mean(it_plain)),
                  'plain_fp64_build_s': t_plain_builds,
                  'plain_fp64_build_note': 'CUDA-event time of the plain loop\'s Fock builds alone (the rest of '
                                           'plain_fp64_s is its host loop, eigensolver and transfers)',
                  'batched_vs_plain_builds_only': {k: t_plain_builds / v['s'] for k, v in runs.items()},
                  **runs,
                  'wall_clock': 'host time around each whole set, GPU synchronised; one-electron set-up excluded; '
                                'batched: best of two runs after one untimed run'}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-scf', action='store_true', help='skip the time-to-converged SCF leg')
    ap.add_argument('--batch', type=int, default=256,
                    help='water clusters in the batched leg (0: skip it)')
    ap.add_argument('--no-batch-scf', action='store_true',
                    help='batched leg: the batched builds only, no SCF of the set')
    ap.add_argument('--no-extra', action='store_true',
                    help='skip the C40H82 and helical-chain build rates')
    ap.add_argument('--autotune', action='store_true',
                    help='time every kernel variant per quartet class and keep the fastest '
                         '(default: the library\'s measured schedule table)')
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    t_main = time.perf_counter()
    legs = {}
    if args.impl == 'reference':
        return run_reference(args)

    from polymer_b200 import build as _build
    _build.build()   # no-op when the in-tree library is up to date
    import numpy as np
    import torch
    import torch.distributed as dist
    from polymer_b200 import capi, fock, scf, system

    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))
    dev = torch.device('cuda', local)

    sysm, p_p, p_c = build_problem(local)
    df = fock.DeviceFock(sysm, local, myid=rank, numprocs=world)
    cen = df.census()
    nc, n = sysm.ncell1, sysm.basis.ncgs
    pp_f = p_p.transpose(-1, -2).contiguous()
    out_c = torch.empty((nc, n, n), dtype=torch.float64, device=dev)
    out_x = torch.empty_like(out_c)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    if args.autotune:
        df.autotune(p_p)   # per-class schedule chosen by timing every variant (untimed set-up)
    cen = df.census()

    def step():
        df.run_fortran(pp_f, None, out_c, out_x)
        if world > 1:
            dist.all_reduce(out_c)
            dist.all_reduce(out_x)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            step()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in evs)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step = float(t.item()) / args.steps
    value = 1000.0 / ms_step

    # ---- roofline of the dominant kernel (one profiled build, untimed above)
    L = capi.lib()
    capi.check(L, L.pfe_context_profile(df.ctx, 1))
    step()
    torch.cuda.synchronize()
    stats = (capi.PfeKernelStat * 64)()
    nst = L.pfe_context_kernel_stats(df.ctx, stats, 64)
    capi.check(L, L.pfe_context_profile(df.ctx, 0))
    kern = [{'cls': '%04d' % s.cls, 'variant': s.variant, 'grid_mult': s.grid_mult, 'ms': s.ms,
             'tuned_ms': list(s.tuned_ms), 'quartets': s.quartets, 'flops': s.flops} for s in stats[:max(nst, 0)]]
    tot_ms = sum(k['ms'] for k in kern) or 1.0
    dom = max(kern, key=lambda k: k['ms']) if kern else None
    peak = measure_fp64_peak(local)
    roof = None
    if dom:
        ach = dom['flops'] / (dom['ms'] * 1e-3) / 1e12
        traffic = ncu_traffic_per_launch()
        kname = ['k_gq', 'k_gq_warp', 'k_gq_block', 'k_gq_wide'][dom['variant']]
        roof = {'bound': 'fp64', 'kernel': '%s<%s>' % (kname, dom['cls']), 'achieved': ach, 'peak': peak,
                'unit': 'TFLOP/s', 'frac': ach / peak if peak else None,
                'peak_source': 'measured in this run: DFMA loop over all SMs (pfe_measure_fp64_peak); '
                               'MEASURED_PEAKS.json has no FP64 figure',
                'share_of_build': dom['ms'] / tot_ms,
                'traffic': traffic.get(dom['cls']) if isinstance(traffic, dict) else None}
        all_flops = sum(k['flops'] for k in kern)
        roof['build_achieved'] = all_flops / (tot_ms * 1e-3) / 1e12

    # ---- the mixed FP32/FP64 recursion (Schwarz x density cutoff 1e-6) on the same
    # density, against the FP64 build (itself checked against the oracle on this
    # workload by tests/test_baseline_configs_gpu.py): max|dF| (F = J - K/2) and
    # dE = tr(P dJ)/2 - tr(P dK)/4 of this density
    mixed = None
    if world == 1:
        dfm = fock.DeviceFock(sysm, local, precision=capi.PFE_PREC_MIXED, mixed_cutoff=1e-6)
        c64, x64 = df(p_p)
        cmx, xmx = dfm(p_p)
        for _ in range(args.warmup):
            dfm(p_p)
        evm = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.fill_(float(k))
            evm[k][0].record(stream)
            dfm.run_fortran(pp_f, None, out_c, out_x)
            evm[k][1].record(stream)
        torch.cuda.synchronize()
        cmm = dfm.census()
        dj, dk = cmx - c64, xmx - x64
        mixed = {'mixed_cutoff': 1e-6, 'build_ms': sum(a.elapsed_time(b) for a, b in evm) / args.steps,
                 'quartets_fp32_fraction': cmm['quartets_fp32'] / max(cmm['quartets'], 1.0),
                 'max_abs_dF': float((dj - 0.5 * dk).abs().max()),
                 'max_abs_dJ': float(dj.abs().max()), 'max_abs_dK': float(dk.abs().max()),
                 'dE': float(0.5 * (p_c[0] * dj[0]).sum() - 0.25 * (p_c[0] * dk[0]).sum()),
                 'against': 'the FP64 build of the same density (pinned to the oracle at this workload by the '
                            'full-size parity tests)'}
        dfm.close()

    # ---- end to end through the host C ABI (pinned host buffers)
    e2e = None
    if world == 1:
        pin_p = torch.empty(pp_f.numel(), dtype=torch.float64).pin_memory()
        pin_p.copy_(pp_f.reshape(-1).cpu())
        pin_c = torch.empty(nc * n * n, dtype=torch.float64).pin_memory()
        pin_x = torch.empty_like(pin_c).pin_memory()
        a, keep = sysm.pfe_args(None, None)
        import ctypes
        a.p_p = ctypes.cast(pin_p.data_ptr(), ctypes.POINTER(ctypes.c_double))
        cp = ctypes.cast(pin_c.data_ptr(), ctypes.POINTER(ctypes.c_double))
        xp = ctypes.cast(pin_x.data_ptr(), ctypes.POINTER(ctypes.c_double))
        for _ in range(args.warmup):
            capi.check(L, L.pfe_fourindex_eri(ctypes.byref(a), cp, xp))
        walls = []
        for k in range(args.steps):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            capi.check(L, L.pfe_fourindex_eri(ctypes.byref(a), cp, xp))
            walls.append(time.perf_counter() - t0)
        e2e = {'value': args.steps / sum(walls), 'unit': 'Fock builds/s',
               'h2d_bytes_per_step': int(pin_p.numel() * 8), 'd2h_bytes_per_step': int(2 * pin_c.numel() * 8),
               'ms_per_step': 1e3 * sum(walls) / args.steps,
               'path': 'pfe_fourindex_eri (host pointers; static inputs cached on the device by content hash)'}

    # ---- time to a converged SCF (1e-8 RMS density): the reference's loop with full FP64
    # builds against the time-to-solution path (commutator DIIS, incremental density-screened
    # builds), both compared by E[P] of the final idempotent density with full FP64 J/K
    legs['build_leg_s'] = time.perf_counter() - t_main
    t_leg = time.perf_counter()
    scf_line = None
    if rank == 0 and world == 1 and not args.no_scf:
        from polymer_b200 import scf
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r_plain = scf.run_scf(sysm, df, device=dev, variational=True)
        torch.cuda.synchronize()
        t_plain = time.perf_counter() - t0
        opts = scf.FastOptions()
        t0 = time.perf_counter()
        r_fast = scf.run_scf_fast(sysm, df, opts=opts, device=dev)
        torch.cuda.synchronize()
        t_fast = time.perf_counter() - t0
        scf_line = {'converged_to': 'RMS density change < %g' % sysm.deck.scfconv,
                    'plain_fp64_s': t_plain, 'plain_iterations': len(r_plain.iterations),
                    'fast_s': t_fast, 'fast_iterations': len(r_fast.iterations),
                    'speedup': t_plain / t_fast,
                    'energy_plain': r_plain.energy_variational, 'energy_fast': r_fast.energy,
                    'abs_dE': abs(r_fast.energy - r_plain.energy_variational),
                    'fast_path': 'commutator DIIS; incremental builds from dP_C with density screening %g, '
                                 'full rebuild every %d; final full FP64 iteration' % (opts.density_tol,
                                                                                      opts.reset_every),
                    'plain_path': "reference loop (nuclear-charge guess, density DIIS), full FP64 builds",
                    'wall_clock': 'host time around each SCF, GPU synchronised'}

    legs['scf_leg_s'] = time.perf_counter() - t_leg
    t_leg = time.perf_counter()
    extra = None
    if rank == 0 and world == 1 and not args.no_extra:
        extra = extra_legs(local, peak)
    legs['extra_leg_s'] = time.perf_counter() - t_leg
    t_leg = time.perf_counter()
    batch = None
    if rank == 0 and world == 1 and args.batch > 0:
        batch = batch_leg(args.batch, local, args.steps, args.warmup, args.autotune, not args.no_batch_scf)
    legs['batch_leg_s'] = time.perf_counter() - t_leg
    t_leg = time.perf_counter()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(sysm, p_p.cpu().numpy())
    legs['cpu_baseline_s'] = time.perf_counter() - t_leg
    legs['total_s'] = time.perf_counter() - t_main

    if rank == 0:
        line = {'metric': METRIC, 'value': value, 'unit': 'Fock builds/s', 'n_gpus': world, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': ms_step, 'higher_is_better': True, 'scaling': 'strong',
                'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
                'config': {'workload': workload_name(), 'npgs': sysm.basis.npgs, 'ncgs': sysm.basis.ncgs,
                           'npshell': sysm.basis.npshell, 'precision': 'fp64',
                           'schedule': 'autotuned' if args.autotune else 'default table',
                           'l2': 'flushed before every timed step (256 MiB write)',
                           'parallelism': 'quartet chunks split over %d GPU(s), NCCL all-reduce of J/K' % world
                           if world > 1 else 'single GPU'},
                'quartets_per_build': cen['quartets'], 'quartets_per_s': cen['quartets'] * value,
                'gpu_launches': args.steps * int(cen['kernel_launches']),
                'roofline': roof, 'mixed': mixed, 'kernels': kern, 'clocks': clk.summary(), 'e2e': e2e, 'scf': scf_line,
                'other_configs': extra, 'batch': batch, 'cpu_baseline': cpu, 'wall_clock_s': legs}
        print(json.dumps(line))
    df.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == '__main__':
    sys.exit(main())
