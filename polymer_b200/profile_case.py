"""Run a few Fock builds of one workload, for a profiler to capture.

    python -m polymer_b200.profile_case c20h42 [--builds 2] [--mixed]
    python -m polymer_b200.profile_case helix  [--builds 2] [--mixed]
    python -m polymer_b200.profile_case water  [--builds 2] [--clusters 32]

One untimed warm-up build, then `--builds` builds, each after a 256 MiB
write that flushes L2 (the same shape as the bench's timed region).  The
workloads:

* c20h42: C20H42 6-31G** (1130 primitives) at INTTOL 1e-10, density from
  one SCF iteration from the nuclear-charge guess;
* helix: helical polyethylene 6-31G at CUTOFF1/CUTOFF2 = 5/10, the
  nuclear-charge guess rotated into P_P_HELIX;
* water: a batch of uneven water clusters in cc-pVDZ (k ~ U{1..16}), the
  batched build from the nuclear-charge guess.

`--mixed` builds with precision MIXED at cutoff 1e-6 (FP32 below the
Schwarz-times-density bound; on the helix, the far cells).  Prints one JSON
line with the mean build time (CUDA events on the launch stream).
"""
import argparse
import json

import torch

from . import fock, geometry, scf, system


def _flush_buf(dev):
    return torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)


def _timed(run, dev, builds):
    flush = _flush_buf(dev)
    run()
    stream = torch.cuda.current_stream(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(builds)]
    for k in range(builds):
        flush.fill_(float(k))
        evs[k][0].record(stream)
        run()
        evs[k][1].record(stream)
    torch.cuda.synchronize(dev)
    return sum(a.elapsed_time(b) for a, b in evs) / max(builds, 1)


def molecule_or_chain(case: str, device: int, builds: int, mixed: bool) -> dict:
    dev = torch.device('cuda', device)
    if case == 'c20h42':
        sysm = system.build_system(geometry.alkane_deck(20, inttol=1e-10), fock.onee)
    else:
        sysm = system.build_system(geometry.polyethylene_deck('6-31G', cutoff1=5, cutoff2=10, kpoints=16),
                                   fock.onee)
    st = scf.HostState(sysm, dev)
    p_c = torch.tensor(scf.guess_density(sysm), dtype=torch.float64, device=dev)
    p_p = scf.decontract(st, p_c)
    p_ph = scf.rotate(st, p_p) if case == 'helix' else None
    kw = {'precision': 1, 'mixed_cutoff': 1e-6} if mixed else {}
    df = fock.DeviceFock(sysm, device, **kw)
    if case == 'c20h42':
        c_c, x_c = df(p_p)
        p_out, _, _, _ = scf.fock_build(st, st.t_c + st.n_c + c_c - 0.5 * x_c)
        p_p = scf.decontract(st, p_out)
    pp = p_p.transpose(-1, -2).contiguous()
    ph = p_ph.transpose(-1, -2).contiguous() if p_ph is not None else None
    nc, n = sysm.ncell1, sysm.basis.ncgs
    out_c = torch.empty((nc, n, n), dtype=torch.float64, device=dev)
    out_x = torch.empty_like(out_c)
    ms = _timed(lambda: df.run_fortran(pp, ph, out_c, out_x), dev, builds)
    cen = df.census()
    df.close()
    return {'case': case, 'mixed': mixed, 'build_ms': ms, 'npgs': sysm.basis.npgs,
            'quartets': cen['quartets'], 'launches_per_build': int(cen['kernel_launches'])}


def water_batch(device: int, builds: int, clusters: int, mixed: bool) -> dict:
    from . import batch_scf
    dev = torch.device('cuda', device)
    systems = [system.build_system(d, fock.onee) for d in geometry.water_batch_decks(clusters)]
    ssys = [systems[k] for k in batch_scf.sorted_order(systems)]
    fb = fock.DeviceBatch(ssys, device)
    if mixed:
        fb.set_screening(mixed_cutoff=1e-6)
    pc = torch.zeros_like(fb.p_c)
    for k, s in enumerate(ssys):
        fb.view(pc, k).copy_(torch.tensor(scf.guess_density(s)[0], device=dev))
    ms = _timed(lambda: fb.run_packed(pc, fb.out_c, fb.out_x), dev, builds)
    cen = fb.census()
    fb.close()
    return {'case': 'water', 'clusters': clusters, 'mixed': mixed, 'build_ms': ms, 'quartets': cen['quartets'],
            'launches_per_build': int(cen['kernel_launches'])}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument('case', choices=['c20h42', 'helix', 'water'])
    ap.add_argument('--builds', type=int, default=2)
    ap.add_argument('--clusters', type=int, default=32)
    ap.add_argument('--mixed', action='store_true')
    ap.add_argument('--device', type=int, default=0)
    a = ap.parse_args(argv)
    from . import build
    build.build()
    torch.cuda.set_device(a.device)
    if a.case == 'water':
        r = water_batch(a.device, a.builds, a.clusters, a.mixed)
    else:
        r = molecule_or_chain(a.case, a.device, a.builds, a.mixed)
    print(json.dumps(r))


if __name__ == '__main__':
    main()
