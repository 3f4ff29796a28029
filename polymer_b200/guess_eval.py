"""The learned-guess experiment on large water clusters: training data,
training, and the held-out comparison against the reference's guess.

Clusters (H2O)_k in cc-pVDZ with k ~ U{8..32}, generated as the batched
workload's clusters are (polymer_b200.geometry.water_deck): training cluster i
from seed 4000+i, held-out cluster i from seed 9000+i (the cluster size drawn
from default_rng([seed, 1])).  Training data are the converged densities of the
batched GPU SCF itself (nuclear-charge guess, each iteration a CUDA graph
replay), the network and its training are those of polymer_b200.guess.

The held-out evaluation runs the batched SCF of the same clusters twice, from
the reference's nuclear-charge guess and from the learned guess (its host-side
features, network evaluation, assembly and purification inside the timed
region), and reports per guess: SCF iterations (mean, max), wall time of the
whole set (GPU synchronised, best of `repeats` runs after one untimed run),
the fallback rate of the learned guess (first commutator error above
BatchOptions.fallback_error: restarted from the nuclear guess) and the largest
energy difference between the two runs' converged energies.

Run: python -m polymer_b200.guess_eval [n_train] [n_heldout] [out.pt] [out.json]
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np
import torch

KMIN, KMAX = 8, 32
# the network trained by train(600, ...) on this configuration
MODEL = os.path.join(os.path.dirname(__file__), 'data', 'guess_water_k8_32.pt')


def cluster_sizes(seeds, kmin: int = KMIN, kmax: int = KMAX):
    return [int(np.random.default_rng([s, 1]).integers(kmin, kmax + 1)) for s in seeds]


def train_seeds(n: int):
    return [4000 + i for i in range(n)]


def heldout_seeds(n: int):
    return [9000 + i for i in range(n)]


def train(n: int, path: str, batch: int = 64, steps: int = 8000, log=print):
    """Converge n training clusters with the batched SCF and train the network on them."""
    from . import guess
    seeds = train_seeds(n)
    t0 = time.perf_counter()
    x, t, w = guess.generate_batched(cluster_sizes(seeds), seeds, batch=batch, log=log)
    t_data = time.perf_counter() - t0
    lg = guess.LearnedGuess()
    t0 = time.perf_counter()
    lg.train(x, t, w, steps=steps, batch=2048, lr=2e-3, log=log)
    t_train = time.perf_counter() - t0
    lg.save(path)
    return lg, {'clusters': n, 'blocks': int(len(x)), 'data_s': t_data, 'train_s': t_train, 'steps': steps}


def evaluate(lg, n: int, batch: int = 64, repeats: int = 1, device: int = 0, log=print):
    """Held-out comparison of the nuclear-charge and the learned guess (see the module notes)."""
    from . import batch_scf, fock, system, guess
    seeds = heldout_seeds(n)
    sizes = cluster_sizes(seeds)
    dev = torch.device('cuda', device)
    out = {'clusters': n, 'k_mean': float(np.mean(sizes)), 'k_min': int(min(sizes)), 'k_max': int(max(sizes))}
    res = {'nuclear': {'s': 0.0, 'it': [], 'e': []}, 'learned': {'s': 0.0, 'it': [], 'e': [], 'fallback': 0}}
    for b0 in range(0, n, batch):
        systems = [system.build_system(guess.sample_cluster(k, s), fock.onee)
                   for k, s in zip(sizes[b0:b0 + batch], seeds[b0:b0 + batch])]
        for name, opts in (('nuclear', batch_scf.BatchOptions()), ('learned', batch_scf.BatchOptions(guess=lg))):
            if b0 == 0:   # one untimed run: allocator pools, lazily loaded kernels
                batch_scf.run_batch_scf(systems, opts, device=device, graph=True)
            best, r = None, None
            for _ in range(repeats):
                torch.cuda.synchronize(dev)
                t0 = time.perf_counter()
                r = batch_scf.run_batch_scf(systems, opts, device=device, graph=True)
                torch.cuda.synchronize(dev)
                dt = time.perf_counter() - t0
                best = dt if best is None else min(best, dt)
            res[name]['s'] += best
            res[name]['it'].extend(int(v) for v in r.iterations)
            res[name]['e'].extend(float(v) for v in r.energy)
            if name == 'learned':
                res[name]['fallback'] += int(r.fallback.sum())
        if log:
            log('held-out %d..%d: nuclear %.1f s, learned %.1f s so far' % (
                b0, b0 + len(systems) - 1, res['nuclear']['s'], res['learned']['s']))
    for name in ('nuclear', 'learned'):
        it = np.array(res[name]['it'])
        out[name] = {'wall_s': res[name]['s'], 'iterations_mean': float(it.mean()), 'iterations_max': int(it.max())}
    out['learned']['fallback_rate'] = res['learned']['fallback'] / float(n)
    out['speedup'] = res['nuclear']['s'] / res['learned']['s']
    out['max_abs_dE'] = float(np.abs(np.array(res['learned']['e']) - np.array(res['nuclear']['e'])).max())
    out['wall_clock'] = 'batched SCF of the whole held-out set per guess, GPU synchronised, batches of %d' % batch
    return out


def main(argv):
    n_train = int(argv[1]) if len(argv) > 1 else 1000
    n_held = int(argv[2]) if len(argv) > 2 else 500
    path = argv[3] if len(argv) > 3 else 'guess_water_k8_32.pt'
    out = argv[4] if len(argv) > 4 else None
    lg, info = train(n_train, path)
    ev = evaluate(lg, n_held)
    line = {'training': info, 'heldout': ev}
    print(json.dumps(line))
    if out:
        with open(out, 'w') as fh:
            json.dump(line, fh, indent=1)


if __name__ == '__main__':
    main(sys.argv)
