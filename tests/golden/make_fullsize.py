"""Generate tests/golden/fullsize_*.npz: the oracle's J and K of the two
largest parity cases, stored as projections so the fixtures stay small.

For C20H42 6-31G** (INTTOL 1e-10, the Fock-build benchmark) and a 16-water
cc-pVDZ cluster (1072 primitives), with the seeded densities that
tests/test_baseline_configs_gpu.py builds, the oracle's (C_C, X_C) are computed
in full on this machine's cores (tests/oracle_pool.py) and stored as
C_C @ R and X_C @ R for a seeded random R (n x 4), with max|C_C|, max|X_C|,
the traces tr(P C_C), tr(P X_C) and sum|C_C|, sum|X_C|.  A GPU build agreeing
element-wise to e with the oracle agrees in every projection to at most
e * ||R[:, k]||_1, which is what the test checks; a wrong element shows up in
all four projections.

Usage (from the repository root): python tests/golden/make_fullsize.py [name ...]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))


def cases():
    import oracle
    from polymer_b200 import geometry, system

    def onee_s(sysm):
        s_p, t_p, _ = oracle.onee_overlap(sysm)
        return s_p, t_p, np.zeros_like(t_p)
    return {
        'c20h42': lambda: (system.build_system(geometry.alkane_deck(20, inttol=1e-10), onee_s), 120),
        'water16': lambda: (system.build_system(geometry.water_deck(16, seed=2001), onee_s), 16),
    }


def density(sysm, seed):
    """The seeded random decontracted density of the parity tests (contracted
    P_C = (A + A^T)*0.3-scaled normal, P_P = CC^T P_C CC)."""
    rng = np.random.default_rng(seed)
    n = sysm.basis.ncgs
    a = rng.normal(size=(n, n)) * 0.3
    pc = a + a.T
    return pc, np.einsum('ai,cab,bj->cij', sysm.basis.cc, pc[None], sysm.basis.cc, optimize=True)


def projector(n):
    return np.random.default_rng(7).normal(size=(n, 4))


def main(names):
    import oracle_pool
    for name, make in cases().items():
        if names and name not in names:
            continue
        sysm, seed = make()
        pc, pp = density(sysm, seed)
        c, x = oracle_pool.fourindex_eri(sysm, pp)
        c, x = c[0], x[0]
        r = projector(sysm.basis.ncgs)
        out = os.path.join(HERE, 'fullsize_%s.npz' % name)
        np.savez_compressed(out, cr=c @ r, xr=x @ r, cmax=np.abs(c).max(), xmax=np.abs(x).max(),
                            ctr=np.sum(pc * c), xtr=np.sum(pc * x), cabs=np.abs(c).sum(), xabs=np.abs(x).sum(),
                            npgs=sysm.basis.npgs, ncgs=sysm.basis.ncgs, seed=seed)
        print('wrote', out)


if __name__ == '__main__':
    main(sys.argv[1:])
