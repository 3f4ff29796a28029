"""Lattice and helical Fock builds on the GPU against the CPU oracle.

Covers the general path of FOURINDEX_ERI (src/pfourindexdirect.f90:224-803):
(Q1,Q2) tickets, Q3 images, the LCEL1 exchange window, the helical density
P_P_HELIX and the C2H back-transform, for a helical chain (180 degree screw),
a translational chain and a 3-D periodic box.  Tolerance as the molecular
parity tests: 1e-11 relative to max|C_C| (plus 1e-13).
"""
import numpy as np
import pytest
import torch

import oracle
from polymer_b200 import fock, geometry, inputdeck, scf, system

pytestmark = pytest.mark.gpu

RTOL = 1e-11


def _density(sysm, seed=1):
    rng = np.random.default_rng(seed)
    n = sysm.basis.ncgs
    pc = rng.normal(size=(sysm.ncell1, n, n)) * 0.1
    for c, q in enumerate(sysm.cells):          # P(-q) = P(q)^T, P(0) symmetric
        cm = sysm.cell_index(-q[0], -q[1], -q[2])
        if cm == c:
            pc[c] = 0.5 * (pc[c] + pc[c].T)
        elif cm < c:
            pc[c] = pc[cm].T
    pp = np.einsum('ai,cab,bj->cij', sysm.basis.cc, pc, sysm.basis.cc, optimize=True)
    st = scf.HostState(sysm)
    ph = scf.rotate(st, torch.tensor(pp))
    return pp, (ph.numpy() if ph is not None else None)


def _cases():
    pe = geometry.polyethylene_deck('STO-3G', cutoff1=1, cutoff2=2, kpoints=4)
    pe631 = geometry.polyethylene_deck('6-31G', cutoff1=1, cutoff2=1, kpoints=4)
    chain = inputdeck.make_deck([1, 1], [[0, 0, 0], [1.4, 0, 0]], '6-31Gss', period=(4.0, 0, 0), kpoints=(4, 0, 0),
                                cutoff1=2, cutoff2=3, inttol=1e-10)
    box = inputdeck.make_deck([1, 1], [[0, 0, 0], [0, 0, 1.4]], 'STO-3G', period=(5.0, 5.5, 6.0), kpoints=(2, 2, 2),
                              cutoff1=1, cutoff2=1, inttol=1e-10)
    return {'helix_sto3g': pe, 'helix_631g': pe631, 'chain_631gss': chain, 'box_sto3g': box}


CASES = _cases()


def _close(got, ref, what):
    scale = np.abs(ref).max()
    err = np.abs(got - ref).max()
    assert err <= RTOL * scale + 1e-13, '%s: max|diff| %.3e (scale %.3e)' % (what, err, scale)


@pytest.mark.parametrize('name', sorted(CASES))
def test_lattice_matches_oracle(name):
    s = system.build_system(CASES[name], oracle.onee)
    pp, ph = _density(s)
    c_ref, x_ref = oracle.fourindex_eri(s, pp, ph)
    c_gpu, x_gpu = fock.fourindex_eri(s, pp, ph)
    _close(c_gpu, c_ref, 'C_C')
    _close(x_gpu, x_ref, 'X_C')


@pytest.mark.parametrize('name', ['helix_sto3g', 'box_sto3g'])
def test_rank_shares_sum_to_the_full_build(name):
    """The TICKET split: C_C/X_C summed over ranks (the caller's MPI_ALLREDUCE) equal one rank's full build."""
    s = system.build_system(CASES[name], oracle.onee)
    pp, ph = _density(s, seed=2)
    c_full, x_full = fock.fourindex_eri(s, pp, ph)
    c_sum = np.zeros_like(c_full)
    x_sum = np.zeros_like(x_full)
    for r in range(3):
        c, x = fock.fourindex_eri(s, pp, ph, myid=r, numprocs=3)
        c_sum += c
        x_sum += x
    _close(c_sum, c_full, 'sum C_C')
    _close(x_sum, x_full, 'sum X_C')


def test_molecular_rank_shares_sum_to_the_full_build():
    s = system.build_system(geometry.alkane_deck(2), oracle.onee)
    rng = np.random.default_rng(4)
    n = s.basis.ncgs
    a = rng.normal(size=(n, n))
    pp = np.einsum('ai,cab,bj->cij', s.basis.cc, (a + a.T)[None], s.basis.cc, optimize=True)
    c_full, x_full = fock.fourindex_eri(s, pp)
    parts = [fock.fourindex_eri(s, pp, myid=r, numprocs=2) for r in range(2)]
    _close(parts[0][0] + parts[1][0], c_full, 'sum C_C')
    _close(parts[0][1] + parts[1][1], x_full, 'sum X_C')


def test_rotate_on_the_gpu_matches_oracle():
    """ROTATE_DENSITYMATRIX (P_P_HELIX) as the SCF runs it on the device, against
    the oracle's restatement (src/pdensitymatrix.f90:516-563)."""
    s = system.build_system(geometry.polyethylene_deck('6-31G', cutoff1=5, cutoff2=10, kpoints=16), oracle.onee)
    rng = np.random.default_rng(9)
    n = s.basis.ncgs
    pp = np.einsum('ai,cab,bj->cij', s.basis.cc, rng.normal(size=(s.ncell1, n, n)) * 0.1, s.basis.cc, optimize=True)
    ref = oracle.rotate_density(s, pp)
    got = scf.rotate(scf.HostState(s, 'cuda'), torch.tensor(pp, device='cuda')).cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize('variant', [0, 1])
@pytest.mark.parametrize('name', ['helix_631g', 'chain_631gss', 'box_sto3g'])
def test_straight_line_and_interpreter_match_oracle(name, variant):
    """Both lattice executions against the oracle: the straight-line kernels
    (one ket per lane, classes up to 64 integrals; variant 0) and the op-table
    interpreter for every class (variant 1), FP64 and with the far cells in FP32."""
    s = system.build_system(CASES[name], oracle.onee)
    pp, ph = _density(s, seed=5)
    c_ref, x_ref = oracle.fourindex_eri(s, pp, ph)
    df = fock.DeviceFock(s)
    df.force_variant(variant)
    dev = torch.device('cuda')
    c_d, x_d = df(torch.tensor(pp, device=dev), torch.tensor(ph, device=dev) if ph is not None else None)
    torch.cuda.synchronize()
    _close(c_d.cpu().numpy(), c_ref, 'C_C variant %d' % variant)
    _close(x_d.cpu().numpy(), x_ref, 'X_C variant %d' % variant)
    df.close()
    dm = fock.DeviceFock(s, precision=1, mixed_cutoff=1e-6)
    dm.force_variant(variant)
    c_m, x_m = dm(torch.tensor(pp, device=dev), torch.tensor(ph, device=dev) if ph is not None else None)
    torch.cuda.synchronize()
    scale = np.abs(c_ref).max()
    assert np.abs(c_m.cpu().numpy() - c_ref).max() <= 1e-6 * scale
    assert np.abs(x_m.cpu().numpy() - x_ref).max() <= 1e-6 * scale
    dm.close()
