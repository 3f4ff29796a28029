"""Parity of the CUDA Fock build with the CPU oracle (FP64 path).

The oracle restates FOURINDEX_ERI in the reference's loop order (no
permutational symmetry, same screening, same Boys evaluation); the CUDA path
uses 8-fold symmetry, a different recursion (HGP) and atomics, so agreement is
to rounding: |dC_C|, |dX_C| <= 1e-11 * max|C_C| + 1e-13 (Hartree).
"""
import numpy as np
import pytest
import torch

import oracle
from conftest import deck_of
from polymer_b200 import capi, fock, geometry, scf, system

pytestmark = pytest.mark.gpu

RTOL = 1e-11


def _random_density(sysm, seed=7):
    rng = np.random.default_rng(seed)
    n = sysm.basis.ncgs
    pc = np.zeros((sysm.ncell1, n, n))
    for c in range(sysm.ncell1):
        a = rng.normal(size=(n, n)) * 0.3
        pc[c] = a + a.T
    if sysm.ncell1 > 1:  # a lattice density obeys P(-q) = P(q)^T
        for c, q in enumerate(sysm.cells):
            cm = sysm.cell_index(-q[0], -q[1], -q[2])
            if cm < c:
                pc[c] = pc[cm].T
    cc = sysm.basis.cc
    return pc, np.einsum('ai,cab,bj->cij', cc, pc, cc, optimize=True)


def _assert_close(got, ref, what):
    scale = np.abs(ref).max()
    err = np.abs(got - ref).max()
    assert err <= RTOL * scale + 1e-13, '%s: max|diff| %.3e vs scale %.3e' % (what, err, scale)


def _sys(deck):
    return system.build_system(deck, oracle.onee)


@pytest.fixture(scope='module')
def water(reference_runs):
    return _sys(deck_of(reference_runs['H2O_CCSD_ccpVDZ']))


@pytest.mark.parametrize('name', ['BH_MBGF', 'FH_finiteT_MBPT_zeroT_HF_ref', 'H2O_CCSD_ccpVDZ'])
def test_host_abi_matches_oracle(reference_runs, name):
    s = _sys(deck_of(reference_runs[name]))
    _, pp = _random_density(s)
    c_ref, x_ref = oracle.fourindex_eri(s, pp)
    c_gpu, x_gpu = fock.fourindex_eri(s, pp)
    _assert_close(c_gpu, c_ref, 'C_C')
    _assert_close(x_gpu, x_ref, 'X_C')


@pytest.mark.parametrize('n,inttol', [(3, 1e-10), (2, 1e-12)])
def test_alkane_screened_matches_oracle(n, inttol):
    """6-31G** (s, sp, d cumulative shells, all 21 quartet classes) with screening."""
    s = _sys(geometry.alkane_deck(n, inttol=inttol))
    _, pp = _random_density(s, seed=n)
    c_ref, x_ref = oracle.fourindex_eri(s, pp)
    c_gpu, x_gpu = fock.fourindex_eri(s, pp)
    _assert_close(c_gpu, c_ref, 'C_C')
    _assert_close(x_gpu, x_ref, 'X_C')


@pytest.mark.parametrize('variant', [0, 1, 2, 3])
@pytest.mark.parametrize('mol', ['alkane', 'water'])
def test_every_execution_variant_matches_oracle(variant, mol, reference_runs):
    """Straight-line, warp-per-quartet and block-per-quartet schedules all agree:
    6-31G** alkane (cumulative sp and d shells: the full op tables) and cc-pVDZ
    water (pure p and d shells: the pure-bra and bra-and-ket tables)."""
    if mol == 'alkane':
        s = _sys(geometry.alkane_deck(2, inttol=1e-12))
    else:
        s = _sys(deck_of(reference_runs['H2O_CCSD_ccpVDZ']))
    _, pp = _random_density(s, seed=5)
    c_ref, x_ref = oracle.fourindex_eri(s, pp)
    df = fock.DeviceFock(s)
    df.force_variant(variant)
    c_d, x_d = df(torch.tensor(pp, device='cuda'))
    torch.cuda.synchronize()
    _assert_close(c_d.cpu().numpy(), c_ref, 'C_C variant %d' % variant)
    _assert_close(x_d.cpu().numpy(), x_ref, 'X_C variant %d' % variant)


def test_device_path_matches_host_path(water):
    pc, pp = _random_density(water, seed=3)
    c_h, x_h = fock.fourindex_eri(water, pp)
    df = fock.DeviceFock(water)
    c_d, x_d = df(torch.tensor(pp, device='cuda'))
    torch.cuda.synchronize()
    _assert_close(c_d.cpu().numpy(), c_h, 'C_C device')
    _assert_close(x_d.cpu().numpy(), x_h, 'X_C device')
    cen = df.census()
    assert cen['quartets'] > 0 and cen['flops'] > 0


def test_onee_matches_oracle(water):
    s_o, t_o, n_o = oracle.onee(water)
    s_g, t_g, n_g = fock.onee(water)
    for g, o, w in ((s_g, s_o, 'S'), (t_g, t_o, 'T'), (n_g, n_o, 'V')):
        assert np.abs(g - o).max() <= 1e-12 * np.abs(o).max() + 1e-14, w


def test_scf_with_cuda_fock_reproduces_reference_energy(reference_runs):
    run = reference_runs['H2O_CCSD_ccpVDZ']
    s = system.build_system(deck_of(run), fock.onee)
    res = scf.run_scf(s, fock.DeviceFock(s), device='cuda')
    assert abs(res.energy - run['expected']['total']) < 2e-10
    assert len(res.iterations) == len(run['expected']['iterations'])


def test_nan_density_is_rejected(water):
    _, pp = _random_density(water)
    pp[0, 3, 4] = np.nan
    with pytest.raises(capi.FockError) as e:
        fock.fourindex_eri(water, pp)
    assert e.value.code == -7


def test_malformed_shell_map_is_rejected(water):
    _, pp = _random_density(water)
    a, keep = water.pfe_args(pp)
    bad = keep['p_shell'].copy(order='F')
    # drop a p component of the first p shell: the shell is no longer cumulative
    s = int(np.nonzero(water.basis.p_shell_ang == 1)[0][0])
    bad[s, 1, 0, 0] = -1
    keep['p_shell'] = bad
    a.p_shell = capi.iptr(bad)
    L = capi.lib()
    c = np.zeros(water.basis.ncgs ** 2)
    x = np.zeros_like(c)
    import ctypes
    rc = L.pfe_fourindex_eri(ctypes.byref(a), capi.dptr(c), capi.dptr(x))
    assert rc == -1 and 'cumulative' in capi.last_error(L)


def _zero_onee(sysm):
    n = sysm.basis.npgs
    z = np.zeros((sysm.ncell1, n, n))
    return z, z.copy(), z.copy()


def test_f_shells_are_refused():
    # cc-pVDZ with an f polarization shell added on oxygen (P_SHELL_ANG = 3): the
    # kernels stop at d and the C ABI says so
    from polymer_b200 import basis
    lib = {k: list(v) for k, v in basis.load_basis_library('cc-pVDZ').items()}
    lib['O'] = lib['O'] + [['F', 1.0, [[1.428, 1.0]]]]
    s = system.build_system(geometry.water_deck(1, seed=1), _zero_onee, library=lib)
    assert int(np.max(s.basis.p_shell_ang)) == 3
    n = s.basis.npgs
    with pytest.raises(capi.FockError) as e:
        fock.fourindex_eri(s, np.zeros((1, n, n)))
    assert e.value.code == -3


def test_helix_in_more_than_one_dimension_is_refused():
    # the reference's 'HELICAL SYMMETRY FOR 1D CRYSTAL ONLY'
    s = system.build_system(geometry.polyethylene_deck('STO-3G', cutoff1=1, cutoff2=1, kpoints=2), oracle.onee)
    n = s.basis.npgs
    pp = np.zeros((s.ncell1, n, n))
    a, keep = s.pfe_args(pp, np.zeros_like(pp))
    a.cel1[1] = 1
    c = np.zeros(s.basis.ncgs ** 2 * s.ncell1 * 3)
    x = np.zeros_like(c)
    import ctypes
    L = capi.lib()
    assert L.pfe_fourindex_eri(ctypes.byref(a), capi.dptr(c), capi.dptr(x)) == -1
