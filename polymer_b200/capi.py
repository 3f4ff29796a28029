"""ctypes mirror of include/polymer_fock.h and the loader of libpolymer_fock.so.

The library is built in-tree (``polymer_b200/_build/libpolymer_fock.so``) by
``polymer_b200.build``.  There is no fallback: if the shared object is missing
or fails to load, :func:`lib` raises, so a Fock build never silently runs
anywhere but the CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# PFE_LIBRARY names another build of the library to load instead (a variant
# compiled with other tuning macros); by default the in-tree build.
LIB_PATH = os.environ.get('PFE_LIBRARY') or os.path.join(HERE, '_build', 'libpolymer_fock.so')

PFE_OK = 0
PFE_PREC_FP64 = 0
PFE_PREC_MIXED = 1
_ERRNAMES = {-1: 'PFE_EINVAL', -2: 'PFE_ECUDA', -3: 'PFE_EUNSUPPORTED', -4: 'PFE_ERANGE',
             -5: 'PFE_ENOMEM', -6: 'PFE_ETIMEOUT', -7: 'PFE_ENAN'}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class PfeArgs(ctypes.Structure):
    _fields_ = [
        ('npgs', ctypes.c_int32), ('ncgs', ctypes.c_int32), ('npshell', ctypes.c_int32),
        ('lmax', ctypes.c_int32),
        ('p_shell', _ip), ('p_shell_ang', _ip),
        ('pgsx', _dp), ('pgsy', _dp), ('pgsz', _dp), ('zt', _dp),
        ('cc', _dp), ('c2h', _dp), ('s_p', _dp), ('p_p', _dp), ('p_p_helix', _dp),
        ('igamma', _dp),
        ('cel1', ctypes.c_int32 * 3), ('cel2', ctypes.c_int32 * 3),
        ('reduced_cel1', ctypes.c_int32 * 3),
        ('period', ctypes.c_double * 3), ('helix', ctypes.c_double),
        ('inttol', ctypes.c_double),
        ('print_level', ctypes.c_int32), ('myid', ctypes.c_int32), ('numprocs', ctypes.c_int32),
        ('precision_mode', ctypes.c_int32), ('mixed_cutoff', ctypes.c_double),
    ]


class PfeOneeArgs(ctypes.Structure):
    _fields_ = [('npgs', ctypes.c_int32), ('npshell', ctypes.c_int32), ('natom', ctypes.c_int32),
                ('p_shell', _ip), ('p_shell_ang', _ip), ('pgs_atom', _ip),
                ('pgsx', _dp), ('pgsy', _dp), ('pgsz', _dp), ('zt', _dp),
                ('iatom', _ip), ('atomx', _dp), ('atomy', _dp), ('atomz', _dp),
                ('cel1', ctypes.c_int32 * 3), ('cel2', ctypes.c_int32 * 3),
                ('period', ctypes.c_double * 3), ('helix', ctypes.c_double),
                ('igamma', _dp)]


class PfeCensus(ctypes.Structure):
    _fields_ = [('quartets', ctypes.c_double), ('quartets_ref', ctypes.c_double),
                ('flops', ctypes.c_double), ('quartets_fp32', ctypes.c_double),
                ('pairs', ctypes.c_int64), ('kernel_launches', ctypes.c_int32)]


class PfeKernelStat(ctypes.Structure):
    _fields_ = [('cls', ctypes.c_int32), ('variant', ctypes.c_int32), ('ms', ctypes.c_float),
                ('tuned_ms', ctypes.c_float * 4), ('quartets', ctypes.c_double), ('flops', ctypes.c_double),
                ('grid_mult', ctypes.c_int32), ('pad_', ctypes.c_int32)]


class FockError(RuntimeError):
    """A non-zero status from the library (the reference would PABORT)."""

    def __init__(self, code: int, msg: str):
        super().__init__('%s (%d): %s' % (_ERRNAMES.get(code, 'PFE_E?'), code, msg))
        self.code = code


def dptr(a: Optional[np.ndarray]):
    if a is None:
        return ctypes.cast(None, _dp)
    assert a.dtype == np.float64 and a.flags['F_CONTIGUOUS'] or a.flags['C_CONTIGUOUS']
    return a.ctypes.data_as(_dp)


def iptr(a: Optional[np.ndarray]):
    if a is None:
        return ctypes.cast(None, _ip)
    assert a.dtype == np.int32
    return a.ctypes.data_as(_ip)


_LIB = None


def lib(path: str = LIB_PATH):
    """Load libpolymer_fock.so; raises if it is absent (no CPU fallback exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError('libpolymer_fock.so not built at %s: run python -c "import polymer_b200.build as b; b.build()"' % path)
    L = ctypes.CDLL(path)
    L.pfe_fourindex_eri.argtypes = [ctypes.POINTER(PfeArgs), _dp, _dp]
    L.pfe_fourindex_eri.restype = ctypes.c_int32
    L.pfe_fourindex_eri_gradient.argtypes = [ctypes.POINTER(PfeArgs), _ip, ctypes.c_int32, _dp, _dp]
    L.pfe_fourindex_eri_gradient.restype = ctypes.c_int32
    L.pfe_last_error.argtypes = [ctypes.c_char_p, ctypes.c_int32]
    L.pfe_last_error.restype = ctypes.c_int32
    L.pfe_context_create.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
    L.pfe_context_create.restype = ctypes.c_int32
    L.pfe_context_destroy.argtypes = [ctypes.c_void_p]
    L.pfe_context_destroy.restype = ctypes.c_int32
    L.pfe_context_setup.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfeArgs)]
    L.pfe_context_setup.restype = ctypes.c_int32
    L.pfe_context_fock.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.pfe_context_fock.restype = ctypes.c_int32
    L.pfe_context_fock_pc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
    L.pfe_context_fock_pc.restype = ctypes.c_int32
    L.pfe_context_set_screening.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double]
    L.pfe_context_set_screening.restype = ctypes.c_int32
    L.pfe_context_primitive_targets.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    L.pfe_context_primitive_targets.restype = ctypes.c_int32
    L.pfe_batch_create.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]
    L.pfe_batch_create.restype = ctypes.c_int32
    L.pfe_batch_setup.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfeArgs), ctypes.c_int32]
    L.pfe_batch_setup.restype = ctypes.c_int32
    L.pfe_batch_offsets.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]
    L.pfe_batch_offsets.restype = ctypes.c_int32
    L.pfe_batch_set_screening.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_double, ctypes.c_double]
    L.pfe_batch_set_screening.restype = ctypes.c_int32
    L.pfe_batch_set_instance_screening.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                                   ctypes.c_double]
    L.pfe_batch_set_instance_screening.restype = ctypes.c_int32
    L.pfe_batch_autotune.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.pfe_batch_autotune.restype = ctypes.c_int32
    L.pfe_batch_schedule.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfeKernelStat), ctypes.c_int32]
    L.pfe_batch_schedule.restype = ctypes.c_int32
    L.pfe_batch_refresh.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.pfe_batch_refresh.restype = ctypes.c_int32
    L.pfe_batch_fock_pc.argtypes = [ctypes.c_void_p] * 5
    L.pfe_batch_fock_pc.restype = ctypes.c_int32
    L.pfe_batch_census.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfeCensus)]
    L.pfe_batch_census.restype = ctypes.c_int32
    L.pfe_batch_destroy.argtypes = [ctypes.c_void_p]
    L.pfe_batch_destroy.restype = ctypes.c_int32
    L.pfe_context_census.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfeCensus)]
    L.pfe_context_census.restype = ctypes.c_int32
    L.pfe_overlap_kinetic.argtypes = [ctypes.POINTER(PfeOneeArgs), _dp, _dp]
    L.pfe_overlap_kinetic.restype = ctypes.c_int32
    L.pfe_nuclear_attraction.argtypes = [ctypes.POINTER(PfeOneeArgs), _dp]
    L.pfe_nuclear_attraction.restype = ctypes.c_int32
    L.pfe_overlap_kinetic_noalloc.argtypes = [ctypes.POINTER(PfeOneeArgs), _dp, _dp]
    L.pfe_overlap_kinetic_noalloc.restype = ctypes.c_int32
    L.pfe_context_profile.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    L.pfe_context_profile.restype = ctypes.c_int32
    L.pfe_context_kernel_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(PfeKernelStat), ctypes.c_int32]
    L.pfe_context_kernel_stats.restype = ctypes.c_int32
    L.pfe_context_autotune.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.pfe_context_autotune.restype = ctypes.c_int32
    L.pfe_context_force_variant.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    L.pfe_context_force_variant.restype = ctypes.c_int32
    L.pfe_measure_fp64_peak.argtypes = [ctypes.c_int32, _dp]
    L.pfe_measure_fp64_peak.restype = ctypes.c_int32
    L.pfe_version.argtypes = []
    L.pfe_version.restype = ctypes.c_char_p
    L.pfe_debug_fail_allocation.argtypes = [ctypes.c_int32]
    L.pfe_debug_fail_allocation.restype = ctypes.c_int32
    _vp, _i32, _i64, _f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    for name, args in (('pfe_mlp_gemm', [_vp, _vp, _vp, _i32, _i32, _i32, _i32, _i32, _i32, _vp]),
                       ('pfe_mlp_bias_act', [_vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp]),
                       ('pfe_mlp_act_grad', [_vp, _vp, _vp, _vp, _i64, _i32, _vp]),
                       ('pfe_mlp_colsum', [_vp, _vp, _i32, _i32, _vp]),
                       ('pfe_mlp_mse', [_vp, _vp, _vp, _f32, _vp, _vp, _i64, _vp]),
                       ('pfe_mlp_adam', [_vp, _vp, _vp, _vp, _vp, _i64, _f32, _f32, _f32, _f32, _i32, _f32, _vp]),
                       ('pfe_mlp_to_bf16', [_vp, _vp, _i64, _vp]),
                       ('pfe_scf_next_density', [_i32, _i32, _i32] + [_vp] * 11),
                       ('pfe_scf_fock_assemble', [_i32, _i32] + [_vp] * 14),
                       ('pfe_scf_commutator', [_i32, _i32, _i32] + [_vp] * 9),
                       ('pfe_scf_diis', [_i32, _i32, _i32] + [_vp] * 9),
                       ('pfe_scf_sp2_init', [_i32, _i32, _vp, _vp, _vp, _vp]),
                       ('pfe_scf_sp2_step', [_i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp]),
                       ('pfe_scf_finish', [_i32, _i32, ctypes.c_double] + [_vp] * 9)):
        getattr(L, name).argtypes = args
        getattr(L, name).restype = ctypes.c_int32
    L.pfe_scf_workspace.argtypes = [_i32, _i32, _i32]
    L.pfe_scf_workspace.restype = ctypes.c_int64
    _LIB = L
    return L


def last_error(L) -> str:
    buf = ctypes.create_string_buffer(1024)
    L.pfe_last_error(buf, 1024)
    return buf.value.decode(errors='replace')


def check(L, code: int) -> None:
    if code != PFE_OK:
        raise FockError(code, last_error(L))


# Exported symbols declared in include/polymer_fock.h (checked by the CPU tests).
EXPORTS = ['pfe_fourindex_eri', 'pfe_last_error', 'pfe_context_create', 'pfe_context_destroy',
           'pfe_context_setup', 'pfe_context_fock', 'pfe_context_census', 'pfe_overlap_kinetic',
           'pfe_nuclear_attraction', 'pfe_context_profile', 'pfe_context_kernel_stats',
           'pfe_measure_fp64_peak', 'pfe_context_autotune', 'pfe_context_force_variant',
           'pfe_version', 'pfe_overlap_kinetic_noalloc', 'pfe_context_fock_pc',
           'pfe_context_primitive_targets', 'pfe_context_set_screening', 'pfe_batch_create', 'pfe_batch_setup',
           'pfe_batch_set_screening', 'pfe_batch_set_instance_screening', 'pfe_batch_offsets', 'pfe_batch_refresh',
           'pfe_batch_autotune', 'pfe_batch_schedule', 'pfe_batch_fock_pc', 'pfe_batch_census', 'pfe_batch_destroy',
           'pfe_fourindex_eri_gradient', 'pfe_debug_fail_allocation']

# Exported symbols declared in include/polymer_guess.h (checked by the CPU tests).
GUESS_EXPORTS = ['pfe_mlp_gemm', 'pfe_mlp_bias_act', 'pfe_mlp_act_grad', 'pfe_mlp_colsum', 'pfe_mlp_mse',
                 'pfe_mlp_adam', 'pfe_mlp_to_bf16']

# Exported symbols declared in include/polymer_scf.h (checked by the CPU tests).
SCF_EXPORTS = ['pfe_scf_workspace', 'pfe_scf_next_density', 'pfe_scf_fock_assemble', 'pfe_scf_commutator',
               'pfe_scf_diis', 'pfe_scf_sp2_init', 'pfe_scf_sp2_step', 'pfe_scf_finish']
