"""C-ABI surface checks that need no GPU.

* every entry point include/polymer_fock.h declares is exported by the built
  libpolymer_fock.so (no compute call is made);
* the ctypes mirrors of pfe_args / pfe_onee_args / pfe_census /
  pfe_kernel_stat have exactly the C layout (offsets measured by compiling a
  probe against the header);
* the ctypes signature of every prototype in include/*.h matches it (count,
  pointers, scalar and return types);
* the Fortran shim's BIND(C) type (fortran/pfourindexdirect_gpu.f90) has
  pfe_args' members in order, with the same kinds and array lengths;
* the one-electron entry points refuse a P_SHELL entry outside 1..NPGS for a
  component a shell reaches with PFE_EINVAL, before any device work (so the
  call returns the same on a machine without a GPU).
"""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from polymer_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, 'include', 'polymer_fock.h')


GUESS_HEADER = os.path.join(ROOT, 'include', 'polymer_guess.h')
SCF_HEADER = os.path.join(ROOT, 'include', 'polymer_scf.h')


def _declared(path=HEADER):
    txt = open(path).read()
    return sorted(set(re.findall(r'\b(pfe_[a-z0-9_]+)\s*\(', txt)))


def test_header_declares_the_exports():
    assert _declared() == sorted(capi.EXPORTS)
    assert _declared(GUESS_HEADER) == sorted(capi.GUESS_EXPORTS)
    assert _declared(SCF_HEADER) == sorted(capi.SCF_EXPORTS)


def test_library_exports_every_symbol():
    lib = build.build()
    out = subprocess.run(['nm', '-D', '--defined-only', lib], capture_output=True, text=True, check=True).stdout
    exported = set(ln.split()[-1] for ln in out.splitlines() if ln.strip())
    missing = [s for s in capi.EXPORTS + capi.GUESS_EXPORTS + capi.SCF_EXPORTS if s not in exported]
    assert not missing, missing


@pytest.mark.parametrize('cname,pyt', [('pfe_args', capi.PfeArgs), ('pfe_onee_args', capi.PfeOneeArgs),
                                       ('pfe_census', capi.PfeCensus), ('pfe_kernel_stat', capi.PfeKernelStat)])
def test_struct_layout_matches_header(cname, pyt):
    fields = [f[0] for f in pyt._fields_]
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "%s"' % HEADER, 'int main(void){',
           'printf("%%zu\\n", sizeof(%s));' % cname]
    for f in fields:
        src.append('printf("%%zu\\n", offsetof(%s, %s));' % (cname, f))
    src.append('return 0;}')
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, 'probe.c')
        exe = os.path.join(d, 'probe')
        open(c, 'w').write('\n'.join(src))
        subprocess.run(['gcc', '-o', exe, c], check=True)
        vals = [int(v) for v in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(pyt)
    for f, off in zip(fields, vals[1:]):
        assert getattr(pyt, f).offset == off, f


def test_ctypes_signatures_match_the_headers():
    # every prototype of include/*.h against the argtypes/restype capi.py sets:
    # argument count, pointer or not, and the scalar type of the rest
    root = os.path.join(os.path.dirname(__file__), '..', 'include')
    hdr = ''.join(open(os.path.join(root, f)).read() for f in sorted(os.listdir(root)) if f.endswith('.h'))
    hdr = re.sub(r'/\*.*?\*/', '', hdr, flags=re.S)
    protos = {m.group(2): (m.group(1), m.group(3))
              for m in re.finditer(r'\b(int32_t|void|double)\s+(pfe_\w+)\s*\(([^)]*)\)\s*;', hdr)}
    assert len(protos) >= len(capi.EXPORTS)
    scalar = {'int32_t': ctypes.c_int32, 'int64_t': ctypes.c_int64, 'double': ctypes.c_double,
              'float': ctypes.c_float}
    L = capi.lib()
    for name, (ret, args) in protos.items():
        fn = getattr(L, name)
        params = [a.strip() for a in args.split(',')] if args.strip() not in ('', 'void') else []
        assert fn.argtypes is not None and len(fn.argtypes) == len(params), name
        for p, t in zip(params, fn.argtypes):
            if '*' in p:
                assert t is ctypes.c_void_p or t is ctypes.c_char_p or issubclass(t, ctypes._Pointer), (name, p)
            else:
                ctype = p.replace('const', '').split()[0]
                assert t is scalar[ctype], (name, p, t)
        if ret != 'void':
            assert fn.restype is scalar[ret], (name, ret)


def test_fortran_shim_type_matches_pfe_args():
    # the BIND(C) type of the Fortran shim fortran/pfourindexdirect_gpu.f90 (no
    # Fortran compiler here to check it): same members, order, kinds and array
    # lengths as pfe_args, whose ctypes mirror the layout test pins to the header
    src = open(os.path.join(ROOT, 'fortran', 'pfourindexdirect_gpu.f90')).read()
    body = src[src.index('TYPE, BIND(C) :: PFE_ARGS'):src.index('END TYPE')]
    kinds = {'INTEGER(C_INT32_T)': ctypes.c_int32, 'REAL(C_DOUBLE)': ctypes.c_double, 'TYPE(C_PTR)': None}
    fortran = []
    for line in body.splitlines()[1:]:
        if not line.strip():
            continue
        m = re.match(r'\s*(INTEGER\(C_INT32_T\)|REAL\(C_DOUBLE\)|TYPE\(C_PTR\))\s*::\s*(.*)', line)
        assert m, line
        for name, n in re.findall(r'(\w+)(?:\((\d+)\))?', m.group(2)):
            fortran.append((name.lower(), kinds[m.group(1)], int(n) if n else 1))
    c = []
    for name, t in capi.PfeArgs._fields_:
        if issubclass(t, ctypes.Array):
            c.append((name, t._type_, t._length_))
        elif issubclass(t, ctypes._Pointer) or t is ctypes.c_void_p:
            c.append((name, None, 1))
        else:
            c.append((name, t, 1))
    assert fortran == c


@pytest.mark.parametrize('bad', [0, -1, 10 ** 6])
@pytest.mark.parametrize('entry', ['pfe_overlap_kinetic', 'pfe_overlap_kinetic_noalloc', 'pfe_nuclear_attraction'])
def test_onee_entry_points_refuse_a_malformed_p_shell(entry, bad):
    import numpy as np

    import oracle
    from polymer_b200 import fock, geometry, system
    sysm = system.build_system(geometry.water_deck(1, seed=2001), oracle.onee)
    b = sysm.basis
    # a component the p shell reaches (its x component) points nowhere
    s = int(np.nonzero(b.p_shell_ang == 1)[0][0])
    a, keep = fock.onee_args(sysm)
    keep['p_shell'][s, 1, 0, 0] = bad
    a.p_shell = capi.iptr(keep['p_shell'])
    n = b.npgs ** 2 * sysm.ncell1
    out1, out2 = np.zeros(n), np.zeros(n)
    L = capi.lib()
    fn = getattr(L, entry)
    if entry == 'pfe_nuclear_attraction':
        rc = fn(ctypes.byref(a), capi.dptr(out1))
    else:
        rc = fn(ctypes.byref(a), capi.dptr(out1), capi.dptr(out2))
    assert rc == -1, (entry, bad, rc)   # PFE_EINVAL
    assert 'P_SHELL' in capi.last_error(L)
    assert not out1.any() and not out2.any()
