"""Build libpolymer_fock.so in-tree for sm_100a with nvcc.

Sources: polymer_b200/csrc/*.cu; the class-specialised ERI header is
regenerated from gen_eri.py first.  Output: polymer_b200/_build/.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
OUT = os.path.join(HERE, '_build')
LIB = os.path.join(OUT, 'libpolymer_fock.so')
# the largest units first: the pool starts them before the small ones
SOURCES = ['pfe_mol_big2.cu', 'pfe_mol_big6.cu', 'pfe_mol_big4.cu', 'pfe_mol_big8.cu', 'pfe_mol_big3.cu',
           'pfe_mol_big7.cu', 'pfe_mol_big1.cu', 'pfe_mol_big5.cu', 'pfe_mol.cu', 'pfe_mol_batch.cu',
           'pfe_mol_mixed.cu', 'pfe_mol_batch_mixed.cu', 'pfe_mol_wide.cu', 'pfe_api.cu', 'pfe_eri.cu', 'pfe_lattice.cu', 'pfe_lattice_sl.cu', 'pfe_grad.cu', 'pfe_onee.cu',
           'pfe_mlp.cu', 'pfe_scf.cu']
NVCC = os.environ.get('NVCC', 'nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC', '-diag-suppress', '177,550'] + \
    os.environ.get('PFE_NVCC_FLAGS', '').split()


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('command failed: %s\n%s\n%s' % (' '.join(cmd), r.stdout[-4000:], r.stderr[-8000:]))
    return r.stdout + r.stderr


def generate():
    gen = os.path.join(CSRC, 'gen_eri.py')
    out = os.path.join(CSRC, 'generated', 'eri_classes.cuh')
    grad = os.path.join(CSRC, 'generated', 'eri_grad_tables.cuh')   # made at build time, not committed
    os.makedirs(os.path.dirname(out), exist_ok=True)
    if any((not os.path.exists(f)) or os.path.getmtime(f) < os.path.getmtime(gen) for f in (out, grad)):
        _run([sys.executable, gen, out, '2'])


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile every CUDA source and link the shared library; returns its path."""
    generate()
    os.makedirs(OUT, exist_ok=True)
    # every unit depends on every header (conservative); a unit is rebuilt when
    # its source or a header is newer than its object
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith('.cuh')]
    headers += [os.path.join(CSRC, 'generated', 'eri_classes.cuh'),
                os.path.join(CSRC, 'generated', 'eri_grad_tables.cuh'),
                os.path.join(os.path.dirname(HERE), 'include', 'polymer_fock.h'),
                os.path.join(os.path.dirname(HERE), 'include', 'polymer_guess.h'),
                os.path.join(os.path.dirname(HERE), 'include', 'polymer_scf.h')]
    newest_header = max(os.path.getmtime(d) for d in headers if os.path.exists(d))
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]

    def stale(src):
        obj = os.path.join(OUT, src.replace('.cu', '.o'))
        return ptxas_info or not os.path.exists(obj) or \
            os.path.getmtime(obj) < max(newest_header, os.path.getmtime(os.path.join(CSRC, src)))

    todo = [s for s in srcs if stale(s)]
    if os.path.exists(LIB) and not todo and \
            os.path.getmtime(LIB) >= max(os.path.getmtime(os.path.join(OUT, s.replace('.cu', '.o'))) for s in srcs):
        return LIB

    def compile_one(src):
        obj = os.path.join(OUT, src.replace('.cu', '.o'))
        if src not in todo:
            return obj
        cmd = [NVCC] + ARCH + FLAGS + (['-Xptxas', '-v'] if ptxas_info else []) + \
            ['-c', os.path.join(CSRC, src), '-o', obj + '.tmp']
        log = _run(cmd)
        os.replace(obj + '.tmp', obj)
        if ptxas_info:
            with open(os.path.join(OUT, src.replace('.cu', '.ptxas.txt')), 'w') as fh:
                fh.write(log)
        return obj

    with cf.ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = LIB + '.tmp'
    _run([NVCC] + ARCH + ['-shared', '-o', tmp] + objs + ['-lcublas'])
    os.replace(tmp, LIB)
    if verbose:
        print('built', LIB)
    return LIB


if __name__ == '__main__':
    print(build(verbose=True, ptxas_info='--ptxas' in sys.argv))
