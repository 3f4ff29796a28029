"""Generate tests/golden/reference_runs.json from the reference's sample runs.

The reference ships no tests; its regression data are sample inputs and their
recorded stdout under data/.  This script (run once, where the reference tree
is present) extracts, for every Hartree-Fock-relevant sample:

* the input deck parsed into plain values (atoms, coordinates, keywords), so
  the test machine does not need the reference tree;
* the size census printed by READ3 (NPGS/NCGS/NPSHELL with ghosts);
* the SCF iteration table (ITR, DIIS, density change, total energy);
* the converged energy components (nuclear repulsion, kinetic, nuclear
  attraction, Coulomb, HF exchange, total);
* for the helical polyethylene sample, the per-cell maximum contracted overlap
  and the nuclear repulsion (its SCF is B3LYP, which this package does not implement).

Usage: python make_golden.py <reference-data-dir> [out.json]
"""
import json
import os
import re
import sys

SAMPLES = {
    'H2O_CCSD_ccpVDZ': 'scf',
    'BH_MBGF': 'scf',
    'FH_finiteT_MBPT_zeroT_HF_ref': 'scf',
    'FH_finiteT_MBPT_finiteT_HF_ref': 'scf',
    'Polyethylene_B3LYP_631G': 'lattice',
}

_NUM = r'(-?\d+\.\d+(?:E[-+]\d+)?)'


def parse_input(text):
    lines = text.splitlines()
    deck = {'geometry': [], 'keywords': {}}
    i = 0
    while i < len(lines):
        toks = lines[i].split()
        i += 1
        if not toks or toks[0].startswith('!'):
            continue
        key = toks[0].upper()
        if key == 'GEOMETRY':
            while i < len(lines):
                t = lines[i].split()
                i += 1
                if not t or t[0] == 'X':
                    break
                deck['geometry'].append([t[0]] + [float(v) for v in t[1:4]])
            continue
        deck['keywords'][key] = lines[i].strip()
        i += 1
    return deck


def parse_output(text, kind):
    out = {}
    m = re.search(r'NUMBER OF PRIMITIVE GAUSSIANS  \(INCLUDING GHOST FUNCTIONS\) =\s+(\d+)', text)
    out['npgs'] = int(m.group(1))
    out['ncgs'] = int(re.search(r'NUMBER OF CONTRACTED GAUSSIANS \(INCLUDING GHOST FUNCTIONS\) =\s+(\d+)', text).group(1))
    out['npshell'] = int(re.search(r'NUMBER OF SHELLS\s+\(INCLUDING GHOST FUNCTIONS\) =\s+(\d+)', text).group(1))
    out['nuclear_repulsion_setup'] = float(re.search(r'NUCLEAR REPULSION ENERGY =\s+' + _NUM, text).group(1))
    if kind == 'scf':
        block = text.split('SELF-CONSISTENT FIELD ITERATION')[1].split('SCF CONVERGED')[0]
        iters = []
        for ln in block.splitlines():
            t = ln.split()
            if len(t) >= 6 and t[0].isdigit() and t[1].isdigit():
                iters.append({'iscf': int(t[0]), 'idiis': int(t[1]), 'density_change': float(t[3]),
                              'energy': float(t[4])})
        out['iterations'] = iters
        tail = text.split('SCF CONVERGED')[1]
        for key, label in (('nuclear_repulsion', 'NUCLEAR REPULSION ENERGY'), ('kinetic', 'KINETIC ENERGY'),
                           ('nuclear_attraction', 'NUCLEAR ATTRACTION ENERGY'), ('coulomb', 'COULOMB ENERGY'),
                           ('exchange', 'HF-EXCHANGE ENERGY'), ('total', 'TOTAL SCF ENERGY')):
            out[key] = float(re.search(label + r'\s+=\s+' + _NUM, tail).group(1))
    else:
        block = text.split('X   MAXIMUM OVERLAP')[1].split('-----')[0]
        out['max_overlap_x'] = [float(ln.split()[1]) for ln in block.strip().splitlines()]
    return out


def main():
    src = sys.argv[1]
    dst = sys.argv[2] if len(sys.argv) > 2 else os.path.join(os.path.dirname(__file__), 'reference_runs.json')
    data = {}
    for name, kind in SAMPLES.items():
        with open(os.path.join(src, name)) as fh:
            deck = parse_input(fh.read())
        with open(os.path.join(src, name + '_out')) as fh:
            res = parse_output(fh.read(), kind)
        data[name] = {'kind': kind, 'deck': deck, 'expected': res,
                      'source': 'data/%s and data/%s_out' % (name, name)}
    with open(dst, 'w') as fh:
        json.dump(data, fh, indent=1)
    print('wrote', dst)


if __name__ == '__main__':
    main()
