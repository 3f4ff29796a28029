"""The generated op tables of the interpreters (polymer_b200/csrc/gen_eri.py),
evaluated on the CPU with the op semantics the kernels use (eval_op):

* a table's levels order its ops by dependency (every source slot of an op is
  a Boys slot or the result of an earlier level);
* the pure-bra table of a class reproduces, bit for bit, every output of the
  full table whose bra components are all top-level, and reads the zero slot
  for the others -- so a chunk whose lower bra components carry no
  coefficient gets the same X from either table; the bra-and-ket table does
  the same for outputs whose bra and ket components are all top-level, and
  drops ops beyond the pure-bra table's;
* the straight-line kernels' register passes: the work each pass executes is
  at least one evaluation and at most npass of them, and the pass counts in
  straight_npass, the launcher table and the large classes' dispatch agree;
* the hand-kept op-table lookups and interpreter dispatch return each class's
  own tables and kernels, for exactly the classes the generator serves.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), '..', 'polymer_b200', 'csrc'))
import gen_eri  # noqa: E402


def _geometry(rng):
    g = {k: rng.normal(size=3) for k in ('PA', 'WP', 'QC', 'WQ', 'AB', 'CD')}
    z, h = rng.uniform(0.3, 2.0, size=2)
    rho = z * h / (z + h)
    G1 = [g['PA'], g['QC'], np.ones(3), np.ones(3)]
    G2 = [g['WP'], g['WQ'], g['AB'], g['CD']]
    X = [0.5 / z, 0.5 / h, 0.0, 0.0]
    Y = [rho / z, rho / h, 0.0, 0.0]
    Z = 0.5 / (z + h)
    return G1, G2, X, Y, Z


def _run(table, L, geo, F):
    """Evaluate a table level by level as the interpreters do: every op of a
    level reads the slots as they were when the level began (a level's ops run
    concurrently), then the level's results are written to their destinations."""
    ops, lev, outs, nslots = table
    G1, G2, X, Y, Z = geo
    v = np.full(nslots, np.nan)
    v[0] = 0.0
    v[1:L + 2] = F
    for lv in range(len(lev) - 1):
        snap = v.copy()
        written = set()
        for o in range(lev[lv], lev[lv + 1]):
            h, s1, s2, s3, s4, s5, dest = ops[o]
            kind, ax, cA, cB = h >> 12, (h >> 10) & 3, (h >> 5) & 31, h & 31
            srcs = [s1, s2] + ([s3, s4] if cA else []) + ([s5] if cB else [])
            assert all(not np.isnan(snap[x]) for x in srcs), 'op reads a slot no earlier level wrote'
            val = G1[kind][ax] * snap[s1] + G2[kind][ax] * snap[s2]
            if cA:
                val += cA * X[kind] * (snap[s3] - Y[kind] * snap[s4])
            if cB:
                val += cB * Z * snap[s5]
            assert dest > L + 1 and dest not in written, 'two ops of a level write one slot'
            written.add(dest)
            v[dest] = val
        # no op of this level read a slot this level overwrites
        for o in range(lev[lv], lev[lv + 1]):
            h, s1, s2, s3, s4, s5, dest = ops[o]
            cA, cB = (h >> 5) & 31, h & 31
            srcs = [s1, s2] + ([s3, s4] if cA else []) + ([s5] if cB else [])
            assert not (set(srcs) & written), 'a slot is read and rewritten within one level'
    return np.array([v[x] for x in outs])


CLASSES = [(1, 0, 1, 0), (1, 1, 1, 0), (2, 1, 1, 0), (2, 0, 2, 0), (2, 2, 1, 0), (2, 1, 2, 1)]


@pytest.mark.parametrize('ket', [False, True], ids=['bra', 'bra_ket'])
@pytest.mark.parametrize('cls', CLASSES)
def test_pure_table_matches_the_full_table(cls, ket):
    LA, LB, LC, LD = cls
    L = sum(cls)
    rng = np.random.default_rng(sum(cls))
    geo = _geometry(rng)
    F = rng.uniform(0.1, 1.0, size=L + 1)
    full = _run(gen_eri.gen_optable(*cls), L, geo, F)
    pure_table = gen_eri.gen_optable(*cls, pure_bra=True, pure_ket=ket)
    if ket:
        assert gen_eri.pure_ket_gains(*cls) == (len(pure_table[0]) <
                                                len(gen_eri.gen_optable(*cls, pure_bra=True)[0]))
    else:
        assert len(pure_table[0]) < len(gen_eri.gen_optable(*cls)[0])
    assert pure_table[3] <= gen_eri.gen_optable(*cls)[3]   # fits the full table's slots
    pure = _run(pure_table, L, geo, F)
    ca, cb, cc, cd = (gen_eri.comps(x) for x in cls)
    k = 0
    for a in ca:
        for b in cb:
            top = (LA == 0 or gen_eri.tot(a) == LA) and (LB == 0 or gen_eri.tot(b) == LB)
            for c in cc:
                for d in cd:
                    if ket:
                        top_k = (LC == 0 or gen_eri.tot(c) == LC) and (LD == 0 or gen_eri.tot(d) == LD)
                    else:
                        top_k = True
                    if top and top_k:
                        assert pure[k] == full[k]
                    else:
                        assert pure[k] == 0.0 and pure_table[2][k] == 0
                    k += 1
    assert k == len(full)


@pytest.mark.parametrize('cls,npass', [((1, 1, 1, 0), 2), ((2, 0, 1, 0), 2), ((2, 1, 1, 1), 14), ((2, 2, 1, 0), 10)])
def test_pass_work_accounting(cls, npass):
    # one pass evaluates the whole recursion once; more passes repeat the ops
    # their outputs share, never less than one evaluation, and skipping the
    # all-lower passes of pure bra shells only removes work
    full, one, n1 = gen_eri.pass_work(*cls, 1)
    assert one == full and n1 == 1
    _, many, n = gen_eri.pass_work(*cls, npass)
    assert n == npass and full <= many <= npass * full
    _, pure, npure = gen_eri.pass_work(*cls, npass, pure_bra=True)
    assert npure <= npass and pure <= many


def test_pass_tables_agree():
    # the pass count of each straight-line class lives in three hand-kept
    # places: straight_npass (census, launch count), the launcher table of the
    # smaller classes and the dispatch of the large ones (one unit per class,
    # FP64 and batch instantiations); they must name the same classes and passes
    import re
    csrc = os.path.join(os.path.dirname(__file__), '..', 'polymer_b200', 'csrc')
    kern = open(os.path.join(csrc, 'pfe_mol_kernels.cuh')).read()
    body = kern[kern.index('static inline int straight_npass'):]
    nums = [int(v) for v in re.findall(r'\d+', body[body.index('{{'):body.index('}};')])]
    npass = [nums[6 * i:6 * i + 6] for i in range(6)]
    cls = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]
    seen = {}
    table = kern[kern.index('static const LaunchFn table[6][6]'):]
    table = table[:table.index('#undef Q')]
    rows = re.findall(r'\{((?:Q\([^)]*\)|nullptr|[\s,])*)\}', table)
    assert len(rows) == 6
    for r, row in enumerate(rows):
        entries = re.findall(r'Q\([^)]*\)|nullptr', row)
        assert len(entries) == 6
        for c, entry in enumerate(entries):
            m = re.match(r'Q\((\d), (\d), (\d), (\d), (\d+)\)', entry)
            if m:
                seen[(r, c)] = tuple(int(v) for v in m.groups())
    big = open(os.path.join(csrc, 'pfe_mol_big1.cu')).read()
    for m in re.finditer(r'case (\d) \* 8 \+ (\d): return &launch_q<(\d), (\d), (\d), (\d), (\d+), false, BATCH>', big):
        key = (int(m.group(1)), int(m.group(2)))
        assert key not in seen
        seen[key] = tuple(int(v) for v in m.groups()[2:])
        inst = 'template void launch_q<%s, %s, %s, %s, %s, false, %%s>' % m.groups()[2:]
        units = ''.join(open(os.path.join(csrc, 'pfe_mol_big%d.cu' % k)).read() for k in range(1, 9))
        for batch in ('false', 'true'):
            assert any(line.startswith(inst % batch) for line in units.splitlines()), inst % batch
    assert len(seen) == sum(1 for row in npass for v in row if v) == 19
    for cb in range(6):
        for ck in range(6):
            if npass[cb][ck] == 0:
                assert (cb, ck) not in seen
            else:
                assert seen[(cb, ck)] == cls[cb] + cls[ck] + (npass[cb][ck],)


def test_table_lookups_match_the_generator():
    # host_optable*, hand-kept: each case returns the table of its own class,
    # the full tables cover every class, the pure-bra ones every bra class with
    # a p or d shell, and the bra-and-ket ones exactly the classes the
    # generator emits them for
    import re
    src = open(os.path.join(os.path.dirname(__file__), '..', 'polymer_b200', 'csrc', 'pfe_eri.cu')).read()
    cls = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (2, 2)]

    def cases(fn, suffix):
        body = src[src.index('const OpTableHost* %s(int cb, int ck) {' % fn):]
        body = body[:body.index('\n}\n')]
        got = set()
        for m in re.finditer(r'case (?:(\d) \* 8 \+ (\d)|0): return &op_(\d{4})%s;' % suffix, body):
            cb, ck = (int(m.group(1)), int(m.group(2))) if m.group(1) else (0, 0)
            assert m.group(3) == '%d%d%d%d' % (cls[cb] + cls[ck]), m.group(0)
            got.add((cb, ck))
        return got

    every = {(cb, ck) for cb in range(6) for ck in range(cb + 1)}
    assert cases('host_optable', '') == every
    assert cases('host_optable_pure', '_pure') == {(b, k) for b, k in every if cls[b][0] >= 1}
    assert cases('host_optable_pure2', '_pure2') == {
        (b, k) for b, k in every if cls[b][0] >= 1 and cls[k][0] >= 1 and gen_eri.pure_ket_gains(*(cls[b] + cls[k]))}
    # the interpreters' template dispatch (variants() of pfe_mol.cu), likewise
    mol = open(os.path.join(os.path.dirname(__file__), '..', 'polymer_b200', 'csrc', 'pfe_mol.cu')).read()
    body = mol[mol.index('static Variants variants(int cb, int ck) {'):]
    body = body[:body.index('\n}\n')]
    got = set()
    for m in re.finditer(r'case (\d+): return V\((\d), (\d), (\d), (\d)\);', body):
        cb, ck = divmod(int(m.group(1)), 8)
        assert tuple(int(v) for v in m.groups()[1:]) == cls[cb] + cls[ck], m.group(0)
        got.add((cb, ck))
    assert got == every


@pytest.mark.parametrize('cls', CLASSES + [(2, 2, 2, 1)])
def test_slot_reuse_keeps_every_output(cls):
    """Slots reused after their value's last reader (compact tables, what the
    kernels run) give every output bit for bit as tables with one slot per
    node, in fewer slots."""
    L = sum(cls)
    rng = np.random.default_rng(7 + L)
    geo = _geometry(rng)
    F = rng.uniform(0.1, 1.0, size=L + 1)
    for pb, pk in ((False, False), (True, False), (True, True)):
        if (pb and cls[0] == 0) or (pk and cls[2] == 0):
            continue
        loose = gen_eri.gen_optable(*cls, pure_bra=pb, pure_ket=pk, compact=False)
        tight = gen_eri.gen_optable(*cls, pure_bra=pb, pure_ket=pk)
        a, b = _run(loose, L, geo, F), _run(tight, L, geo, F)
        assert np.array_equal(a, b)
        assert tight[3] <= loose[3]
        if len(tight[0]) > 1000:   # the large classes: a half to two thirds of the slots
            assert tight[3] < 0.75 * loose[3]
