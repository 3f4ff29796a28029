"""Generate class-specialised ERI device code (Head-Gordon-Pople on Obara-Saika).

For every quartet class (LA,LB|LC,LD) of *cumulative* primitive shells (a shell
of angular momentum L carries all Cartesian components of total power <= L,
as the reference's READ3 builds them), emit one straight-line device function
that, from the Boys values, produces every integral (ab|cd) with |a|<=LA,
|b|<=LB, |c|<=LC, |d|<=LD:

1. Obara-Saika vertical recursion on centre A:
   [e+1i,0|00]^m = PA_i[e0|00]^m + WP_i[e0|00]^{m+1}
                   + e_i/(2z)([e-1i,0|00]^m - (rho/z)[e-1i,0|00]^{m+1})
2. and onto centre C (with the electron-transfer cross term):
   [e0|f+1i,0]^m = QC_i[e0|f0]^m + WQ_i[e0|f0]^{m+1}
                   + f_i/(2h)([e0|f-1i,0]^m - (rho/h)[e0|f-1i,0]^{m+1})
                   + e_i/(2(z+h))[e-1i,0|f0]^{m+1}
3. horizontal recursions (a,b+1i| = (a+1i,b| + AB_i(a,b| and likewise on the ket.

This is the same function the reference evaluates with its two-centre OS
recursion (src/pfourindexdirect.f90:563-690); only the order of operations
differs.  The generator memoises the recursion DAG so only the nodes the
outputs need are emitted, and counts the floating-point operations of each
class (FMA = 2) for the roofline census.

Run: python gen_eri.py <out.cuh> [lmax]  (the build does this).
"""
import itertools
import math
import re
import json
import sys


def comps(L):
    """Cartesian powers of total <= L in the reference's loop order (i1 outer)."""
    out = []
    for i1 in range(L + 1):
        for i2 in range(L + 1 - i1):
            for i3 in range(L + 1 - i1 - i2):
                out.append((i1, i2, i3))
    return out


def tot(t):
    return t[0] + t[1] + t[2]


def dec(t, i, k=1):
    l = list(t)
    l[i] -= k
    return tuple(l)


def inc(t, i):
    l = list(t)
    l[i] += 1
    return tuple(l)


class Gen:
    def __init__(self, LA, LB, LC, LD):
        self.LA, self.LB, self.LC, self.LD = LA, LB, LC, LD
        self.L = LA + LB + LC + LD
        self.lines = []
        self.names = {}
        self.flops = 0
        self.n = 0

    def tmp(self):
        self.n += 1
        return 't%d' % self.n

    def emit(self, expr, flops):
        name = self.tmp()
        self.lines.append('    const R %s = %s;' % (name, expr))
        self.flops += flops
        return name

    # ---- vertical recursion --------------------------------------------------------
    def vrr(self, e, f, m):
        key = ('v', e, f, m)
        if key in self.names:
            return self.names[key]
        if tot(e) == 0 and tot(f) == 0:
            name = 'F[%d]' % m
            self.names[key] = name
            return name
        if tot(f) > 0:
            i = next(k for k in range(3) if f[k] > 0)
            fm = dec(f, i)
            terms = []
            fl = 0
            a = self.vrr(e, fm, m)
            b = self.vrr(e, fm, m + 1)
            expr = 'QC%d * %s + WQ%d * %s' % (i, a, i, b)
            fl += 3
            if fm[i] > 0:
                fmm = dec(fm, i)
                c = self.vrr(e, fmm, m)
                d = self.vrr(e, fmm, m + 1)
                expr += ' + (R)%d * oe * (%s - roe * %s)' % (fm[i], c, d)
                fl += 4
            if e[i] > 0:
                g = self.vrr(dec(e, i), fm, m + 1)
                expr += ' + (R)%d * oze * %s' % (e[i], g)
                fl += 2
            name = self.emit(expr, fl)
        else:
            i = next(k for k in range(3) if e[k] > 0)
            em = dec(e, i)
            a = self.vrr(em, f, m)
            b = self.vrr(em, f, m + 1)
            expr = 'PA%d * %s + WP%d * %s' % (i, a, i, b)
            fl = 3
            if em[i] > 0:
                emm = dec(em, i)
                c = self.vrr(emm, f, m)
                d = self.vrr(emm, f, m + 1)
                expr += ' + (R)%d * oz * (%s - roz * %s)' % (em[i], c, d)
                fl += 4
            name = self.emit(expr, fl)
        self.names[key] = name
        return name

    # ---- horizontal recursions ----------------------------------------------------
    def hrr_bra(self, a, b, f):
        """(a b|f 0]^0."""
        key = ('b', a, b, f)
        if key in self.names:
            return self.names[key]
        if tot(b) == 0:
            name = self.vrr(a, f, 0)
        else:
            i = next(k for k in range(3) if b[k] > 0)
            bm = dec(b, i)
            x = self.hrr_bra(inc(a, i), bm, f)
            y = self.hrr_bra(a, bm, f)
            name = self.emit('%s + AB%d * %s' % (x, i, y), 2)
        self.names[key] = name
        return name

    def hrr_ket(self, a, b, c, d):
        key = ('k', a, b, c, d)
        if key in self.names:
            return self.names[key]
        if tot(d) == 0:
            name = self.hrr_bra(a, b, c)
        else:
            i = next(k for k in range(3) if d[k] > 0)
            dm = dec(d, i)
            x = self.hrr_ket(a, b, inc(c, i), dm)
            y = self.hrr_ket(a, b, c, dm)
            name = self.emit('%s + CD%d * %s' % (x, i, y), 2)
        self.names[key] = name
        return name

    def build(self):
        CA, CB, CC, CDc = comps(self.LA), comps(self.LB), comps(self.LC), comps(self.LD)
        outs = []
        for a in CA:
            for b in CB:
                for c in CC:
                    for d in CDc:
                        outs.append(self.hrr_ket(a, b, c, d))
        return outs


OPS_THRESHOLD = 1600  # classes with more integrals have no straight-line function (op tables only)


def gen_optable(LA, LB, LC, LD, pure_bra=False, pure_ket=False, compact=True):
    """Level-scheduled op table of one class for the block-cooperative interpreter.

    Slot 0 holds zero, slots 1..L+1 the Boys values F[m]; the recursion nodes
    are ordered by dependency level so that all ops of a level can run in
    parallel.  Each op is seven uint16: (kind<<12 | axis<<10 | cA<<5 | cB, s1,
    s2, s3, s4, s5, dest) computing into slot dest
      v = G1*s1 + G2*s2 + cA*X*(s3 - Y*s4) + cB*Z*s5
    with (G1, G2, X, Y, Z) = (PA, WP, 1/2z, rho/z, 0) for kind 0 (VRR on A),
    (QC, WQ, 1/2h, rho/h, 1/2(z+h)) for kind 1 (VRR on C), (1, AB, 0, 0, 0)
    for kind 2 (bra HRR) and (1, CD, 0, 0, 0) for kind 3 (ket HRR).

    With `compact` a node's slot is reused once every reader of its value has
    run: a value last read at level l frees its slot for the writers of levels
    l+1 and later (the readers of one level run concurrently with its writers,
    so a slot never changes hands inside a level), and the outputs keep theirs
    to the end.  That halves the slots of the large classes (the interpreters'
    shared memory); without it every node has a slot of its own.
    """
    L = LA + LB + LC + LD
    nodes = {}     # key -> (kind, axis, cA, cB, [src keys]) ; leaves are ('F', m)
    order = []

    def vrr(e, f, m):
        key = ('v', e, f, m)
        if key in nodes:
            return key
        if tot(e) == 0 and tot(f) == 0:
            return ('F', m)
        if tot(f) > 0:
            i = next(k for k in range(3) if f[k] > 0)
            fm = dec(f, i)
            srcs = [vrr(e, fm, m), vrr(e, fm, m + 1), None, None, None]
            cA = cB = 0
            if fm[i] > 0:
                fmm = dec(fm, i)
                srcs[2], srcs[3] = vrr(e, fmm, m), vrr(e, fmm, m + 1)
                cA = fm[i]
            if e[i] > 0:
                srcs[4] = vrr(dec(e, i), fm, m + 1)
                cB = e[i]
            nodes[key] = (1, i, cA, cB, srcs)
        else:
            i = next(k for k in range(3) if e[k] > 0)
            em = dec(e, i)
            srcs = [vrr(em, f, m), vrr(em, f, m + 1), None, None, None]
            cA = 0
            if em[i] > 0:
                emm = dec(em, i)
                srcs[2], srcs[3] = vrr(emm, f, m), vrr(emm, f, m + 1)
                cA = em[i]
            nodes[key] = (0, i, cA, 0, srcs)
        order.append(key)
        return key

    def hb(a, b, f):
        key = ('b', a, b, f)
        if key in nodes:
            return key
        if tot(b) == 0:
            return vrr(a, f, 0)
        i = next(k for k in range(3) if b[k] > 0)
        bm = dec(b, i)
        nodes[key] = (2, i, 0, 0, [hb(inc(a, i), bm, f), hb(a, bm, f), None, None, None])
        order.append(key)
        return key

    def hk(a, b, c, d):
        key = ('k', a, b, c, d)
        if key in nodes:
            return key
        if tot(d) == 0:
            return hb(a, b, c)
        i = next(k for k in range(3) if d[k] > 0)
        dm = dec(d, i)
        nodes[key] = (3, i, 0, 0, [hk(a, b, inc(c, i), dm), hk(a, b, c, dm), None, None, None])
        order.append(key)
        return key

    def kept(a, b):
        # pure_bra: only the top-level components of the bra shells, for bra shells
        # whose lower components carry no coefficient (the d shells of 6-31G** and
        # cc-pVDZ); the other outputs read slot 0, which holds zero
        return not pure_bra or ((LA == 0 or tot(a) == LA) and (LB == 0 or tot(b) == LB))

    def kept_ket(c, d):
        # pure_ket: the same on the ket shells
        return not pure_ket or ((LC == 0 or tot(c) == LC) and (LD == 0 or tot(d) == LD))

    outs = [hk(a, b, c, d) if kept(a, b) and kept_ket(c, d) else None
            for a in comps(LA) for b in comps(LB) for c in comps(LC) for d in comps(LD)]
    level = {}
    for k in order:   # 'order' is a valid topological order (post-order)
        lv = 0
        for sk in nodes[k][4]:
            if sk is not None and sk[0] != 'F':
                lv = max(lv, level[sk] + 1)
        level[k] = lv
    sorted_keys = sorted(order, key=lambda k: level[k])
    slot = {('F', m): 1 + m for m in range(L + 1)}
    base = L + 2
    nlev = (max(level.values()) + 1) if level else 0
    if compact:
        last = {k: -1 for k in sorted_keys}   # level of the last reader of each node
        for k in sorted_keys:
            for sk in nodes[k][4]:
                if sk is not None and sk[0] != 'F':
                    last[sk] = max(last[sk], level[k])
        for o in outs:
            if o is not None and o[0] != 'F':
                last[o] = nlev   # read after the last level
        free, used, release = [], 0, {}
        for k in sorted_keys:   # level by level
            lv = level[k]
            for r in release.pop(lv, []):
                free.append(r)
            if free:
                sl = free.pop()
            else:
                sl = base + used
                used += 1
            slot[k] = sl
            release.setdefault(max(last[k], lv) + 1, []).append(sl)
        nslots = base + used
    else:
        for n, k in enumerate(sorted_keys):
            slot[k] = base + n
        nslots = base + len(sorted_keys)
    ops = []
    for k in sorted_keys:
        kind, ax, cA, cB, srcs = nodes[k]
        ops.append([(kind << 12) | (ax << 10) | (cA << 5) | cB] + [slot[sk] if sk is not None else 0 for sk in srcs]
                   + [slot[k]])
    lev_start = [0] * (nlev + 1)
    for k in sorted_keys:
        lev_start[level[k] + 1] += 1
    for i in range(nlev):
        lev_start[i + 1] += lev_start[i]
    out_slots = [slot[o] if o is not None else 0 for o in outs]
    assert nslots < 32768   # slot indices share 15 bits with other fields in the wide kernel's output list
    return ops, lev_start, out_slots, nslots


def pure_ket_gains(LA, LB, LC, LD):
    """Whether dropping the ket's lower components too saves ops over the
    pure-bra table (not where the ket's top outputs need them all anyway)."""
    return (len(gen_optable(LA, LB, LC, LD, True, True)[0]) <
            len(gen_optable(LA, LB, LC, LD, True, False)[0]))


def emit_optable(LA, LB, LC, LD, pure_bra=False, pure_ket=False, name=None):
    ops, lev, outs, nslots = gen_optable(LA, LB, LC, LD, pure_bra, pure_ket)
    name = name or 'op_%d%d%d%d%s' % (LA, LB, LC, LD, '_pure2' if pure_ket else ('_pure' if pure_bra else ''))
    lines = ['// (%d%d|%d%d): %d ops in %d levels, %d slots' % (LA, LB, LC, LD, len(ops), len(lev) - 1, nslots)]
    flat = [v for op in ops for v in op] or [0] * 7
    lines.append('static const unsigned short %s_ops[%d] = {%s};' % (name, len(flat), ','.join(map(str, flat))))
    lines.append('static const int %s_levels[%d] = {%s};' % (name, len(lev), ','.join(map(str, lev))))
    lines.append('static const unsigned short %s_out[%d] = {%s};' % (name, len(outs), ','.join(map(str, outs))))
    lines.append('static const OpTableHost %s = {%s_ops, %d, %s_levels, %d, %s_out, %d, %d};' % (
        name, name, len(ops), name, len(lev) - 1, name, len(outs), nslots))
    return '\n'.join(lines)


def used_params(lines):
    txt = '\n'.join(lines)
    return {p: (p in txt) for p in ('PA0', 'PA1', 'PA2', 'WP0', 'WP1', 'WP2', 'QC0', 'QC1', 'QC2',
                                    'WQ0', 'WQ1', 'WQ2', 'AB0', 'AB1', 'AB2', 'CD0', 'CD1', 'CD2',
                                    'oz', 'oe', 'oze', 'roz', 'roe')}


def gen_class(LA, LB, LC, LD):
    g = Gen(LA, LB, LC, LD)
    outs = g.build()
    n = len(outs)
    name = 'eri_%d%d%d%d' % (LA, LB, LC, LD)
    body = []
    body.append('// (%d%d|%d%d) cumulative: %d integrals, %d recursion flops' % (LA, LB, LC, LD, n, g.flops))
    body.append('template <typename R>')
    body.append('__device__ __forceinline__ void %s(const R* __restrict__ F, const EriGeom<R>& g, R* __restrict__ out) {' % name)
    u = used_params(g.lines + outs)
    for p in ('PA', 'WP', 'QC', 'WQ', 'AB', 'CD'):
        for k in range(3):
            if u['%s%d' % (p, k)]:
                body.append('    const R %s%d = g.%s[%d];' % (p, k, p, k))
    for p in ('oz', 'oe', 'oze', 'roz', 'roe'):
        if u[p]:
            body.append('    const R %s = g.%s;' % (p, p))
    body.extend(g.lines)
    for k, o in enumerate(outs):
        body.append('    out[%d] = %s;' % (k, o))
    body.append('}')
    return '\n'.join(body), n, g.flops


def pass_work(LA, LB, LC, LD, npass, pure_bra=False):
    """Recursion flops per primitive quartet that the straight-line kernel of a
    class executes when its outputs are held in `npass` register passes.

    Each pass evaluates only the ops its kept outputs depend on (the rest is dead
    code in that pass), so the work is the sum over passes of those ops.  The
    passes split the bra pairs ab, ordered by (|a|, |b|), into slices of
    ceil(NAB / npass); two-pass (d s| classes split at the level boundary instead
    (k_gq's AB0/AB1).  With `pure_bra` (both bra shells pure: their lower
    components carry no coefficient), passes whose pairs all include a lower
    component skip their work, as k_gq's passes skip their chunks.
    Returns (flops of one full evaluation, flops summed over the executed
    passes, number of executed passes)."""
    g = Gen(LA, LB, LC, LD)
    cost = {}
    emit = g.emit

    def counting_emit(expr, flops):
        name = emit(expr, flops)
        cost[name] = flops
        return name

    g.emit = counting_emit
    outs = g.build()
    deps = {}
    for line in g.lines:
        lhs, rhs = line.split('=', 1)
        deps[lhs.split()[-1]] = re.findall(r'\bt\d+\b', rhs)
    ca, cb, cc, cd = comps(LA), comps(LB), comps(LC), comps(LD)
    nab, ncd = len(ca) * len(cb), len(cc) * len(cd)
    key = [tot(ca[k // len(cb)]) * 8 + tot(cb[k % len(cb)]) for k in range(nab)]
    order = sorted(range(nab), key=lambda k: key[k])   # stable, as AbOrder
    lower = [tot(ca[k // len(cb)]) < LA or tot(cb[k % len(cb)]) < LB for k in range(nab)]
    nlow = sum(lower)
    abp = -(-nab // npass)
    split = npass == 2 and LA == 2 and LB == 0 and nlow * ncd <= 40 and (nab - nlow) * ncd <= 40
    total, executed = 0, 0
    for ps in range(npass):
        a0 = (0 if ps == 0 else nlow) if split else ps * abp
        a1 = (nlow if ps == 0 else nab) if split else min(a0 + abp, nab)
        kept = order[a0:a1]
        if pure_bra and (LA > 0 or LB > 0) and all(lower[k] for k in kept):
            continue
        need, stack = set(), [t for k in kept for i in range(ncd) for t in re.findall(r'\bt\d+\b', outs[k * ncd + i])]
        while stack:
            t = stack.pop()
            if t not in need:
                need.add(t)
                stack.extend(deps[t])
        total += sum(cost[t] for t in need)
        executed += 1
    return g.flops, total, executed


HEADER = '''// Generated by polymer_b200/csrc/gen_eri.py -- do not edit.
// Class-specialised (LA LB|LC LD) electron-repulsion integrals over cumulative
// primitive shells; see the generator for the recursions.
#pragma once

// F1(0) = 1/(2/sqrt(PI)) with the reference's PI = 3.14159265358979
// (src/pfourindexdirect.f90:75-77), as an exactly round-tripping literal.
#define PFE_F1_0 %r
''' % (1.0 / (2.0 / math.sqrt(3.14159265358979)))
HEADER += '''
template <typename R>
struct EriGeom {
  R PA[3], WP[3], QC[3], WQ[3], AB[3], CD[3];
  R oz, oe, oze, roz, roe;   // 1/(2z), 1/(2h), 1/(2(z+h)), rho/z, rho/h
};

'''


GRAD_HEADER = '''// Generated by polymer_b200/csrc/gen_eri.py -- do not edit.
// Op tables of the derivative integrals: class (LA LB|LC LD) with centre A, C
// or D raised by one (cumulative), opg_<LA><LB><LC><LD>_<centre>.
#pragma once
#include "eri_classes.cuh"
'''


def main():
    out = sys.argv[1]
    lmax = int(sys.argv[2]) if len(sys.argv) > 2 else 2
    both = len(sys.argv) > 3 and sys.argv[3] == 'all'
    pieces = [HEADER]
    table = {}
    classes = [(la, lb) for la in range(lmax + 1) for lb in range(la + 1)]
    big = []
    for ib, (LA, LB) in enumerate(classes):
        for ik, (LC, LD) in enumerate(classes):
            if ik > ib and not both:
                continue   # the kernels put the higher pair class on the bra side
            n = ncomp_class = (len(comps(LA)) * len(comps(LB)) * len(comps(LC)) * len(comps(LD)))
            big.append(emit_optable(LA, LB, LC, LD))   # every class can run interpreted
            if LA >= 1:
                big.append(emit_optable(LA, LB, LC, LD, pure_bra=True))
            if LA >= 1 and LC >= 1 and pure_ket_gains(LA, LB, LC, LD):
                big.append(emit_optable(LA, LB, LC, LD, pure_bra=True, pure_ket=True))
            if n > OPS_THRESHOLD:
                g = Gen(LA, LB, LC, LD)
                g.build()
                table['%d%d%d%d' % (LA, LB, LC, LD)] = {'integrals': n, 'recursion_flops': g.flops, 'interpreted': True}
                continue
            code, n, fl = gen_class(LA, LB, LC, LD)
            pieces.append(code + '\n')
            table['%d%d%d%d' % (LA, LB, LC, LD)] = {'integrals': n, 'recursion_flops': fl}
    # op tables of the interpreted classes (host data, uploaded at set-up)
    pieces.append('struct OpTableHost { const unsigned short* ops; int nops; const int* levels; int nlevels;'
                  ' const unsigned short* out; int nout; int nslots; };')
    pieces.extend(big)
    # compile-time dispatch on the class and the per-class flop table
    pieces.append('template <int LA, int LB, int LC, int LD> struct EriFn;')
    for key in sorted(table):
        if table[key].get('interpreted'):
            continue
        la, lb, lc, ld = (int(ch) for ch in key)
        pieces.append('template <> struct EriFn<%d, %d, %d, %d> {\n  template <typename R>\n'
                      '  static __device__ __forceinline__ void run(const R* F, const EriGeom<R>& g, R* out) '
                      '{ eri_%s<R>(F, g, out); }\n};' % (la, lb, lc, ld, key))
    pieces.append('template <int LA, int LB, int LC, int LD, typename R>\n'
                  '__device__ __forceinline__ void eri_dispatch(const R* F, const EriGeom<R>& g, R* out) {\n'
                  '  EriFn<LA, LB, LC, LD>::template run<R>(F, g, out);\n}\n')
    pieces.append('// recursion flops per class (FMA = 2), indexed [la][lb][lc][ld]')
    pieces.append('static inline double eri_recursion_flops(int la, int lb, int lc, int ld) {')
    pieces.append('  switch (((la * 3 + lb) * 3 + lc) * 3 + ld) {')
    for key in sorted(table):
        la, lb, lc, ld = (int(ch) for ch in key)
        pieces.append('    case %d: return %d.0;' % (((la * 3 + lb) * 3 + lc) * 3 + ld, table[key]['recursion_flops']))
    pieces.append('    default: return 0.0;\n  }\n}\n')
    with open(out, 'w') as fh:
        fh.write('\n'.join(pieces))
    # gradient tables: every class with one centre raised by one (A, C or D; B by
    # translational invariance), for the derivative integrals of
    # FOURINDEX_ERI_GRADIENT; a header of their own, read by the gradient unit only
    grad = [GRAD_HEADER]
    for LA, LB in classes:
        for LC, LD in classes:
            if (LC, LD) > (LA, LB) or classes.index((LC, LD)) > classes.index((LA, LB)):
                continue
            for c, cls in (('a', (LA + 1, LB, LC, LD)), ('c', (LA, LB, LC + 1, LD)), ('d', (LA, LB, LC, LD + 1))):
                grad.append(emit_optable(*cls, name='opg_%d%d%d%d_%s' % (LA, LB, LC, LD, c)))
    with open(out.replace('eri_classes.cuh', 'eri_grad_tables.cuh'), 'w') as fh:
        fh.write('\n'.join(grad) + '\n')
    with open(out.replace('.cuh', '_flops.json'), 'w') as fh:
        json.dump(table, fh, indent=1, sort_keys=True)


if __name__ == '__main__':
    main()
