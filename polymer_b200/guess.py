"""Learned initial guess for water clusters (no counterpart in the reference,
whose guess is the nuclear-charge diagonal, src/pdensitymatrix.f90:83-127).

An MLP (polymer_b200/mlp.py: the library's BF16 tensor-core kernels) predicts
the blocks P_AB of the contracted density between atoms A and B, each in the
frame of the water that owns A (origin O, e1 along the H-O-H bisector, e2
along H1 - H2), from frame-fixed features of the pair and of A's neighbours.
Frame blocks are rotated to the laboratory with the exact transformation of
Cartesian Gaussians (so predictions are rotation-covariant), assembled
(symmetrised), and purified in FP64: McWeeny iterations in the orthonormal
(LINDEP) basis, then the occupied natural orbitals.  Training data are
converged densities of the GPU SCF over seeded water clusters.
"""
from __future__ import annotations

import dataclasses
import itertools
import math
import os
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from .system import System

NEIGHBOURS = 10      # nearest atoms of A used as features
MAXF = 15            # functions per atom (O in cc-pVDZ: 3s 2p 1d Cartesian = 15)
R_CUT = 8.0          # bohr: inter-monomer blocks predicted below this A-B distance
NFEAT = 9 + 6 * NEIGHBOURS   # pair (types 4, frame offset 3, distance, same water) + neighbours


def _dfact(n: int) -> int:
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def _norm(pw) -> float:
    return 1.0 / math.sqrt(_dfact(2 * pw[0] - 1) * _dfact(2 * pw[1] - 1) * _dfact(2 * pw[2] - 1))


def _monomials(L: int):
    return [(i, j, L - i - j) for i in range(L, -1, -1) for j in range(L - i, -1, -1)]


def monomial_transforms(L: int, Rs: np.ndarray) -> Tuple[list, np.ndarray]:
    """Q[w] with m_i(R_w u) = sum_j Q[w]_ij m_j(u) for the degree-L monomials, for
    a stack of rotations Rs (nw x 3 x 3): m_i(R u) is the product of the L linear
    forms (R u)_r, one per power of monomial i, and its expansion's term
    u_j1 ... u_jL adds prod_k R[r_k, j_k] to the monomial with those powers."""
    pws = _monomials(L)
    pos = {pw: k for k, pw in enumerate(pws)}
    nw = Rs.shape[0]
    # the monomial of every index tuple (j1..jL), as a 0/1 matrix (3^L x nm)
    fold = np.zeros((3 ** L, len(pws)))
    for t, js in enumerate(itertools.product(range(3), repeat=L)):
        fold[t, pos[(js.count(0), js.count(1), js.count(2))]] = 1.0
    q = np.empty((nw, len(pws), len(pws)))
    for i, pw in enumerate(pws):
        rows = [0] * pw[0] + [1] * pw[1] + [2] * pw[2]
        t = np.ones((nw, 1))
        for r in rows:   # outer product with the next linear form, j_k varying fastest last
            t = (t[:, :, None] * Rs[:, r, None, :]).reshape(nw, -1)
        q[:, i, :] = t @ fold
    return pws, q


def monomial_transform(L: int, R: np.ndarray) -> Tuple[list, np.ndarray]:
    """Q with m_i(R u) = sum_j Q_ij m_j(u) for the degree-L monomials."""
    pws, q = monomial_transforms(L, R[None])
    return pws, q[0]


@dataclasses.dataclass
class AOInfo:
    live: np.ndarray         # (ncgs,) bool: row of CC not all zero
    atom: np.ndarray         # (ncgs,) 0-based atom
    powers: List[tuple]      # Cartesian powers of each contracted function
    groups: List[List[int]]  # contracted functions of one shell instance (same atom, L, radial part)
    atom_funcs: List[List[int]]


def _round10(v: np.ndarray) -> np.ndarray:
    """Python's round(x, 10) of every element (applied once per distinct value)."""
    u, inv = np.unique(v, return_inverse=True)
    return np.array([round(float(x), 10) for x in u])[inv.reshape(-1)] if len(u) else v.copy()


def ao_info(sysm: System) -> AOInfo:
    """Per contracted function: live (a row of CC not all zero), atom and
    Cartesian powers of its largest primitive; functions of one shell instance
    share (atom, L, radial part), the radial part being the sorted (exponent,
    coefficient / norm) pairs rounded to 10 digits.  Groups come in the order of
    their first function."""
    b = sysm.basis
    n = b.ncgs
    cc = np.asarray(b.cc)
    live = np.any(cc != 0.0, axis=1)
    p0 = np.argmax(np.abs(cc), axis=1)
    pw = np.stack([np.asarray(b.pax)[p0], np.asarray(b.pay)[p0], np.asarray(b.paz)[p0]], axis=1).astype(int)
    pw[~live] = 0
    atom = np.where(live, np.asarray(b.pgs_atom)[p0].astype(int) - 1, 0)
    powers: List[tuple] = list(map(tuple, pw.tolist()))
    li = np.nonzero(live)[0]
    groups: List[List[int]] = []
    if len(li):
        # _norm of every row's powers: the double factorials are exact integers
        df = np.array([_dfact(2 * k - 1) for k in range(int(pw.max()) + 1)], dtype=float)
        pl = pw[li]
        norms = 1.0 / np.sqrt(df[pl[:, 0]] * df[pl[:, 1]] * df[pl[:, 2]])
        sub = cc[li]
        r, c = np.nonzero(sub != 0.0)
        zr = _round10(np.asarray(b.zt, dtype=float)[c])
        cr = _round10(sub[r, c] / norms[r])
        o = np.lexsort((cr, zr, r))   # per row, pairs sorted by (exponent, coefficient)
        r, zr, cr = r[o], zr[o], cr[o]
        cnt = np.bincount(r, minlength=len(li))
        slot = np.arange(len(r)) - (np.cumsum(cnt) - cnt)[r]
        key = np.full((len(li), 2 + 2 * int(cnt.max())), np.inf)
        key[:, 0] = atom[li]
        key[:, 1] = pw[li].sum(axis=1)
        key[r, 2 + 2 * slot] = zr
        key[r, 3 + 2 * slot] = cr
        _, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        first = np.full(inv.max() + 1, len(li))
        np.minimum.at(first, inv, np.arange(len(li)))
        for g in np.argsort(first, kind='stable'):
            groups.append(li[inv == g].tolist())
    natom = sysm.deck.natom
    atom_funcs = [np.nonzero(live & (atom == a))[0].tolist() for a in range(natom)]
    return AOInfo(live, atom, powers, groups, atom_funcs)


def frame_transform(info: AOInfo, R: np.ndarray, funcs: List[int], qcache: Optional[dict] = None) -> np.ndarray:
    """U (len(funcs) x len(funcs)) with P_frame = U^T P_lab U for the functions
    `funcs` (whole shell instances), R mapping frame vectors to lab vectors;
    `qcache` keeps the monomial transforms of R per degree across calls."""
    idx = {f: k for k, f in enumerate(funcs)}
    u = np.zeros((len(funcs), len(funcs)))
    cache = qcache if qcache is not None else {}
    for g in info.groups:
        if g[0] not in idx:
            continue
        L = sum(info.powers[g[0]])
        if L not in cache:
            cache[L] = monomial_transform(L, R)
        pws, q = cache[L]
        pos = {pw: k for k, pw in enumerate(pws)}
        for i in g:
            for j in g:
                pi, pj = info.powers[i], info.powers[j]
                u[idx[i], idx[j]] = _norm(pi) * q[pos[pi], pos[pj]] / _norm(pj)
    return u


def water_frames(sysm: System) -> List[Tuple[np.ndarray, np.ndarray, List[int]]]:
    """(origin, R, atoms) of every water: atoms come as O, H, H in the deck; the
    frame's e1 bisects the two O-H bonds, e2 lies in the molecular plane."""
    d = sysm.deck
    nw = d.natom // 3
    xyz = np.array(d.coords, dtype=float)[:3 * nw].reshape(nw, 3, 3)
    o = xyz[:, 0]
    a, c = xyz[:, 1] - o, xyz[:, 2] - o
    e1 = (a + c) / np.linalg.norm(a + c, axis=1, keepdims=True)
    e2 = (a - c) - np.sum((a - c) * e1, axis=1, keepdims=True) * e1
    e2 /= np.linalg.norm(e2, axis=1, keepdims=True)
    e3 = np.cross(e1, e2)
    R = np.stack([e1, e2, e3], axis=2)
    return [(o[m], R[m], [3 * m, 3 * m + 1, 3 * m + 2]) for m in range(nw)]


def _type(z: int) -> np.ndarray:
    return np.array([1.0, 0.0]) if z == 8 else np.array([0.0, 1.0])


def pair_list(sysm: System):
    """(A, B, owner water) of every predicted block: all pairs inside a water and
    pairs closer than R_CUT, each in the frame of A's water (A outer, B inner)."""
    d = sysm.deck
    xyz = np.array(d.coords)
    w = np.arange(d.natom) // 3
    dist = np.linalg.norm(xyz[:, None, :] - xyz[None, :, :], axis=2)
    a, b = np.nonzero((w[:, None] == w[None, :]) | (dist < R_CUT))
    return [(int(i), int(j), int(i) // 3) for i, j in zip(a, b)]


def features(sysm: System, frames, pairs) -> np.ndarray:
    """Per pair (A, B): the types of A and B, B - A in the frame (/4 bohr), its
    length, same-water flag, then the NEIGHBOURS atoms nearest A (other than A
    and B), each as type, offset from A in the frame (/8 bohr) and inverse
    distance; missing neighbours are zero."""
    d = sysm.deck
    xyz = np.array(d.coords)
    z = np.array(d.atoms)
    npair = len(pairs)
    out = np.zeros((npair, NFEAT))
    if npair == 0:
        return out
    A = np.array([q[0] for q in pairs])
    B = np.array([q[1] for q in pairs])
    R = np.stack([fr[1] for fr in frames])[np.array([q[2] for q in pairs])]
    typ = np.where((z == 8)[:, None], np.array([1.0, 0.0]), np.array([0.0, 1.0]))
    rel = np.einsum('pji,pj->pi', R, xyz[B] - xyz[A])
    out[:, 0:2] = typ[A]
    out[:, 2:4] = typ[B]
    out[:, 4:7] = rel / 4.0
    out[:, 7] = np.linalg.norm(rel, axis=1) / 4.0
    out[:, 8] = (A // 3 == B // 3)
    # neighbours of A by distance (each row sorted on its own, as np.argsort of that row)
    order = np.argsort(np.linalg.norm(xyz[:, None, :] - xyz[None, :, :], axis=2), axis=1)[A]
    keep = (order != A[:, None]) & (order != B[:, None])
    pos = np.argsort(~keep, axis=1, kind='stable')[:, :NEIGHBOURS]
    sel = np.take_along_axis(order, pos, 1)
    ok = np.take_along_axis(keep, pos, 1)
    rc = np.einsum('pji,pcj->pci', R, xyz[sel] - xyz[A][:, None, :])
    env = np.concatenate([typ[sel], rc / 8.0, (1.0 / np.maximum(np.linalg.norm(rc, axis=2), 1e-6))[..., None]], axis=2)
    env *= ok[..., None]
    out[:, 9:9 + 6 * sel.shape[1]] = env.reshape(npair, -1)
    return out


def _layout(info: AOInfo, a: int, cache: dict):
    """Atom a's functions as (shell instances by relative index, powers): atoms
    with equal layouts share their frame transforms."""
    key = ('layout', a)
    if key not in cache:
        funcs = info.atom_funcs[a]
        idx = {f: k for k, f in enumerate(funcs)}
        cache[key] = (tuple(tuple(idx[i] for i in g) for g in info.groups if g[0] in idx),
                      tuple(info.powers[f] for f in funcs))
    return cache[key]


def _layout_plan(info: AOInfo, a: int, cache: dict):
    """Atom a's layout and its frame transform as entries per degree L: (row,
    column, monomial row, monomial column, norm ratio) arrays, so that
    U[row, col] = Q_L[mrow, mcol] * ratio, as frame_transform fills it."""
    lay = _layout(info, a, cache)
    key = ('plan', lay)
    if key not in cache:
        groups, pws = lay
        plan: Dict[int, tuple] = {}
        for g in groups:
            L = sum(pws[g[0]])
            pos = {pw: k for k, pw in enumerate(_monomials(L))}
            e = plan.setdefault(L, ([], [], [], [], []))
            for i in g:
                for j in g:
                    e[0].append(i)
                    e[1].append(j)
                    e[2].append(pos[pws[i]])
                    e[3].append(pos[pws[j]])
                    e[4].append(_norm(pws[i]) / _norm(pws[j]))
        cache[key] = (len(pws), {L: tuple(np.array(x) for x in e) for L, e in plan.items()})
    return lay, cache[key]


def frame_transforms(info: AOInfo, frames, natom: int, cache: dict) -> dict:
    """Per atom layout: U of every water's frame (nwater x nf x nf), P_frame =
    U^T P_lab U, the monomial transforms of all frames computed at once per degree."""
    Rs = np.stack([fr[1] for fr in frames]) if frames else np.zeros((0, 3, 3))
    q: Dict[int, np.ndarray] = {}
    out: dict = {}
    for a in range(natom):
        lay, (nf, plan) = _layout_plan(info, a, cache)
        if lay in out or nf == 0:
            continue
        u = np.zeros((len(Rs), nf, nf))
        for L, (ui, uj, mi, mj, ratio) in plan.items():
            if L not in q:
                q[L] = monomial_transforms(L, Rs)[1]
            u[:, ui, uj] = q[L][:, mi, mj] * ratio
        out[lay] = u
    return out


def frame_inverses(info: AOInfo, frames, natom: int, cache: dict) -> dict:
    """Per atom layout: V = U^-1 of every water's frame (nwater x nf x nf)."""
    return {lay: np.linalg.inv(u) for lay, u in frame_transforms(info, frames, natom, cache).items()}


def _pair_groups(info: AOInfo, pairs, natom: int, cache: dict):
    """The pairs grouped by the layouts of their two atoms (first-appearance
    order): per group the pair indices, both layouts, the owner waters and the
    function indices of A (rows) and of B (columns)."""
    lays = [_layout(info, a, cache) for a in range(natom)]
    lay_id = {lay: k for k, lay in enumerate(dict.fromkeys(lays))}
    atom_lay = np.array([lay_id[lay] for lay in lays])
    by_id = {k: lay for lay, k in lay_id.items()}
    maxf = max(1, max(len(f) for f in info.atom_funcs))
    funcs = np.zeros((natom, maxf), dtype=np.int64)
    for a, f in enumerate(info.atom_funcs):
        funcs[a, :len(f)] = f
    P = np.asarray(pairs)
    A, B, M = P[:, 0], P[:, 1], P[:, 2]
    combo = atom_lay[A] * len(lay_id) + atom_lay[B]
    for cb in dict.fromkeys(combo.tolist()):
        ks = np.nonzero(combo == cb)[0]
        la, lb = by_id[cb // len(lay_id)], by_id[cb % len(lay_id)]
        na, nb = len(la[1]), len(lb[1])
        if na == 0 or nb == 0:
            continue
        yield ks, la, lb, M[ks], funcs[A[ks], :na], funcs[B[ks], :nb]


def targets(sysm: System, info: AOInfo, frames, pairs, p_c: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Frame blocks of a converged contracted density, flattened to MAXF x MAXF, and their weights."""
    t = np.zeros((len(pairs), MAXF, MAXF))
    w = np.zeros_like(t)
    if pairs:
        cache: dict = {}
        u = frame_transforms(info, frames, sysm.deck.natom, cache)
        for ks, la, lb, m, r, c in _pair_groups(info, pairs, sysm.deck.natom, cache):
            blk = p_c[r[:, :, None], c[:, None, :]]
            t[ks, :r.shape[1], :c.shape[1]] = u[la][m].transpose(0, 2, 1) @ blk @ u[lb][m]
            w[ks, :r.shape[1], :c.shape[1]] = 1.0
    return t.reshape(len(pairs), -1), w.reshape(len(pairs), -1)


def assemble(sysm: System, info: AOInfo, frames, pairs, pred: np.ndarray) -> np.ndarray:
    """Laboratory contracted density from predicted frame blocks (symmetrised:
    each block enters at (A,B) and, transposed, at (B,A); entries are averaged)."""
    n = sysm.basis.ncgs
    if not pairs:
        return np.zeros((n, n))
    natom = sysm.deck.natom
    cache: dict = {}
    vinv = frame_inverses(info, frames, natom, cache)
    idx, val = [], []
    for ks, la, lb, m, r, c in _pair_groups(info, pairs, natom, cache):
        blk = pred[ks].reshape(-1, MAXF, MAXF)[:, :r.shape[1], :c.shape[1]]
        lab = vinv[la][m].transpose(0, 2, 1) @ (blk @ vinv[lb][m])
        idx.append((r[:, :, None] * n + c[:, None, :]).ravel())
        val.append(lab.ravel())
        idx.append((c[:, None, :] * n + r[:, :, None]).ravel())   # the transpose: (B,A) gets lab[k].T
        val.append(lab.ravel())
    if not idx:
        return np.zeros((n, n))
    idx = np.concatenate(idx)
    acc = np.bincount(idx, weights=np.concatenate(val), minlength=n * n).reshape(n, n)
    cnt = np.bincount(idx, minlength=n * n).reshape(n, n)
    return np.where(cnt > 0, acc / np.maximum(cnt, 1), 0.0)


def purify(st, p_c: torch.Tensor, nocc: int, mcweeny: int = 3) -> torch.Tensor:
    """FP64: D = P/2 in the orthonormal (LINDEP) basis, McWeeny D <- 3D^2 - 2D^3,
    then the projector on its nocc leading natural orbitals; returns P_C."""
    d = st.sys.deck
    c2s, s0 = st.c2s, st.s_c[0]
    e_s, v_s = torch.linalg.eigh(c2s @ s0 @ c2s.T)
    keep = e_s > d.lindep
    w = c2s.T @ (v_s[:, keep] / torch.sqrt(e_s[keep]))
    ws = w.T @ s0
    dm = 0.5 * ws @ p_c @ ws.T
    for _ in range(mcweeny):
        d2 = dm @ dm
        dm = 3.0 * d2 - 2.0 * d2 @ dm
    ev, vec = torch.linalg.eigh(0.5 * (dm + dm.T))
    occ = vec[:, -nocc:]
    co = w @ occ
    return 2.0 * co @ co.T


# ---------------------------------------------------------------- training and use

HIDDEN = (256, 256, 256)


def sample_cluster(k: int, seed: int):
    """A seeded water cluster (cc-pVDZ deck) as used for training and testing."""
    from . import geometry
    return geometry.water_deck(k, seed=seed, basis='cc-pVDZ', inttol=1e-12)


def cluster_data(sysm: System, p_c: Optional[np.ndarray] = None):
    info = ao_info(sysm)
    frames = water_frames(sysm)
    pairs = pair_list(sysm)
    x = features(sysm, frames, pairs)
    if p_c is None:
        return info, frames, pairs, x
    t, w = targets(sysm, info, frames, pairs, p_c)
    return info, frames, pairs, x, t, w


def generate(sizes, seeds, device='cuda', log=None):
    """Converged densities of the GPU SCF for clusters (k, seed): features,
    frame-block targets and weights, concatenated."""
    from . import fock, scf, system
    xs, ts, ws = [], [], []
    for k, seed in zip(sizes, seeds):
        s = system.build_system(sample_cluster(k, seed), fock.onee)
        df = fock.DeviceFock(s)
        r = scf.run_scf_fast(s, df, opts=scf.FastOptions(incremental=False), device=device)
        df.close()
        _, _, _, x, t, w = cluster_data(s, r.p_c[0].cpu().numpy())
        xs.append(x)
        ts.append(t)
        ws.append(w)
        if log:
            log('cluster k=%d seed=%d: %d iterations, %d blocks' % (k, seed, len(r.iterations), len(x)))
    return np.concatenate(xs), np.concatenate(ts), np.concatenate(ws)


def generate_batched(sizes, seeds, batch: int = 128, device: int = 0, log=None):
    """generate() with the batched SCF: clusters converged `batch` at a time
    (nuclear-charge guess, each iteration a CUDA graph replay)."""
    from . import batch_scf, fock, system
    xs, ts, ws = [], [], []
    jobs = list(zip(sizes, seeds))
    for b0 in range(0, len(jobs), batch):
        part = jobs[b0:b0 + batch]
        systems = [system.build_system(sample_cluster(k, seed), fock.onee) for k, seed in part]
        res = batch_scf.run_batch_scf(systems, batch_scf.BatchOptions(), device=device, graph=True)
        for s, p_c in zip(systems, res.p_c):
            _, _, _, x, t, w = cluster_data(s, p_c.cpu().numpy())
            xs.append(x)
            ts.append(t)
            ws.append(w)
        if log:
            log('clusters %d..%d: %d builds, mean %.1f iterations, %d blocks so far'
                % (b0, b0 + len(part) - 1, res.builds, float(res.iterations.mean()), sum(len(x) for x in xs)))
    return np.concatenate(xs), np.concatenate(ts), np.concatenate(ws)


class LearnedGuess:
    """The trained network as an initial-guess callable of scf.FastOptions."""

    def __init__(self, net=None, device='cuda'):
        from .mlp import MLP
        self.device = torch.device(device)
        self.net = net or MLP(NFEAT, HIDDEN, MAXF * MAXF, device=device)

    def train(self, x, t, w, steps=2000, batch=512, lr=2e-3, log=None, seed=0):
        rng = np.random.default_rng(seed)
        xt = torch.tensor(x, dtype=torch.float32)
        tt = torch.tensor(t, dtype=torch.float32)
        wt = torch.tensor(w, dtype=torch.float32)
        n = len(x)
        losses = []
        for step in range(steps):
            idx = torch.tensor(rng.integers(0, n, size=min(batch, n)))
            lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))
            loss, gW, gb = self.net.loss_and_grads(xt[idx], tt[idx], wt[idx])
            self.net.adam_step(gW, gb, lr=lr_t)
            losses.append(loss)
            if log and (step % 200 == 0 or step == steps - 1):
                log('step %d loss %.3e' % (step, loss))
        return losses

    def predict_blocks(self, x: np.ndarray) -> np.ndarray:
        out = []
        for i in range(0, len(x), 16384):
            out.append(self.net.forward(torch.tensor(x[i:i + 16384], dtype=torch.float32)).double())
        return torch.cat(out).cpu().numpy()

    def raw(self, sysm: System) -> np.ndarray:
        """The assembled (unpurified) contracted density of the prediction."""
        info, frames, pairs, x = cluster_data(sysm)
        return assemble(sysm, info, frames, pairs, self.predict_blocks(x))

    def raw_many(self, systems) -> List[np.ndarray]:
        """raw() of several molecules with one network evaluation over all their blocks."""
        data = [cluster_data(s) for s in systems]
        pred = self.predict_blocks(np.concatenate([d[3] for d in data]))
        out, o = [], 0
        for s, (info, frames, pairs, x) in zip(systems, data):
            out.append(assemble(s, info, frames, pairs, pred[o:o + len(pairs)]))
            o += len(pairs)
        return out

    def __call__(self, sysm: System, st) -> torch.Tensor:
        info, frames, pairs, x = cluster_data(sysm)
        p = assemble(sysm, info, frames, pairs, self.predict_blocks(x))
        pc = purify(st, torch.tensor(p, dtype=torch.float64, device=st.device), sysm.deck.nelectrons // 2)
        return pc.unsqueeze(0)

    def save(self, path: str) -> None:
        st = self.net.state()
        st['W'] = [w.to(torch.bfloat16) for w in st['W']]   # the weights the GEMMs use
        torch.save(st, path)

    @classmethod
    def load(cls, path: str, device='cuda') -> 'LearnedGuess':
        from .mlp import MLP
        st = torch.load(path, map_location='cpu')
        g = cls(MLP(st['din'], HIDDEN, st['dout'], device=device), device=device)
        st['W'] = [w.float() for w in st['W']]
        g.net.load(st)
        return g


MODEL = os.path.join(os.path.dirname(__file__), 'data', 'guess_water_ccpvdz.pt')


TRAIN_CLUSTERS = 768


def train_default(path: str = MODEL, log=print, n: int = TRAIN_CLUSTERS) -> 'LearnedGuess':
    """The committed network: `n` clusters, k ~ U{1..16} from default_rng(4999),
    cluster i from seed 5000+i (disjoint from the benchmark's seeds 2001..),
    converged by the batched GPU SCF; 8000 Adam steps of 2048 blocks (cosine
    learning rate from 2e-3)."""
    sizes = [int(k) for k in np.random.default_rng(4999).integers(1, 17, size=n)]
    seeds = [5000 + i for i in range(n)]
    x, t, w = generate_batched(sizes, seeds, log=log)
    lg = LearnedGuess()
    lg.train(x, t, w, steps=8000, batch=2048, lr=2e-3, log=log)
    lg.save(path)
    return lg


if __name__ == '__main__':
    import sys
    train_default(sys.argv[1] if len(sys.argv) > 1 else MODEL)
