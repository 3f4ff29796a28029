"""Unit checks of the oracle against closed forms, independent of the
reference's recorded outputs (which pin it end to end through SCF energies):

* the Boys table IGAMMA(i, m) = F_m(i/20) of FMT_PRELIMINARY, from the oracle
  and from the host mirror, against F_m(T) = Gamma(m+1/2) P(m+1/2, T) /
  (2 T^(m+1/2)) (P the regularised lower incomplete gamma), F_m(0) = 1/(2m+1);
* C_C and X_C of an s-only basis (four centres, two uncontracted s primitives
  each, no screening) against J and K assembled from the closed-form primitive
  integrals (ab|cd) = 2 pi^(5/2) / (zeta eta sqrt(zeta+eta)) K_ab K_cd
  F_0(rho |P-Q|^2), contracted with CC as FOURINDEX_ERI does;
* the (p, s) blocks of C_C and X_C of a basis with a p shell, for a density
  on the s primitives, against the same closed form differentiated in the p
  primitive's centre (a complex step: exact to rounding);
* the (d, s) blocks likewise, from second derivatives of the closed form in
  the d primitive's centre (torch autograd in FP64).
"""
import numpy as np
from scipy.special import erf, gamma, gammainc

import oracle
from polymer_b200 import inputdeck, system


def _boys(m, t):
    t = np.asarray(t, dtype=float)
    out = np.full(t.shape, 1.0 / (2 * m + 1))
    pos = t > 0.0
    out[pos] = gamma(m + 0.5) * gammainc(m + 0.5, t[pos]) / (2.0 * t[pos] ** (m + 0.5))
    return out


def test_boys_table_matches_the_closed_form():
    t = np.arange(1701) / 20.0
    for tab in (oracle.fmt_table(), system.fmt_table()):
        tab = np.asarray(tab)
        assert tab.shape == (1701, 28)
        for m in range(28):
            ref = _boys(m, t)
            assert np.all(np.abs(tab[:, m] - ref) <= 1e-12 * ref), m


def test_s_only_fock_matches_closed_form_integrals():
    lib = {'H': [['S', 1.0, [[1.3, 1.0]]], ['S', 1.0, [[0.35, 1.0]]]]}
    xyz = [[0.0, 0.0, 0.0], [1.4, 0.2, 0.0], [0.3, 1.7, 0.5], [-1.1, 0.6, 1.2]]   # bohr
    deck = inputdeck.make_deck([1, 1, 1, 1], xyz, 'STO-3G', inttol=0.0)
    s = system.build_system(deck, oracle.onee, library=lib)
    b = s.basis
    assert not (np.any(b.pax) or np.any(b.pay) or np.any(b.paz))
    cc = b.cc
    rng = np.random.default_rng(7)
    a = rng.normal(size=(b.ncgs, b.ncgs))
    pp = cc.T @ (a + a.T) @ cc               # a decontracted density, as the reference's P_P
    c_c, x_c = oracle.fourindex_eri(s, pp[None])

    pos, z = b.pgs, b.zt
    zeta = z[:, None] + z[None, :]
    centre = (z[:, None, None] * pos[:, None, :] + z[None, :, None] * pos[None, :, :]) / zeta[..., None]
    kab = np.exp(-z[:, None] * z[None, :] / zeta * ((pos[:, None, :] - pos[None, :, :]) ** 2).sum(-1))
    zz = zeta[:, :, None, None] + zeta[None, None, :, :]
    rho = zeta[:, :, None, None] * zeta[None, None, :, :] / zz
    t = rho * ((centre[:, :, None, None, :] - centre[None, None, :, :, :]) ** 2).sum(-1)
    f0 = _f0(t)
    eri = (2.0 * np.pi ** 2.5 / (zeta[:, :, None, None] * zeta[None, None, :, :] * np.sqrt(zz))
           * kab[:, :, None, None] * kab[None, None, :, :] * f0)
    j_p = np.einsum('pqrs,rs->pq', eri, pp)          # C_P(i,j) += P_P(k,l) (ij|kl)
    k_p = np.einsum('pqrs,rq->ps', eri, pp)          # X_P(i,l) += P_P(k,j) (ij|kl)
    j_c, k_c = cc @ j_p @ cc.T, cc @ k_p @ cc.T
    assert np.abs(c_c[0] - j_c).max() <= 1e-12 * np.abs(j_c).max()
    assert np.abs(x_c[0] - k_c).max() <= 1e-12 * np.abs(k_c).max()


def _f0(t):
    """F_0(t) = sqrt(pi) erf(sqrt t) / (2 sqrt t), also for complex t: the ratio
    is even in sqrt(t), so it does not depend on the branch of the root."""
    r = np.sqrt(t)
    with np.errstate(divide='ignore', invalid='ignore'):
        f = 0.5 * np.sqrt(np.pi) * erf(r) / r
    return np.where(t == 0, 1.0, f)


def _ss_rows(pos, z, p):
    """(p q|r s) of s primitives for one bra primitive p and all q, r, s; pos may
    be complex (the closed form is analytic in the centres)."""
    zeta = z[:, None] + z[None, :]
    centre = (z[:, None, None] * pos[:, None, :] + z[None, :, None] * pos[None, :, :]) / zeta[..., None]
    kab = np.exp(-z[:, None] * z[None, :] / zeta * ((pos[:, None, :] - pos[None, :, :]) ** 2).sum(-1))
    zz = zeta[p][:, None, None] + zeta[None, :, :]
    rho = zeta[p][:, None, None] * zeta[None, :, :] / zz
    t = rho * ((centre[p][:, None, None, :] - centre[None, :, :, :]) ** 2).sum(-1)
    f0 = _f0(t)
    return 2.0 * np.pi ** 2.5 / (zeta[p][:, None, None] * zeta[None] * np.sqrt(zz)) * kab[p][:, None, None] * kab[None] * f0


def test_p_s_blocks_match_the_derivative_of_the_closed_form():
    # a p primitive (x - A_x) e^{-a|r-A|^2} is (1/2a) d/dA_x of the s primitive,
    # so with the density on s primitives only, the (p, s) blocks of J and K are
    # (1/2a) d/dA of s-only sums: taken by a complex step (exact to rounding)
    lib = {'H': [['S', 1.0, [[1.3, 1.0]]], ['S', 1.0, [[0.35, 1.0]]]],
           'He': [['S', 1.0, [[2.1, 1.0]]], ['P', 1.0, [[0.8, 1.0]]]]}
    xyz = [[0.0, 0.0, 0.0], [1.4, 0.2, 0.3], [0.3, 1.7, -0.5]]   # bohr
    s = system.build_system(inputdeck.make_deck([2, 1, 1], xyz, 'STO-3G', inttol=0.0), oracle.onee, library=lib)
    b = s.basis
    cc = b.cc
    lsum = b.pax + b.pay + b.paz
    live = np.any(cc != 0.0, axis=0)
    s_prim = np.nonzero(live & (lsum == 0))[0]
    p_prim = np.nonzero(live & (lsum == 1))[0]
    assert len(p_prim) == 3 and np.all(np.count_nonzero(cc[:, live], axis=0) == 1)
    rng = np.random.default_rng(9)
    pp = np.zeros((b.npgs, b.npgs))
    a = rng.normal(size=(len(s_prim), len(s_prim)))
    pp[np.ix_(s_prim, s_prim)] = a + a.T
    c_c, x_c = oracle.fourindex_eri(s, pp[None])

    zs = b.zt[s_prim]
    h = 1e-30
    for p in p_prim:
        axis = int(np.argmax([b.pax[p], b.pay[p], b.paz[p]]))
        pos = np.vstack([b.pgs[p], b.pgs[s_prim]]).astype(complex)   # row 0: the p primitive's centre
        pos[0, axis] += 1j * h
        z = np.concatenate([[b.zt[p]], zs])
        d = _ss_rows(pos, z, 0)[1:, 1:, 1:].imag / h / (2.0 * b.zt[p])   # (p q|r s), q, r, s over s_prim
        ps = pp[np.ix_(s_prim, s_prim)]
        j_p = np.einsum('qrs,rs->q', d, ps)           # C_P(p, q)
        k_p = np.einsum('qrs,rq->s', d, ps)           # X_P(p, l)
        i = int(np.nonzero(cc[:, p])[0][0])
        for q_k, q in enumerate(s_prim):
            jq = int(np.nonzero(cc[:, q])[0][0])
            scale = cc[i, p] * cc[jq, q]
            assert abs(c_c[0][i, jq] - scale * j_p[q_k]) <= 1e-12 * np.abs(c_c[0]).max()
            assert abs(x_c[0][i, jq] - scale * k_p[q_k]) <= 1e-12 * np.abs(x_c[0]).max()


def test_d_s_blocks_match_second_derivatives_of_the_closed_form():
    # a Cartesian d primitive is a second derivative of the s primitive in its
    # centre: (x-A_x)^2 e = (d2/dA_x2 + 2a) e / (4a^2), (x-A_x)(y-A_y) e =
    # d2/dA_x dA_y e / (4a^2); torch autograd (FP64) differentiates the closed
    # form; with the density on s primitives the (d, s) blocks of C_C and X_C
    # follow, through CC (whichever contracted functions the d shell makes)
    import torch
    lib = {'H': [['S', 1.0, [[1.3, 1.0]]], ['S', 1.0, [[0.35, 1.0]]]],
           'He': [['S', 1.0, [[2.1, 1.0]]], ['D', 1.0, [[0.9, 1.0]]]]}
    xyz = [[0.0, 0.0, 0.0], [1.4, 0.2, 0.3], [0.3, 1.7, -0.5]]   # bohr
    s = system.build_system(inputdeck.make_deck([2, 1, 1], xyz, 'STO-3G', inttol=0.0), oracle.onee, library=lib)
    b = s.basis
    cc = b.cc
    pw = np.stack([b.pax, b.pay, b.paz], axis=1).astype(int)
    live = np.any(cc != 0.0, axis=0)
    s_prim = np.nonzero(live & (pw.sum(1) == 0))[0]
    d_prim = np.nonzero(live & (pw.sum(1) == 2))[0]
    assert len(d_prim) == 6
    rng = np.random.default_rng(10)
    pp = np.zeros((b.npgs, b.npgs))
    a = rng.normal(size=(len(s_prim), len(s_prim)))
    pp[np.ix_(s_prim, s_prim)] = a + a.T
    c_c, x_c = oracle.fourindex_eri(s, pp[None])

    t64 = dict(dtype=torch.float64)
    zs = torch.tensor(b.zt[s_prim], **t64)
    ps = torch.tensor(pp[np.ix_(s_prim, s_prim)], **t64)
    cs = torch.tensor(b.pgs[s_prim], **t64)

    def sums(centre, za):
        # (a q|r s) over s primitives q, r, s for an s primitive a at `centre`,
        # contracted with the density: J row (q) and K row (l)
        zq = za + zs
        pq = (za * centre + zs[:, None] * cs) / zq[:, None]
        kq = torch.exp(-za * zs / zq * ((centre - cs) ** 2).sum(1))
        zrs = zs[:, None] + zs[None, :]
        prs = (zs[:, None, None] * cs[:, None, :] + zs[None, :, None] * cs[None, :, :]) / zrs[..., None]
        krs = torch.exp(-zs[:, None] * zs[None, :] / zrs * ((cs[:, None, :] - cs[None, :, :]) ** 2).sum(-1))
        zz = zq[:, None, None] + zrs[None]
        rho = zq[:, None, None] * zrs[None] / zz
        t = rho * ((pq[:, None, None, :] - prs[None]) ** 2).sum(-1)
        f0 = torch.where(t > 1e-12, 0.5 * np.sqrt(np.pi) * torch.erf(torch.sqrt(t.clamp_min(1e-12))) /
                         torch.sqrt(t.clamp_min(1e-12)), 1.0 - t / 3.0 + t * t / 10.0)
        eri = 2.0 * np.pi ** 2.5 / (zq[:, None, None] * zrs[None] * torch.sqrt(zz)) * kq[:, None, None] * krs[None] * f0
        return torch.cat([torch.einsum('qrs,rs->q', eri, ps), torch.einsum('qrs,rq->s', eri, ps)])

    n_s = len(s_prim)
    c_p = np.zeros((b.npgs, b.npgs))
    x_p = np.zeros((b.npgs, b.npgs))
    for p in d_prim:
        za = float(b.zt[p])
        centre = torch.tensor(b.pgs[p], **t64)
        jac2 = torch.autograd.functional.jacobian(
            lambda c: torch.autograd.functional.jacobian(lambda c2: sums(c2, za), c, create_graph=True), centre)
        axes = [ax for ax in range(3) for _ in range(pw[p][ax])]
        val = jac2[:, axes[0], axes[1]]
        if axes[0] == axes[1]:
            val = val + 2.0 * za * sums(centre, za)
        val = (val / (4.0 * za * za)).detach().numpy()
        c_p[p, s_prim], x_p[p, s_prim] = val[:n_s], val[n_s:]
    rows = np.nonzero(np.any(cc[:, d_prim] != 0.0, axis=1))[0]
    assert len(rows) and not np.any(cc[np.ix_(rows, s_prim)])
    cols = np.nonzero(np.any(cc[:, s_prim] != 0.0, axis=1))[0]
    want_c = (cc @ c_p @ cc.T)[np.ix_(rows, cols)]
    want_x = (cc @ x_p @ cc.T)[np.ix_(rows, cols)]
    assert np.abs(c_c[0][np.ix_(rows, cols)] - want_c).max() <= 1e-12 * np.abs(c_c[0]).max()
    assert np.abs(x_c[0][np.ix_(rows, cols)] - want_x).max() <= 1e-12 * np.abs(x_c[0]).max()
    assert np.abs(want_c).max() > 1e-3 * np.abs(c_c[0]).max()
