/*
 * CPU oracle for the direct Fock build -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's algorithm, used by tests/, the smoke
 * check and bench.py's CPU-baseline leg as the checker.  Nothing in the product
 * (polymer_b200/) links or calls it.
 *
 *   oracle_fmt_table            FMT_PRELIMINARY        src/pbasis.f90:1-27
 *   oracle_overlap_kinetic      OVERLAP_KINETIC(0)     src/ponee.f90:1-160 (S_P, T_P per cell)
 *   oracle_nuclear_attraction   NUCLEAR_ATTRACTION(0)  src/ponee.f90:418-603 (N_P per cell)
 *   oracle_fourindex_eri        FOURINDEX_ERI          src/pfourindexdirect.f90:1-814
 *   oracle_form_p2h             FORM_C2H (P2H part)    src/pbasis.f90:134-413 (p and d)
 *   oracle_rotate_density       ROTATE_DENSITYMATRIX   src/pdensitymatrix.f90:516-563 (P_P_HELIX)
 *
 * oracle_fourindex_eri follows the reference's loop order and formulas: the
 * Obara-Saika index tables (:101-221), the (Q1,Q2) cell-pair ticket split
 * (:224-240), the KL/IJ pair data and Schwarz bounds that exclude component 1
 * (:260-462), the per-Q3 ket rebuild (:469-525), the INTTOL screen (:529), the
 * tabulated/asymptotic Boys function (:543-553), the ket-then-bra VRR
 * (:563-690), J/K accumulation incl. the helical branch (:691-740), the
 * contraction (:765-782) and the C2H transform (:784-803).  The sixteen
 * specialised VRR branches of the reference (:574-690) are written here as one
 * expression with optional terms; they are algebraically identical.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/polymer_fock.h"

#define LMAX 3
#define NPOW (LMAX + 2)           /* P_SHELL power extent 0..LMAX+1 */
#define NT ((LMAX + 1) * (LMAX + 1))
#define NCMP 400                  /* max component pairs of one shell pair (20*20) */
#define MDIM 17                   /* ERI(0:16, ...) */

static const double REF_PI = 3.14159265358979;  /* src/pmodules.f90:7 */
static const double TF[22] = {33, 37, 41, 43, 46, 49, 51, 54, 56, 58, 61, 63,
                              66, 68, 70, 72, 74, 76, 78, 80, 82, 84}; /* src/pmodules.f90:156-159 */

/* ------------------------------------------------------------------ FMT table */
void oracle_fmt_table(double *igamma /* (0:1700,0:27) column-major */) {
  for (int i = 0; i <= 1700; ++i) {
    double a = (double)i / 20.0, b = exp(-a), c = 0.0;
    int k = (int)(50.0 + (double)i / 3.0); /* K=50+I/3. truncated to integer */
    for (int j = k; j >= 0; --j) {
      c = (2.0 * a * c + b) / (double)(2 * j + 1);
      if (j <= 27) igamma[i + 1701 * j] = c;
    }
  }
}

/* ------------------------------------------------------------ index helpers */
typedef struct {
  int npgs, ncgs, npshell;
  const int32_t *p_shell;
} shellmap;

static inline int PSH(const shellmap *m, int s, int i1, int i2, int i3) { /* 0-based prim or -1 */
  int v = m->p_shell[s + m->npshell * (i1 + NPOW * (i2 + NPOW * i3))];
  return v > 0 ? v - 1 : -1;
}

/* Obara-Saika bookkeeping for one (ia,ja) shell-pair type, src/pfourindexdirect.f90:101-221 */
typedef struct {
  int n;                       /* NKL(type) */
  int angsum[NCMP];            /* KLANGINDX */
  int d1[NCMP][3], d2[NCMP][3];
  double d1c[NCMP][3], d2c[NCMP][3];
  int d3[NCMP], d4[NCMP], d5[NCMP], dxyz[NCMP];
  double d4c[NCMP], d5c[NCMP];
  int pw[NCMP][6];             /* (i1,i2,i3,j1,j2,j3) of each component pair */
} ostype;

static ostype *g_types = NULL; /* NT entries */

static void build_types(void) {
  if (g_types) return;
  g_types = (ostype *)calloc(NT, sizeof(ostype));
  static int ijmap[NPOW][NPOW][NPOW][NPOW][NPOW][NPOW];
  for (int ia = 0; ia <= LMAX; ++ia)
    for (int ja = 0; ja <= LMAX; ++ja) {
      ostype *t = &g_types[ia * (LMAX + 1) + ja];
      int n = 0;
      for (int i1 = 0; i1 <= ia; ++i1)
        for (int i2 = 0; i2 <= ia - i1; ++i2)
          for (int i3 = 0; i3 <= ia - i1 - i2; ++i3)
            for (int j1 = 0; j1 <= ja; ++j1)
              for (int j2 = 0; j2 <= ja - j1; ++j2)
                for (int j3 = 0; j3 <= ja - j1 - j2; ++j3) {
                  int c = n++; /* 0-based component index; reference index = c+1 */
                  int I[3] = {i1, i2, i3}, J[3] = {j1, j2, j3};
                  t->angsum[c] = i1 + i2 + i3 + j1 + j2 + j3;
                  ijmap[i1][i2][i3][j1][j2][j3] = c + 1;
                  memcpy(t->pw[c], I, sizeof I);
                  memcpy(t->pw[c] + 3, J, sizeof J);
                  for (int x = 0; x < 3; ++x) {
                    t->d1[c][x] = t->d2[c][x] = 0;
                    t->d1c[c][x] = t->d2c[c][x] = 0.0;
                    if (I[x] >= 1) {
                      int Ir[3] = {i1, i2, i3};
                      Ir[x]--;
                      t->d1[c][x] = ijmap[Ir[0]][Ir[1]][Ir[2]][j1][j2][j3];
                      t->d1c[c][x] = I[x] / 2.0;
                    }
                    if (J[x] >= 1) {
                      int Jr[3] = {j1, j2, j3};
                      Jr[x]--;
                      t->d2[c][x] = ijmap[i1][i2][i3][Jr[0]][Jr[1]][Jr[2]];
                      t->d2c[c][x] = J[x] / 2.0;
                    }
                  }
                  t->d3[c] = t->d4[c] = t->d5[c] = 0;
                  t->d4c[c] = t->d5c[c] = 0.0;
                  t->dxyz[c] = 0;
                  int ax = -1, onI = 0;
                  for (int x = 0; x < 3 && ax < 0; ++x)
                    if (I[x] >= 1) { ax = x; onI = 1; }
                  for (int x = 0; x < 3 && ax < 0; ++x)
                    if (J[x] >= 1) { ax = x; onI = 0; }
                  if (ax >= 0) {
                    t->dxyz[c] = ax + 1;
                    int Ir[3] = {i1, i2, i3}, Jr[3] = {j1, j2, j3};
                    if (onI) {
                      Ir[ax]--;
                      t->d3[c] = ijmap[Ir[0]][Ir[1]][Ir[2]][j1][j2][j3];
                      if (I[ax] >= 2) {
                        int I2[3] = {i1, i2, i3};
                        I2[ax] -= 2;
                        t->d4[c] = ijmap[I2[0]][I2[1]][I2[2]][j1][j2][j3];
                        t->d4c[c] = (I[ax] - 1) / 2.0;
                      }
                      if (J[ax] >= 1) {
                        Jr[ax]--;
                        t->d5[c] = ijmap[Ir[0]][Ir[1]][Ir[2]][Jr[0]][Jr[1]][Jr[2]];
                        t->d5c[c] = J[ax] / 2.0;
                      }
                    } else {
                      Jr[ax]--;
                      t->d3[c] = ijmap[i1][i2][i3][Jr[0]][Jr[1]][Jr[2]];
                      if (J[ax] >= 2) {
                        int J2[3] = {j1, j2, j3};
                        J2[ax] -= 2;
                        t->d4[c] = ijmap[i1][i2][i3][J2[0]][J2[1]][J2[2]];
                        t->d4c[c] = (J[ax] - 1) / 2.0;
                      }
                    }
                  }
                }
      t->n = n;
    }
}

/* ERI(m, kl, ij) scratch, indices 1-based in kl/ij like the reference */
static double *g_eri = NULL;
#define ERI(m, kl, ij) g_eri[(m) + MDIM * ((kl) + (NCMP + 1) * (ij))]

/* per shell-pair data, mirrors COMZ_S / PX_S / OV / QI_CI / PGSK / PGSL / KLT_S / KLANG */
typedef struct {
  double comz, px, py, pz, ov;
  int type, ang;
  int n;
  int pk[NCMP], pl[NCMP];
  double qi[NCMP];
} pairdata;

static void make_pair(const shellmap *m, const int32_t *ang, int K, int L,
                      double cx, double cy, double cz, double dx, double dy, double dz,
                      double zk, double zl, double ov, pairdata *p) {
  double comz = zk + zl;
  double px = (cx * zk + dx * zl) / comz, py = (cy * zk + dy * zl) / comz, pz = (cz * zk + dz * zl) / comz;
  p->comz = comz;
  p->px = px; p->py = py; p->pz = pz;
  p->ov = ov;
  p->ang = ang[K] + ang[L];
  p->type = ang[K] * (LMAX + 1) + ang[L];
  int n = 0;
  for (int i1 = 0; i1 <= ang[K]; ++i1)
    for (int i2 = 0; i2 <= ang[K] - i1; ++i2)
      for (int i3 = 0; i3 <= ang[K] - i1 - i2; ++i3)
        for (int j1 = 0; j1 <= ang[L]; ++j1)
          for (int j2 = 0; j2 <= ang[L] - j1; ++j2)
            for (int j3 = 0; j3 <= ang[L] - j1 - j2; ++j3) {
              p->pk[n] = PSH(m, K, i1, i2, i3);
              p->pl[n] = PSH(m, L, j1, j2, j3);
              double q = 0.0;
              if (i1 >= 1) q = px - cx;
              else if (i2 >= 1) q = py - cy;
              else if (i3 >= 1) q = pz - cz;
              else if (j1 >= 1) q = px - dx;
              else if (j2 >= 1) q = py - dy;
              else if (j3 >= 1) q = pz - dz;
              p->qi[n] = q;
              ++n;
            }
  p->n = n;
}

/* Schwarz bound of a pair: max over components 2..n of sqrt((kl|kl) maxc maxc),
 * src/pfourindexdirect.f90:326-363 (the same code serves IJIJ, :430-462). */
static double pair_schwarz(const pairdata *p, const double *maxc) {
  const ostype *t = &g_types[p->type];
  double largecomz = 2.0 * p->comz, rho = 0.5 * p->comz;
  int ijkl = 2 * p->ang;
  double c2 = 2.0 * sqrt(rho / REF_PI) * p->ov * p->ov;
  double best = 0.0;
  if (ijkl > 0) {
    for (int m = 0; m <= ijkl; ++m) ERI(m, 1, 1) = c2 / (double)(2 * m + 1);
    for (int ij = 1; ij <= t->n; ++ij) {
      if (ij == 1) {
        for (int kl = 2; kl <= t->n; ++kl) {
          int c = kl - 1;
          for (int m = 0; m <= ijkl - t->angsum[c]; ++m) {
            double v = p->qi[c] * ERI(m, t->d3[c], 1);
            if (t->d4[c]) v += t->d4c[c] / p->comz * (ERI(m, t->d4[c], 1) - 0.5 * ERI(m + 1, t->d4[c], 1));
            if (t->d5[c]) v += t->d5c[c] / p->comz * (ERI(m, t->d5[c], 1) - 0.5 * ERI(m + 1, t->d5[c], 1));
            ERI(m, kl, 1) = v;
          }
        }
      } else {
        int b = ij - 1, ax = t->dxyz[b] - 1;
        for (int kl = 1; kl <= t->n; ++kl) {
          int c = kl - 1;
          for (int m = 0; m <= ijkl - t->angsum[b] - t->angsum[c]; ++m) {
            double v = p->qi[b] * ERI(m, kl, t->d3[b]);
            if (t->d4[b]) v += t->d4c[b] / p->comz * (ERI(m, kl, t->d4[b]) - 0.5 * ERI(m + 1, kl, t->d4[b]));
            if (t->d5[b]) v += t->d5c[b] / p->comz * (ERI(m, kl, t->d5[b]) - 0.5 * ERI(m + 1, kl, t->d5[b]));
            if (t->d1[c][ax]) v += t->d1c[c][ax] / largecomz * ERI(m + 1, t->d1[c][ax], t->d3[b]);
            if (t->d2[c][ax]) v += t->d2c[c][ax] / largecomz * ERI(m + 1, t->d2[c][ax], t->d3[b]);
            ERI(m, kl, ij) = v;
          }
        }
      }
    }
    for (int kl = 2; kl <= t->n; ++kl) {
      int c = kl - 1;
      double mk = p->pk[c] >= 0 ? maxc[p->pk[c]] : 0.0, ml = p->pl[c] >= 0 ? maxc[p->pl[c]] : 0.0;
      double a = sqrt(ERI(0, kl, kl) * mk * ml);
      if (a > best) best = a;
    }
  } else {
    best = sqrt(c2 * maxc[p->pk[0]] * maxc[p->pl[0]]);
  }
  return best;
}

static inline double boys_tab(const double *ig, int m, double T, double c2, const double *f1, const double *f2) {
  if (T < TF[m]) {
    int ts = (int)floor(T * 20.0 + 0.5); /* NINT for T >= 0 */
    double h = 0.05 * (double)ts - T;
    const double *g = ig + ts;
#define G(k) g[1701 * (m + (k))]
    return ((((((G(6) * h * 0.166666666666667 + G(5)) * h * 0.2 + G(4)) * h * 0.25 + G(3)) * h *
                 0.333333333333333 + G(2)) * h * 0.5 + G(1)) * h + G(0)) * c2;
#undef G
  }
  return c2 * f1[m] * exp(f2[m] * log(T));
}

/* ---------------------------------------------------------- FOURINDEX_ERI */
/* Bra-shell sampling for the bounded CPU baseline: only I with I % g_stride ==
 * g_offset are processed (1/0 = the whole loop, the reference's semantics). */
static int g_stride = 1, g_offset = 0;

int32_t oracle_fourindex_eri(const pfe_args *a, double *c_c, double *x_c);

int32_t oracle_fourindex_eri_sample(const pfe_args *a, double *c_c, double *x_c, int32_t stride, int32_t offset) {
  g_stride = stride > 0 ? stride : 1;
  g_offset = offset;
  int32_t rc = oracle_fourindex_eri(a, c_c, x_c);
  g_stride = 1;
  g_offset = 0;
  return rc;
}

int32_t oracle_fourindex_eri(const pfe_args *a, double *c_c, double *x_c) {
  build_types();
  if (!g_eri) g_eri = (double *)malloc(sizeof(double) * MDIM * (NCMP + 1) * (NCMP + 1));
  const int npgs = a->npgs, ncgs = a->ncgs, nsh = a->npshell;
  shellmap sm = {npgs, ncgs, nsh, a->p_shell};
  const int c1x = a->cel1[0], c1y = a->cel1[1], c1z = a->cel1[2];
  const int c2x = a->cel2[0], c2y = a->cel2[1], c2z = a->cel2[2];
  const int r1x = a->reduced_cel1[0], r1y = a->reduced_cel1[1], r1z = a->reduced_cel1[2];
  const int n1x = 2 * c1x + 1, n1y = 2 * c1y + 1, n1z = 2 * c1z + 1, ncell1 = n1x * n1y * n1z;
  const int h3 = c2x + c1x; /* P3 arrays span -h3..h3 along x */
  const double helix = a->helix;
  const double *ig = a->igamma;
  const size_t pp = (size_t)npgs * npgs;
#define CELL1(qx, qy, qz) ((size_t)((qx) + c1x) + (size_t)n1x * ((size_t)((qy) + c1y) + (size_t)n1y * ((qz) + c1z)))
#define SP(i, j, qx, qy, qz) a->s_p[(size_t)(i) + (size_t)npgs * (j) + pp * CELL1(qx, qy, qz)]
#define PP(i, j, qx, qy, qz) a->p_p[(size_t)(i) + (size_t)npgs * (j) + pp * CELL1(qx, qy, qz)]
#define PPH(i, j, q2, q1) a->p_p_helix[(size_t)(i) + (size_t)npgs * (j) + pp * ((size_t)((q2) + c2x) + (size_t)(2 * c2x + 1) * ((q1) + h3))]

  double f1[22], f2[22];
  f1[0] = 1.0 / (2.0 / sqrt(REF_PI));
  f2[0] = -0.5;
  for (int i = 1; i <= 16 && i < 22; ++i) {
    f1[i] = f1[i - 1] * (double)(2 * i - 1) / 2.0;
    f2[i] = f2[i - 1] - 1.0;
  }
  for (int i = 17; i < 22; ++i) { f1[i] = f1[i - 1] * (double)(2 * i - 1) / 2.0; f2[i] = f2[i - 1] - 1.0; }

  int nh = 2 * h3 + 1;
  double *p3x = malloc(sizeof(double) * nh), *p3c = malloc(sizeof(double) * nh), *p3s = malloc(sizeof(double) * nh);
  int nhy = 2 * (c2y + c1y) + 1, nhz = 2 * (c2z + c1z) + 1;
  double *p3y = malloc(sizeof(double) * nhy), *p3z = malloc(sizeof(double) * nhz);
  for (int q = -h3; q <= h3; ++q) {
    double ang = (double)q * helix;
    p3x[q + h3] = (double)q * a->period[0];
    p3c[q + h3] = cos(ang);
    p3s[q + h3] = sin(ang);
  }
  for (int q = -(c2y + c1y); q <= c2y + c1y; ++q) p3y[q + c2y + c1y] = (double)q * a->period[1];
  for (int q = -(c2z + c1z); q <= c2z + c1z; ++q) p3z[q + c2z + c1z] = (double)q * a->period[2];
#define P3X(q) p3x[(q) + h3]
#define P3C(q) p3c[(q) + h3]
#define P3S(q) p3s[(q) + h3]
#define P3Y(q) p3y[(q) + c2y + c1y]
#define P3Z(q) p3z[(q) + c2z + c1z]

  double *maxc = calloc(npgs, sizeof(double));
  for (int i = 0; i < npgs; ++i)
    for (int j = 0; j < ncgs; ++j) {
      double v = fabs(a->cc[j + (size_t)ncgs * i]);
      if (v > maxc[i]) maxc[i] = v;
    }
  double *cp = calloc(pp * ncell1, sizeof(double));
  double *xp = calloc(pp * ncell1, sizeof(double));
  pairdata *kl0 = malloc(sizeof(pairdata) * (size_t)nsh * nsh);
  double *klkl = malloc(sizeof(double) * (size_t)nsh * nsh);
  pairdata *ijd = malloc(sizeof(pairdata));
  int *head = malloc(sizeof(int) * nsh);
  for (int s = 0; s < nsh; ++s) head[s] = PSH(&sm, s, 0, 0, 0);
  const double *X = a->pgsx, *Y = a->pgsy, *Z = a->pgsz, *ZT = a->zt;
  int32_t status = PFE_OK;

  int ticket = 0;
  for (int q1x = -r1x; q1x <= r1x; ++q1x)
  for (int q1y = -r1y; q1y <= r1y; ++q1y)
  for (int q1z = -r1z; q1z <= r1z; ++q1z) {
    double p1x = q1x * a->period[0], p1y = q1y * a->period[1], p1z = q1z * a->period[2];
    double p1c = P3C(q1x), p1s = P3S(q1x);
    for (int q2x = -r1x; q2x <= r1x; ++q2x)
    for (int q2y = -r1y; q2y <= r1y; ++q2y)
    for (int q2z = -r1z; q2z <= r1z; ++q2z) {
      ticket += 1;
      if (ticket == a->numprocs) ticket -= a->numprocs;
      if (a->myid != ticket) continue;
      double p2x = q2x * a->period[0], p2y = q2y * a->period[1], p2z = q2z * a->period[2];
      double p2c = P3C(q2x), p2s = P3S(q2x);
      /* KL pair data at (K@0, L@Q2) and their Schwarz bounds */
      for (int K = 0; K < nsh; ++K) {
        int kk = head[K];
        for (int L = 0; L < nsh; ++L) {
          int ll = head[L];
          double dx = X[ll] + p2x, dy = Y[ll] * p2c - Z[ll] * p2s + p2y, dz = Y[ll] * p2s + Z[ll] * p2c + p2z;
          make_pair(&sm, a->p_shell_ang, K, L, X[kk], Y[kk], Z[kk], dx, dy, dz, ZT[kk], ZT[ll],
                    SP(kk, ll, q2x, q2y, q2z), &kl0[K * nsh + L]);
          klkl[K * nsh + L] = pair_schwarz(&kl0[K * nsh + L], maxc);
        }
      }
      for (int I = 0; I < nsh; ++I) {
        if (I % g_stride != g_offset) continue;
        int ii = head[I];
        double ax = X[ii], ay = Y[ii], az = Z[ii];
        for (int J = 0; J < nsh; ++J) {
          int jj = head[J];
          double bx = X[jj] + p1x, by = Y[jj] * p1c - Z[jj] * p1s + p1y, bz = Y[jj] * p1s + Z[jj] * p1c + p1z;
          double sij = SP(ii, jj, q1x, q1y, q1z);
          make_pair(&sm, a->p_shell_ang, I, J, ax, ay, az, bx, by, bz, ZT[ii], ZT[jj], sij, ijd);
          double comz = ijd->comz, px = ijd->px, py = ijd->py, pz = ijd->pz;
          double c1 = sij * 2.0 / sqrt(REF_PI);
          int ijt = ijd->type, ijang = ijd->ang, nij = ijd->n;
          const ostype *tij = &g_types[ijt];
          /* IJIJ reads QI_CI(:,SIJ) as left in the KL scratch (src/pfourindexdirect.f90:436-447):
           * for the first (I,J) of a cell pair that is the (I@0, J@Q2) pair built at :262-312,
           * afterwards the (I@Q3, J@Q3+Q2) pair of the last Q3 of the previous (I,J) rebuild
           * (:469-525).  Exact for molecules; replicated as is for lattices. */
          double ijij;
          {
            pairdata stale;
            int q3lx = (I == 0 && J == 0) ? 0 : c2x, q3ly = (I == 0 && J == 0) ? 0 : c2y,
                q3lz = (I == 0 && J == 0) ? 0 : c2z;
            double sx = X[ii] + P3X(q3lx), sy = Y[ii] * P3C(q3lx) - Z[ii] * P3S(q3lx) + P3Y(q3ly),
                   sz = Y[ii] * P3S(q3lx) + Z[ii] * P3C(q3lx) + P3Z(q3lz);
            int tx = q3lx + q2x, ty = q3ly + q2y, tz = q3lz + q2z;
            double ex = X[jj] + P3X(tx), ey = Y[jj] * P3C(tx) - Z[jj] * P3S(tx) + P3Y(ty),
                   ez = Y[jj] * P3S(tx) + Z[jj] * P3C(tx) + P3Z(tz);
            make_pair(&sm, a->p_shell_ang, I, J, sx, sy, sz, ex, ey, ez, ZT[ii], ZT[jj], sij, &stale);
            memcpy(stale.pk, ijd->pk, sizeof stale.pk);
            memcpy(stale.pl, ijd->pl, sizeof stale.pl);
            stale.comz = comz;
            ijij = pair_schwarz(&stale, maxc);
          }
          for (int q3x = -c2x; q3x <= c2x; ++q3x)
          for (int q3y = -c2y; q3y <= c2y; ++q3y)
          for (int q3z = -c2z; q3z <= c2z; ++q3z) {
            int lcel = (q3x + q2x >= -c1x && q3x + q2x <= c1x && q1x - q3x >= -c1x && q1x - q3x <= c1x) &&
                       (q3y + q2y >= -c1y && q3y + q2y <= c1y && q1y - q3y >= -c1y && q1y - q3y <= c1y) &&
                       (q3z + q2z >= -c1z && q3z + q2z <= c1z && q1z - q3z >= -c1z && q1z - q3z <= c1z);
            for (int K = 0; K < nsh; ++K) {
              int kk = head[K];
              double cx = X[kk] + P3X(q3x), cy = Y[kk] * P3C(q3x) - Z[kk] * P3S(q3x) + P3Y(q3y),
                     cz = Y[kk] * P3S(q3x) + Z[kk] * P3C(q3x) + P3Z(q3z);
              for (int L = 0; L < nsh; ++L) {
                int skl = K * nsh + L;
                if (ijij * klkl[skl] < a->inttol) continue; /* the rebuild is pure data; skip it with the screen */
                int ll = head[L];
                int qx = q3x + q2x, qy = q3y + q2y, qz = q3z + q2z;
                double dx = X[ll] + P3X(qx), dy = Y[ll] * P3C(qx) - Z[ll] * P3S(qx) + P3Y(qy),
                       dz = Y[ll] * P3S(qx) + Z[ll] * P3C(qx) + P3Z(qz);
                pairdata kd;
                make_pair(&sm, a->p_shell_ang, K, L, cx, cy, cz, dx, dy, dz, ZT[kk], ZT[ll],
                          SP(kk, ll, q2x, q2y, q2z), &kd);
                const ostype *tkl = &g_types[kd.type];
                double largecomz = comz + kd.comz;
                double rc1 = kd.comz / largecomz, rc2 = comz / largecomz;
                double rho = comz * rc1;
                int ijkl = ijang + kd.ang;
                double c2 = c1 * sqrt(rho) * kd.ov;
                if (ijkl > 21 || ijkl + 6 > 27) { status = PFE_ERANGE; goto done; }
                double qxx = kd.px, qyy = kd.py, qzz = kd.pz;
                double T = rho * ((qxx - px) * (qxx - px) + (qyy - py) * (qyy - py) + (qzz - pz) * (qzz - pz));
                if (ijkl > 0) {
                  for (int m = 0; m <= ijkl; ++m) ERI(m, 1, 1) = boys_tab(ig, m, T, c2, f1, f2);
                  double wx = (px * comz + qxx * kd.comz) / largecomz, wy = (py * comz + qyy * kd.comz) / largecomz,
                         wz = (pz * comz + qzz * kd.comz) / largecomz;
                  double wp[3] = {wx - px, wy - py, wz - pz}, wq[3] = {wx - qxx, wy - qyy, wz - qzz};
                  for (int kl = 2; kl <= tkl->n; ++kl) {
                    int c = kl - 1, ax3 = tkl->dxyz[c] - 1;
                    for (int m = 0; m <= ijkl - tkl->angsum[c]; ++m) {
                      double v = kd.qi[c] * ERI(m, tkl->d3[c], 1) + wq[ax3] * ERI(m + 1, tkl->d3[c], 1);
                      if (tkl->d4[c]) v += tkl->d4c[c] / kd.comz * (ERI(m, tkl->d4[c], 1) - rc2 * ERI(m + 1, tkl->d4[c], 1));
                      if (tkl->d5[c]) v += tkl->d5c[c] / kd.comz * (ERI(m, tkl->d5[c], 1) - rc2 * ERI(m + 1, tkl->d5[c], 1));
                      ERI(m, kl, 1) = v;
                    }
                  }
                  for (int ij = 2; ij <= nij; ++ij) {
                    int b = ij - 1, ax = tij->dxyz[b] - 1;
                    for (int kl = 1; kl <= tkl->n; ++kl) {
                      int c = kl - 1;
                      for (int m = 0; m <= ijkl - tij->angsum[b] - tkl->angsum[c]; ++m) {
                        double v = ijd->qi[b] * ERI(m, kl, tij->d3[b]) + wp[ax] * ERI(m + 1, kl, tij->d3[b]);
                        if (tij->d4[b]) v += tij->d4c[b] / comz * (ERI(m, kl, tij->d4[b]) - rc1 * ERI(m + 1, kl, tij->d4[b]));
                        if (tij->d5[b]) v += tij->d5c[b] / comz * (ERI(m, kl, tij->d5[b]) - rc1 * ERI(m + 1, kl, tij->d5[b]));
                        if (tkl->d1[c][ax]) v += tkl->d1c[c][ax] / largecomz * ERI(m + 1, tkl->d1[c][ax], tij->d3[b]);
                        if (tkl->d2[c][ax]) v += tkl->d2c[c][ax] / largecomz * ERI(m + 1, tkl->d2[c][ax], tij->d3[b]);
                        ERI(m, kl, ij) = v;
                      }
                    }
                  }
                  if (helix == 0.0) {
                    for (int ij = 1; ij <= nij; ++ij) {
                      int pi = ijd->pk[ij - 1], pj = ijd->pl[ij - 1];
                      double acc = 0.0;
                      for (int kl = 1; kl <= tkl->n; ++kl)
                        acc += PP(kd.pk[kl - 1], kd.pl[kl - 1], q2x, q2y, q2z) * ERI(0, kl, ij);
                      cp[(size_t)pi + (size_t)npgs * pj + pp * CELL1(q1x, q1y, q1z)] += acc;
                    }
                    if (lcel)
                      for (int ij = 1; ij <= nij; ++ij) {
                        int pi = ijd->pk[ij - 1], pj = ijd->pl[ij - 1];
                        for (int kl = 1; kl <= tkl->n; ++kl)
                          xp[(size_t)pi + (size_t)npgs * kd.pl[kl - 1] + pp * CELL1(q3x + q2x, q3y + q2y, q3z + q2z)] +=
                              PP(kd.pk[kl - 1], pj, q1x - q3x, q1y - q3y, q1z - q3z) * ERI(0, kl, ij);
                      }
                  } else {
                    for (int ij = 1; ij <= nij; ++ij) {
                      int pi = ijd->pk[ij - 1], pj = ijd->pl[ij - 1];
                      double acc = 0.0;
                      for (int kl = 1; kl <= tkl->n; ++kl)
                        acc += PPH(kd.pk[kl - 1], kd.pl[kl - 1], q3x, q3x + q2x) * ERI(0, kl, ij);
                      cp[(size_t)pi + (size_t)npgs * pj + pp * CELL1(q1x, q1y, q1z)] += acc;
                    }
                    if (lcel)
                      for (int ij = 1; ij <= nij; ++ij) {
                        int pi = ijd->pk[ij - 1], pj = ijd->pl[ij - 1];
                        for (int kl = 1; kl <= tkl->n; ++kl)
                          xp[(size_t)pi + (size_t)npgs * kd.pl[kl - 1] + pp * CELL1(q3x + q2x, q3y + q2y, q3z + q2z)] +=
                              PPH(kd.pk[kl - 1], pj, q3x, q1x) * ERI(0, kl, ij);
                      }
                  }
                } else { /* all-s quartet: helix does not matter */
                  double e;
                  if (T < TF[0]) e = boys_tab(ig, 0, T, c2, f1, f2);
                  else e = c2 * f1[0] * exp(-0.5 * log(T));
                  int pi = ijd->pk[0], pj = ijd->pl[0];
                  cp[(size_t)pi + (size_t)npgs * pj + pp * CELL1(q1x, q1y, q1z)] += PP(kd.pk[0], kd.pl[0], q2x, q2y, q2z) * e;
                  if (lcel)
                    xp[(size_t)pi + (size_t)npgs * kd.pl[0] + pp * CELL1(q3x + q2x, q3y + q2y, q3z + q2z)] +=
                        PP(kd.pk[0], pj, q1x - q3x, q1y - q3y, q1z - q3z) * e;
                }
              }
            }
          }
        }
      }
    }
  }

  /* contraction C_C = CC . C_P . CC^T per cell, then the helical transform */
  {
    double *w2 = malloc(sizeof(double) * (size_t)ncgs * npgs);
    double *src[2] = {cp, xp};
    double *dst[2] = {c_c, x_c};
    for (int o = 0; o < 2; ++o)
      for (int c = 0; c < ncell1; ++c) {
        const double *W1 = src[o] + pp * c;
        double *W3 = dst[o] + (size_t)ncgs * ncgs * c;
        for (int i = 0; i < ncgs; ++i)
          for (int j = 0; j < npgs; ++j) {
            double s = 0.0;
            for (int k = 0; k < npgs; ++k) s += a->cc[i + (size_t)ncgs * k] * W1[k + (size_t)npgs * j];
            w2[i + (size_t)ncgs * j] = s;
          }
        for (int i = 0; i < ncgs; ++i)
          for (int j = 0; j < ncgs; ++j) {
            double s = 0.0;
            for (int k = 0; k < npgs; ++k) s += w2[i + (size_t)ncgs * k] * a->cc[j + (size_t)ncgs * k];
            W3[i + (size_t)ncgs * j] = s;
          }
      }
    free(w2);
    if (helix != 0.0) {
      double *w = malloc(sizeof(double) * (size_t)ncgs * ncgs);
      size_t cc2 = (size_t)ncgs * ncgs;
      for (int o = 0; o < 2; ++o)
        for (int q = -c1x; q <= c1x; ++q) {
          double *M = dst[o] + cc2 * CELL1(q, 0, 0);
          const double *H = a->c2h + cc2 * (size_t)(q + h3);
          for (int i = 0; i < ncgs; ++i)
            for (int j = 0; j < ncgs; ++j) {
              double s = 0.0;
              for (int jj = 0; jj < ncgs; ++jj) s += H[j + (size_t)ncgs * jj] * M[i + (size_t)ncgs * jj];
              w[i + (size_t)ncgs * j] = s;
            }
          memcpy(M, w, sizeof(double) * cc2);
        }
      free(w);
    }
  }
done:
  free(p3x); free(p3c); free(p3s); free(p3y); free(p3z);
  free(maxc); free(cp); free(xp); free(kl0); free(klkl); free(ijd); free(head);
  return status;
#undef CELL1
#undef SP
#undef PP
#undef PPH
}

/* --------------------------------------------------- one-electron integrals */
typedef struct {
  int32_t npgs, npshell, natom;
  const int32_t *p_shell, *p_shell_ang, *pgs_atom;
  const double *pgsx, *pgsy, *pgsz, *zt;
  const int32_t *iatom;
  const double *atomx, *atomy, *atomz;
  int32_t cel1[3], cel2[3];
  double period[3], helix;
  const double *igamma;
} oracle_onee_args;

/* S1/T1 over powers 0..LMAX+1 of both centres */
#define I6(a1, a2, a3, b1, b2, b3) ((a1) + NPOW * ((a2) + NPOW * ((a3) + NPOW * ((b1) + NPOW * ((b2) + NPOW * (b3))))))

int32_t oracle_overlap_kinetic(const oracle_onee_args *a, double *s_p, double *t_p) {
  shellmap sm = {a->npgs, 0, a->npshell, a->p_shell};
  const int npgs = a->npgs, nsh = a->npshell;
  const int c1x = a->cel1[0], c1y = a->cel1[1], c1z = a->cel1[2];
  const int n1x = 2 * c1x + 1, n1y = 2 * c1y + 1, n1z = 2 * c1z + 1;
  const size_t pp = (size_t)npgs * npgs;
  const double pisub = sqrt(REF_PI * REF_PI * REF_PI);
  static double S1[NPOW * NPOW * NPOW * NPOW * NPOW * NPOW], T1[NPOW * NPOW * NPOW * NPOW * NPOW * NPOW];
  memset(s_p, 0, sizeof(double) * pp * n1x * n1y * n1z);
  memset(t_p, 0, sizeof(double) * pp * n1x * n1y * n1z);
  for (int kx = -c1x; kx <= c1x; ++kx)
  for (int ky = -c1y; ky <= c1y; ++ky)
  for (int kz = -c1z; kz <= c1z; ++kz) {
    double qx = kx * a->period[0], qy = ky * a->period[1], qz = kz * a->period[2];
    double ang = kx * a->helix, cs = cos(ang), sn = sin(ang);
    size_t cell = (size_t)(kx + c1x) + (size_t)n1x * ((size_t)(ky + c1y) + (size_t)n1y * (kz + c1z));
    for (int I = 0; I < nsh; ++I) {
      int ii = PSH(&sm, I, 0, 0, 0);
      double ax = a->pgsx[ii], ay = a->pgsy[ii], az = a->pgsz[ii];
      for (int J = 0; J < nsh; ++J) {
        int jj = PSH(&sm, J, 0, 0, 0);
        double bx = a->pgsx[jj] + qx, by = a->pgsy[jj] * cs - a->pgsz[jj] * sn + qy, bz = a->pgsy[jj] * sn + a->pgsz[jj] * cs + qz;
        double r = (ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz);
        double comz1 = a->zt[ii] + a->zt[jj], comz2 = sqrt(comz1 * comz1 * comz1), gzi = a->zt[ii] * a->zt[jj] / comz1;
        S1[0] = pisub / comz2 * exp(-gzi * r);
        T1[0] = gzi * (3.0 - 2.0 * gzi * r) * S1[0];
        double px = (ax * a->zt[ii] + bx * a->zt[jj]) / comz1, py = (ay * a->zt[ii] + by * a->zt[jj]) / comz1,
               pz = (az * a->zt[ii] + bz * a->zt[jj]) / comz1;
        double PA[3] = {px - ax, py - ay, pz - az}, PB[3] = {px - bx, py - by, pz - bz};
        int LI = a->p_shell_ang[I], LJ = a->p_shell_ang[J];
        for (int i1 = 0; i1 <= LI; ++i1)
        for (int i2 = 0; i2 <= LI - i1; ++i2)
        for (int i3 = 0; i3 <= LI - i1 - i2; ++i3)
        for (int j1 = 0; j1 <= LJ; ++j1)
        for (int j2 = 0; j2 <= LJ - j1; ++j2)
        for (int j3 = 0; j3 <= LJ - j1 - j2; ++j3) {
          if (i1 + i2 + i3 + j1 + j2 + j3 == 0) continue;
          int A[3] = {i1, i2, i3}, B[3] = {j1, j2, j3};
          int ax3 = -1, onA = 0;
          for (int x = 0; x < 3 && ax3 < 0; ++x) if (A[x] >= 1) { ax3 = x; onA = 1; }
          for (int x = 0; x < 3 && ax3 < 0; ++x) if (B[x] >= 1) { ax3 = x; onA = 0; }
          int A1[3] = {i1, i2, i3}, B1[3] = {j1, j2, j3};
          int idx = I6(i1, i2, i3, j1, j2, j3);
          double s, t;
          if (onA) {
            A1[ax3]--;
            int i_m1 = I6(A1[0], A1[1], A1[2], j1, j2, j3);
            s = PA[ax3] * S1[i_m1];
            int A2[3] = {A1[0], A1[1], A1[2]};
            double s_m2 = 0.0, t_m2 = 0.0, s_b = 0.0, t_b = 0.0;
            if (A[ax3] >= 2) { A2[ax3]--; int i_m2 = I6(A2[0], A2[1], A2[2], j1, j2, j3); s_m2 = S1[i_m2]; t_m2 = T1[i_m2]; }
            if (B[ax3] >= 1) { int B2[3] = {j1, j2, j3}; B2[ax3]--; int i_b = I6(A1[0], A1[1], A1[2], B2[0], B2[1], B2[2]); s_b = S1[i_b]; t_b = T1[i_b]; }
            if (A[ax3] >= 2) s += 0.5 * (double)(A[ax3] - 1) / comz1 * s_m2;
            if (B[ax3] >= 1) s += 0.5 * (double)B[ax3] / comz1 * s_b;
            S1[idx] = s;
            t = 2.0 * gzi * S1[idx] + PA[ax3] * T1[i_m1];
            if (A[ax3] >= 2) t += 0.5 * (double)(A[ax3] - 1) / comz1 * t_m2 - (double)(A[ax3] - 1) * gzi / a->zt[ii] * s_m2;
            if (B[ax3] >= 1) t += 0.5 * (double)B[ax3] / comz1 * t_b;
            T1[idx] = t;
          } else {
            B1[ax3]--;
            int i_m1 = I6(i1, i2, i3, B1[0], B1[1], B1[2]);
            s = PB[ax3] * S1[i_m1];
            double s_m2 = 0.0, t_m2 = 0.0;
            if (B[ax3] >= 2) { int B2[3] = {B1[0], B1[1], B1[2]}; B2[ax3]--; int i_m2 = I6(i1, i2, i3, B2[0], B2[1], B2[2]); s_m2 = S1[i_m2]; t_m2 = T1[i_m2]; }
            if (B[ax3] >= 2) s += 0.5 * (double)(B[ax3] - 1) / comz1 * s_m2;
            S1[idx] = s;
            t = 2.0 * gzi * S1[idx] + PB[ax3] * T1[i_m1];
            if (B[ax3] >= 2) t += 0.5 * (double)(B[ax3] - 1) / comz1 * t_m2 - (double)(B[ax3] - 1) * gzi / a->zt[jj] * s_m2;
            T1[idx] = t;
          }
        }
        for (int i1 = 0; i1 <= LI; ++i1)
        for (int i2 = 0; i2 <= LI - i1; ++i2)
        for (int i3 = 0; i3 <= LI - i1 - i2; ++i3)
        for (int j1 = 0; j1 <= LJ; ++j1)
        for (int j2 = 0; j2 <= LJ - j1; ++j2)
        for (int j3 = 0; j3 <= LJ - j1 - j2; ++j3) {
          int pi = PSH(&sm, I, i1, i2, i3), pj = PSH(&sm, J, j1, j2, j3);
          int idx = I6(i1, i2, i3, j1, j2, j3);
          s_p[(size_t)pi + (size_t)npgs * pj + pp * cell] = S1[idx];
          t_p[(size_t)pi + (size_t)npgs * pj + pp * cell] = T1[idx];
        }
      }
    }
  }
  return PFE_OK;
}

int32_t oracle_nuclear_attraction(const oracle_onee_args *a, double *n_p) {
  shellmap sm = {a->npgs, 0, a->npshell, a->p_shell};
  const int npgs = a->npgs, nsh = a->npshell;
  const int c1x = a->cel1[0], c1y = a->cel1[1], c1z = a->cel1[2];
  const int c2x = a->cel2[0], c2y = a->cel2[1], c2z = a->cel2[2];
  const int n1x = 2 * c1x + 1, n1y = 2 * c1y + 1, n1z = 2 * c1z + 1;
  const size_t pp = (size_t)npgs * npgs;
  const double *ig = a->igamma;
  const int MM = 2 * LMAX + 2;
  double f1[2 * LMAX + 2], f2[2 * LMAX + 2];
  f1[0] = 1.0 / (2.0 / sqrt(REF_PI));
  f2[0] = -0.5;
  for (int i = 1; i <= 2 * LMAX + 1; ++i) { f1[i] = f1[i - 1] * (double)(2 * i - 1) / 2.0; f2[i] = f2[i - 1] - 1.0; }
  static double N1[NPOW * NPOW * NPOW * NPOW * NPOW * NPOW * (2 * LMAX + 2)];
  static double N2[NPOW * NPOW * NPOW * NPOW * NPOW * NPOW];
#define N1I(idx, m) N1[(idx) * MM + (m)]
  memset(n_p, 0, sizeof(double) * pp * n1x * n1y * n1z);
  /* S_P at the same cell is needed for the prefactor E1 = 2/sqrt(pi) sqrt(zeta) S_P */
  for (int k1x = -c1x; k1x <= c1x; ++k1x)
  for (int k1y = -c1y; k1y <= c1y; ++k1y)
  for (int k1z = -c1z; k1z <= c1z; ++k1z) {
    double q1x = k1x * a->period[0], q1y = k1y * a->period[1], q1z = k1z * a->period[2];
    double ang = k1x * a->helix, cs = cos(ang), sn = sin(ang);
    size_t cell = (size_t)(k1x + c1x) + (size_t)n1x * ((size_t)(k1y + c1y) + (size_t)n1y * (k1z + c1z));
    for (int I = 0; I < nsh; ++I) {
      int ii = PSH(&sm, I, 0, 0, 0);
      double ax = a->pgsx[ii], ay = a->pgsy[ii], az = a->pgsz[ii];
      for (int J = 0; J < nsh; ++J) {
        int jj = PSH(&sm, J, 0, 0, 0);
        double bx = a->pgsx[jj] + q1x, by = a->pgsy[jj] * cs - a->pgsz[jj] * sn + q1y, bz = a->pgsy[jj] * sn + a->pgsz[jj] * cs + q1z;
        double comz = a->zt[ii] + a->zt[jj];
        double px = (ax * a->zt[ii] + bx * a->zt[jj]) / comz, py = (ay * a->zt[ii] + by * a->zt[jj]) / comz,
               pz = (az * a->zt[ii] + bz * a->zt[jj]) / comz;
        double r = (ax - bx) * (ax - bx) + (ay - by) * (ay - by) + (az - bz) * (az - bz);
        double sab = sqrt(REF_PI * REF_PI * REF_PI) / sqrt(comz * comz * comz) * exp(-a->zt[ii] * a->zt[jj] / comz * r);
        double e1 = 2.0 / sqrt(REF_PI) * sqrt(comz) * sab;
        double PA[3] = {px - ax, py - ay, pz - az}, PB[3] = {px - bx, py - by, pz - bz};
        int LI = a->p_shell_ang[I], LJ = a->p_shell_ang[J];
        memset(N2, 0, sizeof N2);
        for (int k2x = -c2x; k2x <= c2x; ++k2x)
        for (int k2y = -c2y; k2y <= c2y; ++k2y)
        for (int k2z = -c2z; k2z <= c2z; ++k2z) {
          double q2x = k2x * a->period[0], q2y = k2y * a->period[1], q2z = k2z * a->period[2];
          double ang2 = k2x * a->helix, cs2 = cos(ang2), sn2 = sin(ang2);
          for (int k = 0; k < a->natom; ++k) {
            double e2 = -(double)a->iatom[k] * e1;
            double cx = a->atomx[k] + q2x, cy = a->atomy[k] * cs2 - a->atomz[k] * sn2 + q2y,
                   cz = a->atomy[k] * sn2 + a->atomz[k] * cs2 + q2z;
            double T = comz * ((px - cx) * (px - cx) + (py - cy) * (py - cy) + (pz - cz) * (pz - cz));
            double PC[3] = {px - cx, py - cy, pz - cz};
            for (int m = 0; m <= LI + LJ; ++m) N1I(0, m) = boys_tab(ig, m, T, e2, f1, f2);
            N2[0] += N1I(0, 0);
            for (int i1 = 0; i1 <= LI; ++i1)
            for (int i2 = 0; i2 <= LI - i1; ++i2)
            for (int i3 = 0; i3 <= LI - i1 - i2; ++i3)
            for (int j1 = 0; j1 <= LJ; ++j1)
            for (int j2 = 0; j2 <= LJ - j1; ++j2)
            for (int j3 = 0; j3 <= LJ - j1 - j2; ++j3) {
              int mmax = LI + LJ - i1 - i2 - i3 - j1 - j2 - j3;
              if (i1 + i2 + i3 + j1 + j2 + j3 == 0 || mmax < 0) continue;
              int A[3] = {i1, i2, i3}, B[3] = {j1, j2, j3};
              int ax3 = -1, onA = 0;
              for (int x = 0; x < 3 && ax3 < 0; ++x) if (A[x] >= 1) { ax3 = x; onA = 1; }
              for (int x = 0; x < 3 && ax3 < 0; ++x) if (B[x] >= 1) { ax3 = x; onA = 0; }
              int idx = I6(i1, i2, i3, j1, j2, j3);
              for (int m = 0; m <= mmax; ++m) {
                double v;
                if (onA) {
                  int A1[3] = {i1, i2, i3}; A1[ax3]--;
                  int i_m1 = I6(A1[0], A1[1], A1[2], j1, j2, j3);
                  v = PA[ax3] * N1I(i_m1, m) - PC[ax3] * N1I(i_m1, m + 1);
                  if (A[ax3] >= 2) {
                    int A2[3] = {A1[0], A1[1], A1[2]}; A2[ax3]--;
                    int i_m2 = I6(A2[0], A2[1], A2[2], j1, j2, j3);
                    v += 0.5 * (double)(A[ax3] - 1) / comz * (N1I(i_m2, m) - N1I(i_m2, m + 1));
                  }
                  if (B[ax3] >= 1) {
                    int B2[3] = {j1, j2, j3}; B2[ax3]--;
                    int i_b = I6(A1[0], A1[1], A1[2], B2[0], B2[1], B2[2]);
                    v += 0.5 * (double)B[ax3] / comz * (N1I(i_b, m) - N1I(i_b, m + 1));
                  }
                } else {
                  int B1[3] = {j1, j2, j3}; B1[ax3]--;
                  int i_m1 = I6(i1, i2, i3, B1[0], B1[1], B1[2]);
                  v = PB[ax3] * N1I(i_m1, m) - PC[ax3] * N1I(i_m1, m + 1);
                  if (B[ax3] >= 2) {
                    int B2[3] = {B1[0], B1[1], B1[2]}; B2[ax3]--;
                    int i_m2 = I6(i1, i2, i3, B2[0], B2[1], B2[2]);
                    v += 0.5 * (double)(B[ax3] - 1) / comz * (N1I(i_m2, m) - N1I(i_m2, m + 1));
                  }
                }
                N1I(idx, m) = v;
              }
              N2[idx] += N1I(idx, 0);
            }
          }
        }
        for (int i1 = 0; i1 <= LI; ++i1)
        for (int i2 = 0; i2 <= LI - i1; ++i2)
        for (int i3 = 0; i3 <= LI - i1 - i2; ++i3)
        for (int j1 = 0; j1 <= LJ; ++j1)
        for (int j2 = 0; j2 <= LJ - j1; ++j2)
        for (int j3 = 0; j3 <= LJ - j1 - j2; ++j3) {
          int pi = PSH(&sm, I, i1, i2, i3), pj = PSH(&sm, J, j1, j2, j3);
          n_p[(size_t)pi + (size_t)npgs * pj + pp * cell] = N2[I6(i1, i2, i3, j1, j2, j3)];
        }
      }
    }
  }
#undef N1I
  return PFE_OK;
}

/* ------------------------------------------------------- helical density rotation
 *
 * oracle_form_p2h: the primitive half of FORM_C2H (src/pbasis.f90:134-413):
 * P2H(:,:,J) for J = -NH..NH is the identity, except that every p triple
 * (x,y,z starting at a primitive with PAX=1,PAY=0,PAZ=0 that has a contracted
 * function, src/pbasis.f90:196-218) and every d sextet (PAX=2, :220-253) is
 * rotated by HELIX*J about the x axis.  p2c[i] is the contracted row of
 * primitive i (0-based) or -1 (P2C of :165-180).  Output column-major
 * P2H(npgs,npgs,2*NH+1).  f functions are not restated (the kernels take s, p, d).
 */
void oracle_form_p2h(int32_t npgs, const int32_t *pax, const int32_t *pay, const int32_t *paz, const int32_t *p2c,
                     double helix, int32_t nh, double *p2h) {
  const size_t nn = (size_t)npgs * npgs;
  memset(p2h, 0, sizeof(double) * nn * (size_t)(2 * nh + 1));
  for (int32_t j = -nh; j <= nh; ++j) {
    double *P = p2h + nn * (size_t)(j + nh);
#define P2H(a, b) P[(size_t)(a) + (size_t)npgs * (size_t)(b)]
    for (int32_t i = 0; i < npgs; ++i) P2H(i, i) = 1.0;
    if (helix == 0.0) continue;
    const double ang = helix * (double)j, c = cos(ang), s = sin(ang);
    for (int32_t i = 0; i < npgs; ++i) {   /* P ORBITALS */
      if (!(pax[i] == 1 && pay[i] == 0 && paz[i] == 0) || p2c[i] == -1) continue;
      P2H(i, i) = 1.0;
      P2H(i + 1, i + 1) = c;
      P2H(i + 2, i + 2) = c;
      P2H(i + 1, i + 2) = s;
      P2H(i + 2, i + 1) = -s;
    }
    for (int32_t i = 0; i < npgs; ++i) {   /* D ORBITALS */
      if (!(pax[i] == 2 && pay[i] == 0 && paz[i] == 0) || p2c[i] == -1) continue;
      P2H(i, i) = 1.0;
      P2H(i + 1, i + 1) = c * c;
      P2H(i + 1, i + 2) = s * s;
      P2H(i + 1, i + 4) = 2.0 * c * s;
      P2H(i + 2, i + 1) = s * s;
      P2H(i + 2, i + 2) = c * c;
      P2H(i + 2, i + 4) = -2.0 * c * s;
      P2H(i + 3, i + 3) = c;
      P2H(i + 3, i + 5) = s;
      P2H(i + 4, i + 1) = -c * s;
      P2H(i + 4, i + 2) = c * s;
      P2H(i + 4, i + 4) = c * c - s * s;
      P2H(i + 5, i + 3) = -s;
      P2H(i + 5, i + 5) = c;
    }
#undef P2H
  }
}

/*
 * oracle_rotate_density: the P_P_HELIX part of ROTATE_DENSITYMATRIX
 * (src/pdensitymatrix.f90:516-563), in the reference's loop order:
 *   TMP1(I,J) = sum_II P2H(II,I,Q2X) P_P(II,J,Q1X-Q2X)
 *   P_P_HELIX(I,J,Q2X,Q1X) = sum_JJ P2H(JJ,J,Q1X) TMP1(I,JJ)
 * for Q2X in [-CEL2X,CEL2X], Q1X in [-CEL2X-CEL1X, CEL2X+CEL1X] with
 * |Q1X-Q2X| <= CEL1X; every other block is zero.  Layouts (column-major):
 * P_P(npgs,npgs,-cel1x:cel1x) (the x cells of a 1-D chain), P2H(npgs,npgs,
 * -(cel2x+cel1x):+), P_P_HELIX(npgs,npgs,-cel2x:cel2x,-(cel2x+cel1x):+).
 */
void oracle_rotate_density(int32_t npgs, int32_t cel1x, int32_t cel2x, const double *p2h, const double *p_p,
                           double *p_p_helix) {
  const size_t nn = (size_t)npgs * npgs;
  const int32_t h3 = cel1x + cel2x, n2 = 2 * cel2x + 1;
  double *tmp1 = malloc(sizeof(double) * nn);
  memset(p_p_helix, 0, sizeof(double) * nn * (size_t)n2 * (size_t)(2 * h3 + 1));
  for (int32_t q2 = -cel2x; q2 <= cel2x; ++q2)
    for (int32_t q1 = -h3; q1 <= h3; ++q1) {
      if (q1 - q2 < -cel1x || q1 - q2 > cel1x) continue;
      const double *A = p2h + nn * (size_t)(q2 + h3);
      const double *B = p2h + nn * (size_t)(q1 + h3);
      const double *Pq = p_p + nn * (size_t)(q1 - q2 + cel1x);
      double *O = p_p_helix + nn * ((size_t)(q2 + cel2x) + (size_t)n2 * (size_t)(q1 + h3));
      for (int32_t i = 0; i < npgs; ++i)
        for (int32_t j = 0; j < npgs; ++j) {
          double t = 0.0;
          for (int32_t ii = 0; ii < npgs; ++ii) t += A[ii + (size_t)npgs * i] * Pq[ii + (size_t)npgs * j];
          tmp1[i + (size_t)npgs * j] = t;
        }
      for (int32_t i = 0; i < npgs; ++i)
        for (int32_t j = 0; j < npgs; ++j) {
          double t = 0.0;
          for (int32_t jj = 0; jj < npgs; ++jj) t += B[jj + (size_t)npgs * j] * tmp1[i + (size_t)npgs * jj];
          O[i + (size_t)npgs * j] = t;
        }
    }
  free(tmp1);
}
