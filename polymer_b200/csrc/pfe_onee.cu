// One-electron integrals on the device: S_P and T_P (OVERLAP_KINETIC(0),
// src/ponee.f90:1-160) and N_P (NUCLEAR_ATTRACTION(0), src/ponee.f90:418-603)
// over primitive shells, per lattice cell, with the helical image of the second
// centre.  These are set-up inputs of the Fock build (S_P feeds its pair
// prefactors), computed once per geometry.  One thread per (shell pair, cell);
// the Obara-Saika recursions are those of the reference, the Boys function is
// the same tabulated evaluation as the two-electron kernels.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "pfe_common.cuh"

namespace pfe {

// storage index of a Cartesian power triple of total <= 2 (10 slots)
__device__ __forceinline__ int cidx(int a, int b, int c) {
  // order: 000 001 002 010 011 020 100 101 110 200
  const int s = a * 100 + b * 10 + c;
  switch (s) {
    case 0: return 0;
    case 1: return 1;
    case 2: return 2;
    case 10: return 3;
    case 11: return 4;
    case 20: return 5;
    case 100: return 6;
    case 101: return 7;
    case 110: return 8;
    default: return 9;  // 200
  }
}

struct OneeDev {
  int npgs, npshell, natom;
  const int* p_shell;  // Fortran P_SHELL(npshell,0:4,0:4,0:4), 1-based
  const int* ang;
  const double *x, *y, *z, *zt;
  const int* iatom;
  const double *ax, *ay, *az;
  int cel1[3], cel2[3];
  double period[3], helix;
  const double* boys;  // row-major [T][m]
};

__device__ __forceinline__ int psh(const OneeDev& a, int s, int i1, int i2, int i3) {
  return a.p_shell[s + a.npshell * (i1 + NPOW * (i2 + NPOW * i3))] - 1;
}

__global__ void k_overlap_kinetic(OneeDev a, double* __restrict__ s_p, double* __restrict__ t_p) {
  const int n1x = 2 * a.cel1[0] + 1, n1y = 2 * a.cel1[1] + 1, n1z = 2 * a.cel1[2] + 1;
  const long long total = (long long)a.npshell * a.npshell * n1x * n1y * n1z;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= total) return;
  const int I = (int)(t % a.npshell), J = (int)((t / a.npshell) % a.npshell);
  const long long cell = t / ((long long)a.npshell * a.npshell);
  const int kx = (int)(cell % n1x) - a.cel1[0];
  const int ky = (int)((cell / n1x) % n1y) - a.cel1[1];
  const int kz = (int)(cell / ((long long)n1x * n1y)) - a.cel1[2];
  const double qx = kx * a.period[0], qy = ky * a.period[1], qz = kz * a.period[2];
  const double ang = kx * a.helix, cs = cos(ang), sn = sin(ang);
  const int ii = psh(a, I, 0, 0, 0), jj = psh(a, J, 0, 0, 0);
  const double Ax = a.x[ii], Ay = a.y[ii], Az = a.z[ii];
  const double Bx = a.x[jj] + qx, By = a.y[jj] * cs - a.z[jj] * sn + qy, Bz = a.y[jj] * sn + a.z[jj] * cs + qz;
  const double r = (Ax - Bx) * (Ax - Bx) + (Ay - By) * (Ay - By) + (Az - Bz) * (Az - Bz);
  const double z1 = a.zt[ii] + a.zt[jj], z2 = sqrt(z1 * z1 * z1), gzi = a.zt[ii] * a.zt[jj] / z1;
  const double pisub = sqrt(REF_PI * REF_PI * REF_PI);
  double S1[10][10], T1[10][10];
  S1[0][0] = pisub / z2 * exp(-gzi * r);
  T1[0][0] = gzi * (3.0 - 2.0 * gzi * r) * S1[0][0];
  const double Px = (Ax * a.zt[ii] + Bx * a.zt[jj]) / z1, Py = (Ay * a.zt[ii] + By * a.zt[jj]) / z1,
               Pz = (Az * a.zt[ii] + Bz * a.zt[jj]) / z1;
  const double PA[3] = {Px - Ax, Py - Ay, Pz - Az}, PB[3] = {Px - Bx, Py - By, Pz - Bz};
  const int LI = a.ang[I], LJ = a.ang[J];
  for (int i1 = 0; i1 <= LI; ++i1)
    for (int i2 = 0; i2 <= LI - i1; ++i2)
      for (int i3 = 0; i3 <= LI - i1 - i2; ++i3)
        for (int j1 = 0; j1 <= LJ; ++j1)
          for (int j2 = 0; j2 <= LJ - j1; ++j2)
            for (int j3 = 0; j3 <= LJ - j1 - j2; ++j3) {
              if (i1 + i2 + i3 + j1 + j2 + j3 == 0) continue;
              int A[3] = {i1, i2, i3}, B[3] = {j1, j2, j3};
              int ax = -1;
              bool onA = false;
              for (int k = 0; k < 3 && ax < 0; ++k) if (A[k] >= 1) { ax = k; onA = true; }
              for (int k = 0; k < 3 && ax < 0; ++k) if (B[k] >= 1) { ax = k; onA = false; }
              const int ci = cidx(i1, i2, i3), cj = cidx(j1, j2, j3);
              if (onA) {
                int A1[3] = {i1, i2, i3};
                A1[ax]--;
                const int c1 = cidx(A1[0], A1[1], A1[2]);
                double s = PA[ax] * S1[c1][cj];
                double sm2 = 0.0, tm2 = 0.0, sb = 0.0, tb = 0.0;
                if (A[ax] >= 2) {
                  int A2[3] = {A1[0], A1[1], A1[2]};
                  A2[ax]--;
                  const int c2 = cidx(A2[0], A2[1], A2[2]);
                  sm2 = S1[c2][cj];
                  tm2 = T1[c2][cj];
                  s += 0.5 * (double)(A[ax] - 1) / z1 * sm2;
                }
                if (B[ax] >= 1) {
                  int B2[3] = {j1, j2, j3};
                  B2[ax]--;
                  const int cb = cidx(B2[0], B2[1], B2[2]);
                  sb = S1[c1][cb];
                  tb = T1[c1][cb];
                  s += 0.5 * (double)B[ax] / z1 * sb;
                }
                S1[ci][cj] = s;
                double tv = 2.0 * gzi * s + PA[ax] * T1[c1][cj];
                if (A[ax] >= 2) tv += 0.5 * (double)(A[ax] - 1) / z1 * tm2 - (double)(A[ax] - 1) * gzi / a.zt[ii] * sm2;
                if (B[ax] >= 1) tv += 0.5 * (double)B[ax] / z1 * tb;
                T1[ci][cj] = tv;
              } else {
                int B1[3] = {j1, j2, j3};
                B1[ax]--;
                const int c1 = cidx(B1[0], B1[1], B1[2]);
                double s = PB[ax] * S1[ci][c1];
                double sm2 = 0.0, tm2 = 0.0;
                if (B[ax] >= 2) {
                  int B2[3] = {B1[0], B1[1], B1[2]};
                  B2[ax]--;
                  const int c2 = cidx(B2[0], B2[1], B2[2]);
                  sm2 = S1[ci][c2];
                  tm2 = T1[ci][c2];
                  s += 0.5 * (double)(B[ax] - 1) / z1 * sm2;
                }
                S1[ci][cj] = s;
                double tv = 2.0 * gzi * s + PB[ax] * T1[ci][c1];
                if (B[ax] >= 2) tv += 0.5 * (double)(B[ax] - 1) / z1 * tm2 - (double)(B[ax] - 1) * gzi / a.zt[jj] * sm2;
                T1[ci][cj] = tv;
              }
            }
  const size_t pp = (size_t)a.npgs * a.npgs;
  for (int i1 = 0; i1 <= LI; ++i1)
    for (int i2 = 0; i2 <= LI - i1; ++i2)
      for (int i3 = 0; i3 <= LI - i1 - i2; ++i3)
        for (int j1 = 0; j1 <= LJ; ++j1)
          for (int j2 = 0; j2 <= LJ - j1; ++j2)
            for (int j3 = 0; j3 <= LJ - j1 - j2; ++j3) {
              const size_t o = (size_t)psh(a, I, i1, i2, i3) + (size_t)a.npgs * psh(a, J, j1, j2, j3) + pp * cell;
              s_p[o] = S1[cidx(i1, i2, i3)][cidx(j1, j2, j3)];
              t_p[o] = T1[cidx(i1, i2, i3)][cidx(j1, j2, j3)];
            }
}

__global__ void k_nuclear(OneeDev a, double* __restrict__ n_p) {
  const int n1x = 2 * a.cel1[0] + 1, n1y = 2 * a.cel1[1] + 1, n1z = 2 * a.cel1[2] + 1;
  const long long total = (long long)a.npshell * a.npshell * n1x * n1y * n1z;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= total) return;
  const int I = (int)(t % a.npshell), J = (int)((t / a.npshell) % a.npshell);
  const long long cell = t / ((long long)a.npshell * a.npshell);
  const int k1x = (int)(cell % n1x) - a.cel1[0];
  const int k1y = (int)((cell / n1x) % n1y) - a.cel1[1];
  const int k1z = (int)(cell / ((long long)n1x * n1y)) - a.cel1[2];
  const double q1x = k1x * a.period[0], q1y = k1y * a.period[1], q1z = k1z * a.period[2];
  const double ang = k1x * a.helix, cs = cos(ang), sn = sin(ang);
  const int ii = psh(a, I, 0, 0, 0), jj = psh(a, J, 0, 0, 0);
  const double Ax = a.x[ii], Ay = a.y[ii], Az = a.z[ii];
  const double Bx = a.x[jj] + q1x, By = a.y[jj] * cs - a.z[jj] * sn + q1y, Bz = a.y[jj] * sn + a.z[jj] * cs + q1z;
  const double comz = a.zt[ii] + a.zt[jj];
  const double Px = (Ax * a.zt[ii] + Bx * a.zt[jj]) / comz, Py = (Ay * a.zt[ii] + By * a.zt[jj]) / comz,
               Pz = (Az * a.zt[ii] + Bz * a.zt[jj]) / comz;
  const double r = (Ax - Bx) * (Ax - Bx) + (Ay - By) * (Ay - By) + (Az - Bz) * (Az - Bz);
  const double sab = sqrt(REF_PI * REF_PI * REF_PI) / sqrt(comz * comz * comz) * exp(-a.zt[ii] * a.zt[jj] / comz * r);
  const double e1 = 2.0 / sqrt(REF_PI) * sqrt(comz) * sab;
  const double PA[3] = {Px - Ax, Py - Ay, Pz - Az}, PB[3] = {Px - Bx, Py - By, Pz - Bz};
  const int LI = a.ang[I], LJ = a.ang[J];
  double N1[10][10][5];
  double N2[10][10];
  for (int x = 0; x < 10; ++x)
    for (int y = 0; y < 10; ++y) N2[x][y] = 0.0;
  for (int k2x = -a.cel2[0]; k2x <= a.cel2[0]; ++k2x)
    for (int k2y = -a.cel2[1]; k2y <= a.cel2[1]; ++k2y)
      for (int k2z = -a.cel2[2]; k2z <= a.cel2[2]; ++k2z) {
        const double q2x = k2x * a.period[0], q2y = k2y * a.period[1], q2z = k2z * a.period[2];
        const double ang2 = k2x * a.helix, cs2 = cos(ang2), sn2 = sin(ang2);
        for (int k = 0; k < a.natom; ++k) {
          const double e2 = -(double)a.iatom[k] * e1;
          const double Cx = a.ax[k] + q2x, Cy = a.ay[k] * cs2 - a.az[k] * sn2 + q2y, Cz = a.ay[k] * sn2 + a.az[k] * cs2 + q2z;
          const double T = comz * ((Px - Cx) * (Px - Cx) + (Py - Cy) * (Py - Cy) + (Pz - Cz) * (Pz - Cz));
          const double PC[3] = {Px - Cx, Py - Cy, Pz - Cz};
          double F[5];
          switch (LI + LJ) {
            case 0: boys_tab<0>(T, e2, a.boys, F); break;
            case 1: boys_tab<1>(T, e2, a.boys, F); break;
            case 2: boys_tab<2>(T, e2, a.boys, F); break;
            case 3: boys_tab<3>(T, e2, a.boys, F); break;
            default: boys_tab<4>(T, e2, a.boys, F); break;
          }
          for (int m = 0; m <= LI + LJ; ++m) N1[0][0][m] = F[m];
          N2[0][0] += N1[0][0][0];
          for (int i1 = 0; i1 <= LI; ++i1)
            for (int i2 = 0; i2 <= LI - i1; ++i2)
              for (int i3 = 0; i3 <= LI - i1 - i2; ++i3)
                for (int j1 = 0; j1 <= LJ; ++j1)
                  for (int j2 = 0; j2 <= LJ - j1; ++j2)
                    for (int j3 = 0; j3 <= LJ - j1 - j2; ++j3) {
                      const int mmax = LI + LJ - i1 - i2 - i3 - j1 - j2 - j3;
                      if (i1 + i2 + i3 + j1 + j2 + j3 == 0 || mmax < 0) continue;
                      int A[3] = {i1, i2, i3}, B[3] = {j1, j2, j3};
                      int ax = -1;
                      bool onA = false;
                      for (int q = 0; q < 3 && ax < 0; ++q) if (A[q] >= 1) { ax = q; onA = true; }
                      for (int q = 0; q < 3 && ax < 0; ++q) if (B[q] >= 1) { ax = q; onA = false; }
                      const int ci = cidx(i1, i2, i3), cj = cidx(j1, j2, j3);
                      for (int m = 0; m <= mmax; ++m) {
                        double v;
                        if (onA) {
                          int A1[3] = {i1, i2, i3};
                          A1[ax]--;
                          const int c1 = cidx(A1[0], A1[1], A1[2]);
                          v = PA[ax] * N1[c1][cj][m] - PC[ax] * N1[c1][cj][m + 1];
                          if (A[ax] >= 2) {
                            int A2[3] = {A1[0], A1[1], A1[2]};
                            A2[ax]--;
                            const int c2 = cidx(A2[0], A2[1], A2[2]);
                            v += 0.5 * (double)(A[ax] - 1) / comz * (N1[c2][cj][m] - N1[c2][cj][m + 1]);
                          }
                          if (B[ax] >= 1) {
                            int B2[3] = {j1, j2, j3};
                            B2[ax]--;
                            const int cb = cidx(B2[0], B2[1], B2[2]);
                            v += 0.5 * (double)B[ax] / comz * (N1[c1][cb][m] - N1[c1][cb][m + 1]);
                          }
                        } else {
                          int B1[3] = {j1, j2, j3};
                          B1[ax]--;
                          const int c1 = cidx(B1[0], B1[1], B1[2]);
                          v = PB[ax] * N1[ci][c1][m] - PC[ax] * N1[ci][c1][m + 1];
                          if (B[ax] >= 2) {
                            int B2[3] = {B1[0], B1[1], B1[2]};
                            B2[ax]--;
                            const int c2 = cidx(B2[0], B2[1], B2[2]);
                            v += 0.5 * (double)(B[ax] - 1) / comz * (N1[ci][c2][m] - N1[ci][c2][m + 1]);
                          }
                        }
                        N1[ci][cj][m] = v;
                      }
                      N2[ci][cj] += N1[ci][cj][0];
                    }
        }
      }
  const size_t pp = (size_t)a.npgs * a.npgs;
  for (int i1 = 0; i1 <= LI; ++i1)
    for (int i2 = 0; i2 <= LI - i1; ++i2)
      for (int i3 = 0; i3 <= LI - i1 - i2; ++i3)
        for (int j1 = 0; j1 <= LJ; ++j1)
          for (int j2 = 0; j2 <= LJ - j1; ++j2)
            for (int j3 = 0; j3 <= LJ - j1 - j2; ++j3)
              n_p[(size_t)psh(a, I, i1, i2, i3) + (size_t)a.npgs * psh(a, J, j1, j2, j3) + pp * cell] =
                  N2[cidx(i1, i2, i3)][cidx(j1, j2, j3)];
}

template <typename T>
static int upload(std::vector<void*>& owned, const T* h, size_t n, T** d) {
  PFE_CUDA(cudaMalloc((void**)d, sizeof(T) * (n ? n : 1)));
  owned.push_back(*d);
  PFE_CUDA(cudaMemcpy(*d, h, sizeof(T) * n, cudaMemcpyHostToDevice));
  return PFE_OK;
}

// Host-side checks shared by the one-electron entry points, made before any
// device work: the kernels index S_P/T_P/N_P by P_SHELL of every component a
// shell reaches (i1+i2+i3 <= P_SHELL_ANG) and by the shell head P_SHELL(s,0,0,0),
// so each of those entries must name a primitive 1..NPGS.  `need_atoms`: the
// allocating entry point uploads the atom list and the Boys table as well.
static int onee_validate(const pfe_onee_args* a, bool need_atoms) {
  if (!a || a->npgs <= 0 || a->npshell <= 0 || (need_atoms && a->natom <= 0)) {
    set_error("invalid one-electron arguments");
    return PFE_EINVAL;
  }
  if (!a->p_shell || !a->p_shell_ang || !a->pgsx || !a->pgsy || !a->pgsz || !a->zt ||
      (need_atoms && (!a->iatom || !a->atomx || !a->atomy || !a->atomz || !a->igamma))) {
    set_error("a required one-electron array pointer is null");
    return PFE_EINVAL;
  }
  for (int k = 0; k < 3; ++k)
    if (a->cel1[k] < 0 || a->cel2[k] < 0) { set_error("negative cutoff"); return PFE_EINVAL; }
  for (int s = 0; s < a->npshell; ++s) {
    const int L = a->p_shell_ang[s];
    if (L < 0 || L > LMAX_SUPPORTED) {
      set_error("P_SHELL_ANG outside the one-electron kernels (s, p, d)");
      return L < 0 ? PFE_EINVAL : PFE_EUNSUPPORTED;
    }
    for (int i1 = 0; i1 <= L; ++i1)
      for (int i2 = 0; i2 <= L - i1; ++i2)
        for (int i3 = 0; i3 <= L - i1 - i2; ++i3) {
          const int p = a->p_shell[(size_t)s + (size_t)a->npshell * (i1 + NPOW * (i2 + NPOW * i3))];
          if (p < 1 || p > a->npgs) {
            char msg[160];
            std::snprintf(msg, sizeof msg, "P_SHELL(%d,%d,%d,%d) = %d is not a primitive 1..NPGS (%d)", s + 1, i1, i2,
                          i3, p, a->npgs);
            set_error(msg);
            return PFE_EINVAL;
          }
        }
  }
  return PFE_OK;
}

static int onee_run(const pfe_onee_args* a, double* s_p, double* t_p, double* n_p) {
  if (const int v = onee_validate(a, true)) return v;
  std::vector<void*> owned;
  OneeDev d{};
  int rc = PFE_OK;
  const size_t psz = (size_t)a->npshell * NPOW * NPOW * NPOW;
  const int n1 = (2 * a->cel1[0] + 1) * (2 * a->cel1[1] + 1) * (2 * a->cel1[2] + 1);
  const size_t out_n = (size_t)a->npgs * a->npgs * n1;
  double *ds = nullptr, *dt = nullptr, *dn = nullptr;
  std::vector<double> tab((size_t)NIG_T * NIG_M);
  for (int t = 0; t < NIG_T; ++t)
    for (int m = 0; m < NIG_M; ++m) tab[(size_t)t * NIG_M + m] = a->igamma[t + (size_t)NIG_T * m];
  int* dps = nullptr; int* dang = nullptr; int* diat = nullptr;
  double *dx = nullptr, *dy = nullptr, *dz = nullptr, *dzt = nullptr, *dax = nullptr, *day = nullptr, *daz = nullptr, *dboys = nullptr;
  if ((rc = upload(owned, a->p_shell, psz, &dps)) || (rc = upload(owned, a->p_shell_ang, (size_t)a->npshell, &dang)) ||
      (rc = upload(owned, a->pgsx, (size_t)a->npgs, &dx)) || (rc = upload(owned, a->pgsy, (size_t)a->npgs, &dy)) ||
      (rc = upload(owned, a->pgsz, (size_t)a->npgs, &dz)) || (rc = upload(owned, a->zt, (size_t)a->npgs, &dzt)) ||
      (rc = upload(owned, a->iatom, (size_t)a->natom, &diat)) || (rc = upload(owned, a->atomx, (size_t)a->natom, &dax)) ||
      (rc = upload(owned, a->atomy, (size_t)a->natom, &day)) || (rc = upload(owned, a->atomz, (size_t)a->natom, &daz)) ||
      (rc = upload(owned, tab.data(), tab.size(), &dboys)))
    goto done;
  d.npgs = a->npgs; d.npshell = a->npshell; d.natom = a->natom;
  d.p_shell = dps; d.ang = dang; d.x = dx; d.y = dy; d.z = dz; d.zt = dzt;
  d.iatom = diat; d.ax = dax; d.ay = day; d.az = daz; d.boys = dboys;
  for (int k = 0; k < 3; ++k) { d.cel1[k] = a->cel1[k]; d.cel2[k] = a->cel2[k]; d.period[k] = a->period[k]; }
  d.helix = a->helix;
  {
    const long long total = (long long)a->npshell * a->npshell * n1;
    const unsigned grid = (unsigned)((total + 127) / 128);
    if (s_p || t_p) {
      if (cudaMalloc(&ds, sizeof(double) * out_n) != cudaSuccess || cudaMalloc(&dt, sizeof(double) * out_n) != cudaSuccess) {
        set_error("cudaMalloc failed");
        rc = PFE_ENOMEM;
        goto done;
      }
      owned.push_back(ds);
      owned.push_back(dt);
      cudaMemset(ds, 0, sizeof(double) * out_n);
      cudaMemset(dt, 0, sizeof(double) * out_n);
      k_overlap_kinetic<<<grid, 128>>>(d, ds, dt);
      if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        set_error("k_overlap_kinetic failed");
        rc = PFE_ECUDA;
        goto done;
      }
      if (s_p) cudaMemcpy(s_p, ds, sizeof(double) * out_n, cudaMemcpyDeviceToHost);
      if (t_p) cudaMemcpy(t_p, dt, sizeof(double) * out_n, cudaMemcpyDeviceToHost);
    }
    if (n_p) {
      if (cudaMalloc(&dn, sizeof(double) * out_n) != cudaSuccess) { set_error("cudaMalloc failed"); rc = PFE_ENOMEM; goto done; }
      owned.push_back(dn);
      cudaMemset(dn, 0, sizeof(double) * out_n);
      k_nuclear<<<grid, 128>>>(d, dn);
      if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
        set_error("k_nuclear failed");
        rc = PFE_ECUDA;
        goto done;
      }
      cudaMemcpy(n_p, dn, sizeof(double) * out_n, cudaMemcpyDeviceToHost);
    }
  }
done:
  for (void* p : owned) cudaFree(p);
  return rc;
}

// ---------------------------------------------------------------- fixed-scratch variant
//
// pfe_overlap_kinetic_noalloc runs k_overlap_kinetic with all of its device
// data (the shell map, centres, exponents and the S_P/T_P results) staged in
// one statically sized device array of this file instead of cudaMalloc'd
// buffers, for callers that may not allocate device memory once they are
// running (a pre-reserved memory budget, a custom allocator that owns the
// device, a process that must not grow its footprint).  Limit: everything must
// fit in kNoAllocScratchBytes (16 MiB), i.e. 2*npgs^2*cells + the inputs; a
// C20H42 6-31G** molecule (976 primitives) fits, larger inputs are refused.

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;          // held for the whole call: calls share the one buffer
static void* g_noalloc_ptr[64] = {nullptr};

static size_t round256(size_t b) { return (b + 255) & ~size_t(255); }

// Device address of the scratch on the current device.  The first call on a
// device does the set-up (loads the module there, looks up the symbol).
static int noalloc_scratch(void** out) {
  int dev = 0;
  PFE_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) { set_error("device index out of range"); return PFE_EINVAL; }
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("cudaGetSymbolAddress of the fixed scratch failed: ") + cudaGetErrorString(e));
      return PFE_ECUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return PFE_OK;
}

static int onee_noalloc(const pfe_onee_args* a, double* s_p, double* t_p) {
  if (!s_p || !t_p) { set_error("invalid one-electron arguments"); return PFE_EINVAL; }
  if (const int v = onee_validate(a, false)) return v;
  const long long n1 = (long long)(2 * a->cel1[0] + 1) * (2 * a->cel1[1] + 1) * (2 * a->cel1[2] + 1);
  const size_t out_n = (size_t)a->npgs * a->npgs * n1;
  const size_t psz = (size_t)a->npshell * NPOW * NPOW * NPOW;
  // scratch layout: S_P | T_P | x | y | z | zt | P_SHELL | P_SHELL_ANG
  const size_t b_out = round256(sizeof(double) * out_n), b_pg = round256(sizeof(double) * a->npgs);
  const size_t b_ps = round256(sizeof(int) * psz), b_ang = round256(sizeof(int) * a->npshell);
  const size_t need = 2 * b_out + 4 * b_pg + b_ps + b_ang;
  if (need > kNoAllocScratchBytes) {
    char msg[256];
    std::snprintf(msg, sizeof msg,
                  "pfe_overlap_kinetic_noalloc: needs %zu bytes of device scratch, the fixed buffer holds %zu "
                  "(npgs %d, %lld cells); use pfe_overlap_kinetic",
                  need, kNoAllocScratchBytes, a->npgs, n1);
    set_error(msg);
    return PFE_EINVAL;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  void* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc != PFE_OK) return rc;
  unsigned char* p = static_cast<unsigned char*>(base);
  double* ds = reinterpret_cast<double*>(p);
  double* dt = reinterpret_cast<double*>(p + b_out);
  double* dx = reinterpret_cast<double*>(p + 2 * b_out);
  double* dy = reinterpret_cast<double*>(p + 2 * b_out + b_pg);
  double* dz = reinterpret_cast<double*>(p + 2 * b_out + 2 * b_pg);
  double* dzt = reinterpret_cast<double*>(p + 2 * b_out + 3 * b_pg);
  int* dps = reinterpret_cast<int*>(p + 2 * b_out + 4 * b_pg);
  int* dang = reinterpret_cast<int*>(p + 2 * b_out + 4 * b_pg + b_ps);
  PFE_CUDA(cudaMemcpy(dx, a->pgsx, sizeof(double) * a->npgs, cudaMemcpyHostToDevice));
  PFE_CUDA(cudaMemcpy(dy, a->pgsy, sizeof(double) * a->npgs, cudaMemcpyHostToDevice));
  PFE_CUDA(cudaMemcpy(dz, a->pgsz, sizeof(double) * a->npgs, cudaMemcpyHostToDevice));
  PFE_CUDA(cudaMemcpy(dzt, a->zt, sizeof(double) * a->npgs, cudaMemcpyHostToDevice));
  PFE_CUDA(cudaMemcpy(dps, a->p_shell, sizeof(int) * psz, cudaMemcpyHostToDevice));
  PFE_CUDA(cudaMemcpy(dang, a->p_shell_ang, sizeof(int) * a->npshell, cudaMemcpyHostToDevice));
  // S_P/T_P entries of primitives that no shell component reaches stay zero,
  // as with the allocating entry point: clear both results first
  PFE_CUDA(cudaMemset(ds, 0, sizeof(double) * out_n));
  PFE_CUDA(cudaMemset(dt, 0, sizeof(double) * out_n));
  OneeDev d{};
  d.npgs = a->npgs; d.npshell = a->npshell; d.natom = a->natom;
  d.p_shell = dps; d.ang = dang; d.x = dx; d.y = dy; d.z = dz; d.zt = dzt;
  for (int k = 0; k < 3; ++k) { d.cel1[k] = a->cel1[k]; d.cel2[k] = a->cel2[k]; d.period[k] = a->period[k]; }
  d.helix = a->helix;
  const long long total = (long long)a->npshell * a->npshell * n1;
  k_overlap_kinetic<<<(unsigned)((total + 127) / 128), 128>>>(d, ds, dt);
  PFE_CUDA(cudaGetLastError());
  PFE_CUDA(cudaMemcpy(s_p, ds, sizeof(double) * out_n, cudaMemcpyDeviceToHost));
  PFE_CUDA(cudaMemcpy(t_p, dt, sizeof(double) * out_n, cudaMemcpyDeviceToHost));
  return PFE_OK;
}

}  // namespace pfe

extern "C" {
int32_t pfe_overlap_kinetic(const pfe_onee_args* a, double* s_p, double* t_p) { return pfe::onee_run(a, s_p, t_p, nullptr); }
int32_t pfe_nuclear_attraction(const pfe_onee_args* a, double* n_p) { return pfe::onee_run(a, nullptr, nullptr, n_p); }
int32_t pfe_overlap_kinetic_noalloc(const pfe_onee_args* a, double* s_p, double* t_p) { return pfe::onee_noalloc(a, s_p, t_p); }
}
