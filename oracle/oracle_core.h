/*
 * oracle_core.h -- CPU restatement of SALMON's (v1.2.1, ARTED periodic code)
 * real-time hot path.  TEST INFRASTRUCTURE ONLY: this is the checker that the
 * CUDA path is compared against, and the CPU baseline that the benchmark times.
 * Nothing in the shipped library links or calls it.
 *
 * Every routine follows the reference line by line (file:line relative to the
 * SALMON source tree) and keeps its loop order, so that the arithmetic matches
 * the reference up to compiler contraction.  Build with -ffp-contract=off and
 * -fcx-fortran-rules (Fortran complex multiply/divide semantics).
 *
 * Layout (Fortran column-major, 0-based in C):
 *   grid index i = iz + NLz*(iy + NLy*ix)            (preparation/init.f90:20-30)
 *   zu[(ik-NK_s)*nb*NL + ib*NL + i]                  zu(NL,nb,NK_s:NK_e)
 *   kAc[d*NK + ik]                                   kAc(NK,3)
 *   zproj[((ik-NK_s)*Nlma + ilma)*Nps + j]           zproj(Nps,Nlma,NK_s:NK_e)
 */
#ifndef SALMON_ORACLE_CORE_H
#define SALMON_ORACLE_CORE_H

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../include/salmon_gpu.h"

typedef double complex zc;

/* Packed projector tables built like init_projector
 * (modules/opt_variables.f90:233-265): idx_proj holds the 0-based grid index of
 * every sphere point, atom by atom; pseudo_start_idx(ia) is the packed offset
 * of atom ia; nprojector(ia) and idx_lma(ia) give the projectors of atom ia,
 * which the reference assumes are numbered consecutively atom by atom. */
typedef struct orc_proj {
  int NPI;
  int* idx_proj;          /* [NPI] */
  int* pseudo_start_idx;  /* [NI]  */
  int* nprojector;        /* [NI]  */
  int* idx_lma;           /* [NI]  */
} orc_proj;

static __inline__ void orc_proj_init(const sgpu_desc* d, orc_proj* p) {
  int NI = d->NI, i, ia, ioffset;
  p->NPI = 0;
  for (ia = 0; ia < NI; ++ia) p->NPI += d->Mps[ia];
  p->idx_proj = (int*)malloc(sizeof(int) * (p->NPI > 0 ? p->NPI : 1));
  p->pseudo_start_idx = (int*)malloc(sizeof(int) * (NI > 0 ? NI : 1));
  p->nprojector = (int*)calloc(NI > 0 ? NI : 1, sizeof(int));
  p->idx_lma = (int*)malloc(sizeof(int) * (NI > 0 ? NI : 1));
  for (i = 0; i < d->Nlma; ++i) p->nprojector[d->a_tbl[i] - 1] += 1;  /* count_if_integer */
  if (NI > 0) p->idx_lma[0] = 0;
  for (ia = 1; ia < NI; ++ia) p->idx_lma[ia] = p->idx_lma[ia - 1] + p->nprojector[ia - 1];
  ioffset = 0;
  for (ia = 0; ia < NI; ++ia) {
    int j;
    p->pseudo_start_idx[ia] = ioffset;
    for (j = 0; j < d->Mps[ia]; ++j) p->idx_proj[ioffset + j] = d->Jxyz[ia * d->Nps + j] - 1; /* zJxyz */
    ioffset += d->Mps[ia];
  }
}

static __inline__ void orc_proj_free(orc_proj* p) {
  free(p->idx_proj); free(p->pseudo_start_idx); free(p->nprojector); free(p->idx_lma);
}

/* lapt(1:12) = lapx(1:4), lapy(1:4), lapz(1:4)   (opt_variables.f90:136-138) */
static __inline__ void orc_lapt(const sgpu_desc* d, double lapt[12]) {
  int n;
  for (n = 0; n < 4; ++n) { lapt[n] = d->lapx[n + 1]; lapt[4 + n] = d->lapy[n + 1]; lapt[8 + n] = d->lapz[n + 1]; }
}

/* nabt(1:12) = k_d * nab_d(1:4)   (common/hpsi.f90:122-124) */
static __inline__ void orc_nabt(const sgpu_desc* d, const double k[3], double nabt[12]) {
  int n;
  for (n = 0; n < 4; ++n) {
    nabt[n] = k[0] * d->nabx[n + 1]; nabt[4 + n] = k[1] * d->naby[n + 1]; nabt[8 + n] = k[2] * d->nabz[n + 1];
  }
}

static __inline__ int orc_mod(int a, int n) { return ((a % n) + n) % n; }

/* hpsi1_RT_stencil(A,B,C,D,E,F)   stencil/F90/hpsi.f90:27-198 (non-blocked,
 * non-"optimized load" branch :162-190).
 *   F = B E + A E - 0.5 v - zI w,
 *   v = sum_{axis,n} C (E(+n)+E(-n)),  w = sum D (E(+n)-E(-n)),  z, then y, then x. */
static __inline__ void orc_stencil_core(int NLx, int NLy, int NLz, double A, const double* B, const double* C,
                               const double* D, const zc* E, zc* F) {
  int ix, iy, iz;
#define E3(x, y, z) E[(z) + NLz * ((y) + NLy * (x))]
  for (ix = 0; ix < NLx; ++ix)
    for (iy = 0; iy < NLy; ++iy)
      for (iz = 0; iz < NLz; ++iz) {
        int zp[5], zm[5], yp[5], ym[5], xp[5], xm[5], n;
        zc v, w, e;
        for (n = 1; n <= 4; ++n) {
          zp[n] = orc_mod(iz + n, NLz); zm[n] = orc_mod(iz - n, NLz);
          yp[n] = orc_mod(iy + n, NLy); ym[n] = orc_mod(iy - n, NLy);
          xp[n] = orc_mod(ix + n, NLx); xm[n] = orc_mod(ix - n, NLx);
        }
        v = (((C[8] * (E3(ix, iy, zp[1]) + E3(ix, iy, zm[1])) + C[9] * (E3(ix, iy, zp[2]) + E3(ix, iy, zm[2]))) +
              C[10] * (E3(ix, iy, zp[3]) + E3(ix, iy, zm[3]))) + C[11] * (E3(ix, iy, zp[4]) + E3(ix, iy, zm[4])));
        w = (((D[8] * (E3(ix, iy, zp[1]) - E3(ix, iy, zm[1])) + D[9] * (E3(ix, iy, zp[2]) - E3(ix, iy, zm[2]))) +
              D[10] * (E3(ix, iy, zp[3]) - E3(ix, iy, zm[3]))) + D[11] * (E3(ix, iy, zp[4]) - E3(ix, iy, zm[4])));
        v = (((C[4] * (E3(ix, yp[1], iz) + E3(ix, ym[1], iz)) + C[5] * (E3(ix, yp[2], iz) + E3(ix, ym[2], iz))) +
              C[6] * (E3(ix, yp[3], iz) + E3(ix, ym[3], iz))) + C[7] * (E3(ix, yp[4], iz) + E3(ix, ym[4], iz))) + v;
        w = (((D[4] * (E3(ix, yp[1], iz) - E3(ix, ym[1], iz)) + D[5] * (E3(ix, yp[2], iz) - E3(ix, ym[2], iz))) +
              D[6] * (E3(ix, yp[3], iz) - E3(ix, ym[3], iz))) + D[7] * (E3(ix, yp[4], iz) - E3(ix, ym[4], iz))) + w;
        v = (((C[0] * (E3(xp[1], iy, iz) + E3(xm[1], iy, iz)) + C[1] * (E3(xp[2], iy, iz) + E3(xm[2], iy, iz))) +
              C[2] * (E3(xp[3], iy, iz) + E3(xm[3], iy, iz))) + C[3] * (E3(xp[4], iy, iz) + E3(xm[4], iy, iz))) + v;
        w = (((D[0] * (E3(xp[1], iy, iz) - E3(xm[1], iy, iz)) + D[1] * (E3(xp[2], iy, iz) - E3(xm[2], iy, iz))) +
              D[2] * (E3(xp[3], iy, iz) - E3(xm[3], iy, iz))) + D[3] * (E3(xp[4], iy, iz) - E3(xm[4], iy, iz))) + w;
        e = E3(ix, iy, iz);
        F[iz + NLz * (iy + NLy * ix)] = ((B[iz + NLz * (iy + NLy * ix)] * e + A * e) - 0.5 * v) - I * w;
      }
#undef E3
}

/* pseudo_pt(ik,zproj,tpsi,htpsi,spseudo,dpseudo)   common/hpsi.f90:163-207.
 * zproj points at zproj(:,:,ik); spseudo/dpseudo are NPI scratch. */
static __inline__ void orc_pseudo_pt(const sgpu_desc* d, const orc_proj* p, double Hxyz, const zc* zproj,
                                 const zc* tpsi, zc* htpsi, zc* spseudo, zc* dpseudo) {
  int ia, ip, i, j;
  for (i = 0; i < p->NPI; ++i) dpseudo[i] = 0.0;
  for (i = 0; i < p->NPI; ++i) spseudo[i] = tpsi[p->idx_proj[i]];         /* gather */
  for (ia = 0; ia < d->NI; ++ia)
    for (ip = 0; ip < p->nprojector[ia]; ++ip) {
      int ilma = p->idx_lma[ia] + ip, ioffset = p->pseudo_start_idx[ia];
      const zc* zp = zproj + (size_t)ilma * d->Nps;
      zc uVpsi = 0.0;
      for (j = 0; j < d->Mps[ia]; ++j) uVpsi = uVpsi + conj(zp[j]) * spseudo[ioffset + j];
      uVpsi = uVpsi * Hxyz * (double)d->iuV[ilma];
      for (j = 0; j < d->Mps[ia]; ++j) dpseudo[ioffset + j] = dpseudo[ioffset + j] + zp[j] * uVpsi;
    }
  for (i = 0; i < p->NPI; ++i) htpsi[p->idx_proj[i]] = htpsi[p->idx_proj[i]] + dpseudo[i];  /* scatter */
}

/* k2lap0_2 and nabt of hpsi_omp_KB_base (common/hpsi.f90:120-124). */
static __inline__ double orc_k2lap0_2(const sgpu_desc* d, const double k[3]) {
  double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
  return (k2 - (d->lapx[0] + d->lapy[0] + d->lapz[0])) * 0.5;
}

static __inline__ void orc_kvec(const sgpu_desc* d, const double* kAc, int ik /*1-based*/, double k[3]) {
  k[0] = kAc[0 * d->NK + ik - 1]; k[1] = kAc[1 * d->NK + ik - 1]; k[2] = kAc[2 * d->NK + ik - 1];
}

/* zfac(n) = (-zI dt)^n / n!   (RT/hamiltonian.f90:46-49) */
static __inline__ void orc_zfac(double dt, zc zfac[4]) {
  int i;
  zfac[0] = -I * dt;
  for (i = 2; i <= 4; ++i) zfac[i - 1] = zfac[i - 2] * (-I * dt) / (double)i;
}

#endif
