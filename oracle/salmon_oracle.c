/*
 * salmon_oracle.c -- CPU oracle for the SALMON real-time hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, the smoke check and the benchmark's
 * CPU-baseline leg load this library, and only as the checker or the timed CPU
 * baseline; the shipped CUDA library never calls it.
 *
 * Each exported orc_* routine restates one reference routine (file:line
 * relative to the SALMON 1.2.1 source tree), keeping its loop order.  Layouts
 * are described in oracle_core.h.  Parity of the stencil is pinned against the
 * reference's own compiled AVX kernel (oracle/_ref, built by oracle/Makefile).
 */
#include "oracle_core.h"

#include <omp.h>
#include <stdio.h>

/* fd_coef: Nd-th order central-difference coefficients before the 1/H^2, 1/H
 * scaling (preparation/fd_coef.f90:26-73).  lap/nab are indexed n+Nd, n=-Nd..Nd. */
void orc_fd_coef(int Nd, double* lap, double* nab) {
  int i, j, k, n = Nd;
  double t, s, s0;
  for (i = 0; i < 2 * n + 1; ++i) { lap[i] = 0.0; nab[i] = 0.0; }
  s = 0.0;
  for (i = -n; i <= n; ++i) {
    if (i == 0) continue;
    for (j = -n; j <= n; ++j) {
      if (j == i || j == 0) continue;
      s = s + 1.0 / (double)(i * j);
    }
  }
  lap[n] = s;
  for (j = 1; j <= n; ++j) {
    t = 1.0;
    for (i = -n; i <= n; ++i) { if (i == j) continue; t = t * (j - i); }
    s = 0.0;
    for (k = -n; k <= n; ++k) {
      if (k == j || k == 0) continue;
      s0 = 1.0;
      for (i = -n; i <= n; ++i) { if (i == k || i == j || i == 0) continue; s0 = s0 * (-i); }
      s = s + s0;
    }
    lap[n + j] = 2.0 * s / t;
    lap[n - j] = lap[n + j];
  }
  for (j = 1; j <= n; ++j) {
    t = 1.0;
    for (i = -n; i <= n; ++i) { if (i == j) continue; t = t * (j - i); }
    s = 1.0;
    for (i = -n; i <= n; ++i) { if (i == j || i == 0) continue; s = s * (-i); }
    nab[n + j] = s / t;
    nab[n - j] = -nab[n + j];
  }
}

/* hpsi1_RT_stencil on one orbital (stencil/F90/hpsi.f90:27-198). */
void orc_stencil(const sgpu_desc* d, double A, const double* B, const double* C, const double* D,
                 const zc* E, zc* F) {
  orc_stencil_core(d->NLx, d->NLy, d->NLz, A, B, C, D, E, F);
}

/* update_projector_omp (common/projector.f90:49-79).  Writes ekr (Nps,NI,NK_s:NK_e)
 * if ekr != NULL and zproj (Nps,Nlma,NK_s:NK_e). */
void orc_update_projector(const sgpu_desc* d, const double* kAc, zc* ekr, zc* zproj) {
  int NLy = d->NLy, NLz = d->NLz, nkl = d->NK_e - d->NK_s + 1;
  int ikl;
  zc* e = ekr ? ekr : (zc*)malloc(sizeof(zc) * (size_t)d->Nps * d->NI * nkl);
#pragma omp parallel for
  for (ikl = 0; ikl < nkl; ++ikl) {
    int ik = d->NK_s + ikl, ia, j, ilma;
    double k[3];
    orc_kvec(d, kAc, ik, k);
    for (ia = 0; ia < d->NI; ++ia)
      for (j = 0; j < d->Mps[ia]; ++j) {
        int i = d->Jxyz[ia * d->Nps + j] - 1;
        int lx = i / (NLy * NLz), ly = (i / NLz) % NLy, lz = i % NLz;
        int ix = d->Jxx[ia * d->Nps + j], iy = d->Jyy[ia * d->Nps + j], iz = d->Jzz[ia * d->Nps + j];
        double kr = k[0] * (lx * d->Hx - ix * d->aLx) + k[1] * (ly * d->Hy - iy * d->aLy) +
                    k[2] * (lz * d->Hz - iz * d->aLz);
        e[((size_t)ikl * d->NI + ia) * d->Nps + j] = cexp(I * kr);
      }
    for (ilma = 0; ilma < d->Nlma; ++ilma) {
      int a = d->a_tbl[ilma] - 1;
      for (j = 0; j < d->Mps[a]; ++j)
        zproj[((size_t)ikl * d->Nlma + ilma) * d->Nps + j] =
            conj(e[((size_t)ikl * d->NI + a) * d->Nps + j]) * d->uV[(size_t)ilma * d->Nps + j];
    }
  }
  if (!ekr) free(e);
}

/* hpsi_omp_KB_base (common/hpsi.f90:98-208) for orbital tpsi of k-point ik
 * (1-based).  If ttpsi != NULL it receives H tpsi - Vloc tpsi before the
 * nonlocal part is added (hpsi.f90:131-133, subtraction :144-160). */
static void hpsi_base(const sgpu_desc* d, const orc_proj* p, const double* kAc, const double* Vloc,
                      const zc* zproj, int ik, const zc* tpsi, zc* htpsi, zc* ttpsi, zc* sp, zc* dp) {
  double k[3], nabt[12], lapt[12], A, Hxyz = d->Hx * d->Hy * d->Hz;
  int NL = d->NLx * d->NLy * d->NLz, i;
  orc_kvec(d, kAc, ik, k);
  A = orc_k2lap0_2(d, k);
  orc_nabt(d, k, nabt);
  orc_lapt(d, lapt);
  orc_stencil_core(d->NLx, d->NLy, d->NLz, A, Vloc, lapt, nabt, tpsi, htpsi);
  if (ttpsi)
    for (i = 0; i < NL; ++i) ttpsi[i] = htpsi[i] - Vloc[i] * tpsi[i];
  orc_pseudo_pt(d, p, Hxyz, zproj + (size_t)(ik - d->NK_s) * d->Nlma * d->Nps, tpsi, htpsi, sp, dp);
}

/* hpsi_omp_KB_GS / hpsi_omp_KB_RT on one orbital (common/hpsi.f90:33-96). */
void orc_hpsi(const sgpu_desc* d, const double* kAc, const double* Vloc, const zc* zproj, int ik,
              const zc* tpsi, zc* htpsi, zc* ttpsi) {
  orc_proj p;
  zc *sp, *dp;
  orc_proj_init(d, &p);
  sp = (zc*)malloc(sizeof(zc) * (p.NPI + 1));
  dp = (zc*)malloc(sizeof(zc) * (p.NPI + 1));
  hpsi_base(d, &p, kAc, Vloc, zproj, ik, tpsi, htpsi, ttpsi, sp, dp);
  free(sp); free(dp);
  orc_proj_free(&p);
}

/* hamiltonian(zu,flag_current) (RT/hamiltonian.f90:27-123): OpenMP over the
 * (ik,ib) pairs of ik_table/ib_table, four chained hpsi calls into per-thread
 * scratch, then zu += sum zfac(n) t_n.  nthreads<=0 uses the OpenMP default. */
void orc_hamiltonian(const sgpu_desc* d, const double* kAc, const double* Vloc, const zc* zproj, double dt,
                     zc* zu, int nthreads) {
  int NL = d->NLx * d->NLy * d->NLz, NB = d->NBoccmax, nkl = d->NK_e - d->NK_s + 1, NKB = nkl * NB;
  zc zfac[4];
  orc_proj p;
  orc_zfac(dt, zfac);
  orc_proj_init(d, &p);
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    zc* t = (zc*)malloc(sizeof(zc) * (size_t)NL * 4);
    zc* sp = (zc*)malloc(sizeof(zc) * (p.NPI + 1));
    zc* dp = (zc*)malloc(sizeof(zc) * (p.NPI + 1));
    int ikb;
#pragma omp for schedule(static)
    for (ikb = 0; ikb < NKB; ++ikb) {
      int ik = d->NK_s + ikb / NB, ib = ikb % NB, i;
      zc* z = zu + ((size_t)(ik - d->NK_s) * NB + ib) * NL;
      zc *t1 = t, *t2 = t + NL, *t3 = t + 2 * (size_t)NL, *t4 = t + 3 * (size_t)NL;
      memcpy(t4, z, sizeof(zc) * NL);                                  /* init */
      hpsi_base(d, &p, kAc, Vloc, zproj, ik, t4, t1, NULL, sp, dp);
      hpsi_base(d, &p, kAc, Vloc, zproj, ik, t1, t2, NULL, sp, dp);
      hpsi_base(d, &p, kAc, Vloc, zproj, ik, t2, t3, NULL, sp, dp);
      hpsi_base(d, &p, kAc, Vloc, zproj, ik, t3, t4, NULL, sp, dp);
      for (i = 0; i < NL; ++i)                                         /* update */
        z[i] = z[i] + zfac[0] * t1[i] + zfac[1] * t2[i] + zfac[2] * t3[i] + zfac[3] * t4[i];
    }
    free(t); free(sp); free(dp);
  }
  orc_proj_free(&p);
}

/* psi_rho_impl with Sym=1, reduce (common/psi_rho.f90:93-146, sym1 :181-206):
 * rho(i) = sum_{ik,ib} occ(ib,ik) |zu(i,ib,ik)|^2 in (ik,ib) order.
 * nb = second dimension of zu (NBoccmax in RT, NB in GS); the first NBoccmax
 * bands are summed. */
void orc_psi_rho(const sgpu_desc* d, const zc* zu, int nb, double* rho) {
  int NL = d->NLx * d->NLy * d->NLz, i;
#pragma omp parallel for
  for (i = 0; i < NL; ++i) {
    double r = 0.0;
    int ik, ib;
    for (ik = d->NK_s; ik <= d->NK_e; ++ik)
      for (ib = 0; ib < d->NBoccmax; ++ib) {
        zc z = zu[((size_t)(ik - d->NK_s) * nb + ib) * NL + i];
        r = r + (1.0 * d->occ[(ik - 1) * d->NB + ib]) * (creal(z) * creal(z) + cimag(z) * cimag(z));
      }
    rho[i] = r;
  }
}

/* current_stencil(C,E,F,G,H) (stencil/F90/current.f90:16-115):
 * F,G,H = 2 sum_i Im(conj(E_i) sum_{n=1..4} C_n E_{i+n}) along x, y, z. */
static void current_stencil(int NLx, int NLy, int NLz, const double* C, const zc* E, double* F, double* G,
                            double* H) {
  int ix, iy, iz;
  double f = 0, g = 0, h = 0;
#define E3(x, y, z) E[(z) + NLz * ((y) + NLy * (x))]
  for (ix = 0; ix < NLx; ++ix)
    for (iy = 0; iy < NLy; ++iy)
      for (iz = 0; iz < NLz; ++iz) {
        zc w = conj(E3(ix, iy, iz)), v;
        v = (((C[8] * E3(ix, iy, orc_mod(iz + 1, NLz)) + C[9] * E3(ix, iy, orc_mod(iz + 2, NLz))) +
              C[10] * E3(ix, iy, orc_mod(iz + 3, NLz))) + C[11] * E3(ix, iy, orc_mod(iz + 4, NLz)));
        h = h + cimag(w * v);
        v = (((C[4] * E3(ix, orc_mod(iy + 1, NLy), iz) + C[5] * E3(ix, orc_mod(iy + 2, NLy), iz)) +
              C[6] * E3(ix, orc_mod(iy + 3, NLy), iz)) + C[7] * E3(ix, orc_mod(iy + 4, NLy), iz));
        g = g + cimag(w * v);
        v = (((C[0] * E3(orc_mod(ix + 1, NLx), iy, iz) + C[1] * E3(orc_mod(ix + 2, NLx), iy, iz)) +
              C[2] * E3(orc_mod(ix + 3, NLx), iy, iz)) + C[3] * E3(orc_mod(ix + 4, NLx), iy, iz));
        f = f + cimag(w * v);
      }
#undef E3
  *F = f * 2.0; *G = g * 2.0; *H = h * 2.0;
}

/* current(mode='RT') impl: init + stencil + pseudo_pt per orbital, summed over
 * orbitals before the allreduce (RT/current.f90:106-274).  zproj must have
 * been built for the same kAc (current calls update_projector(kac), :125). */
void orc_current(const sgpu_desc* d, const double* kAc, const zc* zproj, const zc* zu, int nb, double* jav) {
  int NL = d->NLx * d->NLy * d->NLz, nkl = d->NK_e - d->NK_s + 1, NKB = nkl * d->NBoccmax;
  int NLy = d->NLy, NLz = d->NLz;
  double Hxyz = d->Hx * d->Hy * d->Hz, aLxyz = d->aLx * d->aLy * d->aLz, IaLxyz = 1.0 / aLxyz;
  double nabt[12], jxs = 0, jys = 0, jzs = 0;
  double* jo = (double*)malloc(sizeof(double) * 3 * NKB);
  int n, ikb;
  for (n = 0; n < 4; ++n) { nabt[n] = d->nabx[n + 1]; nabt[4 + n] = d->naby[n + 1]; nabt[8 + n] = d->nabz[n + 1]; }
#pragma omp parallel for
  for (ikb = 0; ikb < NKB; ++ikb) {
    int ik = d->NK_s + ikb / d->NBoccmax, ib = ikb % d->NBoccmax, i, ilma, j;
    const zc* z = zu + ((size_t)(ik - d->NK_s) * nb + ib) * NL;
    double occ = d->occ[(ik - 1) * d->NB + ib], k[3], jt = 0, jx, jy, jz, jxt, jyt, jzt;
    orc_kvec(d, kAc, ik, k);
    for (i = 0; i < NL; ++i) jt = jt + creal(z[i]) * creal(z[i]) + cimag(z[i]) * cimag(z[i]);   /* init */
    jx = occ * k[0] * jt; jy = occ * k[1] * jt; jz = occ * k[2] * jt;
    current_stencil(d->NLx, d->NLy, d->NLz, nabt, z, &jxt, &jyt, &jzt);                          /* stencil */
    jx = jx + jxt * occ; jy = jy + jyt * occ; jz = jz + jzt * occ;
    jxt = 0; jyt = 0; jzt = 0;                                                                   /* pseudo_pt */
    for (ilma = 0; ilma < d->Nlma; ++ilma) {
      int ia = d->a_tbl[ilma] - 1;
      const zc* zp = zproj + ((size_t)(ik - d->NK_s) * d->Nlma + ilma) * d->Nps;
      zc uVpsi = 0, uVpsix = 0, uVpsiy = 0, uVpsiz = 0;
      for (j = 0; j < d->Mps[ia]; ++j) {
        int ii = d->Jxyz[ia * d->Nps + j] - 1;
        int lx = ii / (NLy * NLz), ly = (ii / NLz) % NLy, lz = ii % NLz;
        double x = lx * d->Hx - d->Jxx[ia * d->Nps + j] * d->aLx;
        double y = ly * d->Hy - d->Jyy[ia * d->Nps + j] * d->aLy;
        double zz = lz * d->Hz - d->Jzz[ia * d->Nps + j] * d->aLz;
        uVpsi = uVpsi + conj(zp[j]) * z[ii];
        uVpsix = uVpsix + conj(zp[j]) * x * z[ii];
        uVpsiy = uVpsiy + conj(zp[j]) * y * z[ii];
        uVpsiz = uVpsiz + conj(zp[j]) * zz * z[ii];
      }
      uVpsi = uVpsi * Hxyz * (double)d->iuV[ilma];
      uVpsix = uVpsix * Hxyz; uVpsiy = uVpsiy * Hxyz; uVpsiz = uVpsiz * Hxyz;
      jxt = jxt + occ * IaLxyz * 2 * cimag(conj(uVpsix) * uVpsi);
      jyt = jyt + occ * IaLxyz * 2 * cimag(conj(uVpsiy) * uVpsi);
      jzt = jzt + occ * IaLxyz * 2 * cimag(conj(uVpsiz) * uVpsi);
    }
    jo[3 * ikb + 0] = jx * Hxyz * IaLxyz + jxt;
    jo[3 * ikb + 1] = jy * Hxyz * IaLxyz + jyt;
    jo[3 * ikb + 2] = jz * Hxyz * IaLxyz + jzt;
  }
  for (ikb = 0; ikb < NKB; ++ikb) { jxs += jo[3 * ikb]; jys += jo[3 * ikb + 1]; jzs += jo[3 * ikb + 2]; }
  jav[0] = jxs; jav[1] = jys; jav[2] = jzs;
  free(jo);
}

/* total_energy_stencil(A,C,D,E,F) (stencil/F90/total_energy.f90:25-188):
 * F = sum_i conj(E_i) (A E_i - 0.5 v - zI w). */
static zc total_energy_stencil(int NLx, int NLy, int NLz, double A, const double* C, const double* D, const zc* E,
                               zc* scratch) {
  int i, NL = NLx * NLy * NLz;
  zc F = 0;
  double B0 = 0.0;
  (void)B0;
  /* z = A E - 0.5 v - zI w is the hpsi stencil with B = 0; reuse it pointwise. */
  {
    double* Bz = (double*)calloc(NL, sizeof(double));
    orc_stencil_core(NLx, NLy, NLz, A, Bz, C, D, E, scratch);
    free(Bz);
  }
  for (i = 0; i < NL; ++i) F = F + conj(E[i]) * scratch[i];
  return F;
}

/* Ekin_l and Enl_l of Total_Energy_omp, CPU branch
 * (common/total_energy.f90:113-122, :172-203).  Ekin includes occ*|kAc|^2/2. */
void orc_energy_terms(const sgpu_desc* d, const double* kAc, const zc* zu, int nb, double* ekin, double* enl) {
  int NL = d->NLx * d->NLy * d->NLz, nkl = d->NK_e - d->NK_s + 1, NKB = nkl * d->NBoccmax, ikb;
  double Hxyz = d->Hx * d->Hy * d->Hz, lap0_2 = -(d->lapx[0] + d->lapy[0] + d->lapz[0]) * 0.5, lapt[12];
  double* eo = (double*)malloc(sizeof(double) * 2 * NKB);
  zc* ekr = (zc*)malloc(sizeof(zc) * (size_t)d->Nps * d->NI * nkl);
  zc* zproj = (zc*)malloc(sizeof(zc) * (size_t)d->Nps * d->Nlma * nkl);
  double ek = 0, en = 0;
  orc_lapt(d, lapt);
  orc_update_projector(d, kAc, ekr, zproj);
#pragma omp parallel
  {
    zc* scratch = (zc*)malloc(sizeof(zc) * NL);
#pragma omp for
    for (ikb = 0; ikb < NKB; ++ikb) {
      int ik = d->NK_s + ikb / d->NBoccmax, ib = ikb % d->NBoccmax, ilma, j;
      const zc* z = zu + ((size_t)(ik - d->NK_s) * nb + ib) * NL;
      double occ = d->occ[(ik - 1) * d->NB + ib], k[3], nabt[12], e_nl = 0;
      zc tpsum;
      orc_kvec(d, kAc, ik, k);
      orc_nabt(d, k, nabt);
      tpsum = total_energy_stencil(d->NLx, d->NLy, d->NLz, lap0_2, lapt, nabt, z, scratch);
      eo[2 * ikb] = creal(occ * tpsum * Hxyz + occ * (k[0] * k[0] + k[1] * k[1] + k[2] * k[2]) / 2.0);
      for (ilma = 0; ilma < d->Nlma; ++ilma) {
        int ia = d->a_tbl[ilma] - 1;
        zc uVpsi = 0;
        for (j = 0; j < d->Mps[ia]; ++j)
          uVpsi = uVpsi + d->uV[(size_t)ilma * d->Nps + j] * ekr[((size_t)(ik - d->NK_s) * d->NI + ia) * d->Nps + j] *
                              z[d->Jxyz[ia * d->Nps + j] - 1];
        uVpsi = uVpsi * Hxyz;
        e_nl = e_nl + occ * (creal(uVpsi) * creal(uVpsi) + cimag(uVpsi) * cimag(uVpsi)) * d->iuV[ilma];
      }
      eo[2 * ikb + 1] = e_nl;
    }
    free(scratch);
  }
  for (ikb = 0; ikb < NKB; ++ikb) { ek += eo[2 * ikb]; en += eo[2 * ikb + 1]; }
  *ekin = ek; *enl = en;
  free(eo); free(ekr); free(zproj);
}

/* Gram_Schmidt_ompk (GS/Gram_Schmidt.f90:32-55) on zu_GS(NL,NB,NK_s:NK_e). */
void orc_gram_schmidt(const sgpu_desc* d, zc* zu) {
  int NL = d->NLx * d->NLy * d->NLz, NB = d->NB, nkl = d->NK_e - d->NK_s + 1, ikl;
  double Hxyz = d->Hx * d->Hy * d->Hz;
#pragma omp parallel for
  for (ikl = 0; ikl < nkl; ++ikl) {
    int ib, ibt, i;
    for (ib = 0; ib < NB; ++ib) {
      zc* b = zu + ((size_t)ikl * NB + ib) * NL;
      double s;
      for (ibt = 0; ibt < ib; ++ibt) {
        const zc* bt = zu + ((size_t)ikl * NB + ibt) * NL;
        zc zov = 0;
        for (i = 0; i < NL; ++i) zov = zov + conj(bt[i]) * b[i];
        zov = zov * Hxyz;
        for (i = 0; i < NL; ++i) b[i] = b[i] - bt[i] * zov;
      }
      s = 0;
      for (i = 0; i < NL; ++i) s = s + (creal(b[i]) * creal(b[i]) + cimag(b[i]) * cimag(b[i]));
      s = s * Hxyz;
      for (i = 0; i < NL; ++i) b[i] = b[i] / sqrt(s);
    }
  }
}

static double zdot_re(const zc* a, const zc* b, int n) {
  zc s = 0;
  int i;
  for (i = 0; i < n; ++i) s = s + conj(a[i]) * b[i];
  return creal(s);
}
static zc zdot(const zc* a, const zc* b, int n) {
  zc s = 0;
  int i;
  for (i = 0; i < n; ++i) s = s + conj(a[i]) * b[i];
  return s;
}
static double znrm2(const zc* a, int n) {
  double s = 0;
  int i;
  for (i = 0; i < n; ++i) s = s + (creal(a[i]) * creal(a[i]) + cimag(a[i]) * cimag(a[i]));
  return s;
}

/* CG_ompk with skip_gsortho='n' (GS/CG.f90:34-139) on zu_GS(NL,NB,NK_s:NK_e).
 * Writes esp_var(NB, NK_s:NK_e) (before the allreduce) and, if iters != NULL,
 * the number of CG iterations each (ib,ik) ran.  zproj must match kAc. */
void orc_cg(const sgpu_desc* d, const double* kAc, const double* Vloc, const zc* zproj, zc* zu, int ncg,
            double* esp_var, int* iters) {
  const double delta_cg = 1.e-15;
  int NL = d->NLx * d->NLy * d->NLz, NB = d->NB, nkl = d->NK_e - d->NK_s + 1, ikl;
  double Hxyz = d->Hx * d->Hy * d->Hz;
  orc_proj p;
  orc_proj_init(d, &p);
#pragma omp parallel
  {
    zc* w = (zc*)malloc(sizeof(zc) * (size_t)NL * 9);
    zc *xk = w, *hxk = w + NL, *gk = w + 2 * (size_t)NL, *pk = w + 3 * (size_t)NL, *pko = w + 4 * (size_t)NL;
    zc *txk = w + 5 * (size_t)NL, *htpsi = w + 6 * (size_t)NL, *ttpsi = w + 7 * (size_t)NL;
    zc* sp = (zc*)malloc(sizeof(zc) * (p.NPI + 1));
    zc* dp = (zc*)malloc(sizeof(zc) * (p.NPI + 1));
#pragma omp for
    for (ikl = 0; ikl < nkl; ++ikl) {
      int ik = d->NK_s + ikl, ib, ibt, iter, i;
      for (ib = 0; ib < NB; ++ib) {
        zc* u = zu + ((size_t)ikl * NB + ib) * NL;
        double s, xkHxk, gkgk = 0, pkHpk, uk, ev;
        zc zs, cx, cp, xkHpk;
        int it_done = 0;
        for (ibt = 0; ibt < ib; ++ibt) {
          const zc* ut = zu + ((size_t)ikl * NB + ibt) * NL;
          s = zdot_re(ut, u, NL) * Hxyz;           /* s is real(8) in the reference (CG.f90:45,70) */
          for (i = 0; i < NL; ++i) u[i] = u[i] - ut[i] * s;
        }
        s = 1.0 / sqrt(znrm2(u, NL) * Hxyz);
        for (i = 0; i < NL; ++i) xk[i] = u[i] * s;
        hpsi_base(d, &p, kAc, Vloc, zproj, ik, xk, hxk, txk, sp, dp);
        xkHxk = zdot_re(xk, hxk, NL) * Hxyz;
        for (iter = 1; iter <= ncg; ++iter) {
          it_done = iter;
          for (i = 0; i < NL; ++i) gk[i] = (hxk[i] - xkHxk * xk[i]);
          for (ibt = 0; ibt < ib; ++ibt) {
            const zc* ut = zu + ((size_t)ikl * NB + ibt) * NL;
            zs = zdot(ut, gk, NL) * Hxyz;
            for (i = 0; i < NL; ++i) gk[i] = gk[i] - ut[i] * zs;
          }
          s = znrm2(gk, NL) * Hxyz;
          if (iter == 1) {
            for (i = 0; i < NL; ++i) pk[i] = gk[i];
          } else {
            uk = s / gkgk;
            for (i = 0; i < NL; ++i) pk[i] = gk[i] + uk * pk[i];
          }
          gkgk = s;
          zs = zdot(xk, pk, NL) * Hxyz;
          for (i = 0; i < NL; ++i) pko[i] = pk[i] - xk[i] * zs;
          s = 1.0 / sqrt(znrm2(pko, NL) * Hxyz);
          for (i = 0; i < NL; ++i) pko[i] = pko[i] * s;
          hpsi_base(d, &p, kAc, Vloc, zproj, ik, pko, htpsi, ttpsi, sp, dp);
          xkHpk = zdot(xk, htpsi, NL) * Hxyz;
          pkHpk = zdot_re(pko, htpsi, NL) * Hxyz;
          ev = 0.5 * ((xkHxk + pkHpk) - sqrt((xkHxk - pkHpk) * (xkHxk - pkHpk) +
                                             4 * (creal(xkHpk) * creal(xkHpk) + cimag(xkHpk) * cimag(xkHpk))));
          cx = xkHpk / (ev - xkHxk);
          cp = 1.0 / sqrt(1.0 + (creal(cx) * creal(cx) + cimag(cx) * cimag(cx)));
          cx = cx * cp;
          if (fabs(ev - xkHxk) < delta_cg) break;
          for (i = 0; i < NL; ++i) {
            xk[i] = cx * xk[i] + cp * pko[i];
            hxk[i] = cx * hxk[i] + cp * htpsi[i];
            txk[i] = cx * txk[i] + cp * ttpsi[i];
          }
          xkHxk = zdot_re(xk, hxk, NL) * Hxyz;
        }
        s = 1.0 / sqrt(znrm2(xk, NL) * Hxyz);
        for (i = 0; i < NL; ++i) u[i] = xk[i] * s;
        hpsi_base(d, &p, kAc, Vloc, zproj, ik, u, htpsi, ttpsi, sp, dp);
        xkHxk = zdot_re(u, htpsi, NL) * Hxyz;
        {
          double r = 0;
          for (i = 0; i < NL; ++i) {
            zc t = htpsi[i] - xkHxk * u[i];
            r = r + (creal(t) * creal(t) + cimag(t) * cimag(t));
          }
          esp_var[ikl * NB + ib] = sqrt(r * Hxyz) * d->occ[(ik - 1) * d->NB + ib];
        }
        if (iters) iters[ikl * NB + ib] = it_done;
      }
    }
    free(w); free(sp); free(dp);
  }
  orc_proj_free(&p);
}

/* Subspace Hamiltonian of diag_omp, omp_loop='k' (GS/diag.f90:109-117) for
 * k-point ik: za(ib2,ib1) = <u_ib2|H u_ib1> Hxyz for ib2>ib1, conjugate above,
 * real diagonal.  za is (NB,NB) column-major.  The eigen-decomposition
 * (zheev, :118) and the rotation (:120-127) are done by the caller. */
void orc_subspace_h(const sgpu_desc* d, const double* kAc, const double* Vloc, const zc* zproj, const zc* zu,
                    int ik, zc* za) {
  int NL = d->NLx * d->NLy * d->NLz, NB = d->NB, ikl = ik - d->NK_s, ib1;
  double Hxyz = d->Hx * d->Hy * d->Hz;
  orc_proj p;
  orc_proj_init(d, &p);
#pragma omp parallel
  {
    zc* h = (zc*)malloc(sizeof(zc) * NL * 2);
    zc* sp = (zc*)malloc(sizeof(zc) * (p.NPI + 1));
    zc* dp = (zc*)malloc(sizeof(zc) * (p.NPI + 1));
#pragma omp for
    for (ib1 = 0; ib1 < NB; ++ib1) {
      const zc* u1 = zu + ((size_t)ikl * NB + ib1) * NL;
      int ib2;
      hpsi_base(d, &p, kAc, Vloc, zproj, ik, u1, h, h + NL, sp, dp);
      for (ib2 = ib1 + 1; ib2 < NB; ++ib2) {
        za[ib1 * NB + ib2] = zdot(zu + ((size_t)ikl * NB + ib2) * NL, h, NL) * Hxyz;
        za[ib2 * NB + ib1] = conj(za[ib1 * NB + ib2]);
      }
      za[ib1 * NB + ib1] = creal(zdot(u1, h, NL) * Hxyz);
    }
    free(h); free(sp); free(dp);
  }
  orc_proj_free(&p);
}

int orc_max_threads(void) { return omp_get_max_threads(); }
