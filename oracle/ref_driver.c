/*
 * ref_driver.c -- drives SALMON's own hand-vectorised AVX stencils
 * (src/ARTED/stencil/C/AVX/{hpsi,current,total_energy}.c, compiled unchanged
 * from the reference tree by oracle/Makefile into oracle/_ref/).
 *
 * TEST INFRASTRUCTURE ONLY: the reference build pins the oracle's stencil
 * restatement and is the CPU baseline of the benchmark's reference arm.
 *
 * The AVX kernels read Intel-Fortran module variables by their mangled names
 * (stencil/C/interop.h:73-83); this file defines them.  No padding is used
 * (PNLy = NLy), so E/F are plain zu-layout orbitals.  The AVX kernels need NLz
 * even (they step z by two complex numbers) and 32-byte aligned arrays.
 */
#include <omp.h>
#include <stdio.h>

#include "oracle_core.h"

/* Fortran module variables the reference C kernels reference. */
int global_variables_mp_nl_, global_variables_mp_nlx_, global_variables_mp_nly_, global_variables_mp_nlz_;
int opt_variables_mp_pnlx_, opt_variables_mp_pnly_, opt_variables_mp_pnlz_;
int *opt_variables_mp_modx_, *opt_variables_mp_mody_, *opt_variables_mp_modz_;

/* Reference entry points (Fortran calling convention: every argument by reference). */
void hpsi1_rt_stencil_(const double* A, const double* B, const double* C, const double* D, const zc* E, zc* F);
void current_stencil_(const double* C, const zc* E, double* F, double* G, double* H);
void total_energy_stencil_(const double* A, const double* C, const double* D, const zc* E, zc* F);

/* Sets the grid module variables and the modx/mody/modz tables of
 * opt_vars_initialize_p2 (modules/opt_variables.f90:155-167). Returns 0 on
 * success, -1 if NLz is odd (the AVX kernels step z by two). */
int ref_set_grid(int NLx, int NLy, int NLz) {
  int i, Nd = 4;
  if (NLz % 2) return -1;
  global_variables_mp_nlx_ = NLx; global_variables_mp_nly_ = NLy; global_variables_mp_nlz_ = NLz;
  global_variables_mp_nl_ = NLx * NLy * NLz;
  opt_variables_mp_pnlx_ = NLx; opt_variables_mp_pnly_ = NLy; opt_variables_mp_pnlz_ = NLz;
  free(opt_variables_mp_modx_); free(opt_variables_mp_mody_); free(opt_variables_mp_modz_);
  opt_variables_mp_modx_ = (int*)malloc(sizeof(int) * (NLx * 2 + Nd));
  opt_variables_mp_mody_ = (int*)malloc(sizeof(int) * (NLy * 2 + Nd));
  opt_variables_mp_modz_ = (int*)malloc(sizeof(int) * (NLz * 2 + Nd));
  for (i = 0; i < NLx * 2 + Nd; ++i) opt_variables_mp_modx_[i] = i % NLx;
  for (i = 0; i < NLy * 2 + Nd; ++i) opt_variables_mp_mody_[i] = i % NLy;
  for (i = 0; i < NLz * 2 + Nd; ++i) opt_variables_mp_modz_[i] = i % NLz;
  return 0;
}

static zc* aligned_zc(size_t n) {
  void* p = NULL;
  if (posix_memalign(&p, 64, sizeof(zc) * (n ? n : 1))) return NULL;
  return (zc*)p;
}

/* The reference AVX stencil on one orbital (E, F must be 32-byte aligned). */
void ref_stencil(double A, const double* B, const double* C, const double* D, const zc* E, zc* F) {
  hpsi1_rt_stencil_(&A, B, C, D, E, F);
}

void ref_current_stencil(const double* C, const zc* E, double* F, double* G, double* H) {
  current_stencil_(C, E, F, G, H);
}

void ref_total_energy_stencil(double A, const double* C, const double* D, const zc* E, zc* F) {
  total_energy_stencil_(&A, C, D, E, F);
}

/* hamiltonian(zu,flag_current) (RT/hamiltonian.f90:27-123) with the reference's
 * AVX stencil for hpsi1_RT_stencil and the pseudo_pt/update restatements of
 * oracle_core.h; OpenMP over ikb with per-thread scratch zhtpsi(PNL,4)
 * (:53-73).  Processes orbitals ikb_s..ikb_e-1 (0-based) only, so that a
 * bounded sample of a workload can be timed.  ref_set_grid must have been
 * called for desc's grid. */
int ref_hamiltonian(const sgpu_desc* d, const double* kAc, const double* Vloc, const zc* zproj, double dt, zc* zu,
                    int ikb_s, int ikb_e, int nthreads) {
  int NL = d->NLx * d->NLy * d->NLz, NB = d->NBoccmax;
  double lapt[12], Hxyz = d->Hx * d->Hy * d->Hz;
  zc zfac[4];
  orc_proj p;
  if (global_variables_mp_nlx_ != d->NLx || global_variables_mp_nly_ != d->NLy || global_variables_mp_nlz_ != d->NLz)
    return -1;
  orc_zfac(dt, zfac);
  orc_lapt(d, lapt);
  orc_proj_init(d, &p);
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    zc* t = aligned_zc((size_t)NL * 4);
    zc* sp = aligned_zc(p.NPI + 1);
    zc* dp = aligned_zc(p.NPI + 1);
    int ikb;
#pragma omp for schedule(static)
    for (ikb = ikb_s; ikb < ikb_e; ++ikb) {
      int ik = d->NK_s + ikb / NB, ib = ikb % NB, i, n;
      zc* z = zu + ((size_t)(ik - d->NK_s) * NB + ib) * NL;
      zc* tn[5];
      double k[3], nabt[12], A;
      const zc* zp = zproj + (size_t)(ik - d->NK_s) * d->Nlma * d->Nps;
      orc_kvec(d, kAc, ik, k);
      A = orc_k2lap0_2(d, k);
      orc_nabt(d, k, nabt);
      tn[0] = t + 3 * (size_t)NL;                               /* zhtpsi(:,4) holds the input */
      for (n = 1; n <= 4; ++n) tn[n] = t + (size_t)(n - 1) * NL;
      memcpy(tn[0], z, sizeof(zc) * NL);                        /* init */
      for (n = 1; n <= 4; ++n) {
        hpsi1_rt_stencil_(&A, Vloc, lapt, nabt, tn[n - 1], tn[n]);
        orc_pseudo_pt(d, &p, Hxyz, zp, tn[n - 1], tn[n], sp, dp);
      }
      for (i = 0; i < NL; ++i)                                  /* update */
        z[i] = z[i] + zfac[0] * t[i] + zfac[1] * t[NL + i] + zfac[2] * t[2 * (size_t)NL + i] +
               zfac[3] * t[3 * (size_t)NL + i];
    }
    free(t); free(sp); free(dp);
  }
  orc_proj_free(&p);
  return 0;
}

int ref_max_threads(void) { return omp_get_max_threads(); }
