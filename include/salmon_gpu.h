/*
 * salmon_gpu.h -- C ABI of the B200 real-time propagation path for SALMON's
 * periodic (ARTED) code.
 *
 * The entry points replace, one for one, the Fortran routines that SALMON 1.2.1
 * calls on its real-time hot path.  Each declaration names the reference routine
 * (file:line, paths relative to the SALMON source tree) whose argument meaning it
 * keeps.  Arrays use the reference's Fortran (column-major) layout, so a Fortran
 * caller passes its module arrays unchanged through ISO_C_BINDING:
 *
 *   zu(NL, NBoccmax, NK_s:NK_e)   complex(8)  orbital (ib,ik) is contiguous
 *   grid index i = iz + NLz*(iy + NLy*ix)  (z is unit stride; init.f90:20-30)
 *   kAc(NK, 3)                    real(8)     all k-points, column-major
 *   occ(NB, NK)                   real(8)
 *
 * Conventions
 *   - Every call returns 0 on success or a negative sgpu_status; it never aborts.
 *     sgpu_last_error() returns a message for the last failure on this thread.
 *     The Fortran shim maps non-zero to err_finalize (ARTED/main.f90:21-33).
 *   - Pointers marked HOST are host memory; DEV are device memory of the
 *     handle's device.  HOST arrays may be pageable or pinned.
 *   - Calls on one handle are serialised on the handle's CUDA stream.  Calls
 *     that return host results synchronise that stream; the rest are
 *     asynchronous (sgpu_synchronize waits).  A handle must not be used from
 *     two host threads at once.
 *   - Orbitals stay resident on the device between calls, as the reference's
 *     OpenACC build keeps zu_t resident (control/control_sc.f90:133-149).
 */
#ifndef SALMON_GPU_H
#define SALMON_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
typedef enum sgpu_status {
  SGPU_OK = 0,
  SGPU_ERR_ARG = -1,      /* invalid argument or size                  */
  SGPU_ERR_CUDA = -2,     /* CUDA runtime error (message has details)  */
  SGPU_ERR_ALLOC = -3,    /* device allocation failed                  */
  SGPU_ERR_STATE = -4,    /* call out of order (e.g. no state loaded)  */
  SGPU_ERR_UNSUPPORTED = -5,
  SGPU_ERR_TIMEOUT = -6   /* a bounded device wait gave up             */
} sgpu_status;

/* ---- precision modes (sgpu_set_precision) -------------------------------- */
enum {
  SGPU_PREC_C128 = 0,     /* complex(8) orbitals, FP64 everywhere                 */
  SGPU_PREC_C64 = 1       /* complex(4) orbitals and stencils; FP64 reductions    */
};

/*
 * System descriptor.  Mirrors the module data that ARTED builds in
 * fd_coef (preparation/fd_coef.f90:20-83), init (preparation/init.f90:20-109),
 * prep_ps_periodic (preparation/prep_ps.f90:80-204) and
 * opt_vars_initialize_p2 (modules/opt_variables.f90:105-179).
 * All pointer members are HOST and are copied by sgpu_create; the caller may
 * free them afterwards.
 */
typedef struct sgpu_desc {
  /* real-space grid (global_variables.f90:41-50) */
  int32_t NLx, NLy, NLz;
  double Hx, Hy, Hz;          /* grid spacing                          */
  double aLx, aLy, aLz;       /* cell lengths                          */
  /* k-points and bands */
  int32_t NK;                 /* total k-points (first dim of kAc, second of occ) */
  int32_t NK_s, NK_e;         /* 1-based k range held by this handle   */
  int32_t NB;                 /* bands in occ (and in GS arrays)       */
  int32_t NBoccmax;           /* occupied bands propagated in RT       */
  /* Nd=4 finite-difference coefficients, already divided by H^2 and H
   * (fd_coef.f90:75-80).  lap*[n] = lap(n) for n=0..4; nab*[n] = nab(n),
   * nab*[0] is ignored. */
  double lapx[5], lapy[5], lapz[5];
  double nabx[5], naby[5], nabz[5];
  /* Kleinman-Bylander nonlocal part (prep_ps.f90:80-204) */
  int32_t NI;                 /* atoms                                  */
  int32_t Nps;                /* max sphere points per atom             */
  int32_t Nlma;               /* projectors in total                    */
  const int32_t* Mps;         /* (NI)      sphere points of each atom   */
  const int32_t* Jxyz;        /* (Nps,NI)  1-based grid index of point j of atom a */
  const int32_t* Jxx;         /* (Nps,NI)  periodic image of the point  */
  const int32_t* Jyy;         /* (Nps,NI)                               */
  const int32_t* Jzz;         /* (Nps,NI)                               */
  const double* uV;           /* (Nps,Nlma) projector values            */
  const int32_t* iuV;         /* (Nlma)    sign of each projector       */
  const int32_t* a_tbl;       /* (Nlma)    1-based atom of each projector */
  const double* occ;          /* (NB,NK)   occupations                  */
} sgpu_desc;

typedef struct sgpu_system* sgpu_handle;

/* ---- lifetime ------------------------------------------------------------ */

/* The argument checks sgpu_create runs on a descriptor (sizes, the k range,
 * the projector tables' index ranges), on the host only: no device call, so a
 * rank can validate its k-block's descriptor before it touches a GPU.  0 or
 * SGPU_ERR_ARG / SGPU_ERR_UNSUPPORTED with the reason in sgpu_last_error.
 * No reference counterpart (the reference checks its input in read_input). */
int sgpu_check_desc(const sgpu_desc* desc);

/* Builds the device copies of every table in *desc on the current CUDA device
 * and allocates the resident orbital array and Taylor workspace.
 * Replaces: opt_vars_initialize_p2 + init_projector
 * (modules/opt_variables.f90:105-179, :233-265) and the OpenACC
 * `enter data` of control/control_sc.f90:133-149. */
int sgpu_create(const sgpu_desc* desc, int precision, sgpu_handle* out);

/* Frees every device buffer of the handle (opt_vars_finalize). */
int sgpu_destroy(sgpu_handle h);

/* Switches the orbital precision (SGPU_PREC_C128 or SGPU_PREC_C64).
 * Resident orbitals are converted.  No reference counterpart: the reference
 * propagates complex(8) only. */
int sgpu_set_precision(sgpu_handle h, int precision);

/* Message of the last failed call on this host thread (never NULL). */
const char* sgpu_last_error(void);

/* Waits for all work queued on the handle's stream. */
int sgpu_synchronize(sgpu_handle h);

/* The handle's cudaStream_t, for callers that time or order work around it. */
void* sgpu_stream(sgpu_handle h);

/* ---- resident state ------------------------------------------------------ */

/* HOST zu(NL,NBoccmax,NK_s:NK_e) -> device.  Replaces the OpenACC
 * `enter data copyin(zu_t)` / `update device(zu)` (control_sc.f90:149,
 * RT/dt_evolve.f90:530). */
int sgpu_set_state(sgpu_handle h, const double* zu /* complex(8), HOST */);

/* The same from a DEV complex(8) array of the same layout, e.g. zu_t that an
 * OpenACC host keeps on the device (`host_data use_device(zu_t)`); no host
 * round trip. */
int sgpu_set_state_dev(sgpu_handle h, const void* zu_dev);

/* device -> HOST zu.  Replaces `update self(zu_t)` (control_sc.f90:215,395,414). */
int sgpu_get_state(sgpu_handle h, double* zu /* complex(8), HOST */);

/* Device pointer of the resident orbitals (complex(8) or complex(4) per the
 * precision), layout zu(NL,NBoccmax,NK_s:NK_e). */
void* sgpu_state_ptr(sgpu_handle h);

/* HOST Vloc(NL) -> device.  Vloc = Vh + Vpsl + Vexc (RT/dt_evolve.f90:206).
 * The values are copied into the handle's pinned staging before the call returns
 * (the caller's array is free again); the device copy is queued on the handle's
 * stream without waiting for the work before it. */
int sgpu_set_vloc(sgpu_handle h, const double* vloc);

/* HOST Vpsl(NL) -> device: the local pseudopotential that sgpu_update_vloc
 * adds (prep_ps.f90 Vpsl). */
int sgpu_set_vpsl(sgpu_handle h, const double* vpsl);

/* The self-consistent local potential of RT/dt_evolve.f90:190-207:
 * Vloc = Vh[rho] + Vpsl + Vexc[rho] on the device, with Vh from the Poisson
 * equation in reciprocal space (Hartree, common/Hartree.f90:20-130) and Vexc
 * from the Perdew-Zunger LDA (exc_cor_pz, xc/builtin_pz.f90:23-80).  rho is
 * HOST (NL), e.g. after the allreduce of sgpu_psi_rho's rho_l over k-ranks;
 * NULL uses the density of the handle's resident orbitals.  eh_exc (HOST [2],
 * may be NULL) receives the Hartree energy 1/2 sum Vh rho Hxyz and the
 * exchange-correlation energy sum exc rho Hxyz.  Grid sizes must be 2^a 3^b <= 96. */
int sgpu_update_vloc(sgpu_handle h, const double* rho, double* eh_exc);

/* sgpu_update_vloc from a DEV density rho_dev(NL) (e.g. after an allreduce on
 * the device), enqueued on the handle's stream and not waited for; eh_exc_dev
 * (DEV [2], may be NULL) receives the Hartree and XC energies. */
int sgpu_update_vloc_dev(sgpu_handle h, const double* rho_dev, double* eh_exc_dev);

/* device -> HOST Vloc(NL) (FP64). */
int sgpu_get_vloc(sgpu_handle h, double* vloc);

/* The enforced-time-reversal-symmetry (etrs) propagator's potential history on
 * the device.  sgpu_vloc_history_reset sets Vloc_old(:,1) = Vloc_old(:,2) =
 * Vloc at the start of a real-time run (control/control_sc.f90:82).
 * sgpu_vloc_extrapolate, between the two half steps of dt_evolve_etrs_omp_KB,
 * replaces Vloc by 3 Vloc - 3 Vloc_old(:,1) + Vloc_old(:,2) and shifts the
 * history (Vloc_old(:,2) = Vloc_old(:,1), Vloc_old(:,1) = the previous Vloc)
 * (RT/dt_evolve.f90:248-252).  A step of the etrs propagator is then
 *   sgpu_update_projector(kAc(t)); sgpu_hamiltonian(dt/2, 0);
 *   sgpu_vloc_extrapolate; sgpu_update_projector(kAc(t+dt));
 *   sgpu_hamiltonian(dt/2, 1); sgpu_update_vloc(NULL)
 * (RT/dt_evolve.f90:218-348 for the LDA functionals). */
int sgpu_vloc_history_reset(sgpu_handle h);
int sgpu_vloc_extrapolate(sgpu_handle h);

/* ---- hot path ------------------------------------------------------------ */

/* Sets k+A(t) for the following hpsi/hamiltonian calls and rebuilds the
 * k-dependent projectors zproj(j,ilma,ik) = conj(exp(i kAc.r)) uV(j,ilma).
 * kAc is HOST (NK,3), staged like sgpu_set_vloc's input (no stream wait).
 * Replaces update_projector(kac) (common/projector.f90:29-115). */
int sgpu_update_projector(sgpu_handle h, const double* kAc);

/* One 4th-order Taylor step of every resident orbital:
 *   zu <- zu + sum_{n=1..4} ((-i dt)^n / n!) H^n zu,
 * with H built from the last sgpu_update_projector / sgpu_set_vloc.
 * flag_current non-zero also computes the stencil part of the current of the
 * new orbitals (sum |psi|^2 and the current_stencil sums, which do not depend
 * on k+A), as the reference does under ARTED_CURRENT_PREPROCESSING
 * (current_omp_KB_ST after the update, RT/hamiltonian.f90:68-70); a following
 * sgpu_current on the unchanged orbitals uses them instead of re-reading the
 * orbitals (current.f90:154-156, :213-224).
 * Replaces hamiltonian(zu,flag_current) (RT/hamiltonian.f90:27-123). */
int sgpu_hamiltonian(sgpu_handle h, double dt, int flag_current);

/* H applied to one HOST orbital of k-point ik (1-based, NK_s<=ik<=NK_e).
 * tpsi, htpsi are complex(8) (NL).  If ttpsi is not NULL it receives
 * H tpsi - Vloc tpsi.  Replaces hpsi_omp_KB_GS / hpsi_omp_KB_RT
 * (common/hpsi.f90:33-96). */
int sgpu_hpsi(sgpu_handle h, int ik, const double* tpsi, double* htpsi, double* ttpsi);

/* H applied to resident-layout DEV orbitals ikb_s..ikb_e (1-based over the
 * (ib,ik) pairs of ik_table/ib_table, init.f90:101-109).  tpsi and htpsi
 * point at orbital ikb_s of arrays laid out like zu, in the handle's
 * precision.  Replaces hpsi_acc_KB_RT_LBLK (common/acc/hpsi.f90:28). */
int sgpu_hpsi_batch(sgpu_handle h, int ikb_s, int ikb_e, const void* tpsi, void* htpsi);

/* ---- reductions (FP64 in every precision mode) --------------------------- */

/* rho_l(NL) = sum_{k,b} occ(b,k) |zu(:,b,k)|^2 over the resident orbitals,
 * before the allreduce.  HOST output.  Replaces psi_rho_impl with Sym=1
 * (common/psi_rho.f90:47-90, sym1 :181-206). */
int sgpu_psi_rho(sgpu_handle h, double* rho_l);

/* Capacity of the fixed scratch of sgpu_psi_rho_static, in doubles (16 MiB):
 * ceil(nb*nk/64) * NL must not exceed it (e.g. NL = 32^3 with up to 4096
 * orbitals, or NL = 48^3 with up to 1152). */
#define SGPU_PSI_RHO_STATIC_SCRATCH_DOUBLES 2097152

/* rho(NL) = sum_{ik<nk, ib<nb} occ[ib + ld_occ*ik] |zu(:,ib,ik)|^2 (FP64) over
 * orbitals the CALLER keeps on the device: zu(NL,nb,nk) complex(8)
 * (precision SGPU_PREC_C128) or complex(4) (SGPU_PREC_C64), occ and rho
 * device arrays; enqueued on `stream` (a cudaStream_t, NULL = the legacy
 * default stream) and not waited for.  occ is indexed from the caller's first
 * local k-point: a rank holding k-points NK_s..NK_e of the reference's
 * occ(NB,NK) passes the device address of occ(1,NK_s) with ld_occ = NB (in
 * OpenACC Fortran: `!$acc host_data use_device(zu_t, occ, rho)` around the
 * call, with occ(1,NK_s) as the argument).  Needs no handle and allocates no
 * device memory: its scratch is a static device array of
 * SGPU_PSI_RHO_STATIC_SCRATCH_DOUBLES doubles, and larger problems are
 * rejected with SGPU_ERR_ARG.  It is meant for hosts that own the orbitals
 * through their own device runtime and cannot allocate at that point.
 * The scratch address is looked up once per CUDA context
 * (cudaGetSymbolAddress, keyed on the context's ID, so a device reset or a
 * host-created context gets a fresh lookup); the first call in a context may
 * load the library's device code, so make it before capturing any stream.  All calls
 * on one device share the scratch: calls whose executions overlap race, so
 * order them (one stream, or events).
 * No counterpart in the reference; the computation is psi_rho_impl with
 * Sym=1 (common/psi_rho.f90:47-90, sym1 :181-206), like sgpu_psi_rho. */
int sgpu_psi_rho_static(int precision, int NL, int nb, int nk, const void* zu, const double* occ, int ld_occ,
                        double* rho, void* stream);

/* The same density into a DEV array rho_dev(NL) of the handle's device,
 * enqueued on the handle's stream and not waited for: the per-rank density
 * that psi_rho.f90:88 allreduces, left on the device for a collective
 * (ncclAllReduce on the handle's stream) and sgpu_update_vloc_dev. */
int sgpu_psi_rho_dev(sgpu_handle h, double* rho_dev);

/* Macroscopic current of the resident orbitals at k+A = kAc (HOST (NK,3));
 * jav(3) HOST, before the allreduce.  Rebuilds the projectors for kAc, as
 * current() does.  Replaces current('RT',...) impl
 * (RT/current.f90:78-292, current_stencil stencil/F90/current.f90:16-115). */
int sgpu_current(sgpu_handle h, const double* kAc, double* jav);

/* The same current into DEV jav_dev[3], enqueued on the handle's stream and
 * not waited for (the per-rank value that current.f90:286 allreduces). */
int sgpu_current_dev(sgpu_handle h, const double* kAc, double* jav_dev);

/* Kinetic and nonlocal energies of the resident orbitals at kAc (HOST):
 *   Ekin = sum occ (Hxyz <psi|T + kAc.nabla|psi> + |kAc|^2/2),
 *   Enl  = sum occ |<uV e^{ikr}|psi>|^2 iuV.
 * Replaces the Ekin_l / Enl_l part of Total_Energy_omp
 * (common/total_energy.f90:113-203, stencil/F90/total_energy.f90:25-188). */
int sgpu_energy_terms(sgpu_handle h, const double* kAc, double* ekin, double* enl);

/* ---- ground state (FP64 in every precision mode) -------------------------- */

/* HOST zu_GS(NL,NB,NK_s:NK_e) -> device (ground-state orbitals, all NB bands). */
int sgpu_gs_set_state(sgpu_handle h, const double* zu_gs);

/* device -> HOST zu_GS(NL,NB,NK_s:NK_e). */
int sgpu_gs_get_state(sgpu_handle h, double* zu_gs);

/* Gram-Schmidt of the ground-state bands of every k-point, band by band
 * against the lower bands.  Replaces Gram_Schmidt_ompk
 * (GS/Gram_Schmidt.f90:32-55). */
int sgpu_gram_schmidt(sgpu_handle h);

/* ncg band-by-band CG iterations on the ground-state orbitals with the
 * Hamiltonian of the last sgpu_update_projector / sgpu_set_vloc.  esp_var
 * (NB,NK_s:NK_e) HOST receives the residual norms times occ before the
 * allreduce (may be NULL); iters (NB,NK_s:NK_e) HOST the CG iterations run per
 * band (may be NULL).  Replaces CG_ompk (GS/CG.f90:34-139). */
int sgpu_cg(sgpu_handle h, int ncg, double* esp_var, int* iters);

/* CG stops iterating a band once its Rayleigh quotient changes by less than
 * delta_cg between iterations; the reference fixes delta_cg = 1e-15
 * (GS/CG.f90:42, :114), which is also the default here.  A smaller value lets
 * CG drive residual norms below ~1e-7. */
int sgpu_set_cg_delta(sgpu_handle h, double delta_cg);

/* Residual norms sqrt(||H u - <u|H|u> u||^2 Hxyz) of every band after the last
 * sgpu_cg, HOST (NB,NK_s:NK_e), without the occupation factor of esp_var (so
 * empty bands are reported too).  No reference counterpart. */
int sgpu_cg_residuals(sgpu_handle h, double* res);

/* Subspace diagonalisation: H_sub(NB,NB) per k-point, its Hermitian
 * eigen-decomposition (ascending eigenvalues) and the rotation of the bands.
 * esp (NB,NK_s:NK_e) HOST receives the eigenvalues (may be NULL).  Replaces
 * diag_omp (GS/diag.f90:22-173); the eigen-solver is a cyclic Jacobi on the GPU
 * in place of LAPACK zheev. */
int sgpu_subspace_diag(sgpu_handle h, double* esp);

/* zu_t(:,1:NBoccmax,:) = zu_GS(:,1:NBoccmax,:) on the device (the start of the
 * real-time run), converted to the handle's precision. */
int sgpu_gs_to_rt(sgpu_handle h);

/* ---- tuning --------------------------------------------------------------- */
enum {
  SGPU_PARAM_NSLAB = 0,       /* CTAs per orbital along x in the stencil pass (1..NLx)              */
  SGPU_PARAM_LAUNCHES = 1,    /* kernels the handle has launched, modulo 2^31 (read; set 0 to reset) */
  SGPU_PARAM_UVPSI_SPLIT = 2, /* warps splitting the points of one projection tile: 1, 2, 4 or 8     */
  SGPU_PARAM_CG_PRECOND = 3,  /* sgpu_cg direction: SGPU_CG_PLAIN, SGPU_CG_TPA or SGPU_CG_LEARNED     */
  SGPU_PARAM_PASS_TABLES = 4, /* stencil pass: 1 stages Vloc and the sphere-index table of each plane
                                 through shared memory with the plane (where it fits), 0 loads them
                                 from global memory one plane ahead                                   */
  SGPU_PARAM_KB_KERNEL = 5,   /* KB term of H psi: 1 band-group tile kernel (32 bands of a k-point per
                                 CTA, pipelined gathers), 2 band-quad kernel (UVPSI_SPLIT warps per
                                 4 bands), 3 the tile kernel's projections over KB_SPLIT point ranges
                                 then a point-parallel field kernel, 0 the tile kernel for
                                 complex(4) when its grid has >= 2 CTAs per SM, else form 3          */
  SGPU_PARAM_PASS_FIXED = 6,  /* stencil pass, complex(4): 1 uses the compile-time plane shapes
                                 (16x16, 16x32, 20x20, 32x32 planes, 48x48 in three y-blocks: 9-plane
                                 ring, constant offsets) where they fit, 0 the generic kernel         */
  SGPU_PARAM_CUR_FIXED = 7,   /* current and energy stencils on 32x32 and 48x48 planes: 1 the
                                 current's march with two rows per thread (32x32 split over two CTAs,
                                 48x48 over six) and the energy's over four / six CTAs, 2 the
                                 current's march with one row per thread (four / six CTAs), 0 the
                                 generic kernels                                                     */
  SGPU_PARAM_TAYLOR_KERNEL = 8, /* Taylor step: 1 four stencil passes over all orbitals (any grid), 2
                                 the orbitals of a band group resident in one CTA's shared memory for
                                 the whole step (16x16, 16x32 and 20x20 planes where they fit), 0 the
                                 resident form where it is the faster one (16x16 planes), else the
                                 passes                                                              */
  SGPU_PARAM_NSP = 9,         /* sphere points of the handle (read only): the union of the
                                 projectors' points, a key of the launch-shape table              */
  SGPU_PARAM_KB_SPLIT = 10    /* KB_KERNEL 3: point ranges of the projections, 1..8; 0 about six
                                 CTAs per SM                                                         */
};

/* CG preconditioners.  PLAIN is the reference's CG_ompk.  TPA multiplies the
 * gradient in reciprocal space by the Teter-Payne-Allan kinetic-energy factor
 * (Phys. Rev. B 40, 12255 (1989)); LEARNED applies the loaded 3D-convolution
 * network (sgpu_net_*) to the TPA-preconditioned gradient, as a learned
 * refinement of it (so TPA is what remains without a network).  Neither has a
 * reference counterpart. */
enum { SGPU_CG_PLAIN = 0, SGPU_CG_TPA = 1, SGPU_CG_LEARNED = 2 };

/* Sets / reads a launch parameter of the handle (the autotuner's knobs).  No
 * reference counterpart; the nearest is auto_blocking
 * (modules/opt_variables.f90:340-353), which picks cache blocking sizes. */
int sgpu_set_param(sgpu_handle h, int param, int value);
int sgpu_get_param(sgpu_handle h, int param, int* value);

/* Autotuner: times `reps` H applications of the resident orbitals (projections,
 * KB field, stencil pass) for every launch shape it knows (x-slabs per orbital
 * 1, 2, 4; KB term by the band-group tile kernel, returned as split 0, or by
 * the band-quad kernel with projection split 1, 2, 4, 8), keeps the fastest in
 * the handle (SGPU_PARAM_NSLAB, SGPU_PARAM_KB_KERNEL, SGPU_PARAM_UVPSI_SPLIT)
 * and returns it (any output pointer may be NULL).  The resident orbitals are not
 * modified.  No reference counterpart; the nearest is auto_blocking
 * (modules/opt_variables.f90:340-353). */
int sgpu_autotune(sgpu_handle h, int reps, int* nslab, int* split, double* ms_per_apply);

/* Step tuner: times whole Taylor steps of length dt (reps per candidate, after a
 * warm-up) on a copy of the resident orbitals, for every launch choice that
 * applies to the handle's grid and precision: the Taylor form
 * (SGPU_PARAM_TAYLOR_KERNEL 2 where the resident form fits, else 1), and for
 * the stencil passes the compile-time plane shapes (SGPU_PARAM_PASS_FIXED),
 * the table staging (SGPU_PARAM_PASS_TABLES), x-slabs (SGPU_PARAM_NSLAB 1, 2,
 * 4) and the KB kernel (tile, split tile with its automatic point ranges, or
 * band quad with split 1, 2, 4, 8).  Keeps the
 * fastest in the handle.  params (HOST [6], may be NULL) receives
 * {taylor_kernel, pass_fixed, pass_tables, nslab, kb_kernel, uvpsi_split};
 * ms_per_step (may be NULL) its time.  The resident orbitals are not modified.
 * No reference counterpart; the nearest is auto_blocking
 * (modules/opt_variables.f90:340-353). */
int sgpu_autotune_step(sgpu_handle h, double dt, int reps, int* params, double* ms_per_step);

/* ---- CG preconditioners (ground state) ------------------------------------ */
/* The TPA preconditioner applied to nvec DEV complex(8) vectors (layout
 * [nvec][NL]); vector v is taken at local k-point kidx[v] (HOST, 0-based; NULL
 * means v) with band kinetic energy tband[v] (HOST).  Test and training hook;
 * sgpu_cg applies the same kernels internally. */
int sgpu_tpa_apply(sgpu_handle h, const void* in_dev, void* out_dev, int nvec, const int* kidx, const double* tband);

/* The learned preconditioner: a 3D convolution network on the periodic grid
 * (conv 1->8, 8->8, 8->1 channels; 3x3x3 kernels with circular padding; no bias
 * or activation), BF16 weights and activations with FP32 accumulation.  It is
 * applied to the real and the imaginary part of a complex vector separately
 * (each scaled by the vector's 1/rms), so K(c g) = c K(g) for complex c.
 * Weights: sgpu_net_weight_count() floats, layer by layer, each [co][ci][tap],
 * tap = (dx+1)*9 + (dy+1)*3 + (dz+1).  No reference counterpart. */
int sgpu_net_weight_count(void);
int sgpu_net_set_weights(sgpu_handle h, const float* w);   /* HOST; resets the optimiser */
int sgpu_net_get_weights(sgpu_handle h, float* w);         /* HOST */
/* out = K(in) for nvec DEV complex(8) vectors [nvec][NL] */
int sgpu_net_apply(sgpu_handle h, const void* in_dev, void* out_dev, int nvec);
/* Mean squared error of K(g) against targets t (both DEV complex(8)
 * [nvec][NL], t scaled like g) and its gradient with respect to the weights
 * (grad HOST, may be NULL; loss HOST, may be NULL). */
int sgpu_net_grad(sgpu_handle h, const void* g_dev, const void* t_dev, int nvec, float* grad, double* loss);
/* One Adam step (learning rate lr) on that loss; loss HOST (may be NULL) is the
 * loss before the step. */
int sgpu_net_train_step(sgpu_handle h, const void* g_dev, const void* t_dev, int nvec, float lr, double* loss);

/* ---- batched systems ------------------------------------------------------ */
/* Several systems (handles on the current device) advanced together.  No
 * reference counterpart: the reference runs one system per process. */
typedef struct sgpu_batch* sgpu_batch_handle;

int sgpu_batch_create(const sgpu_handle* handles, int n, sgpu_batch_handle* out);

/* nsteps Taylor steps of every system, system i with time step dt[i] (HOST,
 * n values), each with the Hamiltonian of its last sgpu_update_projector /
 * sgpu_set_vloc.  The steps of all systems are captured once into a CUDA graph
 * (each system on its own stream) and replayed on later calls with the same
 * dt[] and nsteps; a call with other values, or after a handle's precision
 * changed, captures again (and first waits for the handles' queued work).
 * Asynchronous: later calls on a handle are ordered after the replay. */
int sgpu_batch_step(sgpu_batch_handle b, const double* dt, int nsteps);

/* The batch's cudaStream_t (the replay runs on it). */
void* sgpu_batch_stream(sgpu_batch_handle b);

int sgpu_batch_destroy(sgpu_batch_handle b);

/* ---- instrumentation ----------------------------------------------------- */
/* Kernels that sgpu_time_kernel can time. */
enum {
  SGPU_KERNEL_STENCIL_PASS = 0, /* one H application of every resident orbital (zu -> workspace)     */
  SGPU_KERNEL_TAYLOR_LAST = 1,  /* one Taylor stage (H application + update psi + c H psi), on workspace */
  SGPU_KERNEL_UVPSI = 2,        /* the Kleinman-Bylander projections of every resident orbital       */
  SGPU_KERNEL_PSI_RHO = 3,      /* the density reduction                                             */
  SGPU_KERNEL_KB_FIELD = 4,     /* the Kleinman-Bylander term at the sphere points from the projections */
  SGPU_KERNEL_KB_TERM = 5,      /* projections and KB term in one kernel, as the Taylor step runs them  */
  SGPU_KERNEL_CURRENT_STENCIL = 6, /* the current's stencil sums of every resident orbital             */
  SGPU_KERNEL_CURRENT_PROJ = 7  /* the nonlocal current's weighted projections of every resident orbital */
};

/* Launches `kernel` reps times back to back on the handle's stream between two
 * CUDA events and returns the mean device time per launch.  The resident
 * orbitals are not modified.  Counterpart of the reference's per-kernel timers
 * (misc/timer.f90:34-54, LOG_HPSI_STENCIL etc.), which time on the host. */
int sgpu_time_kernel(sgpu_handle h, int kernel, int reps, double* ms_per_launch);

#ifdef __cplusplus
}
#endif
#endif /* SALMON_GPU_H */
