// Internal declarations of the B200 RT-propagation library (not part of the ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/salmon_gpu.h"

namespace sgpu {

constexpr int KB_USPLIT_MAX = 8;  // point ranges of the split KB projections

// ---------------------------------------------------------------- complex --
template <typename R> struct C2Of;
template <> struct C2Of<float> { using type = float2; };
template <> struct C2Of<double> { using type = double2; };
template <typename R> using C2 = typename C2Of<R>::type;

template <typename R> __host__ __device__ __forceinline__ C2<R> mk(R x, R y) { C2<R> c; c.x = x; c.y = y; return c; }
// cp.async (sm_80+ asynchronous global -> shared copies)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
// hint: bring a contiguous global range into L2 (bulk prefetch; the range must
// lie inside one allocation, start 16-byte aligned and span a multiple of 16 bytes)
__device__ __forceinline__ void prefetch_l2_bulk(const void* gmem, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }


template <typename T> __host__ __device__ __forceinline__ T cadd(T a, T b) { a.x += b.x; a.y += b.y; return a; }
template <typename T> __host__ __device__ __forceinline__ T csub(T a, T b) { a.x -= b.x; a.y -= b.y; return a; }
// a*b
template <typename T> __host__ __device__ __forceinline__ T cmul(T a, T b) {
  T c; c.x = a.x * b.x - a.y * b.y; c.y = a.x * b.y + a.y * b.x; return c;
}
// acc + a*b
template <typename T> __host__ __device__ __forceinline__ T cfma(T a, T b, T acc) {
  acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x)); acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y)); return acc;
}
// acc + conj(a)*b
template <typename T> __host__ __device__ __forceinline__ T cfmaj(T a, T b, T acc) {
  acc.x = fma(a.x, b.x, fma(a.y, b.y, acc.x)); acc.y = fma(a.x, b.y, fma(-a.y, b.x, acc.y)); return acc;
}

__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }
template <typename R> __device__ __forceinline__ C2<R> from_d2(double2 a);
template <> __device__ __forceinline__ float2 from_d2<float>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __device__ __forceinline__ double2 from_d2<double>(double2 a) { return a; }

// Sum of NV doubles over the CTA; the result is valid in every thread.
// sh must hold 32*NV doubles; the call contains __syncthreads().
template <int NV>
__device__ __forceinline__ void block_allsum(double (&v)[NV], double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[warp * NV + k] = v[k];
  __syncthreads();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += sh[w * NV + k];  // fixed order: deterministic
    v[k] = t;
  }
}

// ------------------------------------------------------------ the system --
// Per-handle state: sizes, constants and device buffers.
struct System {
  int dev = 0;
  cudaStream_t stream = nullptr;
  // Kernels launched on `stream` so far (read through SGPU_PARAM_LAUNCHES).
  mutable unsigned long long launches = 0;
  // Incremented whenever the orbital / workspace buffers are reallocated
  // (a captured graph of the handle is then stale).
  unsigned long long gen = 0;
  // The stream for one kernel launch; counts the launch.
  cudaStream_t launch_stream() const {
    ++launches;
    return stream;
  }
  int prec = SGPU_PREC_C128;

  int NLx = 0, NLy = 0, NLz = 0, NL = 0;
  int NK = 0, NK_s = 1, NK_e = 0, nkl = 0, NB = 0, NBocc = 0, norb = 0;
  double H[3] = {0, 0, 0}, aL[3] = {0, 0, 0}, Hxyz = 0, aLxyz = 0;
  double lap[3][5] = {}, nab[3][5] = {};
  int NI = 0, Nps = 0, Nlma = 0, NPI = 0, nitems = 0, ninv = 0;
  int max_mps = 0;                 // largest sphere of one atom (points)

  std::vector<double> occ_h;       // occ(NB,NK)
  std::vector<double> kAc_h;       // last kAc (NK,3)
  bool have_state = false, have_vloc = false, have_proj = false;

  // resident orbitals and Taylor workspace (precision-dependent element size)
  void* zu = nullptr;              // [norb][NL]
  void* tw[3] = {nullptr, nullptr, nullptr};
  size_t elem = 16;                // bytes per complex element

  double* vloc64 = nullptr;        // [NL]
  float* vloc32 = nullptr;         // [NL]
  double* occ_o = nullptr;         // [norb] occupation of each resident orbital
  double* kAc_d = nullptr;         // [nkl][3]

  // Kleinman-Bylander tables (built like init_projector, opt_variables.f90:233-265)
  int* idx_proj = nullptr;         // [NPI] 0-based grid index, atom by atom
  int* atom_off = nullptr;         // [NI+1] packed offset of each atom's points
  double* rpos = nullptr;          // [NPI][3] x,y,z relative to the atom image (projector.f90:61)
  int4* items = nullptr;           // [nitems] {atom, first lma_list slot, count (<=4), 0}
  int* lma_list = nullptr;         // [Nlma] projectors grouped by atom
  int* iuV_d = nullptr;            // [Nlma]
  int* lma_atom = nullptr;         // [Nlma]
  double* uV_d = nullptr;          // [Nlma][Nps]
  double2* zproj64 = nullptr;      // [nkl][Nlma][Nps]
  float2* zproj32 = nullptr;       // [nkl][Nlma][Nps]   (C64 mode)
  // Kleinman-Bylander sphere points sorted by grid index: plane x holds points
  // sp_off[x] .. sp_off[x+1]-1 (at most maxpts); point q has the record
  // rec[2q..2q+1] = {in-plane position, count of the first <= 4 entries, e0, e1},
  // {e2, e3, first continuation, continuation count} with e = ilma<<16 | j
  // (zproj(j,ilma)).  lqi[i] is grid point i's index among its plane's sphere
  // points (-1 if none).  qmap[p] is the sphere-point index of packed projector
  // point p (the gather index into a sphere-value array S).
  int* sp_off = nullptr;           // [NLx+1]
  int4* rec = nullptr;             // [2*nsp]
  int* cont = nullptr;             // entries beyond the 4th of points in several spheres
  int* qmap = nullptr;             // [NPI]
  // KB field on the tensor pipe: kbq[p] = qmap[p] where the sphere point lies in
  // exactly one projector item, else -1; those other points (kb_multi, n_multi
  // of them) are summed entry by entry in a fixed order instead.
  int* kbq = nullptr;              // [NPI]
  int* kb_multi = nullptr;         // [n_multi]
  int n_multi = 0;
  short* lqi = nullptr;            // [NL]
  int nsp = 0, maxpts = 0;
  void* Wbuf = nullptr;            // [W_rows][nsp] KB field (element: complex(8) capacity)
  size_t W_rows = 0;
  void* Sbuf = nullptr;            // [norb][nsp] orbital values at the sphere points
  bool S_valid = false;            // Sbuf holds the sphere values of the resident zu
  double2* U = nullptr;            // [norb][Nlma] projections <uV e^{ikr}|psi> (scaled)
  double2* Uw = nullptr;           // [uvw_split][norb][Nlma][4] weighted projections for the current
  int uvw_split = 1;               // point-range parts of the weighted projections (k_uvpsi_w)

  // reduction scratch
  double* red = nullptr;           // device scratch for partial sums
  size_t red_elems = 0;
  double* red_h = nullptr;         // pinned host mirror
  size_t red_h_elems = 0;
  // pinned staging of the per-step host inputs (Vloc [NL], then k+A [3*nkl]):
  // the copies are asynchronous, and the next call waits on the event of the
  // previous copy before it overwrites its region
  double* in_h = nullptr;
  cudaEvent_t ev_vloc_in = nullptr, ev_kac_in = nullptr;
  bool vloc_in_pending = false, kac_in_pending = false;

  // host<->device staging for one orbital / chunked conversions
  double2* stage = nullptr;        // [stage_elems] complex(8)
  size_t stage_elems = 0;

  // ground state (allocated on first use): zu_GS(NL,NB,NK_s:NK_e) and work space
  double2* gs_zu = nullptr;        // [nkl][NB][NL]
  double2* gs_aux = nullptr;       // [nkl][NB][NL]  H zu_GS, rotation output
  double2* gs_W = nullptr;         // [8][nkl][NL]   CG work vectors
  void* gs_st = nullptr;           // [nkl] CG state
  double2* gs_part = nullptr;      // [nsplit][nkl][NB][NB]
  double2* gs_A = nullptr;         // [nkl][NB][NB]
  double2* gs_V = nullptr;         // [nkl][NB][NB]
  double* gs_w = nullptr;          // [nkl][NB]
  int* gs_sweeps = nullptr;        // [nkl]
  double* occ_gs = nullptr;        // [nkl][NB]
  double* gs_out = nullptr;        // [nkl][NB] device results
  double* gs_h = nullptr;          // pinned host staging [nkl][NB]
  int gs_nsplit = 0;
  bool have_gs = false;
  size_t U_rows = 0;               // orbitals U can hold

  // tuning
  int nslab = 1;                   // x-slabs per orbital in the stencil pass
  int nyblk = 1, NYB = 0;          // y-blocks per plane (planes wider than 512 threads) and their rows
  int* sp_blk = nullptr;           // [NLx*(nyblk+1)] first sphere point of each (plane, y-block)
  int pass_tab = 1;                // stencil pass: Vloc/sphere-index tables through the ring (two-point form)
  int pass_fixed = 1;              // stencil pass: compile-time plane shapes with a 9-plane ring (complex(4))
  int cur_fixed = 1;               // current stencil, 32x32 / 48x48 planes: 1 two rows per thread, 2 one, 0 generic
  int taylor_kernel = 0;           // Taylor step: 0 auto, 1 stencil passes, 2 the shared-memory resident kernel
  // The current's stencil sums {jt, F, G, H} of the resident orbitals, computed by a
  // Taylor step called with flag_current (RT/hamiltonian.f90:68-70): rows
  // cur_part[o][cur_nx][4], valid while cur_valid (the orbitals are unchanged since).
  double* cur_part = nullptr;      // [norb][NLx][4]
  double* nab12 = nullptr;         // [12] nabx(1:4), naby(1:4), nabz(1:4) (device, set at creation)
  int cur_nx = 0;
  bool cur_valid = false;
  // The stencil sums of a flag_current step run on a second stream (they only read
  // the orbitals), overlapping the density and the nonlocal current that follow on
  // `stream`; ev_cur marks their end.  aux_pending: `stream` has not waited for it.
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_step = nullptr, ev_cur = nullptr;
  bool aux_pending = false;
  // Makes `stream` wait for the stencil sums (before anything writes the orbitals
  // or cur_part, or reads cur_part).
  cudaError_t aux_join() {
    if (!aux_pending) return cudaSuccess;
    aux_pending = false;
    return cudaStreamWaitEvent(stream, ev_cur, 0);
  }
  int nsm = 148;                   // SMs of the device
  mutable bool kb_smem_ok = false;  // the KB tile kernels' shared-memory limits are raised for this handle
  int um_split = 4;                // band-quad KB kernel: warps splitting the points of one tile (1, 2, 4, 8)
  int kb_kernel = 0;               // KB term: 0 auto, 1 band-group tile kernel, 2 band-quad kernel, 3 split tile
  int kb_usplit = 0;               // split tile: point ranges of the projections (<= KB_USPLIT_MAX; 0 auto)
  double2* Up = nullptr;           // [Up_rows][Nlma] partial projections of the split tile
  size_t Up_rows = 0;
  int cg_precond = 0;              // ground-state CG preconditioner: 0 none, 1 TPA, 2 learned
  double cg_delta = 1e-15;         // CG stops a band when its Rayleigh quotient moves less than this
  bool net_ready = false;          // a preconditioner network has been loaded
  void* net = nullptr;             // its weights, optimiser state and workspace (k_net.cu)
  double* gs_tb = nullptr;         // [nkl] kinetic energy of the band in CG (TPA)
  double* vpsl = nullptr;          // [NL] local pseudopotential (for the self-consistent Vloc)
  double* rho_d = nullptr;         // [NL] density used by the last potential update
  double* exc_d = nullptr;         // [2] Hartree and exchange-correlation energies
  double* gs_res = nullptr;        // [nkl][NB] residual norms of the last sgpu_cg
  double* vloc_hist = nullptr;     // [2][NL] the etrs potential history Vloc_old(:,1:2) (allocated on first use)
};

// ------------------------------------------------------------ kernel API --
// All launches go to s.stream.  A batch is nb orbitals in[0..nb) laid out like
// zu; orbital b of the batch belongs to local k-point (o_beg + b) / nbk
// (nbk = NBoccmax for the resident orbitals, NB for ground-state arrays, 1 for
// one work vector per k-point).

// U[b][ilma] = Hxyz * (scale_iuv ? iuV : 1) * sum_j conj(zproj(j,ilma,k)) in_b(J_a(j))
cudaError_t launch_uvpsi(const System& s, const void* in, int o_beg, int nb, int nbk, bool scale_iuv, int prec = -1);
// the same projections from sphere values S[b][nsp] exported by a pass
cudaError_t launch_uvpsi_from_S(const System& s, const void* S, int o_beg, int nb, int nbk, bool scale_iuv);
// W[b][q] = sum_entries zproj U[b] at every sphere point (needs U of the batch)
cudaError_t launch_kbfield(const System& s, int o_beg, int nb, int nbk, void* W, int prec = -1);
// U and W of one H application in one kernel (plus the entry-wise kernel for
// points in several projector items): projections from S (from_S, the sphere
// values exported by the previous pass) or gathered from the orbitals `in`.
cudaError_t launch_kb_term(const System& s, const void* in, bool from_S, int o_beg, int nb, int nbk, void* W,
                           int prec = -1);
// dynamic shared memory of the pass kernel
// (nr: ring planes, 0 = the precision's default)
size_t pass_smem_bytes(int prec, int NLy, int NLz, int maxpts, bool with_w, int NLx, int nyblk = 1, int NYB = 0,
                       bool tables = false, int nr = 0);

// One H application: out = H in  (mode 0), with ttpsi (mode 1), or one stage
// of the Taylor step (mode 2): out = in + c H in.  W must hold the KB term of
// `in` (launch_kb_term).
struct PassIO {
  const void* in = nullptr;
  void* out = nullptr;
  void* tt = nullptr;
  const void* W = nullptr;         // KB term at the sphere points ([nb][nsp]) or null (no projectors)
  void* S = nullptr;               // export of the output at the sphere points ([nb][nsp]) or null
  double zc[2] = {0.0, 0.0};       // mode 2: the stage coefficient c (re, im)
};
// The four stage coefficients of a 4th-order Taylor step of length dt:
// 1 + sum_{n=1..4} (-i dt H)^n / n! = prod_{s=0..3} (1 + c_s H).
void taylor_stage_coefs(double dt, double c[4][2]);
// prec = -1 uses the handle's precision; SGPU_PREC_C128 forces FP64 (ground state).
cudaError_t launch_hpsi_pass(const System& s, int mode, const PassIO& io, int o_beg, int nb, int nbk, int prec = -1);
// threads per CTA of the pass kernel for an NLy x NLz plane
// Sets the shared-memory attribute of every stencil-pass kernel the handle can
// launch (needed before capturing its launches into a graph).
cudaError_t prepare_pass(const System& s);
cudaError_t prepare_kb(const System& s);
// Raises a kernel's dynamic shared-memory limit to at least `bytes` (never
// lowers it, so handles of different sizes sharing a kernel keep working).
inline cudaError_t raise_smem_limit(const void* func, size_t bytes) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, func);
  if (e != cudaSuccess) return e;
  if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return cudaSuccess;
  return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}  // shared-memory attribute of the KB tile kernel
bool kb_tile_fits(const System& s);
int pass_block_threads(int NLy, int NLz);

// zproj(j,ilma,k) = conj(exp(i kAc.r)) uV(j,ilma)  for the local k-points.
cudaError_t launch_update_projector(const System& s);

// Precision conversion of n complex elements.
cudaError_t launch_c128_to_c64(const double2* src, float2* dst, size_t n, cudaStream_t st);
cudaError_t launch_c64_to_c128(const float2* src, double2* dst, size_t n, cudaStream_t st);
cudaError_t launch_r64_to_r32(const double* src, float* dst, size_t n, cudaStream_t st);

// rho(NL) = sum_o occ_o |zu_o|^2 into red -> host
cudaError_t launch_psi_rho(System& s, double* rho_dev);
// per-orbital current terms and the final jav(3) (device)
cudaError_t launch_current(System& s, double* jav_dev);
cudaError_t launch_current_proj(System& s);
// reduction scratch (doubles) that launch_current and launch_energy need
size_t current_red_elems(int norb, int NLx);
// per-orbital kinetic and nonlocal energies summed (device, 2 doubles)
cudaError_t launch_energy(System& s, double* e_dev);

// ground state (k_gs.cu)
cudaError_t launch_gram_schmidt(const System& s, double2* zu);
cudaError_t launch_cg_begin(const System& s, double2* zu, double2* W, void* st, int ib);
cudaError_t launch_cg_dot0(const System& s, double2* W, void* st);
cudaError_t launch_cg_pre(const System& s, const double2* zu, double2* W, void* st, int ib, int iter);
cudaError_t launch_cg_post(const System& s, double2* W, void* st, int iter);
cudaError_t launch_cg_end(const System& s, double2* zu, double2* W, int ib);
cudaError_t launch_cg_resid(const System& s, double2* W, const double* occ_gs, double* esp_var, double* res, int ib);
cudaError_t launch_cg_grad(const System& s, const double2* zu, double2* W, void* st, double* tband, int ib);
cudaError_t launch_cg_dir(const System& s, const double2* zu, double2* W, void* st, int ib, int iter);
// Batched 3D FFT (sign -1 forward, +1 backward; normalise divides by NL) of
// nvec grid functions, and the TPA preconditioner applied in place to nvec
// vectors (vector v belongs to k-point v / vecs_per_k; tband_dev[v] its band's
// kinetic energy).  Sizes 2^a 3^b up to 96 per axis.
bool fft_size_ok(int n);
// The learned preconditioner applied in place to nvec vectors (k_net.cu).
cudaError_t launch_precond_net(const System& s, double2* data, int nvec);
// Vloc = Vh[rho] + Vpsl + Vxc[rho] into vloc64/vloc32 (k_xc.cu); energies_dev[2] =
// (Eh, Exc).  Grid sizes 2^a 3^b <= 96.
cudaError_t launch_update_vloc(const System& s, const double* rho_dev, double* energies_dev);
void net_free(System& s);
// The etrs potential history: reset (both entries = Vloc) or extrapolate
// (Vloc <- 3 Vloc - 3 hist1 + hist2, history shifted) on the device.
cudaError_t launch_vloc_history(const System& s, bool extrapolate);
cudaError_t launch_fft3d(const System& s, double2* data, int nvec, int sign, bool normalise);
cudaError_t launch_tpa(const System& s, double2* data, int nvec, const double* tband_dev, int vecs_per_k,
                       const int* kidx_dev = nullptr);
size_t cg_state_bytes();
int cg_work_vectors();
cudaError_t launch_subspace_h(const System& s, const double2* U, const double2* HU, double2* part, int nsplit,
                              double2* za);
cudaError_t launch_jacobi(const System& s, double2* A, double2* V, int max_sweeps, double* w, int* sweeps);
cudaError_t launch_rotate(const System& s, const double2* in, const double2* Z, double2* out);

// Sets the message that sgpu_last_error returns (defined with the C ABI).
void set_last_error(const std::string& msg);

// One Taylor step of every resident orbital on the handle's stream (kernel
// launches only).  gather_first: the first projections gather from the
// orbitals instead of reading the sphere values S of the previous step.
// with_current: also compute the current's stencil sums of the new orbitals
// into cur_part (flag_current of RT/hamiltonian.f90:27).
cudaError_t enqueue_taylor_step(System& s, double dt, bool gather_first, bool with_current = false);
cudaError_t enqueue_taylor_step_on(System& s, void* zu_buf, double dt, bool gather_first, bool with_current);

// The Taylor step with each orbital resident in one CTA's shared memory
// (k_resident.cu): whether the handle's grid and precision have that form, the
// launch (cur: [norb][4] stencil sums or null; S: sphere-value export or null),
// and the shared-memory attribute (before a graph capture).
// resident_step_default: the form the auto setting picks (where it measured faster).
bool resident_step_fits(const System& s);
bool resident_step_default(const System& s);
cudaError_t launch_taylor_resident(const System& s, void* zu, double dt, double* cur, void* S);
cudaError_t prepare_resident(const System& s);
// The current's stencil sums of the resident orbitals into part[o][nx][4]
// (k_reduce.cu; nx returned).
cudaError_t launch_current_stencil(System& s, double* part, int& nx);

}  // namespace sgpu

// The C ABI's opaque handle is the System itself.
struct sgpu_system : public sgpu::System {};
