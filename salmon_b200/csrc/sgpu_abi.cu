// C ABI of the B200 RT-propagation library (include/salmon_gpu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <complex>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "sgpu_internal.cuh"

using sgpu::System;

namespace {

thread_local std::string g_err = "no error";

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? SGPU_ERR_ALLOC : SGPU_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

#define CK(expr)                                          \
  do {                                                    \
    cudaError_t e_ = (expr);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, #expr);   \
  } while (0)

template <typename T>
cudaError_t dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  return cudaMalloc((void**)p, n * sizeof(T));
}

template <typename T>
cudaError_t upload(T** p, const T* h, size_t n, cudaStream_t st) {
  cudaError_t e = dalloc(p, n);
  if (e != cudaSuccess || n == 0) return e;
  return cudaMemcpyAsync(*p, h, n * sizeof(T), cudaMemcpyHostToDevice, st);
}

void free_state_buffers(System* s) {
  cudaFree(s->zu);
  for (auto& t : s->tw) { cudaFree(t); t = nullptr; }
  s->zu = nullptr;
}

int alloc_state_buffers(System* s) {
  ++s->gen;
  const size_t n = (size_t)s->norb * s->NL;
  s->elem = s->prec == SGPU_PREC_C64 ? sizeof(float2) : sizeof(double2);
  CK(cudaMalloc(&s->zu, n * s->elem));
  for (auto& t : s->tw) CK(cudaMalloc(&t, n * s->elem));
  return 0;
}

bool valid(sgpu_handle h) { return h != nullptr; }

// kAc(NK,3) host -> [nkl][3] device of the handle's k range
// Host inputs go through the handle's pinned staging, so the copy is queued on
// the stream without waiting for the work before it; the caller's array is free
// again on return.
int set_kac(System* s, const double* kAc) {
  if (s->kac_in_pending) CK(cudaEventSynchronize(s->ev_kac_in));  // the previous copy has read its staging
  double* loc = s->in_h + s->NL;
  for (int kl = 0; kl < s->nkl; ++kl)
    for (int d = 0; d < 3; ++d) loc[3 * kl + d] = kAc[(size_t)d * s->NK + (s->NK_s - 1 + kl)];
  s->kAc_h.assign(kAc, kAc + 3 * (size_t)s->NK);
  CK(cudaMemcpyAsync(s->kAc_d, loc, 3 * (size_t)s->nkl * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(cudaEventRecord(s->ev_kac_in, s->stream));
  s->kac_in_pending = true;
  return 0;
}

int one_orbital_k(const System* s, int ik) { return (ik - s->NK_s) * s->NBocc; }

// One H application of a batch: projections U (gathered from io.in, or from the
// sphere values S exported by the previous pass), the KB field W at the sphere
// points, then the stencil pass (which may export its output to S).
cudaError_t apply_h(System* s, int mode, sgpu::PassIO io, int o_beg, int nb, int nbk, int prec, bool u_from_S) {
  cudaError_t e;
  if (s->nsp > 0) {
    if ((e = sgpu::launch_kb_term(*s, io.in, u_from_S, o_beg, nb, nbk, s->Wbuf, prec)) != cudaSuccess) return e;
    io.W = s->Wbuf;
  }
  return sgpu::launch_hpsi_pass(*s, mode, io, o_beg, nb, nbk, prec);
}

}  // namespace

// Entry points defined in other files report through the same message slot.
void sgpu::set_last_error(const std::string& msg) { g_err = msg; }

// The Taylor polynomial of RT/hamiltonian.f90:46-49, :114-117,
//   p(H) = 1 + sum_{n=1..4} zfac(n) H^n,   zfac(n) = (-i dt)^n / n!,
// is e4(y) = 1 + y + y^2/2 + y^3/6 + y^4/24 at y = -i dt H.  With y_s the four
// roots of e4, p(H) = prod_s (1 - y/y_s) = prod_s (1 + c_s H), c_s = i dt / y_s:
// the same polynomial, applied as four stages psi <- psi + c_s H psi.  Each stage
// is one H application whose update needs only its own input, so no stage reads
// the earlier Taylor terms (the sum form's last pass reads four arrays and
// writes one).  In FP64 the two forms agree to ~1e-15 relative on the test
// systems; the roots are polished by Newton's method in FP64.
void sgpu::taylor_stage_coefs(double dt, double c[4][2]) {
  using Z = std::complex<double>;
  static const std::array<Z, 4> roots = []() {
    // e4 scaled to a monic quartic: y^4 + 4 y^3 + 12 y^2 + 24 y + 24
    auto p = [](Z y) { return (((y + 4.0) * y + 12.0) * y + 24.0) * y + 24.0; };
    auto dp = [](Z y) { return ((4.0 * y + 12.0) * y + 24.0) * y + 24.0; };
    std::array<Z, 4> r = {Z(0.4, 0.9), Z(0.4, 0.9) * Z(0.4, 0.9), Z(0.4, 0.9) * Z(0.4, 0.9) * Z(0.4, 0.9),
                          Z(0.4, 0.9) * Z(0.4, 0.9) * Z(0.4, 0.9) * Z(0.4, 0.9)};
    for (int it = 0; it < 500; ++it)  // Durand-Kerner: all four roots at once
      for (int i = 0; i < 4; ++i) {
        Z den = 1.0;
        for (int j = 0; j < 4; ++j)
          if (j != i) den *= r[i] - r[j];
        r[i] -= p(r[i]) / den;
      }
    for (auto& y : r)  // Newton polish
      for (int it = 0; it < 3; ++it) y -= p(y) / dp(y);
    // a fixed order: the pair nearer the imaginary axis first, +Im before -Im
    std::sort(r.begin(), r.end(), [](Z a, Z b) {
      if (std::abs(a.real() - b.real()) > 1e-6) return a.real() > b.real();
      return a.imag() > b.imag();
    });
    return r;
  }();
  for (int i = 0; i < 4; ++i) {
    const Z ci = Z(0.0, dt) / roots[i];
    c[i][0] = ci.real();
    c[i][1] = ci.imag();
  }
}

// One Taylor step of every resident orbital, enqueued on the handle's stream
// (kernel launches only, so it can be captured into a CUDA graph): four stages
// zu -> tw0 -> tw1 -> tw0 -> zu.
cudaError_t sgpu::enqueue_taylor_step(System& sys, double dt, bool gather_first, bool with_current) {
  return enqueue_taylor_step_on(sys, sys.zu, dt, gather_first, with_current);
}

// The same step on the orbital array zu_buf (s->zu, or a copy the tuner times:
// tw[2], with tw[0] and tw[1] as the stages' workspace).
cudaError_t sgpu::enqueue_taylor_step_on(System& sys, void* zu_buf, double dt, bool gather_first,
                                         bool with_current) {
  System* s = &sys;
  cudaError_t ej = s->aux_join();  // the previous step's stencil sums still read zu
  if (ej != cudaSuccess) return ej;
  s->cur_valid = false;
  const bool resident = s->taylor_kernel == 2 || (s->taylor_kernel == 0 && sgpu::resident_step_default(*s));
  if (resident) {
    // the whole step on chip, a band group per CTA (it gathers its own projections)
    cudaError_t e = sgpu::launch_taylor_resident(*s, zu_buf, dt, with_current ? s->cur_part : nullptr,
                                                 s->nsp > 0 ? s->Sbuf : nullptr);
    if (e != cudaSuccess) return e;
    s->S_valid = s->nsp > 0;
    s->cur_nx = 1;
    s->cur_valid = with_current;
    return cudaSuccess;
  }
  double c[4][2];
  taylor_stage_coefs(dt, c);
  // Each stage exports its output at the sphere points (S); the next stage's
  // projections read S instead of gathering from the full orbitals.
  const void* ins[4] = {zu_buf, s->tw[0], s->tw[1], s->tw[0]};
  void* outs[4] = {s->tw[0], s->tw[1], s->tw[0], zu_buf};
  cudaError_t e;
  for (int n = 0; n < 4; ++n) {
    sgpu::PassIO io;
    io.in = ins[n];
    io.out = outs[n];
    io.S = s->nsp > 0 ? s->Sbuf : nullptr;
    io.zc[0] = c[n][0];
    io.zc[1] = c[n][1];
    const bool from_S = s->nsp > 0 && (n > 0 || !gather_first);
    e = apply_h(s, 2, io, 0, s->norb, s->NBocc, -1, from_S);
    if (e != cudaSuccess) return e;
  }
  s->S_valid = s->nsp > 0;
  if (with_current && zu_buf == s->zu) {
    // the stencil sums of the new orbitals, right after the update, on the second
    // stream: they overlap whatever the caller queues next on `stream` (the
    // density, the nonlocal current), which only reads the orbitals too
    int nx = 1;
    if ((e = cudaEventRecord(s->ev_step, s->stream)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s->aux, s->ev_step, 0)) != cudaSuccess) return e;
    std::swap(s->stream, s->aux);
    e = sgpu::launch_current_stencil(*s, s->cur_part, nx);
    std::swap(s->stream, s->aux);
    if (e != cudaSuccess) return e;
    if ((e = cudaEventRecord(s->ev_cur, s->aux)) != cudaSuccess) return e;
    s->aux_pending = true;
    s->cur_nx = nx;
    s->cur_valid = true;
  }
  return cudaSuccess;
}

extern "C" {

const char* sgpu_last_error(void) { return g_err.c_str(); }

int sgpu_check_desc(const sgpu_desc* d) {
  if (!d) return fail(SGPU_ERR_ARG, "sgpu_check_desc: null descriptor");
  if (d->NLx < 1 || d->NLy < 1 || d->NLz < 1) return fail(SGPU_ERR_ARG, "sgpu_create: grid sizes must be positive");
  if (d->NK < 1 || d->NK_s < 1 || d->NK_e < d->NK_s || d->NK_e > d->NK)
    return fail(SGPU_ERR_ARG, "sgpu_create: need 1 <= NK_s <= NK_e <= NK");
  if (d->NB < 1 || d->NBoccmax < 1 || d->NBoccmax > d->NB)
    return fail(SGPU_ERR_ARG, "sgpu_create: need 1 <= NBoccmax <= NB");
  if (d->NI < 0 || d->Nlma < 0 || d->Nps < 0 || (d->NI > 0 && d->Nlma > 0 && d->Nps < 1))
    return fail(SGPU_ERR_ARG, "sgpu_create: bad NI/Nps/Nlma");
  if (!d->occ) return fail(SGPU_ERR_ARG, "sgpu_create: occ is NULL");
  if (d->Nlma > 0 && (!d->Mps || !d->Jxyz || !d->Jxx || !d->Jyy || !d->Jzz || !d->uV || !d->iuV || !d->a_tbl))
    return fail(SGPU_ERR_ARG, "sgpu_create: projector tables missing");
  if ((d->NLz % 2 == 0 ? d->NLz / 2 : d->NLz) > 128)
    return fail(SGPU_ERR_UNSUPPORTED, "sgpu_create: NLz too large for the stencil pass");
  const long NL = (long)d->NLx * d->NLy * d->NLz;
  if (NL > (1L << 30)) return fail(SGPU_ERR_ARG, "sgpu_create: grid too large");
  if (d->Nlma > 0) {
    for (int a = 0; a < d->NI; ++a) {
      const int m = d->Mps[a];
      if (m < 0 || m > d->Nps) return fail(SGPU_ERR_ARG, "sgpu_create: Mps out of range");
      for (int j = 0; j < m; ++j) {
        const long gi = (long)d->Jxyz[(size_t)a * d->Nps + j] - 1;
        if (gi < 0 || gi >= NL) return fail(SGPU_ERR_ARG, "sgpu_create: Jxyz out of range");
      }
    }
    for (int l = 0; l < d->Nlma; ++l)
      if (d->a_tbl[l] < 1 || d->a_tbl[l] > d->NI) return fail(SGPU_ERR_ARG, "sgpu_create: a_tbl out of range");
  }
  return 0;
}

int sgpu_create(const sgpu_desc* d, int precision, sgpu_handle* out) {
  if (!d || !out) return fail(SGPU_ERR_ARG, "sgpu_create: null argument");
  *out = nullptr;
  if (precision != SGPU_PREC_C128 && precision != SGPU_PREC_C64)
    return fail(SGPU_ERR_ARG, "sgpu_create: precision must be SGPU_PREC_C128 or SGPU_PREC_C64");
  if (int rc = sgpu_check_desc(d)) return rc;
  if (d->NLx < 1 || d->NLy < 1 || d->NLz < 1) return fail(SGPU_ERR_ARG, "sgpu_create: grid sizes must be positive");
  if (d->NK < 1 || d->NK_s < 1 || d->NK_e < d->NK_s || d->NK_e > d->NK)
    return fail(SGPU_ERR_ARG, "sgpu_create: need 1 <= NK_s <= NK_e <= NK");
  if (d->NB < 1 || d->NBoccmax < 1 || d->NBoccmax > d->NB)
    return fail(SGPU_ERR_ARG, "sgpu_create: need 1 <= NBoccmax <= NB");
  if (d->NI < 0 || d->Nlma < 0 || d->Nps < 0 || (d->NI > 0 && d->Nlma > 0 && d->Nps < 1))
    return fail(SGPU_ERR_ARG, "sgpu_create: bad NI/Nps/Nlma");
  if (!d->occ) return fail(SGPU_ERR_ARG, "sgpu_create: occ is NULL");
  if (d->Nlma > 0 && (!d->Mps || !d->Jxyz || !d->Jxx || !d->Jyy || !d->Jzz || !d->uV || !d->iuV || !d->a_tbl))
    return fail(SGPU_ERR_ARG, "sgpu_create: projector tables missing");
  const int rz = (d->NLz % 2 == 0) ? 2 : 1;
  // planes of more than 512 threads' points are split over y-blocks of >= 4 rows
  const int nzg = d->NLz / rz;
  if (nzg > 128) return fail(SGPU_ERR_UNSUPPORTED, "sgpu_create: NLz too large for the stencil pass");
  int nyblk = 1, NYB = d->NLy;
  if ((long)d->NLy * nzg > 512) {
    nyblk = (d->NLy + 512 / nzg - 1) / (512 / nzg);
    NYB = (d->NLy + nyblk - 1) / nyblk;
  }
  const long NL = (long)d->NLx * d->NLy * d->NLz;
  if (NL > (1L << 30)) return fail(SGPU_ERR_ARG, "sgpu_create: grid too large");

  sgpu_system* s = new (std::nothrow) sgpu_system();
  if (!s) return fail(SGPU_ERR_ALLOC, "sgpu_create: host allocation failed");
  auto bail = [&](int rc) {
    sgpu_destroy(s);
    return rc;
  };
  cudaError_t e = cudaGetDevice(&s->dev);
  if (e != cudaSuccess) { delete s; return cuda_fail(e, "cudaGetDevice"); }
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete s; return cuda_fail(e, "cudaStreamCreate"); }
  if ((e = cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&s->ev_step, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&s->ev_cur, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&s->ev_vloc_in, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&s->ev_kac_in, cudaEventDisableTiming)) != cudaSuccess)
    return bail(cuda_fail(e, "sgpu_create: second stream"));
  {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, dev);
  }

  s->prec = precision;
  s->nyblk = nyblk;
  s->NYB = NYB;
  s->NLx = d->NLx; s->NLy = d->NLy; s->NLz = d->NLz; s->NL = (int)NL;
  s->NK = d->NK; s->NK_s = d->NK_s; s->NK_e = d->NK_e; s->nkl = d->NK_e - d->NK_s + 1;
  s->NB = d->NB; s->NBocc = d->NBoccmax; s->norb = s->nkl * s->NBocc;
  s->H[0] = d->Hx; s->H[1] = d->Hy; s->H[2] = d->Hz;
  s->aL[0] = d->aLx; s->aL[1] = d->aLy; s->aL[2] = d->aLz;
  s->Hxyz = d->Hx * d->Hy * d->Hz;
  s->aLxyz = d->aLx * d->aLy * d->aLz;
  for (int n = 0; n < 5; ++n) {
    s->lap[0][n] = d->lapx[n]; s->lap[1][n] = d->lapy[n]; s->lap[2][n] = d->lapz[n];
    s->nab[0][n] = d->nabx[n]; s->nab[1][n] = d->naby[n]; s->nab[2][n] = d->nabz[n];
  }
  s->NI = d->Nlma > 0 ? d->NI : 0;
  s->Nps = d->Nlma > 0 ? d->Nps : 0;
  s->Nlma = d->Nlma;
  s->occ_h.assign(d->occ, d->occ + (size_t)d->NB * d->NK);

  // ---- projector tables: packed index (init_projector, opt_variables.f90:233-265)
  std::vector<int> atom_off(s->NI + 1, 0), idx_proj;
  std::vector<double> rpos;
  for (int a = 0; a < s->NI; ++a) {
    const int m = d->Mps[a];
    if (m < 0 || m > s->Nps) return bail(fail(SGPU_ERR_ARG, "sgpu_create: Mps out of range"));
    atom_off[a + 1] = atom_off[a] + m;
    s->max_mps = std::max(s->max_mps, m);
    for (int j = 0; j < m; ++j) {
      const int gi = d->Jxyz[(size_t)a * s->Nps + j] - 1;
      if (gi < 0 || gi >= s->NL) return bail(fail(SGPU_ERR_ARG, "sgpu_create: Jxyz out of range"));
      idx_proj.push_back(gi);
      const int lx = gi / (s->NLy * s->NLz), ly = (gi / s->NLz) % s->NLy, lz = gi % s->NLz;
      rpos.push_back(lx * s->H[0] - d->Jxx[(size_t)a * s->Nps + j] * s->aL[0]);
      rpos.push_back(ly * s->H[1] - d->Jyy[(size_t)a * s->Nps + j] * s->aL[1]);
      rpos.push_back(lz * s->H[2] - d->Jzz[(size_t)a * s->Nps + j] * s->aL[2]);
    }
  }
  s->NPI = atom_off[s->NI];
  std::vector<int> lma_atom(s->Nlma), iuv(s->Nlma), lma_list;
  std::vector<int4> items;
  for (int l = 0; l < s->Nlma; ++l) {
    const int a = d->a_tbl[l] - 1;
    if (a < 0 || a >= s->NI) return bail(fail(SGPU_ERR_ARG, "sgpu_create: a_tbl out of range"));
    lma_atom[l] = a;
    iuv[l] = d->iuV[l];
  }
  for (int a = 0; a < s->NI; ++a) {  // projectors grouped by atom, chunks of <= 4
    std::vector<int> mine;
    for (int l = 0; l < s->Nlma; ++l)
      if (lma_atom[l] == a) mine.push_back(l);
    for (size_t c = 0; c < mine.size(); c += 4) {
      const int cnt = (int)std::min<size_t>(4, mine.size() - c);
      items.push_back(make_int4(a, (int)lma_list.size(), cnt, 0));
      for (int q = 0; q < cnt; ++q) lma_list.push_back(mine[c + q]);
    }
  }
  s->nitems = (int)items.size();
  // inverse map: for each grid point the (ilma, j) pairs whose sphere holds it
  std::vector<int> cnt(s->NL + 1, 0);
  for (int l = 0; l < s->Nlma; ++l) {
    const int a = lma_atom[l];
    for (int j = 0; j < d->Mps[a]; ++j) cnt[idx_proj[atom_off[a] + j] + 1]++;
  }
  for (int i = 0; i < s->NL; ++i) cnt[i + 1] += cnt[i];
  std::vector<int2> ent(cnt[s->NL]);
  {
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int l = 0; l < s->Nlma; ++l) {
      const int a = lma_atom[l];
      for (int j = 0; j < d->Mps[a]; ++j) {
        const int gi = idx_proj[atom_off[a] + j];
        ent[fill[gi]++] = make_int2(l * s->Nps + j, l);
      }
    }
  }
  s->ninv = (int)ent.size();
  // sphere points by x-plane with their <= 4 (ilma, j) entries, and the map from
  // packed projector points to sphere points
  std::vector<int> sp_off(s->NLx + 1, 0), q_of(s->NL, -1), qmap(std::max(1, s->NPI), 0);
  std::vector<int4> rec;
  std::vector<int> cont, kbq, kb_multi, qrow;
  {
    if (s->Nps >= 65536 || s->Nlma >= 32768)
      return bail(fail(SGPU_ERR_UNSUPPORTED, "sgpu_create: Nps must be < 65536 and Nlma < 32768"));
    const int NYZ = s->NLy * s->NLz;
    int nsp = 0;
    for (int x = 0; x < s->NLx; ++x) {
      sp_off[x] = nsp;
      for (int i = x * NYZ; i < (x + 1) * NYZ; ++i) {
        const int c = cnt[i + 1] - cnt[i];
        if (c == 0) continue;
        int e[4] = {0, 0, 0, 0};
        const int c0 = (int)cont.size();
        for (int k = 0; k < c; ++k) {
          const int2 en = ent[cnt[i] + k];  // {ilma*Nps + j, ilma}
          const int ek = (en.y << 16) | (en.x - en.y * s->Nps);
          if (k < 4) e[k] = ek;
          else cont.push_back(ek);
        }
        rec.push_back(make_int4(i - x * NYZ, std::min(c, 4), e[0], e[1]));
        rec.push_back(make_int4(e[2], e[3], c0, std::max(c - 4, 0)));
        q_of[i] = nsp++;
        qrow.push_back(i / s->NLz);  // x*NLy + y
      }
    }
    sp_off[s->NLx] = nsp;
    s->nsp = nsp;
    for (int x = 0; x < s->NLx; ++x) s->maxpts = std::max(s->maxpts, sp_off[x + 1] - sp_off[x]);
    for (int p = 0; p < s->NPI; ++p) qmap[p] = q_of[idx_proj[p]];
    // items covering each sphere point (an item covers every point of its atom)
    std::vector<int> icnt(std::max(1, nsp), 0);
    for (const int4& it : items)
      for (int p = atom_off[it.x]; p < atom_off[it.x + 1]; ++p) icnt[qmap[p]]++;
    kbq.resize(std::max(1, s->NPI), -1);
    for (int p = 0; p < s->NPI; ++p) kbq[p] = icnt[qmap[p]] == 1 ? qmap[p] : -1;
    for (int q = 0; q < nsp; ++q)
      if (icnt[q] > 1) kb_multi.push_back(q);
    s->n_multi = (int)kb_multi.size();
    if (s->maxpts > 32767) return bail(fail(SGPU_ERR_UNSUPPORTED, "sgpu_create: more than 32767 sphere points in one x-plane"));
  }
  std::vector<short> lqi(s->NL, (short)-1);
  for (int i = 0; i < s->NL; ++i)
    if (q_of[i] >= 0) lqi[i] = (short)(q_of[i] - sp_off[i / (s->NLy * s->NLz)]);
  for (int pr = 0; pr < 2; ++pr)
    if (sgpu::pass_smem_bytes(pr, s->NLy, s->NLz, s->maxpts, true, s->NLx, s->nyblk, s->NYB) > 227 * 1024)
      return bail(fail(SGPU_ERR_UNSUPPORTED, "sgpu_create: an NLy x NLz plane ring does not fit in shared memory"));
  std::vector<double> uv((size_t)s->Nlma * s->Nps);
  if (s->Nlma) std::memcpy(uv.data(), d->uV, uv.size() * sizeof(double));

  // per-orbital occupations of the resident (ik, ib) pairs
  std::vector<double> occo(s->norb);
  for (int kl = 0; kl < s->nkl; ++kl)
    for (int b = 0; b < s->NBocc; ++b) occo[kl * s->NBocc + b] = s->occ_h[(size_t)(s->NK_s - 1 + kl) * s->NB + b];

  // ---- device buffers
  int rc;
  if ((rc = alloc_state_buffers(s)) != 0) return bail(rc);
#define UP(ptr, vec) \
  do { e = upload(&ptr, vec.data(), vec.size(), s->stream); if (e != cudaSuccess) return bail(cuda_fail(e, "upload " #ptr)); } while (0)
  UP(s->idx_proj, idx_proj);
  UP(s->atom_off, atom_off);
  UP(s->rpos, rpos);
  UP(s->items, items);
  UP(s->lma_list, lma_list);
  UP(s->iuV_d, iuv);
  UP(s->lma_atom, lma_atom);
  UP(s->uV_d, uv);
  UP(s->sp_off, sp_off);
  UP(s->rec, rec);
  UP(s->cont, cont);
  UP(s->qmap, qmap);
  UP(s->kbq, kbq);
  UP(s->kb_multi, kb_multi);
  UP(s->lqi, lqi);
  {  // sp_blk: first sphere point of every (plane, y-block) and the plane end
    const int nb1 = s->nyblk + 1;
    std::vector<int> cnt((size_t)s->NLx * s->nyblk, 0), blk((size_t)s->NLx * nb1, 0);
    for (int r : qrow) cnt[(size_t)(r / s->NLy) * s->nyblk + (r % s->NLy) / s->NYB]++;
    int acc = 0;
    for (int x = 0; x < s->NLx; ++x) {
      for (int yb = 0; yb < s->nyblk; ++yb) {
        blk[(size_t)x * nb1 + yb] = acc;
        acc += cnt[(size_t)x * s->nyblk + yb];
      }
      blk[(size_t)x * nb1 + s->nyblk] = acc;
    }
    UP(s->sp_blk, blk);
  }
  UP(s->occ_o, occo);
#undef UP
  const size_t nz = (size_t)s->nkl * s->Nlma * s->Nps;
  if ((e = dalloc(&s->zproj64, nz)) != cudaSuccess) return bail(cuda_fail(e, "alloc zproj64"));
  if ((e = dalloc(&s->zproj32, nz)) != cudaSuccess) return bail(cuda_fail(e, "alloc zproj32"));
  if ((e = cudaMemsetAsync(s->zproj64, 0, std::max<size_t>(nz, 1) * sizeof(double2), s->stream)) != cudaSuccess)
    return bail(cuda_fail(e, "memset zproj64"));
  if ((e = cudaMemsetAsync(s->zproj32, 0, std::max<size_t>(nz, 1) * sizeof(float2), s->stream)) != cudaSuccess)
    return bail(cuda_fail(e, "memset zproj32"));
  if ((e = dalloc(&s->U, (size_t)s->norb * std::max(1, s->Nlma))) != cudaSuccess) return bail(cuda_fail(e, "alloc U"));
  s->U_rows = (size_t)s->norb;
  if ((e = dalloc(&s->Up, (size_t)sgpu::KB_USPLIT_MAX * s->norb * std::max(1, s->Nlma))) != cudaSuccess)
    return bail(cuda_fail(e, "alloc Up"));
  s->Up_rows = (size_t)sgpu::KB_USPLIT_MAX * s->norb;
  if ((e = cudaMalloc(&s->Sbuf, (size_t)s->norb * std::max(1, s->nsp) * sizeof(double2))) != cudaSuccess)
    return bail(cuda_fail(e, "alloc S"));
  if ((e = cudaMalloc(&s->Wbuf, (size_t)s->norb * std::max(1, s->nsp) * sizeof(double2))) != cudaSuccess)
    return bail(cuda_fail(e, "alloc W"));
  s->W_rows = (size_t)s->norb;
  {  // the weighted projections' point ranges: about eight CTAs per SM, at most one 128-point chunk each
    const long ctas = std::max(1L, (long)s->nitems * s->nkl * ((s->NBocc + 31) / 32));
    const int nch = std::max(1, (s->max_mps + 127) / 128);
    s->uvw_split = (int)std::max(1L, std::min<long>({8L, (8L * s->nsm + ctas - 1) / ctas, (long)nch}));
  }
  if ((e = dalloc(&s->Uw, (size_t)s->uvw_split * s->norb * std::max(1, s->Nlma) * 4)) != cudaSuccess)
    return bail(cuda_fail(e, "alloc Uw"));
  if ((e = dalloc(&s->kAc_d, 3 * (size_t)s->nkl)) != cudaSuccess) return bail(cuda_fail(e, "alloc kAc"));
  if ((e = dalloc(&s->vloc64, s->NL)) != cudaSuccess) return bail(cuda_fail(e, "alloc vloc64"));
  if ((e = dalloc(&s->vloc32, s->NL)) != cudaSuccess) return bail(cuda_fail(e, "alloc vloc32"));
  const size_t nchunk = (s->norb + 63) / 64;
  s->red_elems = std::max<size_t>({nchunk * s->NL, 4 * (size_t)s->norb + 64, (size_t)s->NL + 64,
                                   sgpu::current_red_elems(s->norb, s->NLx)});
  if ((e = dalloc(&s->red, s->red_elems)) != cudaSuccess) return bail(cuda_fail(e, "alloc red"));
  if ((e = dalloc(&s->cur_part, (size_t)s->norb * s->NLx * 4)) != cudaSuccess)
    return bail(cuda_fail(e, "alloc cur_part"));
  {
    double h12[12];
    for (int n = 0; n < 4; ++n)
      for (int dd = 0; dd < 3; ++dd) h12[4 * dd + n] = s->nab[dd][n + 1];
    if ((e = dalloc(&s->nab12, 12)) != cudaSuccess) return bail(cuda_fail(e, "alloc nab12"));
    if ((e = cudaMemcpy(s->nab12, h12, sizeof(h12), cudaMemcpyHostToDevice)) != cudaSuccess)
      return bail(cuda_fail(e, "copy nab12"));
  }
  s->red_h_elems = (size_t)s->NL + 64;
  if ((e = cudaMallocHost((void**)&s->red_h, s->red_h_elems * sizeof(double))) != cudaSuccess)
    return bail(cuda_fail(e, "alloc pinned"));
  if ((e = cudaMallocHost((void**)&s->in_h, ((size_t)s->NL + 3 * (size_t)s->nkl) * sizeof(double))) != cudaSuccess)
    return bail(cuda_fail(e, "alloc pinned inputs"));
  s->stage_elems = std::max<size_t>((size_t)4 * s->NL, std::min<size_t>((size_t)1 << 22, (size_t)s->norb * s->NL));
  if ((e = dalloc(&s->stage, s->stage_elems)) != cudaSuccess) return bail(cuda_fail(e, "alloc stage"));
  // zero kAc until the caller sets one
  std::vector<double> k0(3 * (size_t)s->nkl, 0.0);
  if ((e = cudaMemcpyAsync(s->kAc_d, k0.data(), k0.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream)) !=
      cudaSuccess)
    return bail(cuda_fail(e, "init kAc"));
  if ((e = cudaStreamSynchronize(s->stream)) != cudaSuccess) return bail(cuda_fail(e, "sgpu_create sync"));
  *out = s;
  return 0;
}

int sgpu_destroy(sgpu_handle h) {
  if (!h) return 0;
  System* s = h;
  if (s->stream) cudaStreamSynchronize(s->stream);
  sgpu::net_free(*s);
  free_state_buffers(s);
  void* bufs[] = {s->vloc64, s->vloc32, s->occ_o, s->kAc_d, s->idx_proj, s->atom_off, s->rpos, s->items,
                  s->lma_list, s->iuV_d, s->lma_atom, s->uV_d, s->zproj64, s->zproj32, s->sp_off, s->rec, s->cont, s->qmap, s->kbq, s->kb_multi, s->lqi, s->Sbuf, s->Wbuf,
                  s->U, s->Up, s->Uw, s->red, s->stage, s->cur_part, s->nab12};
  for (void* p : bufs) cudaFree(p);
  void* gbufs[] = {s->gs_zu, s->gs_aux, s->gs_W, s->gs_st, s->gs_part, s->gs_A, s->gs_V, s->gs_w, s->gs_sweeps,
                   s->occ_gs, s->gs_out, s->gs_res, s->gs_tb, s->vpsl, s->rho_d, s->exc_d, s->sp_blk,
                   s->vloc_hist};
  for (void* p : gbufs) cudaFree(p);
  if (s->gs_h) cudaFreeHost(s->gs_h);
  if (s->red_h) cudaFreeHost(s->red_h);
  if (s->aux) cudaStreamSynchronize(s->aux);
  if (s->in_h) cudaFreeHost(s->in_h);
  if (s->ev_vloc_in) cudaEventDestroy(s->ev_vloc_in);
  if (s->ev_kac_in) cudaEventDestroy(s->ev_kac_in);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->aux) cudaStreamDestroy(s->aux);
  if (s->ev_step) cudaEventDestroy(s->ev_step);
  if (s->ev_cur) cudaEventDestroy(s->ev_cur);
  delete h;
  return 0;
}

int sgpu_synchronize(sgpu_handle h) {
  if (!valid(h)) return fail(SGPU_ERR_ARG, "null handle");
  CK(h->aux_join());
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

void* sgpu_stream(sgpu_handle h) { return h ? (void*)h->stream : nullptr; }

void* sgpu_state_ptr(sgpu_handle h) { return h ? h->zu : nullptr; }

int sgpu_set_state(sgpu_handle h, const double* zu) {
  if (!valid(h) || !zu) return fail(SGPU_ERR_ARG, "sgpu_set_state: null argument");
  System* s = h;
  CK(s->aux_join());
  const size_t n = (size_t)s->norb * s->NL;
  if (s->prec == SGPU_PREC_C128) {
    CK(cudaMemcpyAsync(s->zu, zu, n * sizeof(double2), cudaMemcpyHostToDevice, s->stream));
  } else {
    for (size_t off = 0; off < n; off += s->stage_elems) {
      const size_t c = std::min(s->stage_elems, n - off);
      CK(cudaMemcpyAsync(s->stage, zu + 2 * off, c * sizeof(double2), cudaMemcpyHostToDevice, s->stream));
      CK(sgpu::launch_c128_to_c64(s->stage, (float2*)s->zu + off, c, s->stream));
    }
  }
  CK(cudaStreamSynchronize(s->stream));
  s->have_state = true;
  s->S_valid = false;
  s->cur_valid = false;
  return 0;
}

int sgpu_set_state_dev(sgpu_handle h, const void* zu_dev) {
  if (!valid(h) || !zu_dev) return fail(SGPU_ERR_ARG, "sgpu_set_state_dev: null argument");
  CK(h->aux_join());
  System* s = h;
  const size_t n = (size_t)s->norb * s->NL;
  if (s->prec == SGPU_PREC_C128)
    CK(cudaMemcpyAsync(s->zu, zu_dev, n * sizeof(double2), cudaMemcpyDeviceToDevice, s->stream));
  else
    CK(sgpu::launch_c128_to_c64(static_cast<const double2*>(zu_dev), (float2*)s->zu, n, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->have_state = true;
  s->S_valid = false;
  s->cur_valid = false;
  return 0;
}

int sgpu_get_state(sgpu_handle h, double* zu) {
  if (!valid(h) || !zu) return fail(SGPU_ERR_ARG, "sgpu_get_state: null argument");
  System* s = h;
  if (!s->have_state) return fail(SGPU_ERR_STATE, "sgpu_get_state: no state loaded");
  const size_t n = (size_t)s->norb * s->NL;
  if (s->prec == SGPU_PREC_C128) {
    CK(cudaMemcpyAsync(zu, s->zu, n * sizeof(double2), cudaMemcpyDeviceToHost, s->stream));
  } else {
    for (size_t off = 0; off < n; off += s->stage_elems) {
      const size_t c = std::min(s->stage_elems, n - off);
      CK(sgpu::launch_c64_to_c128((const float2*)s->zu + off, s->stage, c, s->stream));
      CK(cudaMemcpyAsync(zu + 2 * off, s->stage, c * sizeof(double2), cudaMemcpyDeviceToHost, s->stream));
    }
  }
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int sgpu_set_precision(sgpu_handle h, int precision) {
  if (!valid(h)) return fail(SGPU_ERR_ARG, "null handle");
  if (precision != SGPU_PREC_C128 && precision != SGPU_PREC_C64) return fail(SGPU_ERR_ARG, "bad precision");
  System* s = h;
  if (precision == s->prec) return 0;
  CK(s->aux_join());
  CK(cudaStreamSynchronize(s->stream));  // zu is freed below
  const size_t n = (size_t)s->norb * s->NL;
  void* old = s->zu;
  const int old_prec = s->prec;
  for (auto& t : s->tw) { cudaFree(t); t = nullptr; }
  s->zu = nullptr;
  s->prec = precision;
  s->S_valid = false;
  s->cur_valid = false;
  s->elem = precision == SGPU_PREC_C64 ? sizeof(float2) : sizeof(double2);
  CK(cudaMalloc(&s->zu, n * s->elem));
  if (s->have_state) {
    if (old_prec == SGPU_PREC_C128)
      CK(sgpu::launch_c128_to_c64((const double2*)old, (float2*)s->zu, n, s->stream));
    else
      CK(sgpu::launch_c64_to_c128((const float2*)old, (double2*)s->zu, n, s->stream));
  }
  CK(cudaStreamSynchronize(s->stream));
  cudaFree(old);
  for (auto& t : s->tw) CK(cudaMalloc(&t, n * s->elem));
  if (s->have_proj) CK(sgpu::launch_update_projector(*s));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int sgpu_set_vloc(sgpu_handle h, const double* vloc) {
  if (!valid(h) || !vloc) return fail(SGPU_ERR_ARG, "sgpu_set_vloc: null argument");
  System* s = h;
  if (s->vloc_in_pending) CK(cudaEventSynchronize(s->ev_vloc_in));  // see set_kac
  std::memcpy(s->in_h, vloc, s->NL * sizeof(double));
  CK(cudaMemcpyAsync(s->vloc64, s->in_h, s->NL * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(cudaEventRecord(s->ev_vloc_in, s->stream));
  s->vloc_in_pending = true;
  CK(sgpu::launch_r64_to_r32(s->vloc64, s->vloc32, s->NL, s->stream));
  s->have_vloc = true;
  return 0;
}

int sgpu_update_projector(sgpu_handle h, const double* kAc) {
  if (!valid(h) || !kAc) return fail(SGPU_ERR_ARG, "sgpu_update_projector: null argument");
  System* s = h;
  int rc = set_kac(s, kAc);
  if (rc) return rc;
  CK(sgpu::launch_update_projector(*s));
  s->have_proj = true;
  return 0;
}

int sgpu_hamiltonian(sgpu_handle h, double dt, int flag_current) {
  if (!valid(h)) return fail(SGPU_ERR_ARG, "null handle");
  System* s = h;
  if (!s->have_state || !s->have_vloc || !s->have_proj)
    return fail(SGPU_ERR_STATE, "sgpu_hamiltonian: state, Vloc and projectors must be set first");
  CK(sgpu::enqueue_taylor_step(*s, dt, !s->S_valid, flag_current != 0));
  return 0;
}

int sgpu_hpsi(sgpu_handle h, int ik, const double* tpsi, double* htpsi, double* ttpsi) {
  if (!valid(h) || !tpsi || !htpsi) return fail(SGPU_ERR_ARG, "sgpu_hpsi: null argument");
  System* s = h;
  if (ik < s->NK_s || ik > s->NK_e) return fail(SGPU_ERR_ARG, "sgpu_hpsi: ik outside NK_s..NK_e");
  if (!s->have_vloc || !s->have_proj) return fail(SGPU_ERR_STATE, "sgpu_hpsi: Vloc and projectors must be set first");
  const size_t NL = s->NL;
  double2* in128 = s->stage;
  double2* out128 = s->stage + NL;
  double2* tt128 = s->stage + 2 * NL;
  CK(cudaMemcpyAsync(in128, tpsi, NL * sizeof(double2), cudaMemcpyHostToDevice, s->stream));
  sgpu::PassIO io;
  const int ob = one_orbital_k(s, ik);
  if (s->prec == SGPU_PREC_C64) {
    // FP32 scratch inside the (unused between calls) Taylor workspace
    float2* in32 = (float2*)s->tw[0];
    float2* out32 = (float2*)s->tw[1];
    float2* tt32 = (float2*)s->tw[2];
    CK(sgpu::launch_c128_to_c64(in128, in32, NL, s->stream));
    io.in = in32; io.out = out32; io.tt = tt32;
    CK(apply_h(s, ttpsi ? 1 : 0, io, ob, 1, s->NBocc, -1, false));
    CK(sgpu::launch_c64_to_c128(out32, out128, NL, s->stream));
    if (ttpsi) CK(sgpu::launch_c64_to_c128(tt32, tt128, NL, s->stream));
  } else {
    io.in = in128; io.out = out128; io.tt = tt128;
    CK(apply_h(s, ttpsi ? 1 : 0, io, ob, 1, s->NBocc, -1, false));
  }
  CK(cudaMemcpyAsync(htpsi, out128, NL * sizeof(double2), cudaMemcpyDeviceToHost, s->stream));
  if (ttpsi) CK(cudaMemcpyAsync(ttpsi, tt128, NL * sizeof(double2), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int sgpu_hpsi_batch(sgpu_handle h, int ikb_s, int ikb_e, const void* tpsi, void* htpsi) {
  if (!valid(h) || !tpsi || !htpsi) return fail(SGPU_ERR_ARG, "sgpu_hpsi_batch: null argument");
  System* s = h;
  if (ikb_s < 1 || ikb_e < ikb_s || ikb_e > s->norb) return fail(SGPU_ERR_ARG, "sgpu_hpsi_batch: bad ikb range");
  if (!s->have_vloc || !s->have_proj) return fail(SGPU_ERR_STATE, "sgpu_hpsi_batch: Vloc and projectors must be set first");
  if (((uintptr_t)tpsi | (uintptr_t)htpsi) % 16 != 0)
    return fail(SGPU_ERR_ARG, "sgpu_hpsi_batch: tpsi and htpsi must be 16-byte aligned");
  const int nb = ikb_e - ikb_s + 1;
  sgpu::PassIO io;
  io.in = tpsi;
  io.out = htpsi;
  if ((size_t)nb > s->U_rows || (size_t)nb > s->W_rows) return fail(SGPU_ERR_ARG, "sgpu_hpsi_batch: batch too large");
  CK(apply_h(s, 0, io, ikb_s - 1, nb, s->NBocc, -1, false));
  return 0;
}

int sgpu_psi_rho(sgpu_handle h, double* rho_l) {
  if (!valid(h) || !rho_l) return fail(SGPU_ERR_ARG, "sgpu_psi_rho: null argument");
  System* s = h;
  if (!s->have_state) return fail(SGPU_ERR_STATE, "sgpu_psi_rho: no state loaded");
  double* out = s->stage ? (double*)s->stage : nullptr;  // NL doubles fit in the stage buffer
  CK(sgpu::launch_psi_rho(*s, out));
  CK(cudaMemcpyAsync(s->red_h, out, s->NL * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  std::memcpy(rho_l, s->red_h, s->NL * sizeof(double));
  return 0;
}

int sgpu_psi_rho_dev(sgpu_handle h, double* rho_dev) {
  if (!valid(h) || !rho_dev) return fail(SGPU_ERR_ARG, "sgpu_psi_rho_dev: null argument");
  System* s = h;
  if (!s->have_state) return fail(SGPU_ERR_STATE, "sgpu_psi_rho_dev: no state loaded");
  CK(sgpu::launch_psi_rho(*s, rho_dev));
  return 0;
}

int sgpu_current_dev(sgpu_handle h, const double* kAc, double* jav_dev) {
  if (!valid(h) || !kAc || !jav_dev) return fail(SGPU_ERR_ARG, "sgpu_current_dev: null argument");
  System* s = h;
  if (!s->have_state) return fail(SGPU_ERR_STATE, "sgpu_current_dev: no state loaded");
  int rc = sgpu_update_projector(h, kAc);  // current() rebuilds the projectors (current.f90:125)
  if (rc) return rc;
  CK(sgpu::launch_current(*s, jav_dev));
  return 0;
}

int sgpu_current(sgpu_handle h, const double* kAc, double* jav) {
  if (!valid(h) || !kAc || !jav) return fail(SGPU_ERR_ARG, "sgpu_current: null argument");
  System* s = h;
  if (!s->have_state) return fail(SGPU_ERR_STATE, "sgpu_current: no state loaded");
  int rc = sgpu_update_projector(h, kAc);  // current() rebuilds the projectors (current.f90:125)
  if (rc) return rc;
  double* out = (double*)s->stage;
  CK(sgpu::launch_current(*s, out));
  CK(cudaMemcpyAsync(s->red_h, out, 3 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  std::memcpy(jav, s->red_h, 3 * sizeof(double));
  return 0;
}

int sgpu_energy_terms(sgpu_handle h, const double* kAc, double* ekin, double* enl) {
  if (!valid(h) || !kAc || !ekin || !enl) return fail(SGPU_ERR_ARG, "sgpu_energy_terms: null argument");
  System* s = h;
  if (!s->have_state) return fail(SGPU_ERR_STATE, "sgpu_energy_terms: no state loaded");
  int rc = sgpu_update_projector(h, kAc);  // Total_Energy_omp calls update_projector(kac) (:122)
  if (rc) return rc;
  double* out = (double*)s->stage;
  CK(sgpu::launch_energy(*s, out));
  CK(cudaMemcpyAsync(s->red_h, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  *ekin = s->red_h[0];
  *enl = s->red_h[1];
  return 0;
}

int sgpu_time_kernel(sgpu_handle h, int kernel, int reps, double* ms_per_launch) {
  if (!valid(h) || !ms_per_launch || reps < 1) return fail(SGPU_ERR_ARG, "sgpu_time_kernel: bad argument");
  System* s = h;
  if (!s->have_state || !s->have_vloc || !s->have_proj)
    return fail(SGPU_ERR_STATE, "sgpu_time_kernel: state, Vloc and projectors must be set first");
  CK(s->aux_join());  // nothing of a flag_current step still runs beside the timed launches
  sgpu::PassIO io;
  io.zc[1] = -1e-3;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  auto launch = [&]() -> cudaError_t {
    switch (kernel) {
      case SGPU_KERNEL_STENCIL_PASS:  // as in the Taylor step: KB field added, sphere values exported
        io.in = s->zu; io.out = s->tw[0]; io.S = s->nsp > 0 ? s->Sbuf : nullptr; io.W = s->nsp > 0 ? s->Wbuf : nullptr;
        return sgpu::launch_hpsi_pass(*s, 0, io, 0, s->norb, s->NBocc);
      case SGPU_KERNEL_TAYLOR_LAST:  // one Taylor stage, tw[0] -> tw[1] (zu untouched)
        io.in = s->tw[0]; io.out = s->tw[1];
        io.S = s->nsp > 0 ? s->Sbuf : nullptr; io.W = s->nsp > 0 ? s->Wbuf : nullptr;
        return sgpu::launch_hpsi_pass(*s, 2, io, 0, s->norb, s->NBocc);
      case SGPU_KERNEL_KB_FIELD:
        return sgpu::launch_kbfield(*s, 0, s->norb, s->NBocc, s->Wbuf);
      case SGPU_KERNEL_UVPSI:  // projections from the exported sphere values (passes 2-4 of a step)
        return sgpu::launch_uvpsi_from_S(*s, s->Sbuf, 0, s->norb, s->NBocc, true);
      case SGPU_KERNEL_PSI_RHO:
        return sgpu::launch_psi_rho(*s, (double*)s->stage);
      case SGPU_KERNEL_KB_TERM:  // projections from S and the KB field in one kernel (as in the Taylor step)
        return sgpu::launch_kb_term(*s, s->zu, true, 0, s->norb, s->NBocc, s->Wbuf);
      case SGPU_KERNEL_CURRENT_STENCIL: {  // into the reduction scratch, not cur_part
        int nx = 1;
        return sgpu::launch_current_stencil(*s, s->red, nx);
      }
      case SGPU_KERNEL_CURRENT_PROJ: {  // from the sphere values, as after a Taylor step
        s->S_valid = s->Sbuf != nullptr;
        const cudaError_t e = sgpu::launch_current_proj(*s);
        s->S_valid = false;
        return e;
      }
      default:
        return cudaErrorInvalidValue;
    }
  };
  s->S_valid = false;           // the timed launches overwrite S with workspace values
  cudaError_t err = launch();  // warm-up (and argument check)
  if (err == cudaSuccess) err = cudaEventRecord(e0, s->stream);
  for (int r = 0; r < reps && err == cudaSuccess; ++r) err = launch();
  if (err == cudaSuccess) err = cudaEventRecord(e1, s->stream);
  if (err == cudaSuccess) err = cudaEventSynchronize(e1);
  float ms = 0;
  if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return cuda_fail(err, "sgpu_time_kernel");
  *ms_per_launch = ms / reps;
  return 0;
}

}  // extern "C"

// ------------------------------------------------------------ ground state --
namespace {

int gs_alloc(System* s) {
  if (s->gs_zu) return 0;
  const size_t nbl = (size_t)s->nkl * s->NB * s->NL;
  const int nt = (s->NB + 15) / 16;
  // split K so that the subspace GEMM has at least ~4 CTAs per SM
  s->gs_nsplit = std::max(1, std::min(64, (4 * 148 + s->nkl * nt * nt - 1) / std::max(1, s->nkl * nt * nt)));
  CK(cudaMalloc(&s->gs_zu, nbl * sizeof(double2)));
  CK(cudaMalloc(&s->gs_aux, nbl * sizeof(double2)));
  CK(cudaMalloc(&s->gs_W, (size_t)sgpu::cg_work_vectors() * s->nkl * s->NL * sizeof(double2)));
  CK(cudaMalloc(&s->gs_st, s->nkl * sgpu::cg_state_bytes()));
  CK(cudaMalloc(&s->gs_part, (size_t)s->gs_nsplit * s->nkl * s->NB * s->NB * sizeof(double2)));
  CK(cudaMalloc(&s->gs_A, (size_t)s->nkl * s->NB * s->NB * sizeof(double2)));
  CK(cudaMalloc(&s->gs_V, (size_t)s->nkl * s->NB * s->NB * sizeof(double2)));
  CK(cudaMalloc(&s->gs_w, (size_t)s->nkl * s->NB * sizeof(double)));
  CK(cudaMalloc(&s->gs_sweeps, (size_t)s->nkl * sizeof(int)));
  CK(cudaMalloc(&s->gs_out, (size_t)s->nkl * s->NB * sizeof(double)));
  CK(cudaMalloc(&s->gs_res, (size_t)s->nkl * s->NB * sizeof(double)));
  CK(cudaMemsetAsync(s->gs_res, 0, (size_t)s->nkl * s->NB * sizeof(double), s->stream));
  CK(cudaMalloc(&s->gs_tb, (size_t)s->nkl * sizeof(double)));
  CK(cudaMallocHost((void**)&s->gs_h, (size_t)s->nkl * s->NB * sizeof(double)));
  std::vector<double> occ((size_t)s->nkl * s->NB);
  for (int kl = 0; kl < s->nkl; ++kl)
    for (int b = 0; b < s->NB; ++b) occ[(size_t)kl * s->NB + b] = s->occ_h[(size_t)(s->NK_s - 1 + kl) * s->NB + b];
  CK(cudaMalloc(&s->occ_gs, occ.size() * sizeof(double)));
  CK(cudaMemcpyAsync(s->occ_gs, occ.data(), occ.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  const size_t rows = std::max((size_t)s->norb, (size_t)s->nkl * s->NB);
  if (rows > s->W_rows) {
    CK(cudaStreamSynchronize(s->stream));
    cudaFree(s->Wbuf);
    s->Wbuf = nullptr;
    CK(cudaMalloc(&s->Wbuf, rows * std::max(1, s->nsp) * sizeof(double2)));
    s->W_rows = rows;
  }
  if (rows > s->U_rows) {
    CK(cudaStreamSynchronize(s->stream));
    cudaFree(s->U);
    s->U = nullptr;
    CK(cudaMalloc(&s->U, rows * std::max(1, s->Nlma) * sizeof(double2)));
    s->U_rows = rows;
  }
  if ((size_t)sgpu::KB_USPLIT_MAX * rows > s->Up_rows) {  // the split KB form's partial projections
    CK(cudaStreamSynchronize(s->stream));
    cudaFree(s->Up);
    s->Up = nullptr;
    CK(cudaMalloc(&s->Up, (size_t)sgpu::KB_USPLIT_MAX * rows * std::max(1, s->Nlma) * sizeof(double2)));
    s->Up_rows = (size_t)sgpu::KB_USPLIT_MAX * rows;
  }
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

// FP64 H applied to a batch of nb vectors of the k-points o/nbk (mode 0 or 1).
// A small batch (CG works on one vector per k-point) is split into x-slabs of at
// least 8 planes so that its pass covers the SMs (the handle's own x-slab setting
// is for the resident orbitals).
int gs_hpsi(System* s, const double2* in, double2* out, double2* tt, int nb, int nbk) {
  sgpu::PassIO io;
  io.in = in;
  io.out = out;
  io.tt = tt;
  const int keep = s->nslab;
  if (s->nyblk == 1) s->nslab = std::max(1, std::min(s->nsm / std::max(1, nb), s->NLx / 8));
  const cudaError_t e = apply_h(s, tt ? 1 : 0, io, 0, nb, nbk, SGPU_PREC_C128, false);
  s->nslab = keep;
  CK(e);
  return 0;
}

int gs_ready(System* s, const char* who) {
  if (!s->have_gs) return fail(SGPU_ERR_STATE, std::string(who) + ": no ground-state orbitals loaded");
  if (!s->have_vloc || !s->have_proj) return fail(SGPU_ERR_STATE, std::string(who) + ": Vloc and projectors must be set first");
  return 0;
}

int gs_copy_out(System* s, const double* dev, double* host) {
  if (!host) return 0;
  const size_t n = (size_t)s->nkl * s->NB;
  CK(cudaMemcpyAsync(s->gs_h, dev, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  std::memcpy(host, s->gs_h, n * sizeof(double));
  return 0;
}

}  // namespace

extern "C" {

int sgpu_gs_set_state(sgpu_handle h, const double* zu_gs) {
  if (!valid(h) || !zu_gs) return fail(SGPU_ERR_ARG, "sgpu_gs_set_state: null argument");
  System* s = h;
  int rc = gs_alloc(s);
  if (rc) return rc;
  CK(cudaMemcpyAsync(s->gs_zu, zu_gs, (size_t)s->nkl * s->NB * s->NL * sizeof(double2), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->have_gs = true;
  return 0;
}

int sgpu_gs_get_state(sgpu_handle h, double* zu_gs) {
  if (!valid(h) || !zu_gs) return fail(SGPU_ERR_ARG, "sgpu_gs_get_state: null argument");
  System* s = h;
  if (!s->have_gs) return fail(SGPU_ERR_STATE, "sgpu_gs_get_state: no ground-state orbitals loaded");
  CK(cudaMemcpyAsync(zu_gs, s->gs_zu, (size_t)s->nkl * s->NB * s->NL * sizeof(double2), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int sgpu_gram_schmidt(sgpu_handle h) {
  if (!valid(h)) return fail(SGPU_ERR_ARG, "null handle");
  System* s = h;
  if (!s->have_gs) return fail(SGPU_ERR_STATE, "sgpu_gram_schmidt: no ground-state orbitals loaded");
  CK(sgpu::launch_gram_schmidt(*s, s->gs_zu));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int sgpu_cg(sgpu_handle h, int ncg, double* esp_var, int* iters) {
  if (!valid(h) || ncg < 1) return fail(SGPU_ERR_ARG, "sgpu_cg: bad argument");
  System* s = h;
  int rc = gs_ready(s, "sgpu_cg");
  if (rc) return rc;
  const size_t NL = s->NL, nk = s->nkl;
  double2* W = s->gs_W;
  auto vec = [&](int which) { return W + (size_t)which * nk * NL; };
  std::vector<int> it_all(iters ? (size_t)s->nkl * s->NB : 0);
  std::vector<char> st_h(s->nkl * sgpu::cg_state_bytes());
  for (int ib = 0; ib < s->NB; ++ib) {
    CK(sgpu::launch_cg_begin(*s, s->gs_zu, W, s->gs_st, ib));
    if ((rc = gs_hpsi(s, vec(0), vec(1), vec(2), s->nkl, 1))) return rc;   // xk -> hxk, txk
    CK(sgpu::launch_cg_dot0(*s, W, s->gs_st));
    for (int iter = 1; iter <= ncg; ++iter) {
      if (s->cg_precond == 0) {  // the reference's CG (CG.f90:85-106)
        CK(sgpu::launch_cg_pre(*s, s->gs_zu, W, s->gs_st, ib, iter));
      } else {                   // preconditioned direction
        CK(sgpu::launch_cg_grad(*s, s->gs_zu, W, s->gs_st, s->gs_tb, ib));
        CK(sgpu::launch_tpa(*s, vec(8), s->nkl, s->gs_tb, 1));                      // kinetic-energy factor
        if (s->cg_precond == 2) CK(sgpu::launch_precond_net(*s, vec(8), s->nkl));  // learned refinement
        CK(sgpu::launch_cg_dir(*s, s->gs_zu, W, s->gs_st, ib, iter));
      }
      if ((rc = gs_hpsi(s, vec(5), vec(6), vec(7), s->nkl, 1))) return rc; // pko -> htpsi, ttpsi
      CK(sgpu::launch_cg_post(*s, W, s->gs_st, iter));
    }
    CK(sgpu::launch_cg_end(*s, s->gs_zu, W, ib));
    if ((rc = gs_hpsi(s, vec(0), vec(6), nullptr, s->nkl, 1))) return rc;  // H u_ib
    CK(sgpu::launch_cg_resid(*s, W, s->occ_gs, s->gs_out, s->gs_res, ib));
    if (iters) {
      CK(cudaMemcpyAsync(st_h.data(), s->gs_st, st_h.size(), cudaMemcpyDeviceToHost, s->stream));
      CK(cudaStreamSynchronize(s->stream));
      for (int k = 0; k < s->nkl; ++k) {
        int v;
        std::memcpy(&v, st_h.data() + k * sgpu::cg_state_bytes() + 2 * sizeof(double) + sizeof(int), sizeof(int));
        it_all[(size_t)k * s->NB + ib] = v;
      }
    }
  }
  if ((rc = gs_copy_out(s, s->gs_out, esp_var))) return rc;
  if (iters) std::memcpy(iters, it_all.data(), it_all.size() * sizeof(int));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int sgpu_set_vpsl(sgpu_handle h, const double* vpsl) {
  if (!valid(h) || !vpsl) return fail(SGPU_ERR_ARG, "sgpu_set_vpsl: null argument");
  System* s = h;
  if (!s->vpsl) {
    CK(cudaMalloc(&s->vpsl, (size_t)s->NL * sizeof(double)));
    CK(cudaMalloc(&s->rho_d, (size_t)s->NL * sizeof(double)));
    CK(cudaMalloc(&s->exc_d, 2 * sizeof(double)));
  }
  CK(cudaMemcpyAsync(s->vpsl, vpsl, (size_t)s->NL * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int sgpu_update_vloc(sgpu_handle h, const double* rho, double* eh_exc) {
  if (!valid(h)) return fail(SGPU_ERR_ARG, "null handle");
  System* s = h;
  if (!s->vpsl) return fail(SGPU_ERR_STATE, "sgpu_update_vloc: call sgpu_set_vpsl first");
  if (!(sgpu::fft_size_ok(s->NLx) && sgpu::fft_size_ok(s->NLy) && sgpu::fft_size_ok(s->NLz)))
    return fail(SGPU_ERR_UNSUPPORTED, "sgpu_update_vloc: grid sizes must be 2^a 3^b <= 96");
  if (rho) {
    CK(cudaMemcpyAsync(s->rho_d, rho, (size_t)s->NL * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  } else {
    if (!s->have_state) return fail(SGPU_ERR_STATE, "sgpu_update_vloc: no state loaded");
    CK(sgpu::launch_psi_rho(*s, s->rho_d));
  }
  CK(sgpu::launch_update_vloc(*s, s->rho_d, s->exc_d));
  if (eh_exc) CK(cudaMemcpyAsync(eh_exc, s->exc_d, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->have_vloc = true;
  return 0;
}

int sgpu_update_vloc_dev(sgpu_handle h, const double* rho_dev, double* eh_exc_dev) {
  if (!valid(h) || !rho_dev) return fail(SGPU_ERR_ARG, "sgpu_update_vloc_dev: null argument");
  System* s = h;
  if (!s->vpsl) return fail(SGPU_ERR_STATE, "sgpu_update_vloc_dev: call sgpu_set_vpsl first");
  if (!(sgpu::fft_size_ok(s->NLx) && sgpu::fft_size_ok(s->NLy) && sgpu::fft_size_ok(s->NLz)))
    return fail(SGPU_ERR_UNSUPPORTED, "sgpu_update_vloc_dev: grid sizes must be 2^a 3^b <= 96");
  CK(sgpu::launch_update_vloc(*s, rho_dev, eh_exc_dev ? eh_exc_dev : s->exc_d));
  s->have_vloc = true;
  return 0;
}

int sgpu_vloc_history_reset(sgpu_handle h) {
  if (!valid(h)) return fail(SGPU_ERR_ARG, "null handle");
  System* s = h;
  if (!s->have_vloc) return fail(SGPU_ERR_STATE, "sgpu_vloc_history_reset: no Vloc set");
  if (!s->vloc_hist) CK(cudaMalloc(&s->vloc_hist, 2 * (size_t)s->NL * sizeof(double)));
  CK(sgpu::launch_vloc_history(*s, false));
  return 0;
}

int sgpu_vloc_extrapolate(sgpu_handle h) {
  if (!valid(h)) return fail(SGPU_ERR_ARG, "null handle");
  System* s = h;
  if (!s->vloc_hist) return fail(SGPU_ERR_STATE, "sgpu_vloc_extrapolate: call sgpu_vloc_history_reset first");
  CK(sgpu::launch_vloc_history(*s, true));
  return 0;
}

int sgpu_get_vloc(sgpu_handle h, double* vloc) {
  if (!valid(h) || !vloc) return fail(SGPU_ERR_ARG, "sgpu_get_vloc: null argument");
  System* s = h;
  if (!s->have_vloc) return fail(SGPU_ERR_STATE, "sgpu_get_vloc: no Vloc set");
  CK(cudaMemcpyAsync(vloc, s->vloc64, (size_t)s->NL * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return 0;
}

int sgpu_set_cg_delta(sgpu_handle h, double delta_cg) {
  if (!valid(h) || !(delta_cg > 0.0)) return fail(SGPU_ERR_ARG, "sgpu_set_cg_delta: need a positive threshold");
  h->cg_delta = delta_cg;
  return 0;
}

int sgpu_cg_residuals(sgpu_handle h, double* res) {
  if (!valid(h) || !res) return fail(SGPU_ERR_ARG, "sgpu_cg_residuals: null argument");
  System* s = h;
  if (!s->have_gs) return fail(SGPU_ERR_STATE, "sgpu_cg_residuals: no ground-state orbitals loaded");
  return gs_copy_out(s, s->gs_res, res);
}

int sgpu_subspace_diag(sgpu_handle h, double* esp) {
  if (!valid(h)) return fail(SGPU_ERR_ARG, "null handle");
  System* s = h;
  int rc = gs_ready(s, "sgpu_subspace_diag");
  if (rc) return rc;
  if ((rc = gs_hpsi(s, s->gs_zu, s->gs_aux, nullptr, s->nkl * s->NB, s->NB))) return rc;
  CK(sgpu::launch_subspace_h(*s, s->gs_zu, s->gs_aux, s->gs_part, s->gs_nsplit, s->gs_A));
  CK(sgpu::launch_jacobi(*s, s->gs_A, s->gs_V, 30, s->gs_w, s->gs_sweeps));
  CK(sgpu::launch_rotate(*s, s->gs_zu, s->gs_A, s->gs_aux));
  std::swap(s->gs_zu, s->gs_aux);
  return gs_copy_out(s, s->gs_w, esp) ? SGPU_ERR_CUDA : (cudaStreamSynchronize(s->stream) == cudaSuccess ? 0 : cuda_fail(cudaGetLastError(), "sgpu_subspace_diag"));
}

int sgpu_gs_to_rt(sgpu_handle h) {
  if (!valid(h)) return fail(SGPU_ERR_ARG, "null handle");
  System* s = h;
  if (!s->have_gs) return fail(SGPU_ERR_STATE, "sgpu_gs_to_rt: no ground-state orbitals loaded");
  CK(s->aux_join());
  const size_t run = (size_t)s->NBocc * s->NL;
  for (int k = 0; k < s->nkl; ++k) {
    const double2* src = s->gs_zu + (size_t)k * s->NB * s->NL;
    if (s->prec == SGPU_PREC_C128)
      CK(cudaMemcpyAsync((double2*)s->zu + (size_t)k * run, src, run * sizeof(double2), cudaMemcpyDeviceToDevice, s->stream));
    else
      CK(sgpu::launch_c128_to_c64(src, (float2*)s->zu + (size_t)k * run, run, s->stream));
  }
  CK(cudaStreamSynchronize(s->stream));
  s->have_state = true;
  s->S_valid = false;
  s->cur_valid = false;
  return 0;
}

}  // extern "C"

extern "C" int sgpu_set_param(sgpu_handle h, int param, int value) {
  if (!valid(h)) return fail(SGPU_ERR_ARG, "null handle");
  System* s = h;
  switch (param) {
    case SGPU_PARAM_NSLAB:
      if (value < 1 || value > s->NLx) return fail(SGPU_ERR_ARG, "sgpu_set_param: nslab must be in 1..NLx");
      s->nslab = value;
      return 0;
    case SGPU_PARAM_CG_PRECOND:
      if (value < 0 || value > 2) return fail(SGPU_ERR_ARG, "sgpu_set_param: CG preconditioner must be 0, 1 or 2");
      if (value >= 1 && !(sgpu::fft_size_ok(s->NLx) && sgpu::fft_size_ok(s->NLy) && sgpu::fft_size_ok(s->NLz)))
        return fail(SGPU_ERR_UNSUPPORTED, "sgpu_set_param: the TPA preconditioner needs grid sizes 2^a 3^b <= 96");
      if (value == 2 && !s->net_ready) return fail(SGPU_ERR_STATE, "sgpu_set_param: no preconditioner network loaded");
      s->cg_precond = value;
      return 0;
    case SGPU_PARAM_UVPSI_SPLIT:
      if (value != 1 && value != 2 && value != 4 && value != 8)
        return fail(SGPU_ERR_ARG, "sgpu_set_param: uvpsi split must be 1, 2, 4 or 8");
      s->um_split = value;
      return 0;
    case SGPU_PARAM_PASS_TABLES:
      if (value != 0 && value != 1) return fail(SGPU_ERR_ARG, "sgpu_set_param: pass tables must be 0 or 1");
      s->pass_tab = value;
      if (sgpu::prepare_pass(*s) != cudaSuccess) return fail(SGPU_ERR_CUDA, "sgpu_set_param: pass setup failed");
      return 0;
    case SGPU_PARAM_KB_KERNEL:
      if (value < 0 || value > 3) return fail(SGPU_ERR_ARG, "sgpu_set_param: KB kernel must be 0 to 3");
      s->kb_kernel = value;
      return 0;
    case SGPU_PARAM_KB_SPLIT:
      if (value < 0 || value > sgpu::KB_USPLIT_MAX) return fail(SGPU_ERR_ARG, "sgpu_set_param: KB split must be 0 to 8");
      s->kb_usplit = value;
      return 0;
    case SGPU_PARAM_CUR_FIXED:
      if (value < 0 || value > 2) return fail(SGPU_ERR_ARG, "sgpu_set_param: current fixed shape must be 0, 1 or 2");
      s->cur_fixed = value;
      return 0;
    case SGPU_PARAM_PASS_FIXED:
      if (value != 0 && value != 1) return fail(SGPU_ERR_ARG, "sgpu_set_param: pass fixed shapes must be 0 or 1");
      s->pass_fixed = value;
      if (sgpu::prepare_pass(*s) != cudaSuccess) return fail(SGPU_ERR_CUDA, "sgpu_set_param: pass setup failed");
      return 0;
    case SGPU_PARAM_TAYLOR_KERNEL:
      if (value < 0 || value > 2) return fail(SGPU_ERR_ARG, "sgpu_set_param: Taylor kernel must be 0, 1 or 2");
      if (value == 2 && !sgpu::resident_step_fits(*s))
        return fail(SGPU_ERR_UNSUPPORTED, "sgpu_set_param: no shared-memory resident Taylor step for this grid");
      s->taylor_kernel = value;
      if (sgpu::prepare_resident(*s) != cudaSuccess) return fail(SGPU_ERR_CUDA, "sgpu_set_param: resident setup failed");
      return 0;
    case SGPU_PARAM_LAUNCHES:
      if (value != 0) return fail(SGPU_ERR_ARG, "sgpu_set_param: the launch counter can only be reset to 0");
      s->launches = 0;
      return 0;
    default:
      return fail(SGPU_ERR_ARG, "sgpu_set_param: unknown parameter");
  }
}

extern "C" int sgpu_get_param(sgpu_handle h, int param, int* value) {
  if (!valid(h) || !value) return fail(SGPU_ERR_ARG, "sgpu_get_param: null argument");
  switch (param) {
    case SGPU_PARAM_NSLAB: *value = h->nslab; return 0;
    case SGPU_PARAM_LAUNCHES: *value = (int)(h->launches & 0x7fffffffULL); return 0;
    case SGPU_PARAM_UVPSI_SPLIT: *value = h->um_split; return 0;
    case SGPU_PARAM_CG_PRECOND: *value = h->cg_precond; return 0;
    case SGPU_PARAM_PASS_TABLES: *value = h->pass_tab; return 0;
    case SGPU_PARAM_KB_KERNEL: *value = h->kb_kernel; return 0;
    case SGPU_PARAM_PASS_FIXED: *value = h->pass_fixed; return 0;
    case SGPU_PARAM_CUR_FIXED: *value = h->cur_fixed; return 0;
    case SGPU_PARAM_TAYLOR_KERNEL: *value = h->taylor_kernel; return 0;
    case SGPU_PARAM_NSP: *value = h->nsp; return 0;
    case SGPU_PARAM_KB_SPLIT: *value = h->kb_usplit; return 0;
    default: return fail(SGPU_ERR_ARG, "sgpu_get_param: unknown parameter");
  }
}

extern "C" int sgpu_autotune(sgpu_handle h, int reps, int* nslab, int* split, double* ms) {
  if (!valid(h) || reps < 1) return fail(SGPU_ERR_ARG, "sgpu_autotune: bad argument");
  System* s = h;
  if (!s->have_state || !s->have_vloc || !s->have_proj)
    return fail(SGPU_ERR_STATE, "sgpu_autotune: state, Vloc and projectors must be set first");
  // one H application as in passes 2-3 of a Taylor step: projections from S,
  // KB field, stencil pass with export; zu -> workspace 0 (zu is not modified)
  sgpu::PassIO io;
  io.in = s->zu;
  io.out = s->tw[0];
  io.S = s->nsp > 0 ? s->Sbuf : nullptr;
  const bool from_S = s->nsp > 0;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int old_slab = s->nslab, old_split = s->um_split, old_kb = s->kb_kernel;
  double best = 1e300;
  int bs = old_slab, bk = old_split;
  cudaError_t err = cudaSuccess;
  for (int ns : {1, 2, 4}) {
    if (ns > 1 && s->NLx / ns < 8) continue;
    for (int sp : {0, 1, 2, 4, 8}) {  // 0: the band-group tile kernel
      if (sp == 0 && !sgpu::kb_tile_fits(*s)) continue;
      s->nslab = ns;
      s->um_split = sp ? sp : old_split;
      s->kb_kernel = sp ? 2 : 1;
      err = apply_h(s, 0, io, 0, s->norb, s->NBocc, -1, from_S);  // warm-up
      if (err == cudaSuccess) err = cudaEventRecord(e0, s->stream);
      for (int r = 0; r < reps && err == cudaSuccess; ++r) err = apply_h(s, 0, io, 0, s->norb, s->NBocc, -1, from_S);
      if (err == cudaSuccess) err = cudaEventRecord(e1, s->stream);
      if (err == cudaSuccess) err = cudaEventSynchronize(e1);
      float t = 0;
      if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
      if (err != cudaSuccess) break;
      if (t / reps < best) { best = t / reps; bs = ns; bk = sp; }
    }
    if (err != cudaSuccess) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s->S_valid = false;  // the timed applications overwrote S
  if (err != cudaSuccess) {
    s->nslab = old_slab;
    s->um_split = old_split;
    s->kb_kernel = old_kb;
    return cuda_fail(err, "sgpu_autotune");
  }
  s->nslab = bs;
  s->um_split = bk ? bk : old_split;
  s->kb_kernel = bk ? 2 : 1;
  if (nslab) *nslab = bs;
  if (split) *split = bk;
  if (ms) *ms = best;
  return 0;
}

// ------------------------------------------------------------ step tuner --
// Times whole Taylor steps on a copy of the orbitals (tw[2]; the resident
// orbitals are not modified) for every combination of the launch choices that
// apply to the handle's shapes, keeps the fastest in the handle and returns it.
extern "C" int sgpu_autotune_step(sgpu_handle h, double dt, int reps, int* params, double* ms_per_step) {
  if (!valid(h) || reps < 1) return fail(SGPU_ERR_ARG, "sgpu_autotune_step: bad argument");
  System* s = h;
  if (!s->have_state || !s->have_vloc || !s->have_proj)
    return fail(SGPU_ERR_STATE, "sgpu_autotune_step: state, Vloc and projectors must be set first");
  const size_t bytes = (size_t)s->norb * s->NL * s->elem;
  CK(cudaMemcpyAsync(s->tw[2], s->zu, bytes, cudaMemcpyDeviceToDevice, s->stream));
  const int old[6] = {s->taylor_kernel, s->pass_fixed, s->pass_tab, s->nslab, s->kb_kernel, s->um_split};
  auto apply = [&](const int* p) {
    s->taylor_kernel = p[0]; s->pass_fixed = p[1]; s->pass_tab = p[2]; s->nslab = p[3]; s->kb_kernel = p[4];
    s->um_split = p[5];
  };
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double best = 1e300;
  int bp[6] = {old[0], old[1], old[2], old[3], old[4], old[5]};
  cudaError_t err = cudaSuccess;
  std::vector<std::array<int, 6>> cands;
  if (sgpu::resident_step_fits(*s)) cands.push_back({2, old[1], old[2], old[3], old[4], old[5]});
  for (int pf : {1, 0})
    for (int pt : {1, 0})
      for (int ns : {1, 2, 4}) {
        if (ns > 1 && s->NLx / ns < 8) continue;
        for (int sp : {-1, 0, 1, 2, 4, 8}) {  // -1: the split tile, 0: the band-group tile kernel
          if (sp <= 0 && !sgpu::kb_tile_fits(*s)) continue;
          cands.push_back({1, pf, pt, ns, sp < 0 ? 3 : (sp ? 2 : 1), sp > 0 ? sp : old[5]});
        }
      }
  for (const auto& c : cands) {
    apply(c.data());
    if ((err = sgpu::prepare_pass(*s)) != cudaSuccess) break;
    if ((err = sgpu::prepare_resident(*s)) != cudaSuccess) break;
    err = sgpu::enqueue_taylor_step_on(*s, s->tw[2], dt, true, false);  // warm-up
    if (err == cudaSuccess) err = cudaEventRecord(e0, s->stream);
    for (int r = 0; r < reps && err == cudaSuccess; ++r)
      err = sgpu::enqueue_taylor_step_on(*s, s->tw[2], dt, r == 0, false);
    if (err == cudaSuccess) err = cudaEventRecord(e1, s->stream);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float t = 0;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
    if (err != cudaSuccess) break;
    if (t / reps < best) {
      best = t / reps;
      for (int k = 0; k < 6; ++k) bp[k] = c[k];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  s->S_valid = false;  // the timed steps overwrote S
  s->cur_valid = false;
  if (err != cudaSuccess) {
    apply(old);
    return cuda_fail(err, "sgpu_autotune_step");
  }
  apply(bp);
  if (sgpu::prepare_pass(*s) != cudaSuccess || sgpu::prepare_resident(*s) != cudaSuccess)
    return fail(SGPU_ERR_CUDA, "sgpu_autotune_step: setup of the chosen shapes failed");
  if (params)
    for (int k = 0; k < 6; ++k) params[k] = bp[k];
  if (ms_per_step) *ms_per_step = best;
  return 0;
}
