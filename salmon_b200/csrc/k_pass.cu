// One Hamiltonian application (and the fused last Taylor pass) for sm_100a.
//
// H psi = (k2lap0_2 + Vloc) psi - 1/2 sum lapt (psi(+n)+psi(-n)) - i sum nabt (psi(+n)-psi(-n))
//         + sum_ilma zproj(:,ilma) U(ilma)
// restates hpsi_omp_KB_base (common/hpsi.f90:98-208): the stencil of
// stencil/F90/hpsi.f90:190 and the Kleinman-Bylander scatter of pseudo_pt (:194-206).
//
// Layout: one CTA per (orbital, x-slab).  A y-z plane of one orbital is a
// contiguous NLy*NLz run in HBM (z unit stride).  Each thread owns RZ
// consecutive z points of one y row and marches along x:
//   * planes stream into a shared-memory ring with cp.async, NR-5 planes ahead
//     of use, so HBM latency is off the critical path;
//   * the thread's own 9 x-neighbours sit in a register queue that rotates by
//     unrolling the march 9 times (no register moves);
//   * y and z neighbours come from the shared-memory plane;
//   * the Kleinman-Bylander term of plane x+1 is assembled during plane x: the
//     (zproj offset, ilma, position) entries of its sphere points are spread over
//     all threads (MAXE lanes per point), their zproj values are loaded one
//     plane ahead, and a segmented warp shuffle sums each point's entries in a
//     fixed order into a shared-memory plane (deterministic, no atomics);
//   * complex(4): every accumulation is a packed FP32x2 FMA (__ffma2_rn).
// Each input element is read from HBM once per pass (the 8 halo planes of a
// slab come from L2), each output element written once.
#include <cuda_runtime.h>

#include <type_traits>
#include <utility>

#include "sgpu_internal.cuh"

namespace sgpu {

template <typename R>
struct PassArgs {
  const C2<R>* in;       // [nb][NL]
  C2<R>* out;            // [nb][NL]   (modes 0,1)
  C2<R>* tt;             // [nb][NL]   (mode 1)
  const C2<R>* t1;       // [nb][NL]   (mode 2)
  const C2<R>* t2;
  C2<R>* zu;             // [nb][NL]   (mode 2, read and written)
  const R* vloc;
  const double* kAc;     // [nkl][3]
  int o_beg, NBocc;
  int NLx, NLy, NLz, NL, SX;
  double lap0sum;        // lapx(0)+lapy(0)+lapz(0)
  C2<R> lap2[12];        // {lap, lap} for lapx(1:4), lapy(1:4), lapz(1:4)
  C2<R> nab2[12];        // {nab, nab} for nabx(1:4), ...
  // Kleinman-Bylander sphere points by plane: points sp_off[x] .. sp_off[x+1]-1
  // of plane x, record q = {pos, cnt, e0, e1}, {e2, e3, -, -}, e = ilma<<16 | j.
  const int* sp_off;
  const int4* rec;
  C2<R>* S;              // [nb][nsp] output at the sphere points (null: no export)
  int nsp;
  const C2<R>* zproj;    // [nkl][Nlma][Nps]
  const double2* U;      // [nb][Nlma]
  int Nlma, Nps;
  C2<R> zf[4];
};

// ------------------------------------------------------------- helpers ---
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ double2 fma2(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ double2 neg2(double2 a) { return make_double2(-a.x, -a.y); }
template <typename R> __device__ __forceinline__ C2<R> splat(R c) { return mk<R>(c, c); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// asynchronous copy of this thread's RZ consecutive points (aligned runs)
template <typename R, int RZ>
__device__ __forceinline__ void cp_run(C2<R>* dst, const C2<R>* src) {
  constexpr int BYTES = RZ * (int)sizeof(C2<R>);
  if constexpr (BYTES == 8) {
    cp_async8(dst, src);
  } else {
#pragma unroll
    for (int k = 0; k < BYTES / 16; ++k)
      cp_async16(reinterpret_cast<char*>(dst) + 16 * k, reinterpret_cast<const char*>(src) + 16 * k);
  }
}

template <typename R, int RZ>
__device__ __forceinline__ void ld_run(C2<R> (&d)[RZ], const C2<R>* p) {
  if constexpr (RZ == 2 && std::is_same<R, float>::value) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    d[0] = make_float2(t.x, t.y);
    d[1] = make_float2(t.z, t.w);
  } else {
#pragma unroll
    for (int r = 0; r < RZ; ++r) d[r] = __ldg(p + r);
  }
}
template <typename R, int RZ>
__device__ __forceinline__ void ld_run_rw(C2<R> (&d)[RZ], const C2<R>* p) {
  if constexpr (RZ == 2 && std::is_same<R, float>::value) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    d[0] = make_float2(t.x, t.y);
    d[1] = make_float2(t.z, t.w);
  } else {
#pragma unroll
    for (int r = 0; r < RZ; ++r) d[r] = p[r];
  }
}
template <typename R, int RZ>
__device__ __forceinline__ void st_run(C2<R>* p, const C2<R> (&d)[RZ]) {
  if constexpr (RZ == 2 && std::is_same<R, float>::value) {
    *reinterpret_cast<float4*>(p) = make_float4(d[0].x, d[0].y, d[1].x, d[1].y);
  } else {
#pragma unroll
    for (int r = 0; r < RZ; ++r) p[r] = d[r];
  }
}
template <typename R, int RZ>
__device__ __forceinline__ void lds_run(C2<R> (&d)[RZ], const C2<R>* p) {
  if constexpr (RZ == 2 && std::is_same<R, float>::value) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    d[0] = make_float2(t.x, t.y);
    d[1] = make_float2(t.z, t.w);
  } else {
#pragma unroll
    for (int r = 0; r < RZ; ++r) d[r] = p[r];
  }
}

__device__ __forceinline__ int wrapi(int a, int n) { a %= n; return a < 0 ? a + n : a; }

template <typename R> struct PassGeom {
  static constexpr int NR = std::is_same<R, float>::value ? 8 : 6;  // ring planes
};

// Kleinman-Bylander term of one sphere point: sum over its <= 4 (ilma, j)
// entries of zproj(j,ilma) U(ilma), in entry order.
template <typename R>
__device__ __forceinline__ C2<R> kb_point(const int4& ra, const int4& rb, const C2<R> (&zv)[4], const C2<R>* Us) {
  const int cnt = ra.y;
  C2<R> acc = mk<R>(0, 0);
  if (cnt > 0) acc = cfma(zv[0], Us[ra.z >> 16], acc);
  if (cnt > 1) acc = cfma(zv[1], Us[ra.w >> 16], acc);
  if (cnt > 2) acc = cfma(zv[2], Us[rb.x >> 16], acc);
  if (cnt > 3) acc = cfma(zv[3], Us[rb.y >> 16], acc);
  return acc;
}
__device__ __forceinline__ int kb_zoff(int e, int Nps) { return (e >> 16) * Nps + (e & 0xffff); }
template <typename R>
__device__ __forceinline__ void kb_load_zproj(const int4& ra, const int4& rb, const C2<R>* zp, int Nps,
                                              C2<R> (&zv)[4]) {
  const int cnt = ra.y;
  zv[0] = cnt > 0 ? __ldg(zp + kb_zoff(ra.z, Nps)) : mk<R>(0, 0);
  zv[1] = cnt > 1 ? __ldg(zp + kb_zoff(ra.w, Nps)) : mk<R>(0, 0);
  zv[2] = cnt > 2 ? __ldg(zp + kb_zoff(rb.x, Nps)) : mk<R>(0, 0);
  zv[3] = cnt > 3 ? __ldg(zp + kb_zoff(rb.y, Nps)) : mk<R>(0, 0);
}
__device__ __forceinline__ void kb_load_rec(const int* sp_off, const int4* rec, int p, int4& ra, int4& rb) {
  const int q = __ldg(sp_off + p) + (int)threadIdx.x;
  if (q < __ldg(sp_off + p + 1)) {
    ra = __ldg(rec + 2 * (size_t)q);
    rb = __ldg(rec + 2 * (size_t)q + 1);
  } else {
    ra = make_int4(0, 0, 0, 0);
    rb = make_int4(0, 0, 0, 0);
  }
}
// points of plane p beyond the first blockDim (rare): direct loads, no pipeline
template <typename R>
__device__ __forceinline__ void kb_plane_rest(const int* sp_off, const int4* rec, int p, const C2<R>* zp, int Nps,
                                              const C2<R>* Us, C2<R>* nlb) {
  const int q1 = __ldg(sp_off + p + 1);
  for (int q = __ldg(sp_off + p) + (int)threadIdx.x + (int)blockDim.x; q < q1; q += blockDim.x) {
    const int4 ra = __ldg(rec + 2 * (size_t)q), rb = __ldg(rec + 2 * (size_t)q + 1);
    C2<R> zv[4];
    kb_load_zproj<R>(ra, rb, zp, Nps, zv);
    nlb[ra.x] = kb_point<R>(ra, rb, zv, Us);
  }
}
// export of plane p's output values at its sphere points: S[q] = ob[pos]
template <typename R>
__device__ __forceinline__ void kb_export(const int* sp_off, const int4* rec, int p, const C2<R>* ob, C2<R>* Sb) {
  const int q1 = __ldg(sp_off + p + 1);
  for (int q = __ldg(sp_off + p) + (int)threadIdx.x; q < q1; q += blockDim.x) Sb[q] = ob[__ldg(rec + 2 * (size_t)q).x];
}

// Common part of one march step: ring wait + refill and the KB pipeline
// (records of plane x+2 are loaded, zproj of plane x+1 requested).
#define PASS_STEP_BEGIN()                                                                                    \
  const int j = x - x_beg;                                                                                   \
  cp_async_wait<NR - 6>(); /* this thread's copies of planes <= x+4 have landed */                           \
  __syncthreads();         /* ... and everyone's; plane x-1 is free; nlb of plane x complete */              \
  const T* pl = ring + (size_t)(j % NR) * NYZ;                                                               \
  {                                                                                                          \
    const int jn = j + NR - 1;                                                                               \
    if (act && jn < nplanes)                                                                                 \
      cp_run<R, RZ>(ring + (size_t)(jn % NR) * NYZ + own, inb + (size_t)wrapi(x_beg + jn, a.NLx) * NYZ + own); \
    cp_async_commit();                                                                                       \
  }                                                                                                          \
  const bool more = x + 1 < x_end;                                                                           \
  T zv[4];                                                                                                   \
  int4 ca, cb;                                                                                               \
  if (more) {                                                                                                \
    kb_load_zproj<R>(ra_n, rb_n, zp, a.Nps, zv);                                                             \
    ca = ra_n;                                                                                               \
    cb = rb_n;                                                                                               \
    if (x + 2 < x_end) kb_load_rec(a.sp_off, a.rec, x + 2, ra_n, rb_n);                                      \
  }                                                                                                          \
  const size_t pbase = (size_t)x * NYZ + own;

// End of a step: export the previous plane's sphere values, finish the KB term of plane x+1.
#define PASS_STEP_END()                                                                                        \
  if (do_export && x > x_beg) kb_export<R>(a.sp_off, a.rec, x - 1, ob + (size_t)((j - 1) & 1) * NYZ, Sb);       \
  if (more) {                                                                                                  \
    T* nln = nlb + (size_t)((j + 1) & 1) * NYZ;                                                                \
    if (ca.y > 0) nln[ca.x] = kb_point<R>(ca, cb, zv, Us);                                                     \
    kb_plane_rest<R>(a.sp_off, a.rec, x + 1, zp, a.Nps, Us, nln);                                              \
  }

// Epilogue of one point run: F = B E + A E - 0.5 v - zI w (stencil/F90/hpsi.f90:190),
// optional ttpsi, + nonlocal term, optional Taylor update, store.
template <typename R, int RZ, int MODE>
__device__ __forceinline__ void pass_store(const PassArgs<R>& a, int b, size_t pbase, R A, const R (&vl)[RZ],
                                           const C2<R> (&c)[RZ], const C2<R> (&v)[RZ], const C2<R> (&w)[RZ],
                                           const C2<R> (&nl)[RZ], C2<R>* obp) {
  using T = C2<R>;
  T res[RZ];
#pragma unroll
  for (int r = 0; r < RZ; ++r) {
    T f;
    f.x = fma(vl[r] + A, c[r].x, fma((R)-0.5, v[r].x, w[r].y));
    f.y = fma(vl[r] + A, c[r].y, fma((R)-0.5, v[r].y, -w[r].x));
    if constexpr (MODE == 1) {  // ttpsi = H tpsi - Vloc tpsi before pseudo_pt (hpsi.f90:131-133)
      a.tt[(size_t)b * a.NL + pbase + r] = mk<R>(fma(-vl[r], c[r].x, f.x), fma(-vl[r], c[r].y, f.y));
    }
    res[r] = cadd(f, nl[r]);  // + pseudo_pt scatter (hpsi.f90:203-206)
  }
  if constexpr (MODE == 2) {  // update (RT/hamiltonian.f90:114-117)
    T ps[RZ], p1[RZ], p2[RZ];
    ld_run_rw<R, RZ>(ps, a.zu + (size_t)b * a.NL + pbase);
    ld_run<R, RZ>(p1, a.t1 + (size_t)b * a.NL + pbase);
    ld_run<R, RZ>(p2, a.t2 + (size_t)b * a.NL + pbase);
#pragma unroll
    for (int r = 0; r < RZ; ++r) {
      T u = ps[r];
      u = cfma(a.zf[0], p1[r], u);
      u = cfma(a.zf[1], p2[r], u);
      u = cfma(a.zf[2], c[r], u);
      u = cfma(a.zf[3], res[r], u);
      res[r] = u;
    }
    st_run<R, RZ>(a.zu + (size_t)b * a.NL + pbase, res);
  } else {
    st_run<R, RZ>(a.out + (size_t)b * a.NL + pbase, res);
  }
  if (obp) st_run<R, RZ>(obp, res);  // for the export of the sphere values
}

// Shared prologue of both pass kernels (ring fill, U, nlb, offsets, first plane's scatter).
#define PASS_PROLOGUE()                                                                                        \
  extern __shared__ __align__(16) unsigned char smem_raw[];                                                    \
  const int NLy = a.NLy, NLz = a.NLz, NYZ = NLy * NLz;                                                         \
  T* ring = reinterpret_cast<T*>(smem_raw);                                                                    \
  T* nlb = ring + (size_t)NR * NYZ;                                                                            \
  T* ob = nlb + 2 * (size_t)NYZ;           /* output planes for the sphere export (if any) */                  \
  const bool do_export = a.S != nullptr;                                                                       \
  T* Us = ob + (do_export ? 2 * (size_t)NYZ : 0);                                                              \
  const int b = blockIdx.x;                                                                                    \
  const int o = a.o_beg + b;                                                                                   \
  const int kl = o / a.NBocc;                                                                                  \
  const double kxd = a.kAc[3 * kl], kyd = a.kAc[3 * kl + 1], kzd = a.kAc[3 * kl + 2];                          \
  const R A = (R)((kxd * kxd + kyd * kyd + kzd * kzd - a.lap0sum) * 0.5); /* k2lap0_2 (hpsi.f90:120-121) */    \
  const T* zp = a.zproj + (size_t)kl * a.Nlma * a.Nps;                                                         \
  const int NZG = NLz / RZ;                                                                                    \
  const int t = threadIdx.x;                                                                                   \
  const int bd = blockDim.x;                                                                                   \
  const bool act = t < NLy * NZG;                                                                              \
  const int y = act ? t / NZG : 0;                                                                             \
  const int z0 = act ? (t - y * NZG) * RZ : 0;                                                                 \
  const int own = y * NLz + z0;                                                                                \
  const int x_beg = blockIdx.y * a.SX;                                                                         \
  const int x_end = min(x_beg + a.SX, a.NLx);                                                                  \
  if (x_beg >= x_end) return; /* whole CTA leaves together */                                                  \
  const int nplanes = x_end - x_beg + 4; /* planes the ring delivers: x_beg .. x_end+3 */                       \
  const T* inb = a.in + (size_t)b * a.NL;                                                                      \
  _Pragma("unroll") for (int n = 0; n < NR - 1; ++n) {                                                         \
    if (act && n < nplanes)                                                                                    \
      cp_run<R, RZ>(ring + (size_t)n * NYZ + own, inb + (size_t)wrapi(x_beg + n, a.NLx) * NYZ + own);          \
    cp_async_commit();                                                                                         \
  }                                                                                                            \
  for (int i = t; i < a.Nlma; i += bd) {                                                                       \
    const double2 u = a.U[(size_t)b * a.Nlma + i];                                                             \
    Us[i] = mk<R>((R)u.x, (R)u.y);                                                                             \
  }                                                                                                            \
  for (int i = t; i < 2 * NYZ; i += bd) nlb[i] = mk<R>(0, 0);                                                  \
  int yo[8];                                                                                                   \
  _Pragma("unroll") for (int n = 1; n <= 4; ++n) {                                                             \
    yo[n - 1] = wrapi(y + n, NLy) * NLz + z0;                                                                  \
    yo[3 + n] = wrapi(y - n, NLy) * NLz + z0;                                                                  \
  }                                                                                                            \
  constexpr int NZZ = RZ + 8; /* z runs start at z0-4, z0-4+RZ, ..., z0+4 */                                   \
  int zoff[NZZ / RZ];                                                                                          \
  _Pragma("unroll") for (int m = 0; m < NZZ / RZ; ++m) zoff[m] = y * NLz + wrapi(z0 + m * RZ - 4, NLz);        \
  T q[9][RZ];                                                                                                  \
  if (act) {                                                                                                   \
    _Pragma("unroll") for (int n = 0; n < 4; ++n)                                                              \
        ld_run<R, RZ>(q[n], inb + (size_t)wrapi(x_beg - 4 + n, a.NLx) * NYZ + own);                            \
  }                                                                                                            \
  R vl[RZ];                                                                                                    \
  if (act) {                                                                                                   \
    _Pragma("unroll") for (int r = 0; r < RZ; ++r) vl[r] = __ldg(a.vloc + (size_t)x_beg * NYZ + own + r);      \
  }                                                                                                            \
  T* Sb = do_export ? a.S + (size_t)b * a.nsp : nullptr;                                                       \
  int4 ra_n, rb_n;                                                                                             \
  __syncthreads(); /* Us and the zeroed nlb are visible */                                                     \
  {                                                                                                            \
    int4 r0a, r0b;                                                                                             \
    kb_load_rec(a.sp_off, a.rec, x_beg, r0a, r0b);                                                             \
    T zv0[4];                                                                                                  \
    kb_load_zproj<R>(r0a, r0b, zp, a.Nps, zv0);                                                                \
    if (r0a.y > 0) nlb[r0a.x] = kb_point<R>(r0a, r0b, zv0, Us);                                                \
    kb_plane_rest<R>(a.sp_off, a.rec, x_beg, zp, a.Nps, Us, nlb);                                              \
    if (x_beg + 1 < x_end) kb_load_rec(a.sp_off, a.rec, x_beg + 1, ra_n, rb_n);                                \
  }

// Nonlocal value of this thread's points of plane x; the slot is zeroed for plane x+2.
template <typename R, int RZ>
__device__ __forceinline__ void take_nl(C2<R>* nlc, C2<R> (&nl)[RZ]) {
  lds_run<R, RZ>(nl, nlc);
  C2<R> zr[RZ];
#pragma unroll
  for (int r = 0; r < RZ; ++r) zr[r] = mk<R>(0, 0);
  st_run<R, RZ>(nlc, zr);
}

// ------------------------------------------------ scalar pass (any grid) ---
// FP64, or FP32 on non-cubic grids: scalar FMAs whose coefficients come from
// the kernel parameters (constant bank); the x queue shifts by register moves.
template <typename R, int RZ, int MODE>
__global__ void __launch_bounds__(512) k_hpsi_pass(const PassArgs<R> a) {
  using T = C2<R>;
  constexpr int NR = PassGeom<R>::NR;
  PASS_PROLOGUE()
  const R kx = (R)kxd, ky = (R)kyd, kz = (R)kzd;

  for (int x = x_beg; x < x_end; ++x) {
    PASS_STEP_BEGIN()
    if (act) {
      if (j == 0) {
#pragma unroll
        for (int n = 4; n < 8; ++n) lds_run<R, RZ>(q[n], ring + (size_t)(n - 4) * NYZ + own);
      }
      lds_run<R, RZ>(q[8], ring + (size_t)((j + 4) % NR) * NYZ + own);
      R vln[RZ];
      if (more) {
#pragma unroll
        for (int r = 0; r < RZ; ++r) vln[r] = __ldg(a.vloc + pbase + NYZ + r);
      }
      T v[RZ], w[RZ], wa[RZ];
#pragma unroll
      for (int r = 0; r < RZ; ++r) { v[r] = mk<R>(0, 0); wa[r] = mk<R>(0, 0); }
#pragma unroll
      for (int m = 0; m < NZZ / RZ; ++m) {  // z: each value feeds every point it neighbours
        T run[RZ];
        if (m * RZ == 4) {
#pragma unroll
          for (int s2 = 0; s2 < RZ; ++s2) run[s2] = q[4][s2];
        } else {
          lds_run<R, RZ>(run, pl + zoff[m]);
        }
#pragma unroll
        for (int s2 = 0; s2 < RZ; ++s2)
#pragma unroll
          for (int r = 0; r < RZ; ++r) {
            const int k = m * RZ + s2 - 4 - r;
            if (k != 0 && k >= -4 && k <= 4) {
              const int n = k > 0 ? k : -k;
              const R cl = a.lap2[7 + n].x;
              const R cn = k > 0 ? a.nab2[7 + n].x : -a.nab2[7 + n].x;
              v[r].x = fma(cl, run[s2].x, v[r].x);
              v[r].y = fma(cl, run[s2].y, v[r].y);
              wa[r].x = fma(cn, run[s2].x, wa[r].x);
              wa[r].y = fma(cn, run[s2].y, wa[r].y);
            }
          }
      }
#pragma unroll
      for (int r = 0; r < RZ; ++r) { w[r] = mk<R>(kz * wa[r].x, kz * wa[r].y); wa[r] = mk<R>(0, 0); }
#pragma unroll
      for (int n = 1; n <= 4; ++n) {  // y
        T rp[RZ], rm[RZ];
        lds_run<R, RZ>(rp, pl + yo[n - 1]);
        lds_run<R, RZ>(rm, pl + yo[3 + n]);
#pragma unroll
        for (int r = 0; r < RZ; ++r) {
          v[r].x = fma(a.lap2[3 + n].x, rp[r].x + rm[r].x, v[r].x);
          v[r].y = fma(a.lap2[3 + n].x, rp[r].y + rm[r].y, v[r].y);
          wa[r].x = fma(a.nab2[3 + n].x, rp[r].x - rm[r].x, wa[r].x);
          wa[r].y = fma(a.nab2[3 + n].x, rp[r].y - rm[r].y, wa[r].y);
        }
      }
#pragma unroll
      for (int r = 0; r < RZ; ++r) { w[r].x = fma(ky, wa[r].x, w[r].x); w[r].y = fma(ky, wa[r].y, w[r].y); wa[r] = mk<R>(0, 0); }
#pragma unroll
      for (int n = 1; n <= 4; ++n)  // x: the register queue
#pragma unroll
        for (int r = 0; r < RZ; ++r) {
          const T p = q[4 + n][r], mm = q[4 - n][r];
          v[r].x = fma(a.lap2[n - 1].x, p.x + mm.x, v[r].x);
          v[r].y = fma(a.lap2[n - 1].x, p.y + mm.y, v[r].y);
          wa[r].x = fma(a.nab2[n - 1].x, p.x - mm.x, wa[r].x);
          wa[r].y = fma(a.nab2[n - 1].x, p.y - mm.y, wa[r].y);
        }
#pragma unroll
      for (int r = 0; r < RZ; ++r) { w[r].x = fma(kx, wa[r].x, w[r].x); w[r].y = fma(kx, wa[r].y, w[r].y); }
      T nl[RZ];
      take_nl<R, RZ>(nlb + (size_t)(j & 1) * NYZ + own, nl);
      pass_store<R, RZ, MODE>(a, b, pbase, A, vl, q[4], v, w, nl, do_export ? ob + (size_t)(j & 1) * NYZ + own : nullptr);
      if (more) {
#pragma unroll
        for (int r = 0; r < RZ; ++r) vl[r] = vln[r];
      }
#pragma unroll
      for (int n = 0; n < 8; ++n)
#pragma unroll
        for (int r = 0; r < RZ; ++r) q[n][r] = q[n + 1][r];
    }
    PASS_STEP_END()
  }
  cp_async_wait<0>();
  if (do_export) {
    __syncthreads();
    kb_export<R>(a.sp_off, a.rec, x_end - 1, ob + (size_t)((x_end - 1 - x_beg) & 1) * NYZ, Sb);
  }
}

// --------------------------------------- packed FP32x2 pass (cubic grids) ---
// complex(4) orbitals on a grid with lapx=lapy=lapz and nabx=naby=nabz (cubic
// cell, equal spacing): per shift n the six neighbours are summed first, so
// v += lap_n (sum of the 3 axes' psi(+n)+psi(-n)) and
// w += nab_n (kx dx + ky dy + kz dz) with d = psi(+n)-psi(-n); every operation is
// a packed FP32x2 instruction on (re, im).  RZ = 2; the x queue rotates by
// unrolling the march 9 times.
template <int MODE>
__global__ void __launch_bounds__(512) k_hpsi_pass_f2(const PassArgs<float> a) {
  using R = float;
  using T = float2;
  constexpr int RZ = 2;
  constexpr int NR = PassGeom<R>::NR;
  PASS_PROLOGUE()
  const T kx2 = splat<R>((R)kxd), ky2 = splat<R>((R)kyd), kz2 = splat<R>((R)kzd);
  const T m1 = splat<R>(-1.0f);

  auto step = [&](auto S_, const int x) {
    constexpr int S = decltype(S_)::value;
    PASS_STEP_BEGIN()
    if (act) {
      if constexpr (S == 0) {
        if (j == 0) {
#pragma unroll
          for (int n = 4; n < 8; ++n) lds_run<R, RZ>(q[n], ring + (size_t)(n - 4) * NYZ + own);
        }
      }
      lds_run<R, RZ>(q[(S + 8) % 9], ring + (size_t)((j + 4) % NR) * NYZ + own);
      R vln[RZ];
      if (more) {
#pragma unroll
        for (int r = 0; r < RZ; ++r) vln[r] = __ldg(a.vloc + pbase + NYZ + r);
      }
      // z runs: zz[4+k] is the value at z0+k, k in [-4, 5]
      T zz[NZZ];
#pragma unroll
      for (int m = 0; m < NZZ / RZ; ++m) {
        if (m == 2) {
          zz[4] = q[(S + 4) % 9][0];
          zz[5] = q[(S + 4) % 9][1];
        } else {
          T run[RZ];
          lds_run<R, RZ>(run, pl + zoff[m]);
          zz[2 * m] = run[0];
          zz[2 * m + 1] = run[1];
        }
      }
      T v[RZ], w[RZ];
#pragma unroll
      for (int r = 0; r < RZ; ++r) { v[r] = mk<R>(0, 0); w[r] = mk<R>(0, 0); }
#pragma unroll
      for (int n = 1; n <= 4; ++n) {
        T rp[RZ], rm[RZ];
        lds_run<R, RZ>(rp, pl + yo[n - 1]);
        lds_run<R, RZ>(rm, pl + yo[3 + n]);
#pragma unroll
        for (int r = 0; r < RZ; ++r) {
          const T zp_ = zz[4 + r + n], zm_ = zz[4 + r - n];
          const T xp_ = q[(S + 4 + n) % 9][r], xm_ = q[(S + 4 - n) % 9][r];
          T sum = __fadd2_rn(zp_, zm_);
          sum = __fadd2_rn(sum, rp[r]);
          sum = __fadd2_rn(sum, rm[r]);
          sum = __fadd2_rn(sum, xp_);
          sum = __fadd2_rn(sum, xm_);
          v[r] = __ffma2_rn(a.lap2[n - 1], sum, v[r]);
          T d = __fmul2_rn(kz2, __ffma2_rn(m1, zm_, zp_));
          d = __ffma2_rn(ky2, __ffma2_rn(m1, rm[r], rp[r]), d);
          d = __ffma2_rn(kx2, __ffma2_rn(m1, xm_, xp_), d);
          w[r] = __ffma2_rn(a.nab2[n - 1], d, w[r]);
        }
      }
      T nl[RZ];
      take_nl<R, RZ>(nlb + (size_t)(j & 1) * NYZ + own, nl);
      T c[RZ];
#pragma unroll
      for (int r = 0; r < RZ; ++r) c[r] = q[(S + 4) % 9][r];
      pass_store<R, RZ, MODE>(a, b, pbase, A, vl, c, v, w, nl, do_export ? ob + (size_t)(j & 1) * NYZ + own : nullptr);
      if (more) {
#pragma unroll
        for (int r = 0; r < RZ; ++r) vl[r] = vln[r];
      }
    }
    PASS_STEP_END()
  };

#ifdef SGPU_PASS_ROTATE9
  for (int x0 = x_beg; x0 < x_end; x0 += 9) {
    step(std::integral_constant<int, 0>{}, x0);
    if (x0 + 1 < x_end) step(std::integral_constant<int, 1>{}, x0 + 1);
    if (x0 + 2 < x_end) step(std::integral_constant<int, 2>{}, x0 + 2);
    if (x0 + 3 < x_end) step(std::integral_constant<int, 3>{}, x0 + 3);
    if (x0 + 4 < x_end) step(std::integral_constant<int, 4>{}, x0 + 4);
    if (x0 + 5 < x_end) step(std::integral_constant<int, 5>{}, x0 + 5);
    if (x0 + 6 < x_end) step(std::integral_constant<int, 6>{}, x0 + 6);
    if (x0 + 7 < x_end) step(std::integral_constant<int, 7>{}, x0 + 7);
    if (x0 + 8 < x_end) step(std::integral_constant<int, 8>{}, x0 + 8);
  }
#else
  for (int x = x_beg; x < x_end; ++x) {
    step(std::integral_constant<int, 0>{}, x);
#pragma unroll
    for (int n = 0; n < 8; ++n)
#pragma unroll
      for (int r = 0; r < RZ; ++r) q[n][r] = q[n + 1][r];
  }
#endif
  cp_async_wait<0>();
  if (do_export) {
    __syncthreads();
    kb_export<R>(a.sp_off, a.rec, x_end - 1, ob + (size_t)((x_end - 1 - x_beg) & 1) * NYZ, Sb);
  }
}

// ------------------------------------------------------------- launch ---
template <typename R, int RZ, int MODE>
static cudaError_t launch_pass_t(const System& s, const PassIO& io, int o_beg, int nb, int nbk) {
  PassArgs<R> a;
  a.in = (const C2<R>*)io.in;
  a.out = (C2<R>*)io.out;
  a.tt = (C2<R>*)io.tt;
  a.t1 = (const C2<R>*)io.t1;
  a.t2 = (const C2<R>*)io.t2;
  a.zu = (C2<R>*)io.zu;
  a.vloc = std::is_same<R, float>::value ? (const R*)s.vloc32 : (const R*)s.vloc64;
  a.kAc = s.kAc_d;
  a.o_beg = o_beg;
  a.NBocc = nbk;
  a.NLx = s.NLx; a.NLy = s.NLy; a.NLz = s.NLz; a.NL = s.NL;
  const int nslab = s.nslab < 1 ? 1 : (s.nslab > s.NLx ? s.NLx : s.nslab);
  a.SX = (s.NLx + nslab - 1) / nslab;
  a.lap0sum = s.lap[0][0] + s.lap[1][0] + s.lap[2][0];
  for (int n = 0; n < 4; ++n)
    for (int d = 0; d < 3; ++d) {
      a.lap2[4 * d + n] = mk<R>((R)s.lap[d][n + 1], (R)s.lap[d][n + 1]);
      a.nab2[4 * d + n] = mk<R>((R)s.nab[d][n + 1], (R)s.nab[d][n + 1]);
    }
  a.sp_off = s.sp_off;
  a.rec = s.rec;
  a.S = (C2<R>*)io.S;
  a.nsp = s.nsp;
  a.zproj = std::is_same<R, float>::value ? (const C2<R>*)s.zproj32 : (const C2<R>*)s.zproj64;
  a.U = s.U;
  a.Nlma = s.Nlma;
  a.Nps = s.Nps;
  for (int n = 0; n < 4; ++n) a.zf[n] = mk<R>((R)io.zfac[n][0], (R)io.zfac[n][1]);
  const int nthr = s.NLy * (s.NLz / RZ);
  const int block = ((nthr + 31) / 32) * 32;
  const size_t smem = sizeof(C2<R>) * ((size_t)(PassGeom<R>::NR + 2 + (io.S ? 2 : 0)) * s.NLy * s.NLz + (s.Nlma > 0 ? s.Nlma : 1));
  auto kern = k_hpsi_pass<R, RZ, MODE>;
  if constexpr (std::is_same<R, float>::value && RZ == 2) {
    if (s.cubic) kern = (decltype(kern))k_hpsi_pass_f2<MODE>;
  }
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  dim3 grid(nb, (s.NLx + a.SX - 1) / a.SX);
  kern<<<grid, block, smem, s.stream>>>(a);
  return cudaGetLastError();
}

template <typename R, int RZ>
static cudaError_t launch_pass_rz(const System& s, int mode, const PassIO& io, int o_beg, int nb, int nbk) {
  switch (mode) {
    case 0: return launch_pass_t<R, RZ, 0>(s, io, o_beg, nb, nbk);
    case 1: return launch_pass_t<R, RZ, 1>(s, io, o_beg, nb, nbk);
    default: return launch_pass_t<R, RZ, 2>(s, io, o_beg, nb, nbk);
  }
}

cudaError_t launch_hpsi_pass(const System& s, int mode, const PassIO& io, int o_beg, int nb, int nbk, int prec) {
  if (nb == 0) return cudaSuccess;
  const bool rz2 = (s.NLz % 2) == 0;
  if ((prec < 0 ? s.prec : prec) == SGPU_PREC_C64)
    return rz2 ? launch_pass_rz<float, 2>(s, mode, io, o_beg, nb, nbk)
               : launch_pass_rz<float, 1>(s, mode, io, o_beg, nb, nbk);
  return rz2 ? launch_pass_rz<double, 2>(s, mode, io, o_beg, nb, nbk)
             : launch_pass_rz<double, 1>(s, mode, io, o_beg, nb, nbk);
}

int pass_block_threads(int NLy, int NLz) {
  const int rz = (NLz % 2) == 0 ? 2 : 1;
  return ((NLy * (NLz / rz) + 31) / 32) * 32;
}

}  // namespace sgpu
