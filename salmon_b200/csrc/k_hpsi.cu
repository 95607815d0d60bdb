// Hamiltonian application and Taylor-step kernels for sm_100a.
//
// H psi = (k2lap0_2 + Vloc) psi - 1/2 sum lapt (psi(+n)+psi(-n)) - i sum nabt (psi(+n)-psi(-n))
//         + sum_ilma zproj(:,ilma) U(ilma)
// restates hpsi_omp_KB_base (common/hpsi.f90:98-208): the stencil of
// stencil/F90/hpsi.f90:190 and the Kleinman-Bylander term of pseudo_pt (:163-207).
//
// Stencil pass layout: one CTA per (orbital, x-slab).  The CTA owns whole y-z
// planes (z unit-stride, so one plane of one orbital is a contiguous
// NLy*NLz run in HBM).  Each thread owns RZ consecutive z points of one y row
// and marches along x keeping its own 9 x-neighbours in a register queue; the
// current plane is staged in shared memory for the y and z neighbours.  Every
// element of the input is read from HBM once per pass (plus the 8 halo planes
// of the slab, served from L2), every output element written once.
#include <cuda_runtime.h>

#include <type_traits>

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
  R lapt[12];            // lapx(1:4), lapy(1:4), lapz(1:4)
  R nabc[12];            // nabx(1:4), naby(1:4), nabz(1:4)
  const int* inv_off;
  const int2* inv_ent;
  const C2<R>* zproj;    // [nkl][Nlma][Nps]
  const double2* U;      // [nb][Nlma]
  int Nlma, Nps;
  C2<R> zf[4];
};

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

// MODE 0: out = H in.   MODE 1: also tt = H in - V in before the nonlocal term.
// MODE 2: zu = zu + zf0 t1 + zf1 t2 + zf2 in + zf3 H in   (RT/hamiltonian.f90:99-122).
template <typename R, int RZ, int MODE>
__global__ void __launch_bounds__(512) k_hpsi_pass(const PassArgs<R> a) {
  using T = C2<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* plane = reinterpret_cast<T*>(smem_raw);
  T* Us = plane + a.NLy * a.NLz;

  const int b = blockIdx.x;
  const int o = a.o_beg + b;
  const int kl = o / a.NBocc;
  const double kxd = a.kAc[3 * kl], kyd = a.kAc[3 * kl + 1], kzd = a.kAc[3 * kl + 2];
  const R A = (R)((kxd * kxd + kyd * kyd + kzd * kzd - a.lap0sum) * 0.5);  // k2lap0_2 (hpsi.f90:120-121)
  // nabt = k_d nab_d (hpsi.f90:122-124) is applied once per axis: w = sum_d k_d sum_n nab_d,n (psi(+n)-psi(-n))
  const R kx = (R)kxd, ky = (R)kyd, kz = (R)kzd;
  for (int i = threadIdx.x; i < a.Nlma; i += blockDim.x) {
    const double2 u = a.U[(size_t)b * a.Nlma + i];
    Us[i] = mk<R>((R)u.x, (R)u.y);
  }

  const int NLy = a.NLy, NLz = a.NLz, NYZ = NLy * NLz;
  const int NZG = NLz / RZ;
  const int t = threadIdx.x;
  const bool act = t < NLy * NZG;
  const int y = act ? t / NZG : 0;
  const int z0 = act ? (t - y * NZG) * RZ : 0;
  const int own = y * NLz + z0;

  // neighbour offsets inside a plane (periodic)
  int yo[8];
#pragma unroll
  for (int n = 1; n <= 4; ++n) {
    yo[n - 1] = wrapi(y + n, NLy) * NLz + z0;
    yo[3 + n] = wrapi(y - n, NLy) * NLz + z0;
  }
  // z neighbours: runs of RZ values starting at z0-4, z0-4+RZ, ..., z0+4
  constexpr int NZZ = RZ + 8;
  int zoff[NZZ];
#pragma unroll
  for (int k = 0; k < NZZ; ++k) zoff[k] = y * NLz + wrapi(z0 + k - 4, NLz);

  const int x_beg = blockIdx.y * a.SX;
  const int x_end = min(x_beg + a.SX, a.NLx);
  if (x_beg >= x_end) return;  // whole CTA leaves together

  const T* inb = a.in + (size_t)b * a.NL;
  T q[9][RZ];
  if (act) {
#pragma unroll
    for (int n = 0; n < 9; ++n) ld_run<R, RZ>(q[n], inb + (size_t)wrapi(x_beg - 4 + n, a.NLx) * NYZ + own);
  }

  for (int x = x_beg; x < x_end; ++x) {
    T nxt[RZ];
    R vl[RZ];
    T ps[RZ], p1[RZ], p2[RZ];
    int e0[RZ], e1[RZ];
    const size_t pbase = (size_t)x * NYZ + own;
    if (act) {
      if (x + 1 < x_end) ld_run<R, RZ>(nxt, inb + (size_t)wrapi(x + 5, a.NLx) * NYZ + own);
#pragma unroll
      for (int r = 0; r < RZ; ++r) {
        vl[r] = __ldg(a.vloc + pbase + r);
        e0[r] = __ldg(a.inv_off + pbase + r);
        e1[r] = __ldg(a.inv_off + pbase + r + 1);
      }
    }
    __syncthreads();  // readers of the previous plane are done
    if (act) st_run<R, RZ>(plane + own, q[4]);
    __syncthreads();
    if (act) {
      // v = sum lapt (psi(+n) + psi(-n)),  w = sum nabt (psi(+n) - psi(-n)): every
      // neighbour value is folded in as soon as it is loaded (4 FMA per value).
      T v[RZ], w[RZ];
#pragma unroll
      for (int r = 0; r < RZ; ++r) {
        v[r] = mk<R>(0, 0);
        w[r] = mk<R>(0, 0);
      }
      // z (unit stride): the runs at z0-4 .. z0+RZ+3 of this row
      {
        T wa[RZ];
#pragma unroll
        for (int r = 0; r < RZ; ++r) wa[r] = mk<R>(0, 0);
#pragma unroll
        for (int m = 0; m < NZZ / RZ; ++m) {
          T run[RZ];
          if (m * RZ == 4) {
#pragma unroll
            for (int s2 = 0; s2 < RZ; ++s2) run[s2] = q[4][s2];
          } else {
            lds_run<R, RZ>(run, plane + zoff[m * RZ]);
          }
#pragma unroll
          for (int s2 = 0; s2 < RZ; ++s2)
#pragma unroll
            for (int r = 0; r < RZ; ++r) {
              const int k = m * RZ + s2 - 4 - r;  // offset of this value from point z0+r
              if (k != 0 && k >= -4 && k <= 4) {
                const int n = k > 0 ? k : -k;
                const R cl = a.lapt[7 + n];
                const R cn = k > 0 ? a.nabc[7 + n] : -a.nabc[7 + n];
                v[r].x = fma(cl, run[s2].x, v[r].x);
                v[r].y = fma(cl, run[s2].y, v[r].y);
                wa[r].x = fma(cn, run[s2].x, wa[r].x);
                wa[r].y = fma(cn, run[s2].y, wa[r].y);
              }
            }
        }
#pragma unroll
        for (int r = 0; r < RZ; ++r) {
          w[r].x = kz * wa[r].x;
          w[r].y = kz * wa[r].y;
        }
      }
      // y (stride NLz): rows y+n and y-n
      {
        T wa[RZ];
#pragma unroll
        for (int r = 0; r < RZ; ++r) wa[r] = mk<R>(0, 0);
#pragma unroll
        for (int n = 1; n <= 4; ++n) {
          T rp[RZ], rm[RZ];
          lds_run<R, RZ>(rp, plane + yo[n - 1]);
          lds_run<R, RZ>(rm, plane + yo[3 + n]);
#pragma unroll
          for (int r = 0; r < RZ; ++r) {
            v[r].x = fma(a.lapt[3 + n], rp[r].x + rm[r].x, v[r].x);
            v[r].y = fma(a.lapt[3 + n], rp[r].y + rm[r].y, v[r].y);
            wa[r].x = fma(a.nabc[3 + n], rp[r].x - rm[r].x, wa[r].x);
            wa[r].y = fma(a.nabc[3 + n], rp[r].y - rm[r].y, wa[r].y);
          }
        }
#pragma unroll
        for (int r = 0; r < RZ; ++r) {
          w[r].x = fma(ky, wa[r].x, w[r].x);
          w[r].y = fma(ky, wa[r].y, w[r].y);
        }
      }
      // x (stride NLy*NLz): the register queue
      {
        T wa[RZ];
#pragma unroll
        for (int r = 0; r < RZ; ++r) wa[r] = mk<R>(0, 0);
#pragma unroll
        for (int n = 1; n <= 4; ++n)
#pragma unroll
          for (int r = 0; r < RZ; ++r) {
            const T p = q[4 + n][r], mm = q[4 - n][r];
            v[r].x = fma(a.lapt[n - 1], p.x + mm.x, v[r].x);
            v[r].y = fma(a.lapt[n - 1], p.y + mm.y, v[r].y);
            wa[r].x = fma(a.nabc[n - 1], p.x - mm.x, wa[r].x);
            wa[r].y = fma(a.nabc[n - 1], p.y - mm.y, wa[r].y);
          }
#pragma unroll
        for (int r = 0; r < RZ; ++r) {
          w[r].x = fma(kx, wa[r].x, w[r].x);
          w[r].y = fma(kx, wa[r].y, w[r].y);
        }
      }
      if constexpr (MODE == 2) {  // operands of the update, loaded late to keep registers free
        ld_run_rw<R, RZ>(ps, a.zu + (size_t)b * a.NL + pbase);
        ld_run<R, RZ>(p1, a.t1 + (size_t)b * a.NL + pbase);
        ld_run<R, RZ>(p2, a.t2 + (size_t)b * a.NL + pbase);
      }

      T res[RZ];
#pragma unroll
      for (int r = 0; r < RZ; ++r) {
        const T c = q[4][r];
        // F = B E + A E - 0.5 v - zI w   (stencil/F90/hpsi.f90:190)
        T f;
        f.x = fma(vl[r], c.x, A * c.x) - (R)0.5 * v[r].x + w[r].y;
        f.y = fma(vl[r], c.y, A * c.y) - (R)0.5 * v[r].y - w[r].x;
        if constexpr (MODE == 1) {  // ttpsi = H tpsi - Vloc tpsi before pseudo_pt (hpsi.f90:131-133)
          T g;
          g.x = f.x - vl[r] * c.x;
          g.y = f.y - vl[r] * c.y;
          a.tt[(size_t)b * a.NL + pbase + r] = g;
        }
        // Kleinman-Bylander scatter: dpseudo = sum_ilma zproj(j,ilma) U(ilma)
        if (e1[r] > e0[r]) {
          T dp = mk<R>(0, 0);
          const T* zp = a.zproj + (size_t)kl * a.Nlma * a.Nps;
          for (int e = e0[r]; e < e1[r]; ++e) {
            const int2 en = __ldg(a.inv_ent + e);
            dp = cfma(__ldg(zp + en.x), Us[en.y], dp);
          }
          f = cadd(f, dp);
        }
        if constexpr (MODE == 2) {  // update (RT/hamiltonian.f90:114-117)
          T u = ps[r];
          u = cfma(a.zf[0], p1[r], u);
          u = cfma(a.zf[1], p2[r], u);
          u = cfma(a.zf[2], c, u);
          u = cfma(a.zf[3], f, u);
          res[r] = u;
        } else {
          res[r] = f;
        }
      }
      if constexpr (MODE == 2)
        st_run<R, RZ>(a.zu + (size_t)b * a.NL + pbase, res);
      else
        st_run<R, RZ>(a.out + (size_t)b * a.NL + pbase, res);

      if (x + 1 < x_end) {
#pragma unroll
        for (int n = 0; n < 8; ++n)
#pragma unroll
          for (int r = 0; r < RZ; ++r) q[n][r] = q[n + 1][r];
#pragma unroll
        for (int r = 0; r < RZ; ++r) q[8][r] = nxt[r];
      }
    }
  }
}

// ----------------------------------------------------------------- uVpsi ---
// U[b][ilma] = Hxyz (iuV) sum_j conj(zproj(j,ilma,k)) in_b(J(j))  (hpsi.f90:188-193)
// The projectors are read in FP64 for either orbital precision.
// One CTA per block of UB orbitals; each warp takes (atom, <=4 projectors)
// items, lanes stride over the atom's sphere points, FP64 accumulation,
// warp-shuffle reduction (deterministic order).
constexpr int UB = 4;

template <typename R>
__global__ void __launch_bounds__(256) k_uvpsi(const C2<R>* __restrict__ in, int nb, int NL, int o_beg, int NBocc,
                                              const double2* __restrict__ zproj, int Nlma, int Nps,
                                              const int* __restrict__ idx_proj, const int* __restrict__ atom_off,
                                              const int4* __restrict__ items, int nitems,
                                              const int* __restrict__ lma_list, const int* __restrict__ iuV,
                                              double scale, int use_iuv, double2* __restrict__ U) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int b0 = blockIdx.x * UB;
  int kl[UB];
  bool valid[UB];
#pragma unroll
  for (int u = 0; u < UB; ++u) {
    valid[u] = (b0 + u) < nb;
    kl[u] = valid[u] ? (o_beg + b0 + u) / NBocc : 0;
  }
  for (int it = warp; it < nitems; it += nw) {
    const int4 item = items[it];
    const int a = item.x, l0 = item.y, np = item.z;
    const int p0 = atom_off[a], mps = atom_off[a + 1] - p0;
    double2 acc[4][UB];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int u = 0; u < UB; ++u) acc[p][u] = make_double2(0, 0);
    int ilma[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) ilma[p] = p < np ? lma_list[l0 + p] : 0;
    for (int j = lane; j < mps; j += 32) {
      const int gi = idx_proj[p0 + j];
      double2 v[UB];
#pragma unroll
      for (int u = 0; u < UB; ++u) v[u] = valid[u] ? to_d2(in[(size_t)(b0 + u) * NL + gi]) : make_double2(0, 0);
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        if (p < np) {
#pragma unroll
          for (int u = 0; u < UB; ++u) {
            const double2 z = __ldg(zproj + ((size_t)kl[u] * Nlma + ilma[p]) * Nps + j);
            acc[p][u] = cfmaj(z, v[u], acc[p][u]);
          }
        }
      }
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int u = 0; u < UB; ++u) {
        double2 s = acc[p][u];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          s.x += __shfl_xor_sync(0xffffffffu, s.x, off);
          s.y += __shfl_xor_sync(0xffffffffu, s.y, off);
        }
        acc[p][u] = s;
      }
    if (lane == 0) {
#pragma unroll
      for (int p = 0; p < 4; ++p)
        if (p < np) {
          const double f = scale * (use_iuv ? (double)iuV[ilma[p]] : 1.0);
#pragma unroll
          for (int u = 0; u < UB; ++u)
            if (valid[u]) U[(size_t)(b0 + u) * Nlma + ilma[p]] = make_double2(acc[p][u].x * f, acc[p][u].y * f);
        }
    }
  }
}

cudaError_t launch_uvpsi(const System& s, const void* in, int o_beg, int nb, bool scale_iuv) {
  if (s.Nlma == 0 || nb == 0) return cudaSuccess;
  const int grid = (nb + UB - 1) / UB;
  if (s.prec == SGPU_PREC_C64)
    k_uvpsi<float><<<grid, 256, 0, s.stream>>>((const float2*)in, nb, s.NL, o_beg, s.NBocc, s.zproj64, s.Nlma, s.Nps,
                                               s.idx_proj, s.atom_off, s.items, s.nitems, s.lma_list, s.iuV_d, s.Hxyz,
                                               scale_iuv ? 1 : 0, s.U);
  else
    k_uvpsi<double><<<grid, 256, 0, s.stream>>>((const double2*)in, nb, s.NL, o_beg, s.NBocc, s.zproj64, s.Nlma,
                                                s.Nps, s.idx_proj, s.atom_off, s.items, s.nitems, s.lma_list, s.iuV_d,
                                                s.Hxyz, scale_iuv ? 1 : 0, s.U);
  return cudaGetLastError();
}

template <typename R, int RZ, int MODE>
static cudaError_t launch_pass_t(const System& s, const PassIO& io, int o_beg, int nb) {
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
  a.NBocc = s.NBocc;
  a.NLx = s.NLx; a.NLy = s.NLy; a.NLz = s.NLz; a.NL = s.NL;
  const int nslab = s.nslab < 1 ? 1 : (s.nslab > s.NLx ? s.NLx : s.nslab);
  a.SX = (s.NLx + nslab - 1) / nslab;
  a.lap0sum = s.lap[0][0] + s.lap[1][0] + s.lap[2][0];
  for (int n = 0; n < 4; ++n)
    for (int d = 0; d < 3; ++d) {
      a.lapt[4 * d + n] = (R)s.lap[d][n + 1];
      a.nabc[4 * d + n] = (R)s.nab[d][n + 1];
    }
  a.inv_off = s.inv_off;
  a.inv_ent = s.inv_ent;
  a.zproj = std::is_same<R, float>::value ? (const C2<R>*)s.zproj32 : (const C2<R>*)s.zproj64;
  a.U = s.U;
  a.Nlma = s.Nlma;
  a.Nps = s.Nps;
  for (int n = 0; n < 4; ++n) a.zf[n] = mk<R>((R)io.zfac[n][0], (R)io.zfac[n][1]);
  const int nthr = s.NLy * (s.NLz / RZ);
  const int block = ((nthr + 31) / 32) * 32;
  const size_t smem = sizeof(C2<R>) * ((size_t)s.NLy * s.NLz + (s.Nlma > 0 ? s.Nlma : 1));
  auto kern = k_hpsi_pass<R, RZ, MODE>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  dim3 grid(nb, (s.NLx + a.SX - 1) / a.SX);
  kern<<<grid, block, smem, s.stream>>>(a);
  return cudaGetLastError();
}

template <typename R, int RZ>
static cudaError_t launch_pass_rz(const System& s, int mode, const PassIO& io, int o_beg, int nb) {
  switch (mode) {
    case 0: return launch_pass_t<R, RZ, 0>(s, io, o_beg, nb);
    case 1: return launch_pass_t<R, RZ, 1>(s, io, o_beg, nb);
    default: return launch_pass_t<R, RZ, 2>(s, io, o_beg, nb);
  }
}

cudaError_t launch_hpsi_pass(const System& s, int mode, const PassIO& io, int o_beg, int nb) {
  if (nb == 0) return cudaSuccess;
  const bool rz2 = (s.NLz % 2) == 0;
  if (s.prec == SGPU_PREC_C64)
    return rz2 ? launch_pass_rz<float, 2>(s, mode, io, o_beg, nb) : launch_pass_rz<float, 1>(s, mode, io, o_beg, nb);
  return rz2 ? launch_pass_rz<double, 2>(s, mode, io, o_beg, nb) : launch_pass_rz<double, 1>(s, mode, io, o_beg, nb);
}

// ------------------------------------------------------ update_projector ---
// ekr = exp(i kAc.r) in FP64, zproj = conj(ekr) uV   (common/projector.f90:55-75)
__global__ void k_update_projector(const double* __restrict__ kAc, const double* __restrict__ rpos,
                                   const int* __restrict__ atom_off, const int* __restrict__ lma_atom,
                                   const double* __restrict__ uV, int Nlma, int Nps, double2* __restrict__ z64,
                                   float2* __restrict__ z32) {
  const int kl = blockIdx.y, ilma = blockIdx.x;
  const int a = lma_atom[ilma];
  const int p0 = atom_off[a], mps = atom_off[a + 1] - p0;
  const double kx = kAc[3 * kl], ky = kAc[3 * kl + 1], kz = kAc[3 * kl + 2];
  for (int j = threadIdx.x; j < Nps; j += blockDim.x) {
    double2 z = make_double2(0, 0);
    if (j < mps) {
      const double* r = rpos + 3 * (size_t)(p0 + j);
      const double kr = kx * r[0] + ky * r[1] + kz * r[2];
      double sn, cs;
      sincos(kr, &sn, &cs);
      const double u = uV[(size_t)ilma * Nps + j];
      z = make_double2(cs * u, -sn * u);
    }
    const size_t off = ((size_t)kl * Nlma + ilma) * Nps + j;
    z64[off] = z;
    if (z32) z32[off] = make_float2((float)z.x, (float)z.y);
  }
}

cudaError_t launch_update_projector(const System& s) {
  if (s.Nlma == 0) return cudaSuccess;
  dim3 grid(s.Nlma, s.nkl);
  k_update_projector<<<grid, 128, 0, s.stream>>>(s.kAc_d, s.rpos, s.atom_off, s.lma_atom, s.uV_d, s.Nlma, s.Nps,
                                                 s.zproj64, s.prec == SGPU_PREC_C64 ? s.zproj32 : nullptr);
  return cudaGetLastError();
}

// ------------------------------------------------------------ conversion ---
__global__ void k_c128_to_c64(const double2* __restrict__ src, float2* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = make_float2((float)src[i].x, (float)src[i].y);
}
__global__ void k_c64_to_c128(const float2* __restrict__ src, double2* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = make_double2(src[i].x, src[i].y);
}

__global__ void k_r64_to_r32(const double* __restrict__ src, float* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

static int conv_grid(size_t n) {
  size_t g = (n + 255) / 256;
  return (int)(g > 148 * 16 ? 148 * 16 : (g < 1 ? 1 : g));
}

cudaError_t launch_c128_to_c64(const double2* src, float2* dst, size_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_c128_to_c64<<<conv_grid(n), 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}
cudaError_t launch_r64_to_r32(const double* src, float* dst, size_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_r64_to_r32<<<conv_grid(n), 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}
cudaError_t launch_c64_to_c128(const float2* src, double2* dst, size_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_c64_to_c128<<<conv_grid(n), 256, 0, st>>>(src, dst, n);
  return cudaGetLastError();
}

}  // namespace sgpu
