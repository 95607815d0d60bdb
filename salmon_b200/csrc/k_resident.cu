// The whole 4th-order Taylor step of an orbital in one CTA's shared memory
// (grids whose orbital fits on chip: 16^3, 20^3, the 16x16x32 supercell).
//
// The Taylor polynomial of RT/hamiltonian.f90:46-49, :99-122 is applied as the
// product of its four linear factors, psi <- psi + c_s H psi (s = 0..3, see
// taylor_stage_coefs), each stage in place in shared memory:
//
//   * the orbital is read from HBM once, written once (and, with the current
//     requested, its stencil sums are reduced on chip too);
//   * a stage first projects its input on the Kleinman-Bylander projectors
//     (U = Hxyz iuV sum_j conj(zproj) psi(J(j)), hpsi.f90:188-193; one warp per
//     projector item, FP64, a fixed-order warp sum), then builds the KB term at
//     every sphere point (W = sum zproj U, hpsi.f90:194-206, entries in table
//     order), then marches along x applying the stencil of
//     stencil/F90/hpsi.f90:190 plus W and the stage update;
//   * the march is in place: a thread owns two consecutive z points of one y
//     row, keeps its column's nine x-neighbours (old values) in a register
//     queue that rotates by renaming (the march is unrolled nine times), reads
//     y and z neighbours from the plane, and writes the plane's new values only
//     after a CTA barrier, when nobody reads the plane's old values any more.
//     The first four planes' old values, needed again at the periodic wrap, are
//     kept in a small thread-private wrap buffer.
//
// CTAs are persistent over orbitals (orbital o = blockIdx.x + i*gridDim.x), so
// the assignment and every sum order are fixed: results are reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "sgpu_internal.cuh"
#include "stencil_ops.cuh"

namespace sgpu {

template <typename R>
struct ResArgs {
  C2<R>* zu;             // [norb][NL] in and out
  const R* vloc;         // [NL]
  const double* kAc;     // [nkl][3]
  int nkl, NBocc, NLx, NL;
  double lap0sum;
  R lapt[12], nabc[12];
  float2 cl2[12], cn2[12];
  double nab64[12];      // nabx(1:4), naby(1:4), nabz(1:4) for the current's stencil sums
  double zc[4][2];       // stage coefficients
  // Kleinman-Bylander tables
  int nitems, Nlma, Nps, nsp;
  const int4* items;     // {atom, first lma_list slot, count <= 4}
  const int* lma_list;
  const int* atom_off;
  const int* idx_proj;   // packed point -> grid index
  const int* iuV;
  double Hxyz;
  const double2* zproj;  // [nkl][Nlma][Nps]
  const int4* rec;       // [2 nsp] entries of each sphere point
  const int* cont;
  const int* sp_off;     // [NLx+1]
  const short* lqi;      // [NL]
  C2<R>* S;              // [norb][nsp] export of the new orbital at the sphere points (null: none)
  double* cur;           // [norb][4] jt, F, G, H of the new orbital (null: none)
};

__host__ __device__ constexpr size_t res_align16(size_t b) { return (b + 15) & ~(size_t)15; }

// NBC bands of one k-point per CTA; V_loc staged in shared memory where it fits.
template <typename R, int GY, int GZ, int NBC_, int RZ_ = 2> struct ResGeom {
  static constexpr bool c64 = std::is_same<R, float>::value;
  static constexpr int NBC = NBC_;
  static constexpr int RZ = RZ_;                        // z points per thread
  static constexpr bool VS = c64 && GY * GZ <= 256;
  static constexpr int NTO = ((GY * GZ / RZ + 31) / 32) * 32;  // threads per band
  static constexpr int NT = NBC * NTO;
};

// shared memory: NBC orbitals, their wrap planes, W at the sphere points and U;
// the sphere-index table, V_loc (when staged), sp_off and the reduction scratch
template <typename R, int GY, int GZ, int NBC, int RZ = 2>
__host__ __device__ inline size_t res_smem_bytes(int NLx, int nsp, int Nlma) {
  using G = ResGeom<R, GY, GZ, NBC, RZ>;
  const size_t e = sizeof(C2<R>), NL = (size_t)NLx * GY * GZ;
  return G::NBC * (res_align16(e * NL) + res_align16(e * 4 * GY * GZ) + res_align16(e * (size_t)nsp) +
                   res_align16(sizeof(double2) * (size_t)Nlma)) +
         res_align16(sizeof(short) * NL) + (G::VS ? res_align16(sizeof(R) * NL) : 0) +
         res_align16(sizeof(int) * (size_t)(NLx + 1)) + 32 * 4 * sizeof(double);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// One CTA advances NBC consecutive bands of one k-point together (lockstep
// marches, one barrier per plane for all of them), so the projector tables each
// stage reads are shared by NBC orbitals through L1.
template <typename R, int GY, int GZ, int NBC_, int RZ_>
__global__ void __launch_bounds__(ResGeom<R, GY, GZ, NBC_, RZ_>::NT, 1) k_taylor_resident(const ResArgs<R> a) {
  using T = C2<R>;
  using G = ResGeom<R, GY, GZ, NBC_, RZ_>;
  constexpr int RZ = G::RZ, NBC = G::NBC, NTO = G::NTO, NT = G::NT;
  constexpr int NLy = GY, NLz = GZ, NYZ = GY * GZ, NZG = GZ / RZ;
  static_assert(GZ % RZ == 0 && (RZ == 1 || RZ == 2), "one or two z points per thread");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NLx = a.NLx, NL = a.NL;
  unsigned char* sp = smem_raw;
  T* P0 = reinterpret_cast<T*>(sp);                 // [NBC][NL]
  sp += NBC * res_align16(sizeof(T) * (size_t)NL);
  T* wrap0 = reinterpret_cast<T*>(sp);              // [NBC][4][NYZ]
  sp += NBC * res_align16(sizeof(T) * 4 * NYZ);
  T* Wq0 = reinterpret_cast<T*>(sp);                // [NBC][nsp]
  const size_t wq_stride = res_align16(sizeof(T) * (size_t)a.nsp) / sizeof(T);
  sp += NBC * res_align16(sizeof(T) * (size_t)a.nsp);
  double2* Us0 = reinterpret_cast<double2*>(sp);    // [NBC][Nlma]
  const size_t us_stride = res_align16(sizeof(double2) * (size_t)a.Nlma) / sizeof(double2);
  sp += NBC * res_align16(sizeof(double2) * (size_t)a.Nlma);
  short* lqs = reinterpret_cast<short*>(sp);        // [NL]
  sp += res_align16(sizeof(short) * (size_t)NL);
  R* vls = reinterpret_cast<R*>(sp);                // [NL] (VS)
  if (G::VS) sp += res_align16(sizeof(R) * (size_t)NL);
  int* spo = reinterpret_cast<int*>(sp);            // [NLx+1]
  sp += res_align16(sizeof(int) * (size_t)(NLx + 1));
  double* red = reinterpret_cast<double*>(sp);      // [NT/32][4]

  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int bs = t / NTO, tl = t - bs * NTO;        // band slot, thread within the band
  T* P = P0 + (size_t)bs * (res_align16(sizeof(T) * (size_t)NL) / sizeof(T));
  T* wrap = wrap0 + (size_t)bs * (res_align16(sizeof(T) * 4 * NYZ) / sizeof(T));
  T* Wq = Wq0 + (size_t)bs * wq_stride;
  const bool act = tl < NYZ / RZ;
  const int y = act ? tl / NZG : 0;
  const int z0 = act ? (tl - y * NZG) * RZ : 0;
  const int own = y * NLz + z0;
  int yo[8];
#pragma unroll
  for (int n = 1; n <= 4; ++n) {
    yo[n - 1] = wrapi(y + n, NLy) * NLz + z0;
    yo[3 + n] = wrapi(y - n, NLy) * NLz + z0;
  }
  constexpr int NZZ = RZ + 8;
  int zoff[NZZ / RZ];
#pragma unroll
  for (int m = 0; m < NZZ / RZ; ++m) zoff[m] = y * NLz + wrapi(z0 + m * RZ - 4, NLz);

  // tables shared by every orbital of the launch
  for (int i = t; i < NL / 2; i += NT) reinterpret_cast<int*>(lqs)[i] = __ldg(reinterpret_cast<const int*>(a.lqi) + i);
  if (G::VS)
    for (int i = t; i < NL; i += NT) vls[i] = __ldg(a.vloc + i);
  for (int i = t; i <= NLx; i += NT) spo[i] = __ldg(a.sp_off + i);

  using KT = typename std::conditional<std::is_same<R, float>::value, float2, double>::type;
  auto CL = [&](int i) -> KT {
    if constexpr (std::is_same<R, float>::value) return a.cl2[i]; else return a.lapt[i];
  };
  auto CN = [&](int i) -> KT {
    if constexpr (std::is_same<R, float>::value) return a.cn2[i]; else return a.nabc[i];
  };

  const int gpk = (a.NBocc + NBC - 1) / NBC;        // band groups per k-point
  const int ngroups = a.nkl * gpk;
  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    const int kl = grp / gpk;
    const int b0 = (grp - kl * gpk) * NBC;
    const int nbg = min(NBC, a.NBocc - b0);         // bands in this group
    const bool band_ok = bs < nbg;
    const int o = kl * a.NBocc + b0 + bs;           // this thread's orbital (if band_ok)
    const double kxd = a.kAc[3 * kl], kyd = a.kAc[3 * kl + 1], kzd = a.kAc[3 * kl + 2];
    const R A = (R)((kxd * kxd + kyd * kyd + kzd * kzd - a.lap0sum) * 0.5);  // k2lap0_2 (hpsi.f90:120-121)
    const KT kx = kpair<R>(kxd), ky = kpair<R>(kyd), kz = kpair<R>(kzd);
    T* zo = a.zu + (size_t)o * NL;
    const double2* zpk = a.zproj + (size_t)kl * a.Nlma * a.Nps;

    // the group's orbitals into shared memory (16-byte cp.async chunks)
    {
      const int nchunk = (int)((sizeof(T) * (size_t)NL) / 16);
      const char* src = reinterpret_cast<const char*>(a.zu + (size_t)(kl * a.NBocc + b0) * NL);
      for (int i = t; i < nbg * nchunk; i += NT) {
        const int b = i / nchunk, c = i - b * nchunk;
        char* dst = reinterpret_cast<char*>(P0 + (size_t)b * (res_align16(sizeof(T) * (size_t)NL) / sizeof(T)));
        cp_async16(dst + 16 * (size_t)c, src + 16 * (size_t)i);
      }
      cp_async_commit();
      cp_async_wait<0>();
    }
    __syncthreads();

    for (int st = 0; st < 4; ++st) {
      const T zc = mk<R>((R)a.zc[st][0], (R)a.zc[st][1]);
      const bool last = st == 3;
      // ---- projections of the stage input: one warp per (projector item, band);
      // the warps of one item are adjacent, so its zproj rows are L1 hits after the first
      for (int task = warp; task < a.nitems * NBC; task += NT / 32) {
        const int it = task / NBC, b = task - it * NBC;
        if (b >= nbg) continue;                     // uniform over the warp
        const T* Pb = P0 + (size_t)b * (res_align16(sizeof(T) * (size_t)NL) / sizeof(T));
        const int4 item = __ldg(a.items + it);
        const int at = item.x, l0 = item.y, np = item.z;
        const int p0 = __ldg(a.atom_off + at), mps = __ldg(a.atom_off + at + 1) - p0;
        int lm[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) lm[p] = p < np ? __ldg(a.lma_list + l0 + p) : 0;
        double ur[4] = {0, 0, 0, 0}, ui[4] = {0, 0, 0, 0};
#pragma unroll 2
        for (int j = lane; j < mps; j += 32) {
          const double2 v = to_d2(Pb[__ldg(a.idx_proj + p0 + j)]);
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            if (p < np) {
              const double2 z = __ldg(zpk + (size_t)lm[p] * a.Nps + j);
              // conj(z) v
              ur[p] = fma(z.x, v.x, fma(z.y, v.y, ur[p]));
              ui[p] = fma(z.x, v.y, fma(-z.y, v.x, ui[p]));
            }
          }
        }
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          if (p < np) {  // np is uniform over the warp
            const double sr = warp_sum(ur[p]), si = warp_sum(ui[p]);
            if (lane == 0) {
              const double f = a.Hxyz * (double)__ldg(a.iuV + lm[p]);
              Us0[(size_t)b * us_stride + lm[p]] = make_double2(sr * f, si * f);
            }
          }
        }
      }
      __syncthreads();
      // ---- KB term at every sphere point for every band of the group (entries in
      // table order; each entry's zproj is loaded once for the group), and the
      // wrap planes (this thread's column of planes 0..3, old values)
      for (int q = t; q < a.nsp; q += NT) {
        const int4 ra = __ldg(a.rec + 2 * (size_t)q), rb = __ldg(a.rec + 2 * (size_t)q + 1);
        const int ne = ra.y + rb.w;
        double2 acc[NBC];
#pragma unroll
        for (int b = 0; b < NBC; ++b) acc[b] = make_double2(0.0, 0.0);
        for (int e = 0; e < ne; ++e) {
          const int en = e < 4 ? (e == 0 ? ra.z : (e == 1 ? ra.w : (e == 2 ? rb.x : rb.y)))
                               : __ldg(a.cont + rb.z + (e - 4));
          const int ilma = en >> 16;
          const double2 z = __ldg(zpk + (size_t)ilma * a.Nps + (en & 0xffff));
#pragma unroll
          for (int b = 0; b < NBC; ++b) acc[b] = cfma(z, Us0[(size_t)b * us_stride + ilma], acc[b]);
        }
#pragma unroll
        for (int b = 0; b < NBC; ++b) Wq0[(size_t)b * wq_stride + q] = mk<R>((R)acc[b].x, (R)acc[b].y);
      }
      if (act) {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          T run[RZ];
          lds_run<R, RZ>(run, P + (size_t)m * NYZ + own);
          st_run<R, RZ>(wrap + (size_t)m * NYZ + own, run);
        }
      }
      __syncthreads();

      // ---- the march: register queue of the thread's column (old values);
      // plane x-4+m sits in q[(P+m) % 9] at phase P
      T q[9][RZ];
      if (act) {
#pragma unroll
        for (int n = 0; n < 8; ++n) lds_run<R, RZ>(q[n], P + (size_t)wrapi(n - 4, NLx) * NYZ + own);
      }
      int x = 0;
      auto step = [&](auto phase) -> bool {
        constexpr int PH = decltype(phase)::value;
        const T* pl = P + (size_t)x * NYZ;
        T res[RZ];
        int lq[RZ];
        if (act) {
          {  // plane x+4 (old): from the orbital, or the wrap buffer past the end
            const int xn = x + 4;
            lds_run<R, RZ>(q[(PH + 8) % 9], xn < NLx ? P + (size_t)xn * NYZ + own : wrap + (size_t)(xn - NLx) * NYZ + own);
          }
          if constexpr (RZ == 2) {
            const int lqv = *reinterpret_cast<const int*>(lqs + (size_t)x * NYZ + own);
            lq[0] = (int)(short)(lqv & 0xffff);
            lq[1] = lqv >> 16;
          } else {
            lq[0] = lqs[(size_t)x * NYZ + own];
          }
          R vl[RZ];
          if constexpr (G::VS) {
#pragma unroll
            for (int r = 0; r < RZ; ++r) vl[r] = vls[(size_t)x * NYZ + own + r];
          } else {
#pragma unroll
            for (int r = 0; r < RZ; ++r) vl[r] = __ldg(a.vloc + (size_t)x * NYZ + own + r);
          }
          T v[RZ], w[RZ], wa[RZ], vy[RZ];
#pragma unroll
          for (int r = 0; r < RZ; ++r) { v[r] = mk<R>(0, 0); wa[r] = mk<R>(0, 0); vy[r] = mk<R>(0, 0); }
          if constexpr (std::is_same<R, float>::value) {
            T zv[NZZ];
#pragma unroll
            for (int m = 0; m < NZZ / RZ; ++m) {
              T run[RZ];
              if (m * RZ == 4) {
#pragma unroll
                for (int s2 = 0; s2 < RZ; ++s2) run[s2] = q[(PH + 4) % 9][s2];
              } else {
                lds_run<R, RZ>(run, pl + zoff[m]);
              }
#pragma unroll
              for (int s2 = 0; s2 < RZ; ++s2) zv[m * RZ + s2] = run[s2];
            }
#pragma unroll
            for (int n = 1; n <= 4; ++n)
#pragma unroll
              for (int r = 0; r < RZ; ++r)
                stencil_pair(v[r], wa[r], zv[4 + r + n], zv[4 + r - n], CL(8 + n - 1), CN(8 + n - 1));
          } else {
#pragma unroll
            for (int m = 0; m < NZZ / RZ; ++m) {
              T run[RZ];
              if (m * RZ == 4) {
#pragma unroll
                for (int s2 = 0; s2 < RZ; ++s2) run[s2] = q[(PH + 4) % 9][s2];
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
                    const R cl = a.lapt[7 + n];
                    const R cn = k > 0 ? a.nabc[7 + n] : -a.nabc[7 + n];
                    v[r].x = fma(cl, run[s2].x, v[r].x);
                    v[r].y = fma(cl, run[s2].y, v[r].y);
                    wa[r].x = fma(cn, run[s2].x, wa[r].x);
                    wa[r].y = fma(cn, run[s2].y, wa[r].y);
                  }
                }
            }
          }
#pragma unroll
          for (int r = 0; r < RZ; ++r) { w[r] = kscale(kz, wa[r], mk<R>(0, 0)); wa[r] = mk<R>(0, 0); }
#pragma unroll
          for (int n = 1; n <= 4; ++n) {  // y
            T rp[RZ], rm[RZ];
            lds_run<R, RZ>(rp, pl + yo[n - 1]);
            lds_run<R, RZ>(rm, pl + yo[3 + n]);
#pragma unroll
            for (int r = 0; r < RZ; ++r) stencil_pair(vy[r], wa[r], rp[r], rm[r], CL(4 + n - 1), CN(4 + n - 1));
          }
#pragma unroll
          for (int r = 0; r < RZ; ++r) { w[r] = kscale(ky, wa[r], w[r]); wa[r] = mk<R>(0, 0); }
#pragma unroll
          for (int n = 1; n <= 4; ++n)  // x: the register queue
#pragma unroll
            for (int r = 0; r < RZ; ++r)
              stencil_pair(v[r], wa[r], q[(PH + 4 + n) % 9][r], q[(PH + 4 - n) % 9][r], CL(n - 1), CN(n - 1));
#pragma unroll
          for (int r = 0; r < RZ; ++r) {
            w[r] = kscale(kx, wa[r], w[r]);
            v[r] = cadd(v[r], vy[r]);
          }
          const T* wpl = Wq + spo[x];
#pragma unroll
          for (int r = 0; r < RZ; ++r) {
            const T c = q[(PH + 4) % 9][r];
            // F = B E + A E - 0.5 v - zI w   (stencil/F90/hpsi.f90:190)
            T f;
            f.x = fma(vl[r] + A, c.x, fma((R)-0.5, v[r].x, w[r].y));
            f.y = fma(vl[r] + A, c.y, fma((R)-0.5, v[r].y, -w[r].x));
            if (lq[r] >= 0) f = cadd(f, wpl[lq[r]]);  // + pseudo_pt scatter (hpsi.f90:203-206)
            res[r] = cfma(zc, f, c);                 // the stage: psi + c H psi
          }
        }
        __syncthreads();  // every thread has read plane x's old values
        if (act) {
          st_run<R, RZ>(P + (size_t)x * NYZ + own, res);
          if (last && band_ok) {
            st_run<R, RZ>(zo + (size_t)x * NYZ + own, res);
            if (a.S) {
              const int q0 = spo[x];
#pragma unroll
              for (int r = 0; r < RZ; ++r)
                if (lq[r] >= 0) a.S[(size_t)o * a.nsp + q0 + lq[r]] = res[r];
            }
          }
        }
        ++x;
        return x < NLx;
      };
      for (;;) {
        if (!step(std::integral_constant<int, 0>{})) break;
        if (!step(std::integral_constant<int, 1>{})) break;
        if (!step(std::integral_constant<int, 2>{})) break;
        if (!step(std::integral_constant<int, 3>{})) break;
        if (!step(std::integral_constant<int, 4>{})) break;
        if (!step(std::integral_constant<int, 5>{})) break;
        if (!step(std::integral_constant<int, 6>{})) break;
        if (!step(std::integral_constant<int, 7>{})) break;
        if (!step(std::integral_constant<int, 8>{})) break;
      }
      __syncthreads();  // the stage's output is complete
    }

    // ---- the current's stencil sums of the new orbitals (current.f90:182-186,
    // stencil/F90/current.f90): jt = sum |psi|^2, F/G/H = sum Im(conj(psi) v_d),
    // v_d = sum_n nab_d(n) psi(+n e_d), FP64, per thread in plane order, then a
    // fixed-order sum over the band's warps.
    if (a.cur) {
      double s4[4] = {0, 0, 0, 0};
      if (act) {
        for (int xx = 0; xx < NLx; ++xx) {
#pragma unroll
          for (int r = 0; r < RZ; ++r) {
            const int i = xx * NYZ + own + r;
            const double2 e = to_d2(P[i]);
            s4[0] = fma(e.x, e.x, fma(e.y, e.y, s4[0]));
            double2 vx = make_double2(0, 0), vyy = make_double2(0, 0), vz = make_double2(0, 0);
#pragma unroll
            for (int n = 1; n <= 4; ++n) {
              const double2 px = to_d2(P[wrapi(xx + n, NLx) * NYZ + own + r]);
              const double2 py = to_d2(P[xx * NYZ + wrapi(y + n, NLy) * NLz + z0 + r]);
              const double2 pz = to_d2(P[xx * NYZ + y * NLz + ((z0 + r + n) % NLz)]);
              vx.x = fma(a.nab64[n - 1], px.x, vx.x);
              vx.y = fma(a.nab64[n - 1], px.y, vx.y);
              vyy.x = fma(a.nab64[3 + n], py.x, vyy.x);
              vyy.y = fma(a.nab64[3 + n], py.y, vyy.y);
              vz.x = fma(a.nab64[7 + n], pz.x, vz.x);
              vz.y = fma(a.nab64[7 + n], pz.y, vz.y);
            }
            // aimag(conjg(e) v) = e.x v.y - e.y v.x
            s4[1] += e.x * vx.y - e.y * vx.x;
            s4[2] += e.x * vyy.y - e.y * vyy.x;
            s4[3] += e.x * vz.y - e.y * vz.x;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) s4[k] = warp_sum(s4[k]);
      if (lane == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[warp * 4 + k] = s4[k];
      __syncthreads();
      if (t < 4 * NBC) {
        const int b = t >> 2, k = t & 3;
        if (b < nbg) {
          double acc = 0.0;
          for (int w2 = 0; w2 < NTO / 32; ++w2) acc += red[(b * (NTO / 32) + w2) * 4 + k];
          a.cur[(size_t)(kl * a.NBocc + b0 + b) * 4 + k] = acc;
        }
      }
    }
    __syncthreads();  // before the next group overwrites P and red
  }
}

// ------------------------------------------------------------------ launch --
template <typename R, int GY, int GZ, int NBC, int RZ = 2>
static size_t res_smem(const System& s) { return res_smem_bytes<R, GY, GZ, NBC, RZ>(s.NLx, s.nsp, s.Nlma); }

template <typename R, int GY, int GZ, int NBC, int RZ>
static cudaError_t launch_res_t(const System& s, void* zu, double dt, double* cur, void* S) {
  using G = ResGeom<R, GY, GZ, NBC, RZ>;
  const size_t smem = res_smem<R, GY, GZ, NBC, RZ>(s);
  auto kern = k_taylor_resident<R, GY, GZ, NBC, RZ>;
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s.stream, &cs);
    if (e != cudaSuccess) return e;
    if (cs == cudaStreamCaptureStatusNone && smem > 48 * 1024) {
      e = raise_smem_limit((const void*)kern, smem);
      if (e != cudaSuccess) return e;
    }
  }
  ResArgs<R> a;
  a.zu = (C2<R>*)zu;
  a.vloc = std::is_same<R, float>::value ? (const R*)s.vloc32 : (const R*)s.vloc64;
  a.kAc = s.kAc_d;
  a.nkl = s.nkl;
  a.NBocc = s.NBocc;
  a.NLx = s.NLx;
  a.NL = s.NL;
  a.lap0sum = s.lap[0][0] + s.lap[1][0] + s.lap[2][0];
  for (int n = 0; n < 4; ++n)
    for (int d = 0; d < 3; ++d) {
      a.lapt[4 * d + n] = (R)s.lap[d][n + 1];
      a.nabc[4 * d + n] = (R)s.nab[d][n + 1];
      a.cl2[4 * d + n] = make_float2((float)s.lap[d][n + 1], (float)s.lap[d][n + 1]);
      a.cn2[4 * d + n] = make_float2((float)s.nab[d][n + 1], (float)s.nab[d][n + 1]);
      a.nab64[4 * d + n] = s.nab[d][n + 1];
    }
  taylor_stage_coefs(dt, a.zc);
  a.nitems = s.nitems;
  a.Nlma = s.Nlma;
  a.Nps = s.Nps;
  a.nsp = s.nsp;
  a.items = s.items;
  a.lma_list = s.lma_list;
  a.atom_off = s.atom_off;
  a.idx_proj = s.idx_proj;
  a.iuV = s.iuV_d;
  a.Hxyz = s.Hxyz;
  a.zproj = s.zproj64;
  a.rec = s.rec;
  a.cont = s.cont;
  a.sp_off = s.sp_off;
  a.lqi = s.lqi;
  a.S = (C2<R>*)S;
  a.cur = cur;
  const int ngroups = s.nkl * ((s.NBocc + NBC - 1) / NBC);
  const int grid = std::min(ngroups, s.nsm);  // one CTA per SM (shared memory), persistent over groups
  kern<<<grid, G::NT, smem, s.launch_stream()>>>(a);
  return cudaGetLastError();
}

// The forms built for each plane shape, widest band group first:
//   complex(4), two z points per thread: 16x16 planes 4 or 2 bands per CTA, 16x32
//   and 20x20 2 or 1;
//   complex(8), one z point per thread (twice the warps of the two-point form at
//   its register count): 16x16 planes 2 or 1 bands, 16x32 and 20x20 1.
// f(tag, GY, GZ, NBC, RZ) is called for the first form whose shared memory fits
// (returns false if none does).
template <typename F>
static bool res_dispatch(const System& s, F&& f) {
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  using I4 = std::integral_constant<int, 4>;
  using I16 = std::integral_constant<int, 16>;
  using I20 = std::integral_constant<int, 20>;
  using I32 = std::integral_constant<int, 32>;
  if (s.NLx < 9 || s.nsp < 1 || s.nitems < 1) return false;
  constexpr size_t cap = 227 * 1024;
  auto tryf = [&](auto tag, auto gy, auto gz, auto nbc, auto rz) {
    using R = decltype(tag);
    if (res_smem<R, decltype(gy)::value, decltype(gz)::value, decltype(nbc)::value, decltype(rz)::value>(s) > cap)
      return false;
    f(tag, gy, gz, nbc, rz);
    return true;
  };
  if (s.prec == SGPU_PREC_C64) {
    if (s.NLy == 16 && s.NLz == 16) return tryf(0.0f, I16{}, I16{}, I4{}, I2{}) || tryf(0.0f, I16{}, I16{}, I2{}, I2{});
    if (s.NLy == 16 && s.NLz == 32) return tryf(0.0f, I16{}, I32{}, I2{}, I2{}) || tryf(0.0f, I16{}, I32{}, I1{}, I2{});
    if (s.NLy == 20 && s.NLz == 20) return tryf(0.0f, I20{}, I20{}, I2{}, I2{}) || tryf(0.0f, I20{}, I20{}, I1{}, I2{});
  } else {
    if (s.NLy == 16 && s.NLz == 16) return tryf(0.0, I16{}, I16{}, I2{}, I1{}) || tryf(0.0, I16{}, I16{}, I1{}, I1{});
    if (s.NLy == 16 && s.NLz == 32) return tryf(0.0, I16{}, I32{}, I1{}, I1{});
    if (s.NLy == 20 && s.NLz == 20) return tryf(0.0, I20{}, I20{}, I1{}, I1{});
  }
  return false;
}

bool resident_step_fits(const System& s) {
  return res_dispatch(s, [](auto, auto, auto, auto, auto) {});
}

// The resident form is the default (SGPU_PARAM_TAYLOR_KERNEL 0) where it measured
// faster than the stencil passes: 16x16 planes (16^3 grid x 64 k x 16 bands:
// complex(4) 0.181 against 0.201 ms per step, complex(8) 0.326 against 0.437 ms).
// Elsewhere it is slower (20^3 x 2048 orbitals: complex(4) 1.27 against 0.73 ms,
// complex(8) 1.95 against 1.47 ms): with one CTA per SM the latency of the
// projector-table loads in each stage's KB phase is not hidden behind other CTAs'
// work, and the 20x20 forms spill.  The step tuner measures both per shape.
bool resident_step_default(const System& s) {
  return s.NLy == 16 && s.NLz == 16 && resident_step_fits(s);
}

cudaError_t launch_taylor_resident(const System& s, void* zu, double dt, double* cur, void* S) {
  cudaError_t e = cudaSuccess;
  const bool ok = res_dispatch(s, [&](auto tag, auto gy, auto gz, auto nbc, auto rz) {
    e = launch_res_t<decltype(tag), decltype(gy)::value, decltype(gz)::value, decltype(nbc)::value,
                     decltype(rz)::value>(s, zu, dt, cur, S);
  });
  if (!ok) return cudaErrorNotSupported;
  return e;
}

cudaError_t prepare_resident(const System& s) {
  cudaError_t e = cudaSuccess;
  res_dispatch(s, [&](auto tag, auto gy, auto gz, auto nbc, auto rz) {
    using R = decltype(tag);
    constexpr int GY = decltype(gy)::value, GZ = decltype(gz)::value, NBC = decltype(nbc)::value;
    constexpr int RZ = decltype(rz)::value;
    const size_t b = res_smem<R, GY, GZ, NBC, RZ>(s);
    if (b > 48 * 1024) e = raise_smem_limit((const void*)k_taylor_resident<R, GY, GZ, NBC, RZ>, b);
  });
  return e;
}

}  // namespace sgpu
