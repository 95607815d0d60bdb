// One Hamiltonian application (and the fused last Taylor pass) for sm_100a.
//
// H psi = (k2lap0_2 + Vloc) psi - 1/2 sum lapt (psi(+n)+psi(-n)) - i sum nabt (psi(+n)-psi(-n))
//         + W,   W = sum_ilma zproj(:,ilma) U(ilma) at the sphere points
// restates hpsi_omp_KB_base (common/hpsi.f90:98-208): the stencil of
// stencil/F90/hpsi.f90:190 plus the Kleinman-Bylander scatter of pseudo_pt
// (:194-206).  W is computed beforehand by k_kbfield (k_hpsi.cu) in a compact
// per-orbital array over the sphere points, ordered by grid index.
//
// Layout: one CTA per (orbital, x-slab).  A y-z plane of one orbital is a
// contiguous NLy*NLz run in HBM (z unit stride).  Each thread owns RZ
// consecutive z points of one y row and marches along x:
//   * planes stream into a shared-memory ring with cp.async, NR-5 planes ahead
//     of use, together with each plane's contiguous chunk of W, so HBM latency
//     is off the critical path;
//   * the thread's own 9 x-neighbours sit in a register queue;
//   * y and z neighbours come from the shared-memory plane;
//   * a point's local sphere index (int16 table, loaded one plane ahead) tells
//     whether to add W and whether to export the output value to S, the
//     compact sphere-value array the next pass's projections read.
// Each input element is read from HBM once per pass (the 8 halo planes of a
// slab come from L2), each output element written once.
#include <cuda_runtime.h>

#include <type_traits>

#include "sgpu_internal.cuh"
#include "stencil_ops.cuh"

namespace sgpu {

template <typename R>
struct PassArgs {
  const C2<R>* in;       // [nb][NL]
  C2<R>* out;            // [nb][NL]
  C2<R>* tt;             // [nb][NL]   (mode 1)
  const R* vloc;
  const double* kAc;     // [nkl][3]
  int o_beg, NBocc;
  int NLx, NLy, NLz, NL, SX;
  double lap0sum;        // lapx(0)+lapy(0)+lapz(0)
  R lapt[12];            // lapx(1:4), lapy(1:4), lapz(1:4)
  R nabc[12];            // nabx(1:4), naby(1:4), nabz(1:4)
  float2 cl2[12], cn2[12];  // complex(4): lapt and nabc as broadcast pairs for the packed FP32 arithmetic
  // Kleinman-Bylander term by plane: plane x's sphere points are
  // sp_off[x] .. sp_off[x+1]-1 (at most maxpts); lqi[i] is the index of grid
  // point i among its plane's sphere points, or -1.
  const int* sp_off;
  // y-blocks (YB form, planes wider than one CTA): each orbital plane is split
  // into nyblk CTAs of NYB rows; sp_blk[x*(nyblk+1) + yb] is the first sphere
  // point of plane x in rows >= yb*NYB (sp_blk[x*(nyblk+1)] = sp_off[x]).
  int NYB, nyblk;
  const int* sp_blk;
  const short* lqi;
  const C2<R>* W;        // [nb][nsp] KB term at the sphere points (null: none)
  C2<R>* S;              // [nb][nsp] export of the output (null: none)
  int nsp, maxpts;
  C2<R> zf;              // mode 2: the Taylor stage coefficient c
};

template <typename R> struct PassGeom {
  static constexpr int NR = std::is_same<R, float>::value ? 8 : 6;  // ring planes
};

size_t pass_smem_bytes(int prec, int NLy, int NLz, int maxpts, bool with_w, int NLx, int nyblk, int NYB,
                       bool tables, int nr) {
  const size_t e = prec == SGPU_PREC_C64 ? sizeof(float2) : sizeof(double2);
  const int NR = nr > 0 ? nr : (prec == SGPU_PREC_C64 ? PassGeom<float>::NR : PassGeom<double>::NR);
  const size_t ryz = nyblk > 1 ? (size_t)(NYB + 8) * NLz : (size_t)NLy * NLz;
  const size_t tyz = nyblk > 1 ? (size_t)NYB * NLz : (size_t)NLy * NLz;
  return e * (size_t)NR * (ryz + (with_w ? (size_t)maxpts : 0)) +
         (tables ? (size_t)NR * tyz * (e / 2 + sizeof(short)) : 0) + sizeof(int) * (size_t)NLx * (nyblk + 1) +
         sizeof(int);
}

// MODE 0: out = H in.   MODE 1: also tt = H in - V in before the nonlocal term.
// MODE 2: out = in + c H in, one linear factor of the Taylor polynomial
// (RT/hamiltonian.f90:46-49, :99-122 evaluated as the product of its four
// linear factors; see enqueue_taylor_step).
//
// YB (planes of more than 512 threads' points): the plane is split over nyblk
// CTAs of NYB rows; each CTA's ring holds its rows and 4 halo rows on each side.
// TB (two-point form): Vloc and the local sphere indices of each owned plane
// travel with the plane through the ring (copy group of the plane) instead of
// being loaded from global memory one plane ahead; this takes the dependent
// global loads off each march step.
//
// GY, GZ (non-zero: the plane shape NLy x NLz at compile time, complex(4), two-point
// table form; GB: the rows of a y-block, with YB): the ring then has one slot per
// unrolled phase (NR = 9), so every ring, table and neighbour offset is a
// compile-time constant and the per-step address arithmetic drops to a few adds.
template <typename R, int RZ, int MODE, bool YB, bool TB, int GY = 0, int GZ = 0, int GB = 0>
__global__ void __launch_bounds__(512) k_hpsi_pass(const PassArgs<R> a) {
  static_assert(!TB || RZ == 2, "table staging copies the two points' entries as one run");
  static_assert(GZ == 0 || (std::is_same<R, float>::value && TB && (YB == (GB > 0))),
                "fixed shapes: complex(4) table form; y-block rows with y-blocks only");
  using T = C2<R>;
  constexpr bool FIXED = GZ > 0;
  constexpr int NR = FIXED ? 9 : PassGeom<R>::NR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NLy = FIXED ? GY : a.NLy, NLz = FIXED ? GZ : a.NLz, NYZ = NLy * NLz;
  const bool with_w = a.W != nullptr;
  const bool do_export = a.S != nullptr;
  const int NYBc = YB ? (FIXED ? GB : a.NYB) : NLy;  // rows of a y-block
  const int nyblk = YB ? (FIXED ? (GY + GB - 1) / GB : a.nyblk) : 1;
  const int RYZ = YB ? (NYBc + 8) * NLz : NYZ;  // ring plane size
  T* ring = reinterpret_cast<T*>(smem_raw);
  T* wring = ring + (size_t)NR * RYZ;  // [NR][maxpts] W chunks of the ring's planes
  constexpr bool tab = TB;
  const int TYZ = YB ? NYBc * NLz : NYZ;  // table plane size (owned rows)
  R* vtab = reinterpret_cast<R*>(wring + (with_w ? (size_t)NR * a.maxpts : 0));  // [NR][TYZ] (tab)
  short* lqtab = reinterpret_cast<short*>(vtab + (tab ? (size_t)NR * TYZ : 0));    // [NR][TYZ] (tab)
  // sp_off[0..NLx] (or sp_blk in the YB form)
  int* spo = reinterpret_cast<int*>(lqtab + (tab ? (size_t)NR * TYZ : 0));
  if constexpr (YB) {
    for (int i = threadIdx.x; i < a.NLx * (nyblk + 1); i += blockDim.x) spo[i] = a.sp_blk[i];
  } else {
    for (int i = threadIdx.x; i <= a.NLx; i += blockDim.x) spo[i] = a.sp_off[i];
  }
  __syncthreads();

  const int b = YB ? blockIdx.x / nyblk : blockIdx.x;
  const int yb = YB ? blockIdx.x - b * nyblk : 0;
  const int y0 = YB ? yb * NYBc : 0;
  const int o = a.o_beg + b;
  const int kl = o / a.NBocc;
  const double kxd = a.kAc[3 * kl], kyd = a.kAc[3 * kl + 1], kzd = a.kAc[3 * kl + 2];
  const R A = (R)((kxd * kxd + kyd * kyd + kzd * kzd - a.lap0sum) * 0.5);  // k2lap0_2 (hpsi.f90:120-121)
  // nabt = k_d nab_d (hpsi.f90:122-124), applied once per axis:
  // w = sum_d k_d sum_n nab_d,n (psi(+n) - psi(-n))
  using KT = typename std::conditional<std::is_same<R, float>::value, float2, double>::type;
  const KT kx = kpair<R>(kxd), ky = kpair<R>(kyd), kz = kpair<R>(kzd);
  // FD coefficients: broadcast pairs for complex(4), scalars for complex(8)
  auto CL = [&](int i) -> KT {
    if constexpr (std::is_same<R, float>::value) return a.cl2[i]; else return a.lapt[i];
  };
  auto CN = [&](int i) -> KT {
    if constexpr (std::is_same<R, float>::value) return a.cn2[i]; else return a.nabc[i];
  };

  const int NZG = NLz / RZ;
  const int t = threadIdx.x;
  const int bd = blockDim.x;
  const int ny_own = YB ? min(NYBc, NLy - y0) : NLy;
  const bool act = t < ny_own * NZG;
  const int yl = act ? t / NZG : 0;  // row in the block
  const int y = y0 + yl;             // row in the plane
  const int z0 = act ? (t - yl * NZG) * RZ : 0;
  const int own = y * NLz + z0;                       // in the plane
  const int own_r = YB ? (4 + yl) * NLz + z0 : own;   // in the ring
  const int own_t = YB ? yl * NLz + z0 : own;         // in the table planes

  const int x_beg = blockIdx.y * a.SX;
  const int x_end = min(x_beg + a.SX, a.NLx);
  if (x_beg >= x_end) return;  // whole CTA leaves together
  const int nplanes = x_end - x_beg + 4;  // planes the ring delivers: x_beg .. x_end+3
  const int nown = x_end - x_beg;         // planes that need W
  const T* inb = a.in + (size_t)b * a.NL;
  const T* Wb = with_w ? a.W + (size_t)b * a.nsp : nullptr;
  T* Sb = do_export ? a.S + (size_t)b * a.nsp : nullptr;

  // plane jn (relative to x_beg) into ring slot sl (= jn modulo the ring), with its W chunk
  auto refill = [&](int jn, int sl) {
    int p = x_beg + jn;
    while (p >= a.NLx) p -= a.NLx;
    if constexpr (YB) {
      if (jn < nplanes) {  // the block's rows and the halo rows, periodic in y
        T* dst = ring + (size_t)sl * RYZ;
        const T* src = inb + (size_t)p * NYZ;
        for (int idx = t; idx < (NYBc + 8) * NZG; idx += bd) {
          const int r = idx / NZG, zz = (idx - r * NZG) * RZ;
          int gy = y0 - 4 + r;
          gy += gy < 0 ? NLy : 0;
          gy -= gy >= NLy ? NLy : 0;
          cp_run<R, RZ>(dst + r * NLz + zz, src + gy * NLz + zz);
        }
      }
    } else {
      if (act && jn < nplanes) cp_run<R, RZ>(ring + (size_t)sl * NYZ + own, inb + (size_t)p * NYZ + own);
    }
    if constexpr (TB) {
      if (act && jn < nown) {
        const size_t g = (size_t)p * NYZ + own;
        R* vd = vtab + (size_t)sl * TYZ + own_t;
        if constexpr (sizeof(R) == 4) cp_async8(vd, a.vloc + g); else cp_async16(vd, a.vloc + g);
        if (with_w || do_export) cp_async4(lqtab + (size_t)sl * TYZ + own_t, a.lqi + g);
      }
    }
    if (with_w && jn < nown) {
      const int q0 = YB ? spo[p * (nyblk + 1) + yb] : spo[p];
      const int q1 = YB ? spo[p * (nyblk + 1) + yb + 1] : spo[p + 1];
      T* dst = wring + (size_t)sl * a.maxpts;
      for (int qq = q0 + t; qq < q1; qq += bd) cp_run<R, 1>(dst + (qq - q0), Wb + qq);
    }
    cp_async_commit();
  };
#pragma unroll 1
  for (int n = 0; n < NR - 1; ++n) refill(n, n);

  int yo[8];  // ring offsets of the y neighbours
#pragma unroll
  for (int n = 1; n <= 4; ++n) {
    yo[n - 1] = (YB ? 4 + yl + n : wrapi(y + n, NLy)) * NLz + z0;
    yo[3 + n] = (YB ? 4 + yl - n : wrapi(y - n, NLy)) * NLz + z0;
  }
  constexpr int NZZ = RZ + 8;  // z runs start at z0-4, z0-4+RZ, ..., z0+4
  int zoff[NZZ / RZ];
#pragma unroll
  for (int m = 0; m < NZZ / RZ; ++m) zoff[m] = (YB ? 4 + yl : y) * NLz + wrapi(z0 + m * RZ - 4, NLz);

  // register queue: in the march step of phase P (plane x = x_beg + 9i + P),
  // plane x-4+m sits in q[(P+m) % 9]; the march is unrolled nine times so the
  // queue rotates by renaming, without register moves.
  T q[9][RZ];
  if (act) {
#pragma unroll
    for (int n = 0; n < 4; ++n) ld_run<R, RZ>(q[n], inb + (size_t)wrapi(x_beg - 4 + n, a.NLx) * NYZ + own);
  }
  R vl[RZ];    // Vloc of the current plane, loaded one plane ahead
  int lq[RZ];  // local sphere indices of the current plane, loaded one plane ahead
#pragma unroll
  for (int r = 0; r < RZ; ++r) { vl[r] = (R)0; lq[r] = -1; }
  if (act && !TB) {
#pragma unroll
    for (int r = 0; r < RZ; ++r) vl[r] = __ldg(a.vloc + (size_t)x_beg * NYZ + own + r);
    if (with_w || do_export) ld_lq<RZ>(lq, a.lqi + (size_t)x_beg * NYZ + own);
  }

  int x = x_beg;
  auto step = [&](auto phase) -> bool {
    constexpr int P = decltype(phase)::value;
    const int j = x - x_beg;
    // ring slot of plane j+k: with one slot per phase (j modulo 9 is P) a constant
    auto slot = [&](int k) -> int { return FIXED ? (P + k) % NR : (j + k) % NR; };
    const int s0 = slot(0);
    cp_async_wait<NR - 6>();  // this thread's copies of planes <= x+4 have landed
    __syncthreads();          // ... and everyone's; the slot of plane x-1 is free
    refill(j + NR - 1, slot(NR - 1));
    const T* pl = ring + (size_t)s0 * RYZ;
    if (act) {
      if constexpr (P == 0) {
        if (j == 0) {
#pragma unroll
          for (int n = 4; n < 8; ++n) lds_run<R, RZ>(q[n], ring + (size_t)(n - 4) * RYZ + own_r);
        }
      }
      lds_run<R, RZ>(q[(P + 8) % 9], ring + (size_t)slot(4) * RYZ + own_r);
      const size_t pbase = (size_t)x * NYZ + own;
      R vln[RZ];
      int lqn[RZ];
#pragma unroll
      for (int r = 0; r < RZ; ++r) { vln[r] = (R)0; lqn[r] = -1; }
      if constexpr (TB) {  // this plane's tables arrived with it (copy group j)
        const R* vs = vtab + (size_t)s0 * TYZ + own_t;
#pragma unroll
        for (int r = 0; r < RZ; ++r) vl[r] = vs[r];
        if (with_w || do_export) {
          const int v2 = *reinterpret_cast<const int*>(lqtab + (size_t)s0 * TYZ + own_t);
          lq[0] = (int)(short)(v2 & 0xffff);
          lq[RZ - 1] = v2 >> 16;
        }
      } else if (x + 1 < x_end) {
#pragma unroll
        for (int r = 0; r < RZ; ++r) vln[r] = __ldg(a.vloc + pbase + NYZ + r);
        if (with_w || do_export) ld_lq<RZ>(lqn, a.lqi + pbase + NYZ);
      }
      T v[RZ], w[RZ], wa[RZ];
#pragma unroll
      for (int r = 0; r < RZ; ++r) { v[r] = mk<R>(0, 0); wa[r] = mk<R>(0, 0); }
      if constexpr (std::is_same<R, float>::value) {
        // z: the values z0-4 .. z0+RZ+3 of plane x (the centre run from the queue), as pairs
        T zv[NZZ];
#pragma unroll
        for (int m = 0; m < NZZ / RZ; ++m) {
          T run[RZ];
          if (m * RZ == 4) {
#pragma unroll
            for (int s2 = 0; s2 < RZ; ++s2) run[s2] = q[(P + 4) % 9][s2];
          } else {
            lds_run<R, RZ>(run, pl + zoff[m]);
          }
#pragma unroll
          for (int s2 = 0; s2 < RZ; ++s2) zv[m * RZ + s2] = run[s2];
        }
#pragma unroll
        for (int n = 1; n <= 4; ++n)
#pragma unroll
          for (int r = 0; r < RZ; ++r) stencil_pair(v[r], wa[r], zv[4 + r + n], zv[4 + r - n], CL(8 + n - 1), CN(8 + n - 1));
      } else {
#pragma unroll
        for (int m = 0; m < NZZ / RZ; ++m) {  // z: each value feeds every point it neighbours, as it arrives
          T run[RZ];
          if (m * RZ == 4) {
#pragma unroll
            for (int s2 = 0; s2 < RZ; ++s2) run[s2] = q[(P + 4) % 9][s2];
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
      // the y terms go to a second accumulator (fixed shapes): two shorter FMA
      // chains (0.469 -> 0.438 ms at 32^3)
      constexpr bool SPLITV = FIXED;
      T vy[RZ];
#pragma unroll
      for (int r = 0; r < RZ; ++r) vy[r] = mk<R>(0, 0);
#pragma unroll
      for (int n = 1; n <= 4; ++n) {  // y
        T rp[RZ], rm[RZ];
        lds_run<R, RZ>(rp, pl + yo[n - 1]);
        lds_run<R, RZ>(rm, pl + yo[3 + n]);
#pragma unroll
        for (int r = 0; r < RZ; ++r) stencil_pair(SPLITV ? vy[r] : v[r], wa[r], rp[r], rm[r], CL(4 + n - 1), CN(4 + n - 1));
      }
#pragma unroll
      for (int r = 0; r < RZ; ++r) { w[r] = kscale(ky, wa[r], w[r]); wa[r] = mk<R>(0, 0); }
#pragma unroll
      for (int n = 1; n <= 4; ++n)  // x: the register queue
#pragma unroll
        for (int r = 0; r < RZ; ++r)
          stencil_pair(v[r], wa[r], q[(P + 4 + n) % 9][r], q[(P + 4 - n) % 9][r], CL(n - 1), CN(n - 1));
#pragma unroll
      for (int r = 0; r < RZ; ++r) w[r] = kscale(kx, wa[r], w[r]);
      if constexpr (SPLITV) {
#pragma unroll
        for (int r = 0; r < RZ; ++r) v[r] = cadd(v[r], vy[r]);
      }

      // plane-relative sphere index lq -> this block's W chunk
      const T* wpl = wring + (size_t)s0 * a.maxpts -
                     (YB ? spo[x * (nyblk + 1) + yb] - spo[x * (nyblk + 1)] : 0);
      T res[RZ];
#pragma unroll
      for (int r = 0; r < RZ; ++r) {
        const T c = q[(P + 4) % 9][r];
        // F = B E + A E - 0.5 v - zI w   (stencil/F90/hpsi.f90:190)
        T f;
        f.x = fma(vl[r] + A, c.x, fma((R)-0.5, v[r].x, w[r].y));
        f.y = fma(vl[r] + A, c.y, fma((R)-0.5, v[r].y, -w[r].x));
        if constexpr (MODE == 1) {  // ttpsi = H tpsi - Vloc tpsi before pseudo_pt (hpsi.f90:131-133)
          a.tt[(size_t)b * a.NL + pbase + r] = mk<R>(fma(-vl[r], c.x, f.x), fma(-vl[r], c.y, f.y));
        }
        if (with_w && lq[r] >= 0) f = cadd(f, wpl[lq[r]]);  // + pseudo_pt scatter (hpsi.f90:203-206)
        res[r] = f;
      }
      if constexpr (MODE == 2) {  // one Taylor stage: out = in + c H in
#pragma unroll
        for (int r = 0; r < RZ; ++r) res[r] = cfma(a.zf, res[r], q[(P + 4) % 9][r]);
      }
      st_run<R, RZ>(a.out + (size_t)b * a.NL + pbase, res);
      if (do_export) {  // the output at the sphere points, for the next projections
        const int q0 = YB ? spo[x * (nyblk + 1)] : spo[x];
#pragma unroll
        for (int r = 0; r < RZ; ++r)
          if (lq[r] >= 0) Sb[q0 + lq[r]] = res[r];
      }
      if constexpr (!TB) {
#pragma unroll
        for (int r = 0; r < RZ; ++r) { vl[r] = vln[r]; lq[r] = lqn[r]; }
      }
    }
    ++x;
    return x < x_end;
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
  cp_async_wait<0>();
}

// ------------------------------------------------------------- launch ---
// Vloc and sphere-index tables through the ring: two-point form, when both
// precisions' rings still fit in shared memory with them
static bool pass_tables(const System& s, int RZ) {
  if (RZ != 2 || !s.pass_tab) return false;
  const int NYB = s.nyblk > 1 ? s.NYB : s.NLy;
  for (int pr = 0; pr < 2; ++pr)
    if (pass_smem_bytes(pr, s.NLy, s.NLz, s.maxpts, true, s.NLx, s.nyblk, NYB, true) > 227 * 1024) return false;
  return true;
}

// plane shapes with a compile-time form (complex(4), table form): the 16^3, 20^3
// and 32^3 grids and the 16x16x32 supercell without y-blocks, 48x48 planes in
// three y-blocks of 16 rows (the 48^3 grid)
static int fixed_shape(int NLy, int NLz, int nyblk, int NYB) {
  if (nyblk > 1) return (NLy == 48 && NLz == 48 && nyblk == 3 && NYB == 16) ? 5 : 0;
  if (NLy == 32 && NLz == 32) return 1;
  if (NLy == 16 && NLz == 16) return 2;
  if (NLy == 16 && NLz == 32) return 3;
  if (NLy == 20 && NLz == 20) return 4;
  return 0;
}

template <typename R, int RZ, int MODE>
static void (*pass_kernel(bool yb, bool tb, int shape))(const PassArgs<R>) {
  if constexpr (RZ == 2 && std::is_same<R, float>::value) {
    if (tb && !yb) {
      switch (shape) {
        case 1: return k_hpsi_pass<R, RZ, MODE, false, true, 32, 32>;
        case 2: return k_hpsi_pass<R, RZ, MODE, false, true, 16, 16>;
        case 3: return k_hpsi_pass<R, RZ, MODE, false, true, 16, 32>;
        case 4: return k_hpsi_pass<R, RZ, MODE, false, true, 20, 20>;
        default: break;
      }
    }
    if (tb && yb && shape == 5) return k_hpsi_pass<R, RZ, MODE, true, true, 48, 48, 16>;
  }
  if constexpr (RZ == 2) {
    if (tb) return yb ? k_hpsi_pass<R, RZ, MODE, true, true> : k_hpsi_pass<R, RZ, MODE, false, true>;
  }
  return yb ? k_hpsi_pass<R, RZ, MODE, true, false> : k_hpsi_pass<R, RZ, MODE, false, false>;
}

// the compile-time shape the pass uses for this system and precision (0: none);
// its 9-plane ring must fit in shared memory
template <typename R, int RZ>
static int pass_shape(const System& s, bool tb) {
  if (!std::is_same<R, float>::value || RZ != 2 || !tb || !s.pass_fixed) return 0;
  const int sh = fixed_shape(s.NLy, s.NLz, s.nyblk, s.NYB);
  const int nyb = s.nyblk > 1 ? s.NYB : s.NLy;
  if (sh && pass_smem_bytes(SGPU_PREC_C64, s.NLy, s.NLz, s.maxpts, true, s.NLx, s.nyblk, nyb, true, 9) > 227 * 1024)
    return 0;
  return sh;
}

template <typename R, int RZ, int MODE>
static cudaError_t launch_pass_t(const System& s, const PassIO& io, int o_beg, int nb, int nbk) {
  PassArgs<R> a;
  a.in = (const C2<R>*)io.in;
  a.out = (C2<R>*)io.out;
  a.tt = (C2<R>*)io.tt;
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
      a.lapt[4 * d + n] = (R)s.lap[d][n + 1];
      a.nabc[4 * d + n] = (R)s.nab[d][n + 1];
      a.cl2[4 * d + n] = make_float2((float)s.lap[d][n + 1], (float)s.lap[d][n + 1]);
      a.cn2[4 * d + n] = make_float2((float)s.nab[d][n + 1], (float)s.nab[d][n + 1]);
    }
  a.sp_off = s.sp_off;
  a.nyblk = s.nyblk;
  a.NYB = s.nyblk > 1 ? s.NYB : s.NLy;
  a.sp_blk = s.sp_blk;
  a.lqi = s.lqi;
  a.W = (const C2<R>*)io.W;
  a.S = (C2<R>*)io.S;
  a.nsp = s.nsp;
  a.maxpts = s.maxpts;
  a.zf = mk<R>((R)io.zc[0], (R)io.zc[1]);
  const int nthr = a.NYB * (s.NLz / RZ);
  const int block = ((nthr + 31) / 32) * 32;
  const bool tb = pass_tables(s, RZ);
  const int shape = pass_shape<R, RZ>(s, tb);
  const size_t smem = pass_smem_bytes(std::is_same<R, float>::value ? SGPU_PREC_C64 : SGPU_PREC_C128, s.NLy, s.NLz,
                                      s.maxpts, io.W != nullptr, s.NLx, s.nyblk, a.NYB, tb, shape ? 9 : 0);
  auto kern = pass_kernel<R, RZ, MODE>(s.nyblk > 1, tb, shape);
  if (smem > 48 * 1024) {
    // set outside stream capture (prepare_pass sets it before a capture)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s.stream, &cs);
    if (e != cudaSuccess) return e;
    if (cs == cudaStreamCaptureStatusNone) {
      e = raise_smem_limit((const void*)kern, smem);
      if (e != cudaSuccess) return e;
    }
  }
  dim3 grid(nb * s.nyblk, (s.NLx + a.SX - 1) / a.SX);
  kern<<<grid, block, smem, s.launch_stream()>>>(a);
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

template <typename R, int RZ>
static cudaError_t prepare_pass_rz(const System& s) {
  const bool yb = s.nyblk > 1, tb = pass_tables(s, RZ);
  const int shape = pass_shape<R, RZ>(s, tb);
  const size_t smem = pass_smem_bytes(std::is_same<R, float>::value ? SGPU_PREC_C64 : SGPU_PREC_C128, s.NLy, s.NLz,
                                      s.maxpts, true, s.NLx, s.nyblk, yb ? s.NYB : s.NLy, tb, shape ? 9 : 0);
  if (smem <= 48 * 1024) return cudaSuccess;
  cudaError_t e;
  if ((e = raise_smem_limit((const void*)pass_kernel<R, RZ, 0>(yb, tb, shape), smem)))
    return e;
  if ((e = raise_smem_limit((const void*)pass_kernel<R, RZ, 1>(yb, tb, shape), smem)))
    return e;
  return raise_smem_limit((const void*)pass_kernel<R, RZ, 2>(yb, tb, shape), smem);
}

cudaError_t prepare_pass(const System& s) {
  const bool rz2 = (s.NLz % 2) == 0;
  cudaError_t e = rz2 ? prepare_pass_rz<float, 2>(s) : prepare_pass_rz<float, 1>(s);
  if (e != cudaSuccess) return e;
  return rz2 ? prepare_pass_rz<double, 2>(s) : prepare_pass_rz<double, 1>(s);
}

int pass_block_threads(int NLy, int NLz) {  // without y-blocks
  const int rz = (NLz % 2) == 0 ? 2 : 1;
  return ((NLy * (NLz / rz) + 31) / 32) * 32;
}

}  // namespace sgpu
