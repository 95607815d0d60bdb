// Kleinman-Bylander projections U, the KB field W at the sphere points and the
// projector update for sm_100a, plus the precision conversions.  The
// Hamiltonian pass itself is in k_pass.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "sgpu_internal.cuh"

namespace sgpu {

// ----------------------------------------------------------------- uVpsi ---
// U[b][ilma] = Hxyz (iuV) sum_j conj(zproj(j,ilma,k)) in_b(J(j))  (hpsi.f90:188-193)
//
// A batched dense contraction on the FP64 tensor pipe (mma.sync m8n8k4 f64).
// For one k-point and one projector item (an atom with <= 4 projectors) the
// complex contraction over the atom's points j is the real product
//     C[8][2nb] = A[8][K] B[K][2nb],
//     A rows 0-3 = Re zproj(j, p), rows 4-7 = Im zproj(j, p)      (p = item projector)
//     B cols 2b, 2b+1 = Re, Im in_b(J(j))
// from which U_re[p][b] = C[p][2b] + C[p+4][2b+1] and U_im[p][b] = C[p][2b+1] - C[p+4][2b].
// A CTA owns one 8x8 tile of C: 4 bands of one k-point ("band quad") and one
// item; its UM_SPLIT warps (a tuning parameter: 1, 2, 4 or 8) split K (the
// atom's points, in chunks of 32) and
// their tiles are added in warp order, so the sum order is fixed
// (deterministic).  Orbital values are converted to FP64 before the MMA: the
// contraction is FP64 for either orbital precision.
constexpr int UM_WARPS = 4;   // band quads per CTA (KB field)
constexpr int UM_UNROLL = 8;  // MMAs (of 4 points) per batch of loads: 32 points

__device__ __forceinline__ void mma_f64_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <typename R, int UM_SPLIT>
__global__ void __launch_bounds__(32 * UM_SPLIT) k_uvpsi(const C2<R>* __restrict__ in, int ld_in, int o_beg, int nb,
                                                        int nbk, int kl0, int nquad_k,
                                                        const double2* __restrict__ zproj, int Nlma, int Nps,
                                                        const int* __restrict__ idx, const int* __restrict__ atom_off,
                                                        const int4* __restrict__ items, const int* __restrict__ lma_list,
                                                        const int* __restrict__ iuV, double scale, int use_iuv,
                                                        double2* __restrict__ U) {
  __shared__ double2 part[UM_SPLIT][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = blockIdx.x;
  const int kq = quad / nquad_k;
  const int kl = kl0 + kq;
  const int b_first = kl * nbk + 4 * (quad - kq * nquad_k);  // absolute orbital of the quad's first band
  const int o_lo = max(o_beg, kl * nbk), o_hi = min(o_beg + nb, (kl + 1) * nbk);
  const int4 item = items[blockIdx.y];
  const int a = item.x, l0 = item.y, np = item.z;
  const int p0 = atom_off[a], mps = atom_off[a + 1] - p0;

  // this lane's B element: row (point) lane%4, column n = lane/4 -> band n/2, part n%2
  const int krow = lane & 3, n = lane >> 2;
  const int ob = b_first + (n >> 1);
  const bool bvalid = ob >= o_lo && ob < o_hi;
  const C2<R>* src = in + (size_t)(bvalid ? ob - o_beg : 0) * ld_in;
  const int bpart = n & 1;
  // this lane's A element: row r = lane/4 -> projector r%4, part r/4; column (point) lane%4
  const int pa = n & 3;
  const bool avalid = pa < np;
  const double* zrow =
      reinterpret_cast<const double*>(zproj + ((size_t)kl * Nlma + (avalid ? lma_list[l0 + pa] : 0)) * Nps) + (n >> 2);

  double c0 = 0.0, c1 = 0.0, e0 = 0.0, e1 = 0.0;  // two accumulator tiles (even / odd MMAs)
  constexpr int PTS = 4 * UM_UNROLL;              // points per chunk (one per lane for the index load)
  constexpr int STRIDE = PTS * UM_SPLIT;
  int j0 = warp * PTS;
  int gl = j0 + lane < mps ? __ldg(idx + p0 + j0 + lane) : 0;
  for (; j0 < mps; j0 += STRIDE) {
    // the next chunk's point indices are loaded one chunk ahead
    const int jn = j0 + STRIDE;
    const int nl = jn + lane < mps ? __ldg(idx + p0 + jn + lane) : 0;
    double av[UM_UNROLL], bv[UM_UNROLL];
#pragma unroll
    for (int u = 0; u < UM_UNROLL; ++u) {
      const int j = j0 + 4 * u + krow;
      const int g = __shfl_sync(0xffffffffu, gl, 4 * u + krow);
      av[u] = 0.0;
      bv[u] = 0.0;
      if (j < mps) {
        if (avalid) av[u] = __ldg(zrow + 2 * (size_t)j);
        if (bvalid) {
          const C2<R> v = src[g];
          bv[u] = bpart ? (double)v.y : (double)v.x;
        }
      }
    }
#pragma unroll
    for (int u = 0; u < UM_UNROLL; u += 2) {
      mma_f64_8x8x4(c0, c1, av[u], bv[u]);
      mma_f64_8x8x4(e0, e1, av[u + 1], bv[u + 1]);
    }
    gl = nl;
  }
  part[warp][lane] = make_double2(c0 + e0, c1 + e1);
  __syncthreads();
  if (warp == 0) {
    double2 t = part[0][lane];
#pragma unroll
    for (int w = 1; w < UM_SPLIT; ++w) {
      t.x += part[w][lane].x;
      t.y += part[w][lane].y;
    }
    // lane holds C[r = lane/4][2*(lane%4) + i]; the Im-zproj rows r+4 sit 16 lanes up
    const double d0 = __shfl_down_sync(0xffffffffu, t.x, 16);
    const double d1 = __shfl_down_sync(0xffffffffu, t.y, 16);
    if (lane < 16) {
      const int p = lane >> 2, o = b_first + (lane & 3);
      if (p < np && o >= o_lo && o < o_hi) {
        const int ilma = lma_list[l0 + p];
        const double f = scale * (use_iuv ? (double)iuV[ilma] : 1.0);
        U[(size_t)(o - o_beg) * Nlma + ilma] = make_double2((t.x + d1) * f, (t.y - d0) * f);
      }
    }
  }
}

template <typename R, int SPLIT>
static cudaError_t launch_uvpsi_split(const System& s, const void* in, int ld_in, const int* idx, int o_beg, int nb,
                                      int nbk, bool scale_iuv) {
  const int kl0 = o_beg / nbk, kl1 = (o_beg + nb - 1) / nbk;
  const int nquad_k = (nbk + 3) / 4;
  const int nquad = (kl1 - kl0 + 1) * nquad_k;
  dim3 grid(nquad, s.nitems);
  k_uvpsi<R, SPLIT><<<grid, 32 * SPLIT, 0, s.launch_stream()>>>((const C2<R>*)in, ld_in, o_beg, nb, nbk, kl0, nquad_k,
                                                                 s.zproj64, s.Nlma, s.Nps, idx, s.atom_off, s.items,
                                                                 s.lma_list, s.iuV_d, s.Hxyz, scale_iuv ? 1 : 0, s.U);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t launch_uvpsi_t(const System& s, const void* in, int ld_in, const int* idx, int o_beg, int nb,
                                  int nbk, bool scale_iuv) {
  switch (s.um_split) {
    case 1: return launch_uvpsi_split<R, 1>(s, in, ld_in, idx, o_beg, nb, nbk, scale_iuv);
    case 2: return launch_uvpsi_split<R, 2>(s, in, ld_in, idx, o_beg, nb, nbk, scale_iuv);
    case 8: return launch_uvpsi_split<R, 8>(s, in, ld_in, idx, o_beg, nb, nbk, scale_iuv);
    default: return launch_uvpsi_split<R, 4>(s, in, ld_in, idx, o_beg, nb, nbk, scale_iuv);
  }
}

cudaError_t launch_uvpsi(const System& s, const void* in, int o_beg, int nb, int nbk, bool scale_iuv, int prec) {
  if (s.Nlma == 0 || nb == 0) return cudaSuccess;
  if ((prec < 0 ? s.prec : prec) == SGPU_PREC_C64)
    return launch_uvpsi_t<float>(s, in, s.NL, s.idx_proj, o_beg, nb, nbk, scale_iuv);
  return launch_uvpsi_t<double>(s, in, s.NL, s.idx_proj, o_beg, nb, nbk, scale_iuv);
}

cudaError_t launch_uvpsi_from_S(const System& s, const void* S, int o_beg, int nb, int nbk, bool scale_iuv) {
  if (s.Nlma == 0 || nb == 0) return cudaSuccess;
  if (s.prec == SGPU_PREC_C64) return launch_uvpsi_t<float>(s, S, s.nsp, s.qmap, o_beg, nb, nbk, scale_iuv);
  return launch_uvpsi_t<double>(s, S, s.nsp, s.qmap, o_beg, nb, nbk, scale_iuv);
}

// ------------------------------------------------------------- KB field ---
// W[b][q] = sum over the (ilma, j) entries of sphere point q of zproj(j,ilma,k) U[b][ilma]
// (the dpseudo of pseudo_pt, common/hpsi.f90:194-200, summed per grid point).
//
// Points inside exactly one projector item (the usual case: non-overlapping
// spheres, <= 4 projectors per atom) go through the FP64 tensor pipe: for one
// k-point, item and band quad the field at 8 points is the real product
//     C[8][8] = A[8][8] B[8][8],
//     A[m][p] = Re zproj(j_m, p), A[m][4+p] = Im zproj(j_m, p),
//     B[p][2b] = Re U[b][p], B[p][2b+1] = Im U[b][p], B[4+p][2b] = -Im U[b][p], B[4+p][2b+1] = Re U[b][p],
// two m8n8k4 MMAs per tile of 8 points; B stays in registers for the warp's
// whole sweep over the atom.  Points that lie in several items are summed
// entry by entry in a fixed order by k_kbfield_multi, so every W element has
// one writer and the result is deterministic.
template <typename R>
__global__ void __launch_bounds__(32 * UM_WARPS) k_kbfield(const double2* __restrict__ U, int o_beg, int nb, int nbk,
                                                          int kl0, int nquad_k, int nquad,
                                                          const double2* __restrict__ zproj, int Nlma, int Nps,
                                                          const int* __restrict__ kbq, const int* __restrict__ atom_off,
                                                          const int4* __restrict__ items,
                                                          const int* __restrict__ lma_list, int nsp,
                                                          C2<R>* __restrict__ W) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = blockIdx.x * UM_WARPS + warp;
  if (quad >= nquad) return;  // whole warp leaves; no block-wide synchronisation follows
  const int kq = quad / nquad_k;
  const int kl = kl0 + kq;
  const int b_first = kl * nbk + 4 * (quad - kq * nquad_k);
  const int o_lo = max(o_beg, kl * nbk), o_hi = min(o_beg + nb, (kl + 1) * nbk);
  const int4 item = items[blockIdx.y];
  const int a = item.x, l0 = item.y, np = item.z;
  const int p0 = atom_off[a], mps = atom_off[a + 1] - p0;

  // B fragment (row p = lane%4, column n = lane/4 -> band n/2, part n%2): constant
  const int p = lane & 3, n = lane >> 2;
  const int ob = b_first + (n >> 1);
  double2 u = make_double2(0.0, 0.0);
  if (p < np && ob >= o_lo && ob < o_hi) u = U[(size_t)(ob - o_beg) * Nlma + lma_list[l0 + p]];
  const double bre = (n & 1) ? u.y : u.x;   // rows of Re zproj
  const double bim = (n & 1) ? u.x : -u.y;  // rows of Im zproj
  // A fragment (row m = lane/4 -> point, column p = lane%4); C: row m, columns 2*(lane%4)+{0,1}
  const double2* zp = zproj + ((size_t)kl * Nlma + (p < np ? lma_list[l0 + p] : 0)) * Nps;
  const int oc = b_first + p;  // the orbital of this lane's C elements
  const bool cvalid = oc >= o_lo && oc < o_hi;
  C2<R>* Wb = W + (size_t)(cvalid ? oc - o_beg : 0) * nsp;
  constexpr int T = 8;  // tiles of 8 points per batch of loads
  for (int j0 = 0; j0 < mps; j0 += 8 * T) {
    double2 z[T];
    int q[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
      const int j = j0 + 8 * t + n;
      z[t] = make_double2(0.0, 0.0);
      q[t] = -1;
      if (j < mps) {
        if (p < np) z[t] = __ldg(zp + j);
        q[t] = __ldg(kbq + p0 + j);
      }
    }
#pragma unroll
    for (int t = 0; t < T; ++t) {
      double c0 = 0.0, c1 = 0.0;
      mma_f64_8x8x4(c0, c1, z[t].x, bre);
      mma_f64_8x8x4(c0, c1, z[t].y, bim);
      if (cvalid && q[t] >= 0) Wb[q[t]] = mk<R>((R)c0, (R)c1);
    }
  }
}

// Points in several projector items: one thread per (listed point, orbital
// group), entries summed in their table order.
constexpr int KU = 4;

__device__ __forceinline__ int kb_entry(const int4& ra, const int4& rb, const int* cont, int e) {
  if (e < 4) return e == 0 ? ra.z : (e == 1 ? ra.w : (e == 2 ? rb.x : rb.y));
  return __ldg(cont + rb.z + (e - 4));
}

template <typename R>
__global__ void __launch_bounds__(256) k_kbfield_multi(const double2* __restrict__ U, int nb, int o_beg, int nbk,
                                                       const double2* __restrict__ zproj, int Nlma, int Nps,
                                                       const int4* __restrict__ rec, const int* __restrict__ cont,
                                                       const int* __restrict__ qlist, int nq, int nsp,
                                                       C2<R>* __restrict__ W) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int b0 = blockIdx.y * KU;
  if (t >= nq) return;
  const int q = qlist[t];
  const int4 ra = __ldg(rec + 2 * (size_t)q), rb = __ldg(rec + 2 * (size_t)q + 1);
  const int ne = ra.y + rb.w;
#pragma unroll
  for (int u = 0; u < KU; ++u) {
    if (b0 + u >= nb) break;
    const int kl = (o_beg + b0 + u) / nbk;
    double2 acc = make_double2(0.0, 0.0);
    for (int e = 0; e < ne; ++e) {
      const int en = kb_entry(ra, rb, cont, e);
      const int ilma = en >> 16;
      const double2 z = __ldg(zproj + ((size_t)kl * Nlma + ilma) * Nps + (en & 0xffff));
      const double2 uu = __ldg(U + (size_t)(b0 + u) * Nlma + ilma);
      acc = cfma(z, uu, acc);
    }
    W[(size_t)(b0 + u) * nsp + q] = mk<R>((R)acc.x, (R)acc.y);
  }
}

template <typename R>
static cudaError_t launch_kbfield_t(const System& s, int o_beg, int nb, int nbk, void* W) {
  const int kl0 = o_beg / nbk, kl1 = (o_beg + nb - 1) / nbk;
  const int nquad_k = (nbk + 3) / 4;
  const int nquad = (kl1 - kl0 + 1) * nquad_k;
  dim3 grid((nquad + UM_WARPS - 1) / UM_WARPS, s.nitems);
  k_kbfield<R><<<grid, 32 * UM_WARPS, 0, s.launch_stream()>>>(s.U, o_beg, nb, nbk, kl0, nquad_k, nquad, s.zproj64,
                                                               s.Nlma, s.Nps, s.kbq, s.atom_off, s.items, s.lma_list,
                                                               s.nsp, (C2<R>*)W);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || s.n_multi == 0) return e;
  dim3 g2((s.n_multi + 255) / 256, (nb + KU - 1) / KU);
  k_kbfield_multi<R><<<g2, 256, 0, s.launch_stream()>>>(s.U, nb, o_beg, nbk, s.zproj64, s.Nlma, s.Nps, s.rec, s.cont,
                                                         s.kb_multi, s.n_multi, s.nsp, (C2<R>*)W);
  return cudaGetLastError();
}

// ------------------------------------------------ projections + KB field ---
// One kernel for U and W of the points inside exactly one item (the KB term
// of one H application): a CTA owns (band quad, item); its UM_SPLIT warps
// first build the 8x8 projection tile over the atom's points (as k_uvpsi,
// summed in warp order), keep U in shared memory (and store it for the
// entry-wise kernel of multi-item points), then sweep the atom's points again
// for W = zproj U (as k_kbfield), so U never makes a round trip through global
// memory between two launches.
template <typename R, int UM_SPLIT>
__global__ void __launch_bounds__(32 * UM_SPLIT) k_kb_fused(const C2<R>* __restrict__ in, int ld_in, int o_beg, int nb,
                                                           int nbk, int kl0, int nquad_k,
                                                           const double2* __restrict__ zproj, int Nlma, int Nps,
                                                           const int* __restrict__ idx, const int* __restrict__ kbq,
                                                           const int* __restrict__ atom_off,
                                                           const int4* __restrict__ items,
                                                           const int* __restrict__ lma_list, const int* __restrict__ iuV,
                                                           double scale, double2* __restrict__ U, int nsp,
                                                           C2<R>* __restrict__ W) {
  __shared__ double2 part[UM_SPLIT][32];
  __shared__ double2 Us[4][4];  // [projector][band of the quad]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = blockIdx.x;
  const int kq = quad / nquad_k;
  const int kl = kl0 + kq;
  const int b_first = kl * nbk + 4 * (quad - kq * nquad_k);
  const int o_lo = max(o_beg, kl * nbk), o_hi = min(o_beg + nb, (kl + 1) * nbk);
  const int4 item = items[blockIdx.y];
  const int a = item.x, l0 = item.y, np = item.z;
  const int p0 = atom_off[a], mps = atom_off[a + 1] - p0;
  const int krow = lane & 3, n = lane >> 2;

  // ---- phase 1: U tile (rows: Re/Im zproj of the item's projectors; columns: Re/Im of 4 bands)
  {
    const int ob = b_first + (n >> 1);
    const bool bvalid = ob >= o_lo && ob < o_hi;
    const C2<R>* src = in + (size_t)(bvalid ? ob - o_beg : 0) * ld_in;
    const int bpart = n & 1;
    const int pa = n & 3;
    const bool avalid = pa < np;
    const double* zrow =
        reinterpret_cast<const double*>(zproj + ((size_t)kl * Nlma + (avalid ? lma_list[l0 + pa] : 0)) * Nps) + (n >> 2);
    double c0 = 0.0, c1 = 0.0, e0 = 0.0, e1 = 0.0;
    constexpr int PTS = 4 * UM_UNROLL;
    constexpr int STRIDE = PTS * UM_SPLIT;
    int j0 = warp * PTS;
    int gl = j0 + lane < mps ? __ldg(idx + p0 + j0 + lane) : 0;
    for (; j0 < mps; j0 += STRIDE) {
      const int jn = j0 + STRIDE;
      const int nl = jn + lane < mps ? __ldg(idx + p0 + jn + lane) : 0;
      double av[UM_UNROLL], bv[UM_UNROLL];
#pragma unroll
      for (int u = 0; u < UM_UNROLL; ++u) {
        const int j = j0 + 4 * u + krow;
        const int g = __shfl_sync(0xffffffffu, gl, 4 * u + krow);
        av[u] = 0.0;
        bv[u] = 0.0;
        if (j < mps) {
          if (avalid) av[u] = __ldg(zrow + 2 * (size_t)j);
          if (bvalid) {
            const C2<R> v = src[g];
            bv[u] = bpart ? (double)v.y : (double)v.x;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < UM_UNROLL; u += 2) {
        mma_f64_8x8x4(c0, c1, av[u], bv[u]);
        mma_f64_8x8x4(e0, e1, av[u + 1], bv[u + 1]);
      }
      gl = nl;
    }
    part[warp][lane] = make_double2(c0 + e0, c1 + e1);
  }
  __syncthreads();
  if (warp == 0) {
    double2 t = part[0][lane];
#pragma unroll
    for (int w = 1; w < UM_SPLIT; ++w) {
      t.x += part[w][lane].x;
      t.y += part[w][lane].y;
    }
    const double d0 = __shfl_down_sync(0xffffffffu, t.x, 16);
    const double d1 = __shfl_down_sync(0xffffffffu, t.y, 16);
    if (lane < 16) {
      const int p = lane >> 2, bq = lane & 3, o = b_first + bq;
      double2 u = make_double2(0.0, 0.0);
      if (p < np && o >= o_lo && o < o_hi) {
        const int ilma = lma_list[l0 + p];
        const double f = scale * (double)iuV[ilma];
        u = make_double2((t.x + d1) * f, (t.y - d0) * f);
        U[(size_t)(o - o_beg) * Nlma + ilma] = u;
      }
      Us[p][bq] = u;
    }
  }
  __syncthreads();

  // ---- phase 2: W at the atom's single-item points, 8 points per pair of MMAs
  {
    const int p = krow;  // B row / A column: projector
    const double2 u = Us[p][n >> 1];
    const double bre = (n & 1) ? u.y : u.x;   // rows of Re zproj
    const double bim = (n & 1) ? u.x : -u.y;  // rows of Im zproj
    const double2* zp = zproj + ((size_t)kl * Nlma + (p < np ? lma_list[l0 + p] : 0)) * Nps;
    const int oc = b_first + p;  // the orbital of this lane's C elements (C column pair 2p, 2p+1)
    const bool cvalid = oc >= o_lo && oc < o_hi;
    C2<R>* Wb = W + (size_t)(cvalid ? oc - o_beg : 0) * nsp;
    constexpr int T = 8;
    for (int j0 = warp * 8 * T; j0 < mps; j0 += UM_SPLIT * 8 * T) {
      double2 z[T];
      int q[T];
#pragma unroll
      for (int t = 0; t < T; ++t) {
        const int j = j0 + 8 * t + n;
        z[t] = make_double2(0.0, 0.0);
        q[t] = -1;
        if (j < mps) {
          if (p < np) z[t] = __ldg(zp + j);
          q[t] = __ldg(kbq + p0 + j);
        }
      }
#pragma unroll
      for (int t = 0; t < T; ++t) {
        double c0 = 0.0, c1 = 0.0;
        mma_f64_8x8x4(c0, c1, z[t].x, bre);
        mma_f64_8x8x4(c0, c1, z[t].y, bim);
        if (cvalid && q[t] >= 0) Wb[q[t]] = mk<R>((R)c0, (R)c1);
      }
    }
  }
}

template <typename R, int SPLIT>
static cudaError_t launch_kb_fused_split(const System& s, const void* in, int ld_in, const int* idx, int o_beg, int nb,
                                         int nbk, void* W) {
  const int kl0 = o_beg / nbk, kl1 = (o_beg + nb - 1) / nbk;
  const int nquad_k = (nbk + 3) / 4;
  const int nquad = (kl1 - kl0 + 1) * nquad_k;
  dim3 grid(nquad, s.nitems);
  k_kb_fused<R, SPLIT><<<grid, 32 * SPLIT, 0, s.launch_stream()>>>(
      (const C2<R>*)in, ld_in, o_beg, nb, nbk, kl0, nquad_k, s.zproj64, s.Nlma, s.Nps, idx, s.kbq, s.atom_off, s.items,
      s.lma_list, s.iuV_d, s.Hxyz, s.U, s.nsp, (C2<R>*)W);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || s.n_multi == 0) return e;
  dim3 g2((s.n_multi + 255) / 256, (nb + KU - 1) / KU);
  k_kbfield_multi<R><<<g2, 256, 0, s.launch_stream()>>>(s.U, nb, o_beg, nbk, s.zproj64, s.Nlma, s.Nps, s.rec, s.cont,
                                                         s.kb_multi, s.n_multi, s.nsp, (C2<R>*)W);
  return cudaGetLastError();
}

// ------------------------------------------------------------ KB tile ---
// Projections and KB field of one projector item for a group of up to 32
// bands of one k-point per CTA: U = Hxyz iuV sum_j conj(zproj) in(J(j)), then
// W = zproj U at the item's single-item points (hpsi.f90:188-206), the
// contractions on the FP64 tensor pipe as in k_uvpsi / k_kbfield.  The atom's
// sphere values (gathered by idx) and its zproj rows stream through a
// three-stage shared-memory pipeline of cp.async copies in chunks of CP points,
// so several chunks of every CTA are in flight; zproj is read from L2 twice per
// (k-point, item, band group) instead of twice per band quad.  KBT_KS warps
// share each band quad (an 8x8 C tile): they split every chunk's points and
// their tiles are added in warp order, so the sums are deterministic.
constexpr int KBT_WARPS = 8;               // band quads per CTA
constexpr int KBT_KS = 2;                  // warps per band quad
constexpr int KBT_BANDS = 4 * KBT_WARPS;   // bands per CTA
constexpr int KBT_NS = 4;                  // pipeline stages
template <typename R>
struct KbtGeom {
  static constexpr bool F = std::is_same<R, float>::value;
  static constexpr int CP = F ? 32 : 16;          // points per chunk
  static constexpr int SROW = CP + (F ? 4 : 2);   // padded band row of a chunk
  static constexpr int ZROW = CP + 2;             // padded projector row of a chunk
  static size_t smem(int Nps) {
    return sizeof(C2<R>) * (size_t)KBT_NS * KBT_BANDS * SROW + sizeof(double2) * (size_t)KBT_NS * 4 * ZROW +
           2 * sizeof(int) * (size_t)Nps;
  }
};

// UONLY: phase 1 alone over the chunk range of split blockIdx.z of nsplit, the
// unscaled sums written to Up[split][o - o_beg][ilma] (k_kb_w adds the splits
// in order, scales, and writes U and W).
template <typename R, bool UONLY = false>
__global__ void __launch_bounds__(32 * KBT_WARPS * KBT_KS) k_kb_tile(const C2<R>* __restrict__ in, int ld_in, int o_beg, int nb,
                                                          int nbk, int kl0, int ngrp, const double2* __restrict__ zproj,
                                                          int Nlma, int Nps, const int* __restrict__ idx,
                                                          const int* __restrict__ kbq, const int* __restrict__ atom_off,
                                                          const int4* __restrict__ items,
                                                          const int* __restrict__ lma_list, const int* __restrict__ iuV,
                                                          double scale, double2* __restrict__ U, int nsp,
                                                          C2<R>* __restrict__ W, int nsplit = 1,
                                                          double2* __restrict__ Up = nullptr) {
  using T = C2<R>;
  constexpr int CP = KbtGeom<R>::CP, SROW = KbtGeom<R>::SROW, ZROW = KbtGeom<R>::ZROW;
  constexpr int NT = 32 * KBT_WARPS * KBT_KS;
  static_assert(NT % CP == 0 && 4 * CP <= NT, "chunk layout: each thread copies one point of several bands");
  static_assert((CP / 4) % (2 * KBT_KS) == 0 && (CP / 8) % KBT_KS == 0, "chunk points split evenly over a quad's warps");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Sb = reinterpret_cast<T*>(smem_raw);                                          // [NS][BANDS][SROW]
  double2* Zb = reinterpret_cast<double2*>(Sb + (size_t)KBT_NS * KBT_BANDS * SROW);  // [NS][4][ZROW]
  int* ixs = reinterpret_cast<int*>(Zb + (size_t)KBT_NS * 4 * ZROW);                // [mps] gather index
  int* kqs = ixs + Nps;                                                              // [mps] W index (-1: multi)
  __shared__ double2 Us[KBT_WARPS][4][4];  // [quad][projector][band]
  __shared__ double2 part[KBT_KS][KBT_WARPS][32];

  const int t = threadIdx.x, lane = t & 31;
  const int warp = (t >> 5) % KBT_WARPS, ks = (t >> 5) / KBT_WARPS;  // band quad, share of the points
  const int kq = blockIdx.x / ngrp, grp = blockIdx.x - kq * ngrp;
  const int kl = kl0 + kq;
  const int o_lo = max(o_beg, kl * nbk + grp * KBT_BANDS);
  const int o_hi = min(min(o_beg + nb, (kl + 1) * nbk), kl * nbk + (grp + 1) * KBT_BANDS);
  if (o_lo >= o_hi) return;  // whole CTA leaves together
  const int nbq = o_hi - o_lo;
  const int4 item = items[blockIdx.y];
  const int a = item.x, l0 = item.y, np = item.z;
  const int p0 = atom_off[a], mps = atom_off[a + 1] - p0;
  const int nch_all = (mps + CP - 1) / CP;
  // chunks [cbeg, nch) of this CTA (UONLY: its split's range, possibly empty)
  const int cps = UONLY ? (nch_all + nsplit - 1) / nsplit : nch_all;
  const int cbeg = UONLY ? min(nch_all, (int)blockIdx.z * cps) : 0;
  const int nch = UONLY ? min(nch_all, cbeg + cps) : nch_all;
  for (int j = cbeg * CP + t; j < min(mps, nch * CP); j += NT) {
    ixs[j] = __ldg(idx + p0 + j);
    if (!UONLY) kqs[j] = __ldg(kbq + p0 + j);
  }
  // the copy role of this thread: point jj of a chunk, for bands bc, bc + NT/CP, ...
  // and (t < 4 CP) projector pz of the zproj rows
  const int jj = t % CP, bc = t / CP;
  const int pz = t / CP;
  const double2* zsrc = (t < 4 * CP && pz < np) ? zproj + ((size_t)kl * Nlma + lma_list[l0 + pz]) * Nps : nullptr;
  __syncthreads();

  auto issue = [&](int c, bool with_s) {  // chunk c into stage c % NS
    if (c < nch) {
      const int s = c % KBT_NS;
      const int j = c * CP + jj;
      if (with_s) {
        T* sd = Sb + (size_t)s * KBT_BANDS * SROW + jj;
        const int g = j < mps ? ixs[j] : 0;
#pragma unroll
        for (int b = bc; b < KBT_BANDS; b += NT / CP) {
          if (b < nbq && j < mps) {
            const T* src = in + (size_t)(o_lo + b - o_beg) * ld_in + g;
            if constexpr (sizeof(T) == 8) cp_async8(sd + b * SROW, src); else cp_async16(sd + b * SROW, src);
          } else {
            sd[b * SROW] = mk<R>(0, 0);
          }
        }
      }
      if (t < 4 * CP) {
        double2* zd = Zb + (size_t)s * 4 * ZROW + pz * ZROW + jj;
        if (zsrc && j < mps) cp_async16(zd, zsrc + j); else *zd = make_double2(0.0, 0.0);
      }
    }
    cp_async_commit();
  };

  // ---- phase 1: the warp's 8x8 tile C = A B over all points (A: zproj rows, B: band values)
  const int krow = lane & 3, n = lane >> 2;
  const int pa = n & 3, zpart = n >> 2;                    // A row n: projector n%4, Re (n<4) / Im
  const int bb = 4 * warp + (n >> 1), bpart = n & 1;       // B column n: band n/2 of the quad, Re/Im
  double c0 = 0.0, c1 = 0.0, e0 = 0.0, e1 = 0.0;
  for (int c = cbeg; c < cbeg + KBT_NS - 1; ++c) issue(c, true);
  for (int c = cbeg; c < nch; ++c) {
    cp_async_wait<KBT_NS - 2>();  // this thread's copies of chunk c have landed
    __syncthreads();              // ... everyone's; the stage of chunk c-1 is free
    issue(c + KBT_NS - 1, true);
    const int s = c % KBT_NS;
    const T* sb = Sb + (size_t)s * KBT_BANDS * SROW + bb * SROW;
    const double* za = reinterpret_cast<const double*>(Zb + (size_t)s * 4 * ZROW + pa * ZROW) + zpart;
#pragma unroll
    for (int u = 2 * ks; u < CP / 4; u += 2 * KBT_KS) {
      const int j = 4 * u + krow;
      const T v0 = sb[j], v1 = sb[j + 4];
      mma_f64_8x8x4(c0, c1, za[2 * j], (double)(bpart ? v0.y : v0.x));
      mma_f64_8x8x4(e0, e1, za[2 * (j + 4)], (double)(bpart ? v1.y : v1.x));
    }
  }
  part[ks][warp][lane] = make_double2(c0 + e0, c1 + e1);
  __syncthreads();
  if (ks == 0) {
    double x0 = part[0][warp][lane].x, x1 = part[0][warp][lane].y;
#pragma unroll
    for (int k2 = 1; k2 < KBT_KS; ++k2) {
      x0 += part[k2][warp][lane].x;
      x1 += part[k2][warp][lane].y;
    }
    const double d0 = __shfl_down_sync(0xffffffffu, x0, 16);
    const double d1 = __shfl_down_sync(0xffffffffu, x1, 16);
    if (UONLY) {
      if (lane < 16) {
        const int p = lane >> 2, bq = lane & 3, o = o_lo + 4 * warp + bq;
        if (p < np && o < o_hi)
          Up[((size_t)blockIdx.z * nb + (o - o_beg)) * Nlma + lma_list[l0 + p]] = make_double2(x0 + d1, x1 - d0);
      }
    } else if (lane < 16) {  // C rows p (Re zproj) and p+4 (Im zproj), columns of band bq
      const int p = lane >> 2, bq = lane & 3, o = o_lo + 4 * warp + bq;
      double2 u = make_double2(0.0, 0.0);
      if (p < np && o < o_hi) {
        const int ilma = lma_list[l0 + p];
        const double f = scale * (double)iuV[ilma];
        u = make_double2((x0 + d1) * f, (x1 - d0) * f);
        U[(size_t)(o - o_beg) * Nlma + ilma] = u;
      }
      Us[warp][p][bq] = u;
    }
  }
  if constexpr (UONLY) {
    cp_async_wait<0>();
    return;
  }
  __syncthreads();  // Us written; every warp is done with the phase-1 stages

  // ---- phase 2: W = zproj U at the item's single-item points, 8 points per pair of MMAs
  const int p = krow;  // B row / A column: projector
  const double2 u = Us[warp][p][n >> 1];
  const double bre = (n & 1) ? u.y : u.x;   // rows of Re zproj
  const double bim = (n & 1) ? u.x : -u.y;  // rows of Im zproj
  const int oc = o_lo + 4 * warp + p;       // the orbital of this lane's C elements
  const bool cvalid = oc < o_hi;
  T* Wb = W + (size_t)(cvalid ? oc - o_beg : 0) * nsp;
  for (int c = 0; c < KBT_NS - 1; ++c) issue(c, false);
  for (int c = 0; c < nch; ++c) {
    cp_async_wait<KBT_NS - 2>();
    __syncthreads();
    issue(c + KBT_NS - 1, false);
    const double2* zb = Zb + (size_t)(c % KBT_NS) * 4 * ZROW + p * ZROW;
#pragma unroll
    for (int t8 = ks; t8 < CP / 8; t8 += KBT_KS) {
      const int jl = 8 * t8 + n, j = c * CP + jl;
      const double2 z = zb[jl];
      double w0 = 0.0, w1 = 0.0;
      mma_f64_8x8x4(w0, w1, z.x, bre);
      mma_f64_8x8x4(w0, w1, z.y, bim);
      if (cvalid && j < mps) {
        const int q = kqs[j];
        if (q >= 0) Wb[q] = mk<R>((R)w0, (R)w1);
      }
    }
  }
  cp_async_wait<0>();
}

template <typename R>
static cudaError_t launch_kb_tile_t(const System& s, const void* in, int ld_in, const int* idx, int o_beg, int nb,
                                    int nbk, void* W) {
  const int kl0 = o_beg / nbk, kl1 = (o_beg + nb - 1) / nbk;
  const int ngrp = (nbk + KBT_BANDS - 1) / KBT_BANDS;
  // the kernel's static shared memory counts against the default limit, so the
  // dynamic limit is raised for every size (once per handle; prepare_kb does it
  // before a stream capture)
  const size_t smem = KbtGeom<R>::smem(s.Nps);
  if (!s.kb_smem_ok) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s.stream, &cs);
    if (e != cudaSuccess) return e;
    if (cs == cudaStreamCaptureStatusNone && (e = prepare_kb(s)) != cudaSuccess) return e;
  }
  dim3 grid((kl1 - kl0 + 1) * ngrp, s.nitems);
  k_kb_tile<R><<<grid, 32 * KBT_WARPS * KBT_KS, smem, s.launch_stream()>>>(
      (const C2<R>*)in, ld_in, o_beg, nb, nbk, kl0, ngrp, s.zproj64, s.Nlma, s.Nps, idx, s.kbq, s.atom_off, s.items,
      s.lma_list, s.iuV_d, s.Hxyz, s.U, s.nsp, (C2<R>*)W);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || s.n_multi == 0) return e;
  dim3 g2((s.n_multi + 255) / 256, (nb + KU - 1) / KU);
  k_kbfield_multi<R><<<g2, 256, 0, s.launch_stream()>>>(s.U, nb, o_beg, nbk, s.zproj64, s.Nlma, s.Nps, s.rec, s.cont,
                                                         s.kb_multi, s.n_multi, s.nsp, (C2<R>*)W);
  return cudaGetLastError();
}

// The KB field from the split projections: one CTA per (k-point, band group of
// 32, projector item, KBW_T of the item's points).  Each thread first issues the
// loads of its point (sphere index, <= 4 zproj entries), then the CTA adds the
// splits' partial projections in order and scales them (the CTAs of the first
// point range also store U for the multi-item points), so both sets of loads are
// in flight together; then W = sum_p zproj_p U_p for every band of the group,
// stored in sphere-point order (consecutive threads, consecutive points: a warp's
// store is 256 contiguous bytes of one band).  The sum over p runs in FP64 in
// projector order.
constexpr int KBW_T = 256;
template <typename R>
__global__ void __launch_bounds__(KBW_T) k_kb_w(int o_beg, int nb, int nbk, int kl0, int ngrp,
                                               const double2* __restrict__ zproj, int Nlma, int Nps,
                                               const int* __restrict__ kbq, const int* __restrict__ atom_off,
                                               const int4* __restrict__ items, const int* __restrict__ lma_list,
                                               const int* __restrict__ iuV, double scale,
                                               const double2* __restrict__ Up, int nsplit, double2* __restrict__ U,
                                               int nsp, C2<R>* __restrict__ W) {
  __shared__ double2 Us[KBT_BANDS][4];
  const int t = threadIdx.x;
  const int kq = blockIdx.x / ngrp, grp = blockIdx.x - kq * ngrp;
  const int kl = kl0 + kq;
  const int o_lo = max(o_beg, kl * nbk + grp * KBT_BANDS);
  const int o_hi = min(min(o_beg + nb, (kl + 1) * nbk), kl * nbk + (grp + 1) * KBT_BANDS);
  const int4 item = items[blockIdx.y];
  const int a = item.x, l0 = item.y, np = item.z;
  const int p0 = atom_off[a], mps = atom_off[a + 1] - p0;
  if (o_lo >= o_hi || (int)blockIdx.z * KBW_T >= mps) return;  // whole CTA leaves together
  const int j = blockIdx.z * KBW_T + t;
  // this thread's point: sphere index (-1: in several items, k_kbfield_multi) and zproj
  const int q = j < mps ? __ldg(kbq + p0 + j) : -1;
  double2 z[4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
    z[p] = (p < np && j < mps) ? __ldg(zproj + ((size_t)kl * Nlma + lma_list[l0 + p]) * Nps + j)
                               : make_double2(0.0, 0.0);
  for (int i = t; i < KBT_BANDS * 4; i += KBW_T) {
    const int b = i >> 2, p = i & 3, o = o_lo + b;
    double2 u = make_double2(0.0, 0.0);
    if (p < np && o < o_hi) {
      const int ilma = lma_list[l0 + p];
      const double2* src = Up + (size_t)(o - o_beg) * Nlma + ilma;
      for (int sp = 0; sp < nsplit; ++sp) {
        const double2 v = src[(size_t)sp * nb * Nlma];
        u.x += v.x;
        u.y += v.y;
      }
      const double f = scale * (double)iuV[ilma];
      u = make_double2(u.x * f, u.y * f);
      if (blockIdx.z == 0) U[(size_t)(o - o_beg) * Nlma + ilma] = u;
    }
    Us[b][p] = u;
  }
  __syncthreads();
  if (q < 0) return;
  C2<R>* Wo = W + (size_t)(o_lo - o_beg) * nsp + q;
  const int nbq = o_hi - o_lo;
#pragma unroll 4
  for (int b = 0; b < nbq; ++b) {
    double2 w = make_double2(0.0, 0.0);
#pragma unroll
    for (int p = 0; p < 4; ++p) w = cfma(z[p], Us[b][p], w);
    Wo[(size_t)b * nsp] = mk<R>((R)w.x, (R)w.y);
  }
}

template <typename R>
static cudaError_t launch_kb_split_t(const System& s, const void* in, int ld_in, const int* idx, int o_beg, int nb,
                                     int nbk, void* W) {
  const int kl0 = o_beg / nbk, kl1 = (o_beg + nb - 1) / nbk;
  const int ngrp = (nbk + KBT_BANDS - 1) / KBT_BANDS;
  const size_t smem = KbtGeom<R>::smem(s.Nps);
  if (!s.kb_smem_ok) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(s.stream, &cs);
    if (e != cudaSuccess) return e;
    if (cs == cudaStreamCaptureStatusNone && (e = prepare_kb(s)) != cudaSuccess) return e;
  }
  // point ranges: KB_SPLIT, or (0) enough for about six CTAs per SM
  const int ctas = (kl1 - kl0 + 1) * ngrp * s.nitems;
  int nsplit = std::max(1, std::min(s.kb_usplit > 0 ? s.kb_usplit : (6 * s.nsm + ctas - 1) / ctas, KB_USPLIT_MAX));
  nsplit = (int)std::min<size_t>((size_t)nsplit, s.Up_rows / std::max(1, nb));  // what the partials' buffer holds
  if (nsplit < 1) return cudaErrorInvalidValue;
  dim3 grid((kl1 - kl0 + 1) * ngrp, s.nitems, nsplit);
  k_kb_tile<R, true><<<grid, 32 * KBT_WARPS * KBT_KS, smem, s.launch_stream()>>>(
      (const C2<R>*)in, ld_in, o_beg, nb, nbk, kl0, ngrp, s.zproj64, s.Nlma, s.Nps, idx, s.kbq, s.atom_off, s.items,
      s.lma_list, s.iuV_d, s.Hxyz, s.U, s.nsp, (C2<R>*)W, nsplit, s.Up);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 gw((kl1 - kl0 + 1) * ngrp, s.nitems, (s.max_mps + KBW_T - 1) / KBW_T);
  k_kb_w<R><<<gw, KBW_T, 0, s.launch_stream()>>>(o_beg, nb, nbk, kl0, ngrp, s.zproj64, s.Nlma, s.Nps, s.kbq,
                                                  s.atom_off, s.items, s.lma_list, s.iuV_d, s.Hxyz, s.Up, nsplit,
                                                  s.U, s.nsp, (C2<R>*)W);
  e = cudaGetLastError();
  if (e != cudaSuccess || s.n_multi == 0) return e;
  dim3 g2((s.n_multi + 255) / 256, (nb + KU - 1) / KU);
  k_kbfield_multi<R><<<g2, 256, 0, s.launch_stream()>>>(s.U, nb, o_beg, nbk, s.zproj64, s.Nlma, s.Nps, s.rec, s.cont,
                                                         s.kb_multi, s.n_multi, s.nsp, (C2<R>*)W);
  return cudaGetLastError();
}

static int kb_tile_ctas(const System& s, int o_beg, int nb, int nbk) {
  const int kl0 = o_beg / nbk, kl1 = (o_beg + nb - 1) / nbk;
  return (kl1 - kl0 + 1) * ((nbk + KBT_BANDS - 1) / KBT_BANDS) * s.nitems;
}

bool kb_tile_fits(const System& s) {  // dynamic + static shared memory of both precisions' kernels
  constexpr size_t stat = sizeof(double2) * (KBT_WARPS * 16 + KBT_KS * KBT_WARPS * 32);
  return KbtGeom<double>::smem(s.Nps) + stat <= 227 * 1024 && KbtGeom<float>::smem(s.Nps) + stat <= 227 * 1024;
}

cudaError_t prepare_kb(const System& s) {
  cudaError_t e = raise_smem_limit((const void*)k_kb_tile<float>, KbtGeom<float>::smem(s.Nps));
  if (e == cudaSuccess) e = raise_smem_limit((const void*)k_kb_tile<double>, KbtGeom<double>::smem(s.Nps));
  if (e == cudaSuccess) e = raise_smem_limit((const void*)k_kb_tile<float, true>, KbtGeom<float>::smem(s.Nps));
  if (e == cudaSuccess) e = raise_smem_limit((const void*)k_kb_tile<double, true>, KbtGeom<double>::smem(s.Nps));
  s.kb_smem_ok = e == cudaSuccess;
  return e;
}

template <typename R>
static cudaError_t launch_kb_fused_t(const System& s, const void* in, int ld_in, const int* idx, int o_beg, int nb,
                                     int nbk, void* W) {
  switch (s.um_split) {
    case 1: return launch_kb_fused_split<R, 1>(s, in, ld_in, idx, o_beg, nb, nbk, W);
    case 2: return launch_kb_fused_split<R, 2>(s, in, ld_in, idx, o_beg, nb, nbk, W);
    case 8: return launch_kb_fused_split<R, 8>(s, in, ld_in, idx, o_beg, nb, nbk, W);
    default: return launch_kb_fused_split<R, 4>(s, in, ld_in, idx, o_beg, nb, nbk, W);
  }
}

cudaError_t launch_kb_term(const System& s, const void* in, bool from_S, int o_beg, int nb, int nbk, void* W,
                           int prec) {
  if (s.Nlma == 0 || nb == 0) return cudaSuccess;
  const void* src = from_S ? s.Sbuf : in;
  const int ld = from_S ? s.nsp : s.NL;
  const int* idx = from_S ? s.qmap : s.idx_proj;
  const bool f = (prec < 0 ? s.prec : prec) == SGPU_PREC_C64;
  // auto: the tile kernel for complex(4) grids of >= 2 CTAs per SM, the split form
  // otherwise.  Measured (B200, KB term per H application): 32^3 x 2048 orbitals
  // complex(4) tile 0.112, split 0.111 ms; complex(8) 0.205 / 0.184 ms; 48^3 x 432
  // 0.102 / 0.079 ms (band quad 0.134) and 0.164 / 0.121 ms; 32^3 x 8 k x 128 bands
  // 0.058 / 0.055 ms (band quad 0.079) and 0.089 / 0.087 ms.  The split projections
  // on the FP64 CUDA cores instead of the MMAs (lanes over points, 4 bands x 4
  // projectors a thread) were slower at every shape (0.163, 0.119, 0.086 ms complex(4)).
  const bool fits = kb_tile_fits(s);
  const bool tile_first = f && kb_tile_ctas(s, o_beg, nb, nbk) >= 2 * s.nsm;
  if (fits && (s.kb_kernel == 3 || (s.kb_kernel == 0 && !tile_first)))
    return f ? launch_kb_split_t<float>(s, src, ld, idx, o_beg, nb, nbk, W)
             : launch_kb_split_t<double>(s, src, ld, idx, o_beg, nb, nbk, W);
  const bool tile = fits && (s.kb_kernel == 1 || s.kb_kernel == 0);
  if (tile)
    return f ? launch_kb_tile_t<float>(s, src, ld, idx, o_beg, nb, nbk, W)
             : launch_kb_tile_t<double>(s, src, ld, idx, o_beg, nb, nbk, W);
  if (f) return launch_kb_fused_t<float>(s, src, ld, idx, o_beg, nb, nbk, W);
  return launch_kb_fused_t<double>(s, src, ld, idx, o_beg, nb, nbk, W);
}

cudaError_t launch_kbfield(const System& s, int o_beg, int nb, int nbk, void* W, int prec) {
  if (s.nsp == 0 || nb == 0) return cudaSuccess;
  if ((prec < 0 ? s.prec : prec) == SGPU_PREC_C64) return launch_kbfield_t<float>(s, o_beg, nb, nbk, W);
  return launch_kbfield_t<double>(s, o_beg, nb, nbk, W);
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
  k_update_projector<<<grid, 128, 0, s.launch_stream()>>>(s.kAc_d, s.rpos, s.atom_off, s.lma_atom, s.uV_d, s.Nlma, s.Nps,
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
