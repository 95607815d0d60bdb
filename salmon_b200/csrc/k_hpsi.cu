// Kleinman-Bylander projections U, the KB field W at the sphere points and the
// projector update for sm_100a, plus the precision conversions.  The
// Hamiltonian pass itself is in k_pass.cu.
#include <cuda_runtime.h>

#include <type_traits>

#include "sgpu_internal.cuh"

namespace sgpu {

// ----------------------------------------------------------------- uVpsi ---
// U[b][ilma] = Hxyz (iuV) sum_j conj(zproj(j,ilma,k)) in_b(J(j))  (hpsi.f90:188-193)
// Grid: (orbital pairs, projector items); an item is one atom with <= 4 of its
// projectors.  The 4 warps of a CTA split the atom's sphere points, accumulate
// in FP64, reduce by warp shuffles and then across warps in a fixed order
// (deterministic).  The projectors are read in FP64 for either orbital precision.
constexpr int UB = 2;
constexpr int UV_WARPS = 4;

template <typename R>
__global__ void __launch_bounds__(32 * UV_WARPS) k_uvpsi(const C2<R>* __restrict__ in, int nb, int NL, int o_beg,
                                                        int nbk, const double2* __restrict__ zproj, int Nlma, int Nps,
                                                        const int* __restrict__ idx_proj, const int* __restrict__ atom_off,
                                                        const int4* __restrict__ items, const int* __restrict__ lma_list,
                                                        const int* __restrict__ iuV, double scale, int use_iuv,
                                                        double2* __restrict__ U) {
  __shared__ double2 red[UV_WARPS][4][UB];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b0 = blockIdx.x * UB;
  const int4 item = items[blockIdx.y];
  const int a = item.x, l0 = item.y, np = item.z;
  const int p0 = atom_off[a], mps = atom_off[a + 1] - p0;
  int kl[UB];
  bool valid[UB];
#pragma unroll
  for (int u = 0; u < UB; ++u) {
    valid[u] = (b0 + u) < nb;
    kl[u] = valid[u] ? (o_beg + b0 + u) / nbk : 0;
  }
  bool samek = true;
#pragma unroll
  for (int u = 1; u < UB; ++u) samek = samek && (!valid[u] || kl[u] == kl[0]);
  int ilma[4];
#pragma unroll
  for (int p = 0; p < 4; ++p) ilma[p] = p < np ? lma_list[l0 + p] : 0;
  double2 acc[4][UB];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int u = 0; u < UB; ++u) acc[p][u] = make_double2(0, 0);
#pragma unroll 4
  for (int j = threadIdx.x; j < mps; j += 32 * UV_WARPS) {
    const int gi = __ldg(idx_proj + p0 + j);
    double2 v[UB];
#pragma unroll
    for (int u = 0; u < UB; ++u) v[u] = valid[u] ? to_d2(in[(size_t)(b0 + u) * NL + gi]) : make_double2(0, 0);
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      if (p < np) {
        if (samek) {
          const double2 z = __ldg(zproj + ((size_t)kl[0] * Nlma + ilma[p]) * Nps + j);
#pragma unroll
          for (int u = 0; u < UB; ++u) acc[p][u] = cfmaj(z, v[u], acc[p][u]);
        } else {
#pragma unroll
          for (int u = 0; u < UB; ++u) {
            const double2 z = __ldg(zproj + ((size_t)kl[u] * Nlma + ilma[p]) * Nps + j);
            acc[p][u] = cfmaj(z, v[u], acc[p][u]);
          }
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
      if (lane == 0) red[warp][p][u] = s;
    }
  __syncthreads();
  if (threadIdx.x < 4 * UB) {
    const int p = threadIdx.x / UB, u = threadIdx.x % UB;
    if (p < np && valid[u]) {
      double2 s = red[0][p][u];
#pragma unroll
      for (int w = 1; w < UV_WARPS; ++w) {
        s.x += red[w][p][u].x;
        s.y += red[w][p][u].y;
      }
      const double f = scale * (use_iuv ? (double)iuV[ilma[p]] : 1.0);
      U[(size_t)(b0 + u) * Nlma + ilma[p]] = make_double2(s.x * f, s.y * f);
    }
  }
}

cudaError_t launch_uvpsi(const System& s, const void* in, int o_beg, int nb, int nbk, bool scale_iuv, int prec) {
  if (s.Nlma == 0 || nb == 0) return cudaSuccess;
  dim3 grid((nb + UB - 1) / UB, s.nitems);
  if ((prec < 0 ? s.prec : prec) == SGPU_PREC_C64)
    k_uvpsi<float><<<grid, 32 * UV_WARPS, 0, s.launch_stream()>>>((const float2*)in, nb, s.NL, o_beg, nbk, s.zproj64, s.Nlma,
                                                         s.Nps, s.idx_proj, s.atom_off, s.items, s.lma_list, s.iuV_d,
                                                         s.Hxyz, scale_iuv ? 1 : 0, s.U);
  else
    k_uvpsi<double><<<grid, 32 * UV_WARPS, 0, s.launch_stream()>>>((const double2*)in, nb, s.NL, o_beg, nbk, s.zproj64, s.Nlma,
                                                          s.Nps, s.idx_proj, s.atom_off, s.items, s.lma_list, s.iuV_d,
                                                          s.Hxyz, scale_iuv ? 1 : 0, s.U);
  return cudaGetLastError();
}

cudaError_t launch_uvpsi_from_S(const System& s, const void* S, int o_beg, int nb, int nbk, bool scale_iuv) {
  if (s.Nlma == 0 || nb == 0) return cudaSuccess;
  dim3 grid((nb + UB - 1) / UB, s.nitems);
  if (s.prec == SGPU_PREC_C64)
    k_uvpsi<float><<<grid, 32 * UV_WARPS, 0, s.launch_stream()>>>((const float2*)S, nb, s.nsp, o_beg, nbk, s.zproj64, s.Nlma,
                                                         s.Nps, s.qmap, s.atom_off, s.items, s.lma_list, s.iuV_d,
                                                         s.Hxyz, scale_iuv ? 1 : 0, s.U);
  else
    k_uvpsi<double><<<grid, 32 * UV_WARPS, 0, s.launch_stream()>>>((const double2*)S, nb, s.nsp, o_beg, nbk, s.zproj64, s.Nlma,
                                                          s.Nps, s.qmap, s.atom_off, s.items, s.lma_list, s.iuV_d,
                                                          s.Hxyz, scale_iuv ? 1 : 0, s.U);
  return cudaGetLastError();
}

// ------------------------------------------------------------- KB field ---
// W[b][q] = sum over the (ilma, j) entries of sphere point q of zproj(j,ilma,k) U[b][ilma]
// (the dpseudo of pseudo_pt, common/hpsi.f90:194-200, already summed per grid
// point), in entry order.  One thread per sphere point and KU orbitals; a
// zproj value is loaded once for orbitals on the same k-point.
constexpr int KU = 4;

__device__ __forceinline__ int kb_entry(const int4& ra, const int4& rb, const int* cont, int e) {
  if (e < 4) return e == 0 ? ra.z : (e == 1 ? ra.w : (e == 2 ? rb.x : rb.y));
  return __ldg(cont + rb.z + (e - 4));
}

template <typename R>
__global__ void __launch_bounds__(256) k_kbfield(const double2* __restrict__ U, int nb, int o_beg, int nbk,
                                                 const C2<R>* __restrict__ zproj, int Nlma, int Nps,
                                                 const int4* __restrict__ rec, const int* __restrict__ cont, int nsp,
                                                 C2<R>* __restrict__ W) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int b0 = blockIdx.y * KU;
  if (q >= nsp) return;
  const int4 ra = __ldg(rec + 2 * (size_t)q), rb = __ldg(rec + 2 * (size_t)q + 1);
  const int ne = ra.y + rb.w;
  int kl[KU];
  bool valid[KU];
#pragma unroll
  for (int u = 0; u < KU; ++u) {
    valid[u] = b0 + u < nb;
    kl[u] = valid[u] ? (o_beg + b0 + u) / nbk : 0;
  }
  bool samek = true;
#pragma unroll
  for (int u = 1; u < KU; ++u) samek = samek && (!valid[u] || kl[u] == kl[0]);
  C2<R> acc[KU];
#pragma unroll
  for (int u = 0; u < KU; ++u) acc[u] = mk<R>(0, 0);
  for (int e = 0; e < ne; ++e) {
    const int en = kb_entry(ra, rb, cont, e);
    const int ilma = en >> 16, zoff = ilma * Nps + (en & 0xffff);
    C2<R> z0 = __ldg(zproj + (size_t)kl[0] * Nlma * Nps + zoff);
#pragma unroll
    for (int u = 0; u < KU; ++u) {
      if (!valid[u]) continue;
      const C2<R> z = samek ? z0 : __ldg(zproj + (size_t)kl[u] * Nlma * Nps + zoff);
      const double2 uu = __ldg(U + (size_t)(b0 + u) * Nlma + ilma);
      acc[u] = cfma(z, mk<R>((R)uu.x, (R)uu.y), acc[u]);
    }
  }
#pragma unroll
  for (int u = 0; u < KU; ++u)
    if (valid[u]) W[(size_t)(b0 + u) * nsp + q] = acc[u];
}

cudaError_t launch_kbfield(const System& s, int o_beg, int nb, int nbk, void* W, int prec) {
  if (s.nsp == 0 || nb == 0) return cudaSuccess;
  dim3 grid((s.nsp + 255) / 256, (nb + KU - 1) / KU);
  if ((prec < 0 ? s.prec : prec) == SGPU_PREC_C64)
    k_kbfield<float><<<grid, 256, 0, s.launch_stream()>>>(s.U, nb, o_beg, nbk, s.zproj32, s.Nlma, s.Nps, s.rec, s.cont, s.nsp,
                                                (float2*)W);
  else
    k_kbfield<double><<<grid, 256, 0, s.launch_stream()>>>(s.U, nb, o_beg, nbk, s.zproj64, s.Nlma, s.Nps, s.rec, s.cont, s.nsp,
                                                 (double2*)W);
  return cudaGetLastError();
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
