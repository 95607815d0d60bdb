// FP64 reductions over the resident orbitals: density, current, energy terms.
// Orbitals may be complex(8) or complex(4); every sum is accumulated in FP64
// in a fixed order (no atomics), so results are reproducible run to run.
#include <cuda_runtime.h>

#include "sgpu_internal.cuh"

namespace sgpu {

// ------------------------------------------------------------- psi_rho ---
// rho(i) = sum_{k,b} occ(b,k) |zu(i,b,k)|^2   (common/psi_rho.f90:93-146, sym1)
// Orbitals are split into chunks; each chunk writes a partial density, and the
// partials are summed in chunk order.
constexpr int RHO_CHUNK = 64;

template <typename R>
__global__ void k_rho_partial(const C2<R>* __restrict__ zu, const double* __restrict__ occ_o, int norb, int NL,
                              double* __restrict__ part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NL) return;
  const int o0 = blockIdx.y * RHO_CHUNK;
  const int o1 = min(o0 + RHO_CHUNK, norb);
  double acc = 0.0;
  int o = o0;
  for (; o + 4 <= o1; o += 4) {
    double2 z[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) z[u] = to_d2(zu[(size_t)(o + u) * NL + i]);
#pragma unroll
    for (int u = 0; u < 4; ++u) acc += occ_o[o + u] * (z[u].x * z[u].x + z[u].y * z[u].y);
  }
  for (; o < o1; ++o) {
    const double2 z = to_d2(zu[(size_t)o * NL + i]);
    acc += occ_o[o] * (z.x * z.x + z.y * z.y);
  }
  part[(size_t)blockIdx.y * NL + i] = acc;
}

__global__ void k_rho_final(const double* __restrict__ part, int nchunk, int NL, double* __restrict__ rho) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NL) return;
  double acc = 0.0;
  for (int c = 0; c < nchunk; ++c) acc += part[(size_t)c * NL + i];
  rho[i] = acc;
}

cudaError_t launch_psi_rho(System& s, double* rho_dev) {
  const int nchunk = (s.norb + RHO_CHUNK - 1) / RHO_CHUNK;
  if ((size_t)nchunk * s.NL > s.red_elems) return cudaErrorInvalidValue;
  dim3 grid((s.NL + 255) / 256, nchunk);
  if (s.prec == SGPU_PREC_C64)
    k_rho_partial<float><<<grid, 256, 0, s.launch_stream()>>>((const float2*)s.zu, s.occ_o, s.norb, s.NL, s.red);
  else
    k_rho_partial<double><<<grid, 256, 0, s.launch_stream()>>>((const double2*)s.zu, s.occ_o, s.norb, s.NL, s.red);
  k_rho_final<<<(s.NL + 255) / 256, 256, 0, s.launch_stream()>>>(s.red, nchunk, s.NL, rho_dev);
  return cudaGetLastError();
}

// ------------------------------------------------------ block reduction ---
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sh /*[32*NV]*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sh[warp * NV + k] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = lane < nw ? sh[lane * NV + k] : 0.0;
#pragma unroll
    for (int k = 0; k < NV; ++k)
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
  }
}

// ------------------------------------------------------------- current ---
// Per orbital: jt = sum |psi|^2 (current.f90:182-186) and the current_stencil
// sums F,G,H = 2 sum Im(conj(psi) sum_n nab_n psi(+n)) (stencil/F90/current.f90).
template <typename R>
__global__ void __launch_bounds__(256) k_current_orb(const C2<R>* __restrict__ zu, int NLx, int NLy, int NLz,
                                                      const double* __restrict__ nab12, double* __restrict__ out) {
  __shared__ double sh[32 * 4];
  const int o = blockIdx.x, NL = NLx * NLy * NLz;
  const C2<R>* E = zu + (size_t)o * NL;
  double nb[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) nb[k] = nab12[k];
  double v[4] = {0, 0, 0, 0};  // jt, F (x), G (y), H (z)
  for (int i = threadIdx.x; i < NL; i += blockDim.x) {
    const int iz = i % NLz, iy = (i / NLz) % NLy, ix = i / (NLy * NLz);
    const double2 e = to_d2(E[i]);
    v[0] += e.x * e.x + e.y * e.y;
    double2 sx = make_double2(0, 0), sy = make_double2(0, 0), sz = make_double2(0, 0);
#pragma unroll
    for (int n = 1; n <= 4; ++n) {
      const int jx = ix + n >= NLx ? ix + n - NLx : ix + n;
      const int jy = iy + n >= NLy ? iy + n - NLy : iy + n;
      const int jz = iz + n >= NLz ? iz + n - NLz : iz + n;
      const double2 ex = to_d2(E[(jx * NLy + iy) * NLz + iz]);
      const double2 ey = to_d2(E[(ix * NLy + jy) * NLz + iz]);
      const double2 ez = to_d2(E[(ix * NLy + iy) * NLz + jz]);
      sx.x += nb[n - 1] * ex.x; sx.y += nb[n - 1] * ex.y;
      sy.x += nb[3 + n] * ey.x; sy.y += nb[3 + n] * ey.y;
      sz.x += nb[7 + n] * ez.x; sz.y += nb[7 + n] * ez.y;
    }
    // aimag(conj(e) * s) = e.x s.y - e.y s.x
    v[1] += e.x * sx.y - e.y * sx.x;
    v[2] += e.x * sy.y - e.y * sy.x;
    v[3] += e.x * sz.y - e.y * sz.x;
  }
  block_sum<4>(v, sh);
  if (threadIdx.x == 0) {
    out[4 * o + 0] = v[0];
    out[4 * o + 1] = 2.0 * v[1];
    out[4 * o + 2] = 2.0 * v[2];
    out[4 * o + 3] = 2.0 * v[3];
  }
}

// Weighted projections for the nonlocal current (current.f90:247-265):
// Uw[o][ilma][w] = sum_j conj(zproj(j,ilma,k)) r_w(j) psi(J(j)), r = (1, x, y, z).
template <typename R>
__global__ void __launch_bounds__(256) k_uvpsi_w(const C2<R>* __restrict__ zu, int NL, int NBocc,
                                                  const double2* __restrict__ zproj, int Nlma, int Nps,
                                                  const int* __restrict__ idx_proj, const int* __restrict__ atom_off,
                                                  const double* __restrict__ rpos, const int4* __restrict__ items,
                                                  int nitems, const int* __restrict__ lma_list,
                                                  double2* __restrict__ Uw) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int o = blockIdx.x, kl = o / NBocc;
  for (int it = warp; it < nitems; it += nw) {
    const int4 item = items[it];
    const int a = item.x, l0 = item.y, np = item.z;
    const int p0 = atom_off[a], mps = atom_off[a + 1] - p0;
    double2 acc[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int w = 0; w < 4; ++w) acc[p][w] = make_double2(0, 0);
    int ilma[4];
#pragma unroll
    for (int p = 0; p < 4; ++p) ilma[p] = p < np ? lma_list[l0 + p] : 0;
    for (int j = lane; j < mps; j += 32) {
      const int gi = idx_proj[p0 + j];
      const double2 e = to_d2(zu[(size_t)o * NL + gi]);
      const double* r = rpos + 3 * (size_t)(p0 + j);
      const double rw[4] = {1.0, r[0], r[1], r[2]};
#pragma unroll
      for (int p = 0; p < 4; ++p)
        if (p < np) {
          const double2 z = zproj[((size_t)kl * Nlma + ilma[p]) * Nps + j];
          // conj(z) * e
          const double2 ze = make_double2(z.x * e.x + z.y * e.y, z.x * e.y - z.y * e.x);
#pragma unroll
          for (int w = 0; w < 4; ++w) {
            acc[p][w].x += rw[w] * ze.x;
            acc[p][w].y += rw[w] * ze.y;
          }
        }
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int w = 0; w < 4; ++w)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          acc[p][w].x += __shfl_xor_sync(0xffffffffu, acc[p][w].x, off);
          acc[p][w].y += __shfl_xor_sync(0xffffffffu, acc[p][w].y, off);
        }
    if (lane == 0)
#pragma unroll
      for (int p = 0; p < 4; ++p)
        if (p < np)
#pragma unroll
          for (int w = 0; w < 4; ++w) Uw[((size_t)o * Nlma + ilma[p]) * 4 + w] = acc[p][w];
  }
}

// Combines the per-orbital terms exactly as current() does (current.f90:182-273)
// and sums over orbitals in a fixed order.
__global__ void k_current_final(const double* __restrict__ orb, const double2* __restrict__ Uw,
                                const double* __restrict__ occ_o, const double* __restrict__ kAc,
                                const int* __restrict__ iuV, int norb, int NBocc, int Nlma, double Hxyz,
                                double IaLxyz, double* __restrict__ jav) {
  __shared__ double sh[32 * 3];
  double v[3] = {0, 0, 0};
  for (int o = threadIdx.x; o < norb; o += blockDim.x) {
    const int kl = o / NBocc;
    const double occ = occ_o[o];
    const double jt = orb[4 * o];
    double j[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) j[d] = occ * kAc[3 * kl + d] * jt + orb[4 * o + 1 + d] * occ;
    double jn[3] = {0, 0, 0};
    for (int l = 0; l < Nlma; ++l) {
      const double2* u = Uw + ((size_t)o * Nlma + l) * 4;
      const double f = Hxyz * (double)iuV[l];
      const double2 u0 = make_double2(u[0].x * f, u[0].y * f);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double2 ud = make_double2(u[1 + d].x * Hxyz, u[1 + d].y * Hxyz);
        // aimag(conjg(ud) * u0)
        jn[d] += occ * IaLxyz * 2.0 * (ud.x * u0.y - ud.y * u0.x);
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] += j[d] * Hxyz * IaLxyz + jn[d];
  }
  block_sum<3>(v, sh);
  if (threadIdx.x == 0) {
    jav[0] = v[0];
    jav[1] = v[1];
    jav[2] = v[2];
  }
}

cudaError_t launch_current(System& s, double* jav_dev) {
  double* orb = s.red;  // [norb][4]
  if ((size_t)4 * s.norb > s.red_elems) return cudaErrorInvalidValue;
  double* nab12 = s.red + 4 * (size_t)s.norb;
  if ((size_t)4 * s.norb + 12 > s.red_elems) return cudaErrorInvalidValue;
  double h[12];
  for (int n = 0; n < 4; ++n)
    for (int d = 0; d < 3; ++d) h[4 * d + n] = s.nab[d][n + 1];
  cudaError_t e = cudaMemcpyAsync(nab12, h, sizeof(h), cudaMemcpyHostToDevice, s.stream);
  if (e != cudaSuccess) return e;
  if (s.prec == SGPU_PREC_C64) {
    k_current_orb<float><<<s.norb, 256, 0, s.launch_stream()>>>((const float2*)s.zu, s.NLx, s.NLy, s.NLz, nab12, orb);
    if (s.Nlma)
      k_uvpsi_w<float><<<s.norb, 256, 0, s.launch_stream()>>>((const float2*)s.zu, s.NL, s.NBocc, s.zproj64, s.Nlma, s.Nps,
                                                     s.idx_proj, s.atom_off, s.rpos, s.items, s.nitems, s.lma_list,
                                                     s.Uw);
  } else {
    k_current_orb<double><<<s.norb, 256, 0, s.launch_stream()>>>((const double2*)s.zu, s.NLx, s.NLy, s.NLz, nab12, orb);
    if (s.Nlma)
      k_uvpsi_w<double><<<s.norb, 256, 0, s.launch_stream()>>>((const double2*)s.zu, s.NL, s.NBocc, s.zproj64, s.Nlma,
                                                      s.Nps, s.idx_proj, s.atom_off, s.rpos, s.items, s.nitems,
                                                      s.lma_list, s.Uw);
  }
  k_current_final<<<1, 256, 0, s.launch_stream()>>>(orb, s.Uw, s.occ_o, s.kAc_d, s.iuV_d, s.norb, s.NBocc, s.Nlma, s.Hxyz,
                                           1.0 / s.aLxyz, jav_dev);
  return cudaGetLastError();
}

// -------------------------------------------------------------- energy ---
// tpsum = sum conj(psi) (lap0_2 psi - 0.5 v - i w)  (stencil/F90/total_energy.f90:93-180)
template <typename R>
__global__ void __launch_bounds__(256) k_ekin_orb(const C2<R>* __restrict__ zu, int NLx, int NLy, int NLz, int NBocc,
                                                   const double* __restrict__ kAc, const double* __restrict__ coef,
                                                   double* __restrict__ out) {
  __shared__ double sh[32 * 2];
  const int o = blockIdx.x, NL = NLx * NLy * NLz, kl = o / NBocc;
  const C2<R>* E = zu + (size_t)o * NL;
  // coef: [0] = lap0_2, [1..12] = lapt, [13..24] = nab
  const double A = coef[0];
  double lapt[12], nabt[12];
#pragma unroll
  for (int n = 0; n < 12; ++n) {
    lapt[n] = coef[1 + n];
    nabt[n] = kAc[3 * kl + n / 4] * coef[13 + n];
  }
  double v2[2] = {0, 0};
  for (int i = threadIdx.x; i < NL; i += blockDim.x) {
    const int iz = i % NLz, iy = (i / NLz) % NLy, ix = i / (NLy * NLz);
    const double2 e = to_d2(E[i]);
    double2 v = make_double2(0, 0), w = make_double2(0, 0);
#pragma unroll
    for (int n = 1; n <= 4; ++n) {
      const int xp = (ix + n) % NLx, xm = (ix - n + 4 * NLx) % NLx;
      const int yp = (iy + n) % NLy, ym = (iy - n + 4 * NLy) % NLy;
      const int zp = (iz + n) % NLz, zm = (iz - n + 4 * NLz) % NLz;
      const double2 a1 = to_d2(E[(xp * NLy + iy) * NLz + iz]), a2 = to_d2(E[(xm * NLy + iy) * NLz + iz]);
      const double2 b1 = to_d2(E[(ix * NLy + yp) * NLz + iz]), b2 = to_d2(E[(ix * NLy + ym) * NLz + iz]);
      const double2 c1 = to_d2(E[(ix * NLy + iy) * NLz + zp]), c2 = to_d2(E[(ix * NLy + iy) * NLz + zm]);
      v.x += lapt[n - 1] * (a1.x + a2.x) + lapt[3 + n] * (b1.x + b2.x) + lapt[7 + n] * (c1.x + c2.x);
      v.y += lapt[n - 1] * (a1.y + a2.y) + lapt[3 + n] * (b1.y + b2.y) + lapt[7 + n] * (c1.y + c2.y);
      w.x += nabt[n - 1] * (a1.x - a2.x) + nabt[3 + n] * (b1.x - b2.x) + nabt[7 + n] * (c1.x - c2.x);
      w.y += nabt[n - 1] * (a1.y - a2.y) + nabt[3 + n] * (b1.y - b2.y) + nabt[7 + n] * (c1.y - c2.y);
    }
    // z = A e - 0.5 v - i w ;  F += conj(e) z
    const double2 z = make_double2(A * e.x - 0.5 * v.x + w.y, A * e.y - 0.5 * v.y - w.x);
    v2[0] += e.x * z.x + e.y * z.y;
    v2[1] += e.x * z.y - e.y * z.x;
  }
  block_sum<2>(v2, sh);
  if (threadIdx.x == 0) {
    out[2 * o] = v2[0];
    out[2 * o + 1] = v2[1];
  }
}

__global__ void k_energy_final(const double* __restrict__ orb, const double2* __restrict__ U,
                               const double* __restrict__ occ_o, const double* __restrict__ kAc,
                               const int* __restrict__ iuV, int norb, int NBocc, int Nlma, double Hxyz,
                               double* __restrict__ e) {
  __shared__ double sh[32 * 2];
  double v[2] = {0, 0};
  for (int o = threadIdx.x; o < norb; o += blockDim.x) {
    const int kl = o / NBocc;
    const double occ = occ_o[o];
    const double k2 = kAc[3 * kl] * kAc[3 * kl] + kAc[3 * kl + 1] * kAc[3 * kl + 1] + kAc[3 * kl + 2] * kAc[3 * kl + 2];
    v[0] += occ * orb[2 * o] * Hxyz + occ * k2 / 2.0;   // real part of occ*tpsum*Hxyz + occ*|k|^2/2
    double en = 0;
    for (int l = 0; l < Nlma; ++l) {
      const double2 u = U[(size_t)o * Nlma + l];      // Hxyz * sum uV ekr psi
      en += occ * (u.x * u.x + u.y * u.y) * (double)iuV[l];
    }
    v[1] += en;
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    e[0] = v[0];
    e[1] = v[1];
  }
}

cudaError_t launch_energy(System& s, double* e_dev) {
  if ((size_t)2 * s.norb + 32 > s.red_elems) return cudaErrorInvalidValue;
  double* orb = s.red;
  double* coef = s.red + 2 * (size_t)s.norb;
  double h[25];
  h[0] = -(s.lap[0][0] + s.lap[1][0] + s.lap[2][0]) * 0.5;
  for (int d = 0; d < 3; ++d)
    for (int n = 0; n < 4; ++n) {
      h[1 + 4 * d + n] = s.lap[d][n + 1];
      h[13 + 4 * d + n] = s.nab[d][n + 1];
    }
  cudaError_t err = cudaMemcpyAsync(coef, h, sizeof(h), cudaMemcpyHostToDevice, s.stream);
  if (err != cudaSuccess) return err;
  if (s.prec == SGPU_PREC_C64)
    k_ekin_orb<float><<<s.norb, 256, 0, s.launch_stream()>>>((const float2*)s.zu, s.NLx, s.NLy, s.NLz, s.NBocc, s.kAc_d, coef, orb);
  else
    k_ekin_orb<double><<<s.norb, 256, 0, s.launch_stream()>>>((const double2*)s.zu, s.NLx, s.NLy, s.NLz, s.NBocc, s.kAc_d, coef,
                                                     orb);
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  // U = Hxyz * sum conj(zproj) psi = Hxyz * sum uV ekr psi  (total_energy.f90:191-197), FP64 projectors
  if (s.Nlma) {
    err = launch_uvpsi(s, s.zu, 0, s.norb, s.NBocc, false);
    if (err != cudaSuccess) return err;
  }
  k_energy_final<<<1, 256, 0, s.launch_stream()>>>(orb, s.U, s.occ_o, s.kAc_d, s.iuV_d, s.norb, s.NBocc, s.Nlma, s.Hxyz, e_dev);
  return cudaGetLastError();
}

}  // namespace sgpu
