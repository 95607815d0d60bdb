// FP64 reductions over the resident orbitals: density, current, energy terms.
// Orbitals may be complex(8) or complex(4); every sum is accumulated in FP64
// in a fixed order (no atomics), so results are reproducible run to run.
#include <cuda_runtime.h>

#include <algorithm>

#include <type_traits>

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
// sums F,G,H = 2 sum Im(conj(psi) sum_n nab_n psi(+n)) (stencil/F90/current.f90),
// with forward neighbours only (n = 1..4), as the reference's stencil has them.
//
// One CTA of NT threads per orbital marches along x.  Thread t owns the plane
// points t, t+NT, ... (P of them); for each it keeps psi at planes x..x+4 in a
// register queue (converted to FP64 once, on load), so the x-neighbours cost
// nothing; plane x is staged in FP64 in shared memory (double-buffered) for the
// y and z neighbours.  Every element is read from HBM once (the four wrap planes
// twice) and converted once; the loads run D planes ahead of their use.  Sums are FP64, per thread in plane order, then a
// fixed-order block sum: out[o][4].
struct Nab12 {
  double v[12];  // nabx(1:4), naby(1:4), nabz(1:4): kernel parameters, read from the parameter bank
};

//
// GY, GZ (non-zero): the plane shape at compile time, so the neighbour offsets are
// shifts and masks the compiler recomputes instead of holding them in registers;
// MB: CTAs per SM the register budget is cut for.
template <typename R, int NT, int P, int D, int GY = 0, int GZ = 0, int MB = 1>
__global__ void __launch_bounds__(NT, MB) k_current_march(const C2<R>* __restrict__ zu, int NLx, int NLy_, int NLz_,
                                                        const Nab12 nab, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NLy = GZ ? GY : NLy_, NLz = GZ ? GZ : NLz_;
  const int NYZ = NLy * NLz;
  double2* buf = reinterpret_cast<double2*>(smem_raw);  // [2][NYZ]
  __shared__ double sh[32 * 4];
  const int o = blockIdx.x, t = threadIdx.x;
  const C2<R>* E = zu + (size_t)o * NLx * NYZ;
  const double* nb = nab.v;
  int yr[P][4], zi[P][4], own[P];
  bool ok[P];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const int i = t + NT * p;
    ok[p] = i < NYZ;
    own[p] = ok[p] ? i : 0;
    const int y = own[p] / NLz, z = own[p] - (own[p] / NLz) * NLz;
#pragma unroll
    for (int n = 1; n <= 4; ++n) {
      int yn = y + n, zn = z + n;
      while (yn >= NLy) yn -= NLy;
      while (zn >= NLz) zn -= NLz;
      yr[p][n - 1] = yn * NLz + z;
      zi[p][n - 1] = y * NLz + zn;
    }
  }
  double2 q[5][P];  // q[m][p]: plane x+m at point p
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    const int xm = m < NLx ? m : m % NLx;
#pragma unroll
    for (int p = 0; p < P; ++p) q[m][p] = ok[p] ? to_d2(__ldg(E + (size_t)xm * NYZ + own[p])) : make_double2(0, 0);
  }
  C2<R> nxt[D][P];  // planes x+5 .. x+4+D in flight
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const int xm = (5 + d) % NLx;
#pragma unroll
    for (int p = 0; p < P; ++p) nxt[d][p] = ok[p] ? __ldg(E + (size_t)xm * NYZ + own[p]) : C2<R>{};
  }
  // a plane's bytes (bulk L2 prefetch needs 16-byte multiples; 0: no prefetch)
  const unsigned pf_bytes = ((size_t)NYZ * sizeof(C2<R>)) % 16 == 0 ? (unsigned)(NYZ * sizeof(C2<R>)) : 0u;
  double v[4] = {0, 0, 0, 0};  // jt, F (x), G (y), H (z)
  for (int x = 0; x < NLx; ++x) {
    double2* pl = buf + (size_t)(x & 1) * NYZ;
#pragma unroll
    for (int p = 0; p < P; ++p)
      if (ok[p]) pl[own[p]] = q[0][p];
    if (t == 0 && pf_bytes) {  // plane x+5+D+4 into L2 for the load issued four steps from now
      prefetch_l2_bulk(E + (size_t)((x + 9 + D) % NLx) * NYZ, pf_bytes);
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < P; ++p) {
      if (!ok[p]) continue;
      const double2 e = q[0][p];
      v[0] += e.x * e.x + e.y * e.y;
      double2 sx = make_double2(0, 0), sy = make_double2(0, 0), sz = make_double2(0, 0);
#pragma unroll
      for (int n = 1; n <= 4; ++n) {
        const double2 ex = q[n][p];
        const double2 ey = pl[yr[p][n - 1]];
        const double2 ez = pl[zi[p][n - 1]];
        sx.x += nb[n - 1] * ex.x; sx.y += nb[n - 1] * ex.y;
        sy.x += nb[3 + n] * ey.x; sy.y += nb[3 + n] * ey.y;
        sz.x += nb[7 + n] * ez.x; sz.y += nb[7 + n] * ez.y;
      }
      // aimag(conj(e) * s) = e.x s.y - e.y s.x
      v[1] += e.x * sx.y - e.y * sx.x;
      v[2] += e.x * sy.y - e.y * sy.x;
      v[3] += e.x * sz.y - e.y * sz.x;
    }
    const int xl = (x + 5 + D) % NLx;  // the plane that enters the pipeline
#pragma unroll
    for (int p = 0; p < P; ++p) {
      q[0][p] = q[1][p];
      q[1][p] = q[2][p];
      q[2][p] = q[3][p];
      q[3][p] = q[4][p];
      q[4][p] = ok[p] ? to_d2(nxt[0][p]) : make_double2(0, 0);
#pragma unroll
      for (int d = 0; d + 1 < D; ++d) nxt[d][p] = nxt[d + 1][p];
      nxt[D - 1][p] = ok[p] ? __ldg(E + (size_t)xl * NYZ + own[p]) : C2<R>{};
    }
  }
  block_sum<4>(v, sh);
  if (t == 0) {
    out[4 * (size_t)o] = v[0];
    out[4 * (size_t)o + 1] = v[1];
    out[4 * (size_t)o + 2] = v[2];
    out[4 * (size_t)o + 3] = v[3];
  }
}

// The x-march with each GY x GZ plane split over NP CTAs of GY/NP rows (one
// point per thread, (GY/NP)*GZ threads): a CTA stages its rows and the four rows
// after them (the forward y-neighbours, read from L2 each step) in FP64 in
// shared memory.  Small CTAs at few registers let several orbitals' marches
// share an SM, so one CTA's barrier waits overlap another's arithmetic.
// out[o][h][4], h = the part.
template <typename R, int GY, int GZ, int NP>
__global__ void __launch_bounds__(GY / NP * GZ) k_current_march_yh(const C2<R>* __restrict__ zu, int NLx,
                                                                  const Nab12 nab, double* __restrict__ out) {
  constexpr int NYH = GY / NP, NT = NYH * GZ, NYZ = GY * GZ, RB = (NYH + 4) * GZ;
  static_assert(NT % 32 == 0 && NT <= 1024 && 4 * GZ <= NT, "one point per thread, halo loaded by the first rows");
  __shared__ double2 buf[2][RB];
  __shared__ double sh[32 * 4];
  const int o = blockIdx.x / NP, h = blockIdx.x - (blockIdx.x / NP) * NP, t = threadIdx.x;
  const C2<R>* E = zu + (size_t)o * NLx * NYZ;
  const double* nb = nab.v;
  const int yl = t / GZ, z = t - (t / GZ) * GZ;
  const int own = (h * NYH + yl) * GZ + z;                           // in the plane
  const int hrow = ((h + 1) * NYH + (t / GZ)) % GY;                   // halo row of threads t < 4 GZ
  const int hsrc = hrow * GZ + z;
  int zo[4];                                                          // z neighbours in the staged rows
#pragma unroll
  for (int n = 1; n <= 4; ++n) zo[n - 1] = yl * GZ + ((z + n) % GZ);
  // register queue: at phase P (plane x = 5i + P) plane x+m sits in q[(P+m) % 5];
  // the march is unrolled five times so the queue rotates by renaming (NLx >= 6)
  double2 q[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) q[m] = to_d2(__ldg(E + (size_t)m * NYZ + own));
  C2<R> nxt = __ldg(E + (size_t)(5 % NLx) * NYZ + own);
  int xn = 6 < NLx ? 6 : 6 - NLx;                                     // the plane loaded next
  double v[4] = {0, 0, 0, 0};
  int x = 0;
  auto step = [&](auto phase) -> bool {
    constexpr int P = decltype(phase)::value;
    double2* pl = buf[x & 1];
    const double2 e = q[P % 5];
    pl[t] = e;
    if (t < 4 * GZ) pl[NT + t] = to_d2(__ldg(E + (size_t)x * NYZ + hsrc));
    __syncthreads();
    v[0] = fma(e.x, e.x, fma(e.y, e.y, v[0]));
    double2 sx = make_double2(0, 0), sy = make_double2(0, 0), sz = make_double2(0, 0);
#pragma unroll
    for (int n = 1; n <= 4; ++n) {
      const double2 ex = q[(P + n) % 5];
      const double2 ey = pl[(yl + n) * GZ + z];
      const double2 ez = pl[zo[n - 1]];
      sx.x = fma(nb[n - 1], ex.x, sx.x); sx.y = fma(nb[n - 1], ex.y, sx.y);
      sy.x = fma(nb[3 + n], ey.x, sy.x); sy.y = fma(nb[3 + n], ey.y, sy.y);
      sz.x = fma(nb[7 + n], ez.x, sz.x); sz.y = fma(nb[7 + n], ez.y, sz.y);
    }
    // aimag(conjg(e) s) = e.x s.y - e.y s.x
    v[1] = fma(e.x, sx.y, fma(-e.y, sx.x, v[1]));
    v[2] = fma(e.x, sy.y, fma(-e.y, sy.x, v[2]));
    v[3] = fma(e.x, sz.y, fma(-e.y, sz.x, v[3]));
    q[P % 5] = to_d2(nxt);  // plane x+5 takes the slot of plane x
    nxt = __ldg(E + (size_t)xn * NYZ + own);
    xn = xn + 1 < NLx ? xn + 1 : 0;
    ++x;
    return x < NLx;
  };
  for (;;) {
    if (!step(std::integral_constant<int, 0>{})) break;
    if (!step(std::integral_constant<int, 1>{})) break;
    if (!step(std::integral_constant<int, 2>{})) break;
    if (!step(std::integral_constant<int, 3>{})) break;
    if (!step(std::integral_constant<int, 4>{})) break;
  }
  block_sum<4>(v, sh);
  if (t == 0) {
    double* d = out + 4 * (size_t)blockIdx.x;
    d[0] = v[0];
    d[1] = v[1];
    d[2] = v[2];
    d[3] = v[3];
  }
}
// The same march with two rows per thread: thread (r, z) owns the points of rows
// 2r and 2r+1, so row 2r+1 is a y-neighbour in registers and the four rows above
// it are read once for both points (six shared-memory loads a point instead of
// eight; the march is bound by shared-memory wavefronts).  Each GY x GZ plane is
// split over NP CTAs of GY/NP rows ((GY/NP/2)*GZ threads) plus four halo rows.
template <typename R, int GY, int GZ, int NP, int MB = 1>
__global__ void __launch_bounds__(GY / NP / 2 * GZ, MB) k_current_march_y2(const C2<R>* __restrict__ zu, int NLx,
                                                                      const Nab12 nab, double* __restrict__ out) {
  constexpr int NYH = GY / NP, NT = NYH / 2 * GZ, NYZ = GY * GZ, RB = (NYH + 4) * GZ;
  static_assert(NYH % 2 == 0 && NT % 32 == 0 && NT <= 1024 && 4 * GZ <= NT, "two rows per thread, halo by the first");
  __shared__ double2 buf[2][RB];
  __shared__ double sh[32 * 4];
  const int o = blockIdx.x / NP, h = blockIdx.x - (blockIdx.x / NP) * NP, t = threadIdx.x;
  const C2<R>* E = zu + (size_t)o * NLx * NYZ;
  const double* nb = nab.v;
  const int y0 = 2 * (t / GZ), z = t - (t / GZ) * GZ;                 // local rows y0, y0 + 1
  const int own = (h * NYH + y0) * GZ + z;                            // row y0 in the plane; y0 + 1 is own + GZ
  const int hsrc = (((h + 1) * NYH + t / GZ) % GY) * GZ + z;          // halo row of threads t < 4 GZ
  int zo[4];                                                          // z + n in a staged row
#pragma unroll
  for (int n = 1; n <= 4; ++n) zo[n - 1] = (z + n) % GZ;
  // register queues as in k_current_march_yh (plane x + m in slot (P + m) % 5)
  double2 qa[5], qb[5];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    qa[m] = to_d2(__ldg(E + (size_t)m * NYZ + own));
    qb[m] = to_d2(__ldg(E + (size_t)m * NYZ + own + GZ));
  }
  C2<R> na = __ldg(E + (size_t)(5 % NLx) * NYZ + own), nb_ = __ldg(E + (size_t)(5 % NLx) * NYZ + own + GZ);
  int xn = 6 < NLx ? 6 : 6 - NLx;
  double v[4] = {0, 0, 0, 0};
  int x = 0;
  auto step = [&](auto phase) -> bool {
    constexpr int P = decltype(phase)::value;
    double2* pl = buf[x & 1];
    const double2 ea = qa[P % 5], eb = qb[P % 5];
    pl[y0 * GZ + z] = ea;
    pl[(y0 + 1) * GZ + z] = eb;
    if (t < 4 * GZ) pl[NYH * GZ + t] = to_d2(__ldg(E + (size_t)x * NYZ + hsrc));
    __syncthreads();
    v[0] = fma(ea.x, ea.x, fma(ea.y, ea.y, fma(eb.x, eb.x, fma(eb.y, eb.y, v[0]))));
    double2 r[5];  // rows y0 + 1 .. y0 + 5 at column z
    r[0] = eb;
#pragma unroll
    for (int k = 1; k < 5; ++k) r[k] = pl[(y0 + 1 + k) * GZ + z];
    double2 sxa = make_double2(0, 0), sya = sxa, sza = sxa, sxb = sxa, syb = sxa, szb = sxa;
#pragma unroll
    for (int n = 1; n <= 4; ++n) {
      const double2 xa = qa[(P + n) % 5], xb = qb[(P + n) % 5];
      const double2 ya = r[n - 1], yb = r[n];
      const double2 za = pl[y0 * GZ + zo[n - 1]], zb = pl[(y0 + 1) * GZ + zo[n - 1]];
      sxa.x = fma(nb[n - 1], xa.x, sxa.x); sxa.y = fma(nb[n - 1], xa.y, sxa.y);
      sxb.x = fma(nb[n - 1], xb.x, sxb.x); sxb.y = fma(nb[n - 1], xb.y, sxb.y);
      sya.x = fma(nb[3 + n], ya.x, sya.x); sya.y = fma(nb[3 + n], ya.y, sya.y);
      syb.x = fma(nb[3 + n], yb.x, syb.x); syb.y = fma(nb[3 + n], yb.y, syb.y);
      sza.x = fma(nb[7 + n], za.x, sza.x); sza.y = fma(nb[7 + n], za.y, sza.y);
      szb.x = fma(nb[7 + n], zb.x, szb.x); szb.y = fma(nb[7 + n], zb.y, szb.y);
    }
    // aimag(conjg(e) s) = e.x s.y - e.y s.x, point a then point b
    v[1] = fma(eb.x, sxb.y, fma(-eb.y, sxb.x, fma(ea.x, sxa.y, fma(-ea.y, sxa.x, v[1]))));
    v[2] = fma(eb.x, syb.y, fma(-eb.y, syb.x, fma(ea.x, sya.y, fma(-ea.y, sya.x, v[2]))));
    v[3] = fma(eb.x, szb.y, fma(-eb.y, szb.x, fma(ea.x, sza.y, fma(-ea.y, sza.x, v[3]))));
    qa[P % 5] = to_d2(na);  // plane x+5 takes the slot of plane x
    qb[P % 5] = to_d2(nb_);
    na = __ldg(E + (size_t)xn * NYZ + own);
    nb_ = __ldg(E + (size_t)xn * NYZ + own + GZ);
    xn = xn + 1 < NLx ? xn + 1 : 0;
    ++x;
    return x < NLx;
  };
  for (;;) {
    if (!step(std::integral_constant<int, 0>{})) break;
    if (!step(std::integral_constant<int, 1>{})) break;
    if (!step(std::integral_constant<int, 2>{})) break;
    if (!step(std::integral_constant<int, 3>{})) break;
    if (!step(std::integral_constant<int, 4>{})) break;
  }
  block_sum<4>(v, sh);
  if (t == 0) {
    double* d = out + 4 * (size_t)blockIdx.x;
    d[0] = v[0];
    d[1] = v[1];
    d[2] = v[2];
    d[3] = v[3];
  }
}
template <typename R, int GY, int GZ, int NP, int MB = 1>
static cudaError_t current_march_y2(System& s, const Nab12& nab, double* out) {
  k_current_march_y2<R, GY, GZ, NP, MB><<<NP * s.norb, GY / NP / 2 * GZ, 0, s.launch_stream()>>>((const C2<R>*)s.zu,
                                                                                             s.NLx, nab, out);
  return cudaGetLastError();
}

template <typename R, int GY, int GZ, int NP>
static cudaError_t current_march_yh(System& s, const Nab12& nab, double* out) {
  k_current_march_yh<R, GY, GZ, NP><<<NP * s.norb, GY / NP * GZ, 0, s.launch_stream()>>>((const C2<R>*)s.zu, s.NLx,
                                                                                          nab, out);
  return cudaGetLastError();
}

// Planes of more than 1024 points: one CTA per (orbital, x-plane), the
// neighbours read through L1/L2 (CTAs of one orbital are adjacent in launch
// order, so the x-planes ahead are L2 hits); part[o][x][4].
template <typename R>
__global__ void __launch_bounds__(256, 2) k_current_plane(const C2<R>* __restrict__ zu, int NLx, int NLy, int NLz,
                                                           const double* __restrict__ nab12, double* __restrict__ part) {
  __shared__ double sh[32 * 4];
  const int o = blockIdx.x / NLx, x = blockIdx.x - (blockIdx.x / NLx) * NLx;
  const int NYZ = NLy * NLz;
  const C2<R>* E = zu + (size_t)o * NLx * NYZ;
  const C2<R>* P0 = E + (size_t)x * NYZ;
  const C2<R>* Px[4];
#pragma unroll
  for (int n = 1; n <= 4; ++n) {
    int xn = x + n;
    while (xn >= NLx) xn -= NLx;
    Px[n - 1] = E + (size_t)xn * NYZ;
  }
  double nb[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) nb[k] = nab12[k];
  double v[4] = {0, 0, 0, 0};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int y = warp; y < NLy; y += nw) {
    int yr[4];
#pragma unroll
    for (int n = 1; n <= 4; ++n) {
      int yn = y + n;
      while (yn >= NLy) yn -= NLy;
      yr[n - 1] = yn * NLz;
    }
    for (int z = lane; z < NLz; z += 32) {
      const int i = y * NLz + z;
      const double2 e = to_d2(__ldg(P0 + i));
      v[0] += e.x * e.x + e.y * e.y;
      double2 sx = make_double2(0, 0), sy = make_double2(0, 0), sz = make_double2(0, 0);
#pragma unroll
      for (int n = 1; n <= 4; ++n) {
        int zn = z + n;
        while (zn >= NLz) zn -= NLz;
        const double2 ex = to_d2(__ldg(Px[n - 1] + i));
        const double2 ey = to_d2(__ldg(P0 + yr[n - 1] + z));
        const double2 ez = to_d2(__ldg(P0 + y * NLz + zn));
        sx.x += nb[n - 1] * ex.x; sx.y += nb[n - 1] * ex.y;
        sy.x += nb[3 + n] * ey.x; sy.y += nb[3 + n] * ey.y;
        sz.x += nb[7 + n] * ez.x; sz.y += nb[7 + n] * ez.y;
      }
      v[1] += e.x * sx.y - e.y * sx.x;
      v[2] += e.x * sy.y - e.y * sy.x;
      v[3] += e.x * sz.y - e.y * sz.x;
    }
  }
  block_sum<4>(v, sh);
  if (threadIdx.x == 0) {
    double* d = part + ((size_t)o * NLx + x) * 4;
    d[0] = v[0];
    d[1] = v[1];
    d[2] = v[2];
    d[3] = v[3];
  }
}

// Weighted projections for the nonlocal current (current.f90:247-265):
// Uw[o][ilma][w] = sum_j conj(zproj(j,ilma,k)) r_w(j) psi(J(j)), r = (1, x, y, z).
// psi(J(j)) is read from src[o*ld + idx[j]]: the compact sphere values S with
// the sphere-point map qmap when they are current, else the orbitals with the
// grid index idx_proj.
// One CTA per (projector item, k-point, group of up to 32 bands of that k-point,
// part of the item's points): the points are split into nsplit contiguous ranges
// of UVW_CH-point chunks so that the grid fills the GPU, and each range writes its
// own partial Uw[part][o][ilma][w] (k_current_comb adds the parts in order).  Per
// chunk, conj(zproj) of the item's projectors, the weights r and the bands' values
// are staged in shared memory (band rows padded by one element: the eight band
// rows a warp reads at one point fall in distinct banks).  Thread (lane, warp)
// takes bands bg, bg+8, bg+16, bg+24 (bg = lane & 7) of projector lane >> 3 over
// every eighth point of the chunk: t = conj(zproj) psi once, then
// Uw[., 0] += t, Uw[., w] += r_w t (12 FP64 operations a band and point instead
// of the 16 of four complex products), and the eight warps' sums are added in
// a fixed order.
constexpr int UVW_CH = 128;
template <typename R> struct UvwGeom {
  static constexpr int SROW = UVW_CH + 1;  // padded band row
  static constexpr size_t stage = sizeof(C2<R>) * 32 * SROW + sizeof(double2) * 4 * UVW_CH +
                                  sizeof(double) * 3 * UVW_CH + sizeof(int) * UVW_CH;
  static constexpr size_t red = sizeof(double2) * 8 * 32 * 9;  // the part sums, eight entries (+1 pad) at a time
  static constexpr size_t smem = stage > red ? stage : red;
};

template <typename R>
__global__ void __launch_bounds__(256, 2) k_uvpsi_w(const C2<R>* __restrict__ src, int ld, int NBocc,
                                                     const double2* __restrict__ zproj, int Nlma, int Nps,
                                                     const int* __restrict__ idx, const int* __restrict__ atom_off,
                                                     const double* __restrict__ rpos, const int4* __restrict__ items,
                                                     const int* __restrict__ lma_list, int nsplit, int norb,
                                                     double2* __restrict__ Uw) {
  constexpr int CH = UVW_CH, SROW = UvwGeom<R>::SROW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C2<R>* ps = reinterpret_cast<C2<R>*>(smem_raw);                          // [32][SROW] band values
  double2* cz = reinterpret_cast<double2*>(ps + 32 * SROW);                // [4][CH] conj(zproj)
  double* rw = reinterpret_cast<double*>(cz + 4 * CH);                     // [CH][3] weights x, y, z
  int* is = reinterpret_cast<int*>(rw + 3 * CH);                           // [CH] gather index
  double2* red = reinterpret_cast<double2*>(smem_raw);                     // [8][32][9] after the sums
  const int t = threadIdx.x, lane = t & 31, part = t >> 5;
  const int bg = lane & 7, pg = lane >> 3;  // bands bg + 8i, projector pg (its 4 weights)
  const int4 item = items[blockIdx.x];
  const int kl = blockIdx.y, b0 = (blockIdx.z / nsplit) * 32, split = blockIdx.z - (blockIdx.z / nsplit) * nsplit;
  const int a = item.x, l0 = item.y, np = item.z;
  const int p0 = atom_off[a], mps = atom_off[a + 1] - p0;
  const int nbr = min(32, NBocc - b0);
  if (nbr <= 0) return;  // whole CTA leaves together
  const int nch = (mps + CH - 1) / CH, cps = (nch + nsplit - 1) / nsplit;
  const int cbeg = min(nch, split * cps), cend = min(nch, cbeg + cps);  // may be empty: zeros are written
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int w = 0; w < 4; ++w) acc[i][w] = make_double2(0.0, 0.0);
  for (int c = cbeg; c < cend; ++c) {
    const int c0 = c * CH, len = min(CH, mps - c0);
    __syncthreads();  // the previous chunk is no longer read
    for (int q = t; q < 4 * CH; q += 256) {  // conj(zproj) of point j, projector p
      const int p = q / CH, j = q - p * CH;
      double2 z = make_double2(0.0, 0.0);
      if (j < len && p < np) z = zproj[((size_t)kl * Nlma + lma_list[l0 + p]) * Nps + c0 + j];
      cz[p * CH + j] = make_double2(z.x, -z.y);
      if (p == 0) {
        const double* r = rpos + 3 * (size_t)(p0 + c0 + j);
        rw[3 * j] = j < len ? r[0] : 0.0;
        rw[3 * j + 1] = j < len ? r[1] : 0.0;
        rw[3 * j + 2] = j < len ? r[2] : 0.0;
        is[j] = j < len ? idx[p0 + c0 + j] : 0;
      }
    }
    __syncthreads();
    const int tot = 32 * len;
    for (int q0 = t; q0 < tot; q0 += 8 * 256) {
      C2<R> vals[8];
      int slot[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int q = q0 + u * 256;
        slot[u] = -1;
        if (q < tot) {
          const int bb = q / len, j = q - bb * len;
          slot[u] = bb * SROW + j;
          vals[u] = bb < nbr ? __ldg(src + (size_t)(kl * NBocc + b0 + bb) * ld + is[j]) : C2<R>{};
        }
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (slot[u] >= 0) ps[slot[u]] = vals[u];
    }
    __syncthreads();
    for (int j = part; j < len; j += 8) {
      const double2 zc = cz[pg * CH + j];
      const double r1 = rw[3 * j], r2 = rw[3 * j + 1], r3 = rw[3 * j + 2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const double2 e = to_d2(ps[(bg + 8 * i) * SROW + j]);
        const double tx = fma(zc.x, e.x, -zc.y * e.y), ty = fma(zc.x, e.y, zc.y * e.x);
        acc[i][0].x += tx;
        acc[i][0].y += ty;
        acc[i][1].x = fma(r1, tx, acc[i][1].x);
        acc[i][1].y = fma(r1, ty, acc[i][1].y);
        acc[i][2].x = fma(r2, tx, acc[i][2].x);
        acc[i][2].y = fma(r2, ty, acc[i][2].y);
        acc[i][3].x = fma(r3, tx, acc[i][3].x);
        acc[i][3].y = fma(r3, ty, acc[i][3].y);
      }
    }
  }
  // the eight warps' sums, eight of a thread's sixteen entries at a time
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    __syncthreads();  // the staging buffers (or the previous half) are no longer read
#pragma unroll
    for (int k = 0; k < 8; ++k) red[(part * 32 + lane) * 9 + k] = acc[2 * half + k / 4][k % 4];
    __syncthreads();
    {  // thread (lane', k): entry k of lane' summed over the parts in order
      const int ln = t >> 3, k = t & 7;
      double2 sum = make_double2(0.0, 0.0);
#pragma unroll
      for (int pp = 0; pp < 8; ++pp) {
        const double2 v = red[(pp * 32 + ln) * 9 + k];
        sum.x += v.x;
        sum.y += v.y;
      }
      const int tb = ln & 7, tp = ln >> 3, i = 2 * half + k / 4, w = k & 3;
      const int b = tb + 8 * i;
      if (tp < np && b < nbr)
        Uw[(((size_t)split * norb + kl * NBocc + b0 + b) * Nlma + lma_list[l0 + tp]) * 4 + w] = sum;
    }
  }
}

// Per orbital, combines the plane sums and the weighted projections exactly as
// current() does (current.f90:182-273): jo[o][d].
// One warp per orbital: lane l takes projectors l, l+32, ... in order, the lanes'
// nonlocal sums are added by a fixed butterfly, and lane 0 adds the plane sums.
constexpr int COMB_T = 256;
__global__ void __launch_bounds__(COMB_T) k_current_comb(const double* __restrict__ part, int nx,
                                                        const double2* __restrict__ Uw, int nsplit,
                                                        const double* __restrict__ occ_o,
                                                        const double* __restrict__ kAc, const int* __restrict__ iuV,
                                                        int norb, int NBocc, int Nlma, double Hxyz, double IaLxyz,
                                                        double* __restrict__ jo) {
  const int o = blockIdx.x * (COMB_T / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (o >= norb) return;  // whole warp
  const double occ = occ_o[o];
  double jn[3] = {0, 0, 0};
  for (int l = lane; l < Nlma; l += 32) {
    double2 u[4];  // the point-range parts of k_uvpsi_w, added in order
#pragma unroll
    for (int w = 0; w < 4; ++w) u[w] = Uw[((size_t)o * Nlma + l) * 4 + w];
    for (int sp = 1; sp < nsplit; ++sp)
#pragma unroll
      for (int w = 0; w < 4; ++w) {
        const double2 v = Uw[(((size_t)sp * norb + o) * Nlma + l) * 4 + w];
        u[w].x += v.x;
        u[w].y += v.y;
      }
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
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) jn[d] += __shfl_xor_sync(0xffffffffu, jn[d], off);
  if (lane == 0) {
    double v[4] = {0, 0, 0, 0};
    for (int x = 0; x < nx; ++x) {  // per-orbital rows of partial sums, in order
      const double* d = part + ((size_t)o * nx + x) * 4;
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] += d[k];
    }
    const int kl = o / NBocc;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double j = occ * kAc[3 * kl + d] * v[0] + 2.0 * v[1 + d] * occ;
      jo[3 * (size_t)o + d] = j * Hxyz * IaLxyz + jn[d];
    }
  }
}

// sum over orbitals in a fixed order
__global__ void k_current_sum(const double* __restrict__ jo, int norb, double* __restrict__ jav) {
  __shared__ double sh[32 * 3];
  double v[3] = {0, 0, 0};
  for (int o = threadIdx.x; o < norb; o += blockDim.x) {
#pragma unroll
    for (int d = 0; d < 3; ++d) v[d] += jo[3 * (size_t)o + d];
  }
  block_sum<3>(v, sh);
  if (threadIdx.x == 0) {
    jav[0] = v[0];
    jav[1] = v[1];
    jav[2] = v[2];
  }
}


// scratch of launch_current (part [norb][NLx][4], jo [norb][3], 12 coefficients)
// and of launch_energy (part [norb][NLx][2], eo [norb][2], 25 coefficients)
size_t current_red_elems(int norb, int NLx) { return (size_t)norb * NLx * 4 + 3 * (size_t)norb + 32; }

template <typename R, int NT, int P, int D, int GY = 0, int GZ = 0, int MB = 1>
static cudaError_t current_march(System& s, const Nab12& nab, double* out) {
  const size_t smem = 2 * (size_t)s.NLy * s.NLz * sizeof(double2);
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(k_current_march<R, NT, P, D, GY, GZ, MB>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_current_march<R, NT, P, D, GY, GZ, MB><<<s.norb, NT, smem, s.launch_stream()>>>((const C2<R>*)s.zu, s.NLx, s.NLy,
                                                                                    s.NLz, nab, out);
  return cudaGetLastError();
}

// the x-marching form up to 1024 points per plane (one point per thread, up to
// 1024 threads within 64 registers: the coefficients live in the parameter
// bank), the plane-parallel form beyond.  Measured at 32^3 x 2048 orbitals
// (complex(4)): 0.60 ms, against 0.61 ms with 512 threads x 2 points and 0.69 ms
// with 256 x 4 (spills).
template <typename R>
static cudaError_t current_stencil(System& s, const Nab12& nab, const double* nab12, double* part, int& nx) {
  const int NYZ = s.NLy * s.NLz;
  nx = 1;
  // 32x32 planes: two CTAs of 16 rows per orbital plane, two rows per thread at
  // three CTAs per SM (value 2: four CTAs of 8 rows, one row per thread).
  // At 32^3 x 2048 orbitals, complex(4): 0.328 against 0.388 ms; two rows per
  // thread at 118 registers (two CTAs per SM) 0.709 ms, one CTA per plane 0.344 ms
  // (complex(8): 0.394 / 0.403 / 0.642 / 0.423 ms)
  if (s.cur_fixed && s.NLy == 32 && s.NLz == 32) {
    if (s.cur_fixed == 2) {
      nx = 4;
      return current_march_yh<R, 32, 32, 4>(s, nab, part);
    }
    nx = 2;
    return current_march_y2<R, 32, 32, 2, 3>(s, nab, part);
  }
  // 48x48 planes (the 48^3 grid): six CTAs of 8 rows per orbital plane (two rows per
  // thread, 192 threads; value 2: one row per thread, 384 threads): 0.284 against
  // 0.313 ms at 432 orbitals, complex(4); 0.298 against 0.328 ms complex(8)
  if (s.cur_fixed && s.NLy == 48 && s.NLz == 48) {
    nx = 6;
    return s.cur_fixed == 2 ? current_march_yh<R, 48, 48, 6>(s, nab, part) : current_march_y2<R, 48, 48, 6>(s, nab, part);
  }
  if (NYZ <= 256) return current_march<R, 256, 1, 1>(s, nab, part);
  if (NYZ <= 512) return current_march<R, 512, 1, 1>(s, nab, part);
  if (NYZ <= 1024) return current_march<R, 1024, 1, 1>(s, nab, part);
  nx = s.NLx;
  k_current_plane<R><<<s.norb * s.NLx, 256, 0, s.launch_stream()>>>((const C2<R>*)s.zu, s.NLx, s.NLy, s.NLz, nab12,
                                                                     part);
  return cudaGetLastError();
}

// The stencil sums {jt, F, G, H} of the resident orbitals into part[o][nx][4].
// The 12 nab coefficients of the plane form live at the end of the handle's
// reduction scratch.
cudaError_t launch_current_stencil(System& s, double* part, int& nx) {
  Nab12 nab;
  for (int n = 0; n < 4; ++n)
    for (int d = 0; d < 3; ++d) nab.v[4 * d + n] = s.nab[d][n + 1];
  nx = 1;
  // s.nab12 (device, set at creation) for the plane form; no scratch shared with
  // work that may run beside this on the handle's other stream
  return s.prec == SGPU_PREC_C64 ? current_stencil<float>(s, nab, s.nab12, part, nx)
                                 : current_stencil<double>(s, nab, s.nab12, part, nx);
}

// The weighted projections of the nonlocal current, Uw[o][ilma][w]
// (current.f90:225-273), from the sphere values when they are current.
cudaError_t launch_current_proj(System& s) {
  if (!s.Nlma || !s.nitems) return cudaSuccess;
  cudaError_t e;
  const size_t smem = s.prec == SGPU_PREC_C64 ? UvwGeom<float>::smem : UvwGeom<double>::smem;
  if (smem > 48 * 1024) {  // set on every call: the attribute is per device
    e = s.prec == SGPU_PREC_C64
            ? cudaFuncSetAttribute(k_uvpsi_w<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
            : cudaFuncSetAttribute(k_uvpsi_w<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const dim3 gu(s.nitems, s.nkl, (s.NBocc + 31) / 32 * s.uvw_split);
  // the compact sphere values are current after every Taylor step: 4x fewer bytes than gathering from zu
  const bool fromS = s.S_valid && s.Sbuf;
  const int ld = fromS ? s.nsp : s.NL;
  const int* idx = fromS ? s.qmap : s.idx_proj;
  if (s.prec == SGPU_PREC_C64)
    k_uvpsi_w<float><<<gu, 256, smem, s.launch_stream()>>>(fromS ? (const float2*)s.Sbuf : (const float2*)s.zu, ld,
                                                            s.NBocc, s.zproj64, s.Nlma, s.Nps, idx, s.atom_off,
                                                            s.rpos, s.items, s.lma_list, s.uvw_split, s.norb,
                                                            s.Uw);
  else
    k_uvpsi_w<double><<<gu, 256, smem, s.launch_stream()>>>(fromS ? (const double2*)s.Sbuf : (const double2*)s.zu,
                                                             ld, s.NBocc, s.zproj64, s.Nlma, s.Nps, idx, s.atom_off,
                                                             s.rpos, s.items, s.lma_list, s.uvw_split, s.norb,
                                                            s.Uw);
  return cudaGetLastError();
}

cudaError_t launch_current(System& s, double* jav_dev) {
  double* part = s.red;                              // [norb][nx][4]
  double* jo = part + (size_t)s.norb * s.NLx * 4;    // [norb][3]
  if ((size_t)s.norb * s.NLx * 4 + 3 * (size_t)s.norb + 12 > s.red_elems) return cudaErrorInvalidValue;
  int nx = 1;
  cudaError_t e;
  if (!s.cur_valid) {
    e = launch_current_stencil(s, part, nx);
    if (e != cudaSuccess) return e;
  }
  if ((e = launch_current_proj(s)) != cudaSuccess) return e;
  if (s.cur_valid) {  // computed by the Taylor step that produced these orbitals (flag_current),
    // on the second stream: the projections above overlap them; the sums wait here
    e = s.aux_join();
    if (e != cudaSuccess) return e;
    part = s.cur_part;
    nx = s.cur_nx;
  }
  k_current_comb<<<(s.norb + COMB_T / 32 - 1) / (COMB_T / 32), COMB_T, 0, s.launch_stream()>>>(part, nx, s.Uw, s.uvw_split, s.occ_o, s.kAc_d, s.iuV_d,
                                                                     s.norb, s.NBocc, s.Nlma, s.Hxyz, 1.0 / s.aLxyz,
                                                                     jo);
  k_current_sum<<<1, 256, 0, s.launch_stream()>>>(jo, s.norb, jav_dev);
  return cudaGetLastError();
}

// -------------------------------------------------------------- energy ---
// tpsum = sum conj(psi) (lap0_2 psi - 0.5 v - i w)  (stencil/F90/total_energy.f90:93-180)
// One CTA per (orbital, x-plane), planes of an orbital adjacent in launch
// order (the neighbour planes are L2 hits), laid out like k_current_plane; the plane's
// two sums go to part[o][x][2] and are added in plane order by k_energy_comb.
template <typename R>
__global__ void __launch_bounds__(256, 2) k_ekin_plane(const C2<R>* __restrict__ zu, int NLx, int NLy, int NLz,
                                                        int NBocc, const double* __restrict__ kAc,
                                                        const double* __restrict__ coef, double* __restrict__ part) {
  __shared__ double sh[32 * 2];
  const int o = blockIdx.x / NLx, x = blockIdx.x - (blockIdx.x / NLx) * NLx, kl = o / NBocc;
  const int NYZ = NLy * NLz;
  const C2<R>* E = zu + (size_t)o * NLx * NYZ;
  const C2<R>* P0 = E + (size_t)x * NYZ;
  const C2<R>* Pp[4];
  const C2<R>* Pm[4];
#pragma unroll
  for (int n = 1; n <= 4; ++n) {
    int xp = x + n, xm = x - n;
    while (xp >= NLx) xp -= NLx;
    while (xm < 0) xm += NLx;
    Pp[n - 1] = E + (size_t)xp * NYZ;
    Pm[n - 1] = E + (size_t)xm * NYZ;
  }
  // coef: [0] = lap0_2, [1..12] = lapt, [13..24] = nab
  const double A = coef[0];
  double lapt[12], nabt[12];
#pragma unroll
  for (int n = 0; n < 12; ++n) {
    lapt[n] = coef[1 + n];
    nabt[n] = kAc[3 * kl + n / 4] * coef[13 + n];
  }
  double v2[2] = {0, 0};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int y = warp; y < NLy; y += nw) {
    int yp[4], ym[4];
#pragma unroll
    for (int n = 1; n <= 4; ++n) {
      int a = y + n, b = y - n;
      while (a >= NLy) a -= NLy;
      while (b < 0) b += NLy;
      yp[n - 1] = a * NLz;
      ym[n - 1] = b * NLz;
    }
    for (int z = lane; z < NLz; z += 32) {
      const int i = y * NLz + z;
      const double2 e = to_d2(__ldg(P0 + i));
      double2 v = make_double2(0, 0), w = make_double2(0, 0);
#pragma unroll
      for (int n = 1; n <= 4; ++n) {
        int zp = z + n, zm = z - n;
        while (zp >= NLz) zp -= NLz;
        while (zm < 0) zm += NLz;
        const double2 a1 = to_d2(__ldg(Pp[n - 1] + i)), a2 = to_d2(__ldg(Pm[n - 1] + i));
        const double2 b1 = to_d2(__ldg(P0 + yp[n - 1] + z)), b2 = to_d2(__ldg(P0 + ym[n - 1] + z));
        const double2 c1 = to_d2(__ldg(P0 + y * NLz + zp)), c2 = to_d2(__ldg(P0 + y * NLz + zm));
        v.x += lapt[n - 1] * (a1.x + a2.x) + lapt[3 + n] * (b1.x + b2.x) + lapt[7 + n] * (c1.x + c2.x);
        v.y += lapt[n - 1] * (a1.y + a2.y) + lapt[3 + n] * (b1.y + b2.y) + lapt[7 + n] * (c1.y + c2.y);
        w.x += nabt[n - 1] * (a1.x - a2.x) + nabt[3 + n] * (b1.x - b2.x) + nabt[7 + n] * (c1.x - c2.x);
        w.y += nabt[n - 1] * (a1.y - a2.y) + nabt[3 + n] * (b1.y - b2.y) + nabt[7 + n] * (c1.y - c2.y);
      }
      // z = A e - 0.5 v - i w ;  F += conj(e) z
      const double2 zz = make_double2(A * e.x - 0.5 * v.x + w.y, A * e.y - 0.5 * v.y - w.x);
      v2[0] += e.x * zz.x + e.y * zz.y;
      v2[1] += e.x * zz.y - e.y * zz.x;
    }
  }
  block_sum<2>(v2, sh);
  if (threadIdx.x == 0) {
    part[((size_t)o * NLx + x) * 2] = v2[0];
    part[((size_t)o * NLx + x) * 2 + 1] = v2[1];
  }
}

// The energy stencil as an x-march (GY x GZ planes split over NP CTAs of GY/NP
// rows, one point per thread): psi at planes x-4..x+4 in a register queue
// (FP64, converted once), plane x staged in FP64 in shared memory with four halo
// rows on each side for the +-y neighbours.  The FD coefficients are kernel
// parameters; k enters through nabt = k_d nab_d.  part[o][h][2].
struct EkinCoef {
  double lap0_2;     // -(lapx(0)+lapy(0)+lapz(0))/2
  double lapt[12];   // lapx(1:4), lapy(1:4), lapz(1:4)
  double nab[12];    // nabx(1:4), naby(1:4), nabz(1:4)
};

template <typename R, int GY, int GZ, int NP>
__global__ void __launch_bounds__(GY / NP * GZ) k_ekin_march_yh(const C2<R>* __restrict__ zu, int NLx, int NBocc,
                                                               const double* __restrict__ kAc, const EkinCoef c,
                                                               double* __restrict__ out) {
  constexpr int NYH = GY / NP, NT = NYH * GZ, NYZ = GY * GZ, RB = (NYH + 8) * GZ;
  static_assert(NT % 32 == 0 && NT <= 1024 && 8 * GZ <= NT, "one point per thread, halos loaded by the first rows");
  __shared__ double2 buf[2][RB];
  __shared__ double sh[32 * 2];
  const int o = blockIdx.x / NP, h = blockIdx.x - (blockIdx.x / NP) * NP, t = threadIdx.x;
  const int kl = o / NBocc;
  const C2<R>* E = zu + (size_t)o * NLx * NYZ;
  double nabt[12];
#pragma unroll
  for (int n = 0; n < 12; ++n) nabt[n] = kAc[3 * kl + n / 4] * c.nab[n];
  const int yl = t / GZ, z = t - (t / GZ) * GZ;
  const int y0 = h * NYH;
  const int own = (y0 + yl) * GZ + z;
  // halo rows of threads t < 8 GZ: rows y0-4..y0-1 then y0+NYH..y0+NYH+3
  const int hr = t / GZ;
  const int hrow = hr < 4 ? (y0 - 4 + hr + GY) % GY : (y0 + NYH + hr - 4) % GY;
  const int hdst = (hr < 4 ? hr : NYH + hr) * GZ + z;
  const int hsrc = hrow * GZ + z;
  double2 q[9];  // q[m]: plane x-4+m
#pragma unroll
  for (int m = 0; m < 9; ++m) q[m] = to_d2(__ldg(E + (size_t)((m - 4 + 4 * NLx) % NLx) * NYZ + own));
  C2<R> nxt = __ldg(E + (size_t)(5 % NLx) * NYZ + own);
  double v2[2] = {0, 0};
  for (int x = 0; x < NLx; ++x) {
    double2* pl = buf[x & 1];
    pl[(4 + yl) * GZ + z] = q[4];
    if (t < 8 * GZ) pl[hdst] = to_d2(__ldg(E + (size_t)x * NYZ + hsrc));
    __syncthreads();
    const double2 e = q[4];
    double2 v = make_double2(0, 0), w = make_double2(0, 0);
#pragma unroll
    for (int n = 1; n <= 4; ++n) {
      const double2 a1 = q[4 + n], a2 = q[4 - n];
      const double2 b1 = pl[(4 + yl + n) * GZ + z], b2 = pl[(4 + yl - n) * GZ + z];
      const double2 c1 = pl[(4 + yl) * GZ + (z + n) % GZ], c2 = pl[(4 + yl) * GZ + (z - n + GZ) % GZ];
      v.x += c.lapt[n - 1] * (a1.x + a2.x) + c.lapt[3 + n] * (b1.x + b2.x) + c.lapt[7 + n] * (c1.x + c2.x);
      v.y += c.lapt[n - 1] * (a1.y + a2.y) + c.lapt[3 + n] * (b1.y + b2.y) + c.lapt[7 + n] * (c1.y + c2.y);
      w.x += nabt[n - 1] * (a1.x - a2.x) + nabt[3 + n] * (b1.x - b2.x) + nabt[7 + n] * (c1.x - c2.x);
      w.y += nabt[n - 1] * (a1.y - a2.y) + nabt[3 + n] * (b1.y - b2.y) + nabt[7 + n] * (c1.y - c2.y);
    }
    // z = A e - 0.5 v - i w ;  F += conj(e) z
    const double2 zz = make_double2(c.lap0_2 * e.x - 0.5 * v.x + w.y, c.lap0_2 * e.y - 0.5 * v.y - w.x);
    v2[0] += e.x * zz.x + e.y * zz.y;
    v2[1] += e.x * zz.y - e.y * zz.x;
#pragma unroll
    for (int m = 0; m < 8; ++m) q[m] = q[m + 1];
    q[8] = to_d2(nxt);
    nxt = __ldg(E + (size_t)((x + 6) % NLx) * NYZ + own);
  }
  block_sum<2>(v2, sh);
  if (t == 0) {
    out[2 * (size_t)blockIdx.x] = v2[0];
    out[2 * (size_t)blockIdx.x + 1] = v2[1];
  }
}

// per orbital: occ Re(tpsum) Hxyz + occ |k|^2/2 and occ sum |U|^2 iuV
__global__ void k_energy_comb(const double* __restrict__ part, int nx, const double2* __restrict__ U,
                              const double* __restrict__ occ_o, const double* __restrict__ kAc,
                              const int* __restrict__ iuV, int norb, int NBocc, int Nlma, double Hxyz,
                              double* __restrict__ eo) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= norb) return;
  double tr = 0;
  for (int x = 0; x < nx; ++x) tr += part[((size_t)o * nx + x) * 2];  // per-orbital rows, in order
  const int kl = o / NBocc;
  const double occ = occ_o[o];
  const double k2 = kAc[3 * kl] * kAc[3 * kl] + kAc[3 * kl + 1] * kAc[3 * kl + 1] + kAc[3 * kl + 2] * kAc[3 * kl + 2];
  double en = 0;
  for (int l = 0; l < Nlma; ++l) {
    const double2 u = U[(size_t)o * Nlma + l];      // Hxyz * sum uV ekr psi
    en += occ * (u.x * u.x + u.y * u.y) * (double)iuV[l];
  }
  eo[2 * (size_t)o] = occ * tr * Hxyz + occ * k2 / 2.0;   // real part of occ*tpsum*Hxyz + occ*|k|^2/2
  eo[2 * (size_t)o + 1] = en;
}

__global__ void k_energy_sum(const double* __restrict__ eo, int norb, double* __restrict__ e) {
  __shared__ double sh[32 * 2];
  double v[2] = {0, 0};
  for (int o = threadIdx.x; o < norb; o += blockDim.x) {
    v[0] += eo[2 * (size_t)o];
    v[1] += eo[2 * (size_t)o + 1];
  }
  block_sum<2>(v, sh);
  if (threadIdx.x == 0) {
    e[0] = v[0];
    e[1] = v[1];
  }
}

cudaError_t launch_energy(System& s, double* e_dev) {
  double* part = s.red;                                // [norb][NLx][2]
  double* eo = part + 2 * (size_t)s.norb * s.NLx;      // [norb][2]
  double* coef = eo + 2 * (size_t)s.norb;              // [25]
  if (2 * (size_t)s.norb * s.NLx + 2 * (size_t)s.norb + 32 > s.red_elems) return cudaErrorInvalidValue;
  double h[25];
  h[0] = -(s.lap[0][0] + s.lap[1][0] + s.lap[2][0]) * 0.5;
  for (int d = 0; d < 3; ++d)
    for (int n = 0; n < 4; ++n) {
      h[1 + 4 * d + n] = s.lap[d][n + 1];
      h[13 + 4 * d + n] = s.nab[d][n + 1];
    }
  cudaError_t err = cudaMemcpyAsync(coef, h, sizeof(h), cudaMemcpyHostToDevice, s.stream);
  if (err != cudaSuccess) return err;
  int nx = s.NLx;
  EkinCoef ec;
  ec.lap0_2 = h[0];
  for (int k = 0; k < 12; ++k) {
    ec.lapt[k] = h[1 + k];
    ec.nab[k] = h[13 + k];
  }
  // 32x32 and 48x48 planes: the x-march over planes split in 8-row parts (SGPU_PARAM_CUR_FIXED)
  if (s.cur_fixed && s.NLy == 32 && s.NLz == 32) {
    nx = 4;
    if (s.prec == SGPU_PREC_C64)
      k_ekin_march_yh<float, 32, 32, 4><<<4 * s.norb, 256, 0, s.launch_stream()>>>((const float2*)s.zu, s.NLx, s.NBocc,
                                                                                   s.kAc_d, ec, part);
    else
      k_ekin_march_yh<double, 32, 32, 4><<<4 * s.norb, 256, 0, s.launch_stream()>>>((const double2*)s.zu, s.NLx,
                                                                                    s.NBocc, s.kAc_d, ec, part);
  } else if (s.cur_fixed && s.NLy == 48 && s.NLz == 48) {
    nx = 6;
    if (s.prec == SGPU_PREC_C64)
      k_ekin_march_yh<float, 48, 48, 6><<<6 * s.norb, 384, 0, s.launch_stream()>>>((const float2*)s.zu, s.NLx, s.NBocc,
                                                                                   s.kAc_d, ec, part);
    else
      k_ekin_march_yh<double, 48, 48, 6><<<6 * s.norb, 384, 0, s.launch_stream()>>>((const double2*)s.zu, s.NLx,
                                                                                    s.NBocc, s.kAc_d, ec, part);
  } else {
    const int gp = s.norb * s.NLx;
    const int bt = s.NLy >= 8 ? 256 : 32 * s.NLy;
    if (s.prec == SGPU_PREC_C64)
      k_ekin_plane<float><<<gp, bt, 0, s.launch_stream()>>>((const float2*)s.zu, s.NLx, s.NLy, s.NLz, s.NBocc, s.kAc_d,
                                                            coef, part);
    else
      k_ekin_plane<double><<<gp, bt, 0, s.launch_stream()>>>((const double2*)s.zu, s.NLx, s.NLy, s.NLz, s.NBocc,
                                                             s.kAc_d, coef, part);
  }
  err = cudaGetLastError();
  if (err != cudaSuccess) return err;
  // U = Hxyz * sum conj(zproj) psi = Hxyz * sum uV ekr psi  (total_energy.f90:191-197), FP64 projectors
  if (s.Nlma) {
    err = launch_uvpsi(s, s.zu, 0, s.norb, s.NBocc, false);
    if (err != cudaSuccess) return err;
  }
  k_energy_comb<<<(s.norb + 127) / 128, 128, 0, s.launch_stream()>>>(part, nx, s.U, s.occ_o, s.kAc_d, s.iuV_d,
                                                                    s.norb, s.NBocc, s.Nlma, s.Hxyz, eo);
  k_energy_sum<<<1, 256, 0, s.launch_stream()>>>(eo, s.norb, e_dev);
  return cudaGetLastError();
}

}  // namespace sgpu
