// Batched 3D FFTs of grid functions and the Teter-Payne-Allan kinetic-energy
// preconditioner applied with them (ground-state CG).
//
// The FFT is a mixed-radix (2, 3) Stockham autosort transform of every line
// along one axis, in shared memory, FP64; a 3D transform is three axis passes.
// Grid sizes must be of the form 2^a 3^b (16, 24, 32, 48, 64, ...), at most
// FFT_NMAX points per axis.
//
// Teter, Payne and Allan, Phys. Rev. B 40, 12255 (1989): the residual is
// multiplied in reciprocal space by
//     K(x) = (27 + 18x + 12x^2 + 8x^3) / (27 + 18x + 12x^2 + 8x^3 + 16x^4),
// x = T(G) / T_band, with T(G) the kinetic energy of the plane wave G at k and
// T_band the kinetic energy of the band being optimised.  T(G) is taken as the
// symbol of the finite-difference kinetic operator of hpsi (the Nd=4
// Laplacian and the k.nabla term on this grid), so that K is consistent with
// the H that CG minimises.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "sgpu_internal.cuh"

namespace sgpu {

constexpr int FFT_NMAX = 96;  // 2 x 16 lines x 96 x 16 B = 48 KB of shared memory
constexpr int FFT_TL = 16;       // lines per CTA
constexpr int FFT_THREADS = 256;

bool fft_size_ok(int n) {
  if (n < 1 || n > FFT_NMAX) return false;
  while (n % 2 == 0) n /= 2;
  while (n % 3 == 0) n /= 3;
  return n == 1;
}

// Lines of one axis: line L of vector v = (lo, li) with L = lo*ninner + li;
// element t sits at v*NL + lo*lo_stride + li + t*stride.
struct FftAxis {
  int n, nlines, ninner, lo_stride, stride;
  bool rows;  // the axis is the contiguous one (load whole rows)
};

__global__ void __launch_bounds__(FFT_THREADS) k_fft_lines(double2* __restrict__ data, int NL, FftAxis ax, int sign,
                                                            double scale) {
  extern __shared__ double2 fsm[];
  const int n = ax.n;
  double2* x = fsm;
  double2* y = fsm + FFT_TL * n;
  const int v = blockIdx.y;
  const int L0 = blockIdx.x * FFT_TL;
  const int nl = min(FFT_TL, ax.nlines - L0);
  double2* base = data + (size_t)v * NL;
  auto addr = [&](int l, int t) -> size_t {
    const int L = L0 + l;
    const int lo = L / ax.ninner, li = L - lo * ax.ninner;
    return (size_t)lo * ax.lo_stride + li + (size_t)t * ax.stride;
  };
  // load: coalesced along the contiguous direction of memory
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    int l, t;
    if (ax.rows) { l = e / n; t = e - l * n; } else { t = e / nl; l = e - t * nl; }
    x[l * n + t] = base[addr(l, t)];
  }
  __syncthreads();
  int Ns = 1;
  int m = n;
  while (m > 1) {
    const int R = (m % 2 == 0) ? 2 : 3;
    m /= R;
    const int nR = n / R;
    for (int e = threadIdx.x; e < nl * nR; e += blockDim.x) {
      const int l = e / nR, j = e - l * nR;
      const int k = j % Ns;
      const double2* xl = x + l * n;
      double2* yl = y + l * n;
      // twiddle exp(sign * 2 pi i k r / (Ns R)) for r = 1..R-1
      double s1, c1;
      sincospi(2.0 * sign * k / (double)(Ns * R), &s1, &c1);
      const int idx = (j / Ns) * Ns * R + k;
      if (R == 2) {
        const double2 a = xl[j];
        const double2 b0 = xl[j + nR];
        const double2 b = make_double2(b0.x * c1 - b0.y * s1, b0.x * s1 + b0.y * c1);
        yl[idx] = make_double2(a.x + b.x, a.y + b.y);
        yl[idx + Ns] = make_double2(a.x - b.x, a.y - b.y);
      } else {
        const double c2 = c1 * c1 - s1 * s1, s2 = 2.0 * s1 * c1;
        const double2 a = xl[j];
        const double2 b0 = xl[j + nR], d0 = xl[j + 2 * nR];
        const double2 b = make_double2(b0.x * c1 - b0.y * s1, b0.x * s1 + b0.y * c1);
        const double2 d = make_double2(d0.x * c2 - d0.y * s2, d0.x * s2 + d0.y * c2);
        // size-3 DFT: w = exp(sign 2 pi i / 3) = -1/2 + sign i sqrt(3)/2
        const double h = 0.86602540378443864676 * sign;
        const double2 sp = make_double2(b.x + d.x, b.y + d.y), sm = make_double2(b.x - d.x, b.y - d.y);
        yl[idx] = make_double2(a.x + sp.x, a.y + sp.y);
        const double2 mid = make_double2(a.x - 0.5 * sp.x, a.y - 0.5 * sp.y);
        yl[idx + Ns] = make_double2(mid.x - h * sm.y, mid.y + h * sm.x);
        yl[idx + 2 * Ns] = make_double2(mid.x + h * sm.y, mid.y - h * sm.x);
      }
    }
    __syncthreads();
    double2* t = x;
    x = y;
    y = t;
    Ns *= R;
  }
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    int l, t;
    if (ax.rows) { l = e / n; t = e - l * n; } else { t = e / nl; l = e - t * nl; }
    const double2 w = x[l * n + t];
    base[addr(l, t)] = make_double2(w.x * scale, w.y * scale);
  }
}

static FftAxis axis_of(const System& s, int d) {
  FftAxis a;
  if (d == 2) {  // z: rows of NLz
    a.n = s.NLz; a.nlines = s.NLx * s.NLy; a.ninner = 1; a.lo_stride = s.NLz; a.stride = 1; a.rows = true;
  } else if (d == 1) {  // y: lines (x, z), stride NLz
    a.n = s.NLy; a.nlines = s.NLx * s.NLz; a.ninner = s.NLz; a.lo_stride = s.NLy * s.NLz; a.stride = s.NLz;
    a.rows = false;
  } else {  // x: lines (y, z), stride NLy*NLz
    a.n = s.NLx; a.nlines = s.NLy * s.NLz; a.ninner = s.NLy * s.NLz; a.lo_stride = 0; a.stride = s.NLy * s.NLz;
    a.rows = false;
  }
  return a;
}

cudaError_t launch_fft3d(const System& s, double2* data, int nvec, int sign, bool normalise) {
  if (!fft_size_ok(s.NLx) || !fft_size_ok(s.NLy) || !fft_size_ok(s.NLz)) return cudaErrorInvalidValue;
  for (int d = 2; d >= 0; --d) {
    const FftAxis a = axis_of(s, d);
    const size_t smem = 2 * (size_t)FFT_TL * a.n * sizeof(double2);
    dim3 grid((a.nlines + FFT_TL - 1) / FFT_TL, nvec);
    k_fft_lines<<<grid, FFT_THREADS, smem, s.launch_stream()>>>(data, s.NL, a, sign, normalise ? 1.0 / a.n : 1.0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Kinetic symbol of the FD operator along one axis for the phase th = 2 pi m / n
// per grid step: -1/2 (lap0 + 2 sum lap_n cos(n th)) + 2 k sum nab_n sin(n th)
__device__ __forceinline__ double fd_symbol(const double* lap, const double* nab, double k, double th) {
  double t = lap[0];
  double g = 0.0;
#pragma unroll
  for (int n = 1; n <= 4; ++n) {
    double sn, cs;
    sincos(n * th, &sn, &cs);
    t += 2.0 * lap[n] * cs;
    g += nab[n] * sn;
  }
  return -0.5 * t + 2.0 * k * g;
}

struct TpaArgs {
  int NLx, NLy, NLz, NL;
  double lap[3][5], nab[3][5];
};

// data[v] (reciprocal space) *= K(T(G)/T_band[v]) with the k-point of vector v
__global__ void k_tpa_scale(double2* __restrict__ data, TpaArgs a, const double* __restrict__ kAc,
                            const double* __restrict__ tband, int kl_of_vec_stride, const int* __restrict__ kidx) {
  const int v = blockIdx.y;
  const int kl = kidx ? kidx[v] : v / kl_of_vec_stride;
  const double kx = kAc[3 * kl], ky = kAc[3 * kl + 1], kz = kAc[3 * kl + 2];
  const double tb = fmax(tband[v], 1e-6);
  const double pi2 = 6.28318530717958647692;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.NL; i += gridDim.x * blockDim.x) {
    const int ix = i / (a.NLy * a.NLz), iy = (i / a.NLz) % a.NLy, iz = i % a.NLz;
    const int mx = ix <= a.NLx / 2 ? ix : ix - a.NLx;
    const int my = iy <= a.NLy / 2 ? iy : iy - a.NLy;
    const int mz = iz <= a.NLz / 2 ? iz : iz - a.NLz;
    const double T = 0.5 * (kx * kx + ky * ky + kz * kz) + fd_symbol(a.lap[0], a.nab[0], kx, pi2 * mx / a.NLx) +
                     fd_symbol(a.lap[1], a.nab[1], ky, pi2 * my / a.NLy) +
                     fd_symbol(a.lap[2], a.nab[2], kz, pi2 * mz / a.NLz);
    const double x = fmax(T, 0.0) / tb;
    const double p = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x));
    const double K = p / (p + 16.0 * x * x * x * x);
    double2* d = data + (size_t)v * a.NL + i;
    *d = make_double2(d->x * K, d->y * K);
  }
}

cudaError_t launch_tpa(const System& s, double2* data, int nvec, const double* tband_dev, int vecs_per_k,
                       const int* kidx_dev) {
  cudaError_t e = launch_fft3d(s, data, nvec, -1, false);
  if (e != cudaSuccess) return e;
  TpaArgs a;
  a.NLx = s.NLx; a.NLy = s.NLy; a.NLz = s.NLz; a.NL = s.NL;
  for (int d = 0; d < 3; ++d)
    for (int n = 0; n < 5; ++n) { a.lap[d][n] = s.lap[d][n]; a.nab[d][n] = s.nab[d][n]; }
  dim3 grid((s.NL + 255) / 256 < 1024 ? (s.NL + 255) / 256 : 1024, nvec);
  k_tpa_scale<<<grid, 256, 0, s.launch_stream()>>>(data, a, s.kAc_d, tband_dev, vecs_per_k, kidx_dev);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return launch_fft3d(s, data, nvec, +1, true);
}

}  // namespace sgpu

extern "C" int sgpu_tpa_apply(sgpu_handle h, const void* in_dev, void* out_dev, int nvec, const int* kidx,
                              const double* tband) {
  using sgpu::System;
  if (!h || !in_dev || !out_dev || !tband || nvec < 1) {
    sgpu::set_last_error("sgpu_tpa_apply: bad argument");
    return SGPU_ERR_ARG;
  }
  System* s = h;
  std::vector<int> kv(nvec);
  for (int v = 0; v < nvec; ++v) {
    kv[v] = kidx ? kidx[v] : v;
    if (kv[v] < 0 || kv[v] >= s->nkl) {
      sgpu::set_last_error("sgpu_tpa_apply: k-point index outside the handle's k range");
      return SGPU_ERR_ARG;
    }
  }
  if (!(sgpu::fft_size_ok(s->NLx) && sgpu::fft_size_ok(s->NLy) && sgpu::fft_size_ok(s->NLz))) {
    sgpu::set_last_error("sgpu_tpa_apply: grid sizes must be 2^a 3^b <= 96");
    return SGPU_ERR_UNSUPPORTED;
  }
  double* tb = nullptr;
  int* kd = nullptr;
  cudaError_t e = cudaMalloc(&tb, (size_t)nvec * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&kd, (size_t)nvec * sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyAsync(tb, tband, (size_t)nvec * sizeof(double), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(kd, kv.data(), (size_t)nvec * sizeof(int), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out_dev, in_dev, (size_t)nvec * s->NL * sizeof(double2), cudaMemcpyDeviceToDevice, s->stream);
  if (e == cudaSuccess) e = sgpu::launch_tpa(*s, (double2*)out_dev, nvec, tb, 1, kd);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cudaFree(tb);
  cudaFree(kd);
  if (e != cudaSuccess) {
    sgpu::set_last_error(std::string("sgpu_tpa_apply: ") + cudaGetErrorString(e));
    return SGPU_ERR_CUDA;
  }
  return 0;
}
