// Self-consistent local potential on the device: Hartree potential by FFT,
// Perdew-Zunger LDA exchange-correlation, and Vloc = Vh + Vpsl + Vexc
// (RT/dt_evolve.f90:190-207 with common/Hartree.f90 and xc/builtin_pz.f90).
#include <cuda_runtime.h>

#include "sgpu_internal.cuh"

namespace sgpu {

// rho (real) -> complex work array
__global__ void k_real_to_complex(const double* __restrict__ r, double2* __restrict__ z, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = make_double2(r[i], 0.0);
}

// rho(G) -> Vh(G) = 4 pi rho(G) / |G|^2 / NL, Vh(0) = 0 (Hartree.f90:71-80); |G| from
// the cell (G_d = 2 pi m_d / aL_d with m_d in [-N/2, N/2), Hartree.f90:38-62 and init.f90:52)
__global__ void k_poisson(double2* __restrict__ z, int NLx, int NLy, int NLz, double bx, double by, double bz) {
  const int NL = NLx * NLy * NLz;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NL) return;
  const int ix = i / (NLy * NLz), iy = (i / NLz) % NLy, iz = i % NLz;
  const int mx = ix < NLx - NLx / 2 ? ix : ix - NLx;
  const int my = iy < NLy - NLy / 2 ? iy : iy - NLy;
  const int mz = iz < NLz - NLz / 2 ? iz : iz - NLz;
  const double gx = mx * bx, gy = my * by, gz = mz * bz;
  const double G2 = gx * gx + gy * gy + gz * gz;
  const double f = (i == 0) ? 0.0 : 4.0 * 3.14159265358979323846 / G2 / NL;
  z[i] = make_double2(z[i].x * f, z[i].y * f);
}

// Perdew and Zunger, Phys. Rev. B 23, 5048 (1981), unpolarised: the exchange
// energy per electron -(3/4)(3/(2 pi))^(2/3)/rs plus the correlation fit
// (gamma/(1 + beta1 sqrt(rs) + beta2 rs) for rs >= 1, A ln rs + B + C rs ln rs + D rs
// below), as PZxc evaluates it (xc/builtin_pz.f90:45-76); vxc = exc + rho dexc/drho.
__device__ __forceinline__ void pz(double rho, double& exc, double& vxc) {  // rho: total density
  const double pi = 3.14159265358979323846;
  const double gammaU = -0.1423, beta1U = 1.0529, beta2U = 0.3334;
  const double AU = 0.0311, BU = -0.048, CU = 0.002, DU = -0.0116;
  const double cx = 0.75 * cbrt((3.0 / (2.0 * pi)) * (3.0 / (2.0 * pi)));
  const double tr = rho + 1e-10;
  const double rs = cbrt(3.0 / (4.0 * pi * tr));
  double e = -cx / rs;
  double de = e / (3.0 * tr);
  if (rs > 1.0) {
    const double sq = sqrt(rs);
    const double den = 1.0 + beta1U * sq + beta2U * rs;
    e += gammaU / den;
    de += gammaU * (0.5 * beta1U * sq + beta2U * rs) / (3.0 * tr) / (den * den);
  } else {
    const double ln = log(rs);
    e += AU * ln + BU + CU * rs * ln + DU * rs;
    de -= rs / (3.0 * tr) * (AU / rs + CU * (ln + 1.0) + DU);
  }
  exc = e;
  vxc = e + rho * de;
}

// Vloc = Re Vh + Vpsl + Vxc; per-block partial sums of (1/2 Vh rho, exc rho) for the energies
__global__ void __launch_bounds__(256) k_vloc(const double2* __restrict__ vh, const double* __restrict__ rho,
                                              const double* __restrict__ vpsl, int NL, double* __restrict__ v64,
                                              float* __restrict__ v32, double* __restrict__ part) {
  __shared__ double sh[64];
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NL; i += gridDim.x * blockDim.x) {
    double exc, vxc;
    pz(rho[i], exc, vxc);
    const double v = vh[i].x + vpsl[i] + vxc;
    v64[i] = v;
    v32[i] = (float)v;
    acc[0] = fma(0.5 * vh[i].x, rho[i], acc[0]);
    acc[1] = fma(exc, rho[i], acc[1]);
  }
  block_allsum<2>(acc, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = acc[0];
    part[2 * blockIdx.x + 1] = acc[1];
  }
}

__global__ void k_sum_pairs(const double* __restrict__ part, int n, double scale, double* __restrict__ out) {
  double a = 0.0, b = 0.0;
  for (int i = 0; i < n; ++i) { a += part[2 * i]; b += part[2 * i + 1]; }
  out[0] = a * scale;
  out[1] = b * scale;
}

constexpr int VLOC_BLOCKS = 148;

cudaError_t launch_update_vloc(const System& s, const double* rho_dev, double* energies_dev) {
  if (!fft_size_ok(s.NLx) || !fft_size_ok(s.NLy) || !fft_size_ok(s.NLz)) return cudaErrorInvalidValue;
  double2* z = s.stage;                               // NL complex work values
  double* part = reinterpret_cast<double*>(s.stage + s.NL);  // 2 x VLOC_BLOCKS partial sums
  const int nb = (s.NL + 255) / 256;
  k_real_to_complex<<<nb, 256, 0, s.launch_stream()>>>(rho_dev, z, s.NL);
  cudaError_t e = launch_fft3d(s, z, 1, -1, false);
  if (e != cudaSuccess) return e;
  const double pi2 = 6.28318530717958647692;
  k_poisson<<<nb, 256, 0, s.launch_stream()>>>(z, s.NLx, s.NLy, s.NLz, pi2 / s.aL[0], pi2 / s.aL[1], pi2 / s.aL[2]);
  if ((e = launch_fft3d(s, z, 1, +1, false)) != cudaSuccess) return e;
  k_vloc<<<VLOC_BLOCKS, 256, 0, s.launch_stream()>>>(z, rho_dev, s.vpsl, s.NL, s.vloc64, s.vloc32, part);
  k_sum_pairs<<<1, 1, 0, s.launch_stream()>>>(part, VLOC_BLOCKS, s.Hxyz, energies_dev);
  return cudaGetLastError();
}

// The etrs potential history (RT/dt_evolve.f90:248-252, control/control_sc.f90:82):
// reset: hist1 = hist2 = Vloc;
// extrapolate: Vnew = 3 Vloc - 3 hist1 + hist2, hist2 = hist1, hist1 = Vloc, Vloc = Vnew
// (in FP64, with the FP32 copy of Vloc refreshed).
__global__ void k_vloc_history(double* __restrict__ v64, float* __restrict__ v32, double* __restrict__ h1,
                               double* __restrict__ h2, int NL, int extrapolate) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < NL; i += gridDim.x * blockDim.x) {
    const double v = v64[i];
    if (extrapolate) {
      const double vn = 3.0 * v - 3.0 * h1[i] + h2[i];
      h2[i] = h1[i];
      h1[i] = v;
      v64[i] = vn;
      v32[i] = (float)vn;
    } else {
      h1[i] = v;
      h2[i] = v;
    }
  }
}

cudaError_t launch_vloc_history(const System& s, bool extrapolate) {
  if (!s.vloc_hist) return cudaErrorInvalidValue;
  k_vloc_history<<<(s.NL + 255) / 256, 256, 0, s.launch_stream()>>>(s.vloc64, s.vloc32, s.vloc_hist,
                                                                     s.vloc_hist + s.NL, s.NL, extrapolate ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace sgpu
