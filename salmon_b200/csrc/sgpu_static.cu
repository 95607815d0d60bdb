// sgpu_psi_rho_static: the density reduction over caller-owned device orbitals
// with its scratch in a fixed, statically sized device array instead of memory
// obtained at run time.
//
// Who cannot allocate, and why.  A host that already keeps the orbitals on the
// device through its own runtime (SALMON's OpenACC build holds zu_t in device
// memory owned by the OpenACC present table) can ask for the density without
// creating a handle, and creating a handle is exactly where this library
// allocates.  Such a host may also have handed almost all of the device memory
// to its own pool, so a fresh cudaMalloc can fail in the middle of a time step;
// and cudaFree synchronises the whole device, which stalls work the host has in
// flight on its other streams.  This entry point therefore performs no device
// allocation or release of any kind: its scratch is reserved when the library's
// device code is loaded.
//
// The cost of that choice is a fixed capacity (SGPU_PSI_RHO_STATIC_SCRATCH_DOUBLES
// partial-density values) and one scratch array per device shared by every
// call: two calls on one device whose executions overlap (different streams
// without an ordering between them, or different host threads) write the same
// scratch and corrupt each other's result.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "sgpu_internal.cuh"

namespace {

constexpr int kChunk = 64;       // orbitals per partial density (the handle path uses the same split)
constexpr int kMaxDevices = 64;  // device ordinals the set-up table covers

// The scratch: ceil(norb / kChunk) partial densities of NL values each.
static __device__ __align__(256) double g_rho_scratch[SGPU_PSI_RHO_STATIC_SCRATCH_DOUBLES];

std::mutex g_setup_mu;
double* g_scratch_of_device[kMaxDevices] = {};

// Partial density of orbitals [o0, o0 + kChunk) at grid point i, accumulated
// in FP64 in orbital order; orbital o = ib + nb * ik has weight occ[ib + ld_occ * ik].
template <typename R>
__global__ void k_rho_partial_static(const sgpu::C2<R>* __restrict__ zu, const double* __restrict__ occ, int ld_occ,
                                     int nb, long long norb, int NL, double* __restrict__ part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NL) return;
  const long long o0 = (long long)blockIdx.y * kChunk;
  const long long o1 = o0 + kChunk < norb ? o0 + kChunk : norb;
  double acc = 0.0;
  for (long long o = o0; o < o1; ++o) {
    const double2 z = sgpu::to_d2(zu[(size_t)o * NL + i]);
    const double w = occ[(o % nb) + (size_t)ld_occ * (o / nb)];
    acc += w * (z.x * z.x + z.y * z.y);
  }
  part[(size_t)blockIdx.y * NL + i] = acc;
}

__global__ void k_rho_sum_static(const double* __restrict__ part, int nchunk, int NL, double* __restrict__ rho) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NL) return;
  double acc = 0.0;
  for (int c = 0; c < nchunk; ++c) acc += part[(size_t)c * NL + i];
  rho[i] = acc;
}

int reject(int code, std::string msg);

// Device address of the scratch on the current device, looked up once per
// device (cudaGetSymbolAddress may load the library's device code, which is
// why the first call on a device should not be made inside stream capture).
int scratch_for_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return reject(SGPU_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return reject(SGPU_ERR_UNSUPPORTED, "device ordinal " + std::to_string(dev) + " is beyond the set-up table (" +
                                            std::to_string(kMaxDevices) + " devices)");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_of_device[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_rho_scratch);
    if (e != cudaSuccess || !p)
      return reject(SGPU_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_scratch_of_device[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_of_device[dev];
  return 0;
}

}  // namespace

namespace {
int reject(int code, std::string msg) {
  sgpu::set_last_error("sgpu_psi_rho_static: " + msg);
  return code;
}
}  // namespace

extern "C" int sgpu_psi_rho_static(int precision, int NL, int nb, int nk, const void* zu, const double* occ,
                                   int ld_occ, double* rho, void* stream) {
  if (precision != SGPU_PREC_C128 && precision != SGPU_PREC_C64)
    return reject(SGPU_ERR_ARG, "precision must be SGPU_PREC_C128 or SGPU_PREC_C64");
  if (NL < 1 || nb < 1 || nk < 1) return reject(SGPU_ERR_ARG, "NL, nb and nk must be positive");
  if (ld_occ < nb) return reject(SGPU_ERR_ARG, "ld_occ must be at least nb");
  if (!zu || !occ || !rho) return reject(SGPU_ERR_ARG, "null device pointer");
  const size_t zalign = precision == SGPU_PREC_C128 ? 16 : 8;
  if ((uintptr_t)zu % zalign || (uintptr_t)occ % 8 || (uintptr_t)rho % 8)
    return reject(SGPU_ERR_ARG, "misaligned device pointer");
  const long long norb = (long long)nb * nk;
  const long long nchunk = (norb + kChunk - 1) / kChunk;
  const long long need = nchunk * (long long)NL;
  if (need > (long long)SGPU_PSI_RHO_STATIC_SCRATCH_DOUBLES || nchunk > 65535)
    return reject(SGPU_ERR_ARG, "needs " + std::to_string(need) + " scratch doubles (ceil(nb*nk/" +
                                    std::to_string(kChunk) + ") x NL); the static maximum is " +
                                    std::to_string((long long)SGPU_PSI_RHO_STATIC_SCRATCH_DOUBLES));
  double* part = nullptr;
  if (int rc = scratch_for_current_device(&part)) return rc;
  // Nothing in the scratch has to start at zero: every partial density row
  // that k_rho_sum_static reads is written in full by k_rho_partial_static
  // earlier on the same stream, so no clearing pass is needed.
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dim3 grid((NL + 255) / 256, (unsigned)nchunk);
  if (precision == SGPU_PREC_C64)
    k_rho_partial_static<float><<<grid, 256, 0, st>>>(static_cast<const float2*>(zu), occ, ld_occ, nb, norb, NL, part);
  else
    k_rho_partial_static<double><<<grid, 256, 0, st>>>(static_cast<const double2*>(zu), occ, ld_occ, nb, norb, NL,
                                                       part);
  k_rho_sum_static<<<(NL + 255) / 256, 256, 0, st>>>(part, (int)nchunk, NL, rho);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return reject(SGPU_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  return 0;
}
