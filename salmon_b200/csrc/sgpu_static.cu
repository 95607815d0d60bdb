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
#include <utility>
#include <vector>

#include "sgpu_internal.cuh"

namespace {

constexpr int kChunk = 64;  // orbitals per partial density (the handle path uses the same split)

// The scratch: ceil(norb / kChunk) partial densities of NL values each.
static __device__ __align__(256) double g_rho_scratch[SGPU_PSI_RHO_STATIC_SCRATCH_DOUBLES];

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

// Set-up: the device address of the scratch, looked up with
// cudaGetSymbolAddress once per context and kept in a small table.  In host code
// the name g_rho_scratch is only a host-side stand-in, never a device address.
// The table is keyed on the unique ID of the CURRENT CUDA context, not on the
// device ordinal: an address belongs to the context it was taken in, so after a
// device reset, or when a host runtime makes its own non-primary context
// current, the first call in that context looks the address up again instead of
// reusing a stale one.  The context ID comes from the driver's cuCtxGetCurrent
// and cuCtxGetId (IDs are never reused within a process), reached through
// cudaGetDriverEntryPoint so that the library does not link libcuda; where that
// fails the address is looked up on every call.  A lookup allocates nothing, but
// the first one in a context may load the library's device code into it, which
// is why the first call in a context must not be made inside stream capture.
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);
std::mutex g_setup_mu;
std::vector<std::pair<unsigned long long, double*>> g_scratch_of_context;

template <typename F>
F driver_fn(const char* name) {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &fn, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    return nullptr;
  return reinterpret_cast<F>(fn);
}

int scratch_for_current_context(double** out) {
  static const CtxGetCurrentFn ctx_get_current = driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
  static const CtxGetIdFn ctx_get_id = driver_fn<CtxGetIdFn>("cuCtxGetId");
  void* ctx = nullptr;
  unsigned long long id = 0;
  const bool keyed = ctx_get_current && ctx_get_id && ctx_get_current(&ctx) == 0 && ctx != nullptr &&
                     ctx_get_id(ctx, &id) == 0;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (keyed)
    for (const auto& e : g_scratch_of_context)
      if (e.first == id) {
        *out = e.second;
        return 0;
      }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_rho_scratch);
  if (e != cudaSuccess || !p)
    return reject(SGPU_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
  *out = static_cast<double*>(p);
  if (keyed) {
    if (g_scratch_of_context.size() >= 256) g_scratch_of_context.clear();  // bounded; entries are only a cache
    g_scratch_of_context.emplace_back(id, *out);
  }
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
  if (int rc = scratch_for_current_context(&part)) return rc;
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
