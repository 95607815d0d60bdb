// The learned CG preconditioner: a 3-layer 3D convolution network on the
// periodic grid, BF16 weights and activations, FP32 accumulation, with its
// inference, training (forward, backward, Adam) and the C ABI around it.
//
//   input   one real field: the real part, or the imaginary part, of the
//           (TPA-preconditioned) CG gradient g of one band, scaled by 1/rms(g)
//   layers  conv 1->8, conv 8->8, conv 8->1; 3x3x3 kernels, circular padding,
//           no bias, no activation function: a learned real linear operator f
//           (a factorised 7x7x7 filter)
//   output  K(g) = (f(Re g) + i f(Im g)) * rms(g): complex-linear, K(c g) = c K(g)
//           for every complex c, as a preconditioner for complex CG must be
//
// Training pairs come from plain CG: the gradient g of a band and the error
// e = (1 - P) psi of that band (P the projector on the converged bands), both
// scaled by 1/rms(g); the loss is the mean squared difference.  Every
// reduction (weight gradients, loss, norms) runs in a fixed order.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "sgpu_internal.cuh"

namespace sgpu {

constexpr int NTAP = 27;
constexpr int NET_C = 8;  // hidden channels
constexpr int NW1 = NET_C * 1 * NTAP, NW2 = NET_C * NET_C * NTAP, NW3 = 1 * NET_C * NTAP;
constexpr int NET_NW = NW1 + NW2 + NW3;  // 2160 weights, layer by layer, [co][ci][tap]

using bf16 = __nv_bfloat16;

struct NetGeom {
  int NLx, NLy, NLz, NL;
};

// tap = (dx+1)*9 + (dy+1)*3 + (dz+1)
__device__ __forceinline__ int nbr(int x, int y, int z, int tap, int sgn, const NetGeom& g) {
  int dx = (tap / 9 - 1) * sgn, dy = ((tap / 3) % 3 - 1) * sgn, dz = (tap % 3 - 1) * sgn;
  int xx = x + dx, yy = y + dy, zz = z + dz;
  xx += xx < 0 ? g.NLx : 0; xx -= xx >= g.NLx ? g.NLx : 0;
  yy += yy < 0 ? g.NLy : 0; yy -= yy >= g.NLy ? g.NLy : 0;
  zz += zz < 0 ? g.NLz : 0; zz -= zz >= g.NLz ? g.NLz : 0;
  return (xx * g.NLy + yy) * g.NLz + zz;
}

__device__ __forceinline__ float tof(float v) { return v; }
__device__ __forceinline__ float tof(bf16 v) { return __bfloat162float(v); }
__device__ __forceinline__ void fromf(float& d, float v) { d = v; }
__device__ __forceinline__ void fromf(bf16& d, float v) { d = __float2bfloat16_rn(v); }

// ---------------------------------------------------------------- forward --
// out[v][i][co] = sum_{tap,ci} W[co][ci][tap] in[v][i + d(tap)][ci]
template <int CI, int CO, typename TI, typename TO>
__global__ void __launch_bounds__(256) k_conv_fwd(const TI* __restrict__ in, const bf16* __restrict__ W,
                                                  TO* __restrict__ out, NetGeom g, int nvec) {
  __shared__ float w[CO * CI * NTAP];
  for (int t = threadIdx.x; t < CO * CI * NTAP; t += blockDim.x) w[t] = __bfloat162float(W[t]);
  __syncthreads();
  const size_t total = (size_t)nvec * g.NL;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int v = (int)(idx / g.NL), i = (int)(idx - (size_t)v * g.NL);
    const int x = i / (g.NLy * g.NLz), y = (i / g.NLz) % g.NLy, z = i % g.NLz;
    const TI* inv = in + (size_t)v * g.NL * CI;
    float acc[CO];
#pragma unroll
    for (int co = 0; co < CO; ++co) acc[co] = 0.f;
    for (int tap = 0; tap < NTAP; ++tap) {
      const TI* p = inv + (size_t)nbr(x, y, z, tap, 1, g) * CI;
      float a[CI];
#pragma unroll
      for (int ci = 0; ci < CI; ++ci) a[ci] = tof(p[ci]);
#pragma unroll
      for (int co = 0; co < CO; ++co)
#pragma unroll
        for (int ci = 0; ci < CI; ++ci) acc[co] = fmaf(w[(co * CI + ci) * NTAP + tap], a[ci], acc[co]);
    }
    TO* o = out + idx * CO;
#pragma unroll
    for (int co = 0; co < CO; ++co) fromf(o[co], acc[co]);
  }
}

// ------------------------------------------------------ backward (input) --
// gin[v][i][ci] = sum_{tap,co} W[co][ci][tap] gout[v][i - d(tap)][co]
template <int CI, int CO>
__global__ void __launch_bounds__(256) k_conv_bwd_data(const float* __restrict__ gout, const bf16* __restrict__ W,
                                                       float* __restrict__ gin, NetGeom g, int nvec) {
  __shared__ float w[CO * CI * NTAP];
  for (int t = threadIdx.x; t < CO * CI * NTAP; t += blockDim.x) w[t] = __bfloat162float(W[t]);
  __syncthreads();
  const size_t total = (size_t)nvec * g.NL;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int v = (int)(idx / g.NL), i = (int)(idx - (size_t)v * g.NL);
    const int x = i / (g.NLy * g.NLz), y = (i / g.NLz) % g.NLy, z = i % g.NLz;
    const float* gv = gout + (size_t)v * g.NL * CO;
    float acc[CI];
#pragma unroll
    for (int ci = 0; ci < CI; ++ci) acc[ci] = 0.f;
    for (int tap = 0; tap < NTAP; ++tap) {
      const float* p = gv + (size_t)nbr(x, y, z, tap, -1, g) * CO;
#pragma unroll
      for (int co = 0; co < CO; ++co) {
        const float go = p[co];
#pragma unroll
        for (int ci = 0; ci < CI; ++ci) acc[ci] = fmaf(w[(co * CI + ci) * NTAP + tap], go, acc[ci]);
      }
    }
    float* o = gin + idx * CI;
#pragma unroll
    for (int ci = 0; ci < CI; ++ci) o[ci] = acc[ci];
  }
}

// ---------------------------------------------------- backward (weights) --
// part[cta][co][ci][tap] = sum over the CTA's x-plane of gout[i][co] in[i + d(tap)][ci];
// the CTA stages input planes x-1, x, x+1 and the output-gradient plane.
template <int CI, int CO>
__global__ void __launch_bounds__(256) k_conv_bwd_w(const float* __restrict__ gout, const bf16* __restrict__ in,
                                                    float* __restrict__ part, NetGeom g) {
  extern __shared__ float nsm[];
  const int NYZ = g.NLy * g.NLz;
  float* sgo = nsm;                                         // [NYZ][CO]
  bf16* sin_ = reinterpret_cast<bf16*>(nsm + NYZ * CO);     // [3][NYZ][CI]
  const int v = blockIdx.y, x = blockIdx.x;
  for (int t = threadIdx.x; t < 3 * NYZ * CI; t += blockDim.x) {
    const int pl = t / (NYZ * CI), r = t - pl * NYZ * CI;
    int xx = x + pl - 1;
    xx += xx < 0 ? g.NLx : 0; xx -= xx >= g.NLx ? g.NLx : 0;
    sin_[t] = in[((size_t)v * g.NL + (size_t)xx * NYZ) * CI + r];
  }
  for (int t = threadIdx.x; t < NYZ * CO; t += blockDim.x) sgo[t] = gout[((size_t)v * g.NL + (size_t)x * NYZ) * CO + t];
  __syncthreads();
  float* pout = part + ((size_t)v * g.NLx + x) * (CO * CI * NTAP);
  for (int wi = threadIdx.x; wi < CO * CI * NTAP; wi += blockDim.x) {
    const int co = wi / (CI * NTAP), ci = (wi / NTAP) % CI, tap = wi % NTAP;
    const int pl = tap / 9, dy = (tap / 3) % 3 - 1, dz = tap % 3 - 1;
    float acc = 0.f;
    for (int y = 0; y < g.NLy; ++y) {
      int yy = y + dy;
      yy += yy < 0 ? g.NLy : 0; yy -= yy >= g.NLy ? g.NLy : 0;
      const bf16* irow = sin_ + ((size_t)pl * NYZ + yy * g.NLz) * CI + ci;
      const float* grow = sgo + (size_t)y * g.NLz * CO + co;
      for (int z = 0; z < g.NLz; ++z) {
        int zz = z + dz;
        zz += zz < 0 ? g.NLz : 0; zz -= zz >= g.NLz ? g.NLz : 0;
        acc = fmaf(grow[z * CO], __bfloat162float(irow[zz * CI]), acc);
      }
    }
    pout[wi] = acc;
  }
}

// dW[w] = sum_c part[c][w], in CTA order
__global__ void k_sum_parts(const float* __restrict__ part, int nparts, int nw, float* __restrict__ dW) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  double acc = 0.0;
  for (int c = 0; c < nparts; ++c) acc += part[(size_t)c * nw + w];
  dW[w] = (float)acc;
}

// ---------------------------------------------------- packing and the loss --
// scale[v] = 1 / rms(g_v) over the NL complex values (one CTA per vector)
__global__ void __launch_bounds__(256) k_vec_invrms(const double2* __restrict__ g, int NL, double* __restrict__ scale) {
  __shared__ double sh[64];
  const double2* p = g + (size_t)blockIdx.x * NL;
  double v[1] = {0.0};
  for (int i = threadIdx.x; i < NL; i += blockDim.x) v[0] = fma(p[i].x, p[i].x, fma(p[i].y, p[i].y, v[0]));
  block_allsum<1>(v, sh);
  if (threadIdx.x == 0) scale[blockIdx.x] = v[0] > 0.0 ? sqrt(NL / v[0]) : 0.0;
}

// vector v -> samples 2v (real part) and 2v+1 (imaginary part), one channel each
template <typename T>
__global__ void k_pack(const double2* __restrict__ g, const double* __restrict__ scale, int NL, int nvec,
                       T* __restrict__ out) {
  const size_t total = (size_t)nvec * NL;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const size_t v = idx / NL, i = idx - v * NL;
    const double s = scale[v];
    fromf(out[(2 * v) * NL + i], (float)(g[idx].x * s));
    fromf(out[(2 * v + 1) * NL + i], (float)(g[idx].y * s));
  }
}

__global__ void k_unpack(const float* __restrict__ y, const double* __restrict__ scale, int NL, int nvec,
                         double2* __restrict__ out) {
  const size_t total = (size_t)nvec * NL;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const size_t v = idx / NL, i = idx - v * NL;
    const double s = scale[v];
    const double inv = s > 0.0 ? 1.0 / s : 0.0;
    out[idx] = make_double2(y[(2 * v) * NL + i] * inv, y[(2 * v + 1) * NL + i] * inv);
  }
}

// gy = 2 (y - t) / count; part[b] = sum over the block's elements of (y - t)^2
__global__ void __launch_bounds__(256) k_mse(const float* __restrict__ y, const float* __restrict__ t, size_t n,
                                             float* __restrict__ gy, double* __restrict__ part) {
  __shared__ double sh[64];
  double v[1] = {0.0};
  const double inv = 2.0 / (double)n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float d = y[i] - t[i];
    gy[i] = (float)(d * inv);
    v[0] += (double)d * d;
  }
  block_allsum<1>(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

__global__ void k_sum_loss(const double* __restrict__ part, int n, double count, double* __restrict__ loss) {
  double a = 0.0;
  for (int i = 0; i < n; ++i) a += part[i];
  *loss = a / count;
}

// Adam (Kingma and Ba, 2015) on the FP32 master weights; BF16 copies for the kernels
__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v2,
                       const float* __restrict__ grad, bf16* __restrict__ wb, int n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gr = grad[i];
  const float mm = b1 * m[i] + (1.f - b1) * gr;
  const float vv = b2 * v2[i] + (1.f - b2) * gr * gr;
  m[i] = mm;
  v2[i] = vv;
  const float wn = w[i] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  w[i] = wn;
  wb[i] = __float2bfloat16_rn(wn);
}

__global__ void k_to_bf16(const float* __restrict__ src, bf16* __restrict__ dst, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __float2bfloat16_rn(src[i]);
}

// ------------------------------------------------------------ workspace --
struct NetState {
  float* w = nullptr;   // FP32 master weights [NET_NW]
  bf16* wb = nullptr;   // BF16 copies used by the kernels
  float *m = nullptr, *v2 = nullptr, *grad = nullptr;
  int adam_t = 0;
  int cap = 0;          // vectors the activation buffers hold
  bf16 *a0 = nullptr, *a1 = nullptr, *a2 = nullptr;
  float *y = nullptr, *t = nullptr, *gy = nullptr, *g2 = nullptr, *g1 = nullptr, *part = nullptr;
  double *scale = nullptr, *lpart = nullptr, *loss = nullptr;
  size_t part_elems = 0;
};

static int grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

static cudaError_t net_reserve(System& s, NetState& ns, int nvec) {
  if (nvec <= ns.cap) return cudaSuccess;
  cudaError_t e = cudaStreamSynchronize(s.stream);
  if (e != cudaSuccess) return e;
  void* bufs[] = {ns.a0, ns.a1, ns.a2, ns.y, ns.t, ns.gy, ns.g2, ns.g1, ns.part, ns.scale, ns.lpart};
  for (void* p : bufs) cudaFree(p);
  const size_t n = (size_t)2 * nvec * s.NL;  // two real samples per vector
  ns.part_elems = (size_t)2 * nvec * s.NLx * NW2;
  if ((e = cudaMalloc(&ns.a0, n * sizeof(bf16)))) return e;
  if ((e = cudaMalloc(&ns.a1, n * NET_C * sizeof(bf16)))) return e;
  if ((e = cudaMalloc(&ns.a2, n * NET_C * sizeof(bf16)))) return e;
  if ((e = cudaMalloc(&ns.y, n * sizeof(float)))) return e;
  if ((e = cudaMalloc(&ns.t, n * sizeof(float)))) return e;
  if ((e = cudaMalloc(&ns.gy, n * sizeof(float)))) return e;
  if ((e = cudaMalloc(&ns.g2, n * NET_C * sizeof(float)))) return e;
  if ((e = cudaMalloc(&ns.g1, n * NET_C * sizeof(float)))) return e;
  if ((e = cudaMalloc(&ns.part, ns.part_elems * sizeof(float)))) return e;
  if ((e = cudaMalloc(&ns.scale, (size_t)nvec * sizeof(double)))) return e;
  if ((e = cudaMalloc(&ns.lpart, (size_t)148 * 32 * sizeof(double)))) return e;
  ns.cap = nvec;
  return cudaSuccess;
}

static NetGeom geom(const System& s) { return NetGeom{s.NLx, s.NLy, s.NLz, s.NL}; }

// input vectors -> a0 (2 real samples per vector, scaled by 1/rms) -> a1 -> a2 -> y
static cudaError_t net_forward(System& s, NetState& ns, const double2* g, int nvec) {
  const NetGeom G = geom(s);
  const int ns2 = 2 * nvec;
  const size_t n = (size_t)ns2 * s.NL;
  k_vec_invrms<<<nvec, 256, 0, s.launch_stream()>>>(g, s.NL, ns.scale);
  k_pack<bf16><<<grid_for(n / 2), 256, 0, s.launch_stream()>>>(g, ns.scale, s.NL, nvec, ns.a0);
  k_conv_fwd<1, NET_C, bf16, bf16><<<grid_for(n), 256, 0, s.launch_stream()>>>(ns.a0, ns.wb, ns.a1, G, ns2);
  k_conv_fwd<NET_C, NET_C, bf16, bf16><<<grid_for(n), 256, 0, s.launch_stream()>>>(ns.a1, ns.wb + NW1, ns.a2, G, ns2);
  k_conv_fwd<NET_C, 1, bf16, float><<<grid_for(n), 256, 0, s.launch_stream()>>>(ns.a2, ns.wb + NW1 + NW2, ns.y, G, ns2);
  return cudaGetLastError();
}

template <int CI, int CO>
static cudaError_t conv_bwd_w(System& s, NetState& ns, const float* gout, const bf16* in, float* dW, int nvec) {
  const NetGeom G = geom(s);
  const size_t smem = (size_t)s.NLy * s.NLz * (3 * CI * sizeof(bf16) + CO * sizeof(float));
  cudaError_t e = cudaFuncSetAttribute(k_conv_bwd_w<CI, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_conv_bwd_w<CI, CO><<<dim3(s.NLx, nvec), 256, smem, s.launch_stream()>>>(gout, in, ns.part, G);
  const int nw = CO * CI * NTAP;
  k_sum_parts<<<(nw + 255) / 256, 256, 0, s.launch_stream()>>>(ns.part, nvec * s.NLx, nw, dW);
  return cudaGetLastError();
}

// loss and gradients of the weights for targets t (complex, scaled like g)
static cudaError_t net_loss_grad(System& s, NetState& ns, const double2* g, const double2* tg, int nvec) {
  cudaError_t e = net_forward(s, ns, g, nvec);
  if (e != cudaSuccess) return e;
  const NetGeom G = geom(s);
  const int ns2 = 2 * nvec;
  const size_t n = (size_t)ns2 * s.NL;
  k_pack<float><<<grid_for(n / 2), 256, 0, s.launch_stream()>>>(tg, ns.scale, s.NL, nvec, ns.t);
  const int nb = grid_for(n);
  k_mse<<<nb, 256, 0, s.launch_stream()>>>(ns.y, ns.t, n, ns.gy, ns.lpart);
  k_sum_loss<<<1, 1, 0, s.launch_stream()>>>(ns.lpart, nb, (double)n, ns.loss);
  if ((e = conv_bwd_w<NET_C, 1>(s, ns, ns.gy, ns.a2, ns.grad + NW1 + NW2, ns2))) return e;
  k_conv_bwd_data<NET_C, 1><<<grid_for(n), 256, 0, s.launch_stream()>>>(ns.gy, ns.wb + NW1 + NW2, ns.g2, G, ns2);
  if ((e = conv_bwd_w<NET_C, NET_C>(s, ns, ns.g2, ns.a1, ns.grad + NW1, ns2))) return e;
  k_conv_bwd_data<NET_C, NET_C><<<grid_for(n), 256, 0, s.launch_stream()>>>(ns.g2, ns.wb + NW1, ns.g1, G, ns2);
  if ((e = conv_bwd_w<1, NET_C>(s, ns, ns.g1, ns.a0, ns.grad, ns2))) return e;
  return cudaGetLastError();
}

static NetState* net_of(System& s) { return static_cast<NetState*>(s.net); }

cudaError_t launch_precond_net(const System& cs, double2* data, int nvec) {
  System& s = const_cast<System&>(cs);
  NetState* ns = net_of(s);
  if (!ns) return cudaErrorInvalidValue;
  cudaError_t e = net_reserve(s, *ns, nvec);
  if (e != cudaSuccess) return e;
  if ((e = net_forward(s, *ns, data, nvec))) return e;
  k_unpack<<<grid_for((size_t)nvec * s.NL), 256, 0, s.launch_stream()>>>(ns->y, ns->scale, s.NL, nvec, data);
  return cudaGetLastError();
}

void net_free(System& s) {
  NetState* ns = net_of(s);
  if (!ns) return;
  void* bufs[] = {ns->w, ns->wb, ns->m, ns->v2, ns->grad, ns->a0, ns->a1, ns->a2, ns->y, ns->t, ns->gy,
                  ns->g2, ns->g1, ns->part, ns->scale, ns->lpart, ns->loss};
  for (void* p : bufs) cudaFree(p);
  delete ns;
  s.net = nullptr;
  s.net_ready = false;
}

}  // namespace sgpu

// ------------------------------------------------------------------ C ABI --
using sgpu::System;

namespace {
int nfail(int code, const std::string& msg) {
  sgpu::set_last_error(msg);
  return code;
}
int ncuda(cudaError_t e, const char* what) {
  return nfail(SGPU_ERR_CUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}
}  // namespace

extern "C" {

int sgpu_net_weight_count(void) { return sgpu::NET_NW; }

int sgpu_net_set_weights(sgpu_handle h, const float* w) {
  if (!h || !w) return nfail(SGPU_ERR_ARG, "sgpu_net_set_weights: null argument");
  System* s = h;
  using namespace sgpu;
  NetState* ns = net_of(*s);
  cudaError_t e;
  if (!ns) {
    ns = new NetState();
    s->net = ns;
    if ((e = cudaMalloc(&ns->w, NET_NW * sizeof(float))) || (e = cudaMalloc(&ns->wb, NET_NW * sizeof(bf16))) ||
        (e = cudaMalloc(&ns->m, NET_NW * sizeof(float))) || (e = cudaMalloc(&ns->v2, NET_NW * sizeof(float))) ||
        (e = cudaMalloc(&ns->grad, NET_NW * sizeof(float))) || (e = cudaMalloc(&ns->loss, sizeof(double)))) {
      net_free(*s);
      return ncuda(e, "sgpu_net_set_weights: alloc");
    }
  }
  if ((e = cudaMemcpyAsync(ns->w, w, NET_NW * sizeof(float), cudaMemcpyHostToDevice, s->stream)) ||
      (e = cudaMemsetAsync(ns->m, 0, NET_NW * sizeof(float), s->stream)) ||
      (e = cudaMemsetAsync(ns->v2, 0, NET_NW * sizeof(float), s->stream)))
    return ncuda(e, "sgpu_net_set_weights");
  k_to_bf16<<<(NET_NW + 255) / 256, 256, 0, s->launch_stream()>>>(ns->w, ns->wb, NET_NW);
  if ((e = cudaStreamSynchronize(s->stream))) return ncuda(e, "sgpu_net_set_weights");
  ns->adam_t = 0;
  s->net_ready = true;
  return 0;
}

int sgpu_net_get_weights(sgpu_handle h, float* w) {
  if (!h || !w) return nfail(SGPU_ERR_ARG, "sgpu_net_get_weights: null argument");
  System* s = h;
  sgpu::NetState* ns = sgpu::net_of(*s);
  if (!ns) return nfail(SGPU_ERR_STATE, "sgpu_net_get_weights: no network loaded");
  cudaError_t e = cudaMemcpyAsync(w, ns->w, sgpu::NET_NW * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  return e == cudaSuccess ? 0 : ncuda(e, "sgpu_net_get_weights");
}

int sgpu_net_apply(sgpu_handle h, const void* in_dev, void* out_dev, int nvec) {
  if (!h || !in_dev || !out_dev || nvec < 1) return nfail(SGPU_ERR_ARG, "sgpu_net_apply: bad argument");
  System* s = h;
  if (!s->net_ready) return nfail(SGPU_ERR_STATE, "sgpu_net_apply: no network loaded");
  cudaError_t e = cudaMemcpyAsync(out_dev, in_dev, (size_t)nvec * s->NL * sizeof(double2), cudaMemcpyDeviceToDevice,
                                  s->stream);
  if (e == cudaSuccess) e = sgpu::launch_precond_net(*s, (double2*)out_dev, nvec);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  return e == cudaSuccess ? 0 : ncuda(e, "sgpu_net_apply");
}

int sgpu_net_grad(sgpu_handle h, const void* g_dev, const void* t_dev, int nvec, float* grad, double* loss) {
  if (!h || !g_dev || !t_dev || nvec < 1) return nfail(SGPU_ERR_ARG, "sgpu_net_grad: bad argument");
  System* s = h;
  sgpu::NetState* ns = sgpu::net_of(*s);
  if (!s->net_ready || !ns) return nfail(SGPU_ERR_STATE, "sgpu_net_grad: no network loaded");
  cudaError_t e = sgpu::net_reserve(*s, *ns, nvec);
  if (e == cudaSuccess) e = sgpu::net_loss_grad(*s, *ns, (const double2*)g_dev, (const double2*)t_dev, nvec);
  if (e == cudaSuccess && grad)
    e = cudaMemcpyAsync(grad, ns->grad, sgpu::NET_NW * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess && loss) e = cudaMemcpyAsync(loss, ns->loss, sizeof(double), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  return e == cudaSuccess ? 0 : ncuda(e, "sgpu_net_grad");
}

int sgpu_net_train_step(sgpu_handle h, const void* g_dev, const void* t_dev, int nvec, float lr, double* loss) {
  if (!h || !g_dev || !t_dev || nvec < 1 || !(lr > 0.f)) return nfail(SGPU_ERR_ARG, "sgpu_net_train_step: bad argument");
  System* s = h;
  sgpu::NetState* ns = sgpu::net_of(*s);
  if (!s->net_ready || !ns) return nfail(SGPU_ERR_STATE, "sgpu_net_train_step: no network loaded");
  cudaError_t e = sgpu::net_reserve(*s, *ns, nvec);
  if (e == cudaSuccess) e = sgpu::net_loss_grad(*s, *ns, (const double2*)g_dev, (const double2*)t_dev, nvec);
  if (e != cudaSuccess) return ncuda(e, "sgpu_net_train_step");
  const float b1 = 0.9f, b2 = 0.999f;
  ns->adam_t += 1;
  const float c1 = 1.f - powf(b1, (float)ns->adam_t), c2 = 1.f - powf(b2, (float)ns->adam_t);
  sgpu::k_adam<<<(sgpu::NET_NW + 255) / 256, 256, 0, s->launch_stream()>>>(ns->w, ns->m, ns->v2, ns->grad, ns->wb,
                                                                           sgpu::NET_NW, lr, b1, b2, 1e-8f, c1, c2);
  e = cudaGetLastError();
  if (e == cudaSuccess && loss) e = cudaMemcpyAsync(loss, ns->loss, sizeof(double), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  return e == cudaSuccess ? 0 : ncuda(e, "sgpu_net_train_step");
}

}  // extern "C"
