// FP64 ground-state kernels: Gram-Schmidt, the band-by-band CG of the
// reference, and the pieces of the subspace diagonalisation (H_sub = U^H H U,
// Hermitian eigen-decomposition, rotation).  Every reduction is a fixed-order
// CTA reduction (deterministic).  Arrays: zu_GS(NL,NB,NK_s:NK_e) complex(8).
#include <cuda_runtime.h>

#include <cooperative_groups.h>

#include <algorithm>

#include "sgpu_internal.cuh"

namespace sgpu {

constexpr int GS_THREADS = 512;

// ------------------------------------------------------------------ groups --
// The Gram-Schmidt and CG kernels run one thread-block cluster per k-point: the
// cluster's C CTAs split the NL points into contiguous slices, and every inner
// product is a fixed-order CTA sum followed by a sum of the C partials in rank
// order, read from each CTA's shared memory over the cluster (distributed
// shared memory); all CTAs of the cluster obtain the same value.  The
// sequential structure of the reference (band by band, each projection on the
// already updated vector) is kept; the cluster only parallelises each vector
// operation over more SMs.  C = 1 is one CTA per k-point.
namespace cgx = cooperative_groups;

struct Grp {
  int k, rank, C, lo, hi;
  int parity;
  double* part;  // [2][4] this CTA's partial sums (shared memory)
};

__device__ __forceinline__ Grp grp_make(int NL, double* part) {
  cgx::cluster_group cl = cgx::this_cluster();
  Grp g;
  g.C = (int)cl.num_blocks();
  g.rank = (int)cl.block_rank();
  g.k = blockIdx.x / g.C;
  const int slice = (NL + g.C - 1) / g.C;
  g.lo = min(NL, g.rank * slice);
  g.hi = min(NL, g.lo + slice);
  g.parity = 0;
  g.part = part;
  return g;
}

// sum of NV doubles over the k-point's cluster, valid in every thread of every CTA
template <int NV>
__device__ __forceinline__ void grp_allsum(Grp& g, double (&v)[NV], double* sh) {
  block_allsum<NV>(v, sh);
  if (g.C == 1) return;
  cgx::cluster_group cl = cgx::this_cluster();
  if (threadIdx.x == 0)
#pragma unroll
    for (int j = 0; j < NV; ++j) g.part[g.parity * 4 + j] = v[j];
  cl.sync();  // every CTA's partial is in place (and every read of this slot from two sums ago is done)
  double t[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) t[j] = 0.0;
  for (int r = 0; r < g.C; ++r) {
    const double* rp = cl.map_shared_rank(g.part, r);
#pragma unroll
    for (int j = 0; j < NV; ++j) t[j] += rp[g.parity * 4 + j];
  }
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = t[j];
  g.parity ^= 1;
}

// before a CTA of a cluster leaves: no other CTA still reads its shared memory
__device__ __forceinline__ void grp_exit(const Grp& g) {
  if (g.C > 1) cgx::this_cluster().sync();
}

// <a|b> over the NL points (the cluster's sum), valid in every thread
__device__ __forceinline__ double2 grp_zdot(Grp& g, const double2* __restrict__ a, const double2* __restrict__ b,
                                            double* sh) {
  double v[2] = {0.0, 0.0};
  for (int i = g.lo + threadIdx.x; i < g.hi; i += blockDim.x) {
    const double2 x = a[i], y = b[i];
    v[0] = fma(x.x, y.x, fma(x.y, y.y, v[0]));
    v[1] = fma(x.x, y.y, fma(-x.y, y.x, v[1]));
  }
  grp_allsum<2>(g, v, sh);
  return make_double2(v[0], v[1]);
}

__device__ __forceinline__ double grp_nrm2(Grp& g, const double2* __restrict__ a, double* sh) {
  double v[1] = {0.0};
  for (int i = g.lo + threadIdx.x; i < g.hi; i += blockDim.x) {
    const double2 x = a[i];
    v[0] = fma(x.x, x.x, fma(x.y, x.y, v[0]));
  }
  grp_allsum<1>(g, v, sh);
  return v[0];
}

#define GRP_FOR(i) for (int i = g.lo + threadIdx.x; i < g.hi; i += blockDim.x)

// ------------------------------------------------------------ Gram-Schmidt --
// Gram_Schmidt_ompk (GS/Gram_Schmidt.f90:32-55): for each band, subtract the
// projections on the lower bands one by one (each projection uses the band as
// already updated), then normalise.  One cluster per k-point.
__global__ void __launch_bounds__(GS_THREADS) k_gram_schmidt(double2* __restrict__ zu, int NB, int NL, double Hxyz) {
  __shared__ double sh[64];
  __shared__ double part[8];
  Grp g = grp_make(NL, part);
  double2* base = zu + (size_t)g.k * NB * NL;
  for (int ib = 0; ib < NB; ++ib) {
    double2* u = base + (size_t)ib * NL;
    for (int ibt = 0; ibt < ib; ++ibt) {
      const double2* ut = base + (size_t)ibt * NL;
      const double2 d = grp_zdot(g, ut, u, sh);
      const double2 zov = make_double2(d.x * Hxyz, d.y * Hxyz);
      GRP_FOR(i) u[i] = csub(u[i], cmul(ut[i], zov));
    }
    const double s = grp_nrm2(g, u, sh) * Hxyz;
    const double inv = 1.0 / sqrt(s);
    GRP_FOR(i) u[i] = make_double2(u[i].x * inv, u[i].y * inv);
  }
  grp_exit(g);
}

// ---------------------------------------------------------------------- CG --
// CG_ompk with skip_gsortho='n' (GS/CG.f90:34-139), split into kernels around
// the H applications; one cluster per k-point works on band ib of its k-point.
// Work vectors W[which][k][NL] (which = xk, hxk, txk, gk, pk, pko, htpsi, ttpsi):
// each kind is a contiguous batch of one vector per k-point for the H pass.
// Every CTA reads the k-point's state at the start of a kernel; rank 0 writes it
// back only after a cluster-wide sum, i.e. after every CTA has read it.
enum { CG_XK = 0, CG_HXK, CG_TXK, CG_GK, CG_PK, CG_PKO, CG_HT, CG_TT, CG_HK, CG_NW };

struct CGState {
  double xkHxk, gkgk;
  int done, iters;
};

__device__ __forceinline__ double2* wv(double2* W, int nkl, int k, int which, int NL) {
  return W + ((size_t)which * nkl + k) * NL;
}

// Orthogonalise band ib against the lower bands with REAL coefficients (s is
// real(8) in the reference, CG.f90:45,70), normalise into xk.
__global__ void __launch_bounds__(GS_THREADS) k_cg_begin(double2* __restrict__ zu, double2* __restrict__ W,
                                                         CGState* __restrict__ st, int ib, int nkl, int NB, int NL,
                                                         double Hxyz) {
  __shared__ double sh[64];
  __shared__ double part[8];
  Grp g = grp_make(NL, part);
  const int k = g.k;
  double2* base = zu + (size_t)k * NB * NL;
  double2* u = base + (size_t)ib * NL;
  for (int ibt = 0; ibt < ib; ++ibt) {
    const double2* ut = base + (size_t)ibt * NL;
    const double s = grp_zdot(g, ut, u, sh).x * Hxyz;
    GRP_FOR(i) u[i] = make_double2(u[i].x - ut[i].x * s, u[i].y - ut[i].y * s);
  }
  const double inv = 1.0 / sqrt(grp_nrm2(g, u, sh) * Hxyz);
  double2* xk = wv(W, nkl, k, CG_XK, NL);
  GRP_FOR(i) xk[i] = make_double2(u[i].x * inv, u[i].y * inv);
  if (g.rank == 0 && threadIdx.x == 0) { st[k].done = 0; st[k].iters = 0; }
  grp_exit(g);
}

// xkHxk = Re <xk|hxk> Hxyz
__global__ void __launch_bounds__(GS_THREADS) k_cg_dot0(double2* __restrict__ W, CGState* __restrict__ st, int nkl,
                                                        int NL, double Hxyz) {
  __shared__ double sh[64];
  __shared__ double part[8];
  Grp g = grp_make(NL, part);
  const int k = g.k;
  const double d = grp_zdot(g, wv(W, nkl, k, CG_XK, NL), wv(W, nkl, k, CG_HXK, NL), sh).x * Hxyz;
  if (g.rank == 0 && threadIdx.x == 0) st[k].xkHxk = d;
  grp_exit(g);
}

// gradient, orthogonalisation against the lower bands, conjugate direction,
// pko = normalised component of pk orthogonal to xk (CG.f90:85-106)
__global__ void __launch_bounds__(GS_THREADS) k_cg_pre(const double2* __restrict__ zu, double2* __restrict__ W,
                                                       CGState* __restrict__ st, int ib, int iter, int nkl, int NB,
                                                       int NL, double Hxyz) {
  __shared__ double sh[64];
  __shared__ double part[8];
  Grp g = grp_make(NL, part);
  const int k = g.k;
  const CGState st0 = st[k];
  if (st0.done) return;  // uniform over the cluster, before any cluster-wide sum
  const double2* base = zu + (size_t)k * NB * NL;
  double2 *xk = wv(W, nkl, k, CG_XK, NL), *hxk = wv(W, nkl, k, CG_HXK, NL), *gk = wv(W, nkl, k, CG_GK, NL);
  double2 *pk = wv(W, nkl, k, CG_PK, NL), *pko = wv(W, nkl, k, CG_PKO, NL);
  const double xkHxk = st0.xkHxk;
  GRP_FOR(i) gk[i] = make_double2(hxk[i].x - xkHxk * xk[i].x, hxk[i].y - xkHxk * xk[i].y);
  for (int ibt = 0; ibt < ib; ++ibt) {
    const double2* ut = base + (size_t)ibt * NL;
    const double2 d = grp_zdot(g, ut, gk, sh);
    const double2 zs = make_double2(d.x * Hxyz, d.y * Hxyz);
    GRP_FOR(i) gk[i] = csub(gk[i], cmul(ut[i], zs));
  }
  const double s = grp_nrm2(g, gk, sh) * Hxyz;
  if (iter == 1) {
    GRP_FOR(i) pk[i] = gk[i];
  } else {
    const double uk = s / st0.gkgk;
    GRP_FOR(i) pk[i] = make_double2(gk[i].x + uk * pk[i].x, gk[i].y + uk * pk[i].y);
  }
  const double2 d = grp_zdot(g, xk, pk, sh);
  if (g.rank == 0 && threadIdx.x == 0) st[k].gkgk = s;
  const double2 zs = make_double2(d.x * Hxyz, d.y * Hxyz);
  GRP_FOR(i) pko[i] = csub(pk[i], cmul(xk[i], zs));
  const double inv = 1.0 / sqrt(grp_nrm2(g, pko, sh) * Hxyz);
  GRP_FOR(i) pko[i] = make_double2(pko[i].x * inv, pko[i].y * inv);
  grp_exit(g);
}

// Preconditioned variant (no reference counterpart; Payne et al., Rev. Mod.
// Phys. 64, 1045 (1992), section V.B): the gradient gk (as above, orthogonal
// to the lower bands) is preconditioned into hk = K gk by a separate kernel
// chain; k_cg_dir orthogonalises hk against the lower bands and xk, and builds
// the conjugate direction with beta = <gk|hk> / <gk|hk>_previous.
// k_cg_grad also records the kinetic energy of xk (T_band, for the TPA form).
__global__ void __launch_bounds__(GS_THREADS) k_cg_grad(const double2* __restrict__ zu, double2* __restrict__ W,
                                                        CGState* __restrict__ st, double* __restrict__ tband, int ib,
                                                        int nkl, int NB, int NL, double Hxyz) {
  __shared__ double sh[64];
  __shared__ double part[8];
  Grp g = grp_make(NL, part);
  const int k = g.k;
  const CGState st0 = st[k];
  if (st0.done) return;
  const double2* base = zu + (size_t)k * NB * NL;
  double2 *xk = wv(W, nkl, k, CG_XK, NL), *hxk = wv(W, nkl, k, CG_HXK, NL), *gk = wv(W, nkl, k, CG_GK, NL);
  double2* hk = wv(W, nkl, k, CG_HK, NL);
  const double xkHxk = st0.xkHxk;
  GRP_FOR(i) gk[i] = make_double2(hxk[i].x - xkHxk * xk[i].x, hxk[i].y - xkHxk * xk[i].y);
  for (int ibt = 0; ibt < ib; ++ibt) {
    const double2* ut = base + (size_t)ibt * NL;
    const double2 d = grp_zdot(g, ut, gk, sh);
    const double2 zs = make_double2(d.x * Hxyz, d.y * Hxyz);
    GRP_FOR(i) gk[i] = csub(gk[i], cmul(ut[i], zs));
  }
  GRP_FOR(i) hk[i] = gk[i];  // the preconditioner works in place on hk
  const double t = grp_zdot(g, xk, wv(W, nkl, k, CG_TXK, NL), sh).x * Hxyz;
  if (g.rank == 0 && threadIdx.x == 0) tband[k] = t;
  grp_exit(g);
}

__global__ void __launch_bounds__(GS_THREADS) k_cg_dir(const double2* __restrict__ zu, double2* __restrict__ W,
                                                       CGState* __restrict__ st, int ib, int iter, int nkl, int NB,
                                                       int NL, double Hxyz) {
  __shared__ double sh[64];
  __shared__ double part[8];
  Grp g = grp_make(NL, part);
  const int k = g.k;
  const CGState st0 = st[k];
  if (st0.done) return;
  const double2* base = zu + (size_t)k * NB * NL;
  double2 *xk = wv(W, nkl, k, CG_XK, NL), *gk = wv(W, nkl, k, CG_GK, NL), *hk = wv(W, nkl, k, CG_HK, NL);
  double2 *pk = wv(W, nkl, k, CG_PK, NL), *pko = wv(W, nkl, k, CG_PKO, NL);
  for (int ibt = 0; ibt < ib; ++ibt) {
    const double2* ut = base + (size_t)ibt * NL;
    const double2 d = grp_zdot(g, ut, hk, sh);
    const double2 zs = make_double2(d.x * Hxyz, d.y * Hxyz);
    GRP_FOR(i) hk[i] = csub(hk[i], cmul(ut[i], zs));
  }
  {
    const double2 d = grp_zdot(g, xk, hk, sh);
    const double2 zs = make_double2(d.x * Hxyz, d.y * Hxyz);
    GRP_FOR(i) hk[i] = csub(hk[i], cmul(xk[i], zs));
  }
  const double s = grp_zdot(g, gk, hk, sh).x * Hxyz;
  if (iter == 1) {
    GRP_FOR(i) pk[i] = hk[i];
  } else {
    const double uk = s / st0.gkgk;
    GRP_FOR(i) pk[i] = make_double2(hk[i].x + uk * pk[i].x, hk[i].y + uk * pk[i].y);
  }
  const double2 d = grp_zdot(g, xk, pk, sh);
  if (g.rank == 0 && threadIdx.x == 0) st[k].gkgk = s;
  const double2 zs = make_double2(d.x * Hxyz, d.y * Hxyz);
  GRP_FOR(i) pko[i] = csub(pk[i], cmul(xk[i], zs));
  const double inv = 1.0 / sqrt(grp_nrm2(g, pko, sh) * Hxyz);
  GRP_FOR(i) pko[i] = make_double2(pko[i].x * inv, pko[i].y * inv);
  grp_exit(g);
}

// 2x2 Rayleigh-Ritz in span{xk, pko} and the update (CG.f90:108-119)
__global__ void __launch_bounds__(GS_THREADS) k_cg_post(double2* __restrict__ W, CGState* __restrict__ st, int iter,
                                                        int nkl, int NL, double Hxyz, double delta_cg) {
  __shared__ double sh[64];
  __shared__ double part[8];
  Grp g = grp_make(NL, part);
  const int k = g.k;
  const CGState st0 = st[k];
  if (st0.done) return;
  double2 *xk = wv(W, nkl, k, CG_XK, NL), *hxk = wv(W, nkl, k, CG_HXK, NL), *txk = wv(W, nkl, k, CG_TXK, NL);
  const double2 *pko = wv(W, nkl, k, CG_PKO, NL), *ht = wv(W, nkl, k, CG_HT, NL), *tt = wv(W, nkl, k, CG_TT, NL);
  const double xkHxk = st0.xkHxk;
  const double2 d1 = grp_zdot(g, xk, ht, sh);
  const double2 xkHpk = make_double2(d1.x * Hxyz, d1.y * Hxyz);
  const double pkHpk = grp_zdot(g, pko, ht, sh).x * Hxyz;
  const double ev = 0.5 * ((xkHxk + pkHpk) - sqrt((xkHxk - pkHpk) * (xkHxk - pkHpk) +
                                                 4 * (xkHpk.x * xkHpk.x + xkHpk.y * xkHpk.y)));
  double2 cx = make_double2(xkHpk.x / (ev - xkHxk), xkHpk.y / (ev - xkHxk));
  const double cp = 1.0 / sqrt(1.0 + (cx.x * cx.x + cx.y * cx.y));
  cx = make_double2(cx.x * cp, cx.y * cp);
  if (g.rank == 0 && threadIdx.x == 0) st[k].iters = iter;
  if (fabs(ev - xkHxk) < delta_cg) {  // delta_cg = 1e-15 in the reference (CG.f90:42,114)
    if (g.rank == 0 && threadIdx.x == 0) st[k].done = 1;
    grp_exit(g);
    return;
  }
  GRP_FOR(i) {
    xk[i] = cfma(cx, xk[i], make_double2(cp * pko[i].x, cp * pko[i].y));
    hxk[i] = cfma(cx, hxk[i], make_double2(cp * ht[i].x, cp * ht[i].y));
    txk[i] = cfma(cx, txk[i], make_double2(cp * tt[i].x, cp * tt[i].y));
  }
  const double x2 = grp_zdot(g, xk, hxk, sh).x * Hxyz;
  if (g.rank == 0 && threadIdx.x == 0) st[k].xkHxk = x2;
  grp_exit(g);
}

// zu(:,ib) = xk / |xk|; the normalised band is also left in xk for the residual
__global__ void __launch_bounds__(GS_THREADS) k_cg_end(double2* __restrict__ zu, double2* __restrict__ W, int ib,
                                                       int nkl, int NB, int NL, double Hxyz) {
  __shared__ double sh[64];
  __shared__ double part[8];
  Grp g = grp_make(NL, part);
  const int k = g.k;
  double2* xk = wv(W, nkl, k, CG_XK, NL);
  double2* u = zu + ((size_t)k * NB + ib) * NL;
  const double inv = 1.0 / sqrt(grp_nrm2(g, xk, sh) * Hxyz);
  GRP_FOR(i) {
    const double2 v = make_double2(xk[i].x * inv, xk[i].y * inv);
    u[i] = v;
    xk[i] = v;
  }
  grp_exit(g);
}

// esp_var(ib,k) = sqrt(||H u - <u|H u> u||^2 Hxyz) occ(ib,k)  (CG.f90:124-126)
__global__ void __launch_bounds__(GS_THREADS) k_cg_resid(double2* __restrict__ W, const double* __restrict__ occ_gs,
                                                         double* __restrict__ esp_var, double* __restrict__ res,
                                                         int ib, int nkl, int NB, int NL, double Hxyz) {
  __shared__ double sh[64];
  __shared__ double part[8];
  Grp g = grp_make(NL, part);
  const int k = g.k;
  const double2 *u = wv(W, nkl, k, CG_XK, NL), *ht = wv(W, nkl, k, CG_HT, NL);
  const double e = grp_zdot(g, u, ht, sh).x * Hxyz;
  double v[1] = {0.0};
  GRP_FOR(i) {
    const double2 r = make_double2(ht[i].x - e * u[i].x, ht[i].y - e * u[i].y);
    v[0] = fma(r.x, r.x, fma(r.y, r.y, v[0]));
  }
  grp_allsum<1>(g, v, sh);
  if (g.rank == 0 && threadIdx.x == 0) {
    esp_var[(size_t)k * NB + ib] = sqrt(v[0] * Hxyz) * occ_gs[(size_t)k * NB + ib];
    res[(size_t)k * NB + ib] = sqrt(v[0] * Hxyz);  // the residual norm itself, for convergence tests
  }
  grp_exit(g);
}

// ------------------------------------------------------------------ launch --
// CTAs per k-point: enough clusters to cover the SMs about once (C <= 16, a
// power of two, slices of at least 1024 points); 16 needs the non-portable
// cluster size, else 8.
static int gs_cluster_size(const System& s) {
  int C = 1;
  while (C < 16 && s.nkl * C * 2 <= s.nsm && s.NL / (C * 2) >= 1024) C *= 2;
  return C;
}

template <typename Kern, typename... Args>
static cudaError_t launch_gs(const System& s, Kern kern, Args... args) {
  int C = gs_cluster_size(s);
  for (;;) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(s.nkl * C);
    cfg.blockDim = dim3(GS_THREADS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s.launch_stream();
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaSuccess;
    if (C > 8) e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, kern, args...);
    if (e == cudaSuccess || C <= 8) return e;
    (void)cudaGetLastError();  // the non-portable size was refused: clear it and use 8
    --s.launches;
    C = 8;
  }
}

cudaError_t launch_gram_schmidt(const System& s, double2* zu) {
  return launch_gs(s, k_gram_schmidt, zu, s.NB, s.NL, s.Hxyz);
}
cudaError_t launch_cg_begin(const System& s, double2* zu, double2* W, void* st, int ib) {
  return launch_gs(s, k_cg_begin, zu, W, (CGState*)st, ib, s.nkl, s.NB, s.NL, s.Hxyz);
}
cudaError_t launch_cg_dot0(const System& s, double2* W, void* st) {
  return launch_gs(s, k_cg_dot0, W, (CGState*)st, s.nkl, s.NL, s.Hxyz);
}
cudaError_t launch_cg_pre(const System& s, const double2* zu, double2* W, void* st, int ib, int iter) {
  return launch_gs(s, k_cg_pre, zu, W, (CGState*)st, ib, iter, s.nkl, s.NB, s.NL, s.Hxyz);
}
cudaError_t launch_cg_post(const System& s, double2* W, void* st, int iter) {
  return launch_gs(s, k_cg_post, W, (CGState*)st, iter, s.nkl, s.NL, s.Hxyz, s.cg_delta);
}
cudaError_t launch_cg_end(const System& s, double2* zu, double2* W, int ib) {
  return launch_gs(s, k_cg_end, zu, W, ib, s.nkl, s.NB, s.NL, s.Hxyz);
}
cudaError_t launch_cg_grad(const System& s, const double2* zu, double2* W, void* st, double* tband, int ib) {
  return launch_gs(s, k_cg_grad, zu, W, (CGState*)st, tband, ib, s.nkl, s.NB, s.NL, s.Hxyz);
}
cudaError_t launch_cg_dir(const System& s, const double2* zu, double2* W, void* st, int ib, int iter) {
  return launch_gs(s, k_cg_dir, zu, W, (CGState*)st, ib, iter, s.nkl, s.NB, s.NL, s.Hxyz);
}
cudaError_t launch_cg_resid(const System& s, double2* W, const double* occ_gs, double* esp_var, double* res, int ib) {
  return launch_gs(s, k_cg_resid, W, occ_gs, esp_var, res, ib, s.nkl, s.NB, s.NL, s.Hxyz);
}
size_t cg_state_bytes() { return sizeof(CGState); }
int cg_work_vectors() { return CG_NW; }

// ------------------------------------------------------ subspace H (ZGEMM) --
// part[sp][k][n][m] = sum_{i in split sp} conj(A[k][m][i]) B[k][n][i]
// A, B: [k][NB][NL].  16x16 output tile per CTA, K split over blockIdx.z.
constexpr int GT = 16, GK = 32;

__global__ void __launch_bounds__(GT * GT) k_zgemm_hn(const double2* __restrict__ A, const double2* __restrict__ B,
                                                     int NB, int NL, int kchunk, double2* __restrict__ part) {
  __shared__ double2 sa[GT][GK + 1], sb[GT][GK + 1];
  const int k = blockIdx.x / ((NB + GT - 1) / GT);
  const int tm = blockIdx.x % ((NB + GT - 1) / GT), tn = blockIdx.y;
  const int sp = blockIdx.z;
  const int tx = threadIdx.x % GT, ty = threadIdx.x / GT;
  const int m = tm * GT + tx, n = tn * GT + ty;
  const int i0 = sp * kchunk, i1 = min(i0 + kchunk, NL);
  const double2* Ak = A + (size_t)k * NB * NL;
  const double2* Bk = B + (size_t)k * NB * NL;
  double2 acc = make_double2(0, 0);
  for (int ib = i0; ib < i1; ib += GK) {
    for (int e = threadIdx.x; e < GT * GK; e += GT * GT) {
      const int r = e / GK, c = e % GK, i = ib + c;
      const int mr = tm * GT + r, nr = tn * GT + r;
      sa[r][c] = (mr < NB && i < i1) ? Ak[(size_t)mr * NL + i] : make_double2(0, 0);
      sb[r][c] = (nr < NB && i < i1) ? Bk[(size_t)nr * NL + i] : make_double2(0, 0);
    }
    __syncthreads();
#pragma unroll 8
    for (int c = 0; c < GK; ++c) acc = cfmaj(sa[tx][c], sb[ty][c], acc);
    __syncthreads();
  }
  const int nkl = gridDim.x / ((NB + GT - 1) / GT);
  if (m < NB && n < NB) part[(((size_t)sp * nkl + k) * NB + n) * NB + m] = acc;
}

// za[k][n][m] = Hxyz * sum_sp part[sp][k][n][m]  then made Hermitian like
// diag_omp builds it (GS/diag.f90:112-116): the lower triangle (m > n) is
// computed, the upper is its conjugate, the diagonal is real.
__global__ void k_zgemm_reduce_herm(const double2* __restrict__ part, int nsplit, int nkl, int NB, double Hxyz,
                                    double2* __restrict__ za) {
  const size_t tot = (size_t)nkl * NB * NB;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e / ((size_t)NB * NB));
    const int n = (int)((e / NB) % NB), m = (int)(e % NB);
    // element (row m, column n) of za(:,:) stored at za[k][n][m] (column-major)
    const int lo_r = m > n ? m : n, lo_c = m > n ? n : m;  // lower-triangle source
    double2 s = make_double2(0, 0);
    for (int sp = 0; sp < nsplit; ++sp) {
      const double2 p = part[(((size_t)sp * nkl + k) * NB + lo_c) * NB + lo_r];
      s.x += p.x;
      s.y += p.y;
    }
    s = make_double2(s.x * Hxyz, s.y * Hxyz);
    if (m == n) s.y = 0.0;
    else if (m < n) s.y = -s.y;
    za[e] = s;
  }
}

cudaError_t launch_subspace_h(const System& s, const double2* U, const double2* HU, double2* part, int nsplit,
                              double2* za) {
  const int nt = (s.NB + GT - 1) / GT;
  const int kchunk = ((s.NL + nsplit - 1) / nsplit + GK - 1) / GK * GK;
  dim3 grid(s.nkl * nt, nt, nsplit);
  k_zgemm_hn<<<grid, GT * GT, 0, s.launch_stream()>>>(U, HU, s.NB, s.NL, kchunk, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const size_t tot = (size_t)s.nkl * s.NB * s.NB;
  k_zgemm_reduce_herm<<<(int)std::min<size_t>((tot + 255) / 256, 4096), 256, 0, s.launch_stream()>>>(part, nsplit, s.nkl, s.NB,
                                                                                             s.Hxyz, za);
  return cudaGetLastError();
}

// ------------------------------------------- Hermitian Jacobi eigensolver --
// Cyclic two-sided Jacobi with the round-robin ordering: each step rotates
// n/2 disjoint index pairs at once (rows, then columns, then the eigenvector
// columns).  For a pair (p,q) with A_pq = |b| e^{i phi}, J = D R with
// D = diag(1, e^{-i phi}) (makes the pair real) and the real Jacobi rotation
// R = [[c, s], [-s, c]], t = sign(tau)/(|tau|+sqrt(1+tau^2)), tau = (a_qq-a_pp)/(2|b|).
// One CTA per k-point; A and V (column-major, [k][col][row]) live in global memory.
// Sweeps stop when the off-diagonal norm is below 1e-15 of the Frobenius norm,
// or after max_sweeps (the count used is written to sweeps[k]).
__device__ __forceinline__ int rr_partner(int i, int step, int n) {
  // round-robin: position 0 fixed, others rotate; returns the partner of index i
  if (i == 0) return 1 + (step % (n - 1));
  int pos = (i - 1 - step) % (n - 1);
  if (pos < 0) pos += n - 1;  // position of i in the rotating ring, 0..n-2
  // positions pair as (ring 0 <-> fixed 0), (ring r <-> ring n-1-r)
  if (pos == 0) return 0;
  const int ppos = n - 1 - pos;
  int idx = (ppos + step) % (n - 1);
  return idx + 1;
}

__global__ void __launch_bounds__(1024) k_jacobi_herm(double2* __restrict__ Aall, double2* __restrict__ Vall, int NB,
                                                      int max_sweeps, double* __restrict__ w, int* __restrict__ sweeps) {
  extern __shared__ double jsh[];
  // rotation parameters per index (owner p < q): c, s, cos(phi), sin(phi), partner
  double* cs = jsh;                      // [NB] c of the pair owned by p
  double* sn = cs + NB;                  // [NB] s
  double* ph_c = sn + NB;                // [NB] cos(phi)
  double* ph_s = ph_c + NB;              // [NB] sin(phi)
  int* partner = (int*)(ph_s + NB);      // [NB]
  __shared__ double sh[64];
  __shared__ int s_conv;
  const int k = blockIdx.x;
  double2* A = Aall + (size_t)k * NB * NB;
  double2* V = Vall + (size_t)k * NB * NB;
#define AE(r, c) A[(size_t)(c) * NB + (r)]
#define VE(r, c) V[(size_t)(c) * NB + (r)]
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) VE(e % NB, e / NB) = make_double2((e % NB) == (e / NB) ? 1.0 : 0.0, 0.0);
  const int n = NB + (NB & 1);  // even count for the round-robin (index NB is a dummy)
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    // convergence test
    double v[2] = {0.0, 0.0};
    for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
      const int r = e % NB, c = e / NB;
      const double2 x = AE(r, c);
      const double m2 = x.x * x.x + x.y * x.y;
      v[0] += m2;
      if (r != c) v[1] += m2;
    }
    block_allsum<2>(v, sh);
    if (threadIdx.x == 0) s_conv = (v[1] <= 1e-30 * v[0]) ? 1 : 0;
    __syncthreads();
    if (s_conv) break;
    for (int step = 0; step < n - 1; ++step) {
      for (int p = threadIdx.x; p < NB; p += blockDim.x) {
        const int q = rr_partner(p, step, n);
        partner[p] = q < NB ? q : -1;
        cs[p] = 1.0; sn[p] = 0.0; ph_c[p] = 1.0; ph_s[p] = 0.0;
        if (q < NB && p < q) {
          const double app = AE(p, p).x, aqq = AE(q, q).x;
          const double2 b = AE(p, q);
          const double ab = sqrt(b.x * b.x + b.y * b.y);
          if (ab > 0.0) {
            const double tau = (aqq - app) / (2.0 * ab);
            const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            const double c = 1.0 / sqrt(1.0 + t * t);
            cs[p] = c; sn[p] = t * c; ph_c[p] = b.x / ab; ph_s[p] = b.y / ab;
          }
        }
      }
      __syncthreads();
      // rows: A <- J^H A  (rows p,q of every column)
      for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
        const int p = e % NB, col = e / NB;
        const int q = partner[p];
        if (q < 0 || p > q) continue;
        const double c = cs[p], s = sn[p];
        const double2 eph = make_double2(ph_c[p], ph_s[p]);  // e^{i phi}
        const double2 ap = AE(p, col), aq = AE(q, col);
        // new_p = c ap - s e^{i phi} aq ; new_q = s ap + c e^{i phi} aq
        const double2 ea = cmul(eph, aq);
        AE(p, col) = make_double2(c * ap.x - s * ea.x, c * ap.y - s * ea.y);
        AE(q, col) = make_double2(s * ap.x + c * ea.x, s * ap.y + c * ea.y);
      }
      __syncthreads();
      // columns: A <- A J, V <- V J  (columns p,q of every row)
      for (int e = threadIdx.x; e < 2 * NB * NB; e += blockDim.x) {
        const int which = e / (NB * NB), rem = e % (NB * NB);
        const int p = rem / NB, row = rem % NB;
        const int q = partner[p];
        if (q < 0 || p > q) continue;
        const double c = cs[p], s = sn[p];
        const double2 emph = make_double2(ph_c[p], -ph_s[p]);  // e^{-i phi}
        double2* M = which ? V : A;
        const double2 xp = M[(size_t)p * NB + row], xq = M[(size_t)q * NB + row];
        // new_p = c xp - s e^{-i phi} xq ; new_q = s xp + c e^{-i phi} xq
        const double2 ex = cmul(emph, xq);
        M[(size_t)p * NB + row] = make_double2(c * xp.x - s * ex.x, c * xp.y - s * ex.y);
        M[(size_t)q * NB + row] = make_double2(s * xp.x + c * ex.x, s * xp.y + c * ex.y);
      }
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) sweeps[k] = sweep;
  // eigenvalues = diag, sorted ascending with the eigenvector columns (like zheev)
  double* wk = w + (size_t)k * NB;
  for (int i = threadIdx.x; i < NB; i += blockDim.x) cs[i] = AE(i, i).x;
  __syncthreads();
  for (int i = threadIdx.x; i < NB; i += blockDim.x) {
    int rank = 0;
    for (int j2 = 0; j2 < NB; ++j2) rank += (cs[j2] < cs[i]) || (cs[j2] == cs[i] && j2 < i);
    partner[i] = rank;
    wk[rank] = cs[i];
  }
  __syncthreads();
  // permuted eigenvectors into A (A is no longer needed)
  for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
    const int row = e % NB, col = e / NB;
    AE(row, partner[col]) = VE(row, col);
  }
#undef AE
#undef VE
}

cudaError_t launch_jacobi(const System& s, double2* A, double2* V, int max_sweeps, double* w, int* sweeps) {
  const size_t smem = (size_t)s.NB * (4 * sizeof(double) + sizeof(int));
  k_jacobi_herm<<<s.nkl, 1024, smem, s.launch_stream()>>>(A, V, s.NB, max_sweeps, w, sweeps);
  return cudaGetLastError();
}

// ------------------------------------------------------------- rotation ---
// out[k][n][i] = sum_m in[k][m][i] Z[k][n][m]   (zutmp(:,ib1) = sum_ib2 zu(:,ib2) za(ib2,ib1), diag.f90:120-126)
constexpr int ROT_NB = 8;
__global__ void __launch_bounds__(256) k_rotate(const double2* __restrict__ in, const double2* __restrict__ Z,
                                                int NB, int NL, double2* __restrict__ out) {
  const int k = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double2* ink = in + (size_t)k * NB * NL;
  const double2* Zk = Z + (size_t)k * NB * NB;
  double2* outk = out + (size_t)k * NB * NL;
  if (i >= NL) return;
  for (int n0 = 0; n0 < NB; n0 += ROT_NB) {
    double2 acc[ROT_NB];
#pragma unroll
    for (int t = 0; t < ROT_NB; ++t) acc[t] = make_double2(0, 0);
    for (int m = 0; m < NB; ++m) {
      const double2 x = ink[(size_t)m * NL + i];
#pragma unroll
      for (int t = 0; t < ROT_NB; ++t)
        if (n0 + t < NB) acc[t] = cfma(x, __ldg(Zk + (size_t)(n0 + t) * NB + m), acc[t]);
    }
#pragma unroll
    for (int t = 0; t < ROT_NB; ++t)
      if (n0 + t < NB) outk[(size_t)(n0 + t) * NL + i] = acc[t];
  }
}

cudaError_t launch_rotate(const System& s, const double2* in, const double2* Z, double2* out) {
  dim3 grid((s.NL + 255) / 256, s.nkl);
  k_rotate<<<grid, 256, 0, s.launch_stream()>>>(in, Z, s.NB, s.NL, out);
  return cudaGetLastError();
}

}  // namespace sgpu
