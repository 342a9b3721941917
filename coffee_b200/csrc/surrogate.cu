// Kernels of the learned warm start (include/coffee_surrogate.h): 3x3x3
// convolutions as BF16 tensor-core implicit GEMMs with FP32 accumulation,
// their gradients, and the elementwise / pooling / loss / Adam kernels of the
// training step.
//
// The convolutions issue mma.sync.m16n8k16 (BF16 in, FP32 accumulate) from
// one warp per 16 output points: the warp's A fragment is 16 points x 16
// input channels of one tap, gathered straight from the channels-last
// activations (two channels per 32-bit load, zero outside the grid), and
// its B fragments are 16 channels x 8 output channels of that tap's
// weights.  The network is small (16-48 channels), so the kernels are
// bound by these gathers through L1, not by the tensor pipe.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "coffee_internal.h"
#include "coffee_surrogate.h"

namespace coffee {
namespace {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ void mma16816(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t ld2(const bf16* p) {
  return __ldg(reinterpret_cast<const unsigned int*>(p));
}

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

struct Grid4 {
  int n, d, h, w;
  __host__ __device__ long long npts() const { return (long long)n * d * h * w; }
};

// (n, z, y, x) of point p
__device__ __forceinline__ void decompose(const Grid4& g, long long p, int& n, int& z, int& y,
                                          int& x) {
  x = (int)(p % g.w);
  long long q = p / g.w;
  y = (int)(q % g.h);
  q /= g.h;
  z = (int)(q % g.d);
  n = (int)(q / g.d);
}

// The point at offset (dz, dy, dx) from (n, z, y, x), or -1 outside the grid.
__device__ __forceinline__ long long neighbour(const Grid4& g, int n, int z, int y, int x, int dz,
                                               int dy, int dx) {
  const int zz = z + dz, yy = y + dy, xx = x + dx;
  if (zz < 0 || zz >= g.d || yy < 0 || yy >= g.h || xx < 0 || xx >= g.w) return -1;
  return (((long long)n * g.d + zz) * g.h + yy) * g.w + xx;
}

// ------------------------------------------------------------ forward
// One warp: points m0 .. m0 + 15, all K = 8 KT output channels.  Thread
// (g = lane / 4, t = lane % 4) gathers A rows g and g + 8 (points m0 + g,
// m0 + g + 8), channels 2t, 2t + 1 and 2t + 8, 2t + 9 of each 16-channel
// chunk; B rows (channels) 2t, 2t + 1, 2t + 8, 2t + 9 of output channel g of
// each 8-channel tile.
template <int KT>
__global__ void __launch_bounds__(128) conv3d_fwd_kernel(const bf16* __restrict__ x, Grid4 g,
                                                         int C, const bf16* __restrict__ wt,
                                                         const float* __restrict__ bias,
                                                         float* __restrict__ z,
                                                         bf16* __restrict__ a, int act,
                                                         float slope) {
  constexpr int K = KT * 8;
  const long long M = g.npts();
  const int lane = threadIdx.x & 31;
  const long long m0 = ((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5) * 16;
  if (m0 >= M) return;
  const int gr = lane >> 2, tq = lane & 3;
  long long p[2] = {m0 + gr, m0 + gr + 8};
  int pn[2], pz[2], py[2], px[2];
  bool pv[2];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    pv[r] = p[r] < M;
    if (pv[r]) decompose(g, p[r], pn[r], pz[r], py[r], px[r]);
    else pn[r] = pz[r] = py[r] = px[r] = 0;
  }
  float acc[KT][4];
#pragma unroll
  for (int j = 0; j < KT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  for (int tap = 0; tap < 27; ++tap) {
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const bf16* src[2];
    bool ok[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const long long q = pv[r] ? neighbour(g, pn[r], pz[r], py[r], px[r], dz, dy, dx) : -1;
      ok[r] = q >= 0;
      src[r] = x + (ok[r] ? q : 0) * (long long)C;
    }
    for (int c0 = 0; c0 < C; c0 += 16) {
      uint32_t A[4];
      A[0] = ok[0] ? ld2(src[0] + c0 + 2 * tq) : 0u;
      A[1] = ok[1] ? ld2(src[1] + c0 + 2 * tq) : 0u;
      A[2] = ok[0] ? ld2(src[0] + c0 + 2 * tq + 8) : 0u;
      A[3] = ok[1] ? ld2(src[1] + c0 + 2 * tq + 8) : 0u;
#pragma unroll
      for (int j = 0; j < KT; ++j) {
        const bf16* wp = wt + ((long long)(j * 8 + gr) * 27 + tap) * C + c0 + 2 * tq;
        const uint32_t B[2] = {ld2(wp), ld2(wp + 8)};
        mma16816(acc[j], A, B);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    if (!pv[r]) continue;
#pragma unroll
    for (int j = 0; j < KT; ++j) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int k = j * 8 + 2 * tq + e;
        const float v = acc[j][2 * r + e] + (bias ? bias[k] : 0.f);
        const long long o = p[r] * K + k;
        if (z) z[o] = v;
        if (a) a[o] = __float2bfloat16_rn(act ? (v > 0.f ? v : slope * v) : v);
      }
    }
  }
}

template <int KT>
void launch_fwd(const bf16* x, Grid4 g, int C, const bf16* w, const float* bias, float* z, bf16* a,
                int act, float slope, cudaStream_t st) {
  const long long warps = (g.npts() + 15) / 16;
  const unsigned blocks = (unsigned)((warps + 3) / 4);
  conv3d_fwd_kernel<KT><<<blocks, 128, 0, st>>>(x, g, C, w, bias, z, a, act, slope);
}

int fwd_dispatch(const bf16* x, Grid4 g, int C, const bf16* w, int K, const float* bias, float* z,
                 bf16* a, int act, float slope, cudaStream_t st) {
  switch (K / 8) {
    case 1: launch_fwd<1>(x, g, C, w, bias, z, a, act, slope, st); break;
    case 2: launch_fwd<2>(x, g, C, w, bias, z, a, act, slope, st); break;
    case 3: launch_fwd<3>(x, g, C, w, bias, z, a, act, slope, st); break;
    case 4: launch_fwd<4>(x, g, C, w, bias, z, a, act, slope, st); break;
    case 5: launch_fwd<5>(x, g, C, w, bias, z, a, act, slope, st); break;
    case 6: launch_fwd<6>(x, g, C, w, bias, z, a, act, slope, st); break;
    case 7: launch_fwd<7>(x, g, C, w, bias, z, a, act, slope, st); break;
    case 8: launch_fwd<8>(x, g, C, w, bias, z, a, act, slope, st); break;
    default: return fail(COFFEE_E_INVALID, "output channels must be 8..64 in steps of 8 (%d)", K);
  }
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

__global__ void flip_weights_kernel(const bf16* __restrict__ w, int K, int C, bf16* __restrict__ wt) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)K * 27 * C;
  if (i >= n) return;
  const int c = (int)(i % C);
  const int tap = (int)((i / C) % 27);
  const int k = (int)(i / (27LL * C));
  wt[((long long)c * 27 + (26 - tap)) * K + k] = w[i];
}

// ------------------------------------------------------- weight gradient
// dw[k, tap, c] = sum_p dy[p, k] x[p + off(tap), c] as a GEMM over points:
// A = dy^T (16 output channels x 16 points), B = shifted x (16 points x 8
// channels).  Warp w of block b sums the points of chunk 4 b + w for one tap
// (blockIdx.y) and 16 output channels (blockIdx.z) and writes its partial
// sums; wgrad_reduce_kernel adds the chunks in order.
constexpr int kWgradChunks = 128;

template <int CT>
__global__ void __launch_bounds__(128) conv3d_wgrad_kernel(const bf16* __restrict__ dy,
                                                           const bf16* __restrict__ x, Grid4 g,
                                                           int K, long long chunk_pts,
                                                           float* __restrict__ part) {
  constexpr int C = CT * 8;
  const long long M = g.npts();
  const int lane = threadIdx.x & 31, gr = lane >> 2, tq = lane & 3;
  const int chunk = blockIdx.x * 4 + (threadIdx.x >> 5);
  const int tap = blockIdx.y;
  const int k0 = blockIdx.z * 16;
  const int dz = tap / 9 - 1, dyo = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
  const long long pbeg = (long long)chunk * chunk_pts;
  const long long pend = min(M, pbeg + chunk_pts);
  float acc[CT][4];
#pragma unroll
  for (int j = 0; j < CT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  const bf16 zero = __float2bfloat16_rn(0.f);
  for (long long q0 = pbeg; q0 < pend; q0 += 16) {
    // this thread's points: q0 + 2t, +1, +8, +9
    const long long qs[4] = {q0 + 2 * tq, q0 + 2 * tq + 1, q0 + 2 * tq + 8, q0 + 2 * tq + 9};
    const bf16* dyp[4];
    const bf16* xp[4];
    bool dv[4], xv[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      dv[s] = qs[s] < pend;
      long long nb = -1;
      if (dv[s]) {
        int n, z, y, xx;
        decompose(g, qs[s], n, z, y, xx);
        nb = neighbour(g, n, z, y, xx, dz, dyo, dx);
      }
      xv[s] = nb >= 0;
      dyp[s] = dy + (dv[s] ? qs[s] : 0) * (long long)K;
      xp[s] = x + (xv[s] ? nb : 0) * (long long)C;
    }
    uint32_t A[4];
    {
      const bf16 d00 = dv[0] ? dyp[0][k0 + gr] : zero, d01 = dv[1] ? dyp[1][k0 + gr] : zero;
      const bf16 d10 = dv[0] ? dyp[0][k0 + gr + 8] : zero, d11 = dv[1] ? dyp[1][k0 + gr + 8] : zero;
      const bf16 d20 = dv[2] ? dyp[2][k0 + gr] : zero, d21 = dv[3] ? dyp[3][k0 + gr] : zero;
      const bf16 d30 = dv[2] ? dyp[2][k0 + gr + 8] : zero, d31 = dv[3] ? dyp[3][k0 + gr + 8] : zero;
      A[0] = pack2(d00, d01);
      A[1] = pack2(d10, d11);
      A[2] = pack2(d20, d21);
      A[3] = pack2(d30, d31);
    }
#pragma unroll
    for (int j = 0; j < CT; ++j) {
      const int c = j * 8 + gr;
      const bf16 x0 = xv[0] ? xp[0][c] : zero, x1 = xv[1] ? xp[1][c] : zero;
      const bf16 x2 = xv[2] ? xp[2][c] : zero, x3 = xv[3] ? xp[3][c] : zero;
      const uint32_t B[2] = {pack2(x0, x1), pack2(x2, x3)};
      mma16816(acc[j], A, B);
    }
  }
#pragma unroll
  for (int j = 0; j < CT; ++j) {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = k0 + gr + (e >= 2 ? 8 : 0);
      const int c = j * 8 + 2 * tq + (e & 1);
      part[(((long long)chunk * K + k) * 27 + tap) * C + c] = acc[j][e];
    }
  }
}

__global__ void wgrad_reduce_kernel(const float* __restrict__ part, long long n, int chunks,
                                    float* __restrict__ dw) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int q = 0; q < chunks; ++q) s += part[(long long)q * n + i];
  dw[i] = s;
}

template <int CT>
void launch_wgrad(const bf16* dy, const bf16* x, Grid4 g, int K, float* part, cudaStream_t st) {
  const long long M = g.npts();
  long long chunk_pts = (M + kWgradChunks - 1) / kWgradChunks;
  chunk_pts = (chunk_pts + 15) / 16 * 16;
  const dim3 grid(kWgradChunks / 4, 27, (unsigned)(K / 16));
  conv3d_wgrad_kernel<CT><<<grid, 128, 0, st>>>(dy, x, g, K, chunk_pts, part);
}

// ------------------------------------------------------------ elementwise

// db[k] = sum over points of dz[p][k], in two deterministic passes: block b
// of bias_grad_part_kernel sums points [b * per, (b + 1) * per) with
// coalesced reads (blockDim = K * R threads: thread t always adds channel
// t % K, rows t / K, t / K + R, ...), reduces its R rows per channel in a
// fixed order and writes g_bias_part[b][k]; bias_grad_sum_kernel adds the
// blocks in order.
constexpr int kBiasBlocks = 296;
constexpr int kBiasMaxK = 64;
__device__ float g_bias_part[kBiasBlocks * kBiasMaxK];

__global__ void bias_grad_part_kernel(const float* __restrict__ dz, long long npts, int K,
                                      long long per) {
  __shared__ float red[256];
  const int t = threadIdx.x, R = blockDim.x / K, k = t % K, r = t / K;
  const long long p0 = blockIdx.x * per, p1 = min(npts, p0 + per);
  float s = 0.f;
  for (long long p = p0 + r; p < p1; p += R) s += dz[p * K + k];
  red[t] = s;
  __syncthreads();
  if (r == 0) {
    float a = 0.f;
    for (int q = 0; q < R; ++q) a += red[q * K + k];
    g_bias_part[blockIdx.x * kBiasMaxK + k] = a;
  }
}

__global__ void bias_grad_sum_kernel(int K, int blocks, float* __restrict__ db) {
  const int k = threadIdx.x;
  if (k >= K) return;
  float s = 0.f;
  for (int b = 0; b < blocks; ++b) s += g_bias_part[b * kBiasMaxK + k];
  db[k] = s;
}

__global__ void leaky_bwd_kernel(const float* __restrict__ da, const float* __restrict__ z,
                                 long long n, float slope, float* __restrict__ dz,
                                 bf16* __restrict__ dzb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = da[i] * (z[i] > 0.f ? 1.f : slope);
    if (dz) dz[i] = v;
    if (dzb) dzb[i] = __float2bfloat16_rn(v);
  }
}

__global__ void pool2_fwd_kernel(const bf16* __restrict__ x, Grid4 g, int C, bf16* __restrict__ y) {
  const Grid4 h{g.n, g.d / 2, g.h / 2, g.w / 2};
  const long long n = h.npts() * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    int nn, z, yy, xx;
    decompose(h, i / C, nn, z, yy, xx);
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long p = (((long long)nn * g.d + 2 * z + (q >> 2)) * g.h + 2 * yy + ((q >> 1) & 1)) *
                              g.w + 2 * xx + (q & 1);
      s += __bfloat162float(x[p * C + c]);
    }
    y[i] = __float2bfloat16_rn(s * 0.125f);
  }
}

__global__ void pool2_bwd_add_kernel(const float* __restrict__ dy, Grid4 g, int C,
                                     float* __restrict__ dx) {
  const Grid4 h{g.n, g.d / 2, g.h / 2, g.w / 2};
  const long long n = g.npts() * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    int nn, z, yy, xx;
    decompose(g, i / C, nn, z, yy, xx);
    const long long p = (((long long)nn * h.d + z / 2) * h.h + yy / 2) * h.w + xx / 2;
    dx[i] += dy[p * C + c] * 0.125f;
  }
}

__global__ void up2_fwd_kernel(const bf16* __restrict__ x, Grid4 g, int C, bf16* __restrict__ y,
                               int cy, int off) {
  const Grid4 f{g.n, g.d * 2, g.h * 2, g.w * 2};
  const long long n = f.npts() * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long long pf = i / C;
    int nn, z, yy, xx;
    decompose(f, pf, nn, z, yy, xx);
    const long long p = (((long long)nn * g.d + z / 2) * g.h + yy / 2) * g.w + xx / 2;
    y[pf * cy + off + c] = x[p * C + c];
  }
}

__global__ void up2_bwd_kernel(const float* __restrict__ dy, Grid4 g, int C, int cy, int off,
                               float* __restrict__ dx) {
  const Grid4 f{g.n, g.d * 2, g.h * 2, g.w * 2};
  const long long n = g.npts() * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    int nn, z, yy, xx;
    decompose(g, i / C, nn, z, yy, xx);
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long p = (((long long)nn * f.d + 2 * z + (q >> 2)) * f.h + 2 * yy + ((q >> 1) & 1)) *
                              f.w + 2 * xx + (q & 1);
      s += dy[p * cy + off + c];
    }
    dx[i] = s;
  }
}

__global__ void channels_copy_kernel(const bf16* __restrict__ src, long long npts, int c,
                                     bf16* __restrict__ dst, int cdst, int doff) {
  const long long n = npts * c;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[(i / c) * cdst + doff + i % c] = src[i];
}

__global__ void channels_add_kernel(const float* __restrict__ dsrc, long long npts, int csrc,
                                    int soff, int c, float* __restrict__ dx) {
  const long long n = npts * c;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dx[i] += dsrc[(i / c) * csrc + soff + i % c];
}

__global__ void mse_kernel(const float* __restrict__ out, const float* __restrict__ tgt,
                           const float* __restrict__ mask, long long npts, int c, double inv,
                           float* __restrict__ dout, double* __restrict__ partial) {
  const long long n = npts * c;
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float m = mask ? mask[i / c] : 1.f;
    const float d = out[i] - tgt[i];
    dout[i] = (float)(2.0 * inv) * m * d;
    s += (double)m * (double)d * (double)d;
  }
  __shared__ double red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0] * inv;
}

__global__ void sum_partials_kernel(const double* __restrict__ partial, int n,
                                    double* __restrict__ out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += partial[i];  // fixed order
    *out = s;
  }
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, long long n, float lr,
                            float b1, float b2, float eps, float c1, float c2,
                            bf16* __restrict__ wb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

__global__ void to_bf16_kernel(const float* __restrict__ s, long long n, bf16* __restrict__ d) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    d[i] = __float2bfloat16_rn(s[i]);
}

unsigned blocks_for(long long n) {
  return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 32));
}

int check_grid(int n, int d, int h, int w) {
  if (n < 1 || d < 1 || h < 1 || w < 1) return fail(COFFEE_E_INVALID, "empty grid");
  return COFFEE_OK;
}

// ------------------------------------------- forward on tcgen05 (sm_100a)
// The same "same" 3x3x3 convolution as conv3d_fwd_kernel on the fifth-
// generation tensor cores, as an implicit GEMM whose A operand is fetched by
// the tensor memory accelerator:
//
//   * A tile is a box of BX x BY x BZ = 128 points of one sample.  For each
//     stage (one tap, cb = 16, 32 or 64 input channels, the widest that
//     divides C) one thread issues a 5D TMA load of the box shifted by the
//     tap's offset, {c0, x0 + dx, y0 + dy, z0 + dz, n}; the TMA unit writes
//     zeros where the shifted box leaves the grid (the convolution's padding)
//     and lays the 128 rows of 2 cb bytes out with the swizzle of that width,
//     which the MMA's K-major SWIZZLE_32B / 64B / 128B descriptor reads; the
//     stage's cb / 16 MMAs (K 16 each) start 32 bytes apart along the rows.
//   * The weights (N, 27, C) are staged once per persistent CTA in the
//     unswizzled K-major layout: 8-row core matrices of 16-byte rows, the two
//     8-channel halves of a K step LBO bytes apart, 8-row groups 128 apart.
//   * Warp 4 produces (TMA into a kTcStages-deep ring, "full" mbarriers with
//     the expected byte count), warp 5 issues tcgen05.mma (M 128, N, K 16,
//     BF16 in, FP32 accumulate) and commits each step to the ring slot's
//     "empty" mbarrier and each tile to its accumulator's "ready" mbarrier;
//     warps 0-3 read the accumulator back with tcgen05.ld (warp w owns rows
//     32 w .. 32 w + 31) and store.  Two accumulators in tensor memory let
//     the epilogue of one tile overlap the MMAs of the next.
//
// Every wait is bounded (a cycle limit, kTcWaitCycles unless a test sets a
// shorter one) and also ends when another role of the CTA has given up: a
// wait that runs out sets g_tc_fault and the host-visible fault word, the
// roles stop issuing work, the producer waits (with the full bound) for
// every load it has in flight and the MMA thread for what it committed, and
// the CTA frees its tensor memory and returns.  The launching call of the
// next convolution reports COFFEE_E_TIMEOUT until the fault is cleared.
constexpr int kTcM = 128;                         // points per tile = MMA M
constexpr int kTcStages = 8;                      // A ring slots at most
constexpr int kTcSlot = 16384;                    // bytes of one A ring slot (64 channels)
#ifndef COFFEE_TC_FWD_CTAS
#define COFFEE_TC_FWD_CTAS 2
#endif
#ifndef COFFEE_TC_CB48
#define COFFEE_TC_CB48 64
#endif
static_assert(COFFEE_TC_CB48 == 16 || COFFEE_TC_CB48 == 64, "48 channels in 16- or 64-channel boxes");
constexpr int kTcThreads = 192;                   // 4 epilogue warps, producer, MMA
constexpr long long kTcWaitCycles = 4000000000LL; // about 2 s at 1.9 GHz

__device__ int g_tc_fault;

// Launch parameters of the waits: the cycle limit, and (for the test of the
// timeout path only) a producer that issues nothing, so that the MMA
// thread's first wait runs out while no copy or MMA is in flight.
struct TcWaitParams {
  long long cycles;
  int stall_producer;
  int* fault;  // host-mapped word, set on a timeout, read by the launching calls
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: start, LBO, SBO (all >> 4), version 1
// (bits 46-47), base offset 0, layout type at bits 61-63 (0 none, 6 32B swizzle)
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo,
                                             uint32_t layout) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46) | ((uint64_t)layout << 61);
}

// instruction descriptor of kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
__host__ __device__ constexpr uint32_t tc_idesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tc_st16(uint32_t addr, uint4 v) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z),
               "r"(v.w)
               : "memory");
}

// Wait for the phase of parity `parity` of the mbarrier at `mbar`; false if
// it did not complete within kTcWaitCycles or another role gave up (*abort).
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity, volatile int* abort,
                                        const TcWaitParams& wp) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (*abort) return false;
    if (clock64() - t0 > wp.cycles) {
      *abort = 1;
      atomicExch(&g_tc_fault, 1);
      if (wp.fault) atomicExch_system(wp.fault, 1);
      return false;
    }
  }
}

// Wait (bounded by kTcWaitCycles) for the phase of parity `parity` of the
// mbarrier at `mbar`, whatever the other roles do: the drain of work in flight.
__device__ __forceinline__ void tc_drain_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  while (clock64() - t0 < kTcWaitCycles) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return;
  }
}

struct TcBox {
  int bx, by, bz;     // box extent (bx * by * bz = 128)
  int tx, ty, tz;     // boxes per sample along x, y, z
};

template <int N, int CB>
__global__ void __launch_bounds__(kTcThreads) conv3d_fwd_tc_kernel(
    const __grid_constant__ CUtensorMap xmap, Grid4 g, int C, const bf16* __restrict__ w,
    const float* __restrict__ bias, float* __restrict__ z, bf16* __restrict__ a, int act,
    float slope, TcBox box, const TcWaitParams wp, const int nslots) {
  static_assert(N % 16 == 0 && N >= 16 && N <= 64, "N = 16, 32, 48 or 64");
  static_assert(CB == 16 || CB == 32 || CB == 64, "boxes of 16, 32 or 64 channels");
  constexpr int NCOLS = N <= 32 ? 32 : 64;  // columns of one accumulator (power of two >= 32)
  constexpr uint32_t kIdesc = tc_idesc(kTcM, N);
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) unsigned long long full_s[kTcStages], empty_s[kTcStages];
  __shared__ __align__(8) unsigned long long ready_s[2], free_s[2];
  __shared__ uint32_t tmem_s;
  __shared__ int abort_s;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cchunks = C / 16, nks = 27 * cchunks;
  // A box: 128 points x cb channels (16, 32 or 64: rows of 32, 64 or 128
  // bytes under the swizzle of that width), cb / 16 MMAs.  A stage (one ring
  // slot, one full / empty barrier pair) holds U = 64 / cb consecutive boxes,
  // so that every stage feeds up to four MMAs: the barrier round trip per
  // stage, not the tensor pipe, bounded the kernel with one box per stage.
  constexpr int sub = CB / 16;
  constexpr int U = 64 / CB;
  constexpr uint32_t boxb = (uint32_t)(kTcM * CB * 2);
  constexpr uint32_t slot = (uint32_t)kTcSlot;
  static_assert(U * boxb == slot, "a stage fills one slot");
  constexpr uint32_t layout = CB == 16 ? 6u : (CB == 32 ? 4u : 2u);  // 32B / 64B / 128B swizzle
  // boxes per tap; a box may reach past C (C = 48 in 64-channel boxes): the
  // TMA unit fills those channels with zeros and no MMA reads them
  const int bchunks = (C + CB - 1) / CB, units = 27 * bchunks, nstage = (units + U - 1) / U;
  const uint32_t stages = (uint32_t)nslots;
  // A ring at the first 1024-byte boundary (the swizzle atoms repeat every
  // 256 to 1024 bytes), the weights after it
  const uint32_t abase = (smem_addr(tc_smem) + 1023u) & ~1023u;
  const uint32_t wbase = abase + stages * slot;
  const uint32_t full0 = smem_addr(full_s), empty0 = smem_addr(empty_s);
  const uint32_t ready0 = smem_addr(ready_s), free0 = smem_addr(free_s);
  volatile int* abort = &abort_s;

  for (int e = tid; e < nks * N * 2; e += blockDim.x) {
    const int s = e / (N * 2), r = e - s * (N * 2), n = r >> 1, h = r & 1;
    const int tap = s / cchunks, c0 = (s - tap * cchunks) * 16;
    const uint4 v =
        __ldg(reinterpret_cast<const uint4*>(w + ((long long)n * 27 + tap) * C + c0 + 8 * h));
    tc_st16(wbase + (uint32_t)(s * N * 32 + h * (N / 8) * 128 + (n / 8) * 128 + (n % 8) * 16), v);
  }
  if (tid == 0) {
    abort_s = 0;
    for (int b = 0; b < kTcStages; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full0 + 8 * b) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty0 + 8 * b) : "memory");
    }
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(ready0 + 8 * b) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(free0 + 8 * b) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_s)),
                 "r"(2 * NCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_s;

  const long long per_n = (long long)box.tx * box.ty * box.tz;
  const long long ntiles = (long long)g.n * per_n;
  auto tile_origin = [&](long long t, int& n, int& x0, int& y0, int& z0) {
    n = (int)(t / per_n);
    long long r = t - (long long)n * per_n;
    z0 = (int)(r / ((long long)box.tx * box.ty)) * box.bz;
    r %= (long long)box.tx * box.ty;
    y0 = (int)(r / box.tx) * box.by;
    x0 = (int)(r % box.tx) * box.bx;
  };

  if (warp == 4) {
    // ---- producer: one TMA load per K step into the ring
    if (lane == 0) {
      uint32_t step = 0, b = 0, ph = 0;  // slot and phase of step: step % stages, (step / stages) & 1
      const uint64_t map = reinterpret_cast<uint64_t>(&xmap);
      for (long long t = blockIdx.x; t < ntiles && !wp.stall_producer; t += gridDim.x) {
        int n, x0, y0, z0;
        tile_origin(t, n, x0, y0, z0);
        bool ok = true;
        int tap = 0, q = 0;
        for (int s = 0; s < nstage && ok; ++s, ++step) {
          if (step >= stages && !tc_wait(empty0 + 8 * b, ph ^ 1u, abort, wp)) {
            ok = false;
            break;
          }
          const int nb = min(U, units - s * U);  // boxes of this stage
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(full0 + 8 * b),
                       "r"((uint32_t)nb * boxb)
                       : "memory");
          for (int j = 0; j < nb; ++j) {
            const int c0 = q * CB;
            const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
            asm volatile(
                "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(abase + b * slot + (uint32_t)j * boxb),
                "l"(map), "r"(c0), "r"(x0 + dx), "r"(y0 + dy), "r"(z0 + dz), "r"(n),
                "r"(full0 + 8 * b)
                : "memory");
            if (++q == bchunks) {
              q = 0;
              ++tap;
            }
          }
          if (++b == stages) {
            b = 0;
            ph ^= 1u;
          }
        }
        if (!ok) break;
      }
      if (*abort) {
        // every load already issued must land before the CTA's memory goes
        // away: the last `stages` steps are the only ones that can be in
        // flight (a slot is reloaded only after its previous load was
        // consumed), and each is the latest phase of its slot's barrier
        const uint32_t first = step > stages ? step - stages : 0;
        for (uint32_t s2 = first; s2 < step; ++s2)
          tc_drain_wait(full0 + 8 * (s2 % stages), (s2 / stages) & 1);
      }
    }
  } else if (warp == 5) {
    // ---- MMA issuer
    if (lane == 0) {
      uint32_t step = 0, tiles = 0, b = 0, ph = 0;
      bool ok = true;
      for (long long t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++tiles) {
        const uint32_t acc = tiles & 1, use = tiles >> 1;
        if (tiles >= 2 && !tc_wait(free0 + 8 * acc, (use - 1) & 1, abort, wp)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + acc * NCOLS;
        int s16 = 0;  // 16-channel K step of the next MMA
        int cq = 0;   // first channel of the next box
        for (int s = 0; s < nstage; ++s, ++step) {
          if (!tc_wait(full0 + 8 * b, ph, abort, wp)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const int nb = min(U, units - s * U);
          for (int jb = 0; jb < nb; ++jb) {
#pragma unroll
            for (int j = 0; j < sub; ++j) {
              if (cq + 16 * j >= C) break;  // past the tensor's channels
              // K slice j of box jb's swizzled rows: the descriptor start moves 32 bytes
              const uint64_t ad =
                  tc_sdesc(abase + b * slot + (uint32_t)jb * boxb + 32u * j, 16, 8u * CB * 2, layout);
              const uint64_t bd = tc_sdesc(wbase + (uint32_t)(s16 * N * 32), (N / 8) * 128, 128, 0);
              asm volatile(
                  "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                  " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
                  "l"(ad), "l"(bd), "r"(kIdesc), "r"(s16 > 0 ? 1 : 0)
                  : "memory");
              ++s16;
            }
            cq += CB;
            if (cq >= C) cq = 0;
          }
          asm volatile(
              "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                  empty0 + 8 * b)
              : "memory");
          if (++b == stages) {
            b = 0;
            ph ^= 1u;
          }
        }
        if (!ok) break;
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                ready0 + 8 * acc)
            : "memory");
      }
      if (!ok && step > 0) {
        // what was committed must finish before the tensor memory is freed:
        // the commit of the last step tracks every MMA issued before it
        const uint32_t last = step - 1;
        tc_drain_wait(empty0 + 8 * (last % stages), (last / stages) & 1);
      }
    }
  } else {
    // ---- epilogue: warps 0-3, row r = tid of the tile's box
    const int bx = tid % box.bx, by = (tid / box.bx) % box.by, bz = tid / (box.bx * box.by);
    uint32_t tiles = 0;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++tiles) {
      const uint32_t acc = tiles & 1;
      if (!tc_wait(ready0 + 8 * acc, (tiles >> 1) & 1, abort, wp)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t r[N];
#pragma unroll
      for (int c16 = 0; c16 < N / 16; ++c16) {
        const uint32_t taddr =
            tmem + ((uint32_t)(warp * 32) << 16) + acc * NCOLS + (uint32_t)(c16 * 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
            "%10, %11, %12, %13, %14, %15}, [%16];\n"
            : "=r"(r[c16 * 16 + 0]), "=r"(r[c16 * 16 + 1]), "=r"(r[c16 * 16 + 2]),
              "=r"(r[c16 * 16 + 3]), "=r"(r[c16 * 16 + 4]), "=r"(r[c16 * 16 + 5]),
              "=r"(r[c16 * 16 + 6]), "=r"(r[c16 * 16 + 7]), "=r"(r[c16 * 16 + 8]),
              "=r"(r[c16 * 16 + 9]), "=r"(r[c16 * 16 + 10]), "=r"(r[c16 * 16 + 11]),
              "=r"(r[c16 * 16 + 12]), "=r"(r[c16 * 16 + 13]), "=r"(r[c16 * 16 + 14]),
              "=r"(r[c16 * 16 + 15])
            : "r"(taddr)
            : "memory");
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(free0 + 8 * acc) : "memory");
      int n, x0, y0, z0;
      tile_origin(t, n, x0, y0, z0);
      const int px = x0 + bx, py = y0 + by, pz = z0 + bz;
      if (px < g.w && py < g.h && pz < g.d) {
        const long long m = (((long long)n * g.d + pz) * g.h + py) * g.w + px;
#pragma unroll
        for (int k4 = 0; k4 < N; k4 += 4) {
          float v[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) v[e] = __uint_as_float(r[k4 + e]) + (bias ? bias[k4 + e] : 0.f);
          if (z) *reinterpret_cast<float4*>(z + m * N + k4) = make_float4(v[0], v[1], v[2], v[3]);
          if (a) {
            __nv_bfloat162 lo, hi;
            lo.x = __float2bfloat16_rn(act ? (v[0] > 0.f ? v[0] : slope * v[0]) : v[0]);
            lo.y = __float2bfloat16_rn(act ? (v[1] > 0.f ? v[1] : slope * v[1]) : v[1]);
            hi.x = __float2bfloat16_rn(act ? (v[2] > 0.f ? v[2] : slope * v[2]) : v[2]);
            hi.y = __float2bfloat16_rn(act ? (v[3] > 0.f ? v[3] : slope * v[3]) : v[3]);
            uint2 pk;
            pk.x = *reinterpret_cast<uint32_t*>(&lo);
            pk.y = *reinterpret_cast<uint32_t*>(&hi);
            *reinterpret_cast<uint2*>(a + m * N + k4) = pk;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(2 * NCOLS)
                 : "memory");
  }
}

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int encode_fn(EncodeTiledFn* fn) {
  static EncodeTiledFn cached = nullptr;
  if (!cached) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    const cudaError_t err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if (err != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
      return fail(COFFEE_E_CUDA, "cuTensorMapEncodeTiled is not available");
    cached = reinterpret_cast<EncodeTiledFn>(p);
  }
  *fn = cached;
  return COFFEE_OK;
}

int pow2_at_least(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

// Wait parameters of the following launches (coffee_conv3d_tc_set_test_wait)
// and the host-mapped fault word the kernels set on a timeout.
long long g_tc_cycles = kTcWaitCycles;
int g_tc_stall = 0;
volatile int* g_tc_fault_host = nullptr;
int* g_tc_fault_dev = nullptr;

int tc_fault_word() {
  if (g_tc_fault_host) return COFFEE_OK;
  void* h = nullptr;
  COFFEE_CUDA_TRY(cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped));
  *static_cast<volatile int*>(h) = 0;
  void* d = nullptr;
  const cudaError_t err = cudaHostGetDevicePointer(&d, h, 0);
  if (err != cudaSuccess) {
    cudaFreeHost(h);
    return fail(COFFEE_E_CUDA, "cudaHostGetDevicePointer: %s", cudaGetErrorString(err));
  }
  g_tc_fault_host = static_cast<volatile int*>(h);
  g_tc_fault_dev = static_cast<int*>(d);
  return COFFEE_OK;
}

template <int N>
int launch_fwd_tc(const bf16* x, Grid4 g, int C, const bf16* w, const float* bias, float* z,
                  bf16* a, int act, float slope, cudaStream_t st) {
  if (int rc = tc_fault_word()) return rc;
  if (*g_tc_fault_host)
    return fail(COFFEE_E_TIMEOUT,
                "an earlier tcgen05 convolution ran out of time waiting on its pipeline "
                "(its results are invalid); clear the fault with coffee_conv3d_tc_fault");
  // CTAs per SM and ring slots: the most CTAs (up to COFFEE_TC_FWD_CTAS)
  // whose shares of the SM's 228 KB (less 1 KB reserved per CTA) hold the
  // weights and at least two slots; as many slots as fit, at most kTcStages
  const size_t wbytes = (size_t)27 * C * N * 2;
  int nslots = 0, ctas = COFFEE_TC_FWD_CTAS;
  for (; ctas >= 1; --ctas) {
    const long long share = std::min<long long>(227 * 1024, 228LL * 1024 / ctas - 1024);
    nslots = (int)std::min<long long>(kTcStages, (share - 1024 - (long long)wbytes) / kTcSlot);
    if (nslots >= 2) break;
  }
  const size_t smem = 1024 + (size_t)nslots * kTcSlot + wbytes;
  // channels per TMA box: the widest that divides C; 48 channels in
  // COFFEE_TC_CB48-channel boxes: 64 (one box per tap, the last 16 channels
  // zero-filled and not multiplied) or 16 (three boxes per tap, no waste)
  const int cb = C == 48 ? COFFEE_TC_CB48 : (C % 64 == 0 ? 64 : (C % 32 == 0 ? 32 : 16));
  if (ctas < 1 || nslots < 2 || smem > 227 * 1024)
    return fail(COFFEE_E_INVALID, "tcgen05 convolution: %d x %d weights exceed shared memory", N,
                C);
  // the box: x extent a power of two in [8, 128], then y, then z
  TcBox box;
  box.bx = std::min(128, std::max(8, pow2_at_least(g.w)));
  box.by = std::min(128 / box.bx, pow2_at_least(g.h));
  box.bz = 128 / (box.bx * box.by);
  box.tx = (g.w + box.bx - 1) / box.bx;
  box.ty = (g.h + box.by - 1) / box.by;
  box.tz = (g.d + box.bz - 1) / box.bz;
  if (box.bz > 256) return fail(COFFEE_E_INVALID, "tcgen05 convolution: box too deep");
  EncodeTiledFn enc;
  if (int rc = encode_fn(&enc)) return rc;
  CUtensorMap map;
  const cuuint64_t dims[5] = {(cuuint64_t)C, (cuuint64_t)g.w, (cuuint64_t)g.h, (cuuint64_t)g.d,
                              (cuuint64_t)g.n};
  const cuuint64_t strides[4] = {(cuuint64_t)C * 2, (cuuint64_t)C * 2 * g.w,
                                 (cuuint64_t)C * 2 * g.w * g.h, (cuuint64_t)C * 2 * g.w * g.h * g.d};
  const cuuint32_t boxdim[5] = {(cuuint32_t)cb, (cuuint32_t)box.bx, (cuuint32_t)box.by,
                                (cuuint32_t)box.bz, 1};
  const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  const CUresult cr = enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16*>(x), dims,
                          strides, boxdim, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          cb == 16 ? CU_TENSOR_MAP_SWIZZLE_32B
                                   : (cb == 32 ? CU_TENSOR_MAP_SWIZZLE_64B
                                               : CU_TENSOR_MAP_SWIZZLE_128B),
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS)
    return fail(COFFEE_E_INVALID, "tcgen05 convolution: tensor map rejected (%d)", (int)cr);
  auto kern = cb == 64 ? conv3d_fwd_tc_kernel<N, 64>
                       : (cb == 32 ? conv3d_fwd_tc_kernel<N, 32> : conv3d_fwd_tc_kernel<N, 16>);
  COFFEE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // all of the unified L1 / shared memory as shared memory, so that the
  // occupancy below counts every CTA that fits
  COFFEE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
  int dev = 0, sms = 0, per_sm = 0;
  COFFEE_CUDA_TRY(cudaGetDevice(&dev));
  COFFEE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  COFFEE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTcThreads, smem));
  // the resident CTAs of one SM must fit its 512 tensor-memory columns
  // together, so that no tcgen05.alloc waits
  // the occupancy query reported one CTA per SM where the shared memory
  // holds `ctas` (and two measured 1.2-1.6x faster): launch for the shared
  // memory's count; CTAs that do not fit simply start later
  per_sm = std::max(per_sm, ctas);
  per_sm = std::max(1, std::min(per_sm, 512 / (2 * (N <= 32 ? 32 : 64))));
  const long long ntiles = (long long)g.n * box.tx * box.ty * box.tz;
  const unsigned blocks = (unsigned)std::min<long long>(ntiles, (long long)sms * per_sm);
  const TcWaitParams wp{g_tc_cycles, g_tc_stall, g_tc_fault_dev};
  kern<<<blocks, kTcThreads, smem, st>>>(map, g, C, w, bias, z, a, act, slope, box, wp, nslots);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}


// ------------------------------------- weight gradient on tcgen05 (sm_100a)
// dW[k][tap][c] = sum over points p of dy[p][k] x[p + tap][c], as a GEMM
// whose reduction runs over points: D (M 128 x N K) += A (M x 16 points) B
// (16 points x N), with M = TPM taps x CBW channels (TPM = 128 / CBW; CBW
// = 16, 32 or 64 channels, a box of 48 channels zero-filled to 64) and N = K
// output channels.  Both operands are stored point-major, so both are
// MN-major: a 128-point box of x shifted by a tap, loaded by TMA with the
// swizzle of its 2 CBW-byte rows, is one MN atom column of A (TPM such
// boxes side by side, LBO apart, one per tap of the CTA's tap group); the
// unshifted dy box is B.  A CTA owns one tap group and a range of boxes:
// it accumulates in tensor memory over all of them (the TMA unit's zero
// fill outside the grid is the convolution's padding, and zero dy rows
// cover ragged boxes), then writes its 128 x N partial sums; a second kernel
// adds the partials of the point ranges in a fixed order (deterministic).
// Roles, ring, bounded waits and the drain on a timeout are those of
// conv3d_fwd_tc_kernel.
constexpr int kWgTcStages = 4;  // ring slots at most
#ifndef COFFEE_WG_CTAS
#define COFFEE_WG_CTAS 2  // CTAs per SM when their rings fit
#endif

template <int CBW, int KN>
__global__ void __launch_bounds__(kTcThreads) conv3d_wgrad_tc_kernel(
    const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap dymap,
    TcBox box, int ngroups, long long nboxes, long long per_chunk, float* __restrict__ part,
    const TcWaitParams wp, const int nslots) {
  static_assert(CBW == 16 || CBW == 32 || CBW == 64, "x boxes of 16, 32 or 64 channels");
  static_assert(KN == 16 || KN == 32 || KN == 64, "16, 32 or 64 output channels");
  constexpr int TPM = 128 / CBW;                        // taps per M tile
  constexpr uint32_t kAbytes = 128u * 128u * 2u;        // TPM boxes of 128 points x CBW
  constexpr uint32_t kTapBox = 128u * CBW * 2u;         // one x box
  constexpr uint32_t kBbytes = 128u * KN * 2u;          // the dy box
  constexpr uint32_t kSlot = kAbytes + kBbytes;         // multiple of 1024
  constexpr uint32_t kLayoutA = CBW == 16 ? 6u : (CBW == 32 ? 4u : 2u);
  constexpr uint32_t kLayoutB = KN == 16 ? 6u : (KN == 32 ? 4u : 2u);
  constexpr int NCOLS = KN <= 32 ? 32 : 64;
  // kind::f16, FP32 accumulator, BF16 operands, A and B MN-major (bits 15, 16)
  constexpr uint32_t kIdesc = tc_idesc(kTcM, KN) | (1u << 15) | (1u << 16);
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) unsigned long long full_s[kWgTcStages], empty_s[kWgTcStages];
  __shared__ __align__(8) unsigned long long ready_s;
  __shared__ uint32_t tmem_s;
  __shared__ int abort_s;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tg = (int)(blockIdx.x % (unsigned)ngroups);
  const long long chunk = blockIdx.x / (unsigned)ngroups;
  const long long b0 = chunk * per_chunk;
  const long long b1 = min(nboxes, b0 + per_chunk);
  const uint32_t base = (smem_addr(tc_smem) + 1023u) & ~1023u;
  const uint32_t full0 = smem_addr(full_s), empty0 = smem_addr(empty_s);
  const uint32_t ready0 = smem_addr(&ready_s);
  volatile int* abort = &abort_s;

  if (tid == 0) {
    abort_s = 0;
    for (int b = 0; b < kWgTcStages; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full0 + 8 * b) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty0 + 8 * b) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(ready0) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_s)),
                 "r"(NCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_s;

  const long long per_n = (long long)box.tx * box.ty * box.tz;
  auto box_origin = [&](long long t, int& n, int& x0, int& y0, int& z0) {
    n = (int)(t / per_n);
    long long r = t - (long long)n * per_n;
    z0 = (int)(r / ((long long)box.tx * box.ty)) * box.bz;
    r %= (long long)box.tx * box.ty;
    y0 = (int)(r / box.tx) * box.by;
    x0 = (int)(r % box.tx) * box.bx;
  };
  const uint32_t nsteps = (uint32_t)max(0LL, b1 - b0);
  const uint32_t stages = (uint32_t)nslots;

  if (warp == 4) {
    // ---- producer: per box, TPM shifted x boxes and the dy box into a slot
    if (lane == 0) {
      uint32_t step = 0;
      const uint64_t xm = reinterpret_cast<uint64_t>(&xmap);
      const uint64_t dm = reinterpret_cast<uint64_t>(&dymap);
      uint32_t b = 0, ph = 0;  // step % stages, (step / stages) & 1
      for (; step < nsteps && !wp.stall_producer; ++step) {
        if (step >= stages && !tc_wait(empty0 + 8 * b, ph ^ 1u, abort, wp)) break;
        int n, x0, y0, z0;
        box_origin(b0 + step, n, x0, y0, z0);
        const uint32_t slot = base + b * kSlot;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(full0 + 8 * b),
                     "r"(kSlot)
                     : "memory");
#pragma unroll 1
        for (int j = 0; j < TPM; ++j) {
          // taps past the last of the group's (the last group is short) load
          // tap 26 again: their rows of the result are not read
          const int tap = min(tg * TPM + j, 26);
          const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
          asm volatile(
              "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
              "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(slot + (uint32_t)j * kTapBox),
              "l"(xm), "r"(0), "r"(x0 + dx), "r"(y0 + dy), "r"(z0 + dz), "r"(n), "r"(full0 + 8 * b)
              : "memory");
        }
        asm volatile(
            "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(slot + kAbytes),
            "l"(dm), "r"(0), "r"(x0), "r"(y0), "r"(z0), "r"(n), "r"(full0 + 8 * b)
            : "memory");
        if (++b == stages) {
          b = 0;
          ph ^= 1u;
        }
      }
      if (*abort) {
        // the loads of the last `stages` steps may be in flight
        const uint32_t first = step > stages ? step - stages : 0;
        for (uint32_t s2 = first; s2 < step; ++s2)
          tc_drain_wait(full0 + 8 * (s2 % stages), (s2 / stages) & 1);
      }
    }
  } else if (warp == 5) {
    // ---- MMA issuer: 8 MMAs of 16 points per box into one accumulator
    if (lane == 0) {
      uint32_t step = 0, b = 0, ph = 0;
      bool ok = true;
      for (; step < nsteps; ++step) {
        if (!tc_wait(full0 + 8 * b, ph, abort, wp)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t slot = base + b * kSlot;
#pragma unroll
        for (int ks = 0; ks < 8; ++ks) {
          // 16 points: two 8-row groups (SBO apart) of every atom
          const uint64_t ad = tc_sdesc(slot + (uint32_t)ks * 32u * CBW, kTapBox, 16u * CBW, kLayoutA);
          const uint64_t bd =
              tc_sdesc(slot + kAbytes + (uint32_t)ks * 32u * KN, kBbytes, 16u * KN, kLayoutB);
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
              "l"(ad), "l"(bd), "r"(kIdesc), "r"((step > 0 || ks > 0) ? 1 : 0)
              : "memory");
        }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                empty0 + 8 * b)
            : "memory");
        if (++b == stages) {
          b = 0;
          ph ^= 1u;
        }
      }
      if (ok && nsteps > 0) {
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                ready0)
            : "memory");
      } else if (!ok && step > 0) {
        const uint32_t last = step - 1;
        tc_drain_wait(empty0 + 8 * (last % stages), (last / stages) & 1);
      }
    }
  } else {
    // ---- epilogue: warp w reads accumulator rows 32 w .. 32 w + 31
    const int m = tid;  // row of D: tap tg * TPM + m / CBW, channel m % CBW
    float* out = part + ((long long)blockIdx.x * 128 + m) * KN;
    if (nsteps > 0 && tc_wait(ready0, 0, abort, wp)) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      uint32_t r[KN];
#pragma unroll
      for (int c16 = 0; c16 < KN / 16; ++c16) {
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c16 * 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
            "%10, %11, %12, %13, %14, %15}, [%16];\n"
            : "=r"(r[c16 * 16 + 0]), "=r"(r[c16 * 16 + 1]), "=r"(r[c16 * 16 + 2]),
              "=r"(r[c16 * 16 + 3]), "=r"(r[c16 * 16 + 4]), "=r"(r[c16 * 16 + 5]),
              "=r"(r[c16 * 16 + 6]), "=r"(r[c16 * 16 + 7]), "=r"(r[c16 * 16 + 8]),
              "=r"(r[c16 * 16 + 9]), "=r"(r[c16 * 16 + 10]), "=r"(r[c16 * 16 + 11]),
              "=r"(r[c16 * 16 + 12]), "=r"(r[c16 * 16 + 13]), "=r"(r[c16 * 16 + 14]),
              "=r"(r[c16 * 16 + 15])
            : "r"(taddr)
            : "memory");
      }
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int n4 = 0; n4 < KN; n4 += 4)
        *reinterpret_cast<float4*>(out + n4) =
            make_float4(__uint_as_float(r[n4]), __uint_as_float(r[n4 + 1]),
                        __uint_as_float(r[n4 + 2]), __uint_as_float(r[n4 + 3]));
    } else {
#pragma unroll
      for (int n4 = 0; n4 < KN; n4 += 4)
        *reinterpret_cast<float4*>(out + n4) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS)
                 : "memory");
  }
}

// dw[k][tap][c] = the sum over the chunks, in chunk order, of the partial
// sums of conv3d_wgrad_tc_kernel (CTA chunk * ngroups + tap / TPM, row
// (tap % TPM) * CBW + c, column k).
__global__ void wgrad_tc_reduce_kernel(const float* __restrict__ part, int K, int C, int CBW,
                                       int ngroups, int nchunks, float* __restrict__ dw) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long n = (long long)K * 27 * C;
  if (i >= n) return;
  const int k = (int)(i / (27 * C)), r = (int)(i % (27 * C)), tap = r / C, c = r % C;
  const int tpm = 128 / CBW, tg = tap / tpm, m = (tap % tpm) * CBW + c;
  float s = 0.f;
  for (int q = 0; q < nchunks; ++q) s += part[(((long long)q * ngroups + tg) * 128 + m) * K + k];
  dw[i] = s;
}

// Most SMs the chunk count is sized for (the workspace bound).
constexpr int kWgTcMaxSms = 192;

// channels of one x box of the tcgen05 weight gradient (0: not supported)
int wgrad_tc_cbw(int C) { return C == 16 ? 16 : (C == 32 ? 32 : ((C == 48 || C == 64) ? 64 : 0)); }

size_t wgrad_tc_workspace(int K, int C) {
  const int cbw = wgrad_tc_cbw(C);
  if (!cbw) return 0;
  const int groups = (27 + 128 / cbw - 1) / (128 / cbw);
  const long long chunks = std::max(1, COFFEE_WG_CTAS * kWgTcMaxSms / groups);
  return (size_t)chunks * groups * 128 * (size_t)K * sizeof(float);
}

template <int CBW, int KN>
int launch_wgrad_tc(const bf16* dy, const bf16* x, Grid4 g, int C, float* dw, float* part,
                    cudaStream_t st) {
  if (int rc = tc_fault_word()) return rc;
  if (*g_tc_fault_host)
    return fail(COFFEE_E_TIMEOUT,
                "an earlier tcgen05 convolution ran out of time waiting on its pipeline "
                "(its results are invalid); clear the fault with coffee_conv3d_tc_fault");
  constexpr int TPM = 128 / CBW;
  const int groups = (27 + TPM - 1) / TPM;
  TcBox box;
  box.bx = std::min(128, std::max(8, pow2_at_least(g.w)));
  box.by = std::min(128 / box.bx, pow2_at_least(g.h));
  box.bz = 128 / (box.bx * box.by);
  box.tx = (g.w + box.bx - 1) / box.bx;
  box.ty = (g.h + box.by - 1) / box.by;
  box.tz = (g.d + box.bz - 1) / box.bz;
  if (box.bz > 256) return fail(COFFEE_E_INVALID, "tcgen05 weight gradient: box too deep");
  const long long nboxes = (long long)g.n * box.tx * box.ty * box.tz;
  int dev = 0, sms = 0;
  COFFEE_CUDA_TRY(cudaGetDevice(&dev));
  COFFEE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  sms = std::min(sms, kWgTcMaxSms);
  // two CTAs per SM when two rings of at least two slots fit (113 KB each),
  // else one with up to kWgTcStages slots
  const size_t slotb = 128u * 128u * 2u + 128u * KN * 2u;
  int wctas = COFFEE_WG_CTAS, nslots = 0;
  for (; wctas >= 1; --wctas) {
    const long long share = std::min<long long>(227 * 1024, 228LL * 1024 / wctas - 1024);
    nslots = (int)std::min<long long>(kWgTcStages, (share - 1024) / (long long)slotb);
    if (nslots >= 2) break;
  }
  if (wctas < 1) return fail(COFFEE_E_INVALID, "tcgen05 weight gradient: ring exceeds shared memory");
  const size_t smem = 1024 + (size_t)nslots * slotb;
  // one wave of wctas CTAs per SM over all tap groups; every chunk non-empty
  long long chunks = std::max(1LL, std::min(nboxes, (long long)(wctas * sms / groups)));
  const long long per_chunk = (nboxes + chunks - 1) / chunks;
  chunks = (nboxes + per_chunk - 1) / per_chunk;
  EncodeTiledFn enc;
  if (int rc = encode_fn(&enc)) return rc;
  auto make = [&](CUtensorMap* map, const bf16* base, int ch, int boxc,
                  CUtensorMapSwizzle sw) -> int {
    const cuuint64_t dims[5] = {(cuuint64_t)ch, (cuuint64_t)g.w, (cuuint64_t)g.h,
                                (cuuint64_t)g.d, (cuuint64_t)g.n};
    const cuuint64_t strides[4] = {(cuuint64_t)ch * 2, (cuuint64_t)ch * 2 * g.w,
                                   (cuuint64_t)ch * 2 * g.w * g.h,
                                   (cuuint64_t)ch * 2 * g.w * g.h * g.d};
    const cuuint32_t boxdim[5] = {(cuuint32_t)boxc, (cuuint32_t)box.bx, (cuuint32_t)box.by,
                                  (cuuint32_t)box.bz, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult cr = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16*>(base),
                            dims, strides, boxdim, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS)
      return fail(COFFEE_E_INVALID, "tcgen05 weight gradient: tensor map rejected (%d)", (int)cr);
    return COFFEE_OK;
  };
  auto swz = [](int bytes) {
    return bytes == 32 ? CU_TENSOR_MAP_SWIZZLE_32B
                       : (bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B);
  };
  CUtensorMap xmap, dymap;
  if (int rc = make(&xmap, x, C, CBW, swz(2 * CBW))) return rc;
  if (int rc = make(&dymap, dy, KN, KN, swz(2 * KN))) return rc;
  auto kern = conv3d_wgrad_tc_kernel<CBW, KN>;
  COFFEE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  COFFEE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared));
  const TcWaitParams wp{g_tc_cycles, g_tc_stall, g_tc_fault_dev};
  const long long blocks = chunks * groups;
  kern<<<(unsigned)blocks, kTcThreads, smem, st>>>(xmap, dymap, box, groups, nboxes, per_chunk,
                                                   part, wp, nslots);
  COFFEE_CUDA_TRY(cudaGetLastError());
  const long long nw = (long long)KN * 27 * C;
  wgrad_tc_reduce_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, st>>>(part, KN, C, CBW, groups,
                                                                        (int)chunks, dw);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

template <int KN>
int wgrad_tc_dispatch_c(const bf16* dy, const bf16* x, Grid4 g, int C, float* dw, float* part,
                        cudaStream_t st) {
  switch (wgrad_tc_cbw(C)) {
    case 16: return launch_wgrad_tc<16, KN>(dy, x, g, C, dw, part, st);
    case 32: return launch_wgrad_tc<32, KN>(dy, x, g, C, dw, part, st);
    case 64: return launch_wgrad_tc<64, KN>(dy, x, g, C, dw, part, st);
    default: return fail(COFFEE_E_INVALID, "tcgen05 weight gradient: input channels 16, 32, 48 or 64 (%d)", C);
  }
}
}  // namespace
}  // namespace coffee

using namespace coffee;

extern "C" int coffee_conv3d_forward(const void* x, int n, int d, int h, int w, int c,
                                     const void* weight, int k, const float* bias, float* z,
                                     void* a, int act, float slope, void* stream) {
  clear_error();
  if (!x || !weight) return fail(COFFEE_E_INVALID, "coffee_conv3d_forward: null argument");
  if (int rc = check_grid(n, d, h, w)) return rc;
  if (c <= 0 || c % 16) return fail(COFFEE_E_INVALID, "input channels must be a multiple of 16");
  return fwd_dispatch(static_cast<const bf16*>(x), Grid4{n, d, h, w}, c,
                      static_cast<const bf16*>(weight), k, bias, z, static_cast<bf16*>(a), act,
                      slope, static_cast<cudaStream_t>(stream));
}

extern "C" int coffee_conv3d_forward_tc(const void* x, int n, int d, int h, int w, int c,
                                        const void* weight, int k, const float* bias, float* z,
                                        void* a, int act, float slope, void* stream) {
  clear_error();
  if (!x || !weight) return fail(COFFEE_E_INVALID, "coffee_conv3d_forward_tc: null argument");
  if (int rc = check_grid(n, d, h, w)) return rc;
  if (c <= 0 || c % 16) return fail(COFFEE_E_INVALID, "input channels must be a multiple of 16");
  if (reinterpret_cast<uintptr_t>(x) % 16 || reinterpret_cast<uintptr_t>(weight) % 16)
    return fail(COFFEE_E_INVALID, "coffee_conv3d_forward_tc: x and weight must be 16-byte aligned");
  if (reinterpret_cast<uintptr_t>(z) % 16 || reinterpret_cast<uintptr_t>(a) % 8)
    return fail(COFFEE_E_INVALID, "coffee_conv3d_forward_tc: z must be 16-byte, a 8-byte aligned");
  const Grid4 g{n, d, h, w};
  const bf16* xb = static_cast<const bf16*>(x);
  const bf16* wb = static_cast<const bf16*>(weight);
  bf16* ab = static_cast<bf16*>(a);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (k) {
    case 16: return launch_fwd_tc<16>(xb, g, c, wb, bias, z, ab, act, slope, st);
    case 32: return launch_fwd_tc<32>(xb, g, c, wb, bias, z, ab, act, slope, st);
    case 48: return launch_fwd_tc<48>(xb, g, c, wb, bias, z, ab, act, slope, st);
    case 64: return launch_fwd_tc<64>(xb, g, c, wb, bias, z, ab, act, slope, st);
    default: return fail(COFFEE_E_INVALID, "output channels must be 16, 32, 48 or 64 (%d)", k);
  }
}

extern "C" int coffee_conv3d_tc_fault(int* fault, int clear) {
  clear_error();
  if (!fault) return fail(COFFEE_E_INVALID, "coffee_conv3d_tc_fault: null argument");
  COFFEE_CUDA_TRY(cudaMemcpyFromSymbol(fault, g_tc_fault, sizeof(int)));
  if (g_tc_fault_host && *g_tc_fault_host) *fault = 1;
  if (clear) {
    const int zero = 0;
    COFFEE_CUDA_TRY(cudaMemcpyToSymbol(g_tc_fault, &zero, sizeof(int)));
    if (g_tc_fault_host) *g_tc_fault_host = 0;
  }
  return COFFEE_OK;
}

extern "C" int coffee_conv3d_tc_set_test_wait(long long cycles, int stall_producer) {
  clear_error();
  if (cycles < 0) return fail(COFFEE_E_INVALID, "wait limit must be >= 0 cycles");
  g_tc_cycles = cycles > 0 ? cycles : kTcWaitCycles;
  g_tc_stall = stall_producer ? 1 : 0;
  return COFFEE_OK;
}

extern "C" int coffee_conv3d_flip_weights(const void* weight, int k, int c, void* wt,
                                          void* stream) {
  clear_error();
  if (!weight || !wt || k <= 0 || c <= 0)
    return fail(COFFEE_E_INVALID, "coffee_conv3d_flip_weights: bad argument");
  const long long n = (long long)k * 27 * c;
  flip_weights_kernel<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const bf16*>(weight), k, c, static_cast<bf16*>(wt));
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_conv3d_backward_data(const void* dy, int n, int d, int h, int w, int k,
                                           const void* wt, int c, float* dx, void* stream) {
  clear_error();
  if (!dy || !wt || !dx) return fail(COFFEE_E_INVALID, "coffee_conv3d_backward_data: null argument");
  if (int rc = check_grid(n, d, h, w)) return rc;
  if (k <= 0 || k % 16) return fail(COFFEE_E_INVALID, "output channels must be a multiple of 16");
  return fwd_dispatch(static_cast<const bf16*>(dy), Grid4{n, d, h, w}, k,
                      static_cast<const bf16*>(wt), c, nullptr, dx, nullptr, 0, 0.f,
                      static_cast<cudaStream_t>(stream));
}

extern "C" size_t coffee_conv3d_backward_weight_workspace(int k, int c) {
  return std::max((size_t)kWgradChunks * (size_t)k * 27 * (size_t)c * sizeof(float),
                  wgrad_tc_workspace(k, c));
}

extern "C" int coffee_conv3d_backward_weight(const void* dy, const void* x, int n, int d, int h,
                                             int w, int k, int c, float* dw, void* workspace,
                                             void* stream) {
  clear_error();
  if (!dy || !x || !dw || !workspace)
    return fail(COFFEE_E_INVALID, "coffee_conv3d_backward_weight: null argument");
  if (int rc = check_grid(n, d, h, w)) return rc;
  if (k <= 0 || k % 16) return fail(COFFEE_E_INVALID, "output channels must be a multiple of 16");
  if (c <= 0 || c % 8) return fail(COFFEE_E_INVALID, "input channels must be a multiple of 8");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const Grid4 g{n, d, h, w};
  float* part = static_cast<float*>(workspace);
  const bf16* dyb = static_cast<const bf16*>(dy);
  const bf16* xb = static_cast<const bf16*>(x);
  switch (c / 8) {
    case 1: launch_wgrad<1>(dyb, xb, g, k, part, st); break;
    case 2: launch_wgrad<2>(dyb, xb, g, k, part, st); break;
    case 3: launch_wgrad<3>(dyb, xb, g, k, part, st); break;
    case 4: launch_wgrad<4>(dyb, xb, g, k, part, st); break;
    case 5: launch_wgrad<5>(dyb, xb, g, k, part, st); break;
    case 6: launch_wgrad<6>(dyb, xb, g, k, part, st); break;
    case 7: launch_wgrad<7>(dyb, xb, g, k, part, st); break;
    case 8: launch_wgrad<8>(dyb, xb, g, k, part, st); break;
    default: return fail(COFFEE_E_INVALID, "input channels must be 8..64 in steps of 8 (%d)", c);
  }
  COFFEE_CUDA_TRY(cudaGetLastError());
  const long long nw = (long long)k * 27 * c;
  wgrad_reduce_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, st>>>(part, nw, kWgradChunks, dw);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_conv3d_backward_weight_tc(const void* dy, const void* x, int n, int d,
                                                int h, int w, int k, int c, float* dw,
                                                void* workspace, void* stream) {
  clear_error();
  if (!dy || !x || !dw || !workspace)
    return fail(COFFEE_E_INVALID, "coffee_conv3d_backward_weight_tc: null argument");
  if (int rc = check_grid(n, d, h, w)) return rc;
  if (reinterpret_cast<uintptr_t>(dy) % 16 || reinterpret_cast<uintptr_t>(x) % 16 ||
      reinterpret_cast<uintptr_t>(workspace) % 16)
    return fail(COFFEE_E_INVALID,
                "coffee_conv3d_backward_weight_tc: dy, x and workspace must be 16-byte aligned");
  if (!wgrad_tc_cbw(c))
    return fail(COFFEE_E_INVALID, "tcgen05 weight gradient: input channels 16, 32, 48 or 64 (%d)", c);
  const Grid4 g{n, d, h, w};
  const bf16* dyb = static_cast<const bf16*>(dy);
  const bf16* xb = static_cast<const bf16*>(x);
  float* part = static_cast<float*>(workspace);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (k) {
    case 16: return wgrad_tc_dispatch_c<16>(dyb, xb, g, c, dw, part, st);
    case 32: return wgrad_tc_dispatch_c<32>(dyb, xb, g, c, dw, part, st);
    case 64: return wgrad_tc_dispatch_c<64>(dyb, xb, g, c, dw, part, st);
    default: return fail(COFFEE_E_INVALID, "tcgen05 weight gradient: output channels 16, 32 or 64 (%d)", k);
  }
}

extern "C" int coffee_bias_grad(const float* dz, long long npts, int k, float* db, void* stream) {
  clear_error();
  if (!dz || !db || npts <= 0 || k <= 0) return fail(COFFEE_E_INVALID, "coffee_bias_grad: bad argument");
  if (k > kBiasMaxK) return fail(COFFEE_E_INVALID, "coffee_bias_grad: at most %d channels", kBiasMaxK);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long per = (npts + kBiasBlocks - 1) / kBiasBlocks;
  const int blocks = (int)((npts + per - 1) / per);
  const int threads = k * std::max(1, 256 / k);
  bias_grad_part_kernel<<<(unsigned)blocks, (unsigned)threads, 0, st>>>(dz, npts, k, per);
  COFFEE_CUDA_TRY(cudaGetLastError());
  bias_grad_sum_kernel<<<1, kBiasMaxK, 0, st>>>(k, blocks, db);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_leaky_backward(const float* da, const float* z, long long count, float slope,
                                     float* dz, void* dz_bf16, void* stream) {
  clear_error();
  if (!da || !z || count <= 0) return fail(COFFEE_E_INVALID, "coffee_leaky_backward: bad argument");
  leaky_bwd_kernel<<<blocks_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      da, z, count, slope, dz, static_cast<bf16*>(dz_bf16));
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_pool2_forward(const void* x, int n, int d, int h, int w, int c, void* y,
                                    void* stream) {
  clear_error();
  if (!x || !y || d % 2 || h % 2 || w % 2) return fail(COFFEE_E_INVALID, "coffee_pool2_forward: bad argument");
  const Grid4 g{n, d, h, w};
  pool2_fwd_kernel<<<blocks_for(g.npts() / 8 * c), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const bf16*>(x), g, c, static_cast<bf16*>(y));
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_pool2_backward_add(const float* dy, int n, int d, int h, int w, int c,
                                         float* dx, void* stream) {
  clear_error();
  if (!dy || !dx || d % 2 || h % 2 || w % 2) return fail(COFFEE_E_INVALID, "coffee_pool2_backward_add: bad argument");
  const Grid4 g{n, d, h, w};
  pool2_bwd_add_kernel<<<blocks_for(g.npts() * c), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dy, g, c, dx);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_up2_forward(const void* x, int n, int d, int h, int w, int c, void* y,
                                  int cy, int off, void* stream) {
  clear_error();
  if (!x || !y || off < 0 || off + c > cy) return fail(COFFEE_E_INVALID, "coffee_up2_forward: bad argument");
  const Grid4 g{n, d, h, w};
  up2_fwd_kernel<<<blocks_for(g.npts() * 8 * c), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const bf16*>(x), g, c, static_cast<bf16*>(y), cy, off);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_up2_backward(const float* dy, int n, int d, int h, int w, int c, int cy,
                                   int off, float* dx, void* stream) {
  clear_error();
  if (!dy || !dx || off < 0 || off + c > cy) return fail(COFFEE_E_INVALID, "coffee_up2_backward: bad argument");
  const Grid4 g{n, d, h, w};
  up2_bwd_kernel<<<blocks_for(g.npts() * c), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dy, g, c, cy, off, dx);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_channels_copy(const void* src, long long npts, int c, void* dst, int cdst,
                                    int doff, void* stream) {
  clear_error();
  if (!src || !dst || doff < 0 || doff + c > cdst) return fail(COFFEE_E_INVALID, "coffee_channels_copy: bad argument");
  channels_copy_kernel<<<blocks_for(npts * c), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const bf16*>(src), npts, c, static_cast<bf16*>(dst), cdst, doff);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_channels_add(const float* dsrc, long long npts, int csrc, int soff, int c,
                                   float* dx, void* stream) {
  clear_error();
  if (!dsrc || !dx || soff < 0 || soff + c > csrc) return fail(COFFEE_E_INVALID, "coffee_channels_add: bad argument");
  channels_add_kernel<<<blocks_for(npts * c), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dsrc, npts, csrc, soff, c, dx);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_mse(const float* out, const float* target, const float* mask,
                          long long npts, int c, double count, float* dout, double* loss,
                          void* stream) {
  clear_error();
  if (!out || !target || !dout || !loss || !(count > 0)) return fail(COFFEE_E_INVALID, "coffee_mse: bad argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the partial sums live in loss[1 .. 256] (the caller provides 257 doubles)
  const unsigned nb = 256;
  mse_kernel<<<nb, 256, 0, st>>>(out, target, mask, npts, c, 1.0 / count, dout, loss + 1);
  sum_partials_kernel<<<1, 32, 0, st>>>(loss + 1, (int)nb, loss);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_adam(float* w, const float* g, float* m, float* v, long long count,
                           float lr, float beta1, float beta2, float eps, int t, void* w_bf16,
                           void* stream) {
  clear_error();
  if (!w || !g || !m || !v || count <= 0 || t < 1) return fail(COFFEE_E_INVALID, "coffee_adam: bad argument");
  const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
  adam_kernel<<<blocks_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      w, g, m, v, count, lr, beta1, beta2, eps, c1, c2, static_cast<bf16*>(w_bf16));
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}

extern "C" int coffee_to_bf16(const float* src, long long count, void* dst, void* stream) {
  clear_error();
  if (!src || !dst || count <= 0) return fail(COFFEE_E_INVALID, "coffee_to_bf16: bad argument");
  to_bf16_kernel<<<blocks_for(count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      src, count, static_cast<bf16*>(dst));
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
}
