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

__global__ void bias_grad_kernel(const float* __restrict__ dz, long long npts, int K,
                                 float* __restrict__ db) {
  const int k = blockIdx.x;
  float s = 0.f;
  for (long long p = threadIdx.x; p < npts; p += blockDim.x) s += dz[p * K + k];
  __shared__ float red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[k] = red[0];
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
// generation tensor cores: D (128 points x N output channels, FP32) lives in
// tensor memory and is built by 27 C / 16 tcgen05.mma steps of K = 16 (one
// tap, 16 input channels each), issued by one thread.  Both operands come
// from shared memory in the K-major, unswizzled canonical layout: 8-row core
// matrices of 16 bytes per row (128 bytes each), the two 8-channel halves of
// a K step LBO bytes apart and consecutive 8-row groups SBO = 128 bytes
// apart.  A CTA is persistent: it stages the whole weight tensor once, then
// walks its share of 128-point tiles.  Per K step the 128 threads gather
// their point's 16 channels (two 16-byte loads, zeros outside the grid) into
// one of kTcStages A buffers; tcgen05.commit arrives on that buffer's
// mbarrier when the MMA reading it is done, which is what a later step
// waits for before refilling it.  The epilogue reads D back with
// tcgen05.ld (warp w owns points 32 w .. 32 w + 31, one per lane).
//
// Every wait is bounded (kTcWaitCycles); a wait that runs out sets
// g_tc_fault, the block stops issuing work, waits (bounded) for what it has
// in flight, frees its tensor memory and returns.
constexpr int kTcM = 128;                // points per tile = MMA M
constexpr int kTcStages = 4;             // A buffers
constexpr int kTcATile = kTcM * 32;      // bytes of one A buffer (128 x 16 BF16)
constexpr long long kTcWaitCycles = 4000000000LL;  // about 2 s at 1.9 GHz

__device__ int g_tc_fault;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: start, LBO, SBO (all >> 4), version 1
// (bits 46-47), base offset 0, no swizzle (bits 61-63 = 0)
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
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

__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
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
    if (clock64() - t0 > kTcWaitCycles) return false;
  }
}

template <int N>
__global__ void __launch_bounds__(128) conv3d_fwd_tc_kernel(const bf16* __restrict__ x, Grid4 g,
                                                            int C, const bf16* __restrict__ w,
                                                            const float* __restrict__ bias,
                                                            float* __restrict__ z,
                                                            bf16* __restrict__ a, int act,
                                                            float slope) {
  static_assert(N % 16 == 0 && N >= 16 && N <= 64, "N = 16, 32, 48 or 64");
  constexpr int NCOLS = N <= 32 ? 32 : 64;  // tensor-memory columns (a power of two >= 32)
  constexpr uint32_t kIdesc = tc_idesc(kTcM, N);
  extern __shared__ __align__(128) unsigned char tc_smem[];
  __shared__ __align__(8) unsigned long long mbar_s[kTcStages];
  __shared__ uint32_t tmem_s;

  const int tid = threadIdx.x, warp = tid >> 5;
  const int cchunks = C / 16, nks = 27 * cchunks;
  const uint32_t wbase = smem_addr(tc_smem);
  const uint32_t abase = wbase + (uint32_t)(nks * N * 32);
  const uint32_t mbar0 = smem_addr(mbar_s);

  // weights (N, 27, C) -> per K step s = tap * cchunks + chunk: row n, half h
  // at s * N * 32 + h * (N / 8) * 128 + (n / 8) * 128 + (n % 8) * 16
  for (int e = tid; e < nks * N * 2; e += blockDim.x) {
    const int s = e / (N * 2), r = e - s * (N * 2), n = r >> 1, h = r & 1;
    const int tap = s / cchunks, c0 = (s - tap * cchunks) * 16;
    const uint4 v =
        __ldg(reinterpret_cast<const uint4*>(w + ((long long)n * 27 + tap) * C + c0 + 8 * h));
    tc_st16(wbase + (uint32_t)(s * N * 32 + h * (N / 8) * 128 + (n / 8) * 128 + (n % 8) * 16), v);
  }
  if (tid == 0) {
    for (int b = 0; b < kTcStages; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar0 + 8 * b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&tmem_s)),
                 "r"(NCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_s;

  const long long M = g.npts();
  const long long ntiles = (M + kTcM - 1) / kTcM;
  uint32_t step = 0;  // K steps issued by this CTA so far (buffer step % kTcStages)
  bool failed = false;
  const uint32_t a_row = (uint32_t)((tid >> 3) * 128 + (tid & 7) * 16);
  for (long long tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    const long long m = tile * kTcM + tid;
    const bool valid = m < M;
    int pn = 0, pz = 0, py = 0, px = 0;
    if (valid) decompose(g, m, pn, pz, py, px);
    auto gather = [&](int s, uint4& v0, uint4& v1) {
      const int tap = s / cchunks, c0 = (s - tap * cchunks) * 16;
      v0 = make_uint4(0u, 0u, 0u, 0u);
      v1 = v0;
      if (valid) {
        const long long q =
            neighbour(g, pn, pz, py, px, tap / 9 - 1, (tap / 3) % 3 - 1, tap % 3 - 1);
        if (q >= 0) {
          const uint4* p = reinterpret_cast<const uint4*>(x + q * C + c0);
          v0 = __ldg(p);
          v1 = __ldg(p + 1);
        }
      }
    };
    uint4 v0, v1;
    gather(0, v0, v1);
    for (int s = 0; s < nks; ++s, ++step) {
      uint4 n0 = v0, n1 = v1;
      if (s + 1 < nks) gather(s + 1, n0, n1);  // the next step's loads overlap this one
      const uint32_t buf = step % kTcStages;
      bool bad = false;
      if (step >= (uint32_t)kTcStages)  // the MMA that last read this buffer is done
        bad = !tc_wait(mbar0 + 8 * buf, ((step / kTcStages) - 1) & 1);
      const uint32_t ab = abase + buf * kTcATile;
      if (!bad) {
        tc_st16(ab + a_row, v0);
        tc_st16(ab + 2048 + a_row, v1);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      if (__syncthreads_or(bad)) {
        failed = true;
        break;
      }
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint64_t ad = tc_sdesc(ab, 2048, 128);
        const uint64_t bd = tc_sdesc(wbase + (uint32_t)(s * N * 32), (N / 8) * 128, 128);
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(kIdesc), "r"(s > 0 ? 1 : 0)
            : "memory");
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                mbar0 + 8 * buf)
            : "memory");
      }
      v0 = n0;
      v1 = n1;
    }
    if (failed) break;
    const uint32_t last = step - 1;  // its commit covers every MMA of the tile
    const bool bad = !tc_wait(mbar0 + 8 * (last % kTcStages), (last / kTcStages) & 1);
    if (__syncthreads_or(bad)) {
      failed = true;
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
    for (int c16 = 0; c16 < N / 16; ++c16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(c16 * 16);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
          "%11, %12, %13, %14, %15}, [%16];\n"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
            "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr)
          : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (valid) {
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          const int k = c16 * 16 + e;
          const float v = __uint_as_float(r[e]) + (bias ? bias[k] : 0.f);
          const long long o = m * N + k;
          if (z) z[o] = v;
          if (a) a[o] = __float2bfloat16_rn(act ? (v > 0.f ? v : slope * v) : v);
        }
      }
    }
    // every thread's reads of D are complete before the next tile's first
    // MMA overwrites it (that MMA is issued after the next step's barrier)
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  }
  if (failed) {
    if (tid == 0) atomicExch(&g_tc_fault, 1);
    // whatever was committed last must finish before the memory is freed
    if (step > 0) (void)tc_wait(mbar0 + 8 * ((step - 1) % kTcStages), ((step - 1) / kTcStages) & 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOLS)
                 : "memory");
  }
}

template <int N>
int launch_fwd_tc(const bf16* x, Grid4 g, int C, const bf16* w, const float* bias, float* z,
                  bf16* a, int act, float slope, cudaStream_t st) {
  const size_t smem = (size_t)27 * C * N * 2 + (size_t)kTcStages * kTcATile;
  if (smem > 200 * 1024)
    return fail(COFFEE_E_INVALID, "tcgen05 convolution: %d x %d weights exceed shared memory", N,
                C);
  auto kern = conv3d_fwd_tc_kernel<N>;
  COFFEE_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, sms = 0, per_sm = 0;
  COFFEE_CUDA_TRY(cudaGetDevice(&dev));
  COFFEE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  COFFEE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem));
  // resident CTAs of one SM must fit its 512 tensor-memory columns together,
  // so that no tcgen05.alloc waits
  per_sm = std::max(1, std::min(per_sm, 512 / (N <= 32 ? 32 : 64)));
  const long long ntiles = (g.npts() + kTcM - 1) / kTcM;
  const unsigned blocks = (unsigned)std::min<long long>(ntiles, (long long)sms * per_sm);
  kern<<<blocks, 128, smem, st>>>(x, g, C, w, bias, z, a, act, slope);
  COFFEE_CUDA_TRY(cudaGetLastError());
  return COFFEE_OK;
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
  if (clear) {
    const int zero = 0;
    COFFEE_CUDA_TRY(cudaMemcpyToSymbol(g_tc_fault, &zero, sizeof(int)));
  }
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
  return (size_t)kWgradChunks * (size_t)k * 27 * (size_t)c * sizeof(float);
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

extern "C" int coffee_bias_grad(const float* dz, long long npts, int k, float* db, void* stream) {
  clear_error();
  if (!dz || !db || npts <= 0 || k <= 0) return fail(COFFEE_E_INVALID, "coffee_bias_grad: bad argument");
  bias_grad_kernel<<<(unsigned)k, 256, 0, static_cast<cudaStream_t>(stream)>>>(dz, npts, k, db);
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
