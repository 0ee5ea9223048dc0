// Kernels of the warm-start surrogate (a small MLP with a learned low-rank
// field basis): a BF16 GEMM with FP32 accumulation and a bias / GELU
// epilogue, the GELU backward, column sums, the masked MSE gradient and an
// Adam step.  Only the surrogate uses them; the DSMC timestep has no
// contraction.
#include <cuda_bf16.h>

#include <cstdint>

#include "dsmc_b200.h"

namespace {

using bf16 = __nv_bfloat16;

constexpr int kBM = 128, kBN = 128, kBK = 32, kPadK = 40;

struct GemmArgs {
  int m, n, k;
  const bf16* a;
  int lda;
  const bf16* b;
  int ldb;
  float* c;
  int ldc;
  float beta;
  const float* bias;
  int act;  // 0 none, 1 GELU
  bf16* cb;
  int ldcb;
  int kchunk;  // K range per blockIdx.z (multiple of kBK)
};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678f)) + z * 0.39894228f * expf(-0.5f * z * z);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[m x n] (+)= A[m x k] B[k x n].  AT: A is stored k x m (row-major), so the
// product uses its transpose; BT: B is stored n x k.  A 128x128 tile per CTA,
// 8 warps of 64x32, K in steps of 32 through shared memory ([m][k] and [n][k]
// so that every fragment pair is one 32-bit load).
template <bool AT, bool BT>
__global__ void __launch_bounds__(256) k_gemm(const GemmArgs g) {
  __shared__ __align__(16) bf16 As[kBM][kPadK];
  __shared__ __align__(16) bf16 Bs[kBN][kPadK];
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int kbeg = blockIdx.z * g.kchunk;
  const int kend = min(g.k, kbeg + g.kchunk);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 2, wn = warp & 3;
  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);

  for (int kb = kbeg; kb < kend; kb += kBK) {
#pragma unroll
    for (int it = 0; it < 2; it++) {
      const int idx = tid + it * 256;
      if (!AT) {
        const int r = idx >> 2, kv = (idx & 3) * 8;
        const int gm = m0 + r, gk = kb + kv;
        uint4 v = zero;
        if (gm < g.m && gk < kend) v = *reinterpret_cast<const uint4*>(g.a + (size_t)gm * g.lda + gk);
        *reinterpret_cast<uint4*>(&As[r][kv]) = v;
      } else {
        const int kk = idx >> 4, mv = (idx & 15) * 8;
        const int gk = kb + kk, gm = m0 + mv;
        uint4 v = zero;
        if (gk < kend && gm < g.m) v = *reinterpret_cast<const uint4*>(g.a + (size_t)gk * g.lda + gm);
        const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
        for (int j = 0; j < 8; j++) As[mv + j][kk] = e[j];
      }
      if (BT) {
        const int r = idx >> 2, kv = (idx & 3) * 8;
        const int gn = n0 + r, gk = kb + kv;
        uint4 v = zero;
        if (gn < g.n && gk < kend) v = *reinterpret_cast<const uint4*>(g.b + (size_t)gn * g.ldb + gk);
        *reinterpret_cast<uint4*>(&Bs[r][kv]) = v;
      } else {
        const int kk = idx >> 4, nv = (idx & 15) * 8;
        const int gk = kb + kk, gn = n0 + nv;
        uint4 v = zero;
        if (gk < kend && gn < g.n) v = *reinterpret_cast<const uint4*>(g.b + (size_t)gk * g.ldb + gn);
        const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
        for (int j = 0; j < 8; j++) Bs[nv + j][kk] = e[j];
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 16) {
      uint32_t af[4][4], bfr[4][2];
      const int c = kk + (lane & 3) * 2;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int r = wm * 64 + i * 16 + (lane >> 2);
        af[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][c]);
        af[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][c]);
        af[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][c + 8]);
        af[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][c + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int nn = wn * 32 + j * 8 + (lane >> 2);
        bfr[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[nn][c]);
        bfr[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[nn][c + 8]);
      }
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], af[i], bfr[j]);
    }
    __syncthreads();
  }

  const bool split = gridDim.z > 1;
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int h = 0; h < 4; h++) {
        const int row = m0 + wm * 64 + i * 16 + (lane >> 2) + (h >> 1) * 8;
        const int col = n0 + wn * 32 + j * 8 + (lane & 3) * 2 + (h & 1);
        if (row >= g.m || col >= g.n) continue;
        const float v = acc[i][j][h];
        if (split) {
          atomicAdd(&g.c[(size_t)row * g.ldc + col], v);
          continue;
        }
        float z = v;
        if (g.bias) z += g.bias[col];
        if (g.c) {
          float* cp = &g.c[(size_t)row * g.ldc + col];
          if (g.beta != 0.f) z += g.beta * *cp;
          *cp = z;
        }
        if (g.cb) g.cb[(size_t)row * g.ldcb + col] = __float2bfloat16(g.act == 1 ? gelu(z) : z);
      }
}

__global__ void k_gelu_backward(const float* z, const float* dh, float* dz, bf16* dzb, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float d = dh[i] * gelu_grad(z[i]);
    if (dz) dz[i] = d;
    if (dzb) dzb[i] = __float2bfloat16(d);
  }
}

// out[col] = sum over rows of x[row * ld + col]
__global__ void k_colsum(const float* x, int rows, int cols, int ld, float* out) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; r++) s += x[(size_t)r * ld + col];
  out[col] = s;
}

// Masked MSE: targets that are NaN carry no loss.  dy = scale * 2 (y - t).
__global__ void k_mse_grad(const float* y, const bf16* t, size_t n, float scale, bf16* dyb, float* dy,
                           double* loss, unsigned long long* count) {
  __shared__ double red[32];
  __shared__ unsigned long long cnt[32];
  double s = 0.0;
  unsigned long long c = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float tv = __bfloat162float(t[i]);
    float g = 0.f;
    if (tv == tv) {
      const float e = y[i] - tv;
      s += (double)e * e;
      c++;
      g = scale * 2.f * e;
    }
    if (dyb) dyb[i] = __float2bfloat16(g);
    if (dy) dy[i] = g;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = s;
    cnt[threadIdx.x >> 5] = c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    unsigned long long b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      a += red[w];
      b += cnt[w];
    }
    if (loss) atomicAdd(loss, a);
    if (count) atomicAdd(count, b);
  }
}

// Adam with decoupled weight decay; also refreshes the BF16 copy.
__global__ void k_adam(float* w, const float* g, float* m, float* v, bf16* wb, size_t n, float lr,
                       float b1, float b2, float eps, float c1, float c2, float wd) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float upd = (mi / c1) / (sqrtf(vi / c2) + eps);
    const float wi = w[i] - lr * (upd + wd * w[i]);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
  }
}

__global__ void k_to_bf16(const float* x, bf16* y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

unsigned grid_1d(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b < 4096 ? (b ? b : 1) : 4096);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace

extern "C" {

int dsmc_gemm_bf16(int m, int n, int k, const void* a, int lda, int a_trans, const void* b, int ldb,
                   int b_trans, float* c, int ldc, float beta, const float* bias, int act, void* c_bf16,
                   int ldcb, int split_k, void* stream) {
  if (m <= 0 || n <= 0 || k <= 0 || !a || !b || (!c && !c_bf16)) return DSMC_ERR_ARG;
  // 16-byte vector loads along the contiguous dimension of each operand
  if (k % 8 || lda % 8 || ldb % 8 || !aligned16(a) || !aligned16(b)) return DSMC_ERR_ARG;
  if ((a_trans && m % 8) || (!b_trans && n % 8)) return DSMC_ERR_ARG;
  if (split_k < 1) split_k = 1;
  if (split_k > 1 && (!c || bias || act || c_bf16)) return DSMC_ERR_ARG;
  GemmArgs g;
  g.m = m; g.n = n; g.k = k;
  g.a = static_cast<const bf16*>(a); g.lda = lda;
  g.b = static_cast<const bf16*>(b); g.ldb = ldb;
  g.c = c; g.ldc = ldc; g.beta = beta;
  g.bias = bias; g.act = act;
  g.cb = static_cast<bf16*>(c_bf16); g.ldcb = ldcb;
  const int ksteps = (k + kBK - 1) / kBK;
  const int per = (ksteps + split_k - 1) / split_k;
  g.kchunk = per * kBK;
  const int splits = (k + g.kchunk - 1) / g.kchunk;
  const dim3 grid((n + kBN - 1) / kBN, (m + kBM - 1) / kBM, splits);
  cudaStream_t s = (cudaStream_t)stream;
  if (!a_trans && !b_trans) k_gemm<false, false><<<grid, 256, 0, s>>>(g);
  else if (!a_trans && b_trans) k_gemm<false, true><<<grid, 256, 0, s>>>(g);
  else if (a_trans && !b_trans) k_gemm<true, false><<<grid, 256, 0, s>>>(g);
  else k_gemm<true, true><<<grid, 256, 0, s>>>(g);
  return cudaGetLastError() == cudaSuccess ? DSMC_OK : DSMC_ERR_CUDA;
}

int dsmc_gelu_backward(const float* z, const float* dh, float* dz, void* dz_bf16, size_t n,
                       void* stream) {
  if (!z || !dh || (!dz && !dz_bf16)) return DSMC_ERR_ARG;
  k_gelu_backward<<<grid_1d(n), 256, 0, (cudaStream_t)stream>>>(z, dh, dz, static_cast<bf16*>(dz_bf16), n);
  return cudaGetLastError() == cudaSuccess ? DSMC_OK : DSMC_ERR_CUDA;
}

int dsmc_colsum(const float* x, int rows, int cols, int ld, float* out, void* stream) {
  if (!x || !out || rows < 0 || cols <= 0) return DSMC_ERR_ARG;
  k_colsum<<<(cols + 255) / 256, 256, 0, (cudaStream_t)stream>>>(x, rows, cols, ld, out);
  return cudaGetLastError() == cudaSuccess ? DSMC_OK : DSMC_ERR_CUDA;
}

int dsmc_mse_grad(const float* y, const void* t_bf16, size_t n, float scale, void* dy_bf16, float* dy,
                  double* loss, unsigned long long* count, void* stream) {
  if (!y || !t_bf16) return DSMC_ERR_ARG;
  k_mse_grad<<<grid_1d(n), 256, 0, (cudaStream_t)stream>>>(y, static_cast<const bf16*>(t_bf16), n, scale,
                                                           static_cast<bf16*>(dy_bf16), dy, loss, count);
  return cudaGetLastError() == cudaSuccess ? DSMC_OK : DSMC_ERR_CUDA;
}

int dsmc_adam_step(float* w, const float* g, float* m, float* v, void* w_bf16, size_t n, float lr,
                   float b1, float b2, float eps, int t, float weight_decay, void* stream) {
  if (!w || !g || !m || !v || t < 1) return DSMC_ERR_ARG;
  const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
  k_adam<<<grid_1d(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, static_cast<bf16*>(w_bf16), n, lr, b1,
                                                       b2, eps, c1, c2, weight_decay);
  return cudaGetLastError() == cudaSuccess ? DSMC_OK : DSMC_ERR_CUDA;
}

int dsmc_to_bf16(const float* x, void* y, size_t n, void* stream) {
  if (!x || !y) return DSMC_ERR_ARG;
  k_to_bf16<<<grid_1d(n), 256, 0, (cudaStream_t)stream>>>(x, static_cast<bf16*>(y), n);
  return cudaGetLastError() == cudaSuccess ? DSMC_OK : DSMC_ERR_CUDA;
}

}  // extern "C"
