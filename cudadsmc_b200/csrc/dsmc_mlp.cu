// Kernels of the warm-start surrogate (a small MLP with a learned low-rank
// field basis): a BF16 GEMM with FP32 accumulation and a bias / GELU
// epilogue, the GELU backward, column sums, the masked MSE gradient and an
// Adam step.  Only the surrogate uses them; the DSMC timestep has no
// contraction.
#include <cuda_bf16.h>

#include <cstdint>

#include "dsmc_b200.h"
#include "dsmc_bulk.cuh"
#include "dsmc_umma.cuh"

// Set by a GEMM whose wait on its tensor-core work ran out (a second);
// dsmc_gemm_check reports and clears it.
__device__ unsigned int g_gemm_failed = 0;

namespace {

using bf16 = __nv_bfloat16;

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
  int kchunk;  // K range per blockIdx.z (multiple of the tile's K step)
};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678f)) + z * 0.39894228f * expf(-0.5f * z * z);
}

// Operand tile of rows [r0, r0 + 128) and k in [k0, k0 + 64) into `dst`:
// TRANS false - stored rows x k (k contiguous, K-major in shared memory);
// TRANS true - stored k x rows (rows contiguous, MN-major).
template <bool TRANS>
__device__ __forceinline__ void umma_load_tile(const bf16* src, int ld, int rows, int r0, int k0, int kend,
                                               bf16* dst) {
  using namespace dsmcb::umma;
  unsigned char* d = reinterpret_cast<unsigned char*>(dst);
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
  for (int it = 0; it < (kBM * kBK / 8) / kThreads; it++) {
    const int c = threadIdx.x + it * kThreads;
    if (!TRANS) {
      const int r = c >> 3, kc = c & 7;
      const int gr = r0 + r, gk = k0 + kc * 8;
      uint4 v = zero;
      if (gr < rows && gk < kend) v = *reinterpret_cast<const uint4*>(src + (size_t)gr * ld + gk);
      *reinterpret_cast<uint4*>(d + kmajor_off((uint32_t)r, (uint32_t)(kc * 8))) = v;
    } else {
      const int kk = c >> 4, rc = c & 15;
      const int gk = k0 + kk, gr = r0 + rc * 8;
      uint4 v = zero;
      if (gk < kend && gr < rows) v = *reinterpret_cast<const uint4*>(src + (size_t)gk * ld + gr);
      *reinterpret_cast<uint4*>(d + mnmajor_off((uint32_t)(rc * 8), (uint32_t)kk)) = v;
    }
  }
}

// C [m x n] (+)= A [m x k] B [k x n] on the tensor cores (tcgen05.mma, the
// accumulator in TMEM): see dsmc_umma.cuh for the tile, the stages and the
// operand layouts.  AT: A is stored k x m (row-major), so the product uses
// its transpose; BT: B is stored n x k.
template <bool AT, bool BT>
__global__ void __launch_bounds__(dsmcb::umma::kThreads, 1) k_gemm_tc(const GemmArgs g) {
  using namespace dsmcb::umma;
  using namespace dsmcb::dev;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Smem& S = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int kbeg = blockIdx.z * g.kchunk;
  const int kend = min(g.k, kbeg + g.kchunk);
  const int ktiles = (kend - kbeg + kBK - 1) / kBK;
  if (tid == 0) {
    mbar_init(&S.mbar[0], 1);
    mbar_init(&S.mbar[1], 1);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(&S.tmem_base, kTmemCols);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = S.tmem_base;
  const uint32_t idesc = instr_desc(AT ? 1u : 0u, BT ? 0u : 1u);
  uint32_t phase0 = 0, phase1 = 0;  // parity of each stage's next completion
  bool ok = true;
  for (int kt = 0; kt < ktiles; kt++) {
    const int s = kt & 1;
    // the stage's MMAs of tile kt - 2 must have read it before it is refilled
    if (kt >= 2) {
      uint32_t& ph = s ? phase1 : phase0;
      ok = mbar_wait_bounded(&S.mbar[s], ph) && ok;
      ph ^= 1u;
    }
    const int k0 = kbeg + kt * kBK;
    umma_load_tile<AT>(g.a, g.lda, g.m, m0, k0, kend, S.a[s]);
    umma_load_tile<!BT>(g.b, g.ldb, g.n, n0, k0, kend, S.b[s]);
    fence_proxy_async();  // the tiles, written by the generic proxy, are read by the tensor cores
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      const uint32_t a0 = su32(S.a[s]), b0 = su32(S.b[s]);
#pragma unroll
      for (int j = 0; j < kBK / 16; j++)
        mma(tmem, smem_desc(a0 + 2u * kLbo * j), smem_desc(b0 + 2u * kLbo * j), idesc,
            (kt > 0 || j > 0) ? 1u : 0u);
      commit(&S.mbar[s]);
    }
  }
  // the last commit completes after every MMA of the tile
  {
    const int sl = (ktiles - 1) & 1;
    ok = mbar_wait_bounded(&S.mbar[sl], sl ? phase1 : phase0) && ok;
  }
  fence_after_sync();
  const bool split = gridDim.z > 1;
  const int row = m0 + 32 * warp + lane;
#pragma unroll 1
  for (int q = 0; q < kBN / 32; q++) {
    float v[32];
    ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(32 * q), v);
    if (row >= g.m) continue;
#pragma unroll
    for (int j = 0; j < 32; j++) {
      const int col = n0 + 32 * q + j;
      if (col >= g.n) continue;
      if (split) {
        atomicAdd(&g.c[(size_t)row * g.ldc + col], v[j]);
        continue;
      }
      float z = v[j];
      if (g.bias) z += g.bias[col];
      if (g.c) {
        float* cp = &g.c[(size_t)row * g.ldc + col];
        if (g.beta != 0.f) z += g.beta * *cp;
        *cp = z;
      }
      if (g.cb) g.cb[(size_t)row * g.ldcb + col] = __float2bfloat16(g.act == 1 ? gelu(z) : z);
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tmem, kTmemCols);
  }
  if (!ok && tid == 0) atomicOr(&g_gemm_failed, 1u);
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

template <bool AT, bool BT>
void launch_tc(dim3 grid, const GemmArgs& g, cudaStream_t s) {
  static bool attr = false;
  const int smem = (int)sizeof(dsmcb::umma::Smem);
  if (!attr) {
    if (cudaFuncSetAttribute(k_gemm_tc<AT, BT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess)
      return;
    attr = true;
  }
  k_gemm_tc<AT, BT><<<grid, dsmcb::umma::kThreads, smem, s>>>(g);
}

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
  using dsmcb::umma::kBK;
  using dsmcb::umma::kBM;
  using dsmcb::umma::kBN;
  const int ksteps = (k + kBK - 1) / kBK;
  const int per = (ksteps + split_k - 1) / split_k;
  g.kchunk = per * kBK;
  const int splits = (k + g.kchunk - 1) / g.kchunk;
  const dim3 grid((n + kBN - 1) / kBN, (m + kBM - 1) / kBM, splits);
  cudaStream_t s = (cudaStream_t)stream;
  if (!a_trans && !b_trans) launch_tc<false, false>(grid, g, s);
  else if (!a_trans && b_trans) launch_tc<false, true>(grid, g, s);
  else if (a_trans && !b_trans) launch_tc<true, false>(grid, g, s);
  else launch_tc<true, true>(grid, g, s);
  return cudaGetLastError() == cudaSuccess ? DSMC_OK : DSMC_ERR_CUDA;
}

int dsmc_gemm_check(void* stream) {
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return DSMC_ERR_CUDA;
  unsigned int f = 0;
  if (cudaMemcpyFromSymbol(&f, g_gemm_failed, sizeof(f)) != cudaSuccess) return DSMC_ERR_CUDA;
  if (!f) return DSMC_OK;
  f = 0;
  if (cudaMemcpyToSymbol(g_gemm_failed, &f, sizeof(f)) != cudaSuccess) return DSMC_ERR_CUDA;
  return DSMC_ERR_DEVICE;
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
