// The reference's -mt collisions on the split step: NTC selections of every
// listed cell drawn from that cell's Mersenne Twister, the variant of
// kernels/mtwister.cu:30-117 (19-word state, middle word 9, one lower bit,
// tempering shifts 12/7/15/18; include/MersenneTwister.h:31-40), as
// ComputeBirdCollisionsDev (kernels/dsmc_kernel.cu:1002-1089) draws them.
//
// Per cell the twister's state is 21 words (iState, mti1, mt[19]) and its
// parameters one uint4 (matrix_a, mask_b, mask_c, seed), the layouts of
// mt_state and mt_struct_stripped.  The pair counts come from the order
// kernel in the reference RNG mode (FP64 fpc, kernels/dsmc_kernel.cu:934),
// which lists every cell with pairs for one lane; this kernel takes the place
// of the HybridTaus selections of k_ntc_w.
#include "dsmc_kernels.cuh"
#include "dsmc_step_dev.cuh"

namespace dsmcb {
namespace {

using namespace dev;

constexpr uint32_t kMtWords = 21;

// GetRandomIntegerFast / GetRandomFloatFast (kernels/mtwister.cu:70-106): the
// ring advances one word per draw.
struct MtRng {
  uint32_t mt[19];
  uint32_t i, mti1;
  uint32_t a, b, c;
  __device__ __forceinline__ void load(const uint32_t* st, uint4 cfg) {
    i = st[0] < 19u ? st[0] : 0u;  // the host checks uploaded states; kept in range regardless
    mti1 = st[1];
#pragma unroll
    for (int k = 0; k < 19; k++) mt[k] = st[2 + k];
    a = cfg.x;
    b = cfg.y;
    c = cfg.z;
  }
  __device__ __forceinline__ void store(uint32_t* st) const {
    st[0] = i;
    st[1] = mti1;
#pragma unroll
    for (int k = 0; k < 19; k++) st[2 + k] = mt[k];
  }
  __device__ __forceinline__ uint32_t u32() {
    uint32_t i1 = i + 1u, im = i + 9u;
    if (i1 >= 19u) i1 -= 19u;
    if (im >= 19u) im -= 19u;
    const uint32_t mti = mti1;
    mti1 = mt[i1];
    uint32_t x = (mti & 0xFFFFFFFEu) | (mti1 & 0x1u);
    x = mt[im] ^ (x >> 1) ^ ((x & 1u) ? a : 0u);
    mt[i] = x;
    i = i1;
    x ^= x >> 12;
    x ^= (x << 7) & b;
    x ^= (x << 15) & c;
    x ^= x >> 18;
    return x;
  }
  __device__ __forceinline__ float f32() { return ((float)u32() + 1.0f) / 4294967296.0f; }
};

// InitTwisterFast (kernels/mtwister.cu:108-117) for twisters [0, n).
__global__ void k_mt_init(const uint4* cfg, uint32_t* state, uint32_t n) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  uint32_t* st = state + (size_t)t * kMtWords;
  uint32_t prev = cfg[t].w;
  st[2] = prev;
  for (uint32_t k = 1; k < 19; k++) {
    prev = 1812433253u * (prev ^ (prev >> 30)) + k;
    st[2 + k] = prev;
  }
  st[0] = 0;
  st[1] = st[2];
}

// InitMaximums (kernels/dsmc_kernel.cu:1104-1120): (sigma g)max from the
// settings, the remainder from one draw of the cell's twister.
__global__ void k_mt_maximums(const uint4* cfg, uint32_t* state, float2* maxrem, float max_rel_vel,
                              uint32_t n) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  MtRng r;
  r.load(state + (size_t)t * kMtWords, cfg[t]);
  maxrem[t] = make_float2(max_rel_vel, r.f32());
  r.store(state + (size_t)t * kMtWords);
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_ntc_mt(const __grid_constant__ StepParams p,
                                                       uint32_t* mt_state, const uint4* mt_cfg) {
  chained_entry();
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t col = 0;
  double sum_g = 0.0;
  const uint32_t nl = p.meta->n_light;
  uint32_t* claims = &p.meta->tile_next2;
  uint32_t next = 0;
  if (lane == 0) next = atomicAdd(claims, 32u);
  for (uint32_t base = __shfl_sync(kFull, next, 0); base < nl;) {
    if (lane == 0) next = atomicAdd(claims, 32u);
    const uint32_t i = base + lane;
    base = __shfl_sync(kFull, next, 0);
    if (i >= nl) continue;
    const uint4 e = p.ntc_light[i];  // cell, first sorted slot, count, pairs
    GlobalVel acc{p.mid.u, p.mid.v, p.mid.w, e.y};
    float2 vm = p.maxrem[e.x];
    uint32_t* st = mt_state + (size_t)e.x * kMtWords;
    MtRng r;
    r.load(st, mt_cfg[e.x]);
    float4 stat = make_float4(0.f, 0.f, 0.f, 0.f);
    ntc_select_reference(p, (int)e.z, acc, r, e.w, vm, stat, col, sum_g);
    r.store(st);
    p.maxrem[e.x] = vm;
  }
  // per-block totals, one atomic each
  __shared__ unsigned long long s_col[WARPS];
  __shared__ double s_g[WARPS];
  const unsigned long long c = warp_sum((unsigned long long)col);
  const double g = warp_sum(sum_g);
  if (lane == 0) {
    s_col[threadIdx.x >> 5] = c;
    s_g[threadIdx.x >> 5] = g;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tc = 0;
    double tg = 0.0;
    for (int w = 0; w < WARPS; w++) {
      tc += s_col[w];
      tg += s_g[w];
    }
    if (tc) atomicAdd(&p.meta->collisions, tc);
    if (tg != 0.0) atomicAdd(&p.meta->sum_g, tg);
  }
}

constexpr int kNtcMtWarps = 8;

}  // namespace

cudaError_t launch_mt_init(const uint4* cfg, uint32_t* state, uint32_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  k_mt_init<<<(n + 255u) / 256u, 256, 0, stream>>>(cfg, state, n);
  return cudaGetLastError();
}

cudaError_t launch_mt_maximums(const uint4* cfg, uint32_t* state, float2* maxrem, float max_rel_vel,
                               uint32_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  k_mt_maximums<<<(n + 255u) / 256u, 256, 0, stream>>>(cfg, state, maxrem, max_rel_vel, n);
  return cudaGetLastError();
}

cudaError_t launch_ntc_mt(const StepParams& p, uint32_t* mt_state, const uint4* mt_cfg,
                          cudaStream_t stream) {
  return launch_chained(k_ntc_mt<kNtcMtWarps>, (uint32_t)num_sms() * 8u, kNtcMtWarps * 32, 0, stream, true, p, mt_state,
                        mt_cfg);
}

}  // namespace dsmcb
