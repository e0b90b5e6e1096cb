// Device helpers shared by the kernel files: complex arithmetic in the
// reference's forms, warp shuffles of complex values, the 1D TMA bulk copy
// with its mbarrier, and block / grid reductions in a fixed order.
#pragma once

#include <cuda_runtime.h>

#include <climits>
#include <cstddef>
#include <cstdint>

namespace fw {
namespace dev {

constexpr double kNearlyZero = 1.0e-60;  // NEARLY_ZERO, lib/std/defs.h:105

__device__ __forceinline__ double2 cz() { return make_double2(0.0, 0.0); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// acc + a b and acc - a b as four fused multiply-adds into the accumulator
// (the sweeps' inner products: two FP64 instructions fewer per entry than
// a product rounded on its own and then added)
__device__ __forceinline__ double2 cmac(double2 acc, double2 a, double2 b) {
  return make_double2(fma(-a.y, b.y, fma(a.x, b.x, acc.x)), fma(a.y, b.x, fma(a.x, b.y, acc.y)));
}
__device__ __forceinline__ double2 cmsub(double2 acc, double2 a, double2 b) {
  return make_double2(fma(a.y, b.y, fma(-a.x, b.x, acc.x)), fma(-a.y, b.x, fma(-a.x, b.y, acc.y)));
}
__device__ __forceinline__ float2 cmac(float2 acc, float2 a, float2 b) {
  return make_float2(fmaf(-a.y, b.y, fmaf(a.x, b.x, acc.x)), fmaf(a.y, b.x, fmaf(a.x, b.y, acc.y)));
}
__device__ __forceinline__ float2 cmsub(float2 acc, float2 a, float2 b) {
  return make_float2(fmaf(a.y, b.y, fmaf(-a.x, b.x, acc.x)), fmaf(-a.y, b.x, fmaf(-a.x, b.y, acc.y)));
}
__device__ __forceinline__ double cabs_ref(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }  // ComplexAbs
__device__ __forceinline__ bool ciszero(double2 a) { return a.x == 0.0 && a.y == 0.0; }           // ISZERO
// ComplexReciprocal / ComplexDivide (lib/std/complex_adv.c:39-52,133-137)
__device__ __forceinline__ double2 crecip_ref(double2 a) {
  const double d = 1.0 / (a.x * a.x + a.y * a.y);
  return make_double2(a.x * d, -(a.y * d));
}
__device__ __forceinline__ double2 cdiv_ref(double2 a, double2 b) { return cmul(a, crecip_ref(b)); }

template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int o);
template <>
__device__ __forceinline__ double2 shfl_xor(double2 v, int o) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}
template <>
__device__ __forceinline__ float2 shfl_xor(float2 v, int o) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
}
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = cadd(v, shfl_xor(v, o));
  return v;
}

template <typename T>
__device__ __forceinline__ T czero();
template <>
__device__ __forceinline__ double2 czero<double2>() {
  return make_double2(0.0, 0.0);
}
template <>
__device__ __forceinline__ float2 czero<float2>() {
  return make_float2(0.0f, 0.0f);
}


template <typename T>
__device__ __forceinline__ T shfl_idx(T v, int src);
template <>
__device__ __forceinline__ double2 shfl_idx(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
template <>
__device__ __forceinline__ float2 shfl_idx(float2 v, int src) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

template <typename T>
__device__ __forceinline__ T from_d2(double2 a);
template <>
__device__ __forceinline__ double2 from_d2<double2>(double2 a) {
  return a;
}
template <>
__device__ __forceinline__ float2 from_d2<float2>(double2 a) {
  return make_float2((float)a.x, (float)a.y);
}


__host__ __device__ inline size_t a16(size_t b) { return (b + 15) & ~(size_t)15; }


__device__ __forceinline__ uint32_t smem_u32(const void *ptr) { return (uint32_t)__cvta_generic_to_shared(ptr); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// 1D bulk copy global -> shared through the TMA unit, into this CTA's own shared memory
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// the same copy with an L2 eviction policy (createpolicy) for its lines
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                              uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}
__device__ __forceinline__ uint64_t l2_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}


__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) r += sh[i];
  return r;  // valid in thread 0
}
__device__ __forceinline__ double block_max(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) r = fmax(r, sh[i]);
  return r;
}

// reduce the per-block partials of field f in a fixed order (one block)
__device__ inline double reduce_partials(const double *part, int nb, int f, bool is_max, double *sh) {
  double v = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    const double x = __ldcg(part + f * nb + i);  // written by other CTAs of this grid
    v = is_max ? fmax(v, x) : v + x;
  }
  double r = is_max ? block_max(v, sh) : block_sum(v, sh);
  __syncthreads();
  if (threadIdx.x == 0) sh[32] = r;
  __syncthreads();
  r = sh[32];
  __syncthreads();
  return r;
}


// True in the last CTA of the grid to get here, after every CTA wrote its
// partials; that CTA then reduces them in block order (deterministic) and
// resets the ticket for the next launch.
__device__ __forceinline__ bool last_cta(uint32_t *ticket) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  return last;
}

// Sum over the subdomain slots of interface DOF g, in subdomain order; a
// shard sums its own subdomains' slots only (all slots when not sharded).

// ---- row blocks of a subdomain envelope staged in shared memory ----------
// A block's stored entries are contiguous in the envelope: one bulk copy
// brings the block into a staging buffer, completing on the buffer's
// mbarrier.  Two buffers alternate; the use counts give the wait parity.
//
// Every wait is bounded.  A wait that gives up raises the error word and
// returns false; the caller then issues no further copy, waits (at the
// normal bound) for the copies already in flight and returns, so that no
// copy into its shared memory outlives it.

constexpr uint32_t kStageWaitTries = 1u << 22;
constexpr uint32_t kStallTestTries = 64;

template <typename T>
struct Stage {
  const T *L;          // the subdomain's envelope (global)
  T *buf0, *buf1;      // shared staging buffers
  uint64_t *bar;       // [3]: one per buffer, and one no copy ever arrives on (the stall test)
  const int2 *blk;     // shared: (first row, first element) of each block, then (nI, entries)
  uint32_t uses0, uses1;  // copies issued into each buffer (warp-uniform)
  int32_t *err;        // error word raised on a wait timeout
  uint64_t policy;     // L2 eviction policy of the next copies (hint != 0)
  int hint;
  int stall;           // test hook: the next wait polls bar[2], which never completes
};

template <typename T>
__device__ __forceinline__ void stage_init(Stage<T> &st, int32_t *err, int stall) {
  st.uses0 = st.uses1 = 0;
  st.err = err;
  st.policy = 0;
  st.hint = 0;
  st.stall = stall;
}

// 16-byte aligned element range of block b
template <typename T>
__device__ __forceinline__ int stage_a0(const Stage<T> &st, int b) {
  constexpr int kA = 16 / (int)sizeof(T);
  return st.blk[b].y & ~(kA - 1);
}

// lane 0 starts the copy of block b into buffer b & 1; all lanes count it
template <typename T>
__device__ __forceinline__ void stage_issue(Stage<T> &st, int b, int lane) {
  constexpr int kA = 16 / (int)sizeof(T);
  const int k = b & 1;
  if (lane == 0) {
    const int a0 = stage_a0(st, b);
    const int n = (st.blk[b + 1].y - a0 + kA - 1) & ~(kA - 1);
    fence_proxy_async();
    mbar_arrive_expect_tx(&st.bar[k], (uint32_t)(n * sizeof(T)));
    if (st.hint)
      bulk_g2s_hint(k ? st.buf1 : st.buf0, st.L + a0, (uint32_t)(n * sizeof(T)), &st.bar[k], st.policy);
    else
      bulk_g2s(k ? st.buf1 : st.buf0, st.L + a0, (uint32_t)(n * sizeof(T)), &st.bar[k]);
  }
  if (k)
    st.uses1 += 1;
  else
    st.uses0 += 1;
}

// true once the last copy into block b's buffer has landed; false (error
// word raised) when the bounded wait gave up
template <typename T>
__device__ __forceinline__ bool stage_wait(Stage<T> &st, int b) {
  const int k = b & 1;
  const uint32_t uses = k ? st.uses1 : st.uses0;
  if (uses == 0) return true;
  uint64_t *bar = &st.bar[k];
  uint32_t parity = (uses - 1u) & 1u, limit = kStageWaitTries;
  if (st.stall) {
    // test hook: a barrier that nothing arrives on, and a short bound
    st.stall = 0;
    bar = &st.bar[2];
    parity = 0;
    limit = kStallTestTries;
  }
  uint32_t tries = 0;
  while (!mbar_try_wait(bar, parity)) {
    if (++tries > limit) {
      *st.err = 1;
      return false;
    }
  }
  return true;
}

// the drain: waits at the normal bound for the last copy into each buffer
template <typename T>
__device__ __forceinline__ void stage_drain(Stage<T> &st) {
  st.stall = 0;
  stage_wait(st, 0);
  stage_wait(st, 1);
}

// lo and start (relative to the subdomain's envelope) of row r0 + lane
__device__ __forceinline__ void stage_row_meta(const int32_t *lo_g, const int64_t *ptr_g, int64_t base, int r0,
                                               int r1, int lane, int &lo, int &pr) {
  const int i = r0 + lane;
  if (i < r1) {
    lo = lo_g[i];
    pr = (int)(ptr_g[i] - base);
  } else {
    lo = INT_MAX / 2;
    pr = 0;
  }
}

}  // namespace dev
}  // namespace fw
