// probe_kernels.cu -- integer-ALU throughput probes: the denominators of the
// distance kernel's roofline.  The distance kernel is bound by 32-bit LOP3
// issue (one acc & ~(a ^ b) per 32 bins per bit plane per pair) with POPC on a
// separate pipe, so its roofline peak is this device's measured LOP3 rate,
// taken in the same process as the timing it is compared with.
#include <cuda_runtime.h>

#include <cstdint>

#include "sk_device.cuh"
#include "sk_runtime.h"

namespace sk {
namespace {

constexpr int kChains = 16;

__global__ void __launch_bounds__(256) lop3_peak_kernel(uint32_t *sink, int iters, uint32_t seed) {
  uint32_t acc[kChains];
  const uint32_t x = seed ^ (threadIdx.x * 0x9E3779B9u) ^ blockIdx.x;
#pragma unroll
  for (int u = 0; u < kChains; ++u) acc[u] = x * (u + 1) + 0x3C6EF372u * u;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < kChains; ++u) {
      asm volatile("lop3.b32 %0, %1, %2, %0, 0x82;" : "+r"(acc[u]) : "r"(x), "r"(acc[(u + 1) % kChains]));
    }
  }
  uint32_t r = 0;
#pragma unroll
  for (int u = 0; u < kChains; ++u) r ^= acc[u];
  if (r == 0x12345678u) sink[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

__global__ void __launch_bounds__(256) popc_peak_kernel(uint32_t *sink, int iters, uint32_t seed) {
  uint32_t v[kChains];
  const uint32_t x = seed ^ (threadIdx.x * 0x9E3779B9u) ^ blockIdx.x;
#pragma unroll
  for (int u = 0; u < kChains; ++u) v[u] = x * (u + 3);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < kChains; ++u) asm volatile("popc.b32 %0, %0;" : "+r"(v[u]));
  }
  uint32_t r = 0;
#pragma unroll
  for (int u = 0; u < kChains; ++u) r += v[u];
  if (r == 0x12345678u) sink[blockIdx.x * blockDim.x + threadIdx.x] = r;
}

template <typename Kern>
sk_status time_probe(sk_ctx *ctx, Kern kern, int iters, double *ops_per_s) {
  const int block = 256;
  const int grid = ctx->sm_count * 8;
  void *sink = nullptr;
  sk_status st = scratch(ctx, kSlotTemp, static_cast<size_t>(grid) * block * 4, &sink);
  if (st != SK_OK) return st;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  kern<<<grid, block, 0, ctx->stream>>>(static_cast<uint32_t *>(sink), iters / 8, 1u);  // warm-up
  cudaEventRecord(e0, ctx->stream);
  kern<<<grid, block, 0, ctx->stream>>>(static_cast<uint32_t *>(sink), iters, 7u);
  cudaEventRecord(e1, ctx->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "ALU probe");
  *ops_per_s = static_cast<double>(grid) * block * iters * kChains / (ms * 1e-3);
  return SK_OK;
}

}  // namespace
}  // namespace sk

extern "C" sk_status sk_probe_alu_peak(sk_ctx *ctx, double *lop3_per_s, double *popc_per_s) {
  if (!ctx) return SK_EINVAL;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  sk::DeviceGuard g(ctx->device);
  double l = 0.0, p = 0.0;
  sk_status st = sk::time_probe(ctx, sk::lop3_peak_kernel, 1 << 16, &l);
  if (st == SK_OK) st = sk::time_probe(ctx, sk::popc_peak_kernel, 1 << 14, &p);
  if (st != SK_OK) return st;
  if (lop3_per_s) *lop3_per_s = l;
  if (popc_per_s) *popc_per_s = p;
  return SK_OK;
}

namespace sk {
namespace {

// Waits on an mbarrier that nothing arrives on, with the same bounded wait the
// distance kernel uses for its stages: the wait gives up after limit_ns and
// the kernel records a timeout in the status word instead of spinning on.
__global__ void wait_limit_kernel(uint64_t limit_ns, DevStatus *status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  const bool landed = mbar_wait_bounded(&bar, 0, limit_ns);   // phase 0 never completes
  if (!landed && threadIdx.x == 0) {
    atomicOr(&status->error, 1u);
    status->where = 2;
  }
}

}  // namespace
}  // namespace sk

extern "C" sk_status sk_probe_wait_limit(sk_ctx *ctx, int32_t limit_ms) {
  if (!ctx) return SK_EINVAL;
  std::lock_guard<std::recursive_mutex> lock(ctx->mu);
  sk::DeviceGuard g(ctx->device);
  if (limit_ms < 1 || limit_ms > 10000) return sk::fail(ctx, SK_EINVAL, "limit_ms outside [1, 10000]");
  sk_status st = sk::begin_call(ctx);
  if (st != SK_OK) return st;
  sk::wait_limit_kernel<<<1, 32, 0, ctx->stream>>>(static_cast<uint64_t>(limit_ms) * 1000000ull,
                                                   ctx->status_dev);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return sk::cuda_fail(ctx, e, "wait probe launch");
  return sk::finish_call(ctx);
}
