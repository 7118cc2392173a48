// FP64 tensor-pipe throughput probe: the denominator of the FP64 roofline.
// Each warp keeps eight independent m16n8k16 accumulators busy; the grid
// covers every SM several times.  Returns TFLOP/s (best of three launches).
#include "cct_internal.cuh"

namespace cct {
namespace {

__device__ __forceinline__ void dmma_16x8x16(double *d, const double *a, const double *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
      "{%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]), "d"(b[0]),
        "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

__global__ void peak_kernel(double *out, int iters) {
  double acc[8][4];
  double a[8], b[4];
  for (int i = 0; i < 8; i++) a[i] = 1e-3 * (threadIdx.x + i);
  for (int i = 0; i < 4; i++) b[i] = 1e-3 * ((int)threadIdx.x - i);
  for (int s = 0; s < 8; s++)
    for (int r = 0; r < 4; r++) acc[s][r] = 0.0;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int s = 0; s < 8; s++) dmma_16x8x16(acc[s], a, b);
  }
  double s = 0.0;
  for (int i = 0; i < 8; i++)
    for (int r = 0; r < 4; r++) s += acc[i][r];
  if (s == 1234.5678) out[0] = s;  // keeps the loop alive
}

// INT8 tensor-pipe probe: one thread per CTA issues back-to-back
// tcgen05.mma kind::i8 (M=128, N=256, K=32) on operands already in shared
// memory, into one TMEM accumulator; the wait for completion is bounded.
__global__ void __launch_bounds__(128, 1) int8_peak_kernel(int iters, int *err) {
  __shared__ __align__(1024) uint8_t ops[128 * 32 + 256 * 32];
  __shared__ uint64_t done;
  __shared__ uint32_t tbase;
  const int warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < (int)sizeof(ops); i += blockDim.x) ops[i] = (uint8_t)(i * 7);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(&tbase)),
                 "r"(256));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 32) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"((uint32_t)__cvta_generic_to_shared(&done)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("fence.proxy.async.shared::cta;");
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tbase;
  if (threadIdx.x == 32) {
    auto desc = [](const void *p) {
      const uint64_t a = (uint32_t)__cvta_generic_to_shared(p);
      return ((a & 0x3FFFF) >> 4) | (1ull << 16) | ((uint64_t)(256 >> 4) << 32) | (1ull << 46) | (6ull << 61);
    };
    const uint64_t da = desc(ops), db = desc(ops + 128 * 32);
    const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(256 >> 3) << 17) | (8u << 24);
    for (int it = 0; it < iters; it++) {
      const uint32_t acc = it > 0 ? 1u : 0u;
      asm volatile(
          "{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p; }" ::"r"(tmem),
          "l"(da), "l"(db), "r"(idesc), "r"(acc));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        (uint32_t)__cvta_generic_to_shared(&done)));
    bool ok = false;
    for (long w = 0; w < (1L << 26) && !ok; w++) {
      uint32_t r;
      asm volatile(
          "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
          : "=r"(r)
          : "r"((uint32_t)__cvta_generic_to_shared(&done))
          : "memory");
      ok = r != 0;
    }
    if (!ok) atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256));
}

}  // namespace

double measure_int8_peak(int device) {
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return 0.0;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  int *err = nullptr;
  cudaEvent_t e0, e1;
  double best = 0.0;
  if (cudaMalloc(&err, 4) == cudaSuccess && cudaMemset(err, 0, 4) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
      cudaEventCreate(&e1) == cudaSuccess) {
    const int iters = 2048, blocks = nsm * 2;
    for (int rep = 0; rep < 4; rep++) {
      cudaEventRecord(e0);
      int8_peak_kernel<<<blocks, 128>>>(iters, err);
      cudaEventRecord(e1);
      if (cudaEventSynchronize(e1) != cudaSuccess) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      const double ops = 2.0 * 128 * 256 * 32 * (double)iters * blocks;
      if (rep > 0 && ms > 0) best = std::max(best, ops / (ms * 1e-3) / 1e12);
    }
    int herr = 0;
    cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost);
    if (herr) best = 0.0;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (err) cudaFree(err);
  cudaSetDevice(prev);
  return best;
}

double measure_fp64_peak(int device) {
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return 0.0;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  double *out = nullptr;
  cudaEvent_t e0, e1;
  double best = 0.0;
  if (cudaMalloc(&out, 8) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) {
    const int iters = 2000, blocks = nsm * 2, threads = 256;
    for (int rep = 0; rep < 4; rep++) {
      cudaEventRecord(e0);
      peak_kernel<<<blocks, threads>>>(out, iters);
      cudaEventRecord(e1);
      if (cudaEventSynchronize(e1) != cudaSuccess) break;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      const double flops = 2.0 * 16 * 8 * 16 * 8.0 * iters * (double)blocks * (threads / 32);
      if (rep > 0 && ms > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  if (out) cudaFree(out);
  cudaSetDevice(prev);
  return best;
}

}  // namespace cct
