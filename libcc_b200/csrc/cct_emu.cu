// W_abc build as split-integer emulated FP64 on the INT8 tensor pipe
// (tcgen05.mma kind::i8, int32 accumulation in tensor memory, sm_100a).
//
// Same three grouped GEMMs per tuple as cct_wbuild_f64.cu,
//   X_g(p,q,s) = sum_k E[x1][p][q][k] F[x2][x3][s][k] + sum_k E[x2][q][p][k] F[x1][x3][s][k].
// Every operand row is written as 2^e * sum_{t=1..S} a_t 2^(-7t), a_t int8 in
// [-127,127] (truncated digits).  The scale e is shared by the two halves: for
// an A row (p,q) it is the largest row exponent of E[x][p][q] and E[x][q][p]
// over all x; for a B row (z,n) the largest over y of F[y][z][n].  Then
//   X(m,n) = 2^(eA(m)+eB(n)) sum_{d=2..S+1} 2^(-7d) D_d,
//   D_d = sum_{halves} sum_{t+u=d} sum_k a_t b_u,
// keeping digit products with t+u <= S+1 (the dropped tail is below
// 2^(-7(S+1)) of |A||B| per term).  Each D_d is an exact int32 accumulation
// (|D_d| <= 2 S K 127^2 < 2^31 for K <= 4096); FP64 enters only when the
// diagonals are scaled and summed in the epilogue.  Digit count S (4..7) is a
// plan option: about 7S - 2 bits of each operand row survive.
//
// Kernel layout (one CTA per 128 x 64 tile of one job):
//   warp 0      TMA producer: per 32-byte K chunk, S digit slices of the A rows
//               (128 x 32 B) and of the B rows (64 x 32 B), SWIZZLE_32B, 4-stage ring
//   warp 1      TMEM owner + MMA issuer (one thread): S(S+1)/2 MMAs per chunk into
//               S diagonal accumulators (64 int32 columns each), both halves
//   warps 2..5  drain: tcgen05.ld each diagonal, scale, sum in FP64, write X once
// With S = 4 the accumulators fit 256 TMEM columns and two CTAs share an SM, so
// one CTA's drain overlaps the other's MMAs.  Every mbarrier wait is bounded; a
// timeout sets the error word and the CTA unwinds, freeing its tensor memory.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "cct_internal.cuh"

namespace cct {
namespace {

constexpr int EBM = 128, EBN = 64, EKC = 32;  // tile rows, tile cols, K bytes per chunk
constexpr int ESTAGES = 4;
constexpr int A_SLICE = EBM * EKC, B_SLICE = EBN * EKC;  // bytes per slice per stage
constexpr long kWaitLimit = 1L << 26;

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
// Bounded wait on a phase parity; false (and *err set) when the limit runs out.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, int *err) {
  for (long it = 0; it < kWaitLimit; it++) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  atomicExch(err, 1);
  return false;
}
__device__ __forceinline__ void tma_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          su32(dst)),
      "l"(map), "r"(su32(bar)), "r"(c0), "r"(c1)
      : "memory");
}
// K-major, SWIZZLE_32B: 8-row x 32-byte atoms, atoms 256 B apart along M.
__device__ __forceinline__ uint64_t desc_sw32(const void *p) {
  const uint64_t a = su32(p);
  return ((a & 0x3FFFF) >> 4) | (1ull << 16) | ((uint64_t)(256 >> 4) << 32) | (1ull << 46) | (6ull << 61);
}

struct EmuArgs {
  const EmuJob *jobs;
  const int16_t *expE, *expF;
  int nu, no, kchunks;
  int64_t NP, rowsE, rowsF;  // rows per slice in the E/E^T and F tensors
  int tiles_n;
  int *err;
};

constexpr int kNoRowExp = -30000;  // exponent of an all-zero row: never the maximum

__device__ __forceinline__ double pow2(int e) {
  // exact 2^e for normal exponents; ldexp covers the subnormal range
  return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52) : ldexp(1.0, e);
}

template <int S>
constexpr int emu_tmem_cols() { return S * kEmuBN <= 256 ? 256 : 512; }
template <int S>
constexpr int emu_ctas_per_sm() { return S * kEmuBN <= 256 ? 2 : 1; }

template <int S>
__global__ void __launch_bounds__(192, emu_ctas_per_sm<S>())
    wbuild_emu_kernel(const __grid_constant__ CUtensorMap mapE, const __grid_constant__ CUtensorMap mapET,
                      const __grid_constant__ CUtensorMap mapF, const EmuArgs args) {
  constexpr uint32_t TCOLS = emu_tmem_cols<S>();
  extern __shared__ __align__(1024) uint8_t emu_smem[];
  uint8_t *base = (uint8_t *)(((uintptr_t)emu_smem + 1023) & ~(uintptr_t)1023);
  uint8_t *sA = base;                                   // [stage][S][128][32]
  uint8_t *sB = base + ESTAGES * S * A_SLICE;           // [stage][S][64][32]
  __shared__ uint64_t full[ESTAGES], empty[ESTAGES], acc_full;
  __shared__ uint32_t tmem_base;

  const EmuJob job = args.jobs[blockIdx.y];
  const int tile_m = blockIdx.x / args.tiles_n, tile_n = blockIdx.x - tile_m * args.tiles_n;
  const int64_t M = (int64_t)args.nu * args.nu;
  const int64_t m0 = (int64_t)tile_m * EBM;
  const int n0 = tile_n * EBN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nh = job.nhalves;
  const int nk = args.kchunks;

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < ESTAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&acc_full, 1);
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;

  if (warp == 0) {
    if (lane == 0) {  // ---------------- TMA producer
      bool ok = true;
      for (int h = 0; h < nh && ok; h++) {
        const CUtensorMap *mA = h == 0 ? &mapE : &mapET;
        const int64_t arow = (int64_t)(h == 0 ? job.x1 : job.x2) * M + m0;
        const int64_t brow = (int64_t)job.fyz[h] * args.NP + n0;
        for (int kc = 0; kc < nk; kc++) {
          const int g = h * nk + kc, st = g % ESTAGES;
          if (g >= ESTAGES && !mbar_wait(&empty[st], ((g / ESTAGES) - 1) & 1, args.err)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&full[st], S * (A_SLICE + B_SLICE));
#pragma unroll
          for (int t = 0; t < S; t++)
            tma_2d(sA + (st * S + t) * A_SLICE, mA, &full[st], kc * EKC, (int)(t * args.rowsE + arow));
#pragma unroll
          for (int t = 0; t < S; t++)
            tma_2d(sB + (st * S + t) * B_SLICE, &mapF, &full[st], kc * EKC, (int)(t * args.rowsF + brow));
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---------------- MMA issuer: both halves into one set of diagonals
      // kind::i8, D s32, A/B s8, K-major, M = 128, N = 64
      const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(EBN >> 3) << 17) | (8u << 24);
      for (int h = 0; h < nh; h++) {
        bool ok = true;
        for (int kc = 0; kc < nk; kc++) {
          const int g = h * nk + kc, st = g % ESTAGES;
          if (!mbar_wait(&full[st], (g / ESTAGES) & 1, args.err)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
          for (int t = 0; t < S; t++) {
            const uint64_t da = desc_sw32(sA + (st * S + t) * A_SLICE);
#pragma unroll
            for (int u = 0; u < S - t; u++) {
              const uint64_t db = desc_sw32(sB + (st * S + u) * B_SLICE);
              const uint32_t dcol = tmem + (uint32_t)((t + u) * EBN);
              const uint32_t accum = (h > 0 || kc > 0 || t > 0) ? 1u : 0u;
              asm volatile(
                  "{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p; }" ::"r"(
                      dcol),
                  "l"(da), "l"(db), "r"(idesc), "r"(accum));
            }
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              su32(&empty[st])));
        }
        if (!ok) break;
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(&acc_full)));
    }
  } else {  // ---------------- drain (warps 2..5 own TMEM lane quarters 2,3,0,1)
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const int64_t m = m0 + row;
    const bool live = m < M;
    // diagonal d = t + u (0-based digits) carries 2^(-7(d+2))
    double cd[S];
#pragma unroll
    for (int d = 0; d < S; d++) cd[d] = pow2(-7 * (d + 2));
    if (mbar_wait(&acc_full, 0, args.err)) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const int eA = live ? args.expE[m] : 0;
      const int16_t *eB = args.expF + (int64_t)job.x3 * args.NP + n0;
      double *xrow = job.out + m * args.NP + n0;
#pragma unroll 1
      for (int c0 = 0; c0 < EBN; c0 += 16) {
        double acc[16];
#pragma unroll
        for (int j = 0; j < 16; j++) acc[j] = 0.0;
#pragma unroll
        for (int d = 0; d < S; d++) {
          uint32_t v[16];
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                "=r"(v[15])
              : "r"(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(d * EBN + c0)));
          asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
          for (int j = 0; j < 16; j++) acc[j] = fma((double)(int32_t)v[j], cd[d], acc[j]);
        }
        if (live) {
#pragma unroll
          for (int j = 0; j < 16; j += 2) {
            const double s0 = acc[j] * pow2(eA + eB[c0 + j]);
            const double s1 = acc[j + 1] * pow2(eA + eB[c0 + j + 1]);
            *reinterpret_cast<double2 *>(xrow + c0 + j) = make_double2(s0, s1);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
}

// ---------------------------------------------------------------------------- slicing
// Pass 1: per-row exponent (rows of length kvalid, one warp per row).
__global__ void row_exp_kernel(const double *__restrict__ src, int64_t rows, int64_t ld, int64_t kvalid,
                               int16_t *__restrict__ eout) {
  const int lane = threadIdx.x & 31;
  int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (; row < rows; row += stride) {
    const double *r = src + row * ld;
    double mx = 0.0;
    for (int64_t k = lane; k < kvalid; k += 32) mx = fmax(mx, fabs(r[k]));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    int e = kNoRowExp;
    if (mx > 0.0) frexp(mx, &e);  // mx = f 2^e, f in [0.5, 1): every |value| < 2^e
    if (lane == 0) eout[row] = (int16_t)e;
  }
}

// Pass 2a: expE[p*nu+q] = max over x of the row exponents of E[x][p][q] and E[x][q][p].
__global__ void shared_exp_e_kernel(const int16_t *__restrict__ rowexp, int no, int nu, int16_t *__restrict__ expE) {
  const int64_t nu2 = (int64_t)nu * nu;
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nu2; m += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = m / nu, q = m - p * nu, mt = q * nu + p;
    int e = kNoRowExp;
    for (int x = 0; x < no; x++) e = max(e, max((int)rowexp[x * nu2 + m], (int)rowexp[x * nu2 + mt]));
    expE[m] = (int16_t)(e == kNoRowExp ? 0 : e);
  }
}

// Pass 2b: expF[z*NP+n] = max over y of the row exponents of F[y][z][n].
__global__ void shared_exp_f_kernel(const int16_t *__restrict__ rowexp, int no, int64_t NP, int16_t *__restrict__ expF) {
  const int64_t n_all = (int64_t)no * NP;
  for (int64_t zn = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; zn < n_all; zn += (int64_t)gridDim.x * blockDim.x) {
    const int64_t z = zn / NP, n = zn - z * NP;
    int e = kNoRowExp;
    for (int y = 0; y < no; y++) e = max(e, (int)rowexp[((int64_t)y * no + z) * NP + n]);
    expF[zn] = (int16_t)(e == kNoRowExp ? 0 : e);
  }
}

// Pass 3: S truncated 7-bit digits of value * 2^-e, |value * 2^-e| < 1.
__device__ __forceinline__ void digits_row(const double *__restrict__ src, int64_t kvalid, int e, int S, int64_t KP8,
                                           int8_t *dst, int64_t slice_stride, int8_t *dstT) {
  const int lane = threadIdx.x & 31;
  for (int64_t k = lane; k < KP8; k += 32) {
    double y = k < kvalid ? ldexp(src[k], -e) : 0.0;
    for (int t = 0; t < S; t++) {
      y *= 128.0;
      const double a = trunc(y);  // |a| <= 127
      y -= a;                     // exact
      dst[t * slice_stride + k] = (int8_t)a;
      if (dstT) dstT[t * slice_stride + k] = (int8_t)a;
    }
  }
}

__global__ void digits_e_kernel(const double *__restrict__ E, int no, int nu, int64_t KP, int64_t KP8, int S,
                                const int16_t *__restrict__ expE, int8_t *__restrict__ E8, int8_t *__restrict__ E8T) {
  const int64_t nu2 = (int64_t)nu * nu, rows = (int64_t)no * nu2;
  int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (; row < rows; row += stride) {
    const int64_t x = row / nu2, rem = row - x * nu2;
    const int64_t r1 = rem / nu, r2 = rem - r1 * nu;
    const int64_t rowT = x * nu2 + r2 * nu + r1;
    digits_row(E + row * KP, nu + no, expE[rem], S, KP8, E8 + row * KP8, rows * KP8, E8T + rowT * KP8);
  }
}

__global__ void digits_f_kernel(const double *__restrict__ F, int no, int nu, int64_t NP, int64_t KP, int64_t KP8,
                                int S, const int16_t *__restrict__ expF, int8_t *__restrict__ F8) {
  const int64_t rows = (int64_t)no * no * NP;
  int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (; row < rows; row += stride) {
    const int64_t z = (row / NP) % no, n = row % NP;
    digits_row(F + row * KP, nu + no, expF[z * NP + n], S, KP8, F8 + row * KP8, rows * KP8, nullptr);
  }
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_encode_mutex;

int get_encode() {
  std::lock_guard<std::mutex> lock(g_encode_mutex);
  if (g_encode) return CCT_OK;
  cudaDriverEntryPointQueryResult qr;
  void *fn = nullptr;
  CCT_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr));
  if (!fn || qr != cudaDriverEntryPointSuccess) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return CCT_ERR_UNSUPPORTED;
  }
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return CCT_OK;
}

int make_map(CUtensorMap *m, const int8_t *base, int64_t rows, int64_t row_bytes, int box_rows) {
  cuuint64_t dims[2] = {(cuuint64_t)row_bytes, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
  cuuint32_t box[2] = {(cuuint32_t)EKC, (cuuint32_t)box_rows};
  cuuint32_t es[2] = {1, 1};
  const CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void *)base, dims, strides, box, es,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
    return CCT_ERR_CUDA;
  }
  return CCT_OK;
}

template <int S>
int launch_emu_s(const EmuOperands &o, const Dims &d, const EmuJob *jobs_dev, int njobs, int *err, cudaStream_t s) {
  constexpr int smem = ESTAGES * S * (A_SLICE + B_SLICE) + 1024;
  static int configured_device = -1;
  int dev = 0;
  CCT_CUDA(cudaGetDevice(&dev));
  if (configured_device != dev) {
    CCT_CUDA(cudaFuncSetAttribute(wbuild_emu_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    // full shared-memory carveout, so reduction CTAs can sit beside a W-build CTA
    CCT_CUDA(cudaFuncSetAttribute(wbuild_emu_kernel<S>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared));
    configured_device = dev;
  }
  EmuArgs a;
  a.jobs = jobs_dev;
  a.expE = o.expE;
  a.expF = o.expF;
  a.nu = d.nu;
  a.no = d.no;
  a.kchunks = (int)(o.KP8 / EKC);
  a.NP = d.NP;
  a.rowsE = (int64_t)d.no * d.nu * d.nu;
  a.rowsF = (int64_t)d.no * d.no * d.NP;
  a.tiles_n = (int)(d.NP / EBN);
  a.err = err;
  const int64_t M = (int64_t)d.nu * d.nu;
  dim3 grid((unsigned)(((M + EBM - 1) / EBM) * a.tiles_n), (unsigned)njobs);
  wbuild_emu_kernel<S><<<grid, 192, smem, s>>>(o.mapE, o.mapET, o.mapF, a);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

}  // namespace

int emu_build_operands(const Dims &d, const double *E, const double *F, EmuOperands *o, cudaStream_t s) {
  if (o->slices < kEmuMinSlices || o->slices > kEmuMaxSlices) {
    set_error("emulation slice count must be in [" + std::to_string(kEmuMinSlices) + ", " +
              std::to_string(kEmuMaxSlices) + "]");
    return CCT_ERR_INVALID;
  }
  if (d.NP % EBN != 0) {
    set_error("emulated plan needs NP to be a multiple of 64");
    return CCT_ERR_INVALID;
  }
  CCT_TRY(get_encode());
  const int64_t rowsE = (int64_t)d.no * d.nu * d.nu, rowsF = (int64_t)d.no * d.no * d.NP;
  auto grid_rows = [](int64_t rows) {
    int64_t b = (rows * 32 + 255) / 256;
    return (int)(b > 148 * 64 ? 148 * 64 : (b < 1 ? 1 : b));
  };
  auto grid_flat = [](int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
  };
  // per-row exponents (expET and expRowF serve as the row tables), shared scales, digits
  row_exp_kernel<<<grid_rows(rowsE), 256, 0, s>>>(E, rowsE, d.KP, d.nu + d.no, o->expET);
  CCT_CUDA(cudaGetLastError());
  row_exp_kernel<<<grid_rows(rowsF), 256, 0, s>>>(F, rowsF, d.KP, d.nu + d.no, o->expRowF);
  CCT_CUDA(cudaGetLastError());
  shared_exp_e_kernel<<<grid_flat((int64_t)d.nu * d.nu), 256, 0, s>>>(o->expET, d.no, d.nu, o->expE);
  CCT_CUDA(cudaGetLastError());
  shared_exp_f_kernel<<<grid_flat((int64_t)d.no * d.NP), 256, 0, s>>>(o->expRowF, d.no, d.NP, o->expF);
  CCT_CUDA(cudaGetLastError());
  digits_e_kernel<<<grid_rows(rowsE), 256, 0, s>>>(E, d.no, d.nu, d.KP, o->KP8, o->slices, o->expE, o->E8, o->E8T);
  CCT_CUDA(cudaGetLastError());
  digits_f_kernel<<<grid_rows(rowsF), 256, 0, s>>>(F, d.no, d.nu, d.NP, d.KP, o->KP8, o->slices, o->expF, o->F8);
  CCT_CUDA(cudaGetLastError());
  CCT_TRY(make_map(&o->mapE, o->E8, (int64_t)o->slices * rowsE, o->KP8, EBM));
  CCT_TRY(make_map(&o->mapET, o->E8T, (int64_t)o->slices * rowsE, o->KP8, EBM));
  CCT_TRY(make_map(&o->mapF, o->F8, (int64_t)o->slices * rowsF, o->KP8, EBN));
  return CCT_OK;
}

int launch_wbuild_emu(const EmuOperands &o, const Dims &d, const EmuJob *jobs_dev, int njobs, int *err,
                      cudaStream_t s) {
  switch (o.slices) {
    case 4: return launch_emu_s<4>(o, d, jobs_dev, njobs, err, s);
    case 5: return launch_emu_s<5>(o, d, jobs_dev, njobs, err, s);
    case 6: return launch_emu_s<6>(o, d, jobs_dev, njobs, err, s);
    case 7: return launch_emu_s<7>(o, d, jobs_dev, njobs, err, s);
    default:
      set_error("unsupported slice count " + std::to_string(o.slices));
      return CCT_ERR_INVALID;
  }
}

}  // namespace cct
