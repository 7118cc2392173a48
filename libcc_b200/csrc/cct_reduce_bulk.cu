// Per-tuple E[4] / v1 reduction over a blocked X, read by bulk copies.
//
// The same reduction as cct_reduce.cu (t1wt3.f90:18-109, t3squa.f:1-113,
// ddcc_aux.f:97-238 of the reference; see that file), for the emulated W build,
// which stores each GEMM output X_g in 8 x 8 x 8 blocks:
//
//   X_g(p, q, s) at (((p/8) nbk + q/8) NS + s/8) 512 + ((p%8) 8 + q%8) 8 + s%8,
//   nbk = ceil(nu / 8), NS = NP / 8,
//
// so every block an orbit needs is one contiguous 4 KB run.  A persistent CTA
// per SM walks the block triples {A <= B <= C} round-robin.  For each it fetches
// the X_g blocks of all six orbit permutations with cp.async.bulk (one
// mbarrier per buffer, up to 18 x 4 KB) and the VOE entries with 8-byte
// cp.async, double-buffered: the loads of the next block triple are in flight
// while the current one is assembled and reduced.  Phase A adds the X terms
// into W in the same order as cct_reduce_block.cuh (term 0, 1, 2[, 3]), and
// phases B and C are that file's, so the results are bitwise those of the
// row-layout reduction.
#include "cct_internal.cuh"
#include "cct_reduce_block.cuh"

namespace cct {
namespace {

using namespace red;

constexpr int kBlk = RB * RB * RB;  // doubles per block
constexpr int kNX = 3;              // X buffers staged per block triple (i>j>k; degenerate tuples use 2)
constexpr int kStageDoubles = kNX * 6 * kBlk;
constexpr int kVoeDoubles = 3 * VPAIR;
constexpr long kBulkWaitLimit = 1L << 26;
// dynamic shared memory: stage[2][kNX][6][512], W[6][512], V[2][3 VPAIR], two mbarriers
constexpr int kBulkSmem = (2 * kStageDoubles + 6 * SL + 2 * kVoeDoubles) * 8 + 2 * 8;

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *b, uint32_t parity) {
  for (long it = 0; it < kBulkWaitLimit; it++)
    if (mbar_test(b, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(su32(dst)),
      "l"(src), "r"(bytes), "r"(su32(bar))
      : "memory");
}

struct BulkArgs {
  int nu, no, nbk;
  int64_t NS;       // s blocks per (P, Q) block row: NP / 8
  int64_t ncta;     // block triples
  const int16_t *table;
  double *xpart, *vpart;
  int *err;
};

// X_g block (P, Q, S) of the blocked layout
__device__ __forceinline__ const double *xblock(const double *X, const BulkArgs &a, int P, int Q, int S) {
  return X + (((int64_t)P * a.nbk + Q) * a.NS + S) * kBlk;
}

// Issues the loads of block triple k into buffer buf: the X_g blocks of every
// distinct orbit permutation (thread 0, one mbarrier) and the VOE entries (every
// thread, one cp.async group).
template <int NXK>
__device__ __forceinline__ void issue_triple(const BulkArgs &a, const TupleDev &t, const double *__restrict__ voe,
                                             int64_t k, double *stage, double *vsm, uint64_t *bar) {
  const int S0 = a.table[3 * k], S1 = a.table[3 * k + 1], S2 = a.table[3 * k + 2];
  if (threadIdx.x == 0) {
    auto Sm = [&](int m) { return sel3(m, S0, S1, S2); };
    int slot[6];
    orbit_slots(S0, S1, S2, slot);
    int nblk = 0;
#pragma unroll
    for (int p = 0; p < 6; p++) nblk += slot[p] == p;
    mbar_expect_tx(bar, (uint32_t)(nblk * NXK * kBlk * 8));
#pragma unroll
    for (int g = 0; g < NXK; g++)
#pragma unroll
      for (int p = 0; p < 6; p++) {
        if (slot[p] != p) continue;
        bulk_load(stage + (g * 6 + p) * kBlk, xblock(t.x[g], a, Sm(pm(p, 0)), Sm(pm(p, 1)), Sm(pm(p, 2))), kBlk * 8,
                  bar);
      }
  }
  stage_voe(a.nu, a.no, t, voe, S0, S1, S2, vsm);
}

template <int KIND>
__global__ void __launch_bounds__(RT, 1) reduce_bulk_kernel(const BulkArgs a, const TupleDev t,
                                                           const double *__restrict__ eh,
                                                           const double *__restrict__ ep,
                                                           const double *__restrict__ voe) {
  constexpr int NXK = KIND == kIJK ? 3 : 2;
  constexpr int NTERM = KIND == kIJK ? 3 : 4;
  extern __shared__ __align__(128) double bsm[];
  double *stage = bsm;                      // [2][kNX][6][512]
  double *Wsm = stage + 2 * kStageDoubles;  // [6][SL]
  double *Vbuf = Wsm + 6 * SL;              // [2][3 VPAIR]
  uint64_t *bar = reinterpret_cast<uint64_t *>(Vbuf + 2 * kVoeDoubles);
  __shared__ int s_abort;
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  __syncthreads();
  int64_t k = blockIdx.x;
  if (k < a.ncta) issue_triple<NXK>(a, t, voe, k, stage, Vbuf, &bar[0]);
  uint32_t it = 0;
  bool next_issued = false;  // at an abort: the prefetch of iteration it + 1 is in flight
  for (; k < a.ncta; it++, k += gridDim.x) {
    const int buf = (int)(it & 1);
    const int64_t kn = k + gridDim.x;
    // prefetch the next triple into the other buffer (read last in iteration
    // it - 1, which ended with a barrier)
    next_issued = kn < a.ncta;
    if (next_issued) {
      issue_triple<NXK>(a, t, voe, kn, stage + (buf ^ 1) * kStageDoubles, Vbuf + (buf ^ 1) * kVoeDoubles,
                        &bar[buf ^ 1]);
      asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this triple's VOE group is done
    } else {
      cp_async_wait_all();
    }
    if (tid == 0 && !mbar_wait_bounded(&bar[buf], (it >> 1) & 1)) {
      atomicExch(a.err, 1);
      s_abort = 1;
    }
    __syncthreads();
    if (s_abort) break;
    const int S0 = a.table[3 * k], S1 = a.table[3 * k + 1], S2 = a.table[3 * k + 2];
    int slot[6];
    orbit_slots(S0, S1, S2, slot);
    const double *st = stage + buf * kStageDoubles;
    // ---- phase A: W(p) = sum over terms of X_g at the term's index placement.
    // Each thread takes elements in the staged block's own order (contiguous
    // reads) and adds them at their place in W (XOR layout).
#pragma unroll
    for (int term = 0; term < NTERM; term++) {
      const int g = term_entry(KIND, term, 0);
      const int al0 = term_entry(KIND, term, 1), al1 = term_entry(KIND, term, 2), al2 = term_entry(KIND, term, 3);
#pragma unroll
      for (int p = 0; p < 6; p++) {
        if (slot[p] != p) continue;
        // the X_g block this term reads for W block p: block coordinates
        // (O_p[al0], O_p[al1], O_p[al2]) = orbit permutation pidx(pm(p, al0), pm(p, al1))
        const int src = slot[pidx(pm(p, al0), pm(p, al1))];
        const double *xs = st + (g * 6 + src) * kBlk;
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int idx = tid + RT * e;
          const int v2 = idx & 7, v1 = (idx >> 3) & 7, v0 = idx >> 6;  // X_g local (p, q, s)
          const double x = xs[idx];
          // W coordinate m takes the X coordinate whose placement al is m
          const int c0 = al0 == 0 ? v0 : (al1 == 0 ? v1 : v2);
          const int c1 = al0 == 1 ? v0 : (al1 == 1 ? v1 : v2);
          const int c2 = al0 == 2 ? v0 : (al1 == 2 ? v1 : v2);
          double *w = Wsm + p * SL + soff(c0, c1, c2);
          if (term == 0)
            *w = x;
          else
            *w += x;
        }
      }
      __syncthreads();
    }
    if (S0 == S1 && S1 == S2 && tid < RB) Wsm[soff(tid, tid, tid)] = 0.0;  // W_aaa = 0 (ZEROT3)
    __syncthreads();
    reduce_block_bc<KIND>(a.nu, t, eh, ep, S0, S1, S2, slot, Wsm, Vbuf + buf * kVoeDoubles, a.xpart + k, a.vpart);
    __syncthreads();  // W, this buffer and phase C's shared sums are free for the next triple
  }
  // on an abort, let the bulk copies still in flight (this iteration's and the
  // prefetch of the next) land before the CTA exits
  if (tid == 0 && s_abort) {
    mbar_wait_bounded(&bar[it & 1], (it >> 1) & 1);
    if (next_issued) mbar_wait_bounded(&bar[(it + 1) & 1], ((it + 1) >> 1) & 1);
  }
  cp_async_wait_all();
}

int g_bulk_sms[64] = {0};

}  // namespace

int launch_reduce_blocked(const Dims &d, const TupleDev &t, const double *eh, const double *ep, const double *voe,
                          const int16_t *cta_table, double *xpart, double *vpart, int *err, cudaStream_t s) {
  int dev = 0;
  CCT_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("device ordinal out of range");
    return CCT_ERR_INVALID;
  }
  static int configured[64] = {0};
  if (!configured[dev]) {
    CCT_CUDA(cudaFuncSetAttribute(reduce_bulk_kernel<kIJK>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBulkSmem));
    CCT_CUDA(cudaFuncSetAttribute(reduce_bulk_kernel<kIJJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBulkSmem));
    CCT_CUDA(cudaFuncSetAttribute(reduce_bulk_kernel<kIIJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBulkSmem));
    CCT_CUDA(cudaDeviceGetAttribute(&g_bulk_sms[dev], cudaDevAttrMultiProcessorCount, dev));
    configured[dev] = 1;
  }
  if (d.NP % RB != 0) {
    set_error("blocked X needs NP a multiple of 8");
    return CCT_ERR_INVALID;
  }
  BulkArgs a;
  a.nu = d.nu;
  a.no = d.no;
  a.nbk = (d.nu + RB - 1) / RB;
  a.NS = d.NP / RB;
  a.ncta = d.ncta;
  a.table = cta_table;
  a.xpart = xpart;
  a.vpart = vpart;
  a.err = err;
  const int grid = (int)(d.ncta < g_bulk_sms[dev] ? d.ncta : g_bulk_sms[dev]);
  switch (t.kind) {
    case kIJK: reduce_bulk_kernel<kIJK><<<grid, RT, kBulkSmem, s>>>(a, t, eh, ep, voe); break;
    case kIJJ: reduce_bulk_kernel<kIJJ><<<grid, RT, kBulkSmem, s>>>(a, t, eh, ep, voe); break;
    default: reduce_bulk_kernel<kIIJ><<<grid, RT, kBulkSmem, s>>>(a, t, eh, ep, voe); break;
  }
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

}  // namespace cct
