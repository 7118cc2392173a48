// W_abc build as split-integer emulated FP64 on the INT8 tensor pipe
// (tcgen05.mma kind::i8, int32 accumulation in tensor memory, sm_100a).
//
// Same three grouped GEMMs per tuple as cct_wbuild_f64.cu,
//   X_g(p,q,s) = sum_k E[x1][p][q][k] F[x2][x3][s][k] + sum_k E[x2][q][p][k] F[x1][x3][s][k].
// Every operand row is written as 2^(e+1) * sum_{t=1..S} a_t 2^(-7t) with
// round-to-nearest digits a_t in [-64, 64]: |v 2^-(e+1)| < 1/2, each digit is
// rint(128 y) of the running remainder y, which stays in [-1/2, 1/2].  The
// scale e is shared by the two halves: for an A row (p,q) it is the largest
// row exponent of E[x][p][q] and E[x][q][p] over all x; for a B row (z,n) the
// largest over y of F[y][z][n].  Then
//   X(m,n) = 2^(eA(m)+eB(n)+2) sum_{d=2..S+1} 2^(-7d) D_d,
//   D_d = sum_{halves} sum_{t+u=d} sum_k a_t b_u,
// keeping digit products with t+u <= S+1 (the dropped tail is below
// 2^(-7(S+1)) of |A||B| per term).  Each D_d is an exact int32 accumulation
// (|D_d| <= 2 S K 64^2 < 2^31 for K <= 4096).  The epilogue combines the
// diagonals exactly in int64 (up to five of them) and enters FP64 with one
// conversion and one power-of-two scaling per element; the sixth and
// seventh diagonals of 6- and 7-digit launches are added in FP64.  Rounded digits leave an
// unbiased remainder: truncated digits (remainder of the value's own sign)
// shrink every product the same way, and that bias adds up over the K sum,
// the a,b,c sum and the tuples into the energy.  On seeded systems the
// rounded digits give E(T) errors 300-700x smaller at the same digit count.
// Digit count S (3..7) is a plan option, or picked per system from an energy
// error target (cct_plan.cu).  An adaptive plan takes S as the maximum and
// gives each work item (row tile, column tile) its own count s <= S from the
// tile's exponents (EmuOperands::tileExp): a tile whose largest row scales sum
// `gap` bits below the plan's top runs s = S - floor(gap / 7) digits,
// s(s+1)/2 digit products per K chunk instead of S(S+1)/2, and its dropped
// products stay below the top tile's.
//
// Operands are pre-tiled (EmuOperands): the digits of one 32-byte K chunk of
// a 128-row A tile, all slices of the operand, are one contiguous run already
// in the tensor core's K-major no-swizzle layout, and likewise for an N-row B
// tile.  A pipeline stage is therefore two bulk copies (cp.async.bulk) of
// large contiguous runs instead of 2S narrow tensor boxes.  The operand may
// hold more slices than a launch runs (an automatic plan builds 7 and runs
// the count its error target needs); the producer then copies the leading
// slices of each chunk.
//
// Merged digit products.  B's slices of one chunk sit back to back in shared
// memory (slice u at u N rows, 8-row core-matrix groups 256 B apart), so the
// slices u0..u0+c-1 form one B operand of c N rows, and the accumulator
// columns of diagonal d sit at d N.  One MMA of A slice t against that operand
// therefore adds A_t B_u into diagonal t+u for all c slices at once: a chunk
// needs, per t, ceil((S-t) N / 256) MMAs of up to 256 columns instead of S-t
// MMAs of N columns (7 instead of 15 at S = 5, N = 80).  An N = 80 MMA is
// bound by its shared-memory operand reads (A 4 KB + B 2.5 KB); a wide one
// reads A once for up to three B slices.
//
// Persistent kernel, one CTA of 64 + 32 NDW threads per SM (NDW = 16 drain
// warps at 80 registers a thread: the drain is latency-bound, and 16 warps
// took a 3-digit tuple from 0.54 to 0.46 ms against 8 warps at 128
// registers), work items (job,
// row tile, column tile) taken round-robin with the column tile fastest, so
// the CTAs in flight share A tiles through L2:
//   warp 0      producer: per stage, one bulk copy of the A digits and one
//               of the B digits (KS K chunks) into a ring of stages; it runs
//               ahead across work items, so the ring never drains between tiles
//   warp 1      TMEM owner + MMA issuer (one thread): per chunk and A slice t,
//               merged MMAs over the B slices 0..s-1-t into the s diagonal
//               accumulators (N int32 columns each)
//   warps 2..   drain (NDW warps): tcgen05.ld one diagonal at a time, sum in
//               int64, hand the tensor memory back to the issuer, then convert,
//               scale and store X in 32-byte stores.  When two accumulator sets fit
//               the tensor memory (2 S N <= 512) the issuer alternates between
//               them, so the next item's MMAs run while the drain reads and
//               stores the last one; with one set they wait for the read.
// Every mbarrier wait is bounded and also ends when another role aborted; a
// timeout sets the error word, the producer waits for its copies in flight,
// the issuer for its MMAs, and the CTA frees its tensor memory and returns.
#include <algorithm>
#include <type_traits>

#include "cct_internal.cuh"

namespace cct {
namespace {

constexpr int EBM = kEmuBM;
constexpr int A_BLK = kEmuABlk;
// A stage holds KS consecutive K chunks (all S digit slices of each), so one
// barrier round trip feeds KS S(S+1)/2 MMAs.  Ring depth: as many stages as
// the shared-memory budget holds, between 2 and 8.
#ifndef CCT_EMU_KS
#define CCT_EMU_KS 2
#endif
#ifndef CCT_EMU_DRAIN_WARPS
#define CCT_EMU_DRAIN_WARPS 16
#endif
#ifndef CCT_EMU_MAXNREG
#define CCT_EMU_MAXNREG 80
#endif
// Ring budget: 200 KB gives a 3-digit, 80-column tile five stages (2% faster
// than four) and 5 digits three (5% faster than two); the reduction CTA that
// used to fit beside the W build no longer does, which costs nothing (the two
// kernels did not overlap usefully).
#ifndef CCT_EMU_SMEM_BUDGET
#define CCT_EMU_SMEM_BUDGET (200 * 1024)
#endif
constexpr int KS = CCT_EMU_KS;
constexpr int NDW = CCT_EMU_DRAIN_WARPS;  // drain warps: NDW/4 per TMEM lane quarter
constexpr int EMU_THREADS = 64 + 32 * NDW;
template <int S, int EBN>
constexpr int emu_stages() {
  return CCT_EMU_SMEM_BUDGET / (KS * S * (A_BLK + EBN * kEmuKC)) > 8   ? 8
         : CCT_EMU_SMEM_BUDGET / (KS * S * (A_BLK + EBN * kEmuKC)) < 2 ? 2
                                                                        : CCT_EMU_SMEM_BUDGET / (KS * S * (A_BLK + EBN * kEmuKC));
}
// Accumulator sets in tensor memory: two when both fit the 512 columns (3
// digits at N = 80, 4 at N = 64), so the MMAs of the next work item go into
// one set while the drain reads the other; else one.
template <int S, int EBN>
constexpr int emu_acc_bufs() { return 2 * S * EBN <= 512 ? 2 : 1; }
template <int S, int EBN>
constexpr uint32_t emu_tmem_cols() { return emu_acc_bufs<S, EBN>() * S * EBN <= 256 ? 256u : 512u; }
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
__device__ __forceinline__ bool mbar_test(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on a phase parity.  Returns false when another role of the CTA
// aborted, or when the limit runs out (then the error word and the abort flag
// are set).
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, int *err, volatile int *abort_flag) {
  for (long it = 0; it < kWaitLimit; it++) {
    if (mbar_test(b, parity)) return true;
    if ((it & 63) == 63 && *abort_flag) return false;
  }
  atomicExch(err, 1);
  *abort_flag = 1;
  return false;
}
// Bounded wait that ignores the abort flag (used to let work in flight land).
__device__ __forceinline__ void mbar_settle(uint64_t *b, uint32_t parity, int *err) {
  for (long it = 0; it < kWaitLimit; it++)
    if (mbar_test(b, parity)) return;
  atomicExch(err, 1);
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(su32(dst)),
      "l"(src), "r"(bytes), "r"(su32(bar))
      : "memory");
}
// K-major, no swizzle: 8-row x 16-byte core matrices; the two K halves of a
// 32-byte chunk 128 B apart (leading offset), 8-row groups 256 B apart (stride
// offset).  Start address and offsets are in 16-byte units.
__device__ __forceinline__ uint64_t desc_kmajor(const void *p) {
  const uint64_t a = su32(p);
  return ((a & 0x3FFFF) >> 4) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(256 >> 4) << 32) | (1ull << 46);
}

// 32-byte store (one whole sector per thread)
__device__ __forceinline__ void st_global_v4(double *p, double a, double b, double c, double d) {
  asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(a), "d"(b), "d"(c), "d"(d) : "memory");
}

// tcgen05.ld of 16 / 8 consecutive 32-bit columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t *v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(addr));
}
__device__ __forceinline__ void tmem_ld4(uint32_t addr, uint32_t *v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
               : "r"(addr));
}
__device__ __forceinline__ void tmem_ld8(uint32_t addr, uint32_t *v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(addr));
}

struct EmuArgs {
  const EmuJob *jobs;
  const int8_t *E8, *E8T, *F8;
  const int16_t *expE, *expF;
  const int *tileExp;  // adaptive plans: see EmuOperands::tileExp; nullptr: every item runs S digits
  unsigned long long *slice_hist;
  int nu, no, njobs, kchunks, tiles_m, tiles_n;
  int sop;  // digit slices stored per K chunk in the operands (>= the S of the launch)
  int64_t NP;   // X row stride; columns at or past it (a partial last N tile) are not stored
  int64_t NPe;  // rows per (y,z) of the B digits and expF: tiles_n * EBN
  int xblocked; // X in 8 x 8 x 8 blocks (xblock_base), else rows of NP
  int *err;
};

constexpr int kNoRowExp = -30000;  // exponent of an all-zero row: never the maximum

// Digits of work item (row tile tm, column tile tn of job z = x3).
template <int S>
__device__ __forceinline__ int item_slices(const EmuArgs &a, int tm, int tn, int z) {
  if (!a.tileExp) return S;
  const int ea = a.tileExp[tm], eb = a.tileExp[a.tiles_m + z * a.tiles_n + tn];
  const int top = a.tileExp[a.tiles_m + a.no * a.tiles_n] + a.tileExp[a.tiles_m + a.no * a.tiles_n + 1];
  if (ea <= kNoRowExp || eb <= kNoRowExp) return 1;  // all-zero rows or columns: X is zero
  const int s = S - (top - (ea + eb)) / 7;
  return s < 1 ? 1 : (s > S ? S : s);
}

__device__ __forceinline__ double pow2(int e) {
  // exact 2^e for normal exponents; ldexp covers the subnormal range
  return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52) : ldexp(1.0, e);
}

template <int S, int EBN>
__global__ void __maxnreg__(CCT_EMU_MAXNREG) wbuild_emu_kernel(const EmuArgs args) {
  static_assert(S * EBN <= 512 && EBN % 16 == 0, "S diagonals of EBN columns must fit the tensor memory");
  constexpr int B_BLK = EBN * kEmuKC;
  constexpr uint32_t TCOLS = emu_tmem_cols<S, EBN>();
  constexpr int NB = emu_acc_bufs<S, EBN>();  // accumulator sets, S * EBN columns each
  constexpr int ST = emu_stages<S, EBN>();
  constexpr int CA = S * A_BLK, CB = S * B_BLK;    // bytes of one K chunk per operand in shared memory
  constexpr int SA = KS * CA, SB = KS * CB;        // bytes of one stage per operand
  constexpr int MPS = 256 / EBN;                   // B slices per merged MMA (N <= 256)
  static_assert(MPS >= 1, "N tile above 256 columns");
  extern __shared__ __align__(1024) uint8_t emu_smem[];
  uint8_t *base = (uint8_t *)(((uintptr_t)emu_smem + 1023) & ~(uintptr_t)1023);
  uint8_t *sA = base;            // [stage][chunk][slice][4096]
  uint8_t *sB = base + ST * SA;  // [stage][chunk][slice][2048]
  __shared__ uint64_t full[ST], empty[ST], acc_full[NB], tmem_empty[NB], mma_done;
  __shared__ uint32_t tmem_base;
  __shared__ int abort_word;
  volatile int *abort_flag = &abort_word;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t M = (int64_t)args.nu * args.nu;
  const int per_job = args.tiles_m * args.tiles_n;
  const int64_t nitems = (int64_t)args.njobs * per_job;
  const int KC = args.kchunks;
  const int64_t GA = (int64_t)args.sop * A_BLK, GB = (int64_t)args.sop * B_BLK;  // bytes of one K chunk in HBM
  const int64_t aslab = (int64_t)args.tiles_m * KC * GA;  // bytes per occupied index
  const int64_t bslab = (int64_t)args.tiles_n * KC * GB;  // bytes per (y,z)
  const bool whole = args.sop == S;  // operand chunks hold exactly the launch's slices

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&tmem_base)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < NB; b++) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&tmem_empty[b], NDW);  // one arrival per drain warp
    }
    mbar_init(&mma_done, 1);
    abort_word = 0;
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;

  if (warp == 0) {
    if (lane == 0) {  // ---------------- producer
      uint32_t g = 0;
      bool ok = true;
      for (int64_t it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
        const int jb = (int)(it / per_job);
        const int rem = (int)(it - (int64_t)jb * per_job);
        const int tm = rem / args.tiles_n, tn = rem - tm * args.tiles_n;
        const EmuJob job = args.jobs[jb];
        const int sl = item_slices<S>(args, tm, tn, job.x3);
        for (int h = 0; h < job.nhalves && ok; h++) {
          const int8_t *A = (h == 0 ? args.E8 + job.x1 * aslab : args.E8T + job.x2 * aslab) + (int64_t)tm * KC * GA;
          const int8_t *B = args.F8 + job.fyz[h] * bslab + (int64_t)tn * KC * GB;
          for (int kc = 0; kc < KC; kc += KS, g++) {
            const int st = (int)(g % ST);
            const uint32_t nch = KC - kc < KS ? (uint32_t)(KC - kc) : (uint32_t)KS;  // the last stage may be short
            if (g >= (uint32_t)ST && !mbar_wait(&empty[st], ((g / ST) - 1) & 1, args.err, abort_flag)) {
              ok = false;
              break;
            }
            if (sl == S && whole) {  // all digits: the stage's chunks are one contiguous run per operand
              mbar_expect_tx(&full[st], nch * (CA + CB));
              bulk_load(sA + st * SA, A + (int64_t)kc * GA, nch * CA, &full[st]);
              bulk_load(sB + st * SB, B + (int64_t)kc * GB, nch * CB, &full[st]);
            } else {  // the leading sl digit slices of each chunk
              mbar_expect_tx(&full[st], nch * (uint32_t)sl * (A_BLK + B_BLK));
              for (uint32_t c = 0; c < nch; c++) {
                bulk_load(sA + st * SA + c * CA, A + (int64_t)(kc + c) * GA, (uint32_t)sl * A_BLK, &full[st]);
                bulk_load(sB + st * SB + c * CB, B + (int64_t)(kc + c) * GB, (uint32_t)sl * B_BLK, &full[st]);
              }
            }
          }
        }
      }
      // let every copy still in flight land before the CTA can exit
      for (uint32_t q = g > (uint32_t)ST ? g - ST : 0; q < g; q++) mbar_settle(&full[q % ST], (q / ST) & 1, args.err);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---------------- MMA issuer
      // kind::i8, D s32, A/B s8, K-major, M = 128; N (bits 17-22, N >> 3) per MMA
      const uint32_t idesc0 = (2u << 4) | (1u << 7) | (1u << 10) | (8u << 24);
      const uint64_t dA0 = desc_kmajor(sA), dB0 = desc_kmajor(sB);
      uint32_t g = 0, n = 0;
      bool ok = true;
      // halves and digit count of an item (global loads: the issuer fetches
      // them one item ahead, so they are not between two items' MMAs)
      auto item_info = [&](int64_t item, int *nhalves, int *slices) {
        const int jb = (int)(item / per_job);
        const int rem = (int)(item - (int64_t)jb * per_job);
        const int tm = rem / args.tiles_n, tn = rem - tm * args.tiles_n;
        const EmuJob &job = args.jobs[jb];
        *nhalves = job.nhalves;
        *slices = item_slices<S>(args, tm, tn, job.x3);
      };
      int nh_next = 0, sl_next = 0;
      if (blockIdx.x < nitems) item_info(blockIdx.x, &nh_next, &sl_next);
      for (int64_t it = blockIdx.x; it < nitems && ok; it += gridDim.x, n++) {
        // item n uses accumulator set ab; the drain of the item that used it
        // last (use - 1 uses ago) has read it
        const int ab = NB == 2 ? (int)(n & 1) : 0;
        const uint32_t use = NB == 2 ? (n >> 1) : n;
        const uint32_t acc = tmem + (uint32_t)(ab * S * EBN);
        if (use > 0 && !mbar_wait(&tmem_empty[ab], (use - 1) & 1, args.err, abort_flag)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const int nh = nh_next, sl = sl_next;
        // the next item's job and digit count, loaded while this item's MMAs issue
        if (it + gridDim.x < nitems) item_info(it + gridDim.x, &nh_next, &sl_next);
        if (args.slice_hist) atomicAdd(args.slice_hist + sl, 1ull);
        for (int h = 0; h < nh && ok; h++) {
          for (int kc = 0; kc < KC; kc += KS, g++) {
            const int st = (int)(g % ST);
            const int nch = KC - kc < KS ? KC - kc : KS;
            if (!mbar_wait(&full[st], (g / ST) & 1, args.err, abort_flag)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int c = 0; c < KS; c++) {
              if (c >= nch) break;
              // descriptor start addresses are linear in 16-byte units
              const uint64_t dA = dA0 + (uint64_t)((st * SA + c * CA) >> 4);
              const uint64_t dB = dB0 + (uint64_t)((st * SB + c * CB) >> 4);
              const uint32_t first = (h == 0 && kc == 0 && c == 0) ? 0u : 1u;  // accumulate flag of the t = 0 row
              // A slice t against B slices u0 .. u0+cnt-1 (one operand of cnt
              // EBN rows) into diagonals t+u0 .. t+u0+cnt-1
              auto mma = [&](int t, int u0, int cnt) {
                const uint32_t idesc = idesc0 | ((uint32_t)((cnt * EBN) >> 3) << 17);
                asm volatile(
                    "{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p; "
                    "}" ::"r"(acc + (uint32_t)((t + u0) * EBN)),
                    "l"(dA + (uint64_t)(t * (A_BLK >> 4))), "l"(dB + (uint64_t)(u0 * (B_BLK >> 4))), "r"(idesc),
                    "r"(t > 0 ? 1u : first));
              };
              // t = 0 first: with the accumulate flag clear it initialises
              // every diagonal of the item; later rows add into them.  Each
              // digit count has a schedule fixed at compile time:
              // straight-line MMAs with constant shapes and offsets, so the
              // single issuing thread spends no time on the partition
              // arithmetic between MMAs.  A slice t meets n = s - t B slices,
              // taken as MMAs of at most MPS slices whose sizes differ by one.
              auto schedule = [&](auto slc) {
                constexpr int SLC = decltype(slc)::value;
#pragma unroll
                for (int t = 0; t < SLC; t++) {
                  const int n = SLC - t;
                  const int parts = (n + MPS - 1) / MPS;
                  const int base = n / parts, extra = n - base * parts;
#pragma unroll
                  for (int q = 0; q < parts; q++) mma(t, q * base + (q < extra ? q : extra), base + (q < extra ? 1 : 0));
                }
              };
              if constexpr (EBN <= 80) {
                switch (sl) {
                  case 1: schedule(std::integral_constant<int, 1>{}); break;
                  case 2: if constexpr (S >= 2) schedule(std::integral_constant<int, 2>{}); break;
                  case 3: if constexpr (S >= 3) schedule(std::integral_constant<int, 3>{}); break;
                  case 4: if constexpr (S >= 4) schedule(std::integral_constant<int, 4>{}); break;
                  case 5: if constexpr (S >= 5) schedule(std::integral_constant<int, 5>{}); break;
                  case 6: if constexpr (S >= 6) schedule(std::integral_constant<int, 6>{}); break;
                  default: if constexpr (S >= 7) schedule(std::integral_constant<int, 7>{}); break;
                }
              } else if (sl == S) {  // the 96-column tile: one fixed schedule (more would spill)
                schedule(std::integral_constant<int, S>{});
              } else {
#pragma unroll
                for (int t = 0; t < S; t++) {
                  if (t >= sl) break;
                  const int n = sl - t;
                  const int parts = (n + MPS - 1) / MPS;
                  const int base = n / parts, extra = n - base * parts;
                  int u0 = 0;
                  for (int q = 0; q < parts; q++) {
                    const int cnt = base + (q < extra ? 1 : 0);
                    mma(t, u0, cnt);
                    u0 += cnt;
                  }
                }
              }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                su32(&empty[st])));
          }
        }
        if (!ok) break;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            su32(&acc_full[ab])));
      }
      // every MMA issued has completed before the tensor memory is freed
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(&mma_done)));
      mbar_settle(&mma_done, 0, args.err);
    }
  } else {  // ---------------- drain: warp w owns TMEM lane quarter w % 4
    constexpr int CW = EBN / (NDW / 4);  // columns per drain warp
    static_assert(CW % 4 == 0, "the drain stores X four columns at a time");
    const int q = warp & 3;
    const int row = q * 32 + lane;
    const int cbase = ((warp - 2) / 4) * CW;
    // diagonal d = t + u (0-based digits) carries 2^(-7(d+2)), times 2^2 for
    // the two operand scales 2^(e+1)
    double cd[S];
#pragma unroll
    for (int d = 0; d < S; d++) cd[d] = pow2(2 - 7 * (d + 2));
    uint32_t n = 0;
    for (int64_t it = blockIdx.x; it < nitems; it += gridDim.x, n++) {
      // everything that does not depend on the MMAs is fetched before the wait
      const int jb = (int)(it / per_job);
      const int rem = (int)(it - (int64_t)jb * per_job);
      const int tm = rem / args.tiles_n, tn = rem - tm * args.tiles_n;
      const EmuJob job = args.jobs[jb];
      const int64_t m = (int64_t)tm * EBM + row;
      const bool live = m < M;
      const int eA = live ? args.expE[m] : 0;
      const int n0 = tn * EBN + cbase;
      const int sl = item_slices<S>(args, tm, tn, job.x3);
      const int ab = NB == 2 ? (int)(n & 1) : 0;
      const uint32_t use = NB == 2 ? (n >> 1) : n;
      // warp-uniform decision: the tcgen05.ld below are .sync.aligned
      if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[ab], use & 1, args.err, abort_flag))) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
      // Up to five digits the diagonals are summed exactly in int64 by
      // Horner's rule, acc = sum_d D_d 2^(7(sl-1-d)) (|D_d| < 2^31: below
      // 2^60), and converted once; 6- and 7-digit launches, and the 96-column
      // tile (whose int64 sums would spill at 80 registers), sum in FP64.
      // acc holds the int64 sum, or the FP64 bits of the FP64 sum.
      constexpr int H = S <= 5 && EBN <= 80 ? S : 0;
      auto cvt = [](long long x) {
        if constexpr (S <= 3) {  // |x| < 2^46: exact through the 2^52 + 2^51 bias
          return __longlong_as_double(x + 0x4338000000000000LL) - 6755399441055744.0;
        } else {
          return __ll2double_rn(x);
        }
      };
      long long acc[CW];
#pragma unroll
      for (int c0 = 0; c0 < CW; c0 += 16) {
        const int w = CW - c0 >= 16 ? 16 : (CW - c0 >= 8 ? 8 : 4);  // chunk widths 16, then 8 or 4
#pragma unroll
        for (int d0 = 0; d0 < S; d0++) {
          if (d0 >= sl) break;  // diagonals past the item's digit count were not written
          uint32_t v[16];
          const uint32_t addr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)((ab * S + d0) * EBN + cbase + c0);
          if (w == 16)
            tmem_ld16(addr, v);
          else if (w == 8)
            tmem_ld8(addr, v);
          else
            tmem_ld4(addr, v);
          asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
          for (int j = 0; j < 16; j++) {
            if (j >= w) continue;
            const long long dv = (long long)(int32_t)v[j];
            if constexpr (H > 0) {
              acc[c0 + j] = d0 == 0 ? dv : (acc[c0 + j] << 7) + dv;
            } else {
              const double a = d0 == 0 ? 0.0 : __longlong_as_double(acc[c0 + j]);
              acc[c0 + j] = __double_as_longlong(fma((double)dv, cd[d0], a));
            }
          }
        }
      }
      // every diagonal is in registers: hand the tensor memory to the next item
      // before the scaling and the stores
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(&tmem_empty[ab]);
      if (live) {
        const int16_t *eB = args.expF + (int64_t)job.x3 * args.NPe + n0;
        const int e0 = eA + (H > 0 ? 2 - 7 * (sl + 1) : 0);
        auto val = [&](int j) { return (H > 0 ? cvt(acc[j]) : __longlong_as_double(acc[j])) * pow2(e0 + eB[j]); };
        // one 32-byte sector per store (a thread owns a row, so 16-byte
        // stores wrote half a sector each and doubled the write traffic)
        if (args.xblocked) {  // a quad of columns (s % 4 == 0) stays inside one block
          const int64_t pp = m / args.nu, qq = m - pp * args.nu;
          double *xb = job.out + xblock_base(pp >> 3, qq >> 3, 0, args.nu, args.NP) + ((pp & 7) * 8 + (qq & 7)) * 8;
#pragma unroll
          for (int j = 0; j < CW; j += 4) {
            const int64_t sc = n0 + j;
            if (sc >= args.NP) break;
            st_global_v4(xb + (sc >> 3) * 512 + (sc & 7), val(j), val(j + 1), val(j + 2), val(j + 3));
          }
        } else {
          double *xrow = job.out + m * args.NP + n0;
#pragma unroll
          for (int j = 0; j < CW; j += 4) {
            if (n0 + j >= args.NP) break;  // NP is a multiple of 4: a quad is stored whole or not at all
            st_global_v4(xrow + j, val(j), val(j + 1), val(j + 2), val(j + 3));
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
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

// Pass 2b: expF[z*NPe+n] = max over y of the row exponents of F[y][z][n]
// (rows n >= NP, the padding of a partial last N tile, are zero).
__global__ void shared_exp_f_kernel(const int16_t *__restrict__ rowexp, int no, int64_t NP, int64_t NPe,
                                    int16_t *__restrict__ expF) {
  const int64_t n_all = (int64_t)no * NPe;
  for (int64_t zn = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; zn < n_all; zn += (int64_t)gridDim.x * blockDim.x) {
    const int64_t z = zn / NPe, n = zn - z * NPe;
    int e = kNoRowExp;
    if (n < NP)
      for (int y = 0; y < no; y++) e = max(e, (int)rowexp[((int64_t)y * no + z) * NP + n]);
    expF[zn] = (int16_t)(e == kNoRowExp ? 0 : e);
  }
}

// Pass 2c (adaptive plans): the largest nonzero row exponent of every A row
// tile (over x and both halves' row orders) and of every B column tile of each
// z (over y): one block per tile.  tile_exp_top_kernel then appends the two
// maxima.
__global__ void tile_exp_kernel(const int16_t *__restrict__ rowexpE, const int16_t *__restrict__ rowexpF, int no,
                                int nu, int64_t NP, int ebn, int tiles_m, int tiles_n, int *__restrict__ tileExp) {
  const int64_t nu2 = (int64_t)nu * nu;
  const int tile = blockIdx.x;
  int e = kNoRowExp;
  if (tile < tiles_m) {
    for (int r = threadIdx.x; r < kEmuBM; r += blockDim.x) {
      const int64_t m = (int64_t)tile * kEmuBM + r;
      if (m >= nu2) break;
      const int64_t p = m / nu, q = m - p * nu, mt = q * nu + p;
      for (int x = 0; x < no; x++) e = max(e, max((int)rowexpE[x * nu2 + m], (int)rowexpE[x * nu2 + mt]));
    }
  } else {
    const int zt = tile - tiles_m, z = zt / tiles_n, tn = zt - z * tiles_n;
    for (int r = threadIdx.x; r < ebn; r += blockDim.x) {
      const int64_t n = (int64_t)tn * ebn + r;
      if (n >= NP) break;
      for (int y = 0; y < no; y++) e = max(e, (int)rowexpF[((int64_t)y * no + z) * NP + n]);
    }
  }
  __shared__ int red[256];
  red[threadIdx.x] = e;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] = max(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) tileExp[tile] = red[0];
}
__global__ void tile_exp_top_kernel(int tiles_m, int nbt, int *__restrict__ tileExp) {
  __shared__ int red[2][256];
  int ea = kNoRowExp, eb = kNoRowExp;
  for (int t = threadIdx.x; t < tiles_m; t += blockDim.x) ea = max(ea, tileExp[t]);
  for (int t = threadIdx.x; t < nbt; t += blockDim.x) eb = max(eb, tileExp[tiles_m + t]);
  red[0][threadIdx.x] = ea;
  red[1][threadIdx.x] = eb;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      red[0][threadIdx.x] = max(red[0][threadIdx.x], red[0][threadIdx.x + w]);
      red[1][threadIdx.x] = max(red[1][threadIdx.x], red[1][threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    tileExp[tiles_m + nbt] = red[0][0];
    tileExp[tiles_m + nbt + 1] = red[1][0];
  }
}

// Byte offset of (row r, K byte kb) inside one tiled block: 8-row x 16-byte
// core matrices, K halves 128 B apart, 8-row groups 256 B apart.
__host__ __device__ constexpr int blk_off(int r, int kb) { return (r >> 3) * 256 + (kb >> 4) * 128 + (r & 7) * 16 + (kb & 15); }

// Pass 3: S rounded 7-bit digits of y = value * 2^-(e+1), |y| < 1/2: each
// digit is rint(128 y) of the running remainder (|digit| <= 64, the remainder
// stays in [-1/2, 1/2]; every step is exact).  A lane takes four consecutive
// K bytes, so each slice gets one 32-bit store; the four bytes are adjacent in
// the tiled layout (kb % 4 == 0).
__device__ __forceinline__ void digits4(const double *__restrict__ src, int64_t k, int64_t kvalid, int e, int S,
                                        uint32_t *w) {
  double y[4];
#pragma unroll
  for (int i = 0; i < 4; i++) y[i] = (k + i) < kvalid ? ldexp(src[k + i], -(e + 1)) : 0.0;
  for (int t = 0; t < S; t++) {
    uint32_t word = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      y[i] *= 128.0;
      const double a = rint(y[i]);  // |a| <= 64
      y[i] -= a;                    // exact, in [-1/2, 1/2]
      word |= (uint32_t)(uint8_t)(int8_t)a << (8 * i);
    }
    w[t] = word;
  }
}

// E digits: row (x, m = r1*nu + r2) goes to E8 at row m and to E8T at row
// r2*nu + r1 of the same occupied index x.
__global__ void digits_e_kernel(const double *__restrict__ E, int no, int nu, int64_t KP, int64_t KP8, int S,
                                int64_t tiles_m, const int16_t *__restrict__ expE, int8_t *__restrict__ E8,
                                int8_t *__restrict__ E8T) {
  const int64_t nu2 = (int64_t)nu * nu, rows = (int64_t)no * nu2;
  const int64_t KC = KP8 / kEmuKC;
  const int lane = threadIdx.x & 31;
  int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (; row < rows; row += stride) {
    const int64_t x = row / nu2, m = row - x * nu2;
    const int64_t r1 = m / nu, r2 = m - r1 * nu;
    const int64_t mt = r2 * nu + r1;
    const int e = expE[m];
    for (int64_t k = 4 * lane; k < KP8; k += 128) {
      uint32_t w[kEmuDigitCap];
      digits4(E + row * KP, k, nu + no, e, S, w);
      const int64_t kc = k / kEmuKC;
      const int kb = (int)(k - kc * kEmuKC);
      const int64_t ba = ((x * tiles_m + m / kEmuBM) * KC + kc) * S * kEmuABlk + blk_off((int)(m % kEmuBM), kb);
      const int64_t bt = ((x * tiles_m + mt / kEmuBM) * KC + kc) * S * kEmuABlk + blk_off((int)(mt % kEmuBM), kb);
      for (int t = 0; t < S; t++) {
        *reinterpret_cast<uint32_t *>(E8 + ba + (int64_t)t * kEmuABlk) = w[t];
        *reinterpret_cast<uint32_t *>(E8T + bt + (int64_t)t * kEmuABlk) = w[t];
      }
    }
  }
}

__global__ void digits_f_kernel(const double *__restrict__ F, int no, int nu, int64_t NP, int64_t NPe, int64_t KP,
                                int64_t KP8, int S, int ebn, const int16_t *__restrict__ expF,
                                int8_t *__restrict__ F8) {
  const int64_t rows = (int64_t)no * no * NP;
  const int64_t KC = KP8 / kEmuKC, tiles_n = NPe / ebn;
  const int64_t bblk = (int64_t)ebn * kEmuKC;
  const int lane = threadIdx.x & 31;
  int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (; row < rows; row += stride) {
    const int64_t yz = row / NP, n = row - yz * NP;
    const int64_t z = yz % no;
    const int e = expF[z * NPe + n];
    for (int64_t k = 4 * lane; k < KP8; k += 128) {
      uint32_t w[kEmuDigitCap];
      digits4(F + row * KP, k, nu + no, e, S, w);
      const int64_t kc = k / kEmuKC;
      const int kb = (int)(k - kc * kEmuKC);
      const int64_t b = ((yz * tiles_n + n / ebn) * KC + kc) * S * bblk + blk_off((int)(n % ebn), kb);
      for (int t = 0; t < S; t++) *reinterpret_cast<uint32_t *>(F8 + b + (int64_t)t * bblk) = w[t];
    }
  }
}

int g_num_sms[64] = {0};

template <int S, int EBN>
int launch_emu_s(const EmuOperands &o, const Dims &d, const EmuJob *jobs_dev, int njobs, int *err, cudaStream_t s,
                 bool blocked) {
  constexpr int smem = emu_stages<S, EBN>() * KS * S * (A_BLK + EBN * kEmuKC) + 1024;
  static int configured_device = -1;
  int dev = 0;
  CCT_CUDA(cudaGetDevice(&dev));
  if (configured_device != dev) {
    CCT_CUDA(cudaFuncSetAttribute(wbuild_emu_kernel<S, EBN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CCT_CUDA(cudaFuncSetAttribute(wbuild_emu_kernel<S, EBN>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared));
    configured_device = dev;
  }
  if (dev < 0 || dev >= 64) {
    set_error("device ordinal out of range");
    return CCT_ERR_INVALID;
  }
  if (g_num_sms[dev] == 0) CCT_CUDA(cudaDeviceGetAttribute(&g_num_sms[dev], cudaDevAttrMultiProcessorCount, dev));
  EmuArgs a;
  a.jobs = jobs_dev;
  a.E8 = o.E8;
  a.E8T = o.E8T;
  a.F8 = o.F8;
  a.expE = o.expE;
  a.expF = o.expF;
  a.tileExp = o.adaptive && !o.tiles_uniform ? o.tileExp : nullptr;
  a.slice_hist = o.slice_hist;
  a.nu = d.nu;
  a.no = d.no;
  a.njobs = njobs;
  a.kchunks = (int)(o.KP8 / kEmuKC);
  a.sop = o.slices;
  a.tiles_m = (int)o.tiles_m;
  a.tiles_n = (int)(o.NPe / EBN);
  if (o.ebn != EBN || o.NPe % EBN != 0 || o.NPe < d.NP || o.slices < S || d.NP % 4 != 0) {
    set_error("emulated N tile mismatch, fewer operand digits than the launch runs, or an X row stride that "
              "is not a multiple of 4 doubles");
    return CCT_ERR_INVALID;
  }
  a.NP = d.NP;
  a.NPe = o.NPe;
  a.xblocked = blocked ? 1 : 0;
  if (blocked && d.NP % 8 != 0) {
    set_error("blocked X needs NP a multiple of 8");
    return CCT_ERR_INVALID;
  }
  a.err = err;
  const int64_t items = (int64_t)njobs * a.tiles_m * a.tiles_n;
  const int grid = (int)(items < g_num_sms[dev] ? items : g_num_sms[dev]);
  wbuild_emu_kernel<S, EBN><<<grid, EMU_THREADS, smem, s>>>(a);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

}  // namespace

int emu_build_operands(const Dims &d, const double *E, const double *F, EmuOperands *o, cudaStream_t s) {
  if (o->slices < kEmuMinSlices || o->slices > kEmuDigitCap) {
    set_error("emulation slice count must be in [" + std::to_string(kEmuMinSlices) + ", " +
              std::to_string(kEmuDigitCap) + "]");
    return CCT_ERR_INVALID;
  }
  if (o->ebn <= 0 || o->NPe % o->ebn != 0 || o->NPe < d.NP || o->KP8 % kEmuKC != 0 || o->slices * o->ebn > 512) {
    set_error("emulated operands need NPe >= NP a multiple of their N tile, KP8 a multiple of 32 and "
              "slices x N <= 512");
    return CCT_ERR_INVALID;
  }
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
  shared_exp_f_kernel<<<grid_flat((int64_t)d.no * o->NPe), 256, 0, s>>>(o->expRowF, d.no, d.NP, o->NPe, o->expF);
  CCT_CUDA(cudaGetLastError());
  // the rows past nu^2 in the last row tile stay zero
  const size_t bytesE = (size_t)o->slices * d.no * o->tiles_m * kEmuBM * o->KP8;
  CCT_CUDA(cudaMemsetAsync(o->E8, 0, bytesE, s));
  CCT_CUDA(cudaMemsetAsync(o->E8T, 0, bytesE, s));
  digits_e_kernel<<<grid_rows(rowsE), 256, 0, s>>>(E, d.no, d.nu, d.KP, o->KP8, o->slices, o->tiles_m, o->expE,
                                                   o->E8, o->E8T);
  CCT_CUDA(cudaGetLastError());
  if (o->NPe > d.NP)  // the padding rows of a partial last N tile stay zero
    CCT_CUDA(cudaMemsetAsync(o->F8, 0, (size_t)o->slices * d.no * d.no * o->NPe * o->KP8, s));
  digits_f_kernel<<<grid_rows(rowsF), 256, 0, s>>>(F, d.no, d.nu, d.NP, o->NPe, d.KP, o->KP8, o->slices, o->ebn,
                                                   o->expF, o->F8);
  CCT_CUDA(cudaGetLastError());
  if (o->adaptive) {
    const int tiles_n = (int)(o->NPe / o->ebn), nbt = d.no * tiles_n;
    tile_exp_kernel<<<(int)o->tiles_m + nbt, 256, 0, s>>>(o->expET, o->expRowF, d.no, d.nu, d.NP, o->ebn,
                                                          (int)o->tiles_m, tiles_n, o->tileExp);
    CCT_CUDA(cudaGetLastError());
    tile_exp_top_kernel<<<1, 256, 0, s>>>((int)o->tiles_m, nbt, o->tileExp);
    CCT_CUDA(cudaGetLastError());
    // item_slices runs S - floor(gap / 7) digits, gap = top - (ea + eb) >= 0:
    // all S everywhere iff no tile is all zero and the smallest pair is within 7
    std::vector<int> te((size_t)o->tiles_m + nbt + 2);
    CCT_CUDA(cudaMemcpyAsync(te.data(), o->tileExp, te.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    CCT_CUDA(cudaStreamSynchronize(s));
    const int top = te[o->tiles_m + nbt] + te[o->tiles_m + nbt + 1];
    const int minA = *std::min_element(te.begin(), te.begin() + o->tiles_m);
    const int minB = *std::min_element(te.begin() + o->tiles_m, te.begin() + o->tiles_m + nbt);
    o->tiles_uniform = minA > kNoRowExp && minB > kNoRowExp && top - (minA + minB) < 7;
  }
  return CCT_OK;
}

int launch_wbuild_emu(const EmuOperands &o, const Dims &d, const EmuJob *jobs_dev, int njobs, int *err,
                      cudaStream_t s, bool blocked) {
  // (digits run, N tile) pairs with digits x N <= 512 tensor-memory columns
  const int key = o.run_slices * 1000 + o.ebn;
  switch (key) {
    case 3064: return launch_emu_s<3, 64>(o, d, jobs_dev, njobs, err, s, blocked);
    case 3080: return launch_emu_s<3, 80>(o, d, jobs_dev, njobs, err, s, blocked);
    case 3096: return launch_emu_s<3, 96>(o, d, jobs_dev, njobs, err, s, blocked);
    case 4064: return launch_emu_s<4, 64>(o, d, jobs_dev, njobs, err, s, blocked);
    case 4080: return launch_emu_s<4, 80>(o, d, jobs_dev, njobs, err, s, blocked);
    case 4096: return launch_emu_s<4, 96>(o, d, jobs_dev, njobs, err, s, blocked);
    case 5064: return launch_emu_s<5, 64>(o, d, jobs_dev, njobs, err, s, blocked);
    case 5080: return launch_emu_s<5, 80>(o, d, jobs_dev, njobs, err, s, blocked);
    case 5096: return launch_emu_s<5, 96>(o, d, jobs_dev, njobs, err, s, blocked);
    case 6064: return launch_emu_s<6, 64>(o, d, jobs_dev, njobs, err, s, blocked);
    case 6080: return launch_emu_s<6, 80>(o, d, jobs_dev, njobs, err, s, blocked);
    case 7064: return launch_emu_s<7, 64>(o, d, jobs_dev, njobs, err, s, blocked);
    default:
      set_error("unsupported (digits, N tile) = (" + std::to_string(o.run_slices) + ", " + std::to_string(o.ebn) +
                ")");
      return CCT_ERR_INVALID;
  }
}

}  // namespace cct
