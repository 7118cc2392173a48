// Batched (T) for many independent systems of uneven size in one persistent
// kernel fed by a device-side work queue.
//
// The reference runs one system per triples.x process; a batch of small
// systems there is a loop of processes (or here, of per-system plans, each
// launching three W-build GEMM jobs and a reduction per tuple).  Small systems
// leave most of a B200 idle per launch.  Here every tuple of every system is
// cut into work items -- one 256 x BN tile of one W-build GEMM job, or one
// block triple of the tuple's reduction -- and a persistent kernel (one CTA
// per SM) takes items from a queue with one atomicAdd each:
//
//   queue order:  WB(g0) WB(g1) RD(g0) WB(g2) RD(g1) ... WB(gL) RD(gL-1) RD(gL)
//
// where WB(g)/RD(g) are the W-build tiles / reduction blocks of tuple group g
// (tuples sorted by cost, largest first, packed into groups by scratch size).
// Dependencies are counters in global memory:
//   * a reduction block of tuple t waits until every W-build tile of t is done;
//   * the last reduction block of t finalizes t (fixed-order sums of its
//     partials), and the last finalized tuple of a system sums the system
//     (Neumaier etd in tuple order, v1, ets) -- the same arithmetic, in the
//     same order, as a single-system plan, so results are bitwise equal;
//   * the X scratch of group g lives in ring slot g % R (R = 6), so a W-build
//     tile of group g waits until every reduction block of group g-R is done
//     (the reduction partials live outside the ring, one slab per tuple).
// Every wait is on items dispensed earlier, which run on live CTAs and whose
// own waits point further back, so the queue cannot deadlock; each wait is
// also bounded (on timeout the error word is set and the item proceeds).
// Data produced inside the kernel is read through L2 (ld.global.cg /
// cp.async.cg), never through the incoherent L1.
//
// A second executor (mode 1) runs the same items as grouped launches: per
// tuple group, one launch of 128-row W-build tiles (three CTAs per SM) on one
// stream, then one launch of its reduction blocks (two CTAs per SM, the last
// block of a tuple finalizing it) on a second stream, the ring slots guarded
// by stream events instead of counters.  Either forward (counter reset plus the
// launches) is captured once in a CUDA graph and replayed.  The executor, the
// W-build N tile (BN) and the tuple order are chosen by ccT_batch_tune, which
// times every candidate on the loaded batch.
//
// A third executor (mode 2, batches created with CCT_PREC_INT8_EMU) is the
// grouped one with the split-integer W build (cct_emu.cu): each system gets an
// emulated single-system plan whose set_inputs calibrates the system's digit
// count to the batch's error target and builds its digit operands; per tuple
// group, one persistent emulated W-build launch per system covers all of that
// system's tuples in the group, and the reduction launches are mode 1's.  Per
// system the energies equal the emulated plan's own forward bitwise.  The
// tuner of an emulated batch times all three executors (each meets the
// target); an FP64 batch never runs the emulated one.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "cct_internal.cuh"
#include "cct_reduce_block.cuh"
#include "cct_wbuild_tile.cuh"

namespace cct {
namespace {

constexpr int kBT = 256;   // threads per batch CTA (8 warps)
constexpr int kBTM = 256;  // W-build tile rows: one 32-row slab per warp
constexpr int kRing = 6;   // X scratch groups in flight
constexpr long kSpinLimit = 1L << 24;
// Batch-wide W-build N tiles; 0 = per system, the least-padding tile of
// kBNChoices (grouped executor only: one W-build launch per tile width).
constexpr int kBatchBN[] = {0, 32, 48, 64};

struct SysDev {
  int no, nu, nb, tiles_m, tiles_n;
  int64_t KP, NP, ncta;
  const double *eh, *ep, *t1, *voe;
  const int16_t *cta_table;
  int64_t tuple_begin, ntuples;  // the system's tuples, consecutive, in reference order
  double *v1;                    // (nu, no) result
};

struct TupleRec {
  int sys, kind, i, j, k, group;
  int wb_items, rd_items;
  double *x[3];
  double *xpart, *vpart;
};

struct BatchArgs {
  const int4 *items;  // {kind 0 = W-build tile / 1 = reduction block, tuple, job slot | block, tile}
  int64_t nitems;
  int *counters;      // [0] queue head, then wb_done[T], rd_done[T], group_rd[G], sys_done[S]
  int ntuple, ngroup;
  const int *group_rd_items;  // reduction blocks per group
  const TupleRec *tuples;
  const GemmJob *jobs;  // [tuple][3]
  const SysDev *sys;
  double *tuple_etd, *tuple_v1;  // per tuple: weight x3, and 3 nu v1 contributions
  const int64_t *tuple_v1_off;
  double *sys_out;               // [sys][3] = ets, etd, ets+etd
  int *err;
  long spin_limit;               // iterations of a bounded counter wait
};

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// Bounded wait for *p >= target.  Once any wait has timed out (*err set) every
// later wait returns at once, so a failure cannot cascade into a long stall.
__device__ void spin_until(const int *p, int target, int *err, long limit) {
  for (long it = 0; it < limit; it++) {
    if (ld_acquire(p) >= target) return;
    if (*(volatile int *)err) return;
    __nanosleep(64);
  }
  atomicExch(err, 1);
}

// Sums of one tuple's reduction partials, in the order of finalize_kernel.
__device__ void finalize_tuple(const TupleRec &T, const SysDev &S, int t, const BatchArgs &A, double *red) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double weight = T.kind == kIJK ? 1.0 : 0.5;
  double s = 0.0;
  for (int64_t c = tid; c < S.ncta; c += kBT) s += __ldcg(T.xpart + c);
  red[tid] = s;
  __syncthreads();
  for (int st = kBT / 2; st > 0; st >>= 1) {
    if (tid < st) red[tid] += red[tid + st];
    __syncthreads();
  }
  if (tid == 0) A.tuple_etd[t] = weight * red[0];
  const int64_t npairs = (int64_t)S.nb * (S.nb + 1) / 2;
  double *tv = A.tuple_v1 + A.tuple_v1_off[t];
  for (int a = warp; a < S.nu; a += kBT / 32) {
    const int X = a / red::RB, la = a - X * red::RB;
    const double *slab = T.vpart + ((int64_t)X * red::RB + la) * 3 * npairs;
#pragma unroll
    for (int col = 0; col < 3; col++) {
      double v = 0.0;
      for (int64_t q = lane; q < npairs; q += 32) v += __ldcg(slab + col * npairs + q);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0) tv[col * S.nu + a] = weight * v;
    }
  }
}

// One system's etd (Neumaier over its tuples in order), v1 and ets -- the
// arithmetic of finalize_kernel and ets_kernel, in the same order.
__device__ void system_sum(const SysDev &S, int s, const BatchArgs &A, double *red) {
  const int tid = threadIdx.x;
  const int nu = S.nu, no = S.no;
  if (tid == 0) {
    double sum = 0.0, comp = 0.0;
    for (int64_t t = S.tuple_begin; t < S.tuple_begin + S.ntuples; t++) {
      const double v = __ldcg(A.tuple_etd + t);
      const double nsum = sum + v;
      comp += fabs(sum) >= fabs(v) ? (sum - nsum) + v : (v - nsum) + sum;
      sum = nsum;
    }
    red[kBT] = sum + comp;
  }
  // thread per v1 element (a, x): the contributions of the system's tuples in
  // order, each tuple's columns i, j, k in that order (as finalize_kernel adds them)
  for (int64_t e = tid; e < (int64_t)nu * no; e += kBT) {
    const int x = (int)(e / nu), a = (int)(e - (int64_t)x * nu);
    double v = 0.0;
    for (int64_t t = S.tuple_begin; t < S.tuple_begin + S.ntuples; t++) {
      const TupleRec &T = A.tuples[t];
      const double *tv = A.tuple_v1 + A.tuple_v1_off[t];
      if (T.i == x) v += __ldcg(tv + a);
      if (T.j == x) v += __ldcg(tv + nu + a);
      if (T.k == x) v += __ldcg(tv + 2 * nu + a);
    }
    S.v1[e] = v;
  }
  __syncthreads();
  double sacc = 0.0;
  const int64_t n = (int64_t)no * nu;
  for (int64_t e = tid; e < n; e += kBT) {
    const int64_t i = e / nu, a = e - (e / nu) * nu;
    sacc += S.t1[i + (int64_t)no * a] * S.v1[a + (int64_t)nu * i];
  }
  red[tid] = sacc;
  __syncthreads();
  for (int st = kBT / 2; st > 0; st >>= 1) {
    if (tid < st) red[tid] += red[tid + st];
    __syncthreads();
  }
  if (tid == 0) {
    const double ets = 2.0 * red[0], etd = red[kBT];
    A.sys_out[3 * s] = ets;
    A.sys_out[3 * s + 1] = etd;
    A.sys_out[3 * s + 2] = ets + etd;
  }
}

template <int BN>
constexpr int batch_smem() {
  return wb::smem_bytes<BN, kBTM>() > red::REDUCE_SMEM ? wb::smem_bytes<BN, kBTM>() : red::REDUCE_SMEM;
}

template <int BN>
__global__ void __launch_bounds__(kBT, 1) batch_kernel(const BatchArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[kBT + 1];
  __shared__ int64_t s_item;
  __shared__ int s_flag;
  int *const wb_done = A.counters + 1;
  int *const rd_done = wb_done + A.ntuple;
  int *const group_rd = rd_done + A.ntuple;
  int *const sys_done = group_rd + A.ngroup;
  for (;;) {
    __syncthreads();  // the previous item is done with shared memory and s_item
    if (threadIdx.x == 0) s_item = atomicAdd(A.counters, 1);
    __syncthreads();
    const int64_t q = s_item;
    if (q >= A.nitems) break;
    const int4 it = A.items[q];
    const int t = it.y;
    const TupleRec &T = A.tuples[t];
    const SysDev &S = A.sys[T.sys];
    if (it.x == 0) {  // ---- one W-build tile
      if (threadIdx.x == 0 && T.group >= kRing)
        spin_until(group_rd + (T.group - kRing), A.group_rd_items[T.group - kRing], A.err, A.spin_limit);
      __syncthreads();
      const int tile_m = it.w / S.tiles_n, tile_n = it.w - tile_m * S.tiles_n;
      wb::wbuild_tile<BN, kBTM>(A.jobs[(int64_t)t * 3 + it.z], S.nu, S.KP, S.nu + S.no, S.NP, tile_m, tile_n, smem);
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) atomicAdd(wb_done + t, 1);
    } else {  // ---- one reduction block
      if (threadIdx.x == 0) spin_until(wb_done + t, T.wb_items, A.err, A.spin_limit);
      __syncthreads();
      __threadfence();
      TupleDev td;
      td.x[0] = T.x[0];
      td.x[1] = T.x[1];
      td.x[2] = T.x[2];
      td.kind = T.kind;
      td.i = T.i;
      td.j = T.j;
      td.k = T.k;
      td.weight = T.kind == kIJK ? 1.0 : 0.5;
      const int c = it.z;
      const int S0 = S.cta_table[3 * c], S1 = S.cta_table[3 * c + 1], S2 = S.cta_table[3 * c + 2];
      double *dsm = reinterpret_cast<double *>(smem);
      if (T.kind == kIJK)
        red::reduce_block<kIJK, true>(S.nu, S.no, S.NP, td, S.eh, S.ep, S.voe, S0, S1, S2, T.xpart + c, T.vpart, dsm);
      else if (T.kind == kIJJ)
        red::reduce_block<kIJJ, true>(S.nu, S.no, S.NP, td, S.eh, S.ep, S.voe, S0, S1, S2, T.xpart + c, T.vpart, dsm);
      else
        red::reduce_block<kIIJ, true>(S.nu, S.no, S.NP, td, S.eh, S.ep, S.voe, S0, S1, S2, T.xpart + c, T.vpart, dsm);
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) {
        atomicAdd(group_rd + T.group, 1);  // this block no longer reads the group's X scratch
        s_flag = atomicAdd(rd_done + t, 1) == T.rd_items - 1;
      }
      __syncthreads();
      if (s_flag) {  // last block of the tuple: finalize it
        __threadfence();
        finalize_tuple(T, S, t, A, red);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) s_flag = atomicAdd(sys_done + T.sys, 1) == S.ntuples - 1;
        __syncthreads();
        if (s_flag) {  // last tuple of the system: sum the system
          __threadfence();
          system_sum(S, T.sys, A, red);
          __threadfence();
        }
      }
    }
  }
}

// ---- grouped executor: per tuple group, one launch of W-build tiles (128-row
// tiles, three CTAs per SM) and one launch of reduction blocks (several CTAs per
// SM); ordering between the launches comes from the stream, so no item waits.
template <int BN>
__global__ void __launch_bounds__(wb::NT, 3) batch_wb_kernel(const BatchArgs A, int64_t item0) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int4 it = A.items[item0 + blockIdx.x];
  const TupleRec &T = A.tuples[it.y];
  const SysDev &S = A.sys[T.sys];
  const int tile_m = it.w / S.tiles_n, tile_n = it.w - tile_m * S.tiles_n;
  wb::wbuild_tile<BN, wb::BM>(A.jobs[(int64_t)it.y * 3 + it.z], S.nu, S.KP, S.nu + S.no, S.NP, tile_m, tile_n, smem);
}

__global__ void __launch_bounds__(kBT, 2) batch_rd_kernel(const BatchArgs A, int64_t item0) {
  extern __shared__ __align__(16) double dsm[];
  __shared__ double red[kBT + 1];
  __shared__ int s_flag;
  int *const rd_done = A.counters + 1 + A.ntuple;
  int *const sys_done = rd_done + A.ntuple + A.ngroup;
  const int4 it = A.items[item0 + blockIdx.x];
  const int t = it.y;
  const TupleRec &T = A.tuples[t];
  const SysDev &S = A.sys[T.sys];
  TupleDev td;
  td.x[0] = T.x[0];
  td.x[1] = T.x[1];
  td.x[2] = T.x[2];
  td.kind = T.kind;
  td.i = T.i;
  td.j = T.j;
  td.k = T.k;
  td.weight = T.kind == kIJK ? 1.0 : 0.5;
  const int c = it.z;
  const int S0 = S.cta_table[3 * c], S1 = S.cta_table[3 * c + 1], S2 = S.cta_table[3 * c + 2];
  if (T.kind == kIJK)
    red::reduce_block<kIJK>(S.nu, S.no, S.NP, td, S.eh, S.ep, S.voe, S0, S1, S2, T.xpart + c, T.vpart, dsm);
  else if (T.kind == kIJJ)
    red::reduce_block<kIJJ>(S.nu, S.no, S.NP, td, S.eh, S.ep, S.voe, S0, S1, S2, T.xpart + c, T.vpart, dsm);
  else
    red::reduce_block<kIIJ>(S.nu, S.no, S.NP, td, S.eh, S.ep, S.voe, S0, S1, S2, T.xpart + c, T.vpart, dsm);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_flag = atomicAdd(rd_done + t, 1) == T.rd_items - 1;
  __syncthreads();
  if (!s_flag) return;
  __threadfence();
  finalize_tuple(T, S, t, A, red);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_flag = atomicAdd(sys_done + T.sys, 1) == S.ntuples - 1;
  __syncthreads();
  if (!s_flag) return;
  __threadfence();
  system_sum(S, T.sys, A, red);
}

template <typename T>
int dmalloc(T **p, size_t n) {
  *p = nullptr;
  CCT_CUDA(cudaMalloc(reinterpret_cast<void **>(p), (n ? n : 1) * sizeof(T)));
  return CCT_OK;
}

}  // namespace
}  // namespace cct

using namespace cct;

struct BatchSystemHost {
  int no = 0, nu = 0;
  Dims d{};
  double *eh = nullptr, *ep = nullptr, *t1 = nullptr, *t2 = nullptr, *vm = nullptr, *voe = nullptr,
         *vvvo = nullptr, *E = nullptr, *F = nullptr, *v1 = nullptr;
  int16_t *cta_table = nullptr;
  int64_t f_np = 0;  // the N padding F was built for
  bool ready = false;
};

struct ccT_batch {
  int device = 0;
  std::vector<BatchSystemHost> sys;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int bn = 0;                             // W-build N tile; 0 = per system
  int order = 0;                          // 0: tuples by cost, largest first; 1: system by system
  int mode = 1;                           // 0: one persistent kernel; 1: grouped launches; 2: grouped, emulated
  ccT_options opt{};                      // creation options (precision, digit target)
  std::vector<ccT_plan *> emu_plans;      // mode 2: per system, the emulated plan (digit operands, digit count)
  struct EmuLaunch {
    int sys;
    int64_t off, njobs;
  };
  std::vector<std::vector<EmuLaunch>> grp_emu;  // mode 2, per group: one W-build launch per system
  EmuJob *emu_jobs = nullptr;
  cudaStream_t stream2 = nullptr;         // reduction launches of the grouped executor
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_wb[kRing] = {}, ev_ring[kRing] = {};
  struct WbRange {
    int64_t begin, count;
    int bn;
  };
  std::vector<std::vector<WbRange>> grp_wb;  // per group: W-build item ranges, one per N tile width
  std::vector<int64_t> grp_rd_begin, grp_rd_count;
  int64_t group_budget = 256ll << 20;     // X scratch bytes per tuple group
  // testing hook (ccT_batch_debug_stall): the reduction blocks of this tuple
  // (position in queue order) wait for one W-build tile more than it has
  int64_t stall_tuple = -1;
  long spin_limit = kSpinLimit;
  bool tuned = false;
  // schedule (device)
  bool scheduled = false;
  int64_t nitems = 0;
  int ntuple = 0, ngroup = 0;
  int4 *items = nullptr;
  int *counters = nullptr;
  int64_t ncounters = 0;
  int *group_rd_items = nullptr;
  TupleRec *tuples = nullptr;
  GemmJob *jobs = nullptr;
  SysDev *sysdev = nullptr;
  double *tuple_etd = nullptr, *tuple_v1 = nullptr, *sys_out = nullptr, *scratch = nullptr;
  int64_t *tuple_v1_off = nullptr;
  int *err = nullptr;
  cudaGraphExec_t graph = nullptr;
  float last_ms = 0.f;
};

namespace {

void free_schedule(ccT_batch *b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  for (void *q : {(void *)b->items, (void *)b->counters, (void *)b->group_rd_items, (void *)b->tuples,
                  (void *)b->jobs, (void *)b->sysdev, (void *)b->tuple_etd, (void *)b->tuple_v1, (void *)b->sys_out,
                  (void *)b->scratch, (void *)b->tuple_v1_off, (void *)b->err, (void *)b->emu_jobs})
    if (q) cudaFree(q);
  b->emu_jobs = nullptr;
  b->items = nullptr;
  b->counters = nullptr;
  b->group_rd_items = nullptr;
  b->tuples = nullptr;
  b->jobs = nullptr;
  b->sysdev = nullptr;
  b->tuple_etd = b->tuple_v1 = b->sys_out = b->scratch = nullptr;
  b->tuple_v1_off = nullptr;
  b->err = nullptr;
  b->scheduled = false;
}

// Dims of one system for the batch N tile.
Dims batch_dims(int no, int nu, int bn) {
  Dims d{};
  d.no = no;
  d.nu = nu;
  d.KP = round_up(nu + no, kKB);
  d.BN = bn;
  d.NP = round_up(nu, bn);
  d.nb = (nu + kRB - 1) / kRB;
  d.ncta = (int64_t)d.nb * (d.nb + 1) * (d.nb + 2) / 6;
  return d;
}

// Mode 2: an emulated plan per system on the batch's device copies of its
// inputs.  Its set_inputs calibrates the digit count to the batch's target and
// builds the digit operands; a forward of its first tuple configures the
// W-build kernel instance it runs, outside any stream capture.
int ensure_emu_plans(ccT_batch *b) {
  b->emu_plans.resize(b->sys.size(), nullptr);
  for (size_t s = 0; s < b->sys.size(); s++) {
    if (b->emu_plans[s]) continue;
    const BatchSystemHost &S = b->sys[s];
    ccT_options o = b->opt;
    o.precision = CCT_PREC_INT8_EMU;
    o.device = b->device;
    o.vvvo_mode = CCT_VVVO_EXPANDED;
    CCT_TRY(ccT_plan_create(&b->emu_plans[s], S.no, S.nu, &o));
    CCT_TRY(ccT_set_inputs(b->emu_plans[s], S.eh, S.ep, S.t1, S.t2, S.vm, S.voe, S.vvvo, CCT_MEM_DEVICE));
    double ets = 0.0, etd = 0.0;
    CCT_TRY(ccT_forward(b->emu_plans[s], 0, 1, &ets, &etd, nullptr));
  }
  return CCT_OK;
}

int build_schedule(ccT_batch *b) {
  free_schedule(b);
  if (b->mode == 2) CCT_TRY(ensure_emu_plans(b));
  const int nsys = (int)b->sys.size();
  struct TH {
    int sys, kind, i, j, k, njobs, group;
    double cost;
    int64_t scratch, x_off, xpart_off, vpart_off;
    int wb_items, rd_items;
  };
  std::vector<TH> th;
  std::vector<int64_t> sys_begin(nsys), sys_count(nsys);
  // F depends on the N tile: rebuild every system's F for this bn
  // (mode 2: the system's emulated plan's dimensions; its X row stride is the plan's)
  for (int s = 0; s < nsys; s++) {
    BatchSystemHost &S = b->sys[s];
    if (b->mode == 2) {
      S.d = plan_dims(b->emu_plans[s]);
      continue;
    }
    const Dims nd = batch_dims(S.no, S.nu, b->bn ? b->bn : choose_bn(S.nu));
    if (S.F && nd.NP != S.f_np) {
      cudaFree(S.F);
      S.F = nullptr;
    }
    S.d = nd;
    if (!S.F) CCT_TRY(dmalloc(&S.F, (size_t)S.no * S.no * nd.NP * nd.KP));
    S.f_np = nd.NP;
    CCT_TRY(launch_build_f(nd, S.t2, S.vm, S.F, b->stream));
  }
  for (int s = 0; s < nsys; s++) {
    const BatchSystemHost &S = b->sys[s];
    const Dims &d = S.d;
    sys_begin[s] = (int64_t)th.size();
    const int64_t nu2 = (int64_t)S.nu * S.nu;
    const int tm = b->mode == 0 ? kBTM : wb::BM;
    const int tiles_m = (int)((nu2 + tm - 1) / tm), tiles_n = (int)(d.NP / d.BN);
    const int64_t npairs = (int64_t)d.nb * (d.nb + 1) / 2;
    for (const Tuple &t : tuple_list(S.no)) {
      TH h{};
      h.sys = s;
      h.kind = t.kind;
      h.i = t.i;
      h.j = t.j;
      h.k = t.k;
      h.njobs = t.kind == kIJK ? 3 : 2;
      h.cost = (double)h.njobs * nu2 * d.NP * d.KP;
      // X, then the reduction partials; rounded to 256 B so every X buffer of
      // the next tuple stays 16-byte aligned (the W-build stores double2)
      h.scratch = round_up(h.njobs * nu2 * d.NP * 8, 256);  // rounded: X buffers stay 16-byte aligned
      h.xpart_off = round_up(d.ncta + (int64_t)d.nb * kRB * 3 * npairs, 32);  // partial doubles (offset later)
      h.wb_items = b->mode == 2 ? 0 : h.njobs * tiles_m * tiles_n;
      h.rd_items = (int)d.ncta;
      th.push_back(h);
    }
    sys_count[s] = (int64_t)th.size() - sys_begin[s];
  }
  const int T = (int)th.size();
  // processing order and groups
  std::vector<int> order(T);
  std::iota(order.begin(), order.end(), 0);
  if (b->order == 0)
    std::stable_sort(order.begin(), order.end(), [&](int u, int v) { return th[u].cost > th[v].cost; });
  std::vector<std::vector<int>> groups;
  int64_t gbytes = 0, ring_slot = 0;
  for (int u : order) {
    if (groups.empty() || gbytes + th[u].scratch > b->group_budget) {
      groups.emplace_back();
      gbytes = 0;
    }
    th[u].group = (int)groups.size() - 1;
    th[u].x_off = gbytes / 8;
    gbytes += th[u].scratch;
    groups.back().push_back(u);
    ring_slot = std::max(ring_slot, gbytes);
  }
  const int G = (int)groups.size();
  const int64_t slot_doubles = ring_slot / 8;
  int64_t npart = 0;
  for (int u = 0; u < T; u++) {
    const int64_t n = th[u].xpart_off;
    th[u].xpart_off = npart;
    npart += n;
  }
  CCT_TRY(dmalloc(&b->scratch, (size_t)slot_doubles * kRing + (size_t)npart));
  double *partials = b->scratch + slot_doubles * kRing;
  // device records
  std::vector<TupleRec> rec(T);
  std::vector<GemmJob> jobs((size_t)T * 3);
  std::vector<int64_t> v1off(T);
  int64_t v1tot = 0;
  for (int u = 0; u < T; u++) {
    const TH &h = th[u];
    const BatchSystemHost &S = b->sys[h.sys];
    const Dims &d = S.d;
    const int64_t nu2 = (int64_t)S.nu * S.nu;
    double *base = b->scratch + (int64_t)(h.group % kRing) * slot_doubles + h.x_off;
    TupleRec r{};
    r.sys = h.sys;
    r.kind = h.kind;
    r.i = h.i;
    r.j = h.j;
    r.k = h.k;
    r.group = h.group;
    r.wb_items = h.wb_items + (u == b->stall_tuple ? 1 : 0);
    r.rd_items = h.rd_items;
    for (int g = 0; g < 3; g++) r.x[g] = base + (int64_t)std::min(g, h.njobs - 1) * nu2 * d.NP;
    r.xpart = partials + h.xpart_off;
    r.vpart = r.xpart + d.ncta;
    rec[u] = r;
    v1off[u] = v1tot;
    v1tot += 3 * S.nu;
    auto Ex = [&](int x) { return S.E + (int64_t)x * nu2 * d.KP; };
    auto Fyz = [&](int y, int z) { return S.F + ((int64_t)y * d.no + z) * d.NP * d.KP; };
    auto G2 = [&](int x1, int x2, int x3, int slot) {
      return GemmJob{Ex(x1), Ex(x2), Fyz(x2, x3), Fyz(x1, x3), r.x[slot], 2, 0};
    };
    auto H1 = [&](int x1, int x2, int x3, int slot) {
      return GemmJob{Ex(x1), Ex(x1), Fyz(x2, x3), Fyz(x2, x3), r.x[slot], 1, 0};
    };
    GemmJob *J = &jobs[(size_t)u * 3];
    if (b->mode == 2) {
      // the emulated executor builds digit-operand jobs below; the FP64 F is not built
    } else if (h.kind == kIJK) {
      J[0] = G2(h.i, h.j, h.k, 0);
      J[1] = G2(h.i, h.k, h.j, 1);
      J[2] = G2(h.j, h.k, h.i, 2);
    } else if (h.kind == kIJJ) {
      J[0] = G2(h.i, h.j, h.j, 0);
      J[1] = H1(h.j, h.j, h.i, 1);
      J[2] = J[1];
    } else {
      J[0] = H1(h.i, h.i, h.k, 0);
      J[1] = G2(h.i, h.k, h.i, 1);
      J[2] = J[1];
    }
  }
  // mode 2: per group and system, the split-integer jobs of the system's
  // tuples in the group (the FP64 jobs above, as digit-operand indices)
  std::vector<EmuJob> ejobs;
  b->grp_emu.assign(G, {});
  if (b->mode == 2) {
    for (int g = 0; g < G; g++) {
      std::vector<std::pair<int, std::vector<int>>> by_sys;  // systems in order of first appearance
      for (int u : groups[g]) {
        auto it = std::find_if(by_sys.begin(), by_sys.end(), [&](const auto &e) { return e.first == th[u].sys; });
        if (it == by_sys.end()) {
          by_sys.push_back({th[u].sys, {}});
          it = by_sys.end() - 1;
        }
        it->second.push_back(u);
      }
      for (const auto &e : by_sys) {
        const int no = b->sys[e.first].no;
        const int64_t off = (int64_t)ejobs.size();
        for (int u : e.second) {
          const TH &h = th[u];
          const TupleRec &r = rec[u];
          // G(x1,x2,x3): E[x1] F[x2][x3] + E[x2]^T F[x1][x3]; H: E[x1] F[x2][x3] alone
          auto G2 = [&](int x1, int x2, int x3, int slot) {
            return EmuJob{x1, x2, {x2 * no + x3, x1 * no + x3}, r.x[slot], 2, x3};
          };
          auto H1 = [&](int x1, int x2, int x3, int slot) {
            return EmuJob{x1, x1, {x2 * no + x3, x2 * no + x3}, r.x[slot], 1, x3};
          };
          if (h.kind == kIJK) {
            ejobs.push_back(G2(h.i, h.j, h.k, 0));
            ejobs.push_back(G2(h.i, h.k, h.j, 1));
            ejobs.push_back(G2(h.j, h.k, h.i, 2));
          } else if (h.kind == kIJJ) {
            ejobs.push_back(G2(h.i, h.j, h.j, 0));
            ejobs.push_back(H1(h.j, h.j, h.i, 1));
          } else {
            ejobs.push_back(H1(h.i, h.i, h.k, 0));
            ejobs.push_back(G2(h.i, h.k, h.i, 1));
          }
        }
        b->grp_emu[g].push_back({e.first, off, (int64_t)ejobs.size() - off});
      }
    }
  }
  // items: WB(g0) WB(g1) RD(g0) WB(g2) RD(g1) ...
  std::vector<int4> items;
  // (grouped executor: WB(g0) RD(g0) WB(g1) RD(g1) ..., one launch per range)
  b->grp_wb.assign(G, {});
  b->grp_rd_begin.assign(G, 0);
  b->grp_rd_count.assign(G, 0);
  auto push_wb = [&](int g) {
    for (int bn : kBNChoices) {  // one range per N tile width (a single one unless bn is per system)
      const int64_t begin = (int64_t)items.size();
      for (int u : groups[g]) {
        if (b->sys[th[u].sys].d.BN != bn) continue;
        const int ntiles = th[u].wb_items / th[u].njobs;
        for (int slot = 0; slot < th[u].njobs; slot++)
          for (int tile = 0; tile < ntiles; tile++) items.push_back(make_int4(0, u, slot, tile));
      }
      if ((int64_t)items.size() > begin) b->grp_wb[g].push_back({begin, (int64_t)items.size() - begin, bn});
    }
  };
  auto push_rd = [&](int g) {
    b->grp_rd_begin[g] = (int64_t)items.size();
    for (int u : groups[g])
      for (int c = 0; c < th[u].rd_items; c++) items.push_back(make_int4(1, u, c, 0));
    b->grp_rd_count[g] = (int64_t)items.size() - b->grp_rd_begin[g];
  };
  if (b->mode == 0) {
    for (int g = 0; g < G; g++) {
      push_wb(g);
      if (g >= 1) push_rd(g - 1);
    }
    push_rd(G - 1);
  } else {
    for (int g = 0; g < G; g++) {
      if (b->mode == 1) push_wb(g);  // mode 2: the emulated launches of grp_emu
      push_rd(g);
    }
  }
  // per-system device records; tuples of a system are consecutive in th
  std::vector<SysDev> sd(nsys);
  for (int s = 0; s < nsys; s++) {
    const BatchSystemHost &S = b->sys[s];
    SysDev v{};
    v.no = S.no;
    v.nu = S.nu;
    v.nb = S.d.nb;
    const int tm = b->mode == 0 ? kBTM : wb::BM;
    v.tiles_m = (int)(((int64_t)S.nu * S.nu + tm - 1) / tm);
    v.tiles_n = (int)(S.d.NP / S.d.BN);
    v.KP = S.d.KP;
    v.NP = S.d.NP;
    v.ncta = S.d.ncta;
    v.eh = S.eh;
    v.ep = S.ep;
    v.t1 = S.t1;
    v.voe = S.voe;
    v.cta_table = S.cta_table;
    v.tuple_begin = sys_begin[s];
    v.ntuples = sys_count[s];
    v.v1 = S.v1;
    sd[s] = v;
  }
  std::vector<int> gnt(G, 0);
  for (int g = 0; g < G; g++)
    for (int u : groups[g]) gnt[g] += th[u].rd_items;
  b->ntuple = T;
  b->ngroup = G;
  b->nitems = (int64_t)items.size();
  b->ncounters = 1 + 2 * (int64_t)T + G + nsys;
  CCT_TRY(dmalloc(&b->items, items.size()));
  CCT_TRY(dmalloc(&b->counters, (size_t)b->ncounters));
  CCT_TRY(dmalloc(&b->group_rd_items, (size_t)G));
  CCT_TRY(dmalloc(&b->tuples, (size_t)T));
  CCT_TRY(dmalloc(&b->jobs, (size_t)T * 3));
  CCT_TRY(dmalloc(&b->sysdev, (size_t)nsys));
  CCT_TRY(dmalloc(&b->tuple_etd, (size_t)T));
  CCT_TRY(dmalloc(&b->tuple_v1, (size_t)v1tot));
  CCT_TRY(dmalloc(&b->tuple_v1_off, (size_t)T));
  CCT_TRY(dmalloc(&b->sys_out, (size_t)3 * nsys));
  CCT_TRY(dmalloc(&b->err, 1));
  CCT_CUDA(cudaMemcpy(b->items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CCT_CUDA(cudaMemcpy(b->group_rd_items, gnt.data(), G * sizeof(int), cudaMemcpyHostToDevice));
  CCT_CUDA(cudaMemcpy(b->tuples, rec.data(), T * sizeof(TupleRec), cudaMemcpyHostToDevice));
  CCT_CUDA(cudaMemcpy(b->jobs, jobs.data(), jobs.size() * sizeof(GemmJob), cudaMemcpyHostToDevice));
  CCT_CUDA(cudaMemcpy(b->sysdev, sd.data(), nsys * sizeof(SysDev), cudaMemcpyHostToDevice));
  CCT_CUDA(cudaMemcpy(b->tuple_v1_off, v1off.data(), T * sizeof(int64_t), cudaMemcpyHostToDevice));
  if (!ejobs.empty()) {
    CCT_TRY(dmalloc(&b->emu_jobs, ejobs.size()));
    CCT_CUDA(cudaMemcpy(b->emu_jobs, ejobs.data(), ejobs.size() * sizeof(EmuJob), cudaMemcpyHostToDevice));
  }
  CCT_CUDA(cudaStreamSynchronize(b->stream));
  b->scheduled = true;
  return CCT_OK;
}

BatchArgs batch_args(ccT_batch *b) {
  BatchArgs a;
  a.items = b->items;
  a.nitems = b->nitems;
  a.counters = b->counters;
  a.ntuple = b->ntuple;
  a.ngroup = b->ngroup;
  a.group_rd_items = b->group_rd_items;
  a.tuples = b->tuples;
  a.jobs = b->jobs;
  a.sys = b->sysdev;
  a.tuple_etd = b->tuple_etd;
  a.tuple_v1 = b->tuple_v1;
  a.tuple_v1_off = b->tuple_v1_off;
  a.sys_out = b->sys_out;
  a.err = b->err;
  a.spin_limit = b->spin_limit;
  return a;
}

// Kernel attributes are set once at batch creation (configure_all), outside any
// stream capture.
template <int BN>
int launch_batch(ccT_batch *b) {
  int nsm = 0;
  CCT_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device));
  const BatchArgs a = batch_args(b);
  CCT_CUDA(cudaMemsetAsync(b->counters, 0, (size_t)b->ncounters * sizeof(int), b->stream));
  CCT_CUDA(cudaMemsetAsync(b->err, 0, sizeof(int), b->stream));
  batch_kernel<BN><<<nsm, kBT, batch_smem<BN>(), b->stream>>>(a);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

// Grouped executor: W-build launches on b->stream, reduction launches on
// b->stream2; group g reuses the X ring slot of group g - kRing only after that
// group's reduction launch.
template <int BN>
int launch_wb_range(const BatchArgs &a, int64_t begin, int64_t count, cudaStream_t s) {
  batch_wb_kernel<BN><<<(unsigned)count, wb::NT, wb::smem_bytes<BN, wb::BM>(), s>>>(a, begin);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

int launch_grouped(ccT_batch *b) {
  const BatchArgs a = batch_args(b);
  CCT_CUDA(cudaMemsetAsync(b->counters, 0, (size_t)b->ncounters * sizeof(int), b->stream));
  CCT_CUDA(cudaMemsetAsync(b->err, 0, sizeof(int), b->stream));
  CCT_CUDA(cudaEventRecord(b->ev_fork, b->stream));
  CCT_CUDA(cudaStreamWaitEvent(b->stream2, b->ev_fork, 0));
  for (int g = 0; g < b->ngroup; g++) {
    const int slot = g % kRing;
    if (g >= kRing) CCT_CUDA(cudaStreamWaitEvent(b->stream, b->ev_ring[slot], 0));
    for (const ccT_batch::EmuLaunch &L : b->grp_emu[g]) {  // mode 2: one emulated launch per system
      const ccT_plan *P = b->emu_plans[L.sys];
      CCT_TRY(launch_wbuild_emu(plan_emu(P), plan_dims(P), b->emu_jobs + L.off, (int)L.njobs, b->err, b->stream));
    }
    for (const ccT_batch::WbRange &r : b->grp_wb[g]) {
      switch (r.bn) {
        case 64: CCT_TRY(launch_wb_range<64>(a, r.begin, r.count, b->stream)); break;
        case 56: CCT_TRY(launch_wb_range<56>(a, r.begin, r.count, b->stream)); break;
        case 48: CCT_TRY(launch_wb_range<48>(a, r.begin, r.count, b->stream)); break;
        case 40: CCT_TRY(launch_wb_range<40>(a, r.begin, r.count, b->stream)); break;
        case 32: CCT_TRY(launch_wb_range<32>(a, r.begin, r.count, b->stream)); break;
        default:
          set_error("unsupported W-build N tile in the batch");
          return CCT_ERR_INVALID;
      }
    }
    CCT_CUDA(cudaEventRecord(b->ev_wb[slot], b->stream));
    CCT_CUDA(cudaStreamWaitEvent(b->stream2, b->ev_wb[slot], 0));
    if (b->grp_rd_count[g] > 0) {
      batch_rd_kernel<<<(unsigned)b->grp_rd_count[g], kBT, red::REDUCE_SMEM, b->stream2>>>(a, b->grp_rd_begin[g]);
      CCT_CUDA(cudaGetLastError());
    }
    CCT_CUDA(cudaEventRecord(b->ev_ring[slot], b->stream2));
  }
  CCT_CUDA(cudaEventRecord(b->ev_join, b->stream2));
  CCT_CUDA(cudaStreamWaitEvent(b->stream, b->ev_join, 0));
  return CCT_OK;
}

int enqueue_forward(ccT_batch *b) {
  if (b->mode == 1 || b->mode == 2) {
    return launch_grouped(b);
  } else {
    switch (b->bn) {
      case 32: return launch_batch<32>(b);
      case 48: return launch_batch<48>(b);
      case 64: return launch_batch<64>(b);
      default: break;
    }
  }
  set_error("unsupported batch N tile");
  return CCT_ERR_INVALID;
}

// Capture counter reset + kernel once; replay afterwards.
int run_forward(ccT_batch *b) {
  if (!b->graph) {
    // configure the kernel attributes outside the capture
    cudaGraph_t g = nullptr;
    CCT_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int s = enqueue_forward(b);
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (s != CCT_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    CCT_CUDA(e);
    const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    CCT_CUDA(ei);
  }
  CCT_CUDA(cudaEventRecord(b->ev0, b->stream));
  CCT_CUDA(cudaGraphLaunch(b->graph, b->stream));
  CCT_CUDA(cudaEventRecord(b->ev1, b->stream));
  return CCT_OK;
}

int batch_inputs_ready(ccT_batch *b) {
  for (size_t s = 0; s < b->sys.size(); s++)
    if (!b->sys[s].ready) {
      set_error("system " + std::to_string(s) + " has no inputs (ccT_batch_set_inputs)");
      return CCT_ERR_STATE;
    }
  return CCT_OK;
}

// Attribute setting must not happen during stream capture: do it up front.
int configure_all(ccT_batch *b) {
  CCT_CUDA(cudaFuncSetAttribute(batch_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, batch_smem<32>()));
  CCT_CUDA(cudaFuncSetAttribute(batch_kernel<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, batch_smem<48>()));
  CCT_CUDA(cudaFuncSetAttribute(batch_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, batch_smem<64>()));
  CCT_CUDA(cudaFuncSetAttribute(batch_wb_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                wb::smem_bytes<32, wb::BM>()));
  CCT_CUDA(cudaFuncSetAttribute(batch_wb_kernel<48>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                wb::smem_bytes<48, wb::BM>()));
  CCT_CUDA(cudaFuncSetAttribute(batch_wb_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                wb::smem_bytes<64, wb::BM>()));
  CCT_CUDA(cudaFuncSetAttribute(batch_wb_kernel<56>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                wb::smem_bytes<56, wb::BM>()));
  CCT_CUDA(cudaFuncSetAttribute(batch_wb_kernel<40>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                wb::smem_bytes<40, wb::BM>()));
  CCT_CUDA(cudaFuncSetAttribute(batch_rd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, red::REDUCE_SMEM));
  CCT_CUDA(cudaFuncSetAttribute(batch_rd_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared));
  (void)b;
  return CCT_OK;
}

struct Guard {
  int prev = 0;
  explicit Guard(int dev) {
    cudaGetDevice(&prev);
    cudaSetDevice(dev);
  }
  ~Guard() { cudaSetDevice(prev); }
};

}  // namespace

extern "C" {

int ccT_batch_create(ccT_batch **out, int64_t nsys, const int64_t *no, const int64_t *nu, const ccT_options *opt) {
  if (!out || nsys < 1 || !no || !nu) {
    set_error("need an output pointer, nsys >= 1 and the no/nu arrays");
    return CCT_ERR_INVALID;
  }
  *out = nullptr;
  ccT_options o;
  ccT_options_default(&o);
  if (opt) o = *opt;
  if (o.precision != CCT_PREC_FP64 && o.precision != CCT_PREC_INT8_EMU) {
    set_error("precision must be CCT_PREC_FP64 or CCT_PREC_INT8_EMU");
    return CCT_ERR_INVALID;
  }
  if (o.precision == CCT_PREC_INT8_EMU &&
      (o.emu_slices < 0 || (o.emu_slices > 0 && (o.emu_slices < kEmuMinSlices || o.emu_slices > kEmuMaxSlices)) ||
       !(o.emu_tol >= 0.0) || !(o.emu_tol_rel >= 0.0))) {
    set_error("emu_slices must be 0 (calibrated) or " + std::to_string(kEmuMinSlices) + ".." +
              std::to_string(kEmuMaxSlices) + ", emu_tol and emu_tol_rel >= 0");
    return CCT_ERR_INVALID;
  }
  int ndev = 0;
  CCT_CUDA(cudaGetDeviceCount(&ndev));
  if (o.device < 0 || o.device >= ndev) {
    set_error("device ordinal out of range");
    return CCT_ERR_INVALID;
  }
  for (int64_t s = 0; s < nsys; s++)
    if (no[s] < 2 || nu[s] < 1 || no[s] > 4096 || nu[s] > 4096) {
      set_error("system " + std::to_string(s) + ": need 2 <= no <= 4096 and 1 <= nu <= 4096");
      return CCT_ERR_INVALID;
    }
  Guard guard(o.device);
  ccT_batch *b = new ccT_batch();
  b->device = o.device;
  b->opt = o;
  b->mode = o.precision == CCT_PREC_INT8_EMU ? 2 : 1;
  auto fail = [&](int st) {
    ccT_batch_destroy(b);
    return st;
  };
  bool ok = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&b->stream2, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreate(&b->ev0) == cudaSuccess && cudaEventCreate(&b->ev1) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) == cudaSuccess;
  for (int r = 0; r < kRing && ok; r++)
    ok = cudaEventCreateWithFlags(&b->ev_wb[r], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&b->ev_ring[r], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    set_error("cannot create the batch streams/events");
    return fail(CCT_ERR_CUDA);
  }
  int st = configure_all(b);
  if (st) return fail(st);
  b->sys.resize(nsys);
  for (int64_t s = 0; s < nsys; s++) {
    BatchSystemHost &S = b->sys[s];
    S.no = (int)no[s];
    S.nu = (int)nu[s];
    S.d = batch_dims(S.no, S.nu, b->bn ? b->bn : choose_bn(S.nu));
    const int64_t n = S.no, v = S.nu, v2 = v * v;
    if ((st = dmalloc(&S.eh, n)) || (st = dmalloc(&S.ep, v)) || (st = dmalloc(&S.t1, n * v)) ||
        (st = dmalloc(&S.t2, v2 * n * n)) || (st = dmalloc(&S.vm, n * v * n * n)) ||
        (st = dmalloc(&S.voe, v2 * n * n)) || (st = dmalloc(&S.vvvo, v * (v + 1) / 2 * v * n)) ||
        (st = dmalloc(&S.E, n * v2 * S.d.KP)) || (st = dmalloc(&S.v1, v * n)) ||
        (st = dmalloc(&S.cta_table, S.d.ncta * 3)))
      return fail(st);
    std::vector<int16_t> table(S.d.ncta * 3);
    int64_t idx = 0;
    for (int C = 0; C < S.d.nb; C++)
      for (int B = 0; B <= C; B++)
        for (int A = 0; A <= B; A++) {
          table[3 * idx] = (int16_t)A;
          table[3 * idx + 1] = (int16_t)B;
          table[3 * idx + 2] = (int16_t)C;
          idx++;
        }
    if (cudaMemcpy(S.cta_table, table.data(), table.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("cannot upload the reduction table");
      return fail(CCT_ERR_CUDA);
    }
  }
  *out = b;
  return CCT_OK;
}

int ccT_batch_set_inputs(ccT_batch *b, int64_t s, const double *eh, const double *ep, const double *t1,
                         const double *t2, const double *vm, const double *voe, const double *vvvo_packed,
                         int32_t mem) {
  if (!b || s < 0 || s >= (int64_t)b->sys.size()) {
    set_error("need a batch and a system index in range");
    return CCT_ERR_INVALID;
  }
  if (!eh || !ep || !t1 || !t2 || !vm || !voe || !vvvo_packed) {
    set_error("an input pointer is NULL");
    return CCT_ERR_INVALID;
  }
  if (mem != CCT_MEM_HOST && mem != CCT_MEM_DEVICE) {
    set_error("mem must be CCT_MEM_HOST or CCT_MEM_DEVICE");
    return CCT_ERR_INVALID;
  }
  Guard guard(b->device);
  BatchSystemHost &S = b->sys[s];
  const int64_t n = S.no, v = S.nu, v2 = v * v;
  if (s < (int64_t)b->emu_plans.size() && b->emu_plans[s]) {  // new inputs: a new calibration
    free_schedule(b);
    ccT_plan_destroy(b->emu_plans[s]);
    b->emu_plans[s] = nullptr;
  }
  const cudaMemcpyKind kind = mem == CCT_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  // device inputs may still be being written on any stream (as ccT_set_inputs)
  if (mem == CCT_MEM_DEVICE) CCT_CUDA(cudaDeviceSynchronize());
  CCT_CUDA(cudaMemcpyAsync(S.eh, eh, n * 8, kind, b->stream));
  CCT_CUDA(cudaMemcpyAsync(S.ep, ep, v * 8, kind, b->stream));
  CCT_CUDA(cudaMemcpyAsync(S.t1, t1, n * v * 8, kind, b->stream));
  CCT_CUDA(cudaMemcpyAsync(S.t2, t2, v2 * n * n * 8, kind, b->stream));
  CCT_CUDA(cudaMemcpyAsync(S.vm, vm, n * v * n * n * 8, kind, b->stream));
  CCT_CUDA(cudaMemcpyAsync(S.voe, voe, v2 * n * n * 8, kind, b->stream));
  CCT_CUDA(cudaMemcpyAsync(S.vvvo, vvvo_packed, v * (v + 1) / 2 * v * n * 8, kind, b->stream));
  CCT_TRY(launch_build_e(S.d, S.vvvo, S.t2, S.E, 0, S.no, b->stream));  // E depends on KP alone
  CCT_CUDA(cudaStreamSynchronize(b->stream));
  free_schedule(b);  // the next forward rebuilds F (for its N tile) and the graph
  S.ready = true;
  return CCT_OK;
}

int ccT_batch_forward(ccT_batch *b, double *ets, double *etd) {
  if (!b) {
    set_error("batch is NULL");
    return CCT_ERR_INVALID;
  }
  CCT_TRY(batch_inputs_ready(b));
  Guard guard(b->device);
  if (!b->scheduled) CCT_TRY(build_schedule(b));
  CCT_TRY(run_forward(b));
  const int nsys = (int)b->sys.size();
  std::vector<double> out(3 * (size_t)nsys);
  int err = 0;
  CCT_CUDA(cudaMemcpyAsync(out.data(), b->sys_out, out.size() * 8, cudaMemcpyDeviceToHost, b->stream));
  CCT_CUDA(cudaMemcpyAsync(&err, b->err, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  CCT_CUDA(cudaStreamSynchronize(b->stream));
  CCT_CUDA(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
  if (err) {
    set_error("a batch work item ran out its bounded wait");
    return CCT_ERR_TIMEOUT;
  }
  for (int s = 0; s < nsys; s++) {
    if (ets) ets[s] = out[3 * s];
    if (etd) etd[s] = out[3 * s + 1];
    if (!std::isfinite(out[3 * s]) || !std::isfinite(out[3 * s + 1])) {
      set_error("E(T) of system " + std::to_string(s) + " is not finite");
      return CCT_ERR_NONFINITE;
    }
  }
  return CCT_OK;
}

int ccT_batch_v1(ccT_batch *b, int64_t s, double *v1_out) {
  if (!b || s < 0 || s >= (int64_t)b->sys.size() || !v1_out) {
    set_error("need a batch, a system index in range and an output pointer");
    return CCT_ERR_INVALID;
  }
  Guard guard(b->device);
  const BatchSystemHost &S = b->sys[s];
  CCT_CUDA(cudaMemcpy(v1_out, S.v1, (size_t)S.nu * S.no * 8, cudaMemcpyDeviceToHost));
  return CCT_OK;
}

int ccT_batch_configure(ccT_batch *b, int32_t mode, int32_t bn, int32_t order, int64_t group_bytes) {
  if (!b) {
    set_error("batch is NULL");
    return CCT_ERR_INVALID;
  }
  bool ok_bn = false;
  for (int c : kBatchBN) ok_bn |= c == bn;
  if (!ok_bn || (order != 0 && order != 1) || mode < 0 || mode > 2 || group_bytes < (1 << 20) ||
      (mode == 0 && bn == 0) || (mode == 2 && bn != 0)) {
    set_error("mode must be 0, 1 or 2, bn 0 (per system; modes 1 and 2), 32, 48 or 64 (modes 0 and 1), "
              "order 0 or 1, group_bytes >= 1 MiB");
    return CCT_ERR_INVALID;
  }
  if (mode == 2 && b->opt.precision != CCT_PREC_INT8_EMU) {
    set_error("mode 2 (emulated W build) needs a batch created with CCT_PREC_INT8_EMU");
    return CCT_ERR_INVALID;
  }
  Guard guard(b->device);
  b->mode = mode;
  b->bn = bn;
  b->order = order;
  b->group_budget = group_bytes;
  free_schedule(b);
  return CCT_OK;
}

int ccT_batch_tune(ccT_batch *b, int32_t *best_mode, int32_t *best_bn, int32_t *best_order, double *best_ms) {
  if (!b) {
    set_error("batch is NULL");
    return CCT_ERR_INVALID;
  }
  CCT_TRY(batch_inputs_ready(b));
  Guard guard(b->device);
  double best = INFINITY;
  int bbn = b->bn, bord = b->order, bmode = b->mode;
  const int last_mode = b->opt.precision == CCT_PREC_INT8_EMU ? 2 : 1;
  for (int mode = 0; mode <= last_mode; mode++)
  for (int bn : kBatchBN)
    for (int order : {0, 1}) {
      if (mode == 0 && bn == 0) continue;  // the persistent kernel has one N tile
      if (mode == 2 && bn != 0) continue;  // the emulated plans keep their own N tiles
      b->mode = mode;
      b->bn = bn;
      b->order = order;
      CCT_TRY(build_schedule(b));
      float ms = 0.f, tot = 0.f;
      for (int rep = 0; rep < 3; rep++) {  // one warm-up, two timed
        CCT_TRY(run_forward(b));
        CCT_CUDA(cudaEventSynchronize(b->ev1));
        CCT_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        if (rep) tot += ms;
      }
      int err = 0;
      CCT_CUDA(cudaMemcpy(&err, b->err, sizeof(int), cudaMemcpyDeviceToHost));
      if (err) {
        set_error("a batch work item ran out its bounded wait while tuning");
        return CCT_ERR_TIMEOUT;
      }
      if (tot / 2 < best) {
        best = tot / 2;
        bmode = mode;
        bbn = bn;
        bord = order;
      }
    }
  b->mode = bmode;
  b->bn = bbn;
  b->order = bord;
  CCT_TRY(build_schedule(b));
  b->tuned = true;
  if (best_mode) *best_mode = bmode;
  if (best_bn) *best_bn = bbn;
  if (best_order) *best_order = bord;
  if (best_ms) *best_ms = best;
  return CCT_OK;
}

double ccT_batch_last_ms(const ccT_batch *b) { return b ? (double)b->last_ms : 0.0; }

int ccT_batch_debug_stall(ccT_batch *b, int64_t tuple, int64_t spin_limit) {
  if (!b) {
    set_error("batch is NULL");
    return CCT_ERR_INVALID;
  }
  if (spin_limit < 0) {
    set_error("spin_limit must be >= 0 (0 = the default)");
    return CCT_ERR_INVALID;
  }
  b->stall_tuple = tuple < 0 ? -1 : tuple;
  b->spin_limit = spin_limit > 0 ? (long)spin_limit : kSpinLimit;
  free_schedule(b);  // the next forward rebuilds the schedule and its graph
  return CCT_OK;
}

int64_t ccT_batch_work_items(const ccT_batch *b) { return b ? b->nitems : 0; }

int ccT_batch_emu_digits(const ccT_batch *b, int64_t s, int32_t *digits) {
  if (!b || s < 0 || s >= (int64_t)b->sys.size() || !digits) {
    set_error("need a batch, a system index in range and an output pointer");
    return CCT_ERR_INVALID;
  }
  if (s >= (int64_t)b->emu_plans.size() || !b->emu_plans[s]) {
    set_error("system " + std::to_string(s) + " has no emulated plan (mode 2 schedule not built)");
    return CCT_ERR_STATE;
  }
  return ccT_emu_digits(b->emu_plans[s], digits, nullptr, nullptr);
}

int ccT_batch_destroy(ccT_batch *b) {
  if (!b) return CCT_OK;
  Guard guard(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->stream2) cudaStreamSynchronize(b->stream2);
  free_schedule(b);
  for (ccT_plan *p : b->emu_plans)
    if (p) ccT_plan_destroy(p);
  for (BatchSystemHost &S : b->sys)
    for (void *q : {(void *)S.eh, (void *)S.ep, (void *)S.t1, (void *)S.t2, (void *)S.vm, (void *)S.voe,
                    (void *)S.vvvo, (void *)S.E, (void *)S.F, (void *)S.v1, (void *)S.cta_table})
      if (q) cudaFree(q);
  for (cudaEvent_t e : {b->ev0, b->ev1, b->ev_fork, b->ev_join})
    if (e) cudaEventDestroy(e);
  for (int r = 0; r < kRing; r++) {
    if (b->ev_wb[r]) cudaEventDestroy(b->ev_wb[r]);
    if (b->ev_ring[r]) cudaEventDestroy(b->ev_ring[r]);
  }
  if (b->stream2) cudaStreamDestroy(b->stream2);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return CCT_OK;
}

}  // extern "C"
