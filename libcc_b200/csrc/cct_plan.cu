// Plan object, tuple scheduler and the exported C ABI.
//
// Replaces the triples driver (src/triples-ijk/triples.F90:1-333,
// src/triples-abc/triples.f90:193-342) for one GPU: the DDI arrays become
// device-resident HBM buffers owned by the plan, the static/dynamic tuple
// partition becomes a host-side tuple list walked in the reference's order,
// and ddi_gsumf becomes fixed-order on-device accumulation.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cct_internal.cuh"

namespace cct {

static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }

std::vector<Tuple> tuple_list(int no) {
  std::vector<Tuple> v;
  // i>j>k in DDCC_T_TASK order (common_functions.f:62-86): i outermost
  for (int i = 0; i < no; i++)
    for (int j = 0; j < i; j++)
      for (int k = 0; k < j; k++) v.push_back({kIJK, i, j, k});
  // then per i, j<i: (i,j,j) and (i,i,j) (triples-abc/triples.f90:286-313)
  for (int i = 0; i < no; i++)
    for (int j = 0; j < i; j++) {
      v.push_back({kIJJ, i, j, j});
      v.push_back({kIIJ, i, i, j});
    }
  return v;
}

}  // namespace cct

using namespace cct;

// X buffer sets: the W-build of tuple t may run while the reductions of
// tuples t-1 .. t-kNBuf+1 are still reading theirs.
constexpr int kNBuf = 3;
// emulated forwards store X in 8 x 8 x 8 blocks (build constant CCT_X_BLOCKED)
#ifndef CCT_X_BLOCKED
#define CCT_X_BLOCKED 1
#endif
constexpr bool kXBlocked = CCT_X_BLOCKED != 0;
#ifndef CCT_SERIAL_REDUCE
#define CCT_SERIAL_REDUCE 1
#endif
constexpr bool kSerialReduce = CCT_SERIAL_REDUCE != 0;
#ifndef CCT_BWD_PRIO
#define CCT_BWD_PRIO 0
#endif

struct ccT_plan {
  int device = 0;
  ccT_options opt{};
  Dims d{};
  cudaStream_t stream = nullptr;      // stream the kernels run on
  cudaStream_t own_stream = nullptr;  // the plan's own stream (ordering, ets)
  cudaStream_t gemm_stream = nullptr; // W-build GEMMs, highest priority
  cudaStream_t red_stream = nullptr;  // reductions, lowest priority: they fill GEMM tail waves
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_gemm[kNBuf] = {}, ev_red[kNBuf] = {};
  int64_t tick = 0;                   // tuples issued so far: selects the X buffer
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // inputs (device copies, reference layouts)
  double *eh = nullptr, *ep = nullptr, *t1 = nullptr, *t2 = nullptr, *vm = nullptr, *voe = nullptr;
  // derived operands
  double *E = nullptr, *F = nullptr;
  double *X[kNBuf][3] = {};  // GEMM outputs, kNBuf tuples in flight
  double *xpart = nullptr, *vpart = nullptr;
  int16_t *cta_table = nullptr;
  double *acc = nullptr;  // [etd_sum, etd_comp, out3[3], v1(nu*no)]
  GemmJob *jobs = nullptr;  // [buffer][tuple][3]
  bool emulated = false;    // INT8 split-integer W-build
  bool packed = false;      // VVVO kept packed (CCT_VVVO_PACKED): no E; vvvo_res and a slab cache instead
  double *vvvo_res = nullptr;
  double *slabs = nullptr;  // packed plans: kSlabs expanded E slabs (nu^2 x KP each), refilled per tuple
  bool emu_auto = false;    // digit count picked by calibration in ccT_set_inputs
  int emu_base_ebn = 0;     // automatic plans: the N tile the kEmuMaxSlices-digit calibration operands use
  double emu_est_err = 0.0, emu_target = 0.0;  // calibrated |dE(T)| bound and its target (Eh)
  EmuOperands emu;
  EmuJob *emu_jobs = nullptr;  // [buffer][tuple][3]
  int *flags = nullptr;
  double *stage = nullptr;  // packed-slice staging for the legacy hook
  std::vector<Tuple> tuples;
  std::vector<char> e_built;  // legacy hook: E[x] built
  bool inputs_ready = false;
  float last_ms = 0.f;
  int64_t last_launches = 0;
  std::vector<double> host_eh, host_ep;
  // opt-in per-kernel profiling: event pairs per launch, grouped by kernel class
  bool profiling = false;
  std::vector<cudaEvent_t> prof_events;
  std::vector<int> prof_class;  // class of each recorded pair
  double kernel_ms[2] = {0.0, 0.0};
  int64_t kernel_launches[2] = {0, 0};
  // backward: buffers and the saved context (range of the last successful forward)
  AdjBuffers adj;
  cudaStream_t bwd_stream = nullptr;   // the dF GEMMs of the backward
  cudaStream_t rec_stream = nullptr;   // the W recompute of the backward
  cudaStream_t pw_stream = nullptr;    // the backward's pointwise chain when it runs below the GEMMs
  cudaEvent_t ev_bwdf[2] = {};
  // backward, per GX set: pointwise pass done / dE GEMM done / dF GEMM done reading it
  cudaEvent_t ev_gx_pw[kGXSets] = {}, ev_gx_e[kGXSets] = {}, ev_gx_f[kGXSets] = {};
  cudaEvent_t ev_rec[kNBuf] = {}, ev_pw[kNBuf] = {};  // X buffer b: W rebuilt / read by the pointwise pass
  int64_t fwd_begin = -1, fwd_end = -1;
  float last_bwd_ms = 0.f;
  // options.keep_w: the W-build output of the last forward, kept for the
  // backward ([t - keep_begin][job slot][nu^2 NP]), and the W-build jobs
  // that write it ([t - keep_begin][3])
  double *xkeep = nullptr;
  size_t xkeep_count = 0;
  GemmJob *keep_jobs = nullptr;
  int64_t keep_jobs_count = 0;
  int64_t keep_begin = -1, keep_end = -1;
};

namespace {

struct DeviceGuard {
  int prev = 0;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    cudaSetDevice(dev);
  }
  ~DeviceGuard() { cudaSetDevice(prev); }
};

template <typename T>
int dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  CCT_CUDA(cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T)));
  return CCT_OK;
}

double *v1_acc(ccT_plan *p) { return p->acc + 5; }

// The FP64 jobs as split-integer jobs: half 0 E[x1] x F[x2][x3], half 1
// E^T[x2] x F[x1][x3], by occupied index instead of by pointer.
int upload_emu_jobs(ccT_plan *p, const std::vector<GemmJob> &jobs, EmuJob *dst) {
  const Dims &d = p->d;
  const int64_t slab = (int64_t)d.nu * d.nu * d.KP, fslab = d.NP * d.KP;
  std::vector<EmuJob> ej(jobs.size());
  for (size_t q = 0; q < jobs.size(); q++) {
    const GemmJob &g = jobs[q];
    EmuJob e{};
    e.x1 = (int)((g.a0 - p->E) / slab);
    e.x2 = (int)((g.a1 - p->E) / slab);
    e.fyz[0] = (int)((g.b0 - p->F) / fslab);
    e.fyz[1] = (int)((g.b1 - p->F) / fslab);
    e.out = g.out;
    e.nhalves = g.nhalves;
    e.x3 = e.fyz[0] % d.no;  // half 0 reads F[x2][x3], half 1 F[x1][x3]
    ej[q] = e;
  }
  CCT_CUDA(cudaMemcpy(dst, ej.data(), ej.size() * sizeof(EmuJob), cudaMemcpyHostToDevice));
  return CCT_OK;
}

// The three W-build GEMM jobs of tuple t (expanded E), writing X slots out[0..2].
void tuple_jobs(const ccT_plan *p, const Tuple &t, double *const out[3], GemmJob J[3]) {
  const Dims &d = p->d;
  const int64_t nu2 = (int64_t)d.nu * d.nu;
  auto Ex = [&](int x) { return p->E + (int64_t)x * nu2 * d.KP; };
  auto Fyz = [&](int y, int z) { return p->F + ((int64_t)y * d.no + z) * d.NP * d.KP; };
  auto G = [&](int x1, int x2, int x3, int slot) {
    return GemmJob{Ex(x1), Ex(x2), Fyz(x2, x3), Fyz(x1, x3), out[slot], 2, 0};
  };
  auto H = [&](int x1, int x2, int x3, int slot) {
    return GemmJob{Ex(x1), Ex(x1), Fyz(x2, x3), Fyz(x2, x3), out[slot], 1, 0};
  };
  if (t.kind == kIJK) {
    J[0] = G(t.i, t.j, t.k, 0);
    J[1] = G(t.i, t.k, t.j, 1);
    J[2] = G(t.j, t.k, t.i, 2);
  } else if (t.kind == kIJJ) {  // (i,j,j): G(i,j,j), H(j,j,i)
    J[0] = G(t.i, t.j, t.j, 0);
    J[1] = H(t.j, t.j, t.i, 1);
    J[2] = H(t.j, t.j, t.i, 2);  // never launched
  } else {  // (i,i,k): H(i,i,k), G(i,k,i)
    J[0] = H(t.i, t.i, t.k, 0);
    J[1] = G(t.i, t.k, t.i, 1);
    J[2] = G(t.i, t.k, t.i, 2);  // never launched
  }
}

int build_jobs(ccT_plan *p) {
  if (p->packed) return CCT_OK;  // jobs name cache slots: built per forward (packed_schedule)
  std::vector<GemmJob> jobs(p->tuples.size() * 3 * kNBuf);
  size_t q = 0;
  for (int buf = 0; buf < kNBuf; buf++)
    for (const Tuple &t : p->tuples) {
      tuple_jobs(p, t, p->X[buf], &jobs[q]);
      q += 3;
    }
  CCT_CUDA(cudaMemcpy(p->jobs, jobs.data(), jobs.size() * sizeof(GemmJob), cudaMemcpyHostToDevice));
  if (p->emulated) CCT_TRY(upload_emu_jobs(p, jobs, p->emu_jobs));
  return CCT_OK;
}

// Packed plans keep kSlabs expanded E slabs in a cache instead of all of E.
// For the tuples [begin, end) in order, a least-recently-used simulation on
// the host gives every slab a tuple needs a slot; (*expand)[t - begin] lists
// the (slot, x) expansions to issue before tuple t's W build, on the stream
// that runs the W builds (so the W build of the tuple before has finished
// reading the slot), and the tuple's jobs, for every X buffer, name the
// slots.  In tuple order i > j > k a tuple usually needs one new slab.
constexpr int kSlabs = 4;
using SlabFills = std::vector<std::vector<std::pair<int, int>>>;

int packed_schedule(ccT_plan *p, int64_t begin, int64_t end, SlabFills *expand) {
  const Dims &d = p->d;
  const int64_t nu2 = (int64_t)d.nu * d.nu, slab = nu2 * d.KP, n = end - begin, ntup = (int64_t)p->tuples.size();
  int slot_x[kSlabs];
  int64_t last[kSlabs];
  for (int c = 0; c < kSlabs; c++) {
    slot_x[c] = -1;
    last[c] = -1;
  }
  expand->assign(n, {});
  auto Fyz = [&](int y, int z) { return p->F + ((int64_t)y * d.no + z) * d.NP * d.KP; };
  std::vector<GemmJob> jobs((size_t)kNBuf * n * 3);
  for (int64_t t = begin; t < end; t++) {
    const Tuple &tu = p->tuples[t];
    const int need[3] = {tu.i, tu.j, tu.k};
    auto needed = [&](int x) { return x == need[0] || x == need[1] || x == need[2]; };
    int slot_of[3];
    for (int q = 0; q < 3; q++) {
      int c = -1;
      for (int c2 = 0; c2 < kSlabs; c2++)
        if (slot_x[c2] == need[q]) c = c2;
      if (c < 0) {  // the least recently used slot holding none of this tuple's slabs (empty slots first)
        for (int c2 = 0; c2 < kSlabs; c2++)
          if (!needed(slot_x[c2]) && (c < 0 || last[c2] < last[c])) c = c2;
        slot_x[c] = need[q];
        (*expand)[t - begin].push_back({c, need[q]});
      }
      last[c] = t;
      slot_of[q] = c;
    }
    auto Ex = [&](int x) {
      const int q = x == need[0] ? 0 : (x == need[1] ? 1 : 2);
      return p->slabs + slot_of[q] * slab;
    };
    for (int buf = 0; buf < kNBuf; buf++) {
      auto G = [&](int x1, int x2, int x3, int sl) {
        return GemmJob{Ex(x1), Ex(x2), Fyz(x2, x3), Fyz(x1, x3), p->X[buf][sl], 2, 0};
      };
      auto H = [&](int x1, int x2, int x3, int sl) {
        return GemmJob{Ex(x1), Ex(x1), Fyz(x2, x3), Fyz(x2, x3), p->X[buf][sl], 1, 0};
      };
      GemmJob *J = &jobs[((size_t)buf * n + (t - begin)) * 3];
      if (tu.kind == kIJK) {
        J[0] = G(tu.i, tu.j, tu.k, 0);
        J[1] = G(tu.i, tu.k, tu.j, 1);
        J[2] = G(tu.j, tu.k, tu.i, 2);
      } else if (tu.kind == kIJJ) {
        J[0] = G(tu.i, tu.j, tu.j, 0);
        J[1] = J[2] = H(tu.j, tu.j, tu.i, 1);
      } else {
        J[0] = H(tu.i, tu.i, tu.k, 0);
        J[1] = J[2] = G(tu.i, tu.k, tu.i, 1);
      }
    }
  }
  for (int buf = 0; buf < kNBuf; buf++)
    CCT_CUDA(cudaMemcpy(p->jobs + 3 * (buf * ntup + begin), jobs.data() + (size_t)buf * n * 3,
                        (size_t)n * 3 * sizeof(GemmJob), cudaMemcpyHostToDevice));
  return CCT_OK;
}

int packed_fill(ccT_plan *p, const std::vector<std::pair<int, int>> &fills, cudaStream_t st) {
  const int64_t slab = (int64_t)p->d.nu * p->d.nu * p->d.KP;
  for (const auto &f : fills) CCT_TRY(launch_build_e_slab(p->d, p->vvvo_res, p->t2, p->slabs + f.first * slab, f.second, st));
  p->last_launches += (int64_t)fills.size();
  return CCT_OK;
}

int check_denominators(ccT_plan *p) {
  // every tuple with work has i>=j>=k not all equal; D_abc <= eh_i+eh_j+eh_k - 3 min(ep)
  const int no = p->d.no, nu = p->d.nu;
  double epmin = p->host_ep[0];
  for (int a = 1; a < nu; a++) epmin = std::fmin(epmin, p->host_ep[a]);
  double worst = -INFINITY;
  for (const Tuple &t : p->tuples) {
    const double dijk = p->host_eh[t.i] + p->host_eh[t.j] + p->host_eh[t.k];
    worst = std::fmax(worst, dijk - 3.0 * epmin);
  }
  (void)no;
  if (!(worst < 0.0)) {
    set_error("denominator e_i+e_j+e_k-e_a-e_b-e_c reaches " + std::to_string(worst) + " >= 0");
    return CCT_ERR_DENOMINATOR;
  }
  return CCT_OK;
}

// Records one event of a profiled launch pair: cls >= 0 opens pair number
// prof_class.size() (event 2q), cls < 0 closes the last opened pair (event 2q+1).
int prof_mark(ccT_plan *p, int cls, cudaStream_t st) {
  if (!p->profiling) return CCT_OK;
  size_t n;
  if (cls >= 0) {
    n = p->prof_class.size() * 2;
  } else {
    if (p->prof_class.empty()) {
      set_error("profiling: close without open");
      return CCT_ERR_STATE;
    }
    n = p->prof_class.size() * 2 - 1;
  }
  while (p->prof_events.size() <= n) {
    cudaEvent_t e;
    CCT_CUDA(cudaEventCreate(&e));
    p->prof_events.push_back(e);
  }
  CCT_CUDA(cudaEventRecord(p->prof_events[n], st));
  if (cls >= 0) p->prof_class.push_back(cls);
  return CCT_OK;
}

int prof_collect(ccT_plan *p) {
  p->kernel_ms[0] = p->kernel_ms[1] = 0.0;
  p->kernel_launches[0] = p->kernel_launches[1] = 0;
  if (!p->profiling) return CCT_OK;
  for (size_t q = 0; q < p->prof_class.size(); q++) {
    float ms = 0.f;
    CCT_CUDA(cudaEventElapsedTime(&ms, p->prof_events[2 * q], p->prof_events[2 * q + 1]));
    p->kernel_ms[p->prof_class[q]] += ms;
    p->kernel_launches[p->prof_class[q]] += 1;
  }
  p->prof_class.clear();
  return CCT_OK;
}

// Orders the plan's GEMM and reduction streams after everything already issued
// on p->stream.
int fork_streams(ccT_plan *p) {
  CCT_CUDA(cudaEventRecord(p->ev_fork, p->stream));
  CCT_CUDA(cudaStreamWaitEvent(p->gemm_stream, p->ev_fork, 0));
  CCT_CUDA(cudaStreamWaitEvent(p->red_stream, p->ev_fork, 0));
  return CCT_OK;
}

// Orders p->stream after every GEMM and reduction issued so far (each GEMM is
// already waited on by the reduction that follows it).
int join_streams(ccT_plan *p) {
  CCT_CUDA(cudaEventRecord(p->ev_join, p->red_stream));
  CCT_CUDA(cudaStreamWaitEvent(p->stream, p->ev_join, 0));
  return CCT_OK;
}

// The W-build GEMMs of tuple tix into X buffer b on stream st: the plan's
// own form, or the FP64 kernel when fp64 is set (emulated plans keep the FP64
// jobs for the backward's recompute and the digit calibration).
// An emulated W build stores X in 8 x 8 x 8 blocks for the reduction
// (blocked), or in rows of NP (ccT_tuple_w, whose W assembly reads rows).
int wbuild_tuple(ccT_plan *p, int64_t tix, int b, bool fp64, cudaStream_t st, bool blocked = kXBlocked) {
  const Tuple &t = p->tuples[tix];
  const int njobs = t.kind == kIJK ? 3 : 2;
  const int64_t ntup = (int64_t)p->tuples.size();
  if (p->emulated && !fp64)
    return launch_wbuild_emu(p->emu, p->d, p->emu_jobs + 3 * (b * ntup + tix), njobs, p->flags + 1, st, blocked);
  return launch_wbuild_f64(p->d, p->jobs + 3 * (b * ntup + tix), njobs, st);
}

// options.keep_w: room and W-build jobs for the X of tuples [begin, end)
// (3 slots a tuple), allocated when that fits in the free device memory with
// a margin of max(2 GB, 10% of the device); *keep says whether it did.
int prepare_keep(ccT_plan *p, int64_t begin, int64_t end, bool *keep) {
  const Dims &d = p->d;
  const int64_t n = end - begin;
  const size_t slab = (size_t)d.nu * d.nu * d.NP;
  const size_t need = (size_t)n * 3 * slab;
  *keep = false;
  if (p->xkeep_count < need) {
    if (p->xkeep) CCT_CUDA(cudaFree(p->xkeep));
    p->xkeep = nullptr;
    p->xkeep_count = 0;
    size_t free_b = 0, total_b = 0;
    CCT_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t margin = std::max<size_t>((size_t)2 << 30, total_b / 10);
    if (need * 8 + margin > free_b) return CCT_OK;  // recompute in the backward
    if (dalloc(&p->xkeep, need) != CCT_OK) {        // (fragmented memory): recompute too
      p->xkeep = nullptr;
      cudaGetLastError();
      return CCT_OK;
    }
    p->xkeep_count = need;
  }
  if (p->keep_jobs_count < 3 * n) {
    if (p->keep_jobs) CCT_CUDA(cudaFree(p->keep_jobs));
    p->keep_jobs = nullptr;
    p->keep_jobs_count = 0;
    CCT_TRY(dalloc(&p->keep_jobs, (size_t)3 * n));
    p->keep_jobs_count = 3 * n;
  }
  std::vector<GemmJob> jobs((size_t)3 * n);
  for (int64_t t = begin; t < end; t++) {
    double *out[3];
    for (int g = 0; g < 3; g++) out[g] = p->xkeep + ((t - begin) * 3 + g) * slab;
    tuple_jobs(p, p->tuples[t], out, &jobs[(size_t)3 * (t - begin)]);
  }
  CCT_CUDA(cudaMemcpy(p->keep_jobs, jobs.data(), jobs.size() * sizeof(GemmJob), cudaMemcpyHostToDevice));
  *keep = true;
  return CCT_OK;
}

// X slot g of the kept W-build output of tuple begin + slot.
double *xkeep_at(const ccT_plan *p, int64_t slot, int g) {
  return p->xkeep + (slot * 3 + g) * (int64_t)p->d.nu * p->d.nu * p->d.NP;
}

// W-build of tuple tix into X buffer b on the GEMM stream, then its reduction on
// the reduction stream.  The GEMM waits until the reduction that last read
// buffer b (two tuples earlier) is done; the reduction waits for its GEMM.
// keep >= 0 (an FP64 plan keeping W for the backward): the W build writes
// the kept slot instead of buffer b.
int run_tuple(ccT_plan *p, int64_t tix, bool fp64 = false, int64_t keep = -1) {
  const Tuple &t = p->tuples[tix];
  const int b = (int)(p->tick % kNBuf);
  p->tick++;
  CCT_CUDA(cudaStreamWaitEvent(p->gemm_stream, p->ev_red[b], 0));
  CCT_TRY(prof_mark(p, CCT_KERNEL_WBUILD, p->gemm_stream));
  if (keep >= 0)
    CCT_TRY(launch_wbuild_f64(p->d, p->keep_jobs + 3 * keep, t.kind == kIJK ? 3 : 2, p->gemm_stream));
  else
    CCT_TRY(wbuild_tuple(p, tix, b, fp64, p->gemm_stream));
  CCT_TRY(prof_mark(p, -1, p->gemm_stream));
  CCT_CUDA(cudaEventRecord(p->ev_gemm[b], p->gemm_stream));
  CCT_CUDA(cudaStreamWaitEvent(p->red_stream, p->ev_gemm[b], 0));
  // emulated W builds fill every SM's shared memory, so the reduction cannot
  // run beside them: it is queued on the W-build stream itself (the
  // reduction stream then only joins).  The step takes the same time as with
  // two streams (667-672 against 662-675 ms for 800 3-digit tuples at
  // no24-nu320), and each kernel's launch time is then its own.
  cudaStream_t rs = p->red_stream;
  if (kSerialReduce && p->emulated && !fp64) rs = p->gemm_stream;
  TupleDev td;
  for (int g = 0; g < 3; g++) td.x[g] = keep >= 0 ? xkeep_at(p, keep, g) : p->X[b][g];
  td.kind = t.kind;
  td.i = t.i;
  td.j = t.j;
  td.k = t.k;
  td.weight = t.kind == kIJK ? 1.0 : 0.5;
  td.blocked = p->emulated && !fp64 && kXBlocked ? 1 : 0;
  CCT_TRY(prof_mark(p, CCT_KERNEL_REDUCE, rs));
  CCT_TRY(launch_reduce(p->d, td, p->eh, p->ep, p->voe, p->cta_table, p->xpart, p->vpart, rs));
  CCT_TRY(launch_finalize(p->d, td, p->xpart, p->vpart, p->acc, v1_acc(p), rs));
  CCT_TRY(prof_mark(p, -1, rs));
  CCT_CUDA(cudaEventRecord(p->ev_red[b], rs));
  if (rs != p->red_stream) CCT_CUDA(cudaStreamWaitEvent(p->red_stream, p->ev_red[b], 0));
  p->last_launches += 3;
  return CCT_OK;
}

// E(T) contribution (etd + ets) of one tuple alone, with the plan's W build or
// the FP64 one.  Leaves the plan's accumulators holding that tuple only.
int tuple_energy(ccT_plan *p, int64_t tix, bool fp64, double *e) {
  const Dims &d = p->d;
  CCT_CUDA(cudaMemsetAsync(p->acc, 0, (5 + (int64_t)d.nu * d.no) * 8, p->stream));
  CCT_CUDA(cudaMemsetAsync(p->flags + 1, 0, 4, p->stream));
  CCT_TRY(fork_streams(p));
  CCT_TRY(run_tuple(p, tix, fp64));
  CCT_TRY(join_streams(p));
  CCT_TRY(launch_ets(d, p->t1, v1_acc(p), p->acc, p->acc + 2, p->stream));
  double out3[3];
  int werr = 0;
  CCT_CUDA(cudaMemcpyAsync(&werr, p->flags + 1, 4, cudaMemcpyDeviceToHost, p->stream));
  CCT_CUDA(cudaMemcpyAsync(out3, p->acc + 2, 3 * 8, cudaMemcpyDeviceToHost, p->stream));
  CCT_CUDA(cudaStreamSynchronize(p->stream));
  if (werr) {
    set_error("an emulated W-build kernel ran out its bounded wait and unwound");
    return CCT_ERR_TIMEOUT;
  }
  *e = out3[0] + out3[1];
  return CCT_OK;
}

// Automatic digit count of an emulated plan.  Up to kCalSamples tuples spread
// evenly over the tuple list run once with the FP64 W build and once per digit
// count, kEmuMinSlices upward.  The error bound for a count assumes every
// tuple errs by the largest sampled |dE| per unit of tuple weight, all with
// the same sign (the weight of an i>j>k tuple is 1, of a degenerate one 1/2),
// times kCalSafety.  The first count whose bound meets
// max(emu_tol, emu_tol_rel |E(T)|), with E(T) extrapolated the same way from
// the FP64 samples, is kept; failing that, the largest count.
constexpr int kCalSamples = 5;
constexpr double kCalSafety = 2.0;
constexpr double kDefaultTol = 1e-8, kDefaultTolRel = 2e-14;

// The widest N tile for S digits whose digits x columns fit the tensor memory
// and which divides NP, starting from the plan's base tile.
int widest_ebn(const ccT_plan *p, int S) {
  int best = p->emu_base_ebn;
  for (int bn : kEmuBNChoices)
    if (S * bn <= 512 && p->d.NP % bn == 0 && bn > best) best = bn;
  return best;
}

// Digit operands of S slices on N tile ebn.
int build_digits(ccT_plan *p, int S, int ebn) {
  p->d.EBN = p->emu.ebn = ebn;
  p->emu.slices = p->emu.run_slices = S;
  return emu_build_operands(p->d, p->E, p->F, &p->emu, p->stream);
}

int calibrate_digits(ccT_plan *p) {
  const int64_t n = (int64_t)p->tuples.size();
  std::vector<int64_t> idx;
  for (int q = 0; q < kCalSamples; q++) {
    const int64_t t = n <= 1 ? 0 : (int64_t)q * (n - 1) / (kCalSamples - 1);
    if (idx.empty() || idx.back() != t) idx.push_back(t);
  }
  auto weight = [&](int64_t t) { return p->tuples[t].kind == kIJK ? 1.0 : 0.5; };
  double wsum_all = 0.0;
  for (const Tuple &t : p->tuples) wsum_all += t.kind == kIJK ? 1.0 : 0.5;
  const bool prof = p->profiling;
  p->profiling = false;
  std::vector<double> e64(idx.size());
  double esum = 0.0, wsum = 0.0;
  int s = CCT_OK;
  for (size_t q = 0; q < idx.size() && s == CCT_OK; q++) {
    s = tuple_energy(p, idx[q], true, &e64[q]);
    esum += e64[q];
    wsum += weight(idx[q]);
  }
  const double e_est = wsum > 0.0 ? esum / wsum * wsum_all : 0.0;
  const double tol = p->opt.emu_tol > 0.0 ? p->opt.emu_tol : kDefaultTol;
  const double rel = p->opt.emu_tol_rel > 0.0 ? p->opt.emu_tol_rel : kDefaultTolRel;
  const double target = std::fmax(tol, rel * std::fabs(e_est));
  // bound of the count the operands are built for now (run_slices)
  auto bound = [&](double *est) {
    double worst = 0.0;
    for (size_t q = 0; q < idx.size() && s == CCT_OK; q++) {
      double e = 0.0;
      s = tuple_energy(p, idx[q], false, &e);
      const double err = std::fabs(e - e64[q]) / weight(idx[q]);
      worst = std::isfinite(err) ? std::fmax(worst, err) : INFINITY;
    }
    *est = kCalSafety * worst * wsum_all;
  };
  int chosen = kEmuMaxSlices;
  double chosen_err = INFINITY;
  int first = kEmuMinSlices;
  // A target of under 3.5 digits' worth of bits relative to |E(T)| (7 bits a
  // digit) is tried at kEmuMinSlices first, on operands built for that count
  // and its own N tile, which are the plan's final operands when it passes.
  // The emulated X does not depend on the N tile or on how many digits the
  // operands hold, so the choice is the one the sweep below would make.
  const double rel_target = e_est != 0.0 ? target / std::fabs(e_est) : 1.0;
  if (s == CCT_OK && std::log2(1.0 / rel_target) < 3.5 * 7) {
    s = build_digits(p, kEmuMinSlices, widest_ebn(p, kEmuMinSlices));
    double est = INFINITY;
    if (s == CCT_OK) bound(&est);
    if (s == CCT_OK && est <= target) {
      chosen = kEmuMinSlices;
      chosen_err = est;
      first = kEmuMaxSlices + 1;  // done
    } else {
      first = kEmuMinSlices + 1;
    }
  }
  if (s == CCT_OK && first <= kEmuMaxSlices) {  // every count on kEmuMaxSlices-digit operands
    s = build_digits(p, kEmuMaxSlices, p->emu_base_ebn);
    for (int sl = first; sl <= kEmuMaxSlices && s == CCT_OK; sl++) {
      p->emu.run_slices = sl;
      double est = INFINITY;
      bound(&est);
      if (s == CCT_OK && (est <= target || sl == kEmuMaxSlices)) {
        chosen = sl;
        chosen_err = est;
        break;
      }
    }
  }
  p->profiling = prof;
  p->emu.run_slices = chosen;
  p->emu_est_err = chosen_err;
  p->emu_target = target;
  return s;
}

// After calibration an automatic plan rebuilds its digit operands for the
// chosen count: only the leading digits (so a pipeline stage is again one
// contiguous copy per operand) and the widest N tile whose digits x columns
// fit the tensor memory and which divides the plan's NP (so F, the X buffers
// and the FP64 jobs keep their layout).  The digits themselves do not depend
// on the count.
int rebuild_for_count(ccT_plan *p) {
  const int S = p->emu.run_slices;
  const int best = widest_ebn(p, S);
  if (S == p->emu.slices && best == p->d.EBN) return CCT_OK;
  return build_digits(p, S, best);
}

[[noreturn]] void legacy_stop(const char *where, int status) {
  std::fprintf(stderr, "libcc_b200: %s failed: %s (%s)\n", where, ccT_status_string(status), last_error());
  std::fflush(stderr);
  std::exit(1);
}

}  // namespace

namespace cct {
const Dims &plan_dims(const ccT_plan *p) { return p->d; }
const EmuOperands &plan_emu(const ccT_plan *p) { return p->emu; }
}  // namespace cct

extern "C" {

void ccT_options_default(ccT_options *opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->precision = CCT_PREC_FP64;
  opt->device = 0;
  opt->check_inputs = 1;
  opt->emu_slices = 0;
  opt->emu_tol = kDefaultTol;
  opt->emu_tol_rel = kDefaultTolRel;
  opt->vvvo_mode = CCT_VVVO_AUTO;
}

const char *ccT_status_string(int status) {
  switch (status) {
    case CCT_OK: return "ok";
    case CCT_ERR_INVALID: return "invalid argument";
    case CCT_ERR_CUDA: return "CUDA error";
    case CCT_ERR_NOMEM: return "device out of memory";
    case CCT_ERR_NONFINITE: return "non-finite input or result";
    case CCT_ERR_DENOMINATOR: return "non-negative orbital-energy denominator";
    case CCT_ERR_STATE: return "call out of order";
    case CCT_ERR_TIMEOUT: return "device wait timed out";
    case CCT_ERR_UNSUPPORTED: return "unsupported option";
    default: return "unknown status";
  }
}

const char *ccT_last_error(void) { return last_error(); }

int64_t ccT_num_tuples(int64_t no) {
  if (no < 0) return 0;
  return no * (no - 1) * (no - 2) / 6 + no * (no - 1);
}

int ccT_plan_create(ccT_plan **out, int64_t no, int64_t nu, const ccT_options *opt) {
  if (!out) {
    set_error("plan pointer is NULL");
    return CCT_ERR_INVALID;
  }
  *out = nullptr;
  if (no < 2 || nu < 1 || no > 4096 || nu > 8 * 32767) {
    set_error("need 2 <= no <= 4096 and 1 <= nu (got no=" + std::to_string(no) + ", nu=" + std::to_string(nu) + ")");
    return CCT_ERR_INVALID;
  }
  if (nu * nu > (int64_t)0x7fffffff) {
    set_error("nu*nu exceeds int32 row indexing");
    return CCT_ERR_INVALID;
  }
  ccT_options o;
  ccT_options_default(&o);
  if (opt) o = *opt;
  if (o.precision != CCT_PREC_FP64 && o.precision != CCT_PREC_INT8_EMU) {
    set_error("unknown precision");
    return CCT_ERR_INVALID;
  }
  if (o.precision == CCT_PREC_INT8_EMU &&
      o.emu_slices != 0 && (o.emu_slices < kEmuMinSlices || o.emu_slices > kEmuMaxSlices)) {
    set_error("emu_slices must be 0 (automatic, the default) or in [" + std::to_string(kEmuMinSlices) + ", " +
              std::to_string(kEmuMaxSlices) + "]");
    return CCT_ERR_INVALID;
  }
  if (!(o.emu_tol >= 0.0) || !(o.emu_tol_rel >= 0.0)) {
    set_error("emu_tol and emu_tol_rel must be >= 0 (0 = default)");
    return CCT_ERR_INVALID;
  }
  if (o.vvvo_mode < CCT_VVVO_AUTO || o.vvvo_mode > CCT_VVVO_PACKED ||
      (o.vvvo_mode == CCT_VVVO_PACKED && o.precision != CCT_PREC_FP64)) {
    set_error("vvvo_mode must be CCT_VVVO_AUTO, _EXPANDED or _PACKED; PACKED needs an FP64 plan");
    return CCT_ERR_INVALID;
  }
  if (o.keep_w != 0 && o.keep_w != 1) {
    set_error("keep_w must be 0 or 1");
    return CCT_ERR_INVALID;
  }
  int ndev = 0;
  CCT_CUDA(cudaGetDeviceCount(&ndev));
  if (o.device < 0 || o.device >= ndev) {
    set_error("device ordinal out of range");
    return CCT_ERR_INVALID;
  }
  DeviceGuard guard(o.device);
  ccT_plan *p = new ccT_plan();
  p->device = o.device;
  p->opt = o;
  Dims &d = p->d;
  d.no = (int)no;
  d.nu = (int)nu;
  d.KP = round_up(nu + no, kKB);
  p->emulated = o.precision == CCT_PREC_INT8_EMU;
  if (p->emulated) {
    // the emulated tile sets NP; the FP64 W-build (the backward's recompute
    // and the digit calibration) takes the widest of its tiles that divides NP (NP is a multiple of 64,
    // 80 or 96, so 64, 40 or 48 always qualifies)
    d.EBN = emu_choose_bn(nu, o.emu_slices ? o.emu_slices : kEmuMaxSlices);
    d.NP = round_up(nu, d.EBN);
    d.BN = 0;
    for (int bn : kBNChoices)
      if (d.NP % bn == 0) {
        d.BN = bn;
        break;
      }
  } else {
    d.EBN = 0;
    d.BN = choose_bn(nu);
    d.NP = round_up(nu, d.BN);
  }
  d.nb = (int)((nu + kRB - 1) / kRB);
  d.ncta = (int64_t)d.nb * (d.nb + 1) * (d.nb + 2) / 6;
  p->tuples = tuple_list((int)no);
  if (!p->emulated) {
    if (o.vvvo_mode == CCT_VVVO_PACKED) {
      p->packed = true;
    } else if (o.vvvo_mode == CCT_VVVO_AUTO) {
      // packed when the expanded operand would take more than half of the free memory
      size_t free_b = 0, total_b = 0;
      if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
        p->packed = (double)no * nu * nu * d.KP * 8.0 > 0.5 * (double)free_b;
    }
  }
  auto fail = [&](int s) {
    ccT_plan_destroy(p);
    return s;
  };
  int s;
  int prio_least = 0, prio_greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest) != cudaSuccess) return fail(CCT_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&p->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithPriority(&p->gemm_stream, cudaStreamNonBlocking, prio_greatest) != cudaSuccess ||
      cudaStreamCreateWithPriority(&p->red_stream, cudaStreamNonBlocking, prio_greatest) != cudaSuccess)
    return fail(CCT_ERR_CUDA);
  p->stream = p->own_stream;
  for (cudaEvent_t *e : {&p->ev_fork, &p->ev_join})
    if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) return fail(CCT_ERR_CUDA);
  for (int b = 0; b < kNBuf; b++)
    if (cudaEventCreateWithFlags(&p->ev_gemm[b], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_red[b], cudaEventDisableTiming) != cudaSuccess)
      return fail(CCT_ERR_CUDA);
  if (cudaEventCreate(&p->ev0) != cudaSuccess || cudaEventCreate(&p->ev1) != cudaSuccess) return fail(CCT_ERR_CUDA);
  const int64_t nu2 = nu * nu;
  if ((s = dalloc(&p->eh, no)) || (s = dalloc(&p->ep, nu)) || (s = dalloc(&p->t1, no * nu)) ||
      (s = dalloc(&p->t2, nu2 * no * no)) || (s = dalloc(&p->vm, no * nu * no * no)) ||
      (s = dalloc(&p->voe, nu2 * no * no)) ||
      (s = p->packed ? dalloc(&p->vvvo_res, nu * (nu + 1) / 2 * nu * no) : dalloc(&p->E, no * nu2 * d.KP)) ||
      (s = p->packed ? dalloc(&p->slabs, kSlabs * nu2 * d.KP) : CCT_OK) ||
      (s = dalloc(&p->F, no * no * d.NP * d.KP)) ||
      (s = dalloc(&p->xpart, d.ncta)) || (s = dalloc(&p->vpart, (int64_t)12 * d.nb * d.nb * (d.nb + 1))) ||
      (s = dalloc(&p->cta_table, d.ncta * 3)) || (s = dalloc(&p->acc, 5 + nu * no)) ||
      (s = dalloc(&p->jobs, p->tuples.size() * 3 * kNBuf)) || (s = dalloc(&p->flags, 4)))
    return fail(s);
  for (int b = 0; b < kNBuf; b++)
    for (int g = 0; g < 3; g++)
      if ((s = dalloc(&p->X[b][g], (p->emulated && kXBlocked ? round_up(nu, kRB) * round_up(nu, kRB) : nu2) * d.NP)))
        return fail(s);
  if (p->emulated) {
    EmuOperands &e = p->emu;
    e.slices = o.emu_slices ? o.emu_slices : kEmuMaxSlices;
    e.run_slices = e.slices;         // an automatic plan lowers it at calibration
    e.ebn = d.EBN;
    e.NPe = d.NP;
    e.adaptive = o.emu_slices == 0;  // automatic: the calibrated count is the maximum, each tile takes what it needs
    p->emu_auto = o.emu_slices == 0;
    p->emu_base_ebn = d.EBN;
    e.KP8 = round_up(nu + no, kEmuKC);
    e.tiles_m = (nu2 + kEmuBM - 1) / kEmuBM;
    const int64_t rowsE = no * nu2, rowsF = no * no * d.NP;
    const int64_t bytesE = e.slices * no * e.tiles_m * kEmuBM * e.KP8;  // row tiles padded to 128 rows
    if ((s = dalloc(&e.E8, bytesE)) || (s = dalloc(&e.E8T, bytesE)) ||
        (s = dalloc(&e.F8, e.slices * rowsF * e.KP8)) || (s = dalloc(&e.expE, rowsE)) ||
        (s = dalloc(&e.expET, rowsE)) || (s = dalloc(&e.expF, rowsF)) || (s = dalloc(&e.expRowF, rowsF)) ||
        (s = dalloc(&p->emu_jobs, p->tuples.size() * 3 * kNBuf)) ||
        (s = dalloc(&e.tileExp, e.tiles_m + no * (d.NP / d.EBN) + 2)) ||
        (s = dalloc(&e.slice_hist, kEmuMaxSlices + 1)))
      return fail(s);
  }
  std::vector<int16_t> table(d.ncta * 3);
  int64_t idx = 0;
  for (int C = 0; C < d.nb; C++)
    for (int B = 0; B <= C; B++)
      for (int A = 0; A <= B; A++) {
        table[3 * idx] = (int16_t)A;
        table[3 * idx + 1] = (int16_t)B;
        table[3 * idx + 2] = (int16_t)C;
        idx++;
      }
  if (cudaMemcpy(p->cta_table, table.data(), table.size() * sizeof(int16_t), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(CCT_ERR_CUDA);
  if ((s = build_jobs(p))) return fail(s);
  p->e_built.assign(no, 0);
  *out = p;
  return CCT_OK;
}

int ccT_set_inputs(ccT_plan *p, const double *eh, const double *ep, const double *t1, const double *t2,
                   const double *vm, const double *voe, const double *vvvo, int32_t mem) {
  if (!p) {
    set_error("plan is NULL");
    return CCT_ERR_INVALID;
  }
  if (!eh || !ep || !t1 || !t2 || !vm || !voe || !vvvo) {
    set_error("an input pointer is NULL");
    return CCT_ERR_INVALID;
  }
  if (mem != CCT_MEM_HOST && mem != CCT_MEM_DEVICE) {
    set_error("mem must be CCT_MEM_HOST or CCT_MEM_DEVICE");
    return CCT_ERR_INVALID;
  }
  DeviceGuard guard(p->device);
  const Dims &d = p->d;
  const int64_t no = d.no, nu = d.nu, nu2 = nu * nu;
  const int64_t nvvvo = nu * (nu + 1) / 2 * nu * no;
  const cudaMemcpyKind kind = mem == CCT_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  p->inputs_ready = false;
  p->fwd_begin = p->fwd_end = -1;
  p->keep_begin = p->keep_end = -1;
  // Device inputs on the plan's own (non-blocking) stream: the caller may
  // still be writing them on any stream, so wait for the whole device.  On a
  // caller stream (ccT_set_stream) the copies are ordered after its work.
  if (mem == CCT_MEM_DEVICE && p->stream == p->own_stream) CCT_CUDA(cudaDeviceSynchronize());
  // From here on a failure is recorded in s and the transient staging buffer
  // is still freed.
  int s = CCT_OK;
  auto cuda = [&](cudaError_t e, const char *what) {
    if (s == CCT_OK && e != cudaSuccess) {
      set_error(std::string(what) + ": " + cudaGetErrorString(e));
      s = e == cudaErrorMemoryAllocation ? CCT_ERR_NOMEM : CCT_ERR_CUDA;
    }
  };
  cuda(cudaMemcpyAsync(p->eh, eh, no * 8, kind, p->stream), "copy eh");
  cuda(cudaMemcpyAsync(p->ep, ep, nu * 8, kind, p->stream), "copy ep");
  cuda(cudaMemcpyAsync(p->t1, t1, no * nu * 8, kind, p->stream), "copy t1");
  cuda(cudaMemcpyAsync(p->t2, t2, nu2 * no * no * 8, kind, p->stream), "copy t2");
  cuda(cudaMemcpyAsync(p->vm, vm, no * nu * no * no * 8, kind, p->stream), "copy vm");
  cuda(cudaMemcpyAsync(p->voe, voe, nu2 * no * no * 8, kind, p->stream), "copy voe");
  const double *vvvo_dev = vvvo;
  double *staged = nullptr;
  if (s == CCT_OK && p->packed) {  // the packed triangle is the resident operand
    cuda(cudaMemcpyAsync(p->vvvo_res, vvvo, nvvvo * 8, kind, p->stream), "copy vvvo");
    vvvo_dev = p->vvvo_res;
  } else if (s == CCT_OK && mem == CCT_MEM_HOST) {
    // the packed VVVO is only needed to build E; stage it in a transient
    // buffer.  Plain cudaMalloc/cudaFree: with the stream-ordered pool this
    // call took 0.12-0.21 s at no=24/nu=320 (3.2 GB staged), 0.08-0.10 s so.
    cuda(cudaMalloc(reinterpret_cast<void **>(&staged), nvvvo * 8), "stage vvvo");
    if (s == CCT_OK) cuda(cudaMemcpyAsync(staged, vvvo, nvvvo * 8, cudaMemcpyHostToDevice, p->stream), "copy vvvo");
    vvvo_dev = staged;
  }
  if (s == CCT_OK && p->opt.check_inputs) {
    cuda(cudaMemsetAsync(p->flags, 0, 16, p->stream), "clear flags");
    if (s == CCT_OK)
      s = launch_check_inputs(d, p->eh, p->ep, p->t1, p->t2, p->vm, p->voe, vvvo_dev, p->flags, p->stream);
  }
  if (s == CCT_OK && !p->packed) s = launch_build_e(d, vvvo_dev, p->t2, p->E, 0, d.no, p->stream);
  if (s == CCT_OK) s = launch_build_f(d, p->t2, p->vm, p->F, p->stream);
  // an automatic plan builds its digit operands during the calibration
  if (s == CCT_OK && p->emulated && !p->emu_auto) s = emu_build_operands(d, p->E, p->F, &p->emu, p->stream);
  if (staged) {
    cudaStreamSynchronize(p->stream);  // E is built (or the stream failed) before the staging buffer goes
    cudaFree(staged);
  }
  if (s != CCT_OK) return s;
  p->host_eh.resize(no);
  p->host_ep.resize(nu);
  int hflags[4] = {0, 0, 0, 0};
  CCT_CUDA(cudaMemcpyAsync(p->host_eh.data(), p->eh, no * 8, cudaMemcpyDeviceToHost, p->stream));
  CCT_CUDA(cudaMemcpyAsync(p->host_ep.data(), p->ep, nu * 8, cudaMemcpyDeviceToHost, p->stream));
  CCT_CUDA(cudaMemcpyAsync(hflags, p->flags, 16, cudaMemcpyDeviceToHost, p->stream));
  CCT_CUDA(cudaStreamSynchronize(p->stream));
  if (p->opt.check_inputs) {
    if (hflags[0]) {
      set_error("an input array holds NaN or Inf");
      return CCT_ERR_NONFINITE;
    }
    CCT_TRY(check_denominators(p));
  }
  std::fill(p->e_built.begin(), p->e_built.end(), 1);
  if (p->emu_auto) {
    int c = calibrate_digits(p);
    if (c == CCT_OK) c = rebuild_for_count(p);
    if (c == CCT_OK) CCT_CUDA(cudaStreamSynchronize(p->stream));
    if (c != CCT_OK) return c;
  }
  p->inputs_ready = true;
  return CCT_OK;
}

int ccT_forward(ccT_plan *p, int64_t begin, int64_t end, double *ets, double *etd, double *v1_out) {
  if (!p) {
    set_error("plan is NULL");
    return CCT_ERR_INVALID;
  }
  if (!p->inputs_ready) {
    set_error("ccT_forward before ccT_set_inputs");
    return CCT_ERR_STATE;
  }
  const int64_t nt = (int64_t)p->tuples.size();
  if (begin < 0 || end > nt || begin > end) {
    set_error("tuple range [" + std::to_string(begin) + ", " + std::to_string(end) + ") outside [0, " +
              std::to_string(nt) + ")");
    return CCT_ERR_INVALID;
  }
  DeviceGuard guard(p->device);
  const Dims &d = p->d;
  p->last_launches = 0;
  CCT_CUDA(cudaMemsetAsync(p->acc, 0, (5 + (int64_t)d.nu * d.no) * 8, p->stream));
  CCT_CUDA(cudaMemsetAsync(p->flags + 1, 0, 4, p->stream));
  if (p->emulated)
    CCT_CUDA(cudaMemsetAsync(p->emu.slice_hist, 0, (kEmuMaxSlices + 1) * sizeof(unsigned long long), p->stream));
  p->keep_begin = p->keep_end = -1;
  bool keep = false;
  if (p->opt.keep_w && !p->emulated && !p->packed && end > begin) CCT_TRY(prepare_keep(p, begin, end, &keep));
  CCT_CUDA(cudaEventRecord(p->ev0, p->stream));
  SlabFills fills;
  if (p->packed) CCT_TRY(packed_schedule(p, begin, end, &fills));
  CCT_TRY(fork_streams(p));
  for (int64_t t = begin; t < end; t++) {
    if (p->packed) CCT_TRY(packed_fill(p, fills[t - begin], p->gemm_stream));
    CCT_TRY(run_tuple(p, t, false, keep ? t - begin : -1));
  }
  CCT_TRY(join_streams(p));
  CCT_TRY(launch_ets(d, p->t1, v1_acc(p), p->acc, p->acc + 2, p->stream));
  p->last_launches += 1;
  CCT_CUDA(cudaEventRecord(p->ev1, p->stream));
  double out3[3];
  int werr = 0;
  CCT_CUDA(cudaMemcpyAsync(&werr, p->flags + 1, 4, cudaMemcpyDeviceToHost, p->stream));
  CCT_CUDA(cudaMemcpyAsync(out3, p->acc + 2, 3 * 8, cudaMemcpyDeviceToHost, p->stream));
  if (v1_out)
    CCT_CUDA(cudaMemcpyAsync(v1_out, v1_acc(p), (int64_t)d.nu * d.no * 8, cudaMemcpyDeviceToHost, p->stream));
  CCT_CUDA(cudaStreamSynchronize(p->stream));
  CCT_CUDA(cudaEventElapsedTime(&p->last_ms, p->ev0, p->ev1));
  CCT_TRY(prof_collect(p));
  if (ets) *ets = out3[0];
  if (etd) *etd = out3[1];
  p->fwd_begin = p->fwd_end = -1;
  if (werr) {
    set_error("an emulated W-build kernel ran out its bounded wait and unwound");
    return CCT_ERR_TIMEOUT;
  }
  if (!std::isfinite(out3[0]) || !std::isfinite(out3[1])) {
    set_error("E(T) is not finite");
    return CCT_ERR_NONFINITE;
  }
  p->fwd_begin = begin;
  p->fwd_end = end;
  if (keep) {
    p->keep_begin = begin;
    p->keep_end = end;
  }
  return CCT_OK;
}

int ccT_backward(ccT_plan *p, int64_t begin, int64_t end, double *d_eh, double *d_ep, double *d_t1, double *d_t2,
                 double *d_vm, double *d_voe, double *d_vvvo, int32_t mem) {
  if (!p) {
    set_error("plan is NULL");
    return CCT_ERR_INVALID;
  }
  if (mem != CCT_MEM_HOST && mem != CCT_MEM_DEVICE) {
    set_error("mem must be CCT_MEM_HOST or CCT_MEM_DEVICE");
    return CCT_ERR_INVALID;
  }
  if (!p->inputs_ready || begin != p->fwd_begin || end != p->fwd_end) {
    set_error("ccT_backward needs a successful ccT_forward over the same tuple range first");
    return CCT_ERR_STATE;
  }
  if (p->d.nu > 4096) {
    set_error("ccT_backward supports nu <= 4096");
    return CCT_ERR_UNSUPPORTED;
  }
  if (p->packed) {
    set_error("ccT_backward needs the expanded VVVO operand (a plan with vvvo_mode CCT_VVVO_EXPANDED)");
    return CCT_ERR_UNSUPPORTED;
  }
  DeviceGuard guard(p->device);
  const Dims &d = p->d;
  if (!p->adj.ready) {
    const int s = adj_alloc(d, &p->adj);
    if (s != CCT_OK) {
      adj_free(&p->adj);
      return s;
    }
  }
  CCT_TRY(adj_configure(p->device));
  if (!p->bwd_stream) {
    // stream priorities of the backward (build constant CCT_BWD_PRIO): 0, the
    // dF GEMM and the recompute at the default priority below the pointwise
    // chain and the dE GEMM; 1, all four at the highest priority; 2, the three
    // GEMM streams at the highest priority and the pointwise chain on a
    // stream of its own at the lowest
    int prio_least = 0, prio_greatest = 0;
    CCT_CUDA(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
    const int prio = CCT_BWD_PRIO >= 1 ? prio_greatest : 0;
    CCT_CUDA(cudaStreamCreateWithPriority(&p->bwd_stream, cudaStreamNonBlocking, prio));
    CCT_CUDA(cudaStreamCreateWithPriority(&p->rec_stream, cudaStreamNonBlocking, prio));
    if (CCT_BWD_PRIO == 2) CCT_CUDA(cudaStreamCreateWithPriority(&p->pw_stream, cudaStreamNonBlocking, prio_least));
    for (cudaEvent_t &e : p->ev_bwdf) CCT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (int g = 0; g < kGXSets; g++)
      for (cudaEvent_t *e : {&p->ev_gx_pw[g], &p->ev_gx_e[g], &p->ev_gx_f[g]})
        CCT_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    for (int b = 0; b < kNBuf; b++) {
      CCT_CUDA(cudaEventCreateWithFlags(&p->ev_rec[b], cudaEventDisableTiming));
      CCT_CUDA(cudaEventCreateWithFlags(&p->ev_pw[b], cudaEventDisableTiming));
    }
  }
  const int64_t ntup = (int64_t)p->tuples.size();
  CCT_CUDA(cudaEventRecord(p->ev0, p->stream));
  CCT_TRY(adj_zero(d, &p->adj, p->stream));
  // dT1 = 2 v1: an emulated plan's v1 is rebuilt from the FP64 W of this pass
  if (p->emulated) CCT_CUDA(cudaMemsetAsync(p->adj.v1, 0, (5 + (size_t)d.nu * d.no) * 8, p->stream));
  // Four streams.  rec_stream rebuilds W of tuple t into X buffer t mod 3,
  // ahead of red_stream, which runs the pointwise adjoint kernels of tuple t
  // (dE/dW, dVOE, deps and dE/dX into GX set t mod 4); bwd_stream then runs
  // the dF GEMM of tuple t, and gemm_stream one dE GEMM for each pair of
  // consecutive tuples (twice the K per output slab, one read-modify-write of
  // dE per pair).  So the latency-bound pointwise chain overlaps the GEMMs of
  // earlier tuples and the recompute of later ones.  Every accumulator is
  // written by one stream only, in tuple order, so the results stay bitwise
  // reproducible.
  CCT_TRY(fork_streams(p));
  cudaStream_t sW = p->rec_stream, sP = p->pw_stream ? p->pw_stream : p->red_stream, sG = p->gemm_stream,
               sF = p->bwd_stream;
  CCT_CUDA(cudaStreamWaitEvent(sF, p->ev_fork, 0));
  CCT_CUDA(cudaStreamWaitEvent(sW, p->ev_fork, 0));
  if (sP != p->red_stream) CCT_CUDA(cudaStreamWaitEvent(sP, p->ev_fork, 0));
  // W kept by the forward (options.keep_w): no recompute, X read from there
  const bool kept = p->keep_begin == begin && p->keep_end == end;
  for (int64_t t = begin; t < end; t++) {
    const Tuple &tu = p->tuples[t];
    const int set = (int)((t - begin) % kGXSets);
    const int xb = (int)((t - begin) % kNBuf);
    double *Xk[3] = {nullptr, nullptr, nullptr};
    if (kept) {
      for (int g = 0; g < 3; g++) Xk[g] = xkeep_at(p, t - begin, g);
    } else {
      if (t - begin >= kNBuf) CCT_CUDA(cudaStreamWaitEvent(sW, p->ev_pw[xb], 0));  // X buffer read by t-3
      CCT_TRY(launch_wbuild_f64(d, p->jobs + 3 * ((int64_t)xb * ntup + t), tu.kind == kIJK ? 3 : 2, sW));
      CCT_CUDA(cudaEventRecord(p->ev_rec[xb], sW));
      CCT_CUDA(cudaStreamWaitEvent(sP, p->ev_rec[xb], 0));
      for (int g = 0; g < 3; g++) Xk[g] = p->X[xb][g];
    }
    if (t - begin >= kGXSets) {  // GX set last read by the GEMMs of tuple t - kGXSets
      CCT_CUDA(cudaStreamWaitEvent(sP, p->ev_gx_e[set], 0));
      CCT_CUDA(cudaStreamWaitEvent(sP, p->ev_gx_f[set], 0));
    }
    CCT_TRY(adj_tuple_pointwise(d, tu, Xk, p->eh, p->ep, p->t1, p->voe, &p->adj, set, sP));
    if (p->emulated) {
      TupleDev td;
      td.x[0] = Xk[0];
      td.x[1] = Xk[1];
      td.x[2] = Xk[2];
      td.kind = tu.kind;
      td.i = tu.i;
      td.j = tu.j;
      td.k = tu.k;
      td.weight = tu.kind == kIJK ? 1.0 : 0.5;
      CCT_TRY(launch_reduce(d, td, p->eh, p->ep, p->voe, p->cta_table, p->xpart, p->vpart, sP));
      CCT_TRY(launch_finalize(d, td, p->xpart, p->vpart, p->adj.v1, p->adj.v1 + 5, sP));
    }
    CCT_CUDA(cudaEventRecord(p->ev_pw[xb], sP));
    CCT_CUDA(cudaEventRecord(p->ev_gx_pw[set], sP));
    CCT_CUDA(cudaStreamWaitEvent(sF, p->ev_gx_pw[set], 0));
    CCT_TRY(adj_tuple_gemm_f(d, tu, p->E, &p->adj, set, sF));
    CCT_CUDA(cudaEventRecord(p->ev_gx_f[set], sF));
    const int pos = (int)((t - begin) % kDEGroup);
    if (pos == kDEGroup - 1 || t == end - 1) {  // the dE GEMM of the group ending at t
      CCT_CUDA(cudaStreamWaitEvent(sG, p->ev_gx_pw[set], 0));  // also covers the group: same stream, earlier
      Tuple group[kDEGroup];
      int sets[kDEGroup];
      for (int u = 0; u <= pos; u++) {
        group[u] = p->tuples[t - pos + u];
        sets[u] = (set + kGXSets - pos + u) % kGXSets;
      }
      CCT_TRY(adj_tuple_gemm_e(d, group, sets, pos + 1, p->F, &p->adj, sG));
      for (int u = 0; u <= pos; u++) CCT_CUDA(cudaEventRecord(p->ev_gx_e[sets[u]], sG));
    }
  }
  // p->stream after every stream (red_stream already waited for rec_stream)
  CCT_CUDA(cudaEventRecord(p->ev_join, sP));
  CCT_CUDA(cudaStreamWaitEvent(p->stream, p->ev_join, 0));
  CCT_CUDA(cudaEventRecord(p->ev_fork, sG));
  CCT_CUDA(cudaStreamWaitEvent(p->stream, p->ev_fork, 0));
  CCT_CUDA(cudaEventRecord(p->ev_bwdf[0], sF));
  CCT_CUDA(cudaStreamWaitEvent(p->stream, p->ev_bwdf[0], 0));
  CCT_TRY(adj_finish(d, p->emulated ? p->adj.v1 + 5 : v1_acc(p), &p->adj, p->stream));
  CCT_CUDA(cudaEventRecord(p->ev1, p->stream));
  const cudaMemcpyKind kind = mem == CCT_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const int64_t no = d.no, nu = d.nu, nu2 = nu * nu;
  const struct {
    double *dst;
    const double *src;
    int64_t n;
  } outs[] = {{d_eh, p->adj.g_eh, no},
              {d_ep, p->adj.g_ep, nu},
              {d_t1, p->adj.g_t1, no * nu},
              {d_t2, p->adj.g_t2, nu2 * no * no},
              {d_vm, p->adj.g_vm, no * nu * no * no},
              {d_voe, p->adj.g_voe, nu2 * no * no},
              {d_vvvo, p->adj.g_vvvo, nu * (nu + 1) / 2 * nu * no}};
  for (const auto &o : outs)
    if (o.dst) CCT_CUDA(cudaMemcpyAsync(o.dst, o.src, (size_t)o.n * 8, kind, p->stream));
  CCT_CUDA(cudaStreamSynchronize(p->stream));
  CCT_CUDA(cudaEventElapsedTime(&p->last_bwd_ms, p->ev0, p->ev1));
  return CCT_OK;
}

double ccT_last_backward_ms(const ccT_plan *p) { return p ? (double)p->last_bwd_ms : 0.0; }

int64_t ccT_kept_tuples(const ccT_plan *p) { return p && p->keep_end > p->keep_begin ? p->keep_end - p->keep_begin : 0; }

int ccT_emu_slice_histogram(ccT_plan *p, int64_t *hist, int32_t n) {
  if (!p || !hist || n < 1) {
    set_error("need a plan, an output array and n >= 1");
    return CCT_ERR_INVALID;
  }
  for (int32_t s = 0; s < n; s++) hist[s] = 0;
  if (!p->emulated) return CCT_OK;
  DeviceGuard guard(p->device);
  unsigned long long h[kEmuMaxSlices + 1];
  CCT_CUDA(cudaStreamSynchronize(p->stream));
  CCT_CUDA(cudaMemcpy(h, p->emu.slice_hist, sizeof(h), cudaMemcpyDeviceToHost));
  for (int32_t s = 0; s < n && s <= kEmuMaxSlices; s++) hist[s] = (int64_t)h[s];
  return CCT_OK;
}

int ccT_emu_digits(const ccT_plan *p, int32_t *digits, double *est_err, double *target) {
  if (!p) {
    set_error("plan is NULL");
    return CCT_ERR_INVALID;
  }
  if (!p->emulated) {
    set_error("ccT_emu_digits: an FP64 plan has no digit count");
    return CCT_ERR_STATE;
  }
  if (digits) *digits = p->emu.run_slices;
  if (est_err) *est_err = p->emu_auto ? p->emu_est_err : 0.0;
  if (target) *target = p->emu_auto ? p->emu_target : 0.0;
  return CCT_OK;
}

int ccT_tuple_w(ccT_plan *p, int64_t tuple, double *w, int32_t mem) {
  if (!p || !w) {
    set_error("need a plan and an output pointer");
    return CCT_ERR_INVALID;
  }
  if (mem != CCT_MEM_HOST && mem != CCT_MEM_DEVICE) {
    set_error("mem must be CCT_MEM_HOST or CCT_MEM_DEVICE");
    return CCT_ERR_INVALID;
  }
  if (!p->inputs_ready) {
    set_error("ccT_tuple_w before ccT_set_inputs");
    return CCT_ERR_STATE;
  }
  if (tuple < 0 || tuple >= (int64_t)p->tuples.size()) {
    set_error("tuple index out of range");
    return CCT_ERR_INVALID;
  }
  DeviceGuard guard(p->device);
  CCT_TRY(adj_configure(p->device));
  const int64_t n3 = (int64_t)p->d.nu * p->d.nu * p->d.nu;
  // X buffer set 0 and the plan's stream, after everything already issued
  CCT_CUDA(cudaStreamSynchronize(p->gemm_stream));
  CCT_CUDA(cudaStreamSynchronize(p->red_stream));
  double *wc = nullptr, *wf = nullptr;
  CCT_CUDA(cudaMalloc(reinterpret_cast<void **>(&wc), n3 * 8));
  int s = CCT_OK;
  if (mem == CCT_MEM_HOST) {
    const cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&wf), n3 * 8);
    if (e != cudaSuccess) {
      set_error(std::string("ccT_tuple_w: ") + cudaGetErrorString(e));
      s = CCT_ERR_NOMEM;
    }
  } else {
    wf = w;
  }
  if (s == CCT_OK) CCT_CUDA(cudaMemsetAsync(p->flags + 1, 0, 4, p->stream));
  if (s == CCT_OK && p->packed) {
    SlabFills fills;
    s = packed_schedule(p, tuple, tuple + 1, &fills);
    if (s == CCT_OK) s = packed_fill(p, fills[0], p->stream);
  }
  if (s == CCT_OK) s = wbuild_tuple(p, tuple, 0, false, p->stream, false);  // rows of NP, as the assembly reads
  if (s == CCT_OK) s = assemble_w_fortran(p->d, p->tuples[tuple], p->X[0], wc, wf, p->stream);
  int werr = 0;
  if (s == CCT_OK && cudaMemcpyAsync(&werr, p->flags + 1, 4, cudaMemcpyDeviceToHost, p->stream) != cudaSuccess)
    s = CCT_ERR_CUDA;
  if (s == CCT_OK && mem == CCT_MEM_HOST &&
      cudaMemcpyAsync(w, wf, n3 * 8, cudaMemcpyDeviceToHost, p->stream) != cudaSuccess)
    s = CCT_ERR_CUDA;
  if (cudaStreamSynchronize(p->stream) != cudaSuccess && s == CCT_OK) s = CCT_ERR_CUDA;
  if (s == CCT_ERR_CUDA) set_error("ccT_tuple_w: a CUDA call failed");
  cudaFree(wc);
  if (mem == CCT_MEM_HOST && wf) cudaFree(wf);
  if (s == CCT_OK && werr) {
    set_error("an emulated W-build kernel ran out its bounded wait and unwound");
    s = CCT_ERR_TIMEOUT;
  }
  return s;
}

int ccT_set_stream(ccT_plan *p, void *cuda_stream) {
  if (!p) {
    set_error("plan is NULL");
    return CCT_ERR_INVALID;
  }
  DeviceGuard guard(p->device);
  CCT_CUDA(cudaStreamSynchronize(p->stream));
  p->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : p->own_stream;
  return CCT_OK;
}

int ccT_time_wbuild(ccT_plan *p, int64_t tuple, int32_t reps, double *ms_per_launch) {
  if (!p || !ms_per_launch || reps < 1) {
    set_error("need a plan, an output pointer and reps >= 1");
    return CCT_ERR_INVALID;
  }
  if (!p->inputs_ready) {
    set_error("ccT_time_wbuild before ccT_set_inputs");
    return CCT_ERR_STATE;
  }
  if (tuple < 0 || tuple >= (int64_t)p->tuples.size()) {
    set_error("tuple index out of range");
    return CCT_ERR_INVALID;
  }
  DeviceGuard guard(p->device);
  const int njobs = p->tuples[tuple].kind == kIJK ? 3 : 2;
  CCT_TRY(fork_streams(p));
  CCT_CUDA(cudaStreamWaitEvent(p->gemm_stream, p->ev_red[0], 0));
  if (p->packed) {  // the tuple's slabs into the cache (not timed)
    SlabFills fills;
    CCT_TRY(packed_schedule(p, tuple, tuple + 1, &fills));
    CCT_TRY(packed_fill(p, fills[0], p->gemm_stream));
  }
  auto launch = [&]() {
    return p->emulated ? launch_wbuild_emu(p->emu, p->d, p->emu_jobs + 3 * tuple, njobs, p->flags + 1, p->gemm_stream,
                                           kXBlocked)
                       : launch_wbuild_f64(p->d, p->jobs + 3 * tuple, njobs, p->gemm_stream);
  };
  CCT_TRY(launch());  // warm
  CCT_CUDA(cudaEventRecord(p->ev0, p->gemm_stream));
  for (int r = 0; r < reps; r++) CCT_TRY(launch());
  CCT_CUDA(cudaEventRecord(p->ev1, p->gemm_stream));
  CCT_CUDA(cudaEventRecord(p->ev_red[0], p->gemm_stream));  // later writers of buffer 0 follow these
  CCT_CUDA(cudaEventSynchronize(p->ev1));
  float ms = 0.f;
  CCT_CUDA(cudaEventElapsedTime(&ms, p->ev0, p->ev1));
  *ms_per_launch = ms / reps;
  return CCT_OK;
}

int ccT_set_profiling(ccT_plan *p, int32_t on) {
  if (!p) {
    set_error("plan is NULL");
    return CCT_ERR_INVALID;
  }
  p->profiling = on != 0;
  p->prof_class.clear();
  return CCT_OK;
}

int ccT_last_kernel_ms(const ccT_plan *p, int32_t cls, double *total_ms, int64_t *launches) {
  if (!p || cls < 0 || cls > 1) {
    set_error("need a plan and kernel class 0 or 1");
    return CCT_ERR_INVALID;
  }
  if (total_ms) *total_ms = p->kernel_ms[cls];
  if (launches) *launches = p->kernel_launches[cls];
  return CCT_OK;
}

double ccT_last_forward_ms(const ccT_plan *p) { return p ? (double)p->last_ms : 0.0; }
int64_t ccT_last_forward_launches(const ccT_plan *p) { return p ? p->last_launches : 0; }

int ccT_plan_destroy(ccT_plan *p) {
  if (!p) return CCT_OK;
  DeviceGuard guard(p->device);
  for (cudaStream_t st : {p->stream, p->gemm_stream, p->red_stream, p->bwd_stream, p->rec_stream})
    if (st) cudaStreamSynchronize(st);
  double *bufs[] = {p->eh, p->ep, p->t1, p->t2, p->vm, p->voe, p->E, p->F, p->xpart, p->vpart, p->acc, p->stage,
                    p->vvvo_res, p->slabs};
  for (double *b : bufs)
    if (b) cudaFree(b);
  for (int b = 0; b < kNBuf; b++)
    for (int g = 0; g < 3; g++)
      if (p->X[b][g]) cudaFree(p->X[b][g]);
  if (p->cta_table) cudaFree(p->cta_table);
  if (p->jobs) cudaFree(p->jobs);
  if (p->xkeep) cudaFree(p->xkeep);
  if (p->keep_jobs) cudaFree(p->keep_jobs);
  if (p->flags) cudaFree(p->flags);
  for (void *b : {(void *)p->emu.E8, (void *)p->emu.E8T, (void *)p->emu.F8, (void *)p->emu.expE,
                  (void *)p->emu.expET, (void *)p->emu.expF, (void *)p->emu.expRowF, (void *)p->emu_jobs,
                  (void *)p->emu.tileExp, (void *)p->emu.slice_hist})
    if (b) cudaFree(b);
  adj_free(&p->adj);
  if (p->ev0) cudaEventDestroy(p->ev0);
  if (p->ev1) cudaEventDestroy(p->ev1);
  for (cudaEvent_t e : p->prof_events) cudaEventDestroy(e);
  for (cudaEvent_t e : {p->ev_fork, p->ev_join})
    if (e) cudaEventDestroy(e);
  for (int b = 0; b < kNBuf; b++) {
    if (p->ev_gemm[b]) cudaEventDestroy(p->ev_gemm[b]);
    if (p->ev_red[b]) cudaEventDestroy(p->ev_red[b]);
  }
  if (p->gemm_stream) cudaStreamDestroy(p->gemm_stream);
  if (p->bwd_stream) cudaStreamDestroy(p->bwd_stream);
  if (p->rec_stream) cudaStreamDestroy(p->rec_stream);
  if (p->pw_stream) cudaStreamDestroy(p->pw_stream);
  for (cudaEvent_t e : p->ev_bwdf)
    if (e) cudaEventDestroy(e);
  for (int b = 0; b < kNBuf; b++) {
    if (p->ev_rec[b]) cudaEventDestroy(p->ev_rec[b]);
    if (p->ev_pw[b]) cudaEventDestroy(p->ev_pw[b]);
  }
  for (int g = 0; g < kGXSets; g++)
    for (cudaEvent_t e : {p->ev_gx_pw[g], p->ev_gx_e[g], p->ev_gx_f[g]})
      if (e) cudaEventDestroy(e);
  if (p->red_stream) cudaStreamDestroy(p->red_stream);
  if (p->own_stream) cudaStreamDestroy(p->own_stream);
  delete p;
  return CCT_OK;
}

double ccT_measure_fp64_peak(int32_t device) { return measure_fp64_peak(device); }
double ccT_measure_int8_peak(int32_t device) { return measure_int8_peak(device); }

// ----------------------------------------------------------------------------- legacy hooks

static ccT_plan *g_hook = nullptr;
static double *g_hook_v1 = nullptr;
static std::mutex g_hook_mutex;

void ijk_gpu_init_(const int64_t *no, const int64_t *nu, const double *eh, const double *ep, double *v1,
                   const double *t2, const double *vm, const double *voe) {
  std::lock_guard<std::mutex> lock(g_hook_mutex);
  if (!no || !nu || !eh || !ep || !v1 || !t2 || !vm || !voe) legacy_stop("ijk_gpu_init", CCT_ERR_INVALID);
  if (g_hook) {
    ccT_plan_destroy(g_hook);
    g_hook = nullptr;
  }
  ccT_plan *p = nullptr;
  ccT_options o;
  ccT_options_default(&o);
  o.vvvo_mode = CCT_VVVO_EXPANDED;  // the driver hook expands each packed slice into E
  int s = ccT_plan_create(&p, *no, *nu, &o);
  if (s) legacy_stop("ijk_gpu_init", s);
  DeviceGuard guard(p->device);
  const int64_t n_o = *no, n_u = *nu, nu2 = n_u * n_u;
  auto up = [&](double *dst, const double *src, int64_t n) {
    if (cudaMemcpy(dst, src, n * 8, cudaMemcpyHostToDevice) != cudaSuccess) legacy_stop("ijk_gpu_init", CCT_ERR_CUDA);
  };
  up(p->eh, eh, n_o);
  up(p->ep, ep, n_u);
  up(p->t2, t2, nu2 * n_o * n_o);
  up(p->vm, vm, n_o * n_u * n_o * n_o);
  up(p->voe, voe, nu2 * n_o * n_o);
  if ((s = launch_build_f(p->d, p->t2, p->vm, p->F, p->stream))) legacy_stop("ijk_gpu_init", s);
  if ((s = dalloc(&p->stage, n_u * (n_u + 1) / 2 * n_u))) legacy_stop("ijk_gpu_init", s);
  if (cudaMemsetAsync(p->acc, 0, (5 + n_u * n_o) * 8, p->stream) != cudaSuccess) legacy_stop("ijk_gpu_init", CCT_ERR_CUDA);
  p->host_eh.assign(eh, eh + n_o);
  p->host_ep.assign(ep, ep + n_u);
  std::fill(p->e_built.begin(), p->e_built.end(), 0);
  p->inputs_ready = true;
  g_hook = p;
  g_hook_v1 = v1;
}

void ijk_gpu_driver_(const int64_t *nu, const int64_t *no, const int64_t *i, const int64_t *j, const int64_t *k,
                     const double *ve_i, const double *ve_j, const double *ve_k, double *t1, const double *eh,
                     const double *ep, double *etd) {
  (void)t1; (void)eh; (void)ep; (void)etd;
  std::lock_guard<std::mutex> lock(g_hook_mutex);
  ccT_plan *p = g_hook;
  if (!p) legacy_stop("ijk_gpu_driver", CCT_ERR_STATE);
  if (!nu || !no || !i || !j || !k || *nu != p->d.nu || *no != p->d.no) legacy_stop("ijk_gpu_driver", CCT_ERR_INVALID);
  const int64_t I = *i - 1, J = *j - 1, K = *k - 1;  // reference indices are 1-based
  if (!(I > J && J > K && K >= 0 && I < p->d.no)) {
    set_error("need i > j > k >= 1 and i <= no");
    legacy_stop("ijk_gpu_driver", CCT_ERR_INVALID);
  }
  DeviceGuard guard(p->device);
  const int64_t slice = (int64_t)p->d.nu * (p->d.nu + 1) / 2 * p->d.nu;
  const int64_t xs[3] = {I, J, K};
  const double *vs[3] = {ve_i, ve_j, ve_k};
  for (int r = 0; r < 3; r++) {
    const int64_t x = xs[r];
    if (p->e_built[x]) continue;
    if (!vs[r]) legacy_stop("ijk_gpu_driver", CCT_ERR_INVALID);
    if (cudaMemcpyAsync(p->stage, vs[r], slice * 8, cudaMemcpyHostToDevice, p->stream) != cudaSuccess)
      legacy_stop("ijk_gpu_driver", CCT_ERR_CUDA);
    int s = launch_build_e_slice(p->d, p->stage, p->t2, p->E, (int)x, p->stream);
    if (s) legacy_stop("ijk_gpu_driver", s);
    if (cudaStreamSynchronize(p->stream) != cudaSuccess) legacy_stop("ijk_gpu_driver", CCT_ERR_CUDA);
    p->e_built[x] = 1;
  }
  // index of (I,J,K) in the tuple list: DDCC_T_TASK order
  const int64_t tix = I * (I - 1) * (I - 2) / 6 + J * (J - 1) / 2 + K;
  int s = fork_streams(p);
  if (!s) s = run_tuple(p, tix);
  if (s) legacy_stop("ijk_gpu_driver", s);
}

void ijk_gpu_finalize_(const int64_t *no, const int64_t *nu, double *etd) {
  std::lock_guard<std::mutex> lock(g_hook_mutex);
  ccT_plan *p = g_hook;
  if (!p) legacy_stop("ijk_gpu_finalize", CCT_ERR_STATE);
  if (!no || !nu || !etd || *no != p->d.no || *nu != p->d.nu) legacy_stop("ijk_gpu_finalize", CCT_ERR_INVALID);
  DeviceGuard guard(p->device);
  const int64_t n = (int64_t)p->d.nu * p->d.no;
  std::vector<double> v1(n);
  double e[2];
  if (join_streams(p) != CCT_OK ||
      cudaMemcpyAsync(e, p->acc, 16, cudaMemcpyDeviceToHost, p->stream) != cudaSuccess ||
      cudaMemcpyAsync(v1.data(), v1_acc(p), n * 8, cudaMemcpyDeviceToHost, p->stream) != cudaSuccess ||
      cudaStreamSynchronize(p->stream) != cudaSuccess)
    legacy_stop("ijk_gpu_finalize", CCT_ERR_CUDA);
  *etd += e[0] + e[1];
  for (int64_t q = 0; q < n; q++) g_hook_v1[q] += v1[q];
  ccT_plan_destroy(p);
  g_hook = nullptr;
  g_hook_v1 = nullptr;
}

void cc_triples_b200_(const int64_t *no, const int64_t *nu, const double *eh, const double *ep, double *v1,
                      const double *t1, const double *t2, const double *vm, const double *voe, const double *vvvo,
                      double *ets, double *etd) {
  if (!no || !nu || !ets || !etd) legacy_stop("cc_triples_b200", CCT_ERR_INVALID);
  ccT_plan *p = nullptr;
  int s = ccT_plan_create(&p, *no, *nu, nullptr);
  if (s) legacy_stop("cc_triples_b200", s);
  s = ccT_set_inputs(p, eh, ep, t1, t2, vm, voe, vvvo, CCT_MEM_HOST);
  if (s == CCT_OK) s = ccT_forward(p, 0, ccT_num_tuples(*no), ets, etd, v1);
  ccT_plan_destroy(p);
  if (s) legacy_stop("cc_triples_b200", s);
}

}  // extern "C"
