// Internal declarations shared by the libcc_b200 translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/libcc_b200.h"

namespace cct {

// ----------------------------------------------------------------------------- errors
void set_error(const std::string &msg);
const char *last_error();

#define CCT_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                \
      ::cct::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                 \
      return e_ == cudaErrorMemoryAllocation ? CCT_ERR_NOMEM : CCT_ERR_CUDA;                \
    }                                                                                       \
  } while (0)

#define CCT_TRY(call)                  \
  do {                                 \
    int s_ = (call);                   \
    if (s_ != CCT_OK) return s_;       \
  } while (0)

// ----------------------------------------------------------------------------- tiling
// W-build GEMM tile (FP64 DMMA kernel).  K is padded to KB; the single-index
// dimension N is tiled by BN, one of kBNChoices, picked per system to minimise
// the padding of nu (choose_bn).
constexpr int kKB = 16;
constexpr int kBNChoices[] = {64, 56, 48, 40, 32};
inline int choose_bn(int64_t nu) {
  int best = 64;
  int64_t best_np = (nu + 63) / 64 * 64;
  for (int bn : kBNChoices) {
    const int64_t np = (nu + bn - 1) / bn * bn;
    if (np < best_np) {
      best = bn;
      best_np = np;
    }
  }
  return best;
}
// Reduction block edge (elements of a, b, c per block).
constexpr int kRB = 8;

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Tuple kinds.  Every tuple is stored as (i,j,k) with i>=j>=k, 0-based.
enum TupleKind : int { kIJK = 0, kIJJ = 1, kIIJ = 2 };

struct Tuple {
  int kind, i, j, k;
};

// Global tuple list in the reference's order (i>j>k in DDCC_T_TASK order, then
// for each i and j<i the (i,j,j) and (i,i,j) tuples).
std::vector<Tuple> tuple_list(int no);

// One W-build GEMM: X(p,q,s) = sum_kappa A0[(p,q)] B0[s] (+ A1[(q,p)] B1[s]).
struct GemmJob {
  const double *a0;   // E + x1*nu*nu*KP  : row (p,q) at ((p*nu+q)*KP)
  const double *a1;   // E + x2*nu*nu*KP  : row (p,q) read as ((q*nu+p)*KP)
  const double *b0;   // F + (x2*no+x3)*NP*KP : row s at s*KP
  const double *b1;   // F + (x1*no+x3)*NP*KP
  double *out;        // X: row (p,q) at (p*nu+q)*NP
  int nhalves;        // 1 or 2
  // packed = 1: the A rows are not read from E but gathered from the packed
  // VVVO triangle (a0/a1 = the nu columns of occupied x1/x2, nutr doubles
  // each) and from t0/t1 = -T2 rows of x1/x2 ([(p,q)][l], no doubles each):
  // E[x][p][q][k] = packed[x*nu + p][tri(k, q)] for k < nu, t[(p*nu+q)*no + k-nu]
  // for nu <= k < nu+no (cct_layout.cu builds E from the same two sources).
  int packed;
  const double *t0, *t1;
};

// Shapes shared by the kernels of one system.
struct Dims {
  int no, nu;
  int64_t KP;   // padded contraction length of one half: round_up(nu+no, kKB)
  int BN;       // N tile of the W-build GEMM (choose_bn)
  int64_t NP;   // padded single-index length: round_up(nu, BN) (emulated: round_up(nu, EBN))
  int EBN;      // N tile of the emulated W-build (emulated plans), else 0
  int nb;       // reduction blocks per index: ceil(nu / kRB)
  int64_t ncta; // canonical block triples: nb(nb+1)(nb+2)/6
};

// Device-side description of one tuple for the reduction kernels.
struct TupleDev {
  const double *x[3];   // X buffers of the tuple's GEMM jobs
  int kind, i, j, k;
  double weight;        // 1 for i>j>k, 1/2 for degenerate tuples
  int blocked = 0;      // X in 8 x 8 x 8 blocks (emulated forward), else rows of NP
};
// X(p,q,s) of a blocked X buffer: block (p/8, q/8, s/8) of 512 doubles at
// ((p/8) nbk + q/8) NP/8 + s/8, element ((p%8) 8 + q%8) 8 + s%8, nbk = ceil(nu/8)
__host__ __device__ __forceinline__ int64_t xblock_base(int64_t P, int64_t Q, int64_t S, int nu, int64_t NP) {
  return ((P * ((nu + 7) / 8) + Q) * (NP / 8) + S) * 512;
}

// ----------------------------------------------------------------------------- INT8 emulation
// Digit count of the split-integer operands (7 bits each).  An automatic plan
// (emu_slices = 0) builds kEmuMaxSlices digits and runs the smallest count in
// [kEmuMinSlices, kEmuMaxSlices] whose calibrated E(T) error meets its target.
constexpr int kEmuMinSlices = 3, kEmuMaxSlices = 7;
constexpr int kEmuDigitCap = kEmuMaxSlices;  // most digits any operand holds
// N tile of the emulated W-build: the tensor memory holds S diagonal
// accumulators of N int32 columns (S N <= 512), and an MMA instruction costs
// about the same up to N ~ 80, so the widest N that pads nu least is used.
constexpr int kEmuBNChoices[] = {96, 80, 64};
inline int emu_choose_bn(int64_t nu, int slices) {
  int best = 64;
  int64_t best_np = (nu + 63) / 64 * 64;
  for (int bn : kEmuBNChoices) {
    if (slices * bn > 512) continue;
    const int64_t np = (nu + bn - 1) / bn * bn;
    if (np < best_np || (np == best_np && bn > best)) {
      best = bn;
      best_np = np;
    }
  }
  return best;
}

// One emulated W-build GEMM: half h multiplies E-digit rows (half 0: E[x1] rows
// (p,q); half 1: E^T[x2] rows (p,q) = E[x2] rows (q,p)) with F-digit rows of
// F[fyz[h] / no][fyz[h] % no].
struct EmuJob {
  int x1, x2;
  int fyz[2];
  double *out;
  int nhalves;
  int x3;  // the index both halves' F rows share: fyz[h] = (x2|x1) * no + x3
};

// Split-integer operands of one plan, stored pre-tiled in the tensor core's
// K-major no-swizzle shared-memory layout, so one pipeline stage (one 32-byte
// K chunk, every digit slice) is a single contiguous bulk copy per operand.
// A block holds one digit slice of one K chunk of one row tile: 8-row x 16-byte
// core matrices, row r / byte kb at (r/8)*256 + (kb/16)*128 + (r%8)*16 + kb%16.
constexpr int kEmuBM = 128;                      // rows per A tile
constexpr int kEmuKC = 32;                       // K bytes per chunk (one kind::i8 MMA)
constexpr int kEmuABlk = kEmuBM * kEmuKC;        // 4096 bytes
// B blocks hold EBN rows: EBN * kEmuKC bytes (2048, 2560 or 3072)
struct EmuOperands {
  int slices = kEmuMaxSlices;                // digit slices stored per K chunk
  int run_slices = kEmuMaxSlices;            // digits the W build runs (<= slices; the calibrated count)
  int ebn = 0;                               // N tile of F8 (rows per B block)
  int64_t NPe = 0;                           // rows per (y,z) in F8 and expF: NP rounded up to ebn
  int64_t KP8 = 0;                           // digit row length: round_up(nu+no, 32)
  int64_t tiles_m = 0;                       // ceil(nu^2 / 128) row tiles per occupied index
  int8_t *E8 = nullptr, *E8T = nullptr;      // [x][tile_m][kchunk][slice][4096]; E8T rows (q,p)
  int8_t *F8 = nullptr;                      // [y*no+z][tile_n][kchunk][slice][ebn*32], NPe / ebn tiles
  // Digit scales shared by both halves of a GEMM, so one set of diagonal
  // accumulators serves the whole contraction: expE[p*nu+q] (symmetric) is the
  // largest row exponent of E[x][p][q] and E[x][q][p] over all x; expF[z*NPe+n]
  // the largest of F[y][z][n] over all y.  expET and expRowF hold the per-row
  // exponents they are reduced from.
  int16_t *expE = nullptr, *expET = nullptr, *expF = nullptr, *expRowF = nullptr;
  // Per-tile digit counts (adaptive plans): tileExp holds the largest nonzero
  // row exponent of every A row tile [tiles_m], of every B column tile
  // [no][tiles_n] (z = x3 of the job), then the maxima of both sets.  A work
  // item (row tile, column tile) whose exponents sum `gap` below the top runs
  // S - floor(gap / 7) digits (at least 1): its dropped digit products stay
  // below the top tile's, so the bound on |X error| is the same everywhere.
  bool adaptive = false;
  // every item of the adaptive plan runs all S digits (no zero tile, every
  // pair of tile exponents within 7 of the top): the W build then skips the
  // per-item lookups, with the same result
  bool tiles_uniform = false;
  int *tileExp = nullptr;
  unsigned long long *slice_hist = nullptr;  // [kEmuMaxSlices + 1] work items per digit count
};

int emu_build_operands(const Dims &d, const double *E, const double *F, EmuOperands *o, cudaStream_t s);
// blocked: X in 8 x 8 x 8 blocks (xblock_base; NP a multiple of 8), else rows of NP
int launch_wbuild_emu(const EmuOperands &o, const Dims &d, const EmuJob *jobs_dev, int njobs, int *err,
                      cudaStream_t s, bool blocked = false);

// ----------------------------------------------------------------------------- launchers
// layout.cu
int launch_build_e(const Dims &d, const double *vvvo_packed, const double *t2, double *E, int x_begin,
                   int x_end, cudaStream_t s);
int launch_build_e_slice(const Dims &d, const double *packed_slice, const double *t2, double *E, int x,
                         cudaStream_t s);
// E[x] alone into slab (nu^2 rows of KP), from the whole packed VVVO
int launch_build_e_slab(const Dims &d, const double *vvvo_packed, const double *t2, double *slab, int x,
                        cudaStream_t s);
int launch_build_f(const Dims &d, const double *t2, const double *vm, double *F, cudaStream_t s);
int launch_check_inputs(const Dims &d, const double *eh, const double *ep, const double *t1, const double *t2,
                        const double *vm, const double *voe, const double *vvvo, int *flags, cudaStream_t s);

// wbuild_f64.cu
int launch_wbuild_f64(const Dims &d, const GemmJob *jobs_dev, int njobs, cudaStream_t s);

// reduce.cu
int launch_reduce(const Dims &d, const TupleDev &t, const double *eh, const double *ep, const double *voe,
                  const int16_t *cta_table, double *xpart, double *vpart, cudaStream_t s);
int launch_finalize(const Dims &d, const TupleDev &t, const double *xpart, const double *vpart,
                    double *etd_acc, double *v1_acc, cudaStream_t s);
int launch_ets(const Dims &d, const double *t1, const double *v1_acc, const double *etd_acc, double *out3,
               cudaStream_t s);

// adjoint.cu: device buffers of the backward pass (allocated at the first ccT_backward)
// backward: the dE GEMM runs once per group of kDEGroup consecutive tuples
// (their shared E slabs get the K of every tuple in one launch); kGXSets GX
// sets, two groups in flight
#ifndef CCT_DE_GROUP
#define CCT_DE_GROUP 2
#endif
constexpr int kDEGroup = CCT_DE_GROUP;
#ifndef CCT_GX_SETS
#define CCT_GX_SETS (2 * CCT_DE_GROUP)
#endif
constexpr int kGXSets = CCT_GX_SETS;
static_assert(kDEGroup >= 1 && kDEGroup <= 4, "dE GEMM groups of 1 to 4 tuples");
static_assert(kGXSets >= kDEGroup && kGXSets % kDEGroup == 0, "the dE GEMM takes the GX sets of whole groups");
struct AdjBuffers {
  bool ready = false;
  double *dE = nullptr, *dF = nullptr;                 // gradients of the GEMM operands E, F
  double *Wf = nullptr, *GW = nullptr;                 // dense nu^3: W, dE/dW (degenerate tuples)
  double *GX[kGXSets][3] = {};                         // dE/dX_g, nu^2 x NP each, kGXSets tuples in flight
  double *part = nullptr;                              // split-K partials of the dF GEMMs
  int64_t nsplit = 0, kchunk = 0;                      // splits of nu^2, rows per split
  double *Q = nullptr;                                 // 9 nu^2 VOE combinations of dE/dW
  double *vpart = nullptr;                             // per-a-chunk partial VOE gradients
  double *eps = nullptr;                               // per-tile sums of M over pairs of axes
  double *v1 = nullptr;                                // FP64 v1 of an emulated plan: 5 + nu*no
  double *g_eh = nullptr, *g_ep = nullptr, *g_t1 = nullptr, *g_t2 = nullptr, *g_vm = nullptr, *g_voe = nullptr,
         *g_vvvo = nullptr;                            // gradients in the input layouts
};
int adj_alloc(const Dims &d, AdjBuffers *b);
void adj_free(AdjBuffers *b);
int adj_configure(int device);
int adj_zero(const Dims &d, AdjBuffers *b, cudaStream_t s);
// Per tuple: the pointwise kernels (W assembly, dE/dW, dVOE, eps, dE/dX into GX
// set `set`), then the backward GEMMs reading that GX set.
int adj_tuple_pointwise(const Dims &d, const Tuple &t, double *const X[3], const double *eh, const double *ep,
                        const double *t1, const double *voe, AdjBuffers *b, int set, cudaStream_t s);
// dE GEMM of one tuple or of two consecutive tuples (GX sets sets[0..ntup-1])
// in one launch, on s; dF GEMM + its split-K sum of one tuple, on s.
int adj_tuple_gemm_e(const Dims &d, const Tuple *t, const int *sets, int ntup, const double *F, AdjBuffers *b,
                     cudaStream_t s);
int adj_tuple_gemm_f(const Dims &d, const Tuple &t, const double *E, AdjBuffers *b, int set, cudaStream_t s);
int adj_finish(const Dims &d, const double *v1, AdjBuffers *b, cudaStream_t s);
// W(a,b,c) of tuple t from its X buffers: into wc in C order (a slowest), then
// into wf in the reference's layout (a fastest).  Needs adj_configure.
int assemble_w_fortran(const Dims &d, const Tuple &t, double *const X[3], double *wc, double *wf, cudaStream_t s);

// cct_plan.cu: the dimensions and split-integer operands of an emulated plan,
// for the batched executor that runs many plans' W builds in grouped launches
const Dims &plan_dims(const ccT_plan *p);
const EmuOperands &plan_emu(const ccT_plan *p);

// peak.cu
double measure_fp64_peak(int device);
double measure_int8_peak(int device);

}  // namespace cct
