/*
 * libcc_b200 -- B200-native (sm_100a) CCSD(T) triples correction E(T).
 *
 * A drop-in for the GPU hooks and the whole-driver entry of libcc's triples.x
 * (ryanolson/libcc, src/triples-ijk).  Plain C ABI: pointers and sizes only.
 *
 * Array conventions (identical to the reference, Fortran column-major):
 *   eh(no), ep(nu), t1(no,nu), t2(nu,nu,no,no), vm(no,nu,no,no),
 *   voe(nu,nu,no,no), v1(nu,no), vvvo packed (nutr, nu*no) with
 *   nutr = nu*(nu+1)/2 and column x*nu+c holding the a>=b triangle of (ab|c x).
 *
 * Two groups of entry points:
 *   1. Fortran-callable legacy hooks (trailing underscore, every argument by
 *      reference, 8-byte integers as under -sdefault64, 1-based occupied
 *      indices).  Like the reference they return nothing and stop the program
 *      with a message on error.
 *   2. The status-returning ccT_* API (0 = success, see ccT_status).
 */
#ifndef LIBCC_B200_H
#define LIBCC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum {
    CCT_OK = 0,
    CCT_ERR_INVALID = 1,     /* bad argument: shape, index, null pointer        */
    CCT_ERR_CUDA = 2,        /* a CUDA runtime call failed                      */
    CCT_ERR_NOMEM = 3,       /* device allocation failed                        */
    CCT_ERR_NONFINITE = 4,   /* input or result holds NaN/Inf                   */
    CCT_ERR_DENOMINATOR = 5, /* some e_i+e_j+e_k-e_a-e_b-e_c >= 0               */
    CCT_ERR_STATE = 6,       /* call out of order (e.g. forward before inputs)  */
    CCT_ERR_TIMEOUT = 7,     /* a bounded device-side wait ran out              */
    CCT_ERR_UNSUPPORTED = 8  /* option not available on this device / build     */
} ccT_status;

typedef enum {
    CCT_PREC_FP64 = 0,       /* native FP64 DMMA contractions                   */
    CCT_PREC_INT8_EMU = 1    /* split-integer emulated FP64 on INT8 tensor cores */
} ccT_precision;

typedef enum { CCT_MEM_HOST = 0, CCT_MEM_DEVICE = 1 } ccT_memory;

typedef struct {
    int32_t precision;       /* ccT_precision                                    */
    int32_t device;          /* CUDA device ordinal                              */
    int32_t check_inputs;    /* 1: reject NaN/Inf inputs and D >= 0 (default 1)  */
    int32_t emu_slices;      /* INT8 emulation: 0 = automatic (default): the plan
                                stores 7 digits and ccT_set_inputs picks the
                                smallest count, 3..7, whose calibrated |dE(T)|
                                meets the target below, each tile then taking
                                at most that many; 3..7 = that many digits on
                                every tile                                      */
    double emu_tol;          /* automatic digits: target |dE(T)| in Eh against the
                                FP64 form (0 = default 1e-8)                    */
    double emu_tol_rel;      /* automatic digits: relative floor; the target is
                                max(emu_tol, emu_tol_rel |E(T)|) (0 = default
                                2e-14, the FP64 evaluation-order round-off)     */
    int32_t vvvo_mode;       /* FP64 plans: CCT_VVVO_AUTO (default), _EXPANDED or
                                _PACKED (see below)                             */
    int32_t keep_w;          /* FP64 plans with expanded VVVO: 1 = ccT_forward
                                keeps every tuple's W-build output (3 nu^2 NP
                                doubles a tuple) on the device when that fits
                                in the free memory, and ccT_backward reads it
                                instead of rebuilding W (same results); 0
                                (default) = the backward rebuilds W         */
} ccT_options;

/* How an FP64 plan holds VVVO.  EXPANDED: ccT_set_inputs expands the packed
 * triangle once into the W build's row operand E (no*nu^2*round_up(nu+no,16)
 * doubles: 6.9 GB at no=24, nu=320).  PACKED: the packed triangle (about half
 * of that) stays resident and the W build gathers each operand row from it
 * while staging a tile, the reference's "transfer NUTR elements at a time
 * which blow up to NU2" (CUDA_OUTLINE.txt:55-60) done inside the tile loader;
 * the results are bitwise those of EXPANDED.  PACKED plans have no backward
 * (the adjoint writes dE of E's size).  AUTO: PACKED when E would take more
 * than half of the free device memory, else EXPANDED.  Emulated plans and the
 * legacy hooks are always EXPANDED. */
enum { CCT_VVVO_AUTO = 0, CCT_VVVO_EXPANDED = 1, CCT_VVVO_PACKED = 2 };

typedef struct ccT_plan ccT_plan;

/* Fill *opt with defaults (FP64, device 0, input checks on, automatic digits
 * with a 1e-8 Eh target). */
void ccT_options_default(ccT_options *opt);

/* Plan for one system of no occupied and nu virtual orbitals.  Allocates the
 * device-resident HBM buffers that replace the DDI arrays. */
int ccT_plan_create(ccT_plan **plan, int64_t no, int64_t nu, const ccT_options *opt);

/* Load the inputs (reference layouts).  mem = CCT_MEM_HOST copies from host
 * memory (pinned memory copies fastest), CCT_MEM_DEVICE reads device pointers
 * already in HBM.  Ordering of device inputs: on the plan's own stream the call
 * first waits for all work on the device (cudaDeviceSynchronize), so inputs
 * written by any stream are complete; after ccT_set_stream(plan, s) the reads
 * are ordered after the work already queued on s, and inputs written on other
 * streams must be complete or ordered before s by the caller.  From host
 * memory the packed VVVO passes through a transient device buffer of its own
 * size, allocated and freed inside the call.  The call returns once the GEMM
 * operands are built; for an automatic emulated plan it also calibrates the
 * digit count (ccT_emu_digits).  Replaces program.F90:195-223 (restart read)
 * plus the DDI put/bcast of T2/VM/VOE/VVVO. */
int ccT_set_inputs(ccT_plan *plan, const double *eh, const double *ep, const double *t1,
                   const double *t2, const double *vm, const double *voe,
                   const double *vvvo_packed, int32_t mem);

/* Number of tuples with work: C(no,3) i>j>k tuples, then no(no-1)/2 (i,j,j)
 * and no(no-1)/2 (i,i,j) tuples (triples.F90:51-53). */
int64_t ccT_num_tuples(int64_t no);

/* Run tuples [begin, end) of the global tuple list (i>j>k in DDCC_T_TASK order,
 * then for each i and j<i the (i,j,j) and (i,i,j) tuples), accumulate
 * etd and v1, and return ets = 2 sum_{i,a} t1(i,a) v1(a,i), etd, and (if
 * v1_out != NULL) v1(nu,no) for this range.  A full range reproduces
 * cc_triples (triples.F90:1-333).  A partial range gives a shard whose
 * ets/etd/v1 sum linearly with the other shards. */
int ccT_forward(ccT_plan *plan, int64_t begin, int64_t end, double *ets, double *etd, double *v1_out);

/* Gradient of E(T) = ets + etd of the tuple range of the preceding ccT_forward
 * (the saved context: same plan, same inputs, same [begin, end)) with respect
 * to every input, written in the input layouts: d_eh (no), d_ep (nu), d_t1
 * (no,nu), d_t2 (nu,nu,no,no), d_vm (no,nu,no,no), d_voe (nu,nu,no,no) and
 * d_vvvo (the packed (nutr, nu*no) layout of ccT_set_inputs).  Together this
 * is the (T) contribution to the CCSD(T) Lagrangian.  W is recomputed per
 * tuple in FP64 whatever the plan's precision (or, with options.keep_w, read
 * from what the forward kept; otherwise nothing of size nu^3 is kept across
 * tuples).  mem says whether the output pointers are host or device
 * memory; any output pointer may be NULL to skip it.  No reference
 * counterpart: the reference computes no gradient.  Returns CCT_ERR_STATE
 * when no ccT_forward over [begin, end) precedes it. */
int ccT_backward(ccT_plan *plan, int64_t begin, int64_t end, double *d_eh, double *d_ep, double *d_t1,
                 double *d_t2, double *d_vm, double *d_voe, double *d_vvvo, int32_t mem);

/* Milliseconds of device time the last ccT_backward spent (CUDA events). */
double ccT_last_backward_ms(const ccT_plan *plan);

/* Tuples whose W-build output the last ccT_forward kept for the backward
 * (options.keep_w): end - begin of its range, or 0 when it kept none (option
 * off, an emulated or packed plan, or not enough free device memory). */
int64_t ccT_kept_tuples(const ccT_plan *plan);

/* Emulated plans: hist[s] = work items (128-row x N-column W tiles) the last
 * ccT_forward ran with s digits per operand, s = 0..n-1.  With emu_slices = 0
 * the calibrated count S is the maximum and every tile takes the digits its
 * exponents need (a tile whose largest row scales sum g bits below the
 * system's top runs max(1, S - floor(g/7)) digits), so the bound on the
 * error of any W entry is the top tile's.  FP64 plans: all zero.  No
 * reference counterpart (the reference has no emulation). */
int ccT_emu_slice_histogram(ccT_plan *plan, int64_t *hist, int32_t n);

/* Emulated plans: the digit count the W build runs (*digits), the calibrated
 * bound on |dE(T)| against the FP64 form at that count (*est_err, Eh) and the
 * target it was picked for (*target, Eh).  Calibration (automatic plans, in
 * ccT_set_inputs): up to five tuples spread over the tuple list are evaluated
 * with the FP64 W build and with every digit count 3..7; the estimate for a
 * count is 2 x (largest per-tuple |dE| / tuple weight) x (sum of the weights of
 * all tuples), i.e. every tuple's error at the worst sampled size and with
 * the same sign.  Fixed-count plans report their count and zeros.  FP64 plans:
 * CCT_ERR_STATE.  No reference counterpart. */
int ccT_emu_digits(const ccT_plan *plan, int32_t *digits, double *est_err, double *target);

/* W_abc of one tuple of the global list as this plan's W build forms it (FP64,
 * or the emulated digits at the plan's count), after the degenerate tuples'
 * symmetrisation and with W_aaa = 0: the V3 array of ijk_tuple_formv3 /
 * ijj_tuple_formv3+SYMT311 / iij_tuple_formv3+SYMT311 followed by ZEROT3
 * (src/triples-abc/ijk_tuple.f90:1-53, ijj_tuple.f90, iij_tuple.f90,
 * ddcc_aux.f:84-94, 217-253), in the reference's layout w(a,b,c) at
 * a + nu*(b + nu*c).  w holds nu^3 doubles; mem says host or device.  A
 * diagnostic (it allocates a transient nu^3 buffer) for checking W against
 * the reference element by element. */
int ccT_tuple_w(ccT_plan *plan, int64_t tuple, double *w, int32_t mem);

/* ---------------------------------------------------------------- batches
 * Many independent systems of uneven (no, nu) evaluated together.  Every tuple
 * of every system is cut into work items (W-build tiles, reduction blocks) that
 * run either in one persistent kernel fed by a device-side work queue (mode 0)
 * or as grouped launches per tuple group on two streams (mode 1); either is
 * captured in a CUDA graph, and ccT_batch_tune picks the faster.  A batch
 * created with opt->precision = CCT_PREC_INT8_EMU also has mode 2 (its
 * default): mode 1 with the emulated W build, each system's digit count
 * calibrated to opt->emu_tol / emu_tol_rel as an emulated plan's (or fixed by
 * opt->emu_slices), and the tuner times all three executors.  No reference
 * counterpart (the reference runs one system per triples.x process); per
 * system the results equal a single-system plan's (of the same precision and
 * digit options) bitwise. */
typedef struct ccT_batch ccT_batch;

int ccT_batch_create(ccT_batch **batch, int64_t nsys, const int64_t *no, const int64_t *nu,
                     const ccT_options *opt);
/* Inputs of system s, same layouts and meaning as ccT_set_inputs. */
int ccT_batch_set_inputs(ccT_batch *batch, int64_t s, const double *eh, const double *ep, const double *t1,
                         const double *t2, const double *vm, const double *voe, const double *vvvo_packed,
                         int32_t mem);
/* E(T) of every system: ets[s], etd[s] (arrays of nsys doubles, or NULL). */
int ccT_batch_forward(ccT_batch *batch, double *ets, double *etd);
/* v1(nu, no) of system s from the last ccT_batch_forward. */
int ccT_batch_v1(ccT_batch *batch, int64_t s, double *v1_out);
/* Fix the schedule: executor mode (0: one persistent kernel taking every work
 * item from a device queue; 1: per tuple group, one launch of W-build tiles and
 * one of reduction blocks on two streams; 2: as 1 with one emulated W-build
 * launch per system in the group, CCT_PREC_INT8_EMU batches only), W-build N
 * tile bn (32, 48 or 64, or 0 = the least-padding tile per system, modes 1
 * and 2; mode 2 takes 0 only),
 * tuple order (0: by cost, largest first; 1: system by system) and X scratch
 * bytes per tuple group. */
int ccT_batch_configure(ccT_batch *batch, int32_t mode, int32_t bn, int32_t order, int64_t group_bytes);
/* Autotune: time every (mode, bn, order) candidate on the loaded inputs, keep
 * the fastest and report it (outputs may be NULL). */
int ccT_batch_tune(ccT_batch *batch, int32_t *best_mode, int32_t *best_bn, int32_t *best_order,
                   double *best_ms);
/* Testing hook of the persistent executor (mode 0): from the next forward on,
 * the reduction blocks of the tuple at position `tuple` of the queue order
 * wait for one W-build tile more than that tuple has, so their bounded
 * counter wait runs out after spin_limit polls (0 = the default limit); the
 * kernel then finishes its queue and the forward returns CCT_ERR_TIMEOUT with
 * the context intact.  tuple < 0 removes the stall.  No reference
 * counterpart (the reference's only failure handling is stop,
 * program.F90:221-222). */
int ccT_batch_debug_stall(ccT_batch *batch, int64_t tuple, int64_t spin_limit);
/* Device milliseconds of the last batch forward (CUDA events around the graph). */
double ccT_batch_last_ms(const ccT_batch *batch);
/* Work items (W-build tiles + reduction blocks) in the current schedule. */
int64_t ccT_batch_work_items(const ccT_batch *batch);
/* Digit count of system s in the emulated executor (after its schedule was
 * built: a mode 2 forward or tune).  CCT_ERR_STATE before. */
int ccT_batch_emu_digits(const ccT_batch *batch, int64_t s, int32_t *digits);
int ccT_batch_destroy(ccT_batch *batch);

/* Launch the plan's kernels on a caller-provided CUDA stream (a cudaStream_t
 * passed as void*); NULL restores the plan's own stream. */
int ccT_set_stream(ccT_plan *plan, void *cuda_stream);

/* Time `reps` back-to-back launches of the W-build contraction of one tuple
 * with CUDA events on the plan's stream; *ms_per_launch gets the mean. */
int ccT_time_wbuild(ccT_plan *plan, int64_t tuple, int32_t reps, double *ms_per_launch);

/* Per-kernel timing of later ccT_forward calls: on != 0 records a CUDA event
 * pair around every launch of each kernel class on the plan's stream. */
int ccT_set_profiling(ccT_plan *plan, int32_t on);

/* Kernel classes for ccT_last_kernel_ms. */
enum { CCT_KERNEL_WBUILD = 0, CCT_KERNEL_REDUCE = 1 };

/* Summed device milliseconds and launch count of one kernel class in the last
 * profiled ccT_forward. */
int ccT_last_kernel_ms(const ccT_plan *plan, int32_t kernel_class, double *total_ms, int64_t *launches);

/* Milliseconds of device time the last ccT_forward spent, measured by CUDA
 * events around its kernels (excludes input upload). */
double ccT_last_forward_ms(const ccT_plan *plan);

/* Kernel launches issued by the last ccT_forward. */
int64_t ccT_last_forward_launches(const ccT_plan *plan);

int ccT_plan_destroy(ccT_plan *plan);

/* Message for a status code, or the last error recorded on this thread. */
const char *ccT_status_string(int status);
const char *ccT_last_error(void);

/* Measured FP64 mma.sync throughput of this device in TFLOP/s (a short
 * microbenchmark; the denominator of the FP64 roofline). */
double ccT_measure_fp64_peak(int32_t device);

/* Measured INT8 tensor-pipe throughput (tcgen05.mma kind::i8, operands
 * resident in shared memory) in tera-ops/s: the denominator of the emulated
 * form's roofline. */
double ccT_measure_int8_peak(int32_t device);

/* ------------------------------------------------------------------ allocation-free reduction
 * No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory: codes that reserve one arena for all their GPU
 * buffers up front, and drivers that must not risk the implicit device
 * synchronisation of cudaMalloc/cudaFree in the middle of their own
 * asynchronous work.
 *
 * Adds the E[4] and E[5] contributions of one tuple (i,j,k), 0-based with
 * i >= j >= k not all equal (weight 1/2 when two are equal), computed from a
 * W_abc the caller already holds on the device (w(a,b,c) at a + nu*(b + nu*c);
 * w(a,a,a) is treated as 0), into the caller's device accumulators:
 * etd_acc[0..1] (sum and compensation term; etd = etd_acc[0] + etd_acc[1]) and
 * v1_acc(nu,no).  eh, ep, voe are device arrays in the reference layouts.
 * Kernels run on cuda_stream (a cudaStream_t as void*, NULL = default stream).
 *
 * It allocates nothing: its per-block partial sums live in one fixed array in
 * the library's device memory, sized for nu <= CCT_NOALLOC_MAX_NU (6.4 MiB,
 * held by every GPU that loads the library until the process exits).  Larger
 * nu is rejected with CCT_ERR_INVALID.  The first call on a device looks up
 * that array's device address (cudaGetSymbolAddress) with the device current,
 * so make the first call before any stream capture.  The looked-up address
 * is kept for the life of the process: do not call the entry point again on
 * a device after cudaDeviceReset (or any teardown of its primary context).
 * All calls share the array: calls whose kernels overlap on the GPU (different
 * streams with no ordering between them) race; calls ordered on one stream
 * are safe. */
#define CCT_NOALLOC_MAX_NU 320
int ccT_reduce_w_noalloc(int64_t no, int64_t nu, int64_t i, int64_t j, int64_t k, const double *w,
                         const double *eh, const double *ep, const double *voe, double *etd_acc,
                         double *v1_acc, void *cuda_stream);

/* ------------------------------------------------------------------ CCSD T1-dressing terms
 * The two routines of the reference's OpenACC CCSD port that contract the
 * same expanded VVVO slices as the triples, for one process holding every
 * occupied index (nothing in the reference tree calls them; they are the CCSD
 * step before (T)).  Arrays are Fortran column-major; mem says whether every
 * pointer is host or device memory; the calls return when the results are in
 * place.  They keep a device workspace between calls (the same buffers every
 * call of a shape, so repeated calls allocate nothing) and are serialised
 * against each other; ccT_ccsd_release_workspace frees it.
 *
 * ccT_ccsd_terms_29_31 replaces terms_29_30_31 (src/triples-ijk/ccsd_acc.f:1-60):
 *   t2(i,b,c,j) += sum_a o1(i,a) [ (c a|b j) - sum_k o1(k,c) vl(k,a,b,j)
 *                                  - sum_k o1(k,b) vr(c,k,a,j) ]
 * with o1 (no,nu), t2 (no,nu,nu,no), vl the DDI array D_VL read as
 * (no,nu,nu,no), vr D_VR_IBT read as (nu,no,nu,no), vvvo packed as for
 * ccT_set_inputs.  (The routine's TRANMD of its scratch buffer at line 33 has
 * no effect on the result and is not reproduced.) */
int ccT_ccsd_terms_29_31(int64_t no, int64_t nu, const double *o1, double *t2, const double *vl,
                         const double *vr, const double *vvvo, int32_t mem);

/* ccT_ccsd_terms_32_35 replaces terms_32_33_34_35 (ccsd_acc.f:64-160) and leaves
 * its arrays as that routine does: t2 (nou x nou, nou = no nu) transposed;
 * o2 (no,nu,nu,no) permuted to o2(x,y,k,l) = o2_in(k,x,y,l), i.e. (nu,nu,no,no);
 * rl (nou x nou) = the transpose of RL(i,y,z,j) = sum_x o1(i,x) (x y|z j); and
 * vm (no,no,no,nu) replaced by vm(x,y,z,a) = vm_in(y,x,z,a)
 * + sum_{p,q} o2_in(x,p,q,z) (a q|p y), the contraction on the FP64 tensor
 * cores.  The reference's update loop (lines 136-144) offsets that sum by one
 * element within each (j, a) block; this adds it where the surrounding
 * permutations put it. */
int ccT_ccsd_terms_32_35(int64_t no, int64_t nu, const double *o1, double *o2, double *t2, double *vm,
                         double *rl, const double *vvvo, int32_t mem);
/* Frees the device workspace the two CCSD-term entry points keep. */
int ccT_ccsd_release_workspace(void);

/* ------------------------------------------------------------------ legacy hooks
 * ijk_gpu_init_    replaces the call at src/triples-ijk/triples_cpu.F90:363
 * ijk_gpu_driver_  replaces src/triples-ijk/ddcc_t_ijk_big_cuda.f:12-14
 * ijk_gpu_finalize_ replaces the call at src/triples-ijk/triples_cpu.F90:497
 * The driver hook receives the packed VVVO columns of i, j and k exactly as
 * triples_cpu.F90:428-450 fetches them (nutr*nu doubles each); it expands and
 * b<->c-swaps them on the device.  Tuple contributions accumulate on the device
 * and are added into the host etd and v1 (the v1 pointer given at init) by
 * ijk_gpu_finalize_. */
void ijk_gpu_init_(const int64_t *no, const int64_t *nu, const double *eh, const double *ep,
                   double *v1, const double *t2, const double *vm, const double *voe);
void ijk_gpu_driver_(const int64_t *nu, const int64_t *no, const int64_t *i, const int64_t *j,
                     const int64_t *k, const double *ve_i, const double *ve_j, const double *ve_k,
                     double *t1, const double *eh, const double *ep, double *etd);
void ijk_gpu_finalize_(const int64_t *no, const int64_t *nu, double *etd);

/* Whole (T) driver with the packed VVVO passed explicitly instead of a DDI
 * handle: the single-GPU form of cc_triples_acc (src/triples-ijk/triples.F90:1)
 * and cc_triples (src/triples-abc/triples.f90:193).  v1 (nu,no) is
 * overwritten; ets and etd are returned as gms_ets/gms_etd are. */
void cc_triples_b200_(const int64_t *no, const int64_t *nu, const double *eh, const double *ep,
                      double *v1, const double *t1, const double *t2, const double *vm,
                      const double *voe, const double *vvvo, double *ets, double *etd);

#ifdef __cplusplus
}
#endif
#endif /* LIBCC_B200_H */
