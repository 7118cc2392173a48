// Per-tuple E[4] (etd) and E[5] v1 reduction.
//
// Reference: t1wt3_ijk (src/triples-ijk/t1wt3.f90:18-109), T3SQUA_SMP
// (src/triples-abc/t3squa.f:1-113), ADT3DEN + DRT1WT3IJK/IJ/JK
// (src/triples-abc/ddcc_aux.f:97-238).  Per tuple (i,j,k) with W_aaa = 0:
//
//   x3 = sum_abc W_abc (8 W_abc - 4(W_acb + W_cba + W_bac) + 2(W_bca + W_cab)) / D_abc
//   v1(a,i) += sum_bc [Z1 VOE(b,c,j,k) + Z2 VOE(b,c,k,j)] / D_abc      (Z1..Z6 as in
//   v1(a,j) += sum_bc [Z3 VOE(b,c,i,k) + Z5 VOE(b,c,k,i)] / D_abc       t1wt3.f90:80-85,
//   v1(a,k) += sum_bc [Z4 VOE(b,c,i,j) + Z6 VOE(b,c,j,i)] / D_abc       summed over all b)
//   etd += w x3,  v1 += w (...),  w = 1 (i>j>k) or 1/2 (i=j or j=k)
//
// The twelve terms arrive as the three GEMM outputs X_g (cct_wbuild_f64.cu),
// so W at all six index permutations is assembled on chip: one CTA owns an
// unordered triple of 8-wide index blocks {A<=B<=C}, assembles W on every
// distinct ordered block of its orbit in shared memory, and evaluates every
// element of those blocks once.  Per-CTA partials are summed by
// finalize_kernel in a fixed order, so results are bitwise reproducible.
#include "cct_internal.cuh"
#include "cct_reduce_block.cuh"

namespace cct {
namespace {

using namespace red;

template <int KIND, bool BLOCKED>
__global__ void __launch_bounds__(RT, 4) reduce_kernel(int nu, int no, int64_t NP, TupleDev t,
                                                      const double *__restrict__ eh, const double *__restrict__ ep,
                                                      const double *__restrict__ voe,
                                                      const int16_t *__restrict__ table, double *__restrict__ xpart,
                                                      double *__restrict__ vpart) {
  extern __shared__ __align__(16) double dyn_smem[];
  const int64_t cta = blockIdx.x;
  reduce_block<KIND, false, BLOCKED>(nu, no, NP, t, eh, ep, voe, table[3 * cta], table[3 * cta + 1], table[3 * cta + 2],
                     xpart + cta, vpart, dyn_smem);
}

// etd_acc[0..1]: Neumaier (sum, compensation); v1_acc(nu, no).
// Block 0 sums the per-CTA x3 partials (thread t takes partials t, t+256, ...
// in order, then a tree over the 256 threads); every other block owns kFinA
// virtual indices a, one warp per (a, column), each summing the column's v1
// partials over all block triples containing a (lane-strided, then a shuffle
// tree), and one thread per a adds the three column sums to v1 in the order
// i, j, k.  The loads of a thread's partials are issued eight at a time ahead
// of its (ordered) adds.
constexpr int kFinA = 8;
constexpr int kFinThreads = 32 * 3 * kFinA;
__global__ void __launch_bounds__(kFinThreads) finalize_kernel(int nu, int nb, int64_t ncta, TupleDev t,
                                                               const double *__restrict__ xpart,
                                                               const double *__restrict__ vpart,
                                                               double *__restrict__ etd_acc,
                                                               double *__restrict__ v1_acc) {
  constexpr int U = 8;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  if (blockIdx.x == 0) {
    __shared__ double red[256];
    if (tid < 256) {
      double s = 0.0;
      for (int64_t c0 = tid; c0 < ncta; c0 += 256 * U) {
        double v[U];
#pragma unroll
        for (int u = 0; u < U; u++) v[u] = c0 + 256 * u < ncta ? xpart[c0 + 256 * u] : 0.0;
#pragma unroll
        for (int u = 0; u < U; u++)
          if (c0 + 256 * u < ncta) s += v[u];
      }
      red[tid] = s;
    }
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
      if (tid < st) red[tid] += red[tid + st];
      __syncthreads();
    }
    if (tid == 0) {
      const double v = t.weight * red[0];
      const double sum = etd_acc[0];
      const double nsum = sum + v;
      const double comp = fabs(sum) >= fabs(v) ? (sum - nsum) + v : (v - nsum) + sum;
      etd_acc[0] = nsum;
      etd_acc[1] += comp;
    }
    return;
  }
  __shared__ double sc[kFinA][3];
  const int warp = tid >> 5, la8 = warp / 3, col = warp - 3 * (warp / 3);
  const int a = (blockIdx.x - 1) * kFinA + la8;
  if (a < nu) {
    const int X = a / RB, la = a - (a / RB) * RB;
    const int64_t npairs = (int64_t)nb * (nb + 1) / 2;
    const double *slab = vpart + (((int64_t)X * RB + la) * 3 + col) * npairs;
    double v = 0.0;
    for (int64_t q0 = lane; q0 < npairs; q0 += 32 * U) {
      double x[U];
#pragma unroll
      for (int u = 0; u < U; u++) x[u] = q0 + 32 * u < npairs ? slab[q0 + 32 * u] : 0.0;
#pragma unroll
      for (int u = 0; u < U; u++)
        if (q0 + 32 * u < npairs) v += x[u];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) sc[la8][col] = v;
  }
  __syncthreads();
  if (tid < kFinA) {
    const int a2 = (blockIdx.x - 1) * kFinA + tid;
    if (a2 < nu) {
      v1_acc[a2 + (int64_t)nu * t.i] += t.weight * sc[tid][0];
      v1_acc[a2 + (int64_t)nu * t.j] += t.weight * sc[tid][1];
      v1_acc[a2 + (int64_t)nu * t.k] += t.weight * sc[tid][2];
    }
  }
}

// out3 = {ets, etd, ets+etd}; ets = 2 sum_{i,a} t1(i,a) v1(a,i) (triples.F90:311-316)
__global__ void ets_kernel(int no, int nu, const double *__restrict__ t1, const double *__restrict__ v1,
                           const double *__restrict__ etd_acc, double *__restrict__ out3) {
  __shared__ double red[256];
  const int tid = threadIdx.x;
  double s = 0.0;
  const int64_t n = (int64_t)no * nu;
  for (int64_t e = tid; e < n; e += 256) {
    const int64_t i = e / nu, a = e - (e / nu) * nu;
    s += t1[i + (int64_t)no * a] * v1[a + (int64_t)nu * i];
  }
  red[tid] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (tid < st) red[tid] += red[tid + st];
    __syncthreads();
  }
  if (tid == 0) {
    const double ets = 2.0 * red[0];
    const double etd = etd_acc[0] + etd_acc[1];
    out3[0] = ets;
    out3[1] = etd;
    out3[2] = ets + etd;
  }
}

}  // namespace

template <int KIND, bool BLOCKED>
int launch_reduce_kind(const Dims &d, const TupleDev &t, const double *eh, const double *ep, const double *voe,
                       const int16_t *cta_table, double *xpart, double *vpart, cudaStream_t s) {
  constexpr int smem = REDUCE_SMEM;
  static int configured_device = -1;
  int dev = 0;
  CCT_CUDA(cudaGetDevice(&dev));
  if (configured_device != dev) {
    CCT_CUDA(cudaFuncSetAttribute(reduce_kernel<KIND, BLOCKED>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CCT_CUDA(cudaFuncSetAttribute(reduce_kernel<KIND, BLOCKED>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared));
    configured_device = dev;
  }
  reduce_kernel<KIND, BLOCKED>
      <<<(unsigned)d.ncta, RT, smem, s>>>(d.nu, d.no, d.NP, t, eh, ep, voe, cta_table, xpart, vpart);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

template <bool BLOCKED>
int launch_reduce_layout(const Dims &d, const TupleDev &t, const double *eh, const double *ep, const double *voe,
                         const int16_t *cta_table, double *xpart, double *vpart, cudaStream_t s) {
  if (t.kind == kIJK) return launch_reduce_kind<kIJK, BLOCKED>(d, t, eh, ep, voe, cta_table, xpart, vpart, s);
  if (t.kind == kIJJ) return launch_reduce_kind<kIJJ, BLOCKED>(d, t, eh, ep, voe, cta_table, xpart, vpart, s);
  return launch_reduce_kind<kIIJ, BLOCKED>(d, t, eh, ep, voe, cta_table, xpart, vpart, s);
}

int launch_reduce(const Dims &d, const TupleDev &t, const double *eh, const double *ep, const double *voe,
                  const int16_t *cta_table, double *xpart, double *vpart, cudaStream_t s) {
  if (t.blocked) {
    if (d.NP % RB) {
      set_error("blocked X needs NP a multiple of 8 (NP = " + std::to_string(d.NP) + ")");
      return CCT_ERR_INVALID;
    }
    return launch_reduce_layout<true>(d, t, eh, ep, voe, cta_table, xpart, vpart, s);
  }
  return launch_reduce_layout<false>(d, t, eh, ep, voe, cta_table, xpart, vpart, s);
}

int launch_finalize(const Dims &d, const TupleDev &t, const double *xpart, const double *vpart, double *etd_acc,
                    double *v1_acc, cudaStream_t s) {
  const int vblocks = (d.nu + kFinA - 1) / kFinA;  // one warp per (virtual index, column)
  finalize_kernel<<<1 + vblocks, kFinThreads, 0, s>>>(d.nu, d.nb, d.ncta, t, xpart, vpart, etd_acc, v1_acc);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

int launch_ets(const Dims &d, const double *t1, const double *v1_acc, const double *etd_acc, double *out3,
               cudaStream_t s) {
  ets_kernel<<<1, 256, 0, s>>>(d.no, d.nu, t1, v1_acc, etd_acc, out3);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

}  // namespace cct
