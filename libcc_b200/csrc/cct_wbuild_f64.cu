// W_abc build on the FP64 tensor pipe (mma.sync .f64, sm_100a).
//
// The reference forms W for one tuple with twelve DGEMMs and four in-place
// nu^3 transposes (ijk_tuple.f90:47-87, ijk_tuple_acc.f90:59-96).  Grouping
// the twelve terms by which index pair comes from the (p,q)-row operand gives
// three GEMMs per tuple, each with a contraction of 2(nu+no):
//
//   X_g(p,q,s) = sum_k E[x1][p][q][k] F[x2][x3][s][k] + sum_k E[x2][q][p][k] F[x1][x3][s][k]
//
// (E, F as built in cct_layout.cu) and W(a,b,c) = X_0(a,b,c) + X_1(a,c,b) + X_2(b,c,a)
// for (x1,x2,x3) = (i,j,k), (i,k,j), (j,k,i).  The trant3 permutations thus
// disappear into the row addressing of the A operand (row (q,p) for the second
// half) and into the reduction's reads; nothing is transposed in HBM.
//
// Kernel: one CTA per 128 x BN output tile of one job (BN in {32..64}, chosen
// per system so nu needs little padding); 4 warps stacked along M, each
// 32 x BN; mma.sync.m16n8k4.f64; a 3-stage cp.async ring of 128x16 / BNx16
// tiles with 16-byte-aligned rows padded to 20 doubles (conflict-free
// fragment loads); two CTAs per SM.
#include "cct_internal.cuh"

namespace cct {
namespace {

constexpr int BM = 128, BK = kKB;
constexpr int WM = 32;
constexpr int NWARP = BM / WM;
constexpr int NT = NWARP * 32;
constexpr int STAGES = 3;
constexpr int LDS = BK + 4;  // padded smem row (doubles)
constexpr int MF = WM / 16;

template <int BN>
constexpr int smem_bytes() {
  return STAGES * (BM + BN) * LDS * 8 + BM * 2 * 4;
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma_16x8x4(double *d, double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

template <int BN>
__global__ void __launch_bounds__(NT, 2) wbuild_f64_kernel(const GemmJob *__restrict__ jobs, int nu, int64_t KP,
                                                           int64_t NP, int tiles_n) {
  constexpr int NF = BN / 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *As = reinterpret_cast<double *>(smem_raw);
  double *Bs = As + STAGES * BM * LDS;
  int *rowoff = reinterpret_cast<int *>(Bs + STAGES * BN * LDS);  // [2][BM] row index into E (or -1)

  const GemmJob job = jobs[blockIdx.y];
  const int tile_m = blockIdx.x / tiles_n, tile_n = blockIdx.x - tile_m * tiles_n;
  const int64_t M = (int64_t)nu * nu;
  const int64_t m0 = (int64_t)tile_m * BM;
  const int n0 = tile_n * BN;
  const int tid = threadIdx.x;

  for (int r = tid; r < BM; r += NT) {
    const int64_t m = m0 + r;
    if (m < M) {
      const int p = (int)(m / nu), q = (int)(m - (int64_t)(m / nu) * nu);
      rowoff[r] = p * nu + q;
      rowoff[BM + r] = q * nu + p;
    } else {
      rowoff[r] = -1;
      rowoff[BM + r] = -1;
    }
  }
  __syncthreads();

  const int ktiles_half = (int)(KP / BK);
  const int ktiles = ktiles_half * job.nhalves;

  auto load_stage = [&](int stage, int kt) {
    const int h = kt >= ktiles_half;
    const int64_t k0 = (int64_t)(kt - h * ktiles_half) * BK;
    const double *abase = h ? job.a1 : job.a0;
    const double *bbase = h ? job.b1 : job.b0;
    double *as = As + stage * BM * LDS;
    double *bs = Bs + stage * BN * LDS;
    const int chunk = tid & 7;  // 8 x 16 B per 16-double row
#pragma unroll
    for (int rr = tid >> 3; rr < BM; rr += NT / 8) {
      const int ro = rowoff[h * BM + rr];
      const double *src = abase + (ro < 0 ? 0 : (int64_t)ro * KP) + k0 + chunk * 2;
      cp_async16(as + rr * LDS + chunk * 2, src, ro < 0 ? 0 : 16);
    }
#pragma unroll
    for (int rr = tid >> 3; rr < BN; rr += NT / 8) {
      const double *src = bbase + (int64_t)(n0 + rr) * KP + k0 + chunk * 2;
      cp_async16(bs + rr * LDS + chunk * 2, src, 16);
    }
  };

  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;

  double acc[MF][NF][4];
#pragma unroll
  for (int i = 0; i < MF; i++)
#pragma unroll
    for (int j = 0; j < NF; j++)
#pragma unroll
      for (int r = 0; r < 4; r++) acc[i][j][r] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; s++) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }

  for (int kt = 0; kt < ktiles; kt++) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + STAGES - 1;
      if (nk < ktiles) load_stage(nk % STAGES, nk);
      cp_async_commit();
    }
    const double *as = As + (kt % STAGES) * BM * LDS + (warp * WM) * LDS;
    const double *bs = Bs + (kt % STAGES) * BN * LDS;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[MF][2], bf[NF];
#pragma unroll
      for (int i = 0; i < MF; i++) {
        af[i][0] = as[(i * 16 + g) * LDS + kk + t];
        af[i][1] = as[(i * 16 + g + 8) * LDS + kk + t];
      }
#pragma unroll
      for (int j = 0; j < NF; j++) bf[j] = bs[(j * 8 + g) * LDS + kk + t];
#pragma unroll
      for (int i = 0; i < MF; i++)
#pragma unroll
        for (int j = 0; j < NF; j++) dmma_16x8x4(acc[i][j], af[i][0], af[i][1], bf[j]);
    }
  }
  cp_async_wait<0>();

  // epilogue: X[(p*nu+q)*NP + s]
#pragma unroll
  for (int i = 0; i < MF; i++) {
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int64_t m = m0 + warp * WM + i * 16 + g + half * 8;
      if (m >= M) continue;
      double *orow = job.out + m * NP + n0 + 2 * t;
#pragma unroll
      for (int j = 0; j < NF; j++) {
        double2 v = make_double2(acc[i][j][2 * half], acc[i][j][2 * half + 1]);
        *reinterpret_cast<double2 *>(orow + j * 8) = v;
      }
    }
  }
}

template <int BN>
int launch_bn(const Dims &d, const GemmJob *jobs_dev, int njobs, cudaStream_t s) {
  constexpr int smem = smem_bytes<BN>();
  static int configured_device = -1;
  int dev = 0;
  CCT_CUDA(cudaGetDevice(&dev));
  if (configured_device != dev) {
    CCT_CUDA(cudaFuncSetAttribute(wbuild_f64_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    configured_device = dev;
  }
  const int64_t M = (int64_t)d.nu * d.nu;
  const int tiles_m = (int)((M + BM - 1) / BM);
  const int tiles_n = (int)(d.NP / BN);
  dim3 grid(tiles_m * tiles_n, njobs);
  wbuild_f64_kernel<BN><<<grid, NT, smem, s>>>(jobs_dev, d.nu, d.KP, d.NP, tiles_n);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

}  // namespace

int launch_wbuild_f64(const Dims &d, const GemmJob *jobs_dev, int njobs, cudaStream_t s) {
  switch (d.BN) {
    case 64: return launch_bn<64>(d, jobs_dev, njobs, s);
    case 56: return launch_bn<56>(d, jobs_dev, njobs, s);
    case 48: return launch_bn<48>(d, jobs_dev, njobs, s);
    case 40: return launch_bn<40>(d, jobs_dev, njobs, s);
    case 32: return launch_bn<32>(d, jobs_dev, njobs, s);
    default:
      set_error("unsupported W-build N tile " + std::to_string(d.BN));
      return CCT_ERR_INVALID;
  }
}

}  // namespace cct
