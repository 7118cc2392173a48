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
// tiles in unpadded, XOR-swizzled rows (conflict-free fragment loads); three
// CTAs per SM.
#include "cct_wbuild_tile.cuh"

namespace cct {
namespace {

using namespace wb;

template <int BN>
__global__ void __launch_bounds__(NT, 3) wbuild_f64_kernel(const GemmJob *__restrict__ jobs, int nu, int64_t KP,
                                                           int64_t KV, int64_t NP, int tiles_n) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tile_m = blockIdx.x / tiles_n, tile_n = blockIdx.x - tile_m * tiles_n;
  wbuild_tile<BN>(jobs[blockIdx.y], nu, KP, KV, NP, tile_m, tile_n, smem_raw);
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
  wbuild_f64_kernel<BN><<<grid, NT, smem, s>>>(jobs_dev, d.nu, d.KP, d.nu + d.no, d.NP, tiles_n);
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
    case 24: return launch_bn<24>(d, jobs_dev, njobs, s);  // the CCSD terms' X_j GEMM (N = no)
    default:
      set_error("unsupported W-build N tile " + std::to_string(d.BN));
      return CCT_ERR_INVALID;
  }
}

}  // namespace cct
