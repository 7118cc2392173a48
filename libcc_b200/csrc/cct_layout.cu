// Device layouts of the (T) inputs.
//
// The reference keeps the packed VVVO integrals in a DDI distributed array and
// fetches, expands (CPYTSQ, common_functions.f:43-60) and b<->c-swaps
// (tranmd_23 / trant3_1) one occupied slice per new i/j/k.  Here every slice
// is expanded once into HBM, already in the operand order the W-build
// contraction reads, and fused with the T2 rows of the K=no contractions:
//
//   E[x][r1][r2][kappa], kappa < nu       : (kappa r2 | r1 x)       (VVVO slice x)
//                        nu <= kappa < nu+no: -T2(r1, r2, kappa-nu, x)
//                        otherwise          : 0 (pad to KP)
//   F[y][z][s][kappa],   kappa < nu       : T2(s, kappa, y, z)
//                        nu <= kappa < nu+no: VM(kappa-nu, s, z, y)
//                        otherwise / s>=nu  : 0 (pad to KP / NP)
//
// With these, the twelve contractions of one tuple become three GEMMs whose
// rows are contiguous in kappa (see cct_wbuild_f64.cu).
#include "cct_internal.cuh"

namespace cct {

namespace {

__device__ __forceinline__ int64_t tri_index(int64_t a, int64_t b) {
  // packed position of the symmetric pair (a,b): CPYTSQ order, row I >= column J
  int64_t I = a > b ? a : b, J = a > b ? b : a;
  return I * (I + 1) / 2 + J;
}

// One warp per E row (x, r1, r2); lanes walk kappa.  E holds the slabs of
// occupied indices e_x0, e_x0 + 1, ... (0: the whole operand).
__global__ void build_e_kernel(const double *__restrict__ vvvo, const double *__restrict__ t2, double *__restrict__ E,
                               int no, int nu, int64_t KP, int x_begin, int x_end, int64_t col_base, int e_x0) {
  const int64_t nu2 = (int64_t)nu * nu;
  const int64_t nrows = (int64_t)(x_end - x_begin) * nu2;
  const int64_t nutr = (int64_t)nu * (nu + 1) / 2;
  const int lane = threadIdx.x & 31;
  int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (; row < nrows; row += stride) {
    const int64_t xr = row / nu2;
    const int x = x_begin + (int)xr;
    const int64_t rem = row - xr * nu2;
    const int r1 = (int)(rem / nu), r2 = (int)(rem - (int64_t)(rem / nu) * nu);
    const double *col = vvvo + ((int64_t)x * nu + r1 - col_base) * nutr;
    double *dst = E + ((int64_t)(x - e_x0) * nu2 + rem) * KP;
    for (int64_t kap = lane; kap < KP; kap += 32) {
      double v = 0.0;
      if (kap < nu) {
        v = col[tri_index(kap, r2)];
      } else if (kap < nu + no) {
        const int64_t l = kap - nu;
        v = -t2[(((int64_t)x * no + l) * nu + r2) * nu + r1];
      }
      dst[kap] = v;
    }
  }
}

// One warp per F row (y, z, s); lanes walk kappa.
__global__ void build_f_kernel(const double *__restrict__ t2, const double *__restrict__ vm, double *__restrict__ F,
                               int no, int nu, int64_t KP, int64_t NP) {
  const int64_t nrows = (int64_t)no * no * NP;
  const int lane = threadIdx.x & 31;
  int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (; row < nrows; row += stride) {
    const int64_t yz = row / NP;
    const int s = (int)(row - yz * NP);
    const int y = (int)(yz / no), z = (int)(yz - (int64_t)(yz / no) * no);
    double *dst = F + row * KP;
    for (int64_t kap = lane; kap < KP; kap += 32) {
      double v = 0.0;
      if (s < nu) {
        if (kap < nu)
          v = t2[(((int64_t)z * no + y) * nu + kap) * nu + s];
        else if (kap < nu + no)
          v = vm[(((int64_t)y * no + z) * nu + s) * no + (kap - nu)];
      }
      dst[kap] = v;
    }
  }
}

// flags[0] |= 1 when any element is NaN/Inf.
__global__ void finite_kernel(const double *__restrict__ p, int64_t n, int *flags) {
  int bad = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    bad |= !isfinite(p[i]);
  bad = __syncthreads_or(bad);
  if (bad && threadIdx.x == 0) atomicOr(flags, 1);
}

int grid_for(int64_t warps) {
  int64_t blocks = (warps * 32 + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  if (blocks < 1) blocks = 1;
  return (int)blocks;
}

}  // namespace

int launch_build_e(const Dims &d, const double *vvvo_packed, const double *t2, double *E, int x_begin, int x_end,
                   cudaStream_t s) {
  if (x_end <= x_begin) return CCT_OK;
  const int64_t rows = (int64_t)(x_end - x_begin) * d.nu * d.nu;
  build_e_kernel<<<grid_for(rows), 256, 0, s>>>(vvvo_packed, t2, E, d.no, d.nu, d.KP, x_begin, x_end, 0, 0);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

int launch_build_e_slice(const Dims &d, const double *packed_slice, const double *t2, double *E, int x,
                         cudaStream_t s) {
  // packed_slice holds the nu columns x*nu .. x*nu+nu-1 only
  const int64_t rows = (int64_t)d.nu * d.nu;
  build_e_kernel<<<grid_for(rows), 256, 0, s>>>(packed_slice, t2, E, d.no, d.nu, d.KP, x, x + 1,
                                                (int64_t)x * d.nu, 0);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

int launch_build_e_slab(const Dims &d, const double *vvvo_packed, const double *t2, double *slab, int x,
                        cudaStream_t s) {
  const int64_t rows = (int64_t)d.nu * d.nu;
  build_e_kernel<<<grid_for(rows), 256, 0, s>>>(vvvo_packed, t2, slab, d.no, d.nu, d.KP, x, x + 1, 0, x);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}


int launch_build_f(const Dims &d, const double *t2, const double *vm, double *F, cudaStream_t s) {
  const int64_t rows = (int64_t)d.no * d.no * d.NP;
  build_f_kernel<<<grid_for(rows), 256, 0, s>>>(t2, vm, F, d.no, d.nu, d.KP, d.NP);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

int launch_check_inputs(const Dims &d, const double *eh, const double *ep, const double *t1, const double *t2,
                        const double *vm, const double *voe, const double *vvvo, int *flags, cudaStream_t s) {
  const int64_t no = d.no, nu = d.nu;
  const struct {
    const double *p;
    int64_t n;
  } arrs[] = {{eh, no},           {ep, nu},           {t1, no * nu},
              {t2, nu * nu * no * no}, {vm, no * nu * no * no}, {voe, nu * nu * no * no},
              {vvvo, nu * (nu + 1) / 2 * nu * no}};
  for (auto &a : arrs) {
    int64_t blocks = (a.n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    finite_kernel<<<(int)(blocks < 1 ? 1 : blocks), 256, 0, s>>>(a.p, a.n, flags);
    CCT_CUDA(cudaGetLastError());
  }
  return CCT_OK;
}

}  // namespace cct
