// CCSD T1-dressing terms of the reference's OpenACC CCSD port
// (src/triples-ijk/ccsd_acc.f: terms_29_30_31, lines 1-60, and
// terms_32_33_34_35, lines 64-160), on one GPU holding every occupied index.
// They contract the same expanded VVVO slices (ab|c j) as the triples W build,
// here with T1 (O1) and T2 (O2) into CCSD residual intermediates.
//
// terms_29_30_31, per occupied j, as the reference's DGEMM / TRANMD / INSITU
// sequence composes (see oracle/oracle.py for the literal sequence):
//   T2(i,y,z,j) += sum_x O1(i,x) G_j(x,y,z),
//   G_j(x,y,z) = (z x|y j) - sum_k O1(k,z) VL(k,x,y,j) - sum_k O1(k,y) VR(z,k,x,j)
// (f4_g_kernel, then f4_o1_kernel: K = nu, bound by its nu^3 reads).
//
// terms_32_33_34_35:
//   t2 <- t2^T as an (nou x nou) matrix                            (TRANSQ)
//   o2(x,y,k,l) <- o2(k,x,y,l)                                     (INSITU 12, 23)
//   RL_pre(i,y,z,j) = sum_x O1(i,x) (x y|z j);  rl <- RL_pre^T     (DGEMM, TRANSQ)
//   vm(x,y,z,a) <- vm(y,x,z,a) + T((x,z), (a,y)),                  (TRANMD 312, update, TRANMD 23)
//   T((k,l), (a,j)) = sum_{x,y} o2(k,x,y,l) (a y|x j)
// T is one GEMM of M = no^2, N = nu no, K = nu^2 for all j at once: the FP64
// tensor-core W-build tile (cct_wbuild_tile.cuh) on row operands laid out
// for it.  The reference's VM update loop (ccsd_acc.f:136-144) adds tmp at
// an offset of one element; this follows the evident intent, VM(k,l,j,a) +=
// tmp((k,l),a).
#include "cct_internal.cuh"

namespace cct {
namespace {

__device__ __forceinline__ int64_t tri_at(int64_t a, int64_t b) {
  const int64_t I = a > b ? a : b, J = a > b ? b : a;  // packed a >= b triangle, row-major (CPYTSQ)
  return I * (I + 1) / 2 + J;
}

int grid_of(int64_t n) {
  int64_t b = (n + 255) / 256;
  return (int)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

// G_j(x,y,z) for terms 29-31 (or, with vl == vr == nullptr and swap set, the
// plain slice (x y|z j) for terms 32-35), Fortran (x fastest)
__global__ void f4_g_kernel(int no, int nu, int j, const double *__restrict__ o1, const double *__restrict__ vl,
                            const double *__restrict__ vr, const double *__restrict__ vvvo, int plain,
                            double *__restrict__ g) {
  const int64_t nu3 = (int64_t)nu * nu * nu, nutr = (int64_t)nu * (nu + 1) / 2;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nu3; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = e % nu, y = (e / nu) % nu, z = e / ((int64_t)nu * nu);
    if (plain) {  // (x y|z j): column j*nu + z, triangle (x, y)
      g[e] = vvvo[((int64_t)j * nu + z) * nutr + tri_at(x, y)];
      continue;
    }
    double v = vvvo[((int64_t)j * nu + y) * nutr + tri_at(z, x)];  // (z x|y j)
    const double *vlc = vl + (int64_t)no * (x + (int64_t)nu * (y + (int64_t)nu * j));
    const double *vrc = vr + z + (int64_t)nu * (int64_t)no * (x + (int64_t)nu * j);
    for (int k = 0; k < no; k++) v -= o1[k + (int64_t)no * z] * vlc[k] + o1[k + (int64_t)no * y] * vrc[(int64_t)nu * k];
    g[e] = v;
  }
}

// out(i, y, z) (+)= sum_x O1(i,x) g(x,y,z) for one j slab of an (no,nu,nu) array
__global__ void f4_o1_kernel(int no, int nu, const double *__restrict__ o1, const double *__restrict__ g,
                             double *__restrict__ out, int accumulate) {
  const int64_t n = (int64_t)no * nu * nu;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % no, yz = e / no;
    const double *gc = g + yz * nu;
    double s = 0.0;
    for (int x = 0; x < nu; x++) s += o1[i + (int64_t)no * x] * gc[x];
    out[e] = accumulate ? out[e] + s : s;
  }
}

// dst = src^T for an n x n column-major matrix
__global__ void f4_transq_kernel(int64_t n, const double *__restrict__ src, double *__restrict__ dst) {
  const int64_t nn = n * n;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e % n, c = e / n;
    dst[e] = src[c + n * r];
  }
}

// o2 (no,nu,nu,no) -> o2b (nu,nu,no,no), o2b(x,y,k,l) = o2(k,x,y,l); also the
// GEMM's row operand apad[(k + no l)][x + nu y] with rows of kp doubles
__global__ void f4_o2_kernel(int no, int nu, int64_t kp, const double *__restrict__ o2, double *__restrict__ o2b,
                             double *__restrict__ apad) {
  const int64_t nu2 = (int64_t)nu * nu, n = nu2 * no * no;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t xy = e % nu2, kl = e / nu2;
    const int64_t x = xy % nu, y = xy / nu, k = kl % no, l = kl / no;
    const double v = o2[k + no * (x + nu * (y + nu * l))];
    o2b[e] = v;
    apad[kl * kp + xy] = v;
  }
}

// the GEMM's column operand: bpad[(a + nu j)][x + nu y] = (a y|x j)
__global__ void f4_b_kernel(int no, int nu, int64_t kp, const double *__restrict__ vvvo, double *__restrict__ bpad) {
  const int64_t nu2 = (int64_t)nu * nu, n = nu2 * nu * no, nutr = (int64_t)nu * (nu + 1) / 2;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t xy = e % nu2, aj = e / nu2;
    const int64_t x = xy % nu, y = xy / nu, a = aj % nu, j = aj / nu;
    bpad[aj * kp + xy] = vvvo[(j * nu + x) * nutr + tri_at(a, y)];
  }
}

// vm_out(x,y,z,a) = vm_in(y,x,z,a) + T[(x + no z) np + (a + nu y)]
__global__ void f4_vm_kernel(int no, int nu, int64_t np, const double *__restrict__ vm_in, const double *__restrict__ t,
                             double *__restrict__ vm_out) {
  const int64_t n = (int64_t)no * no * no * nu;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = e % no, y = (e / no) % no, z = (e / ((int64_t)no * no)) % no, a = e / ((int64_t)no * no * no);
    vm_out[e] = vm_in[y + no * (x + no * (z + no * a))] + t[(x + no * z) * np + (a + nu * y)];
  }
}

struct DevBuf {  // device copies of host arrays (or the caller's device arrays)
  std::vector<void *> owned;
  ~DevBuf() {
    for (void *p : owned) cudaFree(p);
  }
  int get(double **dst, const double *src, int64_t n, int32_t mem, bool upload, cudaStream_t s) {
    if (mem == CCT_MEM_DEVICE) {
      *dst = const_cast<double *>(src);
      return CCT_OK;
    }
    CCT_CUDA(cudaMalloc(reinterpret_cast<void **>(dst), (size_t)(n < 1 ? 1 : n) * 8));
    owned.push_back(*dst);
    if (upload) CCT_CUDA(cudaMemcpyAsync(*dst, src, (size_t)n * 8, cudaMemcpyHostToDevice, s));
    return CCT_OK;
  }
  int tmp(double **dst, int64_t n) {
    CCT_CUDA(cudaMalloc(reinterpret_cast<void **>(dst), (size_t)(n < 1 ? 1 : n) * 8));
    owned.push_back(*dst);
    return CCT_OK;
  }
};

int check_args(int64_t no, int64_t nu, int32_t mem) {
  if (no < 1 || nu < 1 || no > 4096 || nu > 4096 || (mem != CCT_MEM_HOST && mem != CCT_MEM_DEVICE)) {
    set_error("need 1 <= no, nu <= 4096 and mem CCT_MEM_HOST or CCT_MEM_DEVICE");
    return CCT_ERR_INVALID;
  }
  return CCT_OK;
}

}  // namespace
}  // namespace cct

using namespace cct;

extern "C" int ccT_ccsd_terms_29_31(int64_t no, int64_t nu, const double *o1, double *t2, const double *vl,
                                    const double *vr, const double *vvvo, int32_t mem) {
  CCT_TRY(check_args(no, nu, mem));
  if (!o1 || !t2 || !vl || !vr || !vvvo) {
    set_error("an array pointer is NULL");
    return CCT_ERR_INVALID;
  }
  const cudaStream_t s = nullptr;
  const int64_t nu2 = nu * nu, nutr = nu * (nu + 1) / 2;
  DevBuf b;
  double *d_o1, *d_t2, *d_vl, *d_vr, *d_vvvo, *g;
  CCT_TRY(b.get(&d_o1, o1, no * nu, mem, true, s));
  CCT_TRY(b.get(&d_t2, t2, no * nu2 * no, mem, true, s));
  CCT_TRY(b.get(&d_vl, vl, no * nu2 * no, mem, true, s));
  CCT_TRY(b.get(&d_vr, vr, nu * no * nu * no, mem, true, s));
  CCT_TRY(b.get(&d_vvvo, vvvo, nutr * nu * no, mem, true, s));
  CCT_TRY(b.tmp(&g, nu2 * nu));
  for (int j = 0; j < no; j++) {
    f4_g_kernel<<<grid_of(nu2 * nu), 256, 0, s>>>((int)no, (int)nu, j, d_o1, d_vl, d_vr, d_vvvo, 0, g);
    CCT_CUDA(cudaGetLastError());
    f4_o1_kernel<<<grid_of(no * nu2), 256, 0, s>>>((int)no, (int)nu, d_o1, g, d_t2 + (int64_t)j * no * nu2, 1);
    CCT_CUDA(cudaGetLastError());
  }
  if (mem == CCT_MEM_HOST) CCT_CUDA(cudaMemcpyAsync(t2, d_t2, (size_t)no * nu2 * no * 8, cudaMemcpyDeviceToHost, s));
  CCT_CUDA(cudaStreamSynchronize(s));
  return CCT_OK;
}

extern "C" int ccT_ccsd_terms_32_35(int64_t no, int64_t nu, const double *o1, double *o2, double *t2, double *vm,
                                    double *rl, const double *vvvo, int32_t mem) {
  CCT_TRY(check_args(no, nu, mem));
  if (!o1 || !o2 || !t2 || !vm || !rl || !vvvo) {
    set_error("an array pointer is NULL");
    return CCT_ERR_INVALID;
  }
  if (nu * nu < no) {
    set_error("terms_32_35 needs nu^2 >= no");
    return CCT_ERR_INVALID;
  }
  const cudaStream_t s = nullptr;
  const int64_t nu2 = nu * nu, nou = no * nu, n4 = nou * nou, nutr = nu * (nu + 1) / 2;
  DevBuf b;
  double *d_o1, *d_o2, *d_t2, *d_vm, *d_rl, *d_vvvo;
  CCT_TRY(b.get(&d_o1, o1, no * nu, mem, true, s));
  CCT_TRY(b.get(&d_o2, o2, n4, mem, true, s));
  CCT_TRY(b.get(&d_t2, t2, n4, mem, true, s));
  CCT_TRY(b.get(&d_vm, vm, no * no * no * nu, mem, true, s));
  CCT_TRY(b.get(&d_rl, rl, n4, mem, false, s));
  CCT_TRY(b.get(&d_vvvo, vvvo, nutr * nu * no, mem, true, s));
  // TRANSQ(T2) (ccsd_acc.f:83)
  double *tmp;
  CCT_TRY(b.tmp(&tmp, n4 > nu2 * nu ? n4 : nu2 * nu));
  CCT_CUDA(cudaMemcpyAsync(tmp, d_t2, (size_t)n4 * 8, cudaMemcpyDeviceToDevice, s));
  f4_transq_kernel<<<grid_of(n4), 256, 0, s>>>(nou, tmp, d_t2);
  CCT_CUDA(cudaGetLastError());
  // RL_pre(i,y,z,j) = sum_x O1(i,x) (x y|z j) (line 109), then TRANSQ into rl (line 151)
  double *rlpre;
  CCT_TRY(b.tmp(&rlpre, n4));
  for (int j = 0; j < no; j++) {
    f4_g_kernel<<<grid_of(nu2 * nu), 256, 0, s>>>((int)no, (int)nu, j, d_o1, nullptr, nullptr, d_vvvo, 1, tmp);
    CCT_CUDA(cudaGetLastError());
    f4_o1_kernel<<<grid_of(no * nu2), 256, 0, s>>>((int)no, (int)nu, d_o1, tmp, rlpre + (int64_t)j * no * nu2, 0);
    CCT_CUDA(cudaGetLastError());
  }
  f4_transq_kernel<<<grid_of(n4), 256, 0, s>>>(nou, rlpre, d_rl);
  CCT_CUDA(cudaGetLastError());
  // INSITU 12, 23 of O2 (lines 84-85) and the GEMM operands
  Dims g{};
  g.nu = (int)no;                        // M = no^2 rows (k + no l)
  g.KP = round_up(nu2, kKB);             // K = nu^2 (x + nu y), rows padded
  g.no = (int)(nu2 - no);                // valid K = g.nu + g.no = nu^2
  g.BN = choose_bn(nou);
  g.NP = round_up(nou, g.BN);            // N = nu no (a + nu j)
  double *o2in, *apad, *bpad, *t;
  CCT_TRY(b.tmp(&o2in, n4));
  CCT_TRY(b.tmp(&apad, no * no * g.KP));
  CCT_TRY(b.tmp(&bpad, g.NP * g.KP));
  CCT_TRY(b.tmp(&t, no * no * g.NP));
  CCT_CUDA(cudaMemcpyAsync(o2in, d_o2, (size_t)n4 * 8, cudaMemcpyDeviceToDevice, s));
  CCT_CUDA(cudaMemsetAsync(apad, 0, (size_t)no * no * g.KP * 8, s));
  CCT_CUDA(cudaMemsetAsync(bpad, 0, (size_t)g.NP * g.KP * 8, s));
  f4_o2_kernel<<<grid_of(n4), 256, 0, s>>>((int)no, (int)nu, g.KP, o2in, d_o2, apad);
  CCT_CUDA(cudaGetLastError());
  f4_b_kernel<<<grid_of(nu2 * nou), 256, 0, s>>>((int)no, (int)nu, g.KP, d_vvvo, bpad);
  CCT_CUDA(cudaGetLastError());
  // T((k,l),(a,j)) = sum_{x,y} o2b(x,y,k,l) (a y|x j) (line 119 for every j) on the FP64 tensor cores
  GemmJob job{apad, apad, bpad, bpad, t, 1, 0};
  GemmJob *d_job;
  CCT_CUDA(cudaMalloc(reinterpret_cast<void **>(&d_job), sizeof(GemmJob)));
  b.owned.push_back(d_job);
  CCT_CUDA(cudaMemcpyAsync(d_job, &job, sizeof(GemmJob), cudaMemcpyHostToDevice, s));
  CCT_TRY(launch_wbuild_f64(g, d_job, 1, s));
  // VM: TRANMD 312, the update of lines 125-131, TRANMD 23 (lines 86, 154)
  double *vmin;
  CCT_TRY(b.tmp(&vmin, no * no * no * nu));
  CCT_CUDA(cudaMemcpyAsync(vmin, d_vm, (size_t)no * no * no * nu * 8, cudaMemcpyDeviceToDevice, s));
  f4_vm_kernel<<<grid_of(no * no * no * nu), 256, 0, s>>>((int)no, (int)nu, g.NP, vmin, t, d_vm);
  CCT_CUDA(cudaGetLastError());
  if (mem == CCT_MEM_HOST) {
    CCT_CUDA(cudaMemcpyAsync(t2, d_t2, (size_t)n4 * 8, cudaMemcpyDeviceToHost, s));
    CCT_CUDA(cudaMemcpyAsync(o2, d_o2, (size_t)n4 * 8, cudaMemcpyDeviceToHost, s));
    CCT_CUDA(cudaMemcpyAsync(vm, d_vm, (size_t)no * no * no * nu * 8, cudaMemcpyDeviceToHost, s));
    CCT_CUDA(cudaMemcpyAsync(rl, d_rl, (size_t)n4 * 8, cudaMemcpyDeviceToHost, s));
  }
  CCT_CUDA(cudaStreamSynchronize(s));
  return CCT_OK;
}
