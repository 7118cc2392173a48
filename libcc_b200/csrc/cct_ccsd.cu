// CCSD T1-dressing terms of the reference's OpenACC CCSD port
// (src/triples-ijk/ccsd_acc.f: terms_29_30_31, lines 1-60, and
// terms_32_33_34_35, lines 64-160), on one GPU holding every occupied index.
// They contract the same expanded VVVO slices (ab|c j) as the triples W build,
// here with T1 (O1) and T2 (O2) into CCSD residual intermediates.
//
// terms_29_30_31, per occupied j, as the reference's DGEMM / TRANMD / INSITU
// sequence composes (the oracle restates the literal sequence):
//   T2(i,y,z,j) += sum_x O1(i,x) G_j(x,y,z),
//   G_j(x,y,z) = (z x|y j) - sum_k O1(k,z) VL(k,x,y,j) - sum_k O1(k,y) VR(z,k,x,j).
// The O1 contraction is moved inside the two correction terms, so no nu^3 G_j
// is formed:
//   T2(i,y,z,j) += X_j(y,z,i) - sum_k O1(k,z) P_j(i,k,y) - sum_k O1(k,y) Q_j(i,z,k),
//   X_j(p,q,i) = sum_x (x q|p j) O1(i,x),   P_j(i,k,y) = sum_x O1(i,x) VL(k,x,y,j),
//   Q_j(i,z,k) = sum_x O1(i,x) VR(z,k,x,j).
// X_j for all j is one launch of the FP64 W-build tile with its row operand
// gathered from the packed triangle (the packed-VVVO path: row (p,q) of
// occupied j at k is (k q|p j)) against O1 as the column operand: 2 no^2 nu^3
// flops on the tensor pipe instead of 6 no^2 nu^3 on the FP64 units, and the
// packed slices read once instead of an expanded nu^3 slice written and read
// per j.  P and Q (no^2 nu per j) and the combination are small kernels.
//
// terms_32_33_34_35:
//   t2 <- t2^T as an (nou x nou) matrix                            (TRANSQ)
//   o2(x,y,k,l) <- o2(k,x,y,l)                                     (INSITU 12, 23)
//   RL_pre(i,y,z,j) = sum_x O1(i,x) (x y|z j) = X_j(z,y,i);  rl <- RL_pre^T
//                                                                  (DGEMM, TRANSQ)
//   vm(x,y,z,a) <- vm(y,x,z,a) + T((x,z), (a,y)),                  (TRANMD 312, update, TRANMD 23)
//   T((k,l), (a,j)) = sum_{x,y} o2(k,x,y,l) (a y|x j)
// T is one GEMM of M = no^2, N = nu no, K = nu^2 for all j at once: the FP64
// tensor-core W-build tile (cct_wbuild_tile.cuh) on row operands laid out
// for it.  The reference's VM update loop (ccsd_acc.f:136-144) adds tmp at
// an offset of one element; this follows the evident intent, VM(k,l,j,a) +=
// tmp((k,l),a).
#include "cct_internal.cuh"
#include "cct_wbuild_tile.cuh"

#include <map>
#include <mutex>

namespace cct {
namespace {


int grid_of(int64_t n) {
  int64_t b = (n + 255) / 256;
  return (int)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

// O1 as the W-build tile's column operand: o1pad[i][x] = O1(i,x), rows of kp
// doubles, zero past (no, nu)
__global__ void f4_o1pad_kernel(int no, int nu, int64_t kp, int64_t np, const double *__restrict__ o1,
                                double *__restrict__ o1pad) {
  const int64_t n = np * kp;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e / kp, x = e - i * kp;
    o1pad[e] = (i < no && x < nu) ? o1[i + (int64_t)no * x] : 0.0;
  }
}

// P[j][y][k][i] = sum_x O1(i,x) VL(k,x,y,j) and Q[j][z][k][i] = sum_x O1(i,x) VR(z,k,x,j)
__global__ void f4_pq_kernel(int no, int nu, const double *__restrict__ o1, const double *__restrict__ vl,
                             const double *__restrict__ vr, double *__restrict__ P, double *__restrict__ Q) {
  const int64_t n = (int64_t)no * no * nu * no;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < 2 * n; e += (int64_t)gridDim.x * blockDim.x) {
    const int which = e >= n;
    const int64_t r = e - which * n;
    const int64_t i = r % no, k = (r / no) % no, y = (r / ((int64_t)no * no)) % nu, j = r / ((int64_t)no * no * nu);
    double s = 0.0;
    if (!which) {
      const double *v = vl + k + (int64_t)no * (int64_t)nu * (y + (int64_t)nu * j);  // VL(k, x, y, j), x stride no
      for (int x = 0; x < nu; x++) s += o1[i + (int64_t)no * x] * v[(int64_t)no * x];
      P[r] = s;
    } else {
      const double *v = vr + y + (int64_t)nu * (k + (int64_t)no * (int64_t)nu * j);  // VR(z=y, k, x, j), x stride nu no
      for (int x = 0; x < nu; x++) s += o1[i + (int64_t)no * x] * v[(int64_t)nu * no * x];
      Q[r] = s;
    }
  }
}

// The same steps for no <= kNoTile, staged in shared memory so that global
// accesses are coalesced runs.
constexpr int kNoTile = 32;
// P[j][y][.][.] for one (y, j) per CTA: the contiguous VL(., ., y, j) slab and
// O1 pass through shared memory 32 virtual indices x at a time.
__global__ void __launch_bounds__(256) f4_p_tiled_kernel(int no, int nu, const double *__restrict__ o1,
                                                         const double *__restrict__ vl, double *__restrict__ P) {
  constexpr int XC = 32;
  __shared__ double vs[XC][kNoTile], os[XC][kNoTile];
  const int y = blockIdx.x, j = blockIdx.y, tid = threadIdx.x;
  const int i = tid & 31, kq = tid >> 5;
  const double *slab = vl + (int64_t)no * nu * (y + (int64_t)nu * j);  // VL(k, x, y, j) = slab[k + no x]
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int x0 = 0; x0 < nu; x0 += XC) {
    __syncthreads();
    for (int e = tid; e < XC * kNoTile; e += 256) {
      const int x = e / kNoTile, c = e % kNoTile;
      const bool ok = x0 + x < nu && c < no;
      vs[x][c] = ok ? slab[c + (int64_t)no * (x0 + x)] : 0.0;
      os[x][c] = ok ? o1[c + (int64_t)no * (x0 + x)] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int x = 0; x < XC; x++) {
      const double o = os[x][i];
#pragma unroll
      for (int u = 0; u < 4; u++) acc[u] = fma(vs[x][kq + 8 * u], o, acc[u]);
    }
  }
  double *pj = P + ((int64_t)j * nu + y) * no * no;
#pragma unroll
  for (int u = 0; u < 4; u++) {
    const int k = kq + 8 * u;
    if (k < no && i < no) pj[(int64_t)k * no + i] = acc[u];
  }
}

// Q[j][z][.][.] for eight consecutive z and one j per CTA: VR(z..z+7, k, x, j)
// are 64-byte runs, staged 16 x at a time.
__global__ void __launch_bounds__(256) f4_q_tiled_kernel(int no, int nu, const double *__restrict__ o1,
                                                         const double *__restrict__ vr, double *__restrict__ Q) {
  constexpr int XC = 16, ZT = 8;
  __shared__ double vs[XC][kNoTile][ZT], os[XC][kNoTile];
  const int z0 = blockIdx.x * ZT, j = blockIdx.y, tid = threadIdx.x;
  const int i = tid & 31, zz = tid >> 5;
  const int64_t nuno = (int64_t)nu * no;
  double acc[kNoTile];
#pragma unroll
  for (int k = 0; k < kNoTile; k++) acc[k] = 0.0;
  for (int x0 = 0; x0 < nu; x0 += XC) {
    __syncthreads();
    for (int e = tid; e < XC * kNoTile * ZT; e += 256) {
      const int z = e % ZT, k = (e / ZT) % kNoTile, x = e / (ZT * kNoTile);
      const bool ok = x0 + x < nu && k < no && z0 + z < nu;
      vs[x][k][z] = ok ? vr[(z0 + z) + (int64_t)nu * k + nuno * (x0 + x) + nuno * nu * j] : 0.0;
    }
    for (int e = tid; e < XC * kNoTile; e += 256) {
      const int x = e / kNoTile, c = e % kNoTile;
      os[x][c] = (x0 + x < nu && c < no) ? o1[c + (int64_t)no * (x0 + x)] : 0.0;
    }
    __syncthreads();
    for (int x = 0; x < XC; x++) {
      const double o = os[x][i];
#pragma unroll
      for (int k = 0; k < kNoTile; k++) acc[k] = fma(vs[x][k][zz], o, acc[k]);
    }
  }
  const int z = z0 + zz;
  if (z < nu && i < no) {
    double *qz = Q + ((int64_t)j * nu + z) * no * no;
#pragma unroll
    for (int k = 0; k < kNoTile; k++)
      if (k < no) qz[(int64_t)k * no + i] = acc[k];
  }
}

// T2(i,y,z,j) += X_j(y,z,i) - sum_k O1(k,z) P[j][y][k][i] for one (y, j) per
// CTA and every z (P[j][y] in shared memory, O1(., z) through the read-only
// cache: a warp reads one z's column); four z at a time, so their loads are
// in flight together.
__global__ void __launch_bounds__(256) f4_t2p_tiled_kernel(int no, int nu, int64_t np,
                                                           const double *__restrict__ o1,
                                                           const double *__restrict__ X,
                                                           const double *__restrict__ P, double *__restrict__ t2) {
  __shared__ double ps[kNoTile][kNoTile];
  const int y = blockIdx.x, j = blockIdx.y, tid = threadIdx.x;
  const int i = tid & 31, zg = tid >> 5;
  const double *pj = P + ((int64_t)j * nu + y) * no * no;
  for (int e = tid; e < kNoTile * kNoTile; e += 256) {
    const int k = e / kNoTile, c = e % kNoTile;
    ps[k][c] = (k < no && c < no) ? pj[(int64_t)k * no + c] : 0.0;
  }
  __syncthreads();
  if (i >= no) return;
  const int64_t nu2 = (int64_t)nu * nu;
  constexpr int U = 4;
  for (int zb = zg; zb < nu; zb += 8 * U) {
    double v[U], t[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int z = zb + 8 * u;
      v[u] = z < nu ? X[((int64_t)j * nu2 + (int64_t)y * nu + z) * np + i] : 0.0;
      t[u] = z < nu ? t2[i + (int64_t)no * (y + (int64_t)nu * (z + (int64_t)nu * j))] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int z = zb + 8 * u;
      if (z >= nu) break;
      const double *oz = o1 + (int64_t)no * z;
      for (int k = 0; k < no; k++) v[u] -= __ldg(oz + k) * ps[k][i];
      t2[i + (int64_t)no * (y + (int64_t)nu * (z + (int64_t)nu * j))] = t[u] + v[u];
    }
  }
}

// T2(i,y,z,j) -= sum_k O1(k,y) Q[j][z][k][i] for one (z, j) per CTA and every
// y; T2(., ., z, j) over (i, y) is one contiguous run.
__global__ void __launch_bounds__(256) f4_t2q_tiled_kernel(int no, int nu, const double *__restrict__ o1,
                                                           const double *__restrict__ Q, double *__restrict__ t2) {
  __shared__ double qs[kNoTile][kNoTile];
  const int z = blockIdx.x, j = blockIdx.y, tid = threadIdx.x;
  const int i = tid & 31, yg = tid >> 5;
  const double *qz = Q + ((int64_t)j * nu + z) * no * no;
  for (int e = tid; e < kNoTile * kNoTile; e += 256) {
    const int k = e / kNoTile, c = e % kNoTile;
    qs[k][c] = (k < no && c < no) ? qz[(int64_t)k * no + c] : 0.0;
  }
  __syncthreads();
  if (i >= no) return;
  double *tz = t2 + (int64_t)no * nu * (z + (int64_t)nu * j);
  constexpr int U = 4;
  for (int yb = yg; yb < nu; yb += 8 * U) {
    double t[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int y = yb + 8 * u;
      t[u] = y < nu ? tz[i + (int64_t)no * y] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int y = yb + 8 * u;
      if (y >= nu) break;
      const double *oy = o1 + (int64_t)no * y;
      double s = 0.0;
      for (int k = 0; k < no; k++) s = fma(__ldg(oy + k), qs[k][i], s);
      tz[i + (int64_t)no * y] = t[u] - s;
    }
  }
}

// T2(i,y,z,j) += X_j(y,z,i) - sum_k O1(k,z) P[j][y][k][i] - sum_k O1(k,y) Q[j][z][k][i]
__global__ void f4_t2_kernel(int no, int nu, int64_t np, const double *__restrict__ o1, const double *__restrict__ X,
                             const double *__restrict__ P, const double *__restrict__ Q, double *__restrict__ t2) {
  const int64_t nu2 = (int64_t)nu * nu, n = (int64_t)no * nu2 * no;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e % no, y = (e / no) % nu, z = (e / ((int64_t)no * nu)) % nu, j = e / ((int64_t)no * nu2);
    double v = X[(j * nu2 + y * nu + z) * np + i];
    const double *pj = P + (j * nu + y) * no * no + i, *qj = Q + (j * nu + z) * no * no + i;
    for (int k = 0; k < no; k++) v -= o1[k + (int64_t)no * z] * pj[(int64_t)k * no];
    for (int k = 0; k < no; k++) v -= o1[k + (int64_t)no * y] * qj[(int64_t)k * no];
    t2[e] += v;
  }
}

// rl = RL_pre^T as (nou x nou) matrices: rl[(z + nu j) + nou (i + no y)] = X_j(z,y,i)
// (written in order; the X reads are strided)
__global__ void f4_rl_kernel(int no, int nu, int64_t np, const double *__restrict__ X, double *__restrict__ rl) {
  const int64_t nu2 = (int64_t)nu * nu, nou = (int64_t)no * nu, n = nou * nou;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t zj = e % nou, iy = e / nou, z = zj % nu, j = zj / nu, i = iy % no, y = iy / no;
    rl[e] = X[(j * nu2 + z * nu + y) * np + i];
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
  const int64_t nu2 = (int64_t)nu * nu, n = nu2 * no * no, no2 = (int64_t)no * no;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t xy = e % nu2, kl = e / nu2;
    const int64_t x = xy % nu, y = xy / nu, k = kl % no, l = kl / no;
    const double v = o2[k + no * (x + nu * (y + nu * l))];
    o2b[e] = v;
    const int64_t z = xy / kp;  // K split
    apad[(z * no2 + kl) * kp + (xy - z * kp)] = v;
  }
}

// the GEMM's column operand: bpad[split][(a + nu j)][x + nu y] = (a y|x j), rows
// of kp doubles per split (np rows per split).  A transpose through shared
// memory: a CTA reads 32 packed columns (j, x0..x0+31) x 32 consecutive
// triangle entries t0..t0+31 along the columns, and writes each entry (a, y),
// a >= y, as 32 consecutive x of rows (a, j) and (y, j).
constexpr int kTT = 32;
__global__ void __launch_bounds__(256) f4_b_kernel(int no, int nu, int64_t kp, int64_t np,
                                                   const double *__restrict__ vvvo, double *__restrict__ bpad) {
  __shared__ double tile[kTT][kTT + 1];
  const int64_t nutr = (int64_t)nu * (nu + 1) / 2;
  const int64_t x0 = (int64_t)blockIdx.y * kTT, t0 = (int64_t)blockIdx.x * kTT;
  const int j = blockIdx.z;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int xi = ty; xi < kTT; xi += 8) {
    const int64_t x = x0 + xi, t = t0 + tx;
    tile[xi][tx] = (x < nu && t < nutr) ? vvvo[((int64_t)j * nu + x) * nutr + t] : 0.0;
  }
  __syncthreads();
  const int64_t x = x0 + tx;
  if (x >= nu) return;
  for (int ti = ty; ti < kTT; ti += 8) {
    const int64_t t = t0 + ti;
    if (t >= nutr) break;
    // t = a (a + 1) / 2 + y with 0 <= y <= a
    int64_t a = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while (a * (a + 1) / 2 > t) a--;
    while ((a + 1) * (a + 2) / 2 <= t) a++;
    const int64_t y = t - a * (a + 1) / 2;
    const double v = tile[tx][ti];
    const int64_t c1 = x + (int64_t)nu * y, z1 = c1 / kp;  // row (a, j), column (x, y)
    bpad[(z1 * np + a + (int64_t)nu * j) * kp + (c1 - z1 * kp)] = v;
    if (a != y) {
      const int64_t c2 = x + (int64_t)nu * a, z2 = c2 / kp;  // row (y, j), column (x, a)
      bpad[(z2 * np + y + (int64_t)nu * j) * kp + (c2 - z2 * kp)] = v;
    }
  }
}

// vm_out(x,y,z,a) = vm_in(y,x,z,a) + sum over the K splits of T[(x + no z) np + (a + nu y)]
__global__ void f4_vm_kernel(int no, int nu, int64_t np, int nsplit, int64_t tsplit, const double *__restrict__ vm_in,
                             const double *__restrict__ t, double *__restrict__ vm_out) {
  const int64_t n = (int64_t)no * no * no * nu;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = e % no, y = (e / no) % no, z = (e / ((int64_t)no * no)) % no, a = e / ((int64_t)no * no * no);
    const double *tz = t + (x + no * z) * np + (a + nu * y);
    double v = tz[0];
    for (int sp = 1; sp < nsplit; sp++) v += tz[sp * tsplit];
    vm_out[e] = vm_in[y + no * (x + no * (z + no * a))] + v;
  }
}

// Device workspace of the two entry points, kept between calls: a call asks
// for the same sequence of buffers every time, so slot k of entry point e on
// device d (the k-th buffer of the call) is reused, and grown when a call
// needs more; after the first call of a shape nothing is allocated.  The
// entry points are synchronous and serialised by a mutex;
// ccT_ccsd_release_workspace frees the workspace.
struct Workspace {
  std::vector<std::pair<void *, size_t>> slot;
};
std::mutex g_ws_mutex;
std::map<std::pair<int, int>, Workspace> g_ws;

struct DevBuf {  // device copies of host arrays (or the caller's device arrays) and scratch
  std::lock_guard<std::mutex> lock{g_ws_mutex};
  Workspace *ws = nullptr;
  size_t next = 0;
  explicit DevBuf(int entry) {
    int dev = 0;
    cudaGetDevice(&dev);
    ws = &g_ws[{dev, entry}];
  }
  int alloc(void **dst, size_t bytes) {
    if (bytes < 8) bytes = 8;
    if (next == ws->slot.size()) ws->slot.push_back({nullptr, 0});
    std::pair<void *, size_t> &sl = ws->slot[next++];
    if (sl.second < bytes) {
      if (sl.first) CCT_CUDA(cudaFree(sl.first));
      sl = {nullptr, 0};
      CCT_CUDA(cudaMalloc(&sl.first, bytes));
      sl.second = bytes;
    }
    *dst = sl.first;
    return CCT_OK;
  }
  int get(double **dst, const double *src, int64_t n, int32_t mem, bool upload, cudaStream_t s) {
    if (mem == CCT_MEM_DEVICE) {
      *dst = const_cast<double *>(src);
      return CCT_OK;
    }
    CCT_TRY(alloc(reinterpret_cast<void **>(dst), (size_t)n * 8));
    if (upload) CCT_CUDA(cudaMemcpyAsync(*dst, src, (size_t)n * 8, cudaMemcpyHostToDevice, s));
    return CCT_OK;
  }
  int tmp(double **dst, int64_t n) { return alloc(reinterpret_cast<void **>(dst), (size_t)n * 8); }
};

// X_j(p,q,i) = sum_x (x q|p j) O1(i,x) for every occupied j, X_j at x + j nu^2 np,
// row (p,q) at (p nu + q) np: the W-build tile, one packed-row job per j.
int packed_o1_gemm(int64_t no, int64_t nu, const double *d_o1, const double *d_vvvo, DevBuf &b, double **X,
                   int64_t *np_out, cudaStream_t s) {
  const int64_t nutr = nu * (nu + 1) / 2;
  Dims g{};
  g.nu = (int)nu;                  // M = nu^2 rows (p, q)
  g.no = 0;                        // K = nu (the packed part of a row alone)
  g.KP = round_up(nu, kKB);
  // N = no: a 24-column tile when no pads to 24 (no waste at no = 24, where
  // the smallest plan tile, 32, computes a quarter of padding)
  g.BN = round_up(no, 8) == 24 ? 24 : choose_bn((int)no);
  g.NP = round_up(no, g.BN);
  double *o1pad;
  CCT_TRY(b.tmp(&o1pad, g.NP * g.KP));
  CCT_TRY(b.tmp(X, no * nu * nu * g.NP));
  f4_o1pad_kernel<<<grid_of(g.NP * g.KP), 256, 0, s>>>((int)no, (int)nu, g.KP, g.NP, d_o1, o1pad);
  CCT_CUDA(cudaGetLastError());
  std::vector<GemmJob> jobs((size_t)no);
  for (int64_t j = 0; j < no; j++) {
    const double *pj = d_vvvo + j * nu * nutr;  // the nu packed columns of occupied j
    jobs[j] = GemmJob{pj, pj, o1pad, o1pad, *X + j * nu * nu * g.NP, 1, 1, pj, pj};
  }
  GemmJob *d_jobs;
  CCT_TRY(b.alloc(reinterpret_cast<void **>(&d_jobs), jobs.size() * sizeof(GemmJob)));
  CCT_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(GemmJob), cudaMemcpyHostToDevice, s));
  CCT_TRY(launch_wbuild_f64(g, d_jobs, (int)no, s));
  *np_out = g.NP;
  return CCT_OK;
}

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
  DevBuf b(0);
  double *d_o1, *d_t2, *d_vl, *d_vr, *d_vvvo;
  CCT_TRY(b.get(&d_o1, o1, no * nu, mem, true, s));
  CCT_TRY(b.get(&d_t2, t2, no * nu2 * no, mem, true, s));
  CCT_TRY(b.get(&d_vl, vl, no * nu2 * no, mem, true, s));
  CCT_TRY(b.get(&d_vr, vr, nu * no * nu * no, mem, true, s));
  CCT_TRY(b.get(&d_vvvo, vvvo, nutr * nu * no, mem, true, s));
  double *X, *P, *Q;
  int64_t np = 0;
  CCT_TRY(packed_o1_gemm(no, nu, d_o1, d_vvvo, b, &X, &np, s));
  CCT_TRY(b.tmp(&P, no * no * nu * no));
  CCT_TRY(b.tmp(&Q, no * no * nu * no));
  if (no <= kNoTile) {
    f4_p_tiled_kernel<<<dim3((unsigned)nu, (unsigned)no), 256, 0, s>>>((int)no, (int)nu, d_o1, d_vl, P);
    CCT_CUDA(cudaGetLastError());
    f4_q_tiled_kernel<<<dim3((unsigned)((nu + 7) / 8), (unsigned)no), 256, 0, s>>>((int)no, (int)nu, d_o1, d_vr, Q);
    CCT_CUDA(cudaGetLastError());
    f4_t2p_tiled_kernel<<<dim3((unsigned)nu, (unsigned)no), 256, 0, s>>>((int)no, (int)nu, np, d_o1, X, P, d_t2);
    CCT_CUDA(cudaGetLastError());
    f4_t2q_tiled_kernel<<<dim3((unsigned)nu, (unsigned)no), 256, 0, s>>>((int)no, (int)nu, d_o1, Q, d_t2);
    CCT_CUDA(cudaGetLastError());
  } else {
    f4_pq_kernel<<<grid_of(2 * no * no * nu * no), 256, 0, s>>>((int)no, (int)nu, d_o1, d_vl, d_vr, P, Q);
    CCT_CUDA(cudaGetLastError());
    f4_t2_kernel<<<grid_of(no * nu2 * no), 256, 0, s>>>((int)no, (int)nu, np, d_o1, X, P, Q, d_t2);
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
  DevBuf b(1);
  double *d_o1, *d_o2, *d_t2, *d_vm, *d_rl, *d_vvvo;
  CCT_TRY(b.get(&d_o1, o1, no * nu, mem, true, s));
  CCT_TRY(b.get(&d_o2, o2, n4, mem, true, s));
  CCT_TRY(b.get(&d_t2, t2, n4, mem, true, s));
  CCT_TRY(b.get(&d_vm, vm, no * no * no * nu, mem, true, s));
  CCT_TRY(b.get(&d_rl, rl, n4, mem, false, s));
  CCT_TRY(b.get(&d_vvvo, vvvo, nutr * nu * no, mem, true, s));
  // TRANSQ(T2) (ccsd_acc.f:83)
  double *tmp;
  CCT_TRY(b.tmp(&tmp, n4));
  CCT_CUDA(cudaMemcpyAsync(tmp, d_t2, (size_t)n4 * 8, cudaMemcpyDeviceToDevice, s));
  f4_transq_kernel<<<grid_of(n4), 256, 0, s>>>(nou, tmp, d_t2);
  CCT_CUDA(cudaGetLastError());
  // RL_pre(i,y,z,j) = sum_x O1(i,x) (x y|z j) = X_j(z,y,i) (line 109), then TRANSQ into rl (line 151)
  {
    double *X;
    int64_t np = 0;
    CCT_TRY(packed_o1_gemm(no, nu, d_o1, d_vvvo, b, &X, &np, s));
    f4_rl_kernel<<<grid_of(n4), 256, 0, s>>>((int)no, (int)nu, np, X, d_rl);
    CCT_CUDA(cudaGetLastError());
  }
  // INSITU 12, 23 of O2 (lines 84-85) and the GEMM operands.  T has few
  // output tiles (M = no^2) and a long contraction (K = nu^2), so K is split
  // into nsplit ranges, each a job of its own (the operands stored split by
  // split), for whole waves of CTAs; f4_vm_kernel sums the splits in order.
  Dims g{};
  g.nu = (int)no;                        // M = no^2 rows (k + no l)
  g.BN = choose_bn(nou);
  g.NP = round_up(nou, g.BN);            // N = nu no (a + nu j)
  int nsplit = 1;
  {
    int dev = 0, nsm = 148;
    CCT_CUDA(cudaGetDevice(&dev));
    CCT_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int64_t slots = 3 * (int64_t)nsm;  // W-build tile: three CTAs per SM
    const int64_t tiles = ((int64_t)no * no + wb::BM - 1) / wb::BM * (g.NP / g.BN);
    double best = 0.0;
    for (int sp = 1; sp <= 16 && (int64_t)sp * kKB <= nu2; sp++) {
      const int64_t ctas = tiles * sp, waves = (ctas + slots - 1) / slots;
      const double fill = (double)ctas / (double)(waves * slots);
      if (fill > best + 0.02) {
        best = fill;
        nsplit = sp;
      }
    }
  }
  g.KP = round_up((nu2 + nsplit - 1) / nsplit, kKB);  // K per split (x + nu y), zero past nu^2
  g.no = (int)(g.KP - no);                            // every column of a split counts as valid
  double *o2in, *apad, *bpad, *t;
  CCT_TRY(b.tmp(&o2in, n4));
  CCT_TRY(b.tmp(&apad, nsplit * no * no * g.KP));
  CCT_TRY(b.tmp(&bpad, nsplit * g.NP * g.KP));
  CCT_TRY(b.tmp(&t, nsplit * no * no * g.NP));
  CCT_CUDA(cudaMemcpyAsync(o2in, d_o2, (size_t)n4 * 8, cudaMemcpyDeviceToDevice, s));
  CCT_CUDA(cudaMemsetAsync(apad, 0, (size_t)nsplit * no * no * g.KP * 8, s));
  CCT_CUDA(cudaMemsetAsync(bpad, 0, (size_t)nsplit * g.NP * g.KP * 8, s));
  f4_o2_kernel<<<grid_of(n4), 256, 0, s>>>((int)no, (int)nu, g.KP, o2in, d_o2, apad);
  CCT_CUDA(cudaGetLastError());
  {
    const int64_t nutr = nu * (nu + 1) / 2;
    const dim3 grid((unsigned)((nutr + kTT - 1) / kTT), (unsigned)((nu + kTT - 1) / kTT), (unsigned)no);
    f4_b_kernel<<<grid, 256, 0, s>>>((int)no, (int)nu, g.KP, g.NP, d_vvvo, bpad);
  }
  CCT_CUDA(cudaGetLastError());
  // T((k,l),(a,j)) = sum_{x,y} o2b(x,y,k,l) (a y|x j) (line 119 for every j) on the FP64 tensor cores
  std::vector<GemmJob> jobs(nsplit);
  for (int z = 0; z < nsplit; z++) {
    const double *az = apad + (int64_t)z * no * no * g.KP, *bz = bpad + (int64_t)z * g.NP * g.KP;
    jobs[z] = GemmJob{az, az, bz, bz, t + (int64_t)z * no * no * g.NP, 1, 0};
  }
  GemmJob *d_job;
  CCT_TRY(b.alloc(reinterpret_cast<void **>(&d_job), nsplit * sizeof(GemmJob)));
  CCT_CUDA(cudaMemcpyAsync(d_job, jobs.data(), nsplit * sizeof(GemmJob), cudaMemcpyHostToDevice, s));
  CCT_TRY(launch_wbuild_f64(g, d_job, nsplit, s));
  // VM: TRANMD 312, the update of lines 125-131, TRANMD 23 (lines 86, 154)
  double *vmin;
  CCT_TRY(b.tmp(&vmin, no * no * no * nu));
  CCT_CUDA(cudaMemcpyAsync(vmin, d_vm, (size_t)no * no * no * nu * 8, cudaMemcpyDeviceToDevice, s));
  f4_vm_kernel<<<grid_of(no * no * no * nu), 256, 0, s>>>((int)no, (int)nu, g.NP, nsplit, no * no * g.NP, vmin, t,
                                                          d_vm);
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

extern "C" int ccT_ccsd_release_workspace(void) {
  std::lock_guard<std::mutex> lock(g_ws_mutex);
  int prev = 0;
  cudaGetDevice(&prev);
  for (auto &e : g_ws) {
    cudaSetDevice(e.first.first);
    for (auto &sl : e.second.slot)
      if (sl.first) cudaFree(sl.first);
  }
  g_ws.clear();
  cudaSetDevice(prev);
  return CCT_OK;
}
