// Allocation-free E[4]/E[5] reduction of one tuple from a caller-held W_abc.
//
// Some callers cannot let a library allocate device memory: applications that
// carve every device buffer out of one arena they reserve up front (a
// quantum-chemistry package that sizes its GPU memory once for the whole job),
// and drivers that must not risk the implicit device synchronisation a
// cudaMalloc/cudaFree can cause in the middle of their own asynchronous work.
// ccT_reduce_w_noalloc serves them: it takes W, the orbital energies and the
// VVOO integrals already on the device, accumulates into the caller's etd and
// v1 device buffers, and keeps its per-block partial sums in one fixed array
// in the library's own device memory instead of allocating.
//
// The scratch array g_noalloc_scratch is sized for nu <= CCT_NOALLOC_MAX_NU
// (320): ceil(nu/8) = 40 index blocks give 11480 block triples, each with 1
// energy partial and 72 v1 partials, 6,704,320 bytes in all.  Every GPU that
// loads the library holds that much until the process exits.  All calls share
// the one array and it keeps the last call's contents; each call overwrites the
// partials it reads before reading them, so nothing has to start at zero, but
// two calls whose kernels overlap on the GPU (different streams, no ordering
// between them) race on it.
//
// In host code g_noalloc_scratch names a host-side shadow, not device memory:
// the device address comes from cudaGetSymbolAddress, called once per device
// with that device current, the first time the entry point runs on it.  That
// first call should therefore come before any stream capture.
#include <mutex>

#include "cct_internal.cuh"

namespace cct {
namespace {

constexpr int kMaxNu = CCT_NOALLOC_MAX_NU;
constexpr int kRB2 = 8;
constexpr int kMaxNb = (kMaxNu + kRB2 - 1) / kRB2;
constexpr int64_t kMaxTriples = (int64_t)kMaxNb * (kMaxNb + 1) * (kMaxNb + 2) / 6;
constexpr int64_t kScratchDoubles = kMaxTriples * 73;  // x3 partials, then 72 v1 partials per triple

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double *g_scratch_ptr[kMaxDevices] = {nullptr};

constexpr int NT = 256;
constexpr int SLOT = 640;  // padded 8x8x8 block
__device__ __forceinline__ int boff(int l0, int l1, int l2) { return l0 + 9 * l1 + 81 * l2; }

__constant__ int c_perm6[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

__device__ __forceinline__ int perm_id(int p0, int p1) { return p0 * 2 + ((p1 > p0 ? p1 - 1 : p1)); }

// block triple index -> (A <= B <= C), inverse of idx = C(C+1)(C+2)/6 + B(B+1)/2 + A
__device__ void decode_triple(int64_t idx, int *S) {
  int C = 0;
  while ((int64_t)(C + 1) * (C + 2) * (C + 3) / 6 <= idx) C++;
  idx -= (int64_t)C * (C + 1) * (C + 2) / 6;
  int B = 0;
  while ((int64_t)(B + 1) * (B + 2) / 2 <= idx) B++;
  idx -= (int64_t)B * (B + 1) / 2;
  S[0] = (int)idx;
  S[1] = B;
  S[2] = C;
}

__global__ void __launch_bounds__(NT) noalloc_reduce_kernel(int nu, int no, int i, int j, int k,
                                                           const double *__restrict__ w, const double *__restrict__ eh,
                                                           const double *__restrict__ ep,
                                                           const double *__restrict__ voe, double *__restrict__ xpart,
                                                           double *__restrict__ vpart) {
  __shared__ double Wsm[6 * SLOT];
  __shared__ double vloc[3][kRB2][3];
  __shared__ double red[NT / 32];
  __shared__ int slot_of[6];
  __shared__ int pos_of[3];

  const int tid = threadIdx.x;
  const int64_t cta = blockIdx.x;
  int S[3];
  decode_triple(cta, S);
  if (tid < 6) {
    int slot = tid;
    for (int s2 = 0; s2 < tid; s2++)
      if (S[c_perm6[s2][0]] == S[c_perm6[tid][0]] && S[c_perm6[s2][1]] == S[c_perm6[tid][1]] &&
          S[c_perm6[s2][2]] == S[c_perm6[tid][2]]) {
        slot = s2;
        break;
      }
    slot_of[tid] = slot;
  }
  if (tid < 3) pos_of[tid] = (S[0] == S[tid]) ? 0 : ((S[1] == S[tid]) ? 1 : 2);
  if (tid < 3 * kRB2 * 3) (&vloc[0][0][0])[tid] = 0.0;
  __syncthreads();

  // W(a,b,c) at a + nu*(b + nu*c): a is contiguous, so a is the fastest thread index
  for (int sg = 0; sg < 6; sg++) {
    if (slot_of[sg] != sg) continue;
    const int O0 = S[c_perm6[sg][0]], O1 = S[c_perm6[sg][1]], O2 = S[c_perm6[sg][2]];
    for (int idx = tid; idx < 512; idx += NT) {
      const int l0 = idx & 7, l1 = (idx >> 3) & 7, l2 = idx >> 6;
      const int a = kRB2 * O0 + l0, b = kRB2 * O1 + l1, c = kRB2 * O2 + l2;
      double v = 0.0;
      if (a < nu && b < nu && c < nu && !(a == b && b == c)) v = w[a + (int64_t)nu * (b + (int64_t)nu * c)];
      Wsm[sg * SLOT + boff(l0, l1, l2)] = v;  // W_aaa = 0 (ZEROT3)
    }
  }
  __syncthreads();

  const int warp = tid >> 5, lane = tid & 31;
  const double dijk = eh[i] + eh[j] + eh[k];
  const int64_t nu2 = (int64_t)nu * nu;
  const double *voe_jk = voe + ((int64_t)k * no + j) * nu2, *voe_kj = voe + ((int64_t)j * no + k) * nu2;
  const double *voe_ik = voe + ((int64_t)k * no + i) * nu2, *voe_ki = voe + ((int64_t)i * no + k) * nu2;
  const double *voe_ij = voe + ((int64_t)j * no + i) * nu2, *voe_ji = voe + ((int64_t)i * no + j) * nu2;
  double x3 = 0.0;
  for (int sg = 0; sg < 6; sg++) {
    if (slot_of[sg] != sg) continue;
    const int *sp = c_perm6[sg];
    const int O0 = S[sp[0]], O1 = S[sp[1]], O2 = S[sp[2]];
    const int l0 = warp;
    const int a = kRB2 * O0 + l0;
    double ci = 0.0, cj = 0.0, ck = 0.0;
    for (int h = 0; h < 2; h++) {
      const int pi = lane + 32 * h;
      const int l1 = pi & 7, l2 = pi >> 3;
      const int b = kRB2 * O1 + l1, c = kRB2 * O2 + l2;
      if (a >= nu || b >= nu || c >= nu) continue;
      const int lc[3] = {l0, l1, l2};
      double wp[6];
#pragma unroll
      for (int pp = 0; pp < 6; pp++) {
        const int *q = c_perm6[pp];
        const int comp = perm_id(sp[q[0]], sp[q[1]]);
        wp[pp] = Wsm[slot_of[comp] * SLOT + boff(lc[q[0]], lc[q[1]], lc[q[2]])];
      }
      const double wabc = wp[0], wacb = wp[1], wbac = wp[2], wbca = wp[3], wcab = wp[4], wcba = wp[5];
      const double dinv = 1.0 / (dijk - (ep[a] + ep[b] + ep[c]));
      x3 += wabc * (8.0 * wabc - 4.0 * (wacb + wcba + wbac) + 2.0 * (wbca + wcab)) * dinv;
      const double z1 = (wabc - wbac) * 2.0 - wacb + wbca;
      const double z2 = (wacb - wbca) * 2.0 - wabc + wbac;
      const double z3 = (wbac - wabc) * 2.0 - wcab + wcba;
      const double z4 = (wbca - wacb) * 2.0 - wcba + wcab;
      const double z5 = (wcab - wcba) * 2.0 - wbac + wabc;
      const double z6 = (wcba - wcab) * 2.0 - wbca + wacb;
      const int64_t bc = b + (int64_t)nu * c;
      ci += (z1 * voe_jk[bc] + z2 * voe_kj[bc]) * dinv;
      cj += (z3 * voe_ik[bc] + z5 * voe_ki[bc]) * dinv;
      ck += (z4 * voe_ij[bc] + z6 * voe_ji[bc]) * dinv;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      ci += __shfl_down_sync(0xffffffffu, ci, off);
      cj += __shfl_down_sync(0xffffffffu, cj, off);
      ck += __shfl_down_sync(0xffffffffu, ck, off);
    }
    if (lane == 0) {
      const int pos = pos_of[sp[0]];
      vloc[pos][l0][0] += ci;
      vloc[pos][l0][1] += cj;
      vloc[pos][l0][2] += ck;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) x3 += __shfl_down_sync(0xffffffffu, x3, off);
  if (lane == 0) red[warp] = x3;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int q = 0; q < NT / 32; q++) s += red[q];
    xpart[cta] = s;
  }
  if (tid < 72) vpart[cta * 72 + tid] = (&vloc[0][0][0])[tid];
}

__global__ void noalloc_finalize_kernel(int nu, int nb, int64_t ncta, int i, int j, int k, double weight,
                                        const double *__restrict__ xpart, const double *__restrict__ vpart,
                                        double *__restrict__ etd_acc, double *__restrict__ v1_acc) {
  const int tid = threadIdx.x, lane = tid & 31;
  if (blockIdx.x == 0) {
    __shared__ double red[NT];
    double s = 0.0;
    for (int64_t c = tid; c < ncta; c += NT) s += xpart[c];
    red[tid] = s;
    __syncthreads();
    for (int st = NT / 2; st > 0; st >>= 1) {
      if (tid < st) red[tid] += red[tid + st];
      __syncthreads();
    }
    if (tid == 0) {
      const double v = weight * red[0];
      const double sum = etd_acc[0];
      const double nsum = sum + v;
      const double comp = fabs(sum) >= fabs(v) ? (sum - nsum) + v : (v - nsum) + sum;
      etd_acc[0] = nsum;
      etd_acc[1] += comp;
    }
    return;
  }
  const int a = ((blockIdx.x - 1) * blockDim.x + tid) >> 5;
  if (a >= nu) return;
  const int X = a / kRB2, la = a - (a / kRB2) * kRB2;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  int q = 0;
  for (int Y = 0; Y < nb; Y++)
    for (int Z = Y; Z < nb; Z++, q++) {
      if ((q & 31) != lane) continue;
      int A, B, C;
      if (X <= Y) {
        A = X; B = Y; C = Z;
      } else if (X <= Z) {
        A = Y; B = X; C = Z;
      } else {
        A = Y; B = Z; C = X;
      }
      const int64_t idx = (int64_t)C * (C + 1) * (C + 2) / 6 + (int64_t)B * (B + 1) / 2 + A;
      const int pos = (A == X) ? 0 : ((B == X) ? 1 : 2);
      const double *vp = vpart + idx * 72 + pos * 24 + la * 3;
      s0 += vp[0];
      s1 += vp[1];
      s2 += vp[2];
    }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    s0 += __shfl_down_sync(0xffffffffu, s0, off);
    s1 += __shfl_down_sync(0xffffffffu, s1, off);
    s2 += __shfl_down_sync(0xffffffffu, s2, off);
  }
  if (lane == 0) {
    v1_acc[a + (int64_t)nu * i] += weight * s0;
    v1_acc[a + (int64_t)nu * j] += weight * s1;
    v1_acc[a + (int64_t)nu * k] += weight * s2;
  }
}

// Device address of the scratch array on the current device (set up once per device).
int scratch_on_current_device(double **out) {
  int dev = -1;
  CCT_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal beyond the no-alloc set-up table");
    return CCT_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    double *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&ptr), g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      set_error(std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
      return CCT_ERR_CUDA;
    }
    g_scratch_ptr[dev] = ptr;
  }
  *out = g_scratch_ptr[dev];
  return CCT_OK;
}

}  // namespace
}  // namespace cct

using namespace cct;

extern "C" int ccT_reduce_w_noalloc(int64_t no, int64_t nu, int64_t i, int64_t j, int64_t k, const double *w,
                                    const double *eh, const double *ep, const double *voe, double *etd_acc,
                                    double *v1_acc, void *cuda_stream) {
  if (nu < 1 || nu > kMaxNu) {
    set_error("ccT_reduce_w_noalloc: nu = " + std::to_string(nu) + " outside 1.." + std::to_string(kMaxNu) +
              " (the size its fixed scratch array was built for)");
    return CCT_ERR_INVALID;
  }
  if (no < 2 || !(i >= j && j >= k && k >= 0 && i < no) || (i == j && j == k)) {
    set_error("ccT_reduce_w_noalloc: need 0 <= k <= j <= i < no, not all equal");
    return CCT_ERR_INVALID;
  }
  if (!w || !eh || !ep || !voe || !etd_acc || !v1_acc) {
    set_error("ccT_reduce_w_noalloc: a device pointer is NULL");
    return CCT_ERR_INVALID;
  }
  double *scratch = nullptr;
  CCT_TRY(scratch_on_current_device(&scratch));
  const int nb = (int)((nu + kRB2 - 1) / kRB2);
  const int64_t ncta = (int64_t)nb * (nb + 1) * (nb + 2) / 6;
  double *xpart = scratch;
  double *vpart = scratch + ncta;
  const double weight = (i == j || j == k) ? 0.5 : 1.0;
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  noalloc_reduce_kernel<<<(unsigned)ncta, NT, 0, s>>>((int)nu, (int)no, (int)i, (int)j, (int)k, w, eh, ep, voe,
                                                      xpart, vpart);
  CCT_CUDA(cudaGetLastError());
  const int vblocks = (int)((nu * 32 + NT - 1) / NT);
  noalloc_finalize_kernel<<<1 + vblocks, NT, 0, s>>>((int)nu, nb, ncta, (int)i, (int)j, (int)k, weight, xpart, vpart,
                                                     etd_acc, v1_acc);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}
