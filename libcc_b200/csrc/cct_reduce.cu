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

namespace cct {
namespace {

constexpr int RB = kRB;             // 8
constexpr int RT = 256;             // threads per reduction CTA
constexpr int SL = 640;             // doubles per padded 8x8x8 block in smem
__device__ __forceinline__ int soff(int l0, int l1, int l2) { return l0 + 9 * l1 + 81 * l2; }

// the six permutations of three positions, in a fixed order
__constant__ int c_perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

// W assembly per tuple kind: W(x0,x1,x2) += X_g(x_al0, x_al1, x_al2); {g, al0, al1, al2}
//   i>j>k : X0(a,b,c) + X1(a,c,b) + X2(b,c,a)
//   (i,j,j): X0(a,b,c) + X0(a,c,b) + X1(b,c,a) + X1(c,b,a)
//   (i,i,k): X0(a,b,c) + X0(b,a,c) + X1(a,c,b) + X1(b,c,a)
__constant__ int c_terms[3][4][4] = {
    {{0, 0, 1, 2}, {1, 0, 2, 1}, {2, 1, 2, 0}, {0, 0, 0, 0}},
    {{0, 0, 1, 2}, {0, 0, 2, 1}, {1, 1, 2, 0}, {1, 2, 1, 0}},
    {{0, 0, 1, 2}, {0, 1, 0, 2}, {1, 0, 2, 1}, {1, 1, 2, 0}}};

__device__ __forceinline__ int perm_index(int p0, int p1) {
  // index of the permutation whose first two entries are (p0, p1)
  return p0 * 2 + ((p1 > p0 ? p1 - 1 : p1));
}

constexpr int VSL = 6 * 64;  // staged VOE values per slot: 6 planes x 64 (b,c) pairs

__global__ void __launch_bounds__(RT) reduce_kernel(int nu, int no, int64_t NP, TupleDev t,
                                                   const double *__restrict__ eh, const double *__restrict__ ep,
                                                   const double *__restrict__ voe, const int16_t *__restrict__ table,
                                                   double *__restrict__ xpart, double *__restrict__ vpart) {
  extern __shared__ __align__(16) double dyn_smem[];  // REDUCE_SMEM bytes
  double *Wsm = dyn_smem;                             // [6][SL]
  double *Vsm = dyn_smem + 6 * SL;                    // [6][VSL]
  __shared__ double vloc[3][RB][3];
  __shared__ double red[RT / 32];
  __shared__ int slot_of[6];  // perm sigma -> slot holding block O_sigma
  __shared__ int pos_of[3];   // position m -> first position with the same block

  const int tid = threadIdx.x;
  const int64_t cta = blockIdx.x;
  const int S[3] = {table[3 * cta], table[3 * cta + 1], table[3 * cta + 2]};
  // slots are uniform across the CTA: compute them in registers everywhere
  int slot[6];
#pragma unroll
  for (int sg = 0; sg < 6; sg++) {
    slot[sg] = sg;
#pragma unroll
    for (int s2 = 0; s2 < 6; s2++) {
      if (s2 < sg && slot[sg] == sg && S[c_perm[s2][0]] == S[c_perm[sg][0]] && S[c_perm[s2][1]] == S[c_perm[sg][1]] &&
          S[c_perm[s2][2]] == S[c_perm[sg][2]])
        slot[sg] = s2;
    }
  }
  if (tid < 6) slot_of[tid] = slot[tid];
  if (tid < 3) pos_of[tid] = (S[0] == S[tid]) ? 0 : ((S[1] == S[tid]) ? 1 : 2);
  if (tid < 3 * RB * 3) (&vloc[0][0][0])[tid] = 0.0;

  const int nterm = t.kind == kIJK ? 3 : 4;
  const int64_t nu2 = (int64_t)nu * nu;
  const double *planes[6] = {
      voe + ((int64_t)t.k * no + t.j) * nu2, voe + ((int64_t)t.j * no + t.k) * nu2,   // jk, kj
      voe + ((int64_t)t.k * no + t.i) * nu2, voe + ((int64_t)t.i * no + t.k) * nu2,   // ik, ki
      voe + ((int64_t)t.j * no + t.i) * nu2, voe + ((int64_t)t.i * no + t.j) * nu2};  // ij, ji

  // ---- phase 1: issue every global load of this CTA (X terms, staged VOE)
  double xv[6][4][2];
  double vv[6][2];
#pragma unroll
  for (int sg = 0; sg < 6; sg++) {
    const bool live = slot[sg] == sg;
    const int O[3] = {S[c_perm[sg][0]], S[c_perm[sg][1]], S[c_perm[sg][2]]};
#pragma unroll
    for (int term = 0; term < 4; term++) {
      const int *tm = c_terms[t.kind][term];
      const double *X = t.x[tm[0]];
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int idx = tid + RT * e;
        const int u2 = idx & 7, u1 = (idx >> 3) & 7, u0 = idx >> 6;  // u2: X's contiguous index
        const int xp = RB * O[tm[1]] + u0, xq = RB * O[tm[2]] + u1, xs = RB * O[tm[3]] + u2;
        double v = 0.0;
        if (live && term < nterm && xp < nu && xq < nu && xs < nu) v = X[((int64_t)xp * nu + xq) * NP + xs];
        xv[sg][term][e] = v;
      }
    }
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int q = tid + RT * e;  // < 512; only q < VSL used
      const int plane = q >> 6, pair = q & 63;
      const int b = RB * O[1] + (pair & 7), c = RB * O[2] + (pair >> 3);
      double v = 0.0;
      if (live && q < VSL && b < nu && c < nu) v = planes[plane][b + (int64_t)nu * c];
      vv[sg][e] = v;
    }
  }

  // ---- phase 2: assemble W in shared memory, one term at a time (fixed order)
#pragma unroll
  for (int term = 0; term < 4; term++) {
    if (term < nterm) {
#pragma unroll
      for (int sg = 0; sg < 6; sg++) {
        if (slot[sg] != sg) continue;
        const int *tm = c_terms[t.kind][term];
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int idx = tid + RT * e;
          const int u2 = idx & 7, u1 = (idx >> 3) & 7, u0 = idx >> 6;
          int l[3];
          l[tm[1]] = u0;
          l[tm[2]] = u1;
          l[tm[3]] = u2;
          double *w = Wsm + sg * SL + soff(l[0], l[1], l[2]);
          if (term == 0)
            *w = xv[sg][term][e];
          else
            *w += xv[sg][term][e];
        }
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int sg = 0; sg < 6; sg++) {
    if (slot[sg] != sg) continue;
#pragma unroll
    for (int e = 0; e < 2; e++) {
      const int q = tid + RT * e;
      if (q < VSL) Vsm[sg * VSL + q] = vv[sg][e];
    }
  }
  // W_aaa = 0 (ZEROT3): only the all-equal block triple holds diagonal elements
  if (S[0] == S[1] && S[1] == S[2] && tid < RB) Wsm[soff(tid, tid, tid)] = 0.0;
  __syncthreads();

  // ---- phase 3: energy and v1 contributions, all from shared memory
  const int warp = tid >> 5, lane = tid & 31;
  const double dijk = eh[t.i] + eh[t.j] + eh[t.k];
  double x3 = 0.0;
  for (int sg = 0; sg < 6; sg++) {
    if (slot_of[sg] != sg) continue;
    const int *sp = c_perm[sg];
    const int O[3] = {S[sp[0]], S[sp[1]], S[sp[2]]};
    const int l0 = warp;
    const int a = RB * O[0] + l0;
    const double epa = a < nu ? ep[a] : 0.0;
    double ci = 0.0, cj = 0.0, ck = 0.0;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int pi = lane + 32 * h;
      const int l1 = pi & 7, l2 = pi >> 3;
      const int b = RB * O[1] + l1, c = RB * O[2] + l2;
      if (a < nu && b < nu && c < nu) {
        const int lc[3] = {l0, l1, l2};
        double w[6];
#pragma unroll
        for (int pp = 0; pp < 6; pp++) {
          const int *pi3 = c_perm[pp];
          const int comp = perm_index(sp[pi3[0]], sp[pi3[1]]);  // block of the permuted element
          w[pp] = Wsm[slot_of[comp] * SL + soff(lc[pi3[0]], lc[pi3[1]], lc[pi3[2]])];
        }
        // w[0]=abc w[1]=acb w[2]=bac w[3]=bca w[4]=cab w[5]=cba
        const double wabc = w[0], wacb = w[1], wbac = w[2], wbca = w[3], wcab = w[4], wcba = w[5];
        const double dinv = 1.0 / (dijk - (epa + ep[b] + ep[c]));
        x3 += wabc * (8.0 * wabc - 4.0 * (wacb + wcba + wbac) + 2.0 * (wbca + wcab)) * dinv;
        const double z1 = (wabc - wbac) * 2.0 - wacb + wbca;
        const double z2 = (wacb - wbca) * 2.0 - wabc + wbac;
        const double z3 = (wbac - wabc) * 2.0 - wcab + wcba;
        const double z4 = (wbca - wacb) * 2.0 - wcba + wcab;
        const double z5 = (wcab - wcba) * 2.0 - wbac + wabc;
        const double z6 = (wcba - wcab) * 2.0 - wbca + wacb;
        const double *vs = Vsm + sg * VSL + pi;
        ci += (z1 * vs[0] + z2 * vs[64]) * dinv;
        cj += (z3 * vs[128] + z5 * vs[192]) * dinv;
        ck += (z4 * vs[256] + z6 * vs[320]) * dinv;
      }
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

  // ---- CTA partials: warp trees then a fixed-order sum of the 8 warp values
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) x3 += __shfl_down_sync(0xffffffffu, x3, off);
  if (lane == 0) red[warp] = x3;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int w = 0; w < RT / 32; w++) s += red[w];
    xpart[cta] = s;
  }
  if (tid < 3 * RB * 3) vpart[cta * 72 + tid] = (&vloc[0][0][0])[tid];
}

// etd_acc[0..1]: Neumaier (sum, compensation); v1_acc(nu, no).
// Block 0 sums the per-CTA x3 partials; every other warp owns one virtual
// index a and sums its v1 partials over all block triples containing a.
__global__ void finalize_kernel(int nu, int nb, int64_t ncta, TupleDev t, const double *__restrict__ xpart,
                                const double *__restrict__ vpart, double *__restrict__ etd_acc,
                                double *__restrict__ v1_acc) {
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  if (blockIdx.x == 0) {
    __shared__ double red[256];
    double s = 0.0;
    for (int64_t c = tid; c < ncta; c += 256) s += xpart[c];
    red[tid] = s;
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
  const int a = ((blockIdx.x - 1) * blockDim.x + tid) >> 5;
  if (a >= nu) return;
  const int X = a / RB, la = a - (a / RB) * RB;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  int q = 0;
  for (int Y = 0; Y < nb; Y++) {
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
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    s0 += __shfl_down_sync(0xffffffffu, s0, off);
    s1 += __shfl_down_sync(0xffffffffu, s1, off);
    s2 += __shfl_down_sync(0xffffffffu, s2, off);
  }
  if (lane == 0) {
    v1_acc[a + (int64_t)nu * t.i] += t.weight * s0;
    v1_acc[a + (int64_t)nu * t.j] += t.weight * s1;
    v1_acc[a + (int64_t)nu * t.k] += t.weight * s2;
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

int launch_reduce(const Dims &d, const TupleDev &t, const double *eh, const double *ep, const double *voe,
                  const int16_t *cta_table, double *xpart, double *vpart, cudaStream_t s) {
  constexpr int smem = (6 * SL + 6 * VSL) * 8;
  static int configured_device = -1;
  int dev = 0;
  CCT_CUDA(cudaGetDevice(&dev));
  if (configured_device != dev) {
    CCT_CUDA(cudaFuncSetAttribute(reduce_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    configured_device = dev;
  }
  reduce_kernel<<<(unsigned)d.ncta, RT, smem, s>>>(d.nu, d.no, d.NP, t, eh, ep, voe, cta_table, xpart, vpart);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

int launch_finalize(const Dims &d, const TupleDev &t, const double *xpart, const double *vpart, double *etd_acc,
                    double *v1_acc, cudaStream_t s) {
  const int vblocks = (d.nu * 32 + 255) / 256;  // one warp per virtual index
  finalize_kernel<<<1 + vblocks, 256, 0, s>>>(d.nu, d.nb, d.ncta, t, xpart, vpart, etd_acc, v1_acc);
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
