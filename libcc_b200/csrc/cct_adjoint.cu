// Adjoint of the (T) energy: dE(T)/d{eh, ep, T1, T2, VM, VOE, VVVO}.
//
// Per tuple (i,j,k) with weight w (1, or 1/2 for degenerate tuples) and
// d = 1/D_abc, the forward computes (reduction of cct_reduce.cu, the full-sum
// form of t1wt3.f90:46-95 and triples.F90:311-312)
//   E_t = w sum_abc [ W (P W) + sum_m z_m S_m ] d,
//   P W = 8 W_abc - 4 (W_acb + W_cba + W_bac) + 2 (W_bca + W_cab),
//   S_m(a,b,c) = u_x(a) VOE(b,c,y,z),  u_x(a) = 2 T1(x,a),
//   (m; x,y,z) = (1; i,j,k) (2; i,k,j) (3; j,i,k) (4; k,i,j) (5; j,k,i) (6; k,j,i),
// with z_1..z_6 the combinations of t1wt3.f90:80-85.  Because D is symmetric in
// (a,b,c), P is self-adjoint and a W at a permuted index can be moved onto S:
//   dE/dW = w d (2 P W + H),   H = sum_m sum_pi c_pi S_m(pi^-1)     (adj_gw_kernel)
//   dE/dVOE(b,c,y,z) = w sum_a z_m(a,b,c) u_x(a) d      (adj_gw_kernel + adj_voe_sum_kernel)
//   dE/deh_x = -(multiplicity of x in ijk) sum_abc M,  dE/dep_p = sum over the
//   three index positions of M restricted to p,  M = w W (P W + H) d^2
//   (partial sums in adj_gw_kernel, adj_eps_sum_kernel, adj_eps_total_kernel)
//   dE/dT1(x,a) = 2 v1(a,x)                                          (adj_finish)
// W is recomputed per tuple by the forward GEMMs (nothing of size nu^3 is kept
// across tuples).  The W-build GEMM X_g(p,q,s) = sum_h sum_k E[x_h][perm_h(p,q)][k]
// F[fyz_h][s][k] is bilinear, so with G_g = dE/dX_g:
//   dE[x_h][perm_h(r)] += G_g(r,:) F[fyz_h]          (bwd_e_kernel, K = NP)
//   dF[fyz_h]          += G_g^T E[x_h][perm_h(.)]     (bwd_f_kernel, K = nu^2, split-K)
// and dE, dF are scattered back onto packed VVVO, T2 and VM (adj_scatter_*), the
// adjoint of cct_layout.cu.  All sums run in a fixed order (no floating-point
// atomics): gradients are bitwise reproducible.
#include <algorithm>
#include <type_traits>

#include "cct_internal.cuh"

namespace cct {
namespace {

__host__ __device__ constexpr int term_entry(int kind, int term, int f) {
  // W(x0,x1,x2) += X_g(x_al0, x_al1, x_al2): {g, al0, al1, al2} (same table as cct_reduce.cu)
  constexpr int tab[3][4][4] = {{{0, 0, 1, 2}, {1, 0, 2, 1}, {2, 1, 2, 0}, {0, 0, 0, 0}},
                                {{0, 0, 1, 2}, {0, 0, 2, 1}, {1, 1, 2, 0}, {1, 2, 1, 0}},
                                {{0, 0, 1, 2}, {0, 1, 0, 2}, {1, 0, 2, 1}, {1, 1, 2, 0}}};
  return tab[kind][term][f];
}
__host__ __device__ constexpr int nterms(int kind) { return kind == kIJK ? 3 : 4; }

struct AdjTuple {
  const double *x[3];
  int i, j, k;
  double weight;
};

__device__ __forceinline__ int64_t widx(int nu, int a, int b, int c) { return ((int64_t)a * nu + b) * nu + c; }

// ---------------------------------------------------------------------------- W assembly
// Grids of the dense nu^3 kernels: x = 128-wide blocks of c, y = b, z = a.
// W(a,b,c) = sum over the terms of X_g at a permutation of (a,b,c), for one
// tile a in [a0, a0+8), b in [b0, b0+8), c in [c0, c0+32) per CTA (grid x: c
// blocks, y: b blocks, z: a blocks).  Each term's X tile is staged in shared
// memory by coalesced asynchronous copies in its own index order (innermost
// extent and plane padded by one), then summed and written as 256-byte rows.
constexpr int kWA = 8, kWB = 8, kWC = 32;
constexpr int kWThreads = 256;
#ifndef CCT_BWD_F_CTAS_PER_SM
#define CCT_BWD_F_CTAS_PER_SM 3
#endif
constexpr int kWSlot = 2336;  // >= D0 * (D1 * (D2 + 1) + 1) for every order of (8, 8, 32)

__host__ __device__ constexpr int wf_ext(int pos) { return pos == 2 ? kWC : (pos == 1 ? kWB : kWA); }

template <int KIND, int TERM>
__device__ __forceinline__ void wf_load_term(double *dst, const AdjTuple &t, int nu, int64_t NP, const int o[3]) {
  constexpr int g = term_entry(KIND, TERM, 0);
  constexpr int p0 = term_entry(KIND, TERM, 1), p1 = term_entry(KIND, TERM, 2), p2 = term_entry(KIND, TERM, 3);
  constexpr int D0 = wf_ext(p0), D1 = wf_ext(p1), D2 = wf_ext(p2), PL = D1 * (D2 + 1) + 1;
  const double *X = t.x[g];
#pragma unroll
  for (int e = threadIdx.x; e < D0 * D1 * D2; e += kWThreads) {
    const int k = e % D2, j = (e / D2) % D1, i = e / (D1 * D2);
    const int x0 = o[p0] + i, x1 = o[p1] + j, x2 = o[p2] + k;
    const bool ok = x0 < nu && x1 < nu && x2 < nu;
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst + i * PL + j * (D2 + 1) + k);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa),
                 "l"(X + (ok ? ((int64_t)x0 * nu + x1) * NP + x2 : 0)), "r"(ok ? 8 : 0));
  }
}

template <int KIND, int TERM>
__device__ __forceinline__ double wf_term(const double *src, const int l[3]) {
  constexpr int p0 = term_entry(KIND, TERM, 1), p1 = term_entry(KIND, TERM, 2), p2 = term_entry(KIND, TERM, 3);
  constexpr int D1 = wf_ext(p1), D2 = wf_ext(p2), PL = D1 * (D2 + 1) + 1;
  return src[l[p0] * PL + l[p1] * (D2 + 1) + l[p2]];
}

template <int KIND>
__global__ void __launch_bounds__(kWThreads) adj_wfull_kernel(int nu, int64_t NP, AdjTuple t,
                                                              double *__restrict__ Wf) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *S = reinterpret_cast<double *>(smem_raw);
  const int o[3] = {(int)blockIdx.z * kWA, (int)blockIdx.y * kWB, (int)blockIdx.x * kWC};
  wf_load_term<KIND, 0>(S, t, nu, NP, o);
  wf_load_term<KIND, 1>(S + kWSlot, t, nu, NP, o);
  wf_load_term<KIND, 2>(S + 2 * kWSlot, t, nu, NP, o);
  if (nterms(KIND) > 3) wf_load_term<KIND, (nterms(KIND) > 3 ? 3 : 0)>(S + 3 * kWSlot, t, nu, NP, o);
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();
  const int al = threadIdx.x >> 5, cl = threadIdx.x & 31;
  const int a = o[0] + al, c = o[2] + cl;
  if (a >= nu || c >= nu) return;
#pragma unroll
  for (int bl = 0; bl < kWB; bl++) {
    const int b = o[1] + bl;
    if (b >= nu) break;
    const int l[3] = {al, bl, cl};
    double w = wf_term<KIND, 0>(S, l) + wf_term<KIND, 1>(S + kWSlot, l);
    w += wf_term<KIND, 2>(S + 2 * kWSlot, l);
    if (nterms(KIND) > 3) w += wf_term<KIND, (nterms(KIND) > 3 ? 3 : 0)>(S + 3 * kWSlot, l);
    Wf[widx(nu, a, b, c)] = (a == b && b == c) ? 0.0 : w;
  }
}

// W in the reference's layout: wf[(c nu + b) nu + a] = wc[(a nu + b) nu + c],
// one 32 x 32 (a, c) tile of one b per block.
__global__ void w_fortran_kernel(int nu, const double *__restrict__ wc, double *__restrict__ wf) {
  __shared__ double tile[32][33];
  const int b = blockIdx.z, a0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int a = a0 + r, c = c0 + threadIdx.x;
    tile[r][threadIdx.x] = (a < nu && c < nu) ? wc[widx(nu, a, b, c)] : 0.0;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int c = c0 + r, a = a0 + threadIdx.x;
    if (a < nu && c < nu) wf[((int64_t)c * nu + b) * nu + a] = tile[threadIdx.x][r];
  }
}

// ---------------------------------------------------------------------------- dE/dW and M
// S_m at the permuted triple (r0,r1,r2) of (a,b,c): u_x(r0) VOE(r1,r2,y,z).
struct SmTable {
  int x[6], y[6], z[6];
};

// H = sum_m sum_pi c_pi S_m(pi^-1) regrouped by which occupied role R (i, j, k)
// feeds u and at which position p0 of (a,b,c) u is evaluated:
//   H(a,b,c) = sum_R [ u_R(a) Q_R0(b,c) + u_R(b) Q_R1(a,c) + u_R(c) Q_R2(a,b) ],
// each Q a signed sum of VOE planes, some transposed (built per tuple by adj_q_kernel).
constexpr int kQTerms = 8;
struct QTable {
  int n[9];
  int coef[9][kQTerms];
  int64_t plane[9][kQTerms];  // offset of VOE(., ., y, z)
  int trans[9][kQTerms];      // 1: the plane is read as V(s, r)
};

__global__ void adj_q_kernel(int nu, QTable q, const double *__restrict__ voe, double *__restrict__ Q) {
  const int64_t nu2 = (int64_t)nu * nu;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < 9 * nu2; e += (int64_t)gridDim.x * blockDim.x) {
    const int g = (int)(e / nu2);
    const int64_t rs = e - (int64_t)g * nu2;
    const int r = (int)(rs / nu), sidx = (int)(rs - (int64_t)r * nu);
    double v = 0.0;
    for (int u = 0; u < q.n[g]; u++) {
      const double *pl = voe + q.plane[g][u];
      v += (double)q.coef[g][u] * (q.trans[g][u] ? pl[(int64_t)r * nu + sidx] : pl[(int64_t)sidx * nu + r]);
    }
    Q[e] = v;  // Q[g][r][s]
  }
}

// One CTA of 256 threads per tile a in [a0, a0+16), b in [b0, b0+8), c in
// [c0, c0+8) (grid x: c blocks, y: b blocks, z: a chunks).  The six index
// permutations of W the tile needs, u_R(a), ep(a) and the Q_R1(a,c), Q_R2(a,b)
// blocks are staged in shared memory by coalesced asynchronous copies, so no
// W read is strided and the inner loop reads no global memory.  A tile of
// extents (D0, D1, D2) keeps element (i,j,k) at i*(D1*(D2+1)+1) + j*(D2+1) + k:
// both pads are odd, so the strided tile reads of a half-warp spread over the
// banks.  61 KB of shared memory: three CTAs per SM.  Thread (ag, b, c) forms
// dE/dW and M for the four a of its group; then the CTA
//   - writes dE/dW: for i>j>k tuples straight into the three dE/dX buffers,
//     G0(a,b,c) = G1(a,c,b) = G2(b,c,a) = dE/dW(a,b,c), each as row segments
//     (their padding columns stay zero from allocation); for degenerate
//     tuples into GW, which adj_gx_kernel folds,
//   - stores s_m(b,c) = sum_a z_m(a,b,c) u_x(a) d over its 16 a into
//     vpart[chunk][m][c][b] (adj_voe_sum_kernel adds the chunks in order),
//   - sums M over each pair of tile axes into the eps partials
//     EA[bblk][cblk][a], EB[chunk][cblk][b], EC[chunk][bblk][c].
// Every sum runs in a fixed order.
constexpr int kTA = 16, kTB = 8;
constexpr int kAChunk = kTA;
constexpr int kGwThreads = 256;
constexpr int kGwPer = kTA * kTB * kTB / kGwThreads;  // a per thread
template <int D1, int D2>
__device__ __forceinline__ int tix(int i, int j, int k) {
  return i * (D1 * (D2 + 1) + 1) + j * (D2 + 1) + k;
}
template <int D0, int D1, int D2>
constexpr int tsize() { return D0 * (D1 * (D2 + 1) + 1); }
constexpr int kTabc = tsize<kTA, kTB, kTB>();  // W(a,b,c), W(a,c,b)
constexpr int kTbac = tsize<kTB, kTA, kTB>();  // W(b,a,c), W(c,a,b)
constexpr int kTbca = tsize<kTB, kTB, kTA>();  // W(b,c,a), W(c,b,a)
constexpr int kGwSmem = (2 * (kTabc + kTbac + kTbca) + 4 * kTA + 6 * kTA * kTB) * 8;
static_assert(2 * kTbac >= 4 * 6 * 64, "s_m staging fits the W(b,a,c), W(c,a,b) tiles");
static_assert(kTbca >= 2 * kTA * kTB, "M pair sums fit the W(b,c,a) tile");

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem, bool ok) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(ok ? 8 : 0));
}

// Asynchronous 8-byte copies (zero fill outside the nu^3 box): all tiles' loads
// are in flight at once.
template <int D0, int D1, int D2>
__device__ __forceinline__ void gw_load_tile(double *dst, const double *__restrict__ W, int nu, int o0, int o1,
                                             int o2) {
#pragma unroll
  for (int e = threadIdx.x; e < D0 * D1 * D2; e += kGwThreads) {
    const int k = e % D2, j = (e / D2) % D1, i = e / (D1 * D2);
    const int x0 = o0 + i, x1 = o1 + j, x2 = o2 + k;
    const bool ok = x0 < nu && x1 < nu && x2 < nu;
    cp_async8(dst + tix<D1, D2>(i, j, k), W + (ok ? widx(nu, x0, x1, x2) : 0), ok);
  }
}

template <bool SCATTER>
__global__ void __launch_bounds__(kGwThreads, 3)
    adj_gw_kernel(int nu, int no, int64_t NP, AdjTuple t, const double *__restrict__ Wf,
                  const double *__restrict__ eh, const double *__restrict__ ep, const double *__restrict__ t1,
                  const double *__restrict__ Q, double *__restrict__ GW, double *__restrict__ G0,
                  double *__restrict__ G1, double *__restrict__ G2, double *__restrict__ vpart,
                  double *__restrict__ EA, double *__restrict__ EB, double *__restrict__ EC) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *T0 = reinterpret_cast<double *>(smem_raw);  // W(a,b,c) [a][b][c]
  double *T1 = T0 + kTabc;                             // W(a,c,b) [a][c][b]
  double *T2 = T1 + kTabc;                             // W(b,a,c) [b][a][c]
  double *T4 = T2 + kTbac;                             // W(c,a,b) [c][a][b]
  double *T3 = T4 + kTbac;                             // W(b,c,a) [b][c][a]
  double *T5 = T3 + kTbca;                             // W(c,b,a) [c][b][a]
  double *Ua = T5 + kTbca;                             // [3][kTA] u_R(a), then [kTA] ep(a)
  double *Q1s = Ua + 4 * kTA;                          // [3][kTA][8] Q_R1(a, c)
  double *Q2s = Q1s + 3 * kTA * kTB;                   // [3][kTA][8] Q_R2(a, b)
  const int64_t nu2 = (int64_t)nu * nu;
  const int nb = (nu + kTB - 1) / kTB;
  const int cblk = blockIdx.x, bblk = blockIdx.y, ach = blockIdx.z;
  const int c0 = cblk * kTB, b0 = bblk * kTB, a0 = ach * kTA;
  const int tid = threadIdx.x;
  const int xr[3] = {t.i, t.j, t.k};

  gw_load_tile<kTA, kTB, kTB>(T0, Wf, nu, a0, b0, c0);
  gw_load_tile<kTA, kTB, kTB>(T1, Wf, nu, a0, c0, b0);
  gw_load_tile<kTB, kTA, kTB>(T2, Wf, nu, b0, a0, c0);
  gw_load_tile<kTB, kTA, kTB>(T4, Wf, nu, c0, a0, b0);
  gw_load_tile<kTB, kTB, kTA>(T3, Wf, nu, b0, c0, a0);
  gw_load_tile<kTB, kTB, kTA>(T5, Wf, nu, c0, b0, a0);
  for (int e = tid; e < 6 * kTA * kTB; e += kGwThreads) {  // Q_R1(a, c0+x), Q_R2(a, b0+x)
    const int x = e % kTB, al = (e / kTB) % kTA, RR = e / (kTA * kTB);  // RR = 0..5
    const int R = RR % 3, which = RR / 3;
    const int a = a0 + al, y = (which ? b0 : c0) + x;
    const bool ok = a < nu && y < nu;
    cp_async8(Q1s + e, Q + (ok ? (int64_t)(3 * R + 1 + which) * nu2 + (int64_t)a * nu + y : 0), ok);
  }
  asm volatile("cp.async.commit_group;\n" ::);
  if (tid < kTA) {
    const int a = a0 + tid < nu ? a0 + tid : 0;
#pragma unroll
    for (int R = 0; R < 3; R++) Ua[R * kTA + tid] = 2.0 * t1[xr[R] + (int64_t)no * a];
    Ua[3 * kTA + tid] = ep[a];
  }

  const int ag = tid >> 6, bl = (tid >> 3) & 7, cl = tid & 7;
  const int b = b0 + bl, c = c0 + cl;
  const bool bc_ok = b < nu && c < nu;
  const int bs = bc_ok ? b : 0, cs = bc_ok ? c : 0;  // clamped for the per-thread loads
  const double dijk = eh[t.i] + eh[t.j] + eh[t.k];
  double qb0[3], ub[3], uc[3];
#pragma unroll
  for (int R = 0; R < 3; R++) {
    qb0[R] = Q[(int64_t)(3 * R) * nu2 + (int64_t)bs * nu + cs];  // Q_R0(b,c)
    ub[R] = 2.0 * t1[xr[R] + (int64_t)no * bs];
    uc[R] = 2.0 * t1[xr[R] + (int64_t)no * cs];
  }
  const double ebc = ep[bs] + ep[cs];
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();

  double s[6] = {0, 0, 0, 0, 0, 0};
  double gv[kGwPer], mv[kGwPer];
#pragma unroll
  for (int ia = 0; ia < kGwPer; ia++) {
    const int al = ag * kGwPer + ia, a = a0 + al;
    gv[ia] = 0.0;
    mv[ia] = 0.0;
    if (!bc_ok || a >= nu) continue;
    const double wabc = T0[tix<kTB, kTB>(al, bl, cl)];
    const double wacb = T1[tix<kTB, kTB>(al, cl, bl)];
    const double wbac = T2[tix<kTA, kTB>(bl, al, cl)];
    const double wcab = T4[tix<kTA, kTB>(cl, al, bl)];
    const double wbca = T3[tix<kTB, kTA>(bl, cl, al)];
    const double wcba = T5[tix<kTB, kTA>(cl, bl, al)];
    const double pw = 8.0 * wabc - 4.0 * (wacb + wcba + wbac) + 2.0 * (wbca + wcab);
    const double d = 1.0 / (dijk - (Ua[3 * kTA + al] + ebc));
    double h = 0.0;
    double ua[3];
#pragma unroll
    for (int R = 0; R < 3; R++) {
      ua[R] = Ua[R * kTA + al];
      h += ua[R] * qb0[R];
      h += ub[R] * Q1s[(R * kTA + al) * kTB + cl];
      h += uc[R] * Q2s[(R * kTA + al) * kTB + bl];
    }
    const bool diag = (a == b && b == c);
    gv[ia] = diag ? 0.0 : t.weight * d * (2.0 * pw + h);
    mv[ia] = diag ? 0.0 : t.weight * wabc * (pw + h) * d * d;
    const double z[6] = {(wabc - wbac) * 2.0 - wacb + wbca, (wacb - wbca) * 2.0 - wabc + wbac,
                         (wbac - wabc) * 2.0 - wcab + wcba, (wbca - wacb) * 2.0 - wcba + wcab,
                         (wcab - wcba) * 2.0 - wbac + wabc, (wcba - wcab) * 2.0 - wbca + wacb};
    // z_1..z_6 take u from the roles i, i, j, k, j, k
    constexpr int role[6] = {0, 0, 1, 2, 1, 2};
#pragma unroll
    for (int m = 0; m < 6; m++) s[m] = fma(z[m] * d, ua[role[m]], s[m]);
  }
  __syncthreads();  // the W tiles are dead from here on
  double *Gs = T0, *Ms = T1, *Sv = T2, *Rab = T3, *Rac = T3 + kTA * kTB;
#pragma unroll
  for (int ia = 0; ia < kGwPer; ia++) {
    const int al = ag * kGwPer + ia;
    Gs[tix<kTB, kTB>(al, bl, cl)] = gv[ia];
    Ms[tix<kTB, kTB>(al, bl, cl)] = mv[ia];
  }
#pragma unroll
  for (int m = 0; m < 6; m++) Sv[(ag * 6 + m) * 64 + bl * 8 + cl] = s[m];
  __syncthreads();

  // s_m over the chunk: the four a groups in order
  for (int e = tid; e < 6 * 64; e += kGwThreads) {
    const int m = e >> 6, r = e & 63, bj = r & 7, cj = r >> 3;
    const double v = ((Sv[(0 * 6 + m) * 64 + bj * 8 + cj] + Sv[(1 * 6 + m) * 64 + bj * 8 + cj]) +
                      Sv[(2 * 6 + m) * 64 + bj * 8 + cj]) +
                     Sv[(3 * 6 + m) * 64 + bj * 8 + cj];
    if (b0 + bj < nu && c0 + cj < nu) vpart[((int64_t)ach * 6 + m) * nu2 + (int64_t)(c0 + cj) * nu + b0 + bj] = v;
  }
  // M over pairs of tile axes
  if (tid < kTA * kTB) {
    const int al = tid >> 3, x = tid & 7;
    double rb = 0.0, rc = 0.0;
#pragma unroll
    for (int y = 0; y < kTB; y++) {
      rb += Ms[tix<kTB, kTB>(al, x, y)];  // sum over c at b = x
      rc += Ms[tix<kTB, kTB>(al, y, x)];  // sum over b at c = x
    }
    Rab[al * kTB + x] = rb;
    Rac[al * kTB + x] = rc;
  }
  // dE/dX (or dE/dW) as row segments
  for (int e = tid; e < kTA * kTB * kTB; e += kGwThreads) {
    if (SCATTER) {
      {  // G0(a,b,c): c fastest
        const int cj = e & 7, bj = (e >> 3) & 7, aj = e >> 6;
        const int A = a0 + aj, B = b0 + bj, C = c0 + cj;
        if (A < nu && B < nu && C < nu) G0[((int64_t)A * nu + B) * NP + C] = Gs[tix<kTB, kTB>(aj, bj, cj)];
      }
      {  // G1(a,c,b): b fastest
        const int bj = e & 7, cj = (e >> 3) & 7, aj = e >> 6;
        const int A = a0 + aj, B = b0 + bj, C = c0 + cj;
        if (A < nu && B < nu && C < nu) G1[((int64_t)A * nu + C) * NP + B] = Gs[tix<kTB, kTB>(aj, bj, cj)];
      }
      {  // G2(b,c,a): a fastest
        const int aj = e % kTA, cj = (e / kTA) & 7, bj = e / (kTA * kTB);
        const int A = a0 + aj, B = b0 + bj, C = c0 + cj;
        if (A < nu && B < nu && C < nu) G2[((int64_t)B * nu + C) * NP + A] = Gs[tix<kTB, kTB>(aj, bj, cj)];
      }
    } else {
      const int cj = e & 7, bj = (e >> 3) & 7, aj = e >> 6;
      const int A = a0 + aj, B = b0 + bj, C = c0 + cj;
      if (A < nu && B < nu && C < nu) GW[widx(nu, A, B, C)] = Gs[tix<kTB, kTB>(aj, bj, cj)];
    }
  }
  __syncthreads();
  if (tid < kTA) {  // EA: sum over (b, c) per a
    double v = 0.0;
#pragma unroll
    for (int y = 0; y < kTB; y++) v += Rab[tid * kTB + y];
    if (a0 + tid < nu) EA[((int64_t)bblk * nb + cblk) * nu + a0 + tid] = v;
  } else if (tid >= 64 && tid < 64 + kTB) {  // EB: sum over (a, c) per b
    const int x = tid - 64;
    double v = 0.0;
    for (int al = 0; al < kTA; al++) v += Rab[al * kTB + x];
    if (b0 + x < nu) EB[((int64_t)ach * nb + cblk) * nu + b0 + x] = v;
  } else if (tid >= 128 && tid < 128 + kTB) {  // EC: sum over (a, b) per c
    const int x = tid - 128;
    double v = 0.0;
    for (int al = 0; al < kTA; al++) v += Rac[al * kTB + x];
    if (c0 + x < nu) EC[((int64_t)ach * nb + bblk) * nu + c0 + x] = v;
  }
}

// dVOE(b,c,y_m,z_m) += w sum_chunks vpart[chunk][m][c][b], m = 1..6 in order
// (planes of a degenerate tuple may coincide, so one thread owns all six).
// The chunks are summed in order; 24 loads (four chunks of all six m) are in
// flight at a time.
__global__ void adj_voe_sum_kernel(int nu, int no, int nchunk, AdjTuple t, SmTable sm,
                                   const double *__restrict__ vpart, double *__restrict__ gvoe) {
  constexpr int U = 4;
  const int64_t nu2 = (int64_t)nu * nu;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nu2; e += (int64_t)gridDim.x * blockDim.x) {
    // e = c*nu + b
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    int ch = 0;
    for (; ch + U <= nchunk; ch += U) {
      double x[6 * U];  // flat: [m][u]
#pragma unroll
      for (int m = 0; m < 6; m++)
#pragma unroll
        for (int u = 0; u < U; u++) x[m * U + u] = vpart[((int64_t)(ch + u) * 6 + m) * nu2 + e];
#pragma unroll
      for (int m = 0; m < 6; m++)
#pragma unroll
        for (int u = 0; u < U; u++) v[m] += x[m * U + u];
    }
    for (; ch < nchunk; ch++)
#pragma unroll
      for (int m = 0; m < 6; m++) v[m] += vpart[((int64_t)ch * 6 + m) * nu2 + e];
#pragma unroll
    for (int m = 0; m < 6; m++) gvoe[((int64_t)sm.z[m] * no + sm.y[m]) * nu2 + e] += t.weight * v[m];
  }
}

// ---------------------------------------------------------------------------- dE/dX
// G_g(y0,y1,y2) = sum over the terms of X_g of GW at x with x[al_r] = y_r;
// columns y2 >= nu of the padded rows are zero.
template <int KIND>
__global__ void adj_gx_kernel(int nu, int64_t NP, const double *__restrict__ GW, double *G0, double *G1, double *G2) {
  double *G[3] = {G0, G1, G2};
  const int y2 = blockIdx.x * blockDim.x + threadIdx.x, y1 = blockIdx.y, y0 = blockIdx.z;
  if (y2 < NP) {
    const int64_t e = ((int64_t)y0 * nu + y1) * NP + y2;
    double acc[3] = {0.0, 0.0, 0.0};
    if (y2 < nu) {
      const int ys[3] = {y0, y1, y2};
#pragma unroll
      for (int term = 0; term < nterms(KIND); term++) {
        const int g = term_entry(KIND, term, 0);
        int x[3];
        x[term_entry(KIND, term, 1)] = ys[0];
        x[term_entry(KIND, term, 2)] = ys[1];
        x[term_entry(KIND, term, 3)] = ys[2];
        acc[g] += GW[widx(nu, x[0], x[1], x[2])];
      }
    }
    const int ng = KIND == kIJK ? 3 : 2;
#pragma unroll
    for (int g = 0; g < 3; g++)
      if (g < ng) G[g][e] = acc[g];
  }
}

// ---------------------------------------------------------------------------- eps
// dE/dep_p = sum_bc M(p,b,c) + sum_ac M(a,p,c) + sum_ab M(a,b,p) and
// dE/deh_x -= (multiplicity of x) sum_abc M, from the per-tile partials of
// adj_gw_kernel: a warp per p adds EA[.][.][p], EB[.][.][p], EC[.][.][p] (lanes
// stride the partials, then a fixed shuffle tree), and Rp[p] = the EA part.
__global__ void adj_eps_sum_kernel(int nu, int nb, int nch, const double *__restrict__ EA,
                                   const double *__restrict__ EB, const double *__restrict__ EC,
                                   double *__restrict__ gep, double *__restrict__ Rp) {
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (p >= nu) return;
  double va = 0.0, vb = 0.0, vc = 0.0;
  for (int q = lane; q < nb * nb; q += 32) va += EA[(int64_t)q * nu + p];
  for (int q = lane; q < nch * nb; q += 32) {
    vb += EB[(int64_t)q * nu + p];
    vc += EC[(int64_t)q * nu + p];
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    va += __shfl_xor_sync(0xffffffffu, va, off);
    vb += __shfl_xor_sync(0xffffffffu, vb, off);
    vc += __shfl_xor_sync(0xffffffffu, vc, off);
  }
  if (lane == 0) {
    gep[p] += (va + vb) + vc;
    Rp[p] = va;
  }
}

// One warp: sum_abc M = sum_p R1[p], subtracted from eh_i, eh_j, eh_k.
__global__ void adj_eps_total_kernel(int nu, AdjTuple t, const double *__restrict__ R1, double *__restrict__ geh) {
  const int lane = threadIdx.x & 31;
  double tot = 0.0;
  for (int p = lane; p < nu; p += 32) tot += R1[p];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, off);
  if (lane == 0) {
    geh[t.i] -= tot;
    geh[t.j] -= tot;
    geh[t.k] -= tot;
  }
}

// ---------------------------------------------------------------------------- backward GEMMs
constexpr int BBM = 128, BBK = 16;  // N tile BN in {64, 48, 32}, chosen to fit KP
constexpr int BWM = 32;                 // rows per warp
constexpr int BNT = (BBM / BWM) * 32;   // 128 threads
constexpr int BST = 3;                  // cp.async stages
// Fragment loads are 64-bit, served per half-warp (lanes g = 0..3, t = 0..3).
// The dE A tile [m][k] is unpadded (16 doubles a row) with column c of row r
// stored at c ^ 4 (r & 3): the four rows g of a half-warp then hit four
// disjoint 32-byte bank groups.  [k][.] tiles are padded to a row stride of
// 4 (mod 16) doubles instead.
constexpr int LDA_KM = BBM + 4;         // dF A tile [k][m]
template <int BN>
constexpr int ldb_kn() { return BN + 4; }  // B tile [k][n]
__device__ __forceinline__ int aswz(int r, int c) { return r * BBK + (c ^ ((r & 3) << 2)); }

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
// D(16x8) += A(16x8) B(8x8).  Lane (g = lane/4, t = lane%4) holds
// a = {A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]}, b = {B[t][g], B[t+4][g]} and
// d = {D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]}.
__device__ __forceinline__ void dmma_16x8x8(double *d, const double *a, const double *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
// Row m = p*nu + q of a nu^2 x . operand and its (p,q) <-> (q,p) partner, for
// m < 2^24 (nu <= 4096): the float quotient is within one of p, then corrected.
__device__ __forceinline__ int swap_row(int m, int nu, float inv_nu) {
  int p = __float2int_rz(__int2float_rn(m) * inv_nu);
  int q = m - p * nu;
  if (q < 0) {
    p--;
    q += nu;
  } else if (q >= nu) {
    p++;
    q -= nu;
  }
  return q * nu + p;
}

constexpr int kMaxPairs = 6 * kDEGroup;  // (slot, half) pairs of a tuple group: at most 3 x 2 per tuple
constexpr int kMaxOut = 3 * kDEGroup;    // distinct E slabs of a tuple group
struct BwdPair {
  const double *A;  // dE/dX_g (nu^2 x NP)
  const double *B;  // bwd_e: F[fyz] (NP x KP); bwd_f: E[x] (nu^2 x KP)
  int perm;         // 1: (p,q) <-> (q,p) row permutation of the half
  int out;          // output index
};
struct BwdEArgs {
  BwdPair pair[kMaxPairs];
  double *out[kMaxOut];
  int first[kMaxOut + 1], npairs;  // pairs of output o are first[o] .. first[o+1]-1
  int nu;
  int64_t NP, KP;
  int64_t KV;  // columns that are not padding: nu + no
  int tiles_n;
};

// dE[x](r, n) += sum_pairs sum_s A[perm(r)][s] B[s][n]; M = nu^2, N = KP, K = NP per pair.
// 3 CTAs per SM (2 for BN = 64, whose shared memory does not fit three)
template <int BN>
__global__ void __launch_bounds__(BNT, BN == 64 ? 2 : 3) bwd_e_kernel(const BwdEArgs args) {
  constexpr int BBN = BN, LDB_KN = ldb_kn<BN>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *As = reinterpret_cast<double *>(smem_raw);  // [BST][BBM][BBK], swizzled
  double *Bs = As + BST * BBM * BBK;                    // [BST][BBK][LDB_KN]
  int *rows = reinterpret_cast<int *>(Bs + BST * BBK * LDB_KN);  // [2][BBM]: row of A (or -1)
  const int o = blockIdx.y;
  const int tile_m = blockIdx.x / args.tiles_n, tile_n = blockIdx.x - tile_m * args.tiles_n;
  const int nu = args.nu;
  const int64_t M = (int64_t)nu * nu, NP = args.NP, KP = args.KP;
  const int64_t m0 = (int64_t)tile_m * BBM;
  const int n0 = tile_n * BBN;
  const bool full = n0 + BBN - 8 < args.KV;
  const int tid = threadIdx.x;
  const int p_begin = args.first[o], p_end = args.first[o + 1];
  const int kt_per = (int)((NP + BBK - 1) / BBK);  // NP is a multiple of 8, not always of 16
  const int ktiles = kt_per * (p_end - p_begin);

  {
    const float inv_nu = 1.0f / (float)nu;
    for (int r = tid; r < BBM; r += BNT) {
      const int64_t m = m0 + r;
      rows[r] = m < M ? (int)m : -1;
      rows[BBM + r] = m < M ? swap_row((int)m, nu, inv_nu) : -1;
    }
  }
  __syncthreads();

  auto load_stage = [&](int stage, int kt) {
    const int pi = p_begin + kt / kt_per;
    const int64_t k0 = (int64_t)(kt % kt_per) * BBK;
    const BwdPair &pr = args.pair[pi];
    double *as = As + stage * BBM * BBK;
    double *bs = Bs + stage * BBK * LDB_KN;
    const int *rw = rows + pr.perm * BBM;
    const int chunk = tid & 7;  // 8 x 16 B per 16-double row
    const bool kok = k0 + chunk * 2 < NP;
    for (int rr = tid >> 3; rr < BBM; rr += BNT / 8) {
      const int row = rw[rr];
      const bool ok = row >= 0 && kok;
      const double *src = pr.A + (ok ? (int64_t)row * NP + k0 + chunk * 2 : 0);
      cp_async16(as + aswz(rr, chunk * 2), src, ok ? 16 : 0);
    }
    // B tile: 16 rows (s) x BN columns (n)
    for (int c = tid; c < BBK * (BBN / 2); c += BNT) {
      const int rr = c / (BBN / 2), cc = c - rr * (BBN / 2);
      const int n = n0 + cc * 2;
      const bool ok = n < KP && k0 + rr < NP;
      const double *src = pr.B + (ok ? (k0 + rr) * KP + n : 0);
      cp_async16(bs + rr * LDB_KN + cc * 2, src, ok ? 16 : 0);
    }
  };

  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  constexpr int MF = BWM / 16, NF = BBN / 8;
  // The accumulators start from the current dE tile (all loads in flight at
  // once, before the main loop), so the epilogue only stores.
  if (ktiles == 0) return;
  double *out = args.out[o];
  double acc[MF][NF][4];
#pragma unroll
  for (int i = 0; i < MF; i++)
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int64_t m = m0 + warp * BWM + i * 16 + g + half * 8;
#pragma unroll
      for (int j = 0; j < NF; j++) {
        const int n = n0 + j * 8 + 2 * t;
        double2 v = make_double2(0.0, 0.0);
        if (m < M && n < KP) v = *reinterpret_cast<const double2 *>(out + m * KP + n);
        acc[i][j][2 * half] = v.x;
        acc[i][j][2 * half + 1] = v.y;
      }
    }

#pragma unroll
  for (int s = 0; s < BST - 1; s++) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }
  // NFR: n8 fragments computed; the tile's last one is skipped when all its
  // columns are padding (>= nu + no)
  auto mainloop = [&](auto nfr_c) {
    constexpr int NFR = decltype(nfr_c)::value;
    for (int kt = 0; kt < ktiles; kt++) {
      cp_async_wait<BST - 2>();
      __syncthreads();
      {
        const int nk = kt + BST - 1;
        if (nk < ktiles) load_stage(nk % BST, nk);
        cp_async_commit();
      }
      const double *as = As + (kt % BST) * BBM * BBK;
      const double *bs = Bs + (kt % BST) * BBK * LDB_KN;
      // NP is a multiple of 8: the last k-tile of a pair may hold only 8 columns
      const bool half_tile = NP - (int64_t)(kt % kt_per) * BBK <= BBK / 2;
#pragma unroll
      for (int kk = 0; kk < BBK; kk += 8) {
        if (kk >= BBK / 2 && half_tile) break;
        double af[MF][4], bf[NF][2];
#pragma unroll
        for (int i = 0; i < MF; i++) {
          const int r = warp * BWM + i * 16 + g;
          af[i][0] = as[aswz(r, kk + t)];
          af[i][1] = as[aswz(r + 8, kk + t)];
          af[i][2] = as[aswz(r, kk + 4 + t)];
          af[i][3] = as[aswz(r + 8, kk + 4 + t)];
        }
#pragma unroll
        for (int j = 0; j < NFR; j++) {
          bf[j][0] = bs[(kk + t) * LDB_KN + j * 8 + g];
          bf[j][1] = bs[(kk + 4 + t) * LDB_KN + j * 8 + g];
        }
#pragma unroll
        for (int i = 0; i < MF; i++)
#pragma unroll
          for (int j = 0; j < NFR; j++) dmma_16x8x8(acc[i][j], af[i], bf[j]);
      }
    }
  };
  if (full)
    mainloop(std::integral_constant<int, NF>{});
  else
    mainloop(std::integral_constant<int, NF - 1>{});
  cp_async_wait<0>();
#pragma unroll
  for (int i = 0; i < MF; i++) {
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int64_t m = m0 + warp * BWM + i * 16 + g + half * 8;
      if (m >= M) continue;
      double *orow = out + m * KP;
#pragma unroll
      for (int j = 0; j < NF; j++) {
        const int n = n0 + j * 8 + 2 * t;
        if (n < KP)
          *reinterpret_cast<double2 *>(orow + n) = make_double2(acc[i][j][2 * half], acc[i][j][2 * half + 1]);
      }
    }
  }
}

struct BwdFArgs {
  BwdPair pair[6];
  double *part;     // [pair][split][NP][KP]
  int npairs, nsplit;
  int64_t kchunk;   // rows of nu^2 per split (multiple of BBK)
  int nu;
  int64_t NP, KP;
  int64_t KV;       // columns that are not padding: nu + no
  int tiles_n;
};

// part[pair][split](s, n) = sum_{m in split} A[m][s] B[perm(m)][n]; M = NP, N = KP.
template <int BN>
__global__ void __launch_bounds__(BNT, BN == 64 ? 2 : 3) bwd_f_kernel(const BwdFArgs args) {
  constexpr int BBN = BN, LDB_KN = ldb_kn<BN>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *As = reinterpret_cast<double *>(smem_raw);  // [BST][BBK][LDA_KM]
  double *Bs = As + BST * BBK * LDA_KM;                 // [BST][BBK][LDB_KN]
  const int pi = blockIdx.y, split = blockIdx.z;
  const BwdPair &pr = args.pair[pi];
  const int tile_m = blockIdx.x / args.tiles_n, tile_n = blockIdx.x - tile_m * args.tiles_n;
  const int nu = args.nu;
  const float inv_nu = 1.0f / (float)nu;
  const int64_t Mtot = (int64_t)nu * nu, NP = args.NP, KP = args.KP;
  const int64_t s0 = (int64_t)tile_m * BBM;
  const int n0 = tile_n * BBN;
  const bool full = n0 + BBN - 8 < args.KV;  // else the last n8 fragment is all padding
  const int64_t kbeg = (int64_t)split * args.kchunk;
  const int64_t kend = min(kbeg + args.kchunk, Mtot);
  const int ktiles = kend > kbeg ? (int)((kend - kbeg + BBK - 1) / BBK) : 0;
  const int tid = threadIdx.x;

  auto load_stage = [&](int stage, int kt) {
    const int64_t k0 = kbeg + (int64_t)kt * BBK;
    double *as = As + stage * BBK * LDA_KM;
    double *bs = Bs + stage * BBK * LDB_KN;
    // A tile: 16 rows (m) x 128 columns (s): 64 chunks per row
    for (int c = tid; c < BBK * (BBM / 2); c += BNT) {
      const int rr = c / (BBM / 2), cc = c - rr * (BBM / 2);
      const int64_t m = k0 + rr, s = s0 + cc * 2;
      const bool ok = m < kend && s < NP;
      const double *src = pr.A + (ok ? m * NP + s : 0);
      cp_async16(as + rr * LDA_KM + cc * 2, src, ok ? 16 : 0);
    }
    for (int c = tid; c < BBK * (BBN / 2); c += BNT) {
      const int rr = c / (BBN / 2), cc = c - rr * (BBN / 2);
      const int64_t m = k0 + rr;
      const int n = n0 + cc * 2;
      const bool ok = m < kend && n < KP;
      const int64_t row = ok && pr.perm ? (int64_t)swap_row((int)m, nu, inv_nu) : m;
      const double *src = pr.B + (ok ? row * KP + n : 0);
      cp_async16(bs + rr * LDB_KN + cc * 2, src, ok ? 16 : 0);
    }
  };

  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  constexpr int MF = BWM / 16, NF = BBN / 8;
  double acc[MF][NF][4];
#pragma unroll
  for (int i = 0; i < MF; i++)
#pragma unroll
    for (int j = 0; j < NF; j++)
#pragma unroll
      for (int r = 0; r < 4; r++) acc[i][j][r] = 0.0;

#pragma unroll
  for (int s = 0; s < BST - 1; s++) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }
  auto mainloop = [&](auto nfr_c) {  // NFR n8 fragments, as in bwd_e_kernel
    constexpr int NFR = decltype(nfr_c)::value;
    for (int kt = 0; kt < ktiles; kt++) {
      cp_async_wait<BST - 2>();
      __syncthreads();
      {
        const int nk = kt + BST - 1;
        if (nk < ktiles) load_stage(nk % BST, nk);
        cp_async_commit();
      }
      const double *as = As + (kt % BST) * BBK * LDA_KM + warp * BWM;
      const double *bs = Bs + (kt % BST) * BBK * LDB_KN;
#pragma unroll
      for (int kk = 0; kk < BBK; kk += 8) {
        double af[MF][4], bf[NF][2];
#pragma unroll
        for (int i = 0; i < MF; i++) {
          af[i][0] = as[(kk + t) * LDA_KM + i * 16 + g];
          af[i][1] = as[(kk + t) * LDA_KM + i * 16 + g + 8];
          af[i][2] = as[(kk + 4 + t) * LDA_KM + i * 16 + g];
          af[i][3] = as[(kk + 4 + t) * LDA_KM + i * 16 + g + 8];
        }
#pragma unroll
        for (int j = 0; j < NFR; j++) {
          bf[j][0] = bs[(kk + t) * LDB_KN + j * 8 + g];
          bf[j][1] = bs[(kk + 4 + t) * LDB_KN + j * 8 + g];
        }
#pragma unroll
        for (int i = 0; i < MF; i++)
#pragma unroll
          for (int j = 0; j < NFR; j++) dmma_16x8x8(acc[i][j], af[i], bf[j]);
      }
    }
  };
  if (full)
    mainloop(std::integral_constant<int, NF>{});
  else
    mainloop(std::integral_constant<int, NF - 1>{});
  cp_async_wait<0>();
  double *out = args.part + ((int64_t)pi * args.nsplit + split) * NP * KP;
#pragma unroll
  for (int i = 0; i < MF; i++) {
#pragma unroll
    for (int half = 0; half < 2; half++) {
      const int64_t s = s0 + warp * BWM + i * 16 + g + half * 8;
      if (s >= NP) continue;
#pragma unroll
      for (int j = 0; j < NF; j++) {
        const int n = n0 + j * 8 + 2 * t;
        if (n < KP)
          *reinterpret_cast<double2 *>(out + s * KP + n) =
              make_double2(acc[i][j][2 * half], acc[i][j][2 * half + 1]);
      }
    }
  }
}

// dF[out] += sum over the pairs writing it, then over splits, in order.
struct BwdFReduceArgs {
  double *dst[6];
  int first[7];     // pairs of output o: first[o] .. first[o+1]-1 (pairs sorted by output)
  int nout, nsplit;
  int64_t n;        // NP * KP
};
__global__ void bwd_f_reduce_kernel(const BwdFReduceArgs a, const double *__restrict__ part) {
  const int o = blockIdx.y;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < a.n; e += (int64_t)gridDim.x * blockDim.x) {
    double s = a.dst[o][e];
    for (int pi = a.first[o]; pi < a.first[o + 1]; pi++) {
      const double *src = part + (int64_t)pi * a.nsplit * a.n + e;
      int sp = 0;
      for (; sp + 8 <= a.nsplit; sp += 8) {  // eight loads in flight, added in split order
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; u++) v[u] = src[(int64_t)(sp + u) * a.n];
#pragma unroll
        for (int u = 0; u < 8; u++) s += v[u];
      }
      for (; sp < a.nsplit; sp++) s += src[(int64_t)sp * a.n];
    }
    a.dst[o][e] = s;
  }
}

// ---------------------------------------------------------------------------- scatters
// Packed VVVO: column x*nu + r1 holds (I >= J) of (I J | r1 x) at I(I+1)/2 + J, and
// E[x][r1][r2][k] = col[tri(k, r2)] for k < nu; E[x][r1][r2][nu+l] = -T2(r1,r2,l,x).
__global__ void adj_scatter_e_kernel(int nu, int no, int64_t KP, const double *__restrict__ dE,
                                     double *__restrict__ gvvvo, double *__restrict__ gt2) {
  const int64_t nutr = (int64_t)nu * (nu + 1) / 2;
  const int64_t ncol = (int64_t)nu * no;
  const int64_t nu2 = (int64_t)nu * nu;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < ncol * nutr;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t col = e / nutr, tri = e - col * nutr;
    const int x = (int)(col / nu), r1 = (int)(col - (int64_t)x * nu);
    int I = (int)((sqrt(8.0 * (double)tri + 1.0) - 1.0) * 0.5);
    while ((int64_t)I * (I + 1) / 2 > tri) I--;
    while ((int64_t)(I + 1) * (I + 2) / 2 <= tri) I++;
    const int J = (int)(tri - (int64_t)I * (I + 1) / 2);
    const double *row = dE + ((int64_t)x * nu2 + (int64_t)r1 * nu) * KP;  // rows (r1, r2)
    double v = row[(int64_t)J * KP + I];
    if (I != J) v += row[(int64_t)I * KP + J];
    gvvvo[e] += v;
  }
  // T2 part: thread per (x, r1, r2, l)
  const int64_t nt2 = (int64_t)no * nu2 * no;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nt2; e += (int64_t)gridDim.x * blockDim.x) {
    // e enumerates T2(r1, r2, l, x) in its Fortran order
    const int r1 = (int)(e % nu);
    const int64_t rest = e / nu;
    const int r2 = (int)(rest % nu);
    const int64_t lx = rest / nu;
    const int l = (int)(lx % no), x = (int)(lx / no);
    gt2[e] -= dE[((int64_t)x * nu2 + (int64_t)r1 * nu + r2) * KP + nu + l];
  }
}

// F[y][z][s][k] = T2(s,k,y,z) for k < nu; F[y][z][s][nu+l] = VM(l,s,z,y).
__global__ void adj_scatter_f_kernel(int nu, int no, int64_t NP, int64_t KP, const double *__restrict__ dF,
                                     double *__restrict__ gt2, double *__restrict__ gvm) {
  const int64_t nu2 = (int64_t)nu * nu;
  const int64_t nt2 = nu2 * no * no;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nt2; e += (int64_t)gridDim.x * blockDim.x) {
    // T2(s, k, y, z), Fortran order
    const int s = (int)(e % nu);
    const int64_t r = e / nu;
    const int k = (int)(r % nu);
    const int64_t yz = r / nu;
    const int y = (int)(yz % no), z = (int)(yz / no);
    gt2[e] += dF[(((int64_t)y * no + z) * NP + s) * KP + k];
  }
  const int64_t nvm = (int64_t)no * nu * no * no;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nvm; e += (int64_t)gridDim.x * blockDim.x) {
    // VM(l, s, z, y), Fortran order
    const int l = (int)(e % no);
    const int64_t r = e / no;
    const int s = (int)(r % nu);
    const int64_t zy = r / nu;
    const int z = (int)(zy % no), y = (int)(zy / no);
    gvm[e] += dF[(((int64_t)y * no + z) * NP + s) * KP + nu + l];
  }
}

// dT1(x,a) = 2 v1(a,x)
__global__ void adj_t1_kernel(int nu, int no, const double *__restrict__ v1, double *__restrict__ gt1) {
  const int64_t n = (int64_t)nu * no;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(e % no), a = (int)(e / no);
    gt1[e] = 2.0 * v1[(int64_t)x * nu + a];
  }
}

int grid_for(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  return (int)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

template <int BN>
constexpr int smem_e() { return BST * (BBM * BBK + BBK * ldb_kn<BN>()) * 8 + 2 * BBM * 4; }
template <int BN>
constexpr int smem_f() { return BST * (BBK * LDA_KM + BBK * ldb_kn<BN>()) * 8; }
// N tile for an N extent of KP: least padding, ties to the wider tile
inline int bwd_bn(int64_t KP) {
  int best = 64;
  for (int bn : {48, 32})
    if (round_up(KP, bn) < round_up(KP, best)) best = bn;
  return best;
}
template <int BN>
int launch_bwd_e(const BwdEArgs &a, int tiles_m, int nx, cudaStream_t s) {
  bwd_e_kernel<BN><<<dim3(tiles_m * a.tiles_n, nx), BNT, smem_e<BN>(), s>>>(a);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}
template <int BN>
int launch_bwd_f(const BwdFArgs &a, int tiles_m, cudaStream_t s) {
  bwd_f_kernel<BN><<<dim3(tiles_m * a.tiles_n, a.npairs, a.nsplit), BNT, smem_f<BN>(), s>>>(a);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

}  // namespace

int adj_alloc(const Dims &d, AdjBuffers *b) {
  const int64_t no = d.no, nu = d.nu, nu2 = nu * nu, nu3 = nu2 * nu;
  auto al = [](double **p, int64_t n) -> int {
    *p = nullptr;
    CCT_CUDA(cudaMalloc(reinterpret_cast<void **>(p), (size_t)(n < 1 ? 1 : n) * 8));
    return CCT_OK;
  };
  {
    // dF GEMM split-K: about CCT_BWD_F_CTAS_PER_SM CTAs per SM for the 6 pairs
    // of an i>j>k tuple, rounded to whole k-tiles
    int sms = 148, dev = 0;
    CCT_CUDA(cudaGetDevice(&dev));
    CCT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int bn = bwd_bn(d.KP);
    const int64_t tiles = ((d.NP + BBM - 1) / BBM) * ((d.KP + bn - 1) / bn) * 6;
    int64_t ns = (int64_t)(CCT_BWD_F_CTAS_PER_SM * sms) / tiles;
    ns = ns < 1 ? 1 : (ns > (nu2 + BBK - 1) / BBK ? (nu2 + BBK - 1) / BBK : ns);
    b->kchunk = round_up((nu2 + ns - 1) / ns, BBK);
    b->nsplit = (nu2 + b->kchunk - 1) / b->kchunk;
  }
  CCT_TRY(al(&b->dE, no * nu2 * d.KP));
  CCT_TRY(al(&b->dF, no * no * d.NP * d.KP));
  CCT_TRY(al(&b->Wf, nu3));
  CCT_TRY(al(&b->GW, nu3));
  for (int set = 0; set < kGXSets; set++)
    for (int g = 0; g < 3; g++) {
      CCT_TRY(al(&b->GX[set][g], nu2 * d.NP));
      CCT_CUDA(cudaMemset(b->GX[set][g], 0, (size_t)nu2 * d.NP * 8));  // padding columns stay zero
    }
  CCT_TRY(al(&b->part, 6 * b->nsplit * d.NP * d.KP));
  CCT_TRY(al(&b->Q, 9 * nu2));
  CCT_TRY(al(&b->vpart, ((nu + kAChunk - 1) / kAChunk) * 6 * nu2));
  {
    const int64_t nb = (nu + kTB - 1) / kTB, nch = (nu + kTA - 1) / kTA;
    CCT_TRY(al(&b->eps, (nb * nb + 2 * nch * nb + 1) * nu));  // EA, EB, EC, Rp
  }
  CCT_TRY(al(&b->v1, 5 + nu * no));
  CCT_TRY(al(&b->g_eh, no));
  CCT_TRY(al(&b->g_ep, nu));
  CCT_TRY(al(&b->g_t1, no * nu));
  CCT_TRY(al(&b->g_t2, nu2 * no * no));
  CCT_TRY(al(&b->g_vm, no * nu * no * no));
  CCT_TRY(al(&b->g_voe, nu2 * no * no));
  CCT_TRY(al(&b->g_vvvo, nu * (nu + 1) / 2 * nu * no));
  b->ready = true;
  return CCT_OK;
}

void adj_free(AdjBuffers *b) {
  for (int set = 0; set < kGXSets; set++)
    for (int g = 0; g < 3; g++)
      if (b->GX[set][g]) cudaFree(b->GX[set][g]);
  for (double *q : {b->dE, b->dF, b->Wf, b->GW, b->part, b->Q, b->vpart, b->eps, b->v1, b->g_eh,
                    b->g_ep, b->g_t1, b->g_t2, b->g_vm, b->g_voe, b->g_vvvo})
    if (q) cudaFree(q);
  *b = AdjBuffers{};
}

int assemble_w_fortran(const Dims &d, const Tuple &t, double *const X[3], double *wc, double *wf, cudaStream_t s) {
  const int nu = d.nu;
  AdjTuple at;
  at.x[0] = X[0];
  at.x[1] = X[1];
  at.x[2] = X[2];
  at.i = t.i;
  at.j = t.j;
  at.k = t.k;
  at.weight = t.kind == kIJK ? 1.0 : 0.5;
  const dim3 g3((nu + kWC - 1) / kWC, (nu + kWB - 1) / kWB, (nu + kWA - 1) / kWA);
  switch (t.kind) {
    case kIJK: adj_wfull_kernel<kIJK><<<g3, kWThreads, 3 * kWSlot * 8, s>>>(nu, d.NP, at, wc); break;
    case kIJJ: adj_wfull_kernel<kIJJ><<<g3, kWThreads, 4 * kWSlot * 8, s>>>(nu, d.NP, at, wc); break;
    default: adj_wfull_kernel<kIIJ><<<g3, kWThreads, 4 * kWSlot * 8, s>>>(nu, d.NP, at, wc); break;
  }
  CCT_CUDA(cudaGetLastError());
  const dim3 gt((nu + 31) / 32, (nu + 31) / 32, nu);
  w_fortran_kernel<<<gt, dim3(32, 8), 0, s>>>(nu, wc, wf);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

int adj_zero(const Dims &d, AdjBuffers *b, cudaStream_t s) {
  const int64_t no = d.no, nu = d.nu, nu2 = nu * nu;
  CCT_CUDA(cudaMemsetAsync(b->dE, 0, (size_t)no * nu2 * d.KP * 8, s));
  CCT_CUDA(cudaMemsetAsync(b->dF, 0, (size_t)no * no * d.NP * d.KP * 8, s));
  CCT_CUDA(cudaMemsetAsync(b->g_eh, 0, (size_t)no * 8, s));
  CCT_CUDA(cudaMemsetAsync(b->g_ep, 0, (size_t)nu * 8, s));
  CCT_CUDA(cudaMemsetAsync(b->g_voe, 0, (size_t)nu2 * no * no * 8, s));
  return CCT_OK;
}

// The jobs of one tuple as (x1, x2, x3, nhalves) per X slot, as cct_plan.cu's
// build_jobs lays them out.
static void tuple_slots(const Tuple &t, int slots[3][4], int *nslots) {
  auto G = [&](int s, int x1, int x2, int x3) { slots[s][0] = x1, slots[s][1] = x2, slots[s][2] = x3, slots[s][3] = 2; };
  auto H = [&](int s, int x1, int x2, int x3) { slots[s][0] = x1, slots[s][1] = x2, slots[s][2] = x3, slots[s][3] = 1; };
  if (t.kind == kIJK) {
    G(0, t.i, t.j, t.k);
    G(1, t.i, t.k, t.j);
    G(2, t.j, t.k, t.i);
    *nslots = 3;
  } else if (t.kind == kIJJ) {
    G(0, t.i, t.j, t.j);
    H(1, t.j, t.j, t.i);
    *nslots = 2;
  } else {
    H(0, t.i, t.i, t.k);
    G(1, t.i, t.k, t.i);
    *nslots = 2;
  }
}

int adj_tuple_pointwise(const Dims &d, const Tuple &t, double *const X[3], const double *eh, const double *ep,
                        const double *t1, const double *voe, AdjBuffers *b, int set, cudaStream_t s) {
  double *const *GX = b->GX[set];
  const int no = d.no, nu = d.nu;
  const int64_t nu2 = (int64_t)nu * nu;
  AdjTuple at;
  at.x[0] = X[0];
  at.x[1] = X[1];
  at.x[2] = X[2];
  at.i = t.i;
  at.j = t.j;
  at.k = t.k;
  at.weight = t.kind == kIJK ? 1.0 : 0.5;
  SmTable sm;
  const int smx[6][3] = {{t.i, t.j, t.k}, {t.i, t.k, t.j}, {t.j, t.i, t.k},
                         {t.k, t.i, t.j}, {t.j, t.k, t.i}, {t.k, t.j, t.i}};
  for (int m = 0; m < 6; m++) sm.x[m] = smx[m][0], sm.y[m] = smx[m][1], sm.z[m] = smx[m][2];

  const dim3 g3((nu + kWC - 1) / kWC, (nu + kWB - 1) / kWB, (nu + kWA - 1) / kWA);
  switch (t.kind) {
    case kIJK: adj_wfull_kernel<kIJK><<<g3, kWThreads, 3 * kWSlot * 8, s>>>(nu, d.NP, at, b->Wf); break;
    case kIJJ: adj_wfull_kernel<kIJJ><<<g3, kWThreads, 4 * kWSlot * 8, s>>>(nu, d.NP, at, b->Wf); break;
    default: adj_wfull_kernel<kIIJ><<<g3, kWThreads, 4 * kWSlot * 8, s>>>(nu, d.NP, at, b->Wf); break;
  }
  CCT_CUDA(cudaGetLastError());
  {
    // H regrouped by (role of u, position of u): nine signed sums of VOE planes
    constexpr int kAdj[6][4][4] = {{{2, 0, 1, 2}, {-2, 1, 0, 2}, {-1, 0, 2, 1}, {1, 2, 0, 1}},
                                   {{2, 0, 2, 1}, {-2, 2, 0, 1}, {-1, 0, 1, 2}, {1, 1, 0, 2}},
                                   {{2, 1, 0, 2}, {-2, 0, 1, 2}, {-1, 1, 2, 0}, {1, 2, 1, 0}},
                                   {{2, 2, 0, 1}, {-2, 0, 2, 1}, {-1, 2, 1, 0}, {1, 1, 2, 0}},
                                   {{2, 1, 2, 0}, {-2, 2, 1, 0}, {-1, 1, 0, 2}, {1, 0, 1, 2}},
                                   {{2, 2, 1, 0}, {-2, 1, 2, 0}, {-1, 2, 0, 1}, {1, 0, 2, 1}}};
    constexpr int kRole[6] = {0, 0, 1, 2, 1, 2};  // z_1..z_6 take u from i, i, j, k, j, k
    QTable qt{};
    for (int m = 0; m < 6; m++)
      for (int r = 0; r < 4; r++) {
        const int g = kRole[m] * 3 + kAdj[m][r][1];
        if (qt.n[g] >= kQTerms) {
          set_error("adjoint: Q table overflow");
          return CCT_ERR_INVALID;
        }
        const int u = qt.n[g]++;
        qt.coef[g][u] = kAdj[m][r][0];
        qt.plane[g][u] = ((int64_t)sm.z[m] * no + sm.y[m]) * nu2;
        qt.trans[g][u] = kAdj[m][r][2] > kAdj[m][r][3];
      }
    adj_q_kernel<<<grid_for(9 * nu2), 256, 0, s>>>(nu, qt, voe, b->Q);
    CCT_CUDA(cudaGetLastError());
  }
  {
    const int nb = (nu + kTB - 1) / kTB, nch = (nu + kTA - 1) / kTA;
    double *EA = b->eps, *EB = EA + (int64_t)nb * nb * nu, *EC = EB + (int64_t)nch * nb * nu,
           *Rp = EC + (int64_t)nch * nb * nu;
    const dim3 ggrid(nb, nb, nch);
    if (t.kind == kIJK)
      adj_gw_kernel<true><<<ggrid, kGwThreads, kGwSmem, s>>>(nu, no, d.NP, at, b->Wf, eh, ep, t1, b->Q, b->GW, GX[0],
                                                              GX[1], GX[2], b->vpart, EA, EB, EC);
    else
      adj_gw_kernel<false><<<ggrid, kGwThreads, kGwSmem, s>>>(nu, no, d.NP, at, b->Wf, eh, ep, t1, b->Q, b->GW,
                                                               GX[0], GX[1], GX[2], b->vpart, EA, EB, EC);
    CCT_CUDA(cudaGetLastError());
    adj_voe_sum_kernel<<<grid_for(nu2), 256, 0, s>>>(nu, no, nch, at, sm, b->vpart, b->g_voe);
    CCT_CUDA(cudaGetLastError());
    adj_eps_sum_kernel<<<(nu + 7) / 8, 256, 0, s>>>(nu, nb, nch, EA, EB, EC, b->g_ep, Rp);
    CCT_CUDA(cudaGetLastError());
    adj_eps_total_kernel<<<1, 32, 0, s>>>(nu, at, Rp, b->g_eh);
  }
  CCT_CUDA(cudaGetLastError());
  if (t.kind != kIJK) {  // degenerate tuples: two dE/dW permutations feed each dE/dX element
    const dim3 gx((unsigned)((d.NP + 127) / 128), nu, nu);
    if (t.kind == kIJJ)
      adj_gx_kernel<kIJJ><<<gx, 128, 0, s>>>(nu, d.NP, b->GW, GX[0], GX[1], GX[2]);
    else
      adj_gx_kernel<kIIJ><<<gx, 128, 0, s>>>(nu, d.NP, b->GW, GX[0], GX[1], GX[2]);
    CCT_CUDA(cudaGetLastError());
  }
  return CCT_OK;
}

namespace {
// (slot, half) pairs of one tuple: half h of slot g reads E[x] with row
// permutation h and F[fyz]
struct GemmPair {
  int g, h, x, fyz;
};
std::vector<GemmPair> tuple_pairs(const Tuple &t, int no) {
  int slots[3][4], ns = 0;
  tuple_slots(t, slots, &ns);
  std::vector<GemmPair> pairs;
  for (int g = 0; g < ns; g++)
    for (int h = 0; h < slots[g][3]; h++) {
      const int x = h == 0 ? slots[g][0] : slots[g][1];
      const int fyz = (h == 0 ? slots[g][1] : slots[g][0]) * no + slots[g][2];
      pairs.push_back({g, h, x, fyz});
    }
  return pairs;
}
}  // namespace

int adj_tuple_gemm_e(const Dims &d, const Tuple *tu, const int *sets, int ntup, const double *F, AdjBuffers *b,
                     cudaStream_t s) {
  const int nu = d.nu;
  const int64_t nu2 = (int64_t)nu * nu;
  auto Fyz = [&](int yz) { return F + (int64_t)yz * d.NP * d.KP; };
  // dE: outputs in order of first appearance; per output the pairs of the
  // group's tuples in tuple order, each in slot order (a fixed order)
  if (ntup < 1 || ntup > kDEGroup) {
    set_error("adjoint: dE GEMM group size out of range");
    return CCT_ERR_INVALID;
  }
  std::vector<GemmPair> pairs[kDEGroup];
  for (int u = 0; u < ntup; u++) pairs[u] = tuple_pairs(tu[u], d.no);
  BwdEArgs a{};
  int xs[kMaxOut], nx = 0;
  for (int u = 0; u < ntup; u++)
    for (const GemmPair &q : pairs[u]) {
      bool seen = false;
      for (int v = 0; v < nx; v++) seen |= xs[v] == q.x;
      if (!seen) xs[nx++] = q.x;
    }
  int np_ = 0;
  for (int o = 0; o < nx; o++) {
    a.first[o] = np_;
    a.out[o] = b->dE + (int64_t)xs[o] * nu2 * d.KP;
    for (int u = 0; u < ntup; u++)
      for (const GemmPair &q : pairs[u])
        if (q.x == xs[o]) {
          if (np_ >= kMaxPairs) {
            set_error("adjoint: too many GEMM pairs for one dE launch");
            return CCT_ERR_INVALID;
          }
          a.pair[np_++] = BwdPair{b->GX[sets[u]][q.g], Fyz(q.fyz), q.h, o};
        }
  }
  a.first[nx] = np_;
  a.npairs = np_;
  a.nu = nu;
  a.NP = d.NP;
  a.KP = d.KP;
  a.KV = d.nu + d.no;
  const int bn = bwd_bn(d.KP);
  a.tiles_n = (int)((d.KP + bn - 1) / bn);
  const int tiles_m = (int)((nu2 + BBM - 1) / BBM);
  return bn == 64 ? launch_bwd_e<64>(a, tiles_m, nx, s)
                  : bn == 48 ? launch_bwd_e<48>(a, tiles_m, nx, s) : launch_bwd_e<32>(a, tiles_m, nx, s);
}

int adj_tuple_gemm_f(const Dims &d, const Tuple &t, const double *E, AdjBuffers *b, int set, cudaStream_t sf) {
  const int nu = d.nu;
  const int64_t nu2 = (int64_t)nu * nu;
  double *const *GX = b->GX[set];
  auto Ex = [&](int x) { return E + (int64_t)x * nu2 * d.KP; };
  // dF: one partial per pair and split, then a fixed-order sum per output slab
  BwdFArgs a{};
  std::vector<GemmPair> sorted = tuple_pairs(t, d.no);
  std::stable_sort(sorted.begin(), sorted.end(),
                   [](const GemmPair &u, const GemmPair &v) { return u.fyz < v.fyz; });
  BwdFReduceArgs r{};
  int no_ = 0;
  for (size_t q = 0; q < sorted.size(); q++) {
    a.pair[q] = BwdPair{GX[sorted[q].g], Ex(sorted[q].x), sorted[q].h, 0};
    if (q == 0 || sorted[q].fyz != sorted[q - 1].fyz) {
      r.first[no_] = (int)q;
      r.dst[no_] = b->dF + (int64_t)sorted[q].fyz * d.NP * d.KP;
      no_++;
    }
  }
  r.first[no_] = (int)sorted.size();
  r.nout = no_;
  r.nsplit = (int)b->nsplit;
  r.n = d.NP * d.KP;
  a.part = b->part;
  a.npairs = (int)sorted.size();
  a.nsplit = (int)b->nsplit;
  a.kchunk = b->kchunk;
  a.nu = nu;
  a.NP = d.NP;
  a.KP = d.KP;
  a.KV = d.nu + d.no;
  const int bn = bwd_bn(d.KP);
  a.tiles_n = (int)((d.KP + bn - 1) / bn);
  const int tiles_m = (int)((d.NP + BBM - 1) / BBM);
  CCT_TRY(bn == 64 ? launch_bwd_f<64>(a, tiles_m, sf)
                   : bn == 48 ? launch_bwd_f<48>(a, tiles_m, sf) : launch_bwd_f<32>(a, tiles_m, sf));
  bwd_f_reduce_kernel<<<dim3(grid_for(r.n) < 64 ? grid_for(r.n) : 64, r.nout), 256, 0, sf>>>(r, b->part);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

int adj_configure(int device) {
  static int configured = -1;
  if (configured == device) return CCT_OK;
  CCT_CUDA(cudaFuncSetAttribute(adj_wfull_kernel<kIJK>, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * kWSlot * 8));
  CCT_CUDA(cudaFuncSetAttribute(adj_wfull_kernel<kIJJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * kWSlot * 8));
  CCT_CUDA(cudaFuncSetAttribute(adj_wfull_kernel<kIIJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * kWSlot * 8));
  CCT_CUDA(cudaFuncSetAttribute(adj_gw_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGwSmem));
  CCT_CUDA(cudaFuncSetAttribute(adj_gw_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGwSmem));
  CCT_CUDA(cudaFuncSetAttribute(bwd_e_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_e<64>()));
  CCT_CUDA(cudaFuncSetAttribute(bwd_e_kernel<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_e<48>()));
  CCT_CUDA(cudaFuncSetAttribute(bwd_e_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_e<32>()));
  CCT_CUDA(cudaFuncSetAttribute(bwd_f_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_f<64>()));
  CCT_CUDA(cudaFuncSetAttribute(bwd_f_kernel<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_f<48>()));
  CCT_CUDA(cudaFuncSetAttribute(bwd_f_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_f<32>()));
  configured = device;
  return CCT_OK;
}

int adj_finish(const Dims &d, const double *v1, AdjBuffers *b, cudaStream_t s) {
  const int64_t no = d.no, nu = d.nu, nu2 = nu * nu;
  CCT_CUDA(cudaMemsetAsync(b->g_t2, 0, (size_t)nu2 * no * no * 8, s));
  CCT_CUDA(cudaMemsetAsync(b->g_vm, 0, (size_t)no * nu * no * no * 8, s));
  CCT_CUDA(cudaMemsetAsync(b->g_vvvo, 0, (size_t)(nu * (nu + 1) / 2) * nu * no * 8, s));
  const int64_t ne = std::max<int64_t>((nu * (nu + 1) / 2) * nu * no, no * nu2 * no);
  adj_scatter_e_kernel<<<grid_for(ne), 256, 0, s>>>(d.nu, d.no, d.KP, b->dE, b->g_vvvo, b->g_t2);
  CCT_CUDA(cudaGetLastError());
  adj_scatter_f_kernel<<<grid_for(nu2 * no * no), 256, 0, s>>>(d.nu, d.no, d.NP, d.KP, b->dF, b->g_t2, b->g_vm);
  CCT_CUDA(cudaGetLastError());
  adj_t1_kernel<<<grid_for(nu * no), 256, 0, s>>>(d.nu, d.no, v1, b->g_t1);
  CCT_CUDA(cudaGetLastError());
  return CCT_OK;
}

}  // namespace cct
