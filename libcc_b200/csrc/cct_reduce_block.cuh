// One block triple of the per-tuple E[4] / v1 reduction as a device function,
// shared by the per-tuple reduction kernel (cct_reduce.cu) and the persistent
// batch kernel (cct_batch.cu).  See cct_reduce.cu for the algorithm and the
// reference lines it follows.
#pragma once
#include "cct_internal.cuh"

namespace cct {
namespace red {


constexpr int RB = kRB;  // 8
constexpr int RT = 256;  // threads per reduction CTA
constexpr int SL = 512;  // doubles per 8x8x8 block in smem
// Element (l0, l1, l2) of a block: unpadded, with l0 XOR-ed by (l1 + l2) mod 8.
// The term stores of phase A and the orbit reads of phase B put two
// lane-varying coordinates on different axes; the XOR spreads every such pair
// over distinct 8-byte bank pairs of a half-warp (a padded layout with strides
// 1, 9, 81 left the pairs on axes 0 and 2 two-way conflicted).
__host__ __device__ constexpr int soff(int l0, int l1, int l2) { return (l0 ^ ((l1 + l2) & 7)) + 8 * l1 + 64 * l2; }

// The six permutations of three positions, in a fixed order:
// 0:(0,1,2)=abc 1:(0,2,1)=acb 2:(1,0,2)=bac 3:(1,2,0)=bca 4:(2,0,1)=cab 5:(2,1,0)=cba
__host__ __device__ constexpr int pm(int p, int m) {
  return p == 0 ? m : p == 1 ? (m == 0 ? 0 : m == 1 ? 2 : 1) : p == 2 ? (m == 0 ? 1 : m == 1 ? 0 : 2)
       : p == 3 ? (m == 0 ? 1 : m == 1 ? 2 : 0) : p == 4 ? (m == 0 ? 2 : m == 1 ? 0 : 1)
                : (m == 0 ? 2 : m == 1 ? 1 : 0);
}
__host__ __device__ constexpr int pidx(int p0, int p1) { return p0 * 2 + (p1 > p0 ? p1 - 1 : p1); }
// perm value of role r for element pi(x): W(x_{pi(r(0))}, ...) -> index of pi o r
__host__ __device__ constexpr int compose(int pi, int r) { return pidx(pm(pi, pm(r, 0)), pm(pi, pm(r, 1))); }

// W assembly per tuple kind: W(x0,x1,x2) += X_g(x_al0, x_al1, x_al2); {g, al0, al1, al2}
//   i>j>k : X0(a,b,c) + X1(a,c,b) + X2(b,c,a)
//   (i,j,j): X0(a,b,c) + X0(a,c,b) + X1(b,c,a) + X1(c,b,a)
//   (i,i,k): X0(a,b,c) + X0(b,a,c) + X1(a,c,b) + X1(b,c,a)
__host__ __device__ constexpr int term_entry(int kind, int term, int f) {
  constexpr int tab[3][4][4] = {{{0, 0, 1, 2}, {1, 0, 2, 1}, {2, 1, 2, 0}, {0, 0, 0, 0}},
                                {{0, 0, 1, 2}, {0, 0, 2, 1}, {1, 1, 2, 0}, {1, 2, 1, 0}},
                                {{0, 0, 1, 2}, {0, 1, 0, 2}, {1, 0, 2, 1}, {1, 1, 2, 0}}};
  return tab[kind][term][f];
}

template <typename T>
__device__ __forceinline__ T sel3(int m, T v0, T v1, T v2) {
  return m == 0 ? v0 : (m == 1 ? v1 : v2);
}

// VOE staging: three block pairs x two orientations x six planes x 64 entries:
// pair 0 (b,c), 1 (a,c), 2 (a,b); orientation 0 holds VOE(lo, hi, y, z) of the
// pair's lower and higher coordinates, orientation 1 VOE(hi, lo, y, z); planes
// 0..5 = (y,z) = (j,k) (k,j) (i,k) (k,i) (i,j) (j,i).  Every element reads the
// VOE entries t1wt3.f90:80-85 name, so no symmetry of VOE is assumed.
constexpr int VPAIR = 2 * 6 * 64;
__device__ __forceinline__ int nb_of(int nu) { return (nu + RB - 1) / RB; }
constexpr int REDUCE_SMEM = (6 * SL + 3 * VPAIR) * 8;

// 8-byte global->shared copy that does not wait; ok == false stores 0.0.
__device__ __forceinline__ void cp_async8(double *smem, const double *gmem, bool ok) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(ok ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// slot[p]: the first permutation whose ordered block triple equals O_p (so
// equal blocks of a degenerate orbit are assembled once).
__device__ __forceinline__ void orbit_slots(int S0, int S1, int S2, int slot[6]) {
  auto Sm = [&](int m) { return sel3(m, S0, S1, S2); };
#pragma unroll
  for (int p = 0; p < 6; p++) {
    slot[p] = p;
#pragma unroll
    for (int q = 5; q >= 0; q--)
      if (q < p && Sm(pm(q, 0)) == Sm(pm(p, 0)) && Sm(pm(q, 1)) == Sm(pm(p, 1)) && Sm(pm(q, 2)) == Sm(pm(p, 2)))
        slot[p] = q;
  }
}

// VOE staging as asynchronous 8-byte copies (one commit group).
__device__ __forceinline__ void stage_voe(int nu, int no, const TupleDev &t, const double *__restrict__ voe, int S0,
                                          int S1, int S2, double *Vsm) {
  const int tid = threadIdx.x;
  const int64_t nu2 = (int64_t)nu * nu;
#pragma unroll
  for (int it = 0; it < 3 * VPAIR / RT; it++) {
    const int q = tid + RT * it;
    const int pr = q / VPAIR, orient = (q / 384) & 1, plane = (q / 64) % 6, r = q & 63;
    const int Blo = pr == 0 ? S1 : S0, Bhi = pr == 2 ? S1 : S2;  // (b,c), (a,c), (a,b)
    const int f = RB * (orient ? Bhi : Blo) + (r & 7), s2 = RB * (orient ? Blo : Bhi) + (r >> 3);
    const int px = plane == 0 ? t.j : plane == 1 ? t.k : plane == 2 ? t.i : plane == 3 ? t.k : plane == 4 ? t.i : t.j;
    const int py = plane == 0 ? t.k : plane == 1 ? t.j : plane == 2 ? t.k : plane == 3 ? t.i : plane == 4 ? t.j : t.i;
    const bool ok = f < nu && s2 < nu;
    cp_async8(Vsm + q, voe + (ok ? ((int64_t)py * no + px) * nu2 + f + (int64_t)nu * s2 : 0), ok);
  }
  cp_async_commit();
}

template <int KIND>
__device__ __forceinline__ void reduce_block_bc(int nu, const TupleDev &t, const double *__restrict__ eh,
                                                const double *__restrict__ ep, const int S0, const int S1,
                                                const int S2, const int slot[6], const double *Wsm,
                                                const double *Vsm, double *__restrict__ xpart_slot,
                                                double *__restrict__ vpart);

// One CTA per unordered block triple {A<=B<=C}.  Phase A assembles W on every
// distinct ordered block of the orbit in shared memory (term by term, fixed
// order).  Phase B: each thread evaluates orbits -- the six index permutations
// of one (a,b,c) of block (A,B,C) share six W values and one denominator --
// and accumulates E[4] and the v1 updates of all six elements.  Phase C sums
// the per-thread v1 partials in a fixed order.

// COHERENT: X was written by other CTAs of the same (persistent) kernel, so it
// is read through L2 (ld.global.cg) instead of the read-only path.
template <int KIND, bool COHERENT = false>
__device__ __forceinline__ void reduce_block(int nu, int no, int64_t NP, const TupleDev &t,
                                             const double *__restrict__ eh, const double *__restrict__ ep,
                                             const double *__restrict__ voe, const int S0, const int S1,
                                             const int S2, double *__restrict__ xpart_slot,
                                             double *__restrict__ vpart, double *__restrict__ dyn_smem) {
  constexpr int NTERM = KIND == kIJK ? 3 : 4;
  double *Wsm = dyn_smem;             // [6][SL]
  double *Vsm = Wsm + 6 * SL;         // [3][2][6][64]

  const int tid = threadIdx.x;
  auto Sm = [&](int m) { return sel3(m, S0, S1, S2); };
  int slot[6];
  orbit_slots(S0, S1, S2, slot);

  // ---- VOE staging: asynchronous copies, in flight during phase A's X loads
  stage_voe(nu, no, t, voe, S0, S1, S2, Vsm);


  // ---- phase A: W on the orbit blocks, one X term at a time.  Term 0 (the
  // identity placement X0(a,b,c) for every kind) is copied straight into W
  // asynchronously, unless X is being written by other CTAs of this kernel.
#pragma unroll
  for (int term = 0; term < NTERM; term++) {
    const int g = term_entry(KIND, term, 0);
    const int al0 = term_entry(KIND, term, 1), al1 = term_entry(KIND, term, 2), al2 = term_entry(KIND, term, 3);
    const double *X = t.x[0];
    if (g == 1) X = t.x[1];
    if (g == 2) X = t.x[2];
    if (!COHERENT && term == 0) {
#pragma unroll
      for (int p = 0; p < 6; p++) {
        if (slot[p] != p) continue;
        const int O0 = Sm(pm(p, 0)), O1 = Sm(pm(p, 1)), O2 = Sm(pm(p, 2));
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int idx = tid + RT * e;
          const int u2 = idx & 7, u1 = (idx >> 3) & 7, u0 = idx >> 6;
          const int xp = RB * O0 + u0, xq = RB * O1 + u1, xs = RB * O2 + u2;
          const bool ok = xp < nu && xq < nu && xs < nu;
          const int64_t off = t.blocked ? xblock_base(O0, O1, O2, nu, NP) + idx : ((int64_t)xp * nu + xq) * NP + xs;
          cp_async8(Wsm + p * SL + soff(u0, u1, u2), X + (ok ? off : 0), ok);
        }
      }
      cp_async_commit();
      continue;
    }
    double xv[12];  // [6 blocks][2 elements], flat: the compiler kept a 2-D array in local memory
#pragma unroll
    for (int p = 0; p < 6; p++) {
      const bool live = slot[p] == p;
      const int O0 = Sm(pm(p, 0)), O1 = Sm(pm(p, 1)), O2 = Sm(pm(p, 2));
      const int Oa0 = sel3(al0, O0, O1, O2), Oa1 = sel3(al1, O0, O1, O2), Oa2 = sel3(al2, O0, O1, O2);
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int idx = tid + RT * e;
        const int u2 = idx & 7, u1 = (idx >> 3) & 7, u0 = idx >> 6;  // u2: contiguous X index
        const int xp = RB * Oa0 + u0, xq = RB * Oa1 + u1, xs = RB * Oa2 + u2;
        double v = 0.0;
        if (live && xp < nu && xq < nu && xs < nu) {
          const double *src = X + (t.blocked ? xblock_base(Oa0, Oa1, Oa2, nu, NP) + idx
                                             : ((int64_t)xp * nu + xq) * NP + xs);
          v = COHERENT ? __ldcg(src) : __ldg(src);
        }
        xv[2 * p + e] = v;
      }
    }
    if (!COHERENT && term == 1) {
      cp_async_wait_all();  // term 0 is in W
      __syncthreads();
    }
#pragma unroll
    for (int p = 0; p < 6; p++) {
      if (slot[p] != p) continue;
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const int idx = tid + RT * e;
        const int u2 = idx & 7, u1 = (idx >> 3) & 7, u0 = idx >> 6;
        // block coordinate m takes the u whose placement al is m
        const int c0 = al0 == 0 ? u0 : (al1 == 0 ? u1 : u2);
        const int c1 = al0 == 1 ? u0 : (al1 == 1 ? u1 : u2);
        const int c2 = al0 == 2 ? u0 : (al1 == 2 ? u1 : u2);
        double *w = Wsm + p * SL + soff(c0, c1, c2);
        if (term == 0)
          *w = xv[2 * p + e];
        else
          *w += xv[2 * p + e];
      }
    }
    __syncthreads();
  }
  cp_async_wait_all();  // VOE staging (and term 0 when it went asynchronously)
  if (S0 == S1 && S1 == S2 && tid < RB) Wsm[soff(tid, tid, tid)] = 0.0;  // W_aaa = 0 (ZEROT3)
  __syncthreads();

  reduce_block_bc<KIND>(nu, t, eh, ep, S0, S1, S2, slot, Wsm, Vsm, xpart_slot, vpart);
}

// Phases B and C on W (all orbit blocks, XOR layout) and the VOE staging in
// shared memory; ends with the per-CTA x3 partial in *xpart_slot and the v1
// partials in vpart.
template <int KIND>
__device__ __forceinline__ void reduce_block_bc(int nu, const TupleDev &t, const double *__restrict__ eh,
                                                const double *__restrict__ ep, const int S0, const int S1,
                                                const int S2, const int slot[6], const double *Wsm,
                                                const double *Vsm, double *__restrict__ xpart_slot,
                                                double *__restrict__ vpart) {
  __shared__ double red[RT / 32];
  __shared__ double warpA[RT / 32][RB][3], warpB[RT / 32][4][3], warpC[RT / 32][2][3];
  const int tid = threadIdx.x;
  // ---- phase B: orbits
  const double dijk = eh[t.i] + eh[t.j] + eh[t.k];
  double x3 = 0.0;
  double accA[3] = {0.0, 0.0, 0.0}, accB[3] = {0.0, 0.0, 0.0}, accC[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  const int l0 = tid & 7, l1 = (tid >> 3) & 7;
#pragma unroll
  for (int e = 0; e < 2; e++) {
    const int l2 = (tid >> 6) + 4 * e;
    const int a = RB * S0 + l0, b = RB * S1 + l1, c = RB * S2 + l2;
    bool take = a < nu && b < nu && c < nu && !(a == b && b == c);
    if (S0 == S1 && l0 > l1) take = false;  // the orbit is counted from its a<=b member
    if (S1 == S2 && l1 > l2) take = false;  // ... and from its b<=c member
    if (!take) continue;
    const double mult = (a == b || b == c) ? 0.5 : 1.0;  // three distinct elements, each met twice
    const int lc[3] = {l0, l1, l2};
    double w[6];
#pragma unroll
    for (int p = 0; p < 6; p++)
      w[p] = Wsm[slot[p] * SL + soff(lc[pm(p, 0)], lc[pm(p, 1)], lc[pm(p, 2)])];
    const double dinv = mult * __drcp_rn(dijk - (ep[a] + ep[b] + ep[c]));
    // VOE entry offsets of the three index pairs: (lo, hi) in orientation 0, (hi, lo) in 1
    const int rp[3] = {l1 + 8 * l2, l0 + 8 * l2, l0 + 8 * l1};
    const int rpT[3] = {384 + l2 + 8 * l1, 384 + l2 + 8 * l0, 384 + l1 + 8 * l0};
#pragma unroll
    for (int pi = 0; pi < 6; pi++) {
      // element pi(x); its role values: abc acb bac bca cab cba
      const double wabc = w[compose(pi, 0)], wacb = w[compose(pi, 1)], wbac = w[compose(pi, 2)];
      const double wbca = w[compose(pi, 3)], wcab = w[compose(pi, 4)], wcba = w[compose(pi, 5)];
      x3 += wabc * (8.0 * wabc - 4.0 * (wacb + wcba + wbac) + 2.0 * (wbca + wcab)) * dinv;
      const double z1 = (wabc - wbac) * 2.0 - wacb + wbca;
      const double z2 = (wacb - wbca) * 2.0 - wabc + wbac;
      const double z3 = (wbac - wabc) * 2.0 - wcab + wcba;
      const double z4 = (wbca - wacb) * 2.0 - wcba + wcab;
      const double z5 = (wcab - wcba) * 2.0 - wbac + wabc;
      const double z6 = (wcba - wcab) * 2.0 - wbca + wacb;
      // the element's first index is x_{pm(pi,0)}; its (second, third) pair is the
      // other two coordinates, in order (pm(pi,1), pm(pi,2))
      const int first = pm(pi, 0);
      const int pr = first;                         // pair index = the coordinate left out
      const bool flip = pm(pi, 1) > pm(pi, 2);  // the element's (second, third) = (hi, lo)
      const double *v = Vsm + pr * VPAIR + (flip ? rpT[pr] : rp[pr]);
      const double ci = (z1 * v[0] + z2 * v[64]) * dinv;
      const double cj = (z3 * v[128] + z5 * v[192]) * dinv;
      const double ck = (z4 * v[256] + z6 * v[320]) * dinv;
      if (first == 0) {
        accA[0] += ci; accA[1] += cj; accA[2] += ck;
      } else if (first == 1) {
        accB[0] += ci; accB[1] += cj; accB[2] += ck;
      } else {
        accC[e][0] += ci; accC[e][1] += cj; accC[e][2] += ck;
      }
    }
  }
  // ---- phase C: fixed-order sums.  Lane layout: l0 = lane & 7,
  // l1 = (lane >> 3) + 4 (warp & 1), l2 = (warp >> 1) + 4 e.
  const int warp = tid >> 5, lane = tid & 31;
#pragma unroll
  for (int q = 0; q < 3; q++) {
    double va = accA[q], vb = accB[q], vc0 = accC[0][q], vc1 = accC[1][q];
    va += __shfl_xor_sync(0xffffffffu, va, 8);
    va += __shfl_xor_sync(0xffffffffu, va, 16);  // sum over lanes with equal l0
    vb += __shfl_xor_sync(0xffffffffu, vb, 1);
    vb += __shfl_xor_sync(0xffffffffu, vb, 2);
    vb += __shfl_xor_sync(0xffffffffu, vb, 4);   // sum over lanes with equal l1
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      vc0 += __shfl_xor_sync(0xffffffffu, vc0, off);
      vc1 += __shfl_xor_sync(0xffffffffu, vc1, off);
    }
    if (lane < RB) warpA[warp][lane][q] = va;
    if ((lane & 7) == 0) warpB[warp][lane >> 3][q] = vb;
    if (lane == 0) {
      warpC[warp][0][q] = vc0;
      warpC[warp][1][q] = vc1;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) x3 += __shfl_down_sync(0xffffffffu, x3, off);
  if (lane == 0) red[warp] = x3;
  __syncthreads();

  if (tid == 0) {
    double sum = 0.0;
    for (int w2 = 0; w2 < RT / 32; w2++) sum += red[w2];
    *xpart_slot = sum;
  }
  // v1 partials: position pos (first of equal blocks) collects every coordinate m
  // whose block equals it; written to vslab[X][l][col][q], q = the pair of the
  // other two blocks, so every (block, pair) slot has exactly one writer.
  if (tid < 72) {
    const int pos = tid / 24, l = (tid / 3) % 8, col = tid % 3;
    const int posm[3] = {0, S1 == S0 ? 0 : 1, S2 == S0 ? 0 : (S2 == S1 ? 1 : 2)};
    if (posm[pos] == pos) {
      double v = 0.0;
#pragma unroll
      for (int m = 0; m < 3; m++) {
        if (posm[m] != pos) continue;
        if (m == 0) {
          for (int w2 = 0; w2 < RT / 32; w2++) v += warpA[w2][l][col];
        } else if (m == 1) {
          for (int w2 = (l >> 2); w2 < RT / 32; w2 += 2) v += warpB[w2][l & 3][col];
        } else {
          for (int w2 = 2 * (l & 3); w2 < 2 * (l & 3) + 2; w2++) v += warpC[w2][l >> 2][col];
        }
      }
      const int X = pos == 0 ? S0 : (pos == 1 ? S1 : S2);
      const int Y = pos == 0 ? S1 : S0, Z = pos == 2 ? S1 : S2;  // the other two, Y <= Z
      const int64_t npairs = (int64_t)nb_of(nu) * (nb_of(nu) + 1) / 2;
      const int64_t q = (int64_t)Z * (Z + 1) / 2 + Y;
      vpart[(((int64_t)X * RB + l) * 3 + col) * npairs + q] = v;
    }
  }
}

}  // namespace red
}  // namespace cct
