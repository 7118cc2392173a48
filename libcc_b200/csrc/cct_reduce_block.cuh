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
// Element (l0, l1, l2) of a block in shared memory, unpadded.  The term stores
// of phase A and the orbit reads of phase B give a half-warp one coordinate
// with eight values and another with two (2h, 2h+1) on any two of the three
// axes.  The bank pair (word mod 16) is, in bits, l0 ^ (l1 & 6) ^ l2 and
// (l1 ^ l2) & 1: for every ordered pair of axes the four varying bits map to
// it one to one, so none of those accesses has a bank conflict (an XOR of l0
// with l1 + l2 left the pairs on axes (0, 2) and (1, 2) two-way conflicted).
__host__ __device__ constexpr int soff(int l0, int l1, int l2) {
  return 64 * l2 + 8 * (l1 ^ (l2 & 1)) + (l0 ^ (l1 & 6) ^ l2);
}

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
// pair's lower and higher coordinates, orientation 1 VOE(hi, lo, y, z).  The
// copies bring planes (y,z) = (j,k) (k,j) | (i,k) (k,i) | (i,j) (j,i) -- three
// plane pairs (P, P') -- and combine_voe replaces each pair by
// (2P - P', P - 2P'), the two combinations the v1 sums of t1wt3.f90:80-85
// take of it once Z1..Z6 are written as differences of W.  Every element reads
// the VOE entries those lines name, so no symmetry of VOE is assumed.
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

// VOE staging as asynchronous 8-byte copies (one commit group).  A thread
// copies both planes of a plane pair (1152 pairs, five rounds), so after its
// own wait it can combine them (combine_voe) without a barrier.
constexpr int VOE_PAIRS = 3 * 2 * 3 * 64;
// Entry r = u + 8 v holds VOE(lo + u, hi + v) in orientation 0 and
// VOE(hi + u, lo + v) in orientation 1 (u, v < 8); orientation 1 keeps it at
// (u ^ v) + 8 v, so its reads, which vary v across a half-warp, fall on
// distinct bank pairs.
__device__ __forceinline__ int voe_entry(int orient, int u, int v) { return (orient ? u ^ v : u) + 8 * v; }
__device__ __forceinline__ double *voe_pair_slot(double *Vsm, int pq) {
  const int pr = pq / 384, orient = (pq / 192) & 1, k = (pq >> 6) % 3, r = pq & 63;
  return Vsm + pr * VPAIR + orient * 384 + 2 * k * 64 + voe_entry(orient, r & 7, r >> 3);
}
__device__ __forceinline__ void stage_voe(int nu, int no, const TupleDev &t, const double *__restrict__ voe, int S0,
                                          int S1, int S2, double *Vsm) {
  const int tid = threadIdx.x;
  const int64_t nu2 = (int64_t)nu * nu;
#pragma unroll
  for (int it = 0; it < (VOE_PAIRS + RT - 1) / RT; it++) {
    const int pq = tid + RT * it;
    if (pq >= VOE_PAIRS) break;
    const int pr = pq / 384, orient = (pq / 192) & 1, k = (pq >> 6) % 3, r = pq & 63;
    const int Blo = pr == 0 ? S1 : S0, Bhi = pr == 2 ? S1 : S2;  // (b,c), (a,c), (a,b)
    const int f = RB * (orient ? Bhi : Blo) + (r & 7), s2 = RB * (orient ? Blo : Bhi) + (r >> 3);
    const int y = k == 0 ? t.j : t.i, z = k == 2 ? t.j : t.k;  // plane 2k = (y,z), plane 2k+1 = (z,y)
    const bool ok = f < nu && s2 < nu;
    const int64_t e = f + (int64_t)nu * s2;
    double *dst = voe_pair_slot(Vsm, pq);
    cp_async8(dst, voe + (ok ? ((int64_t)z * no + y) * nu2 + e : 0), ok);
    cp_async8(dst + 64, voe + (ok ? ((int64_t)y * no + z) * nu2 + e : 0), ok);
  }
  cp_async_commit();
}

// After the thread's own copies completed: (P, P') -> (2P - P', P - 2P').
__device__ __forceinline__ void combine_voe(double *Vsm) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int it = 0; it < (VOE_PAIRS + RT - 1) / RT; it++) {
    const int pq = tid + RT * it;
    if (pq >= VOE_PAIRS) break;
    double *v = voe_pair_slot(Vsm, pq);
    const double P = v[0], Q = v[64];
    v[0] = fma(2.0, P, -Q);
    v[64] = fma(-2.0, Q, P);
  }
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
// BLOCKED: X in 8 x 8 x 8 blocks (xblock_base), allocated whole for every block
// of round_up(nu, 8)^2 x NP, so every element of a block is read without a
// bounds check: entries of indices >= nu land in W entries that phase B never
// reads (it evaluates only elements whose three indices are < nu).
template <int KIND, bool COHERENT = false, bool BLOCKED = false>
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

  // Blocked X: every X block the CTA will read is one contiguous 4 KB run, so
  // one thread per (term, block) asks L2 for it up front (a bulk prefetch),
  // and all of the CTA's X is in flight before the first term's loads.
  if (BLOCKED && !COHERENT) {
#pragma unroll
    for (int term = 0; term < NTERM; term++) {
      const int g = term_entry(KIND, term, 0);
      const int al0 = term_entry(KIND, term, 1), al1 = term_entry(KIND, term, 2), al2 = term_entry(KIND, term, 3);
#pragma unroll
      for (int p = 0; p < 6; p++) {
        if (tid != 6 * term + p || slot[p] != p) continue;
        const int O0 = Sm(pm(p, 0)), O1 = Sm(pm(p, 1)), O2 = Sm(pm(p, 2));
        const double *blk = t.x[g] + xblock_base(sel3(al0, O0, O1, O2), sel3(al1, O0, O1, O2),
                                                 sel3(al2, O0, O1, O2), nu, NP);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(blk), "r"(SL * 8) : "memory");
      }
    }
  }

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
          const bool ok = BLOCKED || (xp < nu && xq < nu && xs < nu);
          const int64_t off = BLOCKED ? xblock_base(O0, O1, O2, nu, NP) + idx : ((int64_t)xp * nu + xq) * NP + xs;
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
        if (live && (BLOCKED || (xp < nu && xq < nu && xs < nu))) {
          const double *src = X + (BLOCKED ? xblock_base(Oa0, Oa1, Oa2, nu, NP) + idx
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
  combine_voe(Vsm);     // this thread's own plane pairs
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
    // E[4] of the six elements: sum_pi W_pi (8 W_pi - 4 (sum over the three
    // transposed roles) + 2 (the two cyclic roles)).  Transpositions flip the
    // parity of the permutation, cycles keep it, so with Ev / Od the sums of
    // W over the even / odd permutations this is
    //   6 sum_even (W - Ev/3)^2 + 6 sum_odd (W - Od/3)^2 + 4 (Ev - Od)^2.
    const double Ev = w[0] + w[3] + w[4], Od = w[1] + w[2] + w[5];
    const double e3 = Ev * (1.0 / 3.0), o3 = Od * (1.0 / 3.0);
    const double r0 = w[0] - e3, r3 = w[3] - e3, r4 = w[4] - e3;
    const double r1 = w[1] - o3, r2 = w[2] - o3, r5 = w[5] - o3;
    const double sq = fma(r5, r5, fma(r4, r4, fma(r3, r3, fma(r2, r2, fma(r1, r1, r0 * r0)))));
    const double g = Ev - Od;
    x3 = fma(fma(6.0, sq, 4.0 * (g * g)), dinv, x3);
    // v1: with d1 = W_abc - W_bac, d2 = W_bca - W_acb, d3 = W_cba - W_cab of
    // the element (each an even minus an odd permutation, D below),
    //   Z1 V0 + Z2 V1 = d1 (2V0 - V1) + d2 (V0 - 2V1)
    //   Z3 V2 + Z5 V3 = -d1 (2V2 - V3) + d3 (V2 - 2V3)
    //   Z4 V4 + Z6 V5 = d2 (2V4 - V5) - d3 (V4 - 2V5)
    // and the VOE combinations are staged (combine_voe).
    double D[3][3];  // D[e][o] = W(even perm e) - W(odd perm o), evens 0 3 4, odds 1 2 5
#pragma unroll
    for (int ie = 0; ie < 3; ie++)
#pragma unroll
      for (int io = 0; io < 3; io++) D[ie][io] = w[ie == 0 ? 0 : ie + 2] - w[io == 2 ? 5 : io + 1];
    auto diff = [&](int x, int y) {  // W_x - W_y for permutations of opposite parity
      const bool xe = x == 0 || x == 3 || x == 4;
      const int e = xe ? x : y, o = xe ? y : x;
      const double v = D[e == 0 ? 0 : e - 2][o == 5 ? 2 : o - 1];
      return xe ? v : -v;
    };
    // VOE entry offsets of the three index pairs: (lo, hi) in orientation 0, (hi, lo) in 1
    const int rp[3] = {l1 + 8 * l2, l0 + 8 * l2, l0 + 8 * l1};
    const int rpT[3] = {384 + voe_entry(1, l2, l1), 384 + voe_entry(1, l2, l0), 384 + voe_entry(1, l1, l0)};
#pragma unroll
    for (int first = 0; first < 3; first++) {
      // the two elements whose first index is x_first: pi = 2 first (second <
      // third, orientation 0) and 2 first + 1 (orientation 1); their VOE pair is
      // the other two coordinates
      double ci = 0.0, cj = 0.0, ck = 0.0;
#pragma unroll
      for (int flip = 0; flip < 2; flip++) {
        const int pi = 2 * first + flip;
        const double d1 = diff(compose(pi, 0), compose(pi, 2));
        const double d2 = diff(compose(pi, 3), compose(pi, 1));
        const double d3 = diff(compose(pi, 5), compose(pi, 4));
        const double *v = Vsm + first * VPAIR + (flip ? rpT[first] : rp[first]);
        ci = fma(d1, v[0 * 64], fma(d2, v[1 * 64], ci));
        cj = fma(-d1, v[2 * 64], fma(d3, v[3 * 64], cj));
        ck = fma(d2, v[4 * 64], fma(-d3, v[5 * 64], ck));
      }
      if (first == 0) {
        accA[0] = fma(ci, dinv, accA[0]); accA[1] = fma(cj, dinv, accA[1]); accA[2] = fma(ck, dinv, accA[2]);
      } else if (first == 1) {
        accB[0] = fma(ci, dinv, accB[0]); accB[1] = fma(cj, dinv, accB[1]); accB[2] = fma(ck, dinv, accB[2]);
      } else {
        accC[e][0] = fma(ci, dinv, accC[e][0]); accC[e][1] = fma(cj, dinv, accC[e][1]);
        accC[e][2] = fma(ck, dinv, accC[e][2]);
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
