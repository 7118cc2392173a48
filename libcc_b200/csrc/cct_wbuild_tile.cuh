// The FP64 W-build GEMM tile as a device function, shared by the per-tuple
// kernel (cct_wbuild_f64.cu) and the persistent batch kernel (cct_batch.cu).
// See cct_wbuild_f64.cu for the formulation and the reference lines.
#pragma once
#include "cct_internal.cuh"

namespace cct {
namespace wb {

constexpr int BM = 128, BK = kKB;
constexpr int WM = 32;
constexpr int NWARP = BM / WM;
constexpr int NT = NWARP * 32;
constexpr int STAGES = 3;
// Shared tiles are unpadded (16 doubles a row) with column c of row r stored
// at c ^ 4 (r & 3): the 64-bit fragment loads of a half-warp (rows g = 0..3,
// columns t = 0..3) then hit four disjoint 32-byte bank groups, and a CTA
// needs 64-75 KB, so three fit on an SM.
constexpr int LDS = BK;
__device__ __forceinline__ int swz(int r, int c) { return r * LDS + (c ^ ((r & 3) << 2)); }
constexpr int MF = WM / 16;

template <int BN, int TM = BM>
constexpr int smem_bytes() {
  return STAGES * (TM + BN) * LDS * 8 + TM * 2 * 4 + TM * 2 * 2 * 2;  // tiles, row offsets, packed (p, q)
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
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

// One TM x BN output tile (tile_m, tile_n) of one W-build GEMM job, TM/32
// warps of 32 rows each; every thread of the TM-thread CTA calls it.  Each
// KP-long half of the contraction holds KV = nu + no columns and zero
// padding, whose k4 steps are skipped.  smem_raw holds smem_bytes<BN, TM>().
// It starts with a barrier, so a persistent CTA can call it for consecutive
// tiles on the same shared memory.
template <int BN, int TM = BM>
__device__ __forceinline__ void wbuild_tile(const GemmJob &job, int nu, int64_t KP, int64_t KV, int64_t NP,
                                            int tile_m, int tile_n, unsigned char *smem_raw) {
  constexpr int BM = TM, NT = TM;
  constexpr int NF = BN / 8;
  double *As = reinterpret_cast<double *>(smem_raw);
  double *Bs = As + STAGES * BM * LDS;
  int *rowoff = reinterpret_cast<int *>(Bs + STAGES * BN * LDS);  // [2][BM] row index into E (or -1)
  int16_t *rowpq = reinterpret_cast<int16_t *>(rowoff + 2 * BM);   // [2][BM][2] (p, q) of the row (packed jobs)

  const int64_t M = (int64_t)nu * nu;
  const int64_t m0 = (int64_t)tile_m * BM;
  const int n0 = tile_n * BN;
  const int tid = threadIdx.x;

  __syncthreads();
  for (int r = tid; r < BM; r += NT) {
    const int64_t m = m0 + r;
    if (m < M) {
      const int p = (int)(m / nu), q = (int)(m - (int64_t)(m / nu) * nu);
      rowoff[r] = p * nu + q;
      rowoff[BM + r] = q * nu + p;
      rowpq[2 * r] = (int16_t)p;
      rowpq[2 * r + 1] = (int16_t)q;
      rowpq[2 * (BM + r)] = (int16_t)q;
      rowpq[2 * (BM + r) + 1] = (int16_t)p;
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
    if (!job.packed) {
#pragma unroll
      for (int rr = tid >> 3; rr < BM; rr += NT / 8) {
        const int ro = rowoff[h * BM + rr];
        const double *src = abase + (ro < 0 ? 0 : (int64_t)ro * KP) + k0 + chunk * 2;
        cp_async16(as + swz(rr, chunk * 2), src, ro < 0 ? 0 : 16);
      }
    } else {
      // the row's E values gathered one double at a time: the packed
      // triangle holds (k q | p x) at tri(k, q) of column p, the -T2 rows the
      // k >= nu part; past nu + no the row is zero
      const double *tbase = h ? job.t1 : job.t0;
      const int64_t nutr = (int64_t)nu * (nu + 1) / 2;
      const int nov = (int)(KV - nu);
#pragma unroll
      for (int rr = tid >> 3; rr < BM; rr += NT / 8) {
        const int ro = rowoff[h * BM + rr];
        const int pr = rowpq[2 * (h * BM + rr)], qr = rowpq[2 * (h * BM + rr) + 1];
#pragma unroll
        for (int e = 0; e < 2; e++) {
          const int64_t k = k0 + chunk * 2 + e;
          const double *src = abase;
          int bytes = 0;
          if (ro >= 0 && k < nu) {
            src = abase + (int64_t)pr * nutr + (k >= qr ? k * (k + 1) / 2 + qr : (int64_t)qr * (qr + 1) / 2 + k);
            bytes = 8;
          } else if (ro >= 0 && k < KV) {
            src = tbase + (int64_t)ro * nov + (k - nu);
            bytes = 8;
          }
          cp_async8(as + swz(rr, chunk * 2 + e), src, bytes);
        }
      }
    }
#pragma unroll
    for (int rr = tid >> 3; rr < BN; rr += NT / 8) {
      const double *src = bbase + (int64_t)(n0 + rr) * KP + k0 + chunk * 2;
      cp_async16(bs + swz(rr, chunk * 2), src, 16);
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
    // columns of this k-tile below nu + no; the k4 steps past them multiply zero padding
    const int64_t kv = KV - (int64_t)(kt < ktiles_half ? kt : kt - ktiles_half) * BK;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      if (kk >= kv) break;
      double af[MF][2], bf[NF];
#pragma unroll
      for (int i = 0; i < MF; i++) {
        af[i][0] = as[swz(i * 16 + g, kk + t)];
        af[i][1] = as[swz(i * 16 + g + 8, kk + t)];
      }
#pragma unroll
      for (int j = 0; j < NF; j++) bf[j] = bs[swz(j * 8 + g, kk + t)];
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

}  // namespace wb
}  // namespace cct
