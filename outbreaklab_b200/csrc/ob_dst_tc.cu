// ob_dst_tc.cu — bf16x3 tensor-core sine transforms for the pressure solve (tcgen05 + TMA + TMEM), sm_100a.
//
// Each of the four horizontal transforms of solver.js:155-163 is one batched GEMM over all z-planes at once,
// C[m][n] = sum_k F[m][k] Q[n][k]: F is the field with its planes' rows stacked (m = plane * rows + row, K-major) and Q
// the orthonormal DST-II matrix (N x K, K-major). fp32 operands are split into bf16 pairs (x = hi + lo) and the
// product is accumulated in fp32 TMEM as  F_hi Q_hi + F_hi Q_lo + F_lo Q_hi  (the lo*lo term, ~2^-16 relative, is
// dropped): three tcgen05.mma per K step on the same staged tiles.
//
// Layouts (x fastest unless stated) chain the transforms so that every GEMM reads K-major tiles by TMA:
//   rhs split  S_x[k][j][i]   --X-fwd-->  S_y[k][l][j]  --Y-fwd-->  T2[k][m][l] (fp32)
//   --tridiagonal (transposes through shared memory)-->  S_y[k][l][m]  --Y-inv-->  S_x[k][j][l]  --X-inv-->  phi[k][j][i]
// The first three transforms write the field's row index fastest (lane = row: coalesced column stores straight from
// TMEM); the last writes phi row-major.
// Kernel: persistent, one CTA per SM, tiles of 128 field rows x BN outputs (BN <= 256 chosen per transform so the
// output width divides with little padding: 656 -> 3 x 224), 6 warps: warp 0 issues TMA loads into a 2-stage ring
// (hi/lo tiles of both operands, 128-byte swizzle), warp 1 owns TMEM (two 256-column accumulators) and issues the
// MMAs from one thread, warps 2-5 drain one accumulator (tcgen05.ld) while the MMAs fill the other. No TMA
// multicast. Every mbarrier wait is bounded (ob_tc.cuh).
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ob_poisson.cuh"
#include "ob_tc.cuh"

namespace ob {

namespace {
constexpr int BM = 128;                 // tile rows: rows of the field operand (plane x row)
constexpr int BNMAX = 256;              // tile columns: transform outputs (the DST matrix's rows), runtime <= 256
constexpr int BK = 64;                  // K per pipeline stage: one 128-byte swizzled row of bf16
constexpr int STAGES = 2;
constexpr int A_TILE = BM * BK * 2;     // 16 KB per A operand tile (hi or lo)
constexpr int B_TILE = BNMAX * BK * 2;  // 32 KB per B operand tile slot
// the MMA's N for a tile of BN outputs of which `left` remain in its row of tiles: the multiple of 16 covering them,
// at least 32, at most BN
__host__ __device__ constexpr int narrow_n(int BN, int left) {
  const int r = (left + 15) / 16 * 16;
  return left >= BN ? BN : (r < 32 ? (BN < 32 ? BN : 32) : (r < BN ? r : BN));
}
constexpr int STAGE_BYTES = 2 * A_TILE + 2 * B_TILE;
constexpr int STG_LD = 33;                          // row pitch (floats) of the epilogue's transpose buffer
constexpr int STG_BYTES = 4 * 32 * STG_LD * 4;       // 32 x 32 floats per epilogue warp
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/ + STG_BYTES;
constexpr int kThreads = 192;
constexpr uint32_t kTmemCols = 512;     // two accumulators of 256 columns: the epilogue of one tile overlaps the next

// OUT_T_*: element (m, n) of the product goes to out[(plane * N + n) * ld + r], m = plane * R + r (the field's row
// index is the output's fastest index: the layout the next transform reads K-major). OUT_R_*: out[m * ld + n].
enum OutMode { OUT_T_BF16X2 = 0, OUT_T_F32 = 1, OUT_R_F32 = 2, OUT_R_F32_ADD = 3 };

struct TcOut {
  __nv_bfloat16* hi;
  __nv_bfloat16* lo;
  float* f;
  long ld;   // output pitch (elements)
  int R;     // field rows per plane
  int M;     // valid field rows (planes x R)
  int N;     // valid transform outputs
};
// the epilogue that adds into a row-major output reads the old rows of its tile: one thread per row brings the row's
// [n0, n0 + BN) segment into L2, a tile ahead, so that the loads hit L2 instead of waiting on DRAM
__device__ __forceinline__ void prefetch_rows(const TcOut& out, int m, int n0, int BN) {
  if (m >= out.M) return;
  const float* row = out.f + long(m) * out.ld;
  const int c1 = min(out.N, n0 + BN) - 1;
  for (int c = n0; c < c1; c += 32) tc::prefetch_l2(row + c);
  tc::prefetch_l2(row + c1);
}
}  // namespace

// one tile of a transform: its operands, sizes and output, and its corner
struct TileInfo {
  const CUtensorMap* f_hi;
  const CUtensorMap* f_lo;
  const CUtensorMap* q_hi;
  const CUtensorMap* q_lo;
  int K, BN, m0, n0;
  TcOut out;
};

// the tiles of one transform given by kernel parameters
struct OneProblem {
  const CUtensorMap *f_hi, *f_lo, *q_hi, *q_lo;
  int K, BN, ntn, ntiles;
  TcOut out;
  __device__ __forceinline__ int total() const { return ntiles; }
  __device__ __forceinline__ void tile(int t, TileInfo& ti) const {
    ti.f_hi = f_hi; ti.f_lo = f_lo; ti.q_hi = q_hi; ti.q_lo = q_lo;
    ti.K = K; ti.BN = BN; ti.out = out;
    ti.m0 = (t / ntn) * BM;
    ti.n0 = (t % ntn) * BN;
  }
};

// one transform of every member of an ensemble (grouped launch): problem p owns tiles [start[p], start[p+1]); its
// tensor maps live in global memory, written by the host before any launch that reads them
struct alignas(64) GemmProb {
  CUtensorMap f[2];
  CUtensorMap q[2];
  TcOut out;
  int K, BN, ntn, pad;
};
struct GroupProblems {
  const GemmProb* probs;
  const int* start;
  int n;
  __device__ __forceinline__ int total() const { return __ldg(start + n); }
  __device__ __forceinline__ void tile(int t, TileInfo& ti) const {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(start + mid) <= t) lo = mid;
      else hi = mid - 1;
    }
    const GemmProb& P = probs[lo];
    const int r = t - __ldg(start + lo);
    ti.f_hi = &P.f[0]; ti.f_lo = &P.f[1]; ti.q_hi = &P.q[0]; ti.q_lo = &P.q[1];
    ti.K = P.K; ti.BN = P.BN; ti.out = P.out;
    const int ntn = P.ntn;
    ti.m0 = (r / ntn) * BM;
    ti.n0 = (r % ntn) * ti.BN;
  }
};

// Persistent batched transform C[m][n] = sum_k F[m][k] Q[n][k] in bf16x3: F (the field, M x K, K-major) and Q (the
// DST matrix, N x K, K-major) are each given as bf16 hi/lo planes by TMA maps; tiles of BM x BN are taken round-robin
// (n fastest, so that CTAs working at the same time share the field tile through L2). The tiles come from one problem
// (one model's transform) or from a list of problems (the same transform of every member of an ensemble).
// ONE: the correction pass of the refined solve, in plain bf16 (the hi planes alone, one MMA per k-step): its input
// is the residual of a bf16x3 pass, and the correction needs only bf16 accuracy of itself
template <int MODE, bool ONE, class Src>
__device__ __forceinline__ void dst_tc_run(const Src& src, unsigned int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  // the plain-bf16 pass loads hi planes only: its stages are 48 KB, four of them in the two 96 KB stages' space
  constexpr int NST = ONE ? (STAGES * STAGE_BYTES) / (A_TILE + B_TILE) : STAGES;
  constexpr int SB = ONE ? A_TILE + B_TILE : STAGE_BYTES;
  constexpr int BOFF = ONE ? A_TILE : 2 * A_TILE;   // the matrix tile's place in a stage
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty = full + NST;
  uint64_t* tfull = empty + NST;     // [2] accumulator b holds a finished tile
  uint64_t* tempty = tfull + 2;      // [2] the epilogue has drained accumulator b
  uint64_t* done = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = src.total();

  if (threadIdx.x == 0) {
    for (int s = 0; s < NST; s++) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      tc::mbar_init(&tfull[b], 1);
      tc::mbar_init(&tempty[b], 4);  // one arrival per epilogue warp
    }
    tc::mbar_init(done, 1);
    tc::fence_mbar_init();
  }
  if (warp == 0 && lane == 0 && ntiles > 0) {
    TileInfo ti;
    src.tile(blockIdx.x < unsigned(ntiles) ? int(blockIdx.x) : 0, ti);
    tc::prefetch_tmap(ti.f_hi);
    tc::prefetch_tmap(ti.f_lo);
    tc::prefetch_tmap(ti.q_hi);
    tc::prefetch_tmap(ti.q_lo);
  }
  if (warp == 1) {
    tc::tmem_alloc(tmem_slot, kTmemCols);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer
      int g = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        TileInfo ti;
        src.tile(t, ti);
        const uint32_t bytes = ONE ? uint32_t(A_TILE + ti.BN * BK * 2) : uint32_t(2 * A_TILE + 2 * ti.BN * BK * 2);
        const int nk = (ti.K + BK - 1) / BK;
        for (int kt = 0; kt < nk; kt++, g++) {
          const int s = g % NST;
          const uint32_t ph = (g / NST) & 1;
          if (!(ok = tc::mbar_wait(&empty[s], ph ^ 1, err, 1u))) break;
          uint8_t* st = smem + s * SB;
          tc::mbar_expect_tx(&full[s], bytes);
          tc::tma_load_2d(st, ti.f_hi, &full[s], kt * BK, ti.m0);
          if (!ONE) tc::tma_load_2d(st + A_TILE, ti.f_lo, &full[s], kt * BK, ti.m0);
          tc::tma_load_2d(st + BOFF, ti.q_hi, &full[s], kt * BK, ti.n0);
          if (!ONE) tc::tma_load_2d(st + BOFF + B_TILE, ti.q_lo, &full[s], kt * BK, ti.n0);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      int g = 0, it = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, it++) {
        TileInfo ti;
        src.tile(t, ti);
        // the last tile of a row of tiles multiplies only the matrix rows it needs (its N narrowed to a multiple of 16)
        const uint32_t idesc = tc::idesc_bf16_f32(BM, narrow_n(ti.BN, ti.out.N - ti.n0));
        const int nk = (ti.K + BK - 1) / BK;
        const int b = it & 1;
        if (!(ok = tc::mbar_wait(&tempty[b], ((it >> 1) & 1) ^ 1, err, 2u))) break;
        tc::tc_fence_after();
        const uint32_t acc = tmem + uint32_t(b * 256);
        for (int kt = 0; kt < nk; kt++, g++) {
          const int s = g % NST;
          const uint32_t ph = (g / NST) & 1;
          if (!(ok = tc::mbar_wait(&full[s], ph, err, 2u))) break;
          tc::tc_fence_after();
          const uint8_t* st = smem + s * SB;
          const uint64_t dah = tc::desc_k_sw128(tc::smem_u32(st));
          const uint64_t dal = tc::desc_k_sw128(tc::smem_u32(st + A_TILE));
          const uint64_t dbh = tc::desc_k_sw128(tc::smem_u32(st + BOFF));
          const uint64_t dbl = tc::desc_k_sw128(tc::smem_u32(st + BOFF + B_TILE));
          const int ksub = min(BK, ti.K - kt * BK + 15) / 16;  // 16-wide steps holding data (the rest is zero fill)
          for (int kk = 0; kk < ksub; kk++) {
            const uint64_t o = uint64_t(kk * 2);  // 16 bf16 = 32 bytes, >> 4
            tc::mma_bf16(acc, dah + o, dbh + o, idesc, (kt > 0 || kk > 0) ? 1u : 0u);
            if (!ONE) {
              tc::mma_bf16(acc, dah + o, dbl + o, idesc, 1u);
              tc::mma_bf16(acc, dal + o, dbh + o, idesc, 1u);
            }
          }
          tc::mma_commit(&empty[s]);
        }
        if (ok) tc::mma_commit(&tfull[b]);
      }
      tc::mma_commit(done);  // arrives when every MMA issued above has completed
      tc::mbar_wait(done, 0, err, 4u);
    }
  } else {  // epilogue warps 2..5: TMEM lane quadrant = warp % 4
    const int q = warp & 3;
    int it = 0;
    if (MODE == OUT_R_F32_ADD && int(blockIdx.x) < ntiles) {
      TileInfo tn;
      src.tile(blockIdx.x, tn);
      prefetch_rows(tn.out, tn.m0 + q * 32 + lane, tn.n0, tn.BN);
    }
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
      TileInfo ti;
      src.tile(t, ti);
      if (MODE == OUT_R_F32_ADD && t + int(gridDim.x) < ntiles) {   // the next tile's old rows, while this one drains
        TileInfo tn;
        src.tile(t + gridDim.x, tn);
        prefetch_rows(tn.out, tn.m0 + q * 32 + lane, tn.n0, tn.BN);
      }
      const TcOut& out = ti.out;
      const int BN = ti.BN, m0 = ti.m0, n0 = ti.n0;
      const int b = it & 1;
      if (!tc::mbar_wait(&tfull[b], (it >> 1) & 1, err, 8u)) break;
      tc::tc_fence_after();
      const int m = m0 + q * 32 + lane;  // this thread's row of the tile
      const bool mv = m < out.M;
      const int cend = min(out.N, n0 + BN);  // columns past BN belong to the next tile (BN need not be a multiple of 32)
      const int plane = m / out.R, r = m - plane * out.R;
      for (int ch = 0; ch * 32 < BN; ch++) {
        float v[32];
        tc::tmem_ld32(tmem + uint32_t(b * 256) + (uint32_t(q * 32) << 16) + uint32_t(ch * 32), v);
        const int c0 = n0 + ch * 32;
        if (c0 >= cend) continue;
        if (MODE == OUT_T_BF16X2 || MODE == OUT_T_F32) {
          // column by column: the warp's 32 lanes write 32 consecutive field rows of one output row
          if (mv) {
            const long base = long(plane) * out.N * out.ld + r;
#pragma unroll
            for (int c = 0; c < 32; c++) {
              if (c0 + c < cend) {
                const long a = base + long(c0 + c) * out.ld;
                if (MODE == OUT_T_F32) {
                  out.f[a] = v[c];
                } else if (ONE) {  // the next transform of a plain-bf16 pass reads the hi plane alone
                  out.hi[a] = __float2bfloat16_rn(v[c]);
                } else {
                  __nv_bfloat16 h, l;
                  tc::split_bf16(v[c], h, l);
                  out.hi[a] = h;
                  out.lo[a] = l;
                }
              }
            }
          }
        } else {
          // row-major output: the warp's 32 rows x 32 columns go through shared memory so that each store (and,
          // when adding, each load of the old values) covers one row's 32 consecutive columns: 128 bytes
          float* stg = reinterpret_cast<float*>(smem + STAGES * STAGE_BYTES + 256) + q * 32 * STG_LD;
#pragma unroll
          for (int c = 0; c < 32; c++) stg[lane * STG_LD + c] = v[c];
          __syncwarp();
          const bool cv = c0 + lane < cend;
          const int mrow = m0 + q * 32;
          float old[32];
          if (MODE == OUT_R_F32_ADD) {
#pragma unroll
            for (int r = 0; r < 32; r++) old[r] = (cv && mrow + r < out.M) ? out.f[long(mrow + r) * out.ld + c0 + lane] : 0.f;
          }
#pragma unroll
          for (int r = 0; r < 32; r++) {
            if (cv && mrow + r < out.M) {
              const float val = stg[r * STG_LD + lane];
              out.f[long(mrow + r) * out.ld + c0 + lane] = MODE == OUT_R_F32_ADD ? old[r] + val : val;
            }
          }
          __syncwarp();
        }
      }
      // the accumulator is free again once every lane's tcgen05.ld of it has completed
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&tempty[b]);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem, kTmemCols);
  }
}

template <int MODE, bool ONE = false>
__global__ void __launch_bounds__(kThreads, 1)
    k_dst_tc(const __grid_constant__ CUtensorMap tF_hi, const __grid_constant__ CUtensorMap tF_lo,
             const __grid_constant__ CUtensorMap tQ_hi, const __grid_constant__ CUtensorMap tQ_lo, int K, int BN, TcOut out,
             unsigned int* err) {
  const int ntn = (out.N + BN - 1) / BN;
  const OneProblem src{&tF_hi, &tF_lo, &tQ_hi, &tQ_lo, K, BN, ntn, ((out.M + BM - 1) / BM) * ntn, out};
  dst_tc_run<MODE, ONE>(src, err);
}

template <int MODE, bool ONE = false>
__global__ void __launch_bounds__(kThreads, 1) k_dst_tc_grp(const GemmProb* __restrict__ probs, const int* __restrict__ start, int n,
                                                            unsigned int* err) {
  const GroupProblems src{probs, start, n};
  dst_tc_run<MODE, ONE>(src, err);
}

// ---------------------------------------------------------------------------------------------------------------
// fp32 field -> bf16 hi/lo planes with a padded row pitch (rows of `cols` values, pitch ld), zero in the padding
// ---------------------------------------------------------------------------------------------------------------
// ---------------------------------------------------------------------------------------------------------------
// The same transform on tiles of 256 field rows x BN outputs computed by a pair of SMs (a cluster of 2 CTAs running
// tcgen05.mma.cta_group::2, M = 256): each CTA loads its own 128 field rows and half of the DST-matrix tile (BN / 2
// rows), the first CTA issues the MMAs, and each CTA's TMEM holds its 128 rows of the product. Per k-step a CTA then
// loads 32 KB of field and BN x 128 bytes of matrix (60 KB at BN = 224) for the same MMA work per SM as the single-SM
// tile that loads 88 KB: a third less operand traffic through L2, which bounds the single-SM transform. Both CTAs'
// TMA loads (no multicast) count on the first CTA's stage barrier; the first CTA's commits release both CTAs' stages
// and accumulators; the epilogue warps of both CTAs report a drained accumulator to the first CTA. Results equal the
// single-SM kernel's bit for bit (the same bf16 products, accumulated over the same k-steps).
// ---------------------------------------------------------------------------------------------------------------
namespace {
// shared memory: the epilogue's transpose buffers, the barriers, then a ring of as many stages (field hi/lo, half the
// matrix tile hi/lo) as the tile width leaves room for: 3 at BN = 224 or 256, 4 at BN <= 144 (every slot a multiple
// of 1024 bytes, as the 128-byte swizzle wants)
constexpr int MAXST2 = 8;
constexpr int BAR2_OFF = (STG_BYTES + 1023) / 1024 * 1024;
constexpr int RING2_OFF = BAR2_OFF + 1024;
constexpr int SMEM2_BYTES = 227 * 1024;                      // the most a block may use
constexpr int RING2_BYTES = SMEM2_BYTES - 1024 /*align*/ - RING2_OFF;
__host__ __device__ constexpr int half_bytes2(int BN) { return BN / 2 * BK * 2; }
// a stage holds the field's hi (and lo) tile, then the matrix half's hi (and lo): the plain-bf16 pass (ONE) loads hi
// planes only, so its stages are half as large and twice as many fit
__host__ __device__ constexpr int stage2_bytes(int BN, bool one) { return one ? A_TILE + half_bytes2(BN) : 2 * A_TILE + 2 * half_bytes2(BN); }
__host__ __device__ constexpr int b_off2(bool one) { return one ? A_TILE : 2 * A_TILE; }
__host__ __device__ constexpr int stages2(int BN, bool one) {
  return RING2_BYTES / stage2_bytes(BN, one) < MAXST2 ? RING2_BYTES / stage2_bytes(BN, one) : MAXST2;
}
static_assert(stages2(BNMAX, false) >= 3, "three stages at the widest tile");
}  // namespace

// The pair kernel's tile list. Tiles t < base are whole tiles of BN outputs (n fastest); when the persistent grid's
// last round would be at most half full, the tiles of that round are split along N into S sub-tiles of w outputs each
// (tile tt = base + u / S, sub-tile u % S), so that more pairs share the round. A sub-tile multiplies the same bf16
// products over the same k-steps as the whole tile (the same bits); it stops at its tile's last column, so no output
// is written twice.
struct PairSched {
  int ntn, BN, N, base, S, w, total;
  // row tile, first output, MMA width (a multiple of 16) and end of the outputs this tile writes
  __device__ __forceinline__ void at(int t, int& mt, int& n0, int& nv, int& ce) const {
    if (t < base) {
      mt = t / ntn;
      n0 = (t % ntn) * BN;
      ce = min(N, n0 + BN);
      nv = narrow_n(BN, N - n0);
      return;
    }
    const int u = t - base, tt = base + u / S, sub = u - (u / S) * S;
    mt = tt / ntn;
    const int nt0 = (tt % ntn) * BN;
    n0 = nt0 + sub * w;
    ce = min(min(N, nt0 + BN), n0 + w);
    nv = narrow_n(w, ce - n0);
  }
};

template <int MODE, bool ONE = false>
__global__ void __launch_bounds__(kThreads, 1)
    k_dst_tc2(const __grid_constant__ CUtensorMap tF_hi, const __grid_constant__ CUtensorMap tF_lo,
              const __grid_constant__ CUtensorMap tQ_hi, const __grid_constant__ CUtensorMap tQ_lo, int K, PairSched sc, TcOut out,
              unsigned int* err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + BAR2_OFF);
  uint64_t* empty = full + MAXST2;
  uint64_t* tfull = empty + MAXST2;   // [2] accumulator b holds a finished tile (both CTAs)
  uint64_t* tempty = tfull + 2;       // [2] both CTAs' epilogues have drained accumulator b (used in the first CTA)
  uint64_t* done = tempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = tc::cluster_rank();
  const bool lead = rank == 0;
  const int BN = sc.BN, ntiles = sc.total;
  const int pair = int(blockIdx.x >> 1), npairs = int(gridDim.x >> 1);
  const int bh = BN / 2;
  const int nk = (K + BK - 1) / BK;
  const int nst = stages2(BN, ONE), sbytes = stage2_bytes(BN, ONE), hbytes = half_bytes2(BN);
  constexpr int BOFF = b_off2(ONE);
  uint8_t* ring = smem + RING2_OFF;

  if (threadIdx.x == 0) {
    for (int s = 0; s < MAXST2; s++) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      tc::mbar_init(&tfull[b], 1);
      tc::mbar_init(&tempty[b], 8);  // four epilogue warps in each CTA
    }
    tc::mbar_init(done, 1);
    tc::fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tc::prefetch_tmap(&tF_hi);
    tc::prefetch_tmap(&tF_lo);
    tc::prefetch_tmap(&tQ_hi);
    tc::prefetch_tmap(&tQ_lo);
  }
  if (warp == 1) {
    tc::tmem_alloc_pair(tmem_slot, kTmemCols);
    tc::tmem_relinquish_pair();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::cluster_sync();  // both CTAs' barriers exist before a load or an arrival crosses the pair
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {  // TMA producer of this CTA's half of every stage
      const uint32_t bytes = ONE ? 2u * uint32_t(A_TILE + bh * BK * 2) : 2u * uint32_t(2 * A_TILE + 2 * bh * BK * 2);
      int g = 0;
      bool ok = true;
      for (int t = pair; t < ntiles && ok; t += npairs) {
        // the second CTA holds the second half of the N columns the pair's MMAs use
        int mt, nt0, nv, ce;
        sc.at(t, mt, nt0, nv, ce);
        const int m0 = mt * 2 * BM + int(rank) * BM, n0 = nt0 + int(rank) * (nv / 2);
        for (int kt = 0; kt < nk; kt++, g++) {
          const int s = g % nst;
          const uint32_t ph = (g / nst) & 1;
          if (!(ok = tc::mbar_wait(&empty[s], ph ^ 1, err, 1u))) break;
          uint8_t* st = ring + s * sbytes;
          const uint32_t fb = tc::mapa_shared(tc::smem_u32(&full[s]), 0);
          if (lead) tc::mbar_expect_tx(&full[s], bytes);
          tc::tma_load_2d_pair(st, &tF_hi, fb, kt * BK, m0);
          if (!ONE) tc::tma_load_2d_pair(st + A_TILE, &tF_lo, fb, kt * BK, m0);
          tc::tma_load_2d_pair(st + BOFF, &tQ_hi, fb, kt * BK, n0);
          if (!ONE) tc::tma_load_2d_pair(st + BOFF + hbytes, &tQ_lo, fb, kt * BK, n0);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && lead) {  // MMA issuer of the pair
      int g = 0, it = 0;
      bool ok = true;
      for (int t = pair; t < ntiles && ok; t += npairs, it++) {
        int mt, n0, nv, ce;
        sc.at(t, mt, n0, nv, ce);
        const uint32_t idesc = tc::idesc_bf16_f32(2 * BM, nv);
        const int b = it & 1;
        if (!(ok = tc::mbar_wait(&tempty[b], ((it >> 1) & 1) ^ 1, err, 2u))) break;
        tc::tc_fence_after();
        const uint32_t acc = tmem + uint32_t(b * 256);
        for (int kt = 0; kt < nk; kt++, g++) {
          const int s = g % nst;
          const uint32_t ph = (g / nst) & 1;
          if (!(ok = tc::mbar_wait(&full[s], ph, err, 2u))) break;
          tc::tc_fence_after();
          const uint8_t* st = ring + s * sbytes;
          const uint64_t dah = tc::desc_k_sw128(tc::smem_u32(st));
          const uint64_t dal = tc::desc_k_sw128(tc::smem_u32(st + A_TILE));
          const uint64_t dbh = tc::desc_k_sw128(tc::smem_u32(st + BOFF));
          const uint64_t dbl = tc::desc_k_sw128(tc::smem_u32(st + BOFF + hbytes));
          const int ksub = min(BK, K - kt * BK + 15) / 16;
          for (int kk = 0; kk < ksub; kk++) {
            const uint64_t o = uint64_t(kk * 2);
            tc::mma_bf16_pair(acc, dah + o, dbh + o, idesc, (kt > 0 || kk > 0) ? 1u : 0u);
            if (!ONE) {
              tc::mma_bf16_pair(acc, dah + o, dbl + o, idesc, 1u);
              tc::mma_bf16_pair(acc, dal + o, dbh + o, idesc, 1u);
            }
          }
          tc::mma_commit_pair(&empty[s], 0x3);
        }
        if (ok) tc::mma_commit_pair(&tfull[b], 0x3);
      }
      tc::mma_commit_pair(done, 0x1);
      tc::mbar_wait(done, 0, err, 4u);
    }
  } else {  // epilogue warps 2..5 of both CTAs: TMEM lane quadrant = warp % 4, this CTA's 128 rows of the pair tile
    const int q = warp & 3;
    const uint32_t tempty_lead = tc::mapa_shared(tc::smem_u32(tempty), 0);
    int it = 0;
    if (MODE == OUT_R_F32_ADD && pair < ntiles) {
      int mt, n0, nv, ce;
      sc.at(pair, mt, n0, nv, ce);
      prefetch_rows(out, mt * 2 * BM + int(rank) * BM + q * 32 + lane, n0, ce - n0);
    }
    for (int t = pair; t < ntiles; t += npairs, it++) {
      int mt, n0, nv, cend;
      sc.at(t, mt, n0, nv, cend);
      const int m0 = mt * 2 * BM + int(rank) * BM;
      if (MODE == OUT_R_F32_ADD && t + npairs < ntiles) {   // the next tile's old rows, while this one drains
        int mtn, n0n, nvn, cen;
        sc.at(t + npairs, mtn, n0n, nvn, cen);
        prefetch_rows(out, mtn * 2 * BM + int(rank) * BM + q * 32 + lane, n0n, cen - n0n);
      }
      const int b = it & 1;
      if (!tc::mbar_wait(&tfull[b], (it >> 1) & 1, err, 8u)) break;
      tc::tc_fence_after();
      const int m = m0 + q * 32 + lane;
      const bool mv = m < out.M;
      const int plane = m / out.R, r = m - plane * out.R;
      for (int ch = 0; ch * 32 < BN; ch++) {   // a sub-tile's chunks past its end are skipped below
        float v[32];
        tc::tmem_ld32(tmem + uint32_t(b * 256) + (uint32_t(q * 32) << 16) + uint32_t(ch * 32), v);
        const int c0 = n0 + ch * 32;
        if (c0 >= cend) continue;
        if (MODE == OUT_T_BF16X2 || MODE == OUT_T_F32) {
          if (mv) {
            const long base = long(plane) * out.N * out.ld + r;
#pragma unroll
            for (int c = 0; c < 32; c++) {
              if (c0 + c < cend) {
                const long a = base + long(c0 + c) * out.ld;
                if (MODE == OUT_T_F32) {
                  out.f[a] = v[c];
                } else if (ONE) {
                  out.hi[a] = __float2bfloat16_rn(v[c]);
                } else {
                  __nv_bfloat16 h, l;
                  tc::split_bf16(v[c], h, l);
                  out.hi[a] = h;
                  out.lo[a] = l;
                }
              }
            }
          }
        } else {
          float* stg = reinterpret_cast<float*>(smem) + q * 32 * STG_LD;
#pragma unroll
          for (int c = 0; c < 32; c++) stg[lane * STG_LD + c] = v[c];
          __syncwarp();
          const bool cv = c0 + lane < cend;
          const int mrow = m0 + q * 32;
          float old[32];
          if (MODE == OUT_R_F32_ADD) {
#pragma unroll
            for (int rr = 0; rr < 32; rr++) old[rr] = (cv && mrow + rr < out.M) ? out.f[long(mrow + rr) * out.ld + c0 + lane] : 0.f;
          }
          // every staged value read before the first store, so that the 32 row stores issue back to back
          float val[32];
#pragma unroll
          for (int rr = 0; rr < 32; rr++) val[rr] = stg[rr * STG_LD + lane];
#pragma unroll
          for (int rr = 0; rr < 32; rr++)
            if (cv && mrow + rr < out.M) out.f[long(mrow + rr) * out.ld + c0 + lane] = MODE == OUT_R_F32_ADD ? old[rr] + val[rr] : val[rr];
          __syncwarp();
        }
      }
      // the accumulator is free again once both CTAs' epilogue warps have read it
      tc::tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        if (lead) tc::mbar_arrive(&tempty[b]);
        else tc::mbar_arrive_cluster(tempty_lead + uint32_t(b * 8));
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::cluster_sync();  // the second CTA's shared memory and TMEM stay until the pair's last MMA and epilogue are done
  if (warp == 1) {
    tc::tc_fence_after();
    tc::tmem_dealloc_pair(tmem, kTmemCols);
  }
}

__global__ void k_split_rows(const float* __restrict__ src, long rows, int cols, __nv_bfloat16* __restrict__ hi,
                             __nv_bfloat16* __restrict__ lo, int ld) {
  const long n = rows * ld;
  for (long t = blockIdx.x * long(blockDim.x) + threadIdx.x; t < n; t += long(gridDim.x) * blockDim.x) {
    const long r = t / ld;
    const int c = int(t - r * ld);
    const float x = c < cols ? src[r * cols + c] : 0.f;
    tc::split_bf16(x, hi[t], lo[t]);
  }
}

// ---------------------------------------------------------------------------------------------------------------
// residual of the solved field, accumulated in FP64: r = rhs - [rho_c lap_h(phi) + lo phi(k-1) + diag phi + up phi(k+1)]
// with phi = 0 on the faces beyond the grid (antisymmetric ghosts, the operator the sine transforms diagonalise) and
// Neumann in z (lo = 0 at the ground, up = 0 at the lid); written split for the correction solve
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void resid_body(int nx, int ny, int nz, double idx2, const float4* __restrict__ zop, const float* __restrict__ rhs,
                                           const float* __restrict__ phi, __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo,
                                           int ld, const int BX, const int BY, const int BZ) {
  const int i = BX * blockDim.x + threadIdx.x, j = BY, k = BZ;
  if (i >= nx) return;
  const long pl = long(nx) * ny;
  const long o = long(k) * pl + long(j) * nx + i;
  const double p = phi[o];
  const double xm = i > 0 ? double(phi[o - 1]) : -p, xp = i < nx - 1 ? double(phi[o + 1]) : -p;
  const double ym = j > 0 ? double(phi[o - nx]) : -p, yp = j < ny - 1 ? double(phi[o + nx]) : -p;
  const float4 z = __ldg(zop + k);
  const double zm = k > 0 ? double(phi[o - pl]) : 0.0, zp = k < nz - 1 ? double(phi[o + pl]) : 0.0;
  const double Lp = double(z.w) * (xm + xp + ym + yp - 4.0 * p) * idx2 + double(z.x) * zm + double(z.z) * p + double(z.y) * zp;
  const float r = float(double(rhs[o]) - Lp);
  const long t = (long(k) * ny + j) * ld + i;
  tc::split_bf16(r, hi[t], lo[t]);
}
__global__ void k_resid(int nx, int ny, int nz, double idx2, const float4* __restrict__ zop, const float* __restrict__ rhs,
                        const float* __restrict__ phi, __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo, int ld) {
  resid_body(nx, ny, nz, idx2, zop, rhs, phi, hi, lo, ld, blockIdx.x, blockIdx.y, blockIdx.z);
}
// FP64 norms of the residual r = rhs - A phi (A as in resid_body) and of rhs, over a grid-stride loop: each block
// writes (max|r|, sum r^2, max|rhs|, sum rhs^2) to part[4 * blockIdx.x]; k_norm_final combines them in block order
__global__ void __launch_bounds__(256) k_resid_norm(int nx, int ny, int nz, double idx2, const float4* __restrict__ zop,
                                                    const float* __restrict__ rhs, const float* __restrict__ phi,
                                                    double* __restrict__ part) {
  __shared__ double red[4][8];
  const long pl = long(nx) * ny, n = pl * nz;
  double rmax = 0.0, rss = 0.0, bmax = 0.0, bss = 0.0;
  for (long o = blockIdx.x * long(blockDim.x) + threadIdx.x; o < n; o += long(gridDim.x) * blockDim.x) {
    const int k = int(o / pl);
    const long q = o - k * pl;
    const int j = int(q / nx), i = int(q - long(j) * nx);
    const double p = phi[o];
    const double xm = i > 0 ? double(phi[o - 1]) : -p, xp = i < nx - 1 ? double(phi[o + 1]) : -p;
    const double ym = j > 0 ? double(phi[o - nx]) : -p, yp = j < ny - 1 ? double(phi[o + nx]) : -p;
    const float4 z = __ldg(zop + k);
    const double zm = k > 0 ? double(phi[o - pl]) : 0.0, zp = k < nz - 1 ? double(phi[o + pl]) : 0.0;
    const double b = rhs[o];
    const double r = b - (double(z.w) * (xm + xp + ym + yp - 4.0 * p) * idx2 + double(z.x) * zm + double(z.z) * p + double(z.y) * zp);
    rmax = fmax(rmax, fabs(r));
    rss += r * r;
    bmax = fmax(bmax, fabs(b));
    bss += b * b;
  }
  for (int o = 16; o > 0; o >>= 1) {
    rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
    rss += __shfl_xor_sync(0xffffffffu, rss, o);
    bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
    bss += __shfl_xor_sync(0xffffffffu, bss, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) { red[0][w] = rmax; red[1][w] = rss; red[2][w] = bmax; red[3][w] = bss; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0, c = 0, d = 0;
    for (int u = 0; u < int(blockDim.x >> 5); u++) { a = fmax(a, red[0][u]); b += red[1][u]; c = fmax(c, red[2][u]); d += red[3][u]; }
    part[4 * blockIdx.x + 0] = a; part[4 * blockIdx.x + 1] = b; part[4 * blockIdx.x + 2] = c; part[4 * blockIdx.x + 3] = d;
  }
}
__global__ void k_norm_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  double a = 0, b = 0, c = 0, d = 0;
  for (int u = 0; u < nb; u++) { a = fmax(a, part[4 * u]); b += part[4 * u + 1]; c = fmax(c, part[4 * u + 2]); d += part[4 * u + 3]; }
  out[0] = a; out[1] = b; out[2] = c; out[3] = d;
}

// residual of phi for rhs under the solve's operator, in FP64 on the device: rel[0] = max|r| / max|rhs|,
// rel[1] = ||r||_2 / ||rhs||_2 (scratch: 4 * 1024 + 4 doubles)
int poisson_residual(const PoissonPlan& P, const float* rhs, const float* phi, double* scratch, double rel[2], cudaStream_t s) {
  constexpr int nb = 1024;
  k_resid_norm<<<nb, 256, 0, s>>>(P.nx, P.ny, P.nz, 1.0 / (P.dx * P.dx), P.zop, rhs, phi, scratch);
  k_norm_final<<<1, 1, 0, s>>>(scratch, nb, scratch + 4 * nb);
  double h[4];
  if (cudaMemcpyAsync(h, scratch + 4 * nb, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
    set_error("poisson residual: %s", cudaGetErrorString(cudaGetLastError()));
    return OB_ERR_DEVICE;
  }
  rel[0] = h[2] > 0 ? h[0] / h[2] : 0.0;
  rel[1] = h[3] > 0 ? std::sqrt(h[1] / h[3]) : 0.0;
  return OB_OK;
}

struct ResidProb {
  int nx, ny, nz, ld;
  double idx2;
  const float4* zop;
  const float* rhs;
  const float* phi;
  __nv_bfloat16* hi;
  __nv_bfloat16* lo;
};
// grid (x-y blocks of all members, 1, levels): map[blockIdx.x] = (member, bx | by << 16)
__global__ void k_resid_grp(const ResidProb* __restrict__ probs, const uint2* __restrict__ map) {
  const uint2 e = __ldg(map + blockIdx.x);
  const ResidProb& P = probs[e.x];
  resid_body(P.nx, P.ny, P.nz, P.idx2, P.zop, P.rhs, P.phi, P.hi, P.lo, P.ld, int(e.y & 0xffffu), int(e.y >> 16u), int(blockIdx.z));
}

// ---------------------------------------------------------------------------------------------------------------
// tridiagonal solves in z per mode (l, m) (solver.js:70-103): T2[k][m][l] fp32 in, S_y[k][l][m] bf16 hi/lo out.
// Block = 32 modes in l x 16 in m; forward-sweep coefficients and the right-hand side stay in registers; the result
// goes out through a shared-memory transpose so that every thread stores 16 consecutive m (32 bytes per output
// row: whole sectors). The lowest 2 x 2 modes (near-singular:
// Neumann in z, shift ~ -(pi/L)^2) use FP64 factors precomputed on the host at set_density.
// ---------------------------------------------------------------------------------------------------------------
// modes in m per block: 16 (whole 32-byte sectors per output row) while a thread's NZ levels fit in the 128 registers
// of a 512-thread block, else 8
template <int NZ>
constexpr int tri_tm() { return NZ > 40 ? 8 : 16; }
// the reciprocal of a mode's pivot at one level, den = diag + shift * rhoC - lower * c'_{k-1} (solver.js:88-90), with
// c'_{k-1} in the innermost product so that nothing of it is computed ahead of the recurrence; rcp.approx is one
// MUFU instruction, at most 1 ulp from the rounded reciprocal (the pivots are normal numbers: |den| >= the diagonal's
// 1/dz^2 scale)
__device__ __forceinline__ float tri_pivot_rcp(const float4& o, float shift, float cprev) {
  const float den = fmaf(shift, o.w, fmaf(-o.x, cprev, o.z));
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(den));
  return r;
}
template <int NZ>
__device__ __forceinline__ void tri_body(int nxp, int nyp, int ldy, const float* __restrict__ lam, const float4* __restrict__ zop,
                                         const double* __restrict__ low, const float* __restrict__ T2,
                                         __nv_bfloat16* __restrict__ ohi, __nv_bfloat16* __restrict__ olo, const int BX, const int BY) {
  constexpr int KC = 16;  // levels per transpose chunk
  constexpr int TRI_TM = tri_tm<NZ>();
  __shared__ float tile[KC][TRI_TM][33];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
  const int l = BX * 32 + tx, m = BY * TRI_TM + ty;
  const bool act = l < nxp && m < nyp;
  const bool lowm = l < 2 && m < 2;
  const long sxy = long(nxp) * nyp;
  float x[NZ];
  if (act && !lowm) {
    const float shift = __ldg(lam + l) + __ldg(lam + nxp + m);
    const float* h = T2 + long(m) * nxp + l;
#pragma unroll
    for (int k = 0; k < NZ; k++) x[k] = __ldg(h + sxy * k);  // all loads issued up front; d and then x replace them
    float cp[NZ];
    float cprev = 0.f, dprev = 0.f;
#pragma unroll
    for (int k = 0; k < NZ; k++) {
      const float4 o = __ldg(zop + k);
      const float rd = tri_pivot_rcp(o, shift, cprev);
      cprev = o.y * rd;
      dprev = fmaf(-o.x, dprev, x[k]) * rd;
      cp[k] = cprev;
      x[k] = dprev;
    }
#pragma unroll
    for (int k = NZ - 2; k >= 0; k--) x[k] = fmaf(-cp[k], x[k + 1], x[k]);
  } else if (act) {
    // low mode: low[(mode*2 + 0)*NZ + k] = 1/den_k, low[(mode*2 + 1)*NZ + k] = c'_k (FP64, host-factored)
    const int mode = m * 2 + l;
    const double* rd = low + (mode * 2) * NZ;
    const double* cpd = rd + NZ;
    const float* h = T2 + long(m) * nxp + l;
    double d[NZ];
    double dprev = 0.0;
    for (int k = 0; k < NZ; k++) {
      const double lo = double(__ldg(zop + k).x);
      dprev = (double(h[sxy * k]) - lo * dprev) * rd[k];
      d[k] = dprev;
    }
    for (int k = NZ - 2; k >= 0; k--) d[k] = d[k] - cpd[k] * d[k + 1];
#pragma unroll
    for (int k = 0; k < NZ; k++) x[k] = float(d[k]);
  } else {
#pragma unroll
    for (int k = 0; k < NZ; k++) x[k] = 0.f;
  }
  // transposed store, KC levels at a time: every thread then writes 8 consecutive m of one (level, l) row
#pragma unroll
  for (int kc = 0; kc < NZ; kc += KC) {
#pragma unroll
    for (int kk = 0; kk < KC; kk++)
      if (kc + kk < NZ) tile[kk][ty][tx] = x[kc + kk];
    __syncthreads();
    const int nkc = NZ - kc < KC ? NZ - kc : KC;
    for (int t = tid; t < nkc * 32; t += 32 * TRI_TM) {
      const int kk = t >> 5, lx = t & 31;
      const int ll = BX * 32 + lx;
      if (ll < nxp) {
        __align__(16) __nv_bfloat16 h16[TRI_TM], l16[TRI_TM];
#pragma unroll
        for (int u = 0; u < TRI_TM; u++) tc::split_bf16(tile[kk][u][lx], h16[u], l16[u]);
        // rows hold ldy (a multiple of 8) values: 16-byte aligned; columns past nyp land in the row's zero padding
        // when the pitch has room for them, else they are skipped
        const long o = (long(kc + kk) * nxp + ll) * ldy + BY * TRI_TM;
#pragma unroll
        for (int h = 0; h < TRI_TM / 8; h++)
          if (BY * TRI_TM + h * 8 + 8 <= ldy) {
            *reinterpret_cast<uint4*>(ohi + o + h * 8) = *reinterpret_cast<const uint4*>(h16 + h * 8);
            if (olo) *reinterpret_cast<uint4*>(olo + o + h * 8) = *reinterpret_cast<const uint4*>(l16 + h * 8);
          }
      }
    }
    __syncthreads();
  }
}
// ---------------------------------------------------------------------------------------------------------------
// The tridiagonals of one model's solve through shared memory, every transfer a TMA tile (solver.js:70-103).
// A block takes 16 l x 16 m modes (one per thread; warp = 16 consecutive l at two m):
//   1. one 3-D TMA load brings the block's [NZ][16][16] fp32 tile of T2[k][m][l] into shared memory (zero outside);
//   2. each thread runs the Thomas sweep of its mode: c' in registers, d and then x updated in place in the tile
//      (a warp's tile row is 32 consecutive floats: no bank conflicts), the 2 x 2 lowest modes in FP64 with the
//      host-factored coefficients. The z-operator (lower, upper, diagonal, rhoC per level) is a kernel parameter,
//      so every coefficient is a constant-bank operand of the instruction that uses it (no load in the recurrence),
//      and the reciprocal of each pivot is the hardware's rcp.approx (at most 1 ulp from the rounded quotient);
//   3. one barrier later every thread reads the NZ/8 half rows (level, l, 8 m) it will write, splits them into bf16
//      hi / lo (hi alone for a plain-bf16 pass, HI_ONLY) and holds them in registers; after a second barrier they go
//      back into the tile as [NZ][16][16] hi and lo rows, and one thread stores each with one 3-D TMA store into
//      S_y[k][l][m]: 32-byte rows, whole DRAM sectors (rows of 8 m left each sector half written by two blocks, which
//      doubled the L2 write transactions and made L2 fetch sectors back from DRAM).
// 64 registers and NZ KB of shared memory per 256-thread block (NZ <= 40: four blocks per SM), so one block's loads
// overlap another's sweeps and stores.
// ---------------------------------------------------------------------------------------------------------------
constexpr int TRI_TL = 16, TRI_TM = 16;
template <int NZ>
constexpr int tri_smem_bytes() { return NZ * TRI_TM * TRI_TL * 4 + 4 * NZ * 8 /*FP64 low modes*/ + 128 /*align*/ + 16 /*barrier*/; }
// the z-operator by value: (lower, upper, diagonal, rhoC) of each level (solver.js:139-146)
template <int NZ>
struct TriZ {
  float4 z[NZ];
};

// One block's tile (modes l0 .. l0 + 15, m0 .. m0 + 15) given its tensor maps (kernel parameters, or a member's maps
// in global memory) and zop(k), the z-operator of level k (a constant-bank parameter, or a copy in shared memory).
template <int NZ, bool HI_ONLY, class Zop>
__device__ __forceinline__ void tri_tma_tile(const CUtensorMap* tIn, const CUtensorMap* tHi, const CUtensorMap* tLo, int nxp, int nyp,
                                             const float* __restrict__ lam, const Zop& zop, const double* __restrict__ low,
                                             unsigned int* err, const int l0, const int m0, uint8_t* smraw) {
  static_assert(NZ % 8 == 0, "levels come in whole groups of 8");
  float* tile = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
  double* dlow = reinterpret_cast<double*>(tile + NZ * TRI_TM * TRI_TL);   // [4][NZ]: d of the FP64 low modes
  uint64_t* bar = reinterpret_cast<uint64_t*>(dlow + 4 * NZ);
  static_assert(TRI_TL == 16 && TRI_TM == 16, "thread and output mappings below assume 16 x 16 modes");
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4, tid = threadIdx.x;
  if (tid == 0) {
    tc::prefetch_tmap(tIn);
    tc::mbar_init(bar, 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    tc::mbar_expect_tx(bar, NZ * TRI_TM * TRI_TL * 4);
    tc::tma_load_3d(tile, tIn, bar, l0, m0, 0);
  }
  const int l = l0 + tx, m = m0 + ty;
  const bool act = l < nxp && m < nyp;
  // what the sweep needs besides the tile, fetched while the tile is in flight
  const float shift = act ? __ldg(lam + l) + __ldg(lam + nxp + m) : 0.f;
  // one thread waits (bounded) for the tile and tells the others; if it never arrived the error word reports it and
  // every thread leaves before touching the tile
  __shared__ int s_ok;
  if (tid == 0) s_ok = tc::mbar_wait(bar, 0, err, 16u) ? 1 : 0;
  __syncthreads();
  if (!s_ok) return;
  float* col = tile + ty * TRI_TL + tx;           // element k of this mode: col[k * TRI_TM * TRI_TL]
  constexpr int LS = TRI_TM * TRI_TL;
  if (act && !(l < 2 && m < 2)) {
    float cp[NZ];
    float cprev = 0.f, dprev = 0.f;
#pragma unroll
    for (int k = 0; k < NZ; k++) {
      const float4 o = zop(k);
      const float rd = tri_pivot_rcp(o, shift, cprev);
      cprev = o.y * rd;
      dprev = fmaf(-o.x, dprev, col[k * LS]) * rd;
      cp[k] = cprev;
      col[k * LS] = dprev;
      // a compiler fence every 8 levels: the tile reads of later levels (which do not depend on the recurrence) are
      // not all hoisted ahead of it, which would hold NZ more values in registers next to c'
      if ((k & 7) == 7) asm volatile("" ::: "memory");
    }
    float x = dprev;
#pragma unroll
    for (int k = NZ - 2; k >= 0; k--) {
      x = fmaf(-cp[k], x, col[k * LS]);
      col[k * LS] = x;
      if ((k & 7) == 0) asm volatile("" ::: "memory");
    }
  } else if (act) {
    // lowest modes: low[(mode*2 + 0)*NZ + k] = 1/den_k, low[(mode*2 + 1)*NZ + k] = c'_k (FP64, host-factored)
    const int mode = m * 2 + l;
    const double* rd = low + (mode * 2) * NZ;
    const double* cpd = rd + NZ;
    double* d = dlow + mode * NZ;
    double dprev = 0.0;
#pragma unroll 8
    for (int k = 0; k < NZ; k++) {   // the coefficient loads do not depend on the recurrence: unrolled, they overlap
      dprev = (double(col[k * LS]) - double(zop(k).x) * dprev) * __ldg(rd + k);
      d[k] = dprev;
    }
    double x = dprev;
    col[(NZ - 1) * LS] = float(x);
#pragma unroll 8
    for (int k = NZ - 2; k >= 0; k--) {
      x = d[k] - __ldg(cpd + k) * x;
      col[k * LS] = float(x);
    }
  } else {
#pragma unroll
    for (int k = 0; k < NZ; k++) col[k * LS] = 0.f;   // modes past the grid: zeros (the padding of the output rows)
  }
  __syncthreads();
  // transposed output: in group g, warp kk writes level 8 g + kk; lane -> (l = lx, half of the 16 m); a lane reads
  // its 8 m with the pairs of the second half-warp swapped (m ^ 1), so that the two halves hit different banks, and
  // packs them back in order; the split rows are held as packed bf16 pairs until every thread has read the tile
  const int kk = tid >> 5, lx = tid & 15, half = (tid >> 4) & 1;
  constexpr int NG = NZ / 8;
  uint4 ph[NG], pl[HI_ONLY ? 1 : NG];
#pragma unroll
  for (int g = 0; g < NG; g++) {
    const float* src = tile + (g * 8 + kk) * LS + half * 8 * TRI_TL + lx;
    const float* se = src + half * TRI_TL;   // even u reads m = u + half
    const float* so = src - half * TRI_TL;   // odd u reads m = u - half
    float v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) v[u] = (u & 1) ? so[u * TRI_TL] : se[u * TRI_TL];
    uint32_t h[4], lo[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const float a = half ? v[2 * u + 1] : v[2 * u], b = half ? v[2 * u] : v[2 * u + 1];
      const __nv_bfloat162 hh = __floats2bfloat162_rn(a, b);
      h[u] = *reinterpret_cast<const uint32_t*>(&hh);
      if (!HI_ONLY) {
        const float2 hf = __bfloat1622float2(hh);
        const __nv_bfloat162 ll = __floats2bfloat162_rn(a - hf.x, b - hf.y);
        lo[u] = *reinterpret_cast<const uint32_t*>(&ll);
      }
    }
    ph[g] = make_uint4(h[0], h[1], h[2], h[3]);
    if (!HI_ONLY) pl[g] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
  }
  __syncthreads();   // every read of the tile is done before it is overwritten
  uint4* hi = reinterpret_cast<uint4*>(tile);            // [NZ][16 l][16 m] bf16: two uint4 per (level, l)
  uint4* lo = hi + NZ * TRI_TL * 2;
#pragma unroll
  for (int g = 0; g < NG; g++) {
    const int o = ((g * 8 + kk) * TRI_TL + lx) * 2 + half;
    hi[o] = ph[g];
    if (!HI_ONLY) lo[o] = pl[g];
  }
  tc::fence_proxy_async_smem();
  __syncthreads();
  if (tid == 0) {
    tc::tma_store_3d(tHi, hi, m0, l0, 0);
    if (!HI_ONLY) tc::tma_store_3d(tLo, lo, m0, l0, 0);
    tc::bulk_commit();
    tc::bulk_wait_read_all();   // the shared memory stays until the stores have read it
  }
}

template <int NZ, bool HI_ONLY>
__global__ void __launch_bounds__(TRI_TL * TRI_TM, NZ > 40 ? 2 : 4) k_tri_tma(const __grid_constant__ CUtensorMap tIn, const __grid_constant__ CUtensorMap tHi,
                                                          const __grid_constant__ CUtensorMap tLo, int nxp, int nyp,
                                                          const float* __restrict__ lam, const __grid_constant__ TriZ<NZ> Z,
                                                          const double* __restrict__ low, unsigned int* err) {
  extern __shared__ uint8_t smraw[];
  tri_tma_tile<NZ, HI_ONLY>(&tIn, &tHi, &tLo, nxp, nyp, lam, [&](int k) { return Z.z[k]; }, low, err, blockIdx.x * TRI_TL,
                            blockIdx.y * TRI_TM, smraw);
}

// The same tiles for every member of an ensemble: member p owns the blocks [start[p], start[p+1]) of its gx x gy
// tiles; its tensor maps live in global memory (written by the host before any launch that reads them), and its
// z-operator is copied into shared memory for the sweeps (the members' densities differ, so it cannot be a parameter)
struct alignas(64) TriTmaProb {
  CUtensorMap in, hi, lo;
  const float* lam;
  const float4* zop;
  const double* low;
  int nxp, nyp, gx, pad;
};
template <int NZ, bool HI_ONLY>
__global__ void __launch_bounds__(TRI_TL * TRI_TM, NZ > 40 ? 2 : 4) k_tri_tma_grp(const TriTmaProb* __restrict__ probs, const int* __restrict__ start,
                                                                              int n, unsigned int* err) {
  extern __shared__ uint8_t smraw[];
  __shared__ float4 zs[NZ];
  __shared__ int s_mem, s_r;
  if (threadIdx.x == 0) {
    const int b = blockIdx.x;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(start + mid) <= b) lo = mid;
      else hi = mid - 1;
    }
    s_mem = lo;
    s_r = b - __ldg(start + lo);
  }
  __syncthreads();
  const TriTmaProb* P = probs + s_mem;
  for (int k = threadIdx.x; k < NZ; k += blockDim.x) zs[k] = __ldg(P->zop + k);   // read after the tile's first barrier
  const int r = s_r, gx = P->gx;
  tri_tma_tile<NZ, HI_ONLY>(&P->in, &P->hi, &P->lo, P->nxp, P->nyp, P->lam, [&](int k) { return zs[k]; }, P->low, err,
                            (r % gx) * TRI_TL, (r / gx) * TRI_TM, smraw);
}
// the same solve with plain loads and stores (tri_body), for planes whose pitch a tensor map cannot describe (T2's
// row pitch nxp * 4 bytes not a multiple of 16)
template <int NZ>
__global__ void __launch_bounds__(32 * tri_tm<NZ>()) k_tri_tc(int nxp, int nyp, int ldy, const float* __restrict__ lam, const float4* __restrict__ zop,
                                                const double* __restrict__ low, const float* __restrict__ T2,
                                                __nv_bfloat16* __restrict__ ohi, __nv_bfloat16* __restrict__ olo) {
  tri_body<NZ>(nxp, nyp, ldy, lam, zop, low, T2, ohi, olo, blockIdx.x, blockIdx.y);
}
// the tridiagonals of every member of an ensemble: member p owns the linear blocks [start[p], start[p+1])
struct TriProb {
  int nxp, nyp, ldy, gx;
  const float* lam;
  const float4* zop;
  const double* low;
  const float* T2;
  __nv_bfloat16* ohi;
  __nv_bfloat16* olo;
};
template <int NZ>
__global__ void __launch_bounds__(32 * tri_tm<NZ>()) k_tri_tc_grp(const TriProb* __restrict__ probs, const int* __restrict__ start, int n) {
  // one thread finds the block's member; the problem is read from shared memory, so that no register holds it
  // through the sweeps
  __shared__ TriProb P;
  __shared__ int r;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    const int b = blockIdx.x;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(start + mid) <= b) lo = mid;
      else hi = mid - 1;
    }
    P = probs[lo];
    r = b - __ldg(start + lo);
  }
  __syncthreads();
  tri_body<NZ>(P.nxp, P.nyp, P.ldy, P.lam, P.zop, P.low, P.T2, P.ohi, P.olo, r % P.gx, r / P.gx);
}

// ---------------------------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------------------------
typedef CUresult (*PFN_encodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                    const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled get_encode() {
  static PFN_encodeTiled fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_encodeTiled>(p);
  }
  return fn;
}

// 2-D [rows][cols] bf16 with pitch ld (elements), box 64 x box_rows, 128-byte swizzle; reads past cols or rows are
// zero-filled
static bool make_map_2d(CUtensorMap* m, void* base, long rows, long cols, long ld, int box_rows) {
  PFN_encodeTiled enc = get_encode();
  if (!enc) return false;
  cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows)};
  cuuint64_t strides[1] = {cuuint64_t(ld * 2)};
  cuuint32_t box[2] = {BK, cuuint32_t(box_rows)};
  cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 3-D tensor, innermost dimension first: dims[3] elements, pitches (bytes) of dimensions 1 and 2, box[3], no swizzle;
// loads past the tensor read zeros, stores past it are dropped
static bool make_map_3d(CUtensorMap* m, CUtensorMapDataType type, void* base, const long* dims, const long* pitch_bytes,
                        const int* box) {
  PFN_encodeTiled enc = get_encode();
  if (!enc) return false;
  cuuint64_t d[3] = {cuuint64_t(dims[0]), cuuint64_t(dims[1]), cuuint64_t(dims[2])};
  cuuint64_t st[2] = {cuuint64_t(pitch_bytes[0]), cuuint64_t(pitch_bytes[1])};
  cuuint32_t b[3] = {cuuint32_t(box[0]), cuuint32_t(box[1]), cuuint32_t(box[2])};
  cuuint32_t es[3] = {1, 1, 1};
  return enc(m, type, 3, base, d, st, b, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// tile width for N transform outputs: the fewest tiles of at most 256, then the smallest multiple of 16 covering N
static int pick_bn(int N, int cap = BNMAX) {
  const int nt = (N + cap - 1) / cap;
  return ((N + nt - 1) / nt + 15) / 16 * 16;
}

static int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  }
  return n;
}

static void set_smem_attrs() {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_dst_tc<OUT_T_BF16X2>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc<OUT_T_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc<OUT_R_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc<OUT_R_F32_ADD>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc_grp<OUT_T_BF16X2>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc_grp<OUT_T_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc_grp<OUT_R_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc_grp<OUT_R_F32_ADD>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc<OUT_T_BF16X2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc<OUT_T_F32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc<OUT_R_F32_ADD, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc<OUT_R_F32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc_grp<OUT_T_BF16X2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc_grp<OUT_T_F32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc_grp<OUT_R_F32_ADD, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc_grp<OUT_R_F32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    cudaFuncSetAttribute(k_dst_tc2<OUT_T_BF16X2>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES);
    cudaFuncSetAttribute(k_dst_tc2<OUT_T_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES);
    cudaFuncSetAttribute(k_dst_tc2<OUT_R_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES);
    cudaFuncSetAttribute(k_dst_tc2<OUT_R_F32_ADD>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES);
    cudaFuncSetAttribute(k_dst_tc2<OUT_T_BF16X2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES);
    cudaFuncSetAttribute(k_dst_tc2<OUT_T_F32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES);
    cudaFuncSetAttribute(k_dst_tc2<OUT_R_F32_ADD, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES);
    cudaFuncSetAttribute(k_dst_tc2<OUT_R_F32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM2_BYTES);
    cudaFuncSetAttribute(k_tri_tma<16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<16>());
    cudaFuncSetAttribute(k_tri_tma<40, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<40>());
    cudaFuncSetAttribute(k_tri_tma<80, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<80>());
    cudaFuncSetAttribute(k_tri_tma<16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<16>());
    cudaFuncSetAttribute(k_tri_tma_grp<16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<16>());
    cudaFuncSetAttribute(k_tri_tma_grp<40, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<40>());
    cudaFuncSetAttribute(k_tri_tma_grp<80, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<80>());
    cudaFuncSetAttribute(k_tri_tma_grp<16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<16>());
    cudaFuncSetAttribute(k_tri_tma_grp<40, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<40>());
    cudaFuncSetAttribute(k_tri_tma_grp<80, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<80>());
    cudaFuncSetAttribute(k_tri_tma<40, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<40>());
    cudaFuncSetAttribute(k_tri_tma<80, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tri_smem_bytes<80>());
    attr = true;
  }
}

static inline long pad8(long n) { return (n + 7) / 8 * 8; }

struct TcPlan {
  int nx, ny, nz;
  long ldx, ldy;
  __nv_bfloat16* mat = nullptr;  // 8 matrices hi/lo: qix, qiy, qy, qx
  __nv_bfloat16 *sx_hi = nullptr, *sx_lo = nullptr, *sy_hi = nullptr, *sy_lo = nullptr;
  __nv_bfloat16 *rx_hi = nullptr, *rx_lo = nullptr;  // the right-hand side, split (zero outside what is written)
  // the residual of the refined solve, split: a buffer of its own, because the residual fills the padding that the
  // right-hand side leaves zero (the next step's first pass must see zeros there)
  __nv_bfloat16 *rr_hi = nullptr, *rr_lo = nullptr;
  float* t2 = nullptr;
  double* low = nullptr;  // FP64 factors of the 4 lowest modes
  unsigned int* err = nullptr;
  int bnx = 0, bny = 0;   // tile widths of the x and y transforms
  CUtensorMap Q[4][2];    // DST matrices, the B operand: [transform][hi/lo]
  __nv_bfloat16* qmat[4][2] = {};  // their bf16 planes: x-fwd, y-fwd, y-inv, x-inv
  long qld[4] = {};
  int qdim[4] = {};
  CUtensorMap Fx[2], Fy[2], Fr[2], Frr[2];  // fields, the A operand: S_x, S_y, the split right-hand side and residual
  CUtensorMap tri_in, tri_out[2];  // the tridiagonals' tiles: T2[k][m][l] fp32 in, S_y[k][l][m] bf16 hi / lo out
  bool tri_tma = false;
  float4 zh[80] = {};    // the z-operator on the host: the by-value coefficients of k_tri_tma (nz <= 80)
  CUtensorMap Qh[4][2];  // the DST matrices with boxes of half a tile's width: each CTA of a pair loads one half
  bool pairs = true;     // transforms on SM pairs (k_dst_tc2); single-SM tiles (k_dst_tc) when false
};

static void split_host(const float* src, int N, long ld, std::vector<__nv_bfloat16>& hi, std::vector<__nv_bfloat16>& lo) {
  hi.assign(size_t(N) * ld, __float2bfloat16_rn(0.f));
  lo.assign(size_t(N) * ld, __float2bfloat16_rn(0.f));
  for (int r = 0; r < N; r++)
    for (int c = 0; c < N; c++) {
      const float x = src[size_t(r) * N + c];
      const __nv_bfloat16 h = __float2bfloat16_rn(x);
      hi[size_t(r) * ld + c] = h;
      lo[size_t(r) * ld + c] = __float2bfloat16_rn(x - __bfloat162float(h));
    }
}

// the DST matrices' tensor maps for tiles of bnx / bny outputs: full-width boxes for single-SM tiles, half-width boxes
// for SM pairs
static bool matrix_maps(TcPlan* T, int bnx, int bny) {
  T->bnx = bnx;
  T->bny = bny;
  const int bn[4] = {bnx, bny, bny, bnx};
  bool ok = true;
  for (int t = 0; t < 4; t++)
    for (int h = 0; h < 2; h++)
      ok = ok && make_map_2d(&T->Q[t][h], T->qmat[t][h], T->qdim[t], T->qdim[t], T->qld[t], bn[t]) &&
           make_map_2d(&T->Qh[t][h], T->qmat[t][h], T->qdim[t], T->qdim[t], T->qld[t], bn[t] / 2);
  return ok;
}

static int pair_slots();

int PoissonPlan::tc_create() {
  if (!get_encode()) {
    set_error("poisson: cuTensorMapEncodeTiled is unavailable");
    return OB_ERR_DEVICE;
  }
  TcPlan* T = new TcPlan();
  tc = T;
  T->nx = nx; T->ny = ny; T->nz = nz;
  T->ldx = pad8(nx);
  T->ldy = pad8(ny);
  const size_t mx = size_t(nx) * T->ldx, my = size_t(ny) * T->ldy;
  const size_t nsx = size_t(nz) * ny * T->ldx, nsy = size_t(nz) * nx * T->ldy;
  auto al = [&](void** p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess && cudaMemset(*p, 0, bytes) == cudaSuccess; };
  bool ok = al((void**)&T->mat, (4 * mx + 4 * my) * 2) && al((void**)&T->sx_hi, nsx * 2) && al((void**)&T->sx_lo, nsx * 2) &&
            al((void**)&T->rx_hi, nsx * 2) && al((void**)&T->rx_lo, nsx * 2) &&
            al((void**)&T->sy_hi, nsy * 2) && al((void**)&T->sy_lo, nsy * 2) && al((void**)&T->t2, size_t(nz) * nx * ny * 4) &&
            al((void**)&T->low, size_t(8) * nz * 8) && al((void**)&T->err, 16);
  if (ok && precision >= 2) ok = al((void**)&T->rr_hi, nsx * 2) && al((void**)&T->rr_lo, nsx * 2);
  if (!ok) {
    set_error("poisson: out of device memory for the tensor-core path");
    return OB_ERR_OOM;
  }
  // DST matrices in hi/lo bf16 (the fp32 matrices of PoissonPlan::create, split)
  std::vector<float> M(2 * size_t(nx) * nx + 2 * size_t(ny) * ny);
  cudaMemcpy(M.data(), mats, M.size() * 4, cudaMemcpyDeviceToHost);
  // order: qix (x fwd), qiy (y fwd), qy (y inv), qx (x inv)
  const float* src[4] = {M.data() + ofs_qix, M.data() + ofs_qiy, M.data() + ofs_qy, M.data() + ofs_qx};
  const int dim[4] = {nx, ny, ny, nx};
  const long ld[4] = {T->ldx, T->ldy, T->ldy, T->ldx};
  size_t off = 0;
  __nv_bfloat16* mp[4][2];
  for (int t = 0; t < 4; t++) {
    std::vector<__nv_bfloat16> hi, lo;
    split_host(src[t], dim[t], ld[t], hi, lo);
    const size_t n = size_t(dim[t]) * ld[t];
    mp[t][0] = T->mat + off;
    mp[t][1] = T->mat + off + n;
    cudaMemcpy(mp[t][0], hi.data(), n * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(mp[t][1], lo.data(), n * 2, cudaMemcpyHostToDevice);
    off += 2 * n;
    T->qmat[t][0] = mp[t][0];
    T->qmat[t][1] = mp[t][1];
    T->qld[t] = ld[t];
    T->qdim[t] = dim[t];
  }
  ok = matrix_maps(T, pick_bn(nx), pick_bn(ny));
  // A operands, planes stacked: S_x and the split rhs [nz * ny][nx] pitch ldx; S_y [nz * nx][ny] pitch ldy
  ok = ok && make_map_2d(&T->Fx[0], T->sx_hi, long(nz) * ny, nx, T->ldx, BM) && make_map_2d(&T->Fx[1], T->sx_lo, long(nz) * ny, nx, T->ldx, BM);
  ok = ok && make_map_2d(&T->Fr[0], T->rx_hi, long(nz) * ny, nx, T->ldx, BM) && make_map_2d(&T->Fr[1], T->rx_lo, long(nz) * ny, nx, T->ldx, BM);
  if (precision >= 2)
    ok = ok && make_map_2d(&T->Frr[0], T->rr_hi, long(nz) * ny, nx, T->ldx, BM) && make_map_2d(&T->Frr[1], T->rr_lo, long(nz) * ny, nx, T->ldx, BM);
  ok = ok && make_map_2d(&T->Fy[0], T->sy_hi, long(nz) * nx, ny, T->ldy, BM) && make_map_2d(&T->Fy[1], T->sy_lo, long(nz) * nx, ny, T->ldy, BM);
  if (!ok) {
    set_error("poisson: tensor map encoding failed");
    return OB_ERR_DEVICE;
  }
  // the tridiagonals' tiles (k_tri_tma); when T2's row pitch is not a multiple of 16 bytes the plain-load kernel runs
  if ((nz == 16 || nz == 40 || nz == 80) && (long(nx) * 4) % 16 == 0) {
    const long din[3] = {nx, ny, nz}, pin[2] = {long(nx) * 4, long(nx) * ny * 4};
    const int bin[3] = {TRI_TL, TRI_TM, nz};
    const long dout[3] = {T->ldy, nx, nz}, pout[2] = {T->ldy * 2, T->ldy * nx * 2};
    const int bout[3] = {TRI_TM, TRI_TL, nz};
    T->tri_tma = make_map_3d(&T->tri_in, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, T->t2, din, pin, bin) &&
                 make_map_3d(&T->tri_out[0], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, T->sy_hi, dout, pout, bout) &&
                 make_map_3d(&T->tri_out[1], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, T->sy_lo, dout, pout, bout);
  }
  set_smem_attrs();
  pair_slots();   // the occupancy query of the paired transform runs here, outside any stream capture
  return tc_factor_low();
}

// FP64 LU factors of the lowest 2 x 2 modes (rhs independent), from the fp32 eigenvalues and z-operator
int PoissonPlan::tc_factor_low() {
  TcPlan* T = static_cast<TcPlan*>(tc);
  if (!T) return OB_OK;
  std::vector<float> lamh(nx + ny);
  std::vector<float4> zo(nz);
  cudaMemcpy(lamh.data(), lam, lamh.size() * 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(zo.data(), zop, zo.size() * sizeof(float4), cudaMemcpyDeviceToHost);
  for (int k = 0; k < nz && k < 80; k++) T->zh[k] = zo[k];
  std::vector<double> f(size_t(8) * nz);
  for (int mode = 0; mode < 4; mode++) {
    const int l = mode & 1, m = mode >> 1;
    const double shift = double(lamh[l]) + double(lamh[nx + m]);
    double* rd = f.data() + size_t(mode * 2) * nz;
    double* cp = rd + nz;
    double cprev = 0.0;
    for (int k = 0; k < nz; k++) {
      const double den = double(zo[k].z) + shift * double(zo[k].w) - double(zo[k].x) * cprev;
      rd[k] = 1.0 / den;
      cprev = double(zo[k].y) / den;
      cp[k] = cprev;
    }
  }
  if (cudaMemcpy(T->low, f.data(), f.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
    set_error("poisson: low-mode factor upload failed");
    return OB_ERR_DEVICE;
  }
  return OB_OK;
}

void PoissonPlan::tc_destroy() {
  TcPlan* T = static_cast<TcPlan*>(tc);
  if (!T) return;
  for (void* p : {(void*)T->mat, (void*)T->sx_hi, (void*)T->sx_lo, (void*)T->rx_hi, (void*)T->rx_lo, (void*)T->rr_hi, (void*)T->rr_lo,
                  (void*)T->sy_hi, (void*)T->sy_lo, (void*)T->t2, (void*)T->low, (void*)T->err})
    if (p) cudaFree(p);
  delete T;
  tc = nullptr;
}

static cudaLaunchConfig_t pair_config(int pairs, cudaStream_t s, cudaLaunchAttribute* at) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(2 * pairs);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = SMEM2_BYTES;
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 2;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}

// pairs of SMs that can hold a k_dst_tc2 cluster at once (the GPCs' SM counts need not be even); the persistent grid
// is no larger, so that no cluster waits for a second wave
static int pair_slots() {
  static int n = 0;
  if (!n) {
    cudaLaunchAttribute at[1];
    const cudaLaunchConfig_t cfg = pair_config(num_sms() / 2, nullptr, at);
    if (cudaOccupancyMaxActiveClusters(&n, k_dst_tc2<OUT_T_F32>, &cfg) != cudaSuccess || n <= 0) {
      cudaGetLastError();
      n = num_sms() / 2;
    }
    n = std::min(n, num_sms() / 2);
  }
  return n;
}

// the pair kernel's tiles for M field rows and N outputs at width BN over at most max_pairs pairs (the grid, in
// pairs): whole tiles, except that a last round at most half full is split into sub-tiles (2 to 4 per tile, each at
// least 32 outputs wide, none empty)
static PairSched pair_sched(int M, int N, int BN, int max_pairs, int& pairs) {
  PairSched sc{};
  sc.ntn = (N + BN - 1) / BN;
  sc.BN = BN;
  sc.N = N;
  const int T = ((M + 2 * BM - 1) / (2 * BM)) * sc.ntn;
  pairs = std::max(1, std::min(T, max_pairs));
  sc.base = sc.total = T;
  sc.S = 1;
  sc.w = BN;
  const int R = T % pairs, wlast = N - (sc.ntn - 1) * BN;   // tiles of the last round; the narrowest tile's width
  if (R > 0 && 2 * R <= pairs) {
    for (int S = std::min(4, pairs / R); S >= 2; S--) {
      const int w = std::max(32, ((BN + S - 1) / S + 15) / 16 * 16);
      if ((S - 1) * w < wlast) {
        sc.base = T - R;
        sc.S = S;
        sc.w = w;
        sc.total = T - R + R * S;
        break;
      }
    }
  }
  return sc;
}

template <int MODE, bool ONE = false>
static void launch_tc(const CUtensorMap* f, const CUtensorMap* q, int K, int bn, const TcOut& o, unsigned int* err, cudaStream_t s,
                      const CUtensorMap* qh = nullptr) {
  if (qh) {  // SM pairs: tiles of 256 field rows, qh the DST matrix maps with half-width boxes
    int pairs = 0;
    const PairSched sc = pair_sched(o.M, o.N, bn, pair_slots(), pairs);
    cudaLaunchAttribute at[1];
    const cudaLaunchConfig_t cfg = pair_config(pairs, s, at);
    cudaLaunchKernelEx(&cfg, k_dst_tc2<MODE, ONE>, f[0], f[1], qh[0], qh[1], K, sc, o, err);
    return;
  }
  const int tiles = ((o.M + BM - 1) / BM) * ((o.N + bn - 1) / bn);
  k_dst_tc<MODE, ONE><<<std::min(tiles, num_sms()), kThreads, SMEM_BYTES, s>>>(f[0], f[1], q[0], q[1], K, bn, o, err);
}

// the TMA tridiagonals of one pass: the z-operator goes by value (the host copy of set_density's coefficients)
template <int NZ>
static void launch_tri_tma(const TcPlan* T, const float* lam, bool hi_only, cudaStream_t s) {
  TriZ<NZ> Z;
  for (int k = 0; k < NZ; k++) Z.z[k] = T->zh[k];
  const dim3 grid((T->nx + TRI_TL - 1) / TRI_TL, (T->ny + TRI_TM - 1) / TRI_TM);
  if (hi_only) k_tri_tma<NZ, true><<<grid, TRI_TL * TRI_TM, tri_smem_bytes<NZ>(), s>>>(T->tri_in, T->tri_out[0], T->tri_out[1], T->nx, T->ny, lam, Z, T->low, T->err);
  else k_tri_tma<NZ, false><<<grid, TRI_TL * TRI_TM, tri_smem_bytes<NZ>(), s>>>(T->tri_in, T->tri_out[0], T->tri_out[1], T->nx, T->ny, lam, Z, T->low, T->err);
}

// the four transforms and the tridiagonals from a split right-hand side (rx, or the residual rr when add) to phi
// (stored, or added when add)
static void tc_pass(const PoissonPlan& P, TcPlan* T, const float* lam, const float4* zop, float* phi, bool add, cudaStream_t s,
                    bool one = false) {
#define QH(t) (T->pairs ? T->Qh[t] : nullptr)
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const TcOut sy{T->sy_hi, T->sy_lo, nullptr, T->ldy, ny, nz * ny, nx}, t2{nullptr, nullptr, T->t2, nx, nx, nz * nx, ny};
  // X-fwd: field rows (k, j), K = i, outputs l  -> S_y[k][l][j]
  if (one) launch_tc<OUT_T_BF16X2, true>(add ? T->Frr : T->Fr, T->Q[0], nx, T->bnx, sy, T->err, s, QH(0));
  else launch_tc<OUT_T_BF16X2>(add ? T->Frr : T->Fr, T->Q[0], nx, T->bnx, sy, T->err, s, QH(0));
  // Y-fwd: field rows (k, l), K = j, outputs m  -> T2[k][m][l] fp32
  if (one) launch_tc<OUT_T_F32, true>(T->Fy, T->Q[1], ny, T->bny, t2, T->err, s, QH(1));
  else launch_tc<OUT_T_F32>(T->Fy, T->Q[1], ny, T->bny, t2, T->err, s, QH(1));
  // tridiagonals -> S_y[k][l][m]
  // (a plain-bf16 pass writes the hi plane alone: its y-inverse transform reads nothing else)
  if (T->tri_tma) {
    switch (nz) {
      case 16: launch_tri_tma<16>(T, lam, one, s); break;
      case 40: launch_tri_tma<40>(T, lam, one, s); break;
      default: launch_tri_tma<80>(T, lam, one, s); break;
    }
  } else {
    __nv_bfloat16* lo = one ? nullptr : T->sy_lo;
    switch (nz) {
      case 16: k_tri_tc<16><<<dim3((nx + 31) / 32, (ny + tri_tm<16>() - 1) / tri_tm<16>()), dim3(32, tri_tm<16>()), 0, s>>>(nx, ny, int(T->ldy), lam, zop, T->low, T->t2, T->sy_hi, lo); break;
      case 40: k_tri_tc<40><<<dim3((nx + 31) / 32, (ny + tri_tm<40>() - 1) / tri_tm<40>()), dim3(32, tri_tm<40>()), 0, s>>>(nx, ny, int(T->ldy), lam, zop, T->low, T->t2, T->sy_hi, lo); break;
      default: k_tri_tc<80><<<dim3((nx + 31) / 32, (ny + tri_tm<80>() - 1) / tri_tm<80>()), dim3(32, tri_tm<80>()), 0, s>>>(nx, ny, int(T->ldy), lam, zop, T->low, T->t2, T->sy_hi, lo); break;
    }
  }
  // Y-inv: field rows (k, l), K = m, outputs j  -> S_x[k][j][l]
  const TcOut sx{T->sx_hi, T->sx_lo, nullptr, T->ldx, nx, nz * nx, ny};
  if (one) launch_tc<OUT_T_BF16X2, true>(T->Fy, T->Q[2], ny, T->bny, sx, T->err, s, QH(2));
  else launch_tc<OUT_T_BF16X2>(T->Fy, T->Q[2], ny, T->bny, sx, T->err, s, QH(2));
  // X-inv: field rows (k, j), K = l, outputs i  -> phi[k][j][i]
  const TcOut o{nullptr, nullptr, phi, nx, ny, nz * ny, nx};
  if (one && add) launch_tc<OUT_R_F32_ADD, true>(T->Fx, T->Q[3], nx, T->bnx, o, T->err, s, QH(3));
  else if (one) launch_tc<OUT_R_F32, true>(T->Fx, T->Q[3], nx, T->bnx, o, T->err, s, QH(3));
  else if (add) launch_tc<OUT_R_F32_ADD>(T->Fx, T->Q[3], nx, T->bnx, o, T->err, s, QH(3));
  else launch_tc<OUT_R_F32>(T->Fx, T->Q[3], nx, T->bnx, o, T->err, s, QH(3));
#undef QH
}

// precision 1: one bf16x3 pass; precision 2: a second bf16x3 pass on the FP64-accumulated residual (iterative
// refinement); precision 3: the second pass in plain bf16 (the correction is ~5e-4 of the solution, so bf16 accuracy
// of it leaves an error near 5e-4 x 4e-3 of the solution); precision 4: two bf16x3 refinement sweeps, which leave the
// solution within about an fp32 rounding of the exact one (the residual at the floor set by storing phi in fp32).
// rhs: the fp32 right-hand side (nx*ny*nz), needed by precision 2 and by either when the split is not pre-made
// (presplit: the model's divergence pass writes the split into rx itself).
int PoissonPlan::tc_solve(const float* rhs, float* phi, cudaStream_t s) {
  TcPlan* T = static_cast<TcPlan*>(tc);
  if (!T) { set_error("poisson: tensor-core plan missing"); return OB_ERR_INVALID; }
  if (nz != 16 && nz != 40 && nz != 80) { set_error("poisson: the tensor-core path supports nz in {16, 40, 80}"); return OB_ERR_INVALID; }
  if (!presplit || precision >= 2) {
    if (!rhs) { set_error("poisson: right-hand side missing"); return OB_ERR_INVALID; }
  }
  if (!presplit) k_split_rows<<<1184, 256, 0, s>>>(rhs, long(nz) * ny, nx, T->rx_hi, T->rx_lo, int(T->ldx));
  tc_pass(*this, T, lam, zop, phi, false, s, precision == 5);
  if (precision >= 2) {
    const int sweeps = precision == 4 ? 2 : 1;
    for (int sw = 0; sw < sweeps; sw++) {
      k_resid<<<dim3((nx + 127) / 128, ny, nz), 128, 0, s>>>(nx, ny, nz, 1.0 / (dx * dx), zop, rhs, phi, T->rr_hi, T->rr_lo, int(T->ldx));
      tc_pass(*this, T, lam, zop, phi, true, s, precision == 3);
    }
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("poisson tensor-core launch: %s", cudaGetErrorString(e));
    return OB_ERR_DEVICE;
  }
  return OB_OK;
}

int PoissonPlan::tc_set_pairs(bool on) {
  TcPlan* T = static_cast<TcPlan*>(tc);
  if (!T) { set_error("poisson: the SM-pair transforms need a tensor-core precision (1 to 5)"); return OB_ERR_INVALID; }
  T->pairs = on;
  if (on) pair_slots();   // the occupancy query runs here, outside any stream capture
  return OB_OK;
}
int PoissonPlan::tc_set_tile_widths(int bnx, int bny) {
  TcPlan* T = static_cast<TcPlan*>(tc);
  if (!T) { set_error("poisson: tile widths apply to the tensor-core precisions (1 to 5)"); return OB_ERR_INVALID; }
  for (int b : {bnx, bny})
    if (b != 0 && (b < 32 || b > BNMAX || b % 16)) {
      set_error("poisson: tile width %d not 0 (automatic) or a multiple of 16 in 32..%d", b, BNMAX);
      return OB_ERR_INVALID;
    }
  if (!matrix_maps(T, bnx ? bnx : pick_bn(nx), bny ? bny : pick_bn(ny))) {
    set_error("poisson: tensor map encoding failed");
    return OB_ERR_DEVICE;
  }
  return OB_OK;
}
bool PoissonPlan::tc_pairs() const {
  const TcPlan* T = static_cast<const TcPlan*>(tc);
  return T && T->pairs;
}

void PoissonPlan::tc_rhs_split(__nv_bfloat16** hi, __nv_bfloat16** lo, int* ld) const {
  const TcPlan* T = static_cast<const TcPlan*>(tc);
  *hi = T ? T->rx_hi : nullptr;
  *lo = T ? T->rx_lo : nullptr;
  *ld = T ? int(T->ldx) : 0;
}

int PoissonPlan::tc_check() {
  TcPlan* T = static_cast<TcPlan*>(tc);
  if (!T) return OB_OK;
  unsigned int h = 0;
  cudaMemcpy(&h, T->err, sizeof(h), cudaMemcpyDeviceToHost);
  if (h) {
    cudaMemset(T->err, 0, sizeof(unsigned int));
    set_error("poisson: a tensor-core pipeline wait timed out (code %u)", h);
    return OB_ERR_TIMEOUT;
  }
  return OB_OK;
}

// ---------------------------------------------------------------------------------------------------------------
// grouped solve: the same pass of every member of an ensemble in one launch (persistent transforms over the members'
// concatenated tile lists, the tridiagonals and residuals over their concatenated blocks)
// ---------------------------------------------------------------------------------------------------------------
struct TcGroup {
  int n = 0, nz = 0, precision = 1, bn_cap = BNMAX;
  std::vector<PoissonPlan*> plans;
  std::vector<float*> phi;
  std::vector<const float*> rhs;
  GemmProb* d_probs = nullptr;  // [5][n]: x-fwd, y-fwd, y-inv, x-inv, x-fwd of the residual
  int* d_start = nullptr;       // [5][n + 1] tile starts, [n + 1] tridiagonal block starts, [n + 1] residual block starts
  TriProb* d_tri = nullptr;
  TriTmaProb* d_tri_tma = nullptr;  // the TMA tridiagonals' per-member maps, when every member has them
  bool tri_tma = false;
  int tri_tma_blocks = 0;
  ResidProb* d_res = nullptr;
  uint2* d_res_map = nullptr;  // block map of the residual launch
  unsigned int* err = nullptr;
  int tiles[5] = {}, tri_blocks = 0, res_blocks = 0;
  int ctas = 0;  // CTAs of a transform launch (0: one per SM)
};

// problem tables for the tile-width cap (the B operand's box height is the tile width, so its maps are re-encoded)
static int tc_group_build(TcGroup* G) {
  const int n = G->n;
  constexpr int NT = 5;  // transform lists
  std::vector<GemmProb> probs(size_t(NT) * n);
  std::vector<int> start(size_t(NT + 3) * (n + 1), 0);
  std::vector<TriTmaProb> trit(n);
  bool all_tma = true;
  std::vector<TriProb> tri(n);
  std::vector<ResidProb> res(n);
  std::vector<uint2> res_map;
  const int tm = G->nz == 16 ? tri_tm<16>() : G->nz == 40 ? tri_tm<40>() : tri_tm<80>();
  for (int i = 0; i < n; i++) {
    const PoissonPlan* P = G->plans[i];
    TcPlan* T = static_cast<TcPlan*>(P->tc);
    const int nx = P->nx, ny = P->ny, nz = P->nz;
    const int bnx = pick_bn(nx, G->bn_cap), bny = pick_bn(ny, G->bn_cap);
    // the fifth list is the x-fwd transform again, reading the residual (refined solve only)
    const int bn[NT] = {bnx, bny, bny, bnx, bnx}, K[NT] = {nx, ny, ny, nx, nx}, qi[NT] = {0, 1, 2, 3, 0};
    const CUtensorMap* F[NT] = {T->Fr, T->Fy, T->Fy, T->Fx, G->precision >= 2 ? T->Frr : T->Fr};
    const TcOut xfwd{T->sy_hi, T->sy_lo, nullptr, T->ldy, ny, nz * ny, nx};
    const TcOut out[NT] = {xfwd, TcOut{nullptr, nullptr, T->t2, nx, nx, nz * nx, ny}, TcOut{T->sx_hi, T->sx_lo, nullptr, T->ldx, nx, nz * nx, ny},
                           TcOut{nullptr, nullptr, G->phi[i], nx, ny, nz * ny, nx}, xfwd};
    for (int t = 0; t < NT; t++) {
      GemmProb& g = probs[size_t(t) * n + i];
      std::memset(&g, 0, sizeof(g));
      g.f[0] = F[t][0];
      g.f[1] = F[t][1];
      for (int h = 0; h < 2; h++)
        if (!make_map_2d(&g.q[h], T->qmat[qi[t]][h], T->qdim[qi[t]], T->qdim[qi[t]], T->qld[qi[t]], bn[t])) {
          set_error("ensemble solve: tensor map encoding failed");
          return OB_ERR_DEVICE;
        }
      g.out = out[t];
      g.K = K[t];
      g.BN = bn[t];
      g.ntn = (out[t].N + bn[t] - 1) / bn[t];
      const int nt = ((out[t].M + BM - 1) / BM) * g.ntn;
      start[size_t(t) * (n + 1) + i + 1] = start[size_t(t) * (n + 1) + i] + nt;
    }
    {  // the TMA tiles of 16 x 16 modes (k_tri_tma_grp), when this member's plan has their maps
      const int tx16 = (nx + TRI_TL - 1) / TRI_TL, ty16 = (ny + TRI_TM - 1) / TRI_TM;
      all_tma = all_tma && T->tri_tma;
      TriTmaProb& q = trit[i];
      std::memset(&q, 0, sizeof(q));
      if (T->tri_tma) {
        q.in = T->tri_in;
        q.hi = T->tri_out[0];
        q.lo = T->tri_out[1];
      }
      q.lam = P->lam;
      q.zop = P->zop;
      q.low = T->low;
      q.nxp = nx;
      q.nyp = ny;
      q.gx = tx16;
      start[size_t(NT + 2) * (n + 1) + i + 1] = start[size_t(NT + 2) * (n + 1) + i] + tx16 * ty16;
    }
    const int gx = (nx + 31) / 32, gy = (ny + tm - 1) / tm;
    tri[i] = TriProb{nx, ny, int(T->ldy), gx, P->lam, P->zop, T->low, T->t2, T->sy_hi, T->sy_lo};
    start[size_t(NT) * (n + 1) + i + 1] = start[size_t(NT) * (n + 1) + i] + gx * gy;
    const int rgx = (nx + 127) / 128;
    res[i] = ResidProb{nx, ny, nz, int(T->ldx), 1.0 / (P->dx * P->dx), P->zop, G->rhs[i], G->phi[i], T->rr_hi, T->rr_lo};
    for (int by = 0; by < ny; by++)
      for (int bx = 0; bx < rgx; bx++) res_map.push_back(make_uint2(unsigned(i), unsigned(bx) | (unsigned(by) << 16)));
    start[size_t(NT + 1) * (n + 1) + i + 1] = start[size_t(NT + 1) * (n + 1) + i] + rgx * ny;
  }
  for (int t = 0; t < NT; t++) G->tiles[t] = start[size_t(t) * (n + 1) + n];
  G->tri_blocks = start[size_t(NT) * (n + 1) + n];
  G->res_blocks = start[size_t(NT + 1) * (n + 1) + n];
  G->tri_tma = all_tma;
  G->tri_tma_blocks = start[size_t(NT + 2) * (n + 1) + n];
  const bool ok = cudaMemcpy(G->d_probs, probs.data(), probs.size() * sizeof(GemmProb), cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(G->d_start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(G->d_tri, tri.data(), tri.size() * sizeof(TriProb), cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(G->d_tri_tma, trit.data(), trit.size() * sizeof(TriTmaProb), cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(G->d_res, res.data(), res.size() * sizeof(ResidProb), cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(G->d_res_map, res_map.data(), res_map.size() * sizeof(uint2), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    set_error("ensemble solve: problem table upload failed");
    return OB_ERR_DEVICE;
  }
  return OB_OK;
}

void tc_group_destroy(TcGroup* G) {
  if (!G) return;
  for (void* p : {(void*)G->d_probs, (void*)G->d_start, (void*)G->d_tri, (void*)G->d_tri_tma, (void*)G->d_res, (void*)G->d_res_map, (void*)G->err})
    if (p) cudaFree(p);
  delete G;
}

static size_t res_map_blocks(PoissonPlan* const* plans, int n) {
  size_t b = 0;
  for (int i = 0; i < n; i++) b += size_t((plans[i]->nx + 127) / 128) * plans[i]->ny;
  return b;
}

int tc_group_create(PoissonPlan* const* plans, float* const* phi, const float* const* rhs, int n, TcGroup** out) {
  *out = nullptr;
  if (n < 1) { set_error("ensemble solve: no members"); return OB_ERR_INVALID; }
  TcGroup* G = new TcGroup();
  G->n = n;
  G->nz = plans[0]->nz;
  G->precision = plans[0]->precision;
  for (int i = 0; i < n; i++) {
    const PoissonPlan* P = plans[i];
    if (!P->tc || P->precision < 1 || !P->presplit) {
      set_error("ensemble solve: member %d does not use the tensor-core solve with the split right-hand side", i);
      tc_group_destroy(G);
      return OB_ERR_INVALID;
    }
    if (P->nz != G->nz || P->precision != G->precision) {
      set_error("ensemble solve: members must share nz and the solver precision (member %d)", i);
      tc_group_destroy(G);
      return OB_ERR_INVALID;
    }
    if (G->precision >= 2 && !rhs[i]) {
      set_error("ensemble solve: member %d has no fp32 right-hand side for the refinement", i);
      tc_group_destroy(G);
      return OB_ERR_INVALID;
    }
    G->plans.push_back(plans[i]);
    G->phi.push_back(phi[i]);
    G->rhs.push_back(rhs[i]);
  }
  if (G->nz != 16 && G->nz != 40 && G->nz != 80) {
    set_error("ensemble solve: the tensor-core path supports nz in {16, 40, 80}");
    tc_group_destroy(G);
    return OB_ERR_INVALID;
  }
  const bool ok = cudaMalloc(&G->d_probs, size_t(5) * n * sizeof(GemmProb)) == cudaSuccess &&
                  cudaMalloc(&G->d_start, size_t(8) * (n + 1) * sizeof(int)) == cudaSuccess &&
                  cudaMalloc(&G->d_tri, size_t(n) * sizeof(TriProb)) == cudaSuccess &&
                  cudaMalloc(&G->d_tri_tma, size_t(n) * sizeof(TriTmaProb)) == cudaSuccess &&
                  cudaMalloc(&G->d_res, size_t(n) * sizeof(ResidProb)) == cudaSuccess && cudaMalloc(&G->err, 16) == cudaSuccess &&
                  cudaMalloc(&G->d_res_map, res_map_blocks(plans, n) * sizeof(uint2)) == cudaSuccess &&
                  cudaMemset(G->err, 0, 16) == cudaSuccess;
  if (!ok) {
    set_error("ensemble solve: out of device memory");
    tc_group_destroy(G);
    return OB_ERR_OOM;
  }
  set_smem_attrs();
  const int rc = tc_group_build(G);
  if (rc != OB_OK) {
    tc_group_destroy(G);
    return rc;
  }
  *out = G;
  return OB_OK;
}

int tc_group_set_cap(TcGroup* G, int bn_cap) {
  if (bn_cap < 16 || bn_cap > BNMAX || bn_cap % 16) { set_error("ensemble solve: tile width cap %d not in 16..256 (multiple of 16)", bn_cap); return OB_ERR_INVALID; }
  if (bn_cap == G->bn_cap) return OB_OK;
  // the tables are read by launches already queued: wait for them before rewriting
  if (cudaDeviceSynchronize() != cudaSuccess) { set_error("ensemble solve: device error before retiling"); return OB_ERR_DEVICE; }
  G->bn_cap = bn_cap;
  return tc_group_build(G);
}
int tc_group_cap(const TcGroup* G) { return G->bn_cap; }
void tc_group_set_ctas(TcGroup* G, int ctas) { G->ctas = ctas > 0 ? ctas : 0; }

template <int MODE, bool ONE = false>
static void launch_tc_grp(const TcGroup* G, int t, cudaStream_t s) {
  if (G->tiles[t] < 1) return;
  k_dst_tc_grp<MODE, ONE><<<std::min(G->tiles[t], G->ctas ? G->ctas : num_sms()), kThreads, SMEM_BYTES, s>>>(G->d_probs + size_t(t) * G->n,
                                                                                     G->d_start + size_t(t) * (G->n + 1), G->n, G->err);
}

static void tc_group_pass(const TcGroup* G, bool add, cudaStream_t s, bool one = false) {
  const int n = G->n;
  if (one) {
    launch_tc_grp<OUT_T_BF16X2, true>(G, add ? 4 : 0, s);
    launch_tc_grp<OUT_T_F32, true>(G, 1, s);
  } else {
    launch_tc_grp<OUT_T_BF16X2>(G, add ? 4 : 0, s);
    launch_tc_grp<OUT_T_F32>(G, 1, s);
  }
  const int* ts = G->d_start + size_t(5) * (n + 1);
  if (G->tri_tma) {   // TMA tiles; a plain-bf16 pass writes the hi plane alone
    const int* tt = G->d_start + size_t(7) * (n + 1);
    const int nb = G->tri_tma_blocks, th = TRI_TL * TRI_TM;
#define OB_TRI_GRP(NZ)                                                                                        \
    if (one) k_tri_tma_grp<NZ, true><<<nb, th, tri_smem_bytes<NZ>(), s>>>(G->d_tri_tma, tt, n, G->err);      \
    else k_tri_tma_grp<NZ, false><<<nb, th, tri_smem_bytes<NZ>(), s>>>(G->d_tri_tma, tt, n, G->err);
    switch (G->nz) {
      case 16: OB_TRI_GRP(16) break;
      case 40: OB_TRI_GRP(40) break;
      default: OB_TRI_GRP(80) break;
    }
#undef OB_TRI_GRP
  } else switch (G->nz) {
    case 16: k_tri_tc_grp<16><<<G->tri_blocks, dim3(32, tri_tm<16>()), 0, s>>>(G->d_tri, ts, n); break;
    case 40: k_tri_tc_grp<40><<<G->tri_blocks, dim3(32, tri_tm<40>()), 0, s>>>(G->d_tri, ts, n); break;
    default: k_tri_tc_grp<80><<<G->tri_blocks, dim3(32, tri_tm<80>()), 0, s>>>(G->d_tri, ts, n); break;
  }
  if (one) {
    launch_tc_grp<OUT_T_BF16X2, true>(G, 2, s);
    if (add) launch_tc_grp<OUT_R_F32_ADD, true>(G, 3, s);
    else launch_tc_grp<OUT_R_F32, true>(G, 3, s);
  } else {
    launch_tc_grp<OUT_T_BF16X2>(G, 2, s);
    if (add) launch_tc_grp<OUT_R_F32_ADD>(G, 3, s);
    else launch_tc_grp<OUT_R_F32>(G, 3, s);
  }
}

int tc_group_solve(TcGroup* G, cudaStream_t s) {
  tc_group_pass(G, false, s, G->precision == 5);
  if (G->precision >= 2) {
    const int sweeps = G->precision == 4 ? 2 : 1;
    for (int sw = 0; sw < sweeps; sw++) {
      k_resid_grp<<<dim3(G->res_blocks, 1, G->nz), 128, 0, s>>>(G->d_res, G->d_res_map);
      tc_group_pass(G, true, s, G->precision == 3);
    }
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("ensemble solve launch: %s", cudaGetErrorString(e));
    return OB_ERR_DEVICE;
  }
  return OB_OK;
}

int tc_group_check(TcGroup* G) {
  unsigned int h = 0;
  cudaMemcpy(&h, G->err, sizeof(h), cudaMemcpyDeviceToHost);
  if (h) {
    cudaMemset(G->err, 0, sizeof(unsigned int));
    set_error("ensemble solve: a tensor-core pipeline wait timed out (code %u)", h);
    return OB_ERR_TIMEOUT;
  }
  return OB_OK;
}

}  // namespace ob

// ---- diagnostic: one bf16x3 batched transform C[p] = A B[p]^T, host arrays ----
extern "C" int ob_dst_tc_selftest(int M, int N, int K, int planes, const float* A, const float* B, float* C) {
  using namespace ob;
  if (M < 1 || N < 1 || K < 8 || K % 8 || planes < 1) { set_error("ob_dst_tc_selftest: bad sizes"); return OB_ERR_INVALID; }
  if (!get_encode()) { set_error("ob_dst_tc_selftest: no tensor map encoder"); return OB_ERR_DEVICE; }
  const long ld = K;
  std::vector<__nv_bfloat16> ah(size_t(M) * ld), al(size_t(M) * ld), bh(size_t(planes) * N * ld), bl(size_t(planes) * N * ld);
  for (size_t i = 0; i < ah.size(); i++) { ah[i] = __float2bfloat16_rn(A[i]); al[i] = __float2bfloat16_rn(A[i] - __bfloat162float(ah[i])); }
  for (size_t i = 0; i < bh.size(); i++) { bh[i] = __float2bfloat16_rn(B[i]); bl[i] = __float2bfloat16_rn(B[i] - __bfloat162float(bh[i])); }
  __nv_bfloat16 *dah, *dal, *dbh, *dbl;
  float* dc;
  unsigned int* derr;
  cudaMalloc(&dah, ah.size() * 2); cudaMalloc(&dal, al.size() * 2); cudaMalloc(&dbh, bh.size() * 2); cudaMalloc(&dbl, bl.size() * 2);
  cudaMalloc(&dc, size_t(planes) * M * N * 4); cudaMalloc(&derr, 16);
  cudaMemset(derr, 0, 16);
  cudaMemset(dc, 0, size_t(planes) * M * N * 4);
  cudaMemcpy(dah, ah.data(), ah.size() * 2, cudaMemcpyHostToDevice);
  cudaMemcpy(dal, al.data(), al.size() * 2, cudaMemcpyHostToDevice);
  cudaMemcpy(dbh, bh.data(), bh.size() * 2, cudaMemcpyHostToDevice);
  cudaMemcpy(dbl, bl.data(), bl.size() * 2, cudaMemcpyHostToDevice);
  // the test's A (M x K) is the transform matrix (the kernel's B operand); its B planes (planes x N x K) are the field
  const int bn = pick_bn(M);
  CUtensorMap tq[2], tf[2];
  bool ok = make_map_2d(&tq[0], dah, M, K, ld, bn) && make_map_2d(&tq[1], dal, M, K, ld, bn) &&
            make_map_2d(&tf[0], dbh, long(planes) * N, K, ld, BM) && make_map_2d(&tf[1], dbl, long(planes) * N, K, ld, BM);
  int rc = OB_OK;
  if (!ok) { set_error("ob_dst_tc_selftest: tensor map encoding failed"); rc = OB_ERR_DEVICE; }
  if (rc == OB_OK) {
    set_smem_attrs();
    const TcOut o{nullptr, nullptr, dc, N, N, planes * N, M};  // C[p][m][n] = out[(p * M + m) * N + n]
    launch_tc<OUT_T_F32>(tf, tq, K, bn, o, derr, nullptr);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { set_error("ob_dst_tc_selftest: %s", cudaGetErrorString(e)); rc = OB_ERR_DEVICE; }
    unsigned int h = 0;
    cudaMemcpy(&h, derr, 4, cudaMemcpyDeviceToHost);
    if (rc == OB_OK && h) { set_error("ob_dst_tc_selftest: pipeline wait timed out (code %u)", h); rc = OB_ERR_TIMEOUT; }
    if (rc == OB_OK) cudaMemcpy(C, dc, size_t(planes) * M * N * 4, cudaMemcpyDeviceToHost);
  }
  cudaFree(dah); cudaFree(dal); cudaFree(dbh); cudaFree(dbl); cudaFree(dc); cudaFree(derr);
  return rc;
}
