// FP64 trailing update on the integer tensor pipe by digit splitting (see
// ozaki_update.h).
//
//   F[J1:m, J1:m] -= X X^T,   X = F[J1:m, J0:J1]  (K = J1 - J0 <= kOzK)
//
// Digits.  Row a of X is scaled by 2^-e_a with e_a the exponent of its largest
// magnitude (frexp: |X(a, :)| 2^-e_a < 1), and the scaled values d are split
// exactly into kOzSlices signed 7-bit digits: q_i = trunc(128 d), d <- 128 d - q_i
// (every step exact in FP64; |q_i| <= 127).  Then
//   (X X^T)(a, b) = 2^(e_a + e_b) sum_g 2^-7(g + 2) sum_{i + j = g} Q_i(a, :) . Q_j(b, :)
// with i, j counted from 0; the pairs with i + j < kOzSlices are kept (36 of 64
// for 8 slices).  Each inner product of digit rows is an exact integer sum
// (|.| <= 127^2 K <= 8.3e6, a group of at most 8 of them < 2^31), so the only
// roundings are the truncation of the digit expansion and the final FP64
// addition and subtraction: with 8 slices the transients of the solve agree with the FP64
// direct factorization to the level at which two FP64 orderings agree.
//
// k_oz_slice writes the digits of every row, k_oz_update multiplies them on the
// tensor pipe: per CTA one 128 x 64 output tile (a 128 x 128 task-list tile is two
// CTAs), UMMA M = 128, N = 64, K = 32 (tcgen05.mma kind::i8, A and B from shared
// memory, K-major, 64-byte swizzle), one int32 accumulator in tensor memory per
// digit group g = i + j (8 x 64 columns = all 512).  Warp 0 lane 0 loads each
// 64-digit K block of all slices of the tile's 128 rows and 64 columns with two
// TMA boxes (64 x 128 x 8 and 64 x 64 x 8 bytes) into one of two stages; warp 1
// lane 0 issues the 2 x 36 MMAs of a stage and commits them to the stage's
// "empty" mbarrier; warps 2-9 (tensor-memory lane groups 2, 3, 0, 1, twice: one
// warp per 32 rows and 32 columns) wait for the tile's last commit, read the eight
// accumulators of their columns 4 at a time (all eight tcgen05.ld before one wait),
// put groups 0-3 and 4-7 together exactly as 64-bit integers, convert both by
// the magic-number method (no conversion-unit instructions: with a conversion per
// group the epilogue kept that unit 73% busy and held the tensor pipe at 36%),
// add them with one rounding, scale by 2^(e_a + e_b) and subtract from F.  TMA boxes read only this GPU's slice buffer
// (no multicast).  Every mbarrier wait is bounded; a CTA that gives up records
// err[2], waits (bounded) for its own MMAs and frees its tensor memory.
#include "ozaki_update.h"

#include <algorithm>
#include <string>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "symbolic.h"

namespace tdem {
namespace {

constexpr int OM = 128;                  // tile rows (UMMA M)
constexpr int ON = 64;                   // tile columns (UMMA N)
constexpr int OKB = 64;                  // digits (bytes) of K per stage
constexpr int OS = kOzSlices;            // digit slices
constexpr int A_SLICE = OM * OKB;        // 8 KB
constexpr int B_SLICE = ON * OKB;        // 4 KB
constexpr int A_BYTES = OS * A_SLICE;    // 64 KB
constexpr int B_BYTES = OS * B_SLICE;    // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int NST = 2;                   // stages
constexpr int NTHR = 320;                // producer warp, MMA warp, 8 epilogue warps
constexpr int NEPI = NTHR - 64;          // epilogue threads: two per tile row (32 columns each)
constexpr int EC = ON / 2;               // columns per epilogue thread
constexpr int TMEM_COLS = 512;           // OS accumulators of ON columns
constexpr size_t SMEM_BYTES = 1024 /* alignment */ + (size_t)NST * STAGE_BYTES + 256 /* barriers */ +
                              (OM + ON) * sizeof(int) /* exponents */;
constexpr unsigned kWaitLimit = 1u << 22;
static_assert(OS * ON == TMEM_COLS, "one accumulator per digit group fills tensor memory");
static_assert(SMEM_BYTES <= 227 * 1024, "shared memory of one CTA");

// instruction descriptor: D S32, A and B signed 8-bit, both K-major, M = 128, N = 64
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(ON >> 3) << 17) |
                            ((uint32_t)(OM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor of K half ks (32 bytes of each 64-byte row) of a
// K-major operand with 64-byte swizzle at addr (512-byte aligned): stride byte
// offset 512 (8-row groups), version 1, layout SWIZZLE_64B.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, int ks) {
  const uint32_t start = addr + 32 * ks;
  return (uint64_t)((start >> 4) & 0x3FFF) | ((uint64_t)(16 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) |
         (1ull << 46) | (4ull << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("{ .reg .b64 st; mbarrier.arrive.shared::cta.b64 st, [%0]; }" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// 3D tiled TMA load of box (x, y, z) of the map into dst, completing on bar
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
          "r"(dst),
      "l"(map), "r"(bar), "r"(x), "r"(y), "r"(z)
      : "memory");
}
__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accum) {
  asm volatile(
      "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p; }" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// x (|x| < 2^51) as a double without the conversion unit: the bit pattern of
// 2^52 + 2^51 plus x is the double 2^52 + 2^51 + x (unit spacing in [2^52, 2^53)),
// from which the subtraction is exact (the "magic number" conversion).
__device__ __forceinline__ double exact_double(long long x) {
  return __longlong_as_double(0x4338000000000000LL + x) - 6755399441055744.0;
}
// v 2^n: a product with the power of two built from its exponent bits (exact, or
// rounded once like ldexp when the result is subnormal); ldexp outside the range
// of normal powers
__device__ __forceinline__ double scale2(double v, int n) {
  return (n >= -1022 && n <= 1023) ? v * __longlong_as_double((long long)(n + 1023) << 52) : ldexp(v, n);
}

__device__ __forceinline__ int find_task(const int64_t* __restrict__ prefix, int count, int64_t b) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Digits of rows [row0, row0 + 64) of the panel of one front (64 rows per CTA,
// 256 threads): pass 1 finds each row's exponent, pass 2 stages 64 x 64 blocks
// of the panel (coalesced along the rows) and writes 16 digits per thread and
// slice as one 16-byte store; columns in [K, roundup(K, 64)) get zero digits.
__global__ void __launch_bounds__(256) k_oz_slice(const double* __restrict__ L, const int64_t* __restrict__ l_off,
                                                  const int* __restrict__ fm, const int* __restrict__ fk,
                                                  const int* __restrict__ fronts, const int64_t* __restrict__ prefix,
                                                  const int64_t* __restrict__ aux, int count, int j0,
                                                  int8_t* __restrict__ slices, int* __restrict__ exps,
                                                  int64_t nrows_buf) {
  __shared__ double T[64][65];  // [column][row]
  __shared__ double red[4][64];
  __shared__ double scale[64];
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = fm[s], k = fk[s];
  const int J0 = (j0 / kOuter) * kOuter, J1 = min(k, J0 + kOuter), K = J1 - J0;
  const int row0 = J1 + (int)(blockIdx.x - prefix[idx]) * 64;
  const int nrows = min(64, m - row0);
  const int64_t out0 = aux[idx] + (row0 - J1);
  const double* F = L + l_off[s];
  const int t = threadIdx.x, i = t & 63, g = t >> 6;
  double mx = 0.0;
  if (i < nrows)
    for (int kk = g; kk < K; kk += 4) mx = fmax(mx, fabs(F[(row0 + i) + (int64_t)(J0 + kk) * m]));
  red[g][i] = mx;
  __syncthreads();
  if (t < 64) {
    mx = fmax(fmax(red[0][t], red[1][t]), fmax(red[2][t], red[3][t]));
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);  // mx = f 2^e, 0.5 <= f < 1
    scale[t] = ldexp(1.0, -e);
    if (t < nrows) exps[out0 + t] = e;
  }
  __syncthreads();
  const int rr = t >> 2, seg = t & 3;
  for (int kc = 0; kc < K; kc += 64) {
#pragma unroll 4
    for (int j = 0; j < 16; ++j) {
      const int kk = kc + g + 4 * j;
      T[g + 4 * j][i] = (i < nrows && kk < K) ? F[(row0 + i) + (int64_t)(J0 + kk) * m] : 0.0;
    }
    __syncthreads();
    double d[16];
    const double sc = scale[rr];
#pragma unroll
    for (int q = 0; q < 16; ++q) d[q] = T[16 * seg + q][rr] * sc;
#pragma unroll 1
    for (int sl = 0; sl < OS; ++sl) {
      uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const double t8 = d[q] * 128.0;
        const double dg = trunc(t8);
        d[q] = t8 - dg;
        w[q >> 2] |= ((uint32_t)(int)dg & 0xFFu) << (8 * (q & 3));
      }
      if (rr < nrows)
        *reinterpret_cast<int4*>(slices + ((int64_t)sl * nrows_buf + out0 + rr) * kOzK + kc + 16 * seg) =
            make_int4((int)w[0], (int)w[1], (int)w[2], (int)w[3]);
    }
    __syncthreads();
  }
}

// One output tile of the task list: the tile's front and coordinates.  skip: the
// right half of a last 128-column tile past the front (no work).
struct OzTile {
  int s, m, k, J0, J1, nkb, r0, c0, arow, brow;
  bool skip;
};

__device__ __forceinline__ OzTile oz_tile(const int* __restrict__ fm, const int* __restrict__ fk,
                                          const int* __restrict__ fronts, const int64_t* __restrict__ prefix,
                                          const int64_t* __restrict__ aux, int count, int j0, int64_t id) {
  OzTile z;
  const int64_t tile = id >> 1;
  const int idx = find_task(prefix, count, tile);
  z.s = fronts[idx];
  z.m = fm[z.s];
  z.k = fk[z.s];
  z.J0 = (j0 / kOuter) * kOuter;
  z.J1 = min(z.k, z.J0 + kOuter);
  z.nkb = (z.J1 - z.J0 + OKB - 1) / OKB;
  const int64_t t = tile - prefix[idx];
  int bi = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((int64_t)(bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while ((int64_t)bi * (bi + 1) / 2 > t) --bi;
  const int bj = (int)(t - (int64_t)bi * (bi + 1) / 2);
  z.r0 = z.J1 + bi * 128;
  z.c0 = z.J1 + bj * 128 + (int)(id & 1) * ON;
  z.skip = z.c0 >= z.m;
  z.arow = (int)(aux[idx] + (z.r0 - z.J1));
  z.brow = (int)(aux[idx] + (z.c0 - z.J1));
  return z;
}

// Persistent: every CTA takes the tiles blockIdx.x, blockIdx.x + gridDim.x, ... of
// the 2 x ctas tile list (all roles walk the same sequence).  The producer and the
// MMA thread run ahead across tiles through the two-stage ring; the MMAs of a tile
// wait until the epilogue warps have read the previous tile's accumulators out of
// tensor memory ("tmem_free"), and the epilogue's global read-modify-write of a tile
// overlaps the next tile's loads and MMAs.
__global__ void __launch_bounds__(NTHR, 1)
k_oz_update(double* __restrict__ L, double* __restrict__ U, const int64_t* __restrict__ l_off,
            const int64_t* __restrict__ u_off, const int* __restrict__ fm, const int* __restrict__ fk,
            const int* __restrict__ fronts, const int64_t* __restrict__ prefix, const int64_t* __restrict__ aux,
            int count, int64_t ntiles, int j0, const int* __restrict__ exps, int64_t nrows_buf, int* err,
            const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  // 1024-byte aligned operand area (swizzle atoms are 512 bytes)
  unsigned char* ops =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
  // full[NST], empty[NST], acc_full, tmem_free, done
  uint64_t* bars = reinterpret_cast<uint64_t*>(ops + NST * STAGE_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(ops + NST * STAGE_BYTES + 64);
  int* s_fail = reinterpret_cast<int*>(ops + NST * STAGE_BYTES + 68);
  int* s_issued = s_fail + 1;    // K blocks (over all tiles) whose TMA loads were issued
  int* s_consumed = s_fail + 2;  // K blocks whose loads the MMA thread saw complete
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + NST);
  const uint32_t acc_full = smem_u32(bars + 2 * NST), tmem_free = smem_u32(bars + 2 * NST + 1),
                 done_bar = smem_u32(bars + 2 * NST + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int q = 0; q < NST; ++q) {
      mbar_init(full0 + 8 * q, 1);   // the producer's expect_tx arrival (+ the TMA bytes)
      mbar_init(empty0 + 8 * q, 1);  // one tcgen05.commit frees the stage
    }
    mbar_init(acc_full, 1);          // the commit after a tile's last MMAs
    mbar_init(tmem_free, NEPI);      // every epilogue thread, after its tensor-memory reads
    mbar_init(done_bar, 1);
    *s_fail = 0;
    *s_issued = 0;
    *s_consumed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // producer: K block kb of every slice of each tile's rows (A) and columns (B)
    int kbg = 0;
    bool stop = false;
    for (int64_t id = blockIdx.x; id < ntiles && !stop; id += gridDim.x) {
      const OzTile z = oz_tile(fm, fk, fronts, prefix, aux, count, j0, id);
      if (z.skip) continue;
      for (int kb = 0; kb < z.nkb; ++kb, ++kbg) {
        const int st = kbg % NST;
        if (kbg >= NST && !mbar_wait(empty0 + 8 * st, (uint32_t)(((kbg - NST) / NST) & 1))) {
          atomicExch(s_fail, 1);
          stop = true;
          break;
        }
        if (*(volatile int*)s_fail) {
          stop = true;
          break;
        }
        const uint32_t a = smem_u32(ops + st * STAGE_BYTES);
        mbar_expect_tx(full0 + 8 * st, (uint32_t)STAGE_BYTES);
        tma_load_3d(a, &tmA, full0 + 8 * st, kb * OKB, z.arow, 0);
        tma_load_3d(a + A_BYTES, &tmB, full0 + 8 * st, kb * OKB, z.brow, 0);
        *s_issued = kbg + 1;
      }
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: the kept digit pairs (i, j), i + j < OS, into accumulator i + j
    int kbg = 0, tc = 0;
    bool stop = false;
    for (int64_t id = blockIdx.x; id < ntiles && !stop; id += gridDim.x) {
      const OzTile z = oz_tile(fm, fk, fronts, prefix, aux, count, j0, id);
      if (z.skip) continue;
      // the epilogue has read the previous tile's accumulators
      if (tc > 0 && !mbar_wait(tmem_free, (uint32_t)((tc - 1) & 1))) {
        atomicExch(s_fail, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int kb = 0; kb < z.nkb; ++kb, ++kbg) {
        const int st = kbg % NST;
        if (!mbar_wait(full0 + 8 * st, (uint32_t)((kbg / NST) & 1))) {
          atomicExch(s_fail, 1);
          stop = true;
          break;
        }
        *s_consumed = kbg + 1;
        if (*(volatile int*)s_fail) {
          stop = true;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // descriptors of the stage's slice 0; the others differ only in the start
        // address field (bits 0-13, in 16-byte units), so the fully unrolled issue
        // below adds constants
        const uint64_t da0 = sdesc(smem_u32(ops + st * STAGE_BYTES), 0);
        const uint64_t db0 = sdesc(smem_u32(ops + st * STAGE_BYTES + A_BYTES), 0);
        const uint32_t first = kb > 0 ? 1u : 0u;
#pragma unroll
        for (int i = 0; i < OS; ++i) {
#pragma unroll
          for (int j = 0; j < OS - i; ++j) {
#pragma unroll
            for (int ks = 0; ks < OKB / 32; ++ks)
              mma_i8(tmem + (uint32_t)(ON * (i + j)), da0 + (uint64_t)((i * A_SLICE + 32 * ks) >> 4),
                     db0 + (uint64_t)((j * B_SLICE + 32 * ks) >> 4), (ks > 0 || i > 0) ? 1u : first);
          }
        }
        mma_commit(empty0 + 8 * st);
      }
      if (stop) break;
      mma_commit(acc_full);
      ++tc;
    }
    // every MMA issued: arrives once they have completed
    mma_commit(done_bar);
  } else if (warp >= 2) {
    // epilogue: row 32 (warp % 4) + lane of each tile, columns [cb, cb + EC) (warps
    // w and w + 4 share the tensor-memory lanes of their rows and split the columns)
    const int sub = warp & 3, rl = 32 * sub + lane, cb = EC * ((warp - 2) >> 2);
    int tc = 0;
    for (int64_t id = blockIdx.x; id < ntiles; id += gridDim.x) {
      const OzTile z = oz_tile(fm, fk, fronts, prefix, aux, count, j0, id);
      if (z.skip) continue;
      const int r = z.r0 + rl;
      const int ea = ((int64_t)z.arow + rl < nrows_buf) ? exps[z.arow + rl] : 0;
      // the exponents of this thread's 32 columns, one per lane (read before the
      // wait, handed to the other lanes with shuffles)
      const int ebl = ((int64_t)z.brow + cb + lane < nrows_buf) ? exps[z.brow + cb + lane] : 0;
      // one lane per warp polls the barrier (256 threads polling through a tile's
      // MMA phase kept a shared pipe busy and throttled the MMA and load threads);
      // the shuffle is the warp's synchronisation point before its tensor-memory reads
      int got = 1;
      if (lane == 0) got = mbar_wait(acc_full, (uint32_t)(tc & 1)) ? 1 : 0;
      bool ok = __shfl_sync(0xffffffffu, got, 0) != 0 && *(volatile int*)s_fail == 0;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      double v[EC];
      if (ok) {
#pragma unroll
        for (int cc = 0; cc < EC / 4; ++cc) {
          // 4 columns of all eight group accumulators, then one wait
          uint32_t a[OS][4];
#pragma unroll
          for (int g = 0; g < OS; ++g)
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                         : "=r"(a[g][0]), "=r"(a[g][1]), "=r"(a[g][2]), "=r"(a[g][3])
                         : "r"(tmem + ((uint32_t)(32 * sub) << 16) + (uint32_t)(ON * g + cb + 4 * cc)));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            // groups 0-3 and 4-7 put together exactly in 64-bit integers (|a_g| <=
            // 8 * 127^2 * 512 < 2^26, so |hi|, |lo| < 2^47), then one rounding
            long long hi = (int)a[0][q], lo = (int)a[4][q];
#pragma unroll
            for (int g = 1; g < 4; ++g) {
              hi = hi * 128 + (int)a[g][q];
              lo = lo * 128 + (int)a[4 + g][q];
            }
            v[4 * cc + q] = fma(exact_double(hi), 0x1p-35, exact_double(lo) * 0x1p-63);
          }
        }
      }
      // the accumulators are free for the next tile's MMAs
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      mbar_arrive(tmem_free);
      ++tc;
      if (!ok) break;
      {
        const int64_t lo = l_off[z.s], uo = u_off[z.s];
        const int m = z.m, k = z.k;
        const bool live = r < m;
#pragma unroll
        for (int h = 0; h < EC / 8; ++h) {
          double old[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int c = z.c0 + cb + 8 * h + q;
            old[q] = 0.0;
            if (live && c < m && c <= r)
              old[q] = (c < k) ? L[lo + r + (int64_t)c * m] : U[uo + (r - k) + (int64_t)(c - k) * (m - k)];
          }
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int cl = 8 * h + q, c = z.c0 + cb + cl;
            // every lane takes part in the shuffle
            const int eb = __shfl_sync(0xffffffffu, ebl, cl);
            if (live && c < m && c <= r) {
              double* e = (c < k) ? L + lo + r + (int64_t)c * m : U + uo + (r - k) + (int64_t)(c - k) * (m - k);
              *e = old[q] - scale2(v[cl], ea + eb);
            }
          }
        }
      }
    }
  }
  __syncthreads();
  const bool ok = mbar_wait(done_bar, 0u) && *(volatile int*)s_fail == 0;
  if (!ok && tid == 0) {
    atomicExch(err + 2, 1);
    // loads issued but never seen complete by the MMA thread: wait (bounded) for
    // them, so that no copy into this CTA's shared memory outlives it
    for (int kb = *s_consumed; kb < *s_issued; ++kb) mbar_wait(full0 + 8 * (kb % NST), (uint32_t)((kb / NST) & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

}  // namespace

std::string ozaki_setup(OzakiBuffers& ob) {
  static_assert(sizeof(CUtensorMap) <= sizeof(ob.map_a), "tensor map storage");
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess || !fn || q != cudaDriverEntryPointSuccess)
    return "cuTensorMapEncodeTiled not available from the driver";
  auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
  const cuuint64_t dims[3] = {(cuuint64_t)kOzK, (cuuint64_t)ob.rows, (cuuint64_t)OS};
  const cuuint64_t strides[2] = {(cuuint64_t)kOzK, (cuuint64_t)kOzK * (cuuint64_t)ob.rows};
  const cuuint32_t elem[3] = {1, 1, 1};
  const cuuint32_t box_a[3] = {OKB, OM, OS}, box_b[3] = {OKB, ON, OS};
  CUresult r = encode(reinterpret_cast<CUtensorMap*>(ob.map_a), CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, ob.slices, dims,
                      strides, box_a, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return "cuTensorMapEncodeTiled (128-row digit boxes) failed: " + std::to_string((int)r);
  r = encode(reinterpret_cast<CUtensorMap*>(ob.map_b), CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, ob.slices, dims, strides,
             box_b, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return "cuTensorMapEncodeTiled (64-row digit boxes) failed: " + std::to_string((int)r);
  e = cudaFuncSetAttribute(k_oz_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
  if (e != cudaSuccess) return std::string("cudaFuncSetAttribute(k_oz_update): ") + cudaGetErrorString(e);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&ob.sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                 cudaSuccess)
    return "cannot read the SM count";
  return "";
}

void launch_ozaki_slice(const double* L, const int64_t* l_off, const int* m, const int* k, const int* fronts,
                        const int64_t* prefix, const int64_t* aux, int count, int64_t ctas, int j0,
                        const OzakiBuffers& ob, cudaStream_t s) {
  k_oz_slice<<<(unsigned)ctas, 256, 0, s>>>(L, l_off, m, k, fronts, prefix, aux, count, j0, ob.slices, ob.exps,
                                            ob.rows);
}

void launch_ozaki_update(double* L, double* U, const int64_t* l_off, const int64_t* u_off, const int* m,
                         const int* k, const int* fronts, const int64_t* prefix, const int64_t* aux, int count,
                         int64_t ctas, int j0, const OzakiBuffers& ob, int* err, cudaStream_t s) {
  const int64_t ntiles = 2 * ctas;
  const unsigned grid = (unsigned)std::min<int64_t>(ntiles, ob.sms > 0 ? ob.sms : 148);
  k_oz_update<<<grid, NTHR, SMEM_BYTES, s>>>(
      L, U, l_off, u_off, m, k, fronts, prefix, aux, count, ntiles, j0, ob.exps, ob.rows, err,
      *reinterpret_cast<const CUtensorMap*>(ob.map_a), *reinterpret_cast<const CUtensorMap*>(ob.map_b));
}

}  // namespace tdem
