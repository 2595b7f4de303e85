// Trailing update of the FP32 factorization on the 5th-generation tensor cores.
//
//   F[J1:m, J1:m] -= X X^T,   X = F[J1:m, J0:J1]  (K = J1 - J0 <= kOuter)
//
// for every front of a level that reaches the end of an outer panel, on the
// lower-triangle 128 x 128 tiles of its trailing matrix (the same task list as the
// CUDA-core kernel it replaces).  FP32 accuracy comes from 3xTF32: each operand is
// split as x = xb + xs with xb = tf32(x), xs = tf32(x - xb), and the tile is
// accumulated in FP32 in tensor memory as Xb Xb^T + Xb Xs^T + Xs Xb^T (the
// dropped Xs Xs^T term is below FP32 rounding).
//
// CTA = 13 warps.  Warps 0-11 are producers in three groups of four; group g fills
// K stages g, g + 3, ... into its own stage buffer: it reads the 128 rows of both
// operands from global memory (coalesced along rows, any alignment; all loads of
// a stage issued before the first use), splits them and stores both halves with
// 16-byte stores in the K-major 128-byte-swizzled layout that the UMMA
// descriptors describe.  Warp 12 issues tcgen05.mma (M = N = 128, K = 8 per
// instruction) from one lane and commits each stage to an mbarrier that frees the
// stage's buffer.  After the last stage warps 0-7 read the accumulator from tensor
// memory (tcgen05.ld, warp w owns lanes 32 (w % 4) .. + 31) and subtract it from F.
//
// Every wait is bounded; a wait that gives up records err[2] and the CTA skips
// the rest of its work, still waiting (bounded) for its own MMAs and freeing its
// tensor memory before it returns.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "symbolic.h"
#include "tc_update.h"

namespace tdem {
namespace {

constexpr int TM = 128;                  // tile rows (UMMA M) and columns (UMMA N)
constexpr int TKS = 32;                  // K per pipeline stage
constexpr int NSTAGE = 3;                // operand buffers in flight
constexpr int OPB = TM * TKS * 4;        // bytes of one operand half (16 KB)
constexpr int STAGE_BYTES = 4 * OPB;     // A big, A small, B big, B small
constexpr int NGROUP = 3;                // producer groups (one stage buffer each)
constexpr int NPROD = 128 * NGROUP;      // producer threads (4 warps per group)
constexpr int NTHREADS = NPROD + 32;     // + the MMA warp
constexpr size_t SMEM_BYTES = (size_t)NSTAGE * STAGE_BYTES + 1024 /* alignment */ + 256 /* barriers */;
constexpr unsigned kWaitLimit = 1u << 22;
static_assert(NGROUP == NSTAGE, "producer group g owns stage buffer g");

// instruction descriptor: D F32, A/B TF32, both K-major, M = N = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TM >> 3) << 17) |
                            ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// K-major operand half (128 rows x 32 K elements): 16 groups of 8 rows, group at
// (mn / 8) * 1024; row mn % 8 is one 128-byte line of 32 consecutive K elements,
// its 16-byte chunks (4 elements) XOR-swizzled with the row index.  Byte offset of
// chunk c (elements 4c .. 4c + 3) of row mn:
__device__ __forceinline__ uint32_t chunk_off(int mn, int c) {
  const int row = mn & 7;
  return (uint32_t)((mn >> 3) * 1024 + row * 128 + ((c ^ row) << 4));
}

// UMMA shared-memory descriptor of the K = 8 slice ks (32 bytes along each line)
// of an operand half at addr: stride byte offset 1024 (8-row groups), version 1,
// 128-byte swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, int ks) {
  const uint32_t start = addr + 32 * ks;
  return (uint64_t)((start >> 4) & 0x3FFF) | ((uint64_t)(16 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
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

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accum) {
  asm volatile(
      "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p; }" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
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

// Splits 32 values into their TF32 halves and stores them as eight 16-byte chunks
// of row p of both operand halves.
__device__ __forceinline__ void split_store(const float (&v)[TKS], unsigned char* big, unsigned char* small, int p) {
#pragma unroll
  for (int c = 0; c < TKS / 4; ++c) {
    float4 b, sm;
    b.x = tf32_rna(v[4 * c + 0]);
    b.y = tf32_rna(v[4 * c + 1]);
    b.z = tf32_rna(v[4 * c + 2]);
    b.w = tf32_rna(v[4 * c + 3]);
    sm.x = tf32_rna(v[4 * c + 0] - b.x);
    sm.y = tf32_rna(v[4 * c + 1] - b.y);
    sm.z = tf32_rna(v[4 * c + 2] - b.z);
    sm.w = tf32_rna(v[4 * c + 3] - b.w);
    const uint32_t o = chunk_off(p, c);
    *reinterpret_cast<float4*>(big + o) = b;
    *reinterpret_cast<float4*>(small + o) = sm;
  }
}

// Row `row` of the panel, columns [kc, kc + 32) (ld = m; rows >= m and columns >=
// kend read as 0).
__device__ __forceinline__ void load_row(const float* __restrict__ F, int m, int row, int kc, int kend,
                                         float (&v)[TKS]) {
  const bool okr = row < m;
#pragma unroll
  for (int kk = 0; kk < TKS; ++kk) v[kk] = (okr && kc + kk < kend) ? F[row + (int64_t)(kc + kk) * m] : 0.f;
}

__global__ void __launch_bounds__(NTHREADS, 1)
k_syrk_tc(float* __restrict__ L, float* __restrict__ U, const int64_t* __restrict__ l_off,
          const int64_t* __restrict__ u_off, const int* __restrict__ fm, const int* __restrict__ fk,
          const int* __restrict__ fronts, const int64_t* __restrict__ prefix, int count, int j0, int* err) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  // 1024-byte aligned operand area (the 128-byte swizzle repeats every 1024 bytes)
  unsigned char* ops = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(ops + NSTAGE * STAGE_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * NSTAGE);
  int* s_fail = reinterpret_cast<int*>(tmem_slot + 1);
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + NSTAGE);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int idx = find_task(prefix, count, blockIdx.x);
  const int s = fronts[idx];
  const int m = fm[s], k = fk[s];
  const int J0 = (j0 / kOuter) * kOuter, J1 = min(k, J0 + kOuter);
  const int K = J1 - J0;
  const int nst = (K + TKS - 1) / TKS;
  const int64_t t = blockIdx.x - prefix[idx];
  int bi = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((int64_t)(bi + 1) * (bi + 2) / 2 <= t) ++bi;
  while ((int64_t)bi * (bi + 1) / 2 > t) --bi;
  const int bj = (int)(t - (int64_t)bi * (bi + 1) / 2);
  const int r0 = J1 + bi * TM, c0 = J1 + bj * TM;
  const bool diag = bi == bj;
  const float* F = L + l_off[s];

  if (tid == 0) {
    for (int q = 0; q < NSTAGE; ++q) {
      mbar_init(full0 + 8 * q, 128);  // one producer group fills a stage
      mbar_init(empty0 + 8 * q, 1);         // one tcgen05.commit frees it
    }
    *s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TM)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp < NPROD / 32) {
    // producers: group g = warp / 4 takes stages st = g, g + NGROUP, ... in buffer g
    const int g = warp >> 2, p = tid & 127;
    for (int st = g; st < nst; st += NGROUP) {
      const int buf = g;
      if (st >= NSTAGE) {
        // the MMAs of stage st - NSTAGE must have consumed this buffer
        if (!mbar_wait(empty0 + 8 * buf, (uint32_t)(((st - NSTAGE) / NSTAGE) & 1))) {
          atomicExch(s_fail, 1);
          break;
        }
      }
      if (*(volatile int*)s_fail) break;
      unsigned char* base = ops + buf * STAGE_BYTES;
      const int kc = J0 + st * TKS;
      float va[TKS], vb[TKS];
      load_row(F, m, r0 + p, kc, J1, va);
      if (!diag) load_row(F, m, c0 + p, kc, J1, vb);
      split_store(va, base, base + OPB, p);
      if (!diag) split_store(vb, base + 2 * OPB, base + 3 * OPB, p);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(full0 + 8 * buf);
    }
  } else {
    // MMA warp: one elected lane issues and commits
    for (int st = 0; st < nst; ++st) {
      const int buf = st % NSTAGE;
      bool ok = true;
      if (lane == 0) ok = mbar_wait(full0 + 8 * buf, (uint32_t)((st / NSTAGE) & 1));
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
      if (!ok || *(volatile int*)s_fail) {
        if (lane == 0) atomicExch(s_fail, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (lane == 0) {
        const uint32_t base = smem_u32(ops + buf * STAGE_BYTES);
        const uint32_t ab = base, as = base + OPB;
        const uint32_t bb = diag ? ab : base + 2 * OPB, bs = diag ? as : base + 3 * OPB;
#pragma unroll
        for (int ks = 0; ks < TKS / 8; ++ks) {
          mma_tf32(tmem, sdesc(as, ks), sdesc(bb, ks), (st > 0 || ks > 0) ? 1u : 0u);
          mma_tf32(tmem, sdesc(ab, ks), sdesc(bs, ks), 1u);
          mma_tf32(tmem, sdesc(ab, ks), sdesc(bb, ks), 1u);
        }
        mma_commit(empty0 + 8 * buf);
      }
      __syncwarp();
    }
  }

  // all MMAs done: the last stage's commit covers every earlier MMA
  __syncthreads();
  bool ok = *(volatile int*)s_fail == 0;
  if (nst > 0) {
    const int last = nst - 1;
    const bool done = mbar_wait(empty0 + 8 * (last % NSTAGE), (uint32_t)((last / NSTAGE) & 1));
    ok = ok && done;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok && warp < 8 && nst > 0) {
    // epilogue: warp w reads lanes 32 (w % 4) .. of columns [64 (w / 4), + 64)
    const int sub = warp & 3, half = warp >> 2;
    const int r = r0 + 32 * sub + lane;
    const int64_t lo = l_off[s], uo = u_off[s];
#pragma unroll 1
    for (int cc = 0; cc < 2; ++cc) {
      const int col0 = 64 * half + 32 * cc;
      uint32_t v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(tmem + ((uint32_t)(32 * sub) << 16) + (uint32_t)col0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (r < m) {
        // all loads of the 32 columns first, then all stores (the pointers may
        // alias as far as the compiler knows, which would serialise them)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          float old[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int c = c0 + col0 + 16 * h + j;
            old[j] = 0.f;
            if (c < m && c <= r)
              old[j] = (c < k) ? L[lo + r + (int64_t)c * m] : U[uo + (r - k) + (int64_t)(c - k) * (m - k)];
          }
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int c = c0 + col0 + 16 * h + j;
            if (c < m && c <= r) {
              float* e = (c < k) ? L + lo + r + (int64_t)c * m : U + uo + (r - k) + (int64_t)(c - k) * (m - k);
              *e = old[j] - __uint_as_float(v[16 * h + j]);
            }
          }
        }
      }
    }
  }
  if (!ok && tid == 0) atomicExch(err + 2, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TM) : "memory");
  }
}

}  // namespace

std::string tc_update_setup() {
  cudaError_t e = cudaFuncSetAttribute(k_syrk_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
  return e == cudaSuccess ? std::string() : std::string("cudaFuncSetAttribute(k_syrk_tc): ") + cudaGetErrorString(e);
}

void launch_syrk_tc(float* L, float* U, const int64_t* l_off, const int64_t* u_off, const int* m, const int* k,
                    const int* fronts, const int64_t* prefix, int count, int64_t ctas, int j0, int* err,
                    cudaStream_t s) {
  k_syrk_tc<<<(unsigned)ctas, NTHREADS, SMEM_BYTES, s>>>(L, U, l_off, u_off, m, k, fronts, prefix, count, j0, err);
}

}  // namespace tdem
