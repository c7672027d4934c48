// Tensor-core GEMM of the batched DFT operator (c/mfista_dft_lib.c:30-66,
// :253-278 apply A and A^T one vector at a time with dgemv) for sm_100a:
//
//   P[s][b][r] = sum_{k in K-split s} Amat[r][k] * X[b][k]
//
// with both operands K-major in BF16 "split" form, NP planes each
// (Amat = A0 + A1 [+ A2], every plane BF16, the next plane the rounding
// residual of the previous ones), and
//
//   NP = 2:  Amat X ~ A0 X0 + A0 X1 + A1 X0                       (3 MMAs)
//   NP = 3:  Amat X ~ A0 X0 + A0 X1 + A1 X0 + A0 X2 + A1 X1 + A2 X0 (6 MMAs)
//
// per K step, accumulated in FP32 in tensor memory.  The dropped terms and
// the rounding of the planes leave ~2^-16 (NP = 2) or ~2^-24 (NP = 3)
// relative error per product; callers apply it only to the difference
// between an iterate and an FP64 anchor (defect correction), so the solve
// keeps FP64 accuracy.
//
// One CTA computes a 128-row x 64-problem tile over one K split:
//   * one thread issues TMA tile loads (128-byte swizzle) into a 4-stage
//     shared-memory ring, completion tracked by mbarriers;
//   * one thread issues tcgen05.mma (kind::f16, BF16 in, FP32 accumulate,
//     M = 128, N = 64, K = 16) from shared-memory descriptors and frees each
//     stage with tcgen05.commit;
//   * all four warps read the accumulator back with tcgen05.ld (warp w owns
//     TMEM lanes 32w..32w+31 = tile rows) and store FP32 partials, 32
//     consecutive rows per warp store.
// Every wait is bounded (globaltimer); a timeout sets *err and the CTA
// drains what it issued and releases its tensor memory before returning.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "common.cuh"

namespace mf {
namespace tc {

constexpr int kTM = 128;                            // tile rows (MMA M)
constexpr int kTN = 64;                             // tile problems (MMA N)
constexpr int kTK = 64;                             // K per stage: 128 B of BF16
constexpr int kATile = kTM * kTK * 2;               // 16 KB per plane
constexpr int kXTile = kTN * kTK * 2;               // 8 KB per plane

// shared-memory ring of a kernel with NP planes per operand
template <int NP> struct Ring {
  static constexpr int kStageBytes = NP * (kATile + kXTile);
  static constexpr int kStages = NP == 2 ? 4 : 3;
  static constexpr int kSmemBytes = kStages * kStageBytes + 1024;  // + alignment slack
};

// TMA maps of the operand planes (plane p of A, of X)
struct TcMaps {
  CUtensorMap a[3];
  CUtensorMap x[3];
};
constexpr uint32_t kTmemCols = 64;                  // FP32 accumulator: 128 lanes x 64 columns
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s bound on every wait

// tcgen05 instruction descriptor: dense, D = F32 (bits 4-5 = 1), A = B = BF16
// (bits 7-9, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3 at bit 17,
// M >> 4 at bit 24
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTN >> 3) << 17) |
                            ((uint32_t)(kTM >> 4) << 24);

struct TcArgs {
  float* part;      // [nsplit][bpad][rows]
  int rows;         // padded rows (multiple of kTM)
  int bpad;         // padded problems (multiple of kTN)
  int kblocks;      // K blocks (of kTK) per split
  int kblocks_all;  // K blocks in total
  int* err;         // set to 1 when a wait gave up
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// waits for the completion of the barrier phase with this parity; false if
// it has not completed within `limit_ns`
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long limit_ns) {
  const uint32_t a = smem_addr(bar);
  const unsigned long long t0 = now_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (now_ns() - t0 > limit_ns) return false;
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_addr(dst)),
      "l"((unsigned long long)tm), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// shared-memory matrix descriptor of a K-major tile stored with the 128-byte
// swizzle (rows of 128 B, 8-row groups 1024 B apart, tile 1024-B aligned)
__device__ __forceinline__ uint64_t sw128_desc(const void* tile) {
  uint64_t a = smem_addr(tile);
  uint64_t d = (a & 0x3FFFFull) >> 4;   // start address, 16-B units
  d |= 1ull << 16;                      // leading-dimension offset (unused for this layout)
  d |= (uint64_t)(1024 >> 4) << 32;     // stride-dimension offset: one 8-row group
  d |= 1ull << 46;                      // descriptor version of sm_100
  d |= 2ull << 61;                      // 128-byte swizzle
  return d;
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// grid (rows / kTM, nsplit, bpad / kTN), 128 threads, Ring<NP>::kSmemBytes
// dynamic shared memory
template <int NP>
__global__ void __launch_bounds__(128, 1)
    k_gemm_split_bf16(const __grid_constant__ TcMaps maps, TcArgs g, const ProbState* __restrict__ st, int gate,
                      int B) {
  constexpr int kStages = Ring<NP>::kStages;
  constexpr int kStageBytes = Ring<NP>::kStageBytes;
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], accf;
  __shared__ uint32_t tmem_slot;
  __shared__ int s_any;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = blockIdx.x * kTM, split = blockIdx.y, b0 = blockIdx.z * kTN;
  if (threadIdx.x == 0) {
    int any = 0;
    for (int i = 0; i < kTN && b0 + i < B; ++i) any |= gate_ok(st[b0 + i], gate) ? 1 : 0;
    s_any = any;
  }
  __syncthreads();
  if (!s_any) return;  // no problem of this tile is active (uniform over the CTA)
  const int kb0 = split * g.kblocks;
  const int nk = min(g.kblocks, g.kblocks_all - kb0);
  const uint32_t s0 = smem_addr(smem_raw);
  unsigned char* ring = smem_raw + ((1024u - (s0 & 1023u)) & 1023u);  // 1024-B aligned stages

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&accf, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  int failed = 0;

  if (warp == 0 && lane == 0) {
    // TMA producer
    int issued = 0;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % kStages;
      if (kb >= kStages && !mbar_wait(&empty[s], ((kb / kStages) - 1) & 1, kWaitNs)) {
        failed = 1;
        break;
      }
      unsigned char* sb = ring + s * kStageBytes;
      mbar_expect_tx(&full[s], kStageBytes);
      const int kx = (kb0 + kb) * kTK;
#pragma unroll
      for (int p = 0; p < NP; ++p) tma_load_2d(sb + p * kATile, &maps.a[p], kx, row0, &full[s]);
#pragma unroll
      for (int p = 0; p < NP; ++p) tma_load_2d(sb + NP * kATile + p * kXTile, &maps.x[p], kx, b0, &full[s]);
      issued = kb + 1;
    }
    if (failed) {  // let the copies already issued land before the CTA exits
      for (int kb = max(0, issued - kStages); kb < issued; ++kb)
        mbar_wait(&full[kb % kStages], (kb / kStages) & 1, kWaitNs);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: products A_i X_j with i + j < NP, lowest order first
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % kStages;
      if (!mbar_wait(&full[s], (kb / kStages) & 1, kWaitNs)) {
        failed = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      unsigned char* sb = ring + s * kStageBytes;
      uint64_t ad[NP], xd[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p) {
        ad[p] = sw128_desc(sb + p * kATile);
        xd[p] = sw128_desc(sb + NP * kATile + p * kXTile);
      }
#pragma unroll
      for (int j = 0; j < kTK / 16; ++j) {
        const uint64_t dk = (uint64_t)(j * 32) >> 4;  // 16 BF16 = 32 B further along K
        umma_bf16(tmem, ad[0] + dk, xd[0] + dk, (kb > 0 || j > 0) ? 1u : 0u);
#pragma unroll
        for (int ord = 1; ord < NP; ++ord)
#pragma unroll
          for (int i = 0; i <= ord; ++i) umma_bf16(tmem, ad[i] + dk, xd[ord - i] + dk, 1u);
      }
      umma_commit(&empty[s]);  // the stage is free once these MMAs have read it
    }
    umma_commit(&accf);  // fires when every MMA issued above has completed
  }
  __syncwarp();

  // epilogue: TMEM -> registers -> FP32 partials
  const bool acc_ok = mbar_wait(&accf, 0, 2 * kWaitNs);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const bool all_ok = __all_sync(0xffffffffu, acc_ok ? 1 : 0) != 0;
  if (all_ok) {
    float* out = g.part + ((size_t)split * g.bpad + b0) * g.rows + row0 + warp * 32 + lane;
    const uint32_t tw = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c0 = 0; c0 < kTN; c0 += 16) {
      float v[16];
      tmem_ld16(tw + c0, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) out[(size_t)(c0 + j) * g.rows] = v[j];
    }
  }
  if (failed || !all_ok) atomicExch(g.err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// plane p of the split of v: v = P0 + P1 [+ P2], each BF16
template <int NP> __device__ __forceinline__ void split_value(double v, __nv_bfloat16 (&q)[NP]) {
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    q[p] = __double2bfloat16(v);
    v -= (double)__bfloat162float(q[p]);
  }
}

struct Planes {
  __nv_bfloat16* p[3];
};

// BF16 split planes of a column-major FP64 matrix A (M x N, A[m + n M]):
//   rm: [mrow][nk]  rows m, K = n contiguous  -- operand of A x
//   cm: [nrow][mk]  rows n, K = m contiguous  -- operand of A^T r
// (mrow, nrow multiples of the tile rows, nk, mk of the K block; padding is
// zero).  32 x 32 tiles through shared memory so both layouts are written
// with coalesced stores; grid (cdiv(max(mrow, mk), 32), cdiv(max(nrow, nk), 32)),
// 256 threads.
template <int NP>
__global__ void k_split_matrix(const double* __restrict__ A, int M, int N, int mrow, int nk, int nrow, int mk,
                               Planes rm, Planes cm) {
  __shared__ double t[32][33];
  const int m0 = blockIdx.x * 32, n0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  for (int j = ty; j < 32; j += 8) {
    int m = m0 + tx, n = n0 + j;
    t[j][tx] = (m < M && n < N) ? A[(size_t)n * M + m] : 0.0;  // t[n - n0][m - m0]
  }
  __syncthreads();
  for (int j = ty; j < 32; j += 8) {  // cm: row n, consecutive threads along m
    int n = n0 + j, m = m0 + tx;
    if (n < nrow && m < mk) {
      __nv_bfloat16 q[NP];
      split_value<NP>(t[j][tx], q);
#pragma unroll
      for (int p = 0; p < NP; ++p) cm.p[p][(size_t)n * mk + m] = q[p];
    }
  }
  for (int j = ty; j < 32; j += 8) {  // rm: row m, consecutive threads along n
    int m = m0 + j, n = n0 + tx;
    if (m < mrow && n < nk) {
      __nv_bfloat16 q[NP];
      split_value<NP>(t[tx][j], q);
#pragma unroll
      for (int p = 0; p < NP; ++p) rm.p[p][(size_t)m * nk + n] = q[p];
    }
  }
}

// BF16 split planes of a batch of vectors, X[b][k] = src[b][k] - sub[b][k]
// (sub may be null), K-major [bpad][kpad]; problems outside the gate or
// beyond B, and the K padding, are zero
template <int NP>
__global__ void k_split_vectors(const double* __restrict__ src, long sstride, const double* __restrict__ sub,
                                long substride, int K, int kpad, int B, const ProbState* __restrict__ st, int gate,
                                Planes x) {
  const int b = blockIdx.y;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kpad) return;
  double v = 0.0;
  if (b < B && k < K && gate_ok(st[b], gate)) {
    v = src[(size_t)b * sstride + k];
    if (sub) v -= sub[(size_t)b * substride + k];
  }
  __nv_bfloat16 q[NP];
  split_value<NP>(v, q);
#pragma unroll
  for (int p = 0; p < NP; ++p) x.p[p][(size_t)b * kpad + k] = q[p];
}

}  // namespace tc
}  // namespace mf
