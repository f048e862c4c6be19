// Blackwell 5th-generation tensor cores (tcgen05) for the low-precision trailing
// update of the mixed-precision factor:
//
//     C(i, j) += alpha * sum_k A(i, k) B(j, k)      (alpha = -1 in the factor)
//
// with A and B in BF16 (kind::f16) or TF32 (kind::tf32, FP32 words), k-contiguous
// (A(i, k) = a[i*lda + k]), and C in FP32, column-major, FP32 accumulation.  One CTA
// computes a 128 x 128 tile of C:
//   * thread 0 streams 128-row x 128-byte tiles of A and B into a 3-stage shared-
//     memory ring with TMA (cp.async.bulk.tensor.2d, 128-byte swizzle, no multicast);
//   * thread 32 issues tcgen05.mma.cta_group::1 (M = 128, N = 128) on the staged
//     tiles and tcgen05.commit frees each stage when its MMAs are done;
//   * the 128 x 128 FP32 accumulator lives in tensor memory (128 columns allocated
//     by warp 0); after the last k block all four warps read it back with
//     tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows), stage alpha * acc
//     in 32 x 32 blocks of the (now idle) ring buffer, and add them into C with TMA
//     reduce-add stores (cp.reduce.async.bulk.tensor .add), so that the epilogue
//     never waits on a load of C.  Entries masked out by the lower-only rule add 0.
// Every wait is bounded; a wait that gives up records an error word, the CTA waits
// (bounded) for its loads in flight, and the tensor memory is freed on every path.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include "scalar.cuh"

namespace cuchol {
namespace tc {

// Tiles: 128 x 128 outputs, k blocks of 128 bytes per operand row (64 BF16 or 32
// TF32 elements: one 128-byte swizzle atom wide), 3 stages of 2 x 16 KB, so that two
// CTAs share an SM and one's epilogue overlaps the other's loads.
constexpr int BM = 128, BN = 128, ROW_BYTES = 128, STAGES = 3, THREADS = 128;
constexpr int A_STAGE = BM * ROW_BYTES, B_STAGE = BN * ROW_BYTES;   // 16 KB each
constexpr int STAGE_BYTES = A_STAGE + B_STAGE;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;               // + alignment slack
constexpr unsigned kSpinLimit = 1u << 26;              // bounded mbarrier waits: at most 2^26 polls
constexpr unsigned long long kWaitNs = 1000000000ull;   // and at most one second
constexpr int TMEM_COLS = 128;

// Operand element types: BF16 (kind::f16, K = 16 per MMA) and TF32 held in FP32
// words (kind::tf32, K = 8 per MMA); either way one MMA consumes 32 bytes of each
// operand row.
template <typename Op> struct OpKind;
template <> struct OpKind<__nv_bfloat16> {
  static constexpr int BK = 64;
  static constexpr uint32_t fmt = 1;   // BF16
};
template <> struct OpKind<float> {
  static constexpr int BK = 32;
  static constexpr uint32_t fmt = 2;   // TF32
};

struct Params {
  int m, n, k;                      // C region m x n (its TMA map); operands m x k and n x k                      // C region m x n; operands m x k and n x k
  int a_row0, b_row0;               // first operand rows in the tensor maps
  float alpha;                      // C := C + alpha * A B^T (the factor uses -1)
  int lower_only;                   // only C(i, j) with i >= j (region corner on the diagonal)
  int tiles_m, tiles_n;
  int* err;                         // set to 1 when a wait gives up
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// bounded wait (polls and wall-clock time; a poll may suspend the thread for a while)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  unsigned long long t0 = 0;
  for (unsigned it = 0; it < kSpinLimit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    if (it == 0) t0 = global_ns();
    else if ((it & 15u) == 15u && global_ns() - t0 > kWaitNs) return false;
  }
  return false;
}
__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap* map, const void* src, int x, int y) {
  asm volatile("cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.bulk_group [%0, {%2, %3}], [%1];"
               ::"l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(src)), "r"(x), "r"(y)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, uint64_t* bar, void* dst, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major BF16 tile with 128-byte swizzle:
// rows of 128 bytes (64 elements), 8-row swizzle atoms 1024 bytes apart.
//   bits 0-13 start address >> 4, 16-29 leading byte offset >> 4 (unused for this
//   layout, 1), 32-45 stride byte offset >> 4 (1024 >> 4), 46-48 fixed 0b001,
//   61-63 swizzle mode (2 = 128-byte).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor: FP32 accumulator (bits 4-5 = 1), A and B format at bits
// 7-9 and 10-12 (BF16 = 1, TF32 = 2), both K-major (bits 15, 16 = 0), N >> 3 at bits
// 17-22, M >> 4 at bits 24-28.
template <typename Op>
__host__ __device__ constexpr uint32_t idesc() {
  return (1u << 4) | (OpKind<Op>::fmt << 7) | (OpKind<Op>::fmt << 10) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}

template <typename Op>
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate);
template <>
__device__ __forceinline__ void mma<__nv_bfloat16>(uint32_t tmem, uint64_t adesc, uint64_t bdesc,
                                                   uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem), "l"(adesc), "l"(bdesc), "r"(idesc<__nv_bfloat16>()), "r"(accumulate)
      : "memory");
}
template <>
__device__ __forceinline__ void mma<float>(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n"
      ::"r"(tmem), "l"(adesc), "l"(bdesc), "r"(idesc<float>()), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// Tile t of the launch -> (tile row, tile column).  Lower-only regions (m >= n, the
// corner on the diagonal) enumerate only tiles with ti >= tj, row by row, so that
// consecutive CTAs share their A rows.
__device__ __forceinline__ void tile_of(int t, const Params& p, int& ti, int& tj) {
  if (!p.lower_only) {
    ti = t / p.tiles_n;
    tj = t - ti * p.tiles_n;
    return;
  }
  const int tri = p.tiles_n * (p.tiles_n + 1) / 2;   // rows 0 .. tiles_n-1 hold ti + 1 tiles
  if (t < tri) {
    int r = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while (r > 0 && r * (r + 1) / 2 > t) --r;
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    ti = r;
    tj = t - r * (r + 1) / 2;
  } else {
    const int u = t - tri;
    ti = p.tiles_n + u / p.tiles_n;
    tj = u - (u / p.tiles_n) * p.tiles_n;
  }
}

// SPLIT3 (TF32 only): FP32 products to about FP32 accuracy on the TF32 tensor cores.
// Every operand is held as hi = tf32(x) and lo = tf32(x - hi) (x = hi + lo to
// 2^-22 |x|), ma maps the hi values and mb the lo values of one k-major matrix Q
// (A rows from a_row0, B rows from b_row0 of both), and each k block issues
//     lo_A hi_B^T + hi_A lo_B^T + hi_A hi_B^T
// into the same FP32 accumulator (the dropped lo lo^T term is below 2^-22 of the
// product).  A stage then holds four 16 KB tiles, so one CTA per SM.
// UPPER: the region (described, like the lower case, as the logical lower trapezoid
// m x n with its corner on the diagonal) is stored transposed: mc maps the physical
// n x m upper trapezoid of a column-major matrix (the symmetric update of upper
// storage), with a 128-byte swizzle, and each 32 x 32 block is staged transposed.
template <bool SPLIT3> struct Ring {
  static constexpr int STAGE = SPLIT3 ? 2 * (A_STAGE + B_STAGE) : A_STAGE + B_STAGE;
  static constexpr int SMEM = STAGES * STAGE + 1024;
  static constexpr int A_OFF_LO = A_STAGE;                       // SPLIT3 layout: Ahi Alo Bhi Blo
  static constexpr int B_OFF = SPLIT3 ? 2 * A_STAGE : A_STAGE;
};

template <typename Op, bool SPLIT3 = false, bool UPPER = false>
__global__ void __launch_bounds__(THREADS, SPLIT3 ? 1 : 2)
    update_kernel(const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb,
                  const __grid_constant__ CUtensorMap mc, Params p, const int* stop) {
  static_assert(!SPLIT3 || sizeof(Op) == 4, "the split product is for TF32 operands");
  constexpr int BK = OpKind<Op>::BK;
  using RG = Ring<SPLIT3>;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full[STAGES];
  __shared__ __align__(8) uint64_t empty[STAGES];
  __shared__ __align__(8) uint64_t accb;
  __shared__ uint32_t tmem_slot;
  __shared__ int s_consumed, s_fail;

  if (cta_aborted(stop)) return;   // an earlier step failed
  int ti, tj;
  tile_of(blockIdx.x, p, ti, tj);
  const int row0 = ti * BM, col0 = tj * BN;
  uint8_t* base = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kblocks = (p.k + BK - 1) / BK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&accb, 1);
    s_consumed = 0;
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tmem_alloc(&tmem_slot, TMEM_COLS);
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_slot;

  int issued = 0;
  if (threadIdx.x == 0) {
    // TMA producer
    for (int kb = 0; kb < kblocks; ++kb) {
      const int s = kb % STAGES;
      if (kb >= STAGES && !mbar_wait(&empty[s], ((kb / STAGES) & 1) ^ 1)) {
        s_fail = 1;
        break;
      }
      uint8_t* st = base + s * RG::STAGE;
      mbar_expect_tx(&full[s], RG::STAGE);
      if constexpr (SPLIT3) {
        tma_load_2d(&ma, &full[s], st, kb * BK, p.a_row0 + row0);
        tma_load_2d(&mb, &full[s], st + RG::A_OFF_LO, kb * BK, p.a_row0 + row0);
        tma_load_2d(&ma, &full[s], st + RG::B_OFF, kb * BK, p.b_row0 + col0);
        tma_load_2d(&mb, &full[s], st + RG::B_OFF + B_STAGE, kb * BK, p.b_row0 + col0);
      } else {
        tma_load_2d(&ma, &full[s], st, kb * BK, p.a_row0 + row0);
        tma_load_2d(&mb, &full[s], st + RG::B_OFF, kb * BK, p.b_row0 + col0);
      }
      ++issued;
    }
  } else if (threadIdx.x == 32) {
    // MMA issuer: 4 MMAs of 32 bytes of k per stage
    int kb = 0;
    for (; kb < kblocks; ++kb) {
      const int s = kb % STAGES;
      if (!mbar_wait(&full[s], (kb / STAGES) & 1)) {
        s_fail = 1;
        break;
      }
      fence_after();
      const uint32_t a = smem_u32(base + s * RG::STAGE), b = a + RG::B_OFF;
#pragma unroll
      for (int kk = 0; kk < ROW_BYTES / 32; ++kk) {
        if constexpr (SPLIT3) {
          const uint32_t alo = a + RG::A_OFF_LO, blo = b + B_STAGE;
          mma<Op>(tmem, smem_desc(alo + 32 * kk), smem_desc(b + 32 * kk), (kb | kk) != 0 ? 1u : 0u);
          mma<Op>(tmem, smem_desc(a + 32 * kk), smem_desc(blo + 32 * kk), 1u);
          mma<Op>(tmem, smem_desc(a + 32 * kk), smem_desc(b + 32 * kk), 1u);
        } else {
          mma<Op>(tmem, smem_desc(a + 32 * kk), smem_desc(b + 32 * kk), (kb | kk) != 0 ? 1u : 0u);
        }
      }
      mma_commit(&empty[s]);
    }
    s_consumed = kb;
    mma_commit(&accb);   // arrives when every MMA issued above has completed
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_consumed < issued) {
    // a wait gave up: let the loads still in flight land before the CTA exits
    for (int kb = s_consumed; kb < issued; ++kb) mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1);
  }
  const bool acc_ok = mbar_wait(&accb, 0);
  fence_after();
  if (!acc_ok) s_fail = 1;
  __syncthreads();
  const bool ok = s_fail == 0;

  if (ok) {
    // the ring is idle now: warp w stages its 32 x 32 blocks in two 4 KB buffers
    float* stg = reinterpret_cast<float*>(base) + warp * 2048;
    const int r = row0 + 32 * warp + lane;
    const uint32_t trow = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll 1
    for (int cc = 0; cc < BN / 32; ++cc) {
      const int cbase = col0 + 32 * cc;
      if (cbase >= p.n || (p.lower_only && cbase > row0 + BM - 1)) break;   // uniform across the CTA
      float* buf = stg + (cc & 1) * 1024;
      if (cc >= 2) {
        if (lane == 0) bulk_wait_read<1>();   // the reduce that read this buffer is done
        __syncwarp();
      }
      float v[32];
      tmem_ld32(trow + 32 * cc, v);
      if constexpr (UPPER) {
        // transposed block: physical column = this lane's row, 128-byte swizzled rows
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          float4 w;
          w.x = (!p.lower_only || r >= cbase + 4 * q + 0) ? p.alpha * v[4 * q + 0] : 0.f;
          w.y = (!p.lower_only || r >= cbase + 4 * q + 1) ? p.alpha * v[4 * q + 1] : 0.f;
          w.z = (!p.lower_only || r >= cbase + 4 * q + 2) ? p.alpha * v[4 * q + 2] : 0.f;
          w.w = (!p.lower_only || r >= cbase + 4 * q + 3) ? p.alpha * v[4 * q + 3] : 0.f;
          *reinterpret_cast<float4*>(buf + lane * 32 + ((q ^ (lane & 7)) << 2)) = w;
        }
      } else {
#pragma unroll
        for (int i = 0; i < 32; ++i) buf[i * 32 + lane] = (!p.lower_only || r >= cbase + i) ? p.alpha * v[i] : 0.f;
      }
      fence_proxy_async();
      __syncwarp();
      if (lane == 0) {
        if constexpr (UPPER) tma_reduce_add_2d(&mc, buf, cbase, row0 + 32 * warp);
        else tma_reduce_add_2d(&mc, buf, row0 + 32 * warp, cbase);
        bulk_commit();
      }
    }
    if (lane == 0) bulk_wait_read<0>();
    __syncwarp();
  } else if (threadIdx.x == 0) {
    atomicExch(p.err, 1);
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

}  // namespace tc
}  // namespace cuchol
