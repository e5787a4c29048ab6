// Split-precision (3xTF32) GEMM on the 5th-generation tensor cores for the
// FP32 relay factorisation of the mixed mode.
//
//   C (+)= A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T
//
// where X_hi is X with its low 13 mantissa bits cleared (exactly a TF32
// number) and X_lo = X - X_hi.  The three products run as one K loop of
// 3*K over two tensor maps per operand.  Dropping A_lo B_lo^T leaves an error
// near 2^-22 relative per product -- FP32-level -- which the FP64 iterative
// refinement of the relay solve removes.
//
// One CTA computes one 128x128 tile of C (batch index = blockIdx.y):
//   warp 0, one lane : TMA producer (cp.async.bulk.tensor, 128B swizzle)
//                      into a 3-stage shared-memory ring (A,B 16 KB each);
//   warp 1, one lane : issues tcgen05.mma.kind::tf32 (128x128x8) into a
//                      128-column TMEM accumulator, releases each stage with
//                      tcgen05.commit -> mbarrier;
//   all 4 warps      : epilogue, tcgen05.ld 32x32b (warp w owns TMEM lanes /
//                      rows 32w..32w+31) into a swizzled staging tile, then a
//                      TMA reduce-add (C -= acc) or TMA stores (C = acc, hi, lo).
// Every mbarrier wait is bounded: on time-out the kernel records
// MBD_ERR_TIMEOUT, skips the remaining work and still frees its TMEM.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"
#include "wait_limit.cuh"
#include "tc3.h"
#include "../../include/mbd_b200.h"

namespace mbd {
namespace {

constexpr int BM = 128, BN = 128, BK = 32;   // BK fp32 = 128 bytes = one swizzle atom row
constexpr int STAGES = 3;                    // 97 KB: two CTAs per SM overlap epilogue and main loop
constexpr int TILE_BYTES = BM * BK * 4;      // 16 KB
constexpr int STAGE_BYTES = 2 * TILE_BYTES;
constexpr int TMEM_COLS = 128;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded wait for phase `parity` of an mbarrier.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err) {
  const long long lim = wait_limit_cycles();
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > lim || *(volatile int*)err != 0) {
      atomicCAS(err, 0, MBD_ERR_TIMEOUT);
      return false;
    }
  }
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, uint32_t src, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];"
               ::"l"(reinterpret_cast<uint64_t>(map)), "r"(src), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}

__device__ __forceinline__ void tma_reduce_add_3d(const CUtensorMap* map, uint32_t src, int c0, int c1, int c2) {
  asm volatile("cp.reduce.async.bulk.tensor.3d.global.shared::cta.add.bulk_group [%0, {%2, %3, %4}], [%1];"
               ::"l"(reinterpret_cast<uint64_t>(map)), "r"(src), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), LBO unused (1), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                 // LBO (ignored for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;       // SBO
  d |= (uint64_t)1 << 46;                 // version
  d |= (uint64_t)2 << 61;                 // SWIZZLE_128B
  return d;
}

// Instruction descriptor: D = F32, A = B = TF32, both K-major, M = 128, N = 128.
__host__ __device__ constexpr uint32_t idesc_tf32_128x128() {
  return (1u << 4)            // c_format F32
         | (2u << 7)          // a_format TF32
         | (2u << 10)         // b_format TF32
         | ((BN >> 3) << 17)  // N
         | ((BM >> 4) << 24); // M
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

__device__ __forceinline__ void tri_index(int t, int* ti, int* tj) {
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  *ti = i;
  *tj = t - i * (i + 1) / 2;
}

__global__ void __launch_bounds__(128, 2) tc3_gemm_kernel(const __grid_constant__ Tc3Maps maps, Tc3Params p) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  // 1024-byte alignment for the swizzled tiles
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], done_bar;
  __shared__ uint32_t tmem_base_sh;

  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int b = blockIdx.y;
  int tm, tn;
  if (p.mode == TC3_SYRK_LOWER) {
    tri_index(blockIdx.x, &tm, &tn);
  } else {
    tm = blockIdx.x / p.n_tiles_n;
    tn = blockIdx.x % p.n_tiles_n;
  }
  const int k_tiles = p.k / BK;
  const int iters = 3 * k_tiles;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(smem_u32(&full_bar[s]), 1);
      mbar_init(smem_u32(&empty_bar[s]), 1);
    }
    mbar_init(smem_u32(&done_bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_sh;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer ----------------
    const int arow = p.a_row0 + tm * BM, brow = p.b_row0 + tn * BN;
    for (int i = 0; i < iters; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = (uint32_t)((i / STAGES) & 1);
      if (i >= STAGES && !mbar_wait(smem_u32(&empty_bar[s]), ph ^ 1u, p.err)) break;
      const int seg = i / k_tiles, kk = (i % k_tiles) * BK;
      const CUtensorMap* ma = (seg == 2) ? &maps.a_lo : &maps.a_hi;
      const CUtensorMap* mb = (seg == 1) ? &maps.b_lo : &maps.b_hi;
      uint8_t* sa = smem + s * STAGE_BYTES;
      uint8_t* sb = sa + TILE_BYTES;
      const uint32_t fb = smem_u32(&full_bar[s]);
      mbar_expect_tx(fb, STAGE_BYTES);
      tma_load_3d(smem_u32(sa), ma, fb, kk, arow, b);
      tma_load_3d(smem_u32(sb), mb, fb, kk, brow, b);
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t idesc = idesc_tf32_128x128();
    bool ok = true;
    for (int i = 0; i < iters; ++i) {
      const int s = i % STAGES;
      const uint32_t ph = (uint32_t)((i / STAGES) & 1);
      if (!mbar_wait(smem_u32(&full_bar[s]), ph, p.err)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
      const uint32_t sb = sa + TILE_BYTES;
#pragma unroll
      for (int k4 = 0; k4 < BK / 8; ++k4) {   // 8 tf32 = 32 bytes per MMA
        umma_tf32(tmem, umma_desc_sw128(sa + 32 * k4), umma_desc_sw128(sb + 32 * k4), idesc,
                  (i > 0 || k4 > 0) ? 1u : 0u);
      }
      umma_commit(smem_u32(&empty_bar[s]));
    }
    if (ok) umma_commit(smem_u32(&done_bar));
  }
  __syncwarp();
  // ---------------- epilogue ----------------
  // TMEM -> registers -> 128-byte-swizzled staging tile in the (now idle)
  // pipeline shared memory -> one TMA bulk operation per 128x32 chunk:
  // reduce-add of -acc (SYRK) or plain stores of acc and its hi/lo split.
  // The tensor bounds clip rows/columns outside the matrix.
  //   After a wait above gave up, done_bar is never committed: every thread
  // then spends the bounded wait here, by whose end the copies and MMAs
  // issued before the abort have completed, so TMEM is freed below only
  // once nothing in flight can still write it.
  const bool ok = mbar_wait(smem_u32(&done_bar), 0, p.err);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int rl = warp * 32 + lane;                // tile row == TMEM lane
    const int row = tm * BM + rl;                   // row within the C region
    const bool diag_tile = (p.mode == TC3_SYRK_LOWER) && (tm == tn);
    uint8_t* stg0 = smem;                           // 16 KB each
    uint8_t* stg1 = smem + TILE_BYTES;
    uint8_t* stg2 = smem + 2 * TILE_BYTES;
#pragma unroll 1
    for (int cc = 0; cc < BN / 32; ++cc) {
      uint32_t r[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cc * 32), r);
      const int col0 = tn * BN + cc * 32;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        float4 v, h, l;
        float* pv = reinterpret_cast<float*>(&v);
        float* ph = reinterpret_cast<float*>(&h);
        float* pl = reinterpret_cast<float*>(&l);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int col = col0 + 4 * j + u;
          const float x = __uint_as_float(r[4 * j + u]);
          if (p.mode == TC3_SYRK_LOWER) {
            pv[u] = (diag_tile && col > row) ? 0.f : -x;
          } else {
            pv[u] = x;
            ph[u] = tf32_hi(x);
            pl[u] = x - ph[u];
          }
        }
        const uint32_t off = (uint32_t)rl * 128u + ((uint32_t)(j ^ (rl & 7)) << 4);
        *reinterpret_cast<float4*>(stg0 + off) = v;
        if (p.mode != TC3_SYRK_LOWER) {
          *reinterpret_cast<float4*>(stg1 + off) = h;
          *reinterpret_cast<float4*>(stg2 + off) = l;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("bar.sync 1, 128;" ::: "memory");
      if (threadIdx.x == 0) {
        const int gx = p.c_col0 + col0, gy = p.c_row0 + tm * BM;
        if (p.mode == TC3_SYRK_LOWER) {
          tma_reduce_add_3d(&maps.c, smem_u32(stg0), gx, gy, b);
        } else {
          tma_store_3d(&maps.c, smem_u32(stg0), gx, gy, b);
          tma_store_3d(&maps.c_hi, smem_u32(stg1), col0, gy, b);
          tma_store_3d(&maps.c_lo, smem_u32(stg2), col0, gy, b);
        }
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
    }
    if (threadIdx.x == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// hi/lo split of a row block of an FP32 matrix: out[b][r][c] for r in [r0, r0+rows), c < cols.
__global__ void split_kernel(const float* A, size_t a_bstride, int a_ld, int r0, int c0, int rows, int cols,
                             float* hi, float* lo, size_t o_bstride, int o_ld) {
  const int b = blockIdx.y;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)rows * cols) return;
  const int r = (int)(idx / cols), c = (int)(idx % cols);
  const float x = A[(size_t)b * a_bstride + (size_t)(r0 + r) * a_ld + c0 + c];
  const float h = tf32_hi(x);
  hi[(size_t)b * o_bstride + (size_t)(r0 + r) * o_ld + c] = h;
  lo[(size_t)b * o_bstride + (size_t)(r0 + r) * o_ld + c] = x - h;
}

}  // namespace

constexpr size_t kTc3Smem = STAGES * STAGE_BYTES + 1024;

cudaError_t init_tc3_attributes() {
  return cudaFuncSetAttribute(tc3_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTc3Smem);
}

void launch_tc3_gemm(const Tc3Maps& maps, const Tc3Params& p, int tiles, cudaStream_t s) {
  tc3_gemm_kernel<<<dim3(tiles, p.batch), 128, kTc3Smem, s>>>(maps, p);
}

void launch_split(const float* A, size_t a_bstride, int a_ld, int r0, int c0, int rows, int cols, float* hi,
                  float* lo, size_t o_bstride, int o_ld, int batch, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return;
  const size_t total = (size_t)rows * cols;
  split_kernel<<<dim3((unsigned)((total + 255) / 256), batch), 256, 0, s>>>(A, a_bstride, a_ld, r0, c0, rows, cols,
                                                                           hi, lo, o_bstride, o_ld);
}

// ---- tensor maps ----------------------------------------------------------
namespace {
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
  }
  return fn;
}
}  // namespace

// 3-D map over [batch][rows][cols] FP32 (row-major, ld elements, bstride
// elements between batches) with a 32 x 128 box and 128-byte swizzle.
bool make_tc3_map(CUtensorMap* map, const float* base, int rows, int cols, int ld, size_t bstride, int batch) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)batch};
  cuuint64_t strides[2] = {(cuuint64_t)ld * 4, (cuuint64_t)bstride * 4};
  cuuint32_t box[3] = {BK, BM, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

MBD_WAIT_LIMIT_SETTER(set_wait_limit_tc3)

}  // namespace mbd
