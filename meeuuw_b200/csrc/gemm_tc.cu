// BF16 tensor-core GEMM for sm_100a: D[M, N] = A[M, K] * B[N, K]^T, FP32 accumulation in TMEM.
//
// This is the dense-contraction engine of the learned warm start: the U-Net convolutions as
// implicit GEMMs (k_conv3x3_bf16_tc: the A tiles loaded per tap from the activations by 4D TMA)
// and the remaining contractions (weight gradients, small-channel layers) over im2col matrices
// (k_gemm_bf16_tc).  Design:
//   * one CTA per 128 x BN output tile (BN = 32..256), 128 threads;
//   * A and B tiles (64 BF16 of K per row = 128 bytes) are brought into shared memory by TMA
//     (cp.async.bulk.tensor, 128-byte swizzle, this GPU's own memory only) through a 4-stage
//     mbarrier pipeline;
//   * one thread issues tcgen05.mma (kind::f16, M=128, N=BN, K=16; four per 64-wide K block)
//     with both operands described by shared-memory matrix descriptors, accumulating in TMEM;
//     tcgen05.commit releases each stage and finally signals the epilogue;
//   * four warps read the accumulator back with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31,
//     i.e. output rows), apply the epilogue (bias, ReLU, BF16 or FP32 store) and write D;
//   * split-K over blockIdx.z writes FP32 partial tiles that a separate kernel reduces.
// Every wait is bounded: on timeout the kernel sets an error word, drains what it issued (again
// bounded), releases its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "tma.cuh"

namespace mw {

constexpr int GT_THREADS = 128;
constexpr int GT_BM = 128;
constexpr int GT_BK = 64;                 // BF16 elements per K block (128 bytes, one swizzle row)
constexpr int GT_STAGES = 4;
constexpr long long GT_SPIN = 1LL << 26;  // wait bound (iterations)

// wait on an mbarrier phase, bounded by GT_SPIN polls; false on timeout
MW_D bool mbar_wait(uint64_t* bar, uint32_t parity) { return mbar_wait_bounded(bar, parity, GT_SPIN); }

// Shared-memory matrix descriptor, K-major operand with 128-byte swizzle: rows of 128 bytes,
// 8-row atoms of 1024 bytes (stride byte offset), descriptor version 1.
MW_D uint64_t sdesc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                    // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;          // stride byte offset
  d |= (uint64_t)1 << 46;                    // version
  d |= (uint64_t)2 << 61;                    // SWIZZLE_128B
  return d;
}

// The same for 64-byte rows with 64-byte swizzle (8-row atoms of 512 bytes): the K blocks of 32
// BF16 of the implicit convolution over 32-channel tensors.
MW_D uint64_t sdesc_sw64(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(512 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)4 << 61;                    // SWIZZLE_64B
  return d;
}

// Instruction descriptor: kind::f16, A = B = BF16 (K-major), D = F32, M = 128, N = BN.
MW_HD uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

MW_D void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

MW_D void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

MW_D void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

struct GemmEpi {
  int mode;             // MW_GEMM_EPI_*
  int relu;
  const float* bias;    // per output column (may be null)
  void* out;            // bf16 or f32, row-major with leading dimension ldo
  int64_t ldo;
  int64_t split_stride; // elements between split-K partial tiles (MW_GEMM_EPI_F32 with gridDim.z > 1)
};

template <int BN>
__global__ void __launch_bounds__(GT_THREADS, 1)
k_gemm_bf16_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M, int N,
               int kblocks_per_split, int kblocks_total, GemmEpi ep, int32_t* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte alignment for the swizzled tiles
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  constexpr int A_BYTES = GT_BM * GT_BK * 2;          // 16 KB
  constexpr int B_BYTES = BN * GT_BK * 2;
  constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  uint64_t* bars = (uint64_t*)(base + GT_STAGES * STAGE_BYTES);
  uint64_t* full = bars;
  uint64_t* empty = bars + GT_STAGES;
  uint64_t* done = bars + 2 * GT_STAGES;
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * GT_STAGES + 1);
  __shared__ int abort_flag;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * GT_BM, n0 = blockIdx.y * BN;
  const int kb0 = blockIdx.z * kblocks_per_split;
  int kb1 = kb0 + kblocks_per_split;
  if (kb1 > kblocks_total) kb1 = kblocks_total;
  const int nkb = kb1 > kb0 ? kb1 - kb0 : 0;

  if (tid == 0) {
    abort_flag = 0;
    for (int s = 0; s < GT_STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (tid == 0) {
    const uint32_t idesc = idesc_bf16(BN);
    bool ok = true;
    int produced = 0, consumed = 0;
    for (int it = 0; it < nkb + GT_STAGES - 1 && ok; ++it) {
      if (it < nkb) {                                           // produce K block it
        const int s = it % GT_STAGES;
        if (it >= GT_STAGES) ok = mbar_wait(&empty[s], (uint32_t)((it / GT_STAGES - 1) & 1));
        if (!ok) break;
        unsigned char* sa = base + s * STAGE_BYTES;
        mbar_expect_tx(&full[s], STAGE_BYTES);
        tma_load_2d(sa, &tmA, &full[s], (kb0 + it) * GT_BK, m0);
        tma_load_2d(sa + A_BYTES, &tmB, &full[s], (kb0 + it) * GT_BK, n0);
        produced = it + 1;
      }
      const int kc = it - (GT_STAGES - 1);
      if (kc >= 0 && kc < nkb) {                                // consume K block kc
        const int s = kc % GT_STAGES;
        ok = mbar_wait(&full[s], (uint32_t)((kc / GT_STAGES) & 1));
        if (!ok) break;
        consumed = kc + 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t sa = smem_u32(base + s * STAGE_BYTES);
        const uint32_t sb = sa + A_BYTES;
#pragma unroll
        for (int k = 0; k < GT_BK / 16; ++k)
          mma_bf16(tmem, sdesc_sw128(sa + k * 32), sdesc_sw128(sb + k * 32), idesc, (kc > 0 || k > 0) ? 1u : 0u);
        mma_commit(&empty[s]);
      }
    }
    if (!ok) {
      abort_flag = 1;
      set_flag(err, MW_FLAG_ITER_LIMIT);
      // drain: wait (bounded) for the loads already issued but not consumed
      for (int k = consumed; k < produced; ++k) mbar_wait(&full[k % GT_STAGES], (uint32_t)((k / GT_STAGES) & 1));
    }
    mma_commit(done);    // completes when every MMA issued above has finished
  }
  __syncthreads();
  const bool have_acc = nkb > 0;
  bool done_ok = mbar_wait(done, 0);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!done_ok) set_flag(err, MW_FLAG_ITER_LIMIT);
  if (done_ok && !abort_flag) {
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      if (have_acc) tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      else
        for (int i = 0; i < 16; ++i) v[i] = 0.f;
      const int cbase = n0 + c0;
      if (row >= M) {
        // rows past M hold zero-filled A rows: nothing to store
      } else if (ep.mode == MW_GEMM_EPI_F32) {
        float* o = (float*)ep.out + (int64_t)blockIdx.z * ep.split_stride + (int64_t)row * ep.ldo;
        for (int i = 0; i < 16; ++i) {
          const int c = cbase + i;
          if (c < N) o[c] = v[i] + (ep.bias ? ep.bias[c] : 0.f);
        }
      } else {
        __nv_bfloat16* o = (__nv_bfloat16*)ep.out + (int64_t)row * ep.ldo;
        for (int i = 0; i < 16; ++i) {
          const int c = cbase + i;
          if (c >= N) continue;
          float x = v[i] + (ep.bias ? ep.bias[c] : 0.f);
          if (ep.relu) x = fmaxf(x, 0.f);
          o[c] = __float2bfloat16(x);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

// 3x3 'same' convolution as an implicit GEMM: out[p, co] = sum_{tap, c} X[p + tap, c] W[co, tap C + c]
// with the A tile of each K block -- 128 pixels (a band of 128 / W full image rows) x KB channels of
// one tap -- loaded straight from the NHWC activations by a 4D TMA box at the tap's offset (image
// borders read as zero: the box starts at x = -1 or y = -1, or runs past the last row / column), so
// no im2col matrix is written.  K block kb covers taps-major K = tap C + c (the im2col layout), so
// the K blocks, their MMAs and their order are those of the explicit GEMM over im2col(X).  KB = 64
// (C a multiple of 64): 128-byte rows, 128-byte swizzle; KB = 32: 64-byte rows, 64-byte swizzle.
struct ConvGeo {
  int C, W, H;          // input channels, image width and height (W <= 128, 128 % W == 0)
  int band;             // image rows per 128-pixel tile (128 / W)
};

template <int BN, int KB>
__global__ void __launch_bounds__(GT_THREADS, 1)
k_conv3x3_bf16_tc(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmW, ConvGeo cg,
                  int M, int N, GemmEpi ep, int32_t* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  constexpr int A_BYTES = GT_BM * KB * 2;
  constexpr int B_BYTES = BN * KB * 2;
  constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  uint64_t* bars = (uint64_t*)(base + GT_STAGES * STAGE_BYTES);
  uint64_t* full = bars;
  uint64_t* empty = bars + GT_STAGES;
  uint64_t* done = bars + 2 * GT_STAGES;
  uint32_t* tmem_slot = (uint32_t*)(bars + 2 * GT_STAGES + 1);
  __shared__ int abort_flag;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * GT_BM, n0 = blockIdx.y * BN;
  const int hw = cg.H * cg.W;
  const int img = m0 / hw, y0 = (m0 - img * hw) / cg.W;     // tiles never straddle images (hw % 128 == 0)
  const int cpb = cg.C / KB;                                 // K blocks per tap
  const int nkb = 9 * cpb;

  if (tid == 0) {
    abort_flag = 0;
    for (int s = 0; s < GT_STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (tid == 0) {
    const uint32_t idesc = idesc_bf16(BN);
    bool ok = true;
    int produced = 0, consumed = 0;
    for (int it = 0; it < nkb + GT_STAGES - 1 && ok; ++it) {
      if (it < nkb) {                                           // produce K block it
        const int s = it % GT_STAGES;
        if (it >= GT_STAGES) ok = mbar_wait(&empty[s], (uint32_t)((it / GT_STAGES - 1) & 1));
        if (!ok) break;
        unsigned char* sa = base + s * STAGE_BYTES;
        const int tap = it / cpb, c0 = (it - tap * cpb) * KB;
        mbar_expect_tx(&full[s], STAGE_BYTES);
        tma_load_4d(sa, &tmX, &full[s], c0, tap % 3 - 1, y0 + tap / 3 - 1, img);
        tma_load_2d(sa + A_BYTES, &tmW, &full[s], it * KB, n0);
        produced = it + 1;
      }
      const int kc = it - (GT_STAGES - 1);
      if (kc >= 0 && kc < nkb) {                                // consume K block kc
        const int s = kc % GT_STAGES;
        ok = mbar_wait(&full[s], (uint32_t)((kc / GT_STAGES) & 1));
        if (!ok) break;
        consumed = kc + 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t sa = smem_u32(base + s * STAGE_BYTES);
        const uint32_t sb = sa + A_BYTES;
#pragma unroll
        for (int k = 0; k < KB / 16; ++k) {
          const uint64_t da = KB == 64 ? sdesc_sw128(sa + k * 32) : sdesc_sw64(sa + k * 32);
          const uint64_t db = KB == 64 ? sdesc_sw128(sb + k * 32) : sdesc_sw64(sb + k * 32);
          mma_bf16(tmem, da, db, idesc, (kc > 0 || k > 0) ? 1u : 0u);
        }
        mma_commit(&empty[s]);
      }
    }
    if (!ok) {
      abort_flag = 1;
      set_flag(err, MW_FLAG_ITER_LIMIT);
      for (int k = consumed; k < produced; ++k) mbar_wait(&full[k % GT_STAGES], (uint32_t)((k / GT_STAGES) & 1));
    }
    mma_commit(done);
  }
  __syncthreads();
  bool done_ok = mbar_wait(done, 0);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!done_ok) set_flag(err, MW_FLAG_ITER_LIMIT);
  if (done_ok && !abort_flag) {
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      const int cbase = n0 + c0;
      if (row >= M) {
      } else if (ep.mode == MW_GEMM_EPI_F32) {
        float* o = (float*)ep.out + (int64_t)row * ep.ldo;
        for (int i = 0; i < 16; ++i) {
          const int c = cbase + i;
          if (c < N) o[c] = v[i] + (ep.bias ? ep.bias[c] : 0.f);
        }
      } else {
        __nv_bfloat16* o = (__nv_bfloat16*)ep.out + (int64_t)row * ep.ldo;
        for (int i = 0; i < 16; ++i) {
          const int c = cbase + i;
          if (c >= N) continue;
          float x = v[i] + (ep.bias ? ep.bias[c] : 0.f);
          if (ep.relu) x = fmaxf(x, 0.f);
          o[c] = __float2bfloat16(x);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

// out[i] = sum_s part[s * stride + i] (+ bias per column)
__global__ void k_splitk_reduce(int64_t n, int splits, int64_t stride, int ncols, const float* __restrict__ part,
                                const float* __restrict__ bias, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < splits; ++k) s += part[k * stride + i];
    if (bias) s += bias[i % ncols];
    out[i] = s;
  }
}


// 2D row-major BF16 [rows, cols] (cols contiguous), box {64 cols, box_rows rows}, 128B swizzle,
// out-of-bounds rows/cols read as zero.
static int make_map(CUtensorMap* m, const void* ptr, int64_t rows, int64_t cols, int box_rows, int box_k = GT_BK) {
  auto enc = get_encode();
  if (!enc) return MW_ERR_CUDA;
  if (((uintptr_t)ptr & 15) || (cols * 2) % 16) return MW_ERR_BAD_ARG;
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(cols * 2)};
  cuuint32_t box[2] = {(cuuint32_t)box_k, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, box_k == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? MW_OK : MW_ERR_BAD_ARG;
}

// NHWC BF16 activations [B, H, W, C] as a 4D map (C innermost), box {KB channels, W, band, 1}:
// one box is a 128-pixel band of full image rows for one tap; rows and columns outside the image
// read as zero.
static int make_map_nhwc(CUtensorMap* m, const void* ptr, int B, int H, int W, int C, int band, int kb) {
  auto enc = get_encode();
  if (!enc) return MW_ERR_CUDA;
  if (((uintptr_t)ptr & 15) || (C * 2) % 16) return MW_ERR_BAD_ARG;
  cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
  cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)C * 2 * W, (cuuint64_t)C * 2 * W * H};
  cuuint32_t box[4] = {(cuuint32_t)kb, (cuuint32_t)W, (cuuint32_t)band, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(ptr), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, kb == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? MW_OK : MW_ERR_BAD_ARG;
}

template <int BN, int KB>
static int launch_conv(const CUtensorMap& tx, const CUtensorMap& tw, ConvGeo cg, int M, int N, GemmEpi ep,
                       int32_t* err, cudaStream_t s) {
  dim3 grid((M + GT_BM - 1) / GT_BM, (N + BN - 1) / BN, 1);
  const size_t smem = 1024 + GT_STAGES * (GT_BM * KB * 2 + BN * KB * 2) + 256;
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(k_conv3x3_bf16_tc<BN, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return MW_ERR_CUDA;
    attr_set = true;
  }
  k_conv3x3_bf16_tc<BN, KB><<<grid, GT_THREADS, smem, s>>>(tx, tw, cg, M, N, ep, err);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

template <int BN>
static int launch_gemm(const CUtensorMap& ta, const CUtensorMap& tb, int M, int N, int K, int splits, GemmEpi ep,
                       int32_t* err, cudaStream_t s) {
  const int kbt = K / GT_BK;
  const int per = (kbt + splits - 1) / splits;   // splits is pre-adjusted so that none is empty
  dim3 grid((M + GT_BM - 1) / GT_BM, (N + BN - 1) / BN, splits);
  const size_t smem = 1024 + GT_STAGES * (GT_BM * GT_BK * 2 + BN * GT_BK * 2) + 256;
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(k_gemm_bf16_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return MW_ERR_CUDA;
    attr_set = true;
  }
  k_gemm_bf16_tc<BN><<<grid, GT_THREADS, smem, s>>>(ta, tb, M, N, per, kbt, ep, err);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

}  // namespace mw

using namespace mw;

extern "C" {

int mw_gemm_bf16_tn(int32_t M, int32_t N, int32_t K, const void* A, int64_t lda, const void* B, int64_t ldb,
                    mw_gemm_epilogue epi, void* work, size_t work_bytes, int32_t* err, void* stream) {
  if (M <= 0 || N <= 0 || K <= 0 || (K % GT_BK) != 0 || lda < K || ldb < K) return MW_ERR_BAD_ARG;
  if (epi.splits < 1) epi.splits = 1;
  if (epi.splits > K / GT_BK) epi.splits = K / GT_BK;
  {  // every split gets at least one K block
    const int kbt = K / GT_BK, per = (kbt + epi.splits - 1) / epi.splits;
    epi.splits = (kbt + per - 1) / per;
  }
  int BN = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  CUtensorMap ta, tb;
  // A and B may carry row padding (lda >= K): describe them with their full leading dimension
  // and restrict the K extent through the box coordinates (the kernel only reads K blocks < K/64).
  int rc = make_map(&ta, A, M, lda, GT_BM);
  if (rc) return rc;
  rc = make_map(&tb, B, N, ldb, BN);
  if (rc) return rc;
  GemmEpi ep;
  ep.mode = epi.mode;
  ep.relu = epi.relu;
  ep.bias = epi.bias;
  ep.out = epi.out;
  ep.ldo = epi.ldo;
  ep.split_stride = 0;
  cudaStream_t s = (cudaStream_t)stream;
  const bool split = epi.splits > 1;
  if (split) {
    if (epi.mode != MW_GEMM_EPI_F32) return MW_ERR_BAD_ARG;
    const size_t need = (size_t)epi.splits * M * N * sizeof(float);
    if (!work || work_bytes < need) return MW_ERR_WORKSPACE;
    ep.out = work;
    ep.ldo = N;
    ep.bias = nullptr;
    ep.split_stride = (int64_t)M * N;
  }
  switch (BN) {
    case 32: rc = launch_gemm<32>(ta, tb, M, N, K, epi.splits, ep, err, s); break;
    case 64: rc = launch_gemm<64>(ta, tb, M, N, K, epi.splits, ep, err, s); break;
    case 128: rc = launch_gemm<128>(ta, tb, M, N, K, epi.splits, ep, err, s); break;
    default: rc = launch_gemm<256>(ta, tb, M, N, K, epi.splits, ep, err, s); break;
  }
  if (rc) return rc;
  if (split) {
    if (epi.ldo != N) return MW_ERR_BAD_ARG;
    const int64_t n = (int64_t)M * N;
    k_splitk_reduce<<<grid_for(n, 256), 256, 0, s>>>(n, epi.splits, n, N, (const float*)work, epi.bias,
                                                     (float*)epi.out);
    MW_CHECK_LAUNCH();
  }
  return MW_OK;
}

int mw_conv3x3_bf16(int32_t B, int32_t H, int32_t W, int32_t C, const void* X, int32_t N, const void* Wt, int64_t ldw,
                    mw_gemm_epilogue epi, int32_t* err, void* stream) {
  if (B <= 0 || H <= 0 || W <= 0 || N <= 0 || !X || !Wt) return MW_ERR_BAD_ARG;
  if (C <= 0 || C % 32 != 0 || W > GT_BM || GT_BM % W != 0 || ((int64_t)H * W) % GT_BM != 0) return MW_ERR_BAD_ARG;
  if (ldw < 9 * (int64_t)C || epi.splits > 1) return MW_ERR_BAD_ARG;
  const int KB = C % 64 == 0 ? 64 : 32;
  ConvGeo cg;
  cg.C = C; cg.W = W; cg.H = H; cg.band = GT_BM / W;
  const int M = B * H * W;
  int BN = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  CUtensorMap tx, tw;
  int rc = make_map_nhwc(&tx, X, B, H, W, C, cg.band, KB);
  if (rc) return rc;
  rc = make_map(&tw, Wt, N, ldw, BN, KB);
  if (rc) return rc;
  GemmEpi ep;
  ep.mode = epi.mode;
  ep.relu = epi.relu;
  ep.bias = epi.bias;
  ep.out = epi.out;
  ep.ldo = epi.ldo;
  ep.split_stride = 0;
  cudaStream_t s = (cudaStream_t)stream;
  if (KB == 64) {
    switch (BN) {
      case 32: return launch_conv<32, 64>(tx, tw, cg, M, N, ep, err, s);
      case 64: return launch_conv<64, 64>(tx, tw, cg, M, N, ep, err, s);
      case 128: return launch_conv<128, 64>(tx, tw, cg, M, N, ep, err, s);
      default: return launch_conv<256, 64>(tx, tw, cg, M, N, ep, err, s);
    }
  }
  switch (BN) {
    case 32: return launch_conv<32, 32>(tx, tw, cg, M, N, ep, err, s);
    case 64: return launch_conv<64, 32>(tx, tw, cg, M, N, ep, err, s);
    case 128: return launch_conv<128, 32>(tx, tw, cg, M, N, ep, err, s);
    default: return launch_conv<256, 32>(tx, tw, cg, M, N, ep, err, s);
  }
}

size_t mw_gemm_workspace_bytes(int32_t M, int32_t N, int32_t splits) {
  return (size_t)(splits < 1 ? 1 : splits) * M * N * sizeof(float);
}

}  // extern "C"
