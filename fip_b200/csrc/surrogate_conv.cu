// BF16 3x3 convolutions of the learned surrogate on the 5th-generation tensor cores (tcgen05).
//
// Activations are NHWC bf16 with 64 channels and a zero border of kPad pixels around each
// image: row p of the [N * (H + 2 kPad) * (W + 2 kPad)][64] matrix is one (padded) pixel, 128
// bytes. With that layout a 3x3 convolution of dilation d <= kPad is an implicit GEMM whose nine
// taps are plain row shifts of the activation matrix (tap (dy, dx) reads row
// p + d * (dy * Wp + dx), Wp = W + 2 kPad), so every operand tile is one TMA box:
//
//   forward / dgrad   D[128 pixels][64 out] += sum over 9 taps of
//                     A_tap[128 pixels][64 in] (K-major, rows shifted) x B_tap[64 out][64 in]^T
//   wgrad             D[(2 taps x 64 in)][64 out] += sum over pixels of
//                     X_shifted[pixels][64 in]^T x dY[pixels][64 out]   (both MN-major)
//
// Operands are staged in shared memory by TMA with the 128-byte swizzle, one thread issues
// tcgen05.mma (kind::f16, bf16 inputs, fp32 accumulation in tensor memory) and commits to
// mbarriers, and four epilogue warps read the accumulator with tcgen05.ld and apply the fused
// epilogue (bias, residual, ReLU, ReLU-mask of the backward pass, zero border). Persistent CTAs
// (one per SM) double-buffer the accumulators so the epilogue of a work unit overlaps the MMAs of
// the next. A work unit is 1 to 3 adjacent 128-pixel tiles whose MMAs are issued interleaved into
// independent accumulators (measured: the tensor pipe is busy 62% of the time with one tile per
// unit, 76% with two); how many depends on the epilogue (tiles_per_unit). Every mbarrier wait is bounded; on expiry the kernel records an error, stops and
// frees its tensor memory.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "drv.h"
#include "smem_attr.h"
#include "surrogate.h"

namespace fip {
namespace sg {

namespace {

constexpr int C = 64;                   // channels of every activation tensor
constexpr int BM = 128;                 // pixels per forward tile (MMA M)
constexpr int kTapBytes = C * C * 2;    // 8 KB: one tap of the weights, 64 x 64 bf16
constexpr int kWBytes = 9 * kTapBytes;  // 72 KB
// one slab per kernel row: a tile's 128 rows plus the 2 * dilation rows its dx shifts reach
constexpr int kSlabStride = 18 * 1024;  // slabs start on 1024-byte boundaries (swizzle pattern); <= 144 rows
constexpr int kStages = 6;
// multi-tile form: TP > 1 adjacent 128-pixel tiles per work unit, their MMAs interleaved into TP
// independent accumulators; a slab of TP * 128 + 2 dil rows (dil <= 8) comes as 136-row TMA boxes
constexpr int kBoxRows = 136;  // 17 KB, a multiple of 1024 bytes (the swizzle pattern)
// Tiles per work unit by epilogue, measured on 32 x 512 x 512 (ms per convolution, TP = 1 / 2 / 3):
// bias+ReLU 0.92 / 0.77 / 0.74, bias+residual+ReLU 0.95 / 0.94 / 0.97, head 0.97 / 0.82 / 0.70,
// mask 1.03 / 0.93 / 0.95, residual+mask 1.20 / 1.31 / 1.68, plain 0.98 / 0.83 / 0.73. More
// interleaved accumulators keep the tensor pipe busier; epilogues that load the residual or the
// mask per pixel are bound by those loads, and more pixels per unit lengthen them.
template <int EPI>
constexpr int tiles_per_unit() {
  return EPI == EPI_RES_MASK ? 1 : (EPI == EPI_BIAS_RES_RELU || EPI == EPI_MASK) ? 2 : 3;
}
template <int TP>
struct FwdShape {
  static constexpr int kBoxes = TP == 1 ? 1 : (TP * BM + 2 * kMaxDil + kBoxRows - 1) / kBoxRows;
  static constexpr int kStg = TP == 1 ? kStages : (TP == 2 ? 4 : 3);
  static constexpr int kStride = TP == 1 ? kSlabStride : kBoxes * kBoxRows * C * 2;
  static constexpr uint32_t kTmemCols = TP == 1 ? 128u : (TP == 2 ? 256u : 512u);  // two buffers of TP accumulators
  static constexpr int kSmem = kWBytes + kStg * kStride + 1024;
  static_assert(kSmem + 512 <= 232448, "shared memory (dynamic + about 400 bytes static)");
  static_assert(2 * TP * 64 <= (int)kTmemCols, "tensor memory");
};
constexpr int kThreads = 192;           // warp 0: TMA, warp 1: MMA + TMEM owner, warps 2-5: epilogue
constexpr unsigned long long kWaitNs = 2000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait; false after kWaitNs or once another role gave up (*abort).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort) {
  if (mbar_try(b, parity)) return true;
  const uint64_t t0 = gtimer();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try(b, parity)) return true;
    if ((i & 63u) == 0) {
      if (*abort) return false;
      if (gtimer() - t0 > kWaitNs) return false;
    }
  }
}
__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* tm, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// D[tmem] (+)= A[desc_a] x B[desc_b]^T, kind::f16, one CTA
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t desc_a, uint64_t desc_b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(desc_a), "l"(desc_b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor, 128-byte swizzle (layout type 2), sm100 version 1.
// K-major: rows of 128 B along K, 8-row groups 1024 B apart (SBO), LBO unused (1).
// MN-major: rows of 128 B hold 64 M/N elements for one K index, 8-K-row groups 1024 B apart
// (SBO), the next 64 M/N elements `lbo_bytes` further (LBO).
// The swizzle is applied to absolute shared-memory addresses (as TMA writes them), so a matrix
// may start at any row or 16-byte column of a 1024-byte-aligned tile (base offset 0).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46) | (2ull << 61);
}
// Instruction descriptor: bf16 x bf16 -> f32, M x N, majors (0 K, 1 MN).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void record(int* err, int code) {
  if (err) atomicCAS(err, 0, code);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ void unpack8(uint4 u, float (&f)[8]) {
  const __nv_bfloat162* p = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float2 t = __bfloat1622float2(p[i]);
    f[2 * i] = t.x;
    f[2 * i + 1] = t.y;
  }
}

struct FwdArgs {
  const float* bias;        // [64] or null
  const __nv_bfloat16* res; // residual / gradient added before the activation or mask
  const __nv_bfloat16* mask;// ReLU mask source (> 0 passes)
  void* out;                // bf16 [n_pix][64], or f32 [n_pix][4] (EPI_HEAD)
  int n_pix, Hp, Wp;        // padded pixel count, padded image height / width
  int dil, slab_rows;       // dilation, rows of one slab (128 + 2 dil)
  int n_tiles;
  int* err;
};

// ---------------------------------------------------------------------------------------------
// forward / dgrad: out = epilogue(conv3x3(in, weights)) over every padded pixel
// ---------------------------------------------------------------------------------------------
// TP: 128-pixel tiles per work unit (1, or 2: the pair form)
template <int EPI, int TP>
__global__ void __launch_bounds__(kThreads, 1)
    conv3x3_kernel(const __grid_constant__ CUtensorMap tm_act, const __grid_constant__ CUtensorMap tm_w, FwdArgs a) {
  using FS = FwdShape<TP>;
  constexpr int kStages = FS::kStg;
  constexpr int kSlabStride = FS::kStride;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* s_w = smem;                    // 9 taps x 8 KB
  unsigned char* s_a = smem + kWBytes;          // kStages slabs, one per dy
  __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages], w_bar, acc_full[2], acc_empty[2], done_bar;
  __shared__ uint32_t s_tmem;
  __shared__ float s_bias[C];
  __shared__ volatile int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], 1);
    }
    mbar_init(&w_bar, 1);
    for (int i = 0; i < 2; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], 128);
    }
    mbar_init(&done_bar, 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < C) s_bias[tid] = a.bias ? a.bias[tid] : 0.f;
  if (warp == 1) {  // two buffers of TP 64-column fp32 accumulators
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(FS::kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const int Wp = a.Wp;

  if (warp == 0) {
    if (lane == 0) {  // ---- TMA producer ----
      mbar_expect_tx(&w_bar, kWBytes);
      for (int t = 0; t < 9; ++t) tma_2d(s_w + t * kTapBytes, &tm_w, 0, t * C, &w_bar);
      uint32_t it = 0;
      bool ok = true;
      for (int tile = blockIdx.x; ok && tile < a.n_tiles; tile += gridDim.x) {
        const int p0 = tile * BM * TP;
        for (int r = 0; r < 3; ++r, ++it) {  // rows from p0 + dil * (dy * Wp - 1) serve the taps (dy, -1..1)
          const uint32_t st = it % kStages, ph = (it / kStages) & 1u;
          if (!mbar_wait(&empty_bar[st], ph ^ 1u, &s_abort)) {
            record(a.err, 1);
            s_abort = 1;
            ok = false;
            break;
          }
          const int dy = r - 1;
          const int y0 = p0 + a.dil * (dy * Wp - 1);
          if (TP == 1) {
            mbar_expect_tx(&full_bar[st], (uint32_t)a.slab_rows * C * 2);
            tma_2d(s_a + st * kSlabStride, &tm_act, 0, y0, &full_bar[st]);
          } else {
            mbar_expect_tx(&full_bar[st], (uint32_t)(FS::kBoxes * kBoxRows * C * 2));
            for (int b = 0; b < FS::kBoxes; ++b)
              tma_2d(s_a + st * kSlabStride + b * kBoxRows * C * 2, &tm_act, 0, y0 + b * kBoxRows, &full_bar[st]);
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {  // ---- MMA issuer ----
      constexpr uint32_t idesc = idesc_bf16(BM, C, 0, 0);
      bool ok = mbar_wait(&w_bar, 0, &s_abort);
      if (!ok) {
        record(a.err, 2);
        s_abort = 1;
      }
      uint32_t it = 0, lt = 0;
      for (int tile = blockIdx.x; ok && tile < a.n_tiles; tile += gridDim.x, ++lt) {
        const uint32_t acc = lt & 1u;
        if (!mbar_wait(&acc_empty[acc], ((lt >> 1) & 1u) ^ 1u, &s_abort)) {
          record(a.err, 3);
          s_abort = 1;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + acc * (C * TP);
        for (int r = 0; r < 3; ++r, ++it) {
          const uint32_t st = it % kStages, ph = (it / kStages) & 1u;
          if (!mbar_wait(&full_bar[st], ph, &s_abort)) {
            record(a.err, 4);
            s_abort = 1;
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t slab = smem_u32(s_a + st * kSlabStride);
#pragma unroll
          for (int c = 0; c < 3; ++c) {  // tap (dy, dx = c - 1): the slab from row c * dil on
            const uint32_t sa = slab + 128 * c * a.dil, sb = smem_u32(s_w + (3 * r + c) * kTapBytes);
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
              for (int h = 0; h < TP; ++h)  // the TP tiles' MMAs interleaved: independent accumulators
                tc_mma(d + C * h, sdesc(sa + BM * 128 * h + 32 * k, 16, 1024), sdesc(sb + 32 * k, 16, 1024), idesc,
                       (r | c | k) ? 1u : 0u);
          }
          tc_commit(&empty_bar[st]);
        }
        if (!ok) break;
        tc_commit(&acc_full[acc]);
      }
      // all MMAs issued by this thread have completed once done_bar flips
      tc_commit(&done_bar);
      if (!mbar_wait(&done_bar, 0, &s_abort)) record(a.err, 5);
    }
  } else {  // ---- epilogue: warps 2..5 own TMEM lanes 32 * (warp % 4) .. + 31 ----
    const int q = warp & 3;
    const int row = q * 32 + lane;
    uint32_t lt = 0;
    for (int tile = blockIdx.x; tile < a.n_tiles; tile += gridDim.x, ++lt) {
      const uint32_t acc = lt & 1u;
      if (!mbar_wait(&acc_full[acc], (lt >> 1) & 1u, &s_abort)) {
        record(a.err, 6);
        s_abort = 1;
        break;
      }
      tc_fence_after();
      __syncwarp();  // tcgen05.ld is warp-wide: lanes that left the last pixel early meet here
      // the whole buffer (TP accumulators) into registers, then it is released to the MMA warp
      float vv[TP][64];
      const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + acc * (C * TP);
#pragma unroll
      for (int hh = 0; hh < TP; ++hh)
#pragma unroll
        for (int j = 0; j < 4; ++j) tmem_ld16(base + C * hh + 16 * j, *reinterpret_cast<float(*)[16]>(&vv[hh][16 * j]));
      tmem_wait_ld();
      tc_fence_before();
      mbar_arrive(&acc_empty[acc]);
#pragma unroll
      for (int hh = 0; hh < TP; ++hh) {
        const float (&v)[64] = vv[hh];
        do {  // one pixel; lanes that have nothing to write leave through break
          const int p = (tile * TP + hh) * BM + row;
          if (p >= a.n_pix) break;
          const int xx = p % Wp, yy = (p / Wp) % a.Hp;
          const bool interior = xx >= kPad && xx < Wp - kPad && yy >= kPad && yy < a.Hp - kPad;
          if (EPI == EPI_HEAD) {
            float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
            if (interior) o = make_float4(v[0] + s_bias[0], v[1] + s_bias[1], v[2] + s_bias[2], v[3] + s_bias[3]);
            reinterpret_cast<float4*>(a.out)[p] = o;
            break;
          }
          uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(a.out) + (size_t)p * C);
          if (!interior) {
#pragma unroll
            for (int j = 0; j < 8; ++j) dst[j] = make_uint4(0, 0, 0, 0);
            break;
          }
          const uint4* rsrc = (EPI == EPI_BIAS_RES_RELU || EPI == EPI_RES_MASK)
                                  ? reinterpret_cast<const uint4*>(a.res + (size_t)p * C)
                                  : nullptr;
          const uint4* msrc = (EPI == EPI_MASK || EPI == EPI_RES_MASK) ? reinterpret_cast<const uint4*>(a.mask + (size_t)p * C)
                                                                        : nullptr;
          // every load of the pixel before its first store: the stores may alias the sources as far
          // as the compiler knows, so loads left in the loop below would each wait for the one before
          uint4 rv[8], mv[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (rsrc) rv[j] = rsrc[j];
            if (msrc) mv[j] = msrc[j];
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            float x[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) x[i] = v[8 * j + i];
            if (EPI == EPI_BIAS_RELU || EPI == EPI_BIAS_RES_RELU) {
#pragma unroll
              for (int i = 0; i < 8; ++i) x[i] += s_bias[8 * j + i];
            }
            if (rsrc) {
              float r[8];
              unpack8(rv[j], r);
#pragma unroll
              for (int i = 0; i < 8; ++i) x[i] += r[i];
            }
            if (EPI == EPI_BIAS_RELU || EPI == EPI_BIAS_RES_RELU) {
#pragma unroll
              for (int i = 0; i < 8; ++i) x[i] = fmaxf(x[i], 0.f);
            }
            if (msrc) {
              float m[8];
              unpack8(mv[j], m);
#pragma unroll
              for (int i = 0; i < 8; ++i) x[i] = m[i] > 0.f ? x[i] : 0.f;
            }
            dst[j] = make_uint4(pack_bf16(x[0], x[1]), pack_bf16(x[2], x[3]), pack_bf16(x[4], x[5]), pack_bf16(x[6], x[7]));
          }
        } while (0);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(FS::kTmemCols) : "memory");
  }
}

// ---------------------------------------------------------------------------------------------
// wgrad: part[cta][tap][ci][co] = sum over this CTA's pixels of X[p + off(tap)][ci] * dY[p][co]
// ---------------------------------------------------------------------------------------------
constexpr int kWgChunk = 64;                      // pixels per K step block
constexpr int kWgAtom = kWgChunk * C * 2;         // 8 KB
constexpr int kWgStageBytes = 11 * kWgAtom;       // 10 X atoms (tap 8 twice) + dY
constexpr int kWgStages = 2;

struct WgArgs {
  float* part;  // [gridDim.x][9][64][64]
  int n_pix, Wp, dil;
  int n_chunks;
  int* err;
};

__global__ void __launch_bounds__(kThreads, 1)
    conv3x3_wgrad_kernel(const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_dy, WgArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full_bar[kWgStages], empty_bar[kWgStages], acc_full, done_bar;
  __shared__ uint32_t s_tmem;
  __shared__ volatile int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int c0 = (int)((long long)a.n_chunks * blockIdx.x / gridDim.x);
  const int c1 = (int)((long long)a.n_chunks * (blockIdx.x + 1) / gridDim.x);
  if (tid == 0) {
    for (int i = 0; i < kWgStages; ++i) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], 1);
    }
    mbar_init(&acc_full, 1);
    mbar_init(&done_bar, 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {  // five 64-column accumulators (taps 0-1, 2-3, 4-5, 6-7, 8-8)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(512u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  if (warp == 0) {
    if (lane == 0) {
      uint32_t it = 0;
      for (int ch = c0; ch < c1; ++ch, ++it) {
        const uint32_t st = it % kWgStages, ph = (it / kWgStages) & 1u;
        if (!mbar_wait(&empty_bar[st], ph ^ 1u, &s_abort)) {
          record(a.err, 11);
          s_abort = 1;
          break;
        }
        unsigned char* s = smem + st * kWgStageBytes;
        const int p0 = ch * kWgChunk;
        mbar_expect_tx(&full_bar[st], kWgStageBytes);
        for (int j = 0; j < 10; ++j) {
          const int t = j < 9 ? j : 8;
          const int dy = t / 3 - 1, dx = t % 3 - 1;
          tma_2d(s + j * kWgAtom, &tm_x, 0, p0 + a.dil * (dy * a.Wp + dx), &full_bar[st]);
        }
        tma_2d(s + 10 * kWgAtom, &tm_dy, 0, p0, &full_bar[st]);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = idesc_bf16(128, C, 1, 1);
      uint32_t it = 0;
      bool ok = true;
      for (int ch = c0; ch < c1; ++ch, ++it) {
        const uint32_t st = it % kWgStages, ph = (it / kWgStages) & 1u;
        if (!mbar_wait(&full_bar[st], ph, &s_abort)) {
          record(a.err, 12);
          s_abort = 1;
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t s = smem_u32(smem + st * kWgStageBytes);
        const uint32_t sb = s + 10 * kWgAtom;
#pragma unroll
        for (int m = 0; m < 5; ++m) {
#pragma unroll
          for (int k = 0; k < 4; ++k)  // 16 pixels (two 8-row groups) per MMA
            tc_mma(tmem + m * C, sdesc(s + 2 * m * kWgAtom + 2048 * k, kWgAtom, 1024), sdesc(sb + 2048 * k, kWgAtom, 1024),
                   idesc, (ch > c0 || k > 0) ? 1u : 0u);
        }
        tc_commit(&empty_bar[st]);
      }
      if (ok) tc_commit(&acc_full);
      tc_commit(&done_bar);
      if (!mbar_wait(&done_bar, 0, &s_abort)) record(a.err, 13);
    }
  } else {
    const int q = warp & 3;
    const int row = q * 32 + lane;  // accumulator lane: (tap 2m + row / 64, ci = row % 64)
    float* part = a.part + (size_t)blockIdx.x * 9 * C * C;
    const bool have = c1 > c0;
    bool ok = true;
    if (have) {
      ok = mbar_wait(&acc_full, 0, &s_abort);
      if (!ok) {
        record(a.err, 14);
        s_abort = 1;
      }
    }
    tc_fence_after();
    for (int m = 0; m < 5; ++m) {
      const int t = 2 * m + row / 64;
      if (t > 8) continue;
      float* dst = part + ((size_t)t * C + (row % 64)) * C;
      if (!have || !ok) {
        for (int i = 0; i < C; ++i) dst[i] = 0.f;
        continue;
      }
      const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + m * C;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        float v[16];
        tmem_ld16(base + 16 * c, v);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; i += 4) *reinterpret_cast<float4*>(dst + 16 * c + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
  }
}

// dW[tap][co][ci] = sum over CTAs of part[cta][tap][ci][co]
__global__ void wgrad_reduce_kernel(const float* __restrict__ part, int n_parts, float* __restrict__ dw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // over tap, co, ci
  if (i >= 9 * C * C) return;
  const int t = i / (C * C), co = (i / C) % C, ci = i % C;
  float s = 0.f;
  for (int b = 0; b < n_parts; ++b) s += part[((size_t)b * 9 * C + (size_t)t * C + ci) * C + co];
  dw[i] = s;
}

int encode_act_map(CUtensorMap* tm, const void* base, int rows, int box_rows) {
  cuuint64_t dims[2] = {(cuuint64_t)C, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)C * 2};
  cuuint32_t box[2] = {(cuuint32_t)C, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  if (!drv::TensorMapEncodeTiled) return (int)CUDA_ERROR_NOT_INITIALIZED;
  return (int)drv::TensorMapEncodeTiled(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides,
                                        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
}

int g_sms = 0;

}  // namespace

int conv_grid() {
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
  }
  return g_sms;
}

cudaError_t conv3x3(const ConvShape& s, const __nv_bfloat16* in, const __nv_bfloat16* w, const float* bias,
                    const __nv_bfloat16* res, const __nv_bfloat16* mask, void* out, int epi, int* err,
                    cudaStream_t stream) {
  std::string derr;
  if (!drv::load(&derr)) return cudaErrorInitializationError;
  if (s.dil < 1 || s.dil > kMaxDil) return cudaErrorInvalidValue;
  const int n_pix = s.N * (s.H + 2 * kPad) * (s.W + 2 * kPad);
  const int slab_rows = BM + 2 * s.dil;
  CUtensorMap tm_a, tm_w;
  if (encode_act_map(&tm_w, w, 9 * C, C)) return cudaErrorInvalidValue;
  FwdArgs a;
  a.bias = bias;
  a.res = res;
  a.mask = mask;
  a.out = out;
  a.n_pix = n_pix;
  a.Hp = s.H + 2 * kPad;
  a.Wp = s.W + 2 * kPad;
  a.dil = s.dil;
  a.slab_rows = slab_rows;
  a.err = err;
#define FIP_SG_LAUNCH(E)                                                                                  \
  case E: {                                                                                                \
    constexpr int TP = tiles_per_unit<E>();                                                                \
    if (encode_act_map(&tm_a, in, n_pix, TP == 1 ? slab_rows : kBoxRows)) return cudaErrorInvalidValue;   \
    a.n_tiles = (n_pix + BM * TP - 1) / (BM * TP); /* work units of TP tiles */                           \
    const int smem = FwdShape<TP>::kSmem;                                                                  \
    const int grid = std::min(conv_grid(), a.n_tiles);                                                     \
    static std::atomic<uint64_t> cfg{0};                                                                   \
    const cudaError_t e = ensure_dynamic_smem(conv3x3_kernel<E, TP>, smem, cfg);                          \
    if (e != cudaSuccess) return e;                                                                        \
    conv3x3_kernel<E, TP><<<grid, kThreads, smem, stream>>>(tm_a, tm_w, a);                                \
    break;                                                                                                 \
  }
  switch (epi) {
    FIP_SG_LAUNCH(EPI_BIAS_RELU)
    FIP_SG_LAUNCH(EPI_BIAS_RES_RELU)
    FIP_SG_LAUNCH(EPI_HEAD)
    FIP_SG_LAUNCH(EPI_MASK)
    FIP_SG_LAUNCH(EPI_RES_MASK)
    FIP_SG_LAUNCH(EPI_PLAIN)
    default: return cudaErrorInvalidValue;
  }
#undef FIP_SG_LAUNCH
  return cudaGetLastError();
}

size_t wgrad_scratch_floats() { return (size_t)conv_grid() * 9 * C * C; }

cudaError_t conv3x3_wgrad(const ConvShape& s, const __nv_bfloat16* x, const __nv_bfloat16* dy, float* part, float* dw,
                          int* err, cudaStream_t stream) {
  std::string derr;
  if (!drv::load(&derr)) return cudaErrorInitializationError;
  if (s.dil < 1 || s.dil > kMaxDil) return cudaErrorInvalidValue;
  const int n_pix = s.N * (s.H + 2 * kPad) * (s.W + 2 * kPad);
  CUtensorMap tm_x, tm_dy;
  if (encode_act_map(&tm_x, x, n_pix, kWgChunk) || encode_act_map(&tm_dy, dy, n_pix, kWgChunk)) return cudaErrorInvalidValue;
  WgArgs a;
  a.part = part;
  a.n_pix = n_pix;
  a.Wp = s.W + 2 * kPad;
  a.dil = s.dil;
  a.n_chunks = (n_pix + kWgChunk - 1) / kWgChunk;
  a.err = err;
  const int smem = kWgStages * kWgStageBytes + 1024;
  static std::atomic<uint64_t> cfg{0};
  const cudaError_t e = ensure_dynamic_smem(conv3x3_wgrad_kernel, smem, cfg);
  if (e != cudaSuccess) return e;
  const int grid = conv_grid();
  conv3x3_wgrad_kernel<<<grid, kThreads, smem, stream>>>(tm_x, tm_dy, a);
  wgrad_reduce_kernel<<<(9 * C * C + 255) / 256, 256, 0, stream>>>(part, grid, dw);
  return cudaGetLastError();
}

}  // namespace sg
}  // namespace fip
