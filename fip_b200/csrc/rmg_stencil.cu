// sm_100a kernels of the slim shallow-water step (fip's rmg solver).
//
// rmg_step_kernel restates one launch of the reference's rmg_kernel (src/kernels.cu:264-438)
// with the wet/dry mask replaced by an exact active-tile list:
//   * momentum fluxes fx/fy/gx/gy, the semi-implicit Strickler update of qx/qy with the flux
//     limiter (compute_rmg_qx/qy, src/kernels.cu:75-127), the boundary-face holds (:373-376),
//     continuity (:381), the three write sets (:383-406) and the CFL fold (:392-400), all in
//     FP32 with the same expression trees (compiled with -use_fast_math like the reference, so
//     sqrtf/powf/division are the same approximations);
//   * the domain is cut into tiles of 480 columns x 32 rows. A CTA has four consumer warps
//     (each thread owns 4 adjacent columns, a warp 128 columns of which the 120 inner ones are
//     stored) and one producer warp that streams rows of h/qx/qy/terrain/kSt into a ring of 6
//     rows (7 without kSt) in shared memory with TMA (cp.async.bulk.tensor; each CTA loads its own rows).
//     Consumers march north row by row over the staged rows r-1 .. r+2, exchange east/west
//     neighbours with warp shuffles and do the arithmetic on FP32x2 pairs of columns;
//   * work = the concatenation of the active tiles' rows (strip-major), split evenly over the
//     persistent CTAs, so vertically adjacent active tiles are marched without re-staging;
//   * each CTA folds its CFL minimum into ctl->cfl_bits with one atomicMin per warp, flags the
//     tiles whose new state has a nonzero cell (and whether one lies in the tile's first or last
//     columns: FIP_NZ_*), and (every hmax_every iterations) folds hmax.
// Every wait on an mbarrier is bounded (2 s of %globaltimer); on expiry the kernel records
// FIP_DEVERR_* in ctl->error and returns after draining its own copies.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "drv.h"
#include "fip_ctl.h"
#include "rmg_stencil.h"
#include "smem_attr.h"

namespace fip {

namespace {

constexpr float kDH = 0.01f;         // src/kernels.cu:23
constexpr float kEPS = 10e-7f;       // src/kernels.cu:24 (EPS_TROCKEN)
constexpr float kG = 9.81f;          // src/simdata.h:358
constexpr int kNSlotKvar = 6;
constexpr int kNSlotUniform = 7;
constexpr int kNSlotMax = 10;  // ring depth in rows: 6 with the kSt field, else 7 (leaves L1 room beside 3 CTAs)
// two-warp tiles (240 columns, used by ensembles when the autotuner picks them): 5 CTAs per SM,
// deeper rings in their smaller rows
constexpr int kNSlotKvar2 = 8;
constexpr int kNSlotUniform2 = 10;
constexpr int kMinCtas2 = 5;
constexpr int kMinCtas4 = 3;  // resident CTAs per SM (128 registers per thread)
// narrow threads (2 columns each, tiles of 240 columns): half the registers, more CTAs per SM
constexpr int kMinCtasNarrow = 4;  // 95 registers, no spills (5 per SM spill 128 bytes)
constexpr int kNSlotKvarNarrow = 7;
constexpr int kNSlotUniformNarrow = 8;
constexpr int kMaxChunks = 256;
constexpr unsigned long long kWaitNs = 2000000000ull;
constexpr int kNzBand = 4;  // edge-band width of the tile flags a state's scan sets (>= 2, the stencil's reach)

enum { F_H = 0, F_QX = 1, F_QY = 2, F_S = 3, F_K = 4 };

struct StepArgs {
  float* h[2];
  float* qx[2];
  float* qy[2];
  float* hmax;
  FipCtl* ctl;
  const int* list[2];
  const int* chunk_cnt[2];
  unsigned char* nz[2];
  int W, H, pitch;
  int n_sx, n_ty, n_tiles, n_chunks;
  float dx, kst_fixed, no_value;
  // ensembles only: member table, per-member control, member count, tile rows
  const FipEnsMember* members;
  FipEnsCtl* mctl;
  int n_members;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase of `parity` to complete; false after kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63u) == 0 && globaltimer() - t0 > kWaitNs) return false;
  }
}
__device__ __forceinline__ void tma_row(void* dst, const CUtensorMap* tm, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void record_error(FipCtl* ctl, int code) { atomicCAS(&ctl->error, 0, code); }
// Shared-memory values read where they are used: a volatile load is neither hoisted out of the
// row loop nor merged with an earlier one, so the value holds no register between its uses.
__device__ __forceinline__ int lds_at_use(const int* p) { return *reinterpret_cast<const volatile int*>(p); }
__device__ __forceinline__ float ldsf_at_use(const float* p) { return *reinterpret_cast<const volatile float*>(p); }
__device__ __forceinline__ float2 lds2_at_use(const float* p) {
  const volatile float2* q = reinterpret_cast<const volatile float2*>(p);
  return make_float2(q->x, q->y);
}

// FP32x2 arithmetic (sm_100 packed add/mul/fma): a thread owns NC adjacent columns (4, or 2 in
// the narrow-thread form) and applies the same operation to all of them, so each pair of columns
// goes through one instruction. Each component is rounded to nearest with denormals flushed,
// exactly like the scalar operations under -use_fast_math, so every column gets the scalar result.
__device__ __forceinline__ uint64_t pk2(float a, float b) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void un2(uint64_t v, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t mul2(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t r;
  asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
// d = a op b over the N columns; a float2 operand is the same pair for every pair of columns
#define FIP_V2(name, op)                                                                                  \
  template <int N>                                                                                        \
  __device__ __forceinline__ void name(float (&d)[N], const float (&a)[N], const float (&b)[N]) {         \
    _Pragma("unroll") for (int i = 0; i < N; i += 2) un2(op(pk2(a[i], a[i + 1]), pk2(b[i], b[i + 1])), d[i], d[i + 1]); \
  }                                                                                                       \
  template <int N>                                                                                        \
  __device__ __forceinline__ void name(float (&d)[N], const float (&a)[N], float2 b) {                    \
    const uint64_t bb = pk2(b.x, b.y);                                                                    \
    _Pragma("unroll") for (int i = 0; i < N; i += 2) un2(op(pk2(a[i], a[i + 1]), bb), d[i], d[i + 1]);   \
  }                                                                                                       \
  template <int N>                                                                                        \
  __device__ __forceinline__ void name(float (&d)[N], float2 a, const float (&b)[N]) {                    \
    const uint64_t aa = pk2(a.x, a.y);                                                                    \
    _Pragma("unroll") for (int i = 0; i < N; i += 2) un2(op(aa, pk2(b[i], b[i + 1])), d[i], d[i + 1]);   \
  }
FIP_V2(vadd, add2)
FIP_V2(vsub, sub2)
FIP_V2(vmul, mul2)
#undef FIP_V2
// d = a * b + c
template <int N>
__device__ __forceinline__ void vfma(float (&d)[N], const float (&a)[N], const float (&b)[N], const float (&c)[N]) {
#pragma unroll
  for (int i = 0; i < N; i += 2) un2(fma2(pk2(a[i], a[i + 1]), pk2(b[i], b[i + 1]), pk2(c[i], c[i + 1])), d[i], d[i + 1]);
}
template <int N>
__device__ __forceinline__ void vfma(float (&d)[N], const float (&a)[N], float2 b, const float (&c)[N]) {
  const uint64_t bb = pk2(b.x, b.y);
#pragma unroll
  for (int i = 0; i < N; i += 2) un2(fma2(pk2(a[i], a[i + 1]), bb, pk2(c[i], c[i + 1])), d[i], d[i + 1]);
}
template <int N>
__device__ __forceinline__ void vfma(float (&d)[N], float2 a, const float (&b)[N], const float (&c)[N]) {
  const uint64_t aa = pk2(a.x, a.y);
#pragma unroll
  for (int i = 0; i < N; i += 2) un2(fma2(aa, pk2(b[i], b[i + 1]), pk2(c[i], c[i + 1])), d[i], d[i + 1]);
}

__device__ __forceinline__ bool store_row_flag(int r, int ra) { return r >= ra; }

// OR `bits` into the tile flag byte at p: an atomic OR on the aligned 32-bit word that holds it
// (flag arrays are allocated in whole words), so that warps setting different bits of one tile
// do not overwrite each other
__device__ __forceinline__ void tile_flag_or(unsigned char* p, unsigned bits) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  atomicOr(reinterpret_cast<unsigned*>(a & ~static_cast<uintptr_t>(3)), bits << (8u * static_cast<unsigned>(a & 3)));
}

// max(a, b, c) as the reference nests it (max(max(DH, h_i), h_east))
__device__ __forceinline__ float fmax3(float a, float b, float c) { return fmaxf(fmaxf(a, b), c); }
// (1 / a)^2.33 of the friction factor, as the reference writes it (powf of the reciprocal)
__device__ __forceinline__ float pow_inv(float a) { return powf(1.f / a, 2.33f); }

// The NC staged values of `field` at staged column `col` of a ring slot (one 16- or 8-byte
// shared-memory load)
template <int NC, int FB>
__device__ __forceinline__ void ldsv(float (&v)[NC], const unsigned char* slot, int field, int col) {
  if constexpr (NC == 4) {
    const float4 t = *reinterpret_cast<const float4*>(slot + field * FB + col * 4);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  } else {
    const float2 t = *reinterpret_cast<const float2*>(slot + field * FB + col * 4);
    v[0] = t.x;
    v[1] = t.y;
  }
}
// NC values to global memory in one 16- or 8-byte store (p aligned to NC floats)
template <int NC>
__device__ __forceinline__ void stgv(float* p, const float (&v)[NC]) {
  if constexpr (NC == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  else *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
}
// hmax = max(hmax, h) over NC cells (p aligned to NC floats)
template <int NC>
__device__ __forceinline__ void hmax_foldv(float* p, const float (&h)[NC]) {
  if constexpr (NC == 4) {
    float4* q = reinterpret_cast<float4*>(p);
    float4 m = *q;
    m.x = fmaxf(m.x, h[0]);
    m.y = fmaxf(m.y, h[1]);
    m.z = fmaxf(m.z, h[2]);
    m.w = fmaxf(m.w, h[3]);
    *q = m;
  } else {
    float2* q = reinterpret_cast<float2*>(p);
    float2 m = *q;
    m.x = fmaxf(m.x, h[0]);
    m.y = fmaxf(m.y, h[1]);
    *q = m;
  }
}

// Walk of a CTA's share of the active-tile row stream: maximal runs of rows that are
// contiguous in one strip (vertically adjacent active tiles are one run).
struct Walk {
  long long pos, end;
};

__device__ __forceinline__ int list_entry(const int* list, const int* s_prefix, int n_chunks, long long p) {
  int c = 0;
  while (c + 1 < n_chunks && s_prefix[c + 1] <= p) ++c;
  return list[c * FIP_PLAN_CHUNK + (int)(p - s_prefix[c])];
}

__device__ __forceinline__ bool next_run(Walk& w, const int* list, const int* s_prefix, int n_chunks, int n_ty, int H,
                                         int* strip, int* ra, int* rb) {
  while (w.pos < w.end) {
    long long p = w.pos / FIP_TILE_ROWS;
    const int off = (int)(w.pos - p * FIP_TILE_ROWS);
    int tile = list_entry(list, s_prefix, n_chunks, p);
    const int s = tile / n_ty;
    const int ty0 = tile - s * n_ty;
    int ty = ty0;
    // extend over the following list entries while they are the next tile up the same strip
    while ((p + 1) * FIP_TILE_ROWS < w.end && ty + 1 < n_ty &&
           list_entry(list, s_prefix, n_chunks, p + 1) == tile + 1) {
      ++p;
      ++tile;
      ++ty;
    }
    const long long stop = (p + 1) * FIP_TILE_ROWS < w.end ? (p + 1) * FIP_TILE_ROWS : w.end;
    const int r_a = ty0 * FIP_TILE_ROWS + off;
    int r_b = ty * FIP_TILE_ROWS + (int)(stop - p * FIP_TILE_ROWS);
    w.pos = stop;
    if (r_b > H) r_b = H;
    if (r_a >= r_b) continue;  // rows entirely beyond the grid
    *strip = s;
    *ra = r_a;
    *rb = r_b;
    return true;
  }
  return false;
}

// next_run over an ensemble's concatenated tile list: the member of the run's tiles comes from
// the members' first tile indices (s_tbase, n_members + 1 entries); rows are the member's own.
__device__ __forceinline__ bool next_run_ens(Walk& w, const int* list, const int* s_prefix, int n_chunks, int TR,
                                             const FipEnsMember* mem, const int* s_tbase, int n_members, int* member,
                                             int* strip, int* ra, int* rb) {
  while (w.pos < w.end) {
    long long p = w.pos / TR;
    const int off = (int)(w.pos - p * TR);
    int tile = list_entry(list, s_prefix, n_chunks, p);
    int lo = 0, hi = n_members;  // s_tbase[lo] <= tile < s_tbase[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (s_tbase[mid] <= tile) lo = mid;
      else hi = mid;
    }
    const int n_ty = mem[lo].n_ty, H = mem[lo].H;
    const int local = tile - s_tbase[lo];
    const int s = local / n_ty;
    const int ty0 = local - s * n_ty;
    int ty = ty0;
    while ((p + 1) * TR < w.end && ty + 1 < n_ty && list_entry(list, s_prefix, n_chunks, p + 1) == tile + 1) {
      ++p;
      ++tile;
      ++ty;
    }
    const long long stop = (p + 1) * TR < w.end ? (p + 1) * TR : w.end;
    const int r_a = ty0 * TR + off;
    int r_b = ty * TR + (int)(stop - p * TR);
    w.pos = stop;
    if (r_b > H) r_b = H;
    if (r_a >= r_b) continue;
    *member = lo;
    *strip = s;
    *ra = r_a;
    *rb = r_b;
    return true;
  }
  return false;
}

// KW consumer warps per CTA, NC columns per thread (tiles of 30 * NC * KW columns, TRT rows); ENS:
// the grid is a packed ensemble (member table in the arguments, per-member dt, rows, sizes and CFL
// slots). The tile height is a template argument so that the row-to-tile arithmetic compiles to
// shifts and masks. NC = 2 halves the registers a thread holds, so more CTAs fit on an SM.
template <int NC, int KW>
struct StepShape {
  static_assert(NC == 2 || NC == 4, "4 or 2 columns per thread");
  static_assert(KW == 2 || KW == 4, "tiles of 2 or 4 consumer warps");
  static constexpr int kCols = 32 * NC * KW;       // staged columns per row and field
  static constexpr int kFB = kCols * 4;            // bytes of one staged row of one field
  static constexpr int kBoxes = kCols / 256;       // TMA boxes of 256 floats per staged row
  static constexpr int TC = 30 * NC * KW;          // tile columns (lanes 1..30 of each warp store)
  // staged column of the tile's column 0: lanes read [X0 - NC, X0 + TC + NC) of the staged row
  // (the TMA x coordinate, column 0 - X0, stays a multiple of 4 floats)
  static constexpr int X0 = (NC == 4 && KW == 4) ? FIP_SMEM_X0 : 4;
  static constexpr int kMinCtas = NC == 4 ? (KW == 4 ? kMinCtas4 : kMinCtas2) : kMinCtasNarrow;
  // ring depth in rows with and without the kSt field
  static constexpr int kNSlotK = NC == 4 ? (KW == 4 ? kNSlotKvar : kNSlotKvar2) : kNSlotKvarNarrow;
  static constexpr int kNSlotU = NC == 4 ? (KW == 4 ? kNSlotUniform : kNSlotUniform2) : kNSlotUniformNarrow;
  static_assert(kBoxes >= 1 && kCols % 256 == 0, "staged rows are whole 256-float TMA boxes");
  static_assert(X0 >= NC && X0 + TC + NC <= kCols && X0 % 4 == 0, "staged window");
};

template <bool KVAR, bool ENS, int KW, int TRT, int NC>
__global__ void __launch_bounds__((KW + 1) * 32, StepShape<NC, KW>::kMinCtas)
    rmg_step_kernel(const __grid_constant__ CUtensorMap tm_h0, const __grid_constant__ CUtensorMap tm_h1,
                    const __grid_constant__ CUtensorMap tm_qx0, const __grid_constant__ CUtensorMap tm_qx1,
                    const __grid_constant__ CUtensorMap tm_qy0, const __grid_constant__ CUtensorMap tm_qy1,
                    const __grid_constant__ CUtensorMap tm_s, const __grid_constant__ CUtensorMap tm_k,
                    const StepArgs a) {
  using S = StepShape<NC, KW>;
  constexpr int NF = KVAR ? 5 : 4;
  constexpr int kNSlot = KVAR ? S::kNSlotK : S::kNSlotU;
  constexpr int kFB = S::kFB;
  constexpr int kSlotBytes = NF * kFB;
  constexpr int TC = S::TC;
  constexpr int X0 = S::X0;
  constexpr int FULL = (1 << NC) - 1;  // all NC cells of a thread
  static_assert(kNSlot <= kNSlotMax, "ring depth");
  extern __shared__ __align__(1024) unsigned char smem_dyn[];
  __shared__ __align__(8) uint64_t full_bar[kNSlotMax];
  __shared__ __align__(8) uint64_t empty_bar[kNSlotMax];
  __shared__ int s_prefix[kMaxChunks + 1];
  __shared__ int s_hdr[6];
  __shared__ int s_tbase[ENS ? FIP_ENS_MAX_MEMBERS + 1 : 1];
  // ensemble: the current member's H, row offset, tile-flag base, tile rows, no_value, dx and
  // index per consumer warp, read at their few uses so that they hold no registers through the
  // row loop
  __shared__ int s_msc[ENS ? KW : 1][7];
  // ensemble: broadcast operands of the member's packed arithmetic (dt / dx dependent), the same way
  __shared__ __align__(16) float s_mcf[ENS ? KW : 1][12];

  // 1024-byte aligned ring, addressed from the shared array itself so that its loads compile to
  // shared-memory loads (an integer round trip of the address would make them generic loads)
  unsigned char* ring = smem_dyn + ((1024u - (smem_u32(smem_dyn) & 1023u)) & 1023u);
  FipCtl* ctl = a.ctl;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    s_hdr[0] = *((volatile int*)&ctl->stop);
    s_hdr[1] = ctl->parity;
    s_hdr[2] = ctl->iteration;
    s_hdr[3] = __float_as_int(ctl->dt);
    s_hdr[4] = (ctl->hmax_every > 0 && ctl->iteration > 0 && ctl->iteration % ctl->hmax_every == 0) ? 1 : 0;
    s_hdr[5] = ENS ? 0 : ctl->hmax_full;  // ensembles fold every tile (force_all) instead
    for (int i = 0; i < kNSlot; ++i) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], KW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (ENS) {
    for (int i = tid; i <= a.n_members; i += blockDim.x)
      s_tbase[i] = i < a.n_members ? a.members[i].tile_base : a.n_tiles;
  }
  if (tid < 32) {  // prefix over the chunk counts of this step's plan
    const int* cnt = a.chunk_cnt[(ctl->iteration) & 1];
    if (lane == 0) {
      int acc = 0;
      for (int c = 0; c < a.n_chunks; ++c) {
        s_prefix[c] = acc;
        acc += cnt[c];
      }
      s_prefix[a.n_chunks] = acc;
    }
  }
  __syncthreads();
  if (s_hdr[0]) return;

  const int par = s_hdr[1];
  const int it = s_hdr[2];
  const float dt = __int_as_float(s_hdr[3]);
  const bool fold = s_hdr[4] != 0;
  const int* list = a.list[it & 1];
  constexpr int TR = TRT;
  static_assert(TR == 16 || TR == 32 || TR == 64, "tile rows");
  const long long total = (long long)s_prefix[a.n_chunks] * TR;
  const long long G = gridDim.x;
  Walk walk0;
  walk0.pos = total * blockIdx.x / G;
  walk0.end = total * (blockIdx.x + 1) / G;

  if (warp == KW) {
    // ---------------- producer: one elected thread streams rows with TMA ----------------
    if (lane == 0) {
      const CUtensorMap* th = par ? &tm_h1 : &tm_h0;
      const CUtensorMap* tqx = par ? &tm_qx1 : &tm_qx0;
      const CUtensorMap* tqy = par ? &tm_qy1 : &tm_qy0;
      Walk w = walk0;
      uint32_t seq = 0;
      bool ok = true;
      int s, ra, rb, m = 0;
      // test hook (fip_inject_wait_timeout): the first row is never staged, so this CTA's waits
      // for it run out and report FIP_DEVERR_* instead of hanging
      bool skip_first = false;
      if (blockIdx.x == 0 && ctl->inject) {
        skip_first = true;
        ctl->inject = 0;
      }
      while (ok && (ENS ? next_run_ens(w, list, s_prefix, a.n_chunks, TR, a.members, s_tbase, a.n_members, &m, &s,
                                       &ra, &rb)
                        : next_run(w, list, s_prefix, a.n_chunks, a.n_ty, a.H, &s, &ra, &rb))) {
        const int x0 = s * TC - X0;
        const int y0 = ENS ? a.members[m].row_off : 0;
        for (int j = ra - 2; j <= rb + 1; ++j, ++seq) {
          const uint32_t slot = seq % kNSlot;
          const uint32_t ph = (seq / kNSlot) & 1u;
          if (!mbar_wait(&empty_bar[slot], ph ^ 1u)) {
            record_error(ctl, FIP_DEVERR_WAIT_EMPTY);
            ok = false;
            break;
          }
          if (skip_first && seq == 0) continue;
          unsigned char* dst = ring + slot * kSlotBytes;
          mbar_arrive_expect_tx(&full_bar[slot], kSlotBytes);
          const int y = y0 + j;
#pragma unroll
          for (int b = 0; b < S::kBoxes; ++b) {
            tma_row(dst + F_H * kFB + 1024 * b, th, x0 + 256 * b, y, &full_bar[slot]);
            tma_row(dst + F_QX * kFB + 1024 * b, tqx, x0 + 256 * b, y, &full_bar[slot]);
            tma_row(dst + F_QY * kFB + 1024 * b, tqy, x0 + 256 * b, y, &full_bar[slot]);
            tma_row(dst + F_S * kFB + 1024 * b, &tm_s, x0 + 256 * b, y, &full_bar[slot]);
            if (KVAR) tma_row(dst + F_K * kFB + 1024 * b, &tm_k, x0 + 256 * b, y, &full_bar[slot]);
          }
        }
      }
      // drain: never leave the CTA with copies in flight into its shared memory
      const uint32_t n_in_flight = seq < (uint32_t)kNSlot ? seq : (uint32_t)kNSlot;
      for (uint32_t i = 0; i < n_in_flight; ++i) {
        const uint32_t q = seq - 1 - i;
        if (skip_first && q == 0) continue;  // never issued
        if (!mbar_wait(&full_bar[q % kNSlot], (q / kNSlot) & 1u)) {
          record_error(ctl, FIP_DEVERR_WAIT_DRAIN);
          break;
        }
      }
    }
    return;
  }

  // ---------------- consumers ----------------
  // per-scenario scalars: fixed for a single grid, set at every run for an ensemble member
  float dx = a.dx, dtm = dt, kstf = a.kst_fixed, nv = a.no_value;
  int W = a.W, H = a.H, row0 = 0, tbase = 0, nty = a.n_ty;
  const int pitch = a.pitch;
  float dx_inv, dt_inv, fric_u, dtg, dtdx;
  float2 c_dti, c_dx, c_dxi, c_ndxi, c_dt, c_ndtdx;
  auto set_scalars = [&]() {
    dx_inv = 1.f / dx;  // in-kernel, as the reference (:276-277)
    dt_inv = 1.f / dtm;
    fric_u = dtm * kG / (kstf * kstf);  // uniform kSt: dt * G / (kSt * kSt)
    dtg = dtm * kG;                     // kSt_var: (dt * G) / (kSt * kSt)
    // broadcast operands of the packed arithmetic
    c_dti = make_float2(dt_inv, dt_inv);
    c_dx = make_float2(dx, dx);
    c_dxi = make_float2(dx_inv, dx_inv);
    c_ndxi = make_float2(-dx_inv, -dx_inv);
    c_dt = make_float2(dtm, dtm);
    dtdx = dtm * dx_inv;  // dt * dx_inv of the continuity update (:381), left to right
    c_ndtdx = make_float2(-dtdx, -dtdx);
  };
  set_scalars();
  const int scol = X0 - NC + 30 * NC * warp + NC * lane;  // staged column of k = 0
  const bool out_lane = (lane >= 1 && lane <= 30);
  float* const h_out = a.h[par ^ 1];
  float* const qx_out = a.qx[par ^ 1];
  float* const qy_out = a.qy[par ^ 1];
  const float* const h_in = a.h[par];
  unsigned char* const nzs = a.nz[it & 1];
  const float2 c_q = make_float2(0.25f, 0.25f), c_h = make_float2(0.5f, 0.5f), c_one = make_float2(1.f, 1.f);
  const float2 c_g = make_float2(kG, kG), c_zero = make_float2(0.f, 0.f);
  constexpr float kHG = 0.5f * kG;  // the reference's 0.5f * kG prefix, folded at compile time
  const float2 c_hg = make_float2(kHG, kHG), c_nhg = make_float2(-kHG, -kHG);

  // CFL: dx / (sqrt(G h') + max |u|) is monotone in its denominator, so the minimum over the cells
  // is dx over the largest denominator; the division happens once per warp
  float den_max = 0.0f;
  unsigned expacc = 0u;  // largest exponent field of a computed depth
  uint32_t seq = 0;
  Walk w = walk0;
  int s, ra, rb, m = 0;
  while (ENS ? next_run_ens(w, list, s_prefix, a.n_chunks, TR, a.members, s_tbase, a.n_members, &m, &s, &ra, &rb)
             : next_run(w, list, s_prefix, a.n_chunks, a.n_ty, H, &s, &ra, &rb)) {
    if (ENS) {
      const FipEnsMember& M = a.members[m];
      W = M.W;
      H = M.H;
      row0 = M.row_off;
      tbase = M.tile_base;
      nty = M.n_ty;
      dx = M.dx;
      kstf = M.kst_fixed;
      nv = M.no_value;
      dtm = a.mctl[m].dt;
      set_scalars();
      if (lane == 0) {
        s_msc[warp][0] = H;
        s_msc[warp][1] = row0;
        s_msc[warp][2] = tbase;
        s_msc[warp][3] = nty;
        s_msc[warp][4] = __float_as_int(nv);
        s_msc[warp][5] = __float_as_int(dx);
        s_msc[warp][6] = m;
        s_mcf[warp][0] = s_mcf[warp][1] = dt_inv;
        s_mcf[warp][2] = s_mcf[warp][3] = dx;
        s_mcf[warp][4] = s_mcf[warp][5] = dx_inv;
        s_mcf[warp][6] = s_mcf[warp][7] = dtm;
        s_mcf[warp][8] = s_mcf[warp][9] = -dtdx;
        s_mcf[warp][10] = fric_u;
        s_mcf[warp][11] = dtg;
      }
      __syncwarp();
    }
    const int c = s * TC - NC + 30 * NC * warp + NC * lane;  // global column of k = 0
    // NC-bit column masks of the cell sets the reference's kernel writes (src/kernels.cu:383-406)
    int colHm = 0, colQXm = 0, colQYm = 0, colInm = 0;
    bool holdX[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
      const int cc = c + k;
      colHm |= (out_lane && cc >= 1 && cc <= W - 2) << k;
      colQXm |= (out_lane && cc >= 1 && cc <= W - 3) << k;
      colQYm |= (out_lane && cc >= 2 && cc <= W - 3) << k;
      const bool in = out_lane && cc >= 0 && cc < W;
      colInm |= in << k;
      holdX[k] = (cc == 0 || cc == W - 2);
    }
    // ring slots of the staged rows r-1, r, r+1, r+2 (row ra-2 has sequence number seq); the
    // row loop advances them by one slot per row
    uint32_t iS = seq % kNSlot;
    uint32_t i0 = (seq + 1) % kNSlot, i1 = (seq + 2) % kNSlot, i2 = (seq + 3) % kNSlot;
    uint32_t ph2 = ((seq + 3) / kNSlot) & 1u;  // phase of the slot of row r+2
    auto wait_slot = [&](uint32_t q) -> bool {  // warp-uniform: every lane waits, all must succeed
      const bool got = mbar_wait(&full_bar[q % kNSlot], (q / kNSlot) & 1u);
      return __all_sync(0xffffffffu, got);
    };
    auto release_slot = [&](uint32_t slot) {
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty_bar[slot]);
    };

    bool ok = wait_slot(seq) && wait_slot(seq + 1) && wait_slot(seq + 2);
    if (!ok) {
      record_error(ctl, FIP_DEVERR_WAIT_FULL);
      break;
    }
    // ---- prologue: rows ra-2 .. ra ----
    // carried from row to row: only computed quantities; the raw fields of rows r-1 .. r+2 are
    // read from the staged rows again at every row
    float ux0[NC], uxW0, uy0[NC], uyE0, uyS[NC], gxS[NC], gy0[NC], qy2S[NC];
    float lim0[NC], limE0;  // h * dt_inv * dx * 0.25f of row r (and its east neighbour)
    {
      const unsigned char* slA = ring + iS * kSlotBytes;
      const unsigned char* slB = ring + i0 * kSlotBytes;
      const unsigned char* slC = ring + i1 * kSlotBytes;
      float hs[NC], qyS[NC], h0[NC], qx0[NC], qy0[NC], h1[NC];
      ldsv<NC, kFB>(hs, slA, F_H, scol);
      ldsv<NC, kFB>(qyS, slA, F_QY, scol);
      ldsv<NC, kFB>(h0, slB, F_H, scol);
      ldsv<NC, kFB>(qx0, slB, F_QX, scol);
      ldsv<NC, kFB>(qy0, slB, F_QY, scol);
      ldsv<NC, kFB>(h1, slC, F_H, scol);
      const float hE0 = __shfl_down_sync(0xffffffffu, h0[0], 1);
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        uyS[k] = qyS[k] / fmax3(kDH, hs[k], h0[k]);
        ux0[k] = qx0[k] / fmax3(kDH, h0[k], k < NC - 1 ? h0[k + 1] : hE0);
        uy0[k] = qy0[k] / fmax3(kDH, h0[k], h1[k]);
      }
      vmul(lim0, h0, c_dti);
      vmul(lim0, lim0, c_dx);
      vmul(lim0, lim0, c_q);
      uxW0 = __shfl_up_sync(0xffffffffu, ux0[NC - 1], 1);
      uyE0 = __shfl_down_sync(0xffffffffu, uy0[0], 1);
      limE0 = __shfl_down_sync(0xffffffffu, lim0[0], 1);
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        // compute_rmg_gy for row ra-1: uy_i = uy(ra-1), uy_south = uy(ra-2)
        gy0[k] = (uy0[k] + uyS[k] > 0) ? qyS[k] * uyS[k] : qy0[k] * uy0[k];
        gxS[k] = 0.f;
        qy2S[k] = 0.f;
      }
    }
    // rows r-1 .. r+2 stay staged during row r: qy(r-1) and the terrain of row r are read
    // again instead of being carried in registers; row r-1 is released at the end of row r
    unsigned nzacc = 0u;
    for (int r = ra - 1; r < rb; ++r) {
      {  // wait for row r+2
        const bool got = __all_sync(0xffffffffu, mbar_wait(&full_bar[i2], ph2));
        if (!got) {
          record_error(ctl, FIP_DEVERR_WAIT_FULL);
          ok = false;
          break;
        }
      }
      const unsigned char* slS = ring + iS * kSlotBytes;
      const unsigned char* sl0 = ring + i0 * kSlotBytes;
      const unsigned char* sl1 = ring + i1 * kSlotBytes;
      const unsigned char* sl2 = ring + i2 * kSlotBytes;
      float h2r[NC], qx1[NC], qy1[NC], s1[NC], fric[NC], qyS[NC], s0[NC], h0[NC], h1[NC], qx0[NC], qy0[NC];
      ldsv<NC, kFB>(qyS, slS, F_QY, scol);
      ldsv<NC, kFB>(s0, sl0, F_S, scol);
      ldsv<NC, kFB>(h0, sl0, F_H, scol);
      ldsv<NC, kFB>(qx0, sl0, F_QX, scol);
      ldsv<NC, kFB>(qy0, sl0, F_QY, scol);
      ldsv<NC, kFB>(h1, sl1, F_H, scol);
      ldsv<NC, kFB>(h2r, sl2, F_H, scol);
      ldsv<NC, kFB>(qx1, sl1, F_QX, scol);
      ldsv<NC, kFB>(qy1, sl1, F_QY, scol);
      ldsv<NC, kFB>(s1, sl1, F_S, scol);
      if (KVAR) {
        float kk[NC];
        ldsv<NC, kFB>(kk, sl0, F_K, scol);
        vmul(kk, kk, kk);
#pragma unroll
        for (int k = 0; k < NC; ++k) fric[k] = (ENS ? ldsf_at_use(&s_mcf[warp][11]) : dtg) / kk[k];
      } else {
#pragma unroll
        for (int k = 0; k < NC; ++k) fric[k] = ENS ? ldsf_at_use(&s_mcf[warp][10]) : fric_u;
      }
      const float hE0 = __shfl_down_sync(0xffffffffu, h0[0], 1);
      const float hE1 = __shfl_down_sync(0xffffffffu, h1[0], 1);
      const float qxW0 = __shfl_up_sync(0xffffffffu, qx0[NC - 1], 1);
      const float qyE0 = __shfl_down_sync(0xffffffffu, qy0[0], 1);
      const float qySE = __shfl_down_sync(0xffffffffu, qyS[0], 1);
      const float sE0 = __shfl_down_sync(0xffffffffu, s0[0], 1);
      const float qxW1 = __shfl_up_sync(0xffffffffu, qx1[NC - 1], 1);
      float t[NC], u[NC];

      // velocities of row r+1 (src/kernels.cu:351-354) and the clamp factors of row r+1
      float ux1[NC], uy1[NC], lim1[NC];
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        ux1[k] = qx1[k] / fmax3(kDH, h1[k], k < NC - 1 ? h1[k + 1] : hE1);
        uy1[k] = qy1[k] / fmax3(kDH, h1[k], h2r[k]);
      }
      vmul(lim1, h1, ENS ? lds2_at_use(&s_mcf[warp][0]) : c_dti);
      vmul(lim1, lim1, ENS ? lds2_at_use(&s_mcf[warp][2]) : c_dx);
      vmul(lim1, lim1, c_q);
      const float ux1W = __shfl_up_sync(0xffffffffu, ux1[NC - 1], 1);
      const float uy1E = __shfl_down_sync(0xffffffffu, uy1[0], 1);

      float fx[NC], fy[NC], gx[NC], gy1[NC];
      // compute_rmg_fy (:45-54): ux at the cell and its north neighbour
      vadd(t, ux0, ux1);
      vmul(u, t, c_h);
#pragma unroll
      for (int k = 0; k < NC; ++k) fy[k] = t[k] > 0 ? qy0[k] : (k < NC - 1 ? qy0[k + 1] : qyE0);
      vmul(fy, fy, u);
      // compute_rmg_gy for row r+1 (:65-73, called at :359)
      vadd(t, uy1, uy0);
      vmul(u, qy0, uy0);
      vmul(gy1, qy1, uy1);
#pragma unroll
      for (int k = 0; k < NC; ++k) gy1[k] = t[k] > 0 ? u[k] : gy1[k];
      // compute_rmg_gx (:35-43)
#pragma unroll
      for (int k = 0; k < NC; ++k) t[k] = uy0[k] + (k < NC - 1 ? uy0[k + 1] : uyE0);
      vmul(u, t, c_h);
#pragma unroll
      for (int k = 0; k < NC; ++k) gx[k] = t[k] > 0 ? qx0[k] : qx1[k];
      vmul(gx, gx, u);
      // compute_rmg_fx (:56-63): qx * ux of the cell or of its west neighbour
      vmul(u, qx0, ux0);
      const float pqW = qxW0 * uxW0;
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        const float uw = k > 0 ? ux0[k - 1] : uxW0;
        fx[k] = (uw + ux0[k] > 0) ? (k > 0 ? u[k - 1] : pqW) : u[k];
      }
      const float fyW = __shfl_up_sync(0xffffffffu, fy[NC - 1], 1);
      const float fxE = __shfl_down_sync(0xffffffffu, fx[0], 1);

      const int Hr = ENS ? lds_at_use(&s_msc[warp][0]) : H;
      const bool hold_y = (r == 0 || r == Hr - 2);
      // face depths and the mean cross discharges of the friction factor (:83-92, :110-119)
      float ax0[NC], ax1[NC], ay0[NC], ay1[NC], uyx[NC], uxy[NC];
#pragma unroll
      for (int k = 0; k < NC; ++k) t[k] = h0[k] + (k < NC - 1 ? h0[k + 1] : hE0);
      vmul(ax0, t, c_h);
      vadd(t, h0, h1);
      vmul(ay0, t, c_h);
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        ax0[k] = fmaxf(0.f, ax0[k]);
        ax1[k] = fmaxf(ax0[k], kDH);
        ay0[k] = fmaxf(0.f, ay0[k]);
        ay1[k] = fmaxf(ay0[k], kDH);
      }
#pragma unroll
      for (int k = 0; k < NC; ++k) t[k] = qy0[k] + (k < NC - 1 ? qy0[k + 1] : qyE0);
      vadd(t, t, qyS);
#pragma unroll
      for (int k = 0; k < NC; ++k) t[k] = t[k] + (k < NC - 1 ? qyS[k + 1] : qySE);
      vmul(uyx, t, c_q);
      vadd(t, qx0, qx1);
#pragma unroll
      for (int k = 0; k < NC; ++k) t[k] = (t[k] + (k > 0 ? qx0[k - 1] : qxW0)) + (k > 0 ? qx1[k - 1] : qxW1);
      vmul(uxy, t, c_q);
      // friction factors fric * sqrt(ux^2 + uy^2) * (1 / a1)^2.33 (:91-94, :118-121), 0 where both
      // discharges vanish (then the square sum is 0 and the product is 0 for every finite fric).
      // x first, then y: each square sum is dead once its factor is selected (fewer live registers)
      float rx[NC], ry[NC];
      {
        float m2[NC];
        vmul(t, uyx, uyx);
        vfma(m2, qx0, qx0, t);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
          t[k] = sqrtf(m2[k]);
          u[k] = pow_inv(ax1[k]);
        }
        vmul(rx, fric, t);
        vmul(rx, rx, u);
#pragma unroll
        for (int k = 0; k < NC; ++k) rx[k] = (m2[k] == 0.f) ? 0.f : rx[k];
        vmul(t, qy0, qy0);
        vfma(m2, uxy, uxy, t);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
          t[k] = sqrtf(m2[k]);
          u[k] = pow_inv(ay1[k]);
        }
        vmul(ry, fric, t);
        vmul(ry, ry, u);
#pragma unroll
        for (int k = 0; k < NC; ++k) ry[k] = (m2[k] == 0.f) ? 0.f : ry[k];
      }
      // compute_rmg_qx / compute_rmg_qy (:75-127): the same expression trees; 0.5 G h^2 as
      // nhh = (-0.5 G h) h = -(0.5 G h h)
      float qx2[NC], qy2[NC];
      {
        float nch[NC], nhh[NC], dsum[NC];
        vmul(nch, h0, c_nhg);
        vmul(nhh, nch, h0);
        const float nchE = -kHG * hE0;
        // x: -dfx - dgx - dhx + dhg
#pragma unroll
        for (int k = 0; k < NC; ++k) t[k] = (k < NC - 1 ? fx[k + 1] : fxE) - fx[k];
        vmul(dsum, t, c_ndxi);                  // -dfx
        vsub(t, gx, gxS);                       // (gx_i - gx_south)
        vfma(dsum, t, c_ndxi, dsum);            // - dgx
#pragma unroll
        for (int k = 0; k < NC; ++k) {
          t[k] = fmaf(-(k < NC - 1 ? nch[k + 1] : nchE), k < NC - 1 ? h0[k + 1] : hE0, nhh[k]);  // 0.5G hE hE - 0.5G h h
        }
        vfma(dsum, t, c_ndxi, dsum);            // - dhx
#pragma unroll
        for (int k = 0; k < NC; ++k) u[k] = s0[k] - (k < NC - 1 ? s0[k + 1] : sE0);  // -s_east + s_i
        vmul(t, ax0, c_g);
        vmul(t, t, u);
        vfma(dsum, t, ENS ? lds2_at_use(&s_mcf[warp][4]) : c_dxi, dsum);  // + dhg
        vfma(dsum, ENS ? lds2_at_use(&s_mcf[warp][6]) : c_dt, dsum, qx0);  // qx + dt * (...)
        vadd(t, c_one, rx);
#pragma unroll
        for (int k = 0; k < NC; ++k) qx2[k] = dsum[k] / t[k];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
          float q = fminf(qx2[k], lim0[k]);
          q = fmaxf(q, -(k < NC - 1 ? lim0[k + 1] : limE0));
          qx2[k] = holdX[k] ? qx0[k] : q;  // boundary-face holds (:373-376)
        }
        // zeros as +0: fp32div_wrapper returns +0 for a zero dividend, and a quiescent tile then
        // computes exactly the +0 its cells hold (inputs are loaded with +0 for zeros too)
        vadd(qx2, qx2, c_zero);
        // y: -dgy - dfy - dhy + dhg
        vsub(t, gy1, gy0);
        vmul(dsum, t, c_ndxi);                  // -dgy
#pragma unroll
        for (int k = 0; k < NC; ++k) t[k] = fy[k] - (k > 0 ? fy[k - 1] : fyW);
        vfma(dsum, t, c_ndxi, dsum);            // - dfy
        vmul(u, h1, c_hg);
        vfma(t, u, h1, nhh);                    // 0.5G hN hN - 0.5G h h
        vfma(dsum, t, c_ndxi, dsum);            // - dhy
        vsub(u, s0, s1);
        vmul(t, ay0, c_g);
        vmul(t, t, u);
        vfma(dsum, t, ENS ? lds2_at_use(&s_mcf[warp][4]) : c_dxi, dsum);  // + dhg
        vfma(dsum, ENS ? lds2_at_use(&s_mcf[warp][6]) : c_dt, dsum, qy0);  // qy + dt * (...)
        vadd(t, c_one, ry);
#pragma unroll
        for (int k = 0; k < NC; ++k) qy2[k] = dsum[k] / t[k];
#pragma unroll
        for (int k = 0; k < NC; ++k) {
          float q = fminf(qy2[k], lim0[k]);
          q = fmaxf(q, -lim1[k]);
          qy2[k] = hold_y ? qy0[k] : q;
        }
        vadd(qy2, qy2, c_zero);
      }
      const float qx2W = __shfl_up_sync(0xffffffffu, qx2[NC - 1], 1);

      {
        const bool store_row = r >= ra;  // the extra row below a run only feeds qy2S
        int validm = 0;
        const float nvr = ENS ? __int_as_float(lds_at_use(&s_msc[warp][4])) : nv;
        const int Hs = ENS ? lds_at_use(&s_msc[warp][0]) : H;
#pragma unroll
        for (int k = 0; k < NC; ++k) validm |= (s0[k] != nvr) << k;
        const int mH = (store_row && r >= 1 && r <= Hs - 2) ? (colHm & validm) : 0;
        const int mQX = (store_row && r >= 2 && r <= Hs - 3) ? (colQXm & validm) : 0;
        const int mQY = (store_row && r >= 1 && r <= Hs - 3) ? (colQYm & validm) : 0;
        // continuity (:381): h - dt * dx_inv * ((qx_i - qx_W) + (qy_i - qy_S))
        float h2[NC];
#pragma unroll
        for (int k = 0; k < NC; ++k) t[k] = qx2[k] - (k > 0 ? qx2[k - 1] : qx2W);
        vsub(u, qy2, qy2S);
        vadd(t, t, u);
        vfma(h2, ENS ? lds2_at_use(&s_mcf[warp][8]) : c_ndtdx, t, h0);
        // CFL of wet stored cells (:392-396): dx / (sqrt(G h') + max |u|), velocities of the old state
        vmul(t, c_g, h2);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
          const float uw = k > 0 ? ux0[k - 1] : uxW0;
          u[k] = fmaxf(fabsf(uy0[k]), fmaxf(fabsf(uyS[k]), fmaxf(fabsf(ux0[k]), fabsf(uw))));
          t[k] = sqrtf(t[k]);
        }
        vadd(t, t, u);
#pragma unroll
        for (int k = 0; k < NC; ++k) {
          const bool wk = (mH >> k) & 1;
          expacc = max(expacc, __float_as_uint(h2[k]) & 0x7f800000u);  // all-ones exponent: NaN/Inf
          den_max = fmaxf(den_max, (wk && h2[k] > kEPS) ? t[k] : 0.0f);
          nzacc |= (__float_as_uint(h2[k]) | __float_as_uint(qx2[k]) | __float_as_uint(qy2[k])) & 0x7fffffffu;
        }
        const size_t row_off = (size_t)(r + (ENS ? lds_at_use(&s_msc[warp][1]) : 0)) * (size_t)pitch + (size_t)c;
        if (mH == FULL) {
          stgv<NC>(h_out + row_off, h2);
        } else {
#pragma unroll
          for (int k = 0; k < NC; ++k)
            if ((mH >> k) & 1) h_out[row_off + k] = h2[k];
        }
        if (mQX == FULL) {
          stgv<NC>(qx_out + row_off, qx2);
        } else {
#pragma unroll
          for (int k = 0; k < NC; ++k)
            if ((mQX >> k) & 1) qx_out[row_off + k] = qx2[k];
        }
        if (mQY == FULL) {
          stgv<NC>(qy_out + row_off, qy2);
        } else {
#pragma unroll
          for (int k = 0; k < NC; ++k)
            if ((mQY >> k) & 1) qy_out[row_off + k] = qy2[k];
        }
        if (fold && store_row) {  // flood_plains_kernel on the post-boundary state of the last step (:254-262)
          if (colInm == FULL) {
            hmax_foldv<NC>(a.hmax + row_off, h0);
          } else {
#pragma unroll
            for (int k = 0; k < NC; ++k)
              if ((colInm >> k) & 1) a.hmax[row_off + k] = fmaxf(a.hmax[row_off + k], h0[k]);
          }
        }
        // per-tile wet flag for the next plan, flushed at the tile's last row
        if (store_row && ((r + 1) % TR == 0 || r + 1 == rb)) {
          // halo lanes hold the neighbouring strips' cells; columns beyond W (zero-filled loads)
          // can only set flags, never clear them
          if (__any_sync(0xffffffffu, out_lane && nzacc != 0u)) {
            // edge bands: lane 1 of warp 0 holds the tile's first NC columns, lane 30 of warp
            // KW - 1 its last NC (at least the two the stencil reaches); one warp sets each band
            // bit, every warp with a nonzero cell the ANY bit (the conditions are warp-uniform)
            unsigned f = FIP_NZ_ANY;
            if (warp == 0 && __shfl_sync(0xffffffffu, nzacc, 1) != 0u) f |= FIP_NZ_WEST;
            if (warp == KW - 1 && __shfl_sync(0xffffffffu, nzacc, 30) != 0u) f |= FIP_NZ_EAST;
            if (lane == 0) {
              const int tb = ENS ? lds_at_use(&s_msc[warp][2]) : 0, nt = ENS ? lds_at_use(&s_msc[warp][3]) : nty;
              tile_flag_or(nzs + tb + s * nt + r / TR, f);
            }
          }
          nzacc = 0u;
        }
      }

      // the extra row below a run is no part of a tile
      nzacc = store_row_flag(r, ra) ? nzacc : 0u;
      release_slot(iS);
      // next row: slots advance by one
      iS = i0;
      i0 = i1;
      i1 = i2;
      ++i2;
      if (i2 == (uint32_t)kNSlot) {
        i2 = 0;
        ph2 ^= 1u;
      }
      // travel north (:408-433)
#pragma unroll
      for (int k = 0; k < NC; ++k) {
        qy2S[k] = qy2[k];
        gxS[k] = gx[k];
        uyS[k] = uy0[k];
        ux0[k] = ux1[k];
        uy0[k] = uy1[k];
        gy0[k] = gy1[k];
        lim0[k] = lim1[k];
      }
      uxW0 = ux1W;
      uyE0 = uy1E;
      limE0 = __shfl_down_sync(0xffffffffu, lim0[0], 1);
    }
    if (!ok) break;
    release_slot(iS);  // rows rb-1, rb, rb+1
    release_slot(i0);
    release_slot(i1);
    seq += (uint32_t)(rb - ra + 4);
    if (ENS) {  // this member's CFL minimum: warp reduction, one atomicMin per warp and run
      float dm = den_max;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) dm = fmaxf(dm, __shfl_xor_sync(0xffffffffu, dm, off));
      if (lane == 0 && dm > 0.0f) {
        const float cfl = fminf(1.0f, __int_as_float(lds_at_use(&s_msc[warp][5])) / dm);
        if (cfl < 1.0f) atomicMin(&a.mctl[lds_at_use(&s_msc[warp][6])].cfl_bits[it & 1], __float_as_uint(cfl));
      }
      den_max = 0.0f;
    }
  }

  // inactive tiles still fold hmax when the initial state had negative depths
  if (fold && s_hdr[5]) {
    const int ctid = tid;  // consumer thread
    for (int ch = 0; ch < a.n_chunks; ++ch) {
      const int in_chunk = min(FIP_PLAN_CHUNK, a.n_tiles - ch * FIP_PLAN_CHUNK);
      const int n_inact = in_chunk - (s_prefix[ch + 1] - s_prefix[ch]);
      for (int i = blockIdx.x; i < n_inact; i += gridDim.x) {
        const int tile = list[ch * FIP_PLAN_CHUNK + FIP_PLAN_CHUNK - 1 - i];
        const int st = tile / a.n_ty, ty = tile - st * a.n_ty;
        const int c0 = st * TC, r0 = ty * TR;
        for (int e = ctid; e < TC * TR; e += KW * 32) {
          const int rr = r0 + e / TC, cc = c0 + e % TC;
          if (rr < H && cc < W) {
            const size_t o = (size_t)rr * pitch + cc;
            a.hmax[o] = fmaxf(a.hmax[o], h_in[o]);
          }
        }
      }
    }
  }

  // CFL minimum (capped at 1, the reference's initial value): warp reduction of the largest
  // denominator, one atomicMin per warp on the float bits (all positive)
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) den_max = fmaxf(den_max, __shfl_xor_sync(0xffffffffu, den_max, off));
  const bool any_bad = __any_sync(0xffffffffu, expacc == 0x7f800000u);
  if (lane == 0) {
    const float cfl = den_max > 0.0f ? fminf(1.0f, dx / den_max) : 1.0f;
    if (cfl < 1.0f) atomicMin(&ctl->cfl_bits[it & 1], __float_as_uint(cfl));
    if (any_bad) ctl->nonfinite = 1;
  }
}

// Per tile of a tile_cols x tile_rows grid: sticky flag and the FIP_NZ_* flags of buffer
// (h, qx, qy) (into nz0 and nz1). With or_into set, FIP_NZ_ANY is OR-ed into or_into[t] where the
// tile has a nonzero cell instead, and nothing else is written.
// A tile is sticky (computed every step) when
//  * a cell the step never writes holds water within 2 cells of it (the step reads 2 cells
//    around each cell it updates): no_data cells, and the cells within 1 of the edge that the
//    reference's write sets leave out (src/kernels.cu:383-406) -- only boundary conditions change
//    those, and the conditions' own cells are covered next;
//  * it meets a rectangle of `force`: the cells a boundary condition writes, widened by the
//    stencil's reach (or, with force.all_band, any tile within 4 cells of the edge).
// Elsewhere a tile computes zeros where its cells and the cells within 2 of it are all zero,
// which the plan exploits with the flags of each tile (any cell nonzero; any of its first / last
// kNzBand columns nonzero: the stencil sets those from the columns of the first / last thread of
// the tile, 4 or 2, at least the 2 it reaches).
__global__ void init_tiles_kernel(const float* h, const float* qx, const float* qy, const float* sohle, int W, int H,
                                  int pitch, float no_value, int n_ty, int n_tiles, int tile_cols, int tile_rows,
                                  const TileForce force, unsigned char* or_into, unsigned char* sticky,
                                  unsigned char* nz0, unsigned char* nz1) {
  const int t = blockIdx.x;
  if (t >= n_tiles) return;
  const int s = t / n_ty, ty = t - s * n_ty;
  const int c0 = s * tile_cols, r0 = ty * tile_rows;
  const int c1 = min(c0 + tile_cols, W), r1 = min(r0 + tile_rows, H);
  int nz = 0, st = 0;
  if (or_into) {
    for (int e = threadIdx.x; e < tile_cols * tile_rows; e += blockDim.x) {
      const int r = r0 + e / tile_cols, c = c0 + e % tile_cols;
      if (r < r1 && c < c1) {
        const size_t o = (size_t)r * pitch + c;
        nz |= (h[o] != 0.f) || (qx[o] != 0.f) || (qy[o] != 0.f);
      }
    }
    nz = __syncthreads_or(nz);
    if (threadIdx.x == 0 && nz) or_into[t] |= FIP_NZ_ANY;
    return;
  }
  // the tile widened by the stencil's reach of 2 cells, clipped to the grid
  const int x0 = max(c0 - 2, 0), x1 = min(c1 + 2, W), y0 = max(r0 - 2, 0), y1 = min(r1 + 2, H);
  const int ww = x1 - x0;
  int nzw = 0, nze = 0;  // nonzero cells in the tile's first / last kNzBand columns
  for (int e = threadIdx.x; e < ww * (y1 - y0); e += blockDim.x) {
    const int r = y0 + e / ww, c = x0 + e % ww;
    const size_t o = (size_t)r * pitch + c;
    const bool nzc = (h[o] != 0.f) || (qx[o] != 0.f) || (qy[o] != 0.f);
    if (r >= r0 && r < r1 && c >= c0 && c < c1) {
      nz |= nzc;
      if (c < c0 + kNzBand) nzw |= nzc;
      if (c >= c1 - kNzBand) nze |= nzc;
    }
    const bool unwritten = r <= 1 || r >= H - 2 || c <= 1 || c >= W - 2 || sohle[o] == no_value;
    if (nzc && unwritten) st = 1;
  }
  if (threadIdx.x == 0) {
    if (force.all_band) {
      if (r0 < 4 || r1 > H - 4 || c0 < 4 || c1 > W - 4) st = 1;
    } else {
      for (int i = 0; i < force.n; ++i) {
        const int* q = force.rect[i];
        if (q[0] < c1 && q[1] >= c0 && q[2] < r1 && q[3] >= r0) st = 1;
      }
    }
  }
  nz = __syncthreads_or(nz);
  nzw = __syncthreads_or(nzw);
  nze = __syncthreads_or(nze);
  st = __syncthreads_or(st);
  if (threadIdx.x == 0) {
    const unsigned char f = (unsigned char)((nz ? FIP_NZ_ANY : 0) | (nzw ? FIP_NZ_WEST : 0) | (nze ? FIP_NZ_EAST : 0));
    sticky[t] = (unsigned char)st;
    nz0[t] = f;
    nz1[t] = f;
  }
}

__global__ void hmax_fold_kernel(const float* __restrict__ h, float* __restrict__ hmax, int W, int H, int pitch) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (c >= W || r >= H) return;
  const size_t o = (size_t)r * pitch + c;
  hmax[o] = fmaxf(hmax[o], h[o]);
}

constexpr int kVolBlocks = 1184;  // 8 per SM on 148 SMs
constexpr int kVolThreads = 256;

__global__ void volume_partial_kernel(const float* __restrict__ h, int W, int H, int pitch, double* partials) {
  __shared__ double red[kVolThreads];
  double acc = 0.0;
  for (int r = blockIdx.x; r < H; r += gridDim.x) {
    const float* row = h + (size_t)r * pitch;
    for (int c = threadIdx.x; c < W; c += blockDim.x) acc += (double)row[c];
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void flag_negative_kernel(const float* __restrict__ h, int W, int H, int pitch, int* flag) {
  bool neg = false;
  for (int r = blockIdx.x; r < H; r += gridDim.x) {
    const float* row = h + (size_t)r * pitch;
    for (int c = threadIdx.x; c < W; c += blockDim.x) neg |= row[c] < 0.f;
  }
  if (__syncthreads_or(neg) && threadIdx.x == 0) *flag = 1;
}

__global__ void volume_final_kernel(const double* partials, int n, double* out) {
  __shared__ double red[kVolThreads];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

__global__ void sample_gather_kernel(const float* h, const float* qx, const float* qy, const float* sohle, int pitch,
                                     int n, const int* xy_type, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = xy_type[3 * i], y = xy_type[3 * i + 1], t = xy_type[3 * i + 2];
  const size_t o = (size_t)y * pitch + x;
  float v;
  if (t == 0) v = __fadd_rn(h[o], sohle[o]);  // sample(): val += h_sohle (src/main.cpp:62-67)
  else if (t == 1) v = h[o];
  else if (t == 2) v = qx[o];
  else v = qy[o];
  out[i] = v;
}

}  // namespace

void tile_geometry(int W, int H, int tile_cols, int* n_sx, int* n_ty, int* n_tiles, int* n_chunks) {
  *n_sx = (W + tile_cols - 1) / tile_cols;
  *n_ty = (H + FIP_TILE_ROWS - 1) / FIP_TILE_ROWS;
  *n_tiles = *n_sx * *n_ty;
  *n_chunks = (*n_tiles + FIP_PLAN_CHUNK - 1) / FIP_PLAN_CHUNK;
}

static int encode_map(CUtensorMap* tm, float* base, int W, int H, int pitch) {
  cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)H};
  cuuint64_t strides[1] = {(cuuint64_t)pitch * 4};
  cuuint32_t box[2] = {256, 1};
  cuuint32_t estr[2] = {1, 1};
  if (!drv::TensorMapEncodeTiled) return (int)CUDA_ERROR_NOT_INITIALIZED;
  CUresult r = drv::TensorMapEncodeTiled(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr,
                                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (int)r;
}

int make_tensor_maps(StencilState* st) {
  int r = 0;
  for (int b = 0; b < 2; ++b) {
    if ((r = encode_map(&st->tm_h[b], st->h[b], st->W, st->H, st->pitch))) return r;
    if ((r = encode_map(&st->tm_qx[b], st->qx[b], st->W, st->H, st->pitch))) return r;
    if ((r = encode_map(&st->tm_qy[b], st->qy[b], st->W, st->H, st->pitch))) return r;
  }
  if ((r = encode_map(&st->tm_sohle, st->sohle, st->W, st->H, st->pitch))) return r;
  if ((r = encode_map(&st->tm_kst, st->kst ? st->kst : st->sohle, st->W, st->H, st->pitch))) return r;
  return 0;
}

// -0 -> +0 (bit test: denormals and every other value stay as they are)
__device__ __forceinline__ float positive_zero(float v) { return __float_as_uint(v) == 0x80000000u ? 0.f : v; }

// dst0 (and dst1 unless null) = src with -0 -> +0, over the W x H cells of row pitch `pitch`
// (a multiple of 4 floats, 16-byte aligned rows): four cells per thread, the row's last partial
// group cell by cell. src may be dst0.
__global__ void positive_zero_copy_kernel(const float* src, float* dst0, float* dst1, int W, int H, int pitch) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  const int c = 4 * g;
  if (r >= H || c >= W) return;
  const size_t o = (size_t)r * pitch + c;
  if (c + 4 <= W) {
    float4 v = *reinterpret_cast<const float4*>(src + o);
    v.x = positive_zero(v.x);
    v.y = positive_zero(v.y);
    v.z = positive_zero(v.z);
    v.w = positive_zero(v.w);
    *reinterpret_cast<float4*>(dst0 + o) = v;
    if (dst1) *reinterpret_cast<float4*>(dst1 + o) = v;
  } else {
    for (int k = 0; k < W - c; ++k) {
      const float v = positive_zero(src[o + k]);
      dst0[o + k] = v;
      if (dst1) dst1[o + k] = v;
    }
  }
}

cudaError_t launch_positive_zero(float* a, int W, int H, int pitch, cudaStream_t stream) {
  return launch_positive_zero_copy(a, a, nullptr, W, H, pitch, stream);
}

cudaError_t launch_positive_zero_copy(const float* src, float* dst0, float* dst1, int W, int H, int pitch,
                                      cudaStream_t stream) {
  if (W <= 0 || H <= 0) return cudaSuccess;
  const int groups = (W + 3) / 4;
  positive_zero_copy_kernel<<<dim3((groups + 255) / 256, H), 256, 0, stream>>>(src, dst0, dst1, W, H, pitch);
  return cudaGetLastError();
}



int rmg_step_grid(int device, int nc) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return (nc == 2 ? kMinCtasNarrow : kMinCtas4) * sms;
}

int single_tile_cols(int nc) { return nc == 2 ? StepShape<2, 4>::TC : StepShape<4, 4>::TC; }

template <bool KVAR, bool ENS, int KW, int TRT, int NC>
static cudaError_t launch_step_t(const StencilState& st, int grid, cudaStream_t stream) {
  using S = StepShape<NC, KW>;
  constexpr int NF = KVAR ? 5 : 4;
  const int smem = (KVAR ? S::kNSlotK : S::kNSlotU) * NF * S::kFB + 1024;
  static std::atomic<uint64_t> configured{0};
  const cudaError_t e = ensure_dynamic_smem(rmg_step_kernel<KVAR, ENS, KW, TRT, NC>, smem, configured);
  if (e != cudaSuccess) return e;
  StepArgs a;
  for (int b = 0; b < 2; ++b) {
    a.h[b] = st.h[b];
    a.qx[b] = st.qx[b];
    a.qy[b] = st.qy[b];
    a.list[b] = st.list[b];
    a.chunk_cnt[b] = st.chunk_cnt[b];
    a.nz[b] = st.nz[b];
  }
  a.hmax = st.hmax;
  a.ctl = st.ctl;
  a.W = st.W;
  a.H = st.H;
  a.pitch = st.pitch;
  a.n_sx = st.n_sx;
  a.n_ty = st.n_ty;
  a.n_tiles = st.n_tiles;
  a.n_chunks = st.n_chunks;
  a.dx = st.dx;
  a.kst_fixed = st.kst_fixed;
  a.no_value = st.no_value;
  a.members = st.members;
  a.mctl = st.mctl;
  a.n_members = st.n_members;
  rmg_step_kernel<KVAR, ENS, KW, TRT, NC><<<grid, (KW + 1) * 32, smem, stream>>>(
      st.tm_h[0], st.tm_h[1], st.tm_qx[0], st.tm_qx[1], st.tm_qy[0], st.tm_qy[1], st.tm_sohle, st.tm_kst, a);
  return cudaGetLastError();
}

cudaError_t launch_rmg_step(const StencilState& st, int grid, cudaStream_t stream) {
  if (st.n_chunks > kMaxChunks) return cudaErrorInvalidValue;
  constexpr int T = FIP_TILE_ROWS;
  if (!st.members)
    return st.kst ? launch_step_t<true, false, 4, T, 4>(st, grid, stream)
                  : launch_step_t<false, false, 4, T, 4>(st, grid, stream);
  if (st.n_members > FIP_ENS_MAX_MEMBERS) return cudaErrorInvalidValue;
  // ensemble tile shapes: 2 or 4 consumer warps, 16, 32 or 64 rows
#define FIP_ENS_LAUNCH(KW_, TR_, NC_)                                                              \
  if (st.kw == KW_ && st.tile_rows == TR_ && st.nc == NC_)                                         \
    return st.kst ? launch_step_t<true, true, KW_, TR_, NC_>(st, grid, stream)                     \
                  : launch_step_t<false, true, KW_, TR_, NC_>(st, grid, stream);
  FIP_ENS_LAUNCH(4, 32, 4)
  FIP_ENS_LAUNCH(4, 16, 4)
  FIP_ENS_LAUNCH(4, 64, 4)
  FIP_ENS_LAUNCH(2, 32, 4)
  FIP_ENS_LAUNCH(2, 16, 4)
  FIP_ENS_LAUNCH(2, 64, 4)
  FIP_ENS_LAUNCH(4, 32, 2)
  FIP_ENS_LAUNCH(4, 16, 2)
  FIP_ENS_LAUNCH(4, 64, 2)
#undef FIP_ENS_LAUNCH
  return cudaErrorInvalidValue;
}

int rmg_step_grid_kw(int device, int kw, int nc) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return (nc == 2 ? kMinCtasNarrow : kw == 2 ? kMinCtas2 : kMinCtas4) * sms;
}

cudaError_t launch_init_tiles(const StencilState& st, int parity, cudaStream_t stream) {
  init_tiles_kernel<<<st.n_tiles, 256, 0, stream>>>(st.h[parity], st.qx[parity], st.qy[parity], st.sohle, st.W, st.H,
                                                    st.pitch, st.no_value, st.n_ty, st.n_tiles, st.tile_cols,
                                                    FIP_TILE_ROWS, st.force, nullptr, st.sticky, st.nz[0], st.nz[1]);
  return cudaGetLastError();
}

cudaError_t launch_init_tiles_region(const float* h, const float* qx, const float* qy, const float* h_other,
                                     const float* qx_other, const float* qy_other, const float* sohle, int W, int H,
                                     int pitch, float no_value, int tile_cols, int tile_rows, const TileForce& force,
                                     unsigned char* sticky, unsigned char* nz_cur, unsigned char* nz_prev,
                                     cudaStream_t stream) {
  const int n_sx = (W + tile_cols - 1) / tile_cols, n_ty = (H + tile_rows - 1) / tile_rows;
  init_tiles_kernel<<<n_sx * n_ty, 256, 0, stream>>>(h, qx, qy, sohle, W, H, pitch, no_value, n_ty, n_sx * n_ty,
                                                     tile_cols, tile_rows, force, nullptr, sticky, nz_cur, nz_prev);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !h_other) return e;
  // the other buffer becomes the next step's output: a tile must be computed while it is nonzero
  init_tiles_kernel<<<n_sx * n_ty, 256, 0, stream>>>(h_other, qx_other, qy_other, sohle, W, H, pitch, no_value, n_ty,
                                                     n_sx * n_ty, tile_cols, tile_rows, force, nz_prev, nullptr,
                                                     nullptr, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_hmax_fold(const StencilState& st, int parity, cudaStream_t stream) {
  dim3 grid((st.W + 255) / 256, st.H);
  hmax_fold_kernel<<<grid, 256, 0, stream>>>(st.h[parity], st.hmax, st.W, st.H, st.pitch);
  return cudaGetLastError();
}

int volume_partials(const StencilState&) { return kVolBlocks; }

cudaError_t launch_volume(const StencilState& st, int parity, double* partials, double* out, cudaStream_t stream) {
  volume_partial_kernel<<<kVolBlocks, kVolThreads, 0, stream>>>(st.h[parity], st.W, st.H, st.pitch, partials);
  volume_final_kernel<<<1, kVolThreads, 0, stream>>>(partials, kVolBlocks, out);
  return cudaGetLastError();
}

cudaError_t launch_flag_negative(const float* h, int W, int H, int pitch, int* flag, cudaStream_t stream) {
  if (W <= 0 || H <= 0) return cudaSuccess;
  flag_negative_kernel<<<std::min(H, kVolBlocks), kVolThreads, 0, stream>>>(h, W, H, pitch, flag);
  return cudaGetLastError();
}

cudaError_t launch_sample_gather(const StencilState& st, int parity, int n, const int* xy_type, float* out,
                                 cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  sample_gather_kernel<<<(n + 127) / 128, 128, 0, stream>>>(st.h[parity], st.qx[parity], st.qy[parity], st.sohle,
                                                            st.pitch, n, xy_type, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// One rmg step without any device allocation (fip_rmg_step_noalloc in include/fip.h).
//
// Some callers cannot allocate device memory: a host that drives this step from its own time
// loop while other streams keep the GPU busy (cudaFree synchronises the whole device), or a host
// that owns all device memory through its own pool and forbids allocations once it runs. For
// them the step's scratch (control block,
// tile list, per-tile wet flags) lives in the file-scope array below, which every GPU that loads
// the library holds until the process exits. It holds the plan of at most kNoAllocMaxTiles tiles
// of 480 x 32 cells (about 503 million cells); larger grids are rejected. All calls share it and
// it keeps the last call's contents, so each call first rewrites everything the step reads from
// it; calls that overlap on the GPU (several streams, several host threads) race on it.
namespace {

constexpr int kNoAllocMaxTiles = 32768;
constexpr int kNoAllocMaxChunks = kNoAllocMaxTiles / FIP_PLAN_CHUNK;
constexpr size_t kNoAllocCtlOff = 0;
constexpr size_t kNoAllocCntOff = 256;
constexpr size_t kNoAllocListOff = kNoAllocCntOff + sizeof(int) * kNoAllocMaxChunks;
constexpr size_t kNoAllocNzOff = kNoAllocListOff + sizeof(int) * kNoAllocMaxTiles;
constexpr size_t kNoAllocBytes = kNoAllocNzOff + kNoAllocMaxTiles;
static_assert(sizeof(FipCtl) <= kNoAllocCntOff, "control block must fit its slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Rewrites the part of the scratch the step reads: the control block (dt, a fresh CFL minimum,
// no fold, no stop) and the identity plan over all n_tiles tiles.
__global__ void noalloc_setup_kernel(unsigned char* scratch, float dt, int n_tiles, int n_chunks) {
  FipCtl* ctl = reinterpret_cast<FipCtl*>(scratch + kNoAllocCtlOff);
  int* cnt = reinterpret_cast<int*>(scratch + kNoAllocCntOff);
  int* list = reinterpret_cast<int*>(scratch + kNoAllocListOff);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0) {
    ctl->duration = 0.0;
    ctl->next_sample = ctl->next_save = ctl->target = 0.0;
    ctl->dt = dt;
    ctl->last_cfl = 1.0f;
    ctl->iteration = 0;
    ctl->parity = 0;
    ctl->stop = 0;
    ctl->stop_reason = 0;
    ctl->steps_left = 0;
    ctl->variable_dt = 0;
    ctl->stop_on_nonfinite = 0;
    ctl->nonfinite = 0;
    ctl->error = 0;
    ctl->hmax_every = 0;
    ctl->hmax_full = 0;
    ctl->force_all = 1;
    ctl->inject = 0;
    ctl->cfl_bits[0] = ctl->cfl_bits[1] = __float_as_uint(1.0f);
    ctl->post_done = 0u;
  }
  for (int c = tid; c < n_chunks; c += gridDim.x * blockDim.x)
    cnt[c] = min(FIP_PLAN_CHUNK, n_tiles - c * FIP_PLAN_CHUNK);
  for (int t = tid; t < n_tiles; t += gridDim.x * blockDim.x) list[t] = t;
}

// CFL minimum of the step (NaN when a device-side wait ran out).
__global__ void noalloc_finish_kernel(const unsigned char* scratch, float* cfl_out) {
  const FipCtl* ctl = reinterpret_cast<const FipCtl*>(scratch + kNoAllocCtlOff);
  *cfl_out = ctl->error ? __int_as_float(0x7fc00000) : __uint_as_float(ctl->cfl_bits[0]);
}

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {};

// Device address of the scratch on the current device; cudaGetSymbolAddress once per device.
cudaError_t noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_addr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_noalloc_addr[device]);
  return cudaSuccess;
}

}  // namespace

void set_last_error(const std::string& msg);

}  // namespace fip

extern "C" int fip_rmg_step_noalloc(const float* h_in, const float* qx_in, const float* qy_in, const float* terrain,
                                    const float* kst_or_null, float kst_fixed, float* h_out, float* qx_out,
                                    float* qy_out, int W, int H, int pitch, float dx, float dt, float no_value,
                                    float* cfl_out_or_null, void* stream) {
  using namespace fip;
  auto bad = [](int code, const std::string& m) {
    set_last_error(m);
    return code;
  };
  if (W < 4 || H < 4) return bad(-7, "fip_rmg_step_noalloc: the grid must be at least 4 x 4 cells");
  if (pitch < W || (pitch % 4) != 0)
    return bad(-7, "fip_rmg_step_noalloc: pitch must be >= W and a multiple of 4 elements (16 bytes)");
  int n_sx, n_ty, n_tiles, n_chunks;
  tile_geometry(W, H, FIP_TILE_COLS, &n_sx, &n_ty, &n_tiles, &n_chunks);
  if (n_tiles > kNoAllocMaxTiles)
    return bad(-7, "fip_rmg_step_noalloc: a " + std::to_string(W) + " x " + std::to_string(H) + " grid has " +
                       std::to_string(n_tiles) + " tiles of 480 x 32 cells; the static scratch holds at most " +
                       std::to_string(kNoAllocMaxTiles));
  const void* ptrs[] = {h_in, qx_in, qy_in, terrain, h_out, qx_out, qy_out};
  for (const void* p : ptrs)
    if (!p || (reinterpret_cast<uintptr_t>(p) & 15u))
      return bad(-7, "fip_rmg_step_noalloc: every field must be a non-null, 16-byte aligned device pointer");
  if (kst_or_null && (reinterpret_cast<uintptr_t>(kst_or_null) & 15u))
    return bad(-7, "fip_rmg_step_noalloc: kSt grid must be 16-byte aligned");
  if (!(dt > 0.f) || !(dx > 0.f)) return bad(-7, "fip_rmg_step_noalloc: dt and dx must be positive");
  std::string derr;
  if (!drv::load(&derr)) return bad(-3, derr);
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  unsigned char* scratch = nullptr;
  if (e == cudaSuccess) e = noalloc_scratch(device, &scratch);
  if (e != cudaSuccess) return bad(-3, std::string("fip_rmg_step_noalloc: scratch address: ") + cudaGetErrorString(e));

  StencilState st{};
  st.h[0] = const_cast<float*>(h_in);
  st.h[1] = h_out;
  st.qx[0] = const_cast<float*>(qx_in);
  st.qx[1] = qx_out;
  st.qy[0] = const_cast<float*>(qy_in);
  st.qy[1] = qy_out;
  st.sohle = const_cast<float*>(terrain);
  st.kst = const_cast<float*>(kst_or_null);
  st.hmax = nullptr;
  st.ctl = reinterpret_cast<FipCtl*>(scratch + kNoAllocCtlOff);
  st.sticky = nullptr;
  for (int b = 0; b < 2; ++b) {
    st.nz[b] = scratch + kNoAllocNzOff;
    st.list[b] = reinterpret_cast<int*>(scratch + kNoAllocListOff);
    st.chunk_cnt[b] = reinterpret_cast<int*>(scratch + kNoAllocCntOff);
  }
  st.W = W;
  st.H = H;
  st.pitch = pitch;
  st.n_sx = n_sx;
  st.n_ty = n_ty;
  st.n_tiles = n_tiles;
  st.n_chunks = n_chunks;
  st.dx = dx;
  st.kst_fixed = kst_fixed;
  st.no_value = no_value;
  const int tr = make_tensor_maps(&st);
  if (tr) return bad(-3, drv::message((CUresult)tr, "fip_rmg_step_noalloc: cuTensorMapEncodeTiled"));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  noalloc_setup_kernel<<<(n_tiles + 255) / 256, 256, 0, s>>>(scratch, dt, n_tiles, n_chunks);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = launch_rmg_step(st, rmg_step_grid(device, 4), s);
  if (e == cudaSuccess && cfl_out_or_null) {
    noalloc_finish_kernel<<<1, 1, 0, s>>>(scratch, cfl_out_or_null);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return bad(-3, std::string("fip_rmg_step_noalloc: ") + cudaGetErrorString(e));
  return 0;
}
