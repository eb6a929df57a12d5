#include "bc_codegen.h"

#include <nvrtc.h>

#include "drv.h"
#include "rmg_stencil.h"

#include <cstdio>
#include <cstring>
#include <sstream>

namespace fip {

namespace {

const char kCtlHeader[] =
#include "fip_ctl_str.inc"
    ;

// Static part of the program: time-series interpolation and the boundary discharge sum in IEEE
// float with the host's operation order (the reference evaluates both on the host,
// src/timeseries.cpp:14-26 and src/boundary_condition.cpp:6-18), the active-tile planner and
// the control-block advance (controlTimestep, src/main.cpp:25-43).
const char kPostLib[] = R"FIPSRC(
#define FIP_G 9.81f

__device__ __forceinline__ float fip_interp(const float* tv, int n, float time) {
  int lo = 0, hi = n;  // lower_bound: first time not less than `time`
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (tv[mid] < time) lo = mid + 1; else hi = mid;
  }
  if (lo == 0) return tv[n];
  if (lo == n) return tv[2 * n - 1];
  const float dt = __fsub_rn(tv[lo], tv[lo - 1]);
  const float f = __fdiv_rn(__fsub_rn(time, tv[lo - 1]), dt);
  return __fadd_rn(__fmul_rn(f, tv[n + lo]), __fmul_rn(__fsub_rn(1.f, f), tv[n + lo - 1]));
}

// TimeSeries::interp with the whole block finding the bracket: lower_bound = number of table
// times below `time` (one __syncthreads_count per 512 entries instead of a chain of dependent
// loads); every thread returns the same value.
__device__ float fip_interp_block(const float* tv, int n, float time) {
  int lo = 0;
  for (int j0 = 0; j0 < n; j0 += blockDim.x) {
    const int j = j0 + threadIdx.x;
    lo += __syncthreads_count(j < n && tv[j] < time);
  }
  if (lo == 0) return tv[n];
  if (lo == n) return tv[2 * n - 1];
  const float dt = __fsub_rn(tv[lo], tv[lo - 1]);
  const float f = __fdiv_rn(__fsub_rn(time, tv[lo - 1]), dt);
  return __fadd_rn(__fmul_rn(f, tv[n + lo]), __fmul_rn(__fsub_rn(1.f, f), tv[n + lo - 1]));
}

// sequential float sum of sqrt(g a) a over the condition's cells [from, to), a = z - terrain
// (0 below 1 cm), times dx. Terms are evaluated in parallel, summed in order by thread 0.
__device__ float fip_sum_depths(const float* sohle, long long base, long long inc, int from, int to, float z,
                                float dx, float* s_buf) {
  float acc = 0.f;
  for (int c0 = from; c0 < to; c0 += 4096) {
    const int cn = min(4096, to - c0);
    for (int i = threadIdx.x; i < cn; i += blockDim.x) {
      float ah = __fsub_rn(z, sohle[base + (long long)(c0 + i) * inc]);
      if (ah < 0.01f) ah = 0.f;
      s_buf[i] = __fmul_rn(__fsqrt_rn(__fmul_rn(FIP_G, ah)), ah);
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < cn; ++i) acc = __fadd_rn(acc, s_buf[i]);
    __syncthreads();
  }
  return __fmul_rn(acc, dx);
}

// Active tiles of the next step: a tile is computed when a cell within 2 of it (the stencil's
// reach) may have been nonzero after this step -- a cell of the tile itself or of the tiles above
// and below it, or of the facing edge band (FIP_NZ_EAST / FIP_NZ_WEST) of the three tiles beside
// it in each neighbouring strip --, when it had a nonzero cell after the previous step (its cells
// in the output buffer are then not yet equal to the input), or when it is sticky. The flags of
// the previous step are cleared for reuse.
__device__ void fip_plan(const FipPostArgs& a, const FipCtl* ctl, int k, int chunk) {
  __shared__ int s_act[FIP_POST_THREADS / 32];
  __shared__ int s_inact[FIP_POST_THREADS / 32];
  const int t = chunk * FIP_PLAN_CHUNK + threadIdx.x;
  const unsigned char* nzc = a.nz[k & 1];
  unsigned char* nzp = a.nz[(k + 1) & 1];
  const bool valid = t < a.n_tiles;
  bool act = false;
  if (valid) {
    const int sx = t / a.n_ty, ty = t - sx * a.n_ty;
    act = a.sticky[t] || nzp[t] || ctl->force_all;
    for (int ds = -1; ds <= 1 && !act; ++ds) {
      const int s2 = sx + ds;
      if (s2 < 0 || s2 >= a.n_sx) continue;
      const unsigned char need = ds < 0 ? FIP_NZ_EAST : ds > 0 ? FIP_NZ_WEST : FIP_NZ_ANY;
      for (int dy = -1; dy <= 1; ++dy) {
        const int y2 = ty + dy;
        if (y2 < 0 || y2 >= a.n_ty) continue;
        if (nzc[s2 * a.n_ty + y2] & need) { act = true; break; }
      }
    }
    nzp[t] = 0;
  }
  const unsigned ba = __ballot_sync(0xffffffffu, valid && act);
  const unsigned bi = __ballot_sync(0xffffffffu, valid && !act);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { s_act[warp] = __popc(ba); s_inact[warp] = __popc(bi); }
  __syncthreads();
  int base = 0, ibase = 0, total = 0;
  for (int w = 0; w < FIP_POST_THREADS / 32; ++w) {
    if (w < warp) { base += s_act[w]; ibase += s_inact[w]; }
    total += s_act[w];
  }
  int* list = a.list[(k + 1) & 1] + chunk * FIP_PLAN_CHUNK;
  const unsigned below = (1u << lane) - 1u;
  if (valid && act) list[base + __popc(ba & below)] = t;
  if (valid && !act) list[FIP_PLAN_CHUNK - 1 - (ibase + __popc(bi & below))] = t;
  if (threadIdx.x == 0) a.chunk_cnt[(k + 1) & 1][chunk] = total;
}

// duration += dt (double += float), iteration++, buffer swap, controlTimestep for the next
// step from this step's CFL minimum, and the checks that end a batch of steps.
__device__ void fip_advance(FipCtl* ctl) {
  const int k = ctl->iteration;
  const float dt = ctl->dt;
  const float cfl = __uint_as_float(ctl->cfl_bits[k & 1]);
  ctl->cfl_bits[k & 1] = __float_as_uint(1.0f);
  ctl->last_cfl = cfl;
  const double dur = ctl->duration + (double)dt;
  ctl->duration = dur;
  ctl->iteration = k + 1;
  ctl->parity ^= 1;
  if (ctl->variable_dt) {
    float min_cfl = 42.0f;
    if (cfl < min_cfl) min_cfl = cfl;
    const float target = min_cfl * .5f;
    const float dc = 0.001f;
    float d = dt;
    if (d < target && target - d > dc) d *= 1.001f;
    else if (d > target && d - target > dc) d *= 0.99f;
    ctl->dt = d;
  }
  int reason = 0;
  if (--ctl->steps_left <= 0) reason |= FIP_STOP_BUDGET;
  if (dur >= ctl->next_save) reason |= FIP_STOP_SAVE;
  if (dur >= ctl->target) reason |= FIP_STOP_TARGET;
  if (dur >= ctl->next_sample) reason |= FIP_STOP_SAMPLE;
  if (ctl->nonfinite && ctl->stop_on_nonfinite) reason |= FIP_STOP_NONFINITE;
  if (ctl->error) reason |= FIP_STOP_ERROR;
  ctl->post_done = 0u;
  if (reason) {
    ctl->stop_reason = reason;
    __threadfence();
    ctl->stop = 1;
  }
}
)FIPSRC";

const char kPostKernelHead[] = R"FIPSRC(
extern "C" __global__ void __launch_bounds__(FIP_POST_THREADS) fip_post(const FipPostArgs a) {
  __shared__ float s_buf[4096];
  __shared__ float s_val[2];
  FipCtl* ctl = a.ctl;
  if (*((volatile int*)&ctl->stop)) return;
  const bool step_mode = (a.mode == FIP_POST_MODE_STEP);
  // the plan is for the step after k: the coming step in INIT/PLAN mode
  const int k = step_mode ? ctl->iteration : ctl->iteration - 1;
  if (blockIdx.x == 0) {
    if (a.mode == FIP_POST_MODE_PLAN) return;
    const int cur = step_mode ? (ctl->parity ^ 1) : ctl->parity;
    const double t_d = step_mode ? ctl->duration + (double)ctl->dt : ctl->duration;
    const float t = __double2float_rn(t_d);  // TimeSeries::interp(float time)
    float* h = a.h[cur];
    float* qx = a.qx[cur];
    float* qy = a.qy[cur];
    const float* sohle = a.sohle;
    const long long W = a.W, H = a.H, pitch = a.pitch;
    (void)t; (void)W; (void)H; (void)pitch; (void)h; (void)qx; (void)qy; (void)sohle; (void)s_buf; (void)s_val;
)FIPSRC";

const char kPostKernelTail[] = R"FIPSRC(
  } else {
    fip_plan(a, ctl, k, blockIdx.x - 1);
  }
  if (!step_mode) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&ctl->post_done, 1u);
    if (prev == gridDim.x - 1) {
      __threadfence();
      fip_advance(ctl);
    }
  }
}
)FIPSRC";

// Ensemble counterparts of fip_plan / fip_advance. A member whose target duration is reached
// drops out of the plan (its tiles are no longer computed) and keeps the buffer of its last
// state in final_parity; the others step on together with their own dt.
const char kEnsLib[] = R"FIPSRC(
__device__ __forceinline__ int fip_ens_member_of(const FipEnsPostArgs& a, int t) {
  int lo = 0, hi = a.n_members;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (a.members[mid].tile_base <= t) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ void fip_ens_plan(const FipEnsPostArgs& a, const FipCtl* ctl, int k, int chunk, bool step_mode) {
  __shared__ int s_act[FIP_POST_THREADS / 32];
  __shared__ int s_inact[FIP_POST_THREADS / 32];
  const int t = chunk * FIP_PLAN_CHUNK + threadIdx.x;
  const unsigned char* nzc = a.nz[k & 1];
  unsigned char* nzp = a.nz[(k + 1) & 1];
  const bool valid = t < a.n_tiles;
  bool act = false;
  if (valid) {
    const int m = fip_ens_member_of(a, t);
    const FipEnsMember M = a.members[m];
    const FipEnsCtl* mc = a.mctl + m;
    // runs in the next step: active now and, after a step, still short of its target
    bool runs = mc->active != 0;
    if (step_mode && runs) runs = (mc->duration + (double)mc->dt) < mc->target;
    const int local = t - M.tile_base;
    const int sx = local / M.n_ty, ty = local - sx * M.n_ty;
    act = a.sticky[t] || nzp[t] || ctl->force_all;
    for (int ds = -1; ds <= 1 && !act; ++ds) {  // the rule of fip_plan, within the member
      const int s2 = sx + ds;
      if (s2 < 0 || s2 >= M.n_sx) continue;
      const unsigned char need = ds < 0 ? FIP_NZ_EAST : ds > 0 ? FIP_NZ_WEST : FIP_NZ_ANY;
      for (int dy = -1; dy <= 1; ++dy) {
        const int y2 = ty + dy;
        if (y2 < 0 || y2 >= M.n_ty) continue;
        if (nzc[M.tile_base + s2 * M.n_ty + y2] & need) { act = true; break; }
      }
    }
    act = act && runs;
    nzp[t] = 0;
  }
  const unsigned ba = __ballot_sync(0xffffffffu, valid && act);
  const unsigned bi = __ballot_sync(0xffffffffu, valid && !act);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) { s_act[warp] = __popc(ba); s_inact[warp] = __popc(bi); }
  __syncthreads();
  int base = 0, ibase = 0, total = 0;
  for (int w = 0; w < FIP_POST_THREADS / 32; ++w) {
    if (w < warp) { base += s_act[w]; ibase += s_inact[w]; }
    total += s_act[w];
  }
  int* list = a.list[(k + 1) & 1] + chunk * FIP_PLAN_CHUNK;
  const unsigned below = (1u << lane) - 1u;
  if (valid && act) list[base + __popc(ba & below)] = t;
  if (valid && !act) list[FIP_PLAN_CHUNK - 1 - (ibase + __popc(bi & below))] = t;
  if (threadIdx.x == 0) a.chunk_cnt[(k + 1) & 1][chunk] = total;
}

// Whole block: every running member advances its time (double += float) and dt controller
// (controlTimestep, src/main.cpp:25-43) from its own CFL minimum; the ensemble's iteration and
// buffer parity advance once.
__device__ void fip_ens_advance(const FipEnsPostArgs& a) {
  __shared__ int s_running;
  FipCtl* ctl = a.ctl;
  const int k = ctl->iteration;
  const int new_parity = ctl->parity ^ 1;
  if (threadIdx.x == 0) s_running = 0;
  __syncthreads();
  int running = 0;
  for (int m = threadIdx.x; m < a.n_members; m += blockDim.x) {
    FipEnsCtl* mc = a.mctl + m;
    if (!mc->active) continue;
    const float dt = mc->dt;
    const float cfl = __uint_as_float(mc->cfl_bits[k & 1]);
    mc->cfl_bits[k & 1] = __float_as_uint(1.0f);
    mc->last_cfl = cfl;
    const double dur = mc->duration + (double)dt;
    mc->duration = dur;
    mc->iteration += 1;
    if (mc->variable_dt) {
      float min_cfl = 42.0f;
      if (cfl < min_cfl) min_cfl = cfl;
      const float target = min_cfl * .5f;
      const float dc = 0.001f;
      float d = dt;
      if (d < target && target - d > dc) d *= 1.001f;
      else if (d > target && d - target > dc) d *= 0.99f;
      mc->dt = d;
    }
    if (dur >= mc->target) {
      mc->active = 0;
      mc->final_parity = new_parity;
    } else {
      ++running;
    }
  }
  if (running) atomicAdd(&s_running, running);
  __syncthreads();
  if (threadIdx.x == 0) {
    ctl->iteration = k + 1;
    ctl->parity = new_parity;
    int reason = 0;
    if (--ctl->steps_left <= 0) reason |= FIP_STOP_BUDGET;
    if (s_running == 0) reason |= FIP_STOP_TARGET;
    if (ctl->nonfinite && ctl->stop_on_nonfinite) reason |= FIP_STOP_NONFINITE;
    if (ctl->error) reason |= FIP_STOP_ERROR;
    ctl->post_done = 0u;
    if (reason) {
      ctl->stop_reason = reason;
      __threadfence();
      ctl->stop = 1;
    }
  }
}
)FIPSRC";

const char kEnsKernelHead[] = R"FIPSRC(
extern "C" __global__ void __launch_bounds__(FIP_POST_THREADS) fip_ens_post(const FipEnsPostArgs a) {
  __shared__ float s_buf[4096];
  __shared__ float s_val[2];
  __shared__ int s_last;
  FipCtl* ctl = a.ctl;
  if (*((volatile int*)&ctl->stop)) return;
  const bool step_mode = (a.mode == FIP_POST_MODE_STEP);
  const int k = step_mode ? ctl->iteration : ctl->iteration - 1;
  if (blockIdx.x < a.n_members) {
    const int m = blockIdx.x;
    const FipEnsCtl* mc = a.mctl + m;
    if (a.mode != FIP_POST_MODE_PLAN && mc->active) {
      const int cur = step_mode ? (ctl->parity ^ 1) : ctl->parity;
      const double t_d = step_mode ? mc->duration + (double)mc->dt : mc->duration;
      const float t = __double2float_rn(t_d);  // TimeSeries::interp(float time)
      const long long pitch = a.pitch;
      const long long rbase = (long long)a.members[m].row_off * pitch;
      float* h = a.h[cur] + rbase;
      float* qx = a.qx[cur] + rbase;
      float* qy = a.qy[cur] + rbase;
      const float* sohle = a.sohle + rbase;
      (void)t; (void)h; (void)qx; (void)qy; (void)sohle; (void)s_buf; (void)s_val; (void)pitch;
      switch (m) {
)FIPSRC";

const char kEnsKernelTail[] = R"FIPSRC(
      default: break;
      }
    }
  } else {
    fip_ens_plan(a, ctl, k, blockIdx.x - a.n_members, step_mode);
  }
  if (!step_mode) return;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&ctl->post_done, 1u);
    s_last = (prev == gridDim.x - 1) ? 1 : 0;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    fip_ens_advance(a);
  }
}
)FIPSRC";

std::string flit(float v) {  // exact float literal
  uint32_t b;
  std::memcpy(&b, &v, 4);
  char buf[48];
  std::snprintf(buf, sizeof buf, "__int_as_float(0x%08x)", b);
  return buf;
}

const char* side_name(BcSide s) {
  switch (s) {
    case BcSide::left: return "left";
    case BcSide::right: return "right";
    case BcSide::top: return "top";
    default: return "bottom";
  }
}
const char* type_name(BcType t) {
  switch (t) {
    case BcType::z: return "z";
    case BcType::q: return "q";
    case BcType::close: return "close";
    default: return "open";
  }
}

// src_side_* (src/bc_kernel_gen.cpp:11-73): the side's cell, staggered face and inner
// neighbour of boundary cell `tid`, and the discharge arrays (normal q, lateral q_lateral)
struct SideExpr {
  const char *idx, *stag, *nb, *q, *q_lateral;
};
SideExpr side_expr(BcSide side) {
  switch (side) {
    case BcSide::right: return {"tid * pitch + W - 1", "idx - 1", "idx - 1", "qx", "qy"};
    case BcSide::left: return {"tid * pitch", "idx", "idx + 1", "qx", "qy"};
    case BcSide::top: return {"tid + (H - 1) * pitch", "idx - pitch", "idx - pitch", "qy", "qx"};
    default: return {"tid", "idx", "idx + pitch", "qy", "qx"};
  }
}

// One condition's cell loop. Cells of one condition never touch each other's cells, so each
// thread first loads the operands of 4 cells and then stores them, which lets the loads of the
// 4 cells overlap. The arithmetic is the reference's fragment (src_type_*, src/bc_kernel_gen.cpp:
// 75-137) verbatim in effect: no multiply-add pairs, IEEE sqrtf, so the same rounding.
// sign_pitch > 0: the outflow sign of a top/bottom open boundary is +-sign_pitch (the row pitch of
// the scenario's own buffers) instead of the index difference (packed ensemble rows have a wider
// pitch than the member's own buffers).
void emit_cells(std::ostream& o, const BoundaryCondition& bc, bool staggered, long long sign_pitch = 0) {
  const SideExpr e = side_expr(bc.side);
  const char* qi = staggered ? "stg[u]" : "ci[u]";
  o << "      float* const q = " << e.q << ";\n      float* const q_lateral = " << e.q_lateral << ";\n";
  o << "      (void)q_lateral;\n";
  o << "      for (long long t0 = " << bc.from << "; t0 <= " << bc.to << "; t0 += 4LL * FIP_POST_THREADS) {\n";
  o << "        long long ci[4], stg[4], nbr[4];\n        bool on[4];\n        float L0[4], L1[4], L2[4];\n        (void)L2;\n";
  o << "#pragma unroll\n        for (int u = 0; u < 4; ++u) {\n";
  o << "          const long long tid = t0 + (long long)u * FIP_POST_THREADS + threadIdx.x;\n";
  o << "          on[u] = tid <= " << bc.to << ";\n";
  o << "          const long long idx = " << e.idx << ";\n";
  o << "          ci[u] = idx;\n          stg[u] = " << e.stag << ";\n          nbr[u] = " << e.nb << ";\n";
  o << "          L0[u] = L1[u] = L2[u] = 0.f;\n";
  o << "          if (on[u]) {\n";
  switch (bc.type) {
    case BcType::z:
      if (staggered) o << "            L0[u] = sohle[ci[u]]; L1[u] = sohle[nbr[u]];\n";
      else o << "            L0[u] = sohle[ci[u]]; L1[u] = q[nbr[u]]; L2[u] = h[nbr[u]];\n";
      break;
    case BcType::q:
      o << "            L0[u] = sohle[ci[u]]; L1[u] = h[nbr[u]]; L2[u] = sohle[nbr[u]];\n";
      break;
    case BcType::close:
      o << "            L0[u] = q_lateral[nbr[u]]; L1[u] = h[nbr[u]];\n";
      break;
    case BcType::open:
      o << "            L0[u] = h[nbr[u]]; L1[u] = sohle[nbr[u]]; L2[u] = sohle[ci[u]];\n";
      break;
  }
  o << "          }\n        }\n";
  o << "#pragma unroll\n        for (int u = 0; u < 4; ++u) {\n          if (!on[u]) continue;\n";
  switch (bc.type) {
    case BcType::z:
      if (staggered)
        o << "          h[ci[u]] = fmaxf(0.f, zval - L0[u]);\n"
             "          h[nbr[u]] = fmaxf(0.f, zval - L1[u]);\n"
             "          q[stg[u]] = -0.f;\n";
      else
        o << "          const float ah = fmaxf(0.f, zval - L0[u]);\n"
             "          h[ci[u]] = ah;\n"
             "          q[ci[u]] = 0.99f * (L1[u] / fmaxf(L2[u], 0.01f)) * ah;\n";
      break;
    case BcType::q:
      o << "          float ah = zval - L0[u];\n"
           "          if (ah < 0.f) ah = 0.f;\n"
           "          q["
        << qi << "] = sqrtf(FIP_G * ah) * ah * qval;\n";
      if (staggered)
        o << "          if (ah > 0.f) {\n"
             "            const float z_neighbor = L1[u] + L2[u];\n"
             "            h[ci[u]] = fmaxf(ah / 2, z_neighbor - L0[u]);\n"
             "          }\n";
      else
        o << "          if (ah > 0.f) h[ci[u]] = fmaxf(ah / 2, L1[u] + L2[u] - L0[u]);\n";
      break;
    case BcType::close:
      o << "          q[" << qi
        << "] = 0.f;\n"
           "          q_lateral[ci[u]] = L0[u];\n"
           "          h[ci[u]] = L1[u];\n";
      break;
    case BcType::open:
      o << "          const float ah_neighbor = L0[u];\n"
           "          const float z_neighbor = ah_neighbor + L1[u];\n"
        << (sign_pitch > 0 && (bc.side == BcSide::top || bc.side == BcSide::bottom)
                ? std::string("          const float sign = (float)(") + (bc.side == BcSide::top ? "" : "-") +
                      std::to_string(sign_pitch) + "LL);\n"
                : std::string("          const float sign = (float)(ci[u] - nbr[u]);\n"))
        << "          if (ah_neighbor > 0.f) {\n"
           "            q["
        << qi
        << "] = sign * sqrtf(FIP_G * ah_neighbor) * ah_neighbor;\n"
           "            h[ci[u]] = fminf(ah_neighbor, fmaxf(0.f, z_neighbor - L2[u]));\n"
           "          }\n";
      break;
  }
  o << "        }\n      }\n";
}

}  // namespace

void bc_tile_force(const Config& cfg, TileForce* out) {
  // A condition writes, at every position from..to along its side, the side's cell, the inner
  // neighbour and the staggered face: cells within 1 of the edge. The step reads 2 cells around
  // every cell it updates, so the tiles within 3 cells of those are kept active; the margin used
  // is 4 along the side and 6 cells deep.
  constexpr int kAlong = 4, kDeep = 6;
  *out = TileForce{};
  if (cfg.bcs.size() > (size_t)kMaxForceRects) {
    out->all_band = 1;
    return;
  }
  const int W = (int)cfg.W, H = (int)cfg.H;
  for (const BoundaryCondition& bc : cfg.bcs) {
    int* r = out->rect[out->n++];
    const int a0 = bc.from - kAlong, a1 = bc.to + kAlong;
    switch (bc.side) {
      case BcSide::left: r[0] = 0; r[1] = kDeep - 1; r[2] = a0; r[3] = a1; break;
      case BcSide::right: r[0] = W - kDeep; r[1] = W - 1; r[2] = a0; r[3] = a1; break;
      case BcSide::bottom: r[0] = a0; r[1] = a1; r[2] = 0; r[3] = kDeep - 1; break;
      default: r[0] = a0; r[1] = a1; r[2] = H - kDeep; r[3] = H - 1; break;  // top
    }
  }
}

SeriesLayout layout_series(const Config& cfg) {
  SeriesLayout s;
  for (const BoundaryCondition& bc : cfg.bcs) {
    auto put = [&](const TimeSeries& ts, bool has, std::vector<long>& off, std::vector<int>& n) {
      if (!bc.is_series || !has) {
        off.push_back(-1);
        n.push_back(0);
        return;
      }
      off.push_back((long)s.data.size());
      n.push_back((int)ts.t.size());
      s.data.insert(s.data.end(), ts.t.begin(), ts.t.end());
      s.data.insert(s.data.end(), ts.v.begin(), ts.v.end());
    };
    put(bc.z_series, bc.has_z_series, s.z_off, s.z_n);
    put(bc.q_series, bc.has_q_series, s.q_off, s.q_n);
  }
  if (s.data.empty()) s.data.push_back(0.f);
  return s;
}

namespace {

// zval / qval of condition i for the current step (getZ / getQ, src/boundary_condition.cpp:50-77):
// constants for fixed values, device-side interpolation and wet sum for time series. `pitch` is
// the row pitch the generated code indexes with, `series_base` the offset of this scenario's
// tables in a.series, `dx_expr` the expression of the cell size.
void emit_condition_values(std::ostream& o, const Config& cfg, const SeriesLayout& ser, size_t i, long long pitch,
                           long long series_base, const std::string& dx_expr) {
  const BoundaryCondition& bc = cfg.bcs[i];
  if (!bc.is_series) {
    o << "      const float zval = " << flit(cfg.const_z(bc)) << ";\n";
    o << "      const float qval = " << flit(cfg.const_q(bc)) << ";\n";
    return;
  }
  if (ser.z_off[i] >= 0)
    o << "      const float zval = fip_interp_block(a.series + " << series_base + ser.z_off[i] << "L, " << ser.z_n[i]
      << ", t);\n";
  else
    o << "      const float zval = 0.f;\n";
  if (bc.type == BcType::q) {
    long long base = 0, inc = 1;
    switch (bc.side) {
      case BcSide::left: base = 0; inc = pitch; break;
      case BcSide::right: base = (long long)cfg.W - 1; inc = pitch; break;
      case BcSide::top: base = (long long)(cfg.H - 1) * pitch; inc = 1; break;
      case BcSide::bottom: base = 0; inc = 1; break;
    }
    o << "      const float wsum = fip_sum_depths(sohle, " << base << "LL, " << inc << "LL, " << bc.from << ", " << bc.to
      << ", zval, " << dx_expr << ", s_buf);\n";
    o << "      if (threadIdx.x == 0) s_val[1] = wsum;\n      __syncthreads();\n";
    o << "      const float qval = __fdiv_rn(fip_interp_block(a.series + " << series_base + ser.q_off[i] << "L, "
      << ser.q_n[i] << ", t), s_val[1]);\n";
  } else {
    o << "      const float qval = 0.f;\n";
  }
}

}  // namespace

std::string post_kernel_source(const Config& cfg, const SeriesLayout& ser, int pitch) {
  std::ostringstream o;
  o << "// generated by fip_b200 from " << cfg.yaml_path << "\n";
  o << kCtlHeader << kPostLib << kPostKernelHead;
  for (size_t i = 0; i < cfg.bcs.size(); ++i) {
    const BoundaryCondition& bc = cfg.bcs[i];
    o << "    {  // condition " << i << ": " << side_name(bc.side) << " " << type_name(bc.type) << ", cells "
      << bc.from << ".." << bc.to << (bc.is_series ? ", time series" : "") << "\n";
    emit_condition_values(o, cfg, ser, i, pitch, 0, "a.dx");
    o << "      (void)zval; (void)qval;\n";
    emit_cells(o, bc, cfg.staggered());
    o << "      __syncthreads();\n    }\n";
  }
  o << kPostKernelTail;
  return o.str();
}

std::string ensemble_post_kernel_source(const std::vector<const Config*>& cfgs, const std::vector<SeriesLayout>& sers,
                                        const std::vector<long long>& series_base,
                                        const std::vector<FipEnsMember>& members, int pitch) {
  std::ostringstream o;
  o << "// generated by fip_b200 for an ensemble of " << cfgs.size() << " scenarios\n";
  o << kCtlHeader << kPostLib << kEnsLib << kEnsKernelHead;
  for (size_t m = 0; m < cfgs.size(); ++m) {
    const Config& cfg = *cfgs[m];
    o << "      case " << m << ": {  // " << cfg.yaml_path << "\n";
    o << "        const long long W = " << cfg.W << "LL, H = " << cfg.H << "LL;\n        (void)W; (void)H;\n";
    for (size_t i = 0; i < cfg.bcs.size(); ++i) {
      const BoundaryCondition& bc = cfg.bcs[i];
      o << "    {  // condition " << i << ": " << side_name(bc.side) << " " << type_name(bc.type) << ", cells "
        << bc.from << ".." << bc.to << (bc.is_series ? ", time series" : "") << "\n";
      emit_condition_values(o, cfg, sers[m], i, pitch, series_base[m], flit(cfg.dx));
      o << "      (void)zval; (void)qval;\n";
      emit_cells(o, bc, cfg.staggered(), members[m].pitch_ref);
      o << "      __syncthreads();\n    }\n";
    }
    o << "      } break;\n";
  }
  o << kEnsKernelTail;
  return o.str();
}

int compile_post_kernel(const std::string& source, std::string* cubin, std::string* log, std::string* err) {
  nvrtcProgram prog;
  nvrtcResult r = nvrtcCreateProgram(&prog, source.c_str(), "fip_post.cu", 0, nullptr, nullptr);
  if (r != NVRTC_SUCCESS) {
    *err = std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(r);
    return -1;
  }
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--diag-suppress=177"};
  r = nvrtcCompileProgram(prog, 3, opts);
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  log->assign(log_size, '\0');
  if (log_size) nvrtcGetProgramLog(prog, &(*log)[0]);
  if (r != NVRTC_SUCCESS) {
    *err = std::string("NVRTC compile of the boundary-condition kernel failed: ") + nvrtcGetErrorString(r) + "\n" + *log;
    nvrtcDestroyProgram(&prog);
    return -1;
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  cubin->assign(n, '\0');
  nvrtcGetCUBIN(prog, &(*cubin)[0]);
  nvrtcDestroyProgram(&prog);
  return 0;
}

int build_post_kernel(const std::string& source, PostKernel* out, std::string* err, const char* entry) {
  std::string cubin;
  out->source = source;
  if (compile_post_kernel(source, &cubin, &out->log, err)) return -1;
  if (!drv::load(err)) return -1;
  CUresult cr = drv::ModuleLoadData(&out->module, cubin.data());
  if (cr != CUDA_SUCCESS) {
    *err = drv::message(cr, "cuModuleLoadData");
    return -1;
  }
  cr = drv::ModuleGetFunction(&out->fn, out->module, entry);
  if (cr != CUDA_SUCCESS) {
    *err = std::string("cuModuleGetFunction(") + entry + ") failed";
    return -1;
  }
  return 0;
}

void destroy_post_kernel(PostKernel* k) {
  if (k->module && drv::ModuleUnload) drv::ModuleUnload(k->module);
  k->module = nullptr;
  k->fn = nullptr;
}

}  // namespace fip
