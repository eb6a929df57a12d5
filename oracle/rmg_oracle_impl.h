/*
 * Body of the CPU oracle, included by rmg_oracle_f64.c (REAL=double, P=ora64_) and
 * rmg_oracle_f32.c (REAL=float, P=ora32_). TEST INFRASTRUCTURE ONLY: see rmg_oracle.h.
 *
 * The scheme is restated cell by cell from the reference's rmg_kernel with the wet/dry mask off
 * (ENABLE_MASK 0), as pure functions of the input state. Two things in the kernel make that
 * restatement exact rather than approximate:
 *  - the row march and lane shuffles only ever feed the cells the kernel writes with values of
 *    real neighbours (halo lanes/rows are computed but never stored), so every stored value is
 *    the function below of the input state;
 *  - the kernel writes h, qx and qy on three different cell sets (src/kernels.cu:383-406) and
 *    never touches the rest of the output buffer, which therefore keeps whatever the ping-pong
 *    partner held two steps earlier (plus boundary-condition writes). The oracle keeps both
 *    buffers and writes exactly the same cell sets.
 * Two reference grid-size defects are outside this restatement (the reference writes halo-lane
 * garbage): W mod 28 in {2,3,5} (the W-2 column lands on a halo lane of some warp) and
 * H mod 50 in {2,3} (the H-2 row lands on a halo row of a block). Inputs must avoid them when
 * compared against the reference binary.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(P, name)

/* the reference's float constants, promoted (src/kernels.cu:23-24, src/simdata.h:358) */
#define R_DH ((REAL)0.01f)
#define R_G ((REAL)9.81f)
#define R_EPS ((REAL)10e-7f)
#define R_POW ((REAL)2.33f)

typedef struct {
  int side, type, from, to, is_series;
  float z, q;
  int nz, nq;
  float *zt, *zv, *qt, *qv;
} ora_bc_t;

typedef struct {
  double duration;
  REAL* f[4]; /* h, qx, qy (other buffer = state before the step), hmax */
} ora_dump_t;

struct ora_sim {
  int W, H;
  long pitch;
  float dx_f, dt;
  REAL dx, dxi;
  int variable_dt;
  float kst_fixed, no_value;
  float* terr_f; /* host terrain as float (h_sohle): BC values, no_data test, samples */
  REAL* terr;
  REAL* kst; /* NULL: uniform kst_fixed */
  REAL *h[2], *qx[2], *qy[2], *hmax;
  REAL *qx2c, *qy2c; /* computed (held) fluxes of the step, before the write mask */
  REAL *ux, *uy;     /* per-cell velocities of the input state (src/kernels.cu:351-354) */
  int cur;
  double duration;
  int iteration;
  float last_cfl;
  ora_bc_t* bcs;
  int nbc;
  int sampling_interval, npts;
  double sample_timer;
  int *sx, *sy, *stype;
  char* text;
  size_t text_len, text_cap;
  double* save_times;
  int nsave, save_pos;
  ora_dump_t* dumps;
  int ndump;
  int nthreads;
};

#define IDX(s, r, c) ((size_t)(r) * (size_t)(s)->W + (size_t)(c))

static inline REAL fdivw(REAL a, REAL b) { return (a == (REAL)0) ? (REAL)0 : a / b; }
/* max/min as the GPU's fmaxf/fminf: a NaN operand yields the other one, and of two zeros of
   opposite sign max gives +0 and min gives -0 (libm leaves that sign unspecified) */
static inline REAL rmax(REAL a, REAL b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a == b) return signbit(a) ? b : a;
  return a > b ? a : b;
}
static inline REAL rmin(REAL a, REAL b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a == b) return signbit(a) ? a : b;
  return a < b ? a : b;
}
static inline REAL rsqrt_(REAL a) { return sizeof(REAL) == 8 ? (REAL)sqrt(a) : (REAL)sqrtf((float)a); }
static inline REAL rpow(REAL a, REAL b) { return sizeof(REAL) == 8 ? (REAL)pow(a, b) : (REAL)powf((float)a, (float)b); }
static inline REAL rabs(REAL a) { return sizeof(REAL) == 8 ? (REAL)fabs(a) : (REAL)fabsf((float)a); }

/* field access; out-of-grid reads return 0 (never reached by a stored value, see above) */
static inline REAL gv(const struct ora_sim* s, const REAL* a, int r, int c) {
  if (r < 0 || r >= s->H || c < 0 || c >= s->W) return (REAL)0;
  return a[IDX(s, r, c)];
}

typedef struct {
  const struct ora_sim* s;
  const REAL *h, *qx, *qy;
  REAL dt, dti;
} ora_in_t;

/* ah_qx / ah_qy and the velocities (src/kernels.cu:351-354), evaluated once per cell */
static inline REAL ux_eval(const ora_in_t* in, int r, int c) {
  REAL a = rmax(rmax(R_DH, gv(in->s, in->h, r, c)), gv(in->s, in->h, r, c + 1));
  return fdivw(gv(in->s, in->qx, r, c), a);
}
static inline REAL uy_eval(const ora_in_t* in, int r, int c) {
  REAL a = rmax(rmax(R_DH, gv(in->s, in->h, r, c)), gv(in->s, in->h, r + 1, c));
  return fdivw(gv(in->s, in->qy, r, c), a);
}
static inline REAL ux_at(const ora_in_t* in, int r, int c) { return gv(in->s, in->s->ux, r, c); }
static inline REAL uy_at(const ora_in_t* in, int r, int c) { return gv(in->s, in->s->uy, r, c); }
/* compute_rmg_fx (src/kernels.cu:56-63) */
static inline REAL fx_at(const ora_in_t* in, int r, int c) {
  REAL uw = ux_at(in, r, c - 1), ui = ux_at(in, r, c);
  if (uw + ui > 0) return gv(in->s, in->qx, r, c - 1) * uw;
  return gv(in->s, in->qx, r, c) * ui;
}
/* compute_rmg_fy (src/kernels.cu:45-54) */
static inline REAL fy_at(const ora_in_t* in, int r, int c) {
  REAL ui = ux_at(in, r, c), un = ux_at(in, r + 1, c);
  REAL uh = (ui + un) * (REAL)0.5f;
  if (ui + un > 0) return gv(in->s, in->qy, r, c) * uh;
  return gv(in->s, in->qy, r, c + 1) * uh;
}
/* compute_rmg_gx (src/kernels.cu:35-43) */
static inline REAL gx_at(const ora_in_t* in, int r, int c) {
  REAL ui = uy_at(in, r, c), ue = uy_at(in, r, c + 1);
  REAL uh = (ui + ue) * (REAL)0.5f;
  if (ui + ue > 0) return gv(in->s, in->qx, r, c) * uh;
  return gv(in->s, in->qx, r + 1, c) * uh;
}
/* compute_rmg_gy (src/kernels.cu:65-73), called for the cell itself */
static inline REAL gy_at(const ora_in_t* in, int r, int c) {
  REAL ui = uy_at(in, r, c), us = uy_at(in, r - 1, c);
  if (ui + us > 0) return gv(in->s, in->qy, r - 1, c) * us;
  return gv(in->s, in->qy, r, c) * ui;
}
static inline REAL kst_at(const struct ora_sim* s, int r, int c) {
  return s->kst ? s->kst[IDX(s, r, c)] : (REAL)s->kst_fixed;
}
/* Strickler friction factor, discharges not velocities (src/kernels.cu:90-94, :117-121) */
static inline REAL reib_of(REAL dt, REAL k, REAL ux, REAL uy, REAL inv) {
  if (ux == 0 && uy == 0) return 0;
  return dt * R_G / (k * k) * rsqrt_(ux * ux + uy * uy) * rpow(inv, R_POW);
}
/* compute_rmg_qx (src/kernels.cu:75-100) */
static REAL fqx_at(const ora_in_t* in, int r, int c) {
  const struct ora_sim* s = in->s;
  REAL dxi = s->dxi, dt = in->dt;
  REAL dfx = (fx_at(in, r, c + 1) - fx_at(in, r, c)) * dxi;
  REAL dgx = (gx_at(in, r, c) - gx_at(in, r - 1, c)) * dxi;
  REAL hi = gv(s, in->h, r, c), he = gv(s, in->h, r, c + 1);
  REAL a = (hi + he) * (REAL)0.5f;
  a = rmax((REAL)0, a);
  REAL dhg = a * R_G * (-gv(s, s->terr, r, c + 1) + gv(s, s->terr, r, c)) * dxi;
  REAL dhx = ((REAL)0.5f * R_G * he * he - (REAL)0.5f * R_G * hi * hi) * dxi;
  a = rmax(a, R_DH);
  REAL inv = (REAL)1 / a;
  REAL ux = gv(s, in->qx, r, c);
  REAL uy = (gv(s, in->qy, r, c) + gv(s, in->qy, r, c + 1) + gv(s, in->qy, r - 1, c) +
             gv(s, in->qy, r - 1, c + 1)) * (REAL)0.25f;
  REAL reib = reib_of(dt, kst_at(s, r, c), ux, uy, inv);
  REAL qn = fdivw(ux + dt * (-dfx - dgx - dhx + dhg), (REAL)1 + reib);
  qn = rmin(qn, hi * in->dti * s->dx * (REAL)0.25f);
  qn = rmax(qn, -he * in->dti * s->dx * (REAL)0.25f);
  return qn;
}
/* compute_rmg_qy (src/kernels.cu:102-127) */
static REAL fqy_at(const ora_in_t* in, int r, int c) {
  const struct ora_sim* s = in->s;
  REAL dxi = s->dxi, dt = in->dt;
  REAL dgy = (gy_at(in, r + 1, c) - gy_at(in, r, c)) * dxi;
  REAL dfy = (fy_at(in, r, c) - fy_at(in, r, c - 1)) * dxi;
  REAL hi = gv(s, in->h, r, c), hn = gv(s, in->h, r + 1, c);
  REAL a = (hi + hn) * (REAL)0.5f;
  a = rmax((REAL)0, a);
  REAL dhg = a * R_G * (gv(s, s->terr, r, c) - gv(s, s->terr, r + 1, c)) * dxi;
  REAL dhy = ((REAL)0.5f * R_G * hn * hn - (REAL)0.5f * R_G * hi * hi) * dxi;
  a = rmax(a, R_DH);
  REAL inv = (REAL)1 / a;
  REAL ux = (gv(s, in->qx, r, c) + gv(s, in->qx, r + 1, c) + gv(s, in->qx, r, c - 1) +
             gv(s, in->qx, r + 1, c - 1)) * (REAL)0.25f;
  REAL uy = gv(s, in->qy, r, c);
  REAL reib = reib_of(dt, kst_at(s, r, c), ux, uy, inv);
  REAL qn = fdivw(uy + dt * (-dgy - dfy - dhy + dhg), (REAL)1 + reib);
  qn = rmin(qn, hi * in->dti * s->dx * (REAL)0.25f);
  qn = rmax(qn, -hn * in->dti * s->dx * (REAL)0.25f);
  return qn;
}

/* One launch of rmg_kernel (mask off) followed by the pointer swap. Returns the CFL minimum
   over the stored wet cells, initialised to 1 like each warp's dt_cfl_min (:287). */
static float ora_step(struct ora_sim* s) {
  const int W = s->W, H = s->H, in_b = s->cur, out_b = 1 - s->cur;
  ora_in_t in = {s, s->h[in_b], s->qx[in_b], s->qy[in_b], (REAL)s->dt, (REAL)1 / (REAL)s->dt};
  REAL* ho = s->h[out_b];
  REAL* qxo = s->qx[out_b];
  REAL* qyo = s->qy[out_b];
  /* pass 0: velocities of every cell of the input state */
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
  for (int r = 0; r < H; ++r)
    for (int c = 0; c < W; ++c) {
      s->ux[IDX(s, r, c)] = ux_eval(&in, r, c);
      s->uy[IDX(s, r, c)] = uy_eval(&in, r, c);
    }
  /* pass 1: the fluxes the kernel computes, with the boundary-face holds (:373-376) */
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
  for (int r = 0; r <= H - 2; ++r) {
    for (int c = 0; c <= W - 2; ++c) {
      if (r >= 1) s->qx2c[IDX(s, r, c)] = (c == 0 || c == W - 2) ? in.qx[IDX(s, r, c)] : fqx_at(&in, r, c);
      if (c >= 1) s->qy2c[IDX(s, r, c)] = (r == 0 || r == H - 2) ? in.qy[IDX(s, r, c)] : fqy_at(&in, r, c);
    }
  }
  /* pass 2: continuity, stores on the kernel's cell sets, CFL (:378-406) */
  double cfl = 1.0;
#pragma omp parallel for schedule(static) reduction(min : cfl) num_threads(s->nthreads)
  for (int r = 1; r <= H - 2; ++r) {
    for (int c = 1; c <= W - 2; ++c) {
      if (s->terr_f[IDX(s, r, c)] == s->no_value) continue;
      REAL qx2 = s->qx2c[IDX(s, r, c)], qx2w = s->qx2c[IDX(s, r, c - 1)];
      REAL qy2 = s->qy2c[IDX(s, r, c)], qy2s = s->qy2c[IDX(s, r - 1, c)];
      REAL h2 = in.h[IDX(s, r, c)] - in.dt * s->dxi * ((qx2 - qx2w) + (qy2 - qy2s));
      ho[IDX(s, r, c)] = h2;
      if (h2 > R_EPS) {
        REAL umax = rmax(rabs(uy_at(&in, r, c)),
                         rmax(rabs(uy_at(&in, r - 1, c)), rmax(rabs(ux_at(&in, r, c)), rabs(ux_at(&in, r, c - 1)))));
        REAL d = s->dx / (rsqrt_(R_G * h2) + umax);
        if ((double)d < cfl) cfl = (double)d;
      }
      if (r >= 2 && r <= H - 3 && c <= W - 3) qxo[IDX(s, r, c)] = qx2;
      if (r <= H - 3 && c >= 2 && c <= W - 3) qyo[IDX(s, r, c)] = qy2;
    }
  }
  s->cur = out_b;
  return (float)cfl;
}

/* TimeSeries::interp (src/timeseries.cpp:14-26): first key >= time, clamped ends */
static REAL ts_interp(int n, const float* t, const float* v, float time) {
  int lo = 0, hi = n; /* lower_bound */
  while (lo < hi) {
    int mid = (lo + hi) / 2;
    if (t[mid] < time) lo = mid + 1; else hi = mid;
  }
  if (lo == 0) return (REAL)v[0];
  if (lo == n) return (REAL)v[n - 1];
  REAL dt = (REAL)t[lo] - (REAL)t[lo - 1];
  REAL f = ((REAL)time - (REAL)t[lo - 1]) / dt;
  return f * (REAL)v[lo] + ((REAL)1 - f) * (REAL)v[lo - 1];
}

/* BoundaryCondition::getIdxForNthBoundaryCell (src/boundary_condition.cpp:20-40), as (row, col) */
static void bc_cell(const struct ora_sim* s, int side, int n, int* r, int* c) {
  switch (side) {
    case ORA_SIDE_LEFT: *r = n; *c = 0; break;
    case ORA_SIDE_RIGHT: *r = n; *c = s->W - 1; break;
    case ORA_SIDE_TOP: *r = s->H - 1; *c = n; break;
    default: *r = 0; *c = n; break;
  }
}

/* sumWaterDepths (src/boundary_condition.cpp:6-18): host terrain, exclusive `to` */
static REAL sum_water_depths(const struct ora_sim* s, const ora_bc_t* b, REAL z) {
  REAL sum = 0;
  for (int n = b->from; n < b->to; ++n) {
    int r, c;
    bc_cell(s, b->side, n, &r, &c);
    REAL ah = z - (REAL)s->terr_f[IDX(s, r, c)];
    if (ah < (REAL)0.01f) ah = 0;
    sum += rsqrt_(R_G * ah) * ah;
  }
  return sum * s->dx;
}

/* launchBoundaryConditionKernel (src/main.cpp:85-98) with the generated randbed applied one
   condition after the other, in configuration order */
static void ora_apply_bcs(struct ora_sim* s) {
  REAL* h = s->h[s->cur];
  REAL* qx = s->qx[s->cur];
  REAL* qy = s->qy[s->cur];
  const float t = (float)s->duration;
  for (int i = 0; i < s->nbc; ++i) {
    const ora_bc_t* b = &s->bcs[i];
    REAL zval, qval;
    if (b->is_series) {
      zval = b->nz ? ts_interp(b->nz, b->zt, b->zv, t) : 0;
      qval = (b->type == ORA_BC_Q) ? ts_interp(b->nq, b->qt, b->qv, t) / sum_water_depths(s, b, zval) : 0;
    } else {
      zval = (REAL)b->z;
      qval = (b->type == ORA_BC_Q) ? (REAL)b->q / sum_water_depths(s, b, zval) : (REAL)b->q;
    }
    const int vertical = (b->side == ORA_SIDE_TOP || b->side == ORA_SIDE_BOTTOM);
    REAL* q = vertical ? qy : qx;
    REAL* ql = vertical ? qx : qy;
    for (int tid = b->from; tid <= b->to; ++tid) {
      int r, c, rn, cn, rs, cs;
      bc_cell(s, b->side, tid, &r, &c);
      switch (b->side) { /* src_side_* (src/bc_kernel_gen.cpp:11-73) */
        case ORA_SIDE_LEFT: rn = r; cn = 1; rs = r; cs = 0; break;
        case ORA_SIDE_RIGHT: rn = r; cn = s->W - 2; rs = r; cs = s->W - 2; break;
        case ORA_SIDE_TOP: rn = s->H - 2; cn = c; rs = s->H - 2; cs = c; break;
        default: rn = 1; cn = c; rs = 0; cs = c; break;
      }
      size_t idx = IDX(s, r, c), nb = IDX(s, rn, cn), st = IDX(s, rs, cs);
      REAL sidx = (REAL)s->terr_f[idx], snb = (REAL)s->terr_f[nb];
      switch (b->type) {
        case ORA_BC_Z: /* src_type_z_staggered :81-86 */
          h[idx] = rmax(0, zval - sidx);
          h[nb] = rmax(0, zval - snb);
          q[st] = -(REAL)0;
          break;
        case ORA_BC_Q: { /* src_type_q_staggered :97-105 */
          REAL ah = zval - sidx;
          if (ah < 0) ah = 0;
          q[st] = rsqrt_(R_G * ah) * ah * qval;
          if (ah > 0) {
            REAL znb = h[nb] + snb;
            h[idx] = rmax(ah / 2, znb - sidx);
          }
          break;
        }
        case ORA_BC_CLOSE: /* src_type_close_staggered :113-117 */
          q[st] = 0;
          ql[idx] = ql[nb];
          h[idx] = h[nb];
          break;
        default: { /* src_type_open_staggered :129-137; sign = idx - idx_neighbor in the
                      pitched linear index, i.e. +-1 horizontally and +-pitch vertically */
          REAL ahn = h[nb];
          REAL znb = ahn + snb;
          REAL sign = (REAL)(float)(b->side == ORA_SIDE_LEFT ? -1 : b->side == ORA_SIDE_RIGHT ? 1
                                    : b->side == ORA_SIDE_TOP ? s->pitch : -s->pitch);
          if (ahn > 0) {
            q[st] = sign * rsqrt_(R_G * ahn) * ahn;
            h[idx] = rmin(ahn, rmax(0, znb - sidx));
          }
          break;
        }
      }
    }
  }
}

/* controlTimestep (src/main.cpp:25-43); the CFL slots hold the last step's minimum */
static void ora_control(struct ora_sim* s) {
  float min_cfl = 42.0f;
  if (s->last_cfl < min_cfl) min_cfl = s->last_cfl;
  float target = min_cfl * .5f;
  const float dc = 0.001f;
  if (s->dt < target && target - s->dt > dc) s->dt *= 1.001f;
  else if (s->dt > target && s->dt - target > dc) s->dt *= 0.99f;
}

static void text_append(struct ora_sim* s, const char* str) {
  size_t n = strlen(str);
  if (s->text_len + n + 1 > s->text_cap) {
    s->text_cap = (s->text_len + n + 1) * 2 + 256;
    s->text = (char*)realloc(s->text, s->text_cap);
  }
  memcpy(s->text + s->text_len, str, n + 1);
  s->text_len += n;
}

/* sample (src/main.cpp:53-83): "duration;v1;v2;...;\n", default ostream formatting (%g) */
static void ora_sample(struct ora_sim* s) {
  char buf[64];
  snprintf(buf, sizeof buf, "%g;", s->duration);
  text_append(s, buf);
  for (int k = 0; k < s->npts; ++k) {
    size_t i = IDX(s, s->sy[k], s->sx[k]);
    float v;
    switch (s->stype[k]) {
      case 0: v = (float)s->h[s->cur][i] + s->terr_f[i]; break; /* z = h + host terrain */
      case 1: v = (float)s->h[s->cur][i]; break;
      case 2: v = (float)s->qx[s->cur][i]; break;
      default: v = (float)s->qy[s->cur][i]; break;
    }
    snprintf(buf, sizeof buf, "%g;", (double)v);
    text_append(s, buf);
  }
  text_append(s, "\n");
}

static REAL* ora_alloc(size_t n) { return (REAL*)calloc(n ? n : 1, sizeof(REAL)); }

/* dumpDeviceBuffers (src/main.cpp:180-202): d_h2/d_qx2/d_qy2 after the swap, i.e. the state
   before the step that crossed the save time, plus hmax */
static void ora_dump(struct ora_sim* s) {
  size_t n = (size_t)s->W * s->H;
  s->dumps = (ora_dump_t*)realloc(s->dumps, sizeof(ora_dump_t) * (s->ndump + 1));
  ora_dump_t* d = &s->dumps[s->ndump++];
  d->duration = s->duration;
  const REAL* src[4] = {s->h[1 - s->cur], s->qx[1 - s->cur], s->qy[1 - s->cur], s->hmax};
  for (int f = 0; f < 4; ++f) {
    d->f[f] = ora_alloc(n);
    memcpy(d->f[f], src[f], n * sizeof(REAL));
  }
}

/* simulate (src/main.cpp:100-135) */
static void ora_simulate_once(struct ora_sim* s) {
  if (s->variable_dt) ora_control(s);
  if (s->duration >= s->sample_timer && s->sampling_interval > 0) {
    s->sample_timer += s->sampling_interval;
    ora_sample(s);
  }
  if (s->iteration == 0) ora_apply_bcs(s);
  s->last_cfl = ora_step(s);
  s->duration += s->dt;
  s->iteration++;
  ora_apply_bcs(s);
  if (s->iteration % 100 == 0) {
    size_t n = (size_t)s->W * s->H;
    const REAL* h = s->h[s->cur];
    for (size_t i = 0; i < n; ++i) s->hmax[i] = rmax(s->hmax[i], h[i]);
  }
  if (s->save_pos < s->nsave && s->duration >= s->save_times[s->save_pos]) {
    s->save_pos++;
    ora_dump(s);
  }
}

ora_sim* FN(new_sim)(int W, int H, long pitch_elems, float dx, float dt, int variable_dt, float kst_fixed,
                     float no_value, const float* terrain, const float* h0, const float* qx0,
                     const float* qy0, const float* kst_var) {
  if (W < 4 || H < 4) return NULL;
  struct ora_sim* s = (struct ora_sim*)calloc(1, sizeof(struct ora_sim));
  size_t n = (size_t)W * H;
  s->W = W; s->H = H; s->pitch = pitch_elems;
  s->dx_f = dx; s->dx = (REAL)dx; s->dxi = (REAL)1 / (REAL)dx; s->dt = dt;
  s->variable_dt = variable_dt; s->kst_fixed = kst_fixed; s->no_value = no_value;
  s->terr_f = (float*)malloc(n * sizeof(float));
  memcpy(s->terr_f, terrain, n * sizeof(float));
  s->terr = ora_alloc(n);
  for (size_t i = 0; i < n; ++i) s->terr[i] = (REAL)terrain[i];
  if (kst_var) {
    s->kst = ora_alloc(n);
    for (size_t i = 0; i < n; ++i) s->kst[i] = (REAL)kst_var[i];
  }
  for (int b = 0; b < 2; ++b) {
    s->h[b] = ora_alloc(n); s->qx[b] = ora_alloc(n); s->qy[b] = ora_alloc(n);
    for (size_t i = 0; i < n; ++i) {
      s->h[b][i] = h0 ? (REAL)h0[i] : 0;
      s->qx[b][i] = qx0 ? (REAL)qx0[i] : 0;
      s->qy[b][i] = qy0 ? (REAL)qy0[i] : 0;
    }
  }
  s->hmax = ora_alloc(n);
  memcpy(s->hmax, s->h[0], n * sizeof(REAL));
  s->qx2c = ora_alloc(n);
  s->qy2c = ora_alloc(n);
  s->ux = ora_alloc(n);
  s->uy = ora_alloc(n);
  s->last_cfl = 1.0f; /* initDeviceBuffers fills the CFL slots with 1 (src/simdata.cpp:91-94) */
  s->nthreads = 1;
  return s;
}

static float* dup_f(int n, const float* a) {
  if (!n || !a) return NULL;
  float* r = (float*)malloc(sizeof(float) * n);
  memcpy(r, a, sizeof(float) * n);
  return r;
}

int FN(add_bc)(ora_sim* s, int side, int type, int from, int to, int is_series, float z, float q, int nz,
               const float* zt, const float* zv, int nq, const float* qt, const float* qv) {
  int len = (side == ORA_SIDE_LEFT || side == ORA_SIDE_RIGHT) ? s->H : s->W;
  if (from < 0 || to >= len || from > to + 1) return -1;
  if (is_series && type == ORA_BC_Z && nz <= 0) return -2;
  if (is_series && type == ORA_BC_Q && (nz <= 0 || nq <= 0)) return -2;
  s->bcs = (ora_bc_t*)realloc(s->bcs, sizeof(ora_bc_t) * (s->nbc + 1));
  ora_bc_t* b = &s->bcs[s->nbc++];
  memset(b, 0, sizeof *b);
  b->side = side; b->type = type; b->from = from; b->to = to; b->is_series = is_series;
  b->z = z; b->q = q; b->nz = nz; b->nq = nq;
  b->zt = dup_f(nz, zt); b->zv = dup_f(nz, zv); b->qt = dup_f(nq, qt); b->qv = dup_f(nq, qv);
  return 0;
}

void FN(set_sampling)(ora_sim* s, int interval, int npts, const int* xs, const int* ys, const int* types) {
  s->sampling_interval = interval;
  s->sample_timer = 0;
  s->npts = npts;
  s->sx = (int*)realloc(s->sx, sizeof(int) * (npts ? npts : 1));
  s->sy = (int*)realloc(s->sy, sizeof(int) * (npts ? npts : 1));
  s->stype = (int*)realloc(s->stype, sizeof(int) * (npts ? npts : 1));
  for (int k = 0; k < npts; ++k) { s->sx[k] = xs[k]; s->sy[k] = ys[k]; s->stype[k] = types[k]; }
}

static int cmp_d(const void* a, const void* b) {
  double x = *(const double*)a, y = *(const double*)b;
  return (x > y) - (x < y);
}
void FN(set_save_times)(ora_sim* s, int n, const double* times) {
  s->save_times = (double*)realloc(s->save_times, sizeof(double) * (n ? n : 1));
  memcpy(s->save_times, times, sizeof(double) * n);
  qsort(s->save_times, n, sizeof(double), cmp_d);
  s->nsave = n;
  s->save_pos = 0;
}

void FN(set_threads)(ora_sim* s, int n) { s->nthreads = n > 0 ? n : 1; }

int FN(simulate)(ora_sim* s, int n) {
  for (int i = 0; i < n; ++i) ora_simulate_once(s);
  return s->iteration;
}

/* the headless main loop: while (duration < target_duration) simulate(); (src/main.cpp:243) */
int FN(run_to)(ora_sim* s, double target) {
  while (s->duration < target) ora_simulate_once(s);
  return s->iteration;
}

double FN(duration)(const ora_sim* s) { return s->duration; }
float FN(dt)(const ora_sim* s) { return s->dt; }
int FN(iteration)(const ora_sim* s) { return s->iteration; }
float FN(last_cfl)(const ora_sim* s) { return s->last_cfl; }

double FN(volume)(const ora_sim* s) {
  size_t n = (size_t)s->W * s->H;
  double v = 0;
  for (size_t i = 0; i < n; ++i) v += (double)s->h[s->cur][i];
  return v * (double)s->dx_f * (double)s->dx_f;
}

static void to_float(size_t n, const REAL* a, float* out) {
  for (size_t i = 0; i < n; ++i) out[i] = (float)a[i];
}

void FN(get_field)(const ora_sim* s, int which, float* out) {
  size_t n = (size_t)s->W * s->H;
  int o = 1 - s->cur;
  const REAL* src = which == ORA_F_H ? s->h[s->cur] : which == ORA_F_QX ? s->qx[s->cur]
                    : which == ORA_F_QY ? s->qy[s->cur] : which == ORA_F_H_OTHER ? s->h[o]
                    : which == ORA_F_QX_OTHER ? s->qx[o] : which == ORA_F_QY_OTHER ? s->qy[o] : s->hmax;
  to_float(n, src, out);
}

const char* FN(sample_text)(const ora_sim* s) { return s->text ? s->text : ""; }
int FN(dump_count)(const ora_sim* s) { return s->ndump; }
double FN(dump_duration)(const ora_sim* s, int k) { return s->dumps[k].duration; }
void FN(dump_field)(const ora_sim* s, int k, int which, float* out) {
  to_float((size_t)s->W * s->H, s->dumps[k].f[which], out);
}

void FN(free_sim)(ora_sim* s) {
  if (!s) return;
  free(s->terr_f); free(s->terr); free(s->kst); free(s->hmax); free(s->qx2c); free(s->qy2c); free(s->ux); free(s->uy);
  for (int b = 0; b < 2; ++b) { free(s->h[b]); free(s->qx[b]); free(s->qy[b]); }
  for (int i = 0; i < s->nbc; ++i) {
    free(s->bcs[i].zt); free(s->bcs[i].zv); free(s->bcs[i].qt); free(s->bcs[i].qv);
  }
  free(s->bcs); free(s->sx); free(s->sy); free(s->stype); free(s->text); free(s->save_times);
  for (int k = 0; k < s->ndump; ++k)
    for (int f = 0; f < 4; ++f) free(s->dumps[k].f[f]);
  free(s->dumps);
  free(s);
}
