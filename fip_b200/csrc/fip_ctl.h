// Device-resident control block and tile geometry shared by the stencil kernel (nvcc) and the
// NVRTC-generated post-step kernel. The build turns this file into a string literal
// (fip_ctl_str.inc) that is prepended to every generated program, so both sides agree on the
// layout by construction.
//
// One time step of the reference's simulate() (src/main.cpp:100-135) runs as two launches:
//   rmg stencil : momentum + continuity over the active tiles, CFL minimum, per-tile wet flags
//   post kernel : boundary conditions, next active-tile list, dt control, time/iteration
//                 advance and the event checks (sampling, save_state, target duration)
// All per-step scalars live here in device memory, so a captured CUDA graph of many steps needs
// no host round trip. A step whose launches see `stop != 0` does nothing; the host clears it
// after handling the event that set it.
#ifndef FIP_CTL_H
#define FIP_CTL_H

#define FIP_TILE_COLS 480      // output columns per tile (4 consumer warps x 120)
#define FIP_TILE_ROWS 32       // output rows per tile
#define FIP_SMEM_COLS 512      // staged columns per row and field: [c0-16, c0+496)
#define FIP_SMEM_X0 16         // tile column c0 sits at staged column 16
#define FIP_PLAN_CHUNK 512     // tiles planned per post-kernel block / list chunk
#define FIP_POST_THREADS 512

// per-tile flags of a state (one byte per tile): some cell of the tile is nonzero; some cell of
// its first / last few columns is (2 or 4: the stencil reaches 2 cells, so only the first and
// last two columns feed the tiles of the neighbouring strips)
#define FIP_NZ_ANY 1
#define FIP_NZ_WEST 2
#define FIP_NZ_EAST 4

// stop reasons (bit mask)
#define FIP_STOP_BUDGET 1      // the requested number of steps ran
#define FIP_STOP_SAMPLE 2      // duration >= sampling timer: sample before the next step
#define FIP_STOP_SAVE 4        // duration >= next save_state time: dump after this step
#define FIP_STOP_TARGET 8      // duration >= target duration (run-to-end mode)
#define FIP_STOP_NONFINITE 16  // a stored depth was NaN/Inf (when stop_on_nonfinite is set)
#define FIP_STOP_ERROR 32      // a device wait ran out (see `error`)

// device error codes (ctl->error)
#define FIP_DEVERR_WAIT_FULL 1    // consumer gave up waiting for a staged row
#define FIP_DEVERR_WAIT_EMPTY 2   // producer gave up waiting for a free ring slot
#define FIP_DEVERR_WAIT_DRAIN 3   // producer gave up waiting for its own copies on exit

struct FipCtl {
  double duration;      // simulated time after the last completed step (FP64 accumulator)
  double next_sample;   // sampling timer; +inf when sampling is off
  double next_save;     // next save_state time; +inf when none is left
  double target;        // target duration in run-to-end mode; +inf otherwise
  float dt;             // dt of the next step, already passed through the controller
  float last_cfl;       // CFL minimum of the last step (min with 1, like the reference's slots)
  int iteration;        // completed steps
  int parity;           // which ping-pong buffer holds the current state
  int stop;             // nonzero: launches return at once
  int stop_reason;      // FIP_STOP_* bits of the event(s) that set `stop`
  int steps_left;       // step budget of the current host request
  int variable_dt;
  int stop_on_nonfinite;
  int nonfinite;        // sticky: a stored depth was not finite
  int error;            // FIP_DEVERR_* of the first failed wait, 0 if none
  int hmax_every;       // flood-plain cadence in iterations (100 in the reference)
  int hmax_full;        // fold hmax over inactive tiles too (some initial depth < 0)
  int force_all;        // plan every tile as active (no dry-tile skipping)
  unsigned int cfl_bits[2];  // float bits of the running CFL minimum, by iteration parity
  unsigned int post_done;    // last-block-done counter of the post kernel
  int inject;                // test hook: CTA 0 of the next stencil leaves its first row unstaged once
};

#define FIP_POST_MODE_STEP 0   // after a step: BCs at duration+dt, plan, advance the control block
#define FIP_POST_MODE_INIT 1   // before the first step: BCs at duration, plan from the initial state
#define FIP_POST_MODE_PLAN 2   // plan from the current state only (after the host replaced a field)

// Argument block of the generated post kernel (passed by value; same layout on both sides).
struct FipPostArgs {
  float* h[2];
  float* qx[2];
  float* qy[2];
  const float* sohle;
  FipCtl* ctl;
  const unsigned char* sticky;
  unsigned char* nz[2];
  int* list[2];
  int* chunk_cnt[2];
  const float* series;  // time series tables: n times then n values, at per-condition offsets
  int W, H, pitch;
  int n_sx, n_ty, n_tiles, n_chunks;
  int mode;
  float dx;
  int pad_;
};

// ---- batched ensembles: many scenarios stacked in one set of pitched buffers ----
// Member m occupies rows [row_off, row_off + H) of every packed field (columns [0, W)); the rows
// between members and the columns right of W stay zero, so each member reads exactly what its
// own buffers would hold. Its tiles are [tile_base, tile_base + n_sx * n_ty) of the ensemble's
// concatenated tile list, strip-major like a single scenario.
#define FIP_ENS_MAX_MEMBERS 256

struct FipEnsMember {
  int tile_base, n_sx, n_ty;
  int W, H, row_off;
  float dx, kst_fixed, no_value;
  int pitch_ref;  // row pitch (elements) of the member's own buffers: scales top/bottom open outflow
};

// Per-member state of the ensemble's step loop (the members' counterparts of FipCtl's scalars).
struct FipEnsCtl {
  double duration;  // simulated time after the member's last step
  double target;    // the member's target duration
  float dt;         // dt of the member's next step
  float last_cfl;
  int iteration;    // steps the member ran
  int active;       // 1 while duration < target: the member steps with the ensemble
  int variable_dt;
  int final_parity; // buffer holding the member's state once it stopped
  unsigned int cfl_bits[2];
  int pad_[2];
};

// Argument block of the generated ensemble post kernel.
struct FipEnsPostArgs {
  float* h[2];
  float* qx[2];
  float* qy[2];
  const float* sohle;
  FipCtl* ctl;  // ensemble-wide: stop, parity, iteration, budget, errors
  FipEnsCtl* mctl;
  const FipEnsMember* members;
  const unsigned char* sticky;
  unsigned char* nz[2];
  int* list[2];
  int* chunk_cnt[2];
  const float* series;
  int pitch, n_members, n_tiles, n_chunks;
  int tile_cols, tile_rows, mode, pad_;
};

#endif  // FIP_CTL_H
