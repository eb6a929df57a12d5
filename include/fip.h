/*
 * fip_b200 -- C ABI of the B200 (sm_100a) slim shallow-water solver.
 *
 * Drop-in for the simulation loop of fip (fip-ems/fip). The reference has no library
 * interface: its path sits behind globals in namespace SimData (src/simdata.h:333-373) and the
 * functions cited below. Each entry point here replaces the reference code named in its
 * comment, with the same inputs (the YAML parameter file and raw float32 grids of README.md:46-64)
 * and the same outputs (sampling CSV on stdout, save_state dump files).
 *
 * Conventions: every function returns FIP_OK (0) or a negative FIP_ERR_* code and never exits
 * the process; fip_last_error() gives the message of the last failure on the calling thread.
 * A handle owns all device and host memory and one CUDA stream; handles are independent, and a
 * handle is used from one thread at a time. Grids are row-major W x H float32 (row = y, north =
 * +1 row; col = x, east = +1), unpitched on the host side.
 */
#ifndef FIP_B200_FIP_H
#define FIP_B200_FIP_H

#ifdef __cplusplus
extern "C" {
#endif

#define FIP_OK 0
#define FIP_ERR_CONFIG -1          /* invalid parameter file (the reference prints "Config error: ...") */
#define FIP_ERR_IO -2              /* missing or short input file, unwritable dump */
#define FIP_ERR_CUDA -3            /* CUDA runtime / driver error */
#define FIP_ERR_NVRTC -4           /* boundary-condition kernel failed to compile */
#define FIP_ERR_NONFINITE -5       /* a stored depth became NaN/Inf (only with stop_on_nonfinite) */
#define FIP_ERR_DEVICE_TIMEOUT -6  /* a bounded device-side wait ran out; the handle is unusable */
#define FIP_ERR_ARG -7             /* bad argument */

/* fields for fip_get_field */
#define FIP_FIELD_H 0        /* water depth of the current state (d_h1) */
#define FIP_FIELD_QX 1       /* discharge on the east face of each cell (d_qx1) */
#define FIP_FIELD_QY 2       /* discharge on the north face (d_qy1) */
#define FIP_FIELD_HMAX 3     /* flood-plain (maximum depth) map (d_hmax) */
#define FIP_FIELD_H_PREV 4   /* the ping-pong partner buffers (d_h2, d_qx2, d_qy2): the state */
#define FIP_FIELD_QX_PREV 5  /*   before the last step, except cells the step does not write */
#define FIP_FIELD_QY_PREV 6
#define FIP_FIELD_TERRAIN 7  /* d_sohle */
#define FIP_FIELD_Z 8        /* water level h + terrain */

typedef struct fip_handle fip_handle;

typedef struct {
  int device;               /* CUDA device ordinal (default 0) */
  int use_graphs;           /* run batches of steps as captured CUDA graphs (default 1) */
  int all_tiles;            /* compute every tile every step, no dry-tile skipping (default 0) */
  int stop_on_nonfinite;    /* fip_step/fip_run return FIP_ERR_NONFINITE at the first NaN/Inf depth */
  int quiet;                /* write no sampling CSV and no loader warnings (default 0: stdout and
                               stderr, like the reference; errors are always reported) */
  const char* sample_path;  /* write the sampling CSV to this file instead of stdout (NULL) */
} fip_options;

typedef struct {
  int W, H;
  int pitch;                /* device row pitch in elements (cudaMallocPitch, like the reference) */
  int n_tiles;              /* 480 x 32-cell tiles of the domain */
  int active_tiles;         /* tiles computed by the next step */
  int iteration;
  double duration;
  float dt;
  float last_cfl;           /* CFL minimum of the last step (<= 1) */
  int nonfinite;            /* a stored depth has been NaN/Inf */
} fip_info_t;

void fip_default_options(fip_options* opt);

/* SimData::loadSimData + initDeviceBuffers (src/simdata.cpp:238-310, :54-96) and
 * BoundaryConditionKernel::generate (src/bc_kernel_gen.cpp:154-192); also prints the sampling
 * header like main() (src/main.cpp:225-226). */
int fip_init(const char* yaml_path, fip_handle** out);
int fip_init_ex(const char* yaml_path, const fip_options* opt, fip_handle** out);

/* n_steps calls of simulate() (src/main.cpp:100-135): dt control, sampling, compute kernel
 * (launchComputeKernel, src/kernels.cu:441-455), boundary conditions
 * (launchBoundaryConditionKernel, src/main.cpp:85-98), flood plains every 100 iterations
 * (launchFloodPlainKernel, src/kernels.cu:457-463) and save_state dumps. */
int fip_step(fip_handle* h, int n_steps);

/* The headless loop of main(): while (duration < target_duration) simulate();
 * (src/main.cpp:243-246). */
int fip_run(fip_handle* h);

/* dumpDeviceBuffers (src/main.cpp:180-202): <prefix>_{ah,qx,qy,flood_plains}_<int(duration)>_<UTC
 * %Y-%m-%d-%H-%M>, each 2 x size_t (W, H) + W*H float32, of the buffers the reference dumps (the
 * ping-pong partners, i.e. the state before the last step) and hmax. prefix NULL = the YAML name. */
int fip_save(fip_handle* h, const char* prefix_or_null);

/* Same file format, of the current state (d_h1, d_qx1, d_qy1) and hmax; no counterpart in the
 * reference (its dumps always hold the state before the last step). */
int fip_save_current(fip_handle* h, const char* prefix_or_null);

/* sample (src/main.cpp:53-83): one "duration;v1;v2;...;" row of the configured points now. */
int fip_sample(fip_handle* h);

/* FP64 volume sum(h) * dx^2 of the current state (the commented-out volume check of
 * src/main.cpp:139-149, on the device). */
int fip_volume(fip_handle* h, double* out);

/* Copies one field (FIP_FIELD_*) into a caller-provided host buffer of W*H floats
 * (dumpDeviceBuffer, src/main.cpp:170-178). */
int fip_get_field(fip_handle* h, int field, float* host_out);

/* Replaces one field of the current state (FIP_FIELD_H, _QX or _QY) from a host buffer of W*H
 * floats, in both ping-pong buffers like initDeviceBuffers does for the initial state
 * (src/simdata.cpp:82-88); the active tiles are re-planned before the next step. Pinned host
 * memory lets the copy run at the host link's speed. A negative depth in an FIP_FIELD_H upload
 * switches the max-depth fold to the whole grid, as a negative initial depth does at fip_init
 * (checked on the device copy). Returns once the copy is complete, so the caller may reuse the
 * buffer. No counterpart in the reference (which restarts only from files at start-up). */
int fip_set_field(fip_handle* h, int field, const float* host_src);

/* Pipelined state exchange with the host (no counterpart in the reference): for a host that
 * replaces the whole state (h, qx, qy) from its own buffers, runs some steps and reads the state
 * back, over and over, with inputs that do not depend on the previous outputs (restarts,
 * replayed forcing). The host-device copies overlap the steps: the upload of the next state and
 * the download of the last one run on two copy streams of the handle while the steps run.
 *   fip_stage_state: queues the upload of a state (three W x H host grids; pinned memory lets the
 *     copy run at the host link's speed) into one of two staging slots and returns at once. The
 *     host buffers must stay unchanged until the fip_step_exchange that takes the state returns.
 *     At most two states can wait (FIP_ERR_ARG beyond that).
 *   fip_step_exchange: makes the oldest staged state (if any) the current state, exactly as
 *     fip_set_field of the three fields does, runs n_steps steps (fip_step), and queues the
 *     download of the resulting state into the three host buffers (all NULL: no download). It
 *     returns once the steps are done; the downloads of a call are complete when the next call
 *     returns or after fip_exchange_wait.
 *   fip_exchange_wait: waits for every queued copy. */
int fip_stage_state(fip_handle* h, const float* h_src, const float* qx_src, const float* qy_src);
int fip_step_exchange(fip_handle* h, int n_steps, float* h_dst, float* qx_dst, float* qy_dst);
int fip_exchange_wait(fip_handle* h);

/* duration (s, FP64), dt of the next step, completed iterations (SimData::duration/dt/iteration). */
int fip_time(fip_handle* h, double* duration, float* dt, int* iteration);

int fip_info(fip_handle* h, fip_info_t* out);

/* Device time of the two kernels of a step, measured with CUDA events around each launch of
 * n_steps eager (not graph) steps: average ms per launch. No counterpart in the reference. */
int fip_profile_steps(fip_handle* h, int n_steps, float* stencil_ms, float* post_ms);

/* n_steps steps as one CUDA graph, as the step loop runs them, timed with events on the
 * handle's stream: total device ms of the n steps. When stencil_ms or post_ms is given, n_steps
 * more steps run as a second graph with an event record around every launch (which keeps each
 * launch from overlapping the one before it): the average ms per launch of the stencil and of
 * the post kernel (the gap between launches included). Sampling, dumps and the target duration
 * are not checked during these steps (the state advances normally otherwise). No counterpart
 * in the reference. */
int fip_step_timed(fip_handle* h, int n_steps, float* total_ms, float* stencil_ms, float* post_ms);

/* Exact-resume checkpoint (replaces the reference's restart through save_state dumps fed back as
 * z/qx/qy inputs with offset 16, src/main.cpp:154-202 and src/simdata.cpp:266-274, which loses
 * time, dt, hmax and the ping-pong partner and reads the dumped depth as a level). Writes the
 * current and partner h/qx/qy buffers, hmax, simulated time, dt, iteration, sampling timer and
 * save_state position to one file. */
int fip_checkpoint(fip_handle* h, const char* path);
/* Restores a checkpoint into a handle created from the same parameter file (same grid size and
 * terrain, checked); the run then continues bit for bit as if it had never stopped. */
int fip_restore(fip_handle* h, const char* path);

/* Headless colour map of the current state, replacing the reference's OpenGL view
 * (src/vis.cpp, fragment shader src/shaders.h:57-123) with an RGBA8 image seen from straight
 * above: row 0 is the northern edge (grid row H-1), no-data cells are transparent, water deeper
 * than 1 cm is coloured with the MATLAB jet map of min(1, value / vmax), dry cells show the
 * shaded terrain. what: FIP_RENDER_DEPTH, FIP_RENDER_VELOCITY or FIP_RENDER_HMAX; vmax <= 0
 * uses the viewer's default 5 (m or m/s). Writes W*H*4 bytes to rgba_or_null and/or a PNG file. */
#define FIP_RENDER_DEPTH 0
#define FIP_RENDER_VELOCITY 1
#define FIP_RENDER_HMAX 2
int fip_render(fip_handle* h, int what, float vmax, unsigned char* rgba_or_null, const char* png_path_or_null);

/* Test hook of the failure detection (no counterpart in the reference): the next step's stencil
 * leaves the first row of one CTA unstaged, so that CTA's bounded shared-memory waits run out
 * (2 s) and the step returns FIP_ERR_DEVICE_TIMEOUT; the CUDA context stays usable, the handle
 * does not (destroy it). */
int fip_inject_wait_timeout(fip_handle* h);

/* Frees every device and host resource of the handle (the reference leaves this to
 * cudaDeviceReset at exit, src/main.cpp:256). */
void fip_destroy(fip_handle* h);

/* One rmg step of the whole grid on caller-owned device buffers, allocating nothing. No
 * counterpart in the reference. It is for callers that cannot allocate device memory: a host that
 * drives the step from its own time loop while other streams keep the GPU busy (cudaFree
 * synchronises the whole device), or a host whose own memory pool owns all device memory and
 * forbids allocations once it runs.
 * Inputs: h_in, qx_in, qy_in, terrain (and kst_or_null, else the uniform kst_fixed), pitched with
 * `pitch` elements per row (a multiple of 4), 16-byte aligned, W x H cells, W, H >= 4. Outputs:
 * h_out, qx_out, qy_out receive the step on the cells the reference's kernel writes; their other
 * cells are left as the caller set them (give them the input state, like the reference's
 * ping-pong partner). cfl_out_or_null (device float) receives the CFL minimum of the step, or NaN
 * if a bounded device-side wait ran out: a caller that must detect such a timeout passes it (with
 * NULL a timed-out step still returns 0). No boundary conditions, dt control or sampling: this is
 * the stencil alone (the launch of src/kernels.cu:441-455 with the mask off).
 * Scratch: a static device array sized for grids of at most 32768 tiles of 480 x 32 cells (about
 * 503 million cells); larger grids return FIP_ERR_ARG. Every GPU that loads the library holds
 * that array (about 160 KB) until the process exits. The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and keeps it for the life of the process, so
 * make that first call before any stream capture, and do not reset the device (cudaDeviceReset)
 * between calls. Calls share the array and rewrite what the step reads from it each time; calls
 * that overlap on the GPU (other streams or host threads) race on it. Runs on `stream` (a
 * cudaStream_t, NULL for the legacy default stream) on the current device and returns without
 * synchronising. */
int fip_rmg_step_noalloc(const float* h_in, const float* qx_in, const float* qy_in, const float* terrain,
                         const float* kst_or_null, float kst_fixed, float* h_out, float* qx_out, float* qy_out,
                         int W, int H, int pitch, float dx, float dt, float no_value, float* cfl_out_or_null,
                         void* stream);

/* ---- host-only entry points (no GPU needed) ---- */

/* Parses and validates a parameter file and loads its grids, without touching a GPU
 * (validateSimDataConfig + loadSimData, src/simdata.cpp:152-310). Messages as fip_init. */
int fip_validate(const char* yaml_path);

/* The parsed configuration as a JSON object (name, W, H, dx, dt, variable_dt, solver,
 * target_duration, kSt, no_data, kst_var, boundary_conditions, sampling, save_state), written
 * to buf (NUL-terminated, truncated to buflen). Returns the full length or a negative error. */
int fip_config_json(const char* yaml_path, char* buf, int buflen);

/* CUDA source of the boundary-condition program for a parameter file and a device row pitch in
 * elements (BoundaryConditionKernel::generate's source text, src/bc_kernel_gen.cpp:154-178).
 * When compile != 0 it is also compiled with NVRTC for sm_100a (no GPU needed). Returns the
 * source length or a negative error. */
int fip_bc_program(const char* yaml_path, int pitch, int compile, char* buf, int buflen);

/* ---- Batched ensembles (no counterpart in the reference, which runs one scenario per process,
 * src/main.cpp:204-263) ----
 * Many parameter files advanced together: every ensemble step is one stencil launch and one
 * post-kernel launch over all members still short of their target duration. Each member
 * computes exactly what fip_init + fip_step compute for its own file (own dt controller,
 * boundary conditions, flood plains); sampling points and save_state times of the members are
 * ignored. Members are stacked in one set of device buffers; tile shape is chosen by
 * fip_ensemble_autotune or fip_ensemble_set_shape. */
typedef struct fip_ensemble fip_ensemble;

typedef struct {
  int consumer_warps;  /* 2 or 4 warps per tile */
  int tile_cols, tile_rows;  /* tile_cols = 30 * cols_per_thread * consumer_warps */
  int steps;           /* ensemble steps timed in this shape */
  float ms_per_step;   /* device time per ensemble step (CUDA events) */
  int cols_per_thread; /* 4, or 2 (narrow threads: half the registers, more warps per SM) */
} fip_ensemble_tune_t;

typedef struct {
  int n_members, active_members;
  long long cells;     /* sum of the members' W * H */
  int packed_W, packed_rows, pitch;
  int consumer_warps, tile_cols, tile_rows;
  int n_tiles, active_tiles;  /* tiles of all members / computed by the next step */
  int iteration;       /* ensemble steps taken */
  int nonfinite;
  int cols_per_thread;
} fip_ensemble_info_t;

int fip_ensemble_init(const char* const* yaml_paths, int n_members, const fip_options* opt, fip_ensemble** out);
/* n_steps ensemble steps (members that reached their target duration stay as they are). */
int fip_ensemble_step(fip_ensemble* e, int n_steps);
/* Until every member reached its target duration. */
int fip_ensemble_run(fip_ensemble* e);
/* Times steps_per_shape real ensemble steps in each tile shape (the state advances; results
 * do not depend on the shape) and keeps the fastest. Fills up to max_results entries. */
int fip_ensemble_autotune(fip_ensemble* e, int steps_per_shape, fip_ensemble_tune_t* results, int max_results,
                          int* n_results);
int fip_ensemble_set_shape(fip_ensemble* e, int consumer_warps, int tile_rows);
/* The same with the columns per thread (4, or 2 with 4 consumer warps: 240-column tiles). */
int fip_ensemble_set_shape_nc(fip_ensemble* e, int consumer_warps, int tile_rows, int cols_per_thread);
/* n_steps ensemble steps timed with CUDA events on the ensemble's stream. */
int fip_ensemble_step_timed(fip_ensemble* e, int n_steps, float* total_ms);
/* Member field (FIP_FIELD_H .. FIP_FIELD_TERRAIN) into a W x H host buffer. */
int fip_ensemble_get_field(fip_ensemble* e, int member, int field, float* host);
/* Member fields (FIP_FIELD_H, _QX, _QY, _HMAX or _TERRAIN) of all members, one W x H grid after
 * the other, into device memory (sum of the members' W * H floats). */
int fip_ensemble_gather(fip_ensemble* e, int field, float* dev_out);
int fip_ensemble_time(fip_ensemble* e, int member, double* duration, float* dt, int* iteration);
int fip_ensemble_info(fip_ensemble* e, fip_ensemble_info_t* out);
/* fip_render for one member of an ensemble. */
int fip_ensemble_render(fip_ensemble* e, int member, int what, float vmax, unsigned char* rgba_or_null,
                        const char* png_path_or_null);
void fip_ensemble_destroy(fip_ensemble* e);

/* Message of the last failed call on this thread ("" if none). */
const char* fip_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
