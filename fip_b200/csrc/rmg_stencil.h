// Host interface of the sm_100a kernels in rmg_stencil.cu (internal to libfip_b200).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fip_ctl.h"

namespace fip {

// Tiles that are always computed because boundary conditions write near them: inclusive cell
// rectangles (columns c0..c1, rows r0..r1) covering every cell a configured condition writes,
// widened by the stencil's reach. all_band forces every tile within 4 cells of the edge instead
// (more conditions than the list holds).
constexpr int kMaxForceRects = 32;
struct TileForce {
  int n = 0;
  int all_band = 0;
  int rect[kMaxForceRects][4] = {};  // c0, c1, r0, r1
};

// Device buffers and planning scratch of one scenario. Fields are cudaMallocPitch'ed like the
// reference (src/simdata.cpp:63-73): W floats per row, H+3 rows, `pitch` elements per row.
struct StencilState {
  float* h[2];
  float* qx[2];
  float* qy[2];
  float* sohle;
  float* kst;   // nullptr: uniform kst_fixed
  float* hmax;
  FipCtl* ctl;  // device control block
  unsigned char* sticky;  // per tile: always active (boundary-condition cells, static water on cells the step never writes)
  unsigned char* nz[2];   // per tile: FIP_NZ_* flags of the new state, by iteration parity (whole words)
  int* list[2];           // active tiles by chunk (front) / inactive tiles (back), by parity
  int* chunk_cnt[2];      // active tiles per chunk, by parity
  int W, H, pitch;
  int n_sx, n_ty, n_tiles, n_chunks;
  float dx, kst_fixed, no_value;
  CUtensorMap tm_h[2], tm_qx[2], tm_qy[2], tm_sohle, tm_kst;
  // packed ensembles (members != nullptr): member table, per-member control, tile shape
  const FipEnsMember* members = nullptr;
  FipEnsCtl* mctl = nullptr;
  int n_members = 0;
  int tile_rows = FIP_TILE_ROWS;
  int kw = 4;  // consumer warps per CTA: tiles of 30 * nc * kw columns
  int nc = 4;  // columns per thread (4, or 2: narrow threads; ensembles)
  int tile_cols = FIP_TILE_COLS;  // single grids
  TileForce force;  // single grids: tiles the boundary conditions keep active
};

// Geometry of the tile grid for a W x H domain in tiles of tile_cols x FIP_TILE_ROWS cells.
void tile_geometry(int W, int H, int tile_cols, int* n_sx, int* n_ty, int* n_tiles, int* n_chunks);

// Tile columns of a single grid whose threads own nc columns (480 for 4, 240 for 2).
int single_tile_cols(int nc);

// Encodes the TMA descriptors of every field (box 256 x 1 floats). Returns a CUresult.
int make_tensor_maps(StencilState* st);

// One rmg step over the active tiles of the current plan (reads ctl on the device).
cudaError_t launch_rmg_step(const StencilState& st, int grid_ctas, cudaStream_t stream);

// Per-tile sticky flags and the FIP_NZ_* flags of state buffer `parity` (into both nz slots).
cudaError_t launch_init_tiles(const StencilState& st, int parity, cudaStream_t stream);

// The same for one region of a packed ensemble (pointers at the member's first row, flags at its
// first tile) with an explicit tile shape. nz_cur gets the flags of (h, qx, qy); nz_prev those
// of (h, qx, qy) OR of the other ping-pong buffer when h_other is given, so that a tile whose
// output buffer still holds water is computed.
cudaError_t launch_init_tiles_region(const float* h, const float* qx, const float* qy, const float* h_other,
                                     const float* qx_other, const float* qy_other, const float* sohle, int W, int H,
                                     int pitch, float no_value, int tile_cols, int tile_rows, const TileForce& force,
                                     unsigned char* sticky, unsigned char* nz_cur, unsigned char* nz_prev,
                                     cudaStream_t stream);

// CTAs the step kernel runs with for tiles of kw consumer warps and nc columns per thread (3 per
// SM for 4 warps, 5 for 2, 4 for narrow threads).
int rmg_step_grid_kw(int device, int kw, int nc);

// hmax = max(hmax, h[parity]) over the whole grid (the reference's flood_plains_kernel).
cudaError_t launch_hmax_fold(const StencilState& st, int parity, cudaStream_t stream);

// FP64 sum of h[parity] over the grid into *out (device), deterministic order. `partials`
// holds at least volume_partials() doubles.
int volume_partials(const StencilState& st);
cudaError_t launch_volume(const StencilState& st, int parity, double* partials, double* out,
                          cudaStream_t stream);

// Sets *flag (device) to 1 when one of the W x H cells of h (row pitch `pitch` floats) is
// negative; leaves it as it is otherwise.
cudaError_t launch_flag_negative(const float* h, int W, int H, int pitch, int* flag, cudaStream_t stream);

// Gathers n sample values (type 0..3 = z, h, qx, qy; z adds terrain) of buffer `parity`.
cudaError_t launch_sample_gather(const StencilState& st, int parity, int n, const int* xy_type,
                                 float* out, cudaStream_t stream);

// Replaces -0 by +0 in a W x H field of row pitch `pitch` (uploaded states: the step writes +0
// for every zero it computes, so a quiescent tile must hold +0 for skipping it to be exact).
cudaError_t launch_positive_zero(float* a, int W, int H, int pitch, cudaStream_t stream);
// dst0 (and dst1 unless null) = src with -0 -> +0, same geometry (src may be dst0).
cudaError_t launch_positive_zero_copy(const float* src, float* dst0, float* dst1, int W, int H, int pitch,
                                      cudaStream_t stream);

// Number of CTAs the single-grid step kernel runs with (3 per SM with 4 columns per thread, 5
// with 2).
int rmg_step_grid(int device, int nc);

}  // namespace fip
