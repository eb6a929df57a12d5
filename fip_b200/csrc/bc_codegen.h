// Boundary-condition kernel generation (the reference's BoundaryConditionKernel, src/bc_kernel_gen.{h,cpp}).
// The YAML's conditions become one CUDA program, compiled at start-up with NVRTC straight to an
// sm_100a cubin and loaded with the driver API. The program's single kernel, fip_post, runs after
// every step: block 0 applies the conditions one after the other (configuration order), the
// other blocks build the next active-tile list, and the last block to finish advances the
// device control block (time, dt controller, iteration, event checks).
#pragma once
#include <cuda.h>

#include <string>
#include <vector>

#include "config.h"
#include "fip_ctl.h"

namespace fip {

struct TileForce;  // rmg_stencil.h

struct SeriesLayout {
  std::vector<float> data;      // concatenated tables, uploaded to the device
  std::vector<long> z_off, q_off;  // per condition: offset of its z / q table (-1: none)
  std::vector<int> z_n, q_n;
};

SeriesLayout layout_series(const Config& cfg);

// The cells each boundary condition of `cfg` writes (the side's cell, its inner neighbour and the
// staggered face of every position from..to, src/bc_kernel_gen.cpp:10-136), widened by the
// stencil's reach: their tiles are always computed. Tiles elsewhere on the edge are computed
// only while they or their neighbours hold water.
void bc_tile_force(const Config& cfg, TileForce* out);

// CUDA source of the post kernel for `cfg` (pitch in elements: the top/bottom open boundary
// scales its outflow by idx - idx_neighbor = +-pitch, src/bc_kernel_gen.cpp:122, :132).
std::string post_kernel_source(const Config& cfg, const SeriesLayout& ser, int pitch);

// Post kernel of a packed ensemble (fip_ens_post): block m < members applies member m's
// conditions (its rows start at members[m].row_off of the packed buffers with row pitch `pitch`),
// the other blocks plan the next step's tiles, the last block advances every member.
// series_base[m] is the offset of member m's tables in the concatenated series array.
std::string ensemble_post_kernel_source(const std::vector<const Config*>& cfgs, const std::vector<SeriesLayout>& sers,
                                        const std::vector<long long>& series_base,
                                        const std::vector<FipEnsMember>& members, int pitch);

struct PostKernel {
  CUmodule module = nullptr;
  CUfunction fn = nullptr;
  std::string source, log;
};

// NVRTC compile for sm_100a to a cubin (no GPU needed). Returns 0 or a message in *err.
int compile_post_kernel(const std::string& source, std::string* cubin, std::string* log, std::string* err);

// compile_post_kernel + cuModuleLoadData. Returns 0 or a message in *err.
int build_post_kernel(const std::string& source, PostKernel* out, std::string* err,
                      const char* entry = "fip_post");
void destroy_post_kernel(PostKernel* k);

}  // namespace fip
