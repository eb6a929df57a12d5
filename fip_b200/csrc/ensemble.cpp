// Batched ensembles: many scenarios advanced together by one stencil launch and one post-kernel
// launch per step (include/fip.h, fip_ensemble_*). No counterpart in the reference, which runs
// one scenario per process (src/main.cpp:204-263); each member here computes exactly what
// fip_init/fip_step would compute for its own parameter file.
//
// Layout: the members are stacked in one set of pitched buffers as wide as the widest member.
// Member m occupies rows [row_off, row_off + H) and columns [0, W); three zero rows separate the
// members and the columns right of W stay zero, so every load of the stencil (which reaches two
// rows and columns beyond a member's edge) sees what the member's own buffers would hold. One
// set of TMA descriptors covers all members; the tiles of all members form one concatenated
// active-tile list, so a single persistent launch steps the whole ensemble.
//
// Time: every member keeps its own simulated time, dt (variable_dt controller) and CFL slots;
// the ensemble steps all members that are still short of their target duration, and a member
// that reached it drops out of the plan. Batches of steps run as captured CUDA graphs.
//
// Tile shape: consumer warps per CTA (tiles of 240 or 480 columns) and tile rows (16, 32, 64)
// are chosen by fip_ensemble_autotune, which times real steps of the ensemble in each shape
// (results do not depend on the shape, so no state is saved or restored).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "bc_codegen.h"
#include "config.h"
#include "drv.h"
#include "fip.h"
#include "fip_ctl.h"
#include "render.h"
#include "rmg_stencil.h"

namespace fip {
void set_last_error(const std::string& msg);
int render_region(int device, cudaStream_t stream, const float* h, const float* qx, const float* qy,
                  const float* sohle, int W, int H, int pitch, float no_value, int what, float vmax,
                  unsigned char* rgba_or_null, const char* png_path_or_null);
}

namespace {

struct EnsError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void eck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw EnsError(std::string(what) + ": " + cudaGetErrorString(e));
}
void eckd(CUresult r, const char* what) {
  if (r != CUDA_SUCCESS) throw EnsError(fip::drv::message(r, what));
}

int efail(int code, const std::string& m) {
  fip::set_last_error(m);
  return code;
}

constexpr int kGapRows = 3;  // zero rows above, between and below the members

struct Shape {
  int kw, tile_rows;
  int nc = 4;  // columns per thread
  int cols() const { return 30 * nc * kw; }
};
const Shape kShapes[] = {{4, 32, 4}, {4, 16, 4}, {4, 64, 4}, {2, 32, 4}, {2, 16, 4}, {2, 64, 4},
                         {4, 32, 2}, {4, 16, 2}, {4, 64, 2}};

}  // namespace

struct fip_ensemble {
  std::vector<std::unique_ptr<fip::Config>> cfgs;
  fip_options opt;
  int device = 0;
  cudaStream_t stream = nullptr;
  fip::StencilState st{};
  int n = 0;
  int packed_W = 0, total_rows = 0, pitch = 0;
  std::vector<FipEnsMember> mem;  // host copy for the current tile shape
  FipEnsMember* d_mem = nullptr;
  FipEnsCtl* d_mctl = nullptr;
  FipEnsCtl* h_mctl = nullptr;  // pinned mirror
  FipCtl* d_ctl = nullptr;
  FipCtl* h_ctl = nullptr;  // pinned mirror
  float* d_series = nullptr;
  int max_tiles = 0, max_chunks = 0;
  fip::PostKernel post;
  Shape shape{4, 32};
  int grid_ctas = 0;
  bool started = false;
  std::map<int, cudaGraphExec_t> graphs;  // by batch length, for the current shape
  std::vector<fip_ensemble_tune_t> tune;

  ~fip_ensemble();
  void init(const std::vector<std::string>& paths, const fip_options& o);
  void set_shape(Shape s, bool replan);
  void launch_post(int mode);
  void launch_step_pair();
  void launch_batch(int k);
  void read_ctl();
  int run(long long budget, bool to_target);
  int parity_of(int m) const { return h_mctl[m].active ? h_ctl->parity : h_mctl[m].final_parity; }
  void clear_graphs();
};

fip_ensemble::~fip_ensemble() {
  if (device >= 0) cudaSetDevice(device);
  clear_graphs();
  fip::destroy_post_kernel(&post);
  for (int b = 0; b < 2; ++b) {
    cudaFree(st.h[b]);
    cudaFree(st.qx[b]);
    cudaFree(st.qy[b]);
    cudaFree(st.nz[b]);
    cudaFree(st.list[b]);
    cudaFree(st.chunk_cnt[b]);
  }
  cudaFree(st.sohle);
  cudaFree(st.kst);
  cudaFree(st.hmax);
  cudaFree(st.sticky);
  cudaFree(d_mem);
  cudaFree(d_mctl);
  cudaFree(d_ctl);
  cudaFree(d_series);
  if (h_mctl) cudaFreeHost(h_mctl);
  if (h_ctl) cudaFreeHost(h_ctl);
  if (stream) cudaStreamDestroy(stream);
}

void fip_ensemble::clear_graphs() {
  for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
  graphs.clear();
}

void fip_ensemble::init(const std::vector<std::string>& paths, const fip_options& o) {
  opt = o;
  device = o.device;
  n = (int)cfgs.size();
  eck(cudaSetDevice(device), "cudaSetDevice");
  eck(cudaFree(nullptr), "CUDA context");
  std::string derr;
  if (!fip::drv::load(&derr)) throw EnsError(derr);
  eck(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");

  bool any_kvar = false, negative = false;
  packed_W = 0;
  for (const auto& c : cfgs) {
    packed_W = std::max(packed_W, (int)c->W);
    any_kvar |= c->has_kst_var;
    for (float v : c->h0) negative |= (v < 0.f);
  }
  // rows of each member; the pitch of each member's own buffers (the top/bottom open boundary
  // scales its outflow by it, src/bc_kernel_gen.cpp:122, :132)
  mem.assign(n, FipEnsMember{});
  int row = kGapRows;
  for (int m = 0; m < n; ++m) {
    const fip::Config& c = *cfgs[m];
    FipEnsMember& M = mem[m];
    M.W = (int)c.W;
    M.H = (int)c.H;
    M.row_off = row;
    row += (int)c.H + kGapRows;
    M.dx = c.dx;
    M.kst_fixed = c.kst_fixed;
    M.no_value = c.no_data;
    void* probe = nullptr;
    size_t pb = 0;
    eck(cudaMallocPitch(&probe, &pb, c.W * sizeof(float), c.H + 3), "cudaMallocPitch");
    cudaFree(probe);
    M.pitch_ref = (int)(pb / sizeof(float));
  }
  total_rows = row;

  const size_t row_bytes = (size_t)packed_W * sizeof(float);
  size_t pitch_bytes = 0;
  auto alloc_field = [&](float** p) {
    size_t pb = 0;
    eck(cudaMallocPitch((void**)p, &pb, row_bytes, total_rows), "cudaMallocPitch");
    if (pitch_bytes && pb != pitch_bytes) throw EnsError("inconsistent pitch");
    pitch_bytes = pb;
    eck(cudaMemset2D(*p, pb, 0, pb, total_rows), "cudaMemset2D");
  };
  for (int b = 0; b < 2; ++b) {
    alloc_field(&st.h[b]);
    alloc_field(&st.qx[b]);
    alloc_field(&st.qy[b]);
  }
  alloc_field(&st.sohle);
  alloc_field(&st.hmax);
  if (any_kvar) alloc_field(&st.kst);
  if (pitch_bytes % 16) throw EnsError("row pitch is not a multiple of 16 bytes");
  pitch = (int)(pitch_bytes / sizeof(float));
  for (int m = 0; m < n; ++m) {
    const fip::Config& c = *cfgs[m];
    const size_t W = c.W, H = c.H, rb = W * sizeof(float);
    const size_t off = (size_t)mem[m].row_off * pitch;
    auto up = [&](float* dst, const std::vector<float>& src) {
      eck(cudaMemcpy2D(dst + off, pitch_bytes, src.data(), rb, rb, H, cudaMemcpyHostToDevice), "cudaMemcpy2D");
    };
    for (int b = 0; b < 2; ++b) {
      up(st.h[b], c.h0);
      up(st.qx[b], c.qx0);
      up(st.qy[b], c.qy0);
    }
    up(st.hmax, c.h0);
    up(st.sohle, c.terrain);
    if (any_kvar) {
      // a member with a uniform kSt gets it as a grid: (dt * G) / (kSt * kSt) is the same
      // arithmetic in both forms of the kernel
      if (c.has_kst_var) up(st.kst, c.kst);
      else up(st.kst, std::vector<float>(W * H, c.kst_fixed));
    }
  }
  st.W = packed_W;
  st.H = total_rows;
  st.pitch = pitch;
  st.dx = cfgs[0]->dx;
  st.kst_fixed = cfgs[0]->kst_fixed;
  st.no_value = cfgs[0]->no_data;
  eckd((CUresult)fip::make_tensor_maps(&st), "cuTensorMapEncodeTiled");

  // planning buffers for the smallest tiles any shape uses
  max_tiles = 0;
  for (const Shape& s : kShapes) {
    int t = 0;
    for (int m = 0; m < n; ++m)
      t += ((mem[m].W + s.cols() - 1) / s.cols()) * ((mem[m].H + s.tile_rows - 1) / s.tile_rows);
    max_tiles = std::max(max_tiles, t);
  }
  max_chunks = (max_tiles + FIP_PLAN_CHUNK - 1) / FIP_PLAN_CHUNK;
  if (max_chunks > 256) throw std::invalid_argument("ensemble too large: more than 131072 tiles of 240 x 16 cells");
  eck(cudaMalloc((void**)&st.sticky, max_tiles), "cudaMalloc");
  for (int b = 0; b < 2; ++b) {
    eck(cudaMalloc((void**)&st.nz[b], ((size_t)max_tiles + 3) & ~(size_t)3), "cudaMalloc");
    eck(cudaMalloc((void**)&st.list[b], sizeof(int) * (size_t)max_chunks * FIP_PLAN_CHUNK), "cudaMalloc");
    eck(cudaMalloc((void**)&st.chunk_cnt[b], sizeof(int) * max_chunks), "cudaMalloc");
    eck(cudaMemset(st.chunk_cnt[b], 0, sizeof(int) * max_chunks), "cudaMemset");
  }
  eck(cudaMalloc((void**)&d_mem, sizeof(FipEnsMember) * n), "cudaMalloc");

  // time series of all members, concatenated
  std::vector<fip::SeriesLayout> sers;
  std::vector<long long> sbase;
  std::vector<float> all;
  std::vector<const fip::Config*> cp;
  for (int m = 0; m < n; ++m) {
    sers.push_back(fip::layout_series(*cfgs[m]));
    sbase.push_back((long long)all.size());
    all.insert(all.end(), sers.back().data.begin(), sers.back().data.end());
    cp.push_back(cfgs[m].get());
  }
  eck(cudaMalloc((void**)&d_series, all.size() * sizeof(float)), "cudaMalloc");
  eck(cudaMemcpy(d_series, all.data(), all.size() * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy");

  // control blocks
  eck(cudaMallocHost((void**)&h_ctl, sizeof(FipCtl)), "cudaMallocHost");
  std::memset(h_ctl, 0, sizeof(FipCtl));
  h_ctl->next_sample = h_ctl->next_save = h_ctl->target = 1e300;
  h_ctl->stop_on_nonfinite = opt.stop_on_nonfinite ? 1 : 0;
  h_ctl->hmax_every = 100;
  h_ctl->force_all = (opt.all_tiles || negative) ? 1 : 0;  // negative depths: fold hmax over every tile
  eck(cudaMalloc((void**)&d_ctl, sizeof(FipCtl)), "cudaMalloc");
  eck(cudaMemcpy(d_ctl, h_ctl, sizeof(FipCtl), cudaMemcpyHostToDevice), "cudaMemcpy");
  eck(cudaMallocHost((void**)&h_mctl, sizeof(FipEnsCtl) * n), "cudaMallocHost");
  std::memset(h_mctl, 0, sizeof(FipEnsCtl) * n);
  for (int m = 0; m < n; ++m) {
    const fip::Config& c = *cfgs[m];
    FipEnsCtl& mc = h_mctl[m];
    mc.duration = 0.0;
    mc.target = c.target_duration;
    mc.dt = c.dt;
    mc.last_cfl = 1.0f;
    mc.variable_dt = c.variable_dt ? 1 : 0;
    mc.active = (0.0 < c.target_duration) ? 1 : 0;
    const float one = 1.0f;
    std::memcpy(&mc.cfl_bits[0], &one, 4);
    std::memcpy(&mc.cfl_bits[1], &one, 4);
    if (c.variable_dt) {  // controlTimestep at the start of the first simulate(): CFL slots hold 1
      const float target = 1.0f * .5f, dc = 0.001f;
      float d = mc.dt;
      if (d < target && target - d > dc) d *= 1.001f;
      else if (d > target && d - target > dc) d *= 0.99f;
      mc.dt = d;
    }
  }
  eck(cudaMalloc((void**)&d_mctl, sizeof(FipEnsCtl) * n), "cudaMalloc");
  eck(cudaMemcpy(d_mctl, h_mctl, sizeof(FipEnsCtl) * n, cudaMemcpyHostToDevice), "cudaMemcpy");
  st.ctl = d_ctl;
  st.members = d_mem;
  st.mctl = d_mctl;
  st.n_members = n;

  std::string err;
  const std::string src = fip::ensemble_post_kernel_source(cp, sers, sbase, mem, pitch);
  if (fip::build_post_kernel(src, &post, &err, "fip_ens_post")) throw std::invalid_argument("NVRTC:" + err);
  set_shape(Shape{4, 32, 4}, false);
  eck(cudaStreamSynchronize(stream), "init");
  (void)paths;
}

// Tile shape: member table, tile counts, and (replan) the plan of the current state in it.
void fip_ensemble::set_shape(Shape s, bool replan) {
  shape = s;
  const int tc = s.cols();
  int base = 0;
  for (int m = 0; m < n; ++m) {
    FipEnsMember& M = mem[m];
    M.tile_base = base;
    M.n_sx = (M.W + tc - 1) / tc;
    M.n_ty = (M.H + s.tile_rows - 1) / s.tile_rows;
    base += M.n_sx * M.n_ty;
  }
  st.n_tiles = base;
  st.n_chunks = (base + FIP_PLAN_CHUNK - 1) / FIP_PLAN_CHUNK;
  st.n_sx = 0;
  st.n_ty = 1;
  st.kw = s.kw;
  st.nc = s.nc;
  st.tile_rows = s.tile_rows;
  grid_ctas = fip::rmg_step_grid_kw(device, s.kw, s.nc);
  clear_graphs();
  eck(cudaMemcpyAsync(d_mem, mem.data(), sizeof(FipEnsMember) * n, cudaMemcpyHostToDevice, stream), "cudaMemcpy");
  eck(cudaMemsetAsync(st.nz[0], 0, max_tiles, stream), "cudaMemset");
  eck(cudaMemsetAsync(st.nz[1], 0, max_tiles, stream), "cudaMemset");
  // flags of the current state; the plan for the next step reads nz[k & 1] as "after this step"
  // and nz[(k + 1) & 1] as "after the step before", k = iteration - 1 in plan mode
  const int par = h_ctl->parity;
  const int k = h_ctl->iteration - 1;
  unsigned char* nz_cur = st.nz[k & 1];
  unsigned char* nz_prev = st.nz[(k + 1) & 1];
  for (int m = 0; m < n; ++m) {
    const FipEnsMember& M = mem[m];
    const size_t off = (size_t)M.row_off * pitch;
    const bool other = replan;  // after steps the partner buffer may still hold water elsewhere
    fip::TileForce force;
    fip::bc_tile_force(*cfgs[m], &force);
    eck(fip::launch_init_tiles_region(st.h[par] + off, st.qx[par] + off, st.qy[par] + off,
                                      other ? st.h[par ^ 1] + off : nullptr, other ? st.qx[par ^ 1] + off : nullptr,
                                      other ? st.qy[par ^ 1] + off : nullptr, st.sohle + off, M.W, M.H, pitch,
                                      M.no_value, tc, s.tile_rows, force, st.sticky + M.tile_base,
                                      nz_cur + M.tile_base, nz_prev + M.tile_base, stream),
        "init_tiles");
  }
  if (replan) launch_post(FIP_POST_MODE_PLAN);
}

void fip_ensemble::launch_post(int mode) {
  FipEnsPostArgs a;
  std::memset(&a, 0, sizeof a);
  for (int b = 0; b < 2; ++b) {
    a.h[b] = st.h[b];
    a.qx[b] = st.qx[b];
    a.qy[b] = st.qy[b];
    a.nz[b] = st.nz[b];
    a.list[b] = st.list[b];
    a.chunk_cnt[b] = st.chunk_cnt[b];
  }
  a.sohle = st.sohle;
  a.ctl = d_ctl;
  a.mctl = d_mctl;
  a.members = d_mem;
  a.sticky = st.sticky;
  a.series = d_series;
  a.pitch = pitch;
  a.n_members = n;
  a.n_tiles = st.n_tiles;
  a.n_chunks = st.n_chunks;
  a.tile_cols = shape.cols();
  a.tile_rows = shape.tile_rows;
  a.mode = mode;
  void* params[] = {&a};
  eckd(fip::drv::LaunchKernel(post.fn, n + st.n_chunks, 1, 1, FIP_POST_THREADS, 1, 1, 0, (CUstream)stream, params,
                              nullptr),
       "fip_ens_post launch");
}

void fip_ensemble::launch_step_pair() {
  eck(fip::launch_rmg_step(st, grid_ctas, stream), "rmg_step launch");
  launch_post(FIP_POST_MODE_STEP);
}

void fip_ensemble::launch_batch(int k) {
  if (!opt.use_graphs || k == 1) {
    for (int i = 0; i < k; ++i) launch_step_pair();
    return;
  }
  auto it = graphs.find(k);
  if (it == graphs.end()) {
    cudaGraph_t g;
    eck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture");
    for (int i = 0; i < k; ++i) launch_step_pair();
    eck(cudaStreamEndCapture(stream, &g), "capture");
    cudaGraphExec_t ex;
    eck(cudaGraphInstantiate(&ex, g, 0), "cudaGraphInstantiate");
    cudaGraphDestroy(g);
    it = graphs.emplace(k, ex).first;
  }
  eck(cudaGraphLaunch(it->second, stream), "cudaGraphLaunch");
}

void fip_ensemble::read_ctl() {
  eck(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(FipCtl), cudaMemcpyDeviceToHost, stream), "ctl download");
  eck(cudaMemcpyAsync(h_mctl, d_mctl, sizeof(FipEnsCtl) * n, cudaMemcpyDeviceToHost, stream), "ctl download");
  eck(cudaStreamSynchronize(stream), "step");
}

// Up to `budget` ensemble steps, or (to_target) until every member reached its target duration.
int fip_ensemble::run(long long budget, bool to_target) {
  eck(cudaSetDevice(device), "cudaSetDevice");
  if (!started) {
    h_ctl->stop = 0;
    h_ctl->steps_left = 1;
    eck(cudaMemcpyAsync(d_ctl, h_ctl, sizeof(FipCtl), cudaMemcpyHostToDevice, stream), "ctl upload");
    launch_post(FIP_POST_MODE_INIT);  // iteration-0 boundary conditions and the first plan
    started = true;
  }
  bool any = false;
  for (int m = 0; m < n; ++m) any |= h_mctl[m].active != 0;
  if (!any || budget <= 0) return FIP_OK;
  long long left = budget;
  int rc = FIP_OK;
  for (;;) {
    const int chunk = (int)std::min<long long>(left, 1 << 30);
    h_ctl->steps_left = chunk;
    h_ctl->stop = 0;
    h_ctl->stop_reason = 0;
    auto put = [&](size_t offset, size_t bytes) {
      eck(cudaMemcpyAsync(reinterpret_cast<char*>(d_ctl) + offset, reinterpret_cast<char*>(h_ctl) + offset, bytes,
                          cudaMemcpyHostToDevice, stream),
          "ctl upload");
    };
    put(offsetof(FipCtl, stop), 3 * sizeof(int));  // stop, stop_reason, steps_left
    const int it0 = h_ctl->iteration;
    // batches of 64 steps; the device stops a batch when the budget runs out or all members end
    for (;;) {
      const long long rem = h_ctl->steps_left;
      int k = 64;
      while (k > 1 && k > rem) k >>= 1;
      launch_batch(k);
      read_ctl();
      if (h_ctl->error) return efail(FIP_ERR_DEVICE_TIMEOUT, "device wait ran out (code " + std::to_string(h_ctl->error) + ")");
      if (h_ctl->stop) break;
    }
    const int reason = h_ctl->stop_reason;
    left -= h_ctl->iteration - it0;
    if (reason & FIP_STOP_NONFINITE) {
      rc = efail(FIP_ERR_NONFINITE, "a stored water depth is NaN or Inf at ensemble step " + std::to_string(h_ctl->iteration));
      break;
    }
    if (reason & FIP_STOP_TARGET) break;
    if (!to_target && left <= 0) break;
    if (to_target && left <= 0) left = 1LL << 62;
  }
  h_ctl->stop = 0;
  h_ctl->stop_reason = 0;
  eck(cudaMemcpyAsync(&d_ctl->stop, &h_ctl->stop, 2 * sizeof(int), cudaMemcpyHostToDevice, stream), "ctl upload");
  eck(cudaStreamSynchronize(stream), "step");
  return rc;
}

namespace {

int eguard(const std::function<int()>& f) {
  try {
    return f();
  } catch (const EnsError& e) {
    return efail(FIP_ERR_CUDA, e.what());
  } catch (const std::invalid_argument& e) {
    std::string m = e.what();
    if (m.rfind("IO:", 0) == 0) return efail(FIP_ERR_IO, m.substr(3));
    if (m.rfind("NVRTC:", 0) == 0) return efail(FIP_ERR_NVRTC, m.substr(6));
    return efail(FIP_ERR_CONFIG, m);
  } catch (const std::exception& e) {
    return efail(FIP_ERR_CUDA, e.what());
  }
}

}  // namespace

extern "C" {

int fip_ensemble_init(const char* const* yaml_paths, int n_members, const fip_options* opt, fip_ensemble** out) {
  if (!yaml_paths || !out || n_members <= 0) return efail(FIP_ERR_ARG, "fip_ensemble_init: bad argument");
  if (n_members > FIP_ENS_MAX_MEMBERS)
    return efail(FIP_ERR_ARG, "fip_ensemble_init: at most " + std::to_string(FIP_ENS_MAX_MEMBERS) + " members");
  *out = nullptr;
  fip_options o;
  fip_default_options(&o);
  if (opt) o = *opt;
  std::unique_ptr<fip_ensemble> e(new fip_ensemble());
  std::vector<std::string> paths;
  for (int m = 0; m < n_members; ++m) {
    if (!yaml_paths[m]) return efail(FIP_ERR_ARG, "fip_ensemble_init: null path");
    paths.emplace_back(yaml_paths[m]);
    std::unique_ptr<fip::Config> c(new fip::Config());
    std::string err;
    const int rc = fip::load_config(paths.back(), c.get(), &err, o.quiet != 0);
    if (rc == 2) return efail(FIP_ERR_IO, paths.back() + ": " + err);
    if (rc) return efail(FIP_ERR_CONFIG, paths.back() + ": " + err);
    if (c->W < 4 || c->H < 4) return efail(FIP_ERR_CONFIG, paths.back() + ": grids must be at least 4 x 4 cells");
    e->cfgs.push_back(std::move(c));
  }
  const int rc = eguard([&] {
    e->init(paths, o);
    return FIP_OK;
  });
  if (rc) return rc;
  *out = e.release();
  return FIP_OK;
}

int fip_ensemble_step(fip_ensemble* e, int n_steps) {
  if (!e || n_steps < 0) return efail(FIP_ERR_ARG, "bad argument");
  return eguard([&] { return e->run(n_steps, false); });
}

int fip_ensemble_run(fip_ensemble* e) {
  if (!e) return efail(FIP_ERR_ARG, "null ensemble");
  return eguard([&] { return e->run(1LL << 62, true); });
}

int fip_ensemble_autotune(fip_ensemble* e, int steps_per_shape, fip_ensemble_tune_t* results, int max_results,
                          int* n_results) {
  if (!e || steps_per_shape <= 0) return efail(FIP_ERR_ARG, "bad argument");
  return eguard([&] {
    eck(cudaSetDevice(e->device), "cudaSetDevice");
    if (!e->started) {
      int rc = e->run(1, false);
      if (rc) return rc;
    }
    e->tune.clear();
    cudaEvent_t a, b;
    eck(cudaEventCreate(&a), "event");
    eck(cudaEventCreate(&b), "event");
    int best = -1;
    float best_ms = 0.f;
    const int ns = (int)(sizeof(kShapes) / sizeof(kShapes[0]));
    for (int i = 0; i < ns; ++i) {
      bool any = false;
      for (int m = 0; m < e->n; ++m) any |= e->h_mctl[m].active != 0;
      if (!any) break;
      e->set_shape(kShapes[i], true);
      int rc = e->run(2, false);  // graph capture and first launches outside the timing
      if (rc) return rc;
      const int it0 = e->h_ctl->iteration;
      eck(cudaEventRecord(a, e->stream), "event");
      rc = e->run(steps_per_shape, false);
      if (rc) return rc;
      eck(cudaEventRecord(b, e->stream), "event");
      eck(cudaEventSynchronize(b), "event");
      float ms = 0.f;
      eck(cudaEventElapsedTime(&ms, a, b), "event");
      const int ran = e->h_ctl->iteration - it0;
      fip_ensemble_tune_t r;
      r.consumer_warps = kShapes[i].kw;
      r.tile_cols = kShapes[i].cols();
      r.tile_rows = kShapes[i].tile_rows;
      r.cols_per_thread = kShapes[i].nc;
      r.steps = ran;
      r.ms_per_step = ran > 0 ? ms / ran : 0.f;
      e->tune.push_back(r);
      if (ran > 0 && (best < 0 || r.ms_per_step < best_ms)) {
        best = i;
        best_ms = r.ms_per_step;
      }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (best >= 0) e->set_shape(kShapes[best], true);
    if (n_results) *n_results = (int)e->tune.size();
    for (int i = 0; i < (int)e->tune.size() && i < max_results && results; ++i) results[i] = e->tune[i];
    eck(cudaStreamSynchronize(e->stream), "autotune");
    return FIP_OK;
  });
}

int fip_ensemble_set_shape(fip_ensemble* e, int consumer_warps, int tile_rows) {
  return fip_ensemble_set_shape_nc(e, consumer_warps, tile_rows, 4);
}

int fip_ensemble_set_shape_nc(fip_ensemble* e, int consumer_warps, int tile_rows, int cols_per_thread) {
  if (!e) return efail(FIP_ERR_ARG, "null ensemble");
  bool ok = false;
  for (const Shape& s : kShapes)
    ok |= (s.kw == consumer_warps && s.tile_rows == tile_rows && s.nc == cols_per_thread);
  if (!ok)
    return efail(FIP_ERR_ARG,
                 "fip_ensemble_set_shape: consumer_warps must be 2 or 4, tile_rows 16, 32 or 64, and cols_per_thread 4 "
                 "(or 2 with 4 consumer warps)");
  return eguard([&] {
    eck(cudaSetDevice(e->device), "cudaSetDevice");
    e->set_shape(Shape{consumer_warps, tile_rows, cols_per_thread}, e->started);
    eck(cudaStreamSynchronize(e->stream), "set_shape");
    return FIP_OK;
  });
}

int fip_ensemble_step_timed(fip_ensemble* e, int n_steps, float* total_ms) {
  if (!e || n_steps <= 0) return efail(FIP_ERR_ARG, "bad argument");
  return eguard([&] {
    eck(cudaSetDevice(e->device), "cudaSetDevice");
    if (!e->started) {
      int rc = e->run(1, false);
      if (rc) return rc;
    }
    cudaEvent_t a, b;
    eck(cudaEventCreate(&a), "event");
    eck(cudaEventCreate(&b), "event");
    eck(cudaEventRecord(a, e->stream), "event");
    int rc = e->run(n_steps, false);
    eck(cudaEventRecord(b, e->stream), "event");
    eck(cudaEventSynchronize(b), "event");
    float ms = 0.f;
    eck(cudaEventElapsedTime(&ms, a, b), "event");
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (total_ms) *total_ms = ms;
    return rc;
  });
}

int fip_ensemble_get_field(fip_ensemble* e, int member, int field, float* host) {
  if (!e || !host) return efail(FIP_ERR_ARG, "null argument");
  if (member < 0 || member >= e->n) return efail(FIP_ERR_ARG, "fip_ensemble_get_field: member out of range");
  return eguard([&] {
    eck(cudaSetDevice(e->device), "cudaSetDevice");
    const FipEnsMember& M = e->mem[member];
    const int p = e->parity_of(member);
    const float* src = nullptr;
    switch (field) {
      case FIP_FIELD_H: src = e->st.h[p]; break;
      case FIP_FIELD_QX: src = e->st.qx[p]; break;
      case FIP_FIELD_QY: src = e->st.qy[p]; break;
      case FIP_FIELD_HMAX: src = e->st.hmax; break;
      case FIP_FIELD_H_PREV: src = e->st.h[p ^ 1]; break;
      case FIP_FIELD_QX_PREV: src = e->st.qx[p ^ 1]; break;
      case FIP_FIELD_QY_PREV: src = e->st.qy[p ^ 1]; break;
      case FIP_FIELD_TERRAIN: src = e->st.sohle; break;
      default: throw std::invalid_argument("fip_ensemble_get_field: unsupported field");
    }
    const size_t off = (size_t)M.row_off * e->pitch;
    if (field == FIP_FIELD_HMAX) {
      // the flood-plain fold of the member's last step when its iteration is a multiple of 100
      // (the fused fold otherwise happens at the start of its next step)
      const FipEnsCtl& mc = e->h_mctl[member];
      if (mc.iteration > 0 && mc.iteration % 100 == 0) {
        fip::StencilState r{};
        r.h[p] = e->st.h[p] + off;
        r.hmax = e->st.hmax + off;
        r.W = M.W;
        r.H = M.H;
        r.pitch = e->pitch;
        eck(fip::launch_hmax_fold(r, p, e->stream), "hmax");
      }
    }
    const size_t rb = (size_t)M.W * sizeof(float);
    eck(cudaMemcpy2DAsync(host, rb, src + off, (size_t)e->pitch * sizeof(float), rb, M.H, cudaMemcpyDeviceToHost,
                          e->stream),
        "fip_ensemble_get_field");
    eck(cudaStreamSynchronize(e->stream), "fip_ensemble_get_field");
    return FIP_OK;
  });
}

int fip_ensemble_gather(fip_ensemble* e, int field, float* dev_out) {
  if (!e || !dev_out) return efail(FIP_ERR_ARG, "null argument");
  return eguard([&] {
    eck(cudaSetDevice(e->device), "cudaSetDevice");
    size_t off_out = 0;
    for (int m = 0; m < e->n; ++m) {
      const FipEnsMember& M = e->mem[m];
      const int p = e->parity_of(m);
      const float* src = nullptr;
      switch (field) {
        case FIP_FIELD_H: src = e->st.h[p]; break;
        case FIP_FIELD_QX: src = e->st.qx[p]; break;
        case FIP_FIELD_QY: src = e->st.qy[p]; break;
        case FIP_FIELD_HMAX: src = e->st.hmax; break;
        case FIP_FIELD_TERRAIN: src = e->st.sohle; break;
        default: throw std::invalid_argument("fip_ensemble_gather: unsupported field");
      }
      const size_t rb = (size_t)M.W * sizeof(float);
      eck(cudaMemcpy2DAsync(dev_out + off_out, rb, src + (size_t)M.row_off * e->pitch, (size_t)e->pitch * sizeof(float),
                            rb, M.H, cudaMemcpyDeviceToDevice, e->stream),
          "fip_ensemble_gather");
      off_out += (size_t)M.W * M.H;
    }
    eck(cudaStreamSynchronize(e->stream), "fip_ensemble_gather");
    return FIP_OK;
  });
}

int fip_ensemble_time(fip_ensemble* e, int member, double* duration, float* dt, int* iteration) {
  if (!e) return efail(FIP_ERR_ARG, "null ensemble");
  if (member < 0 || member >= e->n) return efail(FIP_ERR_ARG, "fip_ensemble_time: member out of range");
  const FipEnsCtl& mc = e->h_mctl[member];
  if (duration) *duration = mc.duration;
  if (dt) *dt = mc.dt;
  if (iteration) *iteration = mc.iteration;
  return FIP_OK;
}

int fip_ensemble_info(fip_ensemble* e, fip_ensemble_info_t* out) {
  if (!e || !out) return efail(FIP_ERR_ARG, "null argument");
  return eguard([&] {
    std::memset(out, 0, sizeof *out);
    out->n_members = e->n;
    for (int m = 0; m < e->n; ++m) {
      out->active_members += e->h_mctl[m].active != 0;
      out->cells += (long long)e->mem[m].W * e->mem[m].H;
    }
    out->packed_W = e->packed_W;
    out->packed_rows = e->total_rows;
    out->pitch = e->pitch;
    out->consumer_warps = e->shape.kw;
    out->cols_per_thread = e->shape.nc;
    out->tile_cols = e->shape.cols();
    out->tile_rows = e->shape.tile_rows;
    out->n_tiles = e->st.n_tiles;
    out->iteration = e->h_ctl->iteration;
    if (e->started) {
      std::vector<int> cnt(e->st.n_chunks);
      const int k = e->h_ctl->iteration;
      eck(cudaMemcpy(cnt.data(), e->st.chunk_cnt[k & 1], sizeof(int) * cnt.size(), cudaMemcpyDeviceToHost), "info");
      for (int c : cnt) out->active_tiles += c;
    }
    out->nonfinite = e->h_ctl->nonfinite;
    return FIP_OK;
  });
}

int fip_ensemble_render(fip_ensemble* e, int member, int what, float vmax, unsigned char* rgba_or_null,
                        const char* png_path_or_null) {
  if (!e) return efail(FIP_ERR_ARG, "null ensemble");
  if (member < 0 || member >= e->n) return efail(FIP_ERR_ARG, "fip_ensemble_render: member out of range");
  return eguard([&] {
    eck(cudaSetDevice(e->device), "cudaSetDevice");
    if (what == FIP_RENDER_HMAX) {  // the fold of the member's last step, as fip_ensemble_get_field does
      std::vector<float> tmp((size_t)e->mem[member].W * e->mem[member].H);
      const int rc = fip_ensemble_get_field(e, member, FIP_FIELD_HMAX, tmp.data());
      if (rc) return rc;
    }
    const FipEnsMember& M = e->mem[member];
    const int p = e->parity_of(member);
    const size_t off = (size_t)M.row_off * e->pitch;
    const float* src = what == FIP_RENDER_HMAX ? e->st.hmax + off : e->st.h[p] + off;
    return fip::render_region(e->device, e->stream, src, e->st.qx[p] + off, e->st.qy[p] + off, e->st.sohle + off, M.W,
                              M.H, e->pitch, M.no_value, what, vmax, rgba_or_null, png_path_or_null);
  });
}

void fip_ensemble_destroy(fip_ensemble* e) { delete e; }

}  // extern "C"
