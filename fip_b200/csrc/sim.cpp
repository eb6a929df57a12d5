// Simulation handle: device buffers, the batched step loop and the events of the reference's
// simulate() (src/main.cpp:100-135), behind the C ABI of include/fip.h.
//
// A step is two launches on the handle's stream: the rmg stencil (rmg_stencil.cu) and the
// NVRTC-built post kernel (bc_codegen.cpp). All per-step scalars stay on the device (FipCtl), so
// batches of up to 64 steps run as one captured CUDA graph; the post kernel stops a batch
// (ctl->stop) at the steps where the reference samples, dumps or ends the run, and the host
// handles that event and resumes.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "bc_codegen.h"
#include "config.h"
#include "drv.h"
#include "fip.h"
#include "fip_ctl.h"
#include "render.h"
#include "rmg_stencil.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}
void ckd(CUresult r, const char* what) {
  if (r != CUDA_SUCCESS) throw CudaError(fip::drv::message(r, what));
}

constexpr double kInf = std::numeric_limits<double>::infinity();

}  // namespace

namespace fip {
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace fip

namespace {
// NVTX range for the lifetime of a scope (visible under Nsight Systems / ncu --nvtx; a no-op when
// no tool is attached)
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
};
}  // namespace

struct fip_handle {
  fip::Config cfg;
  fip_options opt;
  int device = 0;
  cudaStream_t stream = nullptr;
  fip::StencilState st{};
  fip::PostKernel post;
  fip::SeriesLayout series;
  float* d_series = nullptr;
  FipCtl* d_ctl = nullptr;
  FipCtl* h_ctl = nullptr;  // pinned mirror
  double* d_vol_partials = nullptr;
  double* d_vol = nullptr;
  int* d_sample_idx = nullptr;
  float* d_sample_val = nullptr;
  float* h_sample_val = nullptr;
  int grid_ctas = 0;
  bool started = false;     // the iteration-0 boundary conditions have run
  bool replan = false;      // the host replaced state fields: recompute the active tiles
  double sample_timer = 0;  // Sampling::timer
  size_t save_pos = 0;
  std::map<int, cudaGraphExec_t> graphs;
  std::ostream* out = &std::cout;
  std::unique_ptr<std::ofstream> out_file;
  // pipelined state exchange (fip_stage_state / fip_step_exchange): two pitched input and two
  // output slots of (h, qx, qy), a copy-in and a copy-out stream, events between the streams
  struct Exchange {
    bool ready = false;
    cudaStream_t in = nullptr, out = nullptr;
    float* slot_in[2][3] = {};
    float* slot_out[2][3] = {};
    cudaEvent_t in_ready[2] = {}, in_free[2] = {}, out_ready[2] = {}, out_done[2] = {};
    bool out_pending[2] = {};
    int head = 0, count = 0, out_next = 0;
  } x;

  ~fip_handle();
  void exchange_setup();
  void init(const std::string& yaml, const fip_options& o);
  void write_ctl_fields();
  void read_ctl();
  void launch_post(int mode);
  void launch_step_pair();
  void launch_batch(int k);
  int run_steps(long long budget, bool to_target);
  void sample();
  void dump(const std::string& prefix, bool current);
  void flush_hmax_if_due();
  int steps_hint() const;
};

fip_handle::~fip_handle() {
  if (device >= 0) cudaSetDevice(device);
  if (x.ready) {
    cudaStreamSynchronize(x.in);
    cudaStreamSynchronize(x.out);
    for (int s = 0; s < 2; ++s) {
      for (int f = 0; f < 3; ++f) {
        cudaFree(x.slot_in[s][f]);
        cudaFree(x.slot_out[s][f]);
      }
      cudaEventDestroy(x.in_ready[s]);
      cudaEventDestroy(x.in_free[s]);
      cudaEventDestroy(x.out_ready[s]);
      cudaEventDestroy(x.out_done[s]);
    }
    cudaStreamDestroy(x.in);
    cudaStreamDestroy(x.out);
  }
  for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
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
  cudaFree(d_series);
  cudaFree(d_ctl);
  cudaFree(d_vol_partials);
  cudaFree(d_vol);
  cudaFree(d_sample_idx);
  cudaFree(d_sample_val);
  if (h_ctl) cudaFreeHost(h_ctl);
  if (h_sample_val) cudaFreeHost(h_sample_val);
  if (stream) cudaStreamDestroy(stream);
}

void fip_handle::init(const std::string& yaml, const fip_options& o) {
  opt = o;
  device = o.device;
  ck(cudaSetDevice(device), "cudaSetDevice");
  ck(cudaFree(nullptr), "CUDA context");
  std::string derr;
  if (!fip::drv::load(&derr)) throw CudaError(derr);
  ck(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
  const size_t W = cfg.W, H = cfg.H;
  const size_t row_bytes = W * sizeof(float);
  size_t pitch_bytes = 0;
  // initDeviceBuffers (src/simdata.cpp:54-96): pitched fields of H+3 rows
  auto alloc_field = [&](float** p) {
    size_t pb = 0;
    ck(cudaMallocPitch((void**)p, &pb, row_bytes, H + 3), "cudaMallocPitch");
    if (pitch_bytes && pb != pitch_bytes) throw CudaError("inconsistent pitch");
    pitch_bytes = pb;
    ck(cudaMemset2D(*p, pb, 0, row_bytes, H + 3), "cudaMemset2D");
  };
  for (int b = 0; b < 2; ++b) {
    alloc_field(&st.h[b]);
    alloc_field(&st.qx[b]);
    alloc_field(&st.qy[b]);
  }
  alloc_field(&st.sohle);
  alloc_field(&st.hmax);
  if (cfg.has_kst_var) alloc_field(&st.kst);
  if (pitch_bytes % 16) throw CudaError("row pitch is not a multiple of 16 bytes");
  const int pitch = (int)(pitch_bytes / sizeof(float));
  auto up = [&](float* dst, const std::vector<float>& src) {
    ck(cudaMemcpy2D(dst, pitch_bytes, src.data(), row_bytes, row_bytes, H, cudaMemcpyHostToDevice), "cudaMemcpy2D");
  };
  for (int b = 0; b < 2; ++b) {
    up(st.h[b], cfg.h0);
    up(st.qx[b], cfg.qx0);
    up(st.qy[b], cfg.qy0);
  }
  up(st.hmax, cfg.h0);
  up(st.sohle, cfg.terrain);
  if (cfg.has_kst_var) up(st.kst, cfg.kst);

  st.W = (int)W;
  st.H = (int)H;
  st.pitch = pitch;
  st.dx = cfg.dx;
  st.kst_fixed = cfg.kst_fixed;
  st.no_value = cfg.no_data;
  st.nc = 4;
  st.tile_cols = fip::single_tile_cols(st.nc);
  fip::tile_geometry(st.W, st.H, st.tile_cols, &st.n_sx, &st.n_ty, &st.n_tiles, &st.n_chunks);
  if (st.n_chunks > 256) throw CudaError("grid too large: more than 131072 tiles");
  fip::bc_tile_force(cfg, &st.force);
  ck(cudaMalloc((void**)&st.sticky, st.n_tiles), "cudaMalloc");
  for (int b = 0; b < 2; ++b) {
    ck(cudaMalloc((void**)&st.nz[b], ((size_t)st.n_tiles + 3) & ~(size_t)3), "cudaMalloc");
    ck(cudaMalloc((void**)&st.list[b], sizeof(int) * st.n_chunks * FIP_PLAN_CHUNK), "cudaMalloc");
    ck(cudaMalloc((void**)&st.chunk_cnt[b], sizeof(int) * st.n_chunks), "cudaMalloc");
    ck(cudaMemset(st.chunk_cnt[b], 0, sizeof(int) * st.n_chunks), "cudaMemset");
  }
  ck(cudaMalloc((void**)&d_ctl, sizeof(FipCtl)), "cudaMalloc");
  st.ctl = d_ctl;
  ckd((CUresult)fip::make_tensor_maps(&st), "cuTensorMapEncodeTiled");

  series = fip::layout_series(cfg);
  ck(cudaMalloc((void**)&d_series, series.data.size() * sizeof(float)), "cudaMalloc");
  ck(cudaMemcpy(d_series, series.data.data(), series.data.size() * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy");

  const int vp = fip::volume_partials(st);
  ck(cudaMalloc((void**)&d_vol_partials, sizeof(double) * vp), "cudaMalloc");
  ck(cudaMalloc((void**)&d_vol, sizeof(double)), "cudaMalloc");
  const int np = (int)cfg.points.size();
  if (np) {
    std::vector<int> idx;
    for (const auto& p : cfg.points) {
      idx.push_back(p.x);
      idx.push_back(p.y);
      idx.push_back((int)p.type);
    }
    ck(cudaMalloc((void**)&d_sample_idx, sizeof(int) * idx.size()), "cudaMalloc");
    ck(cudaMemcpy(d_sample_idx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
    ck(cudaMalloc((void**)&d_sample_val, sizeof(float) * np), "cudaMalloc");
    ck(cudaMallocHost((void**)&h_sample_val, sizeof(float) * np), "cudaMallocHost");
  }

  // control block
  ck(cudaMallocHost((void**)&h_ctl, sizeof(FipCtl)), "cudaMallocHost");
  std::memset(h_ctl, 0, sizeof(FipCtl));
  h_ctl->duration = 0.0;
  h_ctl->next_sample = kInf;
  h_ctl->next_save = cfg.save_times.empty() ? kInf : cfg.save_times[0];
  h_ctl->target = kInf;
  h_ctl->dt = cfg.dt;
  h_ctl->last_cfl = 1.0f;
  h_ctl->variable_dt = cfg.variable_dt ? 1 : 0;
  h_ctl->stop_on_nonfinite = opt.stop_on_nonfinite ? 1 : 0;
  h_ctl->hmax_every = 100;
  bool negative = false;
  for (float v : cfg.h0) negative |= (v < 0.f);
  h_ctl->hmax_full = negative ? 1 : 0;
  h_ctl->force_all = opt.all_tiles ? 1 : 0;
  const float one = 1.0f;
  std::memcpy(&h_ctl->cfl_bits[0], &one, 4);
  std::memcpy(&h_ctl->cfl_bits[1], &one, 4);
  if (cfg.variable_dt) {
    // controlTimestep at the start of the first simulate(): the CFL slots hold 1 (src/simdata.cpp:91-94)
    float min_cfl = 42.0f;
    if (1.0f < min_cfl) min_cfl = 1.0f;
    const float target = min_cfl * .5f, dc = 0.001f;
    float d = h_ctl->dt;
    if (d < target && target - d > dc) d *= 1.001f;
    else if (d > target && d - target > dc) d *= 0.99f;
    h_ctl->dt = d;
  }
  ck(cudaMemcpy(d_ctl, h_ctl, sizeof(FipCtl), cudaMemcpyHostToDevice), "cudaMemcpy");
  ck(fip::launch_init_tiles(st, 0, stream), "init_tiles");
  grid_ctas = fip::rmg_step_grid(device, st.nc);

  // boundary-condition program (BoundaryConditionKernel::generate)
  std::string err;
  std::string src = fip::post_kernel_source(cfg, series, pitch);
  if (fip::build_post_kernel(src, &post, &err)) throw std::invalid_argument("NVRTC:" + err);
  ck(cudaStreamSynchronize(stream), "init");

  if (opt.quiet) {
    out = nullptr;
  } else if (opt.sample_path) {
    out_file.reset(new std::ofstream(opt.sample_path));
    if (!*out_file) throw std::invalid_argument(std::string("IO:cannot open ") + opt.sample_path);
    out = out_file.get();
  }
  if (out && !cfg.points.empty()) {  // sampleHeader (src/main.cpp:45-51)
    *out << "t;";
    for (const auto& p : cfg.points) *out << p.label << ";";
    *out << std::endl;
  }
}

// Slots, streams and events of the pipelined exchange, made at its first use.
void fip_handle::exchange_setup() {
  if (x.ready) return;
  const size_t bytes = (size_t)st.pitch * sizeof(float) * (cfg.H + 3);
  ck(cudaStreamCreateWithFlags(&x.in, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaStreamCreateWithFlags(&x.out, cudaStreamNonBlocking), "cudaStreamCreate");
  for (int s = 0; s < 2; ++s) {
    for (int f = 0; f < 3; ++f) {
      ck(cudaMalloc((void**)&x.slot_in[s][f], bytes), "cudaMalloc");
      ck(cudaMalloc((void**)&x.slot_out[s][f], bytes), "cudaMalloc");
    }
    ck(cudaEventCreateWithFlags(&x.in_ready[s], cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&x.in_free[s], cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&x.out_ready[s], cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&x.out_done[s], cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventRecord(x.in_free[s], stream), "cudaEventRecord");
    ck(cudaEventRecord(x.out_done[s], x.out), "cudaEventRecord");
  }
  x.ready = true;
}

// host-owned control fields: event times, step budget, stop flag
void fip_handle::write_ctl_fields() {
  const size_t off = offsetof(FipCtl, duration);
  (void)off;
  // the device owns duration/dt/iteration/parity; write only the fields the host controls
  auto put = [&](size_t offset, size_t bytes) {
    ck(cudaMemcpyAsync(reinterpret_cast<char*>(d_ctl) + offset, reinterpret_cast<char*>(h_ctl) + offset, bytes,
                       cudaMemcpyHostToDevice, stream),
       "ctl upload");
  };
  put(offsetof(FipCtl, next_sample), 3 * sizeof(double));  // next_sample, next_save, target
  put(offsetof(FipCtl, stop), 3 * sizeof(int));            // stop, stop_reason, steps_left
}

void fip_handle::read_ctl() {
  ck(cudaMemcpyAsync(h_ctl, d_ctl, sizeof(FipCtl), cudaMemcpyDeviceToHost, stream), "ctl download");
  ck(cudaStreamSynchronize(stream), "step");
}

void fip_handle::launch_post(int mode) {
  FipPostArgs a;
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
  a.sticky = st.sticky;
  a.series = d_series;
  a.W = st.W;
  a.H = st.H;
  a.pitch = st.pitch;
  a.n_sx = st.n_sx;
  a.n_ty = st.n_ty;
  a.n_tiles = st.n_tiles;
  a.n_chunks = st.n_chunks;
  a.mode = mode;
  a.dx = st.dx;
  void* params[] = {&a};
  ckd(fip::drv::LaunchKernel(post.fn, 1 + st.n_chunks, 1, 1, FIP_POST_THREADS, 1, 1, 0, (CUstream)stream, params, nullptr),
      "fip_post launch");
}

void fip_handle::launch_step_pair() {
  ck(fip::launch_rmg_step(st, grid_ctas, stream), "rmg_step launch");
  launch_post(FIP_POST_MODE_STEP);
}

void fip_handle::launch_batch(int k) {
  if (!opt.use_graphs || k == 1) {
    for (int i = 0; i < k; ++i) launch_step_pair();
    return;
  }
  auto it = graphs.find(k);
  if (it == graphs.end()) {
    cudaGraph_t g;
    ck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture");
    for (int i = 0; i < k; ++i) launch_step_pair();
    ck(cudaStreamEndCapture(stream, &g), "capture");
    cudaGraphExec_t ex;
    ck(cudaGraphInstantiate(&ex, g, 0), "cudaGraphInstantiate");
    cudaGraphDestroy(g);
    it = graphs.emplace(k, ex).first;
  }
  ck(cudaGraphLaunch(it->second, stream), "cudaGraphLaunch");
}

// Steps until the next event can end a batch: exact for fixed dt (same double accumulation as
// the device), a lower estimate for variable dt.
int fip_handle::steps_hint() const {
  double next = std::min(h_ctl->next_sample, std::min(h_ctl->next_save, h_ctl->target));
  const long long budget = h_ctl->steps_left;
  long long n = budget;
  if (next < kInf) {
    double d = h_ctl->duration;
    long long j = 0;
    if (!cfg.variable_dt) {
      const float dt = h_ctl->dt;
      while (j < 64 && d < next) {
        d += dt;
        ++j;
      }
      if (d < next) j = 64;
    } else {
      const double dtmax = (double)h_ctl->dt * 1.07;  // at most +0.1% per step over 64 steps
      j = dtmax > 0 ? (long long)((next - d) / dtmax) : 1;
      if (j < 1) j = 1;
    }
    n = std::min(n, j);
  }
  if (n > 64) n = 64;
  if (n < 1) n = 1;
  int k = 1;
  while (k * 2 <= n) k *= 2;
  return k;
}

void fip_handle::flush_hmax_if_due() {
  if (h_ctl->iteration > 0 && h_ctl->iteration % h_ctl->hmax_every == 0)
    ck(fip::launch_hmax_fold(st, h_ctl->parity, stream), "hmax");
}

void fip_handle::sample() {  // sample (src/main.cpp:53-83)
  if (!out) return;
  Range range("sampling");
  const int np = (int)cfg.points.size();
  if (np) {
    ck(fip::launch_sample_gather(st, h_ctl->parity, np, d_sample_idx, d_sample_val, stream), "sample");
    ck(cudaMemcpyAsync(h_sample_val, d_sample_val, sizeof(float) * np, cudaMemcpyDeviceToHost, stream), "sample");
    ck(cudaStreamSynchronize(stream), "sample");
  }
  *out << h_ctl->duration << ";";
  for (int i = 0; i < np; ++i) *out << h_sample_val[i] << ";";
  *out << std::endl;
}

void fip_handle::dump(const std::string& prefix, bool current) {
  // dumpDeviceBuffers (src/main.cpp:180-202)
  Range range("save_state dump");
  ck(cudaStreamSynchronize(stream), "dump");
  const size_t W = cfg.W, H = cfg.H;
  std::vector<float> buf(W * H);
  char stamp[64];
  std::time_t now = std::time(nullptr);
  std::tm tmv;
  gmtime_r(&now, &tmv);
  std::strftime(stamp, sizeof stamp, "%Y-%m-%d-%H-%M", &tmv);
  const int b = current ? h_ctl->parity : (h_ctl->parity ^ 1);
  const float* src[4] = {st.h[b], st.qx[b], st.qy[b], st.hmax};
  const char* tag[4] = {"_ah_", "_qx_", "_qy_", "_flood_plains_"};
  for (int f = 0; f < 4; ++f) {
    ck(cudaMemcpy2D(buf.data(), W * 4, src[f], (size_t)st.pitch * 4, W * 4, H, cudaMemcpyDeviceToHost), "dump");
    std::string fn = prefix + tag[f] + std::to_string((int)h_ctl->duration) + "_" + stamp;
    std::ofstream file(fn, std::ios::binary);
    if (!file) throw std::invalid_argument("IO:Failed to open file " + fn);
    size_t w = W, hh = H;
    file.write(reinterpret_cast<const char*>(&w), sizeof(size_t));
    file.write(reinterpret_cast<const char*>(&hh), sizeof(size_t));
    file.write(reinterpret_cast<const char*>(buf.data()), (std::streamsize)(W * H * sizeof(float)));
    if (!file) throw std::invalid_argument("IO:write failed: " + fn);
  }
}

// Runs up to `budget` simulate() calls (or until target_duration when to_target).
int fip_handle::run_steps(long long budget, bool to_target) {
  Range range("fip steps");
  ck(cudaSetDevice(device), "cudaSetDevice");
  if (to_target && h_ctl->duration >= cfg.target_duration) return FIP_OK;
  if (budget <= 0) return FIP_OK;
  if (!started) {
    // start of the first simulate(): sampling before the iteration-0 boundary conditions
    if (h_ctl->duration >= sample_timer && cfg.sampling_interval > 0) {
      sample_timer += cfg.sampling_interval;
      sample();
    }
    h_ctl->next_sample = cfg.sampling_interval > 0 ? sample_timer : kInf;
    h_ctl->stop = 0;
    h_ctl->stop_reason = 0;
    h_ctl->steps_left = 1;
    write_ctl_fields();
    Range r0("boundary conditions, iteration 0");
    launch_post(FIP_POST_MODE_INIT);
    started = true;
  }
  if (replan) {
    Range r1("active-tile plan");
    ck(fip::launch_init_tiles(st, h_ctl->parity, stream), "init_tiles");
    launch_post(FIP_POST_MODE_PLAN);
    replan = false;
  }
  h_ctl->target = to_target ? cfg.target_duration : kInf;
  h_ctl->steps_left = budget > (1LL << 30) ? (1 << 30) : (int)budget;
  h_ctl->stop = 0;
  h_ctl->stop_reason = 0;
  write_ctl_fields();
  const int it0 = h_ctl->iteration;
  int rc = FIP_OK;
  for (;;) {
    {
      Range rb("batch: stencil + boundary conditions / plan / dt");
      launch_batch(steps_hint());
      read_ctl();
    }
    if (h_ctl->error) return fail(FIP_ERR_DEVICE_TIMEOUT, "device wait ran out (code " + std::to_string(h_ctl->error) + ")");
    const int reason = h_ctl->stop ? h_ctl->stop_reason : 0;
    bool done = false;
    if (reason & FIP_STOP_SAVE) {  // end of simulate(): dump after hmax
      flush_hmax_if_due();
      ++save_pos;
      dump(cfg.name, false);
      h_ctl->next_save = save_pos < cfg.save_times.size() ? cfg.save_times[save_pos] : kInf;
    }
    if (reason & FIP_STOP_TARGET) done = true;
    if ((reason & FIP_STOP_SAMPLE) && !done) {  // start of the next simulate()
      sample_timer += cfg.sampling_interval;
      sample();
      h_ctl->next_sample = sample_timer;
    }
    if (reason & FIP_STOP_NONFINITE) {
      rc = fail(FIP_ERR_NONFINITE, "a stored water depth is NaN or Inf at iteration " + std::to_string(h_ctl->iteration));
      done = true;
    }
    if (reason & FIP_STOP_BUDGET) done = true;
    const long long ran = h_ctl->iteration - it0;
    if (!done && !to_target && ran >= budget) done = true;
    h_ctl->stop = 0;
    h_ctl->stop_reason = 0;
    h_ctl->steps_left = to_target ? (1 << 30) : (int)(budget - ran);
    write_ctl_fields();
    if (done) break;
  }
  flush_hmax_if_due();
  ck(cudaStreamSynchronize(stream), "step");
  return rc;
}

// ------------------------------------------------------------------------------------------
namespace {

int guard(const std::function<int()>& f) {
  try {
    return f();
  } catch (const CudaError& e) {
    return fail(FIP_ERR_CUDA, e.what());
  } catch (const std::invalid_argument& e) {
    std::string m = e.what();
    if (m.rfind("IO:", 0) == 0) return fail(FIP_ERR_IO, m.substr(3));
    if (m.rfind("NVRTC:", 0) == 0) return fail(FIP_ERR_NVRTC, m.substr(6));
    return fail(FIP_ERR_CONFIG, m);
  } catch (const std::exception& e) {
    return fail(FIP_ERR_CUDA, e.what());
  }
}

}  // namespace

namespace fip {

// Renders one field of a grid (pointers at its first row) to rgba_or_null and/or a PNG file.
int render_region(int device, cudaStream_t stream, const float* h, const float* qx, const float* qy,
                  const float* sohle, int W, int H, int pitch, float no_value, int what, float vmax,
                  unsigned char* rgba_or_null, const char* png_path_or_null) {
  (void)device;
  if (what < FIP_RENDER_DEPTH || what > FIP_RENDER_HMAX) return fail(FIP_ERR_ARG, "fip_render: unknown field to render");
  if (!(vmax > 0.f)) vmax = 5.0f;  // the viewer's default scale: 5 m, 5 m/s (src/vis.cpp:264-265)
  const size_t n = (size_t)W * H * 4;
  unsigned char* d = nullptr;
  ck(cudaMallocAsync((void**)&d, n, stream), "fip_render");
  std::vector<unsigned char> img(n);
  cudaError_t e = launch_render(h, qx, qy, sohle, W, H, pitch, no_value, what, vmax, d, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(img.data(), d, n, cudaMemcpyDeviceToHost, stream);
  cudaFreeAsync(d, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  ck(e, "fip_render");
  if (rgba_or_null) std::memcpy(rgba_or_null, img.data(), n);
  if (png_path_or_null) {
    const std::string err = write_png_rgba(png_path_or_null, img.data(), W, H);
    if (!err.empty()) throw std::invalid_argument("IO:" + err);
  }
  return FIP_OK;
}

}  // namespace fip

extern "C" {

void fip_default_options(fip_options* o) {
  std::memset(o, 0, sizeof *o);
  o->device = 0;
  o->use_graphs = 1;
}

int fip_init_ex(const char* yaml_path, const fip_options* opt, fip_handle** out) {
  if (!yaml_path || !out) return fail(FIP_ERR_ARG, "null argument");
  *out = nullptr;
  g_last_error.clear();
  fip_options o;
  fip_default_options(&o);
  if (opt) o = *opt;
  std::unique_ptr<fip_handle> h(new fip_handle());
  std::string err;
  int rc = fip::load_config(yaml_path, &h->cfg, &err, o.quiet != 0);
  if (rc == 2) return fail(FIP_ERR_IO, err);
  if (rc) return fail(FIP_ERR_CONFIG, err);
  rc = guard([&] {
    h->init(yaml_path, o);
    return FIP_OK;
  });
  if (rc) return rc;
  *out = h.release();
  return FIP_OK;
}

int fip_init(const char* yaml_path, fip_handle** out) { return fip_init_ex(yaml_path, nullptr, out); }

int fip_step(fip_handle* h, int n) {
  if (!h || n < 0) return fail(FIP_ERR_ARG, "bad argument");
  return guard([&] { return h->run_steps(n, false); });
}

int fip_run(fip_handle* h) {
  if (!h) return fail(FIP_ERR_ARG, "null handle");
  return guard([&] { return h->run_steps(std::numeric_limits<long long>::max(), true); });
}

int fip_save(fip_handle* h, const char* prefix) {
  if (!h) return fail(FIP_ERR_ARG, "null handle");
  return guard([&] {
    h->dump(prefix ? prefix : h->cfg.name, false);
    return FIP_OK;
  });
}

int fip_save_current(fip_handle* h, const char* prefix) {
  if (!h) return fail(FIP_ERR_ARG, "null handle");
  return guard([&] {
    h->dump(prefix ? prefix : h->cfg.name, true);
    return FIP_OK;
  });
}

// ---- exact resume ----
// The reference's only restart path is to feed a save_state dump back as z/qx/qy input files
// (offset 16): the dump holds depth while the loader reads z as a level (src/main.cpp:189 vs
// src/simdata.cpp:266-270), the level round trip rounds the depths, and time, dt, iteration,
// hmax and the ping-pong partner are lost. A checkpoint keeps all of it, so a restored run
// continues bit for bit.
namespace {

constexpr char kCkptMagic[8] = {'F', 'I', 'P', 'C', 'K', 'P', 'T', '1'};

struct CkptHeader {
  char magic[8];
  uint32_t version, header_bytes;
  int64_t W, H;
  uint64_t terrain_hash;  // FNV-1a over the terrain floats: the checkpoint belongs to this scenario
  double duration, sample_timer;
  float dt, last_cfl;
  int32_t iteration, parity, save_pos, started, nonfinite, hmax_full;
};

uint64_t fnv1a(const void* p, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  uint64_t x = 1469598103934665603ull;
  for (size_t i = 0; i < n; ++i) x = (x ^ b[i]) * 1099511628211ull;
  return x;
}

}  // namespace

int fip_checkpoint(fip_handle* h, const char* path) {
  if (!h || !path) return fail(FIP_ERR_ARG, "null argument");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(h->stream), "checkpoint");
    const size_t W = h->cfg.W, H = h->cfg.H;
    CkptHeader hd;
    std::memset(&hd, 0, sizeof hd);
    std::memcpy(hd.magic, kCkptMagic, 8);
    hd.version = 1;
    hd.header_bytes = sizeof hd;
    hd.W = (int64_t)W;
    hd.H = (int64_t)H;
    hd.terrain_hash = fnv1a(h->cfg.terrain.data(), W * H * sizeof(float));
    hd.duration = h->h_ctl->duration;
    hd.sample_timer = h->sample_timer;
    hd.dt = h->h_ctl->dt;
    hd.last_cfl = h->h_ctl->last_cfl;
    hd.iteration = h->h_ctl->iteration;
    hd.parity = h->h_ctl->parity;
    hd.save_pos = (int32_t)h->save_pos;
    hd.started = h->started ? 1 : 0;
    hd.nonfinite = h->h_ctl->nonfinite;
    hd.hmax_full = h->h_ctl->hmax_full;
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::invalid_argument(std::string("IO:cannot open ") + path);
    f.write(reinterpret_cast<const char*>(&hd), sizeof hd);
    const int p = hd.parity;
    const float* src[7] = {h->st.h[p], h->st.qx[p], h->st.qy[p], h->st.h[p ^ 1], h->st.qx[p ^ 1], h->st.qy[p ^ 1],
                           h->st.hmax};
    std::vector<float> buf(W * H);
    for (const float* s : src) {
      ck(cudaMemcpy2D(buf.data(), W * 4, s, (size_t)h->st.pitch * 4, W * 4, H, cudaMemcpyDeviceToHost), "checkpoint");
      f.write(reinterpret_cast<const char*>(buf.data()), (std::streamsize)(W * H * sizeof(float)));
    }
    if (!f) throw std::invalid_argument(std::string("IO:write failed: ") + path);
    return FIP_OK;
  });
}

int fip_restore(fip_handle* h, const char* path) {
  if (!h || !path) return fail(FIP_ERR_ARG, "null argument");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    const size_t W = h->cfg.W, H = h->cfg.H;
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::invalid_argument(std::string("IO:cannot open ") + path);
    CkptHeader hd;
    f.read(reinterpret_cast<char*>(&hd), sizeof hd);
    if (!f || std::memcmp(hd.magic, kCkptMagic, 8) != 0 || hd.version != 1 || hd.header_bytes != sizeof hd)
      throw std::invalid_argument(std::string("IO:") + path + " is not a fip_b200 checkpoint");
    if (hd.W != (int64_t)W || hd.H != (int64_t)H)
      throw std::invalid_argument(std::string("checkpoint ") + path + " is for a " + std::to_string(hd.W) + " x " +
                                  std::to_string(hd.H) + " grid");
    if (hd.terrain_hash != fnv1a(h->cfg.terrain.data(), W * H * sizeof(float)))
      throw std::invalid_argument(std::string("checkpoint ") + path + " was written for a different terrain");
    if (hd.parity != 0 && hd.parity != 1) throw std::invalid_argument(std::string("IO:") + path + ": bad parity");
    const int p = hd.parity;
    float* dst[7] = {h->st.h[p], h->st.qx[p], h->st.qy[p], h->st.h[p ^ 1], h->st.qx[p ^ 1], h->st.qy[p ^ 1],
                     h->st.hmax};
    std::vector<float> buf(W * H);
    for (float* d : dst) {
      f.read(reinterpret_cast<char*>(buf.data()), (std::streamsize)(W * H * sizeof(float)));
      if (!f) throw std::invalid_argument(std::string("IO:") + path + " is truncated");
      ck(cudaMemcpy2D(d, (size_t)h->st.pitch * 4, buf.data(), W * 4, W * 4, H, cudaMemcpyHostToDevice), "restore");
    }
    FipCtl* c = h->h_ctl;
    c->duration = hd.duration;
    c->dt = hd.dt;
    c->last_cfl = hd.last_cfl;
    c->iteration = hd.iteration;
    c->parity = p;
    c->nonfinite = hd.nonfinite;
    c->hmax_full = hd.hmax_full;
    c->stop = c->stop_reason = c->error = 0;
    c->post_done = 0u;
    const float one = 1.0f;
    std::memcpy(&c->cfl_bits[0], &one, 4);
    std::memcpy(&c->cfl_bits[1], &one, 4);
    h->sample_timer = hd.sample_timer;
    h->save_pos = (size_t)std::max(0, hd.save_pos);
    h->started = hd.started != 0;
    c->next_save = h->save_pos < h->cfg.save_times.size() ? h->cfg.save_times[h->save_pos] : kInf;
    c->next_sample = (h->started && h->cfg.sampling_interval > 0) ? h->sample_timer : kInf;
    c->target = kInf;
    ck(cudaMemcpyAsync(h->d_ctl, c, sizeof(FipCtl), cudaMemcpyHostToDevice, h->stream), "restore");
    // exact plan of the restored state: a tile is computed when it or a neighbour holds water, or
    // while the partner buffer (the next step's output) still holds water in it
    const int k = hd.iteration - 1;
    ck(fip::launch_init_tiles_region(h->st.h[p], h->st.qx[p], h->st.qy[p], h->st.h[p ^ 1], h->st.qx[p ^ 1],
                                     h->st.qy[p ^ 1], h->st.sohle, h->st.W, h->st.H, h->st.pitch, h->st.no_value,
                                     h->st.tile_cols, FIP_TILE_ROWS, h->st.force, h->st.sticky, h->st.nz[k & 1],
                                     h->st.nz[(k + 1) & 1],
                                     h->stream),
       "init_tiles");
    if (h->started) h->launch_post(FIP_POST_MODE_PLAN);
    h->replan = false;
    ck(cudaStreamSynchronize(h->stream), "restore");
    return FIP_OK;
  });
}

int fip_render(fip_handle* h, int what, float vmax, unsigned char* rgba_or_null, const char* png_path_or_null) {
  if (!h) return fail(FIP_ERR_ARG, "null handle");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    if (what == FIP_RENDER_HMAX) h->flush_hmax_if_due();
    const int p = h->h_ctl->parity;
    const float* src = what == FIP_RENDER_HMAX ? h->st.hmax : h->st.h[p];
    return fip::render_region(h->device, h->stream, src, h->st.qx[p], h->st.qy[p], h->st.sohle, h->st.W, h->st.H,
                              h->st.pitch, h->st.no_value, what, vmax, rgba_or_null, png_path_or_null);
  });
}

int fip_sample(fip_handle* h) {
  if (!h) return fail(FIP_ERR_ARG, "null handle");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    h->sample();
    return FIP_OK;
  });
}

int fip_volume(fip_handle* h, double* outv) {
  if (!h || !outv) return fail(FIP_ERR_ARG, "null argument");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    Range range("volume reduction (FP64)");
    ck(fip::launch_volume(h->st, h->h_ctl->parity, h->d_vol_partials, h->d_vol, h->stream), "volume");
    double v = 0;
    ck(cudaMemcpyAsync(&v, h->d_vol, sizeof(double), cudaMemcpyDeviceToHost, h->stream), "volume");
    ck(cudaStreamSynchronize(h->stream), "volume");
    *outv = v * (double)h->cfg.dx * (double)h->cfg.dx;
    return FIP_OK;
  });
}

int fip_get_field(fip_handle* h, int field, float* dst) {
  if (!h || !dst) return fail(FIP_ERR_ARG, "null argument");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    const int p = h->h_ctl->parity;
    const float* src = nullptr;
    switch (field) {
      case FIP_FIELD_H: src = h->st.h[p]; break;
      case FIP_FIELD_QX: src = h->st.qx[p]; break;
      case FIP_FIELD_QY: src = h->st.qy[p]; break;
      case FIP_FIELD_HMAX: src = h->st.hmax; break;
      case FIP_FIELD_H_PREV: src = h->st.h[p ^ 1]; break;
      case FIP_FIELD_QX_PREV: src = h->st.qx[p ^ 1]; break;
      case FIP_FIELD_QY_PREV: src = h->st.qy[p ^ 1]; break;
      case FIP_FIELD_TERRAIN: src = h->st.sohle; break;
      case FIP_FIELD_Z: src = h->st.h[p]; break;
      default: return fail(FIP_ERR_ARG, "unknown field " + std::to_string(field));
    }
    const size_t W = h->cfg.W, H = h->cfg.H;
    ck(cudaMemcpy2DAsync(dst, W * 4, src, (size_t)h->st.pitch * 4, W * 4, H, cudaMemcpyDeviceToHost, h->stream),
       "fip_get_field");
    ck(cudaStreamSynchronize(h->stream), "fip_get_field");
    if (field == FIP_FIELD_Z)
      for (size_t i = 0; i < W * H; ++i) dst[i] += h->cfg.terrain[i];
    return FIP_OK;
  });
}

int fip_set_field(fip_handle* h, int field, const float* src) {
  if (!h || !src) return fail(FIP_ERR_ARG, "null argument");
  if (field != FIP_FIELD_H && field != FIP_FIELD_QX && field != FIP_FIELD_QY)
    return fail(FIP_ERR_ARG, "fip_set_field: only FIP_FIELD_H, FIP_FIELD_QX and FIP_FIELD_QY can be set");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    const int p = h->h_ctl->parity;
    float* const* bufs = field == FIP_FIELD_H ? h->st.h : field == FIP_FIELD_QX ? h->st.qx : h->st.qy;
    const size_t W = h->cfg.W, H = h->cfg.H, pb = (size_t)h->st.pitch * 4;
    ck(cudaMemcpy2DAsync(bufs[p], pb, src, W * 4, W * 4, H, cudaMemcpyHostToDevice, h->stream), "fip_set_field");
    ck(fip::launch_positive_zero_copy(bufs[p], bufs[p], bufs[p ^ 1], (int)W, (int)H, h->st.pitch, h->stream),
       "fip_set_field");
    if (field == FIP_FIELD_H && !h->h_ctl->hmax_full) {
      // a negative depth anywhere makes the hmax fold cover inactive tiles too; the check runs on
      // the copy in device memory (a host scan of the caller's buffer costs tens of ms on large
      // grids) and the flag comes back into the host mirror before this call returns
      ck(fip::launch_flag_negative(bufs[p], (int)W, (int)H, h->st.pitch, &h->d_ctl->hmax_full, h->stream),
         "fip_set_field");
      ck(cudaMemcpyAsync(&h->h_ctl->hmax_full, &h->d_ctl->hmax_full, sizeof(int), cudaMemcpyDeviceToHost,
                         h->stream),
         "fip_set_field");
    }
    h->replan = true;
    ck(cudaStreamSynchronize(h->stream), "fip_set_field");
    return FIP_OK;
  });
}

int fip_stage_state(fip_handle* h, const float* h_src, const float* qx_src, const float* qy_src) {
  if (!h || !h_src || !qx_src || !qy_src) return fail(FIP_ERR_ARG, "null argument");
  if (h->x.ready && h->x.count == 2) return fail(FIP_ERR_ARG, "fip_stage_state: two states are already staged");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    h->exchange_setup();
    auto& x = h->x;
    const int s = (x.head + x.count) & 1;
    const size_t W = h->cfg.W, H = h->cfg.H, pb = (size_t)h->st.pitch * 4;
    // the slot's previous contents must have been copied into the state first
    ck(cudaStreamWaitEvent(x.in, x.in_free[s], 0), "fip_stage_state");
    const float* src[3] = {h_src, qx_src, qy_src};
    for (int f = 0; f < 3; ++f)
      ck(cudaMemcpy2DAsync(x.slot_in[s][f], pb, src[f], W * 4, W * 4, H, cudaMemcpyHostToDevice, x.in),
         "fip_stage_state");
    ck(cudaEventRecord(x.in_ready[s], x.in), "fip_stage_state");
    ++x.count;
    return FIP_OK;
  });
}

int fip_step_exchange(fip_handle* h, int n_steps, float* h_dst, float* qx_dst, float* qy_dst) {
  if (!h || n_steps < 0) return fail(FIP_ERR_ARG, "bad argument");
  if ((h_dst || qx_dst || qy_dst) && !(h_dst && qx_dst && qy_dst))
    return fail(FIP_ERR_ARG, "fip_step_exchange: give all three outputs or none");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    h->exchange_setup();
    auto& x = h->x;
    const size_t bytes = (size_t)h->st.pitch * 4 * h->cfg.H;
    if (x.count > 0) {  // the oldest staged state becomes the current state, in both buffers
      const int s = x.head;
      const int p = h->h_ctl->parity;
      ck(cudaStreamWaitEvent(h->stream, x.in_ready[s], 0), "fip_step_exchange");
      float* const* bufs[3] = {h->st.h, h->st.qx, h->st.qy};
      for (int f = 0; f < 3; ++f)  // one pass: slot -> both ping-pong buffers, zeros as +0
        ck(fip::launch_positive_zero_copy(x.slot_in[s][f], bufs[f][p], bufs[f][p ^ 1], (int)h->cfg.W, (int)h->cfg.H,
                                          h->st.pitch, h->stream),
           "exchange");
      ck(cudaEventRecord(x.in_free[s], h->stream), "exchange");
      // a negative depth makes the hmax fold cover inactive tiles (as fip_set_field); the flag
      // stays on the device, where the stencil reads it
      ck(fip::launch_flag_negative(h->st.h[p], (int)h->cfg.W, (int)h->cfg.H, h->st.pitch, &h->d_ctl->hmax_full,
                                   h->stream),
         "exchange");
      h->replan = true;
      x.head ^= 1;
      --x.count;
    }
    int rc = n_steps > 0 ? h->run_steps(n_steps, false) : FIP_OK;
    if (rc) return rc;
    // the previous call's downloads end before this call returns
    const int prev = x.out_next ^ 1;
    if (h_dst) {
      const int o = x.out_next;
      const int p = h->h_ctl->parity;
      const size_t W = h->cfg.W, H = h->cfg.H, pb = (size_t)h->st.pitch * 4;
      ck(cudaStreamWaitEvent(h->stream, x.out_done[o], 0), "exchange");
      const float* cur[3] = {h->st.h[p], h->st.qx[p], h->st.qy[p]};
      float* dst[3] = {h_dst, qx_dst, qy_dst};
      for (int f = 0; f < 3; ++f)
        ck(cudaMemcpyAsync(x.slot_out[o][f], cur[f], bytes, cudaMemcpyDeviceToDevice, h->stream), "exchange");
      ck(cudaEventRecord(x.out_ready[o], h->stream), "exchange");
      ck(cudaStreamWaitEvent(x.out, x.out_ready[o], 0), "exchange");
      for (int f = 0; f < 3; ++f)
        ck(cudaMemcpy2DAsync(dst[f], W * 4, x.slot_out[o][f], pb, W * 4, H, cudaMemcpyDeviceToHost, x.out),
           "exchange");
      ck(cudaEventRecord(x.out_done[o], x.out), "exchange");
      x.out_pending[o] = true;
      x.out_next ^= 1;
    }
    if (x.out_pending[prev]) {
      ck(cudaEventSynchronize(x.out_done[prev]), "exchange");
      x.out_pending[prev] = false;
    }
    return FIP_OK;
  });
}

int fip_exchange_wait(fip_handle* h) {
  if (!h) return fail(FIP_ERR_ARG, "null handle");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    if (!h->x.ready) return FIP_OK;
    ck(cudaStreamSynchronize(h->stream), "fip_exchange_wait");
    ck(cudaStreamSynchronize(h->x.in), "fip_exchange_wait");
    ck(cudaStreamSynchronize(h->x.out), "fip_exchange_wait");
    h->x.out_pending[0] = h->x.out_pending[1] = false;
    return FIP_OK;
  });
}

int fip_inject_wait_timeout(fip_handle* h) {
  if (!h) return fail(FIP_ERR_ARG, "null handle");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    h->h_ctl->inject = 1;
    ck(cudaMemcpyAsync(&h->d_ctl->inject, &h->h_ctl->inject, sizeof(int), cudaMemcpyHostToDevice, h->stream),
       "fip_inject_wait_timeout");
    ck(cudaStreamSynchronize(h->stream), "fip_inject_wait_timeout");
    h->h_ctl->inject = 0;  // the device copy is cleared by the stencil that takes it
    return FIP_OK;
  });
}

int fip_time(fip_handle* h, double* duration, float* dt, int* iteration) {
  if (!h) return fail(FIP_ERR_ARG, "null handle");
  if (duration) *duration = h->h_ctl->duration;
  if (dt) *dt = h->h_ctl->dt;
  if (iteration) *iteration = h->h_ctl->iteration;
  return FIP_OK;
}

int fip_info(fip_handle* h, fip_info_t* o) {
  if (!h || !o) return fail(FIP_ERR_ARG, "null argument");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    std::memset(o, 0, sizeof *o);
    o->W = h->st.W;
    o->H = h->st.H;
    o->pitch = h->st.pitch;
    o->n_tiles = h->st.n_tiles;
    if (h->started) {
      std::vector<int> cnt(h->st.n_chunks);
      ck(cudaMemcpy(cnt.data(), h->st.chunk_cnt[h->h_ctl->iteration & 1], sizeof(int) * cnt.size(),
                    cudaMemcpyDeviceToHost),
         "fip_info");
      for (int c : cnt) o->active_tiles += c;
    } else {
      o->active_tiles = -1;
    }
    o->iteration = h->h_ctl->iteration;
    o->duration = h->h_ctl->duration;
    o->dt = h->h_ctl->dt;
    o->last_cfl = h->h_ctl->last_cfl;
    o->nonfinite = h->h_ctl->nonfinite;
    return FIP_OK;
  });
}

int fip_profile_steps(fip_handle* h, int n, float* stencil_ms, float* post_ms) {
  if (!h || n <= 0) return fail(FIP_ERR_ARG, "bad argument");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    if (!h->started) {
      int rc = h->run_steps(1, false);
      if (rc) return rc;
    }
    h->h_ctl->target = kInf;
    h->h_ctl->next_sample = kInf;  // profiling steps skip sampling and saves
    const double save_keep = h->h_ctl->next_save;
    h->h_ctl->next_save = kInf;
    h->h_ctl->steps_left = n;
    h->h_ctl->stop = 0;
    h->h_ctl->stop_reason = 0;
    h->write_ctl_fields();
    std::vector<cudaEvent_t> ev(3 * n);
    for (auto& e : ev) ck(cudaEventCreate(&e), "event");
    for (int i = 0; i < n; ++i) {
      ck(cudaEventRecord(ev[3 * i], h->stream), "event");
      ck(fip::launch_rmg_step(h->st, h->grid_ctas, h->stream), "rmg_step");
      ck(cudaEventRecord(ev[3 * i + 1], h->stream), "event");
      h->launch_post(FIP_POST_MODE_STEP);
      ck(cudaEventRecord(ev[3 * i + 2], h->stream), "event");
    }
    h->read_ctl();
    double s = 0, p = 0;
    for (int i = 0; i < n; ++i) {
      float a = 0, b = 0;
      ck(cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]), "event");
      ck(cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]), "event");
      s += a;
      p += b;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (stencil_ms) *stencil_ms = (float)(s / n);
    if (post_ms) *post_ms = (float)(p / n);
    h->h_ctl->next_save = save_keep;
    h->h_ctl->next_sample = h->cfg.sampling_interval > 0 ? h->sample_timer : kInf;
    h->h_ctl->stop = 0;
    h->h_ctl->stop_reason = 0;
    h->write_ctl_fields();
    ck(cudaStreamSynchronize(h->stream), "profile");
    return FIP_OK;
  });
}

int fip_step_timed(fip_handle* h, int n, float* total_ms, float* stencil_ms, float* post_ms) {
  if (!h || n <= 0) return fail(FIP_ERR_ARG, "bad argument");
  return guard([&] {
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    if (!h->started) {
      int rc = h->run_steps(1, false);
      if (rc) return rc;
    }
    if (h->replan) {
      ck(fip::launch_init_tiles(h->st, h->h_ctl->parity, h->stream), "init_tiles");
      h->launch_post(FIP_POST_MODE_PLAN);
      h->replan = false;
    }
    const double keep_sample = h->h_ctl->next_sample, keep_save = h->h_ctl->next_save;
    h->h_ctl->next_sample = kInf;
    h->h_ctl->next_save = kInf;
    h->h_ctl->target = kInf;
    const bool per_launch = stencil_ms || post_ms;
    h->h_ctl->steps_left = per_launch ? 2 * n : n;
    h->h_ctl->stop = 0;
    h->h_ctl->stop_reason = 0;
    h->write_ctl_fields();
    // One graph of n steps; with `events`, event record nodes (cudaEventRecordExternal) timestamp
    // every launch, which also keeps each launch from overlapping the one before it.
    auto timed = [&](bool events, std::vector<cudaEvent_t>& ev) {
      ev.resize(events ? 2 * n + 1 : 2);
      for (auto& e : ev) ck(cudaEventCreate(&e), "event");
      cudaGraph_t g;
      ck(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "capture");
      ck(cudaEventRecordWithFlags(ev[0], h->stream, cudaEventRecordExternal), "event");
      for (int i = 0; i < n; ++i) {
        ck(fip::launch_rmg_step(h->st, h->grid_ctas, h->stream), "rmg_step");
        if (events) ck(cudaEventRecordWithFlags(ev[2 * i + 1], h->stream, cudaEventRecordExternal), "event");
        h->launch_post(FIP_POST_MODE_STEP);
        if (events) ck(cudaEventRecordWithFlags(ev[2 * i + 2], h->stream, cudaEventRecordExternal), "event");
      }
      if (!events) ck(cudaEventRecordWithFlags(ev[1], h->stream, cudaEventRecordExternal), "event");
      ck(cudaStreamEndCapture(h->stream, &g), "capture");
      cudaGraphExec_t ex;
      ck(cudaGraphInstantiate(&ex, g, 0), "cudaGraphInstantiate");
      cudaGraphDestroy(g);
      ck(cudaGraphUpload(ex, h->stream), "cudaGraphUpload");
      ck(cudaStreamSynchronize(h->stream), "sync");
      ck(cudaGraphLaunch(ex, h->stream), "cudaGraphLaunch");
      ck(cudaStreamSynchronize(h->stream), "sync");
      cudaGraphExecDestroy(ex);
    };
    std::vector<cudaEvent_t> ev_total, ev_each;
    double tot = 0, s = 0, p = 0;
    float x = 0;
    timed(false, ev_total);  // the steps as the step loop runs them
    ck(cudaEventElapsedTime(&x, ev_total[0], ev_total[1]), "event");
    tot = x;
    if (per_launch) {
      timed(true, ev_each);
      for (int i = 0; i < n; ++i) {
        ck(cudaEventElapsedTime(&x, ev_each[2 * i], ev_each[2 * i + 1]), "event");
        s += x;
        ck(cudaEventElapsedTime(&x, ev_each[2 * i + 1], ev_each[2 * i + 2]), "event");
        p += x;
      }
    }
    h->read_ctl();
    for (auto& e : ev_total) cudaEventDestroy(e);
    for (auto& e : ev_each) cudaEventDestroy(e);
    if (total_ms) *total_ms = (float)tot;
    if (stencil_ms) *stencil_ms = (float)(s / n);
    if (post_ms) *post_ms = (float)(p / n);
    const int err = h->h_ctl->error;
    h->h_ctl->next_sample = keep_sample;
    h->h_ctl->next_save = keep_save;
    h->h_ctl->stop = 0;
    h->h_ctl->stop_reason = 0;
    h->write_ctl_fields();
    ck(cudaStreamSynchronize(h->stream), "sync");
    if (err) return fail(FIP_ERR_DEVICE_TIMEOUT, "device wait ran out (code " + std::to_string(err) + ")");
    return FIP_OK;
  });
}

void fip_destroy(fip_handle* h) { delete h; }

const char* fip_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"

// ---- host-only entry points ---------------------------------------------------------------
namespace {

std::string json_str(const std::string& s) {
  std::string r = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') r += '\\';
    if (c == '\n') {
      r += "\\n";
      continue;
    }
    r += c;
  }
  return r + "\"";
}

std::string json_num(double v) {
  if (std::isnan(v)) return "\"nan\"";
  if (std::isinf(v)) return v > 0 ? "\"inf\"" : "\"-inf\"";
  char b[64];
  std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}

int copy_out(const std::string& s, char* buf, int buflen) {
  if (buf && buflen > 0) {
    const int n = (int)std::min<size_t>(s.size(), (size_t)buflen - 1);
    std::memcpy(buf, s.data(), n);
    buf[n] = '\0';
  }
  return (int)s.size();
}

int load_for_host(const char* path, fip::Config* c, bool quiet) {
  if (!path) return fail(FIP_ERR_ARG, "null path");
  std::string err;
  const int rc = fip::load_config(path, c, &err, quiet);
  if (rc == 2) return fail(FIP_ERR_IO, err);
  if (rc) return fail(FIP_ERR_CONFIG, err);
  return FIP_OK;
}

}  // namespace

extern "C" {

int fip_validate(const char* yaml_path) {
  fip::Config c;
  return load_for_host(yaml_path, &c, false);  // validation prints the reference's warnings
}

int fip_config_json(const char* yaml_path, char* buf, int buflen) {
  fip::Config c;
  int rc = load_for_host(yaml_path, &c, true);
  if (rc) return rc;
  static const char* sides[] = {"left", "right", "top", "bottom"};
  static const char* types[] = {"z", "q", "close", "open"};
  static const char* stypes[] = {"z", "h", "qx", "qy"};
  std::ostringstream o;
  o << "{\"name\":" << json_str(c.name) << ",\"W\":" << c.W << ",\"H\":" << c.H << ",\"dx\":" << json_num(c.dx)
    << ",\"dt\":" << json_num(c.dt) << ",\"variable_dt\":" << (c.variable_dt ? "true" : "false")
    << ",\"solver\":" << (c.solver == fip::Solver::rmg ? "\"rmg\"" : "\"cn\"")
    << ",\"target_duration\":" << json_num(c.target_duration) << ",\"kSt\":" << json_num(c.kst_fixed)
    << ",\"no_data\":" << json_num(c.no_data) << ",\"kst_var\":" << (c.has_kst_var ? "true" : "false");
  double hsum = 0;
  for (float v : c.h0) hsum += v;
  o << ",\"h0_sum\":" << json_num(hsum) << ",\"boundary_conditions\":[";
  for (size_t i = 0; i < c.bcs.size(); ++i) {
    const auto& b = c.bcs[i];
    o << (i ? "," : "") << "{\"side\":\"" << sides[(int)b.side] << "\",\"type\":\"" << types[(int)b.type]
      << "\",\"from\":" << b.from << ",\"to\":" << b.to << ",\"series\":" << (b.is_series ? "true" : "false")
      << ",\"z\":" << json_num(b.z) << ",\"q\":" << json_num(b.q);
    if (!b.is_series) o << ",\"qval\":" << json_num(c.const_q(b));
    auto ts = [&](const char* k, const fip::TimeSeries& t, bool has) {
      if (!has) return;
      o << ",\"" << k << "_t\":[";
      for (size_t j = 0; j < t.t.size(); ++j) o << (j ? "," : "") << json_num(t.t[j]);
      o << "],\"" << k << "_v\":[";
      for (size_t j = 0; j < t.v.size(); ++j) o << (j ? "," : "") << json_num(t.v[j]);
      o << "]";
    };
    ts("z", b.z_series, b.has_z_series);
    ts("q", b.q_series, b.has_q_series);
    o << "}";
  }
  o << "],\"sampling_interval\":" << c.sampling_interval << ",\"sampling\":[";
  for (size_t i = 0; i < c.points.size(); ++i)
    o << (i ? "," : "") << "{\"x\":" << c.points[i].x << ",\"y\":" << c.points[i].y
      << ",\"label\":" << json_str(c.points[i].label) << ",\"type\":\"" << stypes[(int)c.points[i].type] << "\"}";
  o << "],\"save_state\":[";
  for (size_t i = 0; i < c.save_times.size(); ++i) o << (i ? "," : "") << json_num(c.save_times[i]);
  o << "]}";
  return copy_out(o.str(), buf, buflen);
}

int fip_bc_program(const char* yaml_path, int pitch, int compile, char* buf, int buflen) {
  fip::Config c;
  int rc = load_for_host(yaml_path, &c, true);
  if (rc) return rc;
  if (pitch < (int)c.W) return fail(FIP_ERR_ARG, "pitch smaller than W");
  fip::SeriesLayout ser = fip::layout_series(c);
  std::string src = fip::post_kernel_source(c, ser, pitch);
  if (compile) {
    std::string cubin, log, err;
    if (fip::compile_post_kernel(src, &cubin, &log, &err)) return fail(FIP_ERR_NVRTC, err);
  }
  return copy_out(src, buf, buflen);
}

}  // extern "C"
