/*
 * CPU oracle for fip's slim shallow-water time step (the `rmg` solver).
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product links, calls or ships this code: it is the
 * checker used by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline / reference
 * arm. Parity of this restatement is pinned against the reference binary itself (oracle/ref.mk
 * builds it into oracle/_ref/) through the golden fixtures in tests/golden/.
 *
 * Two builds of the same source: ora64_* keeps every field value in double (the "FP64 scalar
 * host loop" of the scheme); ora32_* keeps them in float with IEEE operations (no fast-math
 * approximations, so it differs from the GPU by the rounding of sqrt/pow/div only). In both,
 * the time-step controller keeps dt in float and the simulated time in double, exactly as the
 * reference host does (src/simdata.h:338, :342).
 *
 * Reference files followed (paths relative to the fip project root):
 *   src/kernels.cu:30-127   flux and momentum helpers (fp32div_wrapper, compute_rmg_*)
 *   src/kernels.cu:264-438  rmg_kernel: row march, boundary-face holds (:373-376), the cell sets
 *                           it writes (:383-406) and the CFL fold (:392-400); mask off
 *   src/kernels.cu:254-262  flood_plains_kernel (hmax), cadence src/main.cpp:125-128
 *   src/bc_kernel_gen.cpp:11-137  staggered boundary fragments (z, q, close, open)
 *   src/boundary_condition.cpp:6-77  zval/qval per step, sumWaterDepths
 *   src/timeseries.cpp:14-26  clamped linear interpolation
 *   src/main.cpp:25-43, :100-135  controlTimestep and the simulate() ordering
 */
#ifndef FIP_RMG_ORACLE_H
#define FIP_RMG_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { ORA_SIDE_LEFT = 0, ORA_SIDE_RIGHT = 1, ORA_SIDE_TOP = 2, ORA_SIDE_BOTTOM = 3 };
enum { ORA_BC_Z = 0, ORA_BC_Q = 1, ORA_BC_CLOSE = 2, ORA_BC_OPEN = 3 };
enum { ORA_F_H = 0, ORA_F_QX = 1, ORA_F_QY = 2,            /* current state (d_h1 ...)      */
       ORA_F_H_OTHER = 3, ORA_F_QX_OTHER = 4, ORA_F_QY_OTHER = 5, /* other ping-pong buffer   */
       ORA_F_HMAX = 6 };

typedef struct ora_sim ora_sim;

#define ORA_DECLARE(P)                                                                          \
  ora_sim* P##new_sim(int W, int H, long pitch_elems, float dx, float dt, int variable_dt,     \
                      float kst_fixed, float no_value, const float* terrain, const float* h0,   \
                      const float* qx0, const float* qy0, const float* kst_var);                \
  int P##add_bc(ora_sim* s, int side, int type, int from, int to, int is_series, float z,      \
                float q, int nz, const float* zt, const float* zv, int nq, const float* qt,    \
                const float* qv);                                                               \
  void P##set_sampling(ora_sim* s, int interval, int npts, const int* xs, const int* ys,       \
                       const int* types);                                                       \
  void P##set_save_times(ora_sim* s, int n, const double* times);                              \
  void P##set_threads(ora_sim* s, int n);                                                       \
  int P##simulate(ora_sim* s, int n);                                                           \
  int P##run_to(ora_sim* s, double target_duration);                                           \
  double P##duration(const ora_sim* s);                                                         \
  float P##dt(const ora_sim* s);                                                                \
  int P##iteration(const ora_sim* s);                                                           \
  float P##last_cfl(const ora_sim* s);                                                          \
  double P##volume(const ora_sim* s);                                                           \
  void P##get_field(const ora_sim* s, int which, float* out);                                  \
  const char* P##sample_text(const ora_sim* s);                                                 \
  int P##dump_count(const ora_sim* s);                                                          \
  double P##dump_duration(const ora_sim* s, int k);                                            \
  void P##dump_field(const ora_sim* s, int k, int which, float* out);                          \
  void P##free_sim(ora_sim* s);

ORA_DECLARE(ora64_)
ORA_DECLARE(ora32_)

#ifdef __cplusplus
}
#endif
#endif
