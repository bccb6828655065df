// The whole-step interface of one precision build of the engine
// (alfa_step.cu, compiled as alfa::f64 and as alfa::f32).  The C-ABI unit
// (alfa_capi.cu) holds a context of either build behind one alfa_ctx and
// reaches it only through these functions; their arguments are host types
// and FP64 device buffers, whatever the engine's storage precision.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "alfa.h"

#define ALFA_IFACE_DECLS                                                                      \
  struct Ctx;                                                                                 \
  struct Ens;                                                                                 \
  int ctx_create(const alfa_config& cfg, Ctx** out, std::string* err);                        \
  void ctx_destroy(Ctx* c);                                                                   \
  const char* ctx_error(const Ctx* c);                                                        \
  int ctx_fail(Ctx* c, const std::string& m, int code);                                       \
  void ctx_set_stream(Ctx* c, cudaStream_t s);                                                \
  size_t ctx_bytes(const Ctx* c);                                                             \
  void ctx_derived(const Ctx* c, alfa_derived* o);                                            \
  int init_state(Ctx* c, const double* u, const double* v, const double* w, const double* TH); \
  int set_series(Ctx* c, const double* Uadv, const double* Vadv, const double* THadv,          \
                 const double* sfc, int nrows);                                               \
  int set_geowind_series(Ctx* c, const double* Ug, const double* Vg, int nrows);              \
  int init_moisture(Ctx* c, const double* Q);                                                 \
  int set_moisture_series(Ctx* c, const double* Qadv, const double* msfc, int nrows);         \
  int get_moisture(Ctx* c, double* Q);                                                        \
  int step(Ctx* c, int nsteps, int sgs_mode);                                                 \
  int step_graph(Ctx* c, int nsteps);                                                         \
  int get_state(Ctx* c, double* u, double* v, double* w, double* TH, double* p);              \
  int get_diag(Ctx* c, alfa_diag* o);                                                         \
  int stats_sample(Ctx* c, double* acc);                                                      \
  size_t checkpoint_doubles(const Ctx* c);                                                    \
  int save_checkpoint(Ctx* c, double* dst);                                                   \
  int load_checkpoint(Ctx* c, const double* src);                                             \
  int time_kernel(Ctx* c, int which, int reps, double* ms, double* bytes);                    \
  int autotune(Ctx* c, int reps, alfa_tune_entry* out, int max_out, int* n_out);              \
  int set_line_variant(Ctx* c, int axis, int n_in, int n_out, int map, int nout, int variant); \
  int tc_line_apply(Ctx* c, int map, int cut, int n_in, int n_out, double scale,              \
                    long long ncols, const float* X, float* Y);                               \
  void ctx_set_tc_spin(Ctx* c, unsigned long long polls);                                     \
  int ens_create(Ctx* const* members, int n, Ens** out);                                      \
  int ens_step(Ens* E, int nsteps);                                                           \
  int ens_sync(Ens* E);                                                                       \
  int ens_set_stream(Ens* E, cudaStream_t s);                                                 \
  const char* ens_error(const Ens* E);                                                        \
  void ens_destroy(Ens* E);

namespace alfa {
namespace f64 {
ALFA_IFACE_DECLS
}  // namespace f64
namespace f32 {
ALFA_IFACE_DECLS
}  // namespace f32
}  // namespace alfa
