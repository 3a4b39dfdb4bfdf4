// chns_internal.h -- context of the C ABI and the per-size launch tables.
#pragma once

#include <cuda_runtime.h>

#include "../../include/chns.h"

struct chns_ctx;
struct chns_adj;
// an ensemble's step as one persistent cooperative kernel (chns_persist.cu):
// CHNS_ERR_UNSUPPORTED when the members are not all ternary FP32 at 256..1024
struct chns_persist;
int chns_persist_create(chns_ctx* const* members, int count, chns_persist** out);
void chns_persist_destroy(chns_persist* p);
int chns_persist_step(chns_persist* p, cudaStream_t st);
int chns_persist_check(chns_persist* p, cudaStream_t st);
int chns_persist_grid(const chns_persist* p);
void chns_adj_free(chns_ctx* c);
// shared by chns_set_phase_real and the initial conditions (chns_init.cu)
extern "C" int chns_realdbl_to_realbuf(chns_ctx* c);
extern "C" int chns_phase_from_realdbl(chns_ctx* c, int f);
// real-space field f of the state (truncated first if asked) into c->realdbl
extern "C" int chns_field_to_realdbl(chns_ctx* c, int f, int truncate);
// CHNS_FP32_STATE64: the low part of field f after anything but a step or
// chns_set_state has written its float part (zero, and at k = 0 the rest of the
// double k = 0 mode)
extern "C" int chns_statelo_reset(chns_ctx* c, int f);
// the value chns_tune_override set for a knob (-1: the tuned table)
extern "C" int chns_tune_value(int knob);

namespace chns {
// intermediate buffers of a step: G slots (rows 0..jt) and H slots (rows
// 0..n/2), each of width 2n complex (see chns_kernels.cuh)
constexpr int kNumG = 6, kNumH = 4;

// Launchers instantiated per grid size and precision (chns_inst_*.cu).
struct Launchers {
  // one ETD2RK stage (1 or 2) of the context's model; returns launches enqueued
  int (*stage)(chns_ctx* c, int stage);
  // S-layout field -> truncated in place (the sharp cut, or the smooth filter's two products)
  int (*truncate)(chns_ctx* c, void* s);
  // device real (R, nx*ny) -> S-layout spectrum (unnormalised r2c)
  int (*dfft)(chns_ctx* c, const void* real, void* s);
  // S-layout spectrum -> device real (R), c2r * 1/(nx ny)
  int (*ifft)(chns_ctx* c, const void* s, void* real);
  // FFTW-layout double <-> S layout
  int (*from_fftw)(chns_ctx* c, const double* src, void* s);
  int (*to_fftw)(chns_ctx* c, const void* s, double* dst);
  // free energy and kinetic energy reductions (double results in c->red)
  int (*diag)(chns_ctx* c);
  // nb transforms at once: field b at real + b rs (R elements) and s + b ss
  // (complex elements); scratch holds nb n x (n/2+1) complex fields
  int (*dfftb)(chns_ctx* c, const void* real, size_t rs, void* s, size_t ss, int nb, void* scratch);
  int (*ifftb)(chns_ctx* c, const void* s, size_t ss, void* real, size_t rs, int nb, void* scratch);
  // binary adjoint: product adjoints b0 .. b0 + nb - 1 (chns_adj_rows.cuh) formed from the
  // device record table rf (RecFields) and the physical adjoints in[0..4] (Ab, Bb, Fxb,
  // Fyb, fb) and transformed forward into s + b ss (S layout)
  int (*adjprod)(chns_ctx* c, const void* rf, const void* const* in, int b0, int nb, void* s, size_t ss,
                 void* scratch);
  // the largest dynamic shared memory a step kernel of the context needs (bytes)
  size_t (*step_smem)(const chns_ctx* c);
};

const Launchers* launchers_f64(int logn);
const Launchers* launchers_f32(int logn);

}  // namespace chns

struct chns_ctx {
  chns_params p;
  int n, nr, jt;
  bool p1_split;  // P1 with two CTAs per row (chns_tuned.h or chns_tune_override)
  bool p4_grad;   // grad c_i from P2 in real space for P4 (chns_tuned.h or chns_tune_override)
  bool pdl;       // stage kernels as programmatic dependent launches (chns_tuned.h or chns_tune_override)
  bool f32;
  bool st64;   // FP32 context with a double-float state (CHNS_FP32_STATE64)
  size_t rsz;  // bytes per real scalar (4 or 8)
  cudaStream_t stream;
  bool own_stream;
  // device memory
  void* state[3];
  void* statelo[3]; // CHNS_FP32_STATE64: the low float of the state (S layout): state = state[] + statelo[]
  void* saved[3];
  void* nstar[3];   // when set, stage 2 also stores N(u*) there (adjoint recording)
  void* rec;        // when set (binary), the stage also records the forward fields its
                    // adjoint transposes there (chns_kernels.cuh, Bufs::rec)
  void* nw;
  void* g[12];
  void* h[7];
  void* gradr;      // p4_grad: real-space grad c_i of a stage (P2 -> P4), model x n x n complex of the context precision
  void* coef;
  void* tmag;         // chns::TmaG (host): tensor maps of the G slots for the row kernels' TMA tiles
  unsigned int* tma_err;  // device word the row kernels flag a timed-out tile wait in
  int* mrow;
  void* filt;       // SMOOTH filter factors [nx/2+1 rows][nx/2+1 |m|] in the context precision (else null)
  double* filtd;    // the same in double (FP64 contexts: filt itself)
  void* tw;
  double* k0;       // [12] k = 0 modes (FP32 contexts)
  double* stage;    // FFTW-layout double staging, n * nr complex
  void* realbuf;    // n * n reals of the context precision
  double* realdbl;  // n * n doubles
  double* red;      // reduction results
  void* redscratch;
  // host-side parameters
  double k0coef[6];
  double fx, fy;
  double gamma[3], del;
  int force_j;
  double force_hat;
  // launch bookkeeping
  const chns::Launchers* L;
  int launches_per_step;
  cudaGraphExec_t step_graph;
  bool graph_ok;
  void* hostpin;    // pinned staging for host transfers
  size_t hostpin_bytes;
  void* pinned[8];  // host arrays registered by chns_pin_host
  int npinned;
  // discrete-adjoint buffers (allocated by the first chns_adjoint call)
  chns_adj* adj;
  // tracing: when prof_ev is set, every launch of a stage records an event
  cudaEvent_t* prof_ev;
  int* prof_kind;
  int prof_n, prof_max;
};

namespace chns {
// kernel kinds reported by chns_profile_step
enum { KIND_SPEC_INV = 0, KIND_ROW_ADV = 1, KIND_SPEC_FWD_C = 2, KIND_ROW_FORCE = 3, KIND_SPEC_CURL_W = 4,
       KIND_ROW_ADV_B = 5 };
inline void mark(chns_ctx* c, int kind) {
  if (c->prof_ev && c->prof_n < c->prof_max) {
    cudaEventRecord(c->prof_ev[c->prof_n], c->stream);
    c->prof_kind[c->prof_n] = kind;
    c->prof_n++;
  }
}
}  // namespace chns
