// chns_adjoint.cu -- discrete adjoint of n binary ETD2RK steps (chns_adjoint).
//
// Gradient of a final-time functional J(c_T) with respect to the initial spectral
// state (omega_hat_0, c_hat_0) and to nu, lambda (the mobility M) and sigma.
// Reverse sweep with two-level checkpointing: the forward pass keeps the state
// every `ckpt` steps; each segment is recomputed forward from its checkpoint
// (the last one is recorded during the forward pass), keeping per step u_n, the
// stage-1 state u*, N(u_n) and N(u*) (the stage-2 kernels store N(u*) when the
// context's nstar pointers are set).  Reversing a step applies the transposed
// stage-2 update, the transposed right-hand side at u*, the transposed stage-1
// update and the transposed right-hand side at u_n (kernels in
// chns_adjoint.cuh), captured once as a CUDA graph on fixed buffers.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <vector>

#include "chns_adjoint.cuh"
#include "chns_internal.h"

namespace {

using namespace chns;

#define ACK(call)                                 \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return CHNS_ERR_CUDA;  \
  } while (0)

// phi-function derivatives in z = c h: (e^z)' = e^z; phi1 = (e^z-1)/z, phi2 = (e^z-1-z)/z^2
double dphi1(double z) {
  if (fabs(z) < 0.5) {  // sum_{n>=1} n z^{n-1} / (n+1)!
    double s = 0.0, fact = 2.0, zp = 1.0;
    for (int n = 1; n < 24; n++) {
      s += n * zp / fact;
      zp *= z;
      fact *= (n + 2);
    }
    return s;
  }
  return (exp(z) * (z - 1.0) + 1.0) / (z * z);
}
double dphi2(double z) {
  if (fabs(z) < 0.5) {  // sum_{n>=1} n z^{n-1} / (n+2)!
    double s = 0.0, fact = 6.0, zp = 1.0;
    for (int n = 1; n < 24; n++) {
      s += n * zp / fact;
      zp *= z;
      fact *= (n + 3);
    }
    return s;
  }
  return (z * exp(z) - 2.0 * exp(z) + 2.0 + z) / (z * z * z);
}

// d(e, z1, z2)/dc at linear coefficient c: e = e^{ch}, z1 = h phi1(ch), z2 = h phi2(ch)
void dcoef_dc(double c, double h, double* o) {
  const double z = c * h;
  o[0] = h * exp(z);
  o[1] = h * h * dphi1(z);
  o[2] = h * h * dphi2(z);
}

}  // namespace

// Device buffers of the adjoint, kept in the context between calls.
//   spec: NSPEC S-layout fields in one allocation (slot k at k ncx complex)
//   phys: NPHYS real n x n fields in one allocation
//   bscr: scratch of the batched transforms (7 fields)
//   seg:  per step of a segment, 8 fields: u_n, u*, N(u_n), N(u*); two
//         segments' worth when memory allows, so that the recompute of one
//         segment (side stream) overlaps the reversal of the next
struct chns_adj {
  int cap_states;   // slots allocated (ckpt or 2 ckpt)
  int seg_len;      // ckpt the slots were laid out for
  void* seg;
  cudaStream_t side;  // segment recompute
  cudaStream_t fork;  // parallel branch of the captured reverse step
  cudaEvent_t ev_sweep, ev_ready[2], ev_free[2], ev_fork, ev_join;
  void** ckpt;
  double** ckptk0;
  int nckpt_cap;
  void* dcoef;        // [9][nr][nr] double
  double* acc;        // [8]: J, -, dJ/dsigma (loss part), -, nu, lambda, sigma (step part)
  void* spec;
  void* phys;
  void* bscr;
  cudaGraphExec_t rev;  // one reverse step (fixed buffers), or null
  bool rev_tried;
  size_t ncx, nn;
};

namespace {

// Two field sets (0: the state u*, 1: the state u_n of a reversed step), each
// with its own spectral batch, scratch and F[f(c_t)] and its own physical
// forward fields, so that the forward fields at u_n are computed on a branch
// parallel to the transposed right-hand side at u*.
constexpr int SSET = 9;                      // spectral fields per set
enum { SB = 0, SXo = 7, SFFo = 8 };           // batch of 7, scratch, F[f]
enum {
  SY = 2 * SSET,                             // scratch (f_bar spectrum)
  SNBW, SNBC,                                // N*_bar
  SNBAW, SNBAC,                              // N(u_n)_bar
  SGW, SGC,                                  // running gradient (w_bar, c_bar)
  // current step, in the segment slot layout: u_n, u*, N(u_n), N(u*)
  CUW, CUC, CSW, CSC, CNW, CNC, CXW, CXC,
  NSPEC
};
constexpr int PSET = 9;                                    // physical fields per set
enum { PU = 0, PV, PWX, PWY, PCT, PCX, PCY, PMU, PFT };     // forward fields, f(c_t)
enum { PFB = 2 * PSET, PAB, PBB, PFXB, PFYB, PUB, PVB, PWXB, PWYB, PCTB, PCXB, PCYB, NPHYS };
constexpr int SLOT_FIELDS = 8;
constexpr int kLossBlocks = 1024;  // blocks of the loss reduction

template <class R> struct Adj {
  chns_ctx* c;
  chns_adj* a;
  AdjPar<R> P;
  cudaStream_t st;
  size_t ncx, nn;
  int blocks_s, blocks_p;

  cx<R>* S(int k) const { return (cx<R>*)a->spec + (size_t)k * ncx; }
  R* F(int k) const { return (R*)a->phys + (size_t)k * nn; }
  cx<R>* SS(int set, int k) const { return S(set * SSET + k); }
  R* FS(int set, int k) const { return F(set * PSET + k); }
  void* scratch(int set) const { return (char*)a->bscr + (size_t)set * FOP_N * ncx * sizeof(cx<R>); }

  // batched transforms on stream s with the scratch of a field set
  void ifft(cudaStream_t s, int set, const cx<R>* in, R* x, int nb) {
    c->stream = s;
    c->L->ifftb(c, in, ncx, x, nn, nb, scratch(set));
    c->stream = st;
  }
  void dfft(cudaStream_t s, int set, const R* x, cx<R>* out, int nb) {
    c->stream = s;
    c->L->dfftb(c, x, nn, out, ncx, nb, scratch(set));
    c->stream = st;
  }

  // forward fields of the right-hand side at (w, cc) into field set `set`
  void fields(cudaStream_t s, int set, const cx<R>* w, const cx<R>* cc) {
    k_adj_fwd_prep7<R><<<blocks_s, 256, 0, s>>>(P, w, cc, SS(set, SB), ncx);
    ifft(s, set, SS(set, SB), FS(set, PU), FOP_N);
    k_adj_bulk<R><<<blocks_p, 256, 0, s>>>(FS(set, PCT), FS(set, PFT), nn);
    dfft(s, set, FS(set, PFT), SS(set, SFFo), 1);
    k_adj_mu_prep<R><<<blocks_s, 256, 0, s>>>(P, cc, SS(set, SFFo), SS(set, SXo));
    ifft(s, set, SS(set, SXo), FS(set, PMU), 1);
  }

  // (gw, gc) += J_N(state)^T (nbw, nbc) with the forward fields of set `set`
  // (c_hat of the state: cc); parameter partials into acc[4..6].  Scratch of set 0.
  void transpose_rhs(int set, const cx<R>* cc, const cx<R>* nbw, const cx<R>* nbc, cx<R>* gw, cx<R>* gc) {
    double* pacc = a->acc + 4;
    // transposed spectral tail -> A_bar, B_bar, Fx_bar, Fy_bar
    k_adj_tail4<R><<<blocks_s, 256, 0, st>>>(P, nbw, nbc, SS(0, SB), ncx);
    ifft(st, 0, SS(0, SB), F(PAB), 4);
    // mu_bar -> c_bar (s1 k^2), f_bar, lambda and sigma partials
    k_adj_mubar<R><<<blocks_p, 256, 0, st>>>(F(PFXB), F(PFYB), FS(set, PCX), FS(set, PCY), F(PUB), nn);
    dfft(st, 0, F(PUB), SS(0, SXo), 1);
    k_adj_mu<R><<<blocks_s, 256, 0, st>>>(P, SS(0, SXo), cc, SS(set, SFFo), nbc, gc, S(SY), pacc);
    ifft(st, 0, S(SY), F(PFB), 1);
    // products, then C^T of the seven forward fields
    PhysFields<R> pf{FS(set, PU), FS(set, PV), FS(set, PWX), FS(set, PWY), FS(set, PCT), FS(set, PCX),
                     FS(set, PCY), FS(set, PMU)};
    PhysAdj<R> pa{F(PAB), F(PBB), F(PFXB), F(PFYB), F(PFB), F(PUB), F(PVB), F(PWXB), F(PWYB), F(PCTB), F(PCXB),
                  F(PCYB)};
    k_adj_products<R><<<blocks_p, 256, 0, st>>>(pf, pa, nn);
    dfft(st, 0, F(PUB), SS(0, SB), FOP_N);
    k_adj_acc7<R><<<blocks_s, 256, 0, st>>>(P, SS(0, SB), gw, gc, ncx);
  }

  // one reversed step from the current-step slots (CUW..CXC): the transposed
  // stage 2, right-hand side at u*, stage 1 and right-hand side at u_n.  With a
  // fork stream the forward fields at u_n are built on a parallel branch.
  void reverse_step(const R* coef, const double* dcoef, cudaStream_t fork) {
    double* pacc = a->acc + 4;
    cx<R>* gw = S(SGW);
    cx<R>* gc = S(SGC);
    if (fork) {
      cudaEventRecord(a->ev_fork, st);
      cudaStreamWaitEvent(fork, a->ev_fork, 0);
      fields(fork, 1, S(CUW), S(CUC));
      cudaEventRecord(a->ev_join, fork);
    }
    k_adj_etd2<R><<<blocks_s, 256, 0, st>>>(P, coef, dcoef, gw, gc, S(CXW), S(CXC), S(CNW), S(CNC), S(SNBW),
                                            S(SNBC), S(SNBAW), S(SNBAC), pacc);
    fields(st, 0, S(CSW), S(CSC));
    transpose_rhs(0, S(CSC), S(SNBW), S(SNBC), gw, gc);
    k_adj_etd1<R><<<blocks_s, 256, 0, st>>>(P, coef, dcoef, gw, gc, S(CUW), S(CUC), S(CNW), S(CNC), S(SNBAW),
                                            S(SNBAC), pacc);
    if (fork) {
      cudaStreamWaitEvent(st, a->ev_join, 0);
    } else {
      fields(st, 1, S(CUW), S(CUC));
    }
    transpose_rhs(1, S(CUC), S(SNBAW), S(SNBAC), gw, gc);
  }
};

// one forward step that also records u_n, u*, N(u_n) and N(u*) into a segment slot
int record_step(chns_ctx* c, char* slot, size_t fbytes) {
  cudaStream_t st = c->stream;
  ACK(cudaMemcpyAsync(slot, c->state[0], fbytes, cudaMemcpyDeviceToDevice, st));
  ACK(cudaMemcpyAsync(slot + fbytes, c->state[1], fbytes, cudaMemcpyDeviceToDevice, st));
  c->L->stage(c, 1);
  ACK(cudaMemcpyAsync(slot + 2 * fbytes, c->state[0], fbytes, cudaMemcpyDeviceToDevice, st));
  ACK(cudaMemcpyAsync(slot + 3 * fbytes, c->state[1], fbytes, cudaMemcpyDeviceToDevice, st));
  ACK(cudaMemcpyAsync(slot + 4 * fbytes, c->saved[0], fbytes, cudaMemcpyDeviceToDevice, st));
  ACK(cudaMemcpyAsync(slot + 5 * fbytes, c->saved[1], fbytes, cudaMemcpyDeviceToDevice, st));
  c->nstar[0] = slot + 6 * fbytes;
  c->nstar[1] = slot + 7 * fbytes;
  c->L->stage(c, 2);
  c->nstar[0] = nullptr;
  c->nstar[1] = nullptr;
  return CHNS_OK;
}

int snapshot_save(chns_ctx* c, void* dst, double* dstk0) {
  const size_t bytes = (size_t)c->n * c->nr * 2 * c->rsz;
  ACK(cudaMemcpyAsync(dst, c->state[0], bytes, cudaMemcpyDeviceToDevice, c->stream));
  ACK(cudaMemcpyAsync((char*)dst + bytes, c->state[1], bytes, cudaMemcpyDeviceToDevice, c->stream));
  ACK(cudaMemcpyAsync(dstk0, c->k0, 16 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return CHNS_OK;
}
int snapshot_load(chns_ctx* c, const void* src, const double* srck0) {
  const size_t bytes = (size_t)c->n * c->nr * 2 * c->rsz;
  ACK(cudaMemcpyAsync(c->state[0], src, bytes, cudaMemcpyDeviceToDevice, c->stream));
  ACK(cudaMemcpyAsync(c->state[1], (const char*)src + bytes, bytes, cudaMemcpyDeviceToDevice, c->stream));
  ACK(cudaMemcpyAsync(c->k0, srck0, 16 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return CHNS_OK;
}

int adj_alloc(chns_ctx* c, int seglen, int nckpt) {
  if (!c->adj) {
    c->adj = (chns_adj*)calloc(1, sizeof(chns_adj));
    if (!c->adj) return CHNS_ERR_NOMEM;
  }
  chns_adj* a = c->adj;
  const size_t ncx = (size_t)c->n * c->nr, nn = (size_t)c->n * c->n;
  const size_t fbytes = ncx * 2 * c->rsz;  // one S-layout field
  const size_t snap = 2 * fbytes;
  a->ncx = ncx;
  a->nn = nn;
  if (!a->dcoef) {
    if (cudaMalloc(&a->spec, NSPEC * fbytes) != cudaSuccess) return CHNS_ERR_NOMEM;
    if (cudaMalloc(&a->phys, NPHYS * nn * c->rsz) != cudaSuccess) return CHNS_ERR_NOMEM;
    if (cudaMalloc(&a->bscr, 2 * FOP_N * fbytes) != cudaSuccess) return CHNS_ERR_NOMEM;
    // 8 accumulators, then 3 per-block partials of each loss block
    if (cudaMalloc((void**)&a->acc, (8 + 3 * kLossBlocks) * sizeof(double)) != cudaSuccess) return CHNS_ERR_NOMEM;
    // derivative tables of the ETD coefficients: d/dnu (w), d/dlambda, d/dsigma (c)
    const int nr = c->nr;
    const chns_params& p = c->p;
    std::vector<double> d(9 * (size_t)nr * nr);
    const size_t t = (size_t)nr * nr;
    for (int j = 0; j < nr; j++)
      for (int m = 0; m < nr; m++) {
        const double kx = c->fx * m, ky = c->fy * j, ks = kx * kx + ky * ky, k4 = ks * ks;
        double o[3];
        dcoef_dc(-p.nu * ks, p.dt, o);
        for (int q = 0; q < 3; q++) d[q * t + (size_t)j * nr + m] = -ks * o[q];
        dcoef_dc(-1.5 * p.lambda * p.sigma * p.epsilon * k4, p.dt, o);
        for (int q = 0; q < 3; q++) {
          d[(3 + q) * t + (size_t)j * nr + m] = -1.5 * p.sigma * p.epsilon * k4 * o[q];
          d[(6 + q) * t + (size_t)j * nr + m] = -1.5 * p.lambda * p.epsilon * k4 * o[q];
        }
      }
    if (cudaMalloc(&a->dcoef, d.size() * sizeof(double)) != cudaSuccess) return CHNS_ERR_NOMEM;
    if (cudaMemcpy(a->dcoef, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
      return CHNS_ERR_CUDA;
  }
  if (!a->side) {
    if (cudaStreamCreateWithFlags(&a->side, cudaStreamNonBlocking) != cudaSuccess) return CHNS_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&a->fork, cudaStreamNonBlocking) != cudaSuccess) return CHNS_ERR_CUDA;
    ACK(cudaEventCreateWithFlags(&a->ev_sweep, cudaEventDisableTiming));
    ACK(cudaEventCreateWithFlags(&a->ev_fork, cudaEventDisableTiming));
    ACK(cudaEventCreateWithFlags(&a->ev_join, cudaEventDisableTiming));
    for (int b = 0; b < 2; b++) {
      ACK(cudaEventCreateWithFlags(&a->ev_ready[b], cudaEventDisableTiming));
      ACK(cudaEventCreateWithFlags(&a->ev_free[b], cudaEventDisableTiming));
    }
  }
  if (seglen != a->seg_len || a->cap_states < seglen) {
    // two segments of slots if they fit, else one
    if (a->seg) cudaFree(a->seg);
    a->seg = nullptr;
    a->cap_states = 0;
    a->seg_len = 0;
    if (cudaMalloc(&a->seg, SLOT_FIELDS * fbytes * 2 * (size_t)seglen) == cudaSuccess) {
      a->cap_states = 2 * seglen;
    } else {
      cudaGetLastError();
      if (cudaMalloc(&a->seg, SLOT_FIELDS * fbytes * (size_t)seglen) != cudaSuccess) return CHNS_ERR_NOMEM;
      a->cap_states = seglen;
    }
    a->seg_len = seglen;
  }
  if (nckpt > a->nckpt_cap) {
    for (int k = 0; k < a->nckpt_cap; k++) {
      cudaFree(a->ckpt[k]);
      cudaFree(a->ckptk0[k]);
    }
    free(a->ckpt);
    free(a->ckptk0);
    a->ckpt = (void**)calloc(nckpt, sizeof(void*));
    a->ckptk0 = (double**)calloc(nckpt, sizeof(double*));
    if (!a->ckpt || !a->ckptk0) {
      a->nckpt_cap = 0;
      return CHNS_ERR_NOMEM;
    }
    a->nckpt_cap = nckpt;
    for (int k = 0; k < nckpt; k++) {
      if (cudaMalloc(&a->ckpt[k], snap) != cudaSuccess) return CHNS_ERR_NOMEM;
      if (cudaMalloc((void**)&a->ckptk0[k], 16 * sizeof(double)) != cudaSuccess) return CHNS_ERR_NOMEM;
    }
  }
  return CHNS_OK;
}

template <class R>
int adjoint_impl(chns_ctx* c, int nsteps, int ckpt, const double* lw, double* J, double* g_w, double* g_c,
                 double* g_par, int where) {
  const int nseg = (nsteps + ckpt - 1) / ckpt;
  int rc = adj_alloc(c, ckpt, nseg + 1);
  if (rc) return rc;
  chns_adj* a = c->adj;
  Adj<R> A;
  A.c = c;
  A.a = a;
  A.st = c->stream;
  A.ncx = a->ncx;
  A.nn = a->nn;
  A.blocks_s = (int)((A.ncx + 255) / 256);
  A.blocks_p = 1024;
  const chns_params& p = c->p;
  A.P.n = c->n;
  A.P.jt = c->jt;
  A.P.fx = c->fx;
  A.P.fy = c->fy;
  A.P.s1 = (R)(1.5 * p.sigma * p.epsilon);
  A.P.s2 = (R)(24.0 * (p.sigma / p.epsilon));
  A.P.lam = (R)p.lambda;
  A.P.ds1 = 1.5 * p.epsilon;
  A.P.ds2 = 24.0 / p.epsilon;
  A.P.mrow = c->mrow;
  cudaStream_t st = c->stream;
  const size_t bytes = A.ncx * sizeof(cx<R>);
  const R* coef = (const R*)c->coef;
  const double* dcoef = (const double*)a->dcoef;
  ACK(cudaMemsetAsync(a->acc, 0, 8 * sizeof(double), st));

  // forward sweep with checkpoints (checkpoint nseg keeps u_0 for restoring);
  // the last segment is recorded on the way
  char* segbase = (char*)a->seg;
  const size_t slot = SLOT_FIELDS * bytes;
  const int nlast = (nseg - 1) * ckpt;
  const size_t lastbuf = a->cap_states >= 2 * ckpt ? (size_t)((nseg - 1) % 2) * ckpt : 0;
  if ((rc = snapshot_save(c, a->ckpt[nseg], a->ckptk0[nseg]))) return rc;
  for (int n = 0; n < nsteps; n++) {
    if (n % ckpt == 0 && (rc = snapshot_save(c, a->ckpt[n / ckpt], a->ckptk0[n / ckpt]))) return rc;
    rc = n >= nlast ? record_step(c, segbase + (lastbuf + n - nlast) * slot, bytes) : chns_step(c, 1);
    if (rc) return rc;
  }
  // loss at the final state and its gradient (free_energy.c:3-157: c and grad c untruncated)
  {
    k_adj_loss_prep3<R><<<A.blocks_s, 256, 0, st>>>(A.P, (const cx<R>*)c->state[1], A.SS(0, SB), A.ncx);
    A.ifft(st, 0, A.SS(0, SB), A.FS(0, PCT), 3);
    const double inv = 1.0 / ((double)c->n * (double)c->n);
    const double kb = lw[0] * 12.0 * (p.sigma / p.epsilon) * inv;
    const double kg = (lw[1] * 0.75 * p.sigma * p.epsilon + 4.0 * lw[2]) * inv;
    const double dkb = lw[0] * 12.0 / p.epsilon * inv;
    const double dkg = lw[1] * 0.75 * p.epsilon * inv;
    k_adj_loss<R><<<kLossBlocks, 256, 0, st>>>(A.FS(0, PCT), A.FS(0, PCX), A.FS(0, PCY), A.F(PUB), A.F(PVB),
                                               A.F(PWXB), A.nn, kb, kg, dkb, dkg, a->acc + 8);
    k_sum_parts<<<1, 32, 0, st>>>(a->acc + 8, kLossBlocks, a->acc);
    A.dfft(st, 0, A.F(PUB), A.SS(0, SB), 3);
    k_adj_loss_acc3<R><<<A.blocks_s, 256, 0, st>>>(A.P, A.SS(0, SB), A.S(SGC), A.S(SGW), A.ncx);
  }
  // the reversed step as a CUDA graph on its fixed buffers (eager if capture fails)
  if (!a->rev && !a->rev_tried) {
    a->rev_tried = true;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      A.reverse_step(coef, dcoef, a->fork);
      if (cudaStreamEndCapture(st, &g) == cudaSuccess && g) {
        if (cudaGraphInstantiate(&a->rev, g, 0) != cudaSuccess) a->rev = nullptr;
        cudaGraphDestroy(g);
      }
    }
    cudaGetLastError();
  }
  // reverse sweep: each segment but the last is recomputed from its checkpoint
  // on the side stream, recording its steps into segment buffer s % nbuf, then
  // its steps are reversed on the context stream.  With two buffers the
  // recompute of segment s-1 runs while segment s is reversed.
  const int nbuf = a->cap_states >= 2 * ckpt ? 2 : 1;
  cudaStream_t side = a->side;
  ACK(cudaEventRecord(a->ev_sweep, st));
  ACK(cudaStreamWaitEvent(side, a->ev_sweep, 0));
  auto recompute = [&](int s) -> int {
    const int b = s % nbuf, len = (s * ckpt + ckpt <= nsteps) ? ckpt : nsteps - s * ckpt;
    if (s + nbuf <= nseg - 1) ACK(cudaStreamWaitEvent(side, a->ev_free[b], 0));
    c->stream = side;
    int r = snapshot_load(c, a->ckpt[s], a->ckptk0[s]);
    for (int k = 0; k < len && !r; k++) r = record_step(c, segbase + ((size_t)b * ckpt + k) * slot, bytes);
    c->stream = st;
    if (r) return r;
    ACK(cudaEventRecord(a->ev_ready[b], side));
    return CHNS_OK;
  };
  auto reverse = [&](int s) -> int {
    const int b = s % nbuf, len = (s * ckpt + ckpt <= nsteps) ? ckpt : nsteps - s * ckpt;
    if (s != nseg - 1) ACK(cudaStreamWaitEvent(st, a->ev_ready[b], 0));
    for (int k = len - 1; k >= 0; k--) {
      ACK(cudaMemcpyAsync(A.S(CUW), segbase + ((size_t)b * ckpt + k) * slot, slot, cudaMemcpyDeviceToDevice, st));
      if (a->rev) {
        ACK(cudaGraphLaunch(a->rev, st));
      } else {
        A.reverse_step(coef, dcoef, nullptr);
      }
    }
    ACK(cudaEventRecord(a->ev_free[b], st));
    return CHNS_OK;
  };
  for (int s = nseg - 1; s >= 0; s--) {
    if (nbuf == 2) {
      if (s > 0 && (rc = recompute(s - 1))) return rc;
      if ((rc = reverse(s))) return rc;
    } else {
      if ((rc = reverse(s))) return rc;
      if (s > 0 && (rc = recompute(s - 1))) return rc;
    }
  }
  ACK(cudaGetLastError());
  // restore u_0 and return the results
  if ((rc = snapshot_load(c, a->ckpt[nseg], a->ckptk0[nseg]))) return rc;
  double h[8];
  ACK(cudaMemcpyAsync(h, a->acc, sizeof(h), cudaMemcpyDeviceToHost, st));
  ACK(cudaStreamSynchronize(st));
  if (J) *J = h[0];
  if (g_par) {
    g_par[0] = h[4];
    g_par[1] = h[5];
    g_par[2] = h[6] + h[2];  // sigma: through the step and through the loss
  }
  const size_t fb = 2 * (size_t)c->n * c->nr * sizeof(double);
  const cudaMemcpyKind kind = where == CHNS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (g_w) {
    c->L->to_fftw(c, A.S(SGW), c->stage);
    ACK(cudaMemcpyAsync(g_w, c->stage, fb, kind, st));
  }
  if (g_c) {
    c->L->to_fftw(c, A.S(SGC), c->stage);
    ACK(cudaMemcpyAsync(g_c, c->stage, fb, kind, st));
  }
  ACK(cudaStreamSynchronize(st));
  return CHNS_OK;
}

}  // namespace

void chns_adj_free(chns_ctx* c) {
  chns_adj* a = c->adj;
  if (!a) return;
  if (a->rev) cudaGraphExecDestroy(a->rev);
  if (a->side) {
    cudaStreamSynchronize(a->side);
    cudaStreamDestroy(a->side);
    cudaStreamDestroy(a->fork);
    cudaEventDestroy(a->ev_sweep);
    cudaEventDestroy(a->ev_fork);
    cudaEventDestroy(a->ev_join);
    for (int b = 0; b < 2; b++) {
      cudaEventDestroy(a->ev_ready[b]);
      cudaEventDestroy(a->ev_free[b]);
    }
  }
  if (a->spec) cudaFree(a->spec);
  if (a->phys) cudaFree(a->phys);
  if (a->bscr) cudaFree(a->bscr);
  for (int k = 0; k < a->nckpt_cap; k++) {
    cudaFree(a->ckpt[k]);
    cudaFree(a->ckptk0[k]);
  }
  free(a->ckpt);
  free(a->ckptk0);
  if (a->seg) cudaFree(a->seg);
  if (a->dcoef) cudaFree(a->dcoef);
  if (a->acc) cudaFree(a->acc);
  free(a);
  c->adj = nullptr;
}

extern "C" int chns_adjoint(chns_ctx* c, int nsteps, int ckpt, const double* loss_w, double* J, double* g_w,
                            double* g_c, double* g_par, int where) {
  if (!c || nsteps < 1 || ckpt < 1) return CHNS_ERR_ARG;
  if (c->p.model != CHNS_MODEL_BINARY) return CHNS_ERR_UNSUPPORTED;
  const double dflt[3] = {1.0, 1.0, 1.0};
  const double* lw = loss_w ? loss_w : dflt;
  return c->f32 ? adjoint_impl<float>(c, nsteps, ckpt, lw, J, g_w, g_c, g_par, where)
                : adjoint_impl<double>(c, nsteps, ckpt, lw, J, g_w, g_c, g_par, where);
}
