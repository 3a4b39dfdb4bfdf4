// chns_adjoint.cu -- discrete adjoint of n ETD2RK steps (chns_adjoint), binary
// and ternary models.
//
// Gradient of a final-time functional J with respect to the initial spectral
// state (omega_hat_0 and c_hat_0, or c1_hat_0 and c2_hat_0) and to nu, lambda (the
// mobility M) and sigma (binary) or sigma_12, sigma_13, sigma_23 (ternary).  The
// schedule below is shared; Adj (binary) and AdjT3 (ternary) supply the buffers,
// the transposed step and the loss.
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
#include "chns_adjoint_ns.cuh"
#include "chns_adjoint_t.cuh"
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
  cudaGraphExec_t rev[2];  // one reverse step per current-step buffer (fixed buffers), or null
  void* rf;                // binary: RecStep, the record table of the step being reversed
  bool rev_tried;
  size_t ncx, nn;
};

namespace {

// Binary buffers: two spectral field sets of a batch and a scratch field (set 0: the
// loss; set 1: the transposes' work buffers), the loss's physical fields and the named
// ones; a reversed step reads its states and the forward fields the forward step
// recorded in its segment slot, through the table RecStep.
constexpr int SSET = 8;                      // spectral fields per set
enum { SB = 0, SXo = 7 };                     // batch of 7, scratch
enum {
  SY = 2 * SSET,                             // scratch (f_bar spectrum)
  SNBC,                                      // N*_bar, its c part
  SNBAW, SNBAC,                              // N(u_n)_bar
  SGW, SGC,                                  // running gradient (w_bar, c_bar)
  NSPEC
};
constexpr int PSET = 3;                                    // physical fields of the loss's set
enum { PCT = 0, PCX, PCY };                                 // the loss's c, cx, cy
enum { PFB = PSET, PAB, PBB, PFXB, PFYB, PUB, PVB, PWXB, PWYB, PCTB, PCXB, PCYB, NPHYS };
constexpr int kLossBlocks = 1024;  // blocks of the loss reduction
constexpr int kWork = 4;           // field-set index of the transposes' work buffers
constexpr int kAcc = 32;           // accumulators; the loss reduction's per-block partials follow

template <class R> struct Adj {
  static constexpr int NF = 2, NSPEC_ = NSPEC, NPHYS_ = NPHYS, NBSCR = FOP_N, NDCOEF = 9;
  static constexpr int NSPEC_ALL = NSPEC, NPHYS_ALL = NPHYS, NSCR = 2;
  static constexpr int kW = 1;  // field set of the transposes' work buffers
  // the forward step records what the transposes need (REC kernels): per right-hand
  // side REC_REAL real fields and one spectral field, kept with each segment slot
  static constexpr bool REC = true;
  static constexpr int REC_REAL = 8;
  chns_ctx* c;
  chns_adj* a;
  AdjPar<R> P;
  cudaStream_t st;
  size_t ncx, nn;
  int blocks_s, blocks_p;

  cx<R>* grad(int f) const { return S(SGW + f); }
  void setup() {
    const chns_params& p = c->p;
    P.n = c->n;
    P.jt = c->jt;
    P.fx = c->fx;
    P.fy = c->fy;
    P.s1 = (R)(1.5 * p.sigma * p.epsilon);
    P.s2 = (R)(24.0 * (p.sigma / p.epsilon));
    P.lam = (R)p.lambda;
    P.ds1 = 1.5 * p.epsilon;
    P.ds2 = 24.0 / p.epsilon;
    P.mrow = c->mrow;
  }
  // d/dnu of the w coefficients, d/dlambda and d/dsigma of the c coefficients
  static void dcoef_tables(const chns_ctx* c, std::vector<double>& d) {
    const int nr = c->nr;
    const chns_params& p = c->p;
    const size_t t = (size_t)nr * nr;
    d.assign(NDCOEF * t, 0.0);
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
  }
  // loss at the final state and its gradient (free_energy.c:3-157: c and grad c untruncated)
  void loss(const double* lw) {
    const chns_params& p = c->p;
    k_adj_loss_prep3<R><<<blocks_s, 256, 0, st>>>(P, (const cx<R>*)c->state[1], SS(0, SB), ncx);
    ifft(st, 0, SS(0, SB), FS(0, PCT), 3);
    const double inv = 1.0 / ((double)c->n * (double)c->n);
    const double kb = lw[0] * 12.0 * (p.sigma / p.epsilon) * inv;
    const double kg = (lw[1] * 0.75 * p.sigma * p.epsilon + 4.0 * lw[2]) * inv;
    const double dkb = lw[0] * 12.0 / p.epsilon * inv;
    const double dkg = lw[1] * 0.75 * p.epsilon * inv;
    k_adj_loss<R><<<kLossBlocks, 256, 0, st>>>(FS(0, PCT), FS(0, PCX), FS(0, PCY), F(PUB), F(PVB), F(PWXB), nn, kb,
                                               kg, dkb, dkg, a->acc + kAcc);
    k_sum_parts<<<1, 32, 0, st>>>(a->acc + kAcc, kLossBlocks, a->acc);
    dfft(st, 0, F(PUB), SS(0, SB), 3);
    k_adj_loss_acc3<R><<<blocks_s, 256, 0, st>>>(P, SS(0, SB), S(SGC), S(SGW), ncx);
  }
  // h: the accumulators; g_par = dJ/d(nu, lambda, sigma)
  void params(const double* h, double* g_par) const {
    g_par[0] = h[4];
    g_par[1] = h[5];
    g_par[2] = h[6] + h[2];  // sigma: through the step and through the loss
  }

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

  RecStep<R>* table() const { return static_cast<RecStep<R>*>(a->rf); }

  // the transposed right-hand side r (0: at u*, 1: at u_n) from its tail batch
  // (SS(kW, SB), four spectra of N_bar) to the batch of its seven transformed product
  // adjoints in the same place, with the step's record (N_c_bar: nbc); gc += the mu
  // term; parameter partials into acc[4..6]
  void rhs_body(int r, const cx<R>* nbc, cx<R>* gc) {
    const RecFields<R>* rf = &table()->rhs[r];
    double* pacc = a->acc + 4;
    const void* in[5] = {F(PAB), F(PBB), F(PFXB), F(PFYB), F(PFB)};
    ifft(st, kW, SS(kW, SB), F(PAB), 4);  // A_bar, B_bar, Fx_bar, Fy_bar
    // mu_bar (formed in the transform's first pass) -> c_bar (s1 k^2), f_bar, lambda
    // and sigma partials
    c->L->adjprod(c, rf, in, 7, 1, SS(kW, SXo), ncx, scratch(kW));
    k_adj_mu<R><<<blocks_s, 256, 0, st>>>(P, SS(kW, SXo), rf, nbc, gc, S(SY), pacc);
    ifft(st, kW, S(SY), F(PFB), 1);
    // the seven product adjoints, formed in the first pass of their forward transforms
    c->L->adjprod(c, rf, in, 0, FOP_N, SS(kW, SB), ncx, scratch(kW));
  }

  // one reversed step from the step's record (table(): its states u_n, u*, N(u_n),
  // N(u*) and forward fields): the transposed stage 2 with the tail at u*, the
  // right-hand side at u*, its C^T with stage 1 and the tail at u_n, the right-hand
  // side at u_n and its C^T
  void reverse_step(const R* coef, const double* dcoef, cudaStream_t, int) {
    double* pacc = a->acc + 4;
    cx<R>* gw = S(SGW);
    cx<R>* gc = S(SGC);
    k_adj_etd2_tail<R><<<blocks_s, 256, 0, st>>>(P, coef, dcoef, gw, gc, table(), S(SNBC), S(SNBAW), S(SNBAC),
                                                 SS(kW, SB), ncx, pacc);
    rhs_body(0, S(SNBC), gc);
    k_adj_acc7_etd1_tail<R><<<blocks_s, 256, 0, st>>>(P, coef, dcoef, SS(kW, SB), gw, gc, table(), S(SNBAW),
                                                      S(SNBAC), ncx, pacc);
    rhs_body(1, S(SNBAC), gc);
    k_adj_acc7<R><<<blocks_s, 256, 0, st>>>(P, SS(kW, SB), gw, gc, ncx);
  }
  void prime(cudaStream_t, int) {}  // the forward fields are recorded, not rebuilt
};

// ---------------------------------------------------------------------------
// pure Navier-Stokes: state w.  Two field sets as in the binary model (0: u*,
// 1: u_n), each with the batch of the four forward spectra (u, v, wx, wy) and
// their physical fields.
// ---------------------------------------------------------------------------
namespace nsadj {
constexpr int SSET = 4;                        // spectral fields per set (the batch of 4)
enum {
  SA = 2 * SSET,                               // A_bar spectrum
  SNB,                                         // N*_bar
  SNA,                                         // N(u_n)_bar
  SG,                                          // running gradient
  CUR,                                         // current step: u_n, u*, N(u_n), N(u*)
  NSPEC = CUR + 4
};
constexpr int PSET = 4;                        // u, v, wx, wy per set
enum { PA = 2 * PSET, PXB, NPHYS = PXB + 4 };  // A_bar, then the batch of 4 adjoints
}  // namespace nsadj

template <class R> struct AdjNS {
  static constexpr int NF = 1, NSPEC_ = nsadj::NSPEC, NPHYS_ = nsadj::NPHYS, NBSCR = 4, NDCOEF = 3;
  static constexpr int NSPEC_ALL = NSPEC_ + 3 * nsadj::SSET + 4 * NF, NPHYS_ALL = NPHYS_ + 2 * nsadj::PSET, NSCR = 5;
  static constexpr bool REC = false;
  static constexpr int REC_REAL = 0;
  chns_ctx* c;
  chns_adj* a;
  AdjPar<R> P;
  cudaStream_t st;
  size_t ncx, nn;
  int blocks_s, blocks_p;

  cx<R>* S(int k) const { return (cx<R>*)a->spec + (size_t)k * ncx; }
  R* F(int k) const { return (R*)a->phys + (size_t)k * nn; }
  // field sets 0, 1 (parity 0: u*, u_n), 2, 3 (parity 1), 4: the transposes' work
  cx<R>* SS(int set, int k) const {
    return set < 2 ? S(set * nsadj::SSET + k) : S(NSPEC_ + (set - 2) * nsadj::SSET + k);
  }
  R* FS(int set, int k) const { return set < 2 ? F(set * nsadj::PSET + k) : F(NPHYS_ + (set - 2) * nsadj::PSET + k); }
  void* scratch(int set) const { return (char*)a->bscr + (size_t)set * NBSCR * ncx * sizeof(cx<R>); }
  int curbase(int par) const { return par == 0 ? nsadj::CUR : NSPEC_ + 3 * nsadj::SSET; }
  cx<R>* grad(int) const { return S(nsadj::SG); }

  void setup() {
    P.n = c->n;
    P.jt = c->jt;
    P.fx = c->fx;
    P.fy = c->fy;
    P.s1 = P.s2 = P.lam = (R)0;
    P.ds1 = P.ds2 = 0.0;
    P.mrow = c->mrow;
  }
  // d/dnu of the w coefficients (e, z1, z2)
  static void dcoef_tables(const chns_ctx* c, std::vector<double>& d) {
    const int nr = c->nr;
    const size_t t = (size_t)nr * nr;
    d.assign(NDCOEF * t, 0.0);
    for (int j = 0; j < nr; j++)
      for (int m = 0; m < nr; m++) {
        const double kx = c->fx * m, ky = c->fy * j, ks = kx * kx + ky * ky;
        double o[3];
        dcoef_dc(-c->p.nu * ks, c->p.dt, o);
        for (int q = 0; q < 3; q++) d[q * t + (size_t)j * nr + m] = -ks * o[q];
      }
  }
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
  // loss at the final state (w[0] kinetic energy, w[1] enstrophy, both of the
  // truncated fields) and its gradient
  void loss(const double* lw) {
    using namespace nsadj;
    k_adjns_loss_prep3<R><<<blocks_s, 256, 0, st>>>(P, (const cx<R>*)c->state[0], SS(0, 0), ncx);
    ifft(st, 0, SS(0, 0), FS(0, 0), 3);
    const double inv = 1.0 / ((double)c->n * (double)c->n);
    k_adjns_loss<R><<<kLossBlocks, 256, 0, st>>>(FS(0, 0), FS(0, 1), FS(0, 2), F(PXB), F(PXB + 1), F(PXB + 2), nn,
                                                 lw[0] * inv, lw[1] * inv, a->acc + kAcc);
    k_sum_parts<<<1, 32, 0, st>>>(a->acc + kAcc, kLossBlocks, a->acc);
    dfft(st, 0, F(PXB), SS(0, 0), 3);
    k_adjns_loss_acc3<R><<<blocks_s, 256, 0, st>>>(P, SS(0, 0), S(SG), ncx);
  }
  // g_par = dJ/d(nu, lambda, sigma): only nu acts on a pure Navier-Stokes run
  void params(const double* h, double* g_par) const {
    g_par[0] = h[4];
    g_par[1] = 0.0;
    g_par[2] = 0.0;
  }
  void fields(cudaStream_t s, int set, const cx<R>* w) {
    k_adjns_prep4<R><<<blocks_s, 256, 0, s>>>(P, w, SS(set, 0), ncx);
    ifft(s, set, SS(set, 0), FS(set, 0), 4);
  }
  // gw += J_N(state)^T nbw with the forward fields of set `set`.  Scratch of set 0.
  void transpose_rhs(int set, const cx<R>* nbw, cx<R>* gw) {
    using namespace nsadj;
    k_adjns_tail1<R><<<blocks_s, 256, 0, st>>>(P, nbw, S(SA));
    ifft(st, kWork, S(SA), F(PA), 1);
    k_adjns_products<R><<<blocks_p, 256, 0, st>>>(FS(set, 0), FS(set, 1), FS(set, 2), FS(set, 3), F(PA), F(PXB),
                                                  F(PXB + 1), F(PXB + 2), F(PXB + 3), nn);
    dfft(st, kWork, F(PXB), SS(kWork, 0), 4);
    k_adjns_acc4<R><<<blocks_s, 256, 0, st>>>(P, SS(kWork, 0), gw, ncx);
  }
  // one reversed step from current-step buffer `par` (u_n, u*, N(u_n), N(u*)), whose
  // forward fields were built before it; the next step's are built on the fork
  void reverse_step(const R* coef, const double* dcoef, cudaStream_t fork, int par) {
    using namespace nsadj;
    double* pacc = a->acc + 4;
    cx<R>* gw = S(SG);
    const int b = curbase(par);
    const cx<R>* un = S(b);
    const cx<R>* nn_ = S(b + 2);
    const cx<R>* ns_ = S(b + 3);
    if (fork) {
      cudaEventRecord(a->ev_fork, st);
      cudaStreamWaitEvent(fork, a->ev_fork, 0);
      prime(fork, 1 - par);
      cudaEventRecord(a->ev_join, fork);
    }
    k_adjns_etd2<R><<<blocks_s, 256, 0, st>>>(P, coef, dcoef, gw, ns_, nn_, S(SNB), S(SNA), pacc);
    transpose_rhs(2 * par, S(SNB), gw);
    k_adjns_etd1<R><<<blocks_s, 256, 0, st>>>(P, coef, dcoef, gw, un, nn_, S(SNA), pacc);
    transpose_rhs(2 * par + 1, S(SNA), gw);
    if (fork) {
      cudaStreamWaitEvent(st, a->ev_join, 0);
    } else {
      prime(st, 1 - par);
    }
  }
  // forward fields of current-step buffer `par` into sets 2 par (at u*), 2 par + 1 (at u_n)
  void prime(cudaStream_t s, int par) {
    const int b = curbase(par);
    fields(s, 2 * par, S(b + 1));
    fields(s, 2 * par + 1, S(b));
  }
};

// ---------------------------------------------------------------------------
// ternary model: state (w, c1, c2)
// ---------------------------------------------------------------------------
namespace tern {
constexpr int SSET = 14;                       // spectral fields per set
enum { SB = 0, SX = 10, SFF = 12 };             // batch of 10, mu_hat batch of 2, F[muF] batch of 2
enum {
  SYB = 2 * SSET,                              // F[muF]_bar spectra (2)
  SNB = SYB + 2,                               // N*_bar (3)
  SNA = SNB + 3,                               // N(u_n)_bar (3)
  SG = SNA + 3,                                // running gradient (3)
  CUR = SG + 3,                                // current step: u_n, u*, N(u_n), N(u*) (3 each)
  NSPEC = CUR + 12
};
constexpr int PSET = 14;                       // physical fields per set
enum { PF = 0, PMF = 10, PMU = 12 };            // ten forward fields, muF (2), mu (2)
enum { PTAIL = 2 * PSET, PMUB = PTAIL + 5, PMFB = PMUB + 2, PXB = PMFB + 2, NPHYS = PXB + 10 };
}  // namespace tern

template <class R> struct AdjT3 {
  static constexpr int NF = 3, NSPEC_ = tern::NSPEC, NPHYS_ = tern::NPHYS, NBSCR = T_N, NDCOEF = 6;
  static constexpr int NSPEC_ALL = NSPEC_ + 3 * tern::SSET + 4 * NF, NPHYS_ALL = NPHYS_ + 2 * tern::PSET, NSCR = 5;
  static constexpr bool REC = false;
  static constexpr int REC_REAL = 0;
  int cb = tern::CUR;  // current-step buffer of the step being reversed
  chns_ctx* c;
  chns_adj* a;
  AdjParT<R> P;
  cudaStream_t st;
  size_t ncx, nn;
  int blocks_s, blocks_p;

  cx<R>* S(int k) const { return (cx<R>*)a->spec + (size_t)k * ncx; }
  R* F(int k) const { return (R*)a->phys + (size_t)k * nn; }
  // field sets 0, 1 (parity 0: u*, u_n), 2, 3 (parity 1), 4: the transposes' work
  cx<R>* SS(int set, int k) const {
    return set < 2 ? S(set * tern::SSET + k) : S(NSPEC_ + (set - 2) * tern::SSET + k);
  }
  R* FS(int set, int k) const { return set < 2 ? F(set * tern::PSET + k) : F(NPHYS_ + (set - 2) * tern::PSET + k); }
  void* scratch(int set) const { return (char*)a->bscr + (size_t)set * T_N * ncx * sizeof(cx<R>); }
  int curbase(int par) const { return par == 0 ? tern::CUR : NSPEC_ + 3 * tern::SSET; }
  cx<R>* grad(int f) const { return S(tern::SG + f); }
  cx<R>* cu(int f) const { return S(cb + f); }       // u_n
  cx<R>* cs(int f) const { return S(cb + 3 + f); }   // u*
  cx<R>* cn(int f) const { return S(cb + 6 + f); }   // N(u_n)
  cx<R>* cx_(int f) const { return S(cb + 9 + f); }  // N(u*)

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

  void setup() {
    const chns_params& p = c->p;
    P.n = c->n;
    P.jt = c->jt;
    P.fx = c->fx;
    P.fy = c->fy;
    P.mrow = c->mrow;
    P.s1 = P.s2 = P.lam = (R)0;
    P.ds1 = P.ds2 = 0.0;
    const double g1 = c->gamma[0], g2 = c->gamma[1], g3 = c->gamma[2];
    P.g1 = (R)g1;
    P.g2 = (R)g2;
    P.g3 = (R)g3;
    P.kk = (R)(2.0 * c->del / p.epsilon);
    P.xl6 = (R)(6.0 * p.xlambda);
    P.mu1c = (R)(0.75 * g1 * p.epsilon);
    P.mu2c = (R)(0.75 * g2 * p.epsilon);
    P.lg1 = (R)(p.lambda / g1);
    P.lg2 = (R)(p.lambda / g2);
    P.w11 = (R)(1.0 + g3 / g1);
    P.w12 = (R)(g3 / g2);
    P.w21 = (R)(g3 / g1);
    P.w22 = (R)(1.0 + g3 / g2);
  }
  // d/dnu of the w coefficients, d/dlambda of the c coefficients (-0.75 lambda eps k^4)
  static void dcoef_tables(const chns_ctx* c, std::vector<double>& d) {
    const int nr = c->nr;
    const chns_params& p = c->p;
    const size_t t = (size_t)nr * nr;
    d.assign(NDCOEF * t, 0.0);
    for (int j = 0; j < nr; j++)
      for (int m = 0; m < nr; m++) {
        const double kx = c->fx * m, ky = c->fy * j, ks = kx * kx + ky * ky, k4 = ks * ks;
        double o[3];
        dcoef_dc(-p.nu * ks, p.dt, o);
        for (int q = 0; q < 3; q++) d[q * t + (size_t)j * nr + m] = -ks * o[q];
        dcoef_dc(-0.75 * p.lambda * p.epsilon * k4, p.dt, o);
        for (int q = 0; q < 3; q++) d[(3 + q) * t + (size_t)j * nr + m] = -0.75 * p.epsilon * k4 * o[q];
      }
  }

  // forward fields of the right-hand side at (w, c1, c2) into field set `set`
  void fields(cudaStream_t s, int set, const cx<R>* w, const cx<R>* c1, const cx<R>* c2) {
    k_adj3_fwd_prep<R><<<blocks_s, 256, 0, s>>>(P, w, c1, c2, SS(set, tern::SB), ncx);
    ifft(s, set, SS(set, tern::SB), FS(set, tern::PF), T_N);
    k_adj3_bulk<R><<<blocks_p, 256, 0, s>>>(P, FS(set, tern::PF + T_C1), FS(set, tern::PF + T_C2),
                                            FS(set, tern::PMF), nn);
    dfft(s, set, FS(set, tern::PMF), SS(set, tern::SFF), 2);
    k_adj3_mu_prep<R><<<blocks_s, 256, 0, s>>>(P, c1, c2, SS(set, tern::SFF), SS(set, tern::SX), ncx);
    ifft(s, set, SS(set, tern::SX), FS(set, tern::PMU), 2);
  }

  // (gw, g1, g2) += J_N(state)^T (nw, n1, n2) with the forward fields of `set`;
  // parameter sums into acc[8 + 2 ..]
  void transpose_rhs(int set, const cx<R>* c1, const cx<R>* c2, const cx<R>* nw, const cx<R>* n1, const cx<R>* n2) {
    double* pacc = a->acc + 8;
    k_adj3_tail<R><<<blocks_s, 256, 0, st>>>(P, nw, n1, n2, SS(kWork, tern::SB), ncx);
    ifft(st, kWork, SS(kWork, tern::SB), F(tern::PTAIL), 5);
    const int b = tern::PF;
    PhysT<R> pf{FS(set, b + T_U),   FS(set, b + T_V),   FS(set, b + T_WX),  FS(set, b + T_WY),  FS(set, b + T_C1X),
                FS(set, b + T_C1Y), FS(set, b + T_C2X), FS(set, b + T_C2Y), FS(set, tern::PMU), FS(set, tern::PMU + 1)};
    AdjT5<R> at{F(tern::PTAIL), F(tern::PTAIL + 1), F(tern::PTAIL + 2), F(tern::PTAIL + 3), F(tern::PTAIL + 4)};
    k_adj3_products<R><<<blocks_p, 256, 0, st>>>(P, pf, at, F(tern::PXB), F(tern::PMUB), nn, pacc + 2);
    dfft(st, kWork, F(tern::PMUB), SS(kWork, tern::SX), 2);
    k_adj3_mu<R><<<blocks_s, 256, 0, st>>>(P, SS(kWork, tern::SX), c1, c2, SS(set, tern::SFF), n1, n2, grad(1), grad(2),
                                           S(tern::SYB), ncx, pacc + 6);
    ifft(st, kWork, S(tern::SYB), F(tern::PMFB), 2);
    k_adj3_bulk_bar<R><<<blocks_p, 256, 0, st>>>(P, FS(set, b + T_C1), FS(set, b + T_C2), F(tern::PMFB),
                                                 F(tern::PXB), nn, pacc + 10);
    dfft(st, kWork, F(tern::PXB), SS(kWork, tern::SB), T_N);
    k_adj3_acc<R><<<blocks_s, 256, 0, st>>>(P, SS(kWork, tern::SB), grad(0), grad(1), grad(2), ncx);
  }

  // one reversed step from current-step buffer `par`, whose forward fields were
  // built before it; the next step's (buffer 1 - par) are built on the fork
  void reverse_step(const R* coef, const double* dcoef, cudaStream_t fork, int par) {
    double* pacc = a->acc + 8;
    cb = curbase(par);
    if (fork) {
      cudaEventRecord(a->ev_fork, st);
      cudaStreamWaitEvent(fork, a->ev_fork, 0);
      prime(fork, 1 - par);
      cudaEventRecord(a->ev_join, fork);
    }
    CFields3<R> g{{grad(0), grad(1), grad(2)}};
    CFields3<R> nst{{cx_(0), cx_(1), cx_(2)}}, nnn{{cn(0), cn(1), cn(2)}}, un{{cu(0), cu(1), cu(2)}};
    Fields3<R> nbs{{S(tern::SNB), S(tern::SNB + 1), S(tern::SNB + 2)}};
    Fields3<R> nba{{S(tern::SNA), S(tern::SNA + 1), S(tern::SNA + 2)}};
    Fields3<R> gm{{grad(0), grad(1), grad(2)}};
    k_adj3_etd2<R><<<blocks_s, 256, 0, st>>>(P, coef, dcoef, g, nst, nnn, nbs, nba, pacc);
    transpose_rhs(2 * par, cs(1), cs(2), S(tern::SNB), S(tern::SNB + 1), S(tern::SNB + 2));
    k_adj3_etd1<R><<<blocks_s, 256, 0, st>>>(P, coef, dcoef, gm, un, nnn, nba, pacc);
    transpose_rhs(2 * par + 1, cu(1), cu(2), S(tern::SNA), S(tern::SNA + 1), S(tern::SNA + 2));
    if (fork) {
      cudaStreamWaitEvent(st, a->ev_join, 0);
    } else {
      prime(st, 1 - par);
    }
  }
  // forward fields of current-step buffer `par` into sets 2 par (at u*), 2 par + 1 (at u_n)
  void prime(cudaStream_t s, int par) {
    const int b = curbase(par);
    fields(s, 2 * par, S(b + 3), S(b + 4), S(b + 5));
    fields(s, 2 * par + 1, S(b + 0), S(b + 1), S(b + 2));
  }

  void loss(const double* lw) {
    const chns_params& p = c->p;
    k_adj3_loss_prep<R><<<blocks_s, 256, 0, st>>>(P, (const cx<R>*)c->state[1], (const cx<R>*)c->state[2],
                                                  SS(0, tern::SB), ncx);
    ifft(st, 0, SS(0, tern::SB), FS(0, tern::PF), 6);
    const double inv = 1.0 / ((double)c->n * (double)c->n);
    const double kb = lw[0] * (6.0 / p.epsilon) * inv, kg = lw[1] * 0.375 * p.epsilon * inv, kp = lw[2] * inv;
    k_adj3_loss<R><<<kLossBlocks, 256, 0, st>>>(P, FS(0, tern::PF), F(tern::PXB), nn, kb, kg, kp, a->acc + kAcc);
    k_sum_partsn<4><<<1, 32, 0, st>>>(a->acc + kAcc, kLossBlocks, a->acc);
    dfft(st, 0, F(tern::PXB), SS(0, tern::SB), 6);
    k_adj3_loss_acc<R><<<blocks_s, 256, 0, st>>>(P, SS(0, tern::SB), grad(1), grad(2), grad(0), ncx);
  }

  // g_par = dJ/d(nu, lambda, sigma_12, sigma_13, sigma_23), chained through
  // gamma_1 = s12 + s13 - s23, gamma_2 = s12 + s23 - s13, gamma_3 = s13 + s23 - s12
  // (main.c:166-170) and Delta = 6 g1 g2 g3 / (g1 g2 + g1 g3 + g2 g3)
  void params(const double* h, double* g_par) const {
    const chns_params& p = c->p;
    const double* q = h + 8;
    const double g1 = c->gamma[0], g2 = c->gamma[1], g3 = c->gamma[2], eps = p.epsilon, lam = p.lambda;
    double dg[3] = {h[1] + q[11], h[2] + q[12], h[3] + q[13]};
    dg[0] += q[14] * (-1.0 / (g1 * g1));
    dg[1] += q[15] * (-1.0 / (g2 * g2));
    dg[2] += q[16] * (-1.0 / (g3 * g3));
    // weights w11 = 1 + g3/g1, w12 = g3/g2, w21 = g3/g1, w22 = 1 + g3/g2
    dg[0] += (q[2] + q[4]) * (-g3 / (g1 * g1));
    dg[1] += (q[3] + q[5]) * (-g3 / (g2 * g2));
    dg[2] += (q[2] + q[4]) / g1 + (q[3] + q[5]) / g2;
    // 0.75 g_i eps k^2 c_i in mu_i; lambda / g_i in N_ci
    dg[0] += q[6] * 0.75 * eps + q[8] * (-lam / (g1 * g1));
    dg[1] += q[7] * 0.75 * eps + q[9] * (-lam / (g2 * g2));
    // K = 2 Delta / eps
    const double S = g1 * g2 + g1 * g3 + g2 * g3, P3 = g1 * g2 * g3;
    const double dD[3] = {6.0 * (g2 * g3 * S - P3 * (g2 + g3)) / (S * S), 6.0 * (g1 * g3 * S - P3 * (g1 + g3)) / (S * S),
                          6.0 * (g1 * g2 * S - P3 * (g1 + g2)) / (S * S)};
    for (int k = 0; k < 3; k++) dg[k] += q[10] * (2.0 / eps) * dD[k];
    g_par[0] = q[0];
    g_par[1] = q[1] + q[8] / g1 + q[9] / g2;
    g_par[2] = dg[0] + dg[1] - dg[2];
    g_par[3] = dg[0] - dg[1] + dg[2];
    g_par[4] = -dg[0] + dg[1] + dg[2];
  }
};

// one forward step that also records u_n, u*, N(u_n) and N(u*) (nf fields each)
// into a segment slot; with recb > 0 (binary) the stages' REC kernels also record the
// forward fields of the right-hand sides at u_n and at u* (recb bytes each) behind them
int record_step(chns_ctx* c, char* slot, size_t fbytes, int nf, size_t recb) {
  cudaStream_t st = c->stream;
  for (int f = 0; f < nf; f++) ACK(cudaMemcpyAsync(slot + f * fbytes, c->state[f], fbytes, cudaMemcpyDeviceToDevice, st));
  char* rec = slot + 4 * (size_t)nf * fbytes;
  c->rec = recb ? rec : nullptr;
  c->L->stage(c, 1);
  c->rec = recb ? rec + recb : nullptr;
  for (int f = 0; f < nf; f++) {
    ACK(cudaMemcpyAsync(slot + (nf + f) * fbytes, c->state[f], fbytes, cudaMemcpyDeviceToDevice, st));
    ACK(cudaMemcpyAsync(slot + (2 * nf + f) * fbytes, c->saved[f], fbytes, cudaMemcpyDeviceToDevice, st));
    c->nstar[f] = slot + (3 * nf + f) * fbytes;
  }
  c->L->stage(c, 2);
  c->rec = nullptr;
  for (int f = 0; f < 3; f++) c->nstar[f] = nullptr;
  return CHNS_OK;
}

int snapshot_save(chns_ctx* c, void* dst, double* dstk0) {
  const size_t bytes = (size_t)c->n * c->nr * 2 * c->rsz;
  for (int f = 0; f <= c->p.model; f++)
    ACK(cudaMemcpyAsync((char*)dst + f * bytes, c->state[f], bytes, cudaMemcpyDeviceToDevice, c->stream));
  ACK(cudaMemcpyAsync(dstk0, c->k0, 16 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return CHNS_OK;
}
int snapshot_load(chns_ctx* c, const void* src, const double* srck0) {
  const size_t bytes = (size_t)c->n * c->nr * 2 * c->rsz;
  for (int f = 0; f <= c->p.model; f++)
    ACK(cudaMemcpyAsync(c->state[f], (const char*)src + f * bytes, bytes, cudaMemcpyDeviceToDevice, c->stream));
  ACK(cudaMemcpyAsync(c->k0, srck0, 16 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  return CHNS_OK;
}

// bytes of one recorded forward right-hand side (binary) and of one segment slot
template <class A> size_t rec_bytes(const chns_ctx* c) {
  if (!A::REC) return 0;
  const size_t nn = (size_t)c->n * c->n;
  return A::REC_REAL * nn * c->rsz + (size_t)c->n * c->nr * 2 * c->rsz;
}
template <class A> size_t slot_bytes(const chns_ctx* c) {
  return 4 * (size_t)A::NF * c->n * c->nr * 2 * c->rsz + 2 * rec_bytes<A>(c);
}

template <class A> int adj_alloc(chns_ctx* c, int seglen, int nckpt) {
  if (!c->adj) {
    c->adj = (chns_adj*)calloc(1, sizeof(chns_adj));
    if (!c->adj) return CHNS_ERR_NOMEM;
  }
  chns_adj* a = c->adj;
  const size_t ncx = (size_t)c->n * c->nr, nn = (size_t)c->n * c->n;
  const size_t fbytes = ncx * 2 * c->rsz;  // one S-layout field
  const size_t snap = (size_t)A::NF * fbytes;
  a->ncx = ncx;
  a->nn = nn;
  if (!a->dcoef) {
    if (cudaMalloc(&a->spec, A::NSPEC_ALL * fbytes) != cudaSuccess) return CHNS_ERR_NOMEM;
    if (cudaMalloc(&a->phys, A::NPHYS_ALL * nn * c->rsz) != cudaSuccess) return CHNS_ERR_NOMEM;
    if (cudaMalloc(&a->bscr, (size_t)A::NSCR * A::NBSCR * fbytes) != cudaSuccess) return CHNS_ERR_NOMEM;
    if (cudaMalloc((void**)&a->acc, (kAcc + 4 * kLossBlocks) * sizeof(double)) != cudaSuccess) return CHNS_ERR_NOMEM;
    if (cudaMalloc(&a->rf, sizeof(RecStep<double>)) != cudaSuccess) return CHNS_ERR_NOMEM;
    std::vector<double> d;
    A::dcoef_tables(c, d);
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
    const size_t slot = slot_bytes<A>(c);
    if (cudaMalloc(&a->seg, slot * 2 * (size_t)seglen) == cudaSuccess) {
      a->cap_states = 2 * seglen;
    } else {
      cudaGetLastError();
      if (cudaMalloc(&a->seg, slot * (size_t)seglen) != cudaSuccess) return CHNS_ERR_NOMEM;
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

template <class R, class A>
int adjoint_impl(chns_ctx* c, int nsteps, int ckpt, const double* lw, double* J, double* g_w, double* g_c,
                 double* g_par, int where) {
  const int nseg = (nsteps + ckpt - 1) / ckpt;
  int rc = adj_alloc<A>(c, ckpt, nseg + 1);
  if (rc) return rc;
  chns_adj* a = c->adj;
  A ad;
  ad.c = c;
  ad.a = a;
  ad.st = c->stream;
  ad.ncx = a->ncx;
  ad.nn = a->nn;
  ad.blocks_s = (int)((ad.ncx + 255) / 256);
  ad.blocks_p = 1024;
  ad.setup();
  cudaStream_t st = c->stream;
  const size_t bytes = ad.ncx * sizeof(cx<R>);
  const R* coef = (const R*)c->coef;
  const double* dcoef = (const double*)a->dcoef;
  ACK(cudaMemsetAsync(a->acc, 0, kAcc * sizeof(double), st));

  // forward sweep with checkpoints (checkpoint nseg keeps u_0 for restoring);
  // the last segment is recorded on the way
  char* segbase = (char*)a->seg;
  const size_t cur = 4 * (size_t)A::NF * bytes;  // u_n, u*, N(u_n), N(u*)
  const size_t recb = rec_bytes<A>(c), slot = slot_bytes<A>(c);
  const int nlast = (nseg - 1) * ckpt;
  const size_t lastbuf = a->cap_states >= 2 * ckpt ? (size_t)((nseg - 1) % 2) * ckpt : 0;
  if ((rc = snapshot_save(c, a->ckpt[nseg], a->ckptk0[nseg]))) return rc;
  for (int n = 0; n < nsteps; n++) {
    if (n % ckpt == 0 && (rc = snapshot_save(c, a->ckpt[n / ckpt], a->ckptk0[n / ckpt]))) return rc;
    rc = n >= nlast ? record_step(c, segbase + (lastbuf + n - nlast) * slot, bytes, A::NF, recb) : chns_step(c, 1);
    if (rc) return rc;
  }
  ad.loss(lw);
  // the reversed step as a CUDA graph per current-step buffer, on fixed buffers
  // (eager if a capture fails)
  if (!a->rev[0] && !a->rev_tried) {
    a->rev_tried = true;
    bool ok = true;
    for (int par = 0; par < (A::REC ? 1 : 2) && ok; par++) {
      cudaGraph_t g = nullptr;
      ok = false;
      if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        ad.reverse_step(coef, dcoef, a->fork, par);
        if (cudaStreamEndCapture(st, &g) == cudaSuccess && g) {
          ok = cudaGraphInstantiate(&a->rev[par], g, 0) == cudaSuccess;
          cudaGraphDestroy(g);
        }
      }
      if (!ok) a->rev[par] = nullptr;
    }
    if (!ok) {
      for (int par = 0; par < 2; par++) {
        if (a->rev[par]) cudaGraphExecDestroy(a->rev[par]);
        a->rev[par] = nullptr;
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
    for (int k = 0; k < len && !r; k++)
      r = record_step(c, segbase + ((size_t)b * ckpt + k) * slot, bytes, A::NF, recb);
    c->stream = st;
    if (r) return r;
    ACK(cudaEventRecord(a->ev_ready[b], side));
    return CHNS_OK;
  };
  // Binary: the table is pointed at step k's slot and the one graph runs.  Ternary and
  // pure Navier-Stokes: steps alternate between two current-step buffers; while step k
  // (buffer k & 1) is reversed, step k - 1 is already in the other buffer and its
  // forward fields are built on the graph's parallel branch, so no reversed step waits
  // for its own.
  auto reverse = [&](int s) -> int {
    const int b = s % nbuf, len = (s * ckpt + ckpt <= nsteps) ? ckpt : nsteps - s * ckpt;
    if (s != nseg - 1) ACK(cudaStreamWaitEvent(st, a->ev_ready[b], 0));
    auto slot_of = [&](int k) { return segbase + ((size_t)b * ckpt + k) * slot; };
    if constexpr (A::REC) {  // the reversed step reads the slot through the table
      for (int k = len - 1; k >= 0; k--) {
        char* sk = slot_of(k);
        k_adj_set_rec<R><<<1, 1, 0, st>>>(static_cast<RecStep<R>*>(a->rf), (const cx<R>*)sk, ad.ncx,
                                          (const R*)(sk + cur + recb), (const R*)(sk + cur), a->nn);
        if (a->rev[0]) {
          ACK(cudaGraphLaunch(a->rev[0], st));
        } else {
          ad.reverse_step(coef, dcoef, nullptr, 0);
        }
      }
      ACK(cudaEventRecord(a->ev_free[b], st));
      return CHNS_OK;
    } else {
      const int p0 = (len - 1) & 1;
      ACK(cudaMemcpyAsync(ad.S(ad.curbase(p0)), slot_of(len - 1), cur, cudaMemcpyDeviceToDevice, st));
      ad.prime(st, p0);
      for (int k = len - 1; k >= 0; k--) {
        const int par = k & 1;
        if (k > 0)
          ACK(cudaMemcpyAsync(ad.S(ad.curbase(1 - par)), slot_of(k - 1), cur, cudaMemcpyDeviceToDevice, st));
        if (a->rev[par]) {
          ACK(cudaGraphLaunch(a->rev[par], st));
        } else {
          ad.reverse_step(coef, dcoef, nullptr, par);
        }
      }
      ACK(cudaEventRecord(a->ev_free[b], st));
      return CHNS_OK;
    }
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
  double h[kAcc];
  ACK(cudaMemcpyAsync(h, a->acc, sizeof(h), cudaMemcpyDeviceToHost, st));
  ACK(cudaStreamSynchronize(st));
  if (J) *J = h[0];
  if (g_par) ad.params(h, g_par);
  const size_t fb = 2 * (size_t)c->n * c->nr * sizeof(double);
  const cudaMemcpyKind kind = where == CHNS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (g_w) {
    c->L->to_fftw(c, ad.grad(0), c->stage);
    ACK(cudaMemcpyAsync(g_w, c->stage, fb, kind, st));
  }
  // g_c: dJ/dc_hat (binary) or dJ/dc1_hat followed by dJ/dc2_hat (ternary)
  for (int f = 1; g_c && f < A::NF; f++) {
    c->L->to_fftw(c, ad.grad(f), c->stage);
    ACK(cudaMemcpyAsync((char*)g_c + (f - 1) * fb, c->stage, fb, kind, st));
    ACK(cudaStreamSynchronize(st));  // the staging buffer is reused
  }
  ACK(cudaStreamSynchronize(st));
  return CHNS_OK;
}

}  // namespace

void chns_adj_free(chns_ctx* c) {
  chns_adj* a = c->adj;
  if (!a) return;
  for (int p = 0; p < 2; p++)
    if (a->rev[p]) cudaGraphExecDestroy(a->rev[p]);
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
  if (a->rf) cudaFree(a->rf);
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
  // the checkpoints hold the float state; a double state would not be restored
  if (c->st64) return CHNS_ERR_UNSUPPORTED;
  // the transposed passes implement the sharp cut's mask only
  if (c->p.filter != CHNS_FILTER_SHARP) return CHNS_ERR_UNSUPPORTED;
  const double dflt[3] = {1.0, 1.0, 1.0};
  const double* lw = loss_w ? loss_w : dflt;
  if (c->p.model == CHNS_MODEL_NS)
    return c->f32 ? adjoint_impl<float, AdjNS<float>>(c, nsteps, ckpt, lw, J, g_w, g_c, g_par, where)
                  : adjoint_impl<double, AdjNS<double>>(c, nsteps, ckpt, lw, J, g_w, g_c, g_par, where);
  if (c->p.model == CHNS_MODEL_BINARY)
    return c->f32 ? adjoint_impl<float, Adj<float>>(c, nsteps, ckpt, lw, J, g_w, g_c, g_par, where)
                  : adjoint_impl<double, Adj<double>>(c, nsteps, ckpt, lw, J, g_w, g_c, g_par, where);
  return c->f32 ? adjoint_impl<float, AdjT3<float>>(c, nsteps, ckpt, lw, J, g_w, g_c, g_par, where)
                : adjoint_impl<double, AdjT3<double>>(c, nsteps, ckpt, lw, J, g_w, g_c, g_par, where);
}
