// chns_adjoint.cu -- discrete adjoint of n binary ETD2RK steps (chns_adjoint).
//
// Gradient of a final-time functional J(c_T) with respect to the initial spectral
// state (omega_hat_0, c_hat_0) and to nu, lambda (the mobility M) and sigma.
// Reverse sweep with two-level checkpointing: the forward pass keeps the state
// every `ckpt` steps; each segment is recomputed forward from its checkpoint,
// keeping its states, and reversed step by step.  Reversing step n re-runs the
// forward stage kernels to get u* = stage1(u_n), N(u_n) and N(u*), then applies
// the transposed stage-2 update, the transposed right-hand side at u*, the
// transposed stage-1 update and the transposed right-hand side at u_n (kernels
// in chns_adjoint.cuh).
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

struct chns_adj {
  int cap_states;            // segment length the buffers were sized for
  void* seg;                 // segment states: cap_states x 2 S fields (+ k0 in FP32)
  double* segk0;             // cap_states x 16
  void** ckpt;               // checkpoints (host array of device pointers)
  double** ckptk0;
  int nckpt_cap;
  void* dcoef;               // [9][nr][nr] double
  double* acc;               // [4] J, dJ/dlambda, dJ/dsigma accumulators; [0] also nu in etd kernels
  double* pacc;              // [3] nu, lambda, sigma
  void* spec[16];            // S-layout scratch
  void* phys[20];            // real scratch
  size_t ncx, nn;
};

namespace {

template <class R> struct Adj {
  chns_ctx* c;
  chns_adj* a;
  AdjPar<R> P;
  cudaStream_t st;
  size_t ncx, nn;
  int blocks_s, blocks_p;

  cx<R>* S(int k) const { return (cx<R>*)a->spec[k]; }
  R* F(int k) const { return (R*)a->phys[k]; }

  // physical-field slots
  enum { PU = 0, PV, PWX, PWY, PCT, PCX, PCY, PMU, PAB, PBB, PFXB, PFYB, PFB, PUB, PVB, PWXB, PWYB, PCTB, PCXB, PCYB };
  // spectral slots
  enum { SFF = 0, SX, SY, SNW_S, SNC_S, SNW_N, SNC_N, SNBW, SNBC, SNBAW, SNBAC, SUSW, SUSC, SGW, SGC, NSPEC };

  int ifft(const cx<R>* s, R* x) { return c->L->ifft(c, s, x); }
  int dfft(const R* x, cx<R>* s) { return c->L->dfft(c, x, s); }

  // forward physical fields of the right-hand side at state (w, cc)
  void fwd_fields(const cx<R>* w, const cx<R>* cc) {
    const int ops[7] = {FOP_U, FOP_V, FOP_WX, FOP_WY, FOP_CT, FOP_CX, FOP_CY};
    const int dst[7] = {PU, PV, PWX, PWY, PCT, PCX, PCY};
    for (int k = 0; k < 7; k++) {
      k_adj_fwd_prep<R><<<blocks_s, 256, 0, st>>>(ops[k], P, w, cc, nullptr, S(SX));
      ifft(S(SX), F(dst[k]));
    }
    // F[f(c_t)] and mu (surface_tension.c:20-75)
    cudaMemcpyAsync(F(PFB), F(PCT), nn * sizeof(R), cudaMemcpyDeviceToDevice, st);
    k_adj_bulk<R><<<blocks_p, 256, 0, st>>>(F(PFB), nn);
    dfft(F(PFB), S(SFF));
    k_adj_fwd_prep<R><<<blocks_s, 256, 0, st>>>(FOP_MU, P, w, cc, S(SFF), S(SX));
    ifft(S(SX), F(PMU));
  }

  // (gw, gc) += J_N(state)^T (nbw, nbc); parameter partials into pacc
  void vjp(const cx<R>* w, const cx<R>* cc, const cx<R>* nbw, const cx<R>* nbc, cx<R>* gw, cx<R>* gc) {
    fwd_fields(w, cc);
    double* pacc = a->pacc;
    k_adj_param_nc<R><<<blocks_s, 256, 0, st>>>(P, nbc, S(SFF), pacc);
    const int tail_dst[4] = {PAB, PBB, PFXB, PFYB};
    for (int op = 0; op < 4; op++) {
      k_adj_tail<R><<<blocks_s, 256, 0, st>>>(op, P, nbw, nbc, S(SX));
      ifft(S(SX), F(tail_dst[op]));
    }
    // mu_bar -> mu_bar_hat -> c_bar (s1 k^2), f_bar
    k_adj_mubar<R><<<blocks_p, 256, 0, st>>>(F(PFXB), F(PFYB), F(PCX), F(PCY), F(PUB), nn);
    dfft(F(PUB), S(SX));
    k_adj_mu<R><<<blocks_s, 256, 0, st>>>(P, S(SX), cc, S(SFF), nbc, gc, S(SY), pacc);
    ifft(S(SY), F(PFB));
    // products
    PhysFields<R> pf{F(PU), F(PV), F(PWX), F(PWY), F(PCT), F(PCX), F(PCY), F(PMU)};
    PhysAdj<R> pa{F(PAB), F(PBB), F(PFXB), F(PFYB), F(PFB), F(PUB), F(PVB), F(PWXB), F(PWYB), F(PCTB), F(PCXB),
                  F(PCYB)};
    k_adj_products<R><<<blocks_p, 256, 0, st>>>(pf, pa, nn);
    const int ops[7] = {FOP_U, FOP_V, FOP_WX, FOP_WY, FOP_CT, FOP_CX, FOP_CY};
    const int src[7] = {PUB, PVB, PWXB, PWYB, PCTB, PCXB, PCYB};
    for (int k = 0; k < 7; k++) {
      dfft(F(src[k]), S(SX));
      k_adj_acc<R><<<blocks_s, 256, 0, st>>>(ops[k], P, S(SX), gw, gc);
    }
  }
};

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
  const size_t snap = 2 * ncx * 2 * c->rsz;
  a->ncx = ncx;
  a->nn = nn;
  if (!a->dcoef) {
    for (int k = 0; k < 16; k++)
      if (cudaMalloc(&a->spec[k], ncx * 2 * c->rsz) != cudaSuccess) return CHNS_ERR_NOMEM;
    for (int k = 0; k < 20; k++)
      if (cudaMalloc(&a->phys[k], nn * c->rsz) != cudaSuccess) return CHNS_ERR_NOMEM;
    if (cudaMalloc((void**)&a->acc, 8 * sizeof(double)) != cudaSuccess) return CHNS_ERR_NOMEM;
    a->pacc = a->acc + 4;
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
  if (seglen > a->cap_states) {
    if (a->seg) cudaFree(a->seg);
    if (a->segk0) cudaFree(a->segk0);
    if (cudaMalloc(&a->seg, snap * seglen) != cudaSuccess) return CHNS_ERR_NOMEM;
    if (cudaMalloc((void**)&a->segk0, 16 * sizeof(double) * seglen) != cudaSuccess) return CHNS_ERR_NOMEM;
    a->cap_states = seglen;
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
  const size_t bytes = (size_t)c->n * c->nr * 2 * c->rsz;
  const size_t snap = 2 * bytes;
  const R* coef = (const R*)c->coef;
  const double* dcoef = (const double*)a->dcoef;
  ACK(cudaMemsetAsync(a->acc, 0, 8 * sizeof(double), st));

  // forward sweep with checkpoints; checkpoint nseg keeps u_0 for restoring
  if ((rc = snapshot_save(c, a->ckpt[nseg], a->ckptk0[nseg]))) return rc;
  for (int n = 0; n < nsteps; n++) {
    if (n % ckpt == 0 && (rc = snapshot_save(c, a->ckpt[n / ckpt], a->ckptk0[n / ckpt]))) return rc;
    c->L->stage(c, 1);
    c->L->stage(c, 2);
  }
  // loss at the final state and its gradient (free_energy.c:3-157: c and grad c untruncated)
  cx<R>* gradw = A.S(A.SGW);
  cx<R>* gradc = A.S(A.SGC);
  {
    const cx<R>* ch = (const cx<R>*)c->state[1];
    ACK(cudaMemcpyAsync(A.S(A.SX), ch, bytes, cudaMemcpyDeviceToDevice, st));
    A.ifft(A.S(A.SX), A.F(A.PCT));
    k_spec_mul_ik<R><<<A.blocks_s, 256, 0, st>>>(A.P, ch, A.S(A.SX), 0);
    A.ifft(A.S(A.SX), A.F(A.PCX));
    k_spec_mul_ik<R><<<A.blocks_s, 256, 0, st>>>(A.P, ch, A.S(A.SX), 1);
    A.ifft(A.S(A.SX), A.F(A.PCY));
    const double inv = 1.0 / ((double)c->n * (double)c->n);
    const double kb = lw[0] * 12.0 * (p.sigma / p.epsilon) * inv;
    const double kg = (lw[1] * 0.75 * p.sigma * p.epsilon + 4.0 * lw[2]) * inv;
    const double dkb = lw[0] * 12.0 / p.epsilon * inv;
    const double dkg = lw[1] * 0.75 * p.epsilon * inv;
    k_adj_loss<R><<<A.blocks_p, 256, 0, st>>>(A.F(A.PCT), A.F(A.PCX), A.F(A.PCY), A.F(A.PUB), A.F(A.PVB),
                                              A.F(A.PWXB), A.nn, kb, kg, dkb, dkg, a->acc);
    const int srcs[3] = {A.PUB, A.PVB, A.PWXB};
    for (int op = 0; op < 3; op++) {
      A.dfft(A.F(srcs[op]), A.S(A.SX));
      k_adj_loss_acc<R><<<A.blocks_s, 256, 0, st>>>(op, A.P, A.S(A.SX), gradc);
    }
    ACK(cudaMemsetAsync(gradw, 0, bytes, st));
  }
  // reverse sweep
  char* segbase = (char*)a->seg;
  for (int s = nseg - 1; s >= 0; s--) {
    const int n0 = s * ckpt, len = (n0 + ckpt <= nsteps) ? ckpt : nsteps - n0;
    if ((rc = snapshot_load(c, a->ckpt[s], a->ckptk0[s]))) return rc;
    for (int k = 0; k < len; k++) {
      if ((rc = snapshot_save(c, segbase + (size_t)k * snap, a->segk0 + 16 * k))) return rc;
      if (k + 1 < len) {
        c->L->stage(c, 1);
        c->L->stage(c, 2);
      }
    }
    for (int k = len - 1; k >= 0; k--) {
      const cx<R>* un_w = (const cx<R>*)(segbase + (size_t)k * snap);
      const cx<R>* un_c = (const cx<R>*)(segbase + (size_t)k * snap + bytes);
      // u* = stage1(u_n) and N(u_n)
      if ((rc = snapshot_load(c, un_w, a->segk0 + 16 * k))) return rc;
      c->L->stage(c, 1);
      ACK(cudaMemcpyAsync(A.S(A.SNW_N), c->saved[0], bytes, cudaMemcpyDeviceToDevice, st));
      ACK(cudaMemcpyAsync(A.S(A.SNC_N), c->saved[1], bytes, cudaMemcpyDeviceToDevice, st));
      ACK(cudaMemcpyAsync(A.S(A.SUSW), c->state[0], bytes, cudaMemcpyDeviceToDevice, st));
      ACK(cudaMemcpyAsync(A.S(A.SUSC), c->state[1], bytes, cudaMemcpyDeviceToDevice, st));
      // N(u*): stage 1 again from u* (its state update is discarded)
      c->L->stage(c, 1);
      ACK(cudaMemcpyAsync(A.S(A.SNW_S), c->saved[0], bytes, cudaMemcpyDeviceToDevice, st));
      ACK(cudaMemcpyAsync(A.S(A.SNC_S), c->saved[1], bytes, cudaMemcpyDeviceToDevice, st));
      // stage 2 transposed: N*_bar -> (SNBW, SNBC), the N(u_n)_bar part -> (SNBAW, SNBAC)
      k_adj_etd2<R><<<A.blocks_s, 256, 0, st>>>(A.P, coef, dcoef, gradw, gradc, A.S(A.SNW_S), A.S(A.SNC_S),
                                                A.S(A.SNW_N), A.S(A.SNC_N), A.S(A.SNBW), A.S(A.SNBC),
                                                A.S(A.SNBAW), A.S(A.SNBAC), a->pacc);
      // transposed right-hand side at u*
      A.vjp(A.S(A.SUSW), A.S(A.SUSC), A.S(A.SNBW), A.S(A.SNBC), gradw, gradc);
      // stage 1 transposed
      k_adj_etd1<R><<<A.blocks_s, 256, 0, st>>>(A.P, coef, dcoef, gradw, gradc, un_w, un_c, A.S(A.SNW_N),
                                                A.S(A.SNC_N), A.S(A.SNBAW), A.S(A.SNBAC), a->pacc);
      // transposed right-hand side at u_n
      A.vjp(un_w, un_c, A.S(A.SNBAW), A.S(A.SNBAC), gradw, gradc);
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
  if (g_w) {
    c->L->to_fftw(c, gradw, c->stage);
    ACK(cudaMemcpyAsync(g_w, c->stage, fb, where == CHNS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        st));
  }
  if (g_c) {
    c->L->to_fftw(c, gradc, c->stage);
    ACK(cudaMemcpyAsync(g_c, c->stage, fb, where == CHNS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        st));
  }
  ACK(cudaStreamSynchronize(st));
  return CHNS_OK;
}

}  // namespace

void chns_adj_free(chns_ctx* c) {
  chns_adj* a = c->adj;
  if (!a) return;
  for (int k = 0; k < 16; k++)
    if (a->spec[k]) cudaFree(a->spec[k]);
  for (int k = 0; k < 20; k++)
    if (a->phys[k]) cudaFree(a->phys[k]);
  for (int k = 0; k < a->nckpt_cap; k++) {
    cudaFree(a->ckpt[k]);
    cudaFree(a->ckptk0[k]);
  }
  free(a->ckpt);
  free(a->ckptk0);
  if (a->seg) cudaFree(a->seg);
  if (a->segk0) cudaFree(a->segk0);
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
