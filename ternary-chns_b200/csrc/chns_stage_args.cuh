// chns_stage_args.cuh -- the stage kernels' arguments (Par, Bufs) of a context.
#pragma once

#include "chns_internal.h"
#include "chns_kernels.cuh"

namespace chns {

template <class R> Par<R> make_par(const chns_ctx* c) {
  Par<R> P;
  const chns_params& p = c->p;
  P.n = c->n;
  P.jt = c->jt;
  P.fx = c->fx;
  P.fy = c->fy;
  P.scale = (R)(1.0 / (double)(p.nx * p.ny));
  P.st15 = (R)(1.5 * p.sigma * p.epsilon);
  P.st24 = (R)(24.0 * (p.sigma / p.epsilon));
  P.lam = (R)p.lambda;
  const double g1 = c->gamma[0], g2 = c->gamma[1], g3 = c->gamma[2];
  if (p.model == CHNS_MODEL_TERNARY) {
    P.mu1 = (R)(0.75 * g1 * p.epsilon);
    P.mu2 = (R)(0.75 * g2 * p.epsilon);
    P.lg1 = (R)(p.lambda / g1);
    P.lg2 = (R)(p.lambda / g2);
    P.w11 = (R)(1.0 + (g3 / g1));
    P.w12 = (R)(g3 / g2);
    P.w21 = (R)(g3 / g1);
    P.w22 = (R)(1.0 + (g3 / g2));
    P.g1 = (R)g1;
    P.g2 = (R)g2;
    P.g3 = (R)g3;
    P.g1i = (R)(1.0 / g1);
    P.g2i = (R)(1.0 / g2);
    P.g3i = (R)(1.0 / g3);
    P.six_lam = (R)(6.0 * p.xlambda);
    P.fac_mu = (R)(2.0 * c->del / p.epsilon);
  } else {
    P.mu1 = P.mu2 = P.lg1 = P.lg2 = P.w11 = P.w12 = P.w21 = P.w22 = (R)0;
    P.g1 = P.g2 = P.g3 = P.g1i = P.g2i = P.g3i = P.six_lam = P.fac_mu = (R)0;
  }
  P.force_j = c->force_j;
  P.force_hat = (R)c->force_hat;
  for (int k = 0; k < 6; k++) P.k0coef[k] = c->k0coef[k];
  P.mrow = c->mrow;
  P.filt = (const R*)c->filt;
  P.coef = (const R*)c->coef;
  P.tw = (const cx<R>*)c->tw;
  P.k0 = c->k0;
  P.err = c->tma_err;
  return P;
}

template <class R> Bufs<R> make_bufs(const chns_ctx* c) {
  Bufs<R> B;
  B.w = (cx<R>*)c->state[0];
  B.c1 = (cx<R>*)c->state[1];
  B.c2 = (cx<R>*)c->state[2];
  B.sw = (cx<R>*)c->saved[0];
  B.s1 = (cx<R>*)c->saved[1];
  B.s2 = (cx<R>*)c->saved[2];
  B.xw = (cx<R>*)c->nstar[0];
  B.x1 = (cx<R>*)c->nstar[1];
  B.x2 = (cx<R>*)c->nstar[2];
  B.nw = (cx<R>*)c->nw;
  for (int f = 0; f < 3; f++) B.lo[f] = c->st64 ? (cx<R>*)c->statelo[f] : nullptr;
  B.gr = (cx<R>*)c->gradr;
  B.rec = (R*)c->rec;
  for (int k = 0; k < NG; k++) B.g[k] = (cx<R>*)c->g[k];
  for (int k = 0; k < NH; k++) B.h[k] = (cx<R>*)c->h[k];
  return B;
}

}  // namespace chns
