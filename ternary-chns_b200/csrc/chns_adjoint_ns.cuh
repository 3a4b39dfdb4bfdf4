// chns_adjoint_ns.cuh -- kernels of the discrete adjoint of the pure Navier-Stokes
// ETD2RK step (nonlin.c:30-101 without a phase field, etd2rk.c:81-99,155-174).
//
// The forward right-hand side is N_w = -F[u wx + v wy] (+ the constant forcing),
// with u = T[i ky psi], v = T[-i kx psi], psi = w / k^2, wx = T[i kx w],
// wy = T[i ky w] inverse-transformed (T the truncation mask).  Its transpose uses
// the conventions of chns_adjoint.cuh: C^T(x_bar) = (w_j / n^2) dfft(x_bar) for
// x = ifft(X), F^T(X_bar) = n^2 ifft(X_bar / w_j) for X = dfft(x), a complex
// multiplier becomes its conjugate.  The loss of the final state is
//   J = a_ke <|u|^2 / 2> + a_ens <w_t^2 / 2>,   w_t = ifft(T[w]),
// the first term kinetic_energy.c:17-21,43-49,89 (the truncated velocity).
#pragma once

#include "chns_adjoint.cuh"

namespace chns {

// the four truncated spectra u, v, wx, wy of the right-hand side as one batch
template <class R>
__global__ void k_adjns_prep4(const AdjPar<R> P, const cx<R>* __restrict__ w, cx<R>* __restrict__ out, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  cx<R> r[4] = {czero<R>(), czero<R>(), czero<R>(), czero<R>()};
  if (m.in) {
    const cx<R> a = w[idx];
    cx<R> psi = czero<R>();
    if (m.ks > (R)1e-12) psi = mk<R>(rdiv(a.x, m.ks), rdiv(a.y, m.ks));
    r[0] = mul_ik(psi, m.ky);
    r[1] = mul_ik(psi, -m.kx);
    r[2] = mul_ik(a, m.kx);
    r[3] = mul_ik(a, m.ky);
  }
#pragma unroll
  for (int k = 0; k < 4; k++) out[k * ncx + idx] = r[k];
}

// A_bar = F^T(-N_bar): the spectrum -(n^2 / w_j) N_bar, whose inverse transform is A_bar
template <class R>
__global__ void k_adjns_tail1(const AdjPar<R> P, const cx<R>* __restrict__ nw, cx<R>* __restrict__ out) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  out[idx] = cscale(nw[idx], -(R)((double)P.n * (double)P.n) / m.wj);
}

// u_bar = A_bar wx, v_bar = A_bar wy, wx_bar = A_bar u, wy_bar = A_bar v
template <class R>
__global__ void k_adjns_products(const R* __restrict__ u, const R* __restrict__ v, const R* __restrict__ wx,
                                 const R* __restrict__ wy, const R* __restrict__ ab, R* __restrict__ ub,
                                 R* __restrict__ vb, R* __restrict__ wxb, R* __restrict__ wyb, size_t nn) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const R a = ab[k];
    ub[k] = a * wx[k];
    vb[k] = a * wy[k];
    wxb[k] = a * u[k];
    wyb[k] = a * v[k];
  }
}

// gw += C^T of the batch (u_bar, v_bar, wx_bar, wy_bar) through the multipliers of u, v, wx, wy
template <class R>
__global__ void k_adjns_acc4(const AdjPar<R> P, const cx<R>* __restrict__ xb, cx<R>* __restrict__ gw, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m) || !m.in) return;
  const R sc = m.wj / (R)((double)P.n * (double)P.n);
  cx<R> x[4];
#pragma unroll
  for (int k = 0; k < 4; k++) x[k] = cscale(xb[k * ncx + idx], sc);
  cx<R> dw = czero<R>();
  if (m.ks > (R)1e-12) {  // psi_bar = conj(i ky) u_bar + conj(-i kx) v_bar, w_bar += psi_bar / k^2
    const cx<R> a = mul_mik(x[0], m.ky), b = mul_mik(x[1], -m.kx);
    dw = mk<R>(rdiv(a.x + b.x, m.ks), rdiv(a.y + b.y, m.ks));
  }
  const cx<R> ax = mul_mik(x[2], m.kx), ay = mul_mik(x[3], m.ky);
  const cx<R> o = gw[idx];
  gw[idx] = mk<R>(o.x + dw.x + ax.x + ay.x, o.y + dw.y + ax.y + ay.y);
}

// stage 2 transposed (u1 = u* + z2 (N* - N)): N*_bar = z2 u1_bar, N_bar = -z2 u1_bar,
// with dJ/dnu through z2 into acc[0]
template <class R>
__global__ void k_adjns_etd2(const AdjPar<R> P, const R* __restrict__ coef, const double* __restrict__ dcoef,
                             const cx<R>* __restrict__ gw, const cx<R>* __restrict__ nsw, const cx<R>* __restrict__ nw,
                             cx<R>* __restrict__ nbs, cx<R>* __restrict__ nba, double* acc) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  double dnu = 0.0;
  if (mode_of(P, idx, m)) {
    const int nr = P.n / 2 + 1;
    const size_t t = (size_t)nr * nr, o = (size_t)m.row * nr + m.am;
    const R z2 = coef[2 * t + o];
    const cx<R> b = gw[idx];
    nbs[idx] = cscale(b, z2);
    nba[idx] = cscale(b, -z2);
    dnu = dcoef[2 * t + o] * rdot(b, nsw[idx] - nw[idx]);
  }
  block_acc3(dnu, 0.0, 0.0, acc);
}

// stage 1 transposed (u* = e u + z1 N(u)): u_bar = e u*_bar, N_bar += z1 u*_bar,
// with dJ/dnu through e and z1 into acc[0]
template <class R>
__global__ void k_adjns_etd1(const AdjPar<R> P, const R* __restrict__ coef, const double* __restrict__ dcoef,
                             cx<R>* __restrict__ gw, const cx<R>* __restrict__ uw, const cx<R>* __restrict__ nw,
                             cx<R>* __restrict__ nbw, double* acc) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  double dnu = 0.0;
  if (mode_of(P, idx, m)) {
    const int nr = P.n / 2 + 1;
    const size_t t = (size_t)nr * nr, o = (size_t)m.row * nr + m.am;
    const R e = coef[o], z1 = coef[t + o];
    const cx<R> b = gw[idx], a = nbw[idx];
    nbw[idx] = mk<R>(a.x + z1 * b.x, a.y + z1 * b.y);
    gw[idx] = cscale(b, e);
    dnu = dcoef[o] * rdot(b, uw[idx]) + dcoef[t + o] * rdot(b, nw[idx]);
  }
  block_acc3(dnu, 0.0, 0.0, acc);
}

// the truncated u, v and w_t of the loss as one batch
template <class R>
__global__ void k_adjns_loss_prep3(const AdjPar<R> P, const cx<R>* __restrict__ w, cx<R>* __restrict__ out,
                                   size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  cx<R> r[3] = {czero<R>(), czero<R>(), czero<R>()};
  if (m.in) {
    const cx<R> a = w[idx];
    cx<R> psi = czero<R>();
    if (m.ks > (R)1e-12) psi = mk<R>(rdiv(a.x, m.ks), rdiv(a.y, m.ks));
    r[0] = mul_ik(psi, m.ky);
    r[1] = mul_ik(psi, -m.kx);
    r[2] = a;
  }
#pragma unroll
  for (int k = 0; k < 3; k++) out[k * ncx + idx] = r[k];
}

// per point J = ke (u^2 + v^2) / 2 + kz w_t^2 / 2 (ke, kz include 1/n^2), its
// gradient (u_bar, v_bar, wt_bar), and per-block partials of J
template <class R>
__global__ void k_adjns_loss(const R* __restrict__ u, const R* __restrict__ v, const R* __restrict__ wt,
                             R* __restrict__ ub, R* __restrict__ vb, R* __restrict__ wtb, size_t nn, double ke,
                             double kz, double* part) {
  double sj = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const double a = u[k], b = v[k], c = wt[k];
    sj += ke * 0.5 * (a * a + b * b) + kz * 0.5 * c * c;
    ub[k] = (R)(ke * a);
    vb[k] = (R)(ke * b);
    wtb[k] = (R)(kz * c);
  }
  block_part3(sj, 0.0, 0.0, part);
}

// gw = C^T of the loss batch (u_bar, v_bar, wt_bar) through the multipliers of
// u, v and w_t (every mode written: zero outside the truncation disc)
template <class R>
__global__ void k_adjns_loss_acc3(const AdjPar<R> P, const cx<R>* __restrict__ xb, cx<R>* __restrict__ gw,
                                  size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  cx<R> g = czero<R>();
  if (m.in) {
    const R sc = m.wj / (R)((double)P.n * (double)P.n);
    const cx<R> x0 = cscale(xb[idx], sc), x1 = cscale(xb[ncx + idx], sc), x2 = cscale(xb[2 * ncx + idx], sc);
    g = x2;
    if (m.ks > (R)1e-12) {
      const cx<R> a = mul_mik(x0, m.ky), b = mul_mik(x1, -m.kx);
      g = mk<R>(g.x + rdiv(a.x + b.x, m.ks), g.y + rdiv(a.y + b.y, m.ks));
    }
  }
  gw[idx] = g;
}

}  // namespace chns
