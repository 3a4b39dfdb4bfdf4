// chns_adjoint.cuh -- kernels of the discrete adjoint of the binary ETD2RK step.
//
// The adjoint is the exact transpose (over the stored real and imaginary parts of
// the half spectra) of the forward step of nonlin.c / surface_tension.c /
// etd2rk.c.  Its building blocks, with X a half spectrum (n x (n/2+1) stored
// modes) and x a real n x n field:
//   ifft (fft.c:16-31)  : x = C(X)              ->  C^T(x_bar) = (w_j / n^2) dfft(x_bar)
//   dfft (fft.c:11-14)  : X = F(x)              ->  F^T(X_bar) = n^2 ifft(X_bar / w_j)
// where w_j = 2 for 0 < ky index j < n/2 and 1 for j = 0, n/2 (the Hermitian
// extension counts the interior columns twice); a complex multiplier a becomes
// conj(a), a real multiplier and the truncation mask are their own transposes.
// Spectral fields here are in the S layout (row j', column i; see chns_kernels.cuh),
// real fields are n x n row-major.
#pragma once

#include "chns_kernels.cuh"
#include "chns_adj_rows.cuh"

namespace chns {

// scalars of one adjoint evaluation
template <class R> struct AdjPar {
  int n, jt;
  double fx, fy;
  R s1, s2, lam;        // 1.5 sigma eps, 24 sigma / eps, lambda
  double ds1, ds2;      // d s1 / d sigma = 1.5 eps, d s2 / d sigma = 24 / eps
  const int* mrow;
};

template <class R> struct ModeIdx {
  int row, i, am;
  R kx, ky, ks;
  bool in;    // inside the truncation disc
  R wj;       // Hermitian weight of the column ky = row
};

template <class R>
__device__ __forceinline__ bool mode_of(const AdjPar<R>& P, size_t idx, ModeIdx<R>& m) {
  const int n = P.n;
  const size_t total = (size_t)(n / 2 + 1) * n;
  if (idx >= total) return false;
  m.row = (int)(idx / n);
  m.i = (int)(idx % n);
  const int ms = m.i <= n / 2 ? m.i : m.i - n;
  m.am = ms < 0 ? -ms : ms;
  m.kx = (R)(P.fx * (double)ms);
  m.ky = (R)(P.fy * (double)m.row);
  m.ks = radd(rmul(m.kx, m.kx), rmul(m.ky, m.ky));
  m.in = m.row <= P.jt && m.am <= P.mrow[m.row];
  m.wj = (m.row == 0 || m.row == n / 2) ? (R)1 : (R)2;
  return true;
}

template <class R> __device__ __forceinline__ cx<R> cscale(cx<R> a, R s) { return mk<R>(a.x * s, a.y * s); }
// a * (i k)  and  a * conj(i k) = a * (-i k)
template <class R> __device__ __forceinline__ cx<R> mul_ik(cx<R> a, R k) { return mk<R>(-(k * a.y), k * a.x); }
template <class R> __device__ __forceinline__ cx<R> mul_mik(cx<R> a, R k) { return mk<R>(k * a.y, -(k * a.x)); }
template <class R> __device__ __forceinline__ double rdot(cx<R> a, cx<R> b) {
  return (double)a.x * (double)b.x + (double)a.y * (double)b.y;
}

// block sums of 3 doubles written to part[3 blockIdx.x + k] (no atomics: the
// final sum in k_sum_parts has a fixed order, so the result is reproducible)
__device__ __forceinline__ void block_part3(double a0, double a1, double a2, double* part) {
  __shared__ double red[3][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_down_sync(0xffffffffu, a0, o);
    a1 += __shfl_down_sync(0xffffffffu, a1, o);
    a2 += __shfl_down_sync(0xffffffffu, a2, o);
  }
  if (lane == 0) { red[0][wid] = a0; red[1][wid] = a1; red[2][wid] = a2; }
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[threadIdx.x][w];
    part[3 * blockIdx.x + threadIdx.x] = s;
  }
}

// acc[k] += sum over nblk blocks of part[3 b + k], k = 0..2, in a fixed order (one block of 32)
__global__ void k_sum_parts(const double* __restrict__ part, int nblk, double* acc) {
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s += part[3 * b + threadIdx.x];
    acc[threadIdx.x] += s;
  }
}

// block sum of up to 3 doubles, added atomically to acc[0..2]
__device__ __forceinline__ void block_acc3(double a0, double a1, double a2, double* acc) {
  __shared__ double red[3][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_down_sync(0xffffffffu, a0, o);
    a1 += __shfl_down_sync(0xffffffffu, a1, o);
    a2 += __shfl_down_sync(0xffffffffu, a2, o);
  }
  if (lane == 0) { red[0][wid] = a0; red[1][wid] = a1; red[2][wid] = a2; }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    a0 = lane < nw ? red[0][lane] : 0.0;
    a1 = lane < nw ? red[1][lane] : 0.0;
    a2 = lane < nw ? red[2][lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a0 += __shfl_down_sync(0xffffffffu, a0, o);
      a1 += __shfl_down_sync(0xffffffffu, a1, o);
      a2 += __shfl_down_sync(0xffffffffu, a2, o);
    }
    if (lane == 0) {
      if (a0 != 0.0) atomicAdd(acc + 0, a0);
      if (a1 != 0.0) atomicAdd(acc + 1, a1);
      if (a2 != 0.0) atomicAdd(acc + 2, a2);
    }
  }
}

// The seven forward fields whose products the right-hand side forms (nonlin.c:30-48,
// 177-198, surface_tension.c:20-75), in the order of a batch of their adjoints
// (field k at xb + k ncx).
enum { FOP_U = 0, FOP_V, FOP_WX, FOP_WY, FOP_CT, FOP_CX, FOP_CY, FOP_N };

// ---------------------------------------------------------------------------
// adjoint of the spectral tail of nonlin() (nonlin.c:74-101, 232-253,
// surface_tension.c:98-111, curl.c): from N_bar, the four spectra whose F^T
// (= n^2 ifft(X / w)) gives the physical adjoints, as one batch:
//   0 A_bar = -Nw_bar, 1 B_bar = -Nc_bar, 2 Fx_bar = conj(-i ky) Nw_bar,
//   3 Fy_bar = conj(i kx) Nw_bar,
// each scaled by n^2 / w_j (the inverse transform divides by n^2).
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ void tail4_at(const AdjPar<R>& P, const ModeIdx<R>& m, cx<R> a, cx<R> b, cx<R>* out,
                                         size_t ncx, size_t idx) {
  const R sc = (R)((double)P.n * (double)P.n) / m.wj;
  out[idx] = cscale(a, -sc);
  out[ncx + idx] = cscale(b, -sc);
  out[2 * ncx + idx] = cscale(mul_ik(a, m.ky), sc);   // conj(-i ky) = i ky
  out[3 * ncx + idx] = cscale(mul_mik(a, m.kx), sc);  // conj(i kx) = -i kx
}

// the record table of one step from its segment slot (8 S-layout state fields at
// `state`, ncx complex each) and its two records, laid out as the REC kernels write
// them: c_t, u, v, wx, wy, cx, cy, mu (n x n each), then F[f(c_t)]
template <class R>
__global__ void k_adj_set_rec(RecStep<R>* t, const cx<R>* state, size_t ncx, const R* rec_us, const R* rec_un,
                              size_t nn) {
  for (int s = 0; s < 2; s++) {
    const R* b = s == 0 ? rec_us : rec_un;
    RecFields<R>& r = t->rhs[s];
    r.ct = b;
    r.u = b + nn;
    r.v = b + 2 * nn;
    r.wx = b + 3 * nn;
    r.wy = b + 4 * nn;
    r.gx = b + 5 * nn;
    r.gy = b + 6 * nn;
    r.mu = b + 7 * nn;
    r.ff = reinterpret_cast<const cx<R>*>(b + 8 * nn);
    r.cc = state + (s == 0 ? 3 : 1) * ncx;  // c_hat of u*, of u_n
  }
  for (int f = 0; f < 8; f++) t->f[f] = state + f * ncx;
}

// mu_bar_hat = T[(w_j / n^2) dfft(mu_bar)]; c_bar += s1 k^2 mu_bar_hat; the
// spectrum of F[f]'s adjoint, s2 mu_bar_hat - lambda s2 k^2 Nc_bar, scaled
// n^2 / w_j for F^T; lambda_bar and sigma_bar from the mu terms and from
// N_c = -F[B] - lambda s2 k^2 F[f] (nonlin.c:240, 251).
template <class R>
__global__ void k_adj_mu(const AdjPar<R> P, const cx<R>* __restrict__ mub_hat_raw, const RecFields<R>* rf,
                         const cx<R>* __restrict__ nc, cx<R>* __restrict__ gc, cx<R>* __restrict__ fbar_spec,
                         double* acc) {
  const cx<R>* __restrict__ Ff = rf->ff;
  const cx<R>* __restrict__ c = rf->cc;
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  double dl = 0.0, ds = 0.0;
  if (mode_of(P, idx, m)) {
    const R n2 = (R)((double)P.n * (double)P.n);
    cx<R> mb = czero<R>();
    if (m.in) mb = cscale(mub_hat_raw[idx], m.wj / n2);
    const cx<R> g = gc[idx];
    const R q = rmul(P.s1, m.ks);
    gc[idx] = mk<R>(g.x + q * mb.x, g.y + q * mb.y);
    const cx<R> a = c[idx], f = Ff[idx], nb = nc[idx];
    const R d1 = (R)(P.ds1 * (double)m.ks);
    ds = rdot(mb, mk<R>(d1 * a.x + (R)P.ds2 * f.x, d1 * a.y + (R)P.ds2 * f.y));
    const double dn = -(double)m.ks * rdot(nb, f);
    dl = (double)P.s2 * dn;
    ds += (double)P.lam * P.ds2 * dn;
    const R ql = rmul(rmul(P.lam, P.s2), m.ks);
    const cx<R> fb = mk<R>(P.s2 * mb.x - ql * nb.x, P.s2 * mb.y - ql * nb.y);
    fbar_spec[idx] = cscale(fb, n2 / m.wj);
  }
  block_acc3(0.0, dl, ds, acc);
}

// accumulation of C^T(x_bar) = (w_j / n^2) dfft(x_bar) through the multipliers
// of the forward fields into (gw, gc), for the batch of seven x_bar spectra
// (field k at xb + k ncx, order u, v, wx, wy, ct, cx, cy):
//   u = T[i ky psi], v = T[-i kx psi], psi = w / k^2; wx = T[i kx w], wy = T[i ky w];
//   ct = T[c], cx = T[i kx c], cy = T[i ky c]
template <class R>
__device__ __forceinline__ void acc7_at(const AdjPar<R>& P, const ModeIdx<R>& m, const cx<R>* xb, size_t ncx,
                                        size_t idx, cx<R>& gw, cx<R>& gc) {
  const R sc = m.wj / (R)((double)P.n * (double)P.n);
  cx<R> x[FOP_N];
#pragma unroll
  for (int k = 0; k < FOP_N; k++) x[k] = cscale(xb[k * ncx + idx], sc);
  // psi_bar = conj(i ky) u_bar + conj(-i kx) v_bar, w_bar += psi_bar / k^2
  cx<R> dw = czero<R>();
  if (m.ks > (R)1e-12) {
    const cx<R> a = mul_mik(x[FOP_U], m.ky), b = mul_mik(x[FOP_V], -m.kx);
    dw = mk<R>(rdiv(a.x + b.x, m.ks), rdiv(a.y + b.y, m.ks));
  }
  const cx<R> ax = mul_mik(x[FOP_WX], m.kx), ay = mul_mik(x[FOP_WY], m.ky);
  const cx<R> bx = mul_mik(x[FOP_CX], m.kx), by = mul_mik(x[FOP_CY], m.ky);
  gw = mk<R>(gw.x + dw.x + ax.x + ay.x, gw.y + dw.y + ax.y + ay.y);
  gc = mk<R>(gc.x + x[FOP_CT].x + bx.x + by.x, gc.y + x[FOP_CT].y + bx.y + by.y);
}

template <class R>
__global__ void k_adj_acc7(const AdjPar<R> P, const cx<R>* __restrict__ xb, cx<R>* __restrict__ gw,
                           cx<R>* __restrict__ gc, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m) || !m.in) return;
  cx<R> w = gw[idx], c = gc[idx];
  acc7_at(P, m, xb, ncx, idx, w, c);
  gw[idx] = w;
  gc[idx] = c;
}

// ---------------------------------------------------------------------------
// ETD2RK adjoint (etd2rk.c:81-135, 155-212) with parameter derivatives.
// coef [6][nr][nr] (eta_w, z1_w, z2_w, beta_c, z1_c, z2_c); dcoef [9][nr][nr]:
// d(eta_w, z1_w, z2_w)/d nu, d(beta_c, z1_c, z2_c)/d lambda, ... / d sigma.
// ---------------------------------------------------------------------------
// stage 2 (u1 = u* + z2 (N* - N)): N*_bar = z2 u1_bar (its c part kept in nbs_c, the
// transposed tail of the right-hand side at u* into `out`), N_bar = -z2 u1_bar
template <class R>
__global__ void k_adj_etd2_tail(const AdjPar<R> P, const R* __restrict__ coef, const double* __restrict__ dcoef,
                                const cx<R>* __restrict__ gw, const cx<R>* __restrict__ gc,
                                const RecStep<R>* __restrict__ rs, cx<R>* __restrict__ nbs_c,
                                cx<R>* __restrict__ nba_w, cx<R>* __restrict__ nba_c, cx<R>* __restrict__ out,
                                size_t ncx, double* acc) {
  const cx<R>* __restrict__ nw = rs->f[4];
  const cx<R>* __restrict__ nc = rs->f[5];
  const cx<R>* __restrict__ nsw = rs->f[6];
  const cx<R>* __restrict__ nsc = rs->f[7];
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  double dnu = 0.0, dl = 0.0, dsg = 0.0;
  if (mode_of(P, idx, m)) {
    const int nr = P.n / 2 + 1;
    const size_t t = (size_t)nr * nr, o = (size_t)m.row * nr + m.am;
    const R z2w = coef[2 * t + o], z2c = coef[5 * t + o];
    const cx<R> bw = gw[idx], bc = gc[idx];
    const cx<R> sw = cscale(bw, z2w), sc = cscale(bc, z2c);
    nbs_c[idx] = sc;
    nba_w[idx] = cscale(bw, -z2w);
    nba_c[idx] = cscale(bc, -z2c);
    tail4_at(P, m, sw, sc, out, ncx, idx);
    const cx<R> dw = nsw[idx] - nw[idx], dc = nsc[idx] - nc[idx];
    dnu = dcoef[2 * t + o] * rdot(bw, dw);
    dl = dcoef[5 * t + o] * rdot(bc, dc);
    dsg = dcoef[8 * t + o] * rdot(bc, dc);
  }
  block_acc3(dnu, dl, dsg, acc);
}

// C^T of the right-hand side at u* (batch xb: its seven transformed product
// adjoints) into u*_bar = (gw, gc); stage 1 (u* = e u + z1 N(u)): u_bar = e u*_bar,
// N_bar += z1 u*_bar (its c part kept in nbc); the transposed tail of the right-hand
// side at u_n into xb (each thread reads its seven entries before writing four)
template <class R>
__global__ void k_adj_acc7_etd1_tail(const AdjPar<R> P, const R* __restrict__ coef,
                                     const double* __restrict__ dcoef, cx<R>* xb, cx<R>* __restrict__ gw,
                                     cx<R>* __restrict__ gc, const RecStep<R>* __restrict__ rs,
                                     const cx<R>* __restrict__ nbw, cx<R>* __restrict__ nbc, size_t ncx,
                                     double* acc) {
  const cx<R>* __restrict__ uw = rs->f[0];
  const cx<R>* __restrict__ uc = rs->f[1];
  const cx<R>* __restrict__ nw = rs->f[4];
  const cx<R>* __restrict__ nc = rs->f[5];
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  double dnu = 0.0, dl = 0.0, dsg = 0.0;
  if (mode_of(P, idx, m)) {
    const int nr = P.n / 2 + 1;
    const size_t t = (size_t)nr * nr, o = (size_t)m.row * nr + m.am;
    const R ew = coef[0 * t + o], z1w = coef[1 * t + o], ec = coef[3 * t + o], z1c = coef[4 * t + o];
    cx<R> bw = gw[idx], bc = gc[idx];
    if (m.in) acc7_at(P, m, xb, ncx, idx, bw, bc);
    const cx<R> a = nbw[idx], b = nbc[idx];
    const cx<R> na = mk<R>(a.x + z1w * bw.x, a.y + z1w * bw.y), nb = mk<R>(b.x + z1c * bc.x, b.y + z1c * bc.y);
    nbc[idx] = nb;
    gw[idx] = cscale(bw, ew);
    gc[idx] = cscale(bc, ec);
    tail4_at(P, m, na, nb, xb, ncx, idx);
    dnu = dcoef[0 * t + o] * rdot(bw, uw[idx]) + dcoef[1 * t + o] * rdot(bw, nw[idx]);
    dl = dcoef[3 * t + o] * rdot(bc, uc[idx]) + dcoef[4 * t + o] * rdot(bc, nc[idx]);
    dsg = dcoef[6 * t + o] * rdot(bc, uc[idx]) + dcoef[7 * t + o] * rdot(bc, nc[idx]);
  }
  block_acc3(dnu, dl, dsg, acc);
}

// ---------------------------------------------------------------------------
// loss J = a_bulk E_bulk + a_grad E_grad + a_phi <|grad phi|^2>, phi = 2c - 1,
// at the final state (free_energy.c: c and its gradient NOT truncated)
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_adj_loss(const R* __restrict__ c, const R* __restrict__ cxp, const R* __restrict__ cyp,
                           R* __restrict__ cb, R* __restrict__ cxb, R* __restrict__ cyb, size_t nn, double kb,
                           double kg, double dkb, double dkg, double* part) {
  // per point: J = kb c^2 (1-c)^2 + kg (cx^2 + cy^2), kb/kg include 1/n^2;
  // per-block partials of J and of d J / d sigma through kb, kg (dkb, dkg)
  double sj = 0.0, ssg = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const double a = c[k], x = cxp[k], y = cyp[k];
    const double b = a * a * (1.0 - a) * (1.0 - a), g = x * x + y * y;
    sj += kb * b + kg * g;
    ssg += dkb * b + dkg * g;
    cb[k] = (R)(kb * 2.0 * a * (1.0 - a) * (1.0 - 2.0 * a));
    cxb[k] = (R)(kg * 2.0 * x);
    cyb[k] = (R)(kg * 2.0 * y);
  }
  block_part3(sj, 0.0, ssg, part);
}

// the untruncated c, i kx c, i ky c (free_energy.c) as one batch
template <class R>
__global__ void k_adj_loss_prep3(const AdjPar<R> P, const cx<R>* __restrict__ c, cx<R>* __restrict__ out, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  const cx<R> a = c[idx];
  out[idx] = a;
  out[ncx + idx] = mul_ik(a, m.kx);
  out[2 * ncx + idx] = mul_ik(a, m.ky);
}

// gc = (w_j/n^2)(dfft(cb) - i kx dfft(cxb) - i ky dfft(cyb)) from the batch of three; gw = 0
template <class R>
__global__ void k_adj_loss_acc3(const AdjPar<R> P, const cx<R>* __restrict__ xb, cx<R>* __restrict__ gc,
                                cx<R>* __restrict__ gw, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  const R sc = m.wj / (R)((double)P.n * (double)P.n);
  const cx<R> a = cscale(xb[idx], sc);
  const cx<R> b = mul_mik(cscale(xb[ncx + idx], sc), m.kx), d = mul_mik(cscale(xb[2 * ncx + idx], sc), m.ky);
  gc[idx] = mk<R>(a.x + b.x + d.x, a.y + b.y + d.y);
  gw[idx] = czero<R>();
}

}  // namespace chns
