// chns_adjoint_t.cuh -- kernels of the discrete adjoint of the ternary ETD2RK step.
//
// The ternary right-hand side (nonlin.c:255-377, chem_potential.c:12-94,
// surface_tension.c:112-227) at a state (w, c1, c2):
//   u, v, wx, wy, c_i, dx c_i, dy c_i   truncated fields in physical space
//   muF_i(c1, c2)                       bulk potential (chem_potential.c:53-67)
//   mu_i = T[F[muF_i] + 0.75 g_i eps k^2 c_i]
//   M1 = w11 mu1 + w12 mu2, M2 = w21 mu1 + w22 mu2   (surface_tension.c:148-149, 199-200)
//   N_w  = -F[u wx + v wy] + curl F[(c1x M1 + c2x M2, c1y M1 + c2y M2)]
//   N_ci = -F[u ci_x + v ci_y] - (lambda / g_i) k^2 F[muF_i]
// Its transpose uses the same building blocks as the binary adjoint
// (chns_adjoint.cuh): C^T = (w_j/n^2) dfft, F^T = n^2 ifft( / w_j), conjugated
// complex multipliers.  Batches: the ten forward fields (and their adjoints) in
// the order u, v, wx, wy, c1, c1x, c1y, c2, c2x, c2y.
#pragma once

#include "chns_adjoint.cuh"

namespace chns {

enum { T_U = 0, T_V, T_WX, T_WY, T_C1, T_C1X, T_C1Y, T_C2, T_C2X, T_C2Y, T_N };

template <class R> struct AdjParT : AdjPar<R> {
  R g1, g2, g3;          // gamma_i
  R kk;                  // 2 Delta / eps
  R xl6;                 // 6 Xlambda
  R mu1c, mu2c;          // 0.75 gamma_i eps
  R lg1, lg2;            // lambda / gamma_i
  R w11, w12, w21, w22;  // surface-tension weights
};

// block sums of N doubles added atomically to acc[0..N-1]
template <int NV> __device__ __forceinline__ void block_accn(double (&v)[NV], double* acc) {
  __shared__ double red[NV][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) red[k][wid] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[threadIdx.x][w];
    if (s != 0.0) atomicAdd(acc + threadIdx.x, s);
  }
}

// per-block sums of N doubles in part[N blockIdx.x + k] (summed in a fixed order by k_sum_partsn)
template <int NV> __device__ __forceinline__ void block_partn(double (&v)[NV], double* part) {
  __shared__ double red[NV][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; k++) red[k][wid] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[threadIdx.x][w];
    part[NV * blockIdx.x + threadIdx.x] = s;
  }
}

template <int NV> __global__ void k_sum_partsn(const double* __restrict__ part, int nblk, double* acc) {
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s += part[NV * b + threadIdx.x];
    acc[threadIdx.x] += s;
  }
}

// ---------------------------------------------------------------------------
// forward fields
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_adj3_fwd_prep(const AdjParT<R> P, const cx<R>* __restrict__ w, const cx<R>* __restrict__ c1,
                                const cx<R>* __restrict__ c2, cx<R>* __restrict__ out, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  cx<R> r[T_N];
#pragma unroll
  for (int k = 0; k < T_N; k++) r[k] = czero<R>();
  if (m.in) {
    const cx<R> a = w[idx], b = c1[idx], d = c2[idx];
    cx<R> psi = czero<R>();
    if (m.ks > (R)1e-12) psi = mk<R>(rdiv(a.x, m.ks), rdiv(a.y, m.ks));
    r[T_U] = mul_ik(psi, m.ky);
    r[T_V] = mul_ik(psi, -m.kx);
    r[T_WX] = mul_ik(a, m.kx);
    r[T_WY] = mul_ik(a, m.ky);
    r[T_C1] = b;
    r[T_C1X] = mul_ik(b, m.kx);
    r[T_C1Y] = mul_ik(b, m.ky);
    r[T_C2] = d;
    r[T_C2X] = mul_ik(d, m.kx);
    r[T_C2Y] = mul_ik(d, m.ky);
  }
#pragma unroll
  for (int k = 0; k < T_N; k++) out[k * ncx + idx] = r[k];
}

// the ternary bulk potential at one point (chem_potential.c:53-67): muF1, muF2 and
// the intermediate G_k, fc_k used by the transpose
template <class R> struct TernPot {
  R G1, G2, G3, f1, f2, f3, mf1, mf2;
};
template <class R> __device__ __forceinline__ TernPot<R> tern_pot(const AdjParT<R>& P, R c1, R c2) {
  TernPot<R> o;
  const R c3 = (R)1 - c1 - c2;
  const R p = c1 * c2 * c3;
  o.f1 = c1 * ((R)1 - c1) * ((R)1 - (R)2 * c1);
  o.f2 = c2 * ((R)1 - c2) * ((R)1 - (R)2 * c2);
  o.f3 = c3 * ((R)1 - c3) * ((R)1 - (R)2 * c3);
  o.G1 = P.g1 * o.f1 + P.xl6 * p * c2 * c3;
  o.G2 = P.g2 * o.f2 + P.xl6 * p * c1 * c3;
  o.G3 = P.g3 * o.f3 + P.xl6 * p * c1 * c2;
  o.mf1 = ((o.G1 - o.G2) / P.g2 + (o.G1 - o.G3) / P.g3) * P.kk;
  o.mf2 = ((o.G2 - o.G1) / P.g1 + (o.G2 - o.G3) / P.g3) * P.kk;
  return o;
}

template <class R>
__global__ void k_adj3_bulk(const AdjParT<R> P, const R* __restrict__ c1, const R* __restrict__ c2,
                            R* __restrict__ mf, size_t nn) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const TernPot<R> t = tern_pot(P, c1[k], c2[k]);
    mf[k] = t.mf1;
    mf[nn + k] = t.mf2;
  }
}

// mu_hat_i = T[F[muF_i] + 0.75 g_i eps k^2 c_i]  (surface_tension.c:116-128), batch of two
template <class R>
__global__ void k_adj3_mu_prep(const AdjParT<R> P, const cx<R>* __restrict__ c1, const cx<R>* __restrict__ c2,
                               const cx<R>* __restrict__ ff, cx<R>* __restrict__ out, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  cx<R> r1 = czero<R>(), r2 = czero<R>();
  if (m.in) {
    const R q1 = P.mu1c * m.ks, q2 = P.mu2c * m.ks;
    const cx<R> a = c1[idx], b = c2[idx], f1 = ff[idx], f2 = ff[ncx + idx];
    r1 = mk<R>(f1.x + q1 * a.x, f1.y + q1 * a.y);
    r2 = mk<R>(f2.x + q2 * b.x, f2.y + q2 * b.y);
  }
  out[idx] = r1;
  out[ncx + idx] = r2;
}

// ---------------------------------------------------------------------------
// transpose of the right-hand side
// ---------------------------------------------------------------------------
// N_bar -> the five spectra whose F^T are A_bar, B1_bar, B2_bar, Fx_bar, Fy_bar
template <class R>
__global__ void k_adj3_tail(const AdjParT<R> P, const cx<R>* __restrict__ nw, const cx<R>* __restrict__ n1,
                            const cx<R>* __restrict__ n2, cx<R>* __restrict__ out, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  const R sc = (R)((double)P.n * (double)P.n) / m.wj;
  const cx<R> a = nw[idx];
  out[idx] = cscale(a, -sc);
  out[ncx + idx] = cscale(n1[idx], -sc);
  out[2 * ncx + idx] = cscale(n2[idx], -sc);
  out[3 * ncx + idx] = cscale(mul_ik(a, m.ky), sc);   // conj(-i ky) = i ky
  out[4 * ncx + idx] = cscale(mul_mik(a, m.kx), sc);  // conj(i kx) = -i kx
}

template <class R> struct PhysT {
  const R *u, *v, *wx, *wy, *c1x, *c1y, *c2x, *c2y, *mu1, *mu2;
};
template <class R> struct AdjT5 {
  const R *ab, *b1b, *b2b, *fxb, *fyb;
};

// products transposed: the batch of physical adjoints (positions other than c1,
// c2), mu1_bar, mu2_bar, and the sums for the weights w_ij (acc[0..3])
template <class R>
__global__ void k_adj3_products(const AdjParT<R> P, const PhysT<R> F, const AdjT5<R> A, R* __restrict__ xb,
                                R* __restrict__ mub, size_t nn, double* acc) {
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const R ab = A.ab[k], b1 = A.b1b[k], b2 = A.b2b[k], fx = A.fxb[k], fy = A.fyb[k];
    const R u = F.u[k], v = F.v[k], c1x = F.c1x[k], c1y = F.c1y[k], c2x = F.c2x[k], c2y = F.c2y[k];
    const R mu1 = F.mu1[k], mu2 = F.mu2[k];
    const R m1 = P.w11 * mu1 + P.w12 * mu2, m2 = P.w21 * mu1 + P.w22 * mu2;
    xb[T_U * nn + k] = ab * F.wx[k] + b1 * c1x + b2 * c2x;
    xb[T_V * nn + k] = ab * F.wy[k] + b1 * c1y + b2 * c2y;
    xb[T_WX * nn + k] = ab * u;
    xb[T_WY * nn + k] = ab * v;
    xb[T_C1X * nn + k] = b1 * u + fx * m1;
    xb[T_C1Y * nn + k] = b1 * v + fy * m1;
    xb[T_C2X * nn + k] = b2 * u + fx * m2;
    xb[T_C2Y * nn + k] = b2 * v + fy * m2;
    const R m1b = fx * c1x + fy * c1y, m2b = fx * c2x + fy * c2y;
    mub[k] = P.w11 * m1b + P.w21 * m2b;
    mub[nn + k] = P.w12 * m1b + P.w22 * m2b;
    s[0] += (double)m1b * (double)mu1;
    s[1] += (double)m1b * (double)mu2;
    s[2] += (double)m2b * (double)mu1;
    s[3] += (double)m2b * (double)mu2;
  }
  block_accn<4>(s, acc);
}

// mu_bar_hat_i = T[(w_j/n^2) dfft(mu_bar_i)]; c_i_bar += 0.75 g_i eps k^2 mu_bar_hat_i;
// the spectra of F[muF_i]'s adjoints, mu_bar_hat_i - (lambda/g_i) k^2 N_ci_bar, scaled
// n^2 / w_j for F^T; sums (acc[0..3]): <mu_bar_hat_i, k^2 c_i>, <N_ci_bar, -k^2 F[muF_i]>
template <class R>
__global__ void k_adj3_mu(const AdjParT<R> P, const cx<R>* __restrict__ raw, const cx<R>* __restrict__ c1,
                          const cx<R>* __restrict__ c2, const cx<R>* __restrict__ ff, const cx<R>* __restrict__ n1,
                          const cx<R>* __restrict__ n2, cx<R>* __restrict__ g1, cx<R>* __restrict__ g2,
                          cx<R>* __restrict__ fbar, size_t ncx, double* acc) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  if (mode_of(P, idx, m)) {
    const R n2s = (R)((double)P.n * (double)P.n);
    cx<R> mb1 = czero<R>(), mb2 = czero<R>();
    if (m.in) {
      mb1 = cscale(raw[idx], m.wj / n2s);
      mb2 = cscale(raw[ncx + idx], m.wj / n2s);
    }
    const R q1 = P.mu1c * m.ks, q2 = P.mu2c * m.ks;
    const cx<R> a = g1[idx], b = g2[idx];
    g1[idx] = mk<R>(a.x + q1 * mb1.x, a.y + q1 * mb1.y);
    g2[idx] = mk<R>(b.x + q2 * mb2.x, b.y + q2 * mb2.y);
    const cx<R> x1 = c1[idx], x2 = c2[idx], f1 = ff[idx], f2 = ff[ncx + idx], nb1 = n1[idx], nb2 = n2[idx];
    s[0] = (double)m.ks * rdot(mb1, x1);
    s[1] = (double)m.ks * rdot(mb2, x2);
    s[2] = -(double)m.ks * rdot(nb1, f1);
    s[3] = -(double)m.ks * rdot(nb2, f2);
    const R l1 = P.lg1 * m.ks, l2 = P.lg2 * m.ks, sc = n2s / m.wj;
    fbar[idx] = cscale(mk<R>(mb1.x - l1 * nb1.x, mb1.y - l1 * nb1.y), sc);
    fbar[ncx + idx] = cscale(mk<R>(mb2.x - l2 * nb2.x, mb2.y - l2 * nb2.y), sc);
  }
  block_accn<4>(s, acc);
}

// the bulk potential transposed: c1_bar, c2_bar (batch positions T_C1, T_C2) from
// muF1_bar, muF2_bar; sums (acc[0..6]): dK, G_k's gamma_k fc_k terms (3), the
// 1/g_1, 1/g_2, 1/g_3 coefficients (3)
template <class R>
__global__ void k_adj3_bulk_bar(const AdjParT<R> P, const R* __restrict__ c1, const R* __restrict__ c2,
                                const R* __restrict__ mfb, R* __restrict__ xb, size_t nn, double* acc) {
  double s[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const R i1 = (R)1 / P.g1, i2 = (R)1 / P.g2, i3 = (R)1 / P.g3;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const R a = c1[k], b = c2[k], e = (R)1 - a - b;
    const R m1 = mfb[k], m2 = mfb[nn + k];
    const TernPot<R> t = tern_pot(P, a, b);
    // G_k adjoints: muF1 = K((1/g2 + 1/g3) G1 - G2/g2 - G3/g3), muF2 = K((1/g1 + 1/g3) G2 - G1/g1 - G3/g3)
    const R gb1 = P.kk * ((i2 + i3) * m1 - i1 * m2);
    const R gb2 = P.kk * (-i2 * m1 + (i1 + i3) * m2);
    const R gb3 = P.kk * (-i3 * m1 - i3 * m2);
    // dG/dc with c3 = 1 - c1 - c2; f' = 1 - 6c + 6c^2;  q1 = c1 c2^2 c3^2, q2 = c1^2 c2 c3^2, q3 = c1^2 c2^2 c3
    const R fp1 = (R)1 - (R)6 * a + (R)6 * a * a, fp2 = (R)1 - (R)6 * b + (R)6 * b * b;
    const R fp3 = (R)1 - (R)6 * e + (R)6 * e * e;
    const R dq1a = b * b * e * (e - (R)2 * a), dq1b = (R)2 * a * b * e * (e - b);
    const R dq2a = (R)2 * a * b * e * (e - a), dq2b = a * a * e * (e - (R)2 * b);
    const R dq3a = a * b * b * ((R)2 * e - a), dq3b = a * a * b * ((R)2 * e - b);
    const R dG1a = P.g1 * fp1 + P.xl6 * dq1a, dG1b = P.xl6 * dq1b;
    const R dG2a = P.xl6 * dq2a, dG2b = P.g2 * fp2 + P.xl6 * dq2b;
    const R dG3a = -P.g3 * fp3 + P.xl6 * dq3a, dG3b = -P.g3 * fp3 + P.xl6 * dq3b;
    xb[T_C1 * nn + k] = gb1 * dG1a + gb2 * dG2a + gb3 * dG3a;
    xb[T_C2 * nn + k] = gb1 * dG1b + gb2 * dG2b + gb3 * dG3b;
    s[0] += ((double)m1 * (double)t.mf1 + (double)m2 * (double)t.mf2) / (double)P.kk;
    s[1] += (double)gb1 * (double)t.f1;
    s[2] += (double)gb2 * (double)t.f2;
    s[3] += (double)gb3 * (double)t.f3;
    s[4] += (double)m2 * (double)P.kk * (double)(t.G2 - t.G1);
    s[5] += (double)m1 * (double)P.kk * (double)(t.G1 - t.G2);
    s[6] += (double)P.kk * ((double)m1 * (double)(t.G1 - t.G3) + (double)m2 * (double)(t.G2 - t.G3));
  }
  block_accn<7>(s, acc);
}

// C^T of the ten forward fields into (gw, gc1, gc2)
template <class R>
__global__ void k_adj3_acc(const AdjParT<R> P, const cx<R>* __restrict__ xb, cx<R>* __restrict__ gw,
                           cx<R>* __restrict__ g1, cx<R>* __restrict__ g2, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m) || !m.in) return;
  const R sc = m.wj / (R)((double)P.n * (double)P.n);
  cx<R> x[T_N];
#pragma unroll
  for (int k = 0; k < T_N; k++) x[k] = cscale(xb[k * ncx + idx], sc);
  cx<R> dw = czero<R>();
  if (m.ks > (R)1e-12) {
    const cx<R> a = mul_mik(x[T_U], m.ky), b = mul_mik(x[T_V], -m.kx);
    dw = mk<R>(rdiv(a.x + b.x, m.ks), rdiv(a.y + b.y, m.ks));
  }
  const cx<R> ax = mul_mik(x[T_WX], m.kx), ay = mul_mik(x[T_WY], m.ky);
  const cx<R> p1 = mul_mik(x[T_C1X], m.kx), q1 = mul_mik(x[T_C1Y], m.ky);
  const cx<R> p2 = mul_mik(x[T_C2X], m.kx), q2 = mul_mik(x[T_C2Y], m.ky);
  const cx<R> ow = gw[idx], o1 = g1[idx], o2 = g2[idx];
  gw[idx] = mk<R>(ow.x + dw.x + ax.x + ay.x, ow.y + dw.y + ax.y + ay.y);
  g1[idx] = mk<R>(o1.x + x[T_C1].x + p1.x + q1.x, o1.y + x[T_C1].y + p1.y + q1.y);
  g2[idx] = mk<R>(o2.x + x[T_C2].x + p2.x + q2.x, o2.y + x[T_C2].y + p2.y + q2.y);
}

// ---------------------------------------------------------------------------
// ETD2RK transposed for (w, c1, c2): coef [6][nr][nr]; dcoef [6][nr][nr] =
// d(eta_w, z1_w, z2_w)/d nu, d(beta_c, z1_c, z2_c)/d lambda.  acc[0] nu, acc[1] lambda.
// ---------------------------------------------------------------------------
template <class R> struct Fields3 {
  cx<R>* f[3];
};
template <class R> struct CFields3 {
  const cx<R>* f[3];
};

template <class R>
__global__ void k_adj3_etd2(const AdjParT<R> P, const R* __restrict__ coef, const double* __restrict__ dcoef,
                            const CFields3<R> g, const CFields3<R> nst, const CFields3<R> nn_, Fields3<R> nbs,
                            Fields3<R> nba, double* acc) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  double s[2] = {0.0, 0.0};
  if (mode_of(P, idx, m)) {
    const int nr = P.n / 2 + 1;
    const size_t t = (size_t)nr * nr, o = (size_t)m.row * nr + m.am;
#pragma unroll
    for (int f = 0; f < 3; f++) {
      const R z2 = coef[(f == 0 ? 2 : 5) * t + o];
      const cx<R> b = g.f[f][idx];
      nbs.f[f][idx] = cscale(b, z2);
      nba.f[f][idx] = cscale(b, -z2);
      const cx<R> d = nst.f[f][idx] - nn_.f[f][idx];
      s[f == 0 ? 0 : 1] += dcoef[(f == 0 ? 2 : 5) * t + o] * rdot(b, d);
    }
  }
  block_accn<2>(s, acc);
}

template <class R>
__global__ void k_adj3_etd1(const AdjParT<R> P, const R* __restrict__ coef, const double* __restrict__ dcoef,
                            Fields3<R> g, const CFields3<R> u, const CFields3<R> nn_, Fields3<R> nb, double* acc) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  double s[2] = {0.0, 0.0};
  if (mode_of(P, idx, m)) {
    const int nr = P.n / 2 + 1;
    const size_t t = (size_t)nr * nr, o = (size_t)m.row * nr + m.am;
#pragma unroll
    for (int f = 0; f < 3; f++) {
      const int b0 = f == 0 ? 0 : 3;
      const R e = coef[b0 * t + o], z1 = coef[(b0 + 1) * t + o];
      const cx<R> b = g.f[f][idx], a = nb.f[f][idx];
      nb.f[f][idx] = mk<R>(a.x + z1 * b.x, a.y + z1 * b.y);
      g.f[f][idx] = cscale(b, e);
      s[f == 0 ? 0 : 1] += dcoef[b0 * t + o] * rdot(b, u.f[f][idx]) + dcoef[(b0 + 1) * t + o] * rdot(b, nn_.f[f][idx]);
    }
  }
  block_accn<2>(s, acc);
}

// ---------------------------------------------------------------------------
// loss (free_energy.c ternary: c_i and their gradients untruncated):
//   J = a0 (6/eps) <g1 c1^2(1-c1)^2 + g2 c2^2(1-c2)^2 + g3 c3^2 (c1+c2)^2>
//     + a1 0.375 eps <g1 |grad c1|^2 + g2 |grad c2|^2 + g3 |grad c1 + grad c2|^2>
//     + a2 <|grad c1|^2 + |grad c2|^2>
// ---------------------------------------------------------------------------
template <class R>
__global__ void k_adj3_loss_prep(const AdjParT<R> P, const cx<R>* __restrict__ c1, const cx<R>* __restrict__ c2,
                                 cx<R>* __restrict__ out, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  const cx<R> a = c1[idx], b = c2[idx];
  out[idx] = a;
  out[ncx + idx] = mul_ik(a, m.kx);
  out[2 * ncx + idx] = mul_ik(a, m.ky);
  out[3 * ncx + idx] = b;
  out[4 * ncx + idx] = mul_ik(b, m.kx);
  out[5 * ncx + idx] = mul_ik(b, m.ky);
}

// phys: c1, c1x, c1y, c2, c2x, c2y; adjoints written in the same order; per-block
// partials of J and of dJ/dg1, dJ/dg2, dJ/dg3.  kb = a0 (6/eps)/n^2, kg = a1 0.375 eps/n^2,
// kp = a2 / n^2
template <class R>
__global__ void k_adj3_loss(const AdjParT<R> P, const R* __restrict__ ph, R* __restrict__ adj, size_t nn,
                            double kb, double kg, double kp, double* part) {
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  const double g1 = P.g1, g2 = P.g2, g3 = P.g3;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const double a = ph[k], ax = ph[nn + k], ay = ph[2 * nn + k];
    const double b = ph[3 * nn + k], bx = ph[4 * nn + k], by = ph[5 * nn + k];
    const double e = 1.0 - a - b;
    const double ba = a * a * (1.0 - a) * (1.0 - a), bb = b * b * (1.0 - b) * (1.0 - b);
    const double be = e * e * (a + b) * (a + b);
    const double ga = ax * ax + ay * ay, gb = bx * bx + by * by;
    const double sx = ax + bx, sy = ay + by, gs = sx * sx + sy * sy;
    s[0] += kb * (g1 * ba + g2 * bb + g3 * be) + kg * (g1 * ga + g2 * gb + g3 * gs) + kp * (ga + gb);
    s[1] += kb * ba + kg * ga;
    s[2] += kb * bb + kg * gb;
    s[3] += kb * be + kg * gs;
    // d/dc of c^2 (1-c)^2 = 2 c (1-c)(1-2c); c3^2 (c1+c2)^2 = c3^2 (1-c3)^2 with dc3/dci = -1
    const double d3 = 2.0 * e * (1.0 - e) * (1.0 - 2.0 * e);
    adj[k] = (R)(kb * (g1 * 2.0 * a * (1.0 - a) * (1.0 - 2.0 * a) - g3 * d3));
    adj[3 * nn + k] = (R)(kb * (g2 * 2.0 * b * (1.0 - b) * (1.0 - 2.0 * b) - g3 * d3));
    adj[nn + k] = (R)(2.0 * (kg * (g1 * ax + g3 * sx) + kp * ax));
    adj[2 * nn + k] = (R)(2.0 * (kg * (g1 * ay + g3 * sy) + kp * ay));
    adj[4 * nn + k] = (R)(2.0 * (kg * (g2 * bx + g3 * sx) + kp * bx));
    adj[5 * nn + k] = (R)(2.0 * (kg * (g2 * by + g3 * sy) + kp * by));
  }
  block_partn<4>(s, part);
}

// (gc1, gc2) = C^T of the six loss adjoints; gw = 0
template <class R>
__global__ void k_adj3_loss_acc(const AdjParT<R> P, const cx<R>* __restrict__ xb, cx<R>* __restrict__ g1,
                                cx<R>* __restrict__ g2, cx<R>* __restrict__ gw, size_t ncx) {
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  ModeIdx<R> m;
  if (!mode_of(P, idx, m)) return;
  const R sc = m.wj / (R)((double)P.n * (double)P.n);
  const cx<R> a = cscale(xb[idx], sc), ax = mul_mik(cscale(xb[ncx + idx], sc), m.kx),
              ay = mul_mik(cscale(xb[2 * ncx + idx], sc), m.ky);
  const cx<R> b = cscale(xb[3 * ncx + idx], sc), bx = mul_mik(cscale(xb[4 * ncx + idx], sc), m.kx),
              by = mul_mik(cscale(xb[5 * ncx + idx], sc), m.ky);
  g1[idx] = mk<R>(a.x + ax.x + ay.x, a.y + ax.y + ay.y);
  g2[idx] = mk<R>(b.x + bx.x + by.x, b.y + bx.y + by.y);
  gw[idx] = czero<R>();
}

}  // namespace chns
