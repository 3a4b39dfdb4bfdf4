// chns_adj_rows.cuh -- the binary discrete adjoint's record table and its product
// adjoints fused into the first pass of the forward transform that consumes them.
//
// The transposed right-hand side (nonlin.c:207-251, surface_tension.c:57-112 read
// backwards) forms, point by point, the adjoints of the products of the forward
// step from the physical adjoints A_bar, B_bar, Fx_bar, Fy_bar, f_bar and the
// forward fields the forward step recorded:
//   mu_bar = Fx_bar cx + Fy_bar cy                          (surface_tension.c:87-88)
//   u_bar = Ab wx + Bb cx, v_bar = Ab wy + Bb cy, wx_bar = Ab u, wy_bar = Ab v,
//   cx_bar = Bb u + Fxb mu, cy_bar = Bb v + Fyb mu, ct_bar = fb f'(ct)
// and transforms them forward.  k_adj_prod_r2c computes them while it loads the
// rows of its r2c pass, so they never pass through memory as fields of their own.
#pragma once

#include "chns_kernels.cuh"

namespace chns {

// The forward fields of one right-hand side that its transpose needs, as recorded by
// the forward step's REC kernels (n x n real fields and F[f(c_t)] in the S layout),
// and c_hat of the state it was formed at.
template <class R> struct RecFields {
  const R *u, *v, *wx, *wy, *ct, *gx, *gy, *mu;  // gx, gy: grad c
  const cx<R>* ff;
  const cx<R>* cc;
};

// The record of the step being reversed, device-resident so that a captured reversed
// step reads whichever segment slot it is pointed at: the right-hand sides at u*
// (rhs[0]) and at u_n (rhs[1]), and the slot's states in its order u_n (w, c),
// u* (w, c), N(u_n) (w, c), N(u*) (w, c).
template <class R> struct RecStep {
  RecFields<R> rhs[2];
  const cx<R>* f[8];
};

// the physical adjoints a transposed right-hand side has formed (n x n real each)
template <class R> struct AdjIn {
  const R *ab, *bb, *fxb, *fyb, *fb;
};

// product adjoint B (0..6: u, v, wx, wy, ct, cx, cy; 7: mu_bar) at point k
template <int B, class R>
__device__ __forceinline__ R adj_product(const RecFields<R>& F, const AdjIn<R>& A, size_t k) {
  if constexpr (B == 0) return A.ab[k] * F.wx[k] + A.bb[k] * F.gx[k];
  if constexpr (B == 1) return A.ab[k] * F.wy[k] + A.bb[k] * F.gy[k];
  if constexpr (B == 2) return A.ab[k] * F.u[k];
  if constexpr (B == 3) return A.ab[k] * F.v[k];
  if constexpr (B == 4) {
    const R ct = F.ct[k];
    return A.fb[k] * ((R)1 - (R)6 * ct + (R)6 * ct * ct);
  }
  if constexpr (B == 5) return A.bb[k] * F.u[k] + A.fxb[k] * F.mu[k];
  if constexpr (B == 6) return A.bb[k] * F.v[k] + A.fyb[k] * F.mu[k];
  if constexpr (B == 7) return A.fxb[k] * F.gx[k] + A.fyb[k] * F.gy[k];
}

// x-rows i0, i0 + 1 of product adjoint B as the 16 complex values of thread t
template <int N, int B, class R>
__device__ __forceinline__ void adj_product_rows(cx<R>* v, const RecFields<R>& F, const AdjIn<R>& A, int i0,
                                                 bool live, int t) {
  constexpr int NT = N / 16;
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const size_t k = (size_t)i0 * N + t + NT * m;
    v[m] = live ? mk<R>(adj_product<B>(F, A, k), adj_product<B>(F, A, k + N)) : czero<R>();
  }
}

// r2c row pass (two x-rows per transform, H layout out, as k_row_r2c_plain) of
// product adjoint b0 + blockIdx.y, formed from the record rf and the adjoints A
template <int N, class R, int GPC>
__global__ void __launch_bounds__(GPC * (N / 16))
    k_adj_prod_r2c(const RecFields<R>* __restrict__ rf, const AdjIn<R> A, int b0, cx<R>* __restrict__ H,
                   const cx<R>* __restrict__ tw, size_t hs) {
  constexpr int NT = N / 16;
  const int b = b0 + (int)blockIdx.y;
  H += blockIdx.y * hs;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), tw, t);
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int pair = blockIdx.x * GPC + g;
  const bool live = pair < N / 2;
  const int i0 = 2 * pair;
  const RecFields<R> F = *rf;
  cx<R> v[16];
  switch (b) {  // uniform over the block
    case 0: adj_product_rows<N, 0>(v, F, A, i0, live, t); break;
    case 1: adj_product_rows<N, 1>(v, F, A, i0, live, t); break;
    case 2: adj_product_rows<N, 2>(v, F, A, i0, live, t); break;
    case 3: adj_product_rows<N, 3>(v, F, A, i0, live, t); break;
    case 4: adj_product_rows<N, 4>(v, F, A, i0, live, t); break;
    case 5: adj_product_rows<N, 5>(v, F, A, i0, live, t); break;
    case 6: adj_product_rows<N, 6>(v, F, A, i0, live, t); break;
    default: adj_product_rows<N, 7>(v, F, A, i0, live, t); break;
  }
  row_r2c_store<N>(v, H, N, i0, live, t, sh, TW);
}

}  // namespace chns
