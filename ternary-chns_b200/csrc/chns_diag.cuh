// chns_diag.cuh -- free energy and kinetic energy of the state on the GPU.
//
// free_energy.c:3-157: bulk energy of c (NOT truncated) and gradient energy of
// grad c (NOT truncated); kinetic_energy.c:3-144: <|u|^2/2> of the truncated
// velocity and its mean inside each phase (c_t >= 0.5).  One spectral pass
// writes the needed x-inverse-transformed fields (untruncated ones into H
// buffers with all n/2+1 rows, truncated ones into G buffers), one row pass
// does the y inverse transforms and the pointwise sums with double
// accumulators, and a single-block pass sums the per-CTA partials in a fixed
// order (deterministic).
#pragma once

#include "chns_kernels.cuh"

namespace chns {

constexpr int NRED = 8;  // partial sums per CTA

// inverse y transform with direct loads (diagnostics only)
template <int N, class R>
__device__ __forceinline__ void row_c2r_direct(cx<R>* v, RowSrc<R> s, int jt, bool live, int t, cx<R>* sh,
                                               const Tw<R>& tw) {
  constexpr int NT = N / 16;
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int k = t + NT * m;
    const bool cj = k > N / 2;
    const int kk = cj ? N - k : k;
    cx<R> a = czero<R>(), b = czero<R>();
    if (live && kk <= jt) {
      const cx<R>* p = s.base + (size_t)kk * s.stride + s.off;
      a = p[0];
      b = p[1];
    }
    if (kk == 0 || kk == N / 2) { a.y = (R)0; b.y = (R)0; }
    v[m] = cj ? mk<R>(a.x + b.y, b.x - a.y) : mk<R>(a.x - b.y, a.y + b.x);
  }
  fft<N, +1>(v, sh, t, tw);
}

// FILT: SMOOTH_FILTER truncation (P.filt), a variant of its own as in P3
template <int N, class R, int GPC, int MODEL, bool FILT = false>
__global__ void __launch_bounds__(GPC * (N / 16)) k_diag_spec(const Bufs<R> B, const Par<R> P) {
  constexpr int NT = N / 16;
  constexpr int NR = N / 2 + 1;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), P.tw, t);
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int row = blockIdx.x * GPC + g;
  const bool live = row < NR;
  const bool tr = (int)(blockIdx.x * GPC) <= P.jt;  // CTA-uniform: truncated fields needed
  const int mlim = (live && row <= P.jt) ? P.mrow[row] : -1;
  const R ky = (R)(P.fy * (double)row);
  const R sc = P.scale;
  auto kxm = [&](int m) -> R { return (R)(P.fx * (double)sidx<N>(t + NT * m)); };
  cx<R> in[16], v[16];

  if constexpr (MODEL >= MODEL_BINARY) {
#pragma unroll
    for (int f = 0; f < (MODEL == MODEL_TERNARY ? 2 : 1); f++) {
      load_row<N>(in, f == 0 ? B.c1 : B.c2, row, live, t);
      // c, untruncated (free_energy.c:21-22)
#pragma unroll
      for (int m = 0; m < 16; m++) v[m] = mk<R>(in[m].x * sc, in[m].y * sc);
      fft<N, +1>(v, sh, t, TW);
      if (MODEL == MODEL_BINARY) store_row<N>(v, B.h[HF], row, live, t);
      else store_row_pair<N>(v, B.h[HF], row, f, live, t);
      // grad c, untruncated (free_energy.c:72-78 / 107-119)
#pragma unroll
      for (int d = 0; d < 2; d++) {
#pragma unroll
        for (int m = 0; m < 16; m++) {
          const R k = d == 0 ? kxm(m) : ky;
          v[m] = mk<R>(-rmul(k, in[m].y) * sc, rmul(k, in[m].x) * sc);
        }
        fft<N, +1>(v, sh, t, TW);
        store_row_pair<N>(v, B.h[f == 0 ? HAB : HFF], row, d, live, t);
      }
      // truncated c for the phase masks (kinetic_energy.c:23-32)
      if (tr) {
#pragma unroll
        for (int m = 0; m < 16; m++) {
          v[m] = amask<N>(t, m) <= mlim ? mk<R>(in[m].x * sc, in[m].y * sc) : czero<R>();
          if (FILT && amask<N>(t, m) <= mlim) v[m] = smooth2(v[m], P.filt[(size_t)row * NR + amask<N>(t, m)]);
        }
        fft<N, +1>(v, sh, t, TW);
        if (row <= P.jt) {
          if (MODEL == MODEL_BINARY) store_row<N>(v, B.g[GCT], row, live, t);
          else store_row_pair<N>(v, B.g[GCT], row, f, live, t);
        }
      }
    }
  }
  // truncated velocity (kinetic_energy.c:17-21)
  if (tr) {
    load_row<N>(in, B.w, row, live, t);
#pragma unroll
    for (int d = 0; d < 2; d++) {
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const R kx = kxm(m), ks = ksq(kx, ky);
        R a = (R)0, b = (R)0;
        if (ks > (R)1e-12 && amask<N>(t, m) <= mlim) { a = rdiv(in[m].x, ks); b = rdiv(in[m].y, ks); }
        v[m] = d == 0 ? mk<R>(-rmul(ky, b) * sc, rmul(ky, a) * sc) : mk<R>(rmul(kx, b) * sc, -rmul(kx, a) * sc);
        if (FILT && amask<N>(t, m) <= mlim) v[m] = smooth2(v[m], P.filt[(size_t)row * NR + amask<N>(t, m)]);
      }
      fft<N, +1>(v, sh, t, TW);
      if (row <= P.jt) store_row_pair<N>(v, B.g[GUV], row, d, live, t);
    }
  }
}

// per-CTA sums: [0] bulk, [1] grad, [2] eu, [3] eph1, [4] eph2, [5] n1, [6] n2
template <int N, class R, int GPC, int MODEL>
__global__ void __launch_bounds__(GPC * (N / 16)) k_diag_row(const Bufs<R> B, const Par<R> P, double* part) {
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), P.tw, t);
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int pair = blockIdx.x * GPC + g;
  const bool live = pair < N / 2;
  const int i0 = 2 * pair;
  const int jt = P.jt;
  auto pf = [&](cx<R>* base, int i) { return RowSrc<R>{base, 2 * N, 2 * i}; };
  double acc[NRED] = {0, 0, 0, 0, 0, 0, 0, 0};
  cx<R> a[16], b[16], c[16];
  if constexpr (MODEL == MODEL_BINARY) {
    row_c2r_direct<N>(c, RowSrc<R>{B.g[GCT], N, i0}, jt, live, t, sh, TW);  // c_t of x-rows i0, i1
    row_c2r_direct<N>(a, RowSrc<R>{B.h[HF], N, i0}, N / 2, live, t, sh, TW);  // c (untruncated)
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const double c0 = a[m].x, c1 = a[m].y;
      acc[0] += c0 * c0 * (1.0 - c0) * (1.0 - c0) + c1 * c1 * (1.0 - c1) * (1.0 - c1);
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      row_c2r_direct<N>(a, pf(B.g[GUV], i0 + h), jt, live, t, sh, TW);
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const double ke = 0.5 * ((double)a[m].x * a[m].x + (double)a[m].y * a[m].y);
        acc[2] += ke;
        if ((h ? c[m].y : c[m].x) >= (R)0.5) { acc[3] += ke; acc[5] += 1.0; }
      }
      row_c2r_direct<N>(b, pf(B.h[HAB], i0 + h), N / 2, live, t, sh, TW);
#pragma unroll
      for (int m = 0; m < 16; m++) acc[1] += (double)b[m].x * b[m].x + (double)b[m].y * b[m].y;
    }
  } else if constexpr (MODEL == MODEL_TERNARY) {
    const double g1 = P.g1, g2 = P.g2, g3 = P.g3;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int i = i0 + h;
      row_c2r_direct<N>(c, pf(B.g[GCT], i), jt, live, t, sh, TW);  // (c1_t, c2_t)
      row_c2r_direct<N>(a, pf(B.g[GUV], i), jt, live, t, sh, TW);
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const double ke = 0.5 * ((double)a[m].x * a[m].x + (double)a[m].y * a[m].y);
        acc[2] += ke;
        if (c[m].x >= (R)0.5) { acc[3] += ke; acc[5] += 1.0; }
        if (c[m].y >= (R)0.5) { acc[4] += ke; acc[6] += 1.0; }
      }
      row_c2r_direct<N>(a, pf(B.h[HF], i), N / 2, live, t, sh, TW);  // (c1, c2) untruncated
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const double p = a[m].x, q = a[m].y, r = 1.0 - p - q;
        acc[0] += g1 * p * p * (1.0 - p) * (1.0 - p) + g2 * q * q * (1.0 - q) * (1.0 - q) + g3 * r * r * (p + q) * (p + q);
      }
      row_c2r_direct<N>(a, pf(B.h[HAB], i), N / 2, live, t, sh, TW);  // (c1x, c1y)
      row_c2r_direct<N>(b, pf(B.h[HFF], i), N / 2, live, t, sh, TW);  // (c2x, c2y)
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const double x1 = a[m].x, y1 = a[m].y, x2 = b[m].x, y2 = b[m].y;
        acc[1] += g1 * (x1 * x1 + y1 * y1) + g2 * (x2 * x2 + y2 * y2) + g3 * (x1 + x2) * (x1 + x2) +
                  g3 * (y1 + y2) * (y1 + y2);
      }
    }
  } else {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      row_c2r_direct<N>(a, pf(B.g[GUV], i0 + h), jt, live, t, sh, TW);
#pragma unroll
      for (int m = 0; m < 16; m++) acc[2] += 0.5 * ((double)a[m].x * a[m].x + (double)a[m].y * a[m].y);
    }
  }
  if (!live) {
#pragma unroll
    for (int k = 0; k < NRED; k++) acc[k] = 0.0;
  }
  // block reduction in a fixed order
  __syncthreads();
  double* red = reinterpret_cast<double*>(smem_raw);
  const int nthr = blockDim.x;
#pragma unroll
  for (int k = 0; k < NRED; k++) red[k * nthr + threadIdx.x] = acc[k];
  __syncthreads();
  for (int s = nthr / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
#pragma unroll
      for (int k = 0; k < NRED; k++) red[k * nthr + threadIdx.x] += red[k * nthr + threadIdx.x + s];
    }
    __syncthreads();
  }
  for (int k = threadIdx.x; k < NRED; k += nthr) part[(size_t)blockIdx.x * NRED + k] = red[k * nthr];
}

static __global__ void k_diag_final(const double* __restrict__ part, int nblk, double* out) {
  __shared__ double s[NRED][256];
  for (int k = 0; k < NRED; k++) {
    double a = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) a += part[(size_t)b * NRED + k];
    s[k][threadIdx.x] = a;
  }
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int k = 0; k < NRED; k++) s[k][threadIdx.x] += s[k][threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x < NRED) out[threadIdx.x] = s[threadIdx.x][0];
}

}  // namespace chns
