// chns_kernels.cuh -- the fused passes of one ETD2RK stage on sm_100a.
//
// Data layout in HBM (see also chns_api.cu):
//   S layout  : spectral field, row j' (ky index, 0..n/2) of n complex along kx
//               (the transpose of FFTW's n x (n/2+1) layout, global.h:13-14), so
//               the column transforms along x are contiguous rows.
//   G layout  : like S but only rows 0..jt, jt = the last ky row that survives
//               the truncation (functions.c:47-84).  Holds fields that went
//               through the column (x) inverse transform and wait for the row
//               (y) inverse transform.
//   H layout  : like S; holds fields after the row (y) forward transform,
//               waiting for the column (x) forward transform.
//
// One stage (etd2rk.c:28-135 or :146-212) of the binary model is five kernels:
//   P1 spec_inv     : S -> G : velocity, gradients, truncation, 1/(nx ny), x-iFFT
//   P2 row_adv      : G -> H : y-c2r of x-row pairs, u.grad w, u.grad c, f(c), y-r2c
//   P3 spec_fwd_c   : H -> S : x-FFT; mu_hat and its x-iFFT (-> G); N_c; ETD of c
//   P4 row_force    : G -> H : y-c2r of mu and grad c, mu grad c, y-r2c
//   P5 spec_curl_w  : H -> S : x-FFT; curl; N_w; ETD of w
// Ternary adds the chemical potential (chem_potential.c) to P2 and uses two
// row kernels for P2.  Pure Navier-Stokes is P1, P2 and P3-ns.
#pragma once

#include "chns_fft.cuh"

namespace chns {

enum { MODEL_NS = 0, MODEL_BINARY = 1, MODEL_TERNARY = 2 };

// G-layout buffer slots
enum { GU = 0, GV, GDXW, GDYW, GC1, GC2, GDX1, GDY1, GDX2, GDY2, GMU1, GMU2, NG };
// H-layout buffer slots
enum { HA = 0, HB1, HB2, HF1, HF2, HFX, HFY, NH };

template <class R> struct Par {
  int n, jt;               // grid; last G row that can hold a nonzero mode
  double fx, fy;           // factor_x, factor_y (main.c:54-55)
  R scale;                 // 1/(Nx Ny) of ifft (fft.c:22), a power of two
  R st15, st24, lam;       // binary: 1.5 sigma eps, 24 (sigma/eps), lambda
  R mu1, mu2, lg1, lg2;    // ternary: 0.75 gamma_i eps, lambda/gamma_i
  R w11, w12, w21, w22;    // ternary: 1+g3/g1, g3/g2, g3/g1, 1+g3/g2
  R g1, g2, g3, g1i, g2i, g3i, six_lam, fac_mu;  // ternary chemical potential
  int force_j;             // Kolmogorov forcing row (-1: off)
  R force_hat;             // its spectral amplitude, added to N_w at (0, force_j)
  double k0coef[6];        // ETD coefficients at k = 0 (double)
  const int* mrow;         // [n/2+1] largest |m| kept by the truncation per row (-1: none)
  const R* coef;           // [6][n/2+1][n/2+1] ETD coefficients at (row, |m|)
  const cx<R>* tw;         // tw[q] = exp(-2 pi i q / n)
  double* k0;              // FP32 only: k = 0 modes in double [w, c1, c2, sw, s1, s2] x (re, im)
};

template <class R> struct Bufs {
  cx<R>* w;
  cx<R>* c1;
  cx<R>* c2;
  cx<R>* sw;
  cx<R>* s1;
  cx<R>* s2;
  cx<R>* nw;
  cx<R>* g[NG];
  cx<R>* h[NH];
};

// FP32 step kernels are built for two CTAs per SM (<= 128 registers), FP64 for one
#define CHNS_STEP_BOUNDS(N, R, GPC) __launch_bounds__((GPC) * ((N) / 16), sizeof(R) == 4 ? 2 : 1)

template <class R> __device__ __forceinline__ cx<R> czero() { return mk<R>((R)0, (R)0); }

// signed wavenumber index of column i (functions.c:17-24: Nyquist positive)
template <int N> __device__ __forceinline__ int sidx(int i) { return i <= N / 2 ? i : i - N; }

template <class R> __device__ __forceinline__ R ksq(R kx, R ky) { return radd(rmul(kx, kx), rmul(ky, ky)); }

// ---------------------------------------------------------------------------
// row (y) transforms of a pair of x-rows
// ---------------------------------------------------------------------------

// two adjacent complex values (columns i0, i0+1, i0 even): one 16-byte access in FP32
static __device__ __forceinline__ void ld_pair(const cxf* p, cxf& a, cxf& b) {
  const float4 q = __ldg(reinterpret_cast<const float4*>(p));
  a = mk<float>(q.x, q.y);
  b = mk<float>(q.z, q.w);
}
static __device__ __forceinline__ void ld_pair(const cxd* p, cxd& a, cxd& b) {
  const double2 q0 = __ldg(reinterpret_cast<const double2*>(p));
  const double2 q1 = __ldg(reinterpret_cast<const double2*>(p) + 1);
  a = mk<double>(q0.x, q0.y);
  b = mk<double>(q1.x, q1.y);
}
static __device__ __forceinline__ void st_pair(cxf* p, cxf a, cxf b) {
  *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
static __device__ __forceinline__ void st_pair(cxd* p, cxd a, cxd b) {
  reinterpret_cast<double2*>(p)[0] = make_double2(a.x, a.y);
  reinterpret_cast<double2*>(p)[1] = make_double2(b.x, b.y);
}

// Inverse y transform (c2r) of x-rows i0, i0+1 of a G-layout field: builds
// Z = X_{i0} + i X_{i0+1} with the Hermitian extension (Im of the ky = 0 and
// ky = n/2 bins ignored, FFTW's c2r convention) and transforms.  Output:
// v[m] = (x_{i0}[y], x_{i0+1}[y]) at y = t + NT m.
template <int N, class R>
__device__ __forceinline__ void row_c2r(cx<R>* v, const cx<R>* __restrict__ G, int i0, int jt, bool live,
                                        int t, cx<R>* sh, const cx<R>* __restrict__ tw) {
  constexpr int NT = N / 16;
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int k = t + NT * m;
    const bool cj = k > N / 2;
    const int kk = cj ? N - k : k;
    cx<R> a = czero<R>(), b = czero<R>();
    if (live && kk <= jt) ld_pair(G + (size_t)kk * N + i0, a, b);
    if (kk == 0 || kk == N / 2) { a.y = (R)0; b.y = (R)0; }
    v[m] = cj ? mk<R>(a.x + b.y, b.x - a.y) : mk<R>(a.x - b.y, a.y + b.x);
  }
  fft<N, +1>(v, sh, t, tw);
}

// Forward y transform (r2c) of x-rows i0, i0+1 packed as v = a + i b, split
// into the two half spectra and stored to rows 0..n/2 of an H-layout field.
template <int N, class R>
__device__ __forceinline__ void row_r2c_store(cx<R>* v, cx<R>* __restrict__ H, int i0, bool live, int t,
                                              cx<R>* sh, const cx<R>* __restrict__ tw) {
  constexpr int NT = N / 16;
  fft<N, -1>(v, sh, t, tw);
  __syncthreads();
#pragma unroll
  for (int m = 0; m < 16; m++) sh[spad(t + NT * m)] = v[m];
  __syncthreads();
#pragma unroll
  for (int m = 0; m <= 8; m++) {
    const int k = t + NT * m;
    if (k <= N / 2) {
      const cx<R> z = v[m];
      const cx<R> q = sh[spad((N - k) & (N - 1))];
      const cx<R> A = mk<R>((R)0.5 * (z.x + q.x), (R)0.5 * (z.y - q.y));
      const cx<R> B = mk<R>((R)0.5 * (z.y + q.y), (R)0.5 * (q.x - z.x));
      if (live) st_pair(H + (size_t)k * N + i0, A, B);
    }
  }
}

// thread-private frag slots in shared memory: element m of thread t at [t + NT m]
template <int N, class R> struct Frag {
  cx<R>* p;
  __device__ __forceinline__ cx<R>& operator[](int m) const { return p[(threadIdx.x % (N / 16)) + (N / 16) * m]; }
};

// ---------------------------------------------------------------------------
// P1: spectral fan-out + x inverse transform   (S -> G)
// nonlin.c:30-48, velocity.c:12-42, surface_tension.c:20-22,57-75,
// nonlin.c:177-198,259-284, chem_potential.c:256-261
// ---------------------------------------------------------------------------

// What P1 emits, per model, into the G slots.
template <int N, class R, int GPC, int MODEL>
__global__ void CHNS_STEP_BOUNDS(N, R, GPC) k_spec_inv(const Bufs<R> B, const Par<R> P) {
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int row = blockIdx.x * GPC + g;
  const bool live = row <= P.jt;
  const int mlim = live ? P.mrow[row] : -1;
  const R ky = (R)(P.fy * (double)row);
  const R sc = P.scale;

  uint32_t inmask = 0;
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int ms = sidx<N>(t + NT * m);
    if ((ms < 0 ? -ms : ms) <= mlim) inmask |= 1u << m;
  }
  auto kxm = [&](int m) -> R { return (R)(P.fx * (double)sidx<N>(t + NT * m)); };
  auto store = [&](cx<R>* v, int slot) {
    if (live) {
      cx<R>* p = B.g[slot] + (size_t)row * N;
#pragma unroll
      for (int m = 0; m < 16; m++) p[t + NT * m] = v[m];
    }
  };

  cx<R> in[16], v[16];
  // omega_hat
#pragma unroll
  for (int m = 0; m < 16; m++)
    in[m] = ((inmask >> m) & 1) ? B.w[(size_t)row * N + t + NT * m] : czero<R>();
  // u = I ky psi, v = -I kx psi, psi = w / k^2  (velocity.c:12-42)
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const R kx = kxm(m), ks = ksq(kx, ky);
    R a = (R)0, b = (R)0;
    if (ks > (R)1e-12) { a = rdiv(in[m].x, ks); b = rdiv(in[m].y, ks); }
    v[m] = mk<R>(-rmul(ky, b) * sc, rmul(ky, a) * sc);
  }
  fft<N, +1>(v, sh, t, P.tw);
  store(v, GU);
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const R kx = kxm(m), ks = ksq(kx, ky);
    R a = (R)0, b = (R)0;
    if (ks > (R)1e-12) { a = rdiv(in[m].x, ks); b = rdiv(in[m].y, ks); }
    v[m] = mk<R>(rmul(kx, b) * sc, -rmul(kx, a) * sc);
  }
  fft<N, +1>(v, sh, t, P.tw);
  store(v, GV);
  // grad omega: I kx w, I ky w  (nonlin.c:36-37)
#pragma unroll
  for (int m = 0; m < 16; m++) { const R kx = kxm(m); v[m] = mk<R>(-rmul(kx, in[m].y) * sc, rmul(kx, in[m].x) * sc); }
  fft<N, +1>(v, sh, t, P.tw);
  store(v, GDXW);
#pragma unroll
  for (int m = 0; m < 16; m++) v[m] = mk<R>(-rmul(ky, in[m].y) * sc, rmul(ky, in[m].x) * sc);
  fft<N, +1>(v, sh, t, P.tw);
  store(v, GDYW);

  if constexpr (MODEL >= MODEL_BINARY) {
#pragma unroll
    for (int f = 0; f < (MODEL == MODEL_TERNARY ? 2 : 1); f++) {
      const cx<R>* src = f == 0 ? B.c1 : B.c2;
#pragma unroll
      for (int m = 0; m < 16; m++)
        in[m] = ((inmask >> m) & 1) ? src[(size_t)row * N + t + NT * m] : czero<R>();
      // truncated c (surface_tension.c:20-22, nonlin.c:217, chem_potential.c:256-261)
#pragma unroll
      for (int m = 0; m < 16; m++) v[m] = mk<R>(in[m].x * sc, in[m].y * sc);
      fft<N, +1>(v, sh, t, P.tw);
      store(v, f == 0 ? GC1 : GC2);
      // grad c: I kx c, I ky c (surface_tension.c:57-58, nonlin.c:187-188, 272-273, 314-315)
#pragma unroll
      for (int m = 0; m < 16; m++) { const R kx = kxm(m); v[m] = mk<R>(-rmul(kx, in[m].y) * sc, rmul(kx, in[m].x) * sc); }
      fft<N, +1>(v, sh, t, P.tw);
      store(v, f == 0 ? GDX1 : GDX2);
#pragma unroll
      for (int m = 0; m < 16; m++) v[m] = mk<R>(-rmul(ky, in[m].y) * sc, rmul(ky, in[m].x) * sc);
      fft<N, +1>(v, sh, t, P.tw);
      store(v, f == 0 ? GDY1 : GDY2);
    }
  }
}

// ---------------------------------------------------------------------------
// P2: advection products (+ bulk chemical potential) on x-row pairs (G -> H)
// nonlin.c:56-74 (u.grad w), :201-215 (binary u.grad c), :286-300/328-348
// (ternary u.grad c_i); surface_tension.c:24-35 / nonlin.c:217-230 (f(c));
// chem_potential.c:263-320 (ternary mu^F)
// ---------------------------------------------------------------------------

// acc_a = u . (dx_a, dy_a) for NACC pairs of G slots, accumulated in shared memory
// frags, forward transformed to H slots.  PRE selects extra work done first:
// 0 none; 1 binary f(c) -> HF1; 2 ternary mu^F_1, mu^F_2 -> HF1, HF2.
template <class R> struct AdvIO {
  const cx<R>* dx[3];
  const cx<R>* dy[3];
  cx<R>* out[3];
};

template <int N, class R, int GPC, int NACC, int PRE>
__global__ void CHNS_STEP_BOUNDS(N, R, GPC)
k_row_adv(const Bufs<R> B, const Par<R> P, const AdvIO<R> io) {
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  cx<R>* accbase = reinterpret_cast<cx<R>*>(smem_raw) + GPC * FftShape<N>::SMEM;
  const int pair = blockIdx.x * GPC + g;
  const bool live = pair < N / 2;
  const int i0 = 2 * pair;
  const int jt = P.jt;

  cx<R> u[16], v[16];
  if constexpr (PRE == 1) {
    // f(c) = c (1 - c)(1 - 2c) on the truncated c (surface_tension.c:30-31, nonlin.c:225)
    row_c2r<N>(v, B.g[GC1], i0, jt, live, t, sh, P.tw);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const R a = v[m].x, b = v[m].y;
      v[m] = mk<R>(rmul(rmul(a, rsub((R)1, a)), rsub((R)1, rmul((R)2, a))),
                   rmul(rmul(b, rsub((R)1, b)), rsub((R)1, rmul((R)2, b))));
    }
    row_r2c_store<N>(v, B.h[HF1], i0, live, t, sh, P.tw);
  } else if constexpr (PRE == 2) {
    // ternary bulk chemical potentials (chem_potential.c:303-315)
    row_c2r<N>(u, B.g[GC1], i0, jt, live, t, sh, P.tw);
    row_c2r<N>(v, B.g[GC2], i0, jt, live, t, sh, P.tw);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      R o1[2], o2[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const R c1 = h ? u[m].y : u[m].x, c2 = h ? v[m].y : v[m].x;
        const R c3 = rsub(rsub((R)1, c1), c2);
        const R c123 = rmul(rmul(c1, c2), c3);
        const R fc1 = rmul(rmul(c1, rsub((R)1, c1)), rsub((R)1, rmul((R)2, c1)));
        const R fc2 = rmul(rmul(c2, rsub((R)1, c2)), rsub((R)1, rmul((R)2, c2)));
        const R fc3 = rmul(rmul(c3, rsub((R)1, c3)), rsub((R)1, rmul((R)2, c3)));
        const R G1 = radd(rmul(P.g1, fc1), rmul(rmul(rmul(P.six_lam, c123), c2), c3));
        const R G2 = radd(rmul(P.g2, fc2), rmul(rmul(rmul(P.six_lam, c123), c1), c3));
        const R G3 = radd(rmul(P.g3, fc3), rmul(rmul(rmul(P.six_lam, c123), c1), c2));
        const R m1 = radd(rmul(rsub(G1, G2), P.g2i), rmul(rsub(G1, G3), P.g3i));
        const R m2 = radd(rmul(rsub(G2, G1), P.g1i), rmul(rsub(G2, G3), P.g3i));
        o1[h] = rmul(m1, P.fac_mu);
        o2[h] = rmul(m2, P.fac_mu);
      }
      u[m] = mk<R>(o1[0], o1[1]);
      v[m] = mk<R>(o2[0], o2[1]);
    }
    row_r2c_store<N>(u, B.h[HF1], i0, live, t, sh, P.tw);
    row_r2c_store<N>(v, B.h[HF2], i0, live, t, sh, P.tw);
  }

  if constexpr (NACC > 0) {
    // first factor u: acc_a = u * dx_a
    row_c2r<N>(u, B.g[GU], i0, jt, live, t, sh, P.tw);
#pragma unroll
    for (int a = 0; a < NACC; a++) {
      Frag<N, R> acc{accbase + (size_t)(a * GPC + g) * N};
      row_c2r<N>(v, io.dx[a], i0, jt, live, t, sh, P.tw);
#pragma unroll
      for (int m = 0; m < 16; m++) acc[m] = mk<R>(rmul(u[m].x, v[m].x), rmul(u[m].y, v[m].y));
    }
    // second factor: acc_a += v * dy_a, then the forward y transform
    row_c2r<N>(u, B.g[GV], i0, jt, live, t, sh, P.tw);
#pragma unroll
    for (int a = 0; a < NACC; a++) {
      Frag<N, R> acc{accbase + (size_t)(a * GPC + g) * N};
      row_c2r<N>(v, io.dy[a], i0, jt, live, t, sh, P.tw);
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const cx<R> s = acc[m];
        v[m] = mk<R>(radd(s.x, rmul(u[m].x, v[m].x)), radd(s.y, rmul(u[m].y, v[m].y)));
      }
      row_r2c_store<N>(v, io.out[a], i0, live, t, sh, P.tw);
    }
  }
}

// ---------------------------------------------------------------------------
// P4: surface-tension force mu grad c on x-row pairs (G -> H)
// binary surface_tension.c:70-99; ternary :136-160, :188-210 (the two curls of
// the reference are summed before the transform: F[a] + F[b] = F[a + b])
// ---------------------------------------------------------------------------
template <int N, class R, int GPC, int MODEL>
__global__ void CHNS_STEP_BOUNDS(N, R, GPC) k_row_force(const Bufs<R> B, const Par<R> P) {
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  cx<R>* fbase = reinterpret_cast<cx<R>*>(smem_raw) + GPC * FftShape<N>::SMEM;
  const int pair = blockIdx.x * GPC + g;
  const bool live = pair < N / 2;
  const int i0 = 2 * pair;
  const int jt = P.jt;
  cx<R> a[16], b[16];
  if constexpr (MODEL == MODEL_BINARY) {
    row_c2r<N>(a, B.g[GMU1], i0, jt, live, t, sh, P.tw);  // mu_t
#pragma unroll
    for (int d = 0; d < 2; d++) {
      row_c2r<N>(b, B.g[d == 0 ? GDX1 : GDY1], i0, jt, live, t, sh, P.tw);
#pragma unroll
      for (int m = 0; m < 16; m++) b[m] = mk<R>(rmul(b[m].x, a[m].x), rmul(b[m].y, a[m].y));
      row_r2c_store<N>(b, B.h[d == 0 ? HFX : HFY], i0, live, t, sh, P.tw);
    }
  } else {
    // weights w1 = (1+g3/g1) mu1 + (g3/g2) mu2, w2 = (g3/g1) mu1 + (1+g3/g2) mu2
    Frag<N, R> w1{fbase + (size_t)(0 * GPC + g) * N};
    Frag<N, R> w2{fbase + (size_t)(1 * GPC + g) * N};
    row_c2r<N>(a, B.g[GMU1], i0, jt, live, t, sh, P.tw);
    row_c2r<N>(b, B.g[GMU2], i0, jt, live, t, sh, P.tw);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      w1[m] = mk<R>(radd(rmul(P.w11, a[m].x), rmul(P.w12, b[m].x)), radd(rmul(P.w11, a[m].y), rmul(P.w12, b[m].y)));
      w2[m] = mk<R>(radd(rmul(P.w21, a[m].x), rmul(P.w22, b[m].x)), radd(rmul(P.w21, a[m].y), rmul(P.w22, b[m].y)));
    }
#pragma unroll
    for (int d = 0; d < 2; d++) {
      row_c2r<N>(a, B.g[d == 0 ? GDX1 : GDY1], i0, jt, live, t, sh, P.tw);
#pragma unroll
      for (int m = 0; m < 16; m++) { const cx<R> s = w1[m]; a[m] = mk<R>(rmul(a[m].x, s.x), rmul(a[m].y, s.y)); }
      row_c2r<N>(b, B.g[d == 0 ? GDX2 : GDY2], i0, jt, live, t, sh, P.tw);
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const cx<R> s = w2[m];
        a[m] = mk<R>(radd(a[m].x, rmul(b[m].x, s.x)), radd(a[m].y, rmul(b[m].y, s.y)));
      }
      row_r2c_store<N>(a, B.h[d == 0 ? HFX : HFY], i0, live, t, sh, P.tw);
    }
  }
}

// ---------------------------------------------------------------------------
// helpers of the forward spectral passes
// ---------------------------------------------------------------------------

template <int N, class R>
__device__ __forceinline__ void load_row(cx<R>* v, const cx<R>* __restrict__ src, int row, bool live, int t) {
  constexpr int NT = N / 16;
#pragma unroll
  for (int m = 0; m < 16; m++) v[m] = live ? src[(size_t)row * N + t + NT * m] : czero<R>();
}

template <int N, class R>
__device__ __forceinline__ void store_row(const cx<R>* v, cx<R>* __restrict__ dst, int row, bool live, int t) {
  constexpr int NT = N / 16;
  if (live) {
#pragma unroll
    for (int m = 0; m < 16; m++) dst[(size_t)row * N + t + NT * m] = v[m];
  }
}

template <int N, class R> __device__ __forceinline__ int amask(int t, int m) {
  const int ms = sidx<N>(t + (N / 16) * m);
  return ms < 0 ? -ms : ms;
}

// ETD update of one mode (etd2rk.c:99,113,129-130 / 174,188,205-206).
// STAGE 1: u <- u e + N z1, save N.  STAGE 2: u <- u + (N - saved) z2.
template <int STAGE, class R>
__device__ __forceinline__ cx<R> etd(cx<R> u, cx<R> nl, cx<R>* saved, R e, R z1, R z2) {
  if (STAGE == 1) {
    *saved = nl;
    return mk<R>(radd(rmul(u.x, e), rmul(nl.x, z1)), radd(rmul(u.y, e), rmul(nl.y, z1)));
  } else {
    const cx<R> s = *saved;
    return mk<R>(radd(u.x, rmul(rsub(nl.x, s.x), z2)), radd(u.y, rmul(rsub(nl.y, s.y), z2)));
  }
}

// same in double for the FP32 path's k = 0 mode
template <int STAGE>
__device__ __forceinline__ void etd_k0(double* st, double* sv, double nx, double ny, const double* k0c, int off) {
  if (STAGE == 1) {
    sv[0] = nx; sv[1] = ny;
    st[0] = st[0] * k0c[off + 0] + nx * k0c[off + 1];
    st[1] = st[1] * k0c[off + 0] + ny * k0c[off + 1];
  } else {
    st[0] = st[0] + (nx - sv[0]) * k0c[off + 2];
    st[1] = st[1] + (ny - sv[1]) * k0c[off + 2];
  }
}

// ---------------------------------------------------------------------------
// P3 (phase-field models): x forward transforms, N_w partial, mu and its x
// inverse transform, N_c and the ETD update of c  (H -> S, G)
// binary: nonlin.c:74-101 (-F[u.grad w]), surface_tension.c:35-48 (mu_hat),
//         nonlin.c:215-254 (N_c), etd2rk.c:102-113 / 177-188
// ternary: chem_potential.c:319-320 (F[mu^F]), surface_tension.c:116-137,
//          nonlin.c:300-377, etd2rk.c:117-130 / 191-206
// ---------------------------------------------------------------------------
template <int N, class R, int GPC, int MODEL, int STAGE>
__global__ void CHNS_STEP_BOUNDS(N, R, GPC) k_spec_fwd_c(const Bufs<R> B, const Par<R> P) {
  constexpr int NT = N / 16;
  constexpr int NR = N / 2 + 1;
  constexpr bool F32 = sizeof(R) == 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int row = blockIdx.x * GPC + g;
  const bool live = row < NR;
  const int rowc = live ? row : 0;
  const bool do_mu = (int)(blockIdx.x * GPC) <= P.jt;  // CTA-uniform
  const int mlim = (live && row <= P.jt) ? P.mrow[row] : -1;
  const R ky = (R)(P.fy * (double)row);
  const R* cf = P.coef + (size_t)rowc * NR;
  const size_t cstride = (size_t)NR * NR;
  auto kxm = [&](int m) -> R { return (R)(P.fx * (double)sidx<N>(t + NT * m)); };

  cx<R> f[16], c[16], v[16];
  // N_w partial = -F[u.grad w]   (nonlin.c:74, 92)
  load_row<N>(v, B.h[HA], row, live, t);
  fft<N, -1>(v, sh, t, P.tw);
#pragma unroll
  for (int m = 0; m < 16; m++) v[m] = mk<R>(v[m].x * (R)(-1), v[m].y * (R)(-1));
  store_row<N>(v, B.nw, row, live, t);

#pragma unroll
  for (int fld = 0; fld < (MODEL == MODEL_TERNARY ? 2 : 1); fld++) {
    cx<R>* cst = fld == 0 ? B.c1 : B.c2;
    cx<R>* csv = fld == 0 ? B.s1 : B.s2;
    // F[f(c)] (binary) or F[mu^F_i] (ternary)
    load_row<N>(f, B.h[fld == 0 ? HF1 : HF2], row, live, t);
    fft<N, -1>(f, sh, t, P.tw);
    load_row<N>(c, cst, row, live, t);
    if (do_mu) {
      // binary: mu = T[1.5 sigma eps k^2 c + 24 (sigma/eps) F[f]]   (surface_tension.c:45-46)
      // ternary: mu_i = T[F[mu^F_i] + 0.75 gamma_i eps k^2 c_i]     (surface_tension.c:116-128)
#pragma unroll
      for (int m = 0; m < 16; m++) {
        if (amask<N, R>(t, m) <= mlim) {
          const R ks = ksq(kxm(m), ky);
          if (MODEL == MODEL_BINARY) {
            const R q = rmul(P.st15, ks);
            v[m] = mk<R>(radd(rmul(q, c[m].x), rmul(P.st24, f[m].x)) * P.scale,
                         radd(rmul(q, c[m].y), rmul(P.st24, f[m].y)) * P.scale);
          } else {
            const R q = rmul(fld == 0 ? P.mu1 : P.mu2, ks);
            v[m] = mk<R>(radd(f[m].x, rmul(q, c[m].x)) * P.scale, radd(f[m].y, rmul(q, c[m].y)) * P.scale);
          }
        } else {
          v[m] = czero<R>();
        }
      }
      fft<N, +1>(v, sh, t, P.tw);
      if (row <= P.jt) store_row<N>(v, B.g[fld == 0 ? GMU1 : GMU2], row, live, t);
    }
    // N_c  binary: -F[u.grad c] - lambda (24 (sigma/eps) k^2) F[f]   (nonlin.c:240, 251)
    //      ternary: -F[u.grad c_i] - (lambda/gamma_i) k^2 F[mu^F_i]  (nonlin.c:369-370)
    load_row<N>(v, B.h[fld == 0 ? HB1 : HB2], row, live, t);
    fft<N, -1>(v, sh, t, P.tw);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int am = amask<N, R>(t, m);
      const R ks = ksq(kxm(m), ky);
      cx<R> nl;
      if (MODEL == MODEL_BINARY) {
        const R q = rmul(P.st24, ks);
        nl = mk<R>(rsub(-v[m].x, rmul(P.lam, rmul(q, f[m].x))), rsub(-v[m].y, rmul(P.lam, rmul(q, f[m].y))));
      } else {
        const R q = rmul(fld == 0 ? P.lg1 : P.lg2, ks);
        nl = mk<R>(rsub(-v[m].x, rmul(q, f[m].x)), rsub(-v[m].y, rmul(q, f[m].y)));
      }
      const size_t idx = (size_t)rowc * N + t + NT * m;
      const R e = cf[3 * cstride + am], z1 = cf[4 * cstride + am], z2 = cf[5 * cstride + am];
      cx<R> sv;
      if (STAGE == 2) sv = live ? csv[idx] : czero<R>();
      c[m] = etd<STAGE>(c[m], nl, &sv, e, z1, z2);
      if (STAGE == 1 && live) csv[idx] = sv;
      if (F32 && row == 0 && t == 0 && m == 0) {
        double* st = P.k0 + 2 * (1 + fld);
        double* sd = P.k0 + 2 * (4 + fld);
        etd_k0<STAGE>(st, sd, (double)nl.x, (double)nl.y, P.k0coef, 3);
        c[m] = mk<R>((R)st[0], (R)st[1]);
      }
    }
    store_row<N>(c, cst, row, live, t);
  }
}

// ---------------------------------------------------------------------------
// P5 (phase-field models): x forward transforms of the force, curl, N_w and
// the ETD update of w (H -> S)   surface_tension.c:98-111 / 159-173 / 209-223,
// curl.c:16-31, etd2rk.c:88-99 / 162-174
// P3 for pure Navier-Stokes: NACC = 0 (N_w = -F[u.grad w] only)
// ---------------------------------------------------------------------------
template <int N, class R, int GPC, bool CURL, int STAGE>
__global__ void CHNS_STEP_BOUNDS(N, R, GPC) k_spec_curl_w(const Bufs<R> B, const Par<R> P) {
  constexpr int NT = N / 16;
  constexpr int NR = N / 2 + 1;
  constexpr bool F32 = sizeof(R) == 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int row = blockIdx.x * GPC + g;
  const bool live = row < NR;
  const int rowc = live ? row : 0;
  const R ky = (R)(P.fy * (double)row);
  const R* cf = P.coef + (size_t)rowc * NR;
  const size_t cstride = (size_t)NR * NR;
  auto kxm = [&](int m) -> R { return (R)(P.fx * (double)sidx<N>(t + NT * m)); };

  cx<R> a[16], b[16];
  if constexpr (CURL) {
    load_row<N>(a, B.h[HFX], row, live, t);
    fft<N, -1>(a, sh, t, P.tw);
    load_row<N>(b, B.h[HFY], row, live, t);
    fft<N, -1>(b, sh, t, P.tw);
    // N_w = N_w partial + I (kx F[Fy] - ky F[Fx])
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const R kx = kxm(m);
      const R dr = rsub(rmul(kx, b[m].x), rmul(ky, a[m].x));
      const R di = rsub(rmul(kx, b[m].y), rmul(ky, a[m].y));
      const cx<R> p = live ? B.nw[(size_t)row * N + t + NT * m] : czero<R>();
      a[m] = mk<R>(radd(p.x, -di), radd(p.y, dr));
    }
  } else {
    // pure Navier-Stokes: N_w = -F[u.grad w]
    load_row<N>(a, B.h[HA], row, live, t);
    fft<N, -1>(a, sh, t, P.tw);
#pragma unroll
    for (int m = 0; m < 16; m++) a[m] = mk<R>(a[m].x * (R)(-1), a[m].y * (R)(-1));
  }
  if (P.force_j >= 0 && row == P.force_j && t == 0) a[0].x = radd(a[0].x, P.force_hat);
  load_row<N>(b, B.w, row, live, t);
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int am = amask<N, R>(t, m);
    const size_t idx = (size_t)rowc * N + t + NT * m;
    const R e = cf[0 * cstride + am], z1 = cf[1 * cstride + am], z2 = cf[2 * cstride + am];
    cx<R> sv;
    if (STAGE == 2) sv = live ? B.sw[idx] : czero<R>();
    b[m] = etd<STAGE>(b[m], a[m], &sv, e, z1, z2);
    if (STAGE == 1 && live) B.sw[idx] = sv;
    if (F32 && row == 0 && t == 0 && m == 0) {
      etd_k0<STAGE>(P.k0 + 0, P.k0 + 6, (double)a[m].x, (double)a[m].y, P.k0coef, 0);
      b[m] = mk<R>((R)P.k0[0], (R)P.k0[1]);
    }
  }
  store_row<N>(b, B.w, row, live, t);
}

// ---------------------------------------------------------------------------
// layout conversion and plain transforms (fft.c dfft/ifft on the device)
// ---------------------------------------------------------------------------

// FFTW layout (n x (n/2+1), double) -> S layout (R), and back.
template <class R>
__global__ void k_fftw_to_s(const double2* __restrict__ src, cx<R>* __restrict__ dst, int n) {
  __shared__ double2 tile[32][33];
  const int nr = n / 2 + 1;
  const int j0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int i = i0 + k, j = j0 + threadIdx.x;
    if (i < n && j < nr) tile[k][threadIdx.x] = src[(size_t)i * nr + j];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int j = j0 + k, i = i0 + threadIdx.x;
    if (i < n && j < nr) {
      const double2 v = tile[threadIdx.x][k];
      dst[(size_t)j * n + i] = mk<R>((R)v.x, (R)v.y);
    }
  }
}

template <class R>
__global__ void k_s_to_fftw(const cx<R>* __restrict__ src, double2* __restrict__ dst, int n) {
  __shared__ double2 tile[32][33];
  const int nr = n / 2 + 1;
  const int j0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int j = j0 + k, i = i0 + threadIdx.x;
    if (i < n && j < nr) {
      const cx<R> v = src[(size_t)j * n + i];
      tile[threadIdx.x][k] = make_double2((double)v.x, (double)v.y);
    }
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int i = i0 + k, j = j0 + threadIdx.x;
    if (i < n && j < nr) dst[(size_t)i * nr + j] = tile[k][threadIdx.x];
  }
}

// real field (n x n, R, row-major, i = x) -> H layout: y-r2c of x-row pairs
template <int N, class R, int GPC>
__global__ void __launch_bounds__(GPC * (N / 16)) k_row_r2c_plain(const R* __restrict__ x, cx<R>* __restrict__ H,
                                                                  const cx<R>* __restrict__ tw) {
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int pair = blockIdx.x * GPC + g;
  const bool live = pair < N / 2;
  const int i0 = 2 * pair;
  cx<R> v[16];
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int y = t + NT * m;
    v[m] = live ? mk<R>(x[(size_t)i0 * N + y], x[(size_t)(i0 + 1) * N + y]) : czero<R>();
  }
  row_r2c_store<N>(v, H, i0, live, t, sh, tw);
}

// S/H layout row j': x transform in place (DIR), optional scale
template <int N, class R, int GPC, int DIR>
__global__ void __launch_bounds__(GPC * (N / 16)) k_col_plain(const cx<R>* __restrict__ src, cx<R>* __restrict__ dst,
                                                              int nrows, R scale, const cx<R>* __restrict__ tw) {
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int row = blockIdx.x * GPC + g;
  const bool live = row < nrows;
  cx<R> v[16];
  load_row<N>(v, src, row, live, t);
#pragma unroll
  for (int m = 0; m < 16; m++) v[m] = mk<R>(v[m].x * scale, v[m].y * scale);
  fft<N, DIR>(v, sh, t, tw);
  store_row<N>(v, dst, row, live, t);
}

// G layout (all n/2+1 rows) -> real field: y-c2r of x-row pairs
template <int N, class R, int GPC>
__global__ void __launch_bounds__(GPC * (N / 16)) k_row_c2r_plain(const cx<R>* __restrict__ G, R* __restrict__ x,
                                                                  int jt, const cx<R>* __restrict__ tw) {
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int pair = blockIdx.x * GPC + g;
  const bool live = pair < N / 2;
  const int i0 = 2 * pair;
  cx<R> v[16];
  row_c2r<N>(v, G, i0, jt, live, t, sh, tw);
  if (live) {
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int y = t + NT * m;
      x[(size_t)i0 * N + y] = v[m].x;
      x[(size_t)(i0 + 1) * N + y] = v[m].y;
    }
  }
}

}  // namespace chns
