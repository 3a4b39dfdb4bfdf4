// chns_fft.cuh -- register/shared-memory FFT building blocks for sm_100a.
//
// Replaces the reference's FFTW-MPI transforms (fft.c:11-31, plans main.c:193-194).
// A length-N transform (N = 2^p, 32 <= N <= 4096) is done by a "group" of
// NT = N/16 threads; thread t of the group holds the 16 elements
// x[t + NT*m], m = 0..15, in registers.  Stages follow Stockham's autosorting
// decimation-in-time scheme with radix 16 (a radix-2/4/8 stage first when
// log2(N) is not a multiple of 4): every stage reads the pattern x[t + NT*m]
// from shared memory, multiplies by twiddles from a table in global memory,
// does an in-register DFT, and scatters; the last radix-16 stage leaves the
// output in registers, again as X[t + NT*m] (natural order).  One shared-memory
// round trip per stage after the first; the shared array is padded by one
// element every 16 so that all stage patterns are bank-conflict free.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace chns {

template <class R> struct __align__(2 * sizeof(R)) cx {
  R x, y;
};
using cxf = cx<float>;
using cxd = cx<double>;

template <class R> __device__ __forceinline__ cx<R> mk(R a, R b) { cx<R> r; r.x = a; r.y = b; return r; }
template <class R> __device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) { return mk<R>(a.x + b.x, a.y + b.y); }
template <class R> __device__ __forceinline__ cx<R> operator-(cx<R> a, cx<R> b) { return mk<R>(a.x - b.x, a.y - b.y); }
template <class R> __device__ __forceinline__ cx<R> cmul(cx<R> a, cx<R> b) {
  return mk<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <class R> __device__ __forceinline__ cx<R> cmulc(cx<R> a, cx<R> b) {
  return mk<R>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// Rounded arithmetic without contraction: used wherever the reference's
// expression order must be kept (the FFT butterflies are free to use FMA).
static __device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
static __device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
static __device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
static __device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }
static __device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
static __device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
static __device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
static __device__ __forceinline__ float rdiv(float a, float b) { return __fdiv_rn(a, b); }

// multiply by DIR*i: forward transforms use DIR = -1 (kernel exp(-2 pi i jk/N))
template <int DIR, class R> __device__ __forceinline__ cx<R> mul_i(cx<R> a) {
  return DIR < 0 ? mk<R>(a.y, -a.x) : mk<R>(-a.y, a.x);
}

// Butterfly adds.  In FP32 a complex add or subtract is one packed f32x2
// instruction (sm_100a): two IEEE round-to-nearest adds, the results of the
// scalar pair, in half the issue slots of the transforms' dominant operation.
template <class R> __device__ __forceinline__ cx<R> badd(cx<R> a, cx<R> b) { return a + b; }
template <class R> __device__ __forceinline__ cx<R> bsub(cx<R> a, cx<R> b) { return a - b; }
__device__ __forceinline__ cxf badd(cxf a, cxf b) {
  const float2 r = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
  return mk<float>(r.x, r.y);
}
__device__ __forceinline__ cxf bsub(cxf a, cxf b) {
  cxf r;
  asm("{\n\t.reg .b64 p, q, d;\n\tmov.b64 p, {%2, %3};\n\tmov.b64 q, {%4, %5};\n\t"
      "sub.rn.f32x2 d, p, q;\n\tmov.b64 {%0, %1}, d;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}

// t1 + DIR i d and t1 - DIR i d: the swapped components of i d have no packed
// form, so these stay scalar (and need no register moves)
template <int DIR, class R> __device__ __forceinline__ void rot_pm(cx<R>& a, cx<R>& b, cx<R> t1, cx<R> d) {
  if (DIR < 0) {
    a = mk<R>(t1.x + d.y, t1.y - d.x);
    b = mk<R>(t1.x - d.y, t1.y + d.x);
  } else {
    a = mk<R>(t1.x - d.y, t1.y + d.x);
    b = mk<R>(t1.x + d.y, t1.y - d.x);
  }
}

template <int DIR, class R> __device__ __forceinline__ void dft2(cx<R>& a0, cx<R>& a1) {
  cx<R> t = bsub(a0, a1);
  a0 = badd(a0, a1);
  a1 = t;
}

template <int DIR, class R> __device__ __forceinline__ void dft4(cx<R>& a0, cx<R>& a1, cx<R>& a2, cx<R>& a3) {
  const cx<R> t0 = badd(a0, a2), t1 = bsub(a0, a2), t2 = badd(a1, a3), d = bsub(a1, a3);
  a0 = badd(t0, t2);
  a2 = bsub(t0, t2);
  rot_pm<DIR>(a1, a3, t1, d);
}

// dft4 whose third input enters multiplied by DIR i (the W16^4 twiddle of the
// radix-16 and radix-8 stages), folded into the scalar adds
template <int DIR, class R> __device__ __forceinline__ void dft4_i2(cx<R>& a0, cx<R>& a1, cx<R>& a2, cx<R>& a3) {
  cx<R> t0, t1;
  rot_pm<DIR>(t0, t1, a0, a2);  // a0 + DIR i a2, a0 - DIR i a2
  const cx<R> t2 = badd(a1, a3), d = bsub(a1, a3);
  a0 = badd(t0, t2);
  a2 = bsub(t0, t2);
  rot_pm<DIR>(a1, a3, t1, d);
}

// constants of the 16th roots of unity
#define CHNS_C8 0.92387953251128675612818318939678828682241662586364
#define CHNS_S8 0.38268343236508977172845998403039886676134456248563
#define CHNS_R2 0.70710678118654752440084436210484903928483593768847

// v *= W16^(DIR... e), W16 = exp(DIR * 2 pi i / 16) with DIR = -1 forward
template <int DIR, int E, class R> __device__ __forceinline__ cx<R> tw16(cx<R> v) {
  constexpr int e = E & 15;
  const R c8 = (R)CHNS_C8, s8 = (R)CHNS_S8, r2 = (R)CHNS_R2;
  // w = cos(2 pi e/16) + DIR * i sin(2 pi e/16)
  if (e == 0) return v;
  if (e == 4) return mul_i<DIR>(v);
  if (e == 8) return mk<R>(-v.x, -v.y);
  if (e == 12) return mul_i<-DIR>(v);
  R wc, ws;  // cos, sin of 2 pi e / 16
  switch (e) {
    case 1: wc = c8; ws = s8; break;
    case 2: wc = r2; ws = r2; break;
    case 3: wc = s8; ws = c8; break;
    case 5: wc = -s8; ws = c8; break;
    case 6: wc = -r2; ws = r2; break;
    case 7: wc = -c8; ws = s8; break;
    case 9: wc = -c8; ws = -s8; break;
    case 10: wc = -r2; ws = -r2; break;
    case 11: wc = -s8; ws = -c8; break;
    case 13: wc = s8; ws = -c8; break;
    case 14: wc = r2; ws = -r2; break;
    default: wc = c8; ws = -s8; break;  // 15
  }
  ws = DIR < 0 ? -ws : ws;
  return mk<R>(v.x * wc - v.y * ws, v.x * ws + v.y * wc);
}

// In-register DFT of size R_ on v[off + stride*r], r = 0..R_-1; outputs in
// natural order at the same slots.
template <int DIR, int RADIX, int STRIDE, class R> __device__ __forceinline__ void dft(cx<R>* v) {
  if constexpr (RADIX == 2) {
    dft2<DIR>(v[0], v[STRIDE]);
  } else if constexpr (RADIX == 4) {
    dft4<DIR>(v[0], v[STRIDE], v[2 * STRIDE], v[3 * STRIDE]);
  } else if constexpr (RADIX == 8) {
    // 8 = 2 x 4: r = r1 + 2 r2; X[k2 + 4 k1] lands in slot k1 + 2 k2
    cx<R> y[8];
#pragma unroll
    for (int r = 0; r < 8; r++) y[r] = v[r * STRIDE];
    dft4<DIR>(y[0], y[2], y[4], y[6]);
    dft4<DIR>(y[1], y[3], y[5], y[7]);
    y[3] = tw16<DIR, 2>(y[3]);
    y[7] = tw16<DIR, 6>(y[7]);
    dft2<DIR>(y[0], y[1]);
    dft2<DIR>(y[2], y[3]);
    {
      const cx<R> a = y[4], b = y[5];  // (a + DIR i b, a - DIR i b): the W16^4 twiddle folded in
      rot_pm<DIR>(y[4], y[5], a, b);
    }
    dft2<DIR>(y[6], y[7]);
#pragma unroll
    for (int k = 0; k < 8; k++) v[k * STRIDE] = y[(k / 4) + 2 * (k % 4)];
  } else {
    static_assert(RADIX == 16, "radix");
    // 16 = 4 x 4: r = r1 + 4 r2; X[k2 + 4 k1] lands in slot k1 + 4 k2
    cx<R> y[16];
#pragma unroll
    for (int r = 0; r < 16; r++) y[r] = v[r * STRIDE];
#pragma unroll
    for (int r1 = 0; r1 < 4; r1++) dft4<DIR>(y[r1], y[r1 + 4], y[r1 + 8], y[r1 + 12]);
    y[5] = tw16<DIR, 1>(y[5]);
    y[9] = tw16<DIR, 2>(y[9]);
    y[13] = tw16<DIR, 3>(y[13]);
    y[6] = tw16<DIR, 2>(y[6]);
    y[14] = tw16<DIR, 6>(y[14]);
    y[7] = tw16<DIR, 3>(y[7]);
    y[11] = tw16<DIR, 6>(y[11]);
    y[15] = tw16<DIR, 9>(y[15]);
    dft4<DIR>(y[0], y[1], y[2], y[3]);
    dft4<DIR>(y[4], y[5], y[6], y[7]);
    dft4_i2<DIR>(y[8], y[9], y[10], y[11]);  // y[10] carries the W16^4 twiddle
    dft4<DIR>(y[12], y[13], y[14], y[15]);
#pragma unroll
    for (int k = 0; k < 16; k++) v[k * STRIDE] = y[(k / 4) + 4 * (k % 4)];
  }
}

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

// shared-memory slot of element q of one group's buffer (one pad per 16)
static __device__ __forceinline__ int spad(int q) { return q + (q >> 4); }

template <int N> struct FftShape {
  static constexpr int NT = N / 16;                   // threads per transform
  static constexpr int LOGN = ilog2c(N);
  static constexpr int R0 = 1 << (LOGN % 4);         // leading small radix (1 = none)
  static constexpr int N16 = LOGN / 4;               // number of radix-16 stages
  static constexpr int SMEM = N + N / 16;            // complex slots per group
};

// Multiplies u[r], r = 1..15, by w^r (conj for the inverse), w = tw[base]:
// w, w^2, w^4, w^8 are read from the table and the other powers formed by at
// most two complex products.
template <int DIR, class R>
__device__ __forceinline__ void apply_tw16(cx<R>* u, const cx<R>* __restrict__ tw, int base, int mask) {
  const cx<R> w1 = tw[base & mask], w2 = tw[(2 * base) & mask];
  const cx<R> w4 = tw[(4 * base) & mask], w8 = tw[(8 * base) & mask];
  const cx<R> w3 = cmul(w1, w2), w12 = cmul(w8, w4);
  cx<R> w[16];
  w[1] = w1; w[2] = w2; w[3] = w3; w[4] = w4;
  w[5] = cmul(w4, w1); w[6] = cmul(w4, w2); w[7] = cmul(w4, w3);
  w[8] = w8; w[9] = cmul(w8, w1); w[10] = cmul(w8, w2); w[11] = cmul(w8, w3);
  w[12] = w12; w[13] = cmul(w12, w1); w[14] = cmul(w12, w2); w[15] = cmul(w12, w3);
#pragma unroll
  for (int r = 1; r < 16; r++) u[r] = DIR < 0 ? cmul(u[r], w[r]) : cmulc(u[r], w[r]);
}

// Twiddles of the two twiddled stages of a transform, precomputed once per CTA
// and kept in shared memory.  Slot 0 serves the first twiddled radix-16 stage
// (span R0 when R0 > 1, else span 16 when there are three radix-16 stages): its
// base depends only on t mod that span, so it is one table of (at most) 16
// bases x 4 powers shared by the CTA, element (b, q) = w_b^(2^q) at table[4 b + q];
// thread t reads p0[q], p0 = table + 4 (t mod span).  Slot 1 serves the last stage (span
// N/16, base t): thread tid's w^(2^q), q = 0..3, at p1[q * stride], p1 = table
// + 64 + tid.  Slot 0 is first read after the transform's first exchange
// barrier, so its fill needs no barrier of its own.
template <class R> struct Tw {
  const cx<R>* p0;
  const cx<R>* p1;
  int stride;
};

// bytes of the twiddle region of a CTA of `threads` threads
template <int N, class R> __host__ __device__ constexpr size_t tw_smem_bytes(int threads) {
  return (size_t)(64 + 4 * threads) * sizeof(cx<R>);
}

// Fills the CTA's twiddle region from the table tw[q] = exp(-2 pi i q / N)
// (every thread of the CTA calls it).
template <int N, class R>
__device__ __forceinline__ Tw<R> tw_setup(cx<R>* smem, const cx<R>* __restrict__ tw, int t) {
  constexpr int NT = N / 16;
  constexpr int LOGN = ilog2c(N);
  constexpr int R0 = 1 << (LOGN % 4);
  constexpr int N16 = LOGN / 4;
  constexpr bool SLOT0 = (R0 > 1 && N16 >= 2) || N16 >= 3;
  constexpr int SPAN0 = R0 > 1 ? R0 : 16;                       // distinct slot-0 bases
  constexpr int STEP0 = R0 > 1 ? N / (R0 * 16) : N / 256;       // base b is tw[b STEP0]
  const int tid = threadIdx.x, stride = blockDim.x;
  if (SLOT0) {
    for (int e = tid; e < 4 * SPAN0; e += stride) smem[e] = tw[(((e / 4) * STEP0) << (e % 4)) & (N - 1)];
  }
  cx<R>* p1 = smem + 64 + tid;
  if (NT > 1) {
#pragma unroll
    for (int q = 0; q < 4; q++) p1[q * stride] = tw[(t << q) & (N - 1)];
  }
  return Tw<R>{smem + 4 * (t % SPAN0), p1, stride};
}

// Multiplies u[r], r = 1..15, by w^r (conj for the inverse) from the
// precomputed w, w^2, w^4, w^8 of `slot`; other powers by at most two products.
template <int DIR, class R>
__device__ __forceinline__ void apply_tw16_pre(cx<R>* u, const Tw<R>& T, int slot) {
  cx<R> w1, w2, w4, w8;
  if (slot == 0) {
    w1 = T.p0[0]; w2 = T.p0[1]; w4 = T.p0[2]; w8 = T.p0[3];
  } else {
    w1 = T.p1[0]; w2 = T.p1[T.stride]; w4 = T.p1[2 * T.stride]; w8 = T.p1[3 * T.stride];
  }
  const cx<R> w3 = cmul(w1, w2), w12 = cmul(w8, w4);
  cx<R> w[16];
  w[1] = w1; w[2] = w2; w[3] = w3; w[4] = w4;
  w[5] = cmul(w4, w1); w[6] = cmul(w4, w2); w[7] = cmul(w4, w3);
  w[8] = w8; w[9] = cmul(w8, w1); w[10] = cmul(w8, w2); w[11] = cmul(w8, w3);
  w[12] = w12; w[13] = cmul(w12, w1); w[14] = cmul(w12, w2); w[15] = cmul(w12, w3);
#pragma unroll
  for (int r = 1; r < 16; r++) u[r] = DIR < 0 ? cmul(u[r], w[r]) : cmulc(u[r], w[r]);
}

// One Stockham stage: radix RADIX, span NS (product of the earlier radices).
// v holds x[t + NT*m]; writes the stage output to sh (padded).
template <int N, int DIR, int RADIX, int NS, class R>
__device__ __forceinline__ void fft_stage_to_smem(cx<R>* v, cx<R>* sh, int t, const Tw<R>& tw) {
  constexpr int NT = N / 16;
  constexpr int B = 16 / RADIX;  // butterflies per thread
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + NT * b;
    const int k = j % NS;
    cx<R> u[RADIX];
#pragma unroll
    for (int r = 0; r < RADIX; r++) u[r] = v[b + r * B];
    if (NS > 1) {
      // twiddles W_{NS*RADIX}^{k r} = tw[k r N/(NS RADIX)] (conjugated for the inverse)
      static_assert(NS == 1 || RADIX == 16, "twiddled stages are radix 16");
      apply_tw16_pre<DIR>(u, tw, 0);
    }
    dft<DIR, RADIX, 1>(u);
    const int base = (j / NS) * NS * RADIX + k;
#pragma unroll
    for (int q = 0; q < RADIX; q++) sh[spad(base + q * NS)] = u[q];
  }
}

template <int N, class R>
__device__ __forceinline__ void fft_load_smem(cx<R>* v, const cx<R>* sh, int t) {
  constexpr int NT = N / 16;
#pragma unroll
  for (int m = 0; m < 16; m++) v[m] = sh[spad(t + NT * m)];
}

// Last radix-16 stage (NS = N/16): result stays in registers in natural order.
template <int N, int DIR, class R>
__device__ __forceinline__ void fft_last_stage(cx<R>* v, int t, const Tw<R>& tw) {
  constexpr int NS = N / 16;
  if (NS > 1) apply_tw16_pre<DIR>(v, tw, 1);  // j = t < NS, twiddles tw[t r]
  dft<DIR, 16, 1>(v);
}

// Full transform of one group.  All threads of the CTA must call it together
// (it uses __syncthreads); sh is this group's padded buffer of FftShape<N>::SMEM.
// The leading barrier protects the buffer from the previous transform's readers;
// LEAD = false drops it where the caller has just passed a barrier that every
// earlier reader of the buffer had reached.
template <int N, int DIR, class R, bool LEAD = true>
__device__ __forceinline__ void fft(cx<R>* v, cx<R>* sh, int t, const Tw<R>& tw) {
  using S = FftShape<N>;
  if constexpr (S::N16 == 1 && S::R0 == 1) {
    fft_last_stage<N, DIR>(v, t, tw);  // N = 16: single stage
  } else {
    if constexpr (S::R0 > 1) {
      if (LEAD) __syncthreads();
      fft_stage_to_smem<N, DIR, S::R0, 1>(v, sh, t, tw);
      __syncthreads();
      fft_load_smem<N>(v, sh, t);
    }
    if constexpr (S::N16 >= 2) {
      if (LEAD || S::R0 > 1) __syncthreads();
      fft_stage_to_smem<N, DIR, 16, S::R0>(v, sh, t, tw);
      __syncthreads();
      fft_load_smem<N>(v, sh, t);
    }
    if constexpr (S::N16 >= 3) {
      __syncthreads();
      fft_stage_to_smem<N, DIR, 16, S::R0 * 16>(v, sh, t, tw);
      __syncthreads();
      fft_load_smem<N>(v, sh, t);
    }
    static_assert(S::N16 <= 3, "N <= 4096");
    fft_last_stage<N, DIR>(v, t, tw);
  }
}

}  // namespace chns
