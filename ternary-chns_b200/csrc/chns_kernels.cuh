// chns_kernels.cuh -- the fused passes of one ETD2RK stage on sm_100a.
//
// Data layout in HBM (see also chns_api.cu):
//   S layout : spectral field, row j' (ky index 0..n/2) of n complex along kx
//              (the transpose of FFTW's n x (n/2+1) layout, global.h:13-14), so
//              the x transforms read and write contiguous rows.
//   G layout : fields after the x inverse transform, rows 0..jt only (jt = the
//              last ky row that survives the truncation, functions.c:47-84).
//   H layout : fields after the y forward transform, rows 0..n/2.
//   A "pair field" interleaves two fields of the same x index: element
//   [row][2 i + e], e = 0, 1 (row stride 2n).  The y transform of a pair field
//   at x-row i is one complex transform of z = f0 + i f1, so products such as
//   u.grad w = Re(z_uv) Re(z_w) + Im(z_uv) Im(z_w) come straight out of two
//   transforms.  A "plain" field (row stride n) is transformed two x-rows at a
//   time, z = f(i0) + i f(i0+1).
//
// One stage (etd2rk.c:28-135 or :146-212) of the binary model is five kernels:
//   P1 spec_inv    : S -> G : velocity, gradients, truncation, 1/(nx ny), x-iFFT
//   P2 row_adv     : G -> H : y-c2r, u.grad w, u.grad c, f(c), y-r2c
//   P3 spec_fwd_c  : H -> S, G : x-FFT; -F[u.grad w]; mu and its x-iFFT; N_c; ETD of c
//   P4 row_force   : G -> H : y-c2r of mu and grad c, mu grad c, y-r2c
//   P5 spec_curl_w : H -> S : x-FFT; curl; N_w; ETD of w
// Ternary adds the chemical potential (chem_potential.c) to P2.  Pure
// Navier-Stokes is P1, P2 and P5 without the curl.
//
// The row passes stream their inputs through a shared-memory tile filled by TMA
// (cp.async per thread where no tensor map exists): the copy of the next
// transform's input is in flight while the current transform runs.  With a
// float-pair state (FP32 contexts) P3 / P5 also update the state's low parts.
#pragma once

#include <cuda.h>  // CUtensorMap

#include "chns_fft.cuh"

namespace chns {

enum { MODEL_NS = 0, MODEL_BINARY = 1, MODEL_TERNARY = 2 };

// G slots: pair fields (u,v), (dx w, dy w), (dx c1, dy c1), (dx c2, dy c2);
// GCT truncated c (binary plain, ternary pair (c1,c2)); GMU mu (binary plain,
// ternary pair (mu1, mu2)).  Every slot holds rows 0..jt of width 2n.
enum { GUV = 0, GW, GD1, GD2, GCT, GMU, NG };
// H slots: HAB ternary pair (A, B1) = (u.grad w, u.grad c1), binary plain A then
// plain B1 behind it, pure Navier-Stokes plain A; HF binary plain f(c), ternary
// pair (mu^F_1, mu^F_2); HB2 plain u.grad c2; HFF ternary pair (Fx, Fy), binary
// plain Fx then plain Fy behind it.  Every slot holds rows 0..n/2 of width 2n.
enum { HAB = 0, HF, HB2, HFF, NH };

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
  const R* filt;           // SMOOTH_FILTER factors [n/2+1 rows][n/2+1 |m|] (null: the sharp cut)
  const R* coef;           // [6][n/2+1][n/2+1] ETD coefficients at (row, |m|); with a
                           // double-float state, slots 0 and 3 hold e - 1 (expm1) instead of e
  const cx<R>* tw;         // tw[q] = exp(-2 pi i q / n)
  double* k0;              // FP32 only: k = 0 modes in double [w, c1, c2, sw, s1, s2] x (re, im)
  unsigned int* err;       // bit 0: a bounded wait for an asynchronous copy ran out
};

template <class R> struct Bufs {
  cx<R>* w;
  cx<R>* c1;
  cx<R>* c2;
  cx<R>* sw;
  cx<R>* s1;
  cx<R>* s2;
  cx<R>* xw;   // stage 2: N(u*) of w, c1, c2 stored here when not null
  cx<R>* x1;
  cx<R>* x2;
  cx<R>* nw;
  cx<R>* lo[3];  // FP32 contexts with a double-float state: low parts of w, c1, c2 (else null)
  cx<R>* gr;     // (dx c_i, dy c_i) in real space, [field][x-row][y]: written by P2, read by P4
  R* rec;        // binary REC kernels: the adjoint's record of this right-hand side, n x n real
                 // fields c_t, u, v, wx, wy, cx, cy, mu, then F[f(c_t)] in the S layout
  cx<R>* g[NG];
  cx<R>* h[NH];
};

// FP32 step kernels are built for two CTAs per SM (<= 128 registers), FP64 for one
#define CHNS_STEP_BOUNDS(N, R, GPC) __launch_bounds__((GPC) * ((N) / 16), sizeof(R) == 4 ? 2 : 1)

// The five stage kernels are kernels of their own (one launch per pass), or, in a
// translation unit that defines CHNS_STAGE_BODIES before including this header,
// device functions of the same text that a persistent kernel calls once per
// virtual CTA: there CHNS_BX / CHNS_BY read that CTA's index from chns_vblock
// (a shared int[2] that translation unit declares before the include and sets,
// followed by a barrier, before each call) instead of blockIdx.
// CHNS_GRID_DEP: a stage kernel launched with programmatic stream serialization
// (the context's PDL choice) may be scheduled while the kernel before it ends;
// every access to the step's buffers follows this wait for that kernel's
// completion (a no-op for an ordinary launch).  The next kernel is released
// when this one's CTAs exit (an earlier release, right after the wait, made the
// waiting CTAs of the next kernel crowd the SMs: up to 34% slower at 512^2).
// Only the twiddle table, never written by a kernel, is read before it.
#ifdef CHNS_STAGE_BODIES
#define CHNS_GRID_DEP() ((void)0)
#else
#define CHNS_GRID_DEP() asm volatile("griddepcontrol.wait;\n" ::: "memory")
#endif

#ifdef CHNS_STAGE_BODIES
#define CHNS_STAGE_KERNEL(N, R, GPC) __device__ __forceinline__ void
#define CHNS_TMAG_PARAM const TmaG&
#define CHNS_BUFS_PARAM const Bufs<R>&
#define CHNS_PAR_PARAM const Par<R>&
#define CHNS_BX chns_vblock[0]
#define CHNS_BY chns_vblock[1]
#else
#define CHNS_STAGE_KERNEL(N, R, GPC) __global__ void CHNS_STEP_BOUNDS(N, R, GPC)
#define CHNS_TMAG_PARAM const __grid_constant__ TmaG
#define CHNS_BUFS_PARAM const Bufs<R>
#define CHNS_PAR_PARAM const Par<R>
#define CHNS_BX blockIdx.x
#define CHNS_BY blockIdx.y
#endif

template <class R> __device__ __forceinline__ cx<R> czero() { return mk<R>((R)0, (R)0); }

// signed wavenumber index of column i (functions.c:17-24: Nyquist positive)
template <int N> __device__ __forceinline__ int sidx(int i) { return i <= N / 2 ? i : i - N; }

template <class R> __device__ __forceinline__ R ksq(R kx, R ky) { return radd(rmul(kx, kx), rmul(ky, ky)); }

// SMOOTH_FILTER's truncation of one mode (functions.c:69-72): two products by the
// filter factor f, each rounded
template <class R> __device__ __forceinline__ cx<R> smooth2(cx<R> a, R f) {
  a = mk<R>(rmul(a.x, f), rmul(a.y, f));
  return mk<R>(rmul(a.x, f), rmul(a.y, f));
}

// ---------------------------------------------------------------------------
// asynchronous tile copies (cp.async, 16 bytes each) into shared memory
// ---------------------------------------------------------------------------
static __device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
static __device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
static __device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// The input of one y inverse transform: two complex values per G row k at
// base[k * stride + off .. + 1] (a pair field at x-row i: stride 2n, off 2i;
// a plain field at x-rows i0, i0+1: stride n, off i0).
template <class R> struct RowSrc {
  const cx<R>* base;
  int stride, off;
  int map;  // tensor map of the source (TmaG::map), -1: none
};



// Group-cooperative copy of rows 0..jt of `s` into this group's tile
// (2 complex per row) with cp.async; the caller commits.
template <int N, class R>
__device__ __forceinline__ void tile_issue(cx<R>* tile, RowSrc<R> s, int jt, bool live, int t) {
  constexpr int NT = N / 16;
  constexpr int CH = (int)(2 * sizeof(cx<R>) / 16);  // 16-byte chunks per row
  if (!live) return;
  for (int q = t; q < (jt + 1) * CH; q += NT) {
    const int r = q / CH, c = q % CH;
    cp_async16(reinterpret_cast<char*>(tile + 2 * r) + 16 * c,
               reinterpret_cast<const char*>(s.base + (size_t)r * s.stride + s.off) + 16 * c);
  }
}

// Builds Z = X0 + i X1 with the Hermitian extension from a tile (Im of the ky = 0
// and ky = n/2 bins ignored: FFTW's c2r convention).  v[m] holds Z[t + NT m].
template <int N, class R>
__device__ __forceinline__ void build_c2r_input(cx<R>* v, const cx<R>* tile, int jt, int t) {
  constexpr int NT = N / 16;
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int k = t + NT * m;
    const bool cj = k > N / 2;
    const int kk = cj ? N - k : k;
    cx<R> a = czero<R>(), b = czero<R>();
    if (kk <= jt) {
      a = tile[2 * kk];
      b = tile[2 * kk + 1];
    }
    if (kk == 0 || kk == N / 2) { a.y = (R)0; b.y = (R)0; }
    v[m] = cj ? mk<R>(a.x + b.y, b.x - a.y) : mk<R>(a.x - b.y, a.y + b.x);
  }
}

// ---------------------------------------------------------------------------
// TMA tiles of the step's row kernels.  One 2D tensor map per G slot and view
// (pair fields: rows of 2n complex; plain fields: rows of n complex) over rows
// 0..jt, with 64-bit elements (one FP32 complex value, half an FP64 one); a tile
// is nbox boxes of {2 complex, boxr rows} (16 bytes a row in FP32, 32 in FP64),
// rows beyond jt zero-filled.
// One thread per group issues the boxes on the group's mbarrier; every thread
// of the group waits on it (bounded: on timeout the kernel flags *err and goes
// on, so a broken copy ends in an error status, not a hang).
// ---------------------------------------------------------------------------
struct __align__(64) TmaG {
  CUtensorMap map[2 * NG];  // [2 slot + 0]: pair view, [2 slot + 1]: plain view
  int use;                  // maps built; 0: cp.async tiles
  int boxr, nbox;           // rows per box, boxes per tile (nbox * boxr >= jt + 1)
  int ecx;                  // 64-bit elements per complex value (1: FP32, 2: FP64)
  unsigned int* err;        // bit 0: an mbarrier wait timed out
  int spins;                // try_wait rounds of a tile wait (0: kMbarSpins)
  int skip;                 // test hook: issue no tile copies (every tile wait then runs out)
};
constexpr int kMbarSpins = 1 << 18;  // try_wait rounds before a tile wait gives up

static __device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
static __device__ __forceinline__ void mbar_init(uint64_t* mb) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(mb)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// waits for the phase of parity `par` to complete; false on timeout
static __device__ __forceinline__ bool mbar_wait(uint64_t* mb, unsigned par, int spins = kMbarSpins) {
  unsigned ok = 0;
  for (int k = 0; k < spins && !ok; k++)
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(mb)), "r"(par)
        : "memory");
  return ok != 0;
}
// one tile (nbox boxes) of map `map` at complex column x into `tile`, completing on mb
static __device__ __forceinline__ void tma_tile(void* tile, const TmaG& T, int map, int x, uint64_t* mb) {
  const unsigned rowb = (unsigned)(16 * T.ecx);  // bytes of a tile row: two complex values
  const unsigned bytes = (unsigned)(T.nbox * T.boxr) * rowb;
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // earlier generic reads of the tile
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(mb)), "r"(bytes)
               : "memory");
  for (int b = 0; b < T.nbox; b++)
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];\n" ::"r"(smem_u32(tile) + (unsigned)(b * T.boxr) * rowb),
        "l"(reinterpret_cast<uint64_t>(&T.map[map])), "r"(x * T.ecx), "r"(b * T.boxr), "r"(smem_u32(mb))
        : "memory");
}

// One contiguous block (bytes a multiple of 16, both addresses 16-byte aligned)
// into shared memory by the bulk-copy engine, completing on mb; one thread
// issues it.  The fence orders the block's earlier generic-proxy reads (made
// before the barrier that precedes this call) before the asynchronous write.
static __device__ __forceinline__ void bulk_copy(void* smem, const void* gmem, unsigned bytes, uint64_t* mb) {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(mb)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(smem)),
               "l"(gmem), "r"(bytes), "r"(smem_u32(mb))
               : "memory");
}

// Two row buffers of a spectral pass, each refilled by bulk copy while the
// group transforms what it read from the other: the copy of the next input row
// is in flight during a transform instead of its load latency following it.
// Every wait is bounded; one that runs out sets bit 0 of *err.
template <class R> struct RowPrefetch {
  cx<R>* buf[2];
  uint64_t* mb;
  unsigned par[2];
  unsigned int* err;
  bool issuer, live;
  __device__ __forceinline__ void start(int b, const cx<R>* row, int n) {
    if (issuer && live) bulk_copy(buf[b], row, (unsigned)(n * sizeof(cx<R>)), mb + b);
  }
  __device__ __forceinline__ void wait(int b) {
    if (live && !mbar_wait(mb + b, par[b])) atomicOr(err, 1u);
    par[b] ^= 1u;
  }
  template <int N> __device__ __forceinline__ void read(int b, cx<R>* v, int t) const {
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = buf[b][t + (N / 16) * m];
  }
};

// Row buffers of the prefetching spectral passes (binary P3 / P5 in FP32): two
// rows of N complex per group, then their mbarriers.
template <int N, class R, int GPC> __host__ __device__ constexpr size_t prefetch_smem() {
  return (size_t)GPC * 2 * N * sizeof(cx<R>) + (size_t)GPC * 2 * sizeof(uint64_t);
}
template <int N, class R, int GPC>
__device__ __forceinline__ RowPrefetch<R> prefetch_setup(unsigned char* raw, int g, int t, bool live,
                                                         unsigned int* err) {
  cx<R>* pf = reinterpret_cast<cx<R>*>(raw);
  uint64_t* mb = reinterpret_cast<uint64_t*>(raw + (size_t)GPC * 2 * N * sizeof(cx<R>)) + 2 * g;
  if (t == 0) {
    mbar_init(mb);
    mbar_init(mb + 1);
  }
  return RowPrefetch<R>{{pf + (size_t)(2 * g) * N, pf + (size_t)(2 * g + 1) * N}, mb, {0u, 0u}, err, t == 0, live};
}

// Tile state of a row kernel: TMA (contexts with tensor maps) or cp.async.
template <class R> struct TileLoader {
  bool tma;
  uint64_t* mb;  // this group's mbarrier (TMA)
  unsigned par;  // parity of the next phase to wait for
};

// Starts the copy of `s` into `tile` (group g, thread t of the group).
template <int N, class R>
__device__ __forceinline__ void tile_start(TileLoader<R>& L, const TmaG& T, cx<R>* tile, RowSrc<R> s, int jt,
                                           bool live, int t) {
  if (L.tma) {
    if (t == 0 && live && !T.skip) tma_tile(tile, T, s.map, s.off, L.mb);
  } else {
    tile_issue<N>(tile, s, jt, live, t);
    cp_async_commit();
  }
}

// Waits for the copy in flight to `tile` (every thread of the group).
template <class R>
__device__ __forceinline__ void tile_wait(TileLoader<R>& L, const TmaG& T, bool live) {
  if (L.tma) {
    if (live && !mbar_wait(L.mb, L.par, T.spins > 0 ? T.spins : kMbarSpins)) atomicOr(T.err, 1u);
    L.par ^= 1u;
  } else {
    cp_async_wait_all();
  }
}

// build_c2r_input for the reference's cut with a square box (jt = N/4, known at
// compile time): the rows that can be nonzero are fixed per slot m, so no slot
// tests jt or chooses between a row and its conjugate at run time.  Slots 0..3
// read rows k = t + NT m < N/4; slot 4 only row N/4 (t = 0); slots 5..11 lie
// beyond the cut on both sides (zero); slots 12..15 are the conjugates of rows
// N - k in 1..N/4.  Only row 0 (t = 0, m = 0) has its imaginary part dropped.
template <int N, class R>
__device__ __forceinline__ void build_c2r_input_q(cx<R>* v, const cx<R>* tile, int t) {
  constexpr int NT = N / 16;
#pragma unroll
  for (int m = 0; m < 16; m++) {
    if (m >= 5 && m <= 11) {
      v[m] = czero<R>();
      continue;
    }
    const int k = t + NT * m;
    const int kk = m >= 12 ? N - k : k;
    cx<R> a, b;
    if (m == 4 && t != 0) {
      a = czero<R>();
      b = czero<R>();
    } else {
      a = tile[2 * kk];
      b = tile[2 * kk + 1];
    }
    if (m == 0 && t == 0) { a.y = (R)0; b.y = (R)0; }
    v[m] = m >= 12 ? mk<R>(a.x + b.y, b.x - a.y) : mk<R>(a.x - b.y, a.y + b.x);
  }
}

// row_c2r_tiled with the row kernels' tile loader (TMA or cp.async).  With TMA
// every thread has waited on the tile's mbarrier itself, so the tile needs no
// barrier before it is read; the barrier after the reads (before the next copy
// may overwrite the tile) also serves as the transform's leading barrier.
// JT4: the context's cut is the reference's square-box one (jt = N/4).
template <int N, class R, bool JT4 = false>
__device__ __forceinline__ void row_c2r_loaded(cx<R>* v, cx<R>* tile, TileLoader<R>& L, const TmaG& T,
                                               bool has_next, RowSrc<R> next, int jt, bool live, int t, cx<R>* sh,
                                               const Tw<R>& tw) {
  tile_wait(L, T, live);
  if (!L.tma) __syncthreads();
  if (JT4) build_c2r_input_q<N>(v, tile, t);
  else build_c2r_input<N>(v, tile, jt, t);
  __syncthreads();
  if (has_next) tile_start<N>(L, T, tile, next, jt, live, t);
  fft<N, +1, R, false>(v, sh, t, tw);
}

// Inverse y transform of the input already in flight to `tile`; issues the
// copy of `next` (when has_next) as soon as the tile has been read.  Output:
// v[m] = (f0[y], f1[y]) at y = t + NT m.
template <int N, class R>
__device__ __forceinline__ void row_c2r_tiled(cx<R>* v, cx<R>* tile, bool has_next, RowSrc<R> next, int jt,
                                              bool live, int t, cx<R>* sh, const Tw<R>& tw) {
  cp_async_wait_all();
  __syncthreads();
  build_c2r_input<N>(v, tile, jt, t);
  __syncthreads();  // also the transform's leading barrier
  if (has_next) {
    tile_issue<N>(tile, next, jt, live, t);
    cp_async_commit();
  }
  fft<N, +1, R, false>(v, sh, t, tw);
}

// two adjacent complex values (one 16-byte access in FP32)
static __device__ __forceinline__ void st_pair(cxf* p, cxf a, cxf b) {
  *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
static __device__ __forceinline__ void st_pair(cxd* p, cxd a, cxd b) {
  reinterpret_cast<double2*>(p)[0] = make_double2(a.x, a.y);
  reinterpret_cast<double2*>(p)[1] = make_double2(b.x, b.y);
}

// Forward y transform of v = f0 + i f1, split into the two half spectra and
// stored as (F0[k], F1[k]) at base[k * stride + off .. + 1], k = 0..n/2.
template <int N, class R>
__device__ __forceinline__ void row_r2c_store(cx<R>* v, cx<R>* __restrict__ base, int stride, int off, bool live,
                                              int t, cx<R>* sh, const Tw<R>& tw) {
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
      if (live) st_pair(base + (size_t)k * stride + off, A, B);
    }
  }
}

// thread-private real slots in shared memory: element m of thread t at [t + NT m]
template <int N, class R> struct Frag {
  R* p;
  __device__ __forceinline__ R& operator[](int m) const { return p[(threadIdx.x % (N / 16)) + (N / 16) * m]; }
};

// shared memory of a row kernel: GPC transform buffers, GPC tiles, NFRAG real frags per group
template <int N, class R, int GPC> struct RowSmem {
  cx<R>* sh;
  cx<R>* tile;
  R* frag;
  __device__ __forceinline__ RowSmem(unsigned char* raw, int g, int jt) {
    cx<R>* base = reinterpret_cast<cx<R>*>(raw);
    sh = base + g * FftShape<N>::SMEM;
    tile = base + GPC * FftShape<N>::SMEM + (size_t)g * 2 * (jt + 1);
    frag = reinterpret_cast<R*>(base + GPC * FftShape<N>::SMEM + (size_t)GPC * 2 * (jt + 1)) + (size_t)g * N;
  }
  static __host__ __device__ size_t bytes(int jt, int nfrag) {
    return (size_t)GPC * FftShape<N>::SMEM * sizeof(cx<R>) + (size_t)GPC * 2 * (jt + 1) * sizeof(cx<R>) +
           (size_t)nfrag * GPC * N * sizeof(R);
  }
};

// Shared-memory layout of a row kernel with a tile loader: RowSmem after the
// twiddles (aligned to 128 bytes for TMA: the launch adds 128 bytes of slack),
// then one mbarrier per group.  tjt: last tile row (TMA tiles are whole boxes).
template <int N, class R, int GPC> struct LoadedRowSmem {
  RowSmem<N, R, GPC> S;
  uint64_t* mb;
  __device__ __forceinline__ LoadedRowSmem(unsigned char* raw, int g, int tjt, int nfrag)
      : S(raw, g, tjt), mb(reinterpret_cast<uint64_t*>(raw + RowSmem<N, R, GPC>::bytes(tjt, nfrag)) + g) {}
};
static __device__ __forceinline__ unsigned char* align128(unsigned char* p) {
  return p + ((128u - (smem_u32(p) & 127u)) & 127u);
}
// TMA tiles are used when the context has tensor maps and every group's
// tile and box starts on 128 bytes once the layout's base is aligned: the
// transform buffers and the tiles must be whole multiples of 128 bytes.
template <int N, class R, int GPC>
__device__ __forceinline__ bool tma_tiles_ok(const TmaG& T, const unsigned char* /*raw*/) {
  if (!T.use || T.ecx != (int)(sizeof(R) / 4)) return false;
  const size_t sh_bytes = (size_t)GPC * FftShape<N>::SMEM * sizeof(cx<R>);
  const size_t box_bytes = (size_t)T.boxr * 2 * sizeof(cx<R>);
  return sh_bytes % 128 == 0 && box_bytes % 128 == 0;
}
// bytes of a row kernel's shared memory after the twiddles
template <int N, class R, int GPC> size_t loaded_row_smem_bytes(bool tma, int jt, int boxr, int nbox, int nfrag) {
  const int tjt = tma ? nbox * boxr - 1 : jt;
  return RowSmem<N, R, GPC>::bytes(tjt, nfrag) + (size_t)GPC * sizeof(uint64_t) + (tma ? 128 : 0);
}

// ---------------------------------------------------------------------------
// spectral-pass helpers
// ---------------------------------------------------------------------------

template <int N, class R>
__device__ __forceinline__ void load_row(cx<R>* v, const cx<R>* __restrict__ src, int row, bool live, int t) {
  constexpr int NT = N / 16;
#pragma unroll
  for (int m = 0; m < 16; m++) v[m] = live ? src[(size_t)row * N + t + NT * m] : czero<R>();
}

// element e of a pair field's row: src[row][2 i + e]
template <int N, class R>
__device__ __forceinline__ void load_row_pair(cx<R>* v, const cx<R>* __restrict__ src, int row, int e, bool live,
                                              int t) {
  constexpr int NT = N / 16;
#pragma unroll
  for (int m = 0; m < 16; m++) v[m] = live ? src[(size_t)row * 2 * N + 2 * (t + NT * m) + e] : czero<R>();
}

template <int N, class R>
__device__ __forceinline__ void store_row(const cx<R>* v, cx<R>* __restrict__ dst, int row, bool live, int t) {
  constexpr int NT = N / 16;
  if (live) {
#pragma unroll
    for (int m = 0; m < 16; m++) dst[(size_t)row * N + t + NT * m] = v[m];
  }
}

template <int N, class R>
__device__ __forceinline__ void store_row_pair(const cx<R>* v, cx<R>* __restrict__ dst, int row, int e, bool live,
                                               int t) {
  constexpr int NT = N / 16;
  if (live) {
#pragma unroll
    for (int m = 0; m < 16; m++) dst[(size_t)row * 2 * N + 2 * (t + NT * m) + e] = v[m];
  }
}

// REC: x-row xr of recorded real field k (the real or imaginary parts of v)
template <int N, class R>
__device__ __forceinline__ void rec_row(R* rec, int k, int xr, const cx<R>* v, bool im, bool live, int t) {
  constexpr int NT = N / 16;
  if (!live) return;
  R* d = rec + (size_t)k * N * N + (size_t)xr * N + t;
#pragma unroll
  for (int m = 0; m < 16; m++) d[NT * m] = im ? v[m].y : v[m].x;
}

template <int N> __device__ __forceinline__ int amask(int t, int m) {
  const int ms = sidx<N>(t + (N / 16) * m);
  return ms < 0 ? -ms : ms;
}

// ---------------------------------------------------------------------------
// P1: spectral fan-out + x inverse transform   (S -> G)
// nonlin.c:30-48, velocity.c:12-42, surface_tension.c:20-22,57-75,
// nonlin.c:177-198,259-284, chem_potential.c:256-261
// ---------------------------------------------------------------------------
// SPLIT: P1 runs two CTAs per row (grid.y = 2), each with half of the outputs
// (the launcher's choice per grid size, chns_tuned.h; this default is the
// persistent ensemble kernel's)
template <int N> constexpr bool spec_inv_split() { return N <= 1024; }

template <int N, class R, int GPC, int MODEL, bool SPLIT = spec_inv_split<N>()>
CHNS_STAGE_KERNEL(N, R, GPC) k_spec_inv(CHNS_BUFS_PARAM B, CHNS_PAR_PARAM P) {
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), P.tw, t);
  CHNS_GRID_DEP();
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int row = CHNS_BX * GPC + g;
  const bool live = row <= P.jt;
  const int mlim = live ? P.mrow[row] : -1;
  const R ky = (R)(P.fy * (double)row);
  const R sc = P.scale;

  uint32_t inmask = 0;
#pragma unroll
  for (int m = 0; m < 16; m++)
    if (amask<N>(t, m) <= mlim) inmask |= 1u << m;
  auto kxm = [&](int m) -> R { return (R)(P.fx * (double)sidx<N>(t + NT * m)); };

  cx<R> in[16], v[16];
  // outputs: 0 u, 1 v (velocity.c:12-42), 2 dx w, 3 dy w (nonlin.c:36-37); then per
  // phase field: c_t (surface_tension.c:20-22, nonlin.c:217, chem_potential.c:256-261),
  // dx c, dy c (surface_tension.c:57-58, nonlin.c:187-188, 272-273, 314-315).
  // One loop with one inverse transform keeps the kernel small.  The y derivative
  // of c commutes with the x transform (ky is constant along the row), so dy c is
  // i ky times the transformed c_t and gets no transform of its own.
  // SPLIT divides the outputs between the two CTAs of a row (CHNS_BY), half
  // the transforms each: twice the CTAs for rows too few to fill the GPU
  // (measured: 5-8% more steps/s at 256^2-1024^2; at 4096^2 the second read of
  // the input row costs more than it gains).
  // The vorticity's outputs run in the order dx w, dy w, u, v so that w can be
  // turned into psi = w / k^2 in place once (velocity.c:12-42) for both u and v.
  constexpr int NOUT = MODEL == MODEL_NS ? 4 : (MODEL == MODEL_BINARY ? 7 : 10);
  constexpr int OSPLIT = SPLIT ? (MODEL == MODEL_NS ? 2 : (MODEL == MODEL_BINARY ? 3 : 4)) : NOUT;
  const int obeg = CHNS_BY == 0 ? 0 : OSPLIT, oend = CHNS_BY == 0 ? OSPLIT : NOUT;
  bool loaded = false;
#pragma unroll 1
  for (int idx = 0; idx < NOUT; idx++) {
    const int o = idx < 4 ? (idx + 2) % 4 : idx;  // 2, 3, 0, 1, 4, 5, ...
    if (o < obeg || o >= oend) continue;
    if (o == 6 || o == 9) continue;  // dy c: stored with c_t
    if (!loaded || o == 4 || o == 7) {
      const cx<R>* src = o < 4 ? B.w : (o < 7 ? B.c1 : B.c2);
#pragma unroll
      for (int m = 0; m < 16; m++)
        in[m] = ((inmask >> m) & 1) ? src[(size_t)row * N + t + NT * m] : czero<R>();
      // SMOOTH_FILTER: every output of this field is truncated once, so the loaded
      // row is filtered once (the products by f commute with the derivative and
      // velocity factors up to rounding)
      if (P.filt && live) {
        const R* fr = P.filt + (size_t)row * (N / 2 + 1);
#pragma unroll
        for (int m = 0; m < 16; m++) in[m] = smooth2(in[m], fr[amask<N>(t, m)]);
      }
      loaded = true;
    }
    const int q = o < 4 ? o : 4 + (o - 4) % 3;  // 0 u, 1 v, 2 dx, 3 dy (w); 4 c_t, 5 dx, 6 dy (c)
    if (q < 2) {
      // u = I ky psi, v = -I kx psi, psi = w / k^2 (0 where k^2 <= 1e-12)
      if (q == 0) {
#pragma unroll
        for (int m = 0; m < 16; m++) {
          const R ks = ksq(kxm(m), ky);
          in[m] = ks > (R)1e-12 ? mk<R>(rdiv(in[m].x, ks), rdiv(in[m].y, ks)) : czero<R>();
        }
      }
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const R kx = kxm(m), a = in[m].x, b = in[m].y;
        v[m] = q == 0 ? mk<R>(-rmul(ky, b) * sc, rmul(ky, a) * sc) : mk<R>(rmul(kx, b) * sc, -rmul(kx, a) * sc);
      }
    } else if (q == 4) {
#pragma unroll
      for (int m = 0; m < 16; m++) v[m] = mk<R>(in[m].x * sc, in[m].y * sc);
      // ternary FP32 with the sharp cut: c_t without its mean (the k = 0 mode, kept
      // in double and added back in P2's deviation form of mu^F), so that the float
      // transforms round relative to the concentrations' fluctuations rather than to
      // their means (see mu_ternary_dev)
      if (MODEL == MODEL_TERNARY && sizeof(R) == 4 && !P.filt && row == 0 && t == 0) v[0] = czero<R>();
    } else {
      // I kx f, I ky f
      const bool dx = q == 2 || q == 5;
#pragma unroll
      for (int m = 0; m < 16; m++) {
        const R k = dx ? kxm(m) : ky;
        v[m] = mk<R>(-rmul(k, in[m].y) * sc, rmul(k, in[m].x) * sc);
      }
    }
    fft<N, +1>(v, sh, t, TW);
    if (q < 2) store_row_pair<N>(v, B.g[GUV], row, q, live, t);
    else if (q < 4) store_row_pair<N>(v, B.g[GW], row, q - 2, live, t);
    else if (q == 4) {
      if (MODEL == MODEL_BINARY) store_row<N>(v, B.g[GCT], row, live, t);
      else store_row_pair<N>(v, B.g[GCT], row, o < 7 ? 0 : 1, live, t);
#pragma unroll
      for (int m = 0; m < 16; m++) v[m] = mk<R>(-rmul(ky, v[m].y), rmul(ky, v[m].x));
      store_row_pair<N>(v, B.g[o < 7 ? GD1 : GD2], row, 1, live, t);
    } else {
      store_row_pair<N>(v, B.g[o < 7 ? GD1 : GD2], row, q - 5, live, t);
    }
  }
}

// ---------------------------------------------------------------------------
// P2: advection products (+ bulk chemical potential) on x-row pairs (G -> H)
// nonlin.c:56-74 (u.grad w), :201-215 (binary u.grad c), :286-300/328-348
// (ternary u.grad c_i); surface_tension.c:24-35 / nonlin.c:217-230 (f(c));
// chem_potential.c:263-320 (ternary mu^F)
// ---------------------------------------------------------------------------

// binary f(c) = c (1 - c)(1 - 2c)  (surface_tension.c:30-31, nonlin.c:225)
template <class R> __device__ __forceinline__ R bulk_f(R a) {
  return rmul(rmul(a, rsub((R)1, a)), rsub((R)1, rmul((R)2, a)));
}


// ternary mu^F_1, mu^F_2 at one point (chem_potential.c:269-315)
template <class R> __device__ __forceinline__ void mu_ternary(const Par<R>& P, R c1, R c2, R& o1, R& o2) {
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
  o1 = rmul(m1, P.fac_mu);
  o2 = rmul(m2, P.fac_mu);
}

// mu^F_i(c) - mu^F_i(cb) at one point from the mean concentrations cb and the
// deviations c - cb (the ternary FP32 step's c_t carries no mean): the same
// polynomial as mu_ternary, written in the deviations (exact algebra:
// f(x) - f(xb) = dx (f'(xb) + dx (f''(xb)/2 + 2 dx)) for f = x (1-x)(1-2x), and
// x y - xb yb = dx y + xb dy for the products of the Lambda terms), so that the
// result carries float rounding relative to the deviation instead of to mu^F's
// large mean part.  mu^F(cb) is a constant: it only moves the k = 0 mode of
// F[mu^F], which multiplies k^2 = 0 in N_c and adds const * grad c_i to the
// force, whose curl vanishes when the cut has removed the Nyquist modes (the sharp
// cut; with the smooth filter those modes stay and the step keeps the direct form,
// as does FP64, which keeps the reference's arithmetic).  Measured at 4096^2
// (spinodal noise 1/3 +- 0.02, 100 steps): FP32 within 8e-6 of FP64 against 4.7e-5
// for the direct form.  The binary step keeps the direct f(c): on the forced drop
// run (c from 0 to 1) the deviation form made omega 6x further from FP64.
__device__ __forceinline__ void mu_ternary_dev(const Par<float>& P, float ab, float bb, float da, float dbv,
                                               float& o1, float& o2) {
  const float db_ = 1.0f - ab - bb;  // mean c3
  const float dd = -(da + dbv);      // its deviation
  const float a = ab + da, b = bb + dbv, d = db_ + dd;
  auto dfx = [](float xb, float dx) {
    const float f1 = 1.0f - 6.0f * xb + 6.0f * xb * xb, f2 = -3.0f + 6.0f * xb;
    return dx * (f1 + dx * (f2 + 2.0f * dx));
  };
  const float a2 = a * a, b2 = b * b, d2 = d * d;
  const float ab2 = ab * ab, bb2 = bb * bb;
  const float da2 = da * (a + ab), db2 = dbv * (b + bb), dd2 = dd * (d + db_);  // x^2 - xb^2
  const float dQ1 = da * (b2 * d2) + ab * (db2 * d2 + bb2 * dd2);   // a b^2 d^2
  const float dQ2 = dbv * (a2 * d2) + bb * (da2 * d2 + ab2 * dd2);  // a^2 b d^2
  const float dQ3 = dd * (a2 * b2) + db_ * (da2 * b2 + ab2 * db2);  // a^2 b^2 d
  const float G1 = P.g1 * dfx(ab, da) + P.six_lam * dQ1;
  const float G2 = P.g2 * dfx(bb, dbv) + P.six_lam * dQ2;
  const float G3 = P.g3 * dfx(db_, dd) + P.six_lam * dQ3;
  o1 = ((G1 - G2) * P.g2i + (G1 - G3) * P.g3i) * P.fac_mu;
  o2 = ((G2 - G1) * P.g1i + (G2 - G3) * P.g3i) * P.fac_mu;
}

// dot product of two pair-field transforms: f0 g0 + f1 g1 (e.g. ux*tux + uy*tuy)
template <class R> __device__ __forceinline__ R dot2(cx<R> f, cx<R> g) { return radd(rmul(f.x, g.x), rmul(f.y, g.y)); }

// real frags per group of the row kernels (thread-private values kept across
// transforms in shared memory)
template <int MODEL> constexpr int row_adv_frags() { return MODEL == MODEL_BINARY ? 2 : 1; }
template <int MODEL> constexpr int row_force_frags() { return 2; }

// The row kernels run a fixed schedule of inverse y transforms as a loop with
// one call site per transform direction (the unrolled transforms are long, so
// one copy of each keeps the kernel inside the instruction cache).  Step `it`
// of the schedule reads src(it); the copy of src(it + 1) is in flight while
// step it computes.

// binary P2 schedule: 0 c_t (plain, x-rows i0, i1); then per x-row i:
// 1 + 3h: (u, v); 2 + 3h: (dx w, dy w); 3 + 3h: (dx c, dy c); the forward
// transforms of A and B run at 5 and 6 (both x-rows together)
// ternary P2 schedule: 0, 1: (c1_t, c2_t) of x-rows i0, i1; then per x-row:
// 2 + 4h: (u, v); 3 + 4h: (dx w, dy w); 4 + 4h: (dx c1, dy c1); 5 + 4h: (dx c2, dy c2)
// pure Navier-Stokes P2 schedule: per x-row 2h: (u, v); 2h + 1: (dx w, dy w)
template <int MODEL> struct AdvSchedule {
  static constexpr int PRE = MODEL == MODEL_BINARY ? 1 : (MODEL == MODEL_TERNARY ? 2 : 0);
  static constexpr int PER = MODEL == MODEL_TERNARY ? 4 : (MODEL == MODEL_BINARY ? 3 : 2);
  static constexpr int STEPS = PRE + 2 * PER;
};

template <int N, class R, int MODEL>
__device__ __forceinline__ RowSrc<R> adv_src(const Bufs<R>& B, int it, int i0) {
  using Sc = AdvSchedule<MODEL>;
  if (it < Sc::PRE) {
    if (MODEL == MODEL_BINARY) return RowSrc<R>{B.g[GCT], N, i0, 2 * GCT + 1};
    return RowSrc<R>{B.g[GCT], 2 * N, 2 * (i0 + it), 2 * GCT};
  }
  const int q = it - Sc::PRE, h = q / Sc::PER, r = q % Sc::PER;
  const int slot = r == 0 ? GUV : (r == 1 ? GW : (r == 2 ? GD1 : GD2));
  return RowSrc<R>{B.g[slot], 2 * N, 2 * (i0 + h), 2 * slot};
}

// GR: the stage keeps grad c_i in real space for P4 (Bufs::gr), which then
// transforms only mu (the context's choice per grid size, chns_tuned.h)
// REC (binary): also store the real fields the discrete adjoint transposes (Bufs::rec)
template <int N, class R, int GPC, int MODEL, bool JT4 = false, bool GR = false, bool REC = false>
CHNS_STAGE_KERNEL(N, R, GPC) k_row_adv(CHNS_BUFS_PARAM B, CHNS_PAR_PARAM P, CHNS_TMAG_PARAM T) {
  using Sc = AdvSchedule<MODEL>;
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), P.tw, t);
  CHNS_GRID_DEP();
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
  const bool tma = tma_tiles_ok<N, R, GPC>(T, smem_raw);  // CTA-uniform
  if (tma) smem_raw = align128(smem_raw);
  const int jt = P.jt;
  const LoadedRowSmem<N, R, GPC> LS(smem_raw, g, tma ? T.nbox * T.boxr - 1 : jt, row_adv_frags<MODEL>());
  const RowSmem<N, R, GPC>& S = LS.S;
  const int pair = CHNS_BX * GPC + g;
  const bool live = pair < N / 2;
  const int i0 = 2 * pair;
  Frag<N, R> keep{S.frag}, keep2{S.frag + (size_t)N * GPC};
  cx<R> z[16], v[16];
  R a[16];

  TileLoader<R> TL{tma, LS.mb, 0u};
  if (tma && t == 0) mbar_init(TL.mb);
  __syncthreads();
  tile_start<N>(TL, T, S.tile, adv_src<N, R, MODEL>(B, 0, i0), jt, live, t);
#pragma unroll 1
  for (int it = 0; it < Sc::STEPS; it++) {
    const bool more = it + 1 < Sc::STEPS;
    row_c2r_loaded<N, R, JT4>(v, S.tile, TL, T, more, adv_src<N, R, MODEL>(B, more ? it + 1 : it, i0), jt, live, t,
                              S.sh, TW);
    cx<R>* dst = nullptr;
    int stride = 0, off = 0;
    if (it < Sc::PRE) {
      if (MODEL == MODEL_BINARY) {
        if constexpr (REC) {
          rec_row<N>(B.rec, 0, i0, v, false, live, t);
          rec_row<N>(B.rec, 0, i0 + 1, v, true, live, t);
        }
        // f(c_t) of x-rows i0, i1 (surface_tension.c:30-31, nonlin.c:225)
#pragma unroll
        for (int m = 0; m < 16; m++) v[m] = mk<R>(bulk_f(v[m].x), bulk_f(v[m].y));
        dst = B.h[HF]; stride = N; off = i0;
      } else {
        // mu^F_1, mu^F_2 of x-row i0 + it (chem_potential.c:263-320); FP32 from the
        // deviations (P1 left the means out) and the means (the double k = 0 modes)
        bool dev = false;  // CTA-uniform
        if constexpr (sizeof(R) == 4) dev = !P.filt;
        if (dev) {
          if constexpr (sizeof(R) == 4) {
            const double inv = 1.0 / ((double)N * (double)N);
            const float ab = (float)(P.k0[2] * inv), bb = (float)(P.k0[4] * inv);
#pragma unroll
            for (int m = 0; m < 16; m++) {
              float o1, o2;
              mu_ternary_dev(P, ab, bb, v[m].x, v[m].y, o1, o2);
              v[m] = mk<R>(o1, o2);
            }
          }
        } else {
#pragma unroll
          for (int m = 0; m < 16; m++) {
            R o1, o2;
            mu_ternary(P, v[m].x, v[m].y, o1, o2);
            v[m] = mk<R>(o1, o2);
          }
        }
        dst = B.h[HF]; stride = 2 * N; off = 2 * (i0 + it);
      }
    } else {
      const int q = it - Sc::PRE, h = q / Sc::PER, r = q % Sc::PER;
      if constexpr (REC && MODEL == MODEL_BINARY) {  // (u, v), (wx, wy), (cx, cy) of x-row i0 + h
        rec_row<N>(B.rec, 1 + 2 * r, i0 + h, v, false, live, t);
        rec_row<N>(B.rec, 2 + 2 * r, i0 + h, v, true, live, t);
      }
      if (r == 0) {
        // (u, v) of x-row i0 + h
#pragma unroll
        for (int m = 0; m < 16; m++) z[m] = v[m];
      } else if (MODEL == MODEL_BINARY && r != 0) {
        // binary: A = u dx w + v dy w (r = 1, nonlin.c:62) and B = u dx c + v dy c
        // (r = 2, nonlin.c:207).  Those of x-row i0 wait in the group's shared real
        // slots (not registers: at the 128-register bound of two CTAs per SM) until
        // x-row i1's are formed; each field of the two x-rows is then transformed as
        // one complex row and stored as a plain field, A at HAB, B behind it.  The
        // group thus writes both halves of each 16-byte pair of x-rows at once, and
        // P3 reads whole rows.
        // GR: grad c of this x-row stays in real space for P4 (no second transform there)
        if (GR && r == 2) store_row<N>(v, B.gr, i0 + h, live, t);
        Frag<N, R>& kp = r == 1 ? keep : keep2;
        if (h == 0) {
#pragma unroll
          for (int m = 0; m < 16; m++) kp[m] = dot2(z[m], v[m]);
        } else {
#pragma unroll
          for (int m = 0; m < 16; m++) v[m] = mk<R>(kp[m], dot2(z[m], v[m]));
          dst = B.h[HAB] + (r == 1 ? 0 : (size_t)(N / 2 + 1) * N); stride = N; off = i0;
        }
      } else if (r == 1) {
        // A = u dx w + v dy w (nonlin.c:62)
#pragma unroll
        for (int m = 0; m < 16; m++) a[m] = dot2(z[m], v[m]);
        if (MODEL == MODEL_NS) {
          if (h == 0) {
#pragma unroll
            for (int m = 0; m < 16; m++) keep[m] = a[m];
          } else {
#pragma unroll
            for (int m = 0; m < 16; m++) v[m] = mk<R>(keep[m], a[m]);
            dst = B.h[HAB]; stride = N; off = i0;
          }
        }
      } else if (r == 2) {
        // ternary: B1 = u dx c1 + v dy c1 (nonlin.c:292-293), stored with A as a pair field;
        // GR: grad c1 of this x-row stays in real space for P4
        if (GR) store_row<N>(v, B.gr, i0 + h, live, t);
#pragma unroll
        for (int m = 0; m < 16; m++) v[m] = mk<R>(a[m], dot2(z[m], v[m]));
        dst = B.h[HAB]; stride = 2 * N; off = 2 * (i0 + h);
      } else {
        // B2 = u dx c2 + v dy c2 (nonlin.c:334-335) of x-rows i0, i1, transformed together;
        // GR: grad c2 of this x-row stays in real space for P4
        if (GR) store_row<N>(v, B.gr + (size_t)N * N, i0 + h, live, t);
        if (h == 0) {
#pragma unroll
          for (int m = 0; m < 16; m++) keep[m] = dot2(z[m], v[m]);
        } else {
#pragma unroll
          for (int m = 0; m < 16; m++) v[m] = mk<R>(keep[m], dot2(z[m], v[m]));
          dst = B.h[HB2]; stride = N; off = i0;
        }
      }
    }
    if (dst) row_r2c_store<N>(v, dst, stride, off, live, t, S.sh, TW);  // CTA-uniform
  }
}


// ---------------------------------------------------------------------------
// P4: surface-tension force mu grad c on x-row pairs (G -> H)
// binary surface_tension.c:70-99; ternary :136-160, :188-210 (the two curls of
// the reference are summed before the transform: F[a] + F[b] = F[a + b])
// binary schedule: 0 mu_t (plain, x-rows i0, i1); 1 + h: (dx c, dy c) of x-row i0 + h
// ternary schedule: per x-row 3h: (mu1, mu2); 3h + 1: grad c1; 3h + 2: grad c2
// Every step is an inverse transform of its G rows, or with GR only the mu steps
// are, grad c_i being P2's real-space copy (the same transform of the same G
// rows, so the same values bit for bit).
// ---------------------------------------------------------------------------
template <int N, class R, int MODEL>
__device__ __forceinline__ RowSrc<R> force_src(const Bufs<R>& B, int it, int i0) {
  if (MODEL == MODEL_BINARY) {
    if (it == 0) return RowSrc<R>{B.g[GMU], N, i0, 2 * GMU + 1};
    return RowSrc<R>{B.g[GD1], 2 * N, 2 * (i0 + it - 1), 2 * GD1};
  }
  const int h = it / 3, r = it % 3;
  const int slot = r == 0 ? GMU : (r == 1 ? GD1 : GD2);
  return RowSrc<R>{B.g[slot], 2 * N, 2 * (i0 + h), 2 * slot};
}

template <int N, class R, int GPC, int MODEL, bool JT4 = false, bool GR = false, bool REC = false>
CHNS_STAGE_KERNEL(N, R, GPC) k_row_force(CHNS_BUFS_PARAM B, CHNS_PAR_PARAM P, CHNS_TMAG_PARAM T) {
  constexpr int NT = N / 16;
  constexpr int NIN = MODEL == MODEL_BINARY ? 3 : 6;      // steps with an input (binary: a last step only stores)
  constexpr int STEPS = MODEL == MODEL_BINARY ? 4 : 6;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), P.tw, t);
  CHNS_GRID_DEP();
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
  const bool tma = tma_tiles_ok<N, R, GPC>(T, smem_raw);  // CTA-uniform
  if (tma) smem_raw = align128(smem_raw);
  const int jt = P.jt;
  const LoadedRowSmem<N, R, GPC> LS(smem_raw, g, tma ? T.nbox * T.boxr - 1 : jt, row_force_frags<MODEL>());
  const RowSmem<N, R, GPC>& S = LS.S;
  const int pair = CHNS_BX * GPC + g;
  const bool live = pair < N / 2;
  const int i0 = 2 * pair;
  Frag<N, R> w1{S.frag}, w2{S.frag + N * GPC};
  cx<R> a[16], v[16];
  TileLoader<R> TL{tma, LS.mb, 0u};
  if (tma && t == 0) mbar_init(TL.mb);
  __syncthreads();
  tile_start<N>(TL, T, S.tile, force_src<N, R, MODEL>(B, 0, i0), jt, live, t);
#pragma unroll 1
  for (int it = 0; it < STEPS; it++) {
    const bool mu_step = MODEL == MODEL_BINARY ? it == 0 : it % 3 == 0;
    if (!GR && it < NIN) {
      const bool more = it + 1 < NIN;
      row_c2r_loaded<N, R, JT4>(v, S.tile, TL, T, more, force_src<N, R, MODEL>(B, more ? it + 1 : it, i0), jt, live,
                                t, S.sh, TW);
    } else if (GR && mu_step) {
      // mu of the pair (binary) or of x-row i0 + it/3 (ternary: the copy of x-row i1's is in flight after it 0)
      const bool more = MODEL == MODEL_TERNARY && it == 0;
      row_c2r_loaded<N, R, JT4>(v, S.tile, TL, T, more, force_src<N, R, MODEL>(B, more ? 3 : it, i0), jt, live, t,
                                S.sh, TW);
    } else if (GR && it < NIN) {
      // grad c (binary, x-row i0 + it - 1) or grad c_(it%3) (ternary, x-row i0 + it/3)
      const int xr = MODEL == MODEL_BINARY ? i0 + it - 1 : i0 + it / 3;
      const int f = MODEL == MODEL_BINARY ? 0 : it % 3 - 1;
      load_row<N>(v, B.gr + (size_t)f * N * N, xr, live, t);
    }
    bool store = false;
    cx<R>* dst = B.h[HFF];
    int stride = 2 * N, off = 2 * i0;
    if (MODEL == MODEL_BINARY) {
      // tux *= nphi, tuy *= nphi (surface_tension.c:87-88).  Fx and Fy of x-row i0
      // wait in the shared real slots until x-row i1's are formed; each is then
      // transformed for both x-rows as one complex row and stored as a plain field
      // (Fx at HFF, Fy behind it), so the group writes both halves of each 16-byte
      // pair of x-rows at once and P5 reads whole rows.
      if (it == 0) {
        if constexpr (REC) {
          rec_row<N>(B.rec, 7, i0, v, false, live, t);
          rec_row<N>(B.rec, 7, i0 + 1, v, true, live, t);
        }
#pragma unroll
        for (int m = 0; m < 16; m++) a[m] = v[m];  // mu_t of x-rows i0, i1
      } else if (it == 1) {
#pragma unroll
        for (int m = 0; m < 16; m++) {
          w1[m] = rmul(v[m].x, a[m].x);
          w2[m] = rmul(v[m].y, a[m].x);
        }
      } else if (it == 2) {
#pragma unroll
        for (int m = 0; m < 16; m++) {
          const R mu = a[m].y;
          const R fx = rmul(v[m].x, mu), fy = rmul(v[m].y, mu);
          v[m] = mk<R>(w1[m], fx);
          a[m] = mk<R>(w2[m], fy);
        }
        store = true;
        stride = N; off = i0;
      } else {
#pragma unroll
        for (int m = 0; m < 16; m++) v[m] = a[m];
        store = true;
        dst = B.h[HFF] + (size_t)(N / 2 + 1) * N; stride = N; off = i0;
      }
    } else {
      const int h = it / 3, r = it % 3;
      if (r == 0) {
        // w1 = (1+g3/g1) mu1 + (g3/g2) mu2, w2 = (g3/g1) mu1 + (1+g3/g2) mu2 (surface_tension.c:148-149, 199-200)
#pragma unroll
        for (int m = 0; m < 16; m++) {
          w1[m] = radd(rmul(P.w11, v[m].x), rmul(P.w12, v[m].y));
          w2[m] = radd(rmul(P.w21, v[m].x), rmul(P.w22, v[m].y));
        }
      } else if (r == 1) {
#pragma unroll
        for (int m = 0; m < 16; m++) { const R s = w1[m]; a[m] = mk<R>(rmul(v[m].x, s), rmul(v[m].y, s)); }
      } else {
#pragma unroll
        for (int m = 0; m < 16; m++) {
          const R s = w2[m];
          v[m] = mk<R>(radd(a[m].x, rmul(v[m].x, s)), radd(a[m].y, rmul(v[m].y, s)));
        }
        store = true;
        off = 2 * (i0 + h);
      }
    }
    if (store) row_r2c_store<N>(v, dst, stride, off, live, t, S.sh, TW);  // CTA-uniform
  }
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

// s + e = a + b exactly (Knuth's TwoSum, round to nearest)
__device__ __forceinline__ float two_sum(float a, float b, float& e) {
  const float s = __fadd_rn(a, b);
  const float bp = __fsub_rn(s, a);
  const float ap = __fsub_rn(s, bp);
  e = __fadd_rn(__fsub_rn(a, ap), __fsub_rn(b, bp));
  return s;
}

// One component of the ETD update of a float pair u = hi + lo:
// stage 1  u + d, d = u (e - 1) + N z1   (em1 = e - 1 keeps the decay of the slow
//                                         modes that a float e = 1 - O(1e-9) would lose)
// stage 2  u + d, d = (N - saved) z2     (a correction, small against u)
// The increment d is formed in float from hi (lo em1 is below its rounding): its
// rounding, 2^-24 |d|, matters only for
// modes that change fast (|d| ~ |u|), whose errors decay with them; what must not
// be lost is the part of a small d that a float sum hi + d would round away, so
// that sum is error-free (TwoSum) and its error joins lo.  Returns the new hi;
// the new lo in lo_out.
template <int STAGE>
__device__ __forceinline__ float etd_ff1(float hi, float lo, float n, float sv, float em1, float z1, float z2,
                                         float& lo_out) {
  const float d = STAGE == 1 ? __fmaf_rn(hi, em1, __fmul_rn(n, z1)) : __fmul_rn(__fsub_rn(n, sv), z2);
  float se;
  const float sh = two_sum(hi, d, se);
  const float t = __fadd_rn(se, lo);
  const float h = __fadd_rn(sh, t);  // Fast2Sum: |t| <= ulp(sh) but where hi + d cancels
  lo_out = __fsub_rn(t, __fsub_rn(h, sh));
  return h;
}

// ETD update of one mode of an FP32 context whose state is a float pair
// hi + lo (hi the float state the right-hand side reads; l the low part read by
// the caller): returns the new hi, the new low part in lo_out.  N and the saved N
// are float, as the right-hand side.
template <int STAGE>
__device__ __forceinline__ cxf etd_hilo(cxf hi, cxf l, cxf& lo_out, cxf nl, cxf* saved, float em1, float z1,
                                        float z2) {
  const cxf s = STAGE == 2 ? *saved : nl;
  if (STAGE == 1) *saved = nl;
  cxf h;
  h.x = etd_ff1<STAGE>(hi.x, l.x, nl.x, s.x, em1, z1, z2, lo_out.x);
  h.y = etd_ff1<STAGE>(hi.y, l.y, nl.y, s.y, em1, z1, z2, lo_out.y);
  return h;
}

// the same split of a double k = 0 mode (kept in double by FP32 contexts)
__device__ __forceinline__ cxf split_k0(const double* st, cxf* lo) {
  const cxf h = mk<float>((float)st[0], (float)st[1]);
  lo[0] = mk<float>((float)(st[0] - (double)h.x), (float)(st[1] - (double)h.y));
  return h;
}

// ---------------------------------------------------------------------------
// P3 (phase-field models): x forward transforms, N_w partial, mu and its x
// inverse transform, N_c and the ETD update of c  (H -> S, G)
// binary: nonlin.c:74-101 (-F[u.grad w]), surface_tension.c:35-48 (mu_hat),
//         nonlin.c:215-254 (N_c), etd2rk.c:102-113 / 177-188
// ternary: chem_potential.c:319-320 (F[mu^F]), surface_tension.c:116-137,
//          nonlin.c:300-377, etd2rk.c:117-130 / 191-206
// ---------------------------------------------------------------------------
// S64: FP32 context with a double-float state (B.lo; e - 1 in the e slots of
// P.coef).  Only the modes inside the truncation disc carry a low part: the
// modes outside it never reach a right-hand side (every product's inputs are
// truncated), so their float rounding is not amplified; they are updated in
// float with their low part left at zero.
// FILT: the context's truncation is SMOOTH_FILTER's (P.filt), a variant of its own
// so that the sharp cut's kernel carries none of the filter's registers
template <int N, class R, int GPC, int MODEL, int STAGE, bool S64, bool FILT = false, bool REC = false>
CHNS_STAGE_KERNEL(N, R, GPC) k_spec_fwd_c(CHNS_BUFS_PARAM B, CHNS_PAR_PARAM P) {
  constexpr int NT = N / 16;
  constexpr int NR = N / 2 + 1;
  constexpr bool F32 = sizeof(R) == 4;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), P.tw, t);
  CHNS_GRID_DEP();
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int row = CHNS_BX * GPC + g;
  const bool live = row < NR;
  const int rowc = live ? row : 0;
  const bool do_mu = (int)(CHNS_BX * GPC) <= P.jt;  // CTA-uniform
  const int mlim = (live && row <= P.jt) ? P.mrow[row] : -1;
  const R ky = (R)(P.fy * (double)row);
  const R* __restrict__ cf = P.coef + (size_t)rowc * NR;
  const size_t cstride = (size_t)NR * NR;
  auto kxm = [&](int m) -> R { return (R)(P.fx * (double)sidx<N>(t + NT * m)); };

  cx<R> f[16], c[16], v[16];
  // binary FP32: u.grad w, f(c), the state row and u.grad c come by bulk copy
  // into two row buffers, each copy in flight during the preceding transform
  constexpr bool PF = MODEL == MODEL_BINARY && F32;
  RowPrefetch<R> RP{};
  // N_w partial = -F[u.grad w]   (nonlin.c:74, 92); binary: the plain field at HAB
  if constexpr (PF) {
    RP = prefetch_setup<N, R, GPC>(smem_raw + (size_t)GPC * FftShape<N>::SMEM * sizeof(cx<R>), g, t, live, P.err);
    __syncthreads();
    RP.start(0, B.h[HAB] + (size_t)rowc * N, N);
    RP.start(1, B.h[HF] + (size_t)rowc * N, N);
    RP.wait(0);
    RP.template read<N>(0, v, t);
    __syncthreads();  // buffer 0 read by the whole group; also the transform's leading barrier
    RP.start(0, B.c1 + (size_t)rowc * N, N);
    fft<N, -1, R, false>(v, sh, t, TW);
  } else {
    if (MODEL == MODEL_BINARY) load_row<N>(v, B.h[HAB], row, live, t);
    else load_row_pair<N>(v, B.h[HAB], row, 0, live, t);
    fft<N, -1>(v, sh, t, TW);
  }
#pragma unroll
  for (int m = 0; m < 16; m++) v[m] = mk<R>(v[m].x * (R)(-1), v[m].y * (R)(-1));
  store_row<N>(v, B.nw, row, live, t);

#pragma unroll
  for (int fld = 0; fld < (MODEL == MODEL_TERNARY ? 2 : 1); fld++) {
    cx<R>* cst = fld == 0 ? B.c1 : B.c2;
    cx<R>* csv = fld == 0 ? B.s1 : B.s2;
    cx<R>* cx_out = fld == 0 ? B.x1 : B.x2;
    cx<R>* __restrict__ clo = B.lo[1 + fld];
    // F[f(c)] (binary) or F[mu^F_i] (ternary)
    if constexpr (PF) {
      RP.wait(1);
      RP.template read<N>(1, f, t);
      __syncthreads();
      RP.start(1, B.h[HAB] + (size_t)NR * N + (size_t)rowc * N, N);
      fft<N, -1, R, false>(f, sh, t, TW);
      RP.wait(0);
      RP.template read<N>(0, c, t);
    } else {
      if (MODEL == MODEL_BINARY) load_row<N>(f, B.h[HF], row, live, t);
      else load_row_pair<N>(f, B.h[HF], row, fld, live, t);
      fft<N, -1>(f, sh, t, TW);
      load_row<N>(c, cst, row, live, t);
    }
    if constexpr (REC && MODEL == MODEL_BINARY)  // F[f(c_t)] for the adjoint's record
      store_row<N>(f, reinterpret_cast<cx<R>*>(B.rec + (size_t)8 * N * N), row, live, t);
    if (do_mu) {
      // binary: mu = T[1.5 sigma eps k^2 c + 24 (sigma/eps) F[f]]   (surface_tension.c:45-46)
      // ternary: mu_i = T[F[mu^F_i] + 0.75 gamma_i eps k^2 c_i]     (surface_tension.c:116-128)
#pragma unroll
      for (int m = 0; m < 16; m++) {
        if (amask<N>(t, m) <= mlim) {
          const R ks = ksq(kxm(m), ky);
          if (MODEL == MODEL_BINARY) {
            const R q = rmul(P.st15, ks);
            v[m] = mk<R>(radd(rmul(q, c[m].x), rmul(P.st24, f[m].x)) * P.scale,
                         radd(rmul(q, c[m].y), rmul(P.st24, f[m].y)) * P.scale);
          } else {
            const R q = rmul(fld == 0 ? P.mu1 : P.mu2, ks);
            v[m] = mk<R>(radd(f[m].x, rmul(q, c[m].x)) * P.scale, radd(f[m].y, rmul(q, c[m].y)) * P.scale);
          }
          if constexpr (FILT) v[m] = smooth2(v[m], P.filt[(size_t)row * NR + amask<N>(t, m)]);
        } else {
          v[m] = czero<R>();
        }
      }
      fft<N, +1>(v, sh, t, TW);
      if (row <= P.jt) {
        if (MODEL == MODEL_BINARY) store_row<N>(v, B.g[GMU], row, live, t);
        else store_row_pair<N>(v, B.g[GMU], row, fld, live, t);
      }
    }
    // N_c  binary: -F[u.grad c] - lambda (24 (sigma/eps) k^2) F[f]   (nonlin.c:240, 251)
    //      ternary: -F[u.grad c_i] - (lambda/gamma_i) k^2 F[mu^F_i]  (nonlin.c:369-370)
    if constexpr (PF) {
      RP.wait(1);
      RP.template read<N>(1, v, t);
    } else if (MODEL == MODEL_BINARY) load_row<N>(v, B.h[HAB] + (size_t)NR * N, row, live, t);
    else if (fld == 0) load_row_pair<N>(v, B.h[HAB], row, 1, live, t);
    else load_row<N>(v, B.h[HB2], row, live, t);
    fft<N, -1>(v, sh, t, TW);
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int am = amask<N>(t, m);
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
      cx<R> sv;
      if (STAGE == 2) sv = live ? csv[idx] : czero<R>();
      const R e = cf[3 * cstride + am], z1 = cf[4 * cstride + am], z2 = cf[5 * cstride + am];
      if constexpr (S64) {
        if (am <= mlim) {
          cxf lnew;
          c[m] = etd_hilo<STAGE>(c[m], clo[idx], lnew, nl, &sv, e, z1, z2);
          clo[idx] = lnew;  // am <= mlim only on live rows
        } else {
          c[m] = etd<STAGE>(c[m], nl, &sv, (R)1 + e, z1, z2);
        }
      }
      else c[m] = etd<STAGE>(c[m], nl, &sv, e, z1, z2);
      if (STAGE == 1 && live) csv[idx] = sv;
      if (STAGE == 2 && cx_out && live) cx_out[idx] = nl;
      if (F32 && row == 0 && t == 0 && m == 0) {
        double* st = P.k0 + 2 * (1 + fld);
        double* sd = P.k0 + 2 * (4 + fld);
        etd_k0<STAGE>(st, sd, (double)nl.x, (double)nl.y, P.k0coef, 3);
        if constexpr (S64) c[m] = split_k0(st, clo);
        else c[m] = mk<R>((R)st[0], (R)st[1]);
      }
    }
    store_row<N>(c, cst, row, live, t);
  }
}

// ---------------------------------------------------------------------------
// P5: x forward transforms of the force, curl, N_w and the ETD update of w
// (H -> S)   surface_tension.c:98-111 / 159-173 / 209-223, curl.c:16-31,
// etd2rk.c:88-99 / 162-174.  Pure Navier-Stokes (CURL = false):
// N_w = -F[u.grad w] (nonlin.c:74-101) from the plain field in HAB.
// ---------------------------------------------------------------------------
template <int N, class R, int GPC, bool CURL, int STAGE, bool S64, bool PLAINF = false>
CHNS_STAGE_KERNEL(N, R, GPC) k_spec_curl_w(CHNS_BUFS_PARAM B, CHNS_PAR_PARAM P) {
  constexpr int NT = N / 16;
  constexpr int NR = N / 2 + 1;
  constexpr bool F32 = sizeof(R) == 4;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), P.tw, t);
  CHNS_GRID_DEP();
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int row = CHNS_BX * GPC + g;
  const bool live = row < NR;
  const int rowc = live ? row : 0;
  const int mlim = (live && row <= P.jt) ? P.mrow[row] : -1;  // truncation disc of this row (S64)
  const R ky = (R)(P.fy * (double)row);
  const R* __restrict__ cf = P.coef + (size_t)rowc * NR;
  cx<R>* __restrict__ wlo = B.lo[0];
  const size_t cstride = (size_t)NR * NR;
  auto kxm = [&](int m) -> R { return (R)(P.fx * (double)sidx<N>(t + NT * m)); };

  cx<R> a[16], b[16];
  // binary FP32: Fx, Fy, the partial N_w and the state row come by bulk copy
  // into two row buffers, each copy in flight during the preceding transform
  constexpr bool PF = CURL && PLAINF && F32;
  RowPrefetch<R> RP{};
  if constexpr (PF) {
    RP = prefetch_setup<N, R, GPC>(smem_raw + (size_t)GPC * FftShape<N>::SMEM * sizeof(cx<R>), g, t, live, P.err);
    __syncthreads();
    RP.start(0, B.h[HFF] + (size_t)rowc * N, N);
    RP.start(1, B.h[HFF] + (size_t)NR * N + (size_t)rowc * N, N);
    RP.wait(0);
    RP.template read<N>(0, a, t);
    __syncthreads();  // buffer 0 read by the whole group; also the transform's leading barrier
    RP.start(0, B.nw + (size_t)rowc * N, N);
    fft<N, -1, R, false>(a, sh, t, TW);
    RP.wait(1);
    RP.template read<N>(1, b, t);
    __syncthreads();
    RP.start(1, B.w + (size_t)rowc * N, N);
    fft<N, -1, R, false>(b, sh, t, TW);
    RP.wait(0);
    // N_w = N_w partial + I (kx F[Fy] - ky F[Fx])
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const R kx = kxm(m);
      const R dr = rsub(rmul(kx, b[m].x), rmul(ky, a[m].x));
      const R di = rsub(rmul(kx, b[m].y), rmul(ky, a[m].y));
      const cx<R> p = RP.buf[0][t + NT * m];
      a[m] = mk<R>(radd(p.x, -di), radd(p.y, dr));
    }
  } else if constexpr (CURL) {
    // the force: binary (PLAINF) Fx and Fy as plain fields, ternary a pair field
    if (PLAINF) load_row<N>(a, B.h[HFF], row, live, t);
    else load_row_pair<N>(a, B.h[HFF], row, 0, live, t);
    fft<N, -1>(a, sh, t, TW);
    if (PLAINF) load_row<N>(b, B.h[HFF] + (size_t)NR * N, row, live, t);
    else load_row_pair<N>(b, B.h[HFF], row, 1, live, t);
    fft<N, -1>(b, sh, t, TW);
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
    load_row<N>(a, B.h[HAB], row, live, t);
    fft<N, -1>(a, sh, t, TW);
#pragma unroll
    for (int m = 0; m < 16; m++) a[m] = mk<R>(a[m].x * (R)(-1), a[m].y * (R)(-1));
  }
  if (P.force_j >= 0 && row == P.force_j && t == 0) a[0].x = radd(a[0].x, P.force_hat);
  if constexpr (PF) {
    RP.wait(1);
    RP.template read<N>(1, b, t);
  } else {
    load_row<N>(b, B.w, row, live, t);
  }
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int am = amask<N>(t, m);
    const size_t idx = (size_t)rowc * N + t + NT * m;
    cx<R> sv;
    if (STAGE == 2) sv = live ? B.sw[idx] : czero<R>();
    if (STAGE == 2 && B.xw && live) B.xw[idx] = a[m];
    const R e = cf[0 * cstride + am], z1 = cf[1 * cstride + am], z2 = cf[2 * cstride + am];
    if constexpr (S64) {
      if (am <= mlim) {
        cxf lnew;
        b[m] = etd_hilo<STAGE>(b[m], wlo[idx], lnew, a[m], &sv, e, z1, z2);
        wlo[idx] = lnew;  // am <= mlim only on live rows
      } else {
        b[m] = etd<STAGE>(b[m], a[m], &sv, (R)1 + e, z1, z2);
      }
    }
    else b[m] = etd<STAGE>(b[m], a[m], &sv, e, z1, z2);
    if (STAGE == 1 && live) B.sw[idx] = sv;
    if (F32 && row == 0 && t == 0 && m == 0) {
      etd_k0<STAGE>(P.k0 + 0, P.k0 + 6, (double)a[m].x, (double)a[m].y, P.k0coef, 0);
      if constexpr (S64) b[m] = split_k0(P.k0, B.lo[0]);
      else b[m] = mk<R>((R)P.k0[0], (R)P.k0[1]);
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

// real field (n x n, R, row-major, i = x) -> H layout (plain): y-r2c of x-row pairs.
// Batched over blockIdx.y: field b reads x + b xs and writes H + b hs.
template <int N, class R, int GPC>
__global__ void __launch_bounds__(GPC * (N / 16)) k_row_r2c_plain(const R* __restrict__ x, cx<R>* __restrict__ H,
                                                                  const cx<R>* __restrict__ tw, size_t xs, size_t hs) {
  constexpr int NT = N / 16;
  x += blockIdx.y * xs;
  H += blockIdx.y * hs;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), tw, t);
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
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
  row_r2c_store<N>(v, H, N, i0, live, t, sh, TW);
}

// S/H layout row j': x transform (DIR), optional scale; batched over blockIdx.y
template <int N, class R, int GPC, int DIR>
__global__ void __launch_bounds__(GPC * (N / 16)) k_col_plain(const cx<R>* __restrict__ src, cx<R>* __restrict__ dst,
                                                              int nrows, R scale, const cx<R>* __restrict__ tw,
                                                              size_t ss, size_t ds) {
  constexpr int NT = N / 16;
  src += blockIdx.y * ss;
  dst += blockIdx.y * ds;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), tw, t);
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
  cx<R>* sh = reinterpret_cast<cx<R>*>(smem_raw) + g * FftShape<N>::SMEM;
  const int row = blockIdx.x * GPC + g;
  const bool live = row < nrows;
  cx<R> v[16];
  load_row<N>(v, src, row, live, t);
#pragma unroll
  for (int m = 0; m < 16; m++) v[m] = mk<R>(v[m].x * scale, v[m].y * scale);
  fft<N, DIR>(v, sh, t, TW);
  store_row<N>(v, dst, row, live, t);
}

// plain layout (rows 0..n/2) -> real field: y-c2r of x-row pairs; batched over blockIdx.y
template <int N, class R, int GPC>
__global__ void __launch_bounds__(GPC * (N / 16)) k_row_c2r_plain(const cx<R>* __restrict__ G, R* __restrict__ x,
                                                                  const cx<R>* __restrict__ tw, size_t gs, size_t xs) {
  constexpr int NT = N / 16;
  G += blockIdx.y * gs;
  x += blockIdx.y * xs;
  constexpr int JT = N / 2;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<R> TW = tw_setup<N>(reinterpret_cast<cx<R>*>(smem_all), tw, t);
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, R>(blockDim.x);
  const RowSmem<N, R, GPC> S(smem_raw, g, JT);
  const int pair = blockIdx.x * GPC + g;
  const bool live = pair < N / 2;
  const int i0 = 2 * pair;
  cx<R> v[16];
  tile_issue<N>(S.tile, RowSrc<R>{G, N, i0}, JT, live, t);
  cp_async_commit();
  row_c2r_tiled<N>(v, S.tile, false, RowSrc<R>{nullptr, 0, 0}, JT, live, t, S.sh, TW);
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
