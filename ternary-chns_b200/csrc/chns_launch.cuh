// chns_launch.cuh -- host launchers for one grid size and precision.
// Included by chns_inst_<N>.cu, which instantiates Launchers for N.
#pragma once

#include "chns_internal.h"
#include "chns_kernels.cuh"
#include "chns_tuned.h"
#include "chns_diag.cuh"
#include "chns_stage_args.cuh"
#include "chns_adj_rows.cuh"

namespace chns {

// groups (transforms of one row) per CTA: the tuned threads per CTA of
// chns_tuned.h (or CHNS_CTA_THREADS for an autotuner build) over n/16 threads per
// transform, at least 1 and at most n/16
template <int N, class R> constexpr int gpc_of() {
  constexpr int nt = N / 16;
  constexpr int lg = N >= 4096 ? 7 : N >= 2048 ? 6 : N >= 1024 ? 5 : N >= 512 ? 4 : N >= 256 ? 3 : N >= 128 ? 2
                   : N >= 64 ? 1 : 0;
#ifdef CHNS_CTA_THREADS
  constexpr int threads = CHNS_CTA_THREADS;
#else
  constexpr int threads = sizeof(R) == 4 ? kCtaThreadsF32[lg] : kCtaThreadsF64[lg];
#endif
  constexpr int a = threads / nt;
  return a < 1 ? 1 : (a > nt ? nt : a);
}

template <class K> static void set_smem(K kern, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int N, class R> struct Sizes {
  static constexpr int GPC = gpc_of<N, R>();
  static constexpr int NT = N / 16;
  static constexpr int THREADS = GPC * NT;
  static constexpr size_t TW = tw_smem_bytes<N, R>(THREADS);  // precomputed twiddles
  static constexpr size_t FFT_SMEM = TW + (size_t)GPC * FftShape<N>::SMEM * sizeof(cx<R>);
  static constexpr size_t FRAG = (size_t)GPC * N * sizeof(cx<R>);
  static int grid_rows(int rows) { return (rows + GPC - 1) / GPC; }
};

// shared memory of P3 / P5: the transform buffers, plus the row buffers of the
// binary FP32 passes, which prefetch their input rows
template <int N, class R> constexpr size_t spec_smem(bool prefetch) {
  return Sizes<N, R>::FFT_SMEM + (prefetch && sizeof(R) == 4 ? prefetch_smem<N, R, Sizes<N, R>::GPC>() : 0);
}

// launch of a stage kernel; with the context's PDL choice as a programmatic
// dependent launch (the kernel's CHNS_GRID_DEP waits for its predecessor), so
// that it is scheduled while the kernel before it drains
template <class K, class... Args>
static void launch_stage(const chns_ctx* c, K kern, dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                         const Args&... args) {
  if (!c->pdl) {
    kern<<<grid, block, smem, st>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, args...);
}

// the P3 variant of a context: double-float state (FP32 only) and SMOOTH_FILTER
template <int N, class R, int GPC, int MODEL, int STAGE>
static auto spec_fwd_c_kernel(bool s64, bool filt, bool rec) {
  constexpr bool F32 = sizeof(R) == 4;
  if constexpr (MODEL == MODEL_BINARY) {  // the adjoint's recording (sharp cut only)
    if (rec) return s64 ? k_spec_fwd_c<N, R, GPC, MODEL, STAGE, F32, false, true>
                        : k_spec_fwd_c<N, R, GPC, MODEL, STAGE, false, false, true>;
  }
  return s64 ? (filt ? k_spec_fwd_c<N, R, GPC, MODEL, STAGE, F32, true> : k_spec_fwd_c<N, R, GPC, MODEL, STAGE, F32>)
             : (filt ? k_spec_fwd_c<N, R, GPC, MODEL, STAGE, false, true> : k_spec_fwd_c<N, R, GPC, MODEL, STAGE, false>);
}

// the row kernels of a context: the square-box cut's compile-time tile reads
// (JT4) and grad c_i kept in real space from P2 for P4 (GR; pure Navier-Stokes has none)
template <int N, class R, int GPC, int MODEL>
static auto row_adv_kernel(bool jt4, bool gr, bool rec) {
  if constexpr (MODEL == MODEL_NS) {
    return jt4 ? k_row_adv<N, R, GPC, MODEL, true> : k_row_adv<N, R, GPC, MODEL, false>;
  } else {
    if constexpr (MODEL == MODEL_BINARY) {  // the adjoint's recording
      if (rec)
        return jt4 ? (gr ? k_row_adv<N, R, GPC, MODEL, true, true, true> : k_row_adv<N, R, GPC, MODEL, true, false, true>)
                   : (gr ? k_row_adv<N, R, GPC, MODEL, false, true, true> : k_row_adv<N, R, GPC, MODEL, false, false, true>);
    }
    return jt4 ? (gr ? k_row_adv<N, R, GPC, MODEL, true, true> : k_row_adv<N, R, GPC, MODEL, true, false>)
               : (gr ? k_row_adv<N, R, GPC, MODEL, false, true> : k_row_adv<N, R, GPC, MODEL, false, false>);
  }
}
template <int N, class R, int GPC, int MODEL>
static auto row_force_kernel(bool jt4, bool gr, bool rec) {
  if constexpr (MODEL == MODEL_BINARY) {  // the adjoint's recording
    if (rec)
      return jt4 ? (gr ? k_row_force<N, R, GPC, MODEL, true, true, true> : k_row_force<N, R, GPC, MODEL, true, false, true>)
                 : (gr ? k_row_force<N, R, GPC, MODEL, false, true, true> : k_row_force<N, R, GPC, MODEL, false, false, true>);
  }
  return jt4 ? (gr ? k_row_force<N, R, GPC, MODEL, true, true> : k_row_force<N, R, GPC, MODEL, true, false>)
             : (gr ? k_row_force<N, R, GPC, MODEL, false, true> : k_row_force<N, R, GPC, MODEL, false, false>);
}

template <int N, class R> int stage_impl(chns_ctx* c, int stage) {
  using S = Sizes<N, R>;
  constexpr int GPC = S::GPC;
  const Par<R> P = make_par<R>(c);
  const Bufs<R> B = make_bufs<R>(c);
  cudaStream_t st = c->stream;
  const int model = c->p.model;
  const int jt = c->jt;
  const int rows_inv = S::grid_rows(jt + 1);
  const int rows_all = S::grid_rows(N / 2 + 1);
  const int pairs = S::grid_rows(N / 2);
  int launches = 0;
  // FP32 contexts with a double-float state run the P3 / P5 variants that update it
  constexpr bool F32 = sizeof(R) == 4;
  const bool s64 = F32 && c->st64;
  // the row kernels' tiles come by TMA when the context has its tensor maps
  const TmaG& TG = *static_cast<const TmaG*>(c->tmag);
  const bool tma = TG.use != 0;

  // P1: spectral fan-out and x inverse transforms
  if (model == CHNS_MODEL_NS) {
    auto k = c->p1_split ? k_spec_inv<N, R, GPC, MODEL_NS, true> : k_spec_inv<N, R, GPC, MODEL_NS, false>;
    set_smem(k, S::FFT_SMEM);
    launch_stage(c, k, dim3(rows_inv, c->p1_split ? 2 : 1), S::THREADS, S::FFT_SMEM, st, B, P);
  } else if (model == CHNS_MODEL_BINARY) {
    auto k = c->p1_split ? k_spec_inv<N, R, GPC, MODEL_BINARY, true> : k_spec_inv<N, R, GPC, MODEL_BINARY, false>;
    set_smem(k, S::FFT_SMEM);
    launch_stage(c, k, dim3(rows_inv, c->p1_split ? 2 : 1), S::THREADS, S::FFT_SMEM, st, B, P);
  } else {
    auto k = c->p1_split ? k_spec_inv<N, R, GPC, MODEL_TERNARY, true> : k_spec_inv<N, R, GPC, MODEL_TERNARY, false>;
    set_smem(k, S::FFT_SMEM);
    launch_stage(c, k, dim3(rows_inv, c->p1_split ? 2 : 1), S::THREADS, S::FFT_SMEM, st, B, P);
  }
  launches++;
  mark(c, KIND_SPEC_INV);

  // P2: advection products (+ chemical potential).  The reference's cut on a
  // square box (jt = N/4) has row kernels whose tile reads are fixed at compile time.
  const bool jt4 = jt == N / 4;
  if (model == CHNS_MODEL_NS) {
    auto k = row_adv_kernel<N, R, GPC, MODEL_NS>(jt4, c->p4_grad, c->rec != nullptr);
    const size_t sm = S::TW + loaded_row_smem_bytes<N, R, GPC>(tma, jt, TG.boxr, TG.nbox, row_adv_frags<MODEL_NS>());
    set_smem(k, sm);
    launch_stage(c, k, pairs, S::THREADS, sm, st, B, P, TG);
  } else if (model == CHNS_MODEL_BINARY) {
    auto k = row_adv_kernel<N, R, GPC, MODEL_BINARY>(jt4, c->p4_grad, c->rec != nullptr);
    const size_t sm = S::TW + loaded_row_smem_bytes<N, R, GPC>(tma, jt, TG.boxr, TG.nbox, row_adv_frags<MODEL_BINARY>());
    set_smem(k, sm);
    launch_stage(c, k, pairs, S::THREADS, sm, st, B, P, TG);
  } else {
    auto k = row_adv_kernel<N, R, GPC, MODEL_TERNARY>(jt4, c->p4_grad, c->rec != nullptr);
    const size_t sm = S::TW + loaded_row_smem_bytes<N, R, GPC>(tma, jt, TG.boxr, TG.nbox, row_adv_frags<MODEL_TERNARY>());
    set_smem(k, sm);
    launch_stage(c, k, pairs, S::THREADS, sm, st, B, P, TG);
  }
  launches++;
  mark(c, KIND_ROW_ADV);

  if (model == CHNS_MODEL_NS) {
    // pure Navier-Stokes: N_w = -F[u.grad w], ETD of w
    if (stage == 1) {
      auto k = s64 ? k_spec_curl_w<N, R, GPC, false, 1, F32> : k_spec_curl_w<N, R, GPC, false, 1, false>;
      set_smem(k, S::FFT_SMEM);
      launch_stage(c, k, rows_all, S::THREADS, S::FFT_SMEM, st, B, P);
    } else {
      auto k = s64 ? k_spec_curl_w<N, R, GPC, false, 2, F32> : k_spec_curl_w<N, R, GPC, false, 2, false>;
      set_smem(k, S::FFT_SMEM);
      launch_stage(c, k, rows_all, S::THREADS, S::FFT_SMEM, st, B, P);
    }
    mark(c, KIND_SPEC_CURL_W);
    return launches + 1;
  }

  // P3: x forward transforms, mu, N_c, ETD of c
  {
    const bool bin = model == CHNS_MODEL_BINARY;
    const bool filt = c->filt != nullptr;
    const bool rec = c->rec != nullptr;
    auto k = bin ? (stage == 1 ? spec_fwd_c_kernel<N, R, GPC, MODEL_BINARY, 1>(s64, filt, rec)
                               : spec_fwd_c_kernel<N, R, GPC, MODEL_BINARY, 2>(s64, filt, rec))
                 : (stage == 1 ? spec_fwd_c_kernel<N, R, GPC, MODEL_TERNARY, 1>(s64, filt, rec)
                               : spec_fwd_c_kernel<N, R, GPC, MODEL_TERNARY, 2>(s64, filt, rec));
    set_smem(k, spec_smem<N, R>(bin));
    launch_stage(c, k, rows_all, S::THREADS, spec_smem<N, R>(bin), st, B, P);
  }
  launches++;
  mark(c, KIND_SPEC_FWD_C);

  // P4: surface-tension force
  if (model == CHNS_MODEL_BINARY) {
    auto k = row_force_kernel<N, R, GPC, MODEL_BINARY>(jt4, c->p4_grad, c->rec != nullptr);
    const size_t sm = S::TW + loaded_row_smem_bytes<N, R, GPC>(tma, jt, TG.boxr, TG.nbox, row_force_frags<MODEL_BINARY>());
    set_smem(k, sm);
    launch_stage(c, k, pairs, S::THREADS, sm, st, B, P, TG);
  } else {
    auto k = row_force_kernel<N, R, GPC, MODEL_TERNARY>(jt4, c->p4_grad, c->rec != nullptr);
    const size_t sm = S::TW + loaded_row_smem_bytes<N, R, GPC>(tma, jt, TG.boxr, TG.nbox, row_force_frags<MODEL_TERNARY>());
    set_smem(k, sm);
    launch_stage(c, k, pairs, S::THREADS, sm, st, B, P, TG);
  }
  launches++;
  mark(c, KIND_ROW_FORCE);

  // P5: curl, N_w, ETD of w (binary: the force as two plain fields)
  {
    const bool bin = model == CHNS_MODEL_BINARY;
    auto k = stage == 1
                 ? (s64 ? (bin ? k_spec_curl_w<N, R, GPC, true, 1, F32, true> : k_spec_curl_w<N, R, GPC, true, 1, F32>)
                        : (bin ? k_spec_curl_w<N, R, GPC, true, 1, false, true> : k_spec_curl_w<N, R, GPC, true, 1, false>))
                 : (s64 ? (bin ? k_spec_curl_w<N, R, GPC, true, 2, F32, true> : k_spec_curl_w<N, R, GPC, true, 2, F32>)
                        : (bin ? k_spec_curl_w<N, R, GPC, true, 2, false, true> : k_spec_curl_w<N, R, GPC, true, 2, false>));
    set_smem(k, spec_smem<N, R>(bin));
    launch_stage(c, k, rows_all, S::THREADS, spec_smem<N, R>(bin), st, B, P);
  }
  launches++;
  mark(c, KIND_SPEC_CURL_W);
  return launches;
}

// truncation (functions.c:47-84) of an S-layout field in place: the sharp cut
// zeroes |m| > mrow[row]; with filt (SMOOTH_FILTER, :69-72) every mode is
// multiplied by its factor twice
template <class R>
__global__ void k_truncate(cx<R>* s, const int* __restrict__ mrow, const R* __restrict__ filt, int n) {
  const int row = blockIdx.y;
  const int lim = mrow[row];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int ms = i <= n / 2 ? i : n - i;
    const size_t idx = (size_t)row * n + i;
    if (filt) s[idx] = smooth2(s[idx], filt[(size_t)row * (n / 2 + 1) + ms]);
    else if (ms > lim) s[idx] = czero<R>();
  }
}

template <int N, class R> int truncate_impl(chns_ctx* c, void* s) {
  dim3 grid((N + 255) / 256, N / 2 + 1);
  k_truncate<R><<<grid, 256, 0, c->stream>>>((cx<R>*)s, c->mrow, (const R*)c->filt, N);
  return 1;
}

// the largest dynamic shared memory of the step's kernels (P2 / P4 grow with the G rows)
template <int N, class R> size_t step_smem_impl(const chns_ctx* c) {
  using S = Sizes<N, R>;
  constexpr int GPC = S::GPC;
  const TmaG& TG = *static_cast<const TmaG*>(c->tmag);
  const bool tma = TG.use != 0;
  const int model = c->p.model;
  int frags = model == CHNS_MODEL_BINARY    ? row_adv_frags<MODEL_BINARY>()
              : model == CHNS_MODEL_TERNARY ? row_adv_frags<MODEL_TERNARY>()
                                            : row_adv_frags<MODEL_NS>();
  if (model != CHNS_MODEL_NS && row_force_frags<MODEL_BINARY>() > frags) frags = row_force_frags<MODEL_BINARY>();
  const size_t m = S::TW + loaded_row_smem_bytes<N, R, GPC>(tma, c->jt, TG.boxr, TG.nbox, frags);
  const size_t sp = spec_smem<N, R>(true);
  return m > sp ? m : sp;
}

// batched plain transforms: nb fields at strides (in elements of their type);
// scratch holds nb H-layout fields of n x (n/2+1) complex
template <int N, class R> int dfftb_impl(chns_ctx* c, const void* real, size_t rs, void* s, size_t ss, int nb,
                                         void* scratch) {
  using S = Sizes<N, R>;
  constexpr size_t HS = (size_t)N * (N / 2 + 1);
  auto k1 = k_row_r2c_plain<N, R, S::GPC>;
  set_smem(k1, S::FFT_SMEM);
  k1<<<dim3(S::grid_rows(N / 2), nb), S::THREADS, S::FFT_SMEM, c->stream>>>((const R*)real, (cx<R>*)scratch,
                                                                             (const cx<R>*)c->tw, rs, HS);
  auto k2 = k_col_plain<N, R, S::GPC, -1>;
  set_smem(k2, S::FFT_SMEM);
  k2<<<dim3(S::grid_rows(N / 2 + 1), nb), S::THREADS, S::FFT_SMEM, c->stream>>>(
      (const cx<R>*)scratch, (cx<R>*)s, N / 2 + 1, (R)1, (const cx<R>*)c->tw, HS, ss);
  return 2;
}

template <int N, class R> int ifftb_impl(chns_ctx* c, const void* s, size_t ss, void* real, size_t rs, int nb,
                                         void* scratch) {
  using S = Sizes<N, R>;
  constexpr size_t HS = (size_t)N * (N / 2 + 1);
  auto k1 = k_col_plain<N, R, S::GPC, +1>;
  set_smem(k1, S::FFT_SMEM);
  k1<<<dim3(S::grid_rows(N / 2 + 1), nb), S::THREADS, S::FFT_SMEM, c->stream>>>(
      (const cx<R>*)s, (cx<R>*)scratch, N / 2 + 1, (R)(1.0 / ((double)N * (double)N)), (const cx<R>*)c->tw, ss, HS);
  auto k2 = k_row_c2r_plain<N, R, S::GPC>;
  const size_t sm2 = S::TW + RowSmem<N, R, S::GPC>::bytes(N / 2, 0);
  set_smem(k2, sm2);
  k2<<<dim3(S::grid_rows(N / 2), nb), S::THREADS, sm2, c->stream>>>((const cx<R>*)scratch, (R*)real,
                                                                     (const cx<R>*)c->tw, HS, rs);
  return 2;
}

template <int N, class R> int adjprod_impl(chns_ctx* c, const void* rf, const void* const* in, int b0, int nb,
                                           void* s, size_t ss, void* scratch) {
  using S = Sizes<N, R>;
  constexpr size_t HS = (size_t)N * (N / 2 + 1);
  const AdjIn<R> A{(const R*)in[0], (const R*)in[1], (const R*)in[2], (const R*)in[3], (const R*)in[4]};
  auto k1 = k_adj_prod_r2c<N, R, S::GPC>;
  set_smem(k1, S::FFT_SMEM);
  k1<<<dim3(S::grid_rows(N / 2), nb), S::THREADS, S::FFT_SMEM, c->stream>>>((const RecFields<R>*)rf, A, b0,
                                                                             (cx<R>*)scratch, (const cx<R>*)c->tw, HS);
  auto k2 = k_col_plain<N, R, S::GPC, -1>;
  set_smem(k2, S::FFT_SMEM);
  k2<<<dim3(S::grid_rows(N / 2 + 1), nb), S::THREADS, S::FFT_SMEM, c->stream>>>(
      (const cx<R>*)scratch, (cx<R>*)s, N / 2 + 1, (R)1, (const cx<R>*)c->tw, HS, ss);
  return 2;
}

template <int N, class R> int dfft_impl(chns_ctx* c, const void* real, void* s) {
  return dfftb_impl<N, R>(c, real, 0, s, 0, 1, c->h[HAB]);
}

template <int N, class R> int ifft_impl(chns_ctx* c, const void* s, void* real) {
  return ifftb_impl<N, R>(c, s, 0, real, 0, 1, c->h[HF]);
}

template <int N, class R> int from_fftw_impl(chns_ctx* c, const double* src, void* s) {
  dim3 grid((N / 2 + 1 + 31) / 32, (N + 31) / 32);
  k_fftw_to_s<R><<<grid, dim3(32, 8), 0, c->stream>>>((const double2*)src, (cx<R>*)s, N);
  return 1;
}

template <int N, class R> int to_fftw_impl(chns_ctx* c, const void* s, double* dst) {
  dim3 grid((N / 2 + 1 + 31) / 32, (N + 31) / 32);
  k_s_to_fftw<R><<<grid, dim3(32, 8), 0, c->stream>>>((const cx<R>*)s, (double2*)dst, N);
  return 1;
}

template <int N, class R> int diag_impl(chns_ctx* c) {
  using S = Sizes<N, R>;
  const Par<R> P = make_par<R>(c);
  const Bufs<R> B = make_bufs<R>(c);
  const size_t rsm = S::TW + (size_t)NRED * S::THREADS * sizeof(double);
  const size_t sm = S::FFT_SMEM > rsm ? S::FFT_SMEM : rsm;
  const int model = c->p.model;
  const int rows = S::grid_rows(N / 2 + 1);
  const int pairs = S::grid_rows(N / 2);
  double* part = (double*)c->redscratch;
  if (model == CHNS_MODEL_NS) {
    auto k1 = c->filt ? k_diag_spec<N, R, S::GPC, MODEL_NS, true> : k_diag_spec<N, R, S::GPC, MODEL_NS>;
    set_smem(k1, S::FFT_SMEM);
    k1<<<rows, S::THREADS, S::FFT_SMEM, c->stream>>>(B, P);
    auto k2 = k_diag_row<N, R, S::GPC, MODEL_NS>;
    set_smem(k2, sm);
    k2<<<pairs, S::THREADS, sm, c->stream>>>(B, P, part);
  } else if (model == CHNS_MODEL_BINARY) {
    auto k1 = c->filt ? k_diag_spec<N, R, S::GPC, MODEL_BINARY, true> : k_diag_spec<N, R, S::GPC, MODEL_BINARY>;
    set_smem(k1, S::FFT_SMEM);
    k1<<<rows, S::THREADS, S::FFT_SMEM, c->stream>>>(B, P);
    auto k2 = k_diag_row<N, R, S::GPC, MODEL_BINARY>;
    set_smem(k2, sm);
    k2<<<pairs, S::THREADS, sm, c->stream>>>(B, P, part);
  } else {
    auto k1 = c->filt ? k_diag_spec<N, R, S::GPC, MODEL_TERNARY, true> : k_diag_spec<N, R, S::GPC, MODEL_TERNARY>;
    set_smem(k1, S::FFT_SMEM);
    k1<<<rows, S::THREADS, S::FFT_SMEM, c->stream>>>(B, P);
    auto k2 = k_diag_row<N, R, S::GPC, MODEL_TERNARY>;
    set_smem(k2, sm);
    k2<<<pairs, S::THREADS, sm, c->stream>>>(B, P, part);
  }
  k_diag_final<<<1, 256, 0, c->stream>>>(part, pairs, c->red);
  return 3;
}

template <int N, class R> const Launchers* make_launchers() {
  static const Launchers L = {stage_impl<N, R>,     truncate_impl<N, R>, dfft_impl<N, R>,
                              ifft_impl<N, R>,      from_fftw_impl<N, R>, to_fftw_impl<N, R>,
                              diag_impl<N, R>,      dfftb_impl<N, R>,     ifftb_impl<N, R>,
                              adjprod_impl<N, R>,   step_smem_impl<N, R>};
  return &L;
}

}  // namespace chns

#define CHNS_INSTANTIATE(NN)                                                       \
  namespace chns {                                                                 \
  const Launchers* launchers_f64_##NN() { return make_launchers<NN, double>(); } \
  const Launchers* launchers_f32_##NN() { return make_launchers<NN, float>(); }  \
  }
