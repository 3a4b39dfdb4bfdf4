// chns_slab.cu -- the reference's 2D transforms over several GPUs, one slab of
// x-rows per rank (fft.c:11-31 with FFTW-MPI plans, main.c:43-46,193-194).
//
// The reference distributes every field over MPI ranks by x-rows: rank r holds
// local_nx = nx / P rows, x = r local_nx .. (r+1) local_nx - 1, of the real field
// and the same kx-rows of its spectrum (FFTW layout, local_nx x (ny/2+1)).  A
// transform is the rank's local transforms plus two global transposes.  Here
// each rank is one GPU; the transposes are all-to-all exchanges that the host
// issues between the phases below (NCCL over NVLink, or any other all-to-all of
// equal blocks), so the phases themselves touch only this GPU's memory:
//
//   forward  y:      real x-rows -> y-r2c of x-row pairs -> send buffer
//            (exchange)
//            x:      the rank's J ky-rows, all x, from every rank -> x-FFT -> send buffer
//            (exchange)
//            unpack: the rank's kx-rows, all ky, from every rank -> FFTW layout
//   inverse  pack, (exchange), x (inverse, with 1/(nx ny)), (exchange), y (c2r)
//
// Exchange buffers hold P blocks of J x local_nx complex doubles, J = ceil((ny/2+1)
// / P) (the last rank's block is partly padding).  Block q of a y-phase send
// buffer is [jj][xl] (ky = q J + jj, x = rank local_nx + xl); block r of an
// x-phase send buffer is [jj][kl] (ky = rank J + jj, kx = r local_nx + kl).  Row
// k of the y-phase buffer, taken as one array of P J rows of local_nx, is
// therefore ky = k: the y transforms write and read it like a plain field of row
// stride local_nx.  FP64 only, as the reference.
#include <cuda_runtime.h>
#include <math.h>

#include <new>

#include "chns_internal.h"
#include "chns_kernels.cuh"

struct chns_slab {
  int n, nranks, rank, lnx, J;
  chns::cxd* tw;  // tw[q] = exp(-2 pi i q / n)
};

namespace {

using chns::cxd;

template <int N> constexpr int slab_gpc() {
  constexpr int nt = N / 16;
  constexpr int a = 256 / nt;
  return a < 1 ? 1 : (a > nt ? nt : a);
}

template <int N> constexpr size_t slab_fft_smem() {
  return chns::tw_smem_bytes<N, double>(slab_gpc<N>() * (N / 16)) +
         (size_t)slab_gpc<N>() * chns::FftShape<N>::SMEM * sizeof(cxd);
}

// y-r2c of the slab's x-row pairs: rows i0, i0 + 1 of `real` (row stride rs
// doubles) -> (F0[k], F1[k]) at send[k lnx + i0 .. + 1], k = 0 .. N/2
template <int N, int GPC>
__global__ void __launch_bounds__(GPC * (N / 16)) k_slab_y_r2c(const double* __restrict__ real, size_t rs,
                                                                cxd* __restrict__ send, int lnx,
                                                                const cxd* __restrict__ tw) {
  using namespace chns;
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<double> TW = tw_setup<N>(reinterpret_cast<cxd*>(smem_all), tw, t);
  cxd* sh = reinterpret_cast<cxd*>(smem_all + tw_smem_bytes<N, double>(blockDim.x)) + g * FftShape<N>::SMEM;
  const int pair = blockIdx.x * GPC + g;
  const bool live = 2 * pair < lnx;
  const int i0 = 2 * pair;
  cxd v[16];
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int y = t + NT * m;
    v[m] = live ? mk<double>(real[(size_t)i0 * rs + y], real[(size_t)(i0 + 1) * rs + y]) : czero<double>();
  }
  row_r2c_store<N>(v, send, lnx, i0, live, t, sh, TW);
}

// x transforms (DIR) of the rank's ky-rows jj = 0 .. J-1 (ky = rank J + jj <= N/2):
// row jj gathers x = p lnx + xl from block p of recv and scatters kx = r lnx + kl
// to block r of send, both blocks laid out [jj][xl]; inputs scaled by `scale`
template <int N, int GPC, int DIR>
__global__ void __launch_bounds__(GPC * (N / 16)) k_slab_x(const cxd* __restrict__ recv, cxd* __restrict__ send,
                                                            int lnx, int J, int rank, double scale,
                                                            const cxd* __restrict__ tw) {
  using namespace chns;
  constexpr int NT = N / 16;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<double> TW = tw_setup<N>(reinterpret_cast<cxd*>(smem_all), tw, t);
  cxd* sh = reinterpret_cast<cxd*>(smem_all + tw_smem_bytes<N, double>(blockDim.x)) + g * FftShape<N>::SMEM;
  const int jj = blockIdx.x * GPC + g;
  const bool live = jj < J && rank * J + jj <= N / 2;
  cxd v[16];
#pragma unroll
  for (int m = 0; m < 16; m++) {
    const int x = t + NT * m, p = x / lnx, xl = x - p * lnx;
    const cxd a = live ? recv[((size_t)p * J + jj) * lnx + xl] : czero<double>();
    v[m] = mk<double>(a.x * scale, a.y * scale);
  }
  fft<N, DIR>(v, sh, t, TW);
  if (live) {
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int k = t + NT * m, r = k / lnx, kl = k - r * lnx;
      send[((size_t)r * J + jj) * lnx + kl] = v[m];
    }
  }
}

// y-c2r of the slab's x-row pairs from the y-phase buffer (plain field of row
// stride lnx, rows ky = 0 .. N/2): real rows i0, i0 + 1 (row stride rs)
template <int N, int GPC>
__global__ void __launch_bounds__(GPC * (N / 16)) k_slab_y_c2r(const cxd* __restrict__ recv, double* __restrict__ real,
                                                                size_t rs, int lnx, const cxd* __restrict__ tw) {
  using namespace chns;
  constexpr int NT = N / 16;
  constexpr int JT = N / 2;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  const Tw<double> TW = tw_setup<N>(reinterpret_cast<cxd*>(smem_all), tw, t);
  unsigned char* smem_raw = smem_all + tw_smem_bytes<N, double>(blockDim.x);
  const RowSmem<N, double, GPC> S(smem_raw, g, JT);
  const int pair = blockIdx.x * GPC + g;
  const bool live = 2 * pair < lnx;
  const int i0 = 2 * pair;
  cxd v[16];
  tile_issue<N>(S.tile, RowSrc<double>{recv, lnx, i0, -1}, JT, live, t);
  cp_async_commit();
  row_c2r_tiled<N>(v, S.tile, false, RowSrc<double>{nullptr, 0, 0, -1}, JT, live, t, S.sh, TW);
  if (live) {
#pragma unroll
    for (int m = 0; m < 16; m++) {
      const int y = t + NT * m;
      real[(size_t)i0 * rs + y] = v[m].x;
      real[(size_t)(i0 + 1) * rs + y] = v[m].y;
    }
  }
}

// dst[c][r] = src[r][c] for r < rows_out (src: rows_in x cols, dst row stride ld);
// 32 x 32 tiles through shared memory
__global__ void k_slab_transpose(const cxd* __restrict__ src, cxd* __restrict__ dst, int rows, int cols, int ld) {
  __shared__ cxd tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = src[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) dst[(size_t)c * ld + r] = tile[threadIdx.x][k];
  }
}

// the inverse: dst[r][c] = src[c][r] for r < rows (src row stride ld; dst rows x cols)
__global__ void k_slab_transpose_back(const cxd* __restrict__ src, cxd* __restrict__ dst, int rows, int cols, int ld) {
  __shared__ cxd tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = src[(size_t)c * ld + r];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) dst[(size_t)r * cols + c] = tile[threadIdx.x][k];
  }
}

template <class K> bool slab_smem(K k, size_t bytes) {
  return bytes <= 48 * 1024 ||
         cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess;
}

template <int N> int y_r2c(const chns_slab* s, const double* real, size_t rs, cxd* send, cudaStream_t st) {
  constexpr int GPC = slab_gpc<N>();
  auto k = k_slab_y_r2c<N, GPC>;
  if (!slab_smem(k, slab_fft_smem<N>())) return CHNS_ERR_CUDA;
  k<<<(s->lnx / 2 + GPC - 1) / GPC, GPC * (N / 16), slab_fft_smem<N>(), st>>>(real, rs, send, s->lnx, s->tw);
  return CHNS_OK;
}

template <int N> int x_pass(const chns_slab* s, const cxd* recv, cxd* send, int dir, cudaStream_t st) {
  constexpr int GPC = slab_gpc<N>();
  auto k = dir < 0 ? k_slab_x<N, GPC, -1> : k_slab_x<N, GPC, +1>;
  if (!slab_smem(k, slab_fft_smem<N>())) return CHNS_ERR_CUDA;
  const double scale = dir < 0 ? 1.0 : 1.0 / ((double)N * (double)N);  // ifft's 1/(nx ny), a power of two
  k<<<(s->J + GPC - 1) / GPC, GPC * (N / 16), slab_fft_smem<N>(), st>>>(recv, send, s->lnx, s->J, s->rank, scale,
                                                                         s->tw);
  return CHNS_OK;
}

template <int N> int y_c2r(const chns_slab* s, const cxd* recv, double* real, size_t rs, cudaStream_t st) {
  constexpr int GPC = slab_gpc<N>();
  auto k = k_slab_y_c2r<N, GPC>;
  const size_t sm = chns::tw_smem_bytes<N, double>(GPC * (N / 16)) +
                    chns::RowSmem<N, double, GPC>::bytes(N / 2, 0);
  if (!slab_smem(k, sm)) return CHNS_ERR_CUDA;
  k<<<(s->lnx / 2 + GPC - 1) / GPC, GPC * (N / 16), sm, st>>>(recv, real, rs, s->lnx, s->tw);
  return CHNS_OK;
}

int y_r2c_any(const chns_slab* s, const double* real, size_t rs, cxd* send, cudaStream_t st) {
#define C_(N) y_r2c<N>(s, real, rs, send, st)
  switch (s->n) {
    case 32: return C_(32); case 64: return C_(64); case 128: return C_(128); case 256: return C_(256);
    case 512: return C_(512); case 1024: return C_(1024); case 2048: return C_(2048); case 4096: return C_(4096);
  }
#undef C_
  return CHNS_ERR_UNSUPPORTED;
}

int x_any(const chns_slab* s, const cxd* recv, cxd* send, int dir, cudaStream_t st) {
#define C_(N) x_pass<N>(s, recv, send, dir, st)
  switch (s->n) {
    case 32: return C_(32); case 64: return C_(64); case 128: return C_(128); case 256: return C_(256);
    case 512: return C_(512); case 1024: return C_(1024); case 2048: return C_(2048); case 4096: return C_(4096);
  }
#undef C_
  return CHNS_ERR_UNSUPPORTED;
}

int y_c2r_any(const chns_slab* s, const cxd* recv, double* real, size_t rs, cudaStream_t st) {
#define C_(N) y_c2r<N>(s, recv, real, rs, st)
  switch (s->n) {
    case 32: return C_(32); case 64: return C_(64); case 128: return C_(128); case 256: return C_(256);
    case 512: return C_(512); case 1024: return C_(1024); case 2048: return C_(2048); case 4096: return C_(4096);
  }
#undef C_
  return CHNS_ERR_UNSUPPORTED;
}

int launched() { return cudaGetLastError() == cudaSuccess ? CHNS_OK : CHNS_ERR_CUDA; }

}  // namespace

extern "C" {

int chns_slab_create(int n, int nranks, int rank, chns_slab** out) {
  if (!out) return CHNS_ERR_ARG;
  *out = nullptr;
  if (n < 32 || n > 4096 || (n & (n - 1)) != 0) return CHNS_ERR_UNSUPPORTED;
  if (nranks < 1 || rank < 0 || rank >= nranks || n % nranks != 0 || (n / nranks) % 2 != 0) return CHNS_ERR_ARG;
  chns_slab* s = new (std::nothrow) chns_slab;
  if (!s) return CHNS_ERR_NOMEM;
  s->n = n;
  s->nranks = nranks;
  s->rank = rank;
  s->lnx = n / nranks;
  s->J = (n / 2 + 1 + nranks - 1) / nranks;
  s->tw = nullptr;
  cxd* host = new (std::nothrow) cxd[n];
  if (!host) {
    delete s;
    return CHNS_ERR_NOMEM;
  }
  for (int q = 0; q < n; q++) {
    const long double a = 6.283185307179586476925286766559005768L * (long double)q / (long double)n;
    host[q].x = (double)cosl(a);
    host[q].y = (double)-sinl(a);
  }
  int rc = CHNS_OK;
  if (cudaMalloc((void**)&s->tw, (size_t)n * sizeof(cxd)) != cudaSuccess) rc = CHNS_ERR_NOMEM;
  else if (cudaMemcpy(s->tw, host, (size_t)n * sizeof(cxd), cudaMemcpyHostToDevice) != cudaSuccess) rc = CHNS_ERR_CUDA;
  delete[] host;
  if (rc != CHNS_OK) {
    if (s->tw) cudaFree(s->tw);
    delete s;
    return rc;
  }
  *out = s;
  return CHNS_OK;
}

void chns_slab_destroy(chns_slab* s) {
  if (!s) return;
  if (s->tw) cudaFree(s->tw);
  delete s;
}

int chns_slab_sizes(const chns_slab* s, int* local_nx, int* rows_per_rank, size_t* exchange_complex) {
  if (!s) return CHNS_ERR_ARG;
  if (local_nx) *local_nx = s->lnx;
  if (rows_per_rank) *rows_per_rank = s->J;
  if (exchange_complex) *exchange_complex = (size_t)s->nranks * s->J * s->lnx;
  return CHNS_OK;
}

int chns_slab_dfft_y(const chns_slab* s, const double* real, size_t real_stride, double* send, void* stream) {
  if (!s || !real || !send || real_stride < (size_t)s->n) return CHNS_ERR_ARG;
  const int rc = y_r2c_any(s, real, real_stride, (cxd*)send, (cudaStream_t)stream);
  return rc != CHNS_OK ? rc : launched();
}

int chns_slab_dfft_x(const chns_slab* s, const double* recv, double* send, void* stream) {
  if (!s || !recv || !send) return CHNS_ERR_ARG;
  const int rc = x_any(s, (const cxd*)recv, (cxd*)send, -1, (cudaStream_t)stream);
  return rc != CHNS_OK ? rc : launched();
}

int chns_slab_dfft_unpack(const chns_slab* s, const double* recv, double* spec, void* stream) {
  if (!s || !recv || !spec) return CHNS_ERR_ARG;
  const int rows = s->n / 2 + 1;  // ky rows kept of the P J rows
  dim3 grid((s->lnx + 31) / 32, (rows + 31) / 32);
  k_slab_transpose<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>((const cxd*)recv, (cxd*)spec, rows, s->lnx,
                                                                   s->n / 2 + 1);
  return launched();
}

int chns_slab_ifft_pack(const chns_slab* s, const double* spec, double* send, void* stream) {
  if (!s || !spec || !send) return CHNS_ERR_ARG;
  const int rows = s->n / 2 + 1;
  dim3 grid((s->lnx + 31) / 32, (rows + 31) / 32);
  k_slab_transpose_back<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>((const cxd*)spec, (cxd*)send, rows, s->lnx,
                                                                        s->n / 2 + 1);
  return launched();
}

int chns_slab_ifft_x(const chns_slab* s, const double* recv, double* send, void* stream) {
  if (!s || !recv || !send) return CHNS_ERR_ARG;
  const int rc = x_any(s, (const cxd*)recv, (cxd*)send, +1, (cudaStream_t)stream);
  return rc != CHNS_OK ? rc : launched();
}

int chns_slab_ifft_y(const chns_slab* s, const double* recv, double* real, size_t real_stride, void* stream) {
  if (!s || !recv || !real || real_stride < (size_t)s->n) return CHNS_ERR_ARG;
  const int rc = y_c2r_any(s, (const cxd*)recv, real, real_stride, (cudaStream_t)stream);
  return rc != CHNS_OK ? rc : launched();
}

}  // extern "C"
