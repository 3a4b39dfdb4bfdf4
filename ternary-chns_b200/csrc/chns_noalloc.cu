// chns_noalloc.cu -- a 2D r2c transform that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the point where they need a transform:
// code running inside another library's allocator or memory pool, code that must
// not change the device's memory footprint after start-up, or code whose device
// memory is owned by a host application that hands out only the input and
// output buffers.  chns_dfft_noalloc serves them: the caller passes the input and
// output, and the one intermediate field of the transform (the spectrum after the
// y transforms, before the x transforms) lives in a file-scope device array of
// fixed size instead of a context buffer.
//
// Limits and rules (also stated in include/chns.h):
//  * n is a power of two with 32 <= n <= CHNS_NOALLOC_MAX_N (512); larger n is
//    rejected with CHNS_ERR_UNSUPPORTED.  The scratch array is 2 x 257 x 512
//    complex doubles (4.2 MB); every GPU that loads this library holds it until
//    the process exits.
//  * The first call on a device does a one-time set-up for that device: it
//    looks up the device addresses of the arrays (cudaGetSymbolAddress),
//    uploads the twiddle tables (cudaMemcpyToSymbol), loads the kernels of every
//    supported n (so that a first call at a new size later loads no module) and
//    waits for the device (cudaDeviceSynchronize) so that the first transform,
//    on whatever stream the caller passes, reads a complete table.  Make that
//    first call before any stream capture.  The set-up is keyed on the device's
//    current context: after cudaDeviceReset the next call redoes it.
//  * Every call uses the same array.  Each call writes every scratch element it
//    later reads, so no clearing is needed, but calls that overlap on the GPU
//    (other streams, other host threads) race on the array and corrupt each
//    other's results: order them on one stream or synchronise between them.
#include <cuda_runtime.h>
#include <math.h>

#include <mutex>

#include "chns_internal.h"
#include "chns_kernels.cuh"

namespace {

constexpr int kMaxN = CHNS_NOALLOC_MAX_N;
constexpr size_t kField = (size_t)(kMaxN / 2 + 1) * kMaxN;  // complex values per intermediate field
constexpr int kTwTotal = 2 * kMaxN;                        // tables of n = 32..512 back to back (< 2 kMaxN)

static __device__ __align__(256) chns::cxd g_noalloc_scratch[2 * kField];
static __device__ __align__(256) chns::cxd g_noalloc_tw[kTwTotal];

struct DeviceSetup {
  bool done;
  void* ctx;           // the context the set-up was made in (a reset makes a new one)
  chns::cxd* scratch;  // device address of g_noalloc_scratch on this device
  chns::cxd* tw;       // device address of g_noalloc_tw on this device
};
constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

int tw_offset(int n) {  // start of the table of size n inside g_noalloc_tw
  int off = 0;
  for (int m = 32; m < n; m *= 2) off += m;
  return off;
}

template <int N> constexpr int gpc() {
  constexpr int nt = N / 16;
  constexpr int a = 256 / nt;
  return a < nt ? (a < 1 ? 1 : a) : nt;
}

template <int N> constexpr size_t smem_bytes() {
  return chns::tw_smem_bytes<N, double>(gpc<N>() * (N / 16)) +
         (size_t)gpc<N>() * chns::FftShape<N>::SMEM * sizeof(chns::cxd);
}

// Loads the three kernels of size N into the current context and sets their
// shared-memory limit, so that no later call at this size loads a module.
template <int N> bool load_kernels() {
  auto k1 = chns::k_row_r2c_plain<N, double, gpc<N>()>;
  auto k2 = chns::k_col_plain<N, double, gpc<N>(), -1>;
  auto k3 = chns::k_s_to_fftw<double>;
  cudaFuncAttributes a;
  if (cudaFuncGetAttributes(&a, k1) != cudaSuccess || cudaFuncGetAttributes(&a, k2) != cudaSuccess ||
      cudaFuncGetAttributes(&a, k3) != cudaSuccess)
    return false;
  if (smem_bytes<N>() > 48 * 1024 &&
      (cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<N>()) != cudaSuccess ||
       cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes<N>()) != cudaSuccess))
    return false;
  return true;
}

// The current context of the calling thread (cuCtxGetCurrent through the
// runtime's driver entry point; no link against libcuda).
void* current_context() {
  typedef int (*PFN_ctx)(void**);
  static PFN_ctx fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !f)
      return nullptr;
    fn = reinterpret_cast<PFN_ctx>(f);
  }
  void* c = nullptr;
  return fn(&c) == 0 ? c : nullptr;
}

int setup_device(int dev, DeviceSetup** out) {
  if (dev < 0 || dev >= kMaxDevices) return CHNS_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceSetup& s = g_setup[dev];
  if (cudaSetDevice(dev) != cudaSuccess) return CHNS_ERR_CUDA;  // makes the primary context current (CUDA >= 12)
  void* ctx = current_context();
  if (!ctx) return CHNS_ERR_CUDA;
  if (s.done && s.ctx != ctx) s.done = false;  // a cudaDeviceReset made a new context: redo the set-up
  if (!s.done) {
    if (cudaGetSymbolAddress((void**)&s.scratch, g_noalloc_scratch) != cudaSuccess) return CHNS_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&s.tw, g_noalloc_tw) != cudaSuccess) return CHNS_ERR_CUDA;
    static double host[2 * kTwTotal];
    for (int n = 32; n <= kMaxN; n *= 2) {
      const int off = tw_offset(n);
      for (int q = 0; q < n; q++) {
        const long double a = 6.283185307179586476925286766559005768L * (long double)q / (long double)n;
        host[2 * (off + q)] = (double)cosl(a);
        host[2 * (off + q) + 1] = (double)-sinl(a);
      }
    }
    if (cudaMemcpyToSymbol(g_noalloc_tw, host, sizeof(host)) != cudaSuccess) return CHNS_ERR_CUDA;
    if (!load_kernels<32>() || !load_kernels<64>() || !load_kernels<128>() || !load_kernels<256>() ||
        !load_kernels<512>())
      return CHNS_ERR_CUDA;
    // A pageable cudaMemcpyToSymbol may return before its copy lands, and the
    // caller's stream may be a non-blocking one that the legacy stream does not
    // order: wait here so the first transform reads a complete table.
    if (cudaDeviceSynchronize() != cudaSuccess) return CHNS_ERR_CUDA;
    s.ctx = ctx;
    s.done = true;
  }
  *out = &s;
  return CHNS_OK;
}

template <int N> int run(const double* real, double* spec, const DeviceSetup* s, cudaStream_t st) {
  using chns::cxd;
  constexpr int GPC = gpc<N>();
  constexpr int THREADS = GPC * (N / 16);
  constexpr size_t SMEM = smem_bytes<N>();
  cxd* h = s->scratch;           // after the y transforms (H layout)
  cxd* sl = s->scratch + kField;  // after the x transforms (S layout)
  const cxd* tw = s->tw + tw_offset(N);
  auto k1 = chns::k_row_r2c_plain<N, double, GPC>;  // loaded, with its shared-memory limit, by the set-up
  auto k2 = chns::k_col_plain<N, double, GPC, -1>;
  k1<<<(N / 2 + GPC - 1) / GPC, THREADS, SMEM, st>>>(real, h, tw, 0, 0);
  k2<<<(N / 2 + 1 + GPC - 1) / GPC, THREADS, SMEM, st>>>(h, sl, N / 2 + 1, 1.0, tw, 0, 0);
  dim3 grid((N / 2 + 1 + 31) / 32, (N + 31) / 32);
  chns::k_s_to_fftw<double><<<grid, dim3(32, 8), 0, st>>>(sl, (double2*)spec, N);
  return cudaGetLastError() == cudaSuccess ? CHNS_OK : CHNS_ERR_CUDA;
}

}  // namespace

extern "C" int chns_dfft_noalloc(const double* real, double* spec, int n, void* stream) {
  if (!real || !spec) return CHNS_ERR_ARG;
  if (n < 32 || n > kMaxN || (n & (n - 1)) != 0) return CHNS_ERR_UNSUPPORTED;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return CHNS_ERR_CUDA;
  DeviceSetup* s = nullptr;
  int rc = setup_device(dev, &s);
  if (rc != CHNS_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  switch (n) {
    case 32: return run<32>(real, spec, s, st);
    case 64: return run<64>(real, spec, s, st);
    case 128: return run<128>(real, spec, s, st);
    case 256: return run<256>(real, spec, s, st);
    case 512: return run<512>(real, spec, s, st);
  }
  return CHNS_ERR_UNSUPPORTED;
}
