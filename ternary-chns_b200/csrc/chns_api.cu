// chns_api.cu -- the C ABI (include/chns.h): context, tables, state I/O, steps.
//
// Replaces the set-up of the reference's main.c:43-211 (allocation, plans,
// wavenumbers, gamma_i/Delta) and its time-step entry etd2rk() (etd2rk.c:14-224)
// for one GPU.  All tables are computed here on the host in double with the
// reference's operand order (this file is compiled with -ffp-contract=off on
// the host side), then uploaded once.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>
#include <vector>

#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled

#include "chns_internal.h"
#include "chns_kernels.cuh"
#include "chns_tuned.h"

namespace chns {
#define CHNS_DECL(NN)                  \
  const Launchers* launchers_f64_##NN(); \
  const Launchers* launchers_f32_##NN();
CHNS_DECL(32)
CHNS_DECL(64)
CHNS_DECL(128)
CHNS_DECL(256)
CHNS_DECL(512)
CHNS_DECL(1024)
CHNS_DECL(2048)
CHNS_DECL(4096)

const Launchers* launchers_f64(int logn) {
  switch (logn) {
    case 5: return launchers_f64_32();
    case 6: return launchers_f64_64();
    case 7: return launchers_f64_128();
    case 8: return launchers_f64_256();
    case 9: return launchers_f64_512();
    case 10: return launchers_f64_1024();
    case 11: return launchers_f64_2048();
    case 12: return launchers_f64_4096();
  }
  return nullptr;
}
const Launchers* launchers_f32(int logn) {
  switch (logn) {
    case 5: return launchers_f32_32();
    case 6: return launchers_f32_64();
    case 7: return launchers_f32_128();
    case 8: return launchers_f32_256();
    case 9: return launchers_f32_512();
    case 10: return launchers_f32_1024();
    case 11: return launchers_f32_2048();
    case 12: return launchers_f32_4096();
  }
  return nullptr;
}
}  // namespace chns

namespace {

int ilog2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return (1 << l) == n ? l : -1;
}

#define CK(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return CHNS_ERR_CUDA;  \
  } while (0)

// (e^z - 1 - z) / z^2 for the ACCURATE coefficient mode
double phi2_z(double z) {
  if (fabs(z) < 0.5) {
    double term = 0.5, sum = 0.5;
    for (int n = 1; n < 20; n++) {
      term *= z / (double)(n + 2);
      sum += term;
    }
    return sum;
  }
  return (expm1(z) - z) / (z * z);
}

// ETD coefficients of one wavenumber, etd2rk.c:88-97,102-111,117-127 (stage 1)
// and :162-172,177-186,191-203 (stage 2), in the reference's operand order.
// e - 1 of the vorticity (o[0]) and phase-field (o[1]) linear terms at k^2 = ksqr
void etd_em1(const chns_params& p, double ksqr, double* o) {
  o[0] = expm1(-p.nu * p.dt * ksqr);
  double c = 0.0;
  if (p.model == CHNS_MODEL_BINARY) c = -1.5 * p.lambda * p.sigma * p.epsilon * ksqr * ksqr;
  else if (p.model == CHNS_MODEL_TERNARY) c = -0.75 * p.lambda * p.epsilon * ksqr * ksqr;
  o[1] = expm1(p.dt * c);
}

void etd_coefs(const chns_params& p, double ksqr, double* o) {
  const double dt = p.dt, nu = p.nu;
  double c = -nu * ksqr;
  double eta = exp(-nu * dt * ksqr);
  double z1, z2;
  if (p.coef_mode == CHNS_COEF_REFERENCE) {
    z1 = (fabs(c) > 1e-12) ? (eta - 1.0) / c : dt;
    z2 = (fabs(c) > 1e-12) ? (eta - 1.0 - c * dt) / (dt * c * c) : 0.5 * dt;
  } else {
    double z = c * dt;
    z1 = (z != 0.0) ? dt * (expm1(z) / z) : dt;
    z2 = dt * phi2_z(z);
  }
  double beta = 1.0, z1c = dt, z2c = 0.5 * dt;
  if (p.model == CHNS_MODEL_BINARY) {
    c = -1.5 * p.lambda * p.sigma * p.epsilon * ksqr * ksqr;
    beta = exp(dt * c);
    if (p.coef_mode == CHNS_COEF_REFERENCE) {
      z1c = (fabs(c) > 1e-12) ? (beta - 1.0) / c : dt;
      z2c = (fabs(c) != 0.0) ? (beta - 1.0 - c * dt) / (dt * c * c) : 0.5 * dt;
    }
  } else if (p.model == CHNS_MODEL_TERNARY) {
    c = -0.75 * p.lambda * p.epsilon;
    c *= ksqr * ksqr;
    beta = exp(dt * c);
    if (p.coef_mode == CHNS_COEF_REFERENCE) {
      if (fabs(c) > 1e-12) {
        z1c = (beta - 1.0) / c;
        z2c = (beta - 1.0 - c * dt);
        z2c /= (dt * c * c);
      } else {
        z1c = dt;
        z2c = 0.5 * dt;
      }
    }
  }
  if (p.model != CHNS_MODEL_NS && p.coef_mode != CHNS_COEF_REFERENCE) {
    double z = dt * c;
    z1c = (z != 0.0) ? dt * (expm1(z) / z) : dt;
    z2c = dt * phi2_z(z);
  }
  o[0] = eta;
  o[1] = z1;
  o[2] = z2;
  o[3] = beta;
  o[4] = z1c;
  o[5] = z2c;
}

// k^2 of the mode (|kx index| m, ky index j): kx = fx m, ky = fy j (functions.c:11-33;
// the sign of kx does not enter)
double mode_ksq(double fx, double fy, int m, int j) {
  const double kx = fx * m, ky = fy * j;
  return kx * kx + ky * ky;
}

// The truncation table (functions.c:47-84, the sharp cut k^2 > ((nx/dealias_div) fx)^2):
// mrow[j] = the largest |m| kept in ky row j (-1: none), j = 0..nx/2.  Returns jt,
// the last row with a kept mode.
int truncation_rows(const chns_params& p, double fx, double fy, int* mrow) {
  const int n = p.nx, nr = p.nx / 2 + 1;
  if (p.filter == CHNS_FILTER_SMOOTH) {  // functions.c:69-72: no mode is zeroed
    for (int j = 0; j < nr; j++) mrow[j] = n / 2;
    return n / 2;
  }
  const double dax = (p.nx / p.dealias_div) * fx;
  const double dealias = dax * dax;
  int jt = -1;
  for (int j = 0; j < nr; j++) {
    int lim = -1;
    for (int m = 0; m <= n / 2; m++) {
      if (mode_ksq(fx, fy, m, j) > dealias) break;
      lim = m;
    }
    mrow[j] = lim;
    if (lim >= 0) jt = j;
  }
  return jt;
}

// SMOOTH_FILTER factor of the mode (|kx index| m, ky index j), functions.c:53-54,69-72
// with kxmax, kymax of main.c:57-58: exp(-36 (k^2/k^2max)^18) by the host's libm
double filter_factor(const chns_params& p, double fx, double fy, int m, int j) {
  const double kxmax = (p.nx / 2.0) * fx, kymax = (p.ny / 2.0) * fy;
  const double ksqrmax = (double)(kxmax * kxmax + kymax * kymax);
  const double pp = mode_ksq(fx, fy, m, j) / ksqrmax;
  return ::exp(-36.0 * ::pow(pp, 18.0));
}

int validate(const chns_params* p) {
  if (!p) return CHNS_ERR_ARG;
  if (p->model < 0 || p->model > 2) return CHNS_ERR_ARG;
  if (p->precision != CHNS_FP64 && p->precision != CHNS_FP32 && p->precision != CHNS_FP32_STATE64)
    return CHNS_ERR_ARG;
  if (p->nx != p->ny) return CHNS_ERR_UNSUPPORTED;
  const int l = ilog2_exact(p->nx);
  if (l < 5 || l > 12) return CHNS_ERR_UNSUPPORTED;
  if (!(p->lx > 0) || !(p->ly > 0) || !(p->dt > 0) || !(p->nu >= 0)) return CHNS_ERR_ARG;
  if (p->filter != CHNS_FILTER_SHARP && p->filter != CHNS_FILTER_SMOOTH) return CHNS_ERR_ARG;
  // the sharp cut's band must stay below the Nyquist row
  if (p->filter == CHNS_FILTER_SHARP && !(p->dealias_div > 2.0)) return CHNS_ERR_ARG;
  if (p->model != CHNS_MODEL_NS && !(p->epsilon > 0)) return CHNS_ERR_ARG;
  if (p->coef_mode != CHNS_COEF_REFERENCE && p->coef_mode != CHNS_COEF_ACCURATE) return CHNS_ERR_ARG;
  if (p->force_amp != 0.0) {
    const double q = p->force_k * p->ly / (2.0 * M_PI);
    const double r = nearbyint(q);
    if (fabs(q - r) > 1e-9 || r < 1 || r > p->ny / 2) return CHNS_ERR_ARG;
  }
  return CHNS_OK;
}

void free_all(chns_ctx* c) {
  if (!c) return;
  chns_adj_free(c);
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  void* ptrs[] = {c->state[0], c->state[1], c->state[2], c->saved[0], c->saved[1], c->saved[2], c->nw,
                  c->coef, c->mrow, c->tw, c->k0, c->stage, c->realbuf, c->realdbl, c->red, c->redscratch,
                  c->statelo[0], c->statelo[1], c->statelo[2], c->tma_err, c->filt, c->gradr,
                  (void*)c->filtd == c->filt ? nullptr : (void*)c->filtd};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  for (void* q : c->g)
    if (q) cudaFree(q);
  for (void* q : c->h)
    if (q) cudaFree(q);
  delete static_cast<chns::TmaG*>(c->tmag);
  if (c->hostpin) cudaFreeHost(c->hostpin);
  for (int k = 0; k < c->npinned; k++) cudaHostUnregister(c->pinned[k]);
  c->npinned = 0;
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  free(c);
}

// Tensor maps of the G slots for the TMA tiles of the FP32 row kernels (left
// unused, with cp.async tiles instead, when the driver's encoder is unavailable
// or refuses a map).  Each G slot holds rows 0..jt; a tile is nbox boxes of
// {2 complex, boxr rows}.
// chns_tune_override's process-wide choices (-1: the tuned table)
static int g_tune_box_rows = -1, g_tune_p1_split = -1, g_tune_p4_grad = -1, g_tune_pdl = -1;

static int tuned_index(int n) { return ilog2_exact(n) - 5; }

int build_tma(chns_ctx* c) {
  chns::TmaG* T = new (std::nothrow) chns::TmaG();
  if (!T) return CHNS_ERR_NOMEM;
  c->tmag = T;
  T->use = 0;
  T->err = c->tma_err;
  const int rows = c->jt + 1;
  const int li = tuned_index(c->n);
  const int cap = g_tune_box_rows > 0 ? g_tune_box_rows
                                      : (c->f32 ? chns::kTmaBoxRowsF32[li] : chns::kTmaBoxRowsF64[li]);
  T->boxr = rows >= cap ? cap : (rows + 7) / 8 * 8;
  T->nbox = (rows + T->boxr - 1) / T->boxr;
  T->ecx = c->f32 ? 1 : 2;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn) {
    cudaGetLastError();
    return CHNS_OK;
  }
  const auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  for (int k = 0; k < chns::NG; k++)
    for (int v = 0; v < 2; v++) {
      const cuuint64_t width = (v == 0 ? 2 * (cuuint64_t)c->n : (cuuint64_t)c->n) * T->ecx;  // elements per row
      const cuuint64_t dims[2] = {width, (cuuint64_t)rows};
      const cuuint64_t strides[1] = {width * 8};
      const cuuint32_t box[2] = {(cuuint32_t)(2 * T->ecx), (cuuint32_t)T->boxr};
      const cuuint32_t estr[2] = {1, 1};
      if (encode(&T->map[2 * k + v], CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, c->g[k], dims, strides, box, estr,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return CHNS_OK;
    }
  T->use = 1;
  return CHNS_OK;
}

// CHNS_ERR_TIMEOUT when a row kernel flagged a timed-out tile wait (then clears it)
int tma_status(chns_ctx* c) {
  unsigned int h = 0;
  CK(cudaMemcpyAsync(&h, c->tma_err, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (!h) return CHNS_OK;
  CK(cudaMemsetAsync(c->tma_err, 0, sizeof(h), c->stream));
  return CHNS_ERR_TIMEOUT;
}

int dmalloc(void** p, size_t bytes) {
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    *p = nullptr;
    return CHNS_ERR_NOMEM;
  }
  return cudaMemsetAsync(*p, 0, bytes) == cudaSuccess ? CHNS_OK : CHNS_ERR_CUDA;
}

// Copies `bytes` from a host or device pointer to device memory.
int to_device(chns_ctx* c, void* dst, const void* src, size_t bytes, int where) {
  CK(cudaMemcpyAsync(dst, src, bytes, where == CHNS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     c->stream));
  return CHNS_OK;
}
int from_device(chns_ctx* c, void* dst, const void* src, size_t bytes, int where) {
  CK(cudaMemcpyAsync(dst, src, bytes, where == CHNS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     c->stream));
  if (where != CHNS_DEVICE) CK(cudaStreamSynchronize(c->stream));
  return CHNS_OK;
}

__global__ void k_real_d2r_f32(const double* __restrict__ a, float* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void k_real_r2d_f32(const float* __restrict__ a, double* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}
// FP32 contexts keep the k = 0 modes in double: copy (0,0) of FFTW staging <-> k0
// block sums of n doubles (fixed order within and across blocks: reproducible)
__global__ void k_sum_blocks(const double* __restrict__ a, size_t n, double* part) {
  __shared__ double red[32];
  double s = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) s += a[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    part[blockIdx.x] = t;
  }
}
// k0[2 slot] = the field's sum (its unnormalised k = 0 mode), k0[2 slot + 1] = 0
__global__ void k_sum_finish(const double* __restrict__ part, int nb, double* k0, int slot) {
  double t = 0.0;
  for (int b = 0; b < nb; b++) t += part[b];
  k0[2 * slot] = t;
  k0[2 * slot + 1] = 0.0;
}
// b = (float)(a - sum / n): the field without its mean
__global__ void k_real_d2r_f32_dev(const double* __restrict__ a, float* __restrict__ b, size_t n,
                                   const double* __restrict__ k0, int slot) {
  const double mean = k0[2 * slot] / (double)n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)(a[i] - mean);
}
// the float k = 0 mode of an S-layout field from the double one
__global__ void k_k0_to_state(const double* __restrict__ k0, float2* s, int slot) {
  s[0] = make_float2((float)k0[2 * slot], (float)k0[2 * slot + 1]);
}

__global__ void k_k0_set(double* k0, const double* st, int slot) {
  k0[2 * slot] = st[0];
  k0[2 * slot + 1] = st[1];
}
__global__ void k_k0_get(const double* k0, double* st, int slot) {
  st[0] = k0[2 * slot];
  st[1] = k0[2 * slot + 1];
}

// flag |= 1 when any of n reals is NaN or infinite
template <class R> __global__ void k_nonfinite(const R* __restrict__ a, size_t n, unsigned int* flag) {
  bool bad = false;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    bad |= !isfinite(a[i]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

int enqueue_step(chns_ctx* c) {
  int n1 = c->L->stage(c, 1);
  int n2 = c->L->stage(c, 2);
  c->launches_per_step = n1 + n2;
  return CHNS_OK;
}

int build_graph(chns_ctx* c) {
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return CHNS_ERR_CUDA;
  enqueue_step(c);
  if (cudaStreamEndCapture(c->stream, &g) != cudaSuccess) return CHNS_ERR_CUDA;
  cudaError_t e = cudaGraphInstantiate(&c->step_graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    c->step_graph = nullptr;
    return CHNS_ERR_CUDA;
  }
  c->graph_ok = true;
  return CHNS_OK;
}

}  // namespace

extern "C" {

void chns_default_params(chns_params* p, int model, int n) {
  memset(p, 0, sizeof(*p));
  p->model = model;
  p->precision = CHNS_FP64;
  p->nx = p->ny = n;
  p->lx = p->ly = 4.0 * M_PI;  // global.h:20-21
  p->dt = 1e-4;                 // global.h:31
  p->nu = 0.01;                 // global.h:30
  const double dx = p->lx / n;
  p->epsilon = 3.0 * dx;  // global.h:103,131
  if (model == CHNS_MODEL_BINARY) {
    p->sigma = 2.0;    // global.h:102
    p->lambda = 1e-6;  // global.h:104
  } else if (model == CHNS_MODEL_TERNARY) {
    p->sigma12 = 0.2;   // global.h:127-129
    p->sigma23 = 0.45;
    p->sigma13 = 0.2;
    p->lambda = 1e-4;   // global.h:132
    p->xlambda = 2.0;   // global.h:133
  }
  p->dealias_div = 4.0;
  p->coef_mode = CHNS_COEF_REFERENCE;
}

int chns_create(const chns_params* pin, chns_ctx** out) {
  if (!out) return CHNS_ERR_ARG;
  *out = nullptr;
  int rc = validate(pin);
  if (rc != CHNS_OK) return rc;
  chns_ctx* c = (chns_ctx*)calloc(1, sizeof(chns_ctx));
  if (!c) return CHNS_ERR_NOMEM;
  c->p = *pin;
  const chns_params& p = c->p;
  c->n = p.nx;
  c->nr = p.nx / 2 + 1;
  c->f32 = p.precision != CHNS_FP64;
  c->st64 = p.precision == CHNS_FP32_STATE64;
  c->rsz = c->f32 ? 4 : 8;
  {
    const int li = tuned_index(c->n);
    c->p1_split = g_tune_p1_split >= 0 ? g_tune_p1_split != 0
                                       : (c->f32 ? chns::kSpecInvSplitF32[li] : chns::kSpecInvSplitF64[li]) != 0;
    c->p4_grad = p.model != CHNS_MODEL_NS &&
                 (g_tune_p4_grad >= 0 ? g_tune_p4_grad != 0
                                      : (c->f32 ? chns::kP4GradF32[li] : chns::kP4GradF64[li]) != 0);
    c->pdl = g_tune_pdl >= 0 ? g_tune_pdl != 0 : (c->f32 ? chns::kPdlF32[li] : chns::kPdlF64[li]) != 0;
  }
  const int logn = ilog2_exact(c->n);
  c->L = c->f32 ? chns::launchers_f32(logn) : chns::launchers_f64(logn);
  if (!c->L) {
    free(c);
    return CHNS_ERR_UNSUPPORTED;
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    free(c);
    return CHNS_ERR_CUDA;
  }
  c->own_stream = true;

  // wavenumbers (main.c:54-55, functions.c:11-33) and the truncation table (functions.c:47-84)
  const int n = c->n, nr = c->nr;
  c->fx = (2 * M_PI) / p.lx;
  c->fy = (2 * M_PI) / p.ly;
  std::vector<int> mrow(nr, -1);
  c->jt = truncation_rows(p, c->fx, c->fy, mrow.data());
  if (c->jt < 0 || (c->jt >= n / 2 && p.filter == CHNS_FILTER_SHARP)) {
    free_all(c);
    return CHNS_ERR_UNSUPPORTED;
  }
  // ternary surface-tension coefficients (main.c:166-170)
  if (p.model == CHNS_MODEL_TERNARY) {
    c->gamma[0] = (p.sigma12 - p.sigma23 + p.sigma13);
    c->gamma[1] = (p.sigma12 - p.sigma13 + p.sigma23);
    c->gamma[2] = (p.sigma23 - p.sigma12 + p.sigma13);
    c->del = (6.0 * c->gamma[0] * c->gamma[1] * c->gamma[2]);
    c->del /= (c->gamma[0] * c->gamma[1] + c->gamma[0] * c->gamma[2] + c->gamma[1] * c->gamma[2]);
    if (!(c->gamma[0] != 0 && c->gamma[1] != 0 && c->gamma[2] != 0)) {
      free_all(c);
      return CHNS_ERR_ARG;
    }
  }
  // Kolmogorov forcing: curl of F0 sin(kf y) x-hat = -F0 kf cos(kf y); its
  // unnormalised transform is -F0 kf (nx ny / 2) at kx = 0, ky = kf
  c->force_j = -1;
  if (p.force_amp != 0.0) {
    c->force_j = (int)nearbyint(p.force_k * p.ly / (2.0 * M_PI));
    c->force_hat = -p.force_amp * p.force_k * ((double)p.nx * (double)p.ny / 2.0);
  }

  // ETD coefficient tables [6][nr rows][nr |m|]
  const size_t tsz = (size_t)nr * nr;
  std::vector<double> coef(6 * tsz);
  for (int j = 0; j < nr; j++) {
    for (int m = 0; m < nr; m++) {
      double o[6];
      etd_coefs(p, mode_ksq(c->fx, c->fy, m, j), o);
      for (int q = 0; q < 6; q++) coef[q * tsz + (size_t)j * nr + m] = o[q];
    }
  }
  for (int q = 0; q < 6; q++) c->k0coef[q] = coef[q * tsz];

  // twiddles exp(-2 pi i q / n), long double then rounded
  std::vector<double> twd(2 * (size_t)n);
  for (int q = 0; q < n; q++) {
    const long double a = 6.283185307179586476925286766559005768L * (long double)q / (long double)n;
    twd[2 * q] = (double)cosl(a);
    twd[2 * q + 1] = (double)-sinl(a);
  }

  const size_t ncx = (size_t)nr * n;                // complex per S field
  const size_t ngx = (size_t)(c->jt + 1) * 2 * n;   // complex per G slot (pair width)
  const size_t nhx = (size_t)nr * 2 * n;            // complex per H slot (pair width)
  const size_t cxsz = 2 * c->rsz;
  const int nfields = p.model + 1;
  rc = CHNS_OK;
  for (int f = 0; f < 3 && rc == CHNS_OK; f++) {
    if (f < nfields) {
      rc = dmalloc(&c->state[f], ncx * cxsz);
      if (rc == CHNS_OK) rc = dmalloc(&c->saved[f], ncx * cxsz);
      if (rc == CHNS_OK && c->st64) rc = dmalloc(&c->statelo[f], ncx * cxsz);
    }
  }
  if (rc == CHNS_OK) rc = dmalloc(&c->nw, ncx * cxsz);
  for (int k = 0; k < chns::kNumG && rc == CHNS_OK; k++) rc = dmalloc(&c->g[k], ngx * cxsz);
  for (int k = 0; k < chns::kNumH && rc == CHNS_OK; k++) rc = dmalloc(&c->h[k], nhx * cxsz);
  if (rc == CHNS_OK && c->p4_grad) rc = dmalloc(&c->gradr, (size_t)p.model * n * n * cxsz);
  if (rc == CHNS_OK) rc = dmalloc(&c->coef, 6 * tsz * c->rsz);
  if (rc == CHNS_OK) rc = dmalloc((void**)&c->mrow, nr * sizeof(int));
  if (rc == CHNS_OK) rc = dmalloc(&c->tw, (size_t)n * cxsz);
  if (rc == CHNS_OK) rc = dmalloc((void**)&c->k0, 16 * sizeof(double));
  if (rc == CHNS_OK) rc = dmalloc((void**)&c->stage, 2 * ncx * sizeof(double));
  if (rc == CHNS_OK) rc = dmalloc(&c->realbuf, (size_t)n * n * c->rsz);
  if (rc == CHNS_OK) rc = dmalloc((void**)&c->realdbl, (size_t)n * n * sizeof(double));
  if (rc == CHNS_OK) rc = dmalloc((void**)&c->red, 16 * sizeof(double));
  if (rc == CHNS_OK) rc = dmalloc(&c->redscratch, (size_t)(n / 2 + 1) * 8 * sizeof(double));
  if (rc == CHNS_OK) rc = dmalloc((void**)&c->tma_err, sizeof(unsigned int));
  std::vector<double> filt;
  if (rc == CHNS_OK && p.filter == CHNS_FILTER_SMOOTH) {
    filt.resize(tsz);
    for (int j = 0; j < nr; j++)
      for (int m = 0; m < nr; m++) filt[(size_t)j * nr + m] = filter_factor(p, c->fx, c->fy, m, j);
    rc = dmalloc(&c->filt, tsz * c->rsz);
    if (rc == CHNS_OK && c->f32) rc = dmalloc((void**)&c->filtd, tsz * sizeof(double));
    if (rc == CHNS_OK && !c->f32) c->filtd = (double*)c->filt;
  }
  if (rc == CHNS_OK) rc = build_tma(c);
  // the row kernels' shared memory grows with the G rows (all of them with the
  // smooth filter): refuse a context whose kernels would not launch
  if (rc == CHNS_OK) {
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
      rc = CHNS_ERR_CUDA;
    else if (c->L->step_smem(c) > (size_t)optin)
      rc = CHNS_ERR_UNSUPPORTED;
  }
  if (rc != CHNS_OK) {
    free_all(c);
    return rc;
  }
  // uploads (tables converted to the context precision)
  cudaError_t e = cudaSuccess;
  if (c->f32) {
    std::vector<float> cf(coef.begin(), coef.end());
    std::vector<float> tf(twd.begin(), twd.end());
    if (c->st64) {
      // a double-float state is advanced with e - 1 (slots 0 and 3) in place of e
      for (int j = 0; j < nr; j++)
        for (int m = 0; m < nr; m++) {
          const double ks = (c->fx * m) * (c->fx * m) + (c->fy * j) * (c->fy * j);
          double em1[2];
          etd_em1(p, ks, em1);
          cf[0 * tsz + (size_t)j * nr + m] = (float)em1[0];
          cf[3 * tsz + (size_t)j * nr + m] = (float)em1[1];
        }
    }
    e = cudaMemcpy(c->coef, cf.data(), cf.size() * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->tw, tf.data(), tf.size() * 4, cudaMemcpyHostToDevice);
  } else {
    e = cudaMemcpy(c->coef, coef.data(), coef.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->tw, twd.data(), twd.size() * 8, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMemcpy(c->mrow, mrow.data(), nr * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && c->filtd)
    e = cudaMemcpy(c->filtd, filt.data(), tsz * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && c->filt && c->f32) {
    std::vector<float> ff(filt.begin(), filt.end());
    e = cudaMemcpy(c->filt, ff.data(), tsz * sizeof(float), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    free_all(c);
    return CHNS_ERR_CUDA;
  }
  *out = c;
  return CHNS_OK;
}

int chns_etd_coefficients(const chns_params* p, int i, int j, double* out) {
  const int rc = validate(p);
  if (rc != CHNS_OK) return rc;
  if (!out || i < 0 || i >= p->nx || j < 0 || j > p->nx / 2) return CHNS_ERR_ARG;
  const int m = i <= p->nx / 2 ? i : p->nx - i;
  etd_coefs(*p, mode_ksq((2 * M_PI) / p->lx, (2 * M_PI) / p->ly, m, j), out);
  return CHNS_OK;
}

int chns_truncation_rows(const chns_params* p, int* mrow) {
  const int rc = validate(p);
  if (rc != CHNS_OK) return rc;
  if (!mrow) return CHNS_ERR_ARG;
  truncation_rows(*p, (2 * M_PI) / p->lx, (2 * M_PI) / p->ly, mrow);
  return CHNS_OK;
}

int chns_truncation_factor(const chns_params* p, int i, int j, double* f) {
  const int rc = validate(p);
  if (rc != CHNS_OK) return rc;
  if (!f || i < 0 || i >= p->nx || j < 0 || j > p->nx / 2) return CHNS_ERR_ARG;
  const int m = i <= p->nx / 2 ? i : p->nx - i;
  const double fx = (2 * M_PI) / p->lx, fy = (2 * M_PI) / p->ly;
  if (p->filter == CHNS_FILTER_SMOOTH) {
    *f = filter_factor(*p, fx, fy, m, j);
  } else {
    const double dax = (p->nx / p->dealias_div) * fx;
    *f = mode_ksq(fx, fy, m, j) > dax * dax ? 0.0 : 1.0;
  }
  return CHNS_OK;
}

int chns_destroy(chns_ctx* c) {
  if (!c) return CHNS_ERR_ARG;
  cudaStreamSynchronize(c->stream);
  free_all(c);
  return CHNS_OK;
}

int chns_set_stream(chns_ctx* c, void* stream) {
  if (!c) return CHNS_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
  if (c->own_stream) cudaStreamDestroy(c->stream);
  c->stream = (cudaStream_t)stream;
  c->own_stream = false;
  if (c->step_graph) {
    cudaGraphExecDestroy(c->step_graph);
    c->step_graph = nullptr;
    c->graph_ok = false;
  }
  return CHNS_OK;
}

int chns_pin_host(chns_ctx* c, void* ptr, size_t bytes) {
  if (!c || !ptr || !bytes) return CHNS_ERR_ARG;
  for (int k = 0; k < c->npinned; k++)
    if (c->pinned[k] == ptr) return CHNS_OK;
  const cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterDefault);
  if (e == cudaErrorHostMemoryAlreadyRegistered) {
    cudaGetLastError();
    return CHNS_OK;  // page-locked by someone else: nothing to undo later
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return CHNS_ERR_CUDA;
  }
  if (c->npinned == (int)(sizeof(c->pinned) / sizeof(c->pinned[0]))) {
    cudaHostUnregister(ptr);
    return CHNS_ERR_UNSUPPORTED;
  }
  c->pinned[c->npinned++] = ptr;
  return CHNS_OK;
}

int chns_unpin_host(chns_ctx* c, void* ptr) {
  if (!c || !ptr) return CHNS_ERR_ARG;
  for (int k = 0; k < c->npinned; k++)
    if (c->pinned[k] == ptr) {
      cudaHostUnregister(ptr);
      c->pinned[k] = c->pinned[--c->npinned];
      return CHNS_OK;
    }
  return CHNS_ERR_ARG;
}

int chns_synchronize(chns_ctx* c) {
  if (!c) return CHNS_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  return tma_status(c);
}

// FFTW-layout double <-> S-layout double-float pair (hi = float rounding, lo =
// float rounding of the rest): the state of CHNS_FP32_STATE64.  32 x 32 tiles
// transposed through shared memory, as the plain layout conversions.
__global__ void k_fftw_to_hilo(const double2* __restrict__ src, float2* __restrict__ hi, float2* __restrict__ lo,
                               int n) {
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
      const float2 h = make_float2((float)v.x, (float)v.y);
      hi[(size_t)j * n + i] = h;
      lo[(size_t)j * n + i] = make_float2((float)(v.x - (double)h.x), (float)(v.y - (double)h.y));
    }
  }
}

__global__ void k_hilo_to_fftw(const float2* __restrict__ hi, const float2* __restrict__ lo, double2* __restrict__ dst,
                               int n) {
  __shared__ double2 tile[32][33];
  const int nr = n / 2 + 1;
  const int j0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int j = j0 + k, i = i0 + threadIdx.x;
    if (i < n && j < nr) {
      const float2 h = hi[(size_t)j * n + i], l = lo[(size_t)j * n + i];
      tile[threadIdx.x][k] = make_double2((double)h.x + (double)l.x, (double)h.y + (double)l.y);
    }
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int i = i0 + k, j = j0 + threadIdx.x;
    if (i < n && j < nr) dst[(size_t)i * nr + j] = tile[k][threadIdx.x];
  }
}

// low part of the k = 0 mode of field `slot` from its double value
__global__ void k_lo_k0(const float2* __restrict__ hi, float2* __restrict__ lo, const double* k0, int slot) {
  const float2 h = hi[0];
  lo[0] = make_float2((float)(k0[2 * slot] - (double)h.x), (float)(k0[2 * slot + 1] - (double)h.y));
}

static int set_field(chns_ctx* c, int f, const double* src, int where) {
  const size_t bytes = 2 * (size_t)c->n * c->nr * sizeof(double);
  int rc = to_device(c, c->stage, src, bytes, where);
  if (rc) return rc;
  if (c->st64) {
    const dim3 grid((c->nr + 31) / 32, (c->n + 31) / 32);
    k_fftw_to_hilo<<<grid, dim3(32, 8), 0, c->stream>>>((const double2*)c->stage, (float2*)c->state[f],
                                                         (float2*)c->statelo[f], c->n);
    // low parts only inside the sharp cut's disc (the smooth filter keeps every mode)
    if (c->p.filter == CHNS_FILTER_SHARP) c->L->truncate(c, c->statelo[f]);
  } else {
    c->L->from_fftw(c, c->stage, c->state[f]);
  }
  if (c->f32) k_k0_set<<<1, 1, 0, c->stream>>>(c->k0, c->stage, f);
  CK(cudaGetLastError());
  return CHNS_OK;
}

static int get_field(chns_ctx* c, int f, const void* s, double* dst, int where, int k0slot) {
  const size_t bytes = 2 * (size_t)c->n * c->nr * sizeof(double);
  c->L->to_fftw(c, s, c->stage);
  if (c->f32 && k0slot >= 0) k_k0_get<<<1, 1, 0, c->stream>>>(c->k0, c->stage, k0slot);
  CK(cudaGetLastError());
  return from_device(c, dst, c->stage, bytes, where);
}

int chns_set_state(chns_ctx* c, const double* w, const double* c1, const double* c2, int where) {
  if (!c) return CHNS_ERR_ARG;
  const double* src[3] = {w, c1, c2};
  for (int f = 0; f <= c->p.model; f++) {
    if (!src[f]) continue;
    int rc = set_field(c, f, src[f], where);
    if (rc) return rc;
  }
  return chns_synchronize(c);
}

int chns_get_state(chns_ctx* c, double* w, double* c1, double* c2, int where) {
  if (!c) return CHNS_ERR_ARG;
  double* dst[3] = {w, c1, c2};
  for (int f = 0; f <= c->p.model; f++) {
    if (!dst[f]) continue;
    int rc;
    if (c->st64) {
      const dim3 grid((c->nr + 31) / 32, (c->n + 31) / 32);
      k_hilo_to_fftw<<<grid, dim3(32, 8), 0, c->stream>>>((const float2*)c->state[f], (const float2*)c->statelo[f],
                                                          (double2*)c->stage, c->n);
      k_k0_get<<<1, 1, 0, c->stream>>>(c->k0, c->stage, f);
      CK(cudaGetLastError());
      rc = from_device(c, dst[f], c->stage, 2 * (size_t)c->n * c->nr * sizeof(double), where);
    } else {
      rc = get_field(c, f, c->state[f], dst[f], where, f);
    }
    if (rc) return rc;
  }
  return CHNS_OK;
}

int chns_statelo_reset(chns_ctx* c, int f) {
  if (!c->st64) return CHNS_OK;
  const size_t ncx = (size_t)c->n * c->nr;
  CK(cudaMemsetAsync(c->statelo[f], 0, ncx * sizeof(float2), c->stream));
  k_lo_k0<<<1, 1, 0, c->stream>>>((const float2*)c->state[f], (float2*)c->statelo[f], c->k0, f);
  CK(cudaGetLastError());
  return CHNS_OK;
}

// c->realdbl (n x n doubles) in the context precision in c->realbuf
int chns_realdbl_to_realbuf(chns_ctx* c) {
  const size_t nn = (size_t)c->n * c->n;
  if (c->f32) {
    k_real_d2r_f32<<<1024, 256, 0, c->stream>>>(c->realdbl, (float*)c->realbuf, nn);
  } else {
    CK(cudaMemcpyAsync(c->realbuf, c->realdbl, nn * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  }
  return CHNS_OK;
}

// phase field f (0: c / c1, 1: c2) from the real field in c->realdbl: dfft and
// truncation (init.c:221-225, 253-262); FP32 contexts take its k = 0 mode in double
int chns_phase_from_realdbl(chns_ctx* c, int f) {
  if (c->f32) {
    // FP32: the mean (the k = 0 mode) summed in double and kept there; the float
    // transform takes the field without it, so that its rounding is relative to the
    // fluctuations (a spinodal field is a mean of 1/3 or 1/2 with fluctuations of a
    // few per cent: transformed whole, the fluctuations' spectrum carried errors
    // ~1e-5 of itself, the mean's rounding spread over every mode)
    const size_t nn = (size_t)c->n * c->n;
    const int nb = 128;  // c->redscratch holds (n/2+1) 8 >= 136 doubles
    k_sum_blocks<<<nb, 256, 0, c->stream>>>(c->realdbl, nn, (double*)c->redscratch);
    k_sum_finish<<<1, 1, 0, c->stream>>>((const double*)c->redscratch, nb, c->k0, 1 + f);
    k_real_d2r_f32_dev<<<1024, 256, 0, c->stream>>>(c->realdbl, (float*)c->realbuf, nn, c->k0, 1 + f);
    c->L->dfft(c, c->realbuf, c->state[1 + f]);
    c->L->truncate(c, c->state[1 + f]);
    k_k0_to_state<<<1, 1, 0, c->stream>>>(c->k0, (float2*)c->state[1 + f], 1 + f);
  } else {
    int rc = chns_realdbl_to_realbuf(c);
    if (rc) return rc;
    c->L->dfft(c, c->realbuf, c->state[1 + f]);
    c->L->truncate(c, c->state[1 + f]);
  }
  CK(cudaGetLastError());
  return chns_statelo_reset(c, 1 + f);
}

int chns_set_phase_real(chns_ctx* c, const double* p1, const double* p2, int where) {
  if (!c || c->p.model == CHNS_MODEL_NS) return CHNS_ERR_ARG;
  if (!p1 || (c->p.model == CHNS_MODEL_TERNARY && !p2)) return CHNS_ERR_ARG;
  const size_t bytes = (size_t)c->n * c->nr * 2 * c->rsz;
  CK(cudaMemsetAsync(c->state[0], 0, bytes, c->stream));  // init.c:78-87
  if (c->f32) CK(cudaMemsetAsync(c->k0, 0, 2 * sizeof(double), c->stream));
  if (c->st64) CK(cudaMemsetAsync(c->statelo[0], 0, bytes, c->stream));
  const double* src[2] = {p1, p2};
  for (int f = 0; f < c->p.model; f++) {
    const size_t nn = (size_t)c->n * c->n;
    int rc = to_device(c, c->realdbl, src[f], nn * sizeof(double), where);
    if (!rc) rc = chns_phase_from_realdbl(c, f);
    if (rc) return rc;
  }
  CK(cudaGetLastError());
  return chns_synchronize(c);
}

int chns_step(chns_ctx* c, int nsteps) {
  if (!c || nsteps < 0) return CHNS_ERR_ARG;
  if (nsteps == 0) return CHNS_OK;
  if (!c->graph_ok) {
    if (build_graph(c) != CHNS_OK) {
      cudaGetLastError();
      c->graph_ok = false;
    }
  }
  for (int s = 0; s < nsteps; s++) {
    if (c->graph_ok) {
      CK(cudaGraphLaunch(c->step_graph, c->stream));
    } else {
      enqueue_step(c);
    }
  }
  CK(cudaGetLastError());
  return CHNS_OK;
}

int chns_rhs(chns_ctx* c, double* nw, double* nc1, double* nc2, int where) {
  if (!c) return CHNS_ERR_ARG;
  // stage 1 stores N(u) of the current state in the `saved` buffers; run it on
  // a copy of the state and restore the state afterwards
  const size_t bytes = (size_t)c->n * c->nr * 2 * c->rsz;
  void* keep[3] = {nullptr, nullptr, nullptr};
  void* keeplo[3] = {nullptr, nullptr, nullptr};
  double k0keep[12];
  int rc = CHNS_OK;
  for (int f = 0; f <= c->p.model && rc == CHNS_OK; f++) {
    if (cudaMalloc(&keep[f], bytes) != cudaSuccess) rc = CHNS_ERR_NOMEM;
    else if (cudaMemcpyAsync(keep[f], c->state[f], bytes, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
      rc = CHNS_ERR_CUDA;
    if (rc == CHNS_OK && c->st64) {
      if (cudaMalloc(&keeplo[f], bytes) != cudaSuccess) rc = CHNS_ERR_NOMEM;
      else if (cudaMemcpyAsync(keeplo[f], c->statelo[f], bytes, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
        rc = CHNS_ERR_CUDA;
    }
  }
  bool k0kept = false;  // k0keep holds the k = 0 modes (FP32 contexts)
  if (rc == CHNS_OK && c->f32) {
    if (cudaMemcpy(k0keep, c->k0, sizeof(k0keep), cudaMemcpyDeviceToHost) != cudaSuccess) rc = CHNS_ERR_CUDA;
    else k0kept = true;
  }
  const bool ran = rc == CHNS_OK;  // the stage overwrites the state: restore it from the copies
  if (ran) c->L->stage(c, 1);
  double* dst[3] = {nw, nc1, nc2};
  for (int f = 0; f <= c->p.model && rc == CHNS_OK; f++)
    if (dst[f]) rc = get_field(c, f, c->saved[f], dst[f], where, 3 + f);
  // restore the state (a failed restore is reported: the state is then undefined)
  int rrc = CHNS_OK;
  for (int f = 0; f <= c->p.model; f++) {
    if (keep[f]) {
      if (ran && cudaMemcpyAsync(c->state[f], keep[f], bytes, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
        rrc = CHNS_ERR_CUDA;
      if (cudaStreamSynchronize(c->stream) != cudaSuccess) rrc = CHNS_ERR_CUDA;
      cudaFree(keep[f]);
    }
    if (keeplo[f]) {
      if (ran && cudaMemcpyAsync(c->statelo[f], keeplo[f], bytes, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
        rrc = CHNS_ERR_CUDA;
      if (cudaStreamSynchronize(c->stream) != cudaSuccess) rrc = CHNS_ERR_CUDA;
      cudaFree(keeplo[f]);
    }
  }
  if (ran && k0kept && cudaMemcpy(c->k0, k0keep, sizeof(k0keep), cudaMemcpyHostToDevice) != cudaSuccess) rrc = CHNS_ERR_CUDA;
  if (rc == CHNS_OK) rc = rrc;
  if (rc == CHNS_OK) rc = chns_synchronize(c);
  return rc;
}

int chns_dfft(chns_ctx* c, const double* real, double* spec, int where) {
  if (!c || !real || !spec) return CHNS_ERR_ARG;
  int rc = to_device(c, c->realdbl, real, (size_t)c->n * c->n * sizeof(double), where);
  if (!rc) rc = chns_realdbl_to_realbuf(c);
  if (rc) return rc;
  c->L->dfft(c, c->realbuf, c->nw);
  return get_field(c, 0, c->nw, spec, where, -1);
}

int chns_ifft(chns_ctx* c, const double* spec, double* real, int where) {
  if (!c || !real || !spec) return CHNS_ERR_ARG;
  const size_t nn = (size_t)c->n * c->n;
  int rc = to_device(c, c->stage, spec, 2 * (size_t)c->n * c->nr * sizeof(double), where);
  if (rc) return rc;
  c->L->from_fftw(c, c->stage, c->nw);
  c->L->ifft(c, c->nw, c->realbuf);
  if (c->f32) {
    k_real_r2d_f32<<<1024, 256, 0, c->stream>>>((const float*)c->realbuf, c->realdbl, nn);
  } else {
    CK(cudaMemcpyAsync(c->realdbl, c->realbuf, nn * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  }
  CK(cudaGetLastError());
  return from_device(c, real, c->realdbl, nn * sizeof(double), where);
}

// real-space field f of the state (optionally truncated first) in c->realdbl
int chns_field_to_realdbl(chns_ctx* c, int f, int truncate) {
  const size_t nn = (size_t)c->n * c->n;
  const size_t bytes = (size_t)c->n * c->nr * 2 * c->rsz;
  const void* src = c->state[f];
  if (truncate) {
    CK(cudaMemcpyAsync(c->nw, c->state[f], bytes, cudaMemcpyDeviceToDevice, c->stream));
    c->L->truncate(c, c->nw);
    src = c->nw;
  }
  c->L->ifft(c, src, c->realbuf);
  if (c->f32) {
    k_real_r2d_f32<<<1024, 256, 0, c->stream>>>((const float*)c->realbuf, c->realdbl, nn);
  } else {
    CK(cudaMemcpyAsync(c->realdbl, c->realbuf, nn * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  }
  CK(cudaGetLastError());
  return CHNS_OK;
}

int chns_check(chns_ctx* c) {
  if (!c) return CHNS_ERR_ARG;
  unsigned int* flag = (unsigned int*)c->redscratch;
  CK(cudaMemsetAsync(flag, 0, sizeof(unsigned int), c->stream));
  const size_t nr = (size_t)c->n * c->nr * 2;  // reals per spectral field
  for (int f = 0; f <= c->p.model; f++) {
    if (c->f32)
      k_nonfinite<float><<<1024, 256, 0, c->stream>>>((const float*)c->state[f], nr, flag);
    else
      k_nonfinite<double><<<1024, 256, 0, c->stream>>>((const double*)c->state[f], nr, flag);
  }
  if (c->f32) k_nonfinite<double><<<1, 32, 0, c->stream>>>(c->k0, 6, flag);
  CK(cudaGetLastError());
  unsigned int h = 0;
  CK(cudaMemcpyAsync(&h, flag, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (h) return CHNS_ERR_NONFINITE;
  return tma_status(c);
}

int chns_diagnostics(chns_ctx* c, double* out_fe, double* out_ke) {
  if (!c) return CHNS_ERR_ARG;
  c->L->diag(c);
  CK(cudaGetLastError());
  double r[8];
  CK(cudaMemcpyAsync(r, c->red, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const chns_params& p = c->p;
  const double scale = 1.0 / ((double)p.nx * (double)p.ny);
  double fe[2] = {0.0, 0.0};
  if (p.model == CHNS_MODEL_BINARY) {
    fe[0] = r[0] * (12.0 * (p.sigma / p.epsilon)) * scale;  // free_energy.c:39-42
    fe[1] = r[1] * ((0.75 * p.sigma * p.epsilon) * scale);  // free_energy.c:96
  } else if (p.model == CHNS_MODEL_TERNARY) {
    fe[0] = r[0] * (6.0 / p.epsilon) * scale;  // free_energy.c:48-54
    fe[1] = r[1] * (0.375 * p.epsilon * scale);  // free_energy.c:141
  }
  double ke[3];
  ke[0] = r[2] * scale;                   // kinetic_energy.c:94
  ke[1] = r[5] > 0 ? r[3] / r[5] : 0.0;   // kinetic_energy.c:103-106
  ke[2] = r[6] > 0 ? r[4] / r[6] : 0.0;   // kinetic_energy.c:123-131
  if (out_fe) memcpy(out_fe, fe, sizeof(fe));
  if (out_ke) memcpy(out_ke, ke, sizeof(ke));
  for (int k = 0; k < 7; k++)
    if (!isfinite(r[k])) return CHNS_ERR_NONFINITE;
  if (fe[0] >= 100.0) return CHNS_ERR_NONFINITE;  // the reference's blow-up guard (free_energy.c:151-154)
  return CHNS_OK;
}

int chns_launches_per_step(const chns_ctx* c) { return c ? c->launches_per_step : 0; }

int chns_tma_tiles(const chns_ctx* c) { return c && static_cast<const chns::TmaG*>(c->tmag)->use ? 1 : 0; }

int chns_tune_value(int knob) {
  switch (knob) {
    case CHNS_TUNE_TMA_BOX_ROWS: return g_tune_box_rows;
    case CHNS_TUNE_P1_SPLIT: return g_tune_p1_split;
    case CHNS_TUNE_P4_GRAD: return g_tune_p4_grad;
    case CHNS_TUNE_PDL: return g_tune_pdl;
    default: return -1;
  }
}

int chns_tune_override(int knob, int value) {
  if (knob == CHNS_TUNE_TMA_BOX_ROWS) {
    if (value != -1 && (value < 8 || value > 256 || value % 8 != 0)) return CHNS_ERR_ARG;
    g_tune_box_rows = value;
    return CHNS_OK;
  }
  if (knob == CHNS_TUNE_P1_SPLIT || knob == CHNS_TUNE_P4_GRAD || knob == CHNS_TUNE_PDL) {
    if (value != -1 && value != 0 && value != 1) return CHNS_ERR_ARG;
    (knob == CHNS_TUNE_P1_SPLIT ? g_tune_p1_split : knob == CHNS_TUNE_P4_GRAD ? g_tune_p4_grad : g_tune_pdl) = value;
    return CHNS_OK;
  }
  return CHNS_ERR_ARG;
}

int chns_debug_tile_waits(chns_ctx* c, int spins, int skip_copies) {
  if (!c || spins < 0) return CHNS_ERR_ARG;
  chns::TmaG* T = static_cast<chns::TmaG*>(c->tmag);
  if (!T->use) return CHNS_ERR_UNSUPPORTED;
  CK(cudaStreamSynchronize(c->stream));
  T->spins = spins;
  T->skip = skip_copies ? 1 : 0;
  // the captured step holds the kernels' arguments: capture it again
  if (c->step_graph) {
    cudaGraphExecDestroy(c->step_graph);
    c->step_graph = nullptr;
    c->graph_ok = false;
  }
  return CHNS_OK;
}

int chns_profile_step(chns_ctx* c, int reps, float* ms, int* kind, int maxk) {
  if (!c || reps < 1 || !ms || !kind || maxk < 1) return CHNS_ERR_ARG;
  const int cap = 64;
  cudaEvent_t ev[cap + 1];
  int kinds[cap];
  for (int k = 0; k <= cap; k++)
    if (cudaEventCreate(&ev[k]) != cudaSuccess) return CHNS_ERR_CUDA;
  for (int k = 0; k < maxk; k++) ms[k] = 0.0f;
  int nk = 0;
  int rc = CHNS_OK;
  for (int r = 0; r < reps && rc == CHNS_OK; r++) {
    c->prof_ev = ev + 1;
    c->prof_kind = kinds;
    c->prof_n = 0;
    c->prof_max = cap;
    cudaEventRecord(ev[0], c->stream);
    enqueue_step(c);
    nk = c->prof_n;
    c->prof_ev = nullptr;
    if (cudaEventSynchronize(ev[nk]) != cudaSuccess) rc = CHNS_ERR_CUDA;
    for (int k = 0; k < nk && k < maxk && rc == CHNS_OK; k++) {
      float t = 0.0f;
      cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
      ms[k] += t / reps;
      kind[k] = kinds[k];
    }
  }
  c->prof_ev = nullptr;
  for (int k = 0; k <= cap; k++) cudaEventDestroy(ev[k]);
  if (rc != CHNS_OK) return rc;
  return nk < maxk ? nk : maxk;
}

const char* chns_status_string(int s) {
  switch (s) {
    case CHNS_OK: return "ok";
    case CHNS_ERR_ARG: return "bad argument";
    case CHNS_ERR_CUDA: return "CUDA error";
    case CHNS_ERR_NONFINITE: return "non-finite or blown-up state";
    case CHNS_ERR_TIMEOUT: return "device wait timed out";
    case CHNS_ERR_UNSUPPORTED: return "unsupported size or option";
    case CHNS_ERR_NOMEM: return "out of memory";
    case CHNS_ERR_IO: return "file could not be read or written";
  }
  return "unknown status";
}

}  // extern "C"
