// chns_init.cu -- the reference's initial conditions (init.c) on the device.
//
// Vorticity: zero (ZERO_INIT / INIT_READ_DATA, init.c:67-96), the Taylor-Green
// field (TG_INIT, init.c:38-65: u = a (sin x cos y, -cos x sin y), dfft, curl,
// truncation) or the k-space shell field of the remaining branch (init.c:102-182).  Phase fields: the binary centred tanh drop (init.c:231-248) and
// the ternary noise c_i = 1/4 + 0.001 r (init.c:264-292), each followed by dfft
// and truncation as in init.c.  The noise draws are the C library's rand()
// sequence after srand(seed) (the reference seeds 10 + 2 rank), produced on the
// host with a private random_r state because the generator is sequential; the
// fields, transforms and truncation run on the GPU.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "chns_internal.h"
#include "chns_kernels.cuh"

namespace {

#define IK(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return CHNS_ERR_CUDA;  \
  } while (0)

// phi = 0.5 (1 - tanh((r - pi/4.5) / (0.5 eps))), r from the box centre (init.c:240-246)
__global__ void k_init_drop(double* __restrict__ out, int n, double dx, double dy, double lx, double ly,
                            double eps) {
  const size_t nn = (size_t)n * n;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(k / n), j = (int)(k % n);
    const double x = i * dx, y = j * dy;
    const double r = sqrt((x - lx / 2.0) * (x - lx / 2.0) + (y - ly / 2.0) * (y - ly / 2.0));
    out[k] = 0.5 * (1.0 - tanh((r - (M_PI / 4.5)) / (0.5 * eps)));
  }
}

// c = 1/4 + 0.001 rand() / RAND_MAX (init.c:281-287)
__global__ void k_init_noise(const uint32_t* __restrict__ r, double* __restrict__ out, size_t nn, double rmax) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x)
    out[k] = (1.0 / 4.0) + 0.001 * ((double)r[k] / rmax);
}

// u_x (comp 0) or u_y (comp 1) of the Taylor-Green field (init.c:51-55)
__global__ void k_init_tg(double* __restrict__ out, int n, double dx, double dy, double amp, int comp) {
  const size_t nn = (size_t)n * n;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(k / n), j = (int)(k % n);
    const double x = i * dx, y = j * dy;
    const double u = comp == 0 ? sin(x) * cos(y) : -cos(x) * sin(y);
    out[k] = u * amp;
  }
}

// omega_hat = I (kx uy_hat - ky ux_hat) on the S layout (curl.c:16-31)
template <class R>
__global__ void k_init_curl(const chns::cx<R>* __restrict__ ux, const chns::cx<R>* __restrict__ uy,
                            chns::cx<R>* __restrict__ w, int n, double fx, double fy) {
  const size_t total = (size_t)(n / 2 + 1) * n;
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int row = (int)(idx / n), i = (int)(idx % n);
  const R kx = (R)(fx * (double)(i <= n / 2 ? i : i - n)), ky = (R)(fy * (double)row);
  const chns::cx<R> a = ux[idx], b = uy[idx];
  const R re = kx * b.x - ky * a.x, im = kx * b.y - ky * a.y;
  w[idx] = chns::mk<R>(-im, re);
}

// init.c:102-128: modes per shell rint(|k|) (MPI_Allreduce over one rank), the
// ky = 0 and ky = kymax columns counted once, the others twice (their conjugates)
__global__ void k_shell_count(int* __restrict__ den, int n, int kmax, double fx, double fy, double kymax,
                              int* __restrict__ err) {
  const int nr = n / 2 + 1;
  const size_t total = (size_t)n * nr;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / nr), j = (int)(idx % nr);  // FFTW layout: row i (kx), column j (ky)
    const double kx = fx * (double)(i <= n / 2 ? i : i - n), ky = fy * (double)j;
    const double ksqr = chns::radd(chns::rmul(kx, kx), chns::rmul(ky, ky));
    const int ik = (int)rint(sqrt(ksqr));
    if (ik < 0 || ik > kmax) { atomicOr(err, 1); continue; }
    atomicAdd(&den[ik], (ky == 0.0 || ky == kymax) ? 1 : 2);
  }
}

// init.c:130-181 per mode, into the S layout (row j = ky index, column i):
// vk = sqrt(k^4 e^{-2 k^2} / (3 den[round |k|])) nx ny; v1 = v2 = uamp vk (the phase
// factors exp(I 2 pi r) of init.c:156-157 go through the real exp() and are 1);
// u_hat = P v with the projector of init.c:161-175; omega_hat = I (kx uy - ky ux).
template <class R>
__global__ void k_shell_omega(const int* __restrict__ den, chns::cx<R>* __restrict__ w, int n, double fx, double fy,
                              double uamp, int* __restrict__ err) {
  using namespace chns;
  const size_t total = (size_t)(n / 2 + 1) * n;
  const double ncube = (double)n * (double)n;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(idx / n), i = (int)(idx % n);
    const double kx = fx * (double)(i <= n / 2 ? i : i - n), ky = fy * (double)j;
    const double ksqr = radd(rmul(kx, kx), rmul(ky, ky));
    const int ik = (int)round(sqrt(ksqr));
    const double ee = rmul(rmul(ksqr, ksqr), exp(rmul(-2.0, ksqr)));
    const int d = den[ik];
    // an empty shell would make the reference reuse the previous mode's vk
    if (d == 0) { atomicOr(err, 2); continue; }
    const double vk = rmul(sqrt(rdiv(ee, rmul(3.0, (double)d))), ncube);
    const double s = rmul(uamp, vk);
    double p11, p22, p12;
    if (ksqr > 1e-5) {
      p11 = rsub(1.0, rdiv(rmul(kx, kx), ksqr));
      p22 = rsub(1.0, rdiv(rmul(ky, ky), ksqr));
      p12 = rdiv(rmul(-kx, ky), ksqr);
    } else {
      p11 = 1.0 / 2.0;
      p22 = p11;
      p12 = -1.0 / 2.0;
    }
    const double ux = radd(rmul(p11, s), rmul(p12, s));
    const double uy = radd(rmul(p12, s), rmul(p22, s));
    const double dr = rsub(rmul(kx, uy), rmul(ky, ux));  // curl.c:16-31; the imaginary parts are 0
    w[idx] = mk<R>((R)0, (R)dr);
  }
}

int grid_for(size_t nn) {
  const size_t b = (nn + 255) / 256;
  return (int)(b < 4096 ? b : 4096);
}

}  // namespace

extern "C" {

int chns_init_vorticity(chns_ctx* c, int kind, double amplitude) {
  if (!c) return CHNS_ERR_ARG;
  const size_t bytes = (size_t)c->n * c->nr * 2 * c->rsz;
  if (kind == CHNS_INIT_W_ZERO) {
    IK(cudaMemsetAsync(c->state[0], 0, bytes, c->stream));
  } else if (kind == CHNS_INIT_W_TAYLOR_GREEN) {
    const size_t nn = (size_t)c->n * c->n;
    const double dx = c->p.lx / c->n, dy = c->p.ly / c->n;
    // u_x_hat in the partial-N_w buffer and u_y_hat in the saved N_w buffer: both
    // S-layout fields that every model allocates and the next step rewrites
    void* uh[2] = {c->nw, c->saved[0]};
    if (!uh[0] || !uh[1] || !c->realdbl || !c->realbuf) return CHNS_ERR_ARG;
    for (int comp = 0; comp < 2; comp++) {
      k_init_tg<<<grid_for(nn), 256, 0, c->stream>>>(c->realdbl, c->n, dx, dy, amplitude, comp);
      int rc = chns_realdbl_to_realbuf(c);
      if (rc) return rc;
      c->L->dfft(c, c->realbuf, uh[comp]);
    }
    const int blocks = (int)(((size_t)c->n * c->nr + 255) / 256);
    if (c->f32)
      k_init_curl<float><<<blocks, 256, 0, c->stream>>>((const chns::cx<float>*)uh[0], (const chns::cx<float>*)uh[1],
                                                        (chns::cx<float>*)c->state[0], c->n, c->fx, c->fy);
    else
      k_init_curl<double><<<blocks, 256, 0, c->stream>>>((const chns::cx<double>*)uh[0],
                                                         (const chns::cx<double>*)uh[1],
                                                         (chns::cx<double>*)c->state[0], c->n, c->fx, c->fy);
    c->L->truncate(c, c->state[0]);
  } else if (kind == CHNS_INIT_W_SHELL) {
    // the shell counts and an error word live in the context's real buffer
    const double kxmax = (c->n / 2.0) * c->fx, kymax = (c->n / 2.0) * c->fy;
    const int kmax = (int)round(sqrt(kxmax * kxmax + kymax * kymax));
    if ((size_t)(kmax + 2) * sizeof(int) > (size_t)c->n * c->n * c->rsz || !c->realbuf) return CHNS_ERR_UNSUPPORTED;
    int* den = (int*)c->realbuf;
    int* err = den + kmax + 1;
    IK(cudaMemsetAsync(den, 0, (size_t)(kmax + 2) * sizeof(int), c->stream));
    const size_t modes = (size_t)c->n * c->nr;
    k_shell_count<<<grid_for(modes), 256, 0, c->stream>>>(den, c->n, kmax, c->fx, c->fy, kymax, err);
    if (c->f32)
      k_shell_omega<float><<<grid_for(modes), 256, 0, c->stream>>>(den, (chns::cx<float>*)c->state[0], c->n, c->fx,
                                                                   c->fy, amplitude, err);
    else
      k_shell_omega<double><<<grid_for(modes), 256, 0, c->stream>>>(den, (chns::cx<double>*)c->state[0], c->n,
                                                                    c->fx, c->fy, amplitude, err);
    int herr = 0;
    IK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    IK(cudaStreamSynchronize(c->stream));
    if (herr) return CHNS_ERR_UNSUPPORTED;
    c->L->truncate(c, c->state[0]);
  } else {
    return CHNS_ERR_ARG;
  }
  if (c->f32) IK(cudaMemsetAsync(c->k0, 0, 2 * sizeof(double), c->stream));  // the mean vorticity is 0
  if (int rc = chns_statelo_reset(c, 0)) return rc;
  IK(cudaGetLastError());
  return chns_synchronize(c);
}

int chns_init_phase(chns_ctx* c, int kind, unsigned int seed) {
  if (!c || c->p.model == CHNS_MODEL_NS) return CHNS_ERR_ARG;
  const size_t nn = (size_t)c->n * c->n;
  if (kind == CHNS_INIT_C_DROP) {
    if (c->p.model != CHNS_MODEL_BINARY) return CHNS_ERR_ARG;
    k_init_drop<<<grid_for(nn), 256, 0, c->stream>>>(c->realdbl, c->n, c->p.lx / c->n, c->p.ly / c->n, c->p.lx,
                                                     c->p.ly, c->p.epsilon);
    int rc = chns_phase_from_realdbl(c, 0);
    if (rc) return rc;
  } else if (kind == CHNS_INIT_C_NOISE) {
    if (c->p.model != CHNS_MODEL_TERNARY) return CHNS_ERR_ARG;
    // rand() after srand(seed): two draws per grid point in row-major order (rn1, rn2)
    std::vector<uint32_t> r1(nn), r2(nn);
    char statebuf[128];
    struct random_data rd;
    memset(&rd, 0, sizeof(rd));
    if (initstate_r(seed, statebuf, sizeof(statebuf), &rd) != 0) return CHNS_ERR_ARG;
    for (size_t k = 0; k < nn; k++) {
      int32_t a, b;
      random_r(&rd, &a);
      random_r(&rd, &b);
      r1[k] = (uint32_t)a;
      r2[k] = (uint32_t)b;
    }
    // the draws go through the context's real buffer (at least n^2 x 4 bytes)
    const std::vector<uint32_t>* rs[2] = {&r1, &r2};
    for (int f = 0; f < 2; f++) {
      IK(cudaMemcpyAsync(c->realbuf, rs[f]->data(), nn * sizeof(uint32_t), cudaMemcpyHostToDevice, c->stream));
      k_init_noise<<<grid_for(nn), 256, 0, c->stream>>>((const uint32_t*)c->realbuf, c->realdbl, nn,
                                                        (double)RAND_MAX);
      int rc = chns_phase_from_realdbl(c, f);
      if (rc) return rc;
      IK(cudaStreamSynchronize(c->stream));  // before the host draws are released
    }
  } else {
    return CHNS_ERR_ARG;
  }
  IK(cudaGetLastError());
  return chns_synchronize(c);
}

}  // extern "C"
