// chns_diag_extra.cu -- the reference's remaining per-step diagnostics on the device:
// shell spectra (spectrum.c:3-194) and the interface perimeter (perimeter.c:3-271).
//
// spectrum: every stored mode adds its truncated velocity energy, enstrophy and
// phase-field energies to shell (int)(|k|/dk + 0.5) and to the kx / ky bins, with
// the reference's weights (ky = 0 and ky = kymax columns once, the others twice).
// Unlike spectrum.c the state is not truncated in place.  The sums use double
// atomics, so their order (and the last bits) vary from call to call.
// perimeter: thresholds the real-space phase field at 0.5 and counts cells whose
// +x or +y neighbour (periodic) lies on the other side, and cells above it.
#include <cuda_runtime.h>
#include <math.h>

#include <vector>

#include "chns_internal.h"
#include "chns_kernels.cuh"

namespace {

#define DK(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return CHNS_ERR_CUDA;  \
  } while (0)

struct SpecArgs {
  int n, jt, nshell, nph;
  double fx, fy, dk, scale2;
  const int* mrow;
  const double* filt;  // SMOOTH_FILTER factors [row][|m|] in double (null: the sharp cut)
  const double* k0;  // FP32 contexts: k = 0 modes in double, else null
  double* out;       // ek, ensk, phase spectra (nph x nshell), ekx, eky
};

template <class R>
__device__ __forceinline__ void load_mode(const chns::cx<R>* f, size_t idx, double& re, double& im) {
  const chns::cx<R> v = f[idx];
  re = (double)v.x;
  im = (double)v.y;
}

template <class R>
__global__ void k_spectrum(const chns::cx<R>* __restrict__ w, const chns::cx<R>* __restrict__ c1,
                           const chns::cx<R>* __restrict__ c2, const SpecArgs A) {
  const int n = A.n;
  const size_t total = (size_t)(n / 2 + 1) * n;
  const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const int row = (int)(idx / n), i = (int)(idx % n);
  const int m = i <= n / 2 ? i : i - n;
  const double kx = A.fx * (double)m, ky = A.fy * (double)row;
  const double kxsqr = kx * kx, kysqr = ky * ky, ksqr = kxsqr + kysqr;
  const int ik = (int)((sqrt(ksqr) / A.dk) + 0.5);
  const int ikx = (int)((sqrt(kxsqr) / A.dk) + 0.5);
  const int iky = (int)((sqrt(kysqr) / A.dk) + 0.5);
  const int am = m < 0 ? -m : m;
  const bool in = row <= A.jt && am <= A.mrow[row];  // truncation (functions.c:47-84)
  const bool edge = row == 0 || row == n / 2;         // ky == 0 or ky == kymax
  double eu = 0.0;
  if (in && ksqr > 1e-12) {  // velocity.c: psi = w / k^2, ux = i ky psi, uy = -i kx psi
    double wr, wi;
    load_mode(w, idx, wr, wi);
    const double pr = wr / ksqr, pi_ = wi / ksqr;
    double uxr = -ky * pi_, uxi = ky * pr, uyr = kx * pi_, uyi = -kx * pr;
    if (A.filt) {  // functions.c:69-72
      const double f = A.filt[(size_t)row * (n / 2 + 1) + am];
      uxr = (uxr * f) * f; uxi = (uxi * f) * f; uyr = (uyr * f) * f; uyi = (uyi * f) * f;
    }
    eu = (uxr * uxr + uxi * uxi) + (uyr * uyr + uyi * uyi);
  }
  eu *= A.scale2;
  const double ens = eu * ksqr;
  const int ns = A.nshell;
  double* ek = A.out;
  double* ensk = ek + ns;
  double* sph = ensk + ns;
  double* ekx = sph + (size_t)A.nph * ns;
  double* eky = ekx + (n / 2 + 1);
  const double wu = edge ? 0.5 : 1.0;
  if (eu != 0.0) {
    atomicAdd(ek + ik, wu * eu);
    atomicAdd(ensk + ik, wu * ens);
    atomicAdd(ekx + ikx, wu * eu);
    atomicAdd(eky + iky, wu * eu);
  }
  if (A.nph > 0 && in) {
    const double wp = edge ? 1.0 : 2.0;
    double ar, ai, br = 0.0, bi = 0.0;
    load_mode(c1, idx, ar, ai);
    if (A.k0 && idx == 0) {
      ar = A.k0[2];
      ai = A.k0[3];
    }
    if (A.nph == 3) {
      load_mode(c2, idx, br, bi);
      if (A.k0 && idx == 0) {
        br = A.k0[4];
        bi = A.k0[5];
      }
    }
    if (A.filt) {
      const double f = A.filt[(size_t)row * (n / 2 + 1) + am];
      ar = (ar * f) * f; ai = (ai * f) * f; br = (br * f) * f; bi = (bi * f) * f;
    }
    const double e1 = (ar * ar + ai * ai) * A.scale2;
    atomicAdd(sph + ik, wp * e1);
    if (A.nph == 3) {
      const double e2 = (br * br + bi * bi) * A.scale2;
      const double e12 = fabs((ar * br + ai * bi) * A.scale2);
      atomicAdd(sph + ns + ik, wp * e2);
      atomicAdd(sph + 2 * ns + ik, wp * e12);
    }
  }
}

// counts[0] += cells with a sign change towards (i+1, j) or (i, j+1); counts[1] += cells >= 0.5
__global__ void k_perimeter(const double* __restrict__ ph, int n, unsigned long long* counts) {
  const size_t nn = (size_t)n * n;
  unsigned long long a = 0, b = 0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nn; k += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(k / n), j = (int)(k % n);
    const int ip = i + 1 < n ? i + 1 : 0, jp = j + 1 < n ? j + 1 : 0;
    const double s = ph[k] >= 0.5 ? 1.0 : -1.0;
    const double si = ph[(size_t)ip * n + j] >= 0.5 ? 1.0 : -1.0;
    const double sj = ph[(size_t)i * n + jp] >= 0.5 ? 1.0 : -1.0;
    if (s * si < 0.0 || s * sj < 0.0) a++;
    if (s > 0.0) b++;
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (a) atomicAdd(counts, a);
    if (b) atomicAdd(counts + 1, b);
  }
}

int nshell_of(int n) { return (int)lround((double)n / sqrt(2.0) + 1.0); }

}  // namespace

extern "C" {

int chns_spectrum_shells(const chns_ctx* c) { return c ? nshell_of(c->n) : 0; }

int chns_spectrum(chns_ctx* c, double* out) {
  if (!c || !out) return CHNS_ERR_ARG;
  const int n = c->n, ns = nshell_of(n);
  const int nph = c->p.model == CHNS_MODEL_BINARY ? 1 : (c->p.model == CHNS_MODEL_TERNARY ? 3 : 0);
  const size_t len = (size_t)(2 + nph) * ns + 2 * (size_t)(n / 2 + 1);
  double* dev = nullptr;
  if (len * sizeof(double) > 2 * (size_t)c->n * c->nr * sizeof(double)) return CHNS_ERR_UNSUPPORTED;
  dev = c->stage;  // FFTW-layout staging, n (n/2+1) complex doubles: room for the bins
  DK(cudaMemsetAsync(dev, 0, len * sizeof(double), c->stream));
  SpecArgs A;
  A.n = n;
  A.jt = c->jt;
  A.nshell = ns;
  A.nph = nph;
  A.fx = c->fx;
  A.fy = c->fy;
  A.dk = 2.0 * M_PI / c->p.lx;
  const double scale = 1.0 / ((double)c->p.nx * (double)c->p.ny);
  A.scale2 = scale * scale;
  A.mrow = c->mrow;
  A.filt = c->filtd;
  A.k0 = c->f32 ? c->k0 : nullptr;
  A.out = dev;
  const int blocks = (int)(((size_t)n * c->nr + 255) / 256);
  if (c->f32)
    k_spectrum<float><<<blocks, 256, 0, c->stream>>>(
        (const chns::cx<float>*)c->state[0], (const chns::cx<float>*)(nph ? c->state[1] : c->state[0]),
        (const chns::cx<float>*)(nph == 3 ? c->state[2] : c->state[0]), A);
  else
    k_spectrum<double><<<blocks, 256, 0, c->stream>>>(
        (const chns::cx<double>*)c->state[0], (const chns::cx<double>*)(nph ? c->state[1] : c->state[0]),
        (const chns::cx<double>*)(nph == 3 ? c->state[2] : c->state[0]), A);
  DK(cudaGetLastError());
  DK(cudaMemcpyAsync(out, dev, len * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  DK(cudaStreamSynchronize(c->stream));
  return CHNS_OK;
}

int chns_perimeter(chns_ctx* c, double* out) {
  if (!c || !out || c->p.model == CHNS_MODEL_NS) return CHNS_ERR_ARG;
  const double dx = c->p.lx / c->p.nx, dy = c->p.ly / c->p.ny;
  unsigned long long* cnt = (unsigned long long*)c->red;  // 16 doubles of reduction space
  for (int f = 0; f < c->p.model; f++) {
    int rc = chns_field_to_realdbl(c, 1 + f, 0);  // perimeter.c:26-27: ifft of the untruncated state
    if (rc) return rc;
    DK(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), c->stream));
    k_perimeter<<<1024, 256, 0, c->stream>>>(c->realdbl, c->n, cnt);
    unsigned long long h[2];
    DK(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    DK(cudaStreamSynchronize(c->stream));
    const double sp_t = (double)h[0] * dx;                               // perimeter.c:112
    const double sp_0 = 2.0 * sqrt(M_PI * (double)h[1] * dx * dy);       // perimeter.c:113
    double* o = out + 5 * f;
    o[0] = (double)h[0];
    o[1] = (double)h[1];
    o[2] = sp_0;
    o[3] = sp_t;
    o[4] = (sp_t / sp_0) - 1.0;
  }
  return CHNS_OK;
}

}  // extern "C"
