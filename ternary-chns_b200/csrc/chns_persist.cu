// chns_persist.cu -- an ensemble's ETD2RK step as ONE persistent kernel.
//
// The members of an ensemble are independent runs (own sizes, parameters and
// state).  A step of all of them is ten phases (P1..P5 of stage 1, then of
// stage 2); phase k of a member needs phase k-1 of that member complete.  One
// launch per step keeps as many CTAs as fit on every SM (64-thread CTAs, the
// size the single-run kernels of these grids use).  The CTAs take items from a
// queue -- one item is what one CTA of the single-run kernel of a phase does
// for one member -- in phase order, the largest members first; an item of phase
// k waits only for phase k-1 of its own member (a count of that phase's
// finished items), so members overlap their phases as the graph of per-member
// branches lets them.  The stage code is the single-run kernels' own text
// (chns_kernels.cuh compiled as device functions), so every member evolves bit
// for bit as it would alone; only the row passes' tiles come by cp.async (the
// members' TMA maps stay with the members).
//
// Supported: every member ternary, FP32 (plain float state), n = 256, 512 or
// 1024, the reference's cut on a square box (jt = n/4); other ensembles keep
// the graph of per-member branches (chns_ensemble.cu).  Every wait for a
// member's phase is bounded: one that runs out sets bit 1 of the error word,
// which chns_ensemble_synchronize returns as CHNS_ERR_TIMEOUT (the step's
// results are then garbage).
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "chns_internal.h"

// the virtual CTA index the stage bodies read (CHNS_BX, CHNS_BY)
__shared__ int chns_vblock[2];
#define CHNS_STAGE_BODIES 1
#include "chns_kernels.cuh"
#include "chns_stage_args.cuh"

namespace chns {

constexpr int kEnsThreads = 64;               // threads per CTA: one 1024-point transform group
constexpr int kEnsMinCtas = 4;                // CTAs per SM the kernel is built for (registers up to 255)
constexpr int kEnsPhases = 10;                // P1..P5 of stage 1, then of stage 2
constexpr unsigned kBarrierSpins = 1u << 24;  // polls (over a second) before a wait for a phase gives up

template <int N> constexpr int ens_gpc() { return kEnsThreads / (N / 16); }  // transform groups per CTA
// ints of the step's counters: the queue position, done[nm][kEnsPhases], the error word
inline size_t ens_counters(int nm) { return 2 + (size_t)nm * kEnsPhases; }

struct EnsMember {
  Par<float> P;
  Bufs<float> B;
  int n;
};

// items (CTAs of the single-run kernel) of pass k (0..4) of a member of size n
inline int ens_items(int n, int k) {
  const int gpc = kEnsThreads / (n / 16), jt = n / 4;
  auto rows = [&](int r) { return (r + gpc - 1) / gpc; };
  switch (k) {
    case 0: return 2 * rows(jt + 1);  // P1: two CTAs per row block (n <= 1024)
    case 1: return rows(n / 2);       // P2: x-row pairs
    case 2: return rows(n / 2 + 1);   // P3: spectral rows
    case 3: return rows(n / 2);       // P4
    default: return rows(n / 2 + 1);  // P5
  }
}

template <int N> size_t ens_smem() {
  constexpr int GPC = ens_gpc<N>();
  const size_t tw = tw_smem_bytes<N, float>(kEnsThreads);
  const size_t fft = tw + (size_t)GPC * FftShape<N>::SMEM * sizeof(cxf);
  const size_t adv = tw + loaded_row_smem_bytes<N, float, GPC>(false, N / 4, 0, 0, row_adv_frags<MODEL_TERNARY>());
  const size_t frc = tw + loaded_row_smem_bytes<N, float, GPC>(false, N / 4, 0, 0, row_force_frags<MODEL_TERNARY>());
  return std::max(fft, std::max(adv, frc));
}

template <int N>
__device__ __forceinline__ void ens_phase(const EnsMember& M, int ph, int vb, const TmaG& T0) {
  constexpr int GPC = ens_gpc<N>();
  const int k = ph % 5;
  if (threadIdx.x == 0) {
    const int gx = (N / 4 + 1 + GPC - 1) / GPC;  // P1's row blocks
    chns_vblock[0] = k == 0 ? vb % gx : vb;
    chns_vblock[1] = k == 0 ? vb / gx : 0;
  }
  __syncthreads();  // the index is set; the previous item's shared memory is no longer read
  switch (k) {
    case 0: k_spec_inv<N, float, GPC, MODEL_TERNARY>(M.B, M.P); break;
    case 1: k_row_adv<N, float, GPC, MODEL_TERNARY, true>(M.B, M.P, T0); break;
    case 2:
      if (ph < 5) k_spec_fwd_c<N, float, GPC, MODEL_TERNARY, 1, false>(M.B, M.P);
      else k_spec_fwd_c<N, float, GPC, MODEL_TERNARY, 2, false>(M.B, M.P);
      break;
    case 3: k_row_force<N, float, GPC, MODEL_TERNARY, true>(M.B, M.P, T0); break;
    default:
      if (ph < 5) k_spec_curl_w<N, float, GPC, true, 1, false>(M.B, M.P);
      else k_spec_curl_w<N, float, GPC, true, 2, false>(M.B, M.P);
      break;
  }
  __syncthreads();  // every thread is done with chns_vblock before it changes
}

// Waits until `*ctr` reaches `target` (acquire: the counted items' writes are
// then visible).  Bounded: a wait that runs out flags bit 1 of *err.
__device__ __forceinline__ void ens_wait_count(const int* ctr, int target, unsigned int* err) {
  unsigned spins = 0;
  while (true) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(ctr) : "memory");
    if (v >= target) break;
    if (++spins > kBarrierSpins) {
      atomicOr(err, 2u);
      break;
    }
    __nanosleep(32);
  }
}

// Work queue of one step: item q (0 .. off[kEnsPhases * nm] - 1) is item
// q - off[ph nm + r] of phase ph of member r, off being ascending over (ph, r)
// with the phases outermost and the largest members first.  A CTA takes the next
// item from *next; before phase ph > 0 of member r it waits for done[r, ph-1]
// to count all of that phase's items.  Every item an item waits for was taken
// earlier by a running CTA, so the queue always progresses.  ctr: *next, then
// done[nm][kEnsPhases], zero at launch.
__global__ void __launch_bounds__(kEnsThreads, kEnsMinCtas)
    k_ensemble_step(const EnsMember* __restrict__ mem, const int* __restrict__ off, int nm, int* ctr,
                    unsigned int* err, const TmaG* __restrict__ t0) {
  __shared__ int item_s;
  const TmaG& T0 = *t0;
  const int total = off[kEnsPhases * nm];
  int* next = ctr;
  int* done = ctr + 1;
  while (true) {
    if (threadIdx.x == 0) item_s = atomicAdd(next, 1);
    __syncthreads();
    const int item = item_s;
    if (item >= total) break;
    int lo = 0, hi = kEnsPhases * nm - 1;  // the (phase, member) slot that holds `item`
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (off[mid] <= item) lo = mid;
      else hi = mid - 1;
    }
    const int ph = lo / nm, r = lo % nm;
    if (threadIdx.x == 0 && ph > 0) {
      const int prev = (ph - 1) * nm + r;
      ens_wait_count(done + r * kEnsPhases + ph - 1, off[prev + 1] - off[prev], err);
    }
    const EnsMember& M = mem[r];
    switch (M.n) {  // ens_phase's leading barrier also publishes the wait above
      case 256: ens_phase<256>(M, ph, item - off[lo], T0); break;
      case 512: ens_phase<512>(M, ph, item - off[lo], T0); break;
      default: ens_phase<1024>(M, ph, item - off[lo], T0); break;
    }
    // ens_phase ends on a barrier: the item's writes are done; count it
    if (threadIdx.x == 0) {
      asm volatile("fence.acq_rel.gpu;\n" ::: "memory");
      atomicAdd(done + r * kEnsPhases + ph, 1);
    }
  }
}

}  // namespace chns

struct chns_persist {
  chns::EnsMember* mem = nullptr;  // device
  int* off = nullptr;              // device
  int* ctr = nullptr;              // device: the queue position, done[nm][kEnsPhases], then the error word
  int nm = 0, grid = 0;
  size_t smem = 0;
  chns::TmaG* t0 = nullptr;        // device: no tensor maps (use = 0: cp.async tiles)
};

void chns_persist_destroy(chns_persist* p) {
  if (!p) return;
  if (p->mem) cudaFree(p->mem);
  if (p->off) cudaFree(p->off);
  if (p->ctr) cudaFree(p->ctr);
  if (p->t0) cudaFree(p->t0);
  delete p;
}

int chns_persist_create(chns_ctx* const* members, int count, chns_persist** out) {
  using namespace chns;
  *out = nullptr;
  if (count < 1) return CHNS_ERR_ARG;
  for (int i = 0; i < count; i++) {
    const chns_ctx* c = members[i];
    if (c->p.model != CHNS_MODEL_TERNARY || !c->f32 || c->st64 || c->jt != c->n / 4 ||
        (c->n != 256 && c->n != 512 && c->n != 1024))
      return CHNS_ERR_UNSUPPORTED;
  }
  chns_persist* p = new (std::nothrow) chns_persist();
  if (!p) return CHNS_ERR_NOMEM;
  std::vector<int> order(count);
  for (int i = 0; i < count; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return members[a]->n > members[b]->n; });
  std::vector<EnsMember> mem(count);
  std::vector<int> off((size_t)kEnsPhases * count + 1, 0);
  size_t smem = 0;
  for (int r = 0; r < count; r++) {
    const chns_ctx* c = members[order[r]];
    mem[r].P = make_par<float>(c);
    mem[r].B = make_bufs<float>(c);
    mem[r].n = c->n;
    smem = std::max(smem, c->n == 256 ? ens_smem<256>() : c->n == 512 ? ens_smem<512>() : ens_smem<1024>());
  }
  for (int ph = 0; ph < kEnsPhases; ph++)
    for (int r = 0; r < count; r++) {
      const size_t q = (size_t)ph * count + r;
      off[q + 1] = off[q] + ens_items(mem[r].n, ph % 5);
    }
  p->nm = count;
  p->smem = smem;
  int rc = CHNS_OK;
  if (cudaMalloc((void**)&p->mem, sizeof(EnsMember) * count) != cudaSuccess ||
      cudaMalloc((void**)&p->off, sizeof(int) * off.size()) != cudaSuccess ||
      cudaMalloc((void**)&p->ctr, sizeof(int) * ens_counters(count)) != cudaSuccess ||
      cudaMalloc((void**)&p->t0, sizeof(TmaG)) != cudaSuccess)
    rc = CHNS_ERR_NOMEM;
  TmaG none{};
  none.use = 0;
  if (rc == CHNS_OK &&
      (cudaMemcpy(p->mem, mem.data(), sizeof(EnsMember) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(p->off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemset(p->ctr, 0, sizeof(int) * ens_counters(count)) != cudaSuccess ||
       cudaMemcpy(p->t0, &none, sizeof(TmaG), cudaMemcpyHostToDevice) != cudaSuccess))
    rc = CHNS_ERR_CUDA;
  if (rc == CHNS_OK &&
      cudaFuncSetAttribute(k_ensemble_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    rc = CHNS_ERR_CUDA;
  int per_sm = 0, dev = 0, sms = 0;
  if (rc == CHNS_OK &&
      (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ensemble_step, kEnsThreads, smem) != cudaSuccess ||
       cudaGetDevice(&dev) != cudaSuccess ||
       cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess))
    rc = CHNS_ERR_CUDA;
  if (rc == CHNS_OK && per_sm < 1) rc = CHNS_ERR_UNSUPPORTED;
  if (rc != CHNS_OK) {
    cudaGetLastError();
    chns_persist_destroy(p);
    return rc;
  }
  p->grid = per_sm * sms;
  *out = p;
  return CHNS_OK;
}

// one step of every member: the queue counters cleared, then one launch
int chns_persist_step(chns_persist* p, cudaStream_t st) {
  using namespace chns;
  if (cudaMemsetAsync(p->ctr, 0, sizeof(int) * (ens_counters(p->nm) - 1), st) != cudaSuccess) return CHNS_ERR_CUDA;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(p->grid);
  cfg.blockDim = dim3(kEnsThreads);
  cfg.dynamicSmemBytes = p->smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, k_ensemble_step, (const EnsMember*)p->mem, (const int*)p->off, p->nm, p->ctr,
                         (unsigned int*)(p->ctr + ens_counters(p->nm) - 1), (const TmaG*)p->t0) != cudaSuccess)
    return CHNS_ERR_CUDA;
  return CHNS_OK;
}

// the error word: CHNS_ERR_TIMEOUT if a wait for a member's phase ran out (the word is then cleared)
int chns_persist_check(chns_persist* p, cudaStream_t st) {
  unsigned int h = 0;
  unsigned int* e = (unsigned int*)(p->ctr + chns::ens_counters(p->nm) - 1);
  if (cudaMemcpyAsync(&h, e, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return CHNS_ERR_CUDA;
  if (h) {
    if (cudaMemsetAsync(e, 0, sizeof(h), st) != cudaSuccess) return CHNS_ERR_CUDA;
    return CHNS_ERR_TIMEOUT;
  }
  return CHNS_OK;
}

int chns_persist_grid(const chns_persist* p) { return p ? p->grid : 0; }
