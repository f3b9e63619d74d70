// Learned dispatch.
//
// A 6 -> 32 -> 32 -> 4 fp32 MLP (mlp.cuh) predicts, from segment features,
// the log of the device cycles each kernel variant spends on the segment.  It
// is trained online on the per-segment cycles the iteration kernel records,
// with hand-written forward/backward and Adam kernels, and assigns every
// segment the cheapest variant it is capable of.  All variants give
// identical labels, so the choice changes speed only.
//
// Schedule of a handle in LPA_DISPATCH_LEARNED:
//   1. one iteration on the fixed degree-bucket plan: its device time is the
//      yardstick every learned plan must beat;
//   2. kExplore iterations on round-robin plans (segment s runs its
//      ((s + k) mod capable)-th capable variant) -- every step trains the MLP;
//   3. the MLP's plan runs, then (when it differs) the same plan with every
//      capable segment moved to the two-pass kernels -- per-segment costs do
//      not see a kernel's critical path or launch; the faster of the two is
//      the learned plan.  If it is slower than the fixed plan, the handle
//      reverts to the fixed plan (a revert is counted);
//   4. the chosen plan stays frozen; every kRecheck iterations one iteration
//      runs the other plan and the faster of the two is kept.
// Times compared in 3 and 4 are the iteration's kernel busy time on the GPU
// clock (IterArgs::ktime), not host-visible wall time.
// Features: degree, compressed bits, interval fraction, residual count (per
// vertex of the segment), iteration index and the segment's change rate in
// the previous iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mlp.cuh"
#include "runtime.h"

using namespace lpa_mlp;

namespace {

constexpr int kExplore = 4;
constexpr int kRecheck = 64;
constexpr int kTrainSteps = 64;   // Adam steps after each measured iteration
constexpr uint32_t kBatch = 4096;  // minibatch (sampled segments)
constexpr float kLr = 3e-3f;

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

__global__ void k_mlp_features(const float4 *feat, const lpa_dev::Seg *segs, const uint32_t *seg_changed, float it_feat,
                               float *X, uint32_t n) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const float4 f = feat[s];
    const float nv = float(max(1u, segs[s].end - segs[s].begin));
    float *x = X + size_t(s) * kIn;
    x[0] = f.x;
    x[1] = f.y;
    x[2] = f.z;
    x[3] = f.w;
    x[4] = it_feat;
    x[5] = seg_changed ? float(seg_changed[s]) / nv : 0.f;
  }
}

__global__ void k_mlp_targets(const long long *cycles, float *tgt, uint32_t n) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
    tgt[s] = log2f(1.f + float(cycles[s])) / 32.f;
}

// Gradient of sum_k 0.5 (y[var_k] - target_k)^2 over samples k (idx maps a
// sample to its row; when step != 0 rows are sampled by hash), accumulated
// into grad; loss receives the summed loss.
__global__ void k_mlp_grad(const float *__restrict__ P, const float *__restrict__ X, const uint8_t *__restrict__ var,
                           const float *__restrict__ target, uint32_t rows, uint32_t n, uint32_t step, float *grad,
                           float *loss) {
  __shared__ float sP[kParams];
  __shared__ float sG[kParams];
  __shared__ float sL;
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
    sP[i] = P[i];
    sG[i] = 0.f;
  }
  if (threadIdx.x == 0) sL = 0.f;
  __syncthreads();
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const uint32_t s = step ? mix32(k * 0x9E3779B9u + step) % rows : k;
    float x[kIn], h1[kH], h2[kH], y[kOut];
    for (int i = 0; i < kIn; i++) x[i] = X[size_t(s) * kIn + i];
    forward(sP, x, h1, h2, y);
    const int v = var[s];
    const float e = y[v] - target[s];
    atomicAdd(&sL, 0.5f * e * e);
    atomicAdd(&sG[kOffB3 + v], e);
    float dh2[kH];
    for (int j = 0; j < kH; j++) {
      atomicAdd(&sG[kOffW3 + v * kH + j], e * h2[j]);
      dh2[j] = h2[j] > 0.f ? e * sP[kOffW3 + v * kH + j] : 0.f;
    }
    for (int j = 0; j < kH; j++) {
      if (dh2[j] == 0.f) continue;
      atomicAdd(&sG[kOffB2 + j], dh2[j]);
      for (int i = 0; i < kH; i++) atomicAdd(&sG[kOffW2 + j * kH + i], dh2[j] * h1[i]);
    }
    for (int i = 0; i < kH; i++) {
      if (h1[i] <= 0.f) continue;
      float d = 0.f;
      for (int j = 0; j < kH; j++) d += dh2[j] * sP[kOffW2 + j * kH + i];
      if (d == 0.f) continue;
      atomicAdd(&sG[kOffB1 + i], d);
      for (int q = 0; q < kIn; q++) atomicAdd(&sG[kOffW1 + i * kIn + q], d * x[q]);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kParams; i += blockDim.x)
    if (sG[i] != 0.f) atomicAdd(&grad[i], sG[i]);
  if (threadIdx.x == 0 && loss) atomicAdd(loss, sL);
}

__global__ void k_mlp_adam(float *P, float *G, float *M, float *V, float lr, float scale, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
    const float g = G[i] * scale;
    const float m = 0.9f * M[i] + 0.1f * g;
    const float v = 0.999f * V[i] + 0.001f * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
    G[i] = 0.f;
  }
}

__global__ void k_mlp_infer(const float *__restrict__ P, const float *__restrict__ X, const uint8_t *cap,
                            uint8_t *var_out, float *pred, uint32_t n) {
  __shared__ float sP[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) sP[i] = P[i];
  __syncthreads();
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    float x[kIn], h1[kH], h2[kH], y[kOut];
    for (int i = 0; i < kIn; i++) x[i] = X[size_t(s) * kIn + i];
    forward(sP, x, h1, h2, y);
    if (pred)
      for (int o = 0; o < kOut; o++) pred[size_t(s) * kOut + o] = y[o];
    if (var_out) {
      int best = -1;
      for (int o = 0; o < kOut; o++)
        if (((cap[s] >> o) & 1) && (best < 0 || y[o] < y[best])) best = o;
      var_out[s] = uint8_t(best < 0 ? LPA_VARIANT_BLOCK : best);
    }
  }
}

// Deterministic Xavier-uniform initialisation (splitmix64 stream).
void init_params(std::vector<float> &P) {
  P.assign(kParams, 0.f);
  uint64_t s = 0x5eed1234abcdull;
  auto uni = [&]() {
    s += 0x9e3779b97f4a7c15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    return float(double(z >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
  };
  auto fill = [&](int off, int fan_in, int fan_out) {
    const float a = std::sqrt(6.f / float(fan_in + fan_out));
    for (int i = 0; i < fan_in * fan_out; i++) P[size_t(off + i)] = a * uni();
  };
  fill(kOffW1, kIn, kH);
  fill(kOffW2, kH, kH);
  fill(kOffW3, kH, kOut);
  for (int o = 0; o < kOut; o++) P[size_t(kOffB3 + o)] = 0.5f;  // log-cost targets sit near 0.5
}

}  // namespace

enum Phase : int {
  kPhaseFixed = 0,
  kPhaseExplore = 1,
  kPhaseTrial = 2,
  kPhaseLearned = 3,
  kPhaseReverted = 4,
  kPhaseTrialMerged = 5
};

struct Learner {
  float *d_P = nullptr, *d_G = nullptr, *d_M = nullptr, *d_V = nullptr;
  float *d_X = nullptr, *d_T = nullptr, *d_pred = nullptr, *d_loss = nullptr;
  float4 *d_feat = nullptr;
  uint8_t *d_cap = nullptr, *d_var = nullptr;
  std::vector<uint8_t> cap, learned;
  std::vector<uint8_t> merged;  // the MLP's plan with every capable segment on the two-pass kernels
  std::vector<uint8_t> mlp;     // the MLP's own plan (argmin of its predictions), before any trial
  int phase = kPhaseFixed;
  int explore_k = 0;
  int since_check = 0;
  int adam_step = 0;
  double t_fixed = 0, t_learned = 0;
  double loss = 0;
  uint64_t updates = 0, reverts = 0;
  bool ok = false;
};

namespace {

template <class T>
bool dmalloc(T **p, size_t count) {
  return cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(1, count) * sizeof(T)) == cudaSuccess;
}

bool learner_setup(lpa_handle *h) {
  Learner *L = new Learner();
  h->learner = L;
  const size_t ns = h->segs.size();
  bool ok = dmalloc(&L->d_P, kParams) && dmalloc(&L->d_G, kParams) && dmalloc(&L->d_M, kParams) &&
            dmalloc(&L->d_V, kParams) && dmalloc(&L->d_X, ns * kIn) && dmalloc(&L->d_T, ns) &&
            dmalloc(&L->d_pred, ns * kOut) && dmalloc(&L->d_loss, 1) && dmalloc(&L->d_feat, ns) &&
            dmalloc(&L->d_cap, ns) && dmalloc(&L->d_var, ns);
  if (!ok) {
    cudaGetLastError();
    return false;
  }
  std::vector<float> P;
  init_params(P);
  cudaMemcpy(L->d_P, P.data(), kParams * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemset(L->d_G, 0, kParams * sizeof(float));
  cudaMemset(L->d_M, 0, kParams * sizeof(float));
  cudaMemset(L->d_V, 0, kParams * sizeof(float));
  // static features and capability masks
  std::vector<float4> feat(ns);
  L->cap.resize(ns);
  for (size_t s = 0; s < ns; s++) {
    const lpa_rt::SegInfo &si = h->segs[s];
    const float nv = float(std::max<uint32_t>(1, si.end - si.begin));
    const float deg = float(si.arcs) / nv;
    const float bits = si.region == 0 ? float(si.bits) / nv : 32.f * deg;
    const float itv = si.arcs ? float(si.intervals) / float(si.arcs) : 0.f;
    const float res = float(si.arcs - si.intervals) / nv;
    feat[s] = make_float4(std::log2(1.f + deg) / 20.f, std::log2(1.f + bits) / 24.f, itv,
                          std::log2(1.f + res) / 20.f);
    uint8_t m = 0;
    for (int v = 0; v < 4; v++)
      if (lpa_rt::variant_capable(v, si, h->opts.cms_threshold)) m |= uint8_t(1u << v);
    L->cap[s] = m;
  }
  cudaMemcpy(L->d_feat, feat.data(), ns * sizeof(float4), cudaMemcpyHostToDevice);
  cudaMemcpy(L->d_cap, L->cap.data(), ns, cudaMemcpyHostToDevice);
  L->ok = cudaGetLastError() == cudaSuccess;
  return L->ok;
}

void set_plan(lpa_handle *h, const std::vector<uint8_t> &plan) {
  if (plan != h->variant) {
    h->variant = plan;
    lpa_rt_apply_variants(h);
  }
}

void explore_plan(lpa_handle *h, int k, std::vector<uint8_t> &plan) {
  Learner *L = h->learner;
  plan.resize(h->segs.size());
  for (size_t s = 0; s < plan.size(); s++) {
    int opts[4], n = 0;
    for (int v = 0; v < 4; v++)
      if ((L->cap[s] >> v) & 1) opts[n++] = v;
    plan[s] = uint8_t(n ? opts[(s + size_t(k)) % size_t(n)] : h->fixed[s]);
  }
}

void train(lpa_handle *h) {
  Learner *L = h->learner;
  const uint32_t ns = uint32_t(h->segs.size());
  if (!ns) return;
  const int threads = 256;
  const int blocks = int(std::min<uint32_t>((ns + threads - 1) / threads, uint32_t(h->num_sms) * 4));
  const float it_feat = float(std::min<uint64_t>(h->iterations, 32)) / 32.f;
  k_mlp_features<<<blocks, threads, 0, h->stream>>>(L->d_feat, h->d_segs, h->d_seg_changed_prev, it_feat, L->d_X,
                                                      ns);
  k_mlp_targets<<<blocks, threads, 0, h->stream>>>(h->d_seg_cycles, L->d_T, ns);
  cudaMemcpyAsync(L->d_var, h->d_seg_var, ns, cudaMemcpyDeviceToDevice, h->stream);
  const uint32_t nb = std::min<uint32_t>(kBatch, ns);
  const int gb = int(std::min<uint32_t>((nb + 127) / 128, 64));
  cudaMemsetAsync(L->d_loss, 0, sizeof(float), h->stream);
  for (int st = 0; st < kTrainSteps; st++) {
    L->adam_step++;
    k_mlp_grad<<<gb, 128, 0, h->stream>>>(L->d_P, L->d_X, L->d_var, L->d_T, ns, nb, uint32_t(L->adam_step),
                                          L->d_G, st == kTrainSteps - 1 ? L->d_loss : nullptr);
    const float c1 = 1.f - std::pow(0.9f, float(L->adam_step));
    const float c2 = 1.f - std::pow(0.999f, float(L->adam_step));
    k_mlp_adam<<<(kParams + 255) / 256, 256, 0, h->stream>>>(L->d_P, L->d_G, L->d_M, L->d_V, kLr, 1.f / float(nb), c1,
                                                            c2);
    L->updates++;
  }
  float loss = 0;
  cudaMemcpyAsync(&loss, L->d_loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream);
  cudaStreamSynchronize(h->stream);
  L->loss = double(loss) / double(nb);
}

void infer(lpa_handle *h) {
  Learner *L = h->learner;
  const uint32_t ns = uint32_t(h->segs.size());
  const int threads = 128;
  const int blocks = int(std::min<uint32_t>((ns + threads - 1) / threads, uint32_t(h->num_sms) * 8));
  const float it_feat = float(std::min<uint64_t>(h->iterations, 32)) / 32.f;
  k_mlp_features<<<std::max(1, blocks), threads, 0, h->stream>>>(L->d_feat, h->d_segs, h->d_seg_changed_prev, it_feat,
                                                                  L->d_X, ns);
  k_mlp_infer<<<std::max(1, blocks), threads, 0, h->stream>>>(L->d_P, L->d_X, L->d_cap, L->d_var, L->d_pred, ns);
  L->learned.resize(ns);
  cudaMemcpyAsync(L->learned.data(), L->d_var, ns, cudaMemcpyDeviceToHost, h->stream);
  cudaStreamSynchronize(h->stream);
}

}  // namespace

void lpa_learner_free(lpa_handle *h) {
  Learner *L = h->learner;
  if (!L) return;
  for (void *p : {(void *)L->d_P, (void *)L->d_G, (void *)L->d_M, (void *)L->d_V, (void *)L->d_X, (void *)L->d_T,
                  (void *)L->d_pred, (void *)L->d_loss, (void *)L->d_feat, (void *)L->d_cap, (void *)L->d_var})
    if (p) cudaFree(p);
  delete L;
  h->learner = nullptr;
}

void lpa_learner_reset(lpa_handle *h) { lpa_learner_free(h); }

bool lpa_learner_settled(lpa_handle *h) {
  return h->opts.dispatch != LPA_DISPATCH_LEARNED ||
         (h->learner && (h->learner->phase == kPhaseLearned || h->learner->phase == kPhaseReverted));
}

void lpa_learner_before_iteration(lpa_handle *h) {
  h->collect_cycles = false;
  h->learner_spans = false;
  if (h->opts.dispatch != LPA_DISPATCH_LEARNED) return;
  if (!h->learner && !learner_setup(h)) {
    lpa_learner_free(h);
    h->opts.dispatch = LPA_DISPATCH_FIXED;  // no memory for the model: the heuristic stays
    return;
  }
  Learner *L = h->learner;
  std::vector<uint8_t> plan;
  switch (L->phase) {
    case kPhaseFixed:
      plan = h->fixed;
      break;
    case kPhaseExplore:
      explore_plan(h, L->explore_k, plan);
      break;
    case kPhaseTrialMerged:
      plan = L->merged;
      break;
    case kPhaseTrial:
    case kPhaseLearned:
      plan = (L->since_check >= kRecheck) ? h->fixed : L->learned;
      break;
    default:
      plan = (L->since_check >= kRecheck) ? L->learned : h->fixed;
  }
  set_plan(h, plan);
  // per-segment cycles only while the model trains on them (every item's
  // booking is an atomic); the iteration is timed by its kernels' busy spans
  // until the plan is chosen, then only on the iteration before a recheck
  // and on the recheck itself (the spans' atomics cost a 15 us iteration of
  // the road grid 362^2 about a quarter)
  const bool training = L->phase == kPhaseFixed || L->phase == kPhaseExplore;
  const bool settled = L->phase == kPhaseLearned || L->phase == kPhaseReverted;
  h->collect_cycles = training;
  h->learner_spans = !settled || L->since_check + 1 >= kRecheck;
  if (training)
    cudaMemsetAsync(h->d_seg_cycles, 0, std::max<size_t>(1, h->segs.size()) * sizeof(long long), h->stream);
  if (h->learner_spans) {
    cudaMemsetAsync(h->d_ktime, 0xFF, lpa_dev::kBusyKernels * sizeof(unsigned long long), h->stream);  // starts
    cudaMemsetAsync(h->d_ktime + lpa_dev::kBusyKernels, 0, lpa_dev::kBusyKernels * sizeof(unsigned long long),
                    h->stream);  // ends
  }
  std::swap(h->d_seg_changed, h->d_seg_changed_prev);
  cudaMemsetAsync(h->d_seg_changed, 0, std::max<size_t>(1, h->segs.size()) * sizeof(uint32_t), h->stream);
}

void lpa_learner_after_iteration(lpa_handle *h) {
  const bool timed = h->learner_spans;
  h->collect_cycles = false;
  h->learner_spans = false;
  Learner *L = h->learner;
  if (!L || h->opts.dispatch != LPA_DISPATCH_LEARNED) return;
  // The yardstick's clock: the time the iteration's kernels were busy on the GPU
  // (the sum of their spans on the GPU clock).  Unlike the events around the
  // iteration, it leaves out host-side gaps between launches, which a tool
  // such as a profiler can stretch by orders of magnitude.
  double t = h->last_iter_ms;
  unsigned long long span[2 * lpa_dev::kBusyKernels];
  if (!timed) {
    // a settled plan between rechecks: nothing to compare
  } else if (cudaMemcpy(span, h->d_ktime, sizeof(span), cudaMemcpyDeviceToHost) == cudaSuccess) {
    double busy = 0;
    for (int k = 0; k < lpa_dev::kBusyKernels; k++)
      if (span[lpa_dev::kBusyKernels + k] > span[k]) busy += double(span[lpa_dev::kBusyKernels + k] - span[k]) * 1e-6;
    if (busy > 0) t = busy;
  } else {
    cudaGetLastError();
  }
  const bool fixed_now = h->variant == h->fixed;
  switch (L->phase) {
    case kPhaseFixed:
      L->t_fixed = t;
      train(h);
      L->phase = kPhaseExplore;
      L->explore_k = 0;
      break;
    case kPhaseExplore:
      train(h);
      if (++L->explore_k >= kExplore) {
        infer(h);
        L->mlp = L->learned;
        // Per-segment costs do not see a kernel's critical path or its launch:
        // the plan with the MLP's leftovers moved onto the two-pass kernels
        // is a second candidate, and the measured iteration time decides.
        L->merged = L->learned;
        for (size_t s = 0; s < L->merged.size(); s++)
          if (variant_capable(LPA_VARIANT_TWO_PASS, h->segs[s], h->opts.cms_threshold))
            L->merged[s] = LPA_VARIANT_TWO_PASS;
        L->phase = kPhaseTrial;
        L->since_check = 0;
      }
      break;
    case kPhaseTrial:
      L->t_learned = t;
      if (L->merged != L->learned) {
        L->phase = kPhaseTrialMerged;
        break;
      }
      [[fallthrough]];
    case kPhaseTrialMerged:
      if (L->phase == kPhaseTrialMerged && t < L->t_learned) {
        L->learned = L->merged;
        L->t_learned = t;
      }
      if (L->t_learned > L->t_fixed) {
        L->phase = kPhaseReverted;
        L->reverts++;
      } else {
        L->phase = kPhaseLearned;
      }
      L->since_check = 0;
      break;
    case kPhaseLearned:
    case kPhaseReverted:
      if (L->since_check >= kRecheck) {
        // this iteration ran the other plan: compare and choose
        if (fixed_now) L->t_fixed = t;
        else L->t_learned = t;
        const bool learned_wins = L->t_learned <= L->t_fixed;
        if (L->phase == kPhaseLearned && !learned_wins) L->reverts++;
        L->phase = learned_wins ? kPhaseLearned : kPhaseReverted;
        L->since_check = 0;
      } else {
        if (timed) {
          if (fixed_now) L->t_fixed = t;
          else L->t_learned = t;
        }
        L->since_check++;
      }
      break;
  }
}

void lpa_learner_stats(lpa_handle *h, lpa_stats *st) {
  Learner *L = h->learner;
  if (!L) return;
  st->mlp_loss = L->loss;
  st->mlp_updates = L->updates;
  st->dispatch_reverts = L->reverts;
  st->learned_active = (L->phase == kPhaseLearned) ? 1 : 0;
}

// --------------------------------------------------------------- C ABI ---
extern "C" {

lpa_status lpa_mlp_gradient(int device, const float *params, const float *x, const uint8_t *variant,
                            const float *target, size_t n, float *grad_out, float *loss_out) {
  if (!params || !x || !variant || !target || !grad_out || n == 0) return LPA_ERR_INVALID_ARG;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return LPA_ERR_NO_DEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) return LPA_ERR_INVALID_ARG;
  float *dP, *dX, *dT, *dG, *dL;
  uint8_t *dV;
  if (!dmalloc(&dP, kParams) || !dmalloc(&dX, n * kIn) || !dmalloc(&dT, n) || !dmalloc(&dG, kParams) ||
      !dmalloc(&dL, 1) || !dmalloc(&dV, n)) {
    cudaGetLastError();
    return LPA_ERR_OOM;
  }
  cudaMemcpy(dP, params, kParams * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dX, x, n * kIn * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dT, target, n * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dV, variant, n, cudaMemcpyHostToDevice);
  cudaMemset(dG, 0, kParams * 4);
  cudaMemset(dL, 0, 4);
  k_mlp_grad<<<int(std::min<size_t>((n + 127) / 128, 64)), 128>>>(dP, dX, dV, dT, uint32_t(n), uint32_t(n), 0u, dG,
                                                                   dL);
  cudaMemcpy(grad_out, dG, kParams * 4, cudaMemcpyDeviceToHost);
  if (loss_out) cudaMemcpy(loss_out, dL, 4, cudaMemcpyDeviceToHost);
  const cudaError_t e = cudaGetLastError();
  for (void *p : {(void *)dP, (void *)dX, (void *)dT, (void *)dG, (void *)dL, (void *)dV}) cudaFree(p);
  return e == cudaSuccess ? LPA_OK : LPA_ERR_CUDA;
}

lpa_status lpa_mlp_predict(int device, const float *params, const float *x, size_t n, float *out) {
  if (!params || !x || !out || n == 0) return LPA_ERR_INVALID_ARG;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return LPA_ERR_NO_DEVICE;
  }
  if (cudaSetDevice(device) != cudaSuccess) return LPA_ERR_INVALID_ARG;
  float *dP, *dX, *dY;
  if (!dmalloc(&dP, kParams) || !dmalloc(&dX, n * kIn) || !dmalloc(&dY, n * kOut)) {
    cudaGetLastError();
    return LPA_ERR_OOM;
  }
  cudaMemcpy(dP, params, kParams * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dX, x, n * kIn * 4, cudaMemcpyHostToDevice);
  k_mlp_infer<<<int(std::min<size_t>((n + 127) / 128, 256)), 128>>>(dP, dX, nullptr, nullptr, dY, uint32_t(n));
  cudaMemcpy(out, dY, n * kOut * 4, cudaMemcpyDeviceToHost);
  const cudaError_t e = cudaGetLastError();
  for (void *p : {(void *)dP, (void *)dX, (void *)dY}) cudaFree(p);
  return e == cudaSuccess ? LPA_OK : LPA_ERR_CUDA;
}

lpa_status lpa_get_mlp(lpa_handle *h, float *params, size_t n) {
  if (!h || !params || n != size_t(kParams)) return LPA_ERR_INVALID_ARG;
  if (!h->learner) {
    std::vector<float> P;
    init_params(P);
    std::memcpy(params, P.data(), kParams * sizeof(float));
    return LPA_OK;
  }
  return cudaMemcpy(params, h->learner->d_P, kParams * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? LPA_OK
                                                                                               : LPA_ERR_CUDA;
}

lpa_status lpa_get_learned_plan(lpa_handle *h, uint8_t *plan, float *pred, size_t count) {
  if (!h || count != h->segs.size()) return LPA_ERR_INVALID_ARG;
  if (!h->learner) return LPA_ERR_INVALID_ARG;
  if (plan) std::memcpy(plan, h->learner->learned.data(), std::min(count, h->learner->learned.size()));
  if (pred && cudaMemcpy(pred, h->learner->d_pred, count * kOut * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return LPA_ERR_CUDA;
  return LPA_OK;
}

lpa_status lpa_get_mlp_plan(lpa_handle *h, uint8_t *plan, size_t count) {
  if (!h || !plan || count != h->segs.size() || !h->learner || h->learner->mlp.size() != count)
    return LPA_ERR_INVALID_ARG;
  std::memcpy(plan, h->learner->mlp.data(), count);
  return LPA_OK;
}

lpa_status lpa_get_segment_cycles(lpa_handle *h, uint64_t *cycles, size_t count) {
  if (!h || !cycles || count != h->segs.size()) return LPA_ERR_INVALID_ARG;
  return cudaMemcpy(cycles, h->d_seg_cycles, count * 8, cudaMemcpyDeviceToHost) == cudaSuccess ? LPA_OK
                                                                                               : LPA_ERR_CUDA;
}

}  // extern "C"
