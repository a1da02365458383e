// Strategy network: a 3-layer fp32 MLP (16 -> 64 -> 64 -> 8, ReLU) whose
// three softmax heads pick the pivot rule (2 classes), the trim depth (2) and
// the reachability strategy / switch point (4) for a graph from 16 graph
// statistics.  Forward, backward (cross-entropy summed over heads, mean over
// samples) and Adam run in the kernels below; the parameters live on the
// device.  The labels of a decomposition never depend on what it picks.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "scc_capi.h"
#include "scc_gen.h"
#include "scc_internal.h"

namespace {

constexpr int kIn = 16, kH = 64, kOut = 8;
constexpr int kHeads = 3;
__constant__ int c_head_lo[kHeads] = {0, 2, 4};
__constant__ int c_head_n[kHeads] = {2, 2, 4};
constexpr int kW1 = 0, kB1 = kW1 + kIn * kH, kW2 = kB1 + kH, kB2 = kW2 + kH * kH, kW3 = kB2 + kH,
              kB3 = kW3 + kH * kOut, kParams = kB3 + kOut;

// One CTA of 64 threads per sample: thread j owns hidden unit j.
// Writes post-ReLU activations h1, h2 and the logits.
// norm: mean[16] then scale[16]; the normalised input goes to xn (for the
// weight gradient of the first layer).
__global__ void mlp_forward_kernel(const float *__restrict__ p, const float *__restrict__ norm,
                                   const float *__restrict__ x, uint32_t B, float *__restrict__ xn,
                                   float *__restrict__ h1, float *__restrict__ h2, float *__restrict__ logits) {
  __shared__ float sx[kIn], s1[kH], s2[kH];
  const int j = threadIdx.x;
  for (uint32_t s = blockIdx.x; s < B; s += gridDim.x) {
    if (j < kIn) {
      const float v = (x[(size_t)s * kIn + j] - norm[j]) * norm[kIn + j];
      sx[j] = v;
      xn[(size_t)s * kIn + j] = v;
    }
    __syncthreads();
    float a = p[kB1 + j];
    for (int i = 0; i < kIn; ++i) a += sx[i] * p[kW1 + i * kH + j];
    a = a > 0.f ? a : 0.f;
    s1[j] = a;
    h1[(size_t)s * kH + j] = a;
    __syncthreads();
    float b = p[kB2 + j];
    for (int i = 0; i < kH; ++i) b += s1[i] * p[kW2 + i * kH + j];
    b = b > 0.f ? b : 0.f;
    s2[j] = b;
    h2[(size_t)s * kH + j] = b;
    __syncthreads();
    if (j < kOut) {
      float o = p[kB3 + j];
      for (int i = 0; i < kH; ++i) o += s2[i] * p[kW3 + i * kOut + j];
      logits[(size_t)s * kOut + j] = o;
    }
    __syncthreads();
  }
}

// Per-sample backward to the activations: dlogit = (softmax - onehot) / B per
// head, dh2 = W3 dlogit * [h2 > 0], dh1 = W2 dh2 * [h1 > 0]; loss per sample.
__global__ void mlp_backward_act_kernel(const float *__restrict__ p, const int32_t *__restrict__ y, uint32_t B,
                                        const float *__restrict__ h1, const float *__restrict__ h2,
                                        const float *__restrict__ logits, float *__restrict__ dlog,
                                        float *__restrict__ d2, float *__restrict__ d1, float *__restrict__ loss) {
  __shared__ float sd[kOut], sd2[kH];
  const int j = threadIdx.x;
  const float invB = 1.f / (float)B;
  for (uint32_t s = blockIdx.x; s < B; s += gridDim.x) {
    if (j < kHeads) {
      const int lo = c_head_lo[j], nn = c_head_n[j];
      const float *l = logits + (size_t)s * kOut + lo;
      float mx = l[0];
      for (int k = 1; k < nn; ++k) mx = fmaxf(mx, l[k]);
      float z = 0.f;
      for (int k = 0; k < nn; ++k) z += expf(l[k] - mx);
      const int t = y[(size_t)s * kHeads + j];
      float ls = 0.f;
      for (int k = 0; k < nn; ++k) {
        const float pr = expf(l[k] - mx) / z;
        const float g = (pr - (k == t ? 1.f : 0.f)) * invB;
        sd[lo + k] = g;
        dlog[(size_t)s * kOut + lo + k] = g;
        if (k == t) ls = -(l[k] - mx - logf(z));
      }
      atomicAdd(loss, ls * invB);
    }
    __syncthreads();
    float a = 0.f;
    for (int k = 0; k < kOut; ++k) a += p[kW3 + j * kOut + k] * sd[k];
    a = h2[(size_t)s * kH + j] > 0.f ? a : 0.f;
    sd2[j] = a;
    d2[(size_t)s * kH + j] = a;
    __syncthreads();
    float b = 0.f;
    for (int k = 0; k < kH; ++k) b += p[kW2 + j * kH + k] * sd2[k];
    d1[(size_t)s * kH + j] = h1[(size_t)s * kH + j] > 0.f ? b : 0.f;
    __syncthreads();
  }
}

// Parameter gradients: one thread per parameter, summed over the samples.
__global__ void mlp_backward_param_kernel(const float *__restrict__ x, uint32_t B, const float *__restrict__ h1,
                                          const float *__restrict__ h2, const float *__restrict__ dlog,
                                          const float *__restrict__ d2, const float *__restrict__ d1,
                                          float *__restrict__ grad) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < kParams; q += gridDim.x * blockDim.x) {
    float g = 0.f;
    if (q < kB1) {
      const int i = q / kH, j = q % kH;
      for (uint32_t s = 0; s < B; ++s) g += x[(size_t)s * kIn + i] * d1[(size_t)s * kH + j];
    } else if (q < kW2) {
      const int j = q - kB1;
      for (uint32_t s = 0; s < B; ++s) g += d1[(size_t)s * kH + j];
    } else if (q < kB2) {
      const int i = (q - kW2) / kH, j = (q - kW2) % kH;
      for (uint32_t s = 0; s < B; ++s) g += h1[(size_t)s * kH + i] * d2[(size_t)s * kH + j];
    } else if (q < kW3) {
      const int j = q - kB2;
      for (uint32_t s = 0; s < B; ++s) g += d2[(size_t)s * kH + j];
    } else if (q < kB3) {
      const int i = (q - kW3) / kOut, k = (q - kW3) % kOut;
      for (uint32_t s = 0; s < B; ++s) g += h2[(size_t)s * kH + i] * dlog[(size_t)s * kOut + k];
    } else {
      const int k = q - kB3;
      for (uint32_t s = 0; s < B; ++s) g += dlog[(size_t)s * kOut + k];
    }
    grad[q] = g;
  }
}

__global__ void mlp_adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                                float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < kParams; q += gridDim.x * blockDim.x) {
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
  }
}

struct DevArr {
  float *p = nullptr;
  size_t n = 0;
  cudaError_t get(size_t count) {
    if (count <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, count * sizeof(float));
    if (e == cudaSuccess) n = count;
    return e;
  }
  ~DevArr() {
    if (p) cudaFree(p);
  }
};

}  // namespace

struct scc_mlp {
  int device = 0;
  cudaStream_t st = nullptr;
  DevArr params, grad, adam_m, adam_v, norm, x, xn, h1, h2, logits, dlog, d1, d2, loss;
  int32_t *y = nullptr;
  size_t ycap = 0;
  uint64_t step = 0;
};

namespace {

int mlp_fail(cudaError_t e, const char *what) {
  return sccb::set_error(e == cudaErrorMemoryAllocation ? SCC_ERR_NOMEM : SCC_ERR_CUDA, "%s: %s", what,
                         cudaGetErrorString(e));
}
#define MCK(call, what)                                  \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return mlp_fail(e_, what);    \
  } while (0)

int ensure_batch(scc_mlp *m, uint32_t B) {
  MCK(m->x.get((size_t)B * kIn), "alloc");
  MCK(m->xn.get((size_t)B * kIn), "alloc");
  MCK(m->h1.get((size_t)B * kH), "alloc");
  MCK(m->h2.get((size_t)B * kH), "alloc");
  MCK(m->d1.get((size_t)B * kH), "alloc");
  MCK(m->d2.get((size_t)B * kH), "alloc");
  MCK(m->logits.get((size_t)B * kOut), "alloc");
  MCK(m->dlog.get((size_t)B * kOut), "alloc");
  if ((size_t)B * kHeads > m->ycap) {
    if (m->y) cudaFree(m->y);
    m->y = nullptr;
    m->ycap = 0;
    MCK(cudaMalloc(&m->y, (size_t)B * kHeads * sizeof(int32_t)), "alloc");
    m->ycap = (size_t)B * kHeads;
  }
  return SCC_OK;
}

int forward(scc_mlp *m, const float *hx, uint32_t B) {
  int rc = ensure_batch(m, B);
  if (rc) return rc;
  MCK(cudaMemcpyAsync(m->x.p, hx, (size_t)B * kIn * sizeof(float), cudaMemcpyHostToDevice, m->st), "upload");
  const uint32_t grid = B < 4096 ? B : 4096;
  mlp_forward_kernel<<<grid, kH, 0, m->st>>>(m->params.p, m->norm.p, m->x.p, B, m->xn.p, m->h1.p, m->h2.p,
                                            m->logits.p);
  MCK(cudaGetLastError(), "forward launch");
  return SCC_OK;
}

// gradient of the mean loss into m->grad, loss into m->loss
int backward(scc_mlp *m, const int32_t *hy, uint32_t B) {
  MCK(cudaMemcpyAsync(m->y, hy, (size_t)B * kHeads * sizeof(int32_t), cudaMemcpyHostToDevice, m->st), "upload");
  MCK(cudaMemsetAsync(m->loss.p, 0, sizeof(float), m->st), "memset");
  const uint32_t grid = B < 4096 ? B : 4096;
  mlp_backward_act_kernel<<<grid, kH, 0, m->st>>>(m->params.p, m->y, B, m->h1.p, m->h2.p, m->logits.p, m->dlog.p,
                                                   m->d2.p, m->d1.p, m->loss.p);
  MCK(cudaGetLastError(), "backward launch");
  mlp_backward_param_kernel<<<(kParams + 255) / 256, 256, 0, m->st>>>(m->xn.p, B, m->h1.p, m->h2.p, m->dlog.p,
                                                                       m->d2.p, m->d1.p, m->grad.p);
  MCK(cudaGetLastError(), "backward launch");
  return SCC_OK;
}

bool check_labels(const int32_t *y, uint32_t B) {
  const int n[kHeads] = {2, 2, 4};
  for (uint32_t s = 0; s < B; ++s)
    for (int h = 0; h < kHeads; ++h)
      if (y[(size_t)s * kHeads + h] < 0 || y[(size_t)s * kHeads + h] >= n[h]) return false;
  return true;
}

}  // namespace

extern "C" {

int scc_mlp_create(int device, uint64_t seed, scc_mlp **out) {
  sccb::clear_error();
  if (!out) return sccb::set_error(SCC_ERR_INVALID, "null output");
  *out = nullptr;
  scc_mlp *m = new scc_mlp();
  m->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = m->params.get(kParams);
  if (e == cudaSuccess) e = m->grad.get(kParams);
  if (e == cudaSuccess) e = m->adam_m.get(kParams);
  if (e == cudaSuccess) e = m->adam_v.get(kParams);
  if (e == cudaSuccess) e = m->loss.get(1);
  if (e == cudaSuccess) e = m->norm.get(2 * kIn);
  if (e != cudaSuccess) {
    scc_mlp_destroy(m);
    return mlp_fail(e, "mlp setup");
  }
  // He-uniform initialisation from the counter-based generator, zero biases
  std::vector<float> p(kParams, 0.f);
  auto fill = [&](int off, int fan_in, int count) {
    const float lim = std::sqrt(6.f / (float)fan_in);
    for (int i = 0; i < count; ++i) {
      const uint64_t h = sccg::mix64(seed ^ sccg::mix64((uint64_t)(off + i) ^ 0x4d4c50ull));
      p[off + i] = ((float)(h >> 40) / 16777216.f * 2.f - 1.f) * lim;
    }
  };
  fill(kW1, kIn, kIn * kH);
  fill(kW2, kH, kH * kH);
  fill(kW3, kH, kH * kOut);
  cudaMemcpy(m->params.p, p.data(), kParams * sizeof(float), cudaMemcpyHostToDevice);
  float nm[2 * kIn];
  for (int i = 0; i < kIn; ++i) nm[i] = 0.f, nm[kIn + i] = 1.f;
  cudaMemcpy(m->norm.p, nm, sizeof(nm), cudaMemcpyHostToDevice);
  cudaMemset(m->adam_m.p, 0, kParams * sizeof(float));
  cudaMemset(m->adam_v.p, 0, kParams * sizeof(float));
  *out = m;
  return SCC_OK;
}

int scc_mlp_destroy(scc_mlp *m) {
  if (!m) return SCC_OK;
  cudaSetDevice(m->device);
  if (m->st) cudaStreamSynchronize(m->st);
  if (m->y) cudaFree(m->y);
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
  return SCC_OK;
}

uint32_t scc_mlp_param_count(void) { return kParams; }

int scc_mlp_params(scc_mlp *m, float *buf, int get) {
  sccb::clear_error();
  if (!m || !buf) return sccb::set_error(SCC_ERR_INVALID, "null argument");
  MCK(cudaSetDevice(m->device), "cudaSetDevice");
  if (get) {
    MCK(cudaMemcpyAsync(buf, m->params.p, kParams * sizeof(float), cudaMemcpyDeviceToHost, m->st), "download");
  } else {
    MCK(cudaMemcpyAsync(m->params.p, buf, kParams * sizeof(float), cudaMemcpyHostToDevice, m->st), "upload");
    m->step = 0;
    MCK(cudaMemsetAsync(m->adam_m.p, 0, kParams * sizeof(float), m->st), "reset");
    MCK(cudaMemsetAsync(m->adam_v.p, 0, kParams * sizeof(float), m->st), "reset");
  }
  MCK(cudaStreamSynchronize(m->st), "sync");
  return SCC_OK;
}

int scc_mlp_norm(scc_mlp *m, float *mean, float *scale, int get) {
  sccb::clear_error();
  if (!m || !mean || !scale) return sccb::set_error(SCC_ERR_INVALID, "null argument");
  MCK(cudaSetDevice(m->device), "cudaSetDevice");
  float nm[2 * kIn];
  if (get) {
    MCK(cudaMemcpyAsync(nm, m->norm.p, sizeof(nm), cudaMemcpyDeviceToHost, m->st), "download");
    MCK(cudaStreamSynchronize(m->st), "sync");
    std::memcpy(mean, nm, kIn * sizeof(float));
    std::memcpy(scale, nm + kIn, kIn * sizeof(float));
  } else {
    std::memcpy(nm, mean, kIn * sizeof(float));
    std::memcpy(nm + kIn, scale, kIn * sizeof(float));
    MCK(cudaMemcpyAsync(m->norm.p, nm, sizeof(nm), cudaMemcpyHostToDevice, m->st), "upload");
    MCK(cudaStreamSynchronize(m->st), "sync");
  }
  return SCC_OK;
}

int scc_mlp_forward(scc_mlp *m, const float *x, uint32_t B, float *logits) {
  sccb::clear_error();
  if (!m || !x || !logits || B == 0) return sccb::set_error(SCC_ERR_INVALID, "bad argument");
  MCK(cudaSetDevice(m->device), "cudaSetDevice");
  int rc = forward(m, x, B);
  if (rc) return rc;
  MCK(cudaMemcpyAsync(logits, m->logits.p, (size_t)B * kOut * sizeof(float), cudaMemcpyDeviceToHost, m->st),
      "download");
  MCK(cudaStreamSynchronize(m->st), "sync");
  return SCC_OK;
}

int scc_mlp_loss_grad(scc_mlp *m, const float *x, const int32_t *y, uint32_t B, float *loss, float *grad) {
  sccb::clear_error();
  if (!m || !x || !y || B == 0) return sccb::set_error(SCC_ERR_INVALID, "bad argument");
  if (!check_labels(y, B)) return sccb::set_error(SCC_ERR_INVALID, "class index out of range");
  MCK(cudaSetDevice(m->device), "cudaSetDevice");
  int rc = forward(m, x, B);
  if (!rc) rc = backward(m, y, B);
  if (rc) return rc;
  if (loss) MCK(cudaMemcpyAsync(loss, m->loss.p, sizeof(float), cudaMemcpyDeviceToHost, m->st), "download");
  if (grad) MCK(cudaMemcpyAsync(grad, m->grad.p, kParams * sizeof(float), cudaMemcpyDeviceToHost, m->st), "download");
  MCK(cudaStreamSynchronize(m->st), "sync");
  return SCC_OK;
}

int scc_mlp_train(scc_mlp *m, const float *x, const int32_t *y, uint32_t B, uint32_t epochs, uint32_t batch,
                  float lr, uint64_t seed, float *final_loss) {
  sccb::clear_error();
  if (!m || !x || !y || B == 0 || batch == 0) return sccb::set_error(SCC_ERR_INVALID, "bad argument");
  if (!check_labels(y, B)) return sccb::set_error(SCC_ERR_INVALID, "class index out of range");
  MCK(cudaSetDevice(m->device), "cudaSetDevice");
  std::vector<uint32_t> order(B);
  for (uint32_t i = 0; i < B; ++i) order[i] = i;
  std::vector<float> bx((size_t)batch * kIn);
  std::vector<int32_t> by((size_t)batch * kHeads);
  float last = 0.f;
  for (uint32_t ep = 0; ep < epochs; ++ep) {
    for (uint32_t i = B; i > 1; --i) {  // seeded Fisher-Yates shuffle
      const uint32_t j = (uint32_t)(sccg::mix64(seed ^ ((uint64_t)ep << 32) ^ i) % i);
      std::swap(order[i - 1], order[j]);
    }
    for (uint32_t b0 = 0; b0 < B; b0 += batch) {
      const uint32_t nb = B - b0 < batch ? B - b0 : batch;
      for (uint32_t k = 0; k < nb; ++k) {
        std::memcpy(&bx[(size_t)k * kIn], x + (size_t)order[b0 + k] * kIn, kIn * sizeof(float));
        std::memcpy(&by[(size_t)k * kHeads], y + (size_t)order[b0 + k] * kHeads, kHeads * sizeof(int32_t));
      }
      int rc = forward(m, bx.data(), nb);
      if (!rc) rc = backward(m, by.data(), nb);
      if (rc) return rc;
      ++m->step;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
      mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, m->st>>>(m->params.p, m->grad.p, m->adam_m.p, m->adam_v.p, lr,
                                                               b1, b2, 1e-8f, c1, c2);
      MCK(cudaGetLastError(), "adam launch");
    }
    MCK(cudaMemcpyAsync(&last, m->loss.p, sizeof(float), cudaMemcpyDeviceToHost, m->st), "download");
  }
  MCK(cudaStreamSynchronize(m->st), "sync");
  if (final_loss) *final_loss = last;
  return SCC_OK;
}

int scc_mlp_predict(scc_mlp *m, const float *x, uint32_t B, int32_t *choice) {
  sccb::clear_error();
  if (!m || !x || !choice || B == 0) return sccb::set_error(SCC_ERR_INVALID, "bad argument");
  std::vector<float> lg((size_t)B * kOut);
  int rc = scc_mlp_forward(m, x, B, lg.data());
  if (rc) return rc;
  const int lo[kHeads] = {0, 2, 4}, n[kHeads] = {2, 2, 4};
  for (uint32_t s = 0; s < B; ++s)
    for (int h = 0; h < kHeads; ++h) {
      int best = 0;
      for (int k = 1; k < n[h]; ++k)
        if (lg[(size_t)s * kOut + lo[h] + k] > lg[(size_t)s * kOut + lo[h] + best]) best = k;
      choice[(size_t)s * kHeads + h] = best;
    }
  return SCC_OK;
}

int scc_mlp_apply(const int32_t *choice, scc_opts *opts) {
  sccb::clear_error();
  if (!choice || !opts) return sccb::set_error(SCC_ERR_INVALID, "null argument");
  if (choice[0] < 0 || choice[0] > 1 || choice[1] < 0 || choice[1] > 1 || choice[2] < 0 || choice[2] > 3)
    return sccb::set_error(SCC_ERR_INVALID, "choice (%d, %d, %d) out of range", choice[0], choice[1], choice[2]);
  static const int32_t alg[4] = {SCC_ALG_HYBRID, SCC_ALG_HYBRID, SCC_ALG_HYBRID, SCC_ALG_COMBINE};
  static const int32_t sw[4] = {10, 100, 1000, 10};
  opts->pivot_rule = choice[0] ? SCC_PIVOT_MAX_DEGREE : SCC_PIVOT_MIN_ID;
  opts->trim_depth = choice[1] ? 1 : 0;
  opts->alg = alg[choice[2]];
  opts->switch_permille = sw[choice[2]];
  return SCC_OK;
}

}  // extern "C"
