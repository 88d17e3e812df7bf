// hw_mlp.cu -- the learned depth operator's per-point network (no counterpart in the
// reference): 5 features -> 32 -> 32 (tanh) -> K = 4 logits -> softmax weights over K
// reference-depth operators.  FP32 training on the GPU with hand-written kernels:
// forward + loss, backward with per-block parameter-gradient reduction in shared
// memory, and Adam.  Inference writes the per-point weights that replace the
// interpolation weights (gamma_j) of the varying-depth operator HSS.
//
// Per-point training record (kRec floats): 5 features, then K*kBand band matrix
// G[m][j] = C^2(kappa_m, D_j) of the K learned references at the point's band
// wavenumbers kappa_m, then kBand targets T[m] = effective C^2(kappa_m) of the
// 16-reference operator at the point.  Loss per point: mean_m ((sum_j w_j G_mj - T_m)/T_m)^2.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace {

constexpr int kIn = 5, kH = 32, kK = 4, kBand = 8;
constexpr int kRec = kIn + kK * kBand + kBand;   // 45
// parameter layout: W1[kH][kIn], b1[kH], W2[kH][kH], b2[kH], W3[kK][kH], b3[kK]
constexpr int oW1 = 0, ob1 = oW1 + kH * kIn, oW2 = ob1 + kH, ob2 = oW2 + kH * kH, oW3 = ob2 + kH,
              ob3 = oW3 + kK * kH, kParams = ob3 + kK;
constexpr int kBlock = 64;

struct Act {
  float h1[kH], h2[kH], w[kK];
};

__device__ __forceinline__ void forward(const float* __restrict__ P, const float* x, Act& a) {
  for (int i = 0; i < kH; ++i) {
    float s = P[ob1 + i];
    for (int j = 0; j < kIn; ++j) s += P[oW1 + i * kIn + j] * x[j];
    a.h1[i] = tanhf(s);
  }
  for (int i = 0; i < kH; ++i) {
    float s = P[ob2 + i];
    for (int j = 0; j < kH; ++j) s += P[oW2 + i * kH + j] * a.h1[j];
    a.h2[i] = tanhf(s);
  }
  float z[kK], zmax = -1e30f;
  for (int i = 0; i < kK; ++i) {
    float s = P[ob3 + i];
    for (int j = 0; j < kH; ++j) s += P[oW3 + i * kH + j] * a.h2[j];
    z[i] = s;
    zmax = fmaxf(zmax, s);
  }
  float den = 0.f;
  for (int i = 0; i < kK; ++i) {
    z[i] = expf(z[i] - zmax);
    den += z[i];
  }
  for (int i = 0; i < kK; ++i) a.w[i] = z[i] / den;
}

// loss of one record and dL/dz (softmax logits)
__device__ __forceinline__ float loss_and_dz(const float* rec, const float* w, float* dz) {
  const float* G = rec + kIn;
  const float* T = rec + kIn + kK * kBand;
  float dw[kK] = {0.f, 0.f, 0.f, 0.f};
  float L = 0.f;
  for (int m = 0; m < kBand; ++m) {
    float p = 0.f;
    for (int j = 0; j < kK; ++j) p += w[j] * G[m * kK + j];
    const float e = (p - T[m]) / T[m];
    L += e * e;
    const float dp = 2.f * e / (T[m] * kBand);
    for (int j = 0; j < kK; ++j) dw[j] += dp * G[m * kK + j];
  }
  float s = 0.f;
  for (int j = 0; j < kK; ++j) s += w[j] * dw[j];
  for (int j = 0; j < kK; ++j) dz[j] = w[j] * (dw[j] - s);
  return L / kBand;
}

// One pass over n records: loss sum into *loss, parameter gradients (sum over records)
// accumulated into grad (which the caller zeroes).
__global__ void __launch_bounds__(kBlock) k_mlp_grad(const float* __restrict__ P, const float* __restrict__ data,
                                                     int n, float* __restrict__ grad, float* __restrict__ loss) {
  __shared__ float sP[kParams];
  __shared__ float sx[kBlock][kIn], sh1[kBlock][kH], sd1[kBlock][kH], sh2[kBlock][kH], sd2[kBlock][kH],
      sdz[kBlock][kK];
  __shared__ float sl[kBlock];
  for (int i = threadIdx.x; i < kParams; i += kBlock) sP[i] = P[i];
  __syncthreads();
  const int r = blockIdx.x * kBlock + threadIdx.x;
  const int t = threadIdx.x;
  if (r < n) {
    const float* rec = data + size_t(r) * kRec;
    float x[kIn];
    for (int j = 0; j < kIn; ++j) x[j] = rec[j];
    Act a;
    forward(sP, x, a);
    float dz[kK];
    sl[t] = loss_and_dz(rec, a.w, dz);
    // backward through the hidden layers
    float d2[kH], d1[kH];
    for (int i = 0; i < kH; ++i) {
      float s = 0.f;
      for (int k = 0; k < kK; ++k) s += sP[oW3 + k * kH + i] * dz[k];
      d2[i] = s * (1.f - a.h2[i] * a.h2[i]);
    }
    for (int i = 0; i < kH; ++i) {
      float s = 0.f;
      for (int k = 0; k < kH; ++k) s += sP[oW2 + k * kH + i] * d2[k];
      d1[i] = s * (1.f - a.h1[i] * a.h1[i]);
    }
    for (int j = 0; j < kIn; ++j) sx[t][j] = x[j];
    for (int i = 0; i < kH; ++i) {
      sh1[t][i] = a.h1[i];
      sh2[t][i] = a.h2[i];
      sd1[t][i] = d1[i];
      sd2[t][i] = d2[i];
    }
    for (int k = 0; k < kK; ++k) sdz[t][k] = dz[k];
  } else {
    sl[t] = 0.f;
    for (int j = 0; j < kIn; ++j) sx[t][j] = 0.f;
    for (int i = 0; i < kH; ++i) sh1[t][i] = sh2[t][i] = sd1[t][i] = sd2[t][i] = 0.f;
    for (int k = 0; k < kK; ++k) sdz[t][k] = 0.f;
  }
  __syncthreads();
  // parameter gradients: each thread owns parameters p, sums over the block's records
  for (int p = t; p < kParams; p += kBlock) {
    float s = 0.f;
    if (p < ob1) {
      const int i = (p - oW1) / kIn, j = (p - oW1) % kIn;
      for (int q = 0; q < kBlock; ++q) s += sd1[q][i] * sx[q][j];
    } else if (p < oW2) {
      const int i = p - ob1;
      for (int q = 0; q < kBlock; ++q) s += sd1[q][i];
    } else if (p < ob2) {
      const int i = (p - oW2) / kH, j = (p - oW2) % kH;
      for (int q = 0; q < kBlock; ++q) s += sd2[q][i] * sh1[q][j];
    } else if (p < oW3) {
      const int i = p - ob2;
      for (int q = 0; q < kBlock; ++q) s += sd2[q][i];
    } else if (p < ob3) {
      const int i = (p - oW3) / kH, j = (p - oW3) % kH;
      for (int q = 0; q < kBlock; ++q) s += sdz[q][i] * sh2[q][j];
    } else {
      const int i = p - ob3;
      for (int q = 0; q < kBlock; ++q) s += sdz[q][i];
    }
    atomicAdd(grad + p, s);
  }
  if (t == 0) {
    float s = 0.f;
    for (int q = 0; q < kBlock; ++q) s += sl[q];
    atomicAdd(loss, s);
  }
}

// Adam on the mean gradient (grad / n)
__global__ void k_adam(float* __restrict__ P, const float* __restrict__ grad, float* __restrict__ m1,
                       float* __restrict__ m2, float inv_n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  const float g = grad[p] * inv_n;
  m1[p] = b1 * m1[p] + (1.f - b1) * g;
  m2[p] = b2 * m2[p] + (1.f - b2) * g * g;
  const float mh = m1[p] / c1, vh = m2[p] / c2;
  P[p] -= lr * mh / (sqrtf(vh) + eps);
}

__global__ void k_mlp_infer(const float* __restrict__ P, const float* __restrict__ feat, int n,
                            double* __restrict__ w_out) {
  __shared__ float sP[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) sP[i] = P[i];
  __syncthreads();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  float x[kIn];
  for (int j = 0; j < kIn; ++j) x[j] = feat[size_t(r) * kIn + j];
  Act a;
  forward(sP, x, a);
  for (int k = 0; k < kK; ++k) w_out[size_t(k) * n + r] = double(a.w[k]);   // [K][n]
}

std::string g_mlp_err;

}  // namespace

struct hw_mlp {
  float *P = nullptr, *m1 = nullptr, *m2 = nullptr, *grad = nullptr, *loss = nullptr;
  int step = 0;
  int device = 0;
  std::string err;
};

#define MLP_CUDA(call)                                                             \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      mlp->err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
      return 1;                                                                    \
    }                                                                              \
  } while (0)

extern "C" {

int hw_mlp_sizes(int* n_in, int* n_hidden, int* n_out, int* n_band, int* n_params) {
  if (n_in) *n_in = kIn;
  if (n_hidden) *n_hidden = kH;
  if (n_out) *n_out = kK;
  if (n_band) *n_band = kBand;
  if (n_params) *n_params = kParams;
  return kRec;
}

hw_mlp* hw_mlp_create(unsigned long long seed, int device) {
  hw_mlp* mlp = new hw_mlp();
  mlp->device = device;
  if (cudaSetDevice(device) != cudaSuccess) { g_mlp_err = "cudaSetDevice failed"; delete mlp; return nullptr; }
  // Xavier-uniform initialisation from a splitmix64 stream, zero biases
  std::vector<float> p(kParams, 0.f);
  unsigned long long s = seed;
  auto uni = [&]() {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return double(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int fan_out, int fan_in) {
    const double a = std::sqrt(6.0 / (fan_in + fan_out));
    for (int i = 0; i < fan_out * fan_in; ++i) p[off + i] = float((2 * uni() - 1) * a);
  };
  fill(oW1, kH, kIn);
  fill(oW2, kH, kH);
  fill(oW3, kK, kH);
  bool ok = cudaMalloc(&mlp->P, sizeof(float) * kParams) == cudaSuccess &&
            cudaMalloc(&mlp->m1, sizeof(float) * kParams) == cudaSuccess &&
            cudaMalloc(&mlp->m2, sizeof(float) * kParams) == cudaSuccess &&
            cudaMalloc(&mlp->grad, sizeof(float) * kParams) == cudaSuccess &&
            cudaMalloc(&mlp->loss, sizeof(float)) == cudaSuccess &&
            cudaMemcpy(mlp->P, p.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemset(mlp->m1, 0, sizeof(float) * kParams) == cudaSuccess &&
            cudaMemset(mlp->m2, 0, sizeof(float) * kParams) == cudaSuccess;
  if (!ok) { g_mlp_err = "device allocation failed"; delete mlp; return nullptr; }
  return mlp;
}

void hw_mlp_destroy(hw_mlp* mlp) {
  if (!mlp) return;
  cudaFree(mlp->P); cudaFree(mlp->m1); cudaFree(mlp->m2); cudaFree(mlp->grad); cudaFree(mlp->loss);
  delete mlp;
}

const char* hw_mlp_last_error(const hw_mlp* mlp) { return mlp ? mlp->err.c_str() : g_mlp_err.c_str(); }

int hw_mlp_get_params(hw_mlp* mlp, float* out) {
  MLP_CUDA(cudaMemcpy(out, mlp->P, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  return 0;
}

int hw_mlp_set_params(hw_mlp* mlp, const float* in) {
  MLP_CUDA(cudaMemcpy(mlp->P, in, sizeof(float) * kParams, cudaMemcpyHostToDevice));
  mlp->step = 0;
  MLP_CUDA(cudaMemset(mlp->m1, 0, sizeof(float) * kParams));
  MLP_CUDA(cudaMemset(mlp->m2, 0, sizeof(float) * kParams));
  return 0;
}

// Summed loss and parameter gradients over n device-resident records.
int hw_mlp_grad_device(hw_mlp* mlp, const float* data_dev, int n, float* grad_host, float* loss_host) {
  MLP_CUDA(cudaMemset(mlp->grad, 0, sizeof(float) * kParams));
  MLP_CUDA(cudaMemset(mlp->loss, 0, sizeof(float)));
  k_mlp_grad<<<(n + kBlock - 1) / kBlock, kBlock>>>(mlp->P, data_dev, n, mlp->grad, mlp->loss);
  MLP_CUDA(cudaGetLastError());
  if (grad_host) MLP_CUDA(cudaMemcpy(grad_host, mlp->grad, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  if (loss_host) MLP_CUDA(cudaMemcpy(loss_host, mlp->loss, sizeof(float), cudaMemcpyDeviceToHost));
  return 0;
}

// Full-batch-per-chunk Adam training over host records; losses[epoch] = mean loss.
int hw_mlp_train(hw_mlp* mlp, const float* data_host, int n, int epochs, int batch, float lr, float* losses) {
  float* d = nullptr;
  MLP_CUDA(cudaMalloc(&d, sizeof(float) * size_t(n) * kRec));
  MLP_CUDA(cudaMemcpy(d, data_host, sizeof(float) * size_t(n) * kRec, cudaMemcpyHostToDevice));
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int ep = 0; ep < epochs; ++ep) {
    double tot = 0.0;
    for (int off = 0; off < n; off += batch) {
      const int cnt = (off + batch <= n) ? batch : n - off;
      if (cudaMemset(mlp->grad, 0, sizeof(float) * kParams) != cudaSuccess ||
          cudaMemset(mlp->loss, 0, sizeof(float)) != cudaSuccess) { cudaFree(d); mlp->err = "memset"; return 1; }
      k_mlp_grad<<<(cnt + kBlock - 1) / kBlock, kBlock>>>(mlp->P, d + size_t(off) * kRec, cnt, mlp->grad, mlp->loss);
      ++mlp->step;
      const float c1 = 1.f - std::pow(b1, float(mlp->step)), c2 = 1.f - std::pow(b2, float(mlp->step));
      k_adam<<<(kParams + 255) / 256, 256>>>(mlp->P, mlp->grad, mlp->m1, mlp->m2, 1.f / cnt, lr, b1, b2, eps, c1, c2);
      float l = 0.f;
      if (cudaMemcpy(&l, mlp->loss, sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaFree(d); mlp->err = "training kernel failed"; return 1;
      }
      tot += l;
    }
    if (losses) losses[ep] = float(tot / n);
  }
  cudaFree(d);
  return 0;
}

// Per-point softmax weights [K][n] (double) for n feature rows (host in, host out).
int hw_mlp_infer(hw_mlp* mlp, const float* feat_host, int n, double* w_host) {
  float* f = nullptr;
  double* w = nullptr;
  MLP_CUDA(cudaMalloc(&f, sizeof(float) * size_t(n) * kIn));
  MLP_CUDA(cudaMalloc(&w, sizeof(double) * size_t(n) * kK));
  MLP_CUDA(cudaMemcpy(f, feat_host, sizeof(float) * size_t(n) * kIn, cudaMemcpyHostToDevice));
  k_mlp_infer<<<(n + 255) / 256, 256>>>(mlp->P, f, n, w);
  MLP_CUDA(cudaGetLastError());
  MLP_CUDA(cudaMemcpy(w_host, w, sizeof(double) * size_t(n) * kK, cudaMemcpyDeviceToHost));
  cudaFree(f);
  cudaFree(w);
  return 0;
}

// host-buffer convenience for the gradient check
int hw_mlp_grad(hw_mlp* mlp, const float* data_host, int n, float* grad_host, float* loss_host) {
  float* d = nullptr;
  MLP_CUDA(cudaMalloc(&d, sizeof(float) * size_t(n) * kRec));
  MLP_CUDA(cudaMemcpy(d, data_host, sizeof(float) * size_t(n) * kRec, cudaMemcpyHostToDevice));
  const int r = hw_mlp_grad_device(mlp, d, n, grad_host, loss_host);
  cudaFree(d);
  return r;
}

}  // extern "C"
