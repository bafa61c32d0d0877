// v3dm_proposal.cu -- the learned projection of the candidate-proposal matcher.
//
// f(x) = W2 relu(W1 x + b1) + b2 maps a SIFT descriptor x = u / 512 (u the uint8 descriptor)
// to 32 dimensions; the proposal uses the unit vector z = f(x) / |f(x)|.  W1 (64 x 128) and W2
// (32 x 64) are used in BF16, every sum is accumulated in FP32; the optimiser keeps FP32 master
// copies.  Training minimises the symmetric InfoNCE loss over a batch of B matched descriptor
// pairs (a_k, p_k) with temperature T:
//   s_kl = z(a_k) . z(p_l) / T,
//   L = 1/(2B) sum_k (lse_l s_kl - s_kk) + 1/(2B) sum_l (lse_k s_kl - s_ll),
// with hand-written forward, loss, backward and Adam kernels below.  The pairs are matches that
// the exhaustive matcher produced on held-out images.
//
// Cells: C unit centroids in the 32-d space (k-means of training embeddings).  The forward
// kernel also returns, per descriptor, its 'probes' best cells by z . c (ties: lower cell).
// The proposal matcher scores a left descriptor exactly against the right descriptors whose
// best cell is among the left's probed cells.
//
// Flat parameter layout (V3DM_PROJ_PARAMS floats): W1 [64][128], b1 [64], W2 [32][64], b2 [32].
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "v3dm_internal.h"

namespace v3dm {

namespace {

constexpr int kIn = 128, kHid = 64, kOut = 32;
constexpr int kOffW1 = 0, kOffB1 = kHid * kIn, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kOut * kHid;
constexpr int kParams = kOffB2 + kOut;
static_assert(kParams == V3DM_PROJ_PARAMS, "parameter count");
constexpr int kFwdThreads = 128;
constexpr float kNormEps = 1e-12f;

// One thread per descriptor.  The weights are read from shared memory as FP32 values of the
// BF16 weights; the hidden layer is accumulated k-outer so the descriptor is unpacked once.
// Training stores the hidden activations, the normalised output and the norm; inference may
// instead (or also) assign the descriptor to its 'probes' best cells.
__global__ void __launch_bounds__(kFwdThreads)
k_proj_forward(const uint8_t* __restrict__ x, int n, const __nv_bfloat16* __restrict__ w1b, const float* __restrict__ b1,
               const __nv_bfloat16* __restrict__ w2b, const float* __restrict__ b2, float* __restrict__ hOut,
               float* __restrict__ zOut, float* __restrict__ normOut, const float* __restrict__ cells, int nCells,
               int probes, uint8_t* __restrict__ cellOut) {
  extern __shared__ float4 projSmem[];
  auto sW1 = reinterpret_cast<float4(*)[kHid / 4]>(projSmem);                 // W1[:, k] per k, 32 KB
  auto sW2 = reinterpret_cast<float4(*)[kOut / 4]>(projSmem + kIn * kHid / 4);  // W2[:, j] per j, 8 KB
  auto sC = reinterpret_cast<float4(*)[kOut / 4]>(projSmem + kIn * kHid / 4 + kHid * kOut / 4);
  float* sB1 = reinterpret_cast<float*>(projSmem + kIn * kHid / 4 + kHid * kOut / 4 + V3DM_PROJ_MAX_CELLS * kOut / 4);
  float* sB2 = sB1 + kHid;
  for (int i = threadIdx.x; i < kHid * kIn; i += kFwdThreads) {
    const int j = i / kIn, k = i % kIn;  // W1[j][k]
    reinterpret_cast<float*>(sW1)[k * kHid + j] = __bfloat162float(w1b[i]);
  }
  for (int i = threadIdx.x; i < kOut * kHid; i += kFwdThreads) {
    const int o = i / kHid, j = i % kHid;  // W2[o][j]
    reinterpret_cast<float*>(sW2)[j * kOut + o] = __bfloat162float(w2b[i]);
  }
  if (threadIdx.x < kHid) sB1[threadIdx.x] = b1[threadIdx.x];
  if (threadIdx.x < kOut) sB2[threadIdx.x] = b2[threadIdx.x];
  for (int i = threadIdx.x; i < nCells * kOut; i += kFwdThreads) reinterpret_cast<float*>(sC)[i] = cells[i];
  __syncthreads();
  for (int d = blockIdx.x * kFwdThreads + threadIdx.x; d < n; d += gridDim.x * kFwdThreads) {
    float h[kHid];
#pragma unroll
    for (int j = 0; j < kHid; ++j) h[j] = sB1[j];
    const uint4* xd = reinterpret_cast<const uint4*>(x + (size_t)d * kIn);
#pragma unroll 1
    for (int q = 0; q < kIn / 16; ++q) {
      const uint4 xw = __ldg(xd + q);
      const uint32_t words[4] = {xw.x, xw.y, xw.z, xw.w};
#pragma unroll
      for (int wi = 0; wi < 4; ++wi) {
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int k = q * 16 + wi * 4 + b;
          const float xk = (float)((words[wi] >> (8 * b)) & 255u) * (1.0f / 512.0f);
#pragma unroll
          for (int j4 = 0; j4 < kHid / 4; ++j4) {
            const float4 w = sW1[k][j4];
            h[4 * j4 + 0] = fmaf(w.x, xk, h[4 * j4 + 0]);
            h[4 * j4 + 1] = fmaf(w.y, xk, h[4 * j4 + 1]);
            h[4 * j4 + 2] = fmaf(w.z, xk, h[4 * j4 + 2]);
            h[4 * j4 + 3] = fmaf(w.w, xk, h[4 * j4 + 3]);
          }
        }
      }
    }
    float z[kOut];
#pragma unroll
    for (int o = 0; o < kOut; ++o) z[o] = sB2[o];
#pragma unroll
    for (int j = 0; j < kHid; ++j) {
      const float hj = fmaxf(h[j], 0.0f);
      if (hOut) hOut[(size_t)d * kHid + j] = hj;
#pragma unroll
      for (int o4 = 0; o4 < kOut / 4; ++o4) {
        const float4 w = sW2[j][o4];
        z[4 * o4 + 0] = fmaf(w.x, hj, z[4 * o4 + 0]);
        z[4 * o4 + 1] = fmaf(w.y, hj, z[4 * o4 + 1]);
        z[4 * o4 + 2] = fmaf(w.z, hj, z[4 * o4 + 2]);
        z[4 * o4 + 3] = fmaf(w.w, hj, z[4 * o4 + 3]);
      }
    }
    float ss = 0.0f;
#pragma unroll
    for (int o = 0; o < kOut; ++o) ss = fmaf(z[o], z[o], ss);
    const float nrm = sqrtf(ss);
    const float inv = 1.0f / fmaxf(nrm, kNormEps);
#pragma unroll
    for (int o = 0; o < kOut; ++o) z[o] *= inv;
    if (normOut) normOut[d] = nrm;
    if (zOut) {
      float4* zo = reinterpret_cast<float4*>(zOut + (size_t)d * kOut);
#pragma unroll
      for (int o4 = 0; o4 < kOut / 4; ++o4) zo[o4] = make_float4(z[4 * o4], z[4 * o4 + 1], z[4 * o4 + 2], z[4 * o4 + 3]);
    }
    if (cellOut) {
      // the 'probes' best cells by z . c, in order; ties keep the lower cell
      float bs[V3DM_PROJ_MAX_PROBES];
      int bc[V3DM_PROJ_MAX_PROBES];
#pragma unroll
      for (int i = 0; i < V3DM_PROJ_MAX_PROBES; ++i) {
        bs[i] = -INFINITY;
        bc[i] = 0;
      }
      for (int c = 0; c < nCells; ++c) {
        float s = 0.0f;
#pragma unroll
        for (int o4 = 0; o4 < kOut / 4; ++o4) {
          const float4 w = sC[c][o4];
          s = fmaf(w.x, z[4 * o4], s);
          s = fmaf(w.y, z[4 * o4 + 1], s);
          s = fmaf(w.z, z[4 * o4 + 2], s);
          s = fmaf(w.w, z[4 * o4 + 3], s);
        }
        // insertion into the sorted top list (strict '>' keeps earlier cells first on ties)
        int cc = c;
#pragma unroll
        for (int i = 0; i < V3DM_PROJ_MAX_PROBES; ++i) {
          if (i < probes && s > bs[i]) {
            const float ts = bs[i];
            const int tc = bc[i];
            bs[i] = s;
            bc[i] = cc;
            s = ts;
            cc = tc;
          }
        }
      }
      for (int i = 0; i < probes; ++i) cellOut[(size_t)d * probes + i] = (uint8_t)bc[i];
    }
  }
}

constexpr size_t kFwdSmem =
    sizeof(float) * ((size_t)kIn * kHid + (size_t)kHid * kOut + (size_t)V3DM_PROJ_MAX_CELLS * kOut + kHid + kOut);

cudaError_t launch_forward(const uint8_t* x, long long n, const __nv_bfloat16* w1b, const float* b1,
                           const __nv_bfloat16* w2b, const float* b2, float* hOut, float* zOut, float* normOut,
                           const float* cells, int nCells, int probes, uint8_t* cellOut, cudaStream_t s) {
  static bool attrSet[128] = {};  // per device ordinal
  int dev = 0;
  cudaError_t e0 = cudaGetDevice(&dev);
  if (e0 != cudaSuccess) return e0;
  if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
  if (!attrSet[dev]) {
    cudaError_t e = cudaFuncSetAttribute(k_proj_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem);
    if (e != cudaSuccess) return e;
    attrSet[dev] = true;
  }
  if (n <= 0) return cudaSuccess;
  long long blocks = (n + kFwdThreads - 1) / kFwdThreads;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_proj_forward<<<(unsigned)blocks, kFwdThreads, kFwdSmem, s>>>(x, (int)n, w1b, b1, w2b, b2, hOut, zOut, normOut,
                                                                 cells, nCells, probes, cellOut);
  return cudaGetLastError();
}

// Logits s_kl = za_k . zp_l / T of the batch.
__global__ void k_proj_logits(const float* __restrict__ za, const float* __restrict__ zp, int B, float invT,
                              float* __restrict__ S) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)B * B) return;
  const int k = (int)(i / B), l = (int)(i % B);
  const float4* a = reinterpret_cast<const float4*>(za + (size_t)k * kOut);
  const float4* p = reinterpret_cast<const float4*>(zp + (size_t)l * kOut);
  float s = 0.0f;
#pragma unroll
  for (int o4 = 0; o4 < kOut / 4; ++o4) {
    const float4 x = a[o4], y = p[o4];
    s = fmaf(x.x, y.x, s);
    s = fmaf(x.y, y.y, s);
    s = fmaf(x.z, y.z, s);
    s = fmaf(x.w, y.w, s);
  }
  S[i] = s * invT;
}

// Log-sum-exp of every row (blocks 0..B-1) and every column (blocks B..2B-1) of S.
__global__ void __launch_bounds__(256) k_proj_lse(const float* __restrict__ S, int B, float* __restrict__ lseR,
                                                  float* __restrict__ lseC) {
  __shared__ float red[256];
  const bool row = (int)blockIdx.x < B;
  const int r = row ? blockIdx.x : blockIdx.x - B;
  auto at = [&](int t) { return row ? S[(size_t)r * B + t] : S[(size_t)t * B + r]; };
  float m = -INFINITY;
  for (int t = threadIdx.x; t < B; t += 256) m = fmaxf(m, at(t));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  m = red[0];
  __syncthreads();
  float s = 0.0f;
  for (int t = threadIdx.x; t < B; t += 256) s += expf(at(t) - m);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) (row ? lseR : lseC)[r] = m + logf(red[0]);
}

// Gradient of the loss with respect to the normalised embeddings:
//   G_kl = (softmax_row(k)_l + softmax_col(l)_k - 2 [k == l]) / (2B),
//   dza_k = sum_l G_kl zp_l / T,  dzp_l = sum_k G_kl za_k / T.
// Threads 0..B*32-1 produce dza, the next B*32 dzp.  Block 0 also writes the loss.
__global__ void __launch_bounds__(256)
k_proj_demb(const float* __restrict__ S, const float* __restrict__ lseR, const float* __restrict__ lseC,
            const float* __restrict__ za, const float* __restrict__ zp, int B, float invT, float* __restrict__ dza,
            float* __restrict__ dzp, float* __restrict__ loss) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const float scale = 1.0f / (2.0f * (float)B);
  if (i < (long long)B * kOut) {
    const int k = (int)(i / kOut), o = (int)(i % kOut);
    float acc = 0.0f;
    for (int l = 0; l < B; ++l) {
      const float s = S[(size_t)k * B + l];
      float g = expf(s - lseR[k]) + expf(s - lseC[l]) - (k == l ? 2.0f : 0.0f);
      acc = fmaf(g, zp[(size_t)l * kOut + o], acc);
    }
    dza[i] = acc * scale * invT;
  } else if (i < 2LL * B * kOut) {
    const long long j = i - (long long)B * kOut;
    const int l = (int)(j / kOut), o = (int)(j % kOut);
    float acc = 0.0f;
    for (int k = 0; k < B; ++k) {
      const float s = S[(size_t)k * B + l];
      float g = expf(s - lseR[k]) + expf(s - lseC[l]) - (k == l ? 2.0f : 0.0f);
      acc = fmaf(g, za[(size_t)k * kOut + o], acc);
    }
    dzp[j] = acc * scale * invT;
  }
  if (blockIdx.x == 0) {
    __shared__ float red[256];
    float t = 0.0f;
    for (int k = threadIdx.x; k < B; k += 256) t += (lseR[k] - S[(size_t)k * B + k]) + (lseC[k] - S[(size_t)k * B + k]);
    red[threadIdx.x] = t;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) *loss = red[0] * scale;
  }
}

// Back through the normalisation and the second layer, per sample:
//   dz = (dzn - zn (zn . dzn)) / |z|,   dh = (W2^T dz) * [h > 0].
__global__ void k_proj_back_sample(const float* __restrict__ dzn, const float* __restrict__ zn,
                                   const float* __restrict__ nrm, const float* __restrict__ h,
                                   const __nv_bfloat16* __restrict__ w2b, int n, float* __restrict__ dz,
                                   float* __restrict__ dh) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float g[kOut];
  float dot = 0.0f;
#pragma unroll
  for (int o = 0; o < kOut; ++o) dot = fmaf(zn[(size_t)i * kOut + o], dzn[(size_t)i * kOut + o], dot);
  const float inv = 1.0f / fmaxf(nrm[i], kNormEps);
#pragma unroll
  for (int o = 0; o < kOut; ++o) {
    g[o] = (dzn[(size_t)i * kOut + o] - zn[(size_t)i * kOut + o] * dot) * inv;
    dz[(size_t)i * kOut + o] = g[o];
  }
  for (int j = 0; j < kHid; ++j) {
    float a = 0.0f;
#pragma unroll
    for (int o = 0; o < kOut; ++o) a = fmaf(__bfloat162float(w2b[o * kHid + j]), g[o], a);
    dh[(size_t)i * kHid + j] = h[(size_t)i * kHid + j] > 0.0f ? a : 0.0f;
  }
}

// Parameter gradients, one thread per parameter, summed over the n samples in order
// (deterministic):  dW1 = sum dh x^T, db1 = sum dh, dW2 = sum dz h^T, db2 = sum dz.
__global__ void k_proj_wgrad(const uint8_t* __restrict__ x, const float* __restrict__ h,
                             const float* __restrict__ dz, const float* __restrict__ dh, int n,
                             float* __restrict__ grad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kParams) return;
  float acc = 0.0f;
  if (t < kOffB1) {
    const int j = t / kIn, k = t % kIn;
    for (int i = 0; i < n; ++i) acc = fmaf(dh[(size_t)i * kHid + j], (float)x[(size_t)i * kIn + k] * (1.0f / 512.0f), acc);
  } else if (t < kOffW2) {
    const int j = t - kOffB1;
    for (int i = 0; i < n; ++i) acc += dh[(size_t)i * kHid + j];
  } else if (t < kOffB2) {
    const int o = (t - kOffW2) / kHid, j = (t - kOffW2) % kHid;
    for (int i = 0; i < n; ++i) acc = fmaf(dz[(size_t)i * kOut + o], h[(size_t)i * kHid + j], acc);
  } else {
    const int o = t - kOffB2;
    for (int i = 0; i < n; ++i) acc += dz[(size_t)i * kOut + o];
  }
  grad[t] = acc;
}

// Adam step on the FP32 master parameters; refreshes the BF16 weight copies.
__global__ void k_proj_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, float lr, float b1, float b2, float c1, float c2, float eps,
                            __nv_bfloat16* __restrict__ w1b, __nv_bfloat16* __restrict__ w2b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kParams) return;
  const float gt = g[t];
  const float mt = b1 * m[t] + (1.0f - b1) * gt;
  const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  const float wt = w[t] - lr * (mt / c1) / (sqrtf(vt / c2) + eps);
  w[t] = wt;
  if (t < kOffB1) w1b[t] = __float2bfloat16_rn(wt);
  else if (t >= kOffW2 && t < kOffB2) w2b[t - kOffW2] = __float2bfloat16_rn(wt);
}

__global__ void k_proj_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ w1b,
                               __nv_bfloat16* __restrict__ w2b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < kOffB1) w1b[t] = __float2bfloat16_rn(w[t]);
  else if (t >= kOffW2 && t < kOffB2) w2b[t - kOffW2] = __float2bfloat16_rn(w[t]);
}

struct PGuard {
  int prev = -1;
  explicit PGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~PGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

}  // namespace v3dm

using namespace v3dm;

struct v3dm_projection {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* dW = nullptr;                 // FP32 master parameters
  float* dM = nullptr;                 // Adam moments
  float* dV = nullptr;
  float* dG = nullptr;                 // gradient of the last step
  __nv_bfloat16* dW1b = nullptr;       // BF16 weights used by every forward pass
  __nv_bfloat16* dW2b = nullptr;
  int step = 0;
  int nCells = 0;
  float* dCells = nullptr;             // V3DM_PROJ_MAX_CELLS x 32
  // training scratch for batches of up to cap pairs
  int cap = 0;
  uint8_t* dX = nullptr;               // 2 cap x 128 (anchors then positives)
  float* dH = nullptr;                 // 2 cap x 64
  float* dZ = nullptr;                 // 2 cap x 32
  float* dN = nullptr;                 // 2 cap
  float* dS = nullptr;                 // cap x cap logits
  float* dLseR = nullptr;
  float* dLseC = nullptr;
  float* dDZn = nullptr;               // 2 cap x 32
  float* dDZ = nullptr;                // 2 cap x 32
  float* dDH = nullptr;                // 2 cap x 64
  float* dLoss = nullptr;
  float* hLoss = nullptr;              // pinned
};

namespace {

int pfail(cudaError_t e, const char* what, int line) {
  record_cuda_error(e, "v3dm_proposal.cu", line, what);
  return V3DM_ERR_CUDA;
}

#define V3DM_PTRY(expr)                                       \
  do {                                                        \
    cudaError_t e_ = (expr);                                  \
    if (e_ != cudaSuccess) return pfail(e_, #expr, __LINE__); \
  } while (0)

template <class T>
void pfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

void free_scratch(v3dm_projection* p) {
  pfree(p->dX);
  pfree(p->dH);
  pfree(p->dZ);
  pfree(p->dN);
  pfree(p->dS);
  pfree(p->dLseR);
  pfree(p->dLseC);
  pfree(p->dDZn);
  pfree(p->dDZ);
  pfree(p->dDH);
  p->cap = 0;
}

int ensure_scratch(v3dm_projection* p, int B) {
  if (B <= p->cap) return V3DM_OK;
  free_scratch(p);
  const size_t n2 = 2 * (size_t)B;
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&p->dX), n2 * kIn));
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&p->dH), n2 * kHid * sizeof(float)));
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&p->dZ), n2 * kOut * sizeof(float)));
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&p->dN), n2 * sizeof(float)));
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&p->dS), (size_t)B * B * sizeof(float)));
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&p->dLseR), (size_t)B * sizeof(float)));
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&p->dLseC), (size_t)B * sizeof(float)));
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&p->dDZn), n2 * kOut * sizeof(float)));
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&p->dDZ), n2 * kOut * sizeof(float)));
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&p->dDH), n2 * kHid * sizeof(float)));
  p->cap = B;
  return V3DM_OK;
}

// Loss and gradient of the batch in p->dX (B anchors then B positives) into p->dG / p->dLoss.
int loss_grad(v3dm_projection* p, int B, float T) {
  const int n2 = 2 * B;
  const float invT = 1.0f / T;
  V3DM_PTRY(launch_forward(p->dX, n2, p->dW1b, p->dW + kOffB1, p->dW2b, p->dW + kOffB2, p->dH, p->dZ, p->dN,
                           p->dCells, 0, 0, nullptr, p->stream));
  const float* za = p->dZ;
  const float* zp = p->dZ + (size_t)B * kOut;
  const long long nS = (long long)B * B;
  k_proj_logits<<<(unsigned)((nS + 255) / 256), 256, 0, p->stream>>>(za, zp, B, invT, p->dS);
  V3DM_PTRY(cudaGetLastError());
  k_proj_lse<<<2 * B, 256, 0, p->stream>>>(p->dS, B, p->dLseR, p->dLseC);
  V3DM_PTRY(cudaGetLastError());
  const long long nD = 2LL * B * kOut;
  k_proj_demb<<<(unsigned)((nD + 255) / 256), 256, 0, p->stream>>>(p->dS, p->dLseR, p->dLseC, za, zp, B, invT, p->dDZn,
                                                                   p->dDZn + (size_t)B * kOut, p->dLoss);
  V3DM_PTRY(cudaGetLastError());
  k_proj_back_sample<<<(n2 + 127) / 128, 128, 0, p->stream>>>(p->dDZn, p->dZ, p->dN, p->dH, p->dW2b, n2, p->dDZ,
                                                              p->dDH);
  V3DM_PTRY(cudaGetLastError());
  k_proj_wgrad<<<(kParams + 127) / 128, 128, 0, p->stream>>>(p->dX, p->dH, p->dDZ, p->dDH, n2, p->dG);
  V3DM_PTRY(cudaGetLastError());
  return V3DM_OK;
}

int check_batch(const void* a, const void* pos, int B, float T) {
  if (!a || !pos || B < 2 || B > V3DM_PROJ_MAX_BATCH || !(T > 0.0f)) return V3DM_ERR_ARG;
  return V3DM_OK;
}

}  // namespace

// Shared with the batched matcher (v3dm_batch.cu).
namespace v3dm {
cudaError_t proj_assign(const v3dm_projection* p, const uint8_t* dDesc, long long n, int probes, uint8_t* dCells,
                        cudaStream_t s) {
  return launch_forward(dDesc, n, p->dW1b, p->dW + kOffB1, p->dW2b, p->dW + kOffB2, nullptr, nullptr, nullptr,
                        p->dCells, p->nCells, probes, dCells, s);
}
int proj_cells(const v3dm_projection* p) { return p->nCells; }
cudaStream_t proj_stream(const v3dm_projection* p) { return p->stream; }
}  // namespace v3dm

extern "C" {

int v3dm_projection_create(v3dm_projection** out, int device, unsigned long long seed) {
  if (!out) return V3DM_ERR_ARG;
  *out = nullptr;
  int nDev = 0;
  if (cudaGetDeviceCount(&nDev) != cudaSuccess || device < 0 || device >= nDev) return V3DM_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return V3DM_ERR_CUDA;
  if (prop.major != 10) return V3DM_ERR_NO_DEVICE;
  v3dm_projection* p = new (std::nothrow) v3dm_projection();
  if (!p) return V3DM_ERR_ARG;
  p->device = device;
  PGuard g(device);
  bool ok = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(reinterpret_cast<void**>(&p->dW), kParams * sizeof(float)) == cudaSuccess &&
            cudaMalloc(reinterpret_cast<void**>(&p->dM), kParams * sizeof(float)) == cudaSuccess &&
            cudaMalloc(reinterpret_cast<void**>(&p->dV), kParams * sizeof(float)) == cudaSuccess &&
            cudaMalloc(reinterpret_cast<void**>(&p->dG), kParams * sizeof(float)) == cudaSuccess &&
            cudaMalloc(reinterpret_cast<void**>(&p->dW1b), kHid * kIn * sizeof(__nv_bfloat16)) == cudaSuccess &&
            cudaMalloc(reinterpret_cast<void**>(&p->dW2b), kOut * kHid * sizeof(__nv_bfloat16)) == cudaSuccess &&
            cudaMalloc(reinterpret_cast<void**>(&p->dCells), V3DM_PROJ_MAX_CELLS * kOut * sizeof(float)) == cudaSuccess &&
            cudaMalloc(reinterpret_cast<void**>(&p->dLoss), sizeof(float)) == cudaSuccess &&
            cudaMallocHost(reinterpret_cast<void**>(&p->hLoss), sizeof(float)) == cudaSuccess;
  if (ok) {
    // He-uniform initialisation from a seeded generator (host), zero biases.
    std::vector<float> w(kParams, 0.0f);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> u1(-std::sqrt(6.0f / kIn), std::sqrt(6.0f / kIn));
    std::uniform_real_distribution<float> u2(-std::sqrt(6.0f / kHid), std::sqrt(6.0f / kHid));
    for (int i = 0; i < kHid * kIn; ++i) w[kOffW1 + i] = u1(rng);
    for (int i = 0; i < kOut * kHid; ++i) w[kOffW2 + i] = u2(rng);
    ok = cudaMemcpy(p->dW, w.data(), kParams * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(p->dM, 0, kParams * sizeof(float)) == cudaSuccess &&
         cudaMemset(p->dV, 0, kParams * sizeof(float)) == cudaSuccess &&
         cudaMemset(p->dCells, 0, V3DM_PROJ_MAX_CELLS * kOut * sizeof(float)) == cudaSuccess;
    if (ok) {
      k_proj_to_bf16<<<(kParams + 255) / 256, 256, 0, p->stream>>>(p->dW, p->dW1b, p->dW2b);
      ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(p->stream) == cudaSuccess;
    }
  }
  if (!ok) {
    v3dm_projection_destroy(p);
    return V3DM_ERR_CUDA;
  }
  *out = p;
  return V3DM_OK;
}

int v3dm_projection_destroy(v3dm_projection* p) {
  if (!p) return V3DM_ERR_ARG;
  PGuard g(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  free_scratch(p);
  pfree(p->dW);
  pfree(p->dM);
  pfree(p->dV);
  pfree(p->dG);
  pfree(p->dW1b);
  pfree(p->dW2b);
  pfree(p->dCells);
  pfree(p->dLoss);
  if (p->hLoss) cudaFreeHost(p->hLoss);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
  return V3DM_OK;
}

int v3dm_projection_get_params(v3dm_projection* p, float* params) {
  if (!p || !params) return V3DM_ERR_ARG;
  PGuard g(p->device);
  V3DM_PTRY(cudaMemcpyAsync(params, p->dW, kParams * sizeof(float), cudaMemcpyDeviceToHost, p->stream));
  V3DM_PTRY(cudaStreamSynchronize(p->stream));
  return V3DM_OK;
}

int v3dm_projection_set_params(v3dm_projection* p, const float* params) {
  if (!p || !params) return V3DM_ERR_ARG;
  PGuard g(p->device);
  V3DM_PTRY(cudaMemcpyAsync(p->dW, params, kParams * sizeof(float), cudaMemcpyHostToDevice, p->stream));
  V3DM_PTRY(cudaMemsetAsync(p->dM, 0, kParams * sizeof(float), p->stream));
  V3DM_PTRY(cudaMemsetAsync(p->dV, 0, kParams * sizeof(float), p->stream));
  k_proj_to_bf16<<<(kParams + 255) / 256, 256, 0, p->stream>>>(p->dW, p->dW1b, p->dW2b);
  V3DM_PTRY(cudaGetLastError());
  V3DM_PTRY(cudaStreamSynchronize(p->stream));
  p->step = 0;
  return V3DM_OK;
}

int v3dm_projection_loss_grad(v3dm_projection* p, const uint8_t* anchors, const uint8_t* positives, int B,
                              float temperature, float* loss, float* grad) {
  if (!p) return V3DM_ERR_ARG;
  int st = check_batch(anchors, positives, B, temperature);
  if (st != V3DM_OK) return st;
  PGuard g(p->device);
  st = ensure_scratch(p, B);
  if (st != V3DM_OK) return st;
  V3DM_PTRY(cudaMemcpyAsync(p->dX, anchors, (size_t)B * kIn, cudaMemcpyHostToDevice, p->stream));
  V3DM_PTRY(cudaMemcpyAsync(p->dX + (size_t)B * kIn, positives, (size_t)B * kIn, cudaMemcpyHostToDevice, p->stream));
  st = loss_grad(p, B, temperature);
  if (st != V3DM_OK) return st;
  V3DM_PTRY(cudaMemcpyAsync(p->hLoss, p->dLoss, sizeof(float), cudaMemcpyDeviceToHost, p->stream));
  if (grad) V3DM_PTRY(cudaMemcpyAsync(grad, p->dG, kParams * sizeof(float), cudaMemcpyDeviceToHost, p->stream));
  V3DM_PTRY(cudaStreamSynchronize(p->stream));
  if (loss) *loss = *p->hLoss;
  return V3DM_OK;
}

int v3dm_projection_train_step(v3dm_projection* p, const uint8_t* d_anchors, const uint8_t* d_positives, int B,
                               float temperature, float lr, float* loss) {
  if (!p || !(lr > 0.0f)) return V3DM_ERR_ARG;
  int st = check_batch(d_anchors, d_positives, B, temperature);
  if (st != V3DM_OK) return st;
  PGuard g(p->device);
  st = ensure_scratch(p, B);
  if (st != V3DM_OK) return st;
  V3DM_PTRY(cudaMemcpyAsync(p->dX, d_anchors, (size_t)B * kIn, cudaMemcpyDeviceToDevice, p->stream));
  V3DM_PTRY(cudaMemcpyAsync(p->dX + (size_t)B * kIn, d_positives, (size_t)B * kIn, cudaMemcpyDeviceToDevice,
                            p->stream));
  st = loss_grad(p, B, temperature);
  if (st != V3DM_OK) return st;
  ++p->step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)p->step), c2 = 1.0f - std::pow(b2, (float)p->step);
  k_proj_adam<<<(kParams + 255) / 256, 256, 0, p->stream>>>(p->dW, p->dM, p->dV, p->dG, lr, b1, b2, c1, c2, 1e-8f,
                                                            p->dW1b, p->dW2b);
  V3DM_PTRY(cudaGetLastError());
  if (loss) {
    V3DM_PTRY(cudaMemcpyAsync(p->hLoss, p->dLoss, sizeof(float), cudaMemcpyDeviceToHost, p->stream));
    V3DM_PTRY(cudaStreamSynchronize(p->stream));
    *loss = *p->hLoss;
  }
  return V3DM_OK;
}

int v3dm_projection_embed(v3dm_projection* p, const uint8_t* desc, int n, float* z) {
  if (!p || n < 0 || (n > 0 && (!desc || !z))) return V3DM_ERR_ARG;
  if (n == 0) return V3DM_OK;
  PGuard g(p->device);
  uint8_t* dD = nullptr;
  float* dZ = nullptr;
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&dD), (size_t)n * kIn));
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&dZ), (size_t)n * kOut * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpyAsync(dD, desc, (size_t)n * kIn, cudaMemcpyHostToDevice, p->stream);
  if (e == cudaSuccess)
    e = launch_forward(dD, n, p->dW1b, p->dW + kOffB1, p->dW2b, p->dW + kOffB2, nullptr, dZ, nullptr, p->dCells, 0, 0,
                       nullptr, p->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(z, dZ, (size_t)n * kOut * sizeof(float), cudaMemcpyDeviceToHost, p->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
  cudaFree(dD);
  if (dZ) cudaFree(dZ);
  if (e != cudaSuccess) return pfail(e, "embed", __LINE__);
  return V3DM_OK;
}

int v3dm_projection_set_cells(v3dm_projection* p, int nCells, const float* centroids) {
  if (!p || nCells < 1 || nCells > V3DM_PROJ_MAX_CELLS || !centroids) return V3DM_ERR_ARG;
  PGuard g(p->device);
  V3DM_PTRY(cudaMemcpyAsync(p->dCells, centroids, (size_t)nCells * kOut * sizeof(float), cudaMemcpyHostToDevice,
                            p->stream));
  V3DM_PTRY(cudaStreamSynchronize(p->stream));
  p->nCells = nCells;
  return V3DM_OK;
}

int v3dm_projection_assign(v3dm_projection* p, const uint8_t* desc, int n, int probes, uint8_t* cells) {
  if (!p || n < 0 || probes < 1 || probes > V3DM_PROJ_MAX_PROBES || (n > 0 && (!desc || !cells))) return V3DM_ERR_ARG;
  if (p->nCells == 0) return V3DM_ERR_NOT_ALLOCATED;
  if (probes > p->nCells) return V3DM_ERR_ARG;
  if (n == 0) return V3DM_OK;
  PGuard g(p->device);
  uint8_t* dD = nullptr;
  uint8_t* dC = nullptr;
  V3DM_PTRY(cudaMalloc(reinterpret_cast<void**>(&dD), (size_t)n * kIn));
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&dC), (size_t)n * probes);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dD, desc, (size_t)n * kIn, cudaMemcpyHostToDevice, p->stream);
  if (e == cudaSuccess) e = proj_assign(p, dD, n, probes, dC, p->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cells, dC, (size_t)n * probes, cudaMemcpyDeviceToHost, p->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
  cudaFree(dD);
  if (dC) cudaFree(dC);
  if (e != cudaSuccess) return pfail(e, "assign", __LINE__);
  return V3DM_OK;
}

}  // extern "C"
