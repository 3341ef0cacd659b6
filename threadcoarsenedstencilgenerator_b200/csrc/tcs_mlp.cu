// Cost model of the autotuner: a 3-layer perceptron (n_in -> H -> H -> 1, ReLU) in FP32 with
// hand-written forward, backward and Adam kernels.  No counterpart in the reference, whose
// block-shape choice is an exhaustive timed sweep (cuda/benchmark.cpp:223-251, 287-318).
//
// Parameters live in one packed device vector: W1 [n_in x H], b1 [H], W2 [H x H], b2 [H],
// W3 [H x 1], b3 [1] (row-major, input index first).  Every reduction runs in a fixed order, so
// results are deterministic run to run.

#include "tcs.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "tcs_field.h"  // tcs_internal_set_error: the message tcs_last_error returns

namespace {

int mfail(int code, const std::string& msg) {
  tcs_internal_set_error(msg.c_str());
  return code;
}

constexpr int TILE = 32;  // output tile edge of the GEMM kernel
constexpr int TK = 32;    // reduction slice staged in shared memory
constexpr int ROWS_PER_THREAD = 4;

// C[M x N] = act(op(A)[M x K] * op(B)[K x N] + bias), op = transpose when TA / TB.
// A is [M x K] (lda = K) or, transposed, [K x M] (lda = M); B is [K x N] (ldb = N) or [N x K].
// Block 32 x 8 threads; each thread owns 4 rows of one column of a 32 x 32 tile.
template <bool TA, bool TB, bool RELU, bool BIAS>
__global__ void __launch_bounds__(TILE * (TILE / ROWS_PER_THREAD))
    mlp_gemm(const float* __restrict__ A, const float* __restrict__ B,
             const float* __restrict__ bias, float* __restrict__ C, int M, int N, int K) {
  __shared__ float As[TK][TILE + 1];  // As[k][m]
  __shared__ float Bs[TK][TILE + 1];  // Bs[k][n]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int m0 = blockIdx.y * TILE, n0 = blockIdx.x * TILE;
  float acc[ROWS_PER_THREAD] = {0.f, 0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < K; k0 += TK) {
    for (int i = ty; i < TK; i += TILE / ROWS_PER_THREAD) {
      // As[i][tx] = A(m0 + tx, k0 + i); Bs[i][tx] = B(k0 + i, n0 + tx)
      const int m = m0 + tx, k = k0 + i, n = n0 + tx;
      float a = 0.f, b = 0.f;
      if (m < M && k < K) a = TA ? A[(size_t)k * M + m] : A[(size_t)m * K + k];
      if (k < K && n < N) b = TB ? B[(size_t)n * K + k] : B[(size_t)k * N + n];
      As[i][tx] = a;
      Bs[i][tx] = b;
    }
    __syncthreads();
    const int kn = min(TK, K - k0);
    for (int k = 0; k < kn; ++k) {
      const float b = Bs[k][tx];
#pragma unroll
      for (int r = 0; r < ROWS_PER_THREAD; ++r) acc[r] = fmaf(As[k][ty * ROWS_PER_THREAD + r], b, acc[r]);
    }
    __syncthreads();
  }
  const int n = n0 + tx;
  if (n >= N) return;
#pragma unroll
  for (int r = 0; r < ROWS_PER_THREAD; ++r) {
    const int m = m0 + ty * ROWS_PER_THREAD + r;
    if (m >= M) continue;
    float v = acc[r];
    if (BIAS) v += bias[n];
    if (RELU) v = fmaxf(v, 0.f);
    C[(size_t)m * N + n] = v;
  }
}

// dZ = dA * (A > 0): gradient through the ReLU given its output A.
__global__ void mlp_relu_grad(const float* __restrict__ a, float* __restrict__ d, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    if (!(a[i] > 0.f)) d[i] = 0.f;
}

// db[n] = sum over rows m of D[m][n] (one block per column, fixed-order tree).
__global__ void mlp_colsum(const float* __restrict__ D, float* __restrict__ out, int M, int N) {
  __shared__ float red[256];
  const int n = blockIdx.x;
  float s = 0.f;
  for (int m = threadIdx.x; m < M; m += blockDim.x) s += D[(size_t)m * N + n];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w /= 2) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = red[0];
}

// dY = 2 (Y - T) / M and per-block partial sums of (Y - T)^2.
__global__ void mlp_mse_grad(const float* __restrict__ y, const float* __restrict__ t,
                             float* __restrict__ dy, float* __restrict__ partial, int M) {
  __shared__ float red[256];
  float s = 0.f;
  const float scale = 2.f / (float)M;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
    const float e = y[i] - t[i];
    dy[i] = scale * e;
    s = fmaf(e, e, s);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w /= 2) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void mlp_sum(const float* __restrict__ partial, int n, float scale, float* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float s = 0.f;
    for (int i = 0; i < n; ++i) s += partial[i];
    *out = s * scale;
  }
}

// Adam (Kingma & Ba 2015) with bias correction; c1 = 1 - beta1^t, c2 = 1 - beta2^t.
__global__ void mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                         float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps,
                         float c1, float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

constexpr int MSE_BLOCKS = 64;

}  // namespace

struct tcs_mlp {
  unsigned n_in = 0, H = 0, max_batch = 0;
  size_t n_params = 0;
  float* p = nullptr;     // parameters
  float* g = nullptr;     // gradient
  float* m = nullptr;     // Adam first moment
  float* v = nullptr;     // Adam second moment
  float* a1 = nullptr;    // [max_batch x H] layer-1 output (post-ReLU)
  float* a2 = nullptr;    // [max_batch x H] layer-2 output
  float* d1 = nullptr;    // [max_batch x H] gradient scratch
  float* d2 = nullptr;    // [max_batch x H]
  float* y = nullptr;     // [max_batch] prediction
  float* dy = nullptr;    // [max_batch]
  float* partial = nullptr;  // [MSE_BLOCKS + 1] loss partials, loss at [MSE_BLOCKS]
  unsigned long long step = 0;

  size_t off_w1() const { return 0; }
  size_t off_b1() const { return (size_t)n_in * H; }
  size_t off_w2() const { return off_b1() + H; }
  size_t off_b2() const { return off_w2() + (size_t)H * H; }
  size_t off_w3() const { return off_b2() + H; }
  size_t off_b3() const { return off_w3() + H; }
};

namespace {

int rt(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return TCS_OK;
  return mfail(TCS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <bool TA, bool TB, bool RELU, bool BIAS>
void gemm(const float* A, const float* B, const float* bias, float* C, int M, int N, int K, cudaStream_t st) {
  dim3 grid((N + TILE - 1) / TILE, (M + TILE - 1) / TILE);
  dim3 block(TILE, TILE / ROWS_PER_THREAD);
  mlp_gemm<TA, TB, RELU, BIAS><<<grid, block, 0, st>>>(A, B, bias, C, M, N, K);
}

unsigned grid_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (unsigned)(b < 1024 ? (b ? b : 1) : 1024);
}

void forward(tcs_mlp* m, const float* x, int n, cudaStream_t st) {
  const int H = (int)m->H, I = (int)m->n_in;
  gemm<false, false, true, true>(x, m->p + m->off_w1(), m->p + m->off_b1(), m->a1, n, H, I, st);
  gemm<false, false, true, true>(m->a1, m->p + m->off_w2(), m->p + m->off_b2(), m->a2, n, H, H, st);
  gemm<false, false, false, true>(m->a2, m->p + m->off_w3(), m->p + m->off_b3(), m->y, n, 1, H, st);
}

// Gradient of mean((y - t)^2) w.r.t. all parameters into m->g; loss into m->partial[MSE_BLOCKS].
void backward(tcs_mlp* m, const float* x, const float* t, int n, cudaStream_t st) {
  const int H = (int)m->H, I = (int)m->n_in;
  float* g = m->g;
  mlp_mse_grad<<<MSE_BLOCKS, 256, 0, st>>>(m->y, t, m->dy, m->partial, n);
  mlp_sum<<<1, 32, 0, st>>>(m->partial, MSE_BLOCKS, 1.f / (float)n, m->partial + MSE_BLOCKS);
  // layer 3: y = a2 W3 + b3
  gemm<true, false, false, false>(m->a2, m->dy, nullptr, g + m->off_w3(), H, 1, n, st);  // a2^T dy
  mlp_colsum<<<1, 256, 0, st>>>(m->dy, g + m->off_b3(), n, 1);
  gemm<false, true, false, false>(m->dy, m->p + m->off_w3(), nullptr, m->d2, n, H, 1, st);  // dy W3^T
  mlp_relu_grad<<<grid_for((size_t)n * H), 256, 0, st>>>(m->a2, m->d2, (size_t)n * H);
  // layer 2: a2 = relu(a1 W2 + b2)
  gemm<true, false, false, false>(m->a1, m->d2, nullptr, g + m->off_w2(), H, H, n, st);
  mlp_colsum<<<H, 256, 0, st>>>(m->d2, g + m->off_b2(), n, H);
  gemm<false, true, false, false>(m->d2, m->p + m->off_w2(), nullptr, m->d1, n, H, H, st);
  mlp_relu_grad<<<grid_for((size_t)n * H), 256, 0, st>>>(m->a1, m->d1, (size_t)n * H);
  // layer 1: a1 = relu(x W1 + b1)
  gemm<true, false, false, false>(x, m->d1, nullptr, g + m->off_w1(), I, H, n, st);
  mlp_colsum<<<H, 256, 0, st>>>(m->d1, g + m->off_b1(), n, H);
}

int check_batch(const tcs_mlp* m, unsigned n) {
  if (n == 0 || n > m->max_batch)
    return mfail(TCS_ERR_INVALID_VALUE, "batch of " + std::to_string(n) + " rows; the model holds buffers for 1.." +
                                            std::to_string(m->max_batch));
  return TCS_OK;
}

}  // namespace

extern "C" {

int tcs_mlp_create(unsigned n_in, unsigned n_hidden, unsigned max_batch, tcs_mlp** out) {
  if (!out) return mfail(TCS_ERR_INVALID_VALUE, "NULL output");
  *out = nullptr;
  if (n_in == 0 || n_hidden == 0 || max_batch == 0 || n_in > 4096 || n_hidden > 4096)
    return mfail(TCS_ERR_INVALID_VALUE, "layer sizes must be 1..4096 and max_batch >= 1");
  tcs_mlp* m = new tcs_mlp();
  m->n_in = n_in;
  m->H = n_hidden;
  m->max_batch = max_batch;
  m->n_params = m->off_b3() + 1;
  const size_t act = (size_t)max_batch * n_hidden;
  float** bufs[] = {&m->p, &m->g, &m->m, &m->v, &m->a1, &m->a2, &m->d1, &m->d2, &m->y, &m->dy, &m->partial};
  const size_t sizes[] = {m->n_params, m->n_params, m->n_params, m->n_params, act, act, act, act,
                          max_batch, max_batch, MSE_BLOCKS + 1};
  for (int i = 0; i < 11; ++i) {
    cudaError_t e = cudaMalloc((void**)bufs[i], sizes[i] * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(*bufs[i], 0, sizes[i] * sizeof(float));
    if (e != cudaSuccess) {
      tcs_mlp_destroy(m);
      return rt(e, "tcs_mlp_create");
    }
  }
  *out = m;
  return TCS_OK;
}

int tcs_mlp_param_count(const tcs_mlp* m, unsigned* count) {
  if (!m || !count) return mfail(TCS_ERR_INVALID_VALUE, "NULL argument");
  *count = (unsigned)m->n_params;
  return TCS_OK;
}

int tcs_mlp_set_params(tcs_mlp* m, const float* host, unsigned n) {
  if (!m || !host) return mfail(TCS_ERR_INVALID_VALUE, "NULL argument");
  if (n != m->n_params) return mfail(TCS_ERR_INVALID_VALUE, "expected " + std::to_string(m->n_params) + " parameters");
  int rc = rt(cudaMemcpy(m->p, host, n * sizeof(float), cudaMemcpyHostToDevice), "tcs_mlp_set_params");
  if (rc) return rc;
  m->step = 0;
  if ((rc = rt(cudaMemset(m->m, 0, n * sizeof(float)), "tcs_mlp_set_params"))) return rc;
  return rt(cudaMemset(m->v, 0, n * sizeof(float)), "tcs_mlp_set_params");
}

int tcs_mlp_get_params(const tcs_mlp* m, float* host, unsigned n) {
  if (!m || !host) return mfail(TCS_ERR_INVALID_VALUE, "NULL argument");
  if (n != m->n_params) return mfail(TCS_ERR_INVALID_VALUE, "expected " + std::to_string(m->n_params) + " parameters");
  return rt(cudaMemcpy(host, m->p, n * sizeof(float), cudaMemcpyDeviceToHost), "tcs_mlp_get_params");
}

int tcs_mlp_forward(tcs_mlp* m, const float* x, unsigned n, float* y, void* stream) {
  if (!m || !x || !y) return mfail(TCS_ERR_INVALID_VALUE, "NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  // Inputs of any length: batches of at most max_batch rows through the activation buffers.
  for (unsigned r0 = 0; r0 < n; r0 += m->max_batch) {
    const unsigned nb = std::min(m->max_batch, n - r0);
    forward(m, x + (size_t)r0 * m->n_in, (int)nb, st);
    int rc = rt(cudaMemcpyAsync(y + r0, m->y, nb * sizeof(float), cudaMemcpyDeviceToDevice, st), "tcs_mlp_forward");
    if (rc) return rc;
  }
  return rt(cudaGetLastError(), "tcs_mlp_forward");
}

int tcs_mlp_gradient(tcs_mlp* m, const float* x, const float* t, unsigned n, float* grad, float* loss,
                     void* stream) {
  if (!m || !x || !t) return mfail(TCS_ERR_INVALID_VALUE, "NULL argument");
  int rc = check_batch(m, n);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  forward(m, x, (int)n, st);
  backward(m, x, t, (int)n, st);
  if (grad &&
      (rc = rt(cudaMemcpyAsync(grad, m->g, m->n_params * sizeof(float), cudaMemcpyDeviceToDevice, st),
               "tcs_mlp_gradient")))
    return rc;
  if (loss) {
    if ((rc = rt(cudaMemcpyAsync(loss, m->partial + MSE_BLOCKS, sizeof(float), cudaMemcpyDeviceToHost, st),
                 "tcs_mlp_gradient")))
      return rc;
    if ((rc = rt(cudaStreamSynchronize(st), "tcs_mlp_gradient"))) return rc;
  }
  return rt(cudaGetLastError(), "tcs_mlp_gradient");
}

int tcs_mlp_adam_step(tcs_mlp* m, const float* x, const float* t, unsigned n, float lr, float beta1,
                      float beta2, float eps, float* loss, void* stream) {
  int rc = tcs_mlp_gradient(m, x, t, n, nullptr, loss, stream);
  if (rc) return rc;
  m->step += 1;
  const float c1 = 1.f - (float)std::pow((double)beta1, (double)m->step);
  const float c2 = 1.f - (float)std::pow((double)beta2, (double)m->step);
  mlp_adam<<<grid_for(m->n_params), 256, 0, (cudaStream_t)stream>>>(m->p, m->g, m->m, m->v, m->n_params, lr,
                                                                      beta1, beta2, eps, c1, c2);
  return rt(cudaGetLastError(), "tcs_mlp_adam_step");
}

int tcs_mlp_destroy(tcs_mlp* m) {
  if (!m) return TCS_OK;
  float* bufs[] = {m->p, m->g, m->m, m->v, m->a1, m->a2, m->d1, m->d2, m->y, m->dy, m->partial};
  for (float* b : bufs)
    if (b) cudaFree(b);
  delete m;
  return TCS_OK;
}

}  // extern "C"
