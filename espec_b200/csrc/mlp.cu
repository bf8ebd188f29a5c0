// mlp.cu -- kernels of the learned warm start for the eigensolver: a small
// multilayer perceptron (forward, backward, Adam) and the dense products that
// move eigenvectors in and out of its output basis.
//
// The network maps the 5 parameters of a potential to the coefficients of
// the lowest eigenvectors in a fixed product basis phi_i(x) chi_j(y); it is
// trained on eigenvectors produced by the plain eigensolver (eig.cu).  The
// layers are tiny (5 -> 128 -> 128 -> 4 nb), so the products run as tiled
// SIMT kernels: one 64 x 64 output tile per 256-thread CTA, 16-deep k tiles
// staged in shared memory, 4 x 4 outputs per thread.
#include <cuda_runtime.h>

#include "espec_gpu.h"
#include "espec_internal.h"

namespace espec {
namespace {

constexpr int TM = 64, TN = 64, TK = 16;

// C[M,N] = alpha op(A)[M,K] op(B)[K,N] + beta C; op = transpose when ta/tb.
// Row-major: A is [M,K] (or [K,M] when ta), B is [K,N] (or [N,K] when tb).
template <typename T>
__global__ void __launch_bounds__(256) gemm_kernel(int M, int N, int K, T alpha, const T* A,
                                                   int lda, int ta, const T* B, int ldb, int tb,
                                                   T beta, T* C, int ldc) {
  __shared__ T As[TK][TM + 1];
  __shared__ T Bs[TK][TN + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
  for (int k0 = 0; k0 < K; k0 += TK) {
    for (int e = threadIdx.x; e < TK * TM; e += 256) {
      const int kk = e / TM, mm = e % TM;
      const int gm = m0 + mm, gk = k0 + kk;
      T v = T(0);
      if (gm < M && gk < K) v = ta ? A[(long)gk * lda + gm] : A[(long)gm * lda + gk];
      As[kk][mm] = v;
    }
    for (int e = threadIdx.x; e < TK * TN; e += 256) {
      const int kk = e / TN, nn = e % TN;
      const int gn = n0 + nn, gk = k0 + kk;
      T v = T(0);
      if (gn < N && gk < K) v = tb ? B[(long)gn * ldb + gk] : B[(long)gk * ldb + gn];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gn = n0 + tx + 16 * j;
      if (gn >= N) continue;
      T* c = C + (long)gm * ldc + gn;
      *c = beta == T(0) ? alpha * acc[i][j] : alpha * acc[i][j] + beta * *c;
    }
  }
}

// y = x + b (row broadcast), then tanh when act
__global__ void bias_act_kernel(float* y, const float* b, int rows, int cols, int act) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)rows * cols) return;
  float v = y[i] + b[i % cols];
  y[i] = act ? tanhf(v) : v;
}

// dz = dy * (1 - y^2), y = tanh(z)
__global__ void tanh_back_kernel(float* dz, const float* y, long count) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  dz[i] = dz[i] * (1.0f - y[i] * y[i]);
}

// db[c] = sum_r dy[r, c] (fixed order over rows)
__global__ void colsum_kernel(const float* dy, int rows, int cols, float* db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += dy[(long)r * cols + c];
  db[c] = s;
}

// loss = mean over rows of sum (y - t)^2 / cols; dy = 2 (y - t) / (rows cols)
__global__ void mse_kernel(const float* y, const float* t, int rows, int cols, float* dy,
                           float* row_loss) {
  const int r = blockIdx.x;
  float s = 0.0f;
  const float sc = 2.0f / ((float)rows * (float)cols);
  for (int c = threadIdx.x; c < cols; c += blockDim.x) {
    const float d = y[(long)r * cols + c] - t[(long)r * cols + c];
    dy[(long)r * cols + c] = sc * d;
    s += d * d;
  }
  __shared__ float red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) row_loss[r] = red[0] / ((float)rows * (float)cols);
}

// Adam (Kingma & Ba, 2015) with bias correction folded into the step size
__global__ void adam_kernel(float* w, const float* g, float* m1, float* m2, long count, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// the same with (lr, c1, c2) read from device memory, so that one captured
// training step can be replayed with a new step size and bias correction
__global__ void adam_dev_kernel(float* w, const float* g, float* m1, float* m2, long count,
                                const float* hyper, float b1, float b2, float eps) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float lr = hyper[0], c1 = hyper[1], c2 = hyper[2];
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

// product basis: B[(i*nby + j), (x + nx*y)] = phi[i][x] chi[j][y]
__global__ void outer_basis_kernel(const double* phi, int nbx, int nx, const double* chi, int nby,
                                   int ny, double* B) {
  const long n = (long)nx * ny;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= n * nbx * nby) return;
  const long b = gid / n, k = gid % n;
  const int i = (int)(b / nby), j = (int)(b % nby);
  const int x = (int)(k % nx), y = (int)(k / nx);
  B[gid] = phi[(long)i * nx + x] * chi[(long)j * ny + y];
}

__global__ void f64_to_f32_kernel(const double* a, float* b, long count, double scale) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) b[i] = (float)(a[i] * scale);
}

__global__ void f32_to_f64_kernel(const float* a, double* b, long count, double scale) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) b[i] = (double)a[i] * scale;
}

inline unsigned blocks(long count, int bs = 256) { return (unsigned)((count + bs - 1) / bs); }

}  // namespace
}  // namespace espec

using namespace espec;

#define MLP_CK()                                                           \
  do {                                                                     \
    cudaError_t e_ = cudaGetLastError();                                   \
    if (e_ != cudaSuccess) return set_cuda_error("mlp kernel launch", e_); \
  } while (0)

template <typename T>
static int gemm_launch(int M, int N, int K, T alpha, const T* A, int lda, int ta, const T* B,
                       int ldb, int tb, T beta, T* C, int ldc, void* stream) {
  if (M <= 0 || N <= 0 || K < 0 || !A || !B || !C) return set_error(ESPEC_EINVAL, "bad GEMM");
  dim3 grid((N + TN - 1) / TN, (M + TM - 1) / TM);
  gemm_kernel<T><<<grid, 256, 0, (cudaStream_t)stream>>>(M, N, K, alpha, A, lda, ta, B, ldb, tb,
                                                         beta, C, ldc);
  MLP_CK();
  return ESPEC_OK;
}

extern "C" int espec_gemm_f64(int M, int N, int K, double alpha, const double* A, int lda, int ta,
                              const double* B, int ldb, int tb, double beta, double* C, int ldc,
                              void* stream) {
  return gemm_launch<double>(M, N, K, alpha, A, lda, ta, B, ldb, tb, beta, C, ldc, stream);
}

extern "C" int espec_gemm_f32(int M, int N, int K, float alpha, const float* A, int lda, int ta,
                              const float* B, int ldb, int tb, float beta, float* C, int ldc,
                              void* stream) {
  return gemm_launch<float>(M, N, K, alpha, A, lda, ta, B, ldb, tb, beta, C, ldc, stream);
}

extern "C" int espec_mlp_bias_act(float* y, const float* b, int rows, int cols, int act,
                                  void* stream) {
  bias_act_kernel<<<blocks((long)rows * cols), 256, 0, (cudaStream_t)stream>>>(y, b, rows, cols,
                                                                              act);
  MLP_CK();
  return ESPEC_OK;
}

extern "C" int espec_mlp_tanh_back(float* dz, const float* y, long count, void* stream) {
  tanh_back_kernel<<<blocks(count), 256, 0, (cudaStream_t)stream>>>(dz, y, count);
  MLP_CK();
  return ESPEC_OK;
}

extern "C" int espec_mlp_colsum(const float* dy, int rows, int cols, float* db, void* stream) {
  colsum_kernel<<<blocks(cols), 256, 0, (cudaStream_t)stream>>>(dy, rows, cols, db);
  MLP_CK();
  return ESPEC_OK;
}

extern "C" int espec_mlp_mse(const float* y, const float* t, int rows, int cols, float* dy,
                             float* row_loss, void* stream) {
  mse_kernel<<<rows, 256, 0, (cudaStream_t)stream>>>(y, t, rows, cols, dy, row_loss);
  MLP_CK();
  return ESPEC_OK;
}

extern "C" int espec_mlp_adam(float* w, const float* g, float* m1, float* m2, long count,
                              float lr, float b1, float b2, float eps, int step, void* stream) {
  if (step < 1) return set_error(ESPEC_EINVAL, "Adam step counts from 1");
  float c1 = 1.0f, c2 = 1.0f, p1 = 1.0f, p2 = 1.0f;
  for (int i = 0; i < step; ++i) {
    p1 *= b1;
    p2 *= b2;
  }
  c1 = 1.0f - p1;
  c2 = 1.0f - p2;
  adam_kernel<<<blocks(count), 256, 0, (cudaStream_t)stream>>>(w, g, m1, m2, count, lr, b1, b2,
                                                               eps, c1, c2);
  MLP_CK();
  return ESPEC_OK;
}

extern "C" int espec_mlp_adam_dev(float* w, const float* g, float* m1, float* m2, long count,
                                  const float* hyper, float b1, float b2, float eps,
                                  void* stream) {
  adam_dev_kernel<<<blocks(count), 256, 0, (cudaStream_t)stream>>>(w, g, m1, m2, count, hyper, b1,
                                                                   b2, eps);
  MLP_CK();
  return ESPEC_OK;
}

extern "C" int espec_outer_basis(const double* phi, int nbx, int nx, const double* chi, int nby,
                                 int ny, double* B, void* stream) {
  const long count = (long)nx * ny * nbx * nby;
  outer_basis_kernel<<<blocks(count), 256, 0, (cudaStream_t)stream>>>(phi, nbx, nx, chi, nby, ny,
                                                                      B);
  MLP_CK();
  return ESPEC_OK;
}

extern "C" int espec_convert(const void* src, void* dst, long count, int to_f32, double scale,
                             void* stream) {
  if (to_f32)
    f64_to_f32_kernel<<<blocks(count), 256, 0, (cudaStream_t)stream>>>(
        (const double*)src, (float*)dst, count, scale);
  else
    f32_to_f64_kernel<<<blocks(count), 256, 0, (cudaStream_t)stream>>>(
        (const float*)src, (double*)dst, count, scale);
  MLP_CK();
  return ESPEC_OK;
}
