// mlp.cu -- dense products and loss kernels of the learned warm start for the
// eigensolver: FP64/FP32 GEMMs that move eigenvectors in and out of the
// network's output basis (projection onto and expansion in a product basis
// phi_a(x) chi_b(y), separable), the mean-squared-error loss and the
// bias-gradient column sums.  The network's own products run on the tensor
// cores (mlp_tc.cu).  The GEMMs are tiled SIMT kernels: one 64 x 64 output
// tile per 256-thread CTA, 16-deep k tiles staged in shared memory, 4 x 4
// outputs per thread.
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

// db[c] = sum_r dy[r, c]: 32 columns x 8 row phases per CTA, each phase sums
// rows r = phase mod 8 in order, then the 8 partials are added in order
// (deterministic)
__global__ void colsum_kernel(const float* dy, int rows, int cols, float* db) {
  __shared__ float part[8][33];
  const int c = blockIdx.x * 32 + threadIdx.x;
  float s = 0.0f;
  if (c < cols)
    for (int r = threadIdx.y; r < rows; r += 8) s += dy[(long)r * cols + c];
  part[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && c < cols) {
    float t = 0.0f;
#pragma unroll
    for (int p = 0; p < 8; ++p) t += part[p][threadIdx.x];
    db[c] = t;
  }
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

// separable basis transform of one 2D vector per CTA (x fastest in psi,
// coefficient index a nb + b for phi_a(x) chi_b(y)); shared memory holds
// phi^T [nx][nb], chi^T [ny][nb] and the half-transformed [ny][nb] block.
// project: c = scale sum_{x,y} phi_a(x) chi_b(y) psi(x, y)  (psi f64 -> c f32)
// expand:  psi(x, y) = scale sum_{a,b} phi_a(x) chi_b(y) c_ab  (c f32 -> psi f64)
constexpr int kSepThreads = 256;

__global__ void __launch_bounds__(kSepThreads) sep_basis_kernel(int dir, int nx, int ny, int nb,
                                                                const float* phi, const float* chi,
                                                                double* psi, float* c,
                                                                float scale) {
  extern __shared__ float sep_sm[];
  float* phiT = sep_sm;           // [nx][nb]
  float* chiT = phiT + nx * nb;   // [ny][nb]
  float* half = chiT + ny * nb;   // [ny][nb]
  const long v = blockIdx.x;
  const long n = (long)nx * ny;
  for (int e = threadIdx.x; e < nx * nb; e += kSepThreads) {
    const int a = e / nx, x = e % nx;
    phiT[x * nb + a] = phi[e];
  }
  for (int e = threadIdx.x; e < ny * nb; e += kSepThreads) {
    const int b = e / ny, y = e % ny;
    chiT[y * nb + b] = chi[e];
  }
  __syncthreads();
  double* pv = psi + v * n;
  float* cv = c + v * (long)nb * nb;
  if (dir == 0) {
    // half[y][a] = sum_x psi(x, y) phi_a(x)
    for (int e = threadIdx.x; e < ny * nb; e += kSepThreads) {
      const int y = e / nb, a = e % nb;
      const double* row = pv + (long)y * nx;
      float s = 0.0f;
      for (int x = 0; x < nx; ++x) s = fmaf((float)row[x], phiT[x * nb + a], s);
      half[e] = s;
    }
    __syncthreads();
    // c[a][b] = sum_y chi_b(y) half[y][a]
    for (int e = threadIdx.x; e < nb * nb; e += kSepThreads) {
      const int a = e / nb, b = e % nb;
      float s = 0.0f;
      for (int y = 0; y < ny; ++y) s = fmaf(chiT[y * nb + b], half[y * nb + a], s);
      cv[e] = scale * s;
    }
  } else {
    // half[y][a] = sum_b chi_b(y) c[a][b]
    for (int e = threadIdx.x; e < ny * nb; e += kSepThreads) {
      const int y = e / nb, a = e % nb;
      const float* ca = cv + (long)a * nb;
      float s = 0.0f;
      for (int b = 0; b < nb; ++b) s = fmaf(chiT[y * nb + b], ca[b], s);
      half[e] = s;
    }
    __syncthreads();
    // psi(x, y) = sum_a phi_a(x) half[y][a]
    for (long e = threadIdx.x; e < n; e += kSepThreads) {
      const int y = (int)(e / nx), x = (int)(e % nx);
      float s = 0.0f;
      for (int a = 0; a < nb; ++a) s = fmaf(phi[(long)a * nx + x], half[y * nb + a], s);
      pv[e] = (double)(scale * s);
    }
  }
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

extern "C" int espec_mlp_colsum(const float* dy, int rows, int cols, float* db, void* stream) {
  colsum_kernel<<<(unsigned)((cols + 31) / 32), dim3(32, 8), 0, (cudaStream_t)stream>>>(dy, rows,
                                                                                       cols, db);
  MLP_CK();
  return ESPEC_OK;
}

extern "C" int espec_mlp_mse(const float* y, const float* t, int rows, int cols, float* dy,
                             float* row_loss, void* stream) {
  mse_kernel<<<rows, 256, 0, (cudaStream_t)stream>>>(y, t, rows, cols, dy, row_loss);
  MLP_CK();
  return ESPEC_OK;
}

extern "C" int espec_sep_basis(int dir, int nvec, int nx, int ny, int nb, const float* phi,
                               const float* chi, double* psi, float* c, float scale,
                               void* stream) {
  if (nvec < 0 || nx < 1 || ny < 1 || nb < 1 || !phi || !chi || !psi || !c)
    return set_error(ESPEC_EINVAL, "bad basis transform");
  const size_t smem = sizeof(float) * (size_t)nb * (nx + 2 * ny);
  if (smem > 200 * 1024) return set_error(ESPEC_EINVAL, "basis tables exceed shared memory");
  if (nvec == 0) return ESPEC_OK;
  cudaError_t e = cudaFuncSetAttribute(sep_basis_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return set_cuda_error("cudaFuncSetAttribute", e);
  sep_basis_kernel<<<nvec, kSepThreads, smem, (cudaStream_t)stream>>>(dir ? 1 : 0, nx, ny, nb,
                                                                     phi, chi, psi, c, scale);
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
