// mlp_tc.cu -- the warm-start network's products on the 5th-generation tensor
// cores, and the element-wise kernels of its BF16 training step.
//
// The network (5 potential parameters -> 3 x 256 GELU -> coefficients of the
// four lowest eigenvectors) keeps FP32 master weights and trains with BF16
// copies of weights, activations and back-propagated gradients as GEMM
// operands; every product accumulates in FP32.
//
// GEMM: C[M,N] (f32) = alpha op(A) op(B) + beta C, A and B bfloat16.  One CTA
// of 128 threads owns a 128 x BN output tile whose FP32 accumulator lives in
// tensor memory (TMEM lane = tile row, column = tile column).  K advances in
// stages of 64: all threads stage the A and B tiles in shared memory as
// "core matrices" (8 x 16 bytes, no swizzle; K-major or MN-major, whichever
// keeps the source's 16-byte runs whole) with vector loads, one thread
// issues four tcgen05.mma (M = 128, N = BN, K = 16, kind::f16 with BF16
// inputs) and commits them to an mbarrier; the next stage is staged into the
// other buffer while they run.  The epilogue reads the accumulator with
// tcgen05.ld (one warp per 32 TMEM lanes).  Every mbarrier wait is bounded:
// on timeout the kernel records it in a device status word, skips the
// epilogue and still releases its TMEM.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "espec_gpu.h"
#include "espec_internal.h"

namespace espec {
namespace {

constexpr int kBM = 128;         // tile rows = TMEM lanes
constexpr int kBK = 64;          // k per stage: four MMAs of k = 16
constexpr int kTcThreads = 128;  // four warps, one per 32 TMEM lanes
constexpr long kWaitLimit = 1L << 22;

__device__ int g_tc_status;  // non-zero: a bounded wait gave up (sticky until read)

struct TcGemm {
  int M, N, K;
  float alpha, beta;
  const uint16_t* A;
  int lda, ta;
  const uint16_t* B;
  int ldb, tb;
  float* C;
  int ldc;
  int a_vec, b_vec;  // 16-byte loads allowed: ld % 8 == 0 and a 16-byte aligned base
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor of a K-major, no-swizzle operand: start
// address, leading byte offset (between the two 8-element k chunks of one
// MMA), stride byte offset (between 8-row groups), descriptor version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) |
         ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulator, BF16 A and B, A / B K-major (0)
// or MN-major (1) at bits 15 / 16, N >> 3 at bit 17, M >> 4 at bit 24
template <int BN>
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t a_mn, uint32_t b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn << 15) | (b_mn << 16) |
         ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(kBM >> 4) << 24);
}

__device__ __forceinline__ uint32_t pack2(uint16_t lo, uint16_t hi) {
  return (uint32_t)lo | ((uint32_t)hi << 16);
}

// Operand tile of R rows (M or N) x 64 k as 8 x 8 core matrices of 16-byte
// rows: core matrix (row group g, k group q) at q * 16 R + g * 128 bytes, so
// that one descriptor serves both forms (stride byte offset 128 between row
// groups, leading byte offset 16 R between k groups).
//  * kcontig source (element (row, k) at X[row ld + k]): K-major core
//    matrices, 16-byte row = 8 consecutive k of one row;
//  * otherwise (element at X[k ld + row]): MN-major core matrices, 16-byte
//    row = 8 consecutive rows at one k.
// Either way a 16-byte row is 16 contiguous source bytes, loaded as one
// vector when vec (aligned, in bounds) and element by element at the edges
// (rows >= nrows, k >= K read as zero).  Consecutive threads take
// consecutive 16-byte pieces of the source.
template <int R>
__device__ __forceinline__ void stage_tile(uint8_t* dst, const uint16_t* X, int ld, bool kcontig,
                                           bool vec, int row0, int nrows, int k0, int K) {
  constexpr int kIter = R * (kBK / 8) / kTcThreads;  // 16-byte pieces per thread
  uint4 v[kIter];
  int off[kIter];
  // all loads first (independent, in flight together), then the stores
#pragma unroll
  for (int i = 0; i < kIter; ++i) {
    const int it = threadIdx.x + i * kTcThreads;
    if (kcontig) {
      const int r = it / (kBK / 8), q = it % (kBK / 8);
      const int row = row0 + r, kb = k0 + 8 * q;
      off[i] = q * (R * 16) + (r >> 3) * 128 + (r & 7) * 16;
      if (vec && row < nrows && kb + 8 <= K) {
        v[i] = __ldg(reinterpret_cast<const uint4*>(X + (long)row * ld + kb));
      } else {
        uint16_t e[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
          e[j] = (row < nrows && kb + j < K) ? X[(long)row * ld + kb + j] : (uint16_t)0;
        v[i] = make_uint4(pack2(e[0], e[1]), pack2(e[2], e[3]), pack2(e[4], e[5]),
                          pack2(e[6], e[7]));
      }
    } else {
      const int g = it % (R / 8), k = it / (R / 8);
      const int kk = k0 + k, m = row0 + 8 * g;
      off[i] = (k >> 3) * (R * 16) + g * 128 + (k & 7) * 16;
      if (vec && kk < K && m + 8 <= nrows) {
        v[i] = __ldg(reinterpret_cast<const uint4*>(X + (long)kk * ld + m));
      } else {
        uint16_t e[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
          e[j] = (kk < K && m + j < nrows) ? X[(long)kk * ld + m + j] : (uint16_t)0;
        v[i] = make_uint4(pack2(e[0], e[1]), pack2(e[2], e[3]), pack2(e[4], e[5]),
                          pack2(e[6], e[7]));
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kIter; ++i) *reinterpret_cast<uint4*>(dst + off[i]) = v[i];
}

// bounded wait for the completion of the mbarrier phase with this parity
__device__ __forceinline__ bool wait_phase(uint64_t* bar, uint32_t parity,
                                           long limit = kWaitLimit) {
  const uint32_t a = smem_u32(bar);
  for (long i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (i > 64) __nanosleep(64);
  }
  atomicExch(&g_tc_status, 1);
  return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

template <int BN>
constexpr size_t tc_smem_bytes() {
  return 1024 + 2 * (size_t)(kBM + BN) * kBK * 2 + 64;
}

template <int BN>
__global__ void __launch_bounds__(kTcThreads) gemm_bf16_tc(TcGemm g) {
  static_assert(BN == 128 || BN == 256, "TMEM columns: a power of two, N tile of one MMA");
  constexpr int kA = kBM * kBK * 2, kB = BN * kBK * 2;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sA[2] = {base, base + kA};
  uint8_t* sB[2] = {base + 2 * kA, base + 2 * kA + kB};
  uint64_t* bar = (uint64_t*)(base + 2 * (kA + kB));
  uint32_t* tmem_slot = (uint32_t*)(bar + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN;
  const bool a_kc = !g.ta, b_kc = g.tb != 0;

  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar + 1)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  stage_tile<kBM>(sA[0], g.A, g.lda, a_kc, g.a_vec, m0, g.M, 0, g.K);
  stage_tile<BN>(sB[0], g.B, g.ldb, b_kc, g.b_vec, n0, g.N, 0, g.K);
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const int nk = (g.K + kBK - 1) / kBK;
  const uint32_t idesc = idesc_bf16<BN>(a_kc ? 0u : 1u, b_kc ? 0u : 1u);
  bool ok = true;
  for (int kt = 0; kt < nk; ++kt) {
    const int b = kt & 1;
    if (threadIdx.x == 0) {
      const uint32_t a0 = smem_u32(sA[b]), b0 = smem_u32(sB[b]);
#pragma unroll
      for (int j = 0; j < kBK / 16; ++j) {
        const uint64_t da = smem_desc(a0 + j * 2 * (kBM * 16), kBM * 16, 128);
        const uint64_t db = smem_desc(b0 + j * 2 * (BN * 16), BN * 16, 128);
        const uint32_t acc = (kt > 0 || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
              smem_u32(bar + b))
          : "memory");
    }
    if (kt + 1 < nk) {
      // the other buffer was read by the MMAs of stage kt - 1
      if (kt >= 1) ok = wait_phase(bar + (b ^ 1), ((kt - 1) >> 1) & 1) && ok;
      stage_tile<kBM>(sA[b ^ 1], g.A, g.lda, a_kc, g.a_vec, m0, g.M, (kt + 1) * kBK, g.K);
      stage_tile<BN>(sB[b ^ 1], g.B, g.ldb, b_kc, g.b_vec, n0, g.N, (kt + 1) * kBK, g.K);
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    }
  }
  // the last two commits (every earlier one was waited for above)
  if (nk >= 2) ok = wait_phase(bar + ((nk - 2) & 1), ((nk - 2) >> 1) & 1) && ok;
  if (nk >= 1) ok = wait_phase(bar + ((nk - 1) & 1), ((nk - 1) >> 1) & 1) && ok;
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  ok = __syncthreads_and(ok) != 0;
  if (ok && nk >= 1) {
    const int row = m0 + warp * 32 + lane;
    float* crow = g.C + (long)row * g.ldc;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t r[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
      if (row < g.M) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int n = n0 + c0 + j;
          if (n < g.N) {
            float v = g.alpha * __uint_as_float(r[j]);
            if (g.beta != 0.0f) v = fmaf(g.beta, crow[n], v);
            crow[n] = v;
          }
        }
      }
    }
  } else if (nk == 0) {  // empty sum: C = beta C
    for (int e = threadIdx.x; e < kBM * BN; e += kTcThreads) {
      const int row = m0 + e / BN, n = n0 + e % BN;
      if (row < g.M && n < g.N) {
        float* c = g.C + (long)row * g.ldc + n;
        *c = g.beta == 0.0f ? 0.0f : g.beta * *c;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(BN));
}

__device__ __forceinline__ uint16_t bf16_bits(float v) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}

// GELU(z) = z Phi(z), Phi the standard normal distribution function
__device__ __forceinline__ float gelu(float z) {
  return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
         z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// z += b (row broadcast); h = bf16(gelu(z)) when act, else bf16(z) (h optional)
__global__ void bias_gelu_kernel(float* z, const float* b, int rows, int cols, int act,
                                 uint16_t* h) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)rows * cols) return;
  const float v = z[i] + b[i % cols];
  z[i] = v;
  if (h) h[i] = bf16_bits(act ? gelu(v) : v);
}

// dh <- dh gelu'(z); dzb = bf16(dh)
__global__ void gelu_back_kernel(float* dh, const float* z, long count, uint16_t* dzb) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float d = dh[i] * gelu_grad(z[i]);
  dh[i] = d;
  dzb[i] = bf16_bits(d);
}

__global__ void to_bf16_kernel(const float* x, uint16_t* y, long count) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) y[i] = bf16_bits(x[i]);
}

// Adam on the FP32 master weights, (lr, 1 - b1^t, 1 - b2^t) from device memory,
// and the BF16 copy the products use
__global__ void adam_bf16_kernel(float* w, const float* g, float* m1, float* m2, long count,
                                 const float* hyper, float b1, float b2, float eps, uint16_t* wb) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float lr = hyper[0], c1 = hyper[1], c2 = hyper[2];
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  const float nw = w[i] - lr * (a / c1) / (sqrtf(b / c2) + eps);
  w[i] = nw;
  if (wb) wb[i] = bf16_bits(nw);
}

inline unsigned nblk(long count) { return (unsigned)((count + 255) / 256); }

template <int BN>
int launch_tc(const TcGemm& g, cudaStream_t st) {
  static DeviceFlags attr;
  {
    const cudaError_t e = set_max_smem_once(attr, gemm_bf16_tc<BN>, tc_smem_bytes<BN>());
    if (e != cudaSuccess) return set_cuda_error("cudaFuncSetAttribute", e);
  }
  dim3 grid((g.N + BN - 1) / BN, (g.M + kBM - 1) / kBM);
  gemm_bf16_tc<BN><<<grid, kTcThreads, tc_smem_bytes<BN>(), st>>>(g);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error("tensor-core GEMM launch", e);
  return ESPEC_OK;
}

}  // namespace
}  // namespace espec

using namespace espec;

#define TC_CK()                                                                \
  do {                                                                         \
    cudaError_t e_ = cudaGetLastError();                                       \
    if (e_ != cudaSuccess) return set_cuda_error("mlp bf16 kernel launch", e_); \
  } while (0)

extern "C" int espec_gemm_bf16(int M, int N, int K, float alpha, const void* A, int lda, int ta,
                               const void* B, int ldb, int tb, float beta, float* C, int ldc,
                               void* stream) {
  if (M <= 0 || N <= 0 || K < 0 || !C || (K > 0 && (!A || !B)))
    return set_error(ESPEC_EINVAL, "bad GEMM");
  if (lda < (ta ? M : K) || ldb < (tb ? K : N) || ldc < N)
    return set_error(ESPEC_EINVAL, "leading dimension smaller than the row length");
  auto vec_ok = [](const void* p, int ld) { return ld % 8 == 0 && ((uintptr_t)p & 15) == 0; };
  TcGemm g{M, N, K, alpha, beta, (const uint16_t*)A, lda, ta ? 1 : 0, (const uint16_t*)B, ldb,
           tb ? 1 : 0, C, ldc, vec_ok(A, lda) ? 1 : 0, vec_ok(B, ldb) ? 1 : 0};
  // N tiles of 256 only when that still gives a CTA per SM
  const long tiles256 = (long)((N + 255) / 256) * ((M + kBM - 1) / kBM);
  return (N > 128 && tiles256 >= 148) ? launch_tc<256>(g, (cudaStream_t)stream)
                                      : launch_tc<128>(g, (cudaStream_t)stream);
}

namespace espec {
namespace {
// One thread waits, with the GEMM's bounded wait, on an mbarrier that nothing
// arrives on and no copy or MMA is attached to: the wait must give up after
// `polls` polls and set the status word.  The barrier is invalidated before
// the CTA exits.
__global__ void mbar_timeout_probe(long polls, int* gave_up) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    const bool ok = wait_phase(&bar, 0u, polls);
    *gave_up = ok ? 0 : 1;
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(&bar)) : "memory");
  }
}
}  // namespace
}  // namespace espec

extern "C" int espec_selftest_mbar_wait(long polls, int* gave_up) {
  if (polls < 1 || !gave_up) return set_error(ESPEC_EINVAL, "polls must be positive");
  int* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(int));
  if (e != cudaSuccess) return set_cuda_error("cudaMalloc", e);
  mbar_timeout_probe<<<1, 32>>>(polls, d);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(gave_up, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return set_cuda_error("mbarrier wait self-test", e);
  return ESPEC_OK;
}

extern "C" int espec_gemm_bf16_status(int* timed_out) {
  if (!timed_out) return set_error(ESPEC_EINVAL, "null argument");
  int v = 0, zero = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_tc_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_tc_status, &zero, sizeof(int));
  if (e != cudaSuccess) return set_cuda_error("tensor-core GEMM status", e);
  *timed_out = v;
  return ESPEC_OK;
}

extern "C" int espec_mlp_bias_gelu(float* z, const float* b, int rows, int cols, int act,
                                   void* h_bf16, void* stream) {
  bias_gelu_kernel<<<nblk((long)rows * cols), 256, 0, (cudaStream_t)stream>>>(
      z, b, rows, cols, act, (uint16_t*)h_bf16);
  TC_CK();
  return ESPEC_OK;
}

extern "C" int espec_mlp_gelu_back(float* dh, const float* z, long count, void* dz_bf16,
                                   void* stream) {
  gelu_back_kernel<<<nblk(count), 256, 0, (cudaStream_t)stream>>>(dh, z, count,
                                                                   (uint16_t*)dz_bf16);
  TC_CK();
  return ESPEC_OK;
}

extern "C" int espec_to_bf16(const float* x, void* y, long count, void* stream) {
  to_bf16_kernel<<<nblk(count), 256, 0, (cudaStream_t)stream>>>(x, (uint16_t*)y, count);
  TC_CK();
  return ESPEC_OK;
}

extern "C" int espec_mlp_adam_bf16(float* w, const float* g, float* m1, float* m2, long count,
                                   const float* hyper, float b1, float b2, float eps, void* w_bf16,
                                   void* stream) {
  adam_bf16_kernel<<<nblk(count), 256, 0, (cudaStream_t)stream>>>(w, g, m1, m2, count, hyper, b1,
                                                                  b2, eps, (uint16_t*)w_bf16);
  TC_CK();
  return ESPEC_OK;
}
