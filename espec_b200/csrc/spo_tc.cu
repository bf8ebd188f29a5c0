// spo_tc.cu -- 256-point split-operator packets with the FFT as dense DFT
// GEMMs on the 5th-generation tensor cores (mixed form: FP32 state, lifting
// phases; no counterpart in the reference, whose FFT is Singleton's fft3d.f
// called from spofft.f:142-160).
//
// Four-step transform of N = 256 = 16 x 16 points, n = n1 + 16 n2 and
// k = k1 + 16 k2 (forward sign +, as fft3d.f with ISN = +1):
//   stage A: Y[n1, k1]  = sum_n2 x[n1 + 16 n2] W16^(n2 k1)     (GEMM)
//   twiddle: Y[n1, k1] *= W256^(n1 k1)                          (lifting rotation)
//   stage B: X[k1 + 16 k2] = sum_n1 Y[n1, k1] W16^(n1 k2)      (GEMM)
// One CTA of 128 threads propagates 8 packets for the whole time loop: row
// r = 16 p + s of every GEMM is packet p's line s, its 16 complex values
// the 32 K (or N) entries (real parts, then imaginary parts) -- M = 128,
// N = 32, K = 32 per stage, the 32 x 32 real form of the 16-point DFT as B.
// Thread r keeps its line in registers; the line of stage A (rows n1) and of
// stage B (rows k1) are transposes of each other, exchanged through shared
// memory once per transform.  The inverse transform runs stages B and A with
// the conjugate matrix in reverse; the kinetic phase sits between the two
// transforms on thread (p, k1)'s frequencies k1 + 16 k2.
//
// Precision: fixed-point slices, so that the tensor cores add exactly.  Each
// row of data is scaled by a power of two 2^-e to |y| < 1 and cut into three
// BF16 slices y = a0 + a1 + a2 + r, a_i an integer multiple of 2^-8(i+1)
// (|a0| <= 1, |a1| <= 2^-9, |a2| <= 2^-17, each slice rounded to nearest, the
// residual |r| <= 2^-25 unbiased); the DFT matrix, |b| <= 1, is cut the same
// way into four slices b0..b3 (32 bits: the forward and inverse matrices are
// each other's inverse to 2^-33, so no fixed per-step bias remains).  The
// products of order i + j = 0, 1, 2, 3 accumulate in four separate TMEM
// accumulators: within one order every term is a multiple of 2^-8(i+j+2) and
// the 32-term sums span at most 23 bits, so each accumulator holds its exact
// sum whatever rounding the tensor cores' FP32 adders use (truncating adders
// left a bias of ~1e-7 per step in C(t) when all orders shared one
// accumulator).  The row is then P0 + (P1 + (P2 + P3)), rounded to nearest,
// times 2^e.  Nine products, 18 tcgen05.mma (kind::f16, M = 128, N = 32,
// K = 16) per stage, issued by one thread and committed to an mbarrier whose
// waits are bounded; the accumulators are read back with tcgen05.ld (warp w:
// TMEM lanes 32w .. 32w + 31).  Operand tiles are "core matrices" of 8 rows x
// 16 bytes without swizzle, K-major, the layout the warm-start GEMM
// (mlp_tc.cu) uses.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cfloat>

#include "espec_gpu.h"
#include "espec_internal.h"
#include "spo1d.cuh"

namespace espec {
namespace {

constexpr int kN = 256;          // points per packet
constexpr int kL = 16;           // line length (and number of lines) of a packet
constexpr int kRows = 128;       // GEMM rows = threads = 8 packets x 16 lines
constexpr int kPk = kRows / kL;  // packets per CTA
constexpr int kK = 32;           // real K (and N) of one stage
constexpr int kAcc = 4;          // accumulators: product orders 0..3
constexpr int kASl = 3;          // slices of a data row
constexpr int kBSl = 4;          // slices of the DFT matrix
constexpr int kTmemCols = kAcc * 32;
static_assert(kTmemCols == 128, "TMEM allocations are powers of two >= 32 columns");
constexpr long kTcWaitLimit = 1L << 22;
constexpr int kStage = 33;       // staging row stride in floats (conflict-free columns)

// shared-memory layout (bytes from a 1024-aligned base)
constexpr int kATile = kRows * kK * 2;             // one BF16 split of the A tile: 8 KB
constexpr int kBTile = kK * kK * 2;                // one BF16 split of a DFT matrix: 2 KB
constexpr int kOffA = 0;                           // kASl slices
constexpr int kOffB = kOffA + kASl * kATile;       // 2 directions x kBSl slices
constexpr int kOffStage = kOffB + 2 * kBSl * kBTile;  // 128 x 33 floats
constexpr int kOffBar = kOffStage + kRows * kStage * 4;
constexpr int kSmemBytes = 1024 + kOffBar + 64;

__device__ int g_tc_spo_status;  // non-zero: a bounded wait gave up (sticky until read)

__device__ __forceinline__ uint32_t su32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (row, k) of a K-major tile of R rows
template <int R>
__device__ __forceinline__ int core_off(int row, int k) {
  return (k >> 3) * (16 * R) + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) |
         ((uint64_t)(sbo >> 4) << 32) | (1ull << 46);
}

// FP32 accumulator, BF16 A and B (both K-major), N = 32, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kK >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);

__device__ __forceinline__ uint16_t bf16_bits(float v) {  // v exact in BF16
  return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}

// y (|y| < 1) = a0 + a1 + a2 + r: a_i = round(y_i 2^(8i+8)) 2^-(8i+8) of the
// remainder y_i, an integer of at most 8 bits times a power of two (exact in
// BF16); every difference is exact in FP32
__device__ __forceinline__ void slice3(float y, uint16_t& h, uint16_t& m, uint16_t& l) {
  const float a0 = rintf(y * 256.0f) * (1.0f / 256.0f);
  const float r1 = y - a0;
  const float a1 = rintf(r1 * 65536.0f) * (1.0f / 65536.0f);
  const float r2 = r1 - a1;
  const float a2 = rintf(r2 * 16777216.0f) * (1.0f / 16777216.0f);
  h = bf16_bits(a0);
  m = bf16_bits(a1);
  l = bf16_bits(a2);
}

__device__ __forceinline__ uint32_t pk2(uint16_t a, uint16_t b) {
  return (uint32_t)a | ((uint32_t)b << 16);
}

// row r of the A tile (three slices) from its 16 complex values; returns
// the row's scale 2^e (the GEMM's output row is scaled back by it)
__device__ __forceinline__ float write_row(uint8_t* a, int r, const cpx<float>* v) {
  float mx = 0.0f;
#pragma unroll
  for (int j = 0; j < kL; ++j) mx = fmaxf(mx, fmaxf(fabsf(v[j].x), fabsf(v[j].y)));
  // mx 2^-e in [0.5, 1) for a normal mx (clamped to keep 2^e and 2^-e normal)
  int e = 0;
  if (mx > 0.0f && mx <= FLT_MAX) e = max(-126, min(126, ((__float_as_int(mx) >> 23) & 0xff) - 126));
  const float down = __int_as_float((127 - e) << 23);
#pragma unroll
  for (int q = 0; q < 4; ++q) {  // k group: 8 consecutive K entries
    uint16_t h[8], m[8], l[8];
#pragma unroll
    for (int e8 = 0; e8 < 8; ++e8) {
      const int k = 8 * q + e8;
      const float x = k < kL ? v[k].x : v[k - kL].y;
      slice3(x * down, h[e8], m[e8], l[e8]);
    }
    const int off = core_off<kRows>(r, 8 * q);
    *reinterpret_cast<uint4*>(a + off) =
        make_uint4(pk2(h[0], h[1]), pk2(h[2], h[3]), pk2(h[4], h[5]), pk2(h[6], h[7]));
    *reinterpret_cast<uint4*>(a + kATile + off) =
        make_uint4(pk2(m[0], m[1]), pk2(m[2], m[3]), pk2(m[4], m[5]), pk2(m[6], m[7]));
    *reinterpret_cast<uint4*>(a + 2 * kATile + off) =
        make_uint4(pk2(l[0], l[1]), pk2(l[2], l[3]), pk2(l[4], l[5]), pk2(l[6], l[7]));
  }
  return __int_as_float((127 + e) << 23);
}

__device__ __forceinline__ bool wait_parity(uint64_t* bar, uint32_t parity) {
  const uint32_t a = su32(bar);
  for (long i = 0; i < kTcWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (i > 64) __nanosleep(32);
  }
  atomicExch(&g_tc_spo_status, 1);
  return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&f)[32]) {
  uint32_t r[32];
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
#pragma unroll
  for (int j = 0; j < 32; ++j) f[j] = __uint_as_float(r[j]);
}

struct TcCta {
  uint8_t* a;       // A tile, 3 splits
  uint8_t* b;       // B tiles [dir][split]
  float* stage;     // transpose staging
  uint64_t* bar;
  uint32_t tmem;
  uint32_t phase;   // parity of the next mbarrier completion
  bool ok;

  // the A tile written by every thread -> 18 MMAs (dir 0 forward, 1 inverse)
  // into the four order accumulators -> this thread's row, P0 + (P1 + (P2 +
  // P3)) times the row's scale
  __device__ __forceinline__ void gemm(int dir, float (&d)[32], float scale) {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (threadIdx.x == 0 && ok) {
      const uint32_t a0 = su32(a), b0 = su32(b + dir * kBSl * kBTile);
      // (A slice, B slice) of the nine products kept, by order i + j; the
      // first product of an order starts its accumulator
      constexpr int pa[9] = {0, 1, 0, 2, 1, 0, 2, 1, 0};
      constexpr int pb[9] = {0, 0, 1, 0, 1, 2, 1, 2, 3};
#pragma unroll
      for (int q = 0; q < 9; ++q)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int ord = pa[q] + pb[q];
          const bool first = (q == 0 || pa[q - 1] + pb[q - 1] != ord) && j == 0;
          const uint64_t da = sdesc(a0 + pa[q] * kATile + j * 2 * (kRows * 16), kRows * 16, 128);
          const uint64_t db = sdesc(b0 + pb[q] * kBTile + j * 2 * (kK * 16), kK * 16, 128);
          const uint32_t acc = first ? 0u : 1u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
                  tmem + (uint32_t)(ord * 32)),
              "l"(da), "l"(db), "r"(kIdesc), "r"(acc));
        }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
              su32(bar))
          : "memory");
    }
    if (ok) {
      ok = wait_parity(bar, phase) && ok;
      phase ^= 1u;
    }
    ok = __syncthreads_and(ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const int w = threadIdx.x >> 5;
    if (ok) {
      const uint32_t lane = tmem + ((uint32_t)(w * 32) << 16);
      float e[32];
      tmem_ld32(lane + 96, d);
      tmem_ld32(lane + 64, e);
#pragma unroll
      for (int j = 0; j < 32; ++j) d[j] = __fadd_rn(e[j], d[j]);
      tmem_ld32(lane + 32, e);
#pragma unroll
      for (int j = 0; j < 32; ++j) d[j] = __fadd_rn(e[j], d[j]);
      tmem_ld32(lane, e);
#pragma unroll
      for (int j = 0; j < 32; ++j) d[j] = __fmul_rn(__fadd_rn(e[j], d[j]), scale);
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) d[j] = 0.0f;
    }
  }

  // out[c] = this thread's column of the 16 lines of its packet
  __device__ __forceinline__ void transpose(const cpx<float>* in, cpx<float>* out) {
    const int t = threadIdx.x, p = t >> 4, s = t & 15;
    __syncthreads();  // the staging rows of the last transpose have been read
#pragma unroll
    for (int c = 0; c < kL; ++c) {
      stage[t * kStage + c] = in[c].x;
      stage[t * kStage + kL + c] = in[c].y;
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kL; ++c) {
      const float* row = stage + (kL * p + c) * kStage;
      out[c] = mk(row[s], row[kL + s]);
    }
  }
};

// The 32 x 32 real form of the 16-point DFT in K-major BF16 slices (four,
// cut from the FP64 value): B[n][k] (row = output index N, column = input
// index K); dir 1 conjugate.
__device__ void build_dft_tiles(uint8_t* b) {
  for (int e = threadIdx.x; e < 2 * kK * kK; e += blockDim.x) {
    const int dir = e / (kK * kK), nn = (e / kK) % kK, kk = e % kK;
    const int kout = nn % kL, kin = kk % kL;
    double s, c;
    sincospi(2.0 * (double)((kout * kin) % kL) / kL, &s, &c);
    if (dir) s = -s;
    // out re = in re c - in im s ; out im = in re s + in im c
    double v;
    if (nn < kL) v = kk < kL ? c : -s;
    else v = kk < kL ? s : c;
    uint8_t* base = b + dir * kBSl * kBTile;
    const int off = core_off<kK>(nn, kk);
    double r = v, sc = 256.0;
#pragma unroll
    for (int i = 0; i < kBSl; ++i, sc *= 256.0) {
      const double bi = rint(r * sc) / sc;  // an integer of <= 8 bits times 2^-(8i+8)
      r -= bi;
      *reinterpret_cast<uint16_t*>(base + i * kBTile + off) = bf16_bits((float)bi);
    }
  }
}

__global__ void __launch_bounds__(kRows, 1) spo_tc256_kernel(SpoArgs<float> a, int npk) {
  using TB = Tab<float>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  TcCta cta;
  cta.a = base + kOffA;
  cta.b = base + kOffB;
  cta.stage = reinterpret_cast<float*>(base + kOffStage);
  cta.bar = reinterpret_cast<uint64_t*>(base + kOffBar);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(base + kOffBar + 8);
  cta.phase = 0;
  cta.ok = true;

  const int t = threadIdx.x, w = t >> 5, p = t >> 4, s = t & 15;
  const int pk_index = blockIdx.x * kPk + p;
  const bool live = pk_index < npk;
  const SpoPacket pk = a.pk[live ? pk_index : 0];
  const int base_pt = pk.off;
  double2* cout = a.c_out + pk.c_off;

  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(su32(cta.bar)));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     su32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  build_dft_tiles(cta.b);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  cta.tmem = *tmem_slot;

  // this thread's tables: x-space slot j is point s + 16 j, k-space slot j
  // (thread s = k1) is frequency s + 16 j, stored at final position 16 s + j
  RotF tw[kL];  // W256^(s c), forward sign
#pragma unroll
  for (int c = 0; c < kL; ++c) tw[c] = make_rotf(6.283185307179586476925287 * (double)(s * c) / kN);
  // The per-point tables stay in global memory and are read every step
  // (a CTA's 2048 points x 32 B stay in L1); registers hold the state and the
  // twiddles.  Rows of absent packets (the last CTA) read packet 0's tables
  // and propagate zeros.
  const int xb = base_pt + s;             // x-space slot j: point xb + 16 j
  const int kb = base_pt + kL * s;        // k-space slot j: final position kb + j
  cpx<float> v[kL];
  double c0r = 0.0;
#pragma unroll
  for (int j = 0; j < kL; ++j) {
    const double2 p0 = live ? (a.psi_start ? a.psi_start[xb + kL * j] : a.psi0[xb + kL * j])
                            : make_double2(0.0, 0.0);
    c0r += p0.x * p0.x + p0.y * p0.y;
    v[j] = mk((float)p0.x, (float)p0.y);
  }
  // C(0) = <psi0|psi0> over the packet's 16 threads (a resumed run writes no C(0))
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) c0r += __shfl_xor_sync(0xffffffffu, c0r, o);
  if (live && s == 0 && !a.psi_start) cout[0] = make_double2(c0r, 0.0);

  bool finite = true;
  for (int step = 1; step <= a.nsteps; ++step) {
    // x-space phase (h at the first step, then the merged g)
    {
      const TB::phase_t* ph = step == 1 ? a.tab.h : a.tab.g;
#pragma unroll
      for (int j = 0; j < kL; ++j) v[j] = TB::apply(ph[xb + kL * j], v[j]);
    }
    float d[32];
    cpx<float> y[kL];
    // forward stage A: lines s over n2 -> Y[n1 = s][k1 = c]
    cta.gemm(0, d, write_row(cta.a, t, v));
#pragma unroll
    for (int c = 0; c < kL; ++c) y[c] = rot<false>(tw[c], mk(d[c], d[kL + c]));
    cta.transpose(y, v);  // thread (p, k1 = s): Y[n1 = c][k1]
    // forward stage B: -> X[k1 + 16 k2], k2 = c; kinetic phase
    cta.gemm(0, d, write_row(cta.a, t, v));
#pragma unroll
    for (int c = 0; c < kL; ++c) v[c] = TB::apply(a.tab.k[kb + c], mk(d[c], d[kL + c]));
    // inverse stage B: -> Y[n1 = c][k1 = s], conjugate twiddle
    cta.gemm(1, d, write_row(cta.a, t, v));
#pragma unroll
    for (int c = 0; c < kL; ++c) y[c] = rot<true>(tw[c], mk(d[c], d[kL + c]));
    cta.transpose(y, v);  // thread (p, n1 = s): Y[n1][k1 = c]
    // inverse stage A: -> x[s + 16 n2], n2 = c
    cta.gemm(1, d, write_row(cta.a, t, v));
#pragma unroll
    for (int c = 0; c < kL; ++c) v[c] = mk(d[c], d[kL + c]);
    // C(t) = sum w x: FP32 products per thread, FP64 over the packet's threads
    float pr = 0.0f, pi = 0.0f;
#pragma unroll
    for (int j = 0; j < kL; ++j) {
      const TB::weight_t wj = a.tab.w[xb + kL * j];
      pr = fmaf(wj.x, v[j].x, fmaf(-wj.y, v[j].y, pr));
      pi = fmaf(wj.x, v[j].y, fmaf(wj.y, v[j].x, pi));
    }
    double cr = pr, ci = pi;
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      cr += __shfl_xor_sync(0xffffffffu, cr, o);
      ci += __shfl_xor_sync(0xffffffffu, ci, o);
    }
    if (live && s == 0) {
      finite = finite && isfinite(cr) && isfinite(ci);
      cout[step] = make_double2(cr, ci);
    }
    if (!cta.ok) break;
  }
  if (live && s == 0 && !finite && a.nonfinite) atomicAdd(a.nonfinite, 1);
  if (live && a.psi_out && cta.ok) {
#pragma unroll
    for (int j = 0; j < kL; ++j) {
      const int x = xb + kL * j;
      const cpx<float> o = a.nsteps > 0 ? TB::apply(a.tab.hm[x], v[j]) : v[j];
      a.psi_out[x] = make_double2((double)o.x, (double)o.y);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (w == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(cta.tmem),
                 "r"(kTmemCols));
}

}  // namespace

// final-layout frequency of position f = 16 s + j: s + 16 j
void spo_tc256_final_freq(int* kap) {
  for (int f = 0; f < kN; ++f) kap[f] = (f >> 4) + kL * (f & 15);
}

cudaError_t spo_tc256_launch(const SpoArgs<float>& a, int npk, cudaStream_t st) {
  static DeviceFlags attr;
  cudaError_t e = set_max_smem_once(attr, spo_tc256_kernel, kSmemBytes);
  if (e != cudaSuccess) return e;
  const int grid = (npk + kPk - 1) / kPk;
  if (grid < 1) return cudaSuccess;
  spo_tc256_kernel<<<grid, kRows, kSmemBytes, st>>>(a, npk);
  return cudaGetLastError();
}

int spo_tc_status(int* timed_out) {
  int v = 0, zero = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_tc_spo_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_tc_spo_status, &zero, sizeof(int));
  if (e != cudaSuccess) return set_cuda_error("tensor-core split-operator status", e);
  *timed_out = v;
  return ESPEC_OK;
}

}  // namespace espec
