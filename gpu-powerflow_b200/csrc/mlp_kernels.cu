// mlp_kernels.cu -- BF16 training and inference kernels of the warm-start MLP.
//
// The network predicts each scenario's Newton starting point (Va, Vm) from its
// loads.  Its dense layers are GEMM-shaped, so they run on the 5th-generation
// tensor cores:
//
//   k_gemm_bf16   C[M,N] = A[M,K] * B[N,K]^T, A and B bf16 and K-contiguous,
//                 fp32 accumulation in tensor memory.  One CTA computes a
//                 128 x BN tile: a producer thread streams 128 x 64 tiles of
//                 A and BN x 64 tiles of B into shared memory with TMA
//                 (128-byte swizzle, mbarrier ring), an MMA thread issues
//                 tcgen05.mma (M = 128, N = BN, K = 16 per instruction) into
//                 a BN-column TMEM accumulator, and the four warps read the
//                 accumulator back (tcgen05.ld 32x32b) for a fused epilogue.
//                 Three shapes: BN = 128 with a 3-stage ring and two CTAs
//                 per SM when the 128 x 128 tiles fill the 148 SMs (the
//                 second CTA's loads overlap the first one's MMAs); BN = 224
//                 with a 4-stage ring, one CTA per SM, when those tiles fill
//                 80-100 % of the SMs in a single wave (the output layer:
//                 8 x 17 tiles instead of 8 x 29 in 1.6 waves; a partial last
//                 column tile reads zeros past N and stores nothing there);
//                 else BN = 64 tiles, twice as many CTAs for the narrow
//                 1024-wide hidden layers.  Epilogues:
//                   EPI_F32        out = acc                         (fp32)
//                   EPI_BIAS_F32   out = acc + bias                  (fp32)
//                   EPI_BIAS_GELU  z = acc + bias; aux = z; out = gelu(z)  (bf16)
//                   EPI_DGELU      out = acc * gelu'(aux)            (bf16)
//                 With a_kblocks > 0, B = [B_hi | B_lo] (2K columns) against A
//                 (K columns) gives A (B_hi + B_lo)^T in one accumulator,
//                 the split-weight output layer (bf16 hi + bf16 lo carry
//                 about 16 mantissa bits of the fp32 weights): on the
//                 128 x 224 shape each stage holds A's k-block with both of
//                 its B k-blocks (A read once); on the others the A tile of
//                 k-block kb is A's k-block kb mod a_kblocks.
//                 Every mbarrier wait is bounded.  On a timeout the kernel
//                 raises the error flag, stops issuing, waits (bounded) for
//                 the TMA loads and MMAs it already issued, writes NaN into
//                 the output tiles it could not finish, and frees its TMEM
//                 before returning.
//
// plus the small element-wise and reduction kernels of a training step
// (transpose, loss gradient, bias gradient, Adam).  GELU is the exact
// erf form, 0.5 z (1 + erf(z / sqrt 2)).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>

#include "cupf_mlp.h"
#include "tcgen05.cuh"

namespace cupf_b200 {
namespace {

using namespace tc;

constexpr int kBM = 128, kBK = 64, kThreads = 128;
constexpr uint32_t kTileA = kBM * kBK * 2;     // 16 KB A tile per stage

// shared memory of one CTA: 1 KB alignment slack, the ring (an A tile and NB
// B tiles per stage), the barriers
template <int BN, int STAGES, int NB = 1>
constexpr size_t gemm_smem() {
  return 1024 + (size_t)STAGES * (kTileA + (uint32_t)NB * BN * kBK * 2) + 256;  // + barriers, TMEM slot, fail flag
}

enum { EPI_F32 = 0, EPI_BIAS_F32 = 1, EPI_BIAS_GELU = 2, EPI_DGELU = 3 };

// ---- TMA ----
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];\n" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major bf16 tile written by TMA with
// the 128-byte swizzle: rows of 64 elements (128 B), 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t smem_desc_sw128(const void* tile) {
  const uint64_t addr = smem_u32(tile);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;      // start address
  d |= (uint64_t)1 << 16;            // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset: next 8-row group
  d |= (uint64_t)1 << 46;            // descriptor version for tcgen05
  d |= (uint64_t)2 << 61;            // 128-byte swizzle
  return d;
}

// Instruction descriptor: bf16 x bf16 -> fp32, both operands K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4)                     // D format fp32
         | (1u << 7)                   // A format bf16
         | (1u << 10)                  // B format bf16
         | ((uint32_t)(n >> 3) << 17)  // N / 8
         | ((uint32_t)(m >> 4) << 24); // M / 16
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.3989422804014327f * expf(-0.5f * z * z);
}

struct GemmArgs {
  int M, N, K;
  void* out;           // [M][ldo] fp32 or bf16
  long long ldo;
  const float* bias;   // [N]
  __nv_bfloat16* aux;  // [M][ldaux] pre-activations (written by EPI_BIAS_GELU, read by EPI_DGELU)
  long long ldaux;
  int epi;
  int a_kblocks;  // > 0: A's k-block index wraps modulo a_kblocks (split-weight B)
  int* error;
  long long spin_limit;  // mbarrier polls before a wait gives up
  int stall_loads;       // failure-path test: the producer issues no loads, so the MMA thread's wait runs out
};

// tensor-memory columns of a BN-column accumulator (a power of two, >= 32)
template <int BN>
__host__ __device__ constexpr uint32_t tmem_cols() {
  return BN <= 32 ? 32u : BN <= 64 ? 64u : BN <= 128 ? 128u : 256u;
}

// NB = 2 (split weights, a_kblocks > 0): each stage holds A's k-block kb and
// both B k-blocks that multiply it, kb (hi) and a_kblocks + kb (lo), so A is
// read once for the two products; NB = 1 with a_kblocks > 0 reads A's
// k-blocks twice instead (k-block kb of B against A's kb mod a_kblocks).
template <int BN, int STAGES, int MINB, int NB = 1>
__global__ void __launch_bounds__(kThreads, MINB)
    k_gemm_bf16(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs g) {
  static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "accumulator width: 32..256 columns in steps of 32");
  static_assert(NB == 1 || NB == 2, "one B tile per stage, or the hi and lo tiles of split weights");
  constexpr uint32_t kTileB = (uint32_t)BN * kBK * 2;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sA = base;
  unsigned char* sB = base + STAGES * kTileA;  // [stage][NB] tiles
  uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * (kTileA + NB * kTileB));
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  int* s_fail = reinterpret_cast<int*>(tslot + 1);  // some thread's wait ran out

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * BN;
  const int nk = NB == 2 ? g.a_kblocks : g.K / kBK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(done, 1);
    *s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) tmem_alloc(tslot, tmem_cols<BN>());
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  bool ok = true;
  // programmatic dependent launch: the next kernel on the stream may start
  // its own set-up now; this CTA's first read of memory that an earlier
  // kernel writes (the producer's first load) waits for that kernel to
  // finish, and every store here follows that load
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");

  if (threadIdx.x == 0) {
    // producer: stage s holds k-block kb; refill it once the MMAs of kb - STAGES are done
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    int issued = 0;
    for (int kb = 0; kb < (g.stall_loads ? 0 : nk); ++kb) {
      const int s = kb % STAGES;
      if (kb >= STAGES && !mbar_wait(empty + s, ((kb / STAGES) - 1) & 1, g.spin_limit)) {
        ok = false;
        break;
      }
      mbar_expect_tx(full + s, kTileA + NB * kTileB);
      const int ka = NB == 1 && g.a_kblocks > 0 ? kb % g.a_kblocks : kb;
      tma_load_2d(sA + s * kTileA, &ta, ka * kBK, m0, full + s);
#pragma unroll
      for (int h = 0; h < NB; ++h)
        tma_load_2d(sB + (s * NB + h) * kTileB, &tb, (kb + h * g.a_kblocks) * kBK, n0, full + s);
      issued = kb + 1;
    }
    if (!ok) {
      // drain: the last load issued into each stage is the only one that can
      // still be in flight there (nothing newer was issued into that stage);
      // wait (bounded) for it before the CTA releases its shared memory
      for (int kb = issued - 1; kb >= 0 && kb >= issued - STAGES; --kb)
        mbar_wait(full + kb % STAGES, (kb / STAGES) & 1, g.spin_limit);
    }
  } else if (threadIdx.x == 32) {
    // MMA issuer
    constexpr uint32_t idesc = idesc_bf16(kBM, BN);
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (!mbar_wait(full + s, (kb / STAGES) & 1, g.spin_limit)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const uint64_t da = smem_desc_sw128(sA + s * kTileA);
#pragma unroll
      for (int h = 0; h < NB; ++h) {
        const uint64_t db = smem_desc_sw128(sB + (s * NB + h) * kTileB);
#pragma unroll
        for (int k = 0; k < kBK / 16; ++k)  // K = 16 per instruction: advance 32 bytes inside the swizzled row
          tc_mma(tmem, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc, (kb > 0 || h > 0 || k > 0) ? 1u : 0u);
      }
      tc_commit(empty + s);
    }
    tc_commit(done);  // arrives once every MMA issued above has completed
  }
  if (!ok) {
    atomicExch(g.error, 1);
    atomicExch(s_fail, 1);
  }

  // every lane waits, then the warp agrees, so the .sync.aligned loads below
  // run warp-converged
  const bool have = __all_sync(0xffffffffu, mbar_wait(done, 0, g.spin_limit));
  if (!have && lane == 0) {
    atomicExch(g.error, 2);
    atomicExch(s_fail, 1);
  }
  __syncthreads();
  tc_fence_after();
  if (*s_fail) {
    // a wait ran out, so the accumulator is not known to be complete: mark
    // this tile's outputs as not-a-number (the warm start treats a
    // non-finite prediction as missing and solves that scenario from flat
    // start); the host reads the raised flag
    const int row = m0 + warp * 32 + lane;
    for (int c = 0; c < BN && n0 + c < g.N; ++c) {
      if (g.epi == EPI_F32 || g.epi == EPI_BIAS_F32)
        static_cast<float*>(g.out)[(size_t)row * g.ldo + n0 + c] = __int_as_float(0x7fc00000);
      else
        static_cast<__nv_bfloat16*>(g.out)[(size_t)row * g.ldo + n0 + c] = __ushort_as_bfloat16((unsigned short)0x7fc0);
    }
    // MMAs issued before the timeout may still be writing the accumulator:
    // one more bounded wait before the tensor memory is released
    if (!have) mbar_wait(done, 0, g.spin_limit);
  } else {
    const int row = m0 + warp * 32 + lane;
    const uint32_t tl = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < BN && n0 + c0 < g.N; c0 += 32) {  // (N - n0 is a multiple of 32)
      float v[32];
      tmem_ld32(tl + (uint32_t)c0, v);
      const int col = n0 + c0;
      if (g.epi == EPI_F32 || g.epi == EPI_BIAS_F32) {
        if (g.epi == EPI_BIAS_F32)
#pragma unroll
          for (int i = 0; i < 32; ++i) v[i] += g.bias[col + i];
        float4* o = reinterpret_cast<float4*>(static_cast<float*>(g.out) + (size_t)row * g.ldo + col);
#pragma unroll
        for (int i = 0; i < 8; ++i) o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
      } else {
        __nv_bfloat16* aux = g.aux ? g.aux + (size_t)row * g.ldaux + col : nullptr;
        __align__(16) __nv_bfloat16 ob[32];
        if (g.epi == EPI_BIAS_GELU) {
          __align__(16) __nv_bfloat16 zb[32];
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const float z = v[i] + g.bias[col + i];
            zb[i] = __float2bfloat16(z);
            ob[i] = __float2bfloat16(gelu(z));
          }
          if (aux)  // inference keeps no pre-activations
#pragma unroll
            for (int i = 0; i < 4; ++i) reinterpret_cast<uint4*>(aux)[i] = reinterpret_cast<const uint4*>(zb)[i];
        } else {  // EPI_DGELU
          __align__(16) __nv_bfloat16 zb[32];
#pragma unroll
          for (int i = 0; i < 4; ++i) reinterpret_cast<uint4*>(zb)[i] = reinterpret_cast<const uint4*>(aux)[i];
#pragma unroll
          for (int i = 0; i < 32; ++i) ob[i] = __float2bfloat16(v[i] * gelu_grad(__bfloat162float(zb[i])));
        }
        uint4* o = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(g.out) + (size_t)row * g.ldo + col);
#pragma unroll
        for (int i = 0; i < 4; ++i) o[i] = reinterpret_cast<const uint4*>(ob)[i];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, tmem_cols<BN>());
}

// ---- element-wise / reduction kernels ----

// out[c][r] = in[r][c] for a rows x cols bf16 matrix with row stride ld (32 x 32 tiles through shared memory)
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ in, long long ld, __nv_bfloat16* __restrict__ out,
                                 int rows, int cols) {
  __shared__ __nv_bfloat16 t[32][33];
  const int c = blockIdx.x * 32 + threadIdx.x;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = blockIdx.y * 32 + i;
    if (r < rows && c < cols) t[i][threadIdx.x] = in[(size_t)r * ld + c];
  }
  __syncthreads();
  const int r = blockIdx.y * 32 + threadIdx.x;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int cc = blockIdx.x * 32 + i;
    if (r < rows && cc < cols) out[(size_t)cc * rows + r] = t[threadIdx.x][i];
  }
}

// features: x[b][k] = bf16((raw[b][k] - mean[k]) * inv_std[k]) for k < n_in, 0 for n_in <= k < width
// (x has row stride ldx)
__global__ void k_standardize(const float* __restrict__ raw, const float* __restrict__ mean,
                              const float* __restrict__ inv_std, __nv_bfloat16* __restrict__ x, long long ldx, int B,
                              int n_in, int width) {
  const long long n = (long long)B * width;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i % width);
    const long long b = i / width;
    x[b * ldx + k] = __float2bfloat16(k < n_in ? (raw[b * n_in + k] - mean[k]) * inv_std[k] : 0.0f);
  }
}

// Power-flow load features, standardized, straight from Sbus: column k is
// Re(sgen_k - S_bk) for k < n, Im(sgen_{k-n} - S_b(k-n)) for n <= k < 2n,
// extra[k - 2n] for the next n_extra columns (fixed inputs such as PV
// setpoints), then zero padding to width.  Rows r >= B repeat row B - 1.
__global__ void k_load_features(const double* __restrict__ sbus, long long sbus_stride, const double* __restrict__ sgen,
                                const float* __restrict__ extra, int n, int n_extra, const float* __restrict__ mean,
                                const float* __restrict__ inv_std, __nv_bfloat16* __restrict__ x, long long ldx,
                                int B, int width) {
  // block y = one row of x (scenario r; rows past B repeat the last one).  A
  // thread reads bus k's complex injection once (16 bytes) and writes both
  // of its features, P at column k and Q at column n + k.
  const long long r = blockIdx.y;
  const long long b = r < B ? r : B - 1;
  const double2* s = reinterpret_cast<const double2*>(sbus) + b * sbus_stride;
  const double2* sg = reinterpret_cast<const double2*>(sgen);
  __nv_bfloat16* xr = x + r * ldx;
  const int n_in = 2 * n + n_extra;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const double2 v = s[k], g = sg[k];
    const double fp = g.x - v.x, fq = g.y - v.y;
    xr[k] = __float2bfloat16(((float)fp - mean[k]) * inv_std[k]);
    xr[n + k] = __float2bfloat16(((float)fq - mean[n + k]) * inv_std[n + k]);
  }
  for (int k = 2 * n + blockIdx.x * blockDim.x + threadIdx.x; k < width; k += gridDim.x * blockDim.x)
    xr[k] = __float2bfloat16(k < n_in ? ((float)(double)extra[k - 2 * n] - mean[k]) * inv_std[k] : 0.0f);
}

// mean-squared-error gradient on the first n_out columns:
// g = 2 (pred - target) / (B n_out) in bf16 (0 in padding), loss += sum (pred - target)^2 / (B n_out)
__global__ void k_mse_grad(const float* __restrict__ pred, int ld, const float* __restrict__ target, int n_out, int B,
                           __nv_bfloat16* __restrict__ grad, float* __restrict__ loss) {
  const long long n = (long long)B * ld;
  const float scale = 1.0f / ((float)B * (float)n_out);
  float local = 0.0f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(i % ld);
    const long long b = i / ld;
    float gval = 0.0f;
    if (k < n_out) {
      const float d = pred[i] - target[b * n_out + k];
      gval = 2.0f * d * scale;
      local += d * d * scale;
    }
    grad[i] = __float2bfloat16(gval);
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, local);
}

// column sums of a bf16 [rows][cols] matrix into fp32 [cols]
__global__ void k_col_sum_bf16(const __nv_bfloat16* __restrict__ g, int rows, int cols, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.0f;
  for (int r = 0; r < rows; ++r) s += __bfloat162float(g[(size_t)r * cols + c]);
  out[c] = s;
}

// Adam on fp32 master weights; refreshes the bf16 copy used by the GEMMs.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ grad, float* __restrict__ m,
                       float* __restrict__ v, __nv_bfloat16* __restrict__ w16, long long n, float lr, float b1,
                       float b2, float eps, float bc1, float bc2, float weight_decay) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = grad[i] + weight_decay * w[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16(wi);
  }
}

// ---- host side ----

thread_local std::string g_err;

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  if (!fn) throw std::runtime_error("cuTensorMapEncodeTiled is not available");
  return fn;
}

// [rows][k] bf16 with row stride ld, K contiguous, boxes of box_rows rows x 64 elements, 128-byte swizzle
CUtensorMap make_map(const void* ptr, int rows, int k, long long ld, int box_rows) {
  CUtensorMap m;
  const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box,
                               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw std::runtime_error("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}

int* error_flag() {
  static std::mutex mu;
  static std::map<int, int*> flags;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  int*& f = flags[dev];
  if (!f) {
    if (cudaMalloc(&f, sizeof(int)) != cudaSuccess) throw std::runtime_error("error flag allocation failed");
    cudaMemset(f, 0, sizeof(int));
  }
  return f;
}

// Wait bound of the GEMM's mbarrier polls and the failure-path test switch
// (mlp_set_wait_test); read at each launch.
std::atomic<long long> g_spin_limit{kSpinLimit};
std::atomic<int> g_stall_loads{0};

// the tile shapes: wide grids; grids with fewer 128 x 128 tiles than SMs;
// and grids whose 128 x 224 tiles fill 80-100 % of the SMs in one wave (one
// CTA per SM, a 4-stage ring of 44 KB stages), where 128 x 128 tiles two per
// SM would leave a partly filled second wave (the network's output layer)
constexpr int kWideBN = 128, kWideStages = 3, kWideMinBlocks = 2;
constexpr int kNarrowBN = 64, kNarrowStages = 4, kNarrowMinBlocks = 2;
constexpr int kTallBN = 224, kTallStages = 4, kTallMinBlocks = 1;
constexpr int kTallSplitStages = 3;  // stages of A + hi + lo tiles (72 KB each)
constexpr int kSMs = 148;

template <int BN, int STAGES, int MINB, int NB = 1>
void set_smem_attribute() {
  const cudaError_t e = cudaFuncSetAttribute(k_gemm_bf16<BN, STAGES, MINB, NB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)gemm_smem<BN, STAGES, NB>());
  if (e != cudaSuccess) throw std::runtime_error(std::string("gemm smem attribute: ") + cudaGetErrorString(e));
}

void configure_gemm() {
  static std::mutex mu;
  static std::map<int, bool> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return;
  set_smem_attribute<kWideBN, kWideStages, kWideMinBlocks>();
  set_smem_attribute<kNarrowBN, kNarrowStages, kNarrowMinBlocks>();
  set_smem_attribute<kTallBN, kTallStages, kTallMinBlocks>();
  set_smem_attribute<kTallBN, kTallSplitStages, kTallMinBlocks, 2>();
  done[dev] = true;
}

template <int BN, int STAGES, int MINB, int NB = 1>
void launch_shape(const void* A, long long lda, int ka_cols, const void* B, long long ldb, GemmArgs g,
                  cudaStream_t stream) {
  const CUtensorMap ta = make_map(A, g.M, ka_cols, lda, kBM), tb = make_map(B, g.N, g.K, ldb, BN);
  g.spin_limit = g_spin_limit.load();
  g.stall_loads = g_stall_loads.load();
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((g.N + BN - 1) / BN, g.M / kBM);  // a partial last column tile reads zeros past N
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = gemm_smem<BN, STAGES, NB>();
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;  // overlap the previous kernel's tail
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, k_gemm_bf16<BN, STAGES, MINB, NB>, ta, tb, g);
  if (e != cudaSuccess) throw std::runtime_error(std::string("gemm launch: ") + cudaGetErrorString(e));
}

// A has ka_cols columns (== g.K unless A's k-blocks wrap); M, N multiples of 128
void launch_gemm(const void* A, long long lda, int ka_cols, const void* B, long long ldb, const GemmArgs& g,
                 cudaStream_t stream) {
  configure_gemm();
  const long long tall = (long long)(g.M / kBM) * ((g.N + kTallBN - 1) / kTallBN);
  if ((long long)(g.M / kBM) * (g.N / 128) >= kSMs && tall <= kSMs && 5 * tall >= 4 * kSMs) {
    if (g.a_kblocks > 0)
      launch_shape<kTallBN, kTallSplitStages, kTallMinBlocks, 2>(A, lda, ka_cols, B, ldb, g, stream);
    else
      launch_shape<kTallBN, kTallStages, kTallMinBlocks>(A, lda, ka_cols, B, ldb, g, stream);
  }
  else if ((long long)(g.M / kBM) * (g.N / 128) >= kSMs)
    launch_shape<kWideBN, kWideStages, kWideMinBlocks>(A, lda, ka_cols, B, ldb, g, stream);
  else
    launch_shape<kNarrowBN, kNarrowStages, kNarrowMinBlocks>(A, lda, ka_cols, B, ldb, g, stream);
}

unsigned grid1d(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16); }

template <typename F>
int guarded(F&& f) {
  try {
    f();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      g_err = cudaGetErrorString(e);
      return 2;
    }
    return 0;
  } catch (const std::exception& ex) {
    g_err = ex.what();
    return 1;
  }
}

}  // namespace
}  // namespace cupf_b200

using namespace cupf_b200;

extern "C" {

const char* mlp_last_error() { return g_err.c_str(); }

int mlp_gemm_bf16(const void* A, long long lda, const void* B, long long ldb, int M, int N, int K, int epi,
                  void* out, long long ldo, const float* bias, void* aux, long long ldaux, void* stream) {
  return guarded([&] {
    if (M <= 0 || N <= 0 || K <= 0 || M % kBM || N % 128 || K % kBK)
      throw std::invalid_argument("mlp_gemm_bf16: M and N must be multiples of 128, K of 64");
    if (epi < EPI_F32 || epi > EPI_DGELU) throw std::invalid_argument("mlp_gemm_bf16: unknown epilogue");
    if ((epi == EPI_BIAS_F32 || epi == EPI_BIAS_GELU) && !bias) throw std::invalid_argument("mlp_gemm_bf16: bias missing");
    if (epi == EPI_DGELU && (!aux || ldaux < N)) throw std::invalid_argument("mlp_gemm_bf16: aux missing");
    if (epi == EPI_BIAS_GELU && aux && ldaux < N) throw std::invalid_argument("mlp_gemm_bf16: aux row stride < N");
    if (lda < K || ldb < K || ldo < N || lda % 8 || ldb % 8 || ldo % 8)
      throw std::invalid_argument("mlp_gemm_bf16: leading dimensions must be >= the row length and multiples of 8");
    if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(out)) & 15)
      throw std::invalid_argument("mlp_gemm_bf16: operands must be 16-byte aligned");
    GemmArgs g{M, N, K, out, ldo, bias, static_cast<__nv_bfloat16*>(aux), ldaux, epi, 0, error_flag(), kSpinLimit, 0};
    launch_gemm(A, lda, K, B, ldb, g, static_cast<cudaStream_t>(stream));
  });
}

int mlp_gemm_bf16_split(const void* A, long long lda, const void* B, long long ldb, int M, int N, int K, int epi,
                        void* out, long long ldo, const float* bias, void* stream) {
  return guarded([&] {
    if (M <= 0 || N <= 0 || K <= 0 || M % kBM || N % 128 || K % kBK)
      throw std::invalid_argument("mlp_gemm_bf16_split: M and N must be multiples of 128, K of 64");
    if (epi != EPI_F32 && epi != EPI_BIAS_F32)
      throw std::invalid_argument("mlp_gemm_bf16_split: only the fp32 epilogues keep the split's precision");
    if (epi == EPI_BIAS_F32 && !bias) throw std::invalid_argument("mlp_gemm_bf16_split: bias missing");
    if (lda < K || ldb < 2LL * K || ldo < N || lda % 8 || ldb % 8 || ldo % 8)
      throw std::invalid_argument("mlp_gemm_bf16_split: need lda >= K, ldb >= 2K, ldo >= N, all multiples of 8");
    if ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) | reinterpret_cast<uintptr_t>(out)) & 15)
      throw std::invalid_argument("mlp_gemm_bf16_split: operands must be 16-byte aligned");
    GemmArgs g{M, N, 2 * K, out, ldo, bias, nullptr, 0, epi, K / kBK, error_flag(), kSpinLimit, 0};
    launch_gemm(A, lda, K, B, ldb, g, static_cast<cudaStream_t>(stream));
  });
}

int mlp_set_wait_test(long long spin_limit, int stall_loads) {
  if (spin_limit < 1 || (stall_loads != 0 && stall_loads != 1)) {
    g_err = "mlp_set_wait_test: spin_limit must be positive and stall_loads 0 or 1";
    return 1;
  }
  g_spin_limit.store(spin_limit);
  g_stall_loads.store(stall_loads);
  return 0;
}

int mlp_error_flag(int* out_host, int reset) {
  return guarded([&] {
    int* f = error_flag();
    if (cudaMemcpy(out_host, f, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      throw std::runtime_error("error flag read failed");
    if (reset) cudaMemset(f, 0, sizeof(int));
  });
}

int mlp_transpose_bf16(const void* in, long long ld, void* out, int rows, int cols, void* stream) {
  return guarded([&] {
    if (ld < cols) throw std::invalid_argument("mlp_transpose_bf16: ld must be >= cols");
    dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    k_transpose_bf16<<<grid, dim3(32, 8), 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(in), ld, static_cast<__nv_bfloat16*>(out), rows, cols);
  });
}

int mlp_standardize(const float* raw, const float* mean, const float* inv_std, void* x, long long ldx, int B,
                    int n_in, int width, void* stream) {
  return guarded([&] {
    if (ldx < width || width < n_in) throw std::invalid_argument("mlp_standardize: need n_in <= width <= ldx");
    k_standardize<<<grid1d((long long)B * width), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        raw, mean, inv_std, static_cast<__nv_bfloat16*>(x), ldx, B, n_in, width);
  });
}

int mlp_load_features(const double* sbus, long long sbus_stride, const double* sgen, const float* extra, int n,
                      int n_extra, const float* mean, const float* inv_std, void* x, long long ldx, int B, int rows,
                      int width, void* stream) {
  return guarded([&] {
    if (!sbus || !sgen || !mean || !inv_std || !x || (n_extra > 0 && !extra))
      throw std::invalid_argument("mlp_load_features: null pointer");
    if (n <= 0 || n_extra < 0 || B <= 0 || rows < B || width < 2 * n + n_extra || ldx < width || sbus_stride < n)
      throw std::invalid_argument("mlp_load_features: inconsistent sizes");
    if (rows > 65535) throw std::invalid_argument("mlp_load_features: more than 65535 rows");
    if ((reinterpret_cast<uintptr_t>(sbus) | reinterpret_cast<uintptr_t>(sgen)) & 15)
      throw std::invalid_argument("mlp_load_features: sbus and sgen must be 16-byte aligned (complex128 elements)");
    const int per_row = std::max(n, width - 2 * n);
    const dim3 grid((unsigned)std::min((per_row + 255) / 256, 8), (unsigned)rows);
    k_load_features<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        sbus, sbus_stride, sgen, extra, n, n_extra, mean, inv_std, static_cast<__nv_bfloat16*>(x), ldx, B, width);
  });
}

int mlp_mse_grad(const float* pred, int ld, const float* target, int n_out, int B, void* grad, float* loss,
                 void* stream) {
  return guarded([&] {
    k_mse_grad<<<grid1d((long long)B * ld), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        pred, ld, target, n_out, B, static_cast<__nv_bfloat16*>(grad), loss);
  });
}

int mlp_col_sum_bf16(const void* g, int rows, int cols, float* out, void* stream) {
  return guarded([&] {
    k_col_sum_bf16<<<(cols + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(g), rows, cols, out);
  });
}

int mlp_adam(float* w, const float* grad, float* m, float* v, void* w_bf16, long long n, float lr, float b1, float b2,
             float eps, int step, float weight_decay, void* stream) {
  return guarded([&] {
    const float bc1 = 1.0f - std::pow(b1, (float)step), bc2 = 1.0f - std::pow(b2, (float)step);
    k_adam<<<grid1d(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(w, grad, m, v, static_cast<__nv_bfloat16*>(w_bf16),
                                                                      n, lr, b1, b2, eps, bc1, bc2, weight_decay);
  });
}

}  // extern "C"
