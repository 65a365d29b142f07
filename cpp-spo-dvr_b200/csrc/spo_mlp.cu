// The learned potential (include/spo_mlp.h): a BF16 multilayer perceptron whose products run on the
// B200 tensor cores through tcgen05.mma, FP32 accumulators in tensor memory.
//
// One GEMM kernel serves the forward pass and both backward products: C[M x N] = A[M x K] B[N x K]^T
// with A and B BF16, K-major (row-major with K contiguous), K a multiple of 64, N <= 256:
//   - a block of 128 threads owns 128 rows of C; warp 0 allocates 256 tensor-memory columns;
//   - per K chunk of 64, the threads stage A (128 x 64) and B (N x 64) in shared memory in the
//     canonical K-major layout without swizzle (8-row x 16-byte core matrices: K chunks LBO bytes
//     apart, 8-row groups SBO = 128 bytes apart), make the writes visible to the tensor core
//     (fence.proxy.async), and one thread issues four tcgen05.mma (M 128, N, K 16) and a
//     tcgen05.commit on the stage's mbarrier; two stages alternate, so chunk k + 1 is staged while
//     the tensor core multiplies chunk k (a stage is rewritten after its previous commit, bounded wait);
//   - epilogue: each warp reads its 32 accumulator lanes (tcgen05.ld 32x32b, 16 columns at a time)
//     and writes FP32, BF16, or bias + SiLU (pre-activation FP32, activation BF16);
//   - split K: blockIdx.y takes a share of the K chunks and writes its own FP32 partial, summed in a
//     fixed order afterwards (weight gradients, where K is the batch).
// Everything else (output layer, loss, SiLU derivative, transposes, Adam) is plain SIMT, with fixed-
// order reductions so that a training run is repeatable.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/spo_b200.h"
#include "../../include/spo_mlp.h"

namespace {

using bf16 = __nv_bfloat16;

struct MlpError : std::runtime_error {
  int code;
  MlpError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void ck(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) throw MlpError(SPO_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e));
  if (e != cudaSuccess) throw MlpError(SPO_ERR_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}
void need(bool c, const std::string& m) {
  if (!c) throw MlpError(SPO_ERR_INVALID, m);
}

// ------------------------------------------------------------------------------------------------
// tcgen05 / mbarrier primitives
// ------------------------------------------------------------------------------------------------
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
constexpr int kWaitLimit = 1 << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = smem_addr(bar);
  for (int i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Warp-wide: allocates `cols` tensor-memory columns, the address written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t addr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(addr), "r"(cols) : "memory");
}
// Shared-memory matrix descriptor, K-major without swizzle (version 1, base offset 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// D[tmem] (+)= A[smem] B[smem]^T, BF16 inputs, FP32 accumulate (one thread issues).
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}
// Arrives on the barrier when this thread's earlier tcgen05.mma have completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}
// Warp-wide: 16 consecutive FP32 columns of the warp's 32 lanes (one lane per thread).
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace tc

enum Epilogue { kEpiF32 = 0, kEpiBf16 = 1, kEpiBiasSilu = 2 };

struct GemmArgs {
  const bf16* a;
  long long lda;
  const bf16* b;
  long long ldb;
  int m, n, k;
  int epi;
  float* c;  // kEpiF32 (split K: partial y at c + y * c_split_stride), kEpiBiasSilu: pre-activation
  long long ldc, c_split_stride;
  const float* bias;
  bf16* out16;  // kEpiBf16: the product; kEpiBiasSilu: the activation
  long long ld16;
  int* error_flag;
};

constexpr int kBM = 128, kBK = 64, kBNMax = 256;
constexpr std::size_t kStageBytes = static_cast<std::size_t>(kBM + kBNMax) * kBK * 2;  // one A and one B chunk
constexpr std::size_t kGemmSmem = 2 * kStageBytes + 64;                                  // two stages, barriers
// At most two blocks per SM: the number whose 256 tensor-memory columns fit the SM's 512 together.
constexpr std::size_t kGemmLaunchSmem = kGemmSmem;
static_assert(3 * kGemmLaunchSmem > 228 * 1024, "two blocks per SM at most");

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }

// Two stages: while the tensor core multiplies chunk k (stage k % 2), the threads stage chunk k + 1 in
// the other buffer, after the commit of chunk k - 1 (its previous user) has arrived.
__global__ void __launch_bounds__(128) gemm_tn_kernel(GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * kStageBytes);  // one per stage
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tc::tmem_alloc(tslot, 256);
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::mbar_init(bar + 1, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  const int m0 = blockIdx.x * kBM;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(g.n >> 3) << 17) |
                         (static_cast<uint32_t>(kBM >> 4) << 24);
  const int nk = g.k / kBK;
  const int kc_first = static_cast<int>(static_cast<long long>(nk) * blockIdx.y / gridDim.y);
  const int kc_last = static_cast<int>(static_cast<long long>(nk) * (blockIdx.y + 1) / gridDim.y);
  // A: core (r8, kc) at (kc * 16 + r8) * 128; B: core (r8, kc) at (kc * 32 + r8) * 128
  // All of a thread's 16-byte loads of a chunk are issued before the first is stored.
  auto stage = [&](int st, int kc) {
    unsigned char* As = smem + st * kStageBytes;
    unsigned char* Bs = As + kBM * kBK * 2;
    const int k0 = kc * kBK;
    constexpr int NA = kBM * 8 / 128, NB = kBNMax * 8 / 128;
    uint4 va[NA], vb[NB];
#pragma unroll
    for (int i = 0; i < NA; ++i) {
      const int p = tid + 128 * i, r = p >> 3, c = p & 7;
      va[i] = m0 + r < g.m ? *reinterpret_cast<const uint4*>(g.a + static_cast<long long>(m0 + r) * g.lda + k0 + 8 * c)
                           : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      const int p = tid + 128 * i, r = p >> 3, c = p & 7;
      if (p < g.n * 8) vb[i] = *reinterpret_cast<const uint4*>(g.b + static_cast<long long>(r) * g.ldb + k0 + 8 * c);
    }
#pragma unroll
    for (int i = 0; i < NA; ++i) {
      const int p = tid + 128 * i, r = p >> 3, c = p & 7;
      *reinterpret_cast<uint4*>(As + (c * (kBM / 8) + (r >> 3)) * 128 + (r & 7) * 16) = va[i];
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      const int p = tid + 128 * i, r = p >> 3, c = p & 7;
      if (p < g.n * 8) *reinterpret_cast<uint4*>(Bs + (c * (kBNMax / 8) + (r >> 3)) * 128 + (r & 7) * 16) = vb[i];
    }
    tc::fence_proxy_async();  // the generic writes, visible to the tensor core
  };
  uint32_t parity = 0;   // bit s: the phase parity of stage s's barrier
  uint32_t pending = 0;  // bit s: a commit on stage s's barrier not yet waited for
  bool failed = false;
  if (kc_first < kc_last) stage(0, kc_first);
  tc::fence_before_sync();
  __syncthreads();
  for (int kc = kc_first; kc < kc_last; ++kc) {
    const int st = (kc - kc_first) & 1;
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t a0 = tc::smem_addr(smem + st * kStageBytes);
      const uint32_t b0 = a0 + kBM * kBK * 2;
#pragma unroll
      for (int s = 0; s < kBK / 16; ++s) {
        const uint64_t ad = tc::smem_desc(a0 + 2 * s * (kBM / 8) * 128, (kBM / 8) * 128, 128);
        const uint64_t bd = tc::smem_desc(b0 + 2 * s * (kBNMax / 8) * 128, (kBNMax / 8) * 128, 128);
        tc::mma_bf16(tmem, ad, bd, idesc, (kc > kc_first || s > 0) ? 1u : 0u);
      }
      tc::commit(bar + st);
    }
    pending |= 1u << st;
    if (kc + 1 < kc_last) {
      // the other stage's previous chunk (kc - 1) must be multiplied before it is overwritten
      bool ok = true;
      if (kc > kc_first) {
        ok = tc::mbar_wait(bar + (st ^ 1), parity >> (st ^ 1) & 1u);
        if (ok) {
          parity ^= 1u << (st ^ 1);
          pending &= ~(1u << (st ^ 1));
        }
      }
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      stage(st ^ 1, kc + 1);
    }
    tc::fence_before_sync();
    __syncthreads();
  }
  // The last chunk's commit: it arrives when every earlier tcgen05.mma of the issuing thread has
  // completed, so the accumulator is final (the second-to-last commit needs no wait of its own).
  if (!failed && kc_last > kc_first) {
    const int last = (kc_last - kc_first - 1) & 1;
    const bool ok = tc::mbar_wait(bar + last, parity >> last & 1u);
    if (ok) pending = 0;  // the last commit arrives after every earlier MMA of the issuing thread
    failed = __syncthreads_or(!ok) != 0;
  }
  tc::fence_after_sync();
  if (failed) {
    if (tid == 0) atomicExch(g.error_flag, 1);
    // bounded waits for the MMAs in flight, so that none still writes the accumulator when it is freed
    for (int k = 0; k < 2; ++k)
      if (pending >> k & 1u) tc::mbar_wait(bar + k, parity >> k & 1u);
  } else if (kc_last > kc_first) {
    const int row = m0 + warp * 32 + lane;
    for (int j = 0; j < g.n / 16; ++j) {
      uint32_t r[16];
      tc::tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(j * 16), r);
      if (row < g.m) {
        if (g.epi == kEpiF32) {
          float* dst = g.c + blockIdx.y * g.c_split_stride + static_cast<long long>(row) * g.ldc + j * 16;
#pragma unroll
          for (int e = 0; e < 16; e += 4)
            *reinterpret_cast<float4*>(dst + e) = make_float4(__uint_as_float(r[e]), __uint_as_float(r[e + 1]),
                                                              __uint_as_float(r[e + 2]), __uint_as_float(r[e + 3]));
        } else if (g.epi == kEpiBf16) {
          bf16* dst = g.out16 + static_cast<long long>(row) * g.ld16 + j * 16;
#pragma unroll
          for (int e = 0; e < 16; ++e) dst[e] = __float2bfloat16_rn(__uint_as_float(r[e]));
        } else {
          float* zd = g.c + static_cast<long long>(row) * g.ldc + j * 16;
          bf16* ad = g.out16 + static_cast<long long>(row) * g.ld16 + j * 16;
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const float z = __uint_as_float(r[e]) + g.bias[j * 16 + e];
            zd[e] = z;
            ad[e] = __float2bfloat16_rn(silu(z));
          }
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 256);
}

// ------------------------------------------------------------------------------------------------
// SIMT kernels
// ------------------------------------------------------------------------------------------------
// x (n x n_in, FP32) rows idx[i] (or i) -> BF16 rows of width w (zero-padded).
__global__ void gather_inputs_kernel(const float* __restrict__ x, int n_in, const long long* __restrict__ idx,
                                     long long rows, int w, bf16* __restrict__ out) {
  const long long total = rows * w;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long i = t / w;
    const int c = static_cast<int>(t - i * w);
    const long long src = idx ? idx[i] : i;
    out[t] = __float2bfloat16_rn(c < n_in ? x[src * n_in + c] : 0.0f);
  }
}
__global__ void gather_targets_kernel(const float* __restrict__ y, const long long* __restrict__ idx, long long rows,
                                      float* __restrict__ out) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < rows;
       i += static_cast<long long>(gridDim.x) * blockDim.x)
    out[i] = y[idx ? idx[i] : i];
}

// out[i] = sum_k a[i][k] w[k] + b, one warp per row, fixed order (lane-strided sums, then a fixed tree).
__global__ void output_layer_kernel(const bf16* __restrict__ a, int w, const float* __restrict__ wo,
                                    const float* __restrict__ bo, long long rows, float* __restrict__ out) {
  const long long row = blockIdx.x * static_cast<long long>(blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (row >= rows) return;
  float s = 0.0f;
  for (int k = lane; k < w; k += 32) s += __bfloat162float(a[row * w + k]) * wo[k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[row] = s + bo[0];
}

// d[i] = 2 (out[i] - y[i]) / rows; the squared errors summed per block in a fixed order.
__global__ void loss_kernel(const float* __restrict__ out, const float* __restrict__ y, long long rows,
                            float* __restrict__ d, double* __restrict__ block_sums) {
  __shared__ double part[256];
  double s = 0.0;
  for (long long i = blockIdx.x * 256ll + threadIdx.x; i < rows; i += 256ll * gridDim.x) {
    const float e = out[i] - y[i];
    d[i] = 2.0f * e / static_cast<float>(rows);
    s += static_cast<double>(e) * e;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) block_sums[blockIdx.x] = part[0];
}

// Column sums over rows, one block per column, fixed order: sum_i v(i, col).
// mode 0: gw_out[col] = sum_i d[i] a[i][col]; mode 1: gb[col] = sum_i dzf[i][col] (FP32 matrix).
__global__ void column_sums_kernel(int mode, const float* __restrict__ d, const bf16* __restrict__ a,
                                   const float* __restrict__ m32, int w, long long rows, float* __restrict__ out) {
  __shared__ float part[256];
  const int col = blockIdx.x;
  float s = 0.0f;
  for (long long i = threadIdx.x; i < rows; i += 256) {
    s += mode == 0 ? d[i] * __bfloat162float(a[i * w + col]) : m32[i * w + col];
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) part[threadIdx.x] += part[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[col] = part[0];
}

// Gradient into the last hidden activation: g[i][k] = d[i] w_out[k] (FP32).
__global__ void output_backward_kernel(const float* __restrict__ d, const float* __restrict__ wo, int w,
                                       long long rows, float* __restrict__ g) {
  const long long total = rows * w;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long i = t / w;
    g[t] = d[i] * wo[t - i * w];
  }
}

// dz = g * SiLU'(z), kept in FP32 (bias gradient) and BF16 (the products), both row-major.
__global__ void silu_backward_kernel(const float* __restrict__ g, const bf16* __restrict__ g16, const float* __restrict__ z,
                                     long long total, float* __restrict__ dz, bf16* __restrict__ dz16) {
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float zz = z[t];
    const float s = 1.0f / (1.0f + __expf(-zz));
    const float gv = g ? g[t] : __bfloat162float(g16[t]);
    const float v = gv * s * (1.0f + zz * (1.0f - s));
    dz[t] = v;
    dz16[t] = __float2bfloat16_rn(v);
  }
}

// out[c][r] = in[r][c] for an R x C BF16 matrix (32 x 32 tiles through shared memory).
__global__ void transpose_kernel(const bf16* __restrict__ in, long long rows, int cols, bf16* __restrict__ out) {
  __shared__ bf16 tile[32][33];
  const long long r0 = static_cast<long long>(blockIdx.y) * 32;
  const int c0 = blockIdx.x * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const long long r = r0 + k;
    const int c = c0 + threadIdx.x;
    tile[k][threadIdx.x] = (r < rows && c < cols) ? in[r * cols + c] : __float2bfloat16_rn(0.0f);
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k;
    const long long r = r0 + threadIdx.x;
    if (c < cols && r < rows) out[static_cast<long long>(c) * rows + r] = tile[threadIdx.x][k];
  }
}

// out[i] = sum over the split partials in order.
__global__ void sum_partials_kernel(const float* __restrict__ parts, int n_parts, long long stride, long long n,
                                    float* __restrict__ out) {
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    float s = 0.0f;
    for (int p = 0; p < n_parts; ++p) s += parts[p * stride + t];
    out[t] = s;
  }
}

// Adam on FP32 parameters.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float c1, float c2,
                            float eps) {
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float gt = g[t];
    const float mt = b1 * m[t] + (1.0f - b1) * gt;
    const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
  }
}

// BF16 copies of a weight matrix W (rows x cols): row-major and transposed.
__global__ void weights_to_bf16_kernel(const float* __restrict__ w, int rows, int cols, bf16* __restrict__ wb,
                                       bf16* __restrict__ wt) {
  const long long total = static_cast<long long>(rows) * cols;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(t / cols), c = static_cast<int>(t - static_cast<long long>(r) * cols);
    const bf16 h = __float2bfloat16_rn(w[t]);
    wb[t] = h;
    wt[static_cast<long long>(c) * rows + r] = h;
  }
}

unsigned grid_for(long long n, int threads = 256) {
  return static_cast<unsigned>(std::min<long long>(std::max<long long>((n + threads - 1) / threads, 1), 148 * 16));
}

// ------------------------------------------------------------------------------------------------
// The network
// ------------------------------------------------------------------------------------------------
template <typename U>
struct DevBuf {
  U* p = nullptr;
  std::size_t n = 0;
  void alloc(std::size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    n = count;
    ck(cudaMalloc(&p, sizeof(U) * std::max<std::size_t>(count, 1)), "cudaMalloc");
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

struct Layer {
  int in, out;
  DevBuf<float> w, b, gw, gb, mw, vw, mb, vb;
  DevBuf<bf16> wb, wt;
};

}  // namespace

struct spo_mlp {
  std::string err;
  int device = 0;
  int n_in = 0, in_pad = 0, width = 0, depth = 0;
  cudaStream_t stream = nullptr;
  std::vector<std::unique_ptr<Layer>> layers;
  DevBuf<float> wo, bo, gwo, gbo, mwo, vwo, mbo, vbo;
  DevBuf<int> error_flag;
  // per-batch work space (capacity rows)
  long long cap = 0;
  DevBuf<bf16> x16;                        // rows x in_pad
  std::vector<std::unique_ptr<DevBuf<float>>> z;   // per layer: rows x width (pre-activation)
  std::vector<std::unique_ptr<DevBuf<bf16>>> act;  // per layer: rows x width (activation)
  DevBuf<float> out, yb, d, g32, dz32, partials;
  DevBuf<double> loss_parts;
  DevBuf<bf16> g16, dz16, dzt, at;
  DevBuf<long long> idx;
  long long step = 0;

  ~spo_mlp() {
    if (stream) cudaStreamDestroy(stream);
  }

  long long parameter_count() const {
    long long n = 0;
    for (const auto& l : layers) n += static_cast<long long>(l->in) * l->out + l->out;
    return n + width + 1;
  }

  void ensure_capacity(long long rows) {
    if (rows <= cap) return;
    cap = ((rows + 127) / 128) * 128;
    x16.alloc(cap * in_pad);
    z.clear();
    act.clear();
    for (int l = 0; l < depth; ++l) {
      z.push_back(std::make_unique<DevBuf<float>>());
      z.back()->alloc(cap * width);
      act.push_back(std::make_unique<DevBuf<bf16>>());
      act.back()->alloc(cap * width);
    }
    out.alloc(cap);
    yb.alloc(cap);
    d.alloc(cap);
    g32.alloc(cap * width);
    dz32.alloc(cap * width);
    g16.alloc(cap * width);
    dz16.alloc(cap * width);
    dzt.alloc(cap * width);
    at.alloc(cap * std::max(width, in_pad));
    idx.alloc(cap);
    loss_parts.alloc(256);
  }

  void refresh_bf16() {
    for (auto& l : layers)
      weights_to_bf16_kernel<<<grid_for(static_cast<long long>(l->in) * l->out), 256, 0, stream>>>(l->w.p, l->out, l->in,
                                                                                                   l->wb.p, l->wt.p);
    ck(cudaGetLastError(), "weights_to_bf16");
  }

  void gemm(const bf16* a, long long lda, const bf16* b, long long ldb, int m, int n, int k, int epi, float* c,
            long long ldc, const float* bias, bf16* out16, long long ld16, int splits = 1, long long split_stride = 0) {
    need(k % kBK == 0 && n % 16 == 0 && n >= 16 && n <= kBNMax && lda % 8 == 0 && ldb % 8 == 0, "gemm shape");
    GemmArgs g{a, lda, b, ldb, m, n, k, epi, c, ldc, split_stride, bias, out16, ld16, error_flag.p};
    const dim3 grid(static_cast<unsigned>((m + kBM - 1) / kBM), static_cast<unsigned>(splits));
    gemm_tn_kernel<<<grid, 128, kGemmLaunchSmem, stream>>>(g);
    ck(cudaGetLastError(), "gemm launch");
  }

  // Forward pass of `rows` rows already in x16; output in out.
  void forward(long long rows) {
    const bf16* a = x16.p;
    int k = in_pad;
    for (int l = 0; l < depth; ++l) {
      Layer& L = *layers[l];
      gemm(a, k, L.wb.p, L.in, static_cast<int>(rows), width, k, kEpiBiasSilu, z[l]->p, width, L.b.p, act[l]->p, width);
      a = act[l]->p;
      k = width;
    }
    output_layer_kernel<<<static_cast<unsigned>((rows + 7) / 8), 256, 0, stream>>>(act[depth - 1]->p, width, wo.p, bo.p,
                                                                                  rows, out.p);
    ck(cudaGetLastError(), "output layer");
  }

  // Loss and all gradients for `rows` rows in x16 / yb. Returns the loss.
  double backward(long long rows) {
    const unsigned lb = static_cast<unsigned>(std::min<long long>((rows + 255) / 256, 256));
    loss_kernel<<<lb, 256, 0, stream>>>(out.p, yb.p, rows, d.p, loss_parts.p);
    column_sums_kernel<<<width, 256, 0, stream>>>(0, d.p, act[depth - 1]->p, nullptr, width, rows, gwo.p);
    column_sums_kernel<<<1, 256, 0, stream>>>(1, nullptr, nullptr, d.p, 1, rows, gbo.p);
    output_backward_kernel<<<grid_for(rows * width), 256, 0, stream>>>(d.p, wo.p, width, rows, g32.p);
    ck(cudaGetLastError(), "output backward");
    const int splits = static_cast<int>(std::min<long long>(64, rows / kBK));
    for (int l = depth - 1; l >= 0; --l) {
      Layer& L = *layers[l];
      const bool first_grad = l == depth - 1;
      silu_backward_kernel<<<grid_for(rows * width), 256, 0, stream>>>(first_grad ? g32.p : nullptr, g16.p, z[l]->p,
                                                                      rows * width, dz32.p, dz16.p);
      column_sums_kernel<<<width, 256, 0, stream>>>(1, nullptr, nullptr, dz32.p, width, rows, L.gb.p);
      // gW = dz^T a_in : A = dz^T (width x rows), B = a_in^T (in x rows), K = rows
      const bf16* a_in = l == 0 ? x16.p : act[l - 1]->p;
      const dim3 tb(32, 8);
      transpose_kernel<<<dim3((width + 31) / 32, static_cast<unsigned>((rows + 31) / 32)), tb, 0, stream>>>(
          dz16.p, rows, width, dzt.p);
      transpose_kernel<<<dim3((L.in + 31) / 32, static_cast<unsigned>((rows + 31) / 32)), tb, 0, stream>>>(
          a_in, rows, L.in, at.p);
      ck(cudaGetLastError(), "transposes");
      const long long wsz = static_cast<long long>(L.out) * L.in;
      gemm(dzt.p, rows, at.p, rows, L.out, L.in, static_cast<int>(rows), kEpiF32, partials.p, L.in, nullptr, nullptr, 0,
           splits, wsz);
      sum_partials_kernel<<<grid_for(wsz), 256, 0, stream>>>(partials.p, splits, wsz, wsz, L.gw.p);
      ck(cudaGetLastError(), "sum partials");
      if (l > 0) {
        // d a_in = dz W : A = dz (rows x width), B = W^T (in x width)
        gemm(dz16.p, width, L.wt.p, L.out, static_cast<int>(rows), L.in, width, kEpiBf16, nullptr, 0, nullptr, g16.p,
             L.in);
      }
    }
    std::vector<double> parts(lb);
    ck(cudaMemcpyAsync(parts.data(), loss_parts.p, sizeof(double) * lb, cudaMemcpyDeviceToHost, stream), "loss");
    ck(cudaStreamSynchronize(stream), "backward");
    check_flag();
    double s = 0.0;
    for (double p : parts) s += p;
    return s / static_cast<double>(rows);
  }

  void check_flag() {
    int f = 0;
    ck(cudaMemcpy(&f, error_flag.p, sizeof(int), cudaMemcpyDeviceToHost), "error flag");
    if (f) {
      ck(cudaMemset(error_flag.p, 0, sizeof(int)), "error flag");
      throw MlpError(SPO_ERR_TIMEOUT, "mlp: a bounded wait for the tensor cores gave up");
    }
  }

  void load_rows(const float* x_dev, const float* y_dev, const long long* idx_dev, long long rows) {
    gather_inputs_kernel<<<grid_for(rows * in_pad), 256, 0, stream>>>(x_dev, n_in, idx_dev, rows, in_pad, x16.p);
    if (y_dev) gather_targets_kernel<<<grid_for(rows), 256, 0, stream>>>(y_dev, idx_dev, rows, yb.p);
    ck(cudaGetLastError(), "gather");
  }

  void adam(float lr) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f - std::pow(b1, static_cast<float>(step)), c2 = 1.0f - std::pow(b2, static_cast<float>(step));
    for (auto& l : layers) {
      const long long nw = static_cast<long long>(l->in) * l->out;
      adam_kernel<<<grid_for(nw), 256, 0, stream>>>(l->w.p, l->gw.p, l->mw.p, l->vw.p, nw, lr, b1, b2, c1, c2, eps);
      adam_kernel<<<grid_for(l->out), 256, 0, stream>>>(l->b.p, l->gb.p, l->mb.p, l->vb.p, l->out, lr, b1, b2, c1, c2, eps);
    }
    adam_kernel<<<grid_for(width), 256, 0, stream>>>(wo.p, gwo.p, mwo.p, vwo.p, width, lr, b1, b2, c1, c2, eps);
    adam_kernel<<<1, 256, 0, stream>>>(bo.p, gbo.p, mbo.p, vbo.p, 1, lr, b1, b2, c1, c2, eps);
    ck(cudaGetLastError(), "adam");
    refresh_bf16();
  }

  // Parameter transfer in the documented order.
  template <typename F>
  void for_each_param(F&& f) {
    for (auto& l : layers) {
      f(l->w, l->gw, static_cast<long long>(l->in) * l->out);
      f(l->b, l->gb, l->out);
    }
    f(wo, gwo, width);
    f(bo, gbo, 1);
  }
};

namespace {
std::string g_mlp_error;

template <typename F>
int guarded_mlp(spo_mlp* m, F&& f) {
  if (!m) return SPO_ERR_INVALID;
  try {
    ck(cudaSetDevice(m->device), "cudaSetDevice");
    f();
    return SPO_OK;
  } catch (const MlpError& e) {
    m->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    m->err = e.what();
    return SPO_ERR_DEVICE;
  }
}

// splitmix64, for the initial weights and the batch order.
struct SplitMix {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};
}  // namespace

extern "C" {

const char* spo_mlp_last_error(const spo_mlp* m) { return m ? m->err.c_str() : g_mlp_error.c_str(); }

int spo_mlp_create(int n_in, int width, int depth, unsigned long long seed, int device, spo_mlp** out) {
  if (!out) return SPO_ERR_INVALID;
  *out = nullptr;
  auto m = std::make_unique<spo_mlp>();
  try {
    need(n_in >= 1 && n_in <= 64, "spo_mlp_create: n_in must be 1..64");
    need(width == 64 || width == 128 || width == 256, "spo_mlp_create: width must be 64, 128 or 256");
    need(depth >= 1 && depth <= 8, "spo_mlp_create: depth must be 1..8");
    m->device = device;
    ck(cudaSetDevice(device), "cudaSetDevice");
    int major = 0;
    ck(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device), "compute capability");
    need(major >= 10, "spo_mlp_create: needs an sm_100 device (tcgen05)");
    ck(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaFuncSetAttribute(gemm_tn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            static_cast<int>(kGemmLaunchSmem)),
       "gemm smem");
    m->n_in = n_in;
    m->in_pad = 64;
    m->width = width;
    m->depth = depth;
    SplitMix rng{seed};
    auto init = [&](DevBuf<float>& buf, long long n, double scale) {
      std::vector<float> h(static_cast<std::size_t>(n));
      for (auto& v : h) v = static_cast<float>((2.0 * rng.uniform() - 1.0) * scale);
      buf.alloc(static_cast<std::size_t>(n));
      ck(cudaMemcpy(buf.p, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "init");
    };
    auto zeros = [&](DevBuf<float>& buf, long long n) {
      buf.alloc(static_cast<std::size_t>(n));
      ck(cudaMemset(buf.p, 0, sizeof(float) * n), "init");
    };
    for (int l = 0; l < depth; ++l) {
      auto L = std::make_unique<Layer>();
      L->in = l == 0 ? m->in_pad : width;
      L->out = width;
      const long long nw = static_cast<long long>(L->in) * L->out;
      const int fan_in = l == 0 ? n_in : width;
      init(L->w, nw, 1.0 / std::sqrt(static_cast<double>(fan_in)));
      if (l == 0) {  // the padded input columns carry no weight
        std::vector<float> h(static_cast<std::size_t>(nw));
        ck(cudaMemcpy(h.data(), L->w.p, sizeof(float) * nw, cudaMemcpyDeviceToHost), "init");
        for (int r = 0; r < L->out; ++r)
          for (int c = n_in; c < L->in; ++c) h[static_cast<std::size_t>(r) * L->in + c] = 0.0f;
        ck(cudaMemcpy(L->w.p, h.data(), sizeof(float) * nw, cudaMemcpyHostToDevice), "init");
      }
      zeros(L->b, L->out);
      zeros(L->gw, nw);
      zeros(L->gb, L->out);
      zeros(L->mw, nw);
      zeros(L->vw, nw);
      zeros(L->mb, L->out);
      zeros(L->vb, L->out);
      L->wb.alloc(static_cast<std::size_t>(nw));
      L->wt.alloc(static_cast<std::size_t>(nw));
      m->layers.push_back(std::move(L));
    }
    init(m->wo, width, 1.0 / std::sqrt(static_cast<double>(width)));
    zeros(m->bo, 1);
    zeros(m->gwo, width);
    zeros(m->gbo, 1);
    zeros(m->mwo, width);
    zeros(m->vwo, width);
    zeros(m->mbo, 1);
    zeros(m->vbo, 1);
    m->error_flag.alloc(1);
    ck(cudaMemset(m->error_flag.p, 0, sizeof(int)), "error flag");
    m->partials.alloc(static_cast<std::size_t>(64) * width * std::max(width, m->in_pad));
    m->refresh_bf16();
    ck(cudaStreamSynchronize(m->stream), "create");
  } catch (const MlpError& e) {
    g_mlp_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_mlp_error = e.what();
    return SPO_ERR_DEVICE;
  }
  *out = m.release();
  return SPO_OK;
}

int spo_mlp_destroy(spo_mlp* m) {
  if (!m) return SPO_OK;
  cudaSetDevice(m->device);
  delete m;
  return SPO_OK;
}

int spo_mlp_parameter_count(const spo_mlp* m, long long* n) {
  if (!m || !n) return SPO_ERR_INVALID;
  *n = m->parameter_count();
  return SPO_OK;
}

int spo_mlp_input_width(const spo_mlp* m, int* n) {
  if (!m || !n) return SPO_ERR_INVALID;
  *n = m->in_pad;
  return SPO_OK;
}

int spo_mlp_get_parameters(spo_mlp* m, float* out) {
  return guarded_mlp(m, [&] {
    need(out != nullptr, "null pointer");
    long long off = 0;
    m->for_each_param([&](DevBuf<float>& p, DevBuf<float>&, long long n) {
      ck(cudaMemcpy(out + off, p.p, sizeof(float) * n, cudaMemcpyDeviceToHost), "get parameters");
      off += n;
    });
  });
}

int spo_mlp_set_parameters(spo_mlp* m, const float* in) {
  return guarded_mlp(m, [&] {
    need(in != nullptr, "null pointer");
    long long off = 0;
    m->for_each_param([&](DevBuf<float>& p, DevBuf<float>&, long long n) {
      ck(cudaMemcpy(p.p, in + off, sizeof(float) * n, cudaMemcpyHostToDevice), "set parameters");
      off += n;
    });
    m->refresh_bf16();
    ck(cudaStreamSynchronize(m->stream), "set parameters");
  });
}

int spo_mlp_predict(spo_mlp* m, const float* x, long long n, float* y) {
  return guarded_mlp(m, [&] {
    need(x && y && n > 0, "spo_mlp_predict: bad arguments");
    constexpr long long chunk = 1 << 16;
    m->ensure_capacity(std::min(n, chunk));
    DevBuf<float> xd;
    xd.alloc(static_cast<std::size_t>(std::min(n, chunk) * m->n_in));
    for (long long i0 = 0; i0 < n; i0 += chunk) {
      const long long rows = std::min(chunk, n - i0);
      ck(cudaMemcpyAsync(xd.p, x + i0 * m->n_in, sizeof(float) * rows * m->n_in, cudaMemcpyHostToDevice, m->stream),
         "upload");
      m->load_rows(xd.p, nullptr, nullptr, rows);
      m->forward(rows);
      ck(cudaMemcpyAsync(y + i0, m->out.p, sizeof(float) * rows, cudaMemcpyDeviceToHost, m->stream), "download");
      ck(cudaStreamSynchronize(m->stream), "predict");
    }
    m->check_flag();
  });
}

int spo_mlp_gradients(spo_mlp* m, const float* x, const float* y, long long n, double* loss, float* grad) {
  return guarded_mlp(m, [&] {
    need(x && y && grad && n >= kBK && n <= 65536 && n % kBK == 0,
         "spo_mlp_gradients: n must be a multiple of 64, at most 65536");
    m->ensure_capacity(n);
    DevBuf<float> xd, yd;
    xd.alloc(static_cast<std::size_t>(n * m->n_in));
    yd.alloc(static_cast<std::size_t>(n));
    ck(cudaMemcpy(xd.p, x, sizeof(float) * n * m->n_in, cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(yd.p, y, sizeof(float) * n, cudaMemcpyHostToDevice), "upload");
    m->load_rows(xd.p, yd.p, nullptr, n);
    m->forward(n);
    const double l = m->backward(n);
    if (loss) *loss = l;
    long long off = 0;
    m->for_each_param([&](DevBuf<float>&, DevBuf<float>& g, long long cnt) {
      ck(cudaMemcpy(grad + off, g.p, sizeof(float) * cnt, cudaMemcpyDeviceToHost), "gradients");
      off += cnt;
    });
  });
}

int spo_mlp_train(spo_mlp* m, const float* x, const float* y, long long n, int epochs, int batch, float lr,
                  unsigned long long seed, double* last_epoch_loss) {
  return guarded_mlp(m, [&] {
    need(x && y && n >= batch && epochs > 0 && batch >= 128 && batch % 128 == 0 && batch <= 65536 && lr > 0.0f,
         "spo_mlp_train: bad arguments");
    m->ensure_capacity(batch);
    DevBuf<float> xd, yd;
    DevBuf<long long> perm;
    xd.alloc(static_cast<std::size_t>(n * m->n_in));
    yd.alloc(static_cast<std::size_t>(n));
    perm.alloc(static_cast<std::size_t>(n));
    ck(cudaMemcpy(xd.p, x, sizeof(float) * n * m->n_in, cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(yd.p, y, sizeof(float) * n, cudaMemcpyHostToDevice), "upload");
    SplitMix rng{seed};
    std::vector<long long> order(static_cast<std::size_t>(n));
    const long long steps_per_epoch = n / batch;
    const long long total_steps = steps_per_epoch * epochs;
    long long t = 0;
    double epoch_loss = 0.0;
    for (int e = 0; e < epochs; ++e) {
      for (long long i = 0; i < n; ++i) order[i] = i;
      for (long long i = n - 1; i > 0; --i) std::swap(order[i], order[rng.next() % static_cast<uint64_t>(i + 1)]);
      ck(cudaMemcpy(perm.p, order.data(), sizeof(long long) * n, cudaMemcpyHostToDevice), "order");
      epoch_loss = 0.0;
      for (long long s = 0; s < steps_per_epoch; ++s, ++t) {
        const double frac = static_cast<double>(t) / static_cast<double>(std::max<long long>(total_steps - 1, 1));
        const float rate = static_cast<float>(lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.14159265358979 * frac))));
        m->load_rows(xd.p, yd.p, perm.p + s * batch, batch);
        m->forward(batch);
        epoch_loss += m->backward(batch);
        m->adam(rate);
      }
      epoch_loss /= static_cast<double>(steps_per_epoch);
    }
    ck(cudaStreamSynchronize(m->stream), "train");
    m->check_flag();
    if (last_epoch_loss) *last_epoch_loss = epoch_loss;
  });
}

}  // extern "C"
