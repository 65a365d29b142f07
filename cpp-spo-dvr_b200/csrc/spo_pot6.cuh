// Potential step of the interaction region, mixed form, with both theta contractions on the fifth-
// generation tensor cores (tcgen05.mma, kind::tf32, FP32 accumulators in tensor memory)
// (src/propagation/potential_operator.cpp:84-135, angular_transform.cpp:54-114).
//
// Per mJ block m the forward contraction dvr[c, theta] = sum_J M_m[theta, J] f[c, J] is a real matrix
// (the Gauss-Legendre/Legendre matrix) applied to a batch of complex columns. Here it is a GEMM whose
// rows are the real and imaginary parts of 64 (x, y) columns of one (Z, r) point (M = 128 rows, row
// 2c + comp), whose K is the block's J (padded to 8 or 16) and whose N = 16 is theta:
//     D_m[row, theta] = sum_J A_m[row, J] B_m[theta, J]
// and the transposed contraction f'[c, J] = sum_theta M_m[theta, J] x[c, theta] is the same shape with
// K = theta and N = J (padded to 16). FP32 accuracy from TF32 tensor cores (split precision): every
// operand is split into a TF32 high part (round to nearest) and the TF32-rounded remainder, and each
// product is formed as a_hi b_lo + a_lo b_hi + a_hi b_hi (the a_lo b_lo term, ~2^-22 relative, is
// dropped), accumulated in FP32.
//
// Tensor memory holds the item's whole DVR intermediate: 31 blocks x 16 theta = 496 of the 512 columns,
// lane = row. One block of 256 threads per SM (one item at a time):
//   forward: for each block m, the threads stage A_m (hi and lo, canonical K-major layout without
//            swizzle: 8-row x 16-byte core matrices) from the item's wave packet in shared memory,
//            scaled on the way (absorbers, rot(dt/2), the specular wave into the initial channel); one
//            thread issues the block's tcgen05.mma into columns 16m..16m+15 and commits to an mbarrier;
//            two A stages alternate. The wave packet arrives in 64-state chunks by bulk asynchronous
//            copies (cp.async.bulk, two chunk buffers), issued as soon as a buffer is no longer read.
//   phi:     each thread takes 4 (column, theta) lines: tcgen05.ld of its lane's values of two adjacent
//            theta for all 31 blocks, one shuffle with the partner lane (the other component) to form
//            complex values, DFT over phi (sign +1), times exp(i A) (read from L2, where it was
//            prefetched when the item started), DFT (sign -1), one shuffle back, tcgen05.st in place.
//   back:    for each slot m, the threads read its 16 theta columns from tensor memory, split them into
//            the A stage, one thread issues the transposed contraction into the same 16 columns; while
//            it runs the previous slot's result is read back, multiplied by rot(dt/2) and stored.
// The projection onto the specular grid is projection_finalize_kernel's (after this kernel), as for
// potential3/4/5.
//
// Every wait on an mbarrier is bounded. A block whose wait gives up sets *error_flag, waits (bounded)
// for its copies and tensor-core work in flight, frees its tensor memory and returns; the host reads the
// flag after the step.
#pragma once

#include <cstdint>

#include "spo_pot5.cuh"

namespace spo {

namespace pot6 {

using pot5::smem_addr;

// Round to TF32 (10 explicit mantissa bits, nearest, ties away from zero).
__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Warp-wide tensor-memory allocation of `cols` columns (address written to *slot), and its release.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t addr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(addr), "r"(cols) : "memory");
}

// Shared-memory matrix descriptor: K-major, no swizzle (version 1, base offset 0). lbo: bytes between
// core matrices adjacent in K; sbo: bytes between core matrices adjacent in M (or N).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B (K-major), N, M = 128.
constexpr uint32_t idesc_tf32(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(n >> 3) << 17) | ((128u >> 4) << 24);
}

// D[tmem] (+)= A[smem] B[smem]^T, TF32 inputs, FP32 accumulation; issued by one thread.
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
      : "memory");
}

// Arrives on the mbarrier when every earlier tcgen05.mma of this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

// Warp-wide tensor-memory loads/stores of the warp's 32 lanes (one lane per thread), consecutive columns.
__device__ __forceinline__ void tmem_ld2(uint32_t addr, uint32_t& a, uint32_t& b) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(a), "=r"(b) : "r"(addr));
}
__device__ __forceinline__ void tmem_ld8(uint32_t addr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(addr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_st2(uint32_t addr, uint32_t a, uint32_t b) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(addr), "r"(a), "r"(b) : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// The square rotational basis of a heteronuclear run with JMax = MJMax = NT - 1: blocks mJ = -(NT-1) ..
// NT-1 in this order, block b holding J = |mJ| .. NT-1 (NT - |mJ| states) at consecutive FBR indices.
template <int NT>
struct Basis {
  static constexpr int kBlocks = 2 * NT - 1;
  static constexpr int kRot = NT * NT;
  static constexpr int nj(int b) { return NT - (b < NT - 1 ? NT - 1 - b : b - (NT - 1)); }
  static constexpr int first(int b) { return b == 0 ? 0 : first(b - 1) + nj(b - 1); }
  static constexpr int kpad(int b) { return nj(b) <= 8 ? 8 : 16; }
  // Offset (floats, per limb) of block b's forward B matrix: kpad(b) x 16 values.
  static constexpr int bf_offset(int b) { return b == 0 ? 0 : bf_offset(b - 1) + kpad(b - 1) * 16; }
  static constexpr int kBfFloats = bf_offset(kBlocks - 1) + kpad(kBlocks - 1) * 16;
  static constexpr int kBbFloats = kBlocks * 16 * 16;  // N = 16 (J, padded) x K = 16 (theta) per block
};

}  // namespace pot6

template <typename T>
struct Pot6Args {
  PotArgs<T> p;          // psi, chi, sizes, scaling tables, exp(i A), symmetry maps
  const float* bf;       // forward B matrices, hi then lo (Basis::kBfFloats each), canonical layout
  const float* bb;       // transposed-contraction B matrices, hi then lo (Basis::kBbFloats each)
  int tiles;             // 64-column tiles per (Z, r) point
  long long n_items;     // nz_potential * nr * tiles
  int identity_maps;
  int poll_limit;        // polls before a wait on an mbarrier gives up
  unsigned extra_tx;     // bytes announced beyond those copied (0; a failure-detection test sets it so that
                         // a chunk's barrier phase cannot complete and the wait gives up)
};

constexpr int kPot6Tile = 64;                // columns per item (M = 128 rows: real and imaginary parts)
constexpr int kPot6Threads = 256;
constexpr int kPot6RawStride = 64 * 8 + 16;  // bytes per column of a 64-state chunk (16-byte pad)

// Shared memory of potential6_kernel (bytes): B forward and transposed (hi, lo), two A stages (hi, lo:
// 128 rows x 16 K each), two raw chunk buffers (64 columns x 64 states), two opt_r rot(dt/2) rows and two
// rot(dt/2) rows (item parity; each with its low parts, see cmul2), the item's incoming amplitudes, block
// tables (4 x 32 ints), barriers.
template <int NT>
constexpr std::size_t pot6_smem() {
  using B = pot6::Basis<NT>;
  return 4 * 2 * static_cast<std::size_t>(B::kBfFloats + B::kBbFloats) + 2 * 2 * 128 * 16 * 4 +
         2 * static_cast<std::size_t>(kPot6Tile) * kPot6RawStride + 8 * 8 * static_cast<std::size_t>(B::kRot) +
         8 * kPot6Tile + 4 * 32 * 4 + 64;
}

template <int NPHI, int NT>
__global__ void __launch_bounds__(kPot6Threads, 1) potential6_kernel(Pot6Args<float> g, int* __restrict__ error_flag) {
  using V = float2;
  using Bs = pot6::Basis<NT>;
  static_assert(NT == 16, "tiles of 16 theta (N = 16, two K steps of 8)");
  static_assert(NPHI >= 2 * NT - 1, "every mJ block has its phi slot");
  constexpr int NB = Bs::kBlocks;
  constexpr int NROT = Bs::kRot;
  constexpr int NCHUNK = NROT / 64;
  static_assert(NROT % 64 == 0, "64-state chunks");
  constexpr uint32_t kIdesc = pot6::idesc_tf32(16);
  constexpr uint32_t kStageLimb = 128 * 16 * 4;  // bytes of one limb of an A stage

  const PotArgs<float>& a = g.p;
  extern __shared__ __align__(1024) unsigned char smem[];
  float* const bf_s = reinterpret_cast<float*>(smem);                // [limb][Bs::kBfFloats]
  float* const bb_s = bf_s + 2 * Bs::kBfFloats;                      // [limb][Bs::kBbFloats]
  unsigned char* const astage = reinterpret_cast<unsigned char*>(bb_s + 2 * Bs::kBbFloats);  // [stage][limb]
  unsigned char* const raw = astage + 2 * 2 * kStageLimb;           // [buffer][column][64 states]
  V* const before_s = reinterpret_cast<V*>(raw + 2 * kPot6Tile * kPot6RawStride);  // [parity][hi, lo][irot]
  V* const rot_s = before_s + 4 * NROT;                             // [parity][hi, lo][irot]
  V* const sp_s = rot_s + 4 * NROT;                                 // [c]: sp2sc(c) chi(point)
  int* const tab = reinterpret_cast<int*>(sp_s + kPot6Tile);        // [nj | first | kpad | bf offset][block]
  uint64_t* const bars = reinterpret_cast<uint64_t*>(tab + 4 * 32);  // raw[2], fwd[2], bwd[2]
  uint32_t* const tslot = reinterpret_cast<uint32_t*>(bars + 6);
  uint64_t* const bar_raw = bars;
  uint64_t* const bar_fwd = bars + 2;
  uint64_t* const bar_bwd = bars + 4;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n_rot = a.n_rot;  // == NROT (checked on the host)
  const int n_xy = a.n_xy;
  const int i0 = a.initial_channel;

  if (warp == 0) pot6::tmem_alloc(tslot, 512);
  if (tid == 0) {
    for (int k = 0; k < 6; ++k) pot5::mbar_init(bars + k, 1);
    pot5::mbar_init_fence();
    static_for<0, NB>([&](auto bb) {
      constexpr int b = SPO_CV(bb);
      tab[b] = Bs::nj(b);
      tab[32 + b] = Bs::first(b);
      tab[64 + b] = Bs::kpad(b);
      tab[96 + b] = Bs::bf_offset(b);
    });
  }
  for (int k = tid; k < 2 * (Bs::kBfFloats + Bs::kBbFloats) / 4; k += kPot6Threads)
    reinterpret_cast<float4*>(bf_s)[k] = reinterpret_cast<const float4*>(g.bf)[k];  // bf and bb are adjacent
  pot5::fence_proxy_async();  // the B matrices, visible to the tensor core
  pot6::fence_before_sync();
  __syncthreads();
  pot6::fence_after_sync();
  const uint32_t tmem = *tslot;

  // Phase parities: bit k of `par` is the parity of the next phase of bars[k] to wait for.
  uint32_t par = 0;
  bool failed = false;
  // Outstanding work, for the bounded clean-up of a block that gives up: raw buffers with a copy issued
  // and not waited for (bits 0, 1); MMA barriers with a commit not waited for (bits 2-5).
  uint32_t pending = 0;

  auto item_of = [&](long long item, int& izr, int& c0, int& ncol) {
    izr = static_cast<int>(item / g.tiles);
    c0 = static_cast<int>(item - static_cast<long long>(izr) * g.tiles) * kPot6Tile;
    ncol = min(kPot6Tile, n_xy - c0);
  };
  // Chunk q of the item's columns into raw buffer q % 2 (thread 0): ncol copies of 512 bytes, plus for
  // q = 0 the item's opt_r rot(dt/2) row and its rot(dt/2) row (into rot_s[rp]).
  auto issue_chunk = [&](long long item, int q, int rp) {
    int izr, c0, ncol;
    item_of(item, izr, c0, ncol);
    const int ir = izr % a.nr;
    const int buf = q & 1;
    const uint32_t bytes = static_cast<uint32_t>(ncol) * 512u + (q == 0 ? 4u * NROT * 8u : 0u) + g.extra_tx;
    pot5::fence_proxy_async();
    pot5::mbar_arrive_tx(bar_raw + buf, bytes);
    const V* src = a.psi + (static_cast<long long>(izr) * n_xy + c0) * NROT + 64 * q;
    for (int c = 0; c < ncol; ++c)
      pot5::bulk_copy(raw + (buf * kPot6Tile + c) * kPot6RawStride, src + static_cast<long long>(c) * NROT, 512u,
                      bar_raw + buf);
    if (q == 0) {  // the rows and their low parts (the n_scale entries after the table)
      const long long row = static_cast<long long>(ir) * NROT, n_scale = static_cast<long long>(a.nr) * NROT;
      pot5::bulk_copy(before_s + rp * 2 * NROT, a.before + row, NROT * 8u, bar_raw + buf);
      pot5::bulk_copy(before_s + rp * 2 * NROT + NROT, a.before + n_scale + row, NROT * 8u, bar_raw + buf);
      pot5::bulk_copy(rot_s + rp * 2 * NROT, a.rot_half + row, NROT * 8u, bar_raw + buf);
      pot5::bulk_copy(rot_s + rp * 2 * NROT + NROT, a.rot_half + n_scale + row, NROT * 8u, bar_raw + buf);
    }
  };
  // The item's wave packet (ncol * 2 KB, contiguous) and exp(i A) rows into L2.
  auto prefetch_psi = [&](long long item) {
    int izr, c0, ncol;
    item_of(item, izr, c0, ncol);
    const unsigned char* src =
        reinterpret_cast<const unsigned char*>(a.psi + (static_cast<long long>(izr) * n_xy + c0) * NROT);
    const int pieces = (ncol * NROT * 8 + 16383) / 16384;
    for (int k = lane; k < pieces; k += 32) {
      const int bytes = min(16384, ncol * NROT * 8 - k * 16384);
      pot5::prefetch_l2(src + k * 16384, static_cast<uint32_t>(bytes));
    }
  };
  auto prefetch_exp = [&](long long item) {
    int izr, c0, ncol;
    item_of(item, izr, c0, ncol);
    for (int c = lane; c < ncol; c += 32) {
      const int ixy = c0 + c;
      const int rep = g.identity_maps ? ixy : __ldg(a.rep_of + ixy);
      const long long e0 = (static_cast<long long>(izr) * a.n_rep + rep) * NT * NPHI;
      pot5::prefetch_l2(a.expia + e0, static_cast<uint32_t>(NT * NPHI * 8));
      pot5::prefetch_l2(a.exp_mod + e0, static_cast<uint32_t>(NT * NPHI * 2));
    }
  };
  // A bounded wait by every thread on bars[k]; true for the whole block when one of them gave up.
  auto wait_bar = [&](int k) {
    const bool ok = pot5::mbar_wait(bars + k, par >> k & 1u, g.poll_limit);
    if (ok) {  // a phase that did not complete stays pending for the clean-up
      par ^= 1u << k;
      pending &= ~(1u << k);
    }
    return __syncthreads_or(!ok) != 0;
  };

  long long item = blockIdx.x;
  int rp = 0;  // parity of the item count: the rot(dt/2) row the current item reads
  if (item < g.n_items && tid == 0) {
    issue_chunk(item, 0, 0);
    issue_chunk(item, 1, 0);
  }
  if (item < g.n_items) pending |= 3u;

  // Thread roles. Staging (forward): t -> comp = t & 1, column c = (t >> 1) & 63, quad pair p = t >> 7.
  const int st_comp = tid & 1, st_c = (tid >> 1) & 63, st_p = tid >> 7;
  // Tensor-memory lanes: warp w reads lanes 32 (w % 4) .. + 31; row = 2c + comp.
  const int q4 = warp & 3, half = warp >> 2;
  const int row = 32 * q4 + lane;
  const int t_c = row >> 1, t_comp = row & 1;
  const uint32_t lane_addr = tmem + (static_cast<uint32_t>(32 * q4) << 16);

  for (; item < g.n_items && !failed; item += gridDim.x, rp ^= 1) {
    int izr, c0, ncol;
    item_of(item, izr, c0, ncol);
    const long long next = item + gridDim.x;
    if (warp == 0) prefetch_exp(item);
    if (warp == 1 && next < g.n_items) prefetch_psi(next);
    const float oz = a.opt_z[izr / a.nr];
    // the item's opt_r (and its low part), the scale of its opt_r rot(dt/2) row (see fmul_t)
    const V sb = a.before[2 * static_cast<long long>(a.nr) * NROT + static_cast<long long>(izr % a.nr) * NROT];
    const V one = make_float2(1.f, 0.f);
    if (tid < kPot6Tile)
      sp_s[tid] = tid < ncol ? cmul2(a.chi[izr], a.sp2sc[c0 + tid], a.sp2sc[n_xy + c0 + tid]) : make_float2(0.f, 0.f);
    uint32_t waited = 0;  // raw chunks of this item already waited for

    // ------------------------------------------------------------------ forward contraction
    for (int b = 0; b < NB && !failed; ++b) {
      const int s = b & 1;
      const int nj = tab[b], first = tab[32 + b], kpad = tab[64 + b];
      if (b >= 2 && wait_bar(2 + s)) { failed = true; break; }  // the MMAs of block b - 2 read this stage
      const int qlo = first >> 6, qhi = (first + nj - 1) >> 6;
      for (int q = qlo; q <= qhi; ++q)
        if (!(waited >> q & 1u)) {
          if (wait_bar(q & 1)) { failed = true; break; }
          waited |= 1u << q;
        }
      if (failed) break;
      // Stage A_b: thread (c, comp, p) reads the 4 states of quad 2p + comp of column c, scales them,
      // and after one exchange with its partner lane writes row 2c + comp of quads 2p and 2p + 1.
      if (st_p < kpad / 8) {
        const int kq = 2 * st_p + st_comp;
        V w[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int j = 4 * kq + e;
          const int irot = first + j;
          w[e] = make_float2(0.f, 0.f);
          if (j < nj && st_c < ncol) {
            const int qq = irot >> 6;
            const V v = *reinterpret_cast<const V*>(raw + ((qq & 1) * kPot6Tile + st_c) * kPot6RawStride +
                                                    (irot & 63) * 8);
            w[e] = cscale(fmul_parts(v, before_s[rp * 2 * NROT + irot], before_s[rp * 2 * NROT + NROT + irot], sb), oz);
            if (irot == i0)
              w[e] = cadd(w[e], fmul_parts(sp_s[st_c], rot_s[rp * 2 * NROT + i0], rot_s[rp * 2 * NROT + NROT + i0], one));
          }
        }
        // exchange: comp 0 keeps the real parts (its quad, and the partner's), comp 1 the imaginary parts
        float mine[4], other[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float send = st_comp ? w[e].x : w[e].y;
          const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
          mine[e] = st_comp ? w[e].y : w[e].x;  // my component of my quad
          other[e] = recv;                       // my component of the partner's quad
        }
        const int r = 2 * st_c + st_comp;
        unsigned char* stg = astage + s * 2 * kStageLimb;
#pragma unroll
        for (int u = 0; u < 2; ++u) {  // quads 2p (u = 0) and 2p + 1
          const float* src = (u == st_comp) ? mine : other;
          float hi[4], lo[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            hi[e] = pot6::tf32_round(src[e]);
            lo[e] = pot6::tf32_round(src[e] - hi[e]);
          }
          const int kqq = 2 * st_p + u;
          const uint32_t off = static_cast<uint32_t>((kqq * 16 + (r >> 3)) * 128 + (r & 7) * 16);
          *reinterpret_cast<float4*>(stg + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
          *reinterpret_cast<float4*>(stg + kStageLimb + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
        }
      }
      pot5::fence_proxy_async();
      pot6::fence_before_sync();
      __syncthreads();
      if (tid == 0) {
        pot6::fence_after_sync();
        const uint32_t a_hi = pot5::smem_addr(astage + s * 2 * kStageLimb), a_lo = a_hi + kStageLimb;
        const uint32_t b_hi = pot5::smem_addr(bf_s + tab[96 + b]), b_lo = b_hi + 4u * Bs::kBfFloats;
        const uint32_t d = tmem + 16u * b;
        for (int ks = 0; ks < kpad / 8; ++ks) {
          const uint64_t ah = pot6::smem_desc(a_hi + ks * 4096u, 2048u, 128u);
          const uint64_t al = pot6::smem_desc(a_lo + ks * 4096u, 2048u, 128u);
          const uint64_t bh = pot6::smem_desc(b_hi + ks * 512u, 256u, 128u);
          const uint64_t bl = pot6::smem_desc(b_lo + ks * 512u, 256u, 128u);
          pot6::mma_tf32(d, ah, bl, kIdesc, ks > 0 ? 1u : 0u);
          pot6::mma_tf32(d, al, bh, kIdesc, 1u);
          pot6::mma_tf32(d, ah, bh, kIdesc, 1u);
        }
        pot6::mma_commit(bar_fwd + s);
      }
      pending |= 1u << (2 + s);
      // A raw chunk no later block reads is refilled: the chunk two ahead, or the next item's first two.
      const int q_next = b + 1 < NB ? (tab[32 + b + 1] >> 6) : NCHUNK;
      for (int q = qlo; q < q_next; ++q) {
        if (q + 2 < NCHUNK) {
          if (tid == 0) issue_chunk(item, q + 2, rp);
          pending |= 1u << (q & 1);
        } else if (next < g.n_items && q + 2 - NCHUNK < 2) {
          if (tid == 0) issue_chunk(next, q + 2 - NCHUNK, rp ^ 1);
          pending |= 1u << (q & 1);
        }
      }
    }
    if (failed) break;
    // every forward MMA has completed when the last block's commit arrives; the other barrier's last
    // commit has then arrived too
    if (wait_bar(2 + ((NB - 1) & 1))) { failed = true; break; }
    if (wait_bar(2 + ((NB - 2) & 1))) { failed = true; break; }
    pot6::fence_after_sync();

    // ------------------------------------------------------------------ phi: DFT, exp(i A), DFT^-1
    {
      const bool valid = t_c < ncol;
      const int ixy = c0 + t_c;
      const int rep = valid ? (g.identity_maps ? ixy : __ldg(a.rep_of + ixy)) : 0;
      for (int pp = 0; pp < 4; ++pp) {
        const int th0 = 8 * half + 2 * pp;   // the pair's two lines: theta th0 (comp 0) and th0 + 1 (comp 1)
        const int th = th0 + t_comp;        // this thread's line
        const long long e0 = ((static_cast<long long>(izr) * a.n_rep + rep) * NT + th) * NPHI;
        const V* eg = a.expia + e0;
        V e[NPHI];
        float em[NPHI];  // the entries' modulus corrections (see exp_mul)
        if (valid && g.identity_maps) {
#pragma unroll
          for (int h = 0; h < NPHI / 2; ++h) {
            const float4 qv = __ldg(reinterpret_cast<const float4*>(eg + 2 * h));
            e[2 * h] = make_float2(qv.x, qv.y);
            e[2 * h + 1] = make_float2(qv.z, qv.w);
          }
#pragma unroll
          for (int h = 0; h < NPHI; ++h) em[h] = __half2float(__ldg(a.exp_mod + e0 + h)) * 5.9604644775390625e-8f;
        } else if (valid) {
          const int* map = a.phi_map + ixy * NPHI;
#pragma unroll
          for (int h = 0; h < NPHI; ++h) {
            const int pm = __ldg(map + h);
            e[h] = __ldg(eg + pm);
            em[h] = __half2float(__ldg(a.exp_mod + e0 + pm)) * 5.9604644775390625e-8f;
          }
        } else {
#pragma unroll
          for (int h = 0; h < NPHI; ++h) {
            e[h] = make_float2(0.f, 0.f);
            em[h] = 0.f;
          }
        }
        uint32_t v0[NB], v1[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) pot6::tmem_ld2(lane_addr + 16u * b + th0, v0[b], v1[b]);
        pot6::tmem_wait_ld();
        V x[NPHI];
#pragma unroll
        for (int p = 0; p < NPHI; ++p) x[p] = make_float2(0.f, 0.f);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          const float f0 = __uint_as_float(v0[b]), f1 = __uint_as_float(v1[b]);
          const float recv = __shfl_xor_sync(0xffffffffu, t_comp ? f0 : f1, 1);
          const int mj = b - (NT - 1);
          x[mj >= 0 ? mj : NPHI + mj] = t_comp ? make_float2(recv, f1) : make_float2(f0, recv);
        }
        rdft<NPHI, +1>(x);
#pragma unroll
        for (int p = 0; p < NPHI; ++p)  // x (1 + g)(1 + m), g the table entry (see exp_mul)
          x[p] = cadd(x[p], cmul2(x[p], e[p], make_float2(em[p] * (1.0f + e[p].x), em[p] * e[p].y)));
        rdft<NPHI, -1>(x);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          const int mj = b - (NT - 1);
          const V y = x[mj >= 0 ? mj : NPHI + mj];
          const float recv = __shfl_xor_sync(0xffffffffu, t_comp ? y.x : y.y, 1);
          // comp 0 stores (Re line th0, Re line th0 + 1), comp 1 (Im line th0, Im line th0 + 1)
          const uint32_t lo = __float_as_uint(t_comp ? recv : y.x), hi = __float_as_uint(t_comp ? y.y : recv);
          pot6::tmem_st2(lane_addr + 16u * b + th0, lo, hi);
        }
      }
      pot6::tmem_wait_st();
    }
    pot6::fence_before_sync();
    __syncthreads();
    pot6::fence_after_sync();

    // ------------------------------------------------------------------ transposed contraction
    const V* rot_row = rot_s + rp * 2 * NROT;  // then its NROT low parts
    auto epilogue = [&](int b) {
      // the slot's 16 J columns (comp part) of this thread's lane, J = 8 half .. + 7
      uint32_t u[8];
      pot6::tmem_ld8(lane_addr + 16u * b + 8u * half, u);
      pot6::tmem_wait_ld();
      const int nj = tab[b], first = tab[32 + b];
      V* out = a.psi + (static_cast<long long>(izr) * n_xy + c0 + t_c) * NROT + first;
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2) {
        const float ev = __uint_as_float(u[2 * s2]), od = __uint_as_float(u[2 * s2 + 1]);
        const float recv = __shfl_xor_sync(0xffffffffu, t_comp ? ev : od, 1);
        // comp 0: J = 8 half + 2 s2 (Re ev, Im recv); comp 1: J + 1 (Re recv, Im od)
        const int j = 8 * half + 2 * s2 + t_comp;
        const V y = t_comp ? make_float2(recv, od) : make_float2(ev, recv);
        if (j < nj && t_c < ncol) out[j] = fmul_parts(y, rot_row[first + j], rot_row[NROT + first + j], one);
      }
    };
    for (int b = 0; b < NB && !failed; ++b) {
      const int s = b & 1;
      // stage A'_b: this lane's 8 theta (8 half .. + 7), split into hi and lo
      {
        uint32_t u[8];
        pot6::tmem_ld8(lane_addr + 16u * b + 8u * half, u);
        pot6::tmem_wait_ld();
        unsigned char* stg = astage + s * 2 * kStageLimb;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
          float hi[4], lo[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float v = __uint_as_float(u[4 * kk + e]);
            hi[e] = pot6::tf32_round(v);
            lo[e] = pot6::tf32_round(v - hi[e]);
          }
          const int kq = 2 * half + kk;
          const uint32_t off = static_cast<uint32_t>((kq * 16 + (row >> 3)) * 128 + (row & 7) * 16);
          *reinterpret_cast<float4*>(stg + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
          *reinterpret_cast<float4*>(stg + kStageLimb + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);
        }
      }
      pot5::fence_proxy_async();
      pot6::fence_before_sync();
      __syncthreads();
      if (tid == 0) {
        pot6::fence_after_sync();
        const uint32_t a_hi = pot5::smem_addr(astage + s * 2 * kStageLimb), a_lo = a_hi + kStageLimb;
        const uint32_t b_hi = pot5::smem_addr(bb_s + b * 256), b_lo = b_hi + 4u * Bs::kBbFloats;
        const uint32_t d = tmem + 16u * b;
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          const uint64_t ah = pot6::smem_desc(a_hi + ks * 4096u, 2048u, 128u);
          const uint64_t al = pot6::smem_desc(a_lo + ks * 4096u, 2048u, 128u);
          const uint64_t bh = pot6::smem_desc(b_hi + ks * 512u, 256u, 128u);
          const uint64_t bl = pot6::smem_desc(b_lo + ks * 512u, 256u, 128u);
          pot6::mma_tf32(d, ah, bl, kIdesc, ks > 0 ? 1u : 0u);
          pot6::mma_tf32(d, al, bh, kIdesc, 1u);
          pot6::mma_tf32(d, ah, bh, kIdesc, 1u);
        }
        pot6::mma_commit(bar_bwd + s);
      }
      pending |= 1u << (4 + s);
      if (b >= 1) {
        if (wait_bar(4 + (s ^ 1))) { failed = true; break; }
        pot6::fence_after_sync();
        epilogue(b - 1);
      }
    }
    if (failed) break;
    if (wait_bar(4 + ((NB - 1) & 1))) { failed = true; break; }
    pot6::fence_after_sync();
    epilogue(NB - 1);
    pot6::fence_before_sync();
  }

  if (failed) {
    if (tid == 0) atomicExch(error_flag, 1);
    // bounded waits for this block's copies and tensor-core work in flight
    for (int k = 0; k < 6; ++k)
      if (pending >> k & 1u) pot5::mbar_wait(bars + k, par >> k & 1u, g.poll_limit);
  }
  pot6::fence_before_sync();
  __syncthreads();
  pot6::fence_after_sync();
  if (warp == 0) pot6::tmem_dealloc(tmem, 512);
}

}  // namespace spo
