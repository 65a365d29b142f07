// Potential step of the interaction region, mixed form, with the item data moved by bulk asynchronous
// copies (src/propagation/potential_operator.cpp:84-135, angular_transform.cpp:54-114).
//
// potential4_kernel loads each item's wave packet and exp(i A) rows with ordinary per-thread loads when
// it needs them; with 12 warps per SM that keeps too few bytes in flight (1.8 TB/s on configuration 3).
// This kernel issues them one item ahead with cp.async.bulk (global -> shared, completion counted in
// bytes on an mbarrier), so the copies of item k + 1 run while item k computes:
//   - psi: the CB columns of the item (n_rot contiguous values each) into the F buffer, column c at
//     F + c (n_rot + 2) (the 16-byte pad puts the columns on different banks); issued for item k + 1
//     as soon as item k's forward sums have read F;
//   - exp(i A): each thread's phi line (NPHI contiguous values of its column's representative) into its
//     own row of E (rows of NPHI + 2 values: 16-byte loads of 8 consecutive rows on distinct banks);
//     issued for item k + 1 when item k's phi phase is done.
//   - the item's rows of the scaling tables (opt_r rot(dt/2) and rot(dt/2) at its r point) with the
//     columns; its opt_z value, incoming specular amplitude and sp2sc coefficients into registers when
//     the copies are issued, so that no global load sits on the path between two barriers.
// Per item: wait for F; scale it in place (absorbers, rot(dt/2), the specular wave into the initial
// channel); forward theta sums (potential4's tiles, F read column-major); wait for E; phi DFT, exp(i A),
// inverse DFT; transposed theta sums, rot(dt/2), store. The matrix rows are staged in shared memory as
// in potential4 (about 105 KB per block on configuration 3: two blocks per SM). The projection onto the
// specular grid is projection_finalize_kernel's.
//
// Every wait on an mbarrier is bounded. A block whose wait gives up sets *error_flag, waits (bounded)
// for the copies it has in flight and returns as a whole; the host reads the flag after the step.
#pragma once

#include <cstdint>

#include "spo_pot4.cuh"

namespace spo {

namespace pot5 {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrives on the barrier, announcing `bytes` more bytes of asynchronous copies for the current phase.
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 state;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 state, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 state;\n\t"
      "mbarrier.arrive.shared::cta.b64 state, [%0];\n\t}" ::"r"(smem_addr(bar))
      : "memory");
}

// Waits for the phase with the given parity to complete; false after `limit` polls (kWaitLimit by default).
constexpr int kWaitLimit = 1 << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = kWaitLimit) {
  const uint32_t addr = smem_addr(bar);
  for (int i = 0; i < limit; ++i) {
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

// Orders this thread's earlier shared-memory accesses before later asynchronous-proxy writes to them.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Asks for `bytes` (a multiple of 16, 16-byte aligned) of global memory to be brought into L2.
__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global to this CTA's
// shared memory, completing `bytes` on the barrier.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

}  // namespace pot5

// Shared memory of potential5_kernel: 2 barriers (padded to 32 bytes), F (CB columns of n_rot + 2
// values), E (NT CB rows of NPHI + 2 values), X (NPHI padded slot blocks), the scaling rows with their
// low parts (one opt_r rot(dt/2) row, two rot(dt/2) rows, CB incoming amplitudes), the matrix rows (n_rot rows of NT + 4),
// irot -> slot (n_rot ints), the slot sizes and first rows (2 NPHI ints), the schedule (8 sched_len ints).
// The L2E form keeps neither E nor the scaling rows in shared memory.
template <typename T>
constexpr std::size_t pot5_smem(int n_rot, int nphi, int nt, int cb, int sched_len, bool l2e = false) {
  return 32 + sizeof(Vec<T>) * (static_cast<std::size_t>(cb) * (n_rot + 2) +
                                (l2e ? 0 : static_cast<std::size_t>(nt) * cb * (nphi + 2)) +
                                static_cast<std::size_t>(nphi) * pot4_slot_stride<T>(nt, cb) +
                                (l2e ? 0 : 6) * static_cast<std::size_t>(n_rot) + cb) +
         sizeof(T) * static_cast<std::size_t>(n_rot) * (nt + 4) +
         sizeof(int) * (static_cast<std::size_t>(n_rot) + 2 * nphi + 8 * sched_len);
}

// The theta contractions use the matrix as a 12-bit high part (staged in shared memory) plus the FP32
// rounding of the rest (read through L1), each term as fma(hi, x, fma(lo, x, acc)): hi + lo is the FP64
// matrix to ~2^-36, and the lo products (~2^-13 of a term) stay well above the rounding unit of the sum, so
// the sums round without bias. With the matrix rounded to FP32 alone (even with each rotational state's
// sum of squares kept), the forward and transposed contractions of a physical wave packet (few rotational
// states with turning relative phases, smooth in theta, the potential varying with theta) changed its norm
// by up to ~1e-8 per step, the same sign every step: 5e-5 in P_reaction over 20000 steps of configuration 3.
// With hi + lo as an FP32 value and its small remainder, the remainders lie below half an ulp of the
// running sum and are rounded away.
//
// L2E: the exp(i A) rows are not staged in shared memory; each item's block of them is prefetched into
// L2 one item ahead (cp.async.bulk.prefetch.L2) and every thread reads its row from there at the start of
// its phi phase; the opt_r rot(dt/2) values of a thread's rotational states come one item ahead into
// registers, and its rot(dt/2) values (with their low parts) are read through L1 at the start of the back
// sums. That leaves ~72 KB of shared memory per block: three blocks (12 warps) per SM instead of two.
template <typename T, int NPHI, int NT, int CB, bool L2E = false>
__global__ void __launch_bounds__(NT * CB, L2E ? 3 : 2) potential5_kernel(Pot4Args<T> g, int* __restrict__ error_flag) {
  using V = Vec<T>;
  static_assert(sizeof(T) == 4, "the mixed form");
  static_assert(NT * CB == 128 && NT % 4 == 0 && CB % 2 == 0, "tile shape");
  constexpr int NTH = NT * CB;
  constexpr int LDL = NT + 4;
  constexpr int QUADS = NT / 4;
  constexpr int PAIRS = CB / 2;
  static_assert(QUADS * PAIRS == 16, "a slot tile is one half-warp");
  constexpr int SS = pot4_slot_stride<T>(NT, CB);
  constexpr int ERS = NPHI + 2;  // E row stride (values)
  const PotArgs<T>& a = g.p;
  const int n_rot = a.n_rot;
  const int FCS = n_rot + 2;     // F column stride (values); n_rot is even
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);  // 0: F, 1: E
  V* const F = reinterpret_cast<V*>(smem_raw + 32);  // [c][irot], columns of FCS values
  V* E = F + CB * FCS;                     // [line][phi], line = thread (not with L2E)
  V* X = E + (L2E ? 0 : NTH * ERS);        // [p][theta][c], slot blocks of SS values
  // The scaling rows hold each value and its low part (see cmul2): rows of n_rot values, then n_rot low parts.
  V* Bf = X + NPHI * SS;                   // [irot]: opt_r rot(dt/2) at the item's r point (not with L2E)
  V* R = Bf + (L2E ? 0 : 2 * n_rot);       // [item parity][irot]: rot(dt/2) at the item's r point (not with L2E)
  V* SP = R + (L2E ? 0 : 4 * n_rot);       // [c]: sp2sc(c) * chi, the item's incoming amplitudes
  T* L = reinterpret_cast<T*>(SP + CB);    // [irot][position of theta], rows of LDL
  int* irot_slot = reinterpret_cast<int*>(L + n_rot * LDL);
  int* s_nj = irot_slot + n_rot;           // [slot]: J count
  int* s_first = s_nj + NPHI;              // [slot]: first irot
  int* sched = s_first + NPHI;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int k = 0; k < 2; ++k) pot5::mbar_init(bars + k, NTH);
    pot5::mbar_init_fence();
  }
  for (int k = tid; k < n_rot * LDL; k += NTH) L[k] = g.leg_rows12[k];
  for (int k = tid; k < n_rot; k += NTH) irot_slot[k] = g.irot_slot[k];
  for (int k = tid; k < NPHI; k += NTH) {
    s_nj[k] = g.slot_nj[k];
    s_first[k] = g.slot_nj[k] > 0 ? g.slot_first[k] : 0;
  }
  for (int k = tid; k < 8 * g.sched_len; k += NTH) sched[k] = g.fwd_sched[k];
  __syncthreads();

  const int fc = tid % PAIRS;
  const int fq = (tid / PAIRS) % QUADS;
  const int fg = tid / 16;
  const int line_c = tid % CB;
  const int line_t = tid / CB;
  const int nt_table = g.nt_table;
  const int i0 = a.initial_channel;
  const uint32_t col_bytes = static_cast<uint32_t>(n_rot * sizeof(V));
  constexpr uint32_t row_bytes = NPHI * sizeof(V);
  // The item's opt_z value, incoming amplitude chi(point) and (threads c < CB) sp2sc(column c), loaded
  // when the item's copies are issued and used in its scaling phase.
  T oz = 0;
  V chi_in = cmake<V>(0, 0), sp_in = cmake<V>(0, 0), sp_lo = cmake<V>(0, 0);
  V bq[2] = {cmake<V>(0, 0), cmake<V>(0, 0)};  // L2E: opt_r rot(dt/2) of irot tid and tid + NTH
  V bql[2] = {cmake<V>(0, 0), cmake<V>(0, 0)};  // and their low parts
  V sb = cmake<V>(1, 0);  // the item's opt_r (and its low part): the scale of its opt_r rot(dt/2) row (fmul_t)
  const V one = cmake<V>(1, 0);
  const long long n_scale = static_cast<long long>(a.nr) * n_rot;  // entries of the scaling tables

  auto item_columns = [&](long long item, int& izr, int& c0, int& ncol) {
    izr = static_cast<int>(item / g.chunks);
    c0 = static_cast<int>(item - static_cast<long long>(izr) * g.chunks) * CB;
    ncol = min(CB, a.n_xy - c0);
  };
  // Every thread arrives on each barrier once per phase; the threads that copy announce their bytes.
  // Threads c < ncol copy column c; in the staged form thread CB the opt_r rot(dt/2) row, thread CB + 1 the
  // rot(dt/2) row (into R[parity]), CB + 2 its low parts, CB + 3 those of the opt_r rot(dt/2) row.
  auto issue_psi = [&](long long item, int parity_r) {
    int izr, c0, ncol;
    item_columns(item, izr, c0, ncol);
    const int ir = izr % a.nr;
    if (tid < ncol) {
      pot5::fence_proxy_async();
      pot5::mbar_arrive_tx(bars, col_bytes + (tid == 0 ? g.extra_tx : 0u));
      pot5::bulk_copy(F + tid * FCS, a.psi + (static_cast<long long>(izr) * a.n_xy + c0 + tid) * n_rot, col_bytes,
                      bars);
    } else if (!L2E && tid >= CB && tid <= CB + 3) {
      pot5::fence_proxy_async();
      pot5::mbar_arrive_tx(bars, col_bytes);
      const long long row = static_cast<long long>(ir) * n_rot;
      if (tid == CB)
        pot5::bulk_copy(Bf, a.before + row, col_bytes, bars);
      else if (tid == CB + 3)
        pot5::bulk_copy(Bf + n_rot, a.before + n_scale + row, col_bytes, bars);
      else if (tid == CB + 1)
        pot5::bulk_copy(R + parity_r * 2 * n_rot, a.rot_half + row, col_bytes, bars);
      else
        pot5::bulk_copy(R + parity_r * 2 * n_rot + n_rot, a.rot_half + n_scale + row, col_bytes, bars);
    } else {
      pot5::mbar_arrive(bars);
    }
    if constexpr (L2E) {
#pragma unroll
      for (int u = 0; u < 2; ++u)
        if (tid + u * NTH < n_rot) {
          bq[u] = a.before[static_cast<long long>(ir) * n_rot + tid + u * NTH];
          bql[u] = a.before[n_scale + static_cast<long long>(ir) * n_rot + tid + u * NTH];
        }
    }
    oz = a.opt_z[izr / a.nr];
    sb = a.before[2 * n_scale + static_cast<long long>(ir) * n_rot];
    chi_in = a.chi[izr];
    if (tid < ncol) {
      sp_in = a.sp2sc[c0 + tid];
      sp_lo = a.sp2sc[a.n_xy + c0 + tid];
    }
  };
  auto issue_exp = [&](long long item) {
    int izr, c0, ncol;
    item_columns(item, izr, c0, ncol);
    if constexpr (L2E) {  // column tid's rows (nt_table NPHI contiguous values) into L2
      if (tid < ncol) {
        const int ixy = c0 + tid;
        const int rep = g.identity_maps ? ixy : __ldg(a.rep_of + ixy);
        const long long e0 = (static_cast<long long>(izr) * a.n_rep + rep) * nt_table * NPHI;
        pot5::prefetch_l2(a.expia + e0, static_cast<uint32_t>(nt_table * row_bytes));
        // and the rows' modulus corrections (see exp_mul): 2 bytes per entry
        if ((nt_table * NPHI) % 8 == 0) pot5::prefetch_l2(a.exp_mod + e0, static_cast<uint32_t>(nt_table * NPHI * 2));
      }
      return;
    }
    if (line_c < ncol && line_t < nt_table) {
      const int ixy = c0 + line_c;
      const int rep = g.identity_maps ? ixy : __ldg(a.rep_of + ixy);
      pot5::fence_proxy_async();
      pot5::mbar_arrive_tx(bars + 1, row_bytes);
      pot5::bulk_copy(E + tid * ERS, a.expia + ((static_cast<long long>(izr) * a.n_rep + rep) * nt_table + line_t) * NPHI,
                      row_bytes, bars + 1);
    } else {
      pot5::mbar_arrive(bars + 1);
    }
  };
  // A bounded wait by every thread; true (for the whole block) when one of them gave up.
  auto wait_failed = [&](uint64_t* bar, uint32_t parity) {
    const bool ok = pot5::mbar_wait(bar, parity, g.poll_limit);
    return __syncthreads_or(!ok) != 0;
  };
  // Phase parities (bit 0: F, bit 1: E) and copies issued but not yet waited for (same bits).
  uint32_t parity = 0, pending = 0;
  auto give_up = [&]() {
    if (tid == 0) atomicExch(error_flag, 1);
    // bounded waits for this block's copies in flight, so that none lands after the block has left
    for (int k = 0; k < 2; ++k)
      if (pending >> k & 1u) pot5::mbar_wait(bars + k, parity >> k & 1u, g.poll_limit);
  };

  long long item = blockIdx.x;
  int rp = 0;  // parity of the item count: the R row the current item reads
  if (item < g.n_items) {
    issue_psi(item, rp);
    issue_exp(item);
    pending = L2E ? 1u : 3u;
  }
  for (; item < g.n_items; item += gridDim.x, rp ^= 1) {
    int izr, c0, ncol;
    item_columns(item, izr, c0, ncol);
    const long long col_base = static_cast<long long>(izr) * a.n_xy + c0;
    const int ir_item = izr % a.nr;
    // rot(dt/2) at the item's r point, then its n_rot low parts
    const V* rh_row = L2E ? a.rot_half + static_cast<long long>(ir_item) * n_rot : R + rp * 2 * n_rot;
    const long long rh_lo = L2E ? n_scale : n_rot;
    if (tid < CB) SP[tid] = cmul2(chi_in, sp_in, sp_lo);  // the previous item's scaling phase has read SP

    // ---- wait for the columns and rows, scale the columns in place (absorbers, rot(dt/2), the
    // specular wave into the initial channel)
    if (wait_failed(bars, parity & 1u)) {
      give_up();
      return;
    }
    parity ^= 1u;
    pending &= ~1u;
    // Two rotational states per pass, all their loads before the first store (the compiler cannot tell
    // that the runtime-strided stores to F miss the later loads, and would otherwise serialise them).
    {
      const V rot_i0 = rh_row[i0], rot_i0_lo = rh_row[rh_lo + i0];
      const V sbi = sb;
      for (int ia = tid; ia < n_rot; ia += 2 * NTH) {
        const int ib = ia + NTH;
        const bool has_b = ib < n_rot;
        const int irs[2] = {ia, has_b ? ib : ia};
        V b[2], bl[2], v[2][CB];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if constexpr (L2E) {
            b[u] = ia == tid ? bq[u] : a.before[static_cast<long long>(ir_item) * n_rot + irs[u]];
            bl[u] = ia == tid ? bql[u] : a.before[n_scale + static_cast<long long>(ir_item) * n_rot + irs[u]];
          } else {
            b[u] = Bf[irs[u]];
            bl[u] = Bf[n_rot + irs[u]];
          }
#pragma unroll
          for (int c = 0; c < CB; ++c) v[u][c] = F[c * FCS + irs[u]];
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          if (u == 1 && !has_b) break;
          const bool at_i0 = irs[u] == i0;
#pragma unroll
          for (int c = 0; c < CB; ++c) {
            V w = cmake<V>(0, 0);
            if (c < ncol) {
              w = cscale(fmul_parts(v[u][c], b[u], bl[u], sbi), oz);
              if (at_i0) w = cadd(w, fmul_parts(SP[c], rot_i0, rot_i0_lo, one));  // the specular wave into the initial channel
            }
            F[c * FCS + irs[u]] = w;
          }
        }
      }
    }
    __syncthreads();
    const long long next = item + gridDim.x;

    // ---- forward theta contraction
    for (int s = 0; s < g.sched_len; ++s) {
      const int slot = sched[fg * g.sched_len + s];
      if (slot < 0) continue;
      const int nj = s_nj[slot];
      const int first = s_first[slot];
      T acc[4][4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[q][r] = 0;
      const V* f0p = F + (2 * fc) * FCS + first;
      const V* f1p = f0p + FCS;
      const T* lp = L + first * LDL + 4 * fq;                 // the entries' 12-bit high parts
      const T* lq = g.leg_rows_lo + first * LDL + 4 * fq;     // and the rest (through L1)
      for (int j = 0; j < nj; ++j) {
        T l[4], m[4];
        ld4(lp + j * LDL, l);
        ld4(lq + j * LDL, m);
        const V f0 = f0p[j];
        const V f1 = f1p[j];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          acc[q][0] = fmaf(l[q], f0.x, fmaf(m[q], f0.x, acc[q][0]));
          acc[q][1] = fmaf(l[q], f0.y, fmaf(m[q], f0.y, acc[q][1]));
          acc[q][2] = fmaf(l[q], f1.x, fmaf(m[q], f1.x, acc[q][2]));
          acc[q][3] = fmaf(l[q], f1.y, fmaf(m[q], f1.y, acc[q][3]));
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        st2c(X + slot * SS + (fq + QUADS * q) * CB + 2 * fc, cmake<V>(acc[q][0], acc[q][1]),
             cmake<V>(acc[q][2], acc[q][3]));
    }
    __syncthreads();
    // the next item's columns (every thread has finished reading F)
    if (next < g.n_items) {
      issue_psi(next, rp ^ 1);
      pending |= 1u;
    }

    // ---- phi transform, exp(i A), inverse phi transform
    if constexpr (L2E) {
      if (line_c < ncol && line_t < nt_table) {  // padding lines (theta >= nt_table) hold zeros
        const int ixy = c0 + line_c;
        const int rep = g.identity_maps ? ixy : __ldg(a.rep_of + ixy);
        const long long e0 = ((static_cast<long long>(izr) * a.n_rep + rep) * nt_table + line_t) * NPHI;
        const V* eg = a.expia + e0;
        V* xl = X + line_t * CB + line_c;
        V x[NPHI];
        if (g.identity_maps) {
          V e[NPHI];  // this line's row from L2, requested before the transform
          static_for<0, NPHI / 2>([&](auto h) {
            constexpr int P = 2 * SPO_CV(h);
            const float4 q = __ldg(reinterpret_cast<const float4*>(eg + P));
            e[P] = cmake<V>(q.x, q.y);
            e[P + 1] = cmake<V>(q.z, q.w);
          });
          if constexpr (sizeof(T) == 4 && NPHI % 8 == 0) {  // the row's corrections, 16 bytes per load
            uint32_t mw[NPHI / 2];
            static_for<0, NPHI / 8>([&](auto h) {
              const uint4 q = __ldg(reinterpret_cast<const uint4*>(a.exp_mod + e0) + SPO_CV(h));
              mw[4 * SPO_CV(h)] = q.x;
              mw[4 * SPO_CV(h) + 1] = q.y;
              mw[4 * SPO_CV(h) + 2] = q.z;
              mw[4 * SPO_CV(h) + 3] = q.w;
            });
            static_for<0, NPHI>([&](auto p) { x[SPO_CV(p)] = xl[SPO_CV(p) * SS]; });
            rdft<NPHI, +1>(x);
            static_for<0, NPHI / 2>([&](auto h) {
              constexpr int P = 2 * SPO_CV(h);
              x[P] = exp_mul_m(x[P], e[P], mod_lo(mw[SPO_CV(h)]));
              x[P + 1] = exp_mul_m(x[P + 1], e[P + 1], mod_hi(mw[SPO_CV(h)]));
            });
          } else {
            static_for<0, NPHI>([&](auto p) { x[SPO_CV(p)] = xl[SPO_CV(p) * SS]; });
            rdft<NPHI, +1>(x);
            static_for<0, NPHI>([&](auto p) { x[SPO_CV(p)] = exp_mul(x[SPO_CV(p)], e[SPO_CV(p)], a.exp_mod, e0 + SPO_CV(p)); });
          }
        } else {
          const int* map = a.phi_map + ixy * NPHI;
          static_for<0, NPHI>([&](auto p) { x[SPO_CV(p)] = xl[SPO_CV(p) * SS]; });
          rdft<NPHI, +1>(x);
          static_for<0, NPHI>([&](auto p) {
            const int pm = __ldg(map + SPO_CV(p));
            x[SPO_CV(p)] = exp_mul(x[SPO_CV(p)], eg[pm], a.exp_mod, e0 + pm);
          });
        }
        rdft<NPHI, -1>(x);
        static_for<0, NPHI>([&](auto p) { xl[SPO_CV(p) * SS] = x[SPO_CV(p)]; });
      }
    } else {
    if (wait_failed(bars + 1, parity >> 1 & 1u)) {
      give_up();
      return;
    }
    parity ^= 2u;
    pending &= ~2u;
    if (line_c < ncol && line_t < nt_table) {  // padding lines (theta >= nt_table) hold zeros
      const int ixy = c0 + line_c;
      V* xl = X + line_t * CB + line_c;
      const V* el = E + tid * ERS;
      const int rep = g.identity_maps ? ixy : __ldg(a.rep_of + ixy);
      const long long e0 = ((static_cast<long long>(izr) * a.n_rep + rep) * nt_table + line_t) * NPHI;
      V x[NPHI];
      static_for<0, NPHI>([&](auto p) { x[SPO_CV(p)] = xl[SPO_CV(p) * SS]; });
      rdft<NPHI, +1>(x);
      if (g.identity_maps) {
        static_for<0, NPHI / 2>([&](auto h) {
          constexpr int P = 2 * SPO_CV(h);
          V ea, eb;
          ld2c(el + P, ea, eb);
          x[P] = exp_mul(x[P], ea, a.exp_mod, e0 + P);
          x[P + 1] = exp_mul(x[P + 1], eb, a.exp_mod, e0 + P + 1);
        });
      } else {
        const int* map = a.phi_map + ixy * NPHI;
        static_for<0, NPHI>([&](auto p) {
          const int pm = __ldg(map + SPO_CV(p));
          x[SPO_CV(p)] = exp_mul(x[SPO_CV(p)], el[pm], a.exp_mod, e0 + pm);
        });
      }
      rdft<NPHI, -1>(x);
      static_for<0, NPHI>([&](auto p) { xl[SPO_CV(p) * SS] = x[SPO_CV(p)]; });
    }
    }
    __syncthreads();
    // the next item's exp(i A) rows (every thread has read its row of this item)
    if (next < g.n_items) {
      issue_exp(next);
      if (!L2E) pending |= 2u;
    }

    // ---- transposed theta contraction, rot(dt/2), store: two rotational states per pass (irot and
    // irot + NTH), their sums interleaved as independent chains
    for (int ia = tid; ia < n_rot; ia += 2 * NTH) {
      const int ib = ia + NTH;
      const bool has_b = ib < n_rot;
      const int ibb = has_b ? ib : ia;
      const V rh[2] = {rh_row[ia], rh_row[ibb]}, rhl[2] = {rh_row[rh_lo + ia], rh_row[rh_lo + ibb]};
      T acc[2][CB][2];
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int c = 0; c < CB; ++c) acc[u][c][0] = acc[u][c][1] = 0;
      const V* ys[2] = {X + irot_slot[ia] * SS, X + irot_slot[ibb] * SS};
      const T* lrow[2] = {L + ia * LDL, L + ibb * LDL};                          // 12-bit high parts
      const T* lrest[2] = {g.leg_rows_lo + ia * LDL, g.leg_rows_lo + ibb * LDL};  // the rest, through L1
#pragma unroll 1
      for (int kq = 0; kq < QUADS; ++kq) {
        T l[2][4], m[2][4];
        ld4(lrow[0] + 4 * kq, l[0]);
        ld4(lrow[1] + 4 * kq, l[1]);
        ld4(lrest[0] + 4 * kq, m[0]);
        ld4(lrest[1] + 4 * kq, m[1]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
#pragma unroll
          for (int c = 0; c < CB; c += 2) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              V y0, y1;
              ld2c(ys[u] + (kq + QUADS * q) * CB + c, y0, y1);
              acc[u][c][0] = fmaf(l[u][q], y0.x, fmaf(m[u][q], y0.x, acc[u][c][0]));
              acc[u][c][1] = fmaf(l[u][q], y0.y, fmaf(m[u][q], y0.y, acc[u][c][1]));
              acc[u][c + 1][0] = fmaf(l[u][q], y1.x, fmaf(m[u][q], y1.x, acc[u][c + 1][0]));
              acc[u][c + 1][1] = fmaf(l[u][q], y1.y, fmaf(m[u][q], y1.y, acc[u][c + 1][1]));
            }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int irot = u == 0 ? ia : ib;
        if (u == 1 && !has_b) break;
#pragma unroll
        for (int c = 0; c < CB; ++c)
          if (c < ncol) a.psi[(col_base + c) * n_rot + irot] = fmul_parts(cmake<V>(acc[u][c][0], acc[u][c][1]), rh[u], rhl[u], one);
      }
    }
  }
}

}  // namespace spo
