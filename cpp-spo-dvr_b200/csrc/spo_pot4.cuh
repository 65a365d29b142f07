// Potential step of the interaction region as a persistent kernel with register-tiled theta
// contractions (src/propagation/potential_operator.cpp:84-135, angular_transform.cpp:54-114).
//
// One block per SM slot loops over work items (a (Z, r) point and a chunk of CB (x, y) columns),
// NT * CB = 128 threads. The angular matrix M_m[theta, J] = sqrt(w_theta / nphi) P_J^m(theta) has one
// row per rotational state irot (its block m, its J), padded to NT + 4 values, so that the 16-byte
// loads of consecutive rows fall on distinct bank groups; within a row theta is stored in the order in
// which the forward tiles take it. The mixed form stages it in shared memory once per block, FP64 reads
// it through L1 (pot4_matrix_shared). Per item:
//   load:    F[irot][c] = opt_Z before(ir, irot) psi(c, irot), plus rot(dt/2) e0(c) chi(ir, iz) in the
//            initial channel (potential_operator.cpp:116-123);
//   forward: X[p][theta][c] = sum_J M_m[theta, J] F[first_m + J][c] for the slot p of every mJ block m,
//            each thread a tile of 4 theta (strided by NT / 4) x 2 columns (16 FMAs per two 16-byte
//            loads, conflict-free stores). The slots are
//            dealt to half-warps in +m / -m pairs (equal trip counts within a warp), balanced over the
//            warps by their J counts; slots without basis functions are written as zeros;
//   phi:     thread (theta, c) takes its line of NPHI slots into registers: DFT (sign +1), times
//            exp(i A) of the column's representative at the mapped phi, DFT (sign -1), back in place;
//   back:    thread irot sums over theta for all CB columns (one matrix element reused CB times, the
//            CB slot values of one theta read as 16-byte vectors), times rot(dt/2), stores psi;
//   projection onto the specular grid: projection_finalize_kernel, after this kernel.
// The back sums take theta in the tiles' order (not ascending), so the result agrees with the other
// potential kernels to rounding.
#pragma once

#include "spo_regfft.cuh"

namespace spo {

template <typename T>
struct Pot4Args {
  PotArgs<T> p;              // pointers and sizes shared with the other potential kernels
  const T* leg_rows;         // n_rot rows of NT + 4: M_m[theta, J] of irot = first_m + J, theta at position
                             // (theta % (NT / 4)) * 4 + theta / (NT / 4)
  // potential5 (mixed form): the same rows as a 12-bit high part and the FP32 rounding of the rest, so that
  // hi + lo is the FP64 matrix to ~2^-36 and each term's lo product stays well above the rounding unit of
  // the running sum (see potential5_kernel)
  const T* leg_rows12;
  const T* leg_rows_lo;
  const int* slot_first;     // per phi slot: first irot of its mJ block
  const int* slot_nj;        // per phi slot: J count (0: no basis functions)
  const int* irot_slot;      // per irot: its phi slot
  const int* fwd_sched;      // per half-warp group g (8 groups): sched_len entries, a slot or -1 (nothing)
  int sched_len;
  int chunks;                // column chunks per point
  long long n_items;         // nz_potential * nr * chunks
  int identity_maps;
  int nt_table;              // theta points of the exp(i A) table (potential5: NT, or fewer with the rest
                             // of the tile padding)
  int poll_limit;            // potential5: polls before a wait on an mbarrier gives up
  unsigned extra_tx;         // potential5: bytes announced beyond those copied (0; a failure-detection test
                             // sets it so that a barrier phase cannot complete and the wait gives up)
};

// 4 consecutive real values (16-byte aligned) and 2 consecutive complex values.
SPO_HD void ld4(const float* p, float (&o)[4]) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w;
}
SPO_HD void ld4(const double* p, double (&o)[4]) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
SPO_HD void ld2c(const float2* p, float2& a, float2& b) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  a = make_float2(q.x, q.y);
  b = make_float2(q.z, q.w);
}
SPO_HD void ld2c(const double2* p, double2& a, double2& b) {
  a = p[0];
  b = p[1];
}
SPO_HD void st2c(float2* p, float2 a, float2 b) { *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y); }
SPO_HD void st2c(double2* p, double2 a, double2 b) {
  p[0] = a;
  p[1] = b;
}

// X holds one block of NT * CB values per phi slot, each followed by 16 bytes of padding: the back sums
// of a warp read the blocks of two or three slots at once, which then start on different banks.
template <typename T>
constexpr int pot4_slot_stride(int nt, int cb) {
  return nt * cb + static_cast<int>(16 / sizeof(Vec<T>));
}

// Where the matrix rows live: shared memory in the mixed form (20 KB on config 2); in FP64 (40 KB) they
// are read through L1 instead, so that two FP64 blocks fit per SM (10.3 against 12.7 ms per launch on
// config 2, where the mixed form is fastest with them staged).
template <typename T>
constexpr bool pot4_matrix_shared() {
  return sizeof(T) == 4;
}

// Shared memory of potential4_kernel: F (n_rot CB), X (NPHI padded slot blocks), the matrix rows
// (n_rot (NT + 4), when staged), irot -> slot (n_rot ints), the schedule (8 sched_len ints).
template <typename T>
constexpr std::size_t pot4_smem(int n_rot, int nphi, int nt, int cb, int sched_len) {
  return sizeof(Vec<T>) * (static_cast<std::size_t>(n_rot) * cb + static_cast<std::size_t>(nphi) * pot4_slot_stride<T>(nt, cb)) +
         (pot4_matrix_shared<T>() ? sizeof(T) * static_cast<std::size_t>(n_rot) * (nt + 4) : 0) +
         sizeof(int) * (static_cast<std::size_t>(n_rot) + 8 * sched_len);
}

template <typename T, int NPHI, int NT, int CB>
__global__ void __launch_bounds__(NT * CB, sizeof(T) == 4 ? 3 : 1) potential4_kernel(Pot4Args<T> g) {
  using V = Vec<T>;
  static_assert(NT * CB == 128 && NT % 4 == 0 && CB % 2 == 0, "tile shape");
  constexpr int NTH = NT * CB;
  constexpr int LDL = NT + 4;
  constexpr int QUADS = NT / 4;       // theta sets of 4 per slot tile
  constexpr int PAIRS = CB / 2;       // column pairs per slot tile
  static_assert(QUADS * PAIRS == 16, "a slot tile is one half-warp");
  constexpr int SS = pot4_slot_stride<T>(NT, CB);  // X values per slot block
  const PotArgs<T>& a = g.p;
  const int n_rot = a.n_rot;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* F = reinterpret_cast<V*>(smem_raw);                   // [irot][c]
  V* X = F + n_rot * CB;                                   // [p][theta][c], slot blocks of SS values
  constexpr bool L_SHARED = pot4_matrix_shared<T>();
  T* Ls = reinterpret_cast<T*>(X + NPHI * SS);             // [irot][position of theta], rows of LDL
  // the mixed form's matrix as 12-bit high parts plus the rest, as potential5 uses it
  const T* rows = sizeof(T) == 4 ? g.leg_rows12 : g.leg_rows;
  const T* L = L_SHARED ? Ls : rows;
  int* irot_slot = reinterpret_cast<int*>(Ls + (L_SHARED ? n_rot * LDL : 0));
  int* sched = irot_slot + n_rot;                          // [group][k]
  const int tid = threadIdx.x;
  if constexpr (L_SHARED)
    for (int k = tid; k < n_rot * LDL; k += NTH) Ls[k] = rows[k];
  for (int k = tid; k < n_rot; k += NTH) irot_slot[k] = g.irot_slot[k];
  for (int k = tid; k < 8 * g.sched_len; k += NTH) sched[k] = g.fwd_sched[k];
  __syncthreads();
  // Forward tile of this thread: column pair fc (fastest), theta set fq = {fq + QUADS q, q < 4} (the
  // matrix row holds these four at positions 4 fq .. 4 fq + 3), half-warp group fg. The 8 threads of a
  // 16-byte store phase then write two adjacent theta rows of X: distinct banks.
  const int fc = tid % PAIRS;
  const int fq = (tid / PAIRS) % QUADS;
  const int fg = tid / 16;
  // phi line of this thread
  const int line_c = tid % CB;
  const int line_t = tid / CB;
  const int i0 = a.initial_channel;
  // Load tasks: task k = (irot k / PAIRS, column pair k % PAIRS); a warp's 32 tasks store 512
  // contiguous bytes of F.
  const int n_tasks = n_rot * PAIRS;
  auto load_task = [&](long long col_base, int ncol, int k, V& v0, V& v1) {
    const int irot = k / PAIRS;
    const int c = 2 * (k - irot * PAIRS);
    v0 = c < ncol ? a.psi[(col_base + c) * n_rot + irot] : cmake<V>(0, 0);
    v1 = c + 1 < ncol ? a.psi[(col_base + c + 1) * n_rot + irot] : cmake<V>(0, 0);
  };
  auto item_columns = [&](long long item, int& izr, int& c0, int& ncol, long long& col_base) {
    izr = static_cast<int>(item / g.chunks);
    const int chunk = static_cast<int>(item - static_cast<long long>(izr) * g.chunks);
    c0 = chunk * CB;
    ncol = min(CB, a.n_xy - c0);
    col_base = static_cast<long long>(izr) * a.n_xy + c0;
  };

  for (long long item = blockIdx.x; item < g.n_items; item += gridDim.x) {
    int izr, c0, ncol;
    long long col_base;
    item_columns(item, izr, c0, ncol, col_base);
    const int ir = izr % a.nr;
    const int iz = izr / a.nr;
    const T oz = a.opt_z[iz];
    // No barrier here: F is read only by the forward phase, which ended before the previous item's
    // second barrier; X is rewritten only after this item's first barrier.

    // ---- load: absorbers, rot(dt/2), the specular wave into the initial channel
    auto store_task = [&](int k, V v0, V v1) {
      const int irot = k / PAIRS;
      const int c = 2 * (k - irot * PAIRS);
      const long long n_scale = static_cast<long long>(a.nr) * n_rot;  // entries of the scaling tables
      v0 = c < ncol ? cscale(fmul_t(v0, a.before, n_scale, ir * n_rot + irot), oz) : cmake<V>(0, 0);
      v1 = c + 1 < ncol ? cscale(fmul_t(v1, a.before, n_scale, ir * n_rot + irot), oz) : cmake<V>(0, 0);
      if (irot == i0) {
        const V incoming = a.chi[izr];
        if (c < ncol) v0 = cadd(v0, fmul_t(cmul_t(incoming, a.sp2sc, a.n_xy, c0 + c), a.rot_half, n_scale, ir * n_rot + i0));
        if (c + 1 < ncol)
          v1 = cadd(v1, fmul_t(cmul_t(incoming, a.sp2sc, a.n_xy, c0 + c + 1), a.rot_half, n_scale, ir * n_rot + i0));
      }
      st2c(F + irot * CB + c, v0, v1);
    };
    // FP64: batches of 4 tasks, all their loads issued before the first is used (in the mixed form the
    // registers are taken by the exp(i A) line of the phase after next: batching there spills).
    constexpr int LB = sizeof(T) == 4 ? 1 : 4;
    for (int k0 = tid; k0 < n_tasks; k0 += NTH * LB) {
      V v0[LB], v1[LB];
#pragma unroll
      for (int i = 0; i < LB; ++i) {
        const int k = k0 + NTH * i;
        if (k < n_tasks) load_task(col_base, ncol, k, v0[i], v1[i]);
      }
#pragma unroll
      for (int i = 0; i < LB; ++i) {
        const int k = k0 + NTH * i;
        if (k < n_tasks) store_task(k, v0[i], v1[i]);
      }
    }
    __syncthreads();

    const bool has_line = line_c < ncol;

    // ---- forward theta contraction
    for (int k = 0; k < g.sched_len; ++k) {
      const int slot = sched[fg * g.sched_len + k];
      if (slot < 0) continue;  // the other half-warp has a slot here
      const int nj = __ldg(g.slot_nj + slot);
      const int first = nj > 0 ? __ldg(g.slot_first + slot) : 0;
      T acc[4][4];  // [theta q][re c0, im c0, re c1, im c1]
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[q][r] = 0;
      const T* lp = L + first * LDL + 4 * fq;
      const V* fp = F + first * CB + 2 * fc;
      for (int j = 0; j < nj; ++j) {
        T l[4];
        ld4(lp + j * LDL, l);
        V f0, f1;
        ld2c(fp + j * CB, f0, f1);
        if constexpr (sizeof(T) == 4) {
          T m[4];
          ld4(g.leg_rows_lo + (first + j) * LDL + 4 * fq, m);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            acc[q][0] = fmaf(l[q], f0.x, fmaf(m[q], f0.x, acc[q][0]));
            acc[q][1] = fmaf(l[q], f0.y, fmaf(m[q], f0.y, acc[q][1]));
            acc[q][2] = fmaf(l[q], f1.x, fmaf(m[q], f1.x, acc[q][2]));
            acc[q][3] = fmaf(l[q], f1.y, fmaf(m[q], f1.y, acc[q][3]));
          }
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            acc[q][0] += l[q] * f0.x;
            acc[q][1] += l[q] * f0.y;
            acc[q][2] += l[q] * f1.x;
            acc[q][3] += l[q] * f1.y;
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        st2c(X + slot * SS + (fq + QUADS * q) * CB + 2 * fc, cmake<V>(acc[q][0], acc[q][1]),
             cmake<V>(acc[q][2], acc[q][3]));
    }
    // Mixed form: exp(i A) of this thread's phi line (no symmetry maps), requested before the barrier,
    // so that the loads overlap the other threads' last forward tiles (FP64 has no registers to spare).
    constexpr bool EARLY_EXP = sizeof(T) == 4;
    V e[EARLY_EXP ? NPHI : 1];
    const bool direct = EARLY_EXP && g.identity_maps && has_line;
    if (direct) {
      const V* ep = a.expia + ((static_cast<long long>(izr) * a.n_rep + c0 + line_c) * NT + line_t) * NPHI;
      static_for<0, NPHI / 2>([&](auto h) { ld2c(ep + 2 * SPO_CV(h), e[2 * SPO_CV(h)], e[2 * SPO_CV(h) + 1]); });
    }
    __syncthreads();

    // ---- phi transform, exp(i A), inverse phi transform, one line per thread
    if (has_line) {
      const int ixy = c0 + line_c;
      V x[NPHI];
      V* xl = X + line_t * CB + line_c;
      static_for<0, NPHI>([&](auto p) { x[SPO_CV(p)] = xl[SPO_CV(p) * SS]; });
      rdft<NPHI, +1>(x);
      if (direct) {
        const long long e0 = ((static_cast<long long>(izr) * a.n_rep + c0 + line_c) * NT + line_t) * NPHI;
        if constexpr (EARLY_EXP)
          static_for<0, NPHI>([&](auto p) { x[SPO_CV(p)] = exp_mul(x[SPO_CV(p)], e[SPO_CV(p)], a.exp_mod, e0 + SPO_CV(p)); });
      } else if (g.identity_maps) {
        const long long e0 = ((static_cast<long long>(izr) * a.n_rep + ixy) * NT + line_t) * NPHI;
        const V* ep = a.expia + e0;
        static_for<0, NPHI / 2>([&](auto h) {
          constexpr int P = 2 * SPO_CV(h);
          V ea, eb;
          ld2c(ep + P, ea, eb);
          x[P] = exp_mul(x[P], ea, a.exp_mod, e0 + P);
          x[P + 1] = exp_mul(x[P + 1], eb, a.exp_mod, e0 + P + 1);
        });
      } else {
        const long long e0 = ((static_cast<long long>(izr) * a.n_rep + __ldg(a.rep_of + ixy)) * NT + line_t) * NPHI;
        const int* map = a.phi_map + ixy * NPHI;
        static_for<0, NPHI>([&](auto p) {
          const long long ei = e0 + __ldg(map + SPO_CV(p));
          x[SPO_CV(p)] = exp_mul(x[SPO_CV(p)], __ldg(a.expia + ei), a.exp_mod, ei);
        });
      }
      rdft<NPHI, -1>(x);
      static_for<0, NPHI>([&](auto p) { xl[SPO_CV(p) * SS] = x[SPO_CV(p)]; });
    }
    __syncthreads();

    // ---- transposed theta contraction, rot(dt/2), store
    for (int irot = tid; irot < n_rot; irot += NTH) {
      const int slot = irot_slot[irot];
      T acc[CB][2];
#pragma unroll
      for (int c = 0; c < CB; ++c) acc[c][0] = acc[c][1] = 0;
      const T* lrow = L + irot * LDL;
      const V* ys = X + slot * SS;
#pragma unroll 1
      for (int kq = 0; kq < QUADS; ++kq) {
        T l[4], m[4] = {0, 0, 0, 0};
        ld4(lrow + 4 * kq, l);  // theta kq + QUADS q, q < 4
        if constexpr (sizeof(T) == 4) ld4(g.leg_rows_lo + irot * LDL + 4 * kq, m);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const V* y = ys + (kq + QUADS * q) * CB;
#pragma unroll
          for (int c = 0; c < CB; c += 2) {
            V y0, y1;
            ld2c(y + c, y0, y1);
            if constexpr (sizeof(T) == 4) {
              acc[c][0] = fmaf(l[q], y0.x, fmaf(m[q], y0.x, acc[c][0]));
              acc[c][1] = fmaf(l[q], y0.y, fmaf(m[q], y0.y, acc[c][1]));
              acc[c + 1][0] = fmaf(l[q], y1.x, fmaf(m[q], y1.x, acc[c + 1][0]));
              acc[c + 1][1] = fmaf(l[q], y1.y, fmaf(m[q], y1.y, acc[c + 1][1]));
            } else {
              acc[c][0] += l[q] * y0.x;
              acc[c][1] += l[q] * y0.y;
              acc[c + 1][0] += l[q] * y1.x;
              acc[c + 1][1] += l[q] * y1.y;
            }
          }
        }
      }
      const long long n_scale = static_cast<long long>(a.nr) * n_rot;
#pragma unroll
      for (int c = 0; c < CB; ++c)
        if (c < ncol)
          a.psi[(col_base + c) * n_rot + irot] = fmul_t(cmake<V>(acc[c][0], acc[c][1]), a.rot_half, n_scale, ir * n_rot + irot);
    }
  }
}

}  // namespace spo
