// Potential step of the interaction region as a persistent kernel with register-tiled theta
// contractions (src/propagation/potential_operator.cpp:84-135, angular_transform.cpp:54-114).
//
// One block per SM slot loops over work items (a (Z, r) point and a chunk of CB (x, y) columns),
// NT * CB = 128 threads. The angular matrix M_m[theta, J] = sqrt(w_theta / nphi) P_J^m(theta) is
// staged in shared memory once per block, one row per rotational state irot (its block m, its J),
// theta contiguous and the row padded to NT + 4 values, so that the 16-byte loads of consecutive
// rows fall on distinct bank groups. Per item:
//   load:    F[irot][c] = opt_Z before(ir, irot) psi(c, irot), plus rot(dt/2) e0(c) chi(ir, iz) in the
//            initial channel (potential_operator.cpp:116-123);
//   forward: X[p][theta][c] = sum_J M_m[theta, J] F[first_m + J][c] for the slot p of every mJ block m,
//            each thread a tile of 4 theta x 2 columns (16 FMAs per two 16-byte loads). The slots are
//            dealt to half-warps in +m / -m pairs (equal trip counts within a warp), balanced over the
//            warps by their J counts; slots without basis functions are written as zeros;
//   phi:     thread (theta, c) takes its line of NPHI slots into registers: DFT (sign +1), times
//            exp(i A) of the column's representative at the mapped phi, DFT (sign -1), back in place;
//   back:    thread irot sums over theta for all CB columns (one matrix element reused CB times, the
//            CB slot values of one theta read as 16-byte vectors), times rot(dt/2), stores psi;
//   projection onto the specular grid: projection_finalize_kernel, after this kernel.
// Every column goes through the same operations in the same order as in potential3_kernel, so the two
// kernels give the same wave packet bit for bit.
#pragma once

#include "spo_regfft.cuh"

namespace spo {

template <typename T>
struct Pot4Args {
  PotArgs<T> p;              // pointers and sizes shared with the other potential kernels
  const T* leg_rows;         // n_rot rows of NT + 4: M_m[theta, J] of irot = first_m + J, theta contiguous
  const int* slot_first;     // per phi slot: first irot of its mJ block
  const int* slot_nj;        // per phi slot: J count (0: no basis functions)
  const int* irot_slot;      // per irot: its phi slot
  const int* fwd_sched;      // per half-warp group g (8 groups): sched_len entries, a slot or -1 (nothing)
  int sched_len;
  int chunks;                // column chunks per point
  long long n_items;         // nz_potential * nr * chunks
  int identity_maps;
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

// Shared memory of potential4_kernel: F (n_rot CB), X (NPHI NT CB), the matrix rows (n_rot (NT + 4)),
// irot -> slot (n_rot ints), the schedule (8 sched_len ints).
template <typename T>
constexpr std::size_t pot4_smem(int n_rot, int nphi, int nt, int cb, int sched_len) {
  return sizeof(Vec<T>) * (static_cast<std::size_t>(n_rot) * cb + static_cast<std::size_t>(nphi) * nt * cb) +
         sizeof(T) * static_cast<std::size_t>(n_rot) * (nt + 4) + sizeof(int) * (static_cast<std::size_t>(n_rot) + 8 * sched_len);
}

template <typename T, int NPHI, int NT, int CB>
__global__ void __launch_bounds__(NT * CB) potential4_kernel(Pot4Args<T> g) {
  using V = Vec<T>;
  static_assert(NT * CB == 128 && NT % 4 == 0 && CB % 2 == 0, "tile shape");
  constexpr int NTH = NT * CB;
  constexpr int LDL = NT + 4;
  constexpr int QUADS = NT / 4;       // theta quads per slot tile
  constexpr int PAIRS = CB / 2;       // column pairs per slot tile
  static_assert(QUADS * PAIRS == 16, "a slot tile is one half-warp");
  const PotArgs<T>& a = g.p;
  const int n_rot = a.n_rot;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V* F = reinterpret_cast<V*>(smem_raw);                   // [irot][c]
  V* X = F + n_rot * CB;                                   // [p][theta][c]
  T* L = reinterpret_cast<T*>(X + NPHI * NT * CB);         // [irot][theta], rows of LDL
  int* irot_slot = reinterpret_cast<int*>(L + n_rot * LDL);
  int* sched = irot_slot + n_rot;                          // [group][k]
  const int tid = threadIdx.x;
  for (int k = tid; k < n_rot * LDL; k += NTH) L[k] = g.leg_rows[k];
  for (int k = tid; k < n_rot; k += NTH) irot_slot[k] = g.irot_slot[k];
  for (int k = tid; k < 8 * g.sched_len; k += NTH) sched[k] = g.fwd_sched[k];
  __syncthreads();
  // forward tile of this thread: theta quad fq, column pair fc, half-warp group fg
  const int fq = tid % QUADS;
  const int fc = (tid / QUADS) % PAIRS;
  const int fg = tid / 16;
  // phi line of this thread
  const int line_c = tid % CB;
  const int line_t = tid / CB;
  const int i0 = a.initial_channel;

  for (long long item = blockIdx.x; item < g.n_items; item += gridDim.x) {
    const int izr = static_cast<int>(item / g.chunks);
    const int chunk = static_cast<int>(item - static_cast<long long>(izr) * g.chunks);
    const int ir = izr % a.nr;
    const int iz = izr / a.nr;
    const int c0 = chunk * CB;
    const int ncol = min(CB, a.n_xy - c0);
    const long long col_base = static_cast<long long>(izr) * a.n_xy + c0;
    const T oz = a.opt_z[iz];
    // No barrier here: F is read only by the forward phase, which ended before the previous item's
    // second barrier; X is rewritten only after this item's first barrier.

    // ---- load
    for (int irot = tid; irot < n_rot; irot += NTH) {
      const V b = a.before[ir * n_rot + irot];
      V v[CB];
#pragma unroll
      for (int c = 0; c < CB; ++c) {
        v[c] = c < ncol ? cscale(cmul(b, a.psi[(col_base + c) * n_rot + irot]), oz) : cmake<V>(0, 0);
      }
      if (irot == i0) {
        const V incoming = a.chi[izr];
        const V rot_i0 = a.rot_half[ir * n_rot + i0];
#pragma unroll
        for (int c = 0; c < CB; ++c)
          if (c < ncol) v[c] = cadd(v[c], cmul(rot_i0, cmul(a.sp2sc[c0 + c], incoming)));
      }
#pragma unroll
      for (int c = 0; c < CB; c += 2) st2c(F + irot * CB + c, v[c], v[c + 1]);
    }
    __syncthreads();

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
        for (int e = 0; e < 4; ++e) acc[q][e] = 0;
      const T* lp = L + first * LDL + 4 * fq;
      const V* fp = F + first * CB + 2 * fc;
      for (int j = 0; j < nj; ++j) {
        T l[4];
        ld4(lp + j * LDL, l);
        V f0, f1;
        ld2c(fp + j * CB, f0, f1);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          acc[q][0] += l[q] * f0.x;
          acc[q][1] += l[q] * f0.y;
          acc[q][2] += l[q] * f1.x;
          acc[q][3] += l[q] * f1.y;
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
        st2c(X + (slot * NT + 4 * fq + q) * CB + 2 * fc, cmake<V>(acc[q][0], acc[q][1]), cmake<V>(acc[q][2], acc[q][3]));
    }
    __syncthreads();

    // ---- phi transform, exp(i A), inverse phi transform, one line per thread
    if (line_c < ncol) {
      const int ixy = c0 + line_c;
      V x[NPHI];
      static_for<0, NPHI>([&](auto p) { x[SPO_CV(p)] = X[(SPO_CV(p) * NT + line_t) * CB + line_c]; });
      rdft<NPHI, +1>(x);
      if (g.identity_maps) {
        const V* e = a.expia + ((static_cast<long long>(izr) * a.n_rep + ixy) * NT + line_t) * NPHI;
        static_for<0, NPHI / 2>([&](auto h) {
          constexpr int P = 2 * SPO_CV(h);
          V e0, e1;
          ld2c(e + P, e0, e1);
          x[P] = cmul(e0, x[P]);
          x[P + 1] = cmul(e1, x[P + 1]);
        });
      } else {
        const V* e = a.expia + ((static_cast<long long>(izr) * a.n_rep + __ldg(a.rep_of + ixy)) * NT + line_t) * NPHI;
        const int* map = a.phi_map + ixy * NPHI;
        static_for<0, NPHI>([&](auto p) { x[SPO_CV(p)] = cmul(__ldg(e + __ldg(map + SPO_CV(p))), x[SPO_CV(p)]); });
      }
      rdft<NPHI, -1>(x);
      static_for<0, NPHI>([&](auto p) { X[(SPO_CV(p) * NT + line_t) * CB + line_c] = x[SPO_CV(p)]; });
    }
    __syncthreads();

    // ---- transposed theta contraction, rot(dt/2), store, projection share
    for (int irot = tid; irot < n_rot; irot += NTH) {
      const int slot = irot_slot[irot];
      T acc[CB][2];
#pragma unroll
      for (int c = 0; c < CB; ++c) acc[c][0] = acc[c][1] = 0;
      const T* lrow = L + irot * LDL;
      const V* ys = X + slot * NT * CB;
#pragma unroll 1
      for (int tq = 0; tq < NT; tq += 4) {
        T l[4];
        ld4(lrow + tq, l);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const V* y = ys + (tq + q) * CB;
#pragma unroll
          for (int c = 0; c < CB; c += 2) {
            V y0, y1;
            ld2c(y + c, y0, y1);
            acc[c][0] += l[q] * y0.x;
            acc[c][1] += l[q] * y0.y;
            acc[c + 1][0] += l[q] * y1.x;
            acc[c + 1][1] += l[q] * y1.y;
          }
        }
      }
      const V rh = a.rot_half[ir * n_rot + irot];
#pragma unroll
      for (int c = 0; c < CB; ++c)
        if (c < ncol) a.psi[(col_base + c) * n_rot + irot] = cmul(rh, cmake<V>(acc[c][0], acc[c][1]));
    }
  }
}

}  // namespace spo
