// Host side of the B200 split-operator backend, shared by the translation units of the library: the
// error and table helpers, the kernel launchers and the Step<T> class (one wave packet resident in HBM).
// Step<float> and Step<double> are instantiated in spo_step_f32.cu and spo_step_f64.cu (compiled in
// parallel); spo_b200.cu holds the C ABI.
//
// One sub-step of the reference's schedule (src/propagation/split_operator.cpp:17-21,
// split_operator_schedule.cpp:7-13) is, on the device:
//   specular grid   3 axis passes: r forward | Z forward * factor * inverse | r inverse (+ W factors)
//   T_Z             1 axis pass over psi (Z forward * exp(-i T_Z dt) * inverse)
//   T_r             1 axis pass over psi (r forward * exp(-i T_r dt) * inverse)
//   T_xy (+ W gas)  1 pass over psi, 2D (x, y) FFT per (Z, r) point, gas-phase W fused
//   W interaction   1 pass over the interaction region (theta contraction, phi FFTs, exp(iA))
// T_Z and T_r are applied separably: the reference's 2D factor zr_kinetic is the product
// z_kinetic * r_kinetic (src/propagation/propagation_tables.cpp:157-162), so
// F_zr^-1 (z r) F_zr = (F_Z^-1 z F_Z)(F_r^-1 r F_r) exactly, up to rounding.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/spo_b200.h"
#include "spo_kernels.cuh"
#include "spo_regfft.cuh"
#include "spo_pot4.cuh"
#include "spo_pot5.cuh"
#include "spo_pot6.cuh"
#include "spo_persist.cuh"

namespace spo_host {

using cplx = std::complex<double>;

inline thread_local std::string g_create_error;

struct SpoError : std::runtime_error {
  int code;
  SpoError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) throw SpoError(SPO_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e));
  if (e != cudaSuccess) throw SpoError(SPO_ERR_DEVICE, std::string(what) + ": " + cudaGetErrorString(e));
}

inline void require(bool ok, const std::string& what) {
  if (!ok) throw SpoError(SPO_ERR_INVALID, what);
}

// Radices of a valid FFT length (2^h 3^i 5^j 7^k 11^m), fours first.
inline spo::FftPlan make_plan(int n) {
  spo::FftPlan p{};
  p.n = n;
  int m = n;
  auto push = [&](int r) {
    require(p.n_stages < spo::kMaxStages, "FFT length " + std::to_string(n) + " has too many factors");
    p.radix[p.n_stages++] = r;
  };
  while (m % 4 == 0) push(4), m /= 4;
  for (const int r : {2, 3, 5, 7, 11})
    while (m % r == 0) push(r), m /= r;
  require(m == 1, "FFT length " + std::to_string(n) + " is not 2^h 3^i 5^j 7^k 11^m");
  return p;
}

// exp(-2 pi i k / n), k < n, in FP64 (exact on the axes).
inline std::vector<cplx> twiddles(int n) {
  std::vector<cplx> t(n);
  for (int k = 0; k < n; ++k) {
    if (k == 0) t[k] = {1, 0};
    else if (4 * k == n) t[k] = {0, -1};
    else if (2 * k == n) t[k] = {-1, 0};
    else if (4 * k == 3 * n) t[k] = {0, 1};
    else {
      const double a = 2.0 * M_PI * k / n;
      t[k] = {std::cos(a), -std::sin(a)};
    }
  }
  return t;
}

inline std::vector<cplx> complex_array(const double* p, std::size_t n, const char* name) {
  require(p != nullptr, std::string("descriptor array ") + name + " is null");
  std::vector<cplx> v(n);
  for (std::size_t i = 0; i < n; ++i) v[i] = {p[2 * i], p[2 * i + 1]};
  return v;
}
inline std::vector<double> real_array(const double* p, std::size_t n, const char* name) {
  require(p != nullptr, std::string("descriptor array ") + name + " is null");
  return std::vector<double>(p, p + n);
}
inline std::vector<int> int_array(const int* p, std::size_t n, const char* name) {
  require(p != nullptr, std::string("descriptor array ") + name + " is null");
  return std::vector<int>(p, p + n);
}

// Owned device allocations of a handle.
class DeviceArena {
 public:
  ~DeviceArena() {
    for (void* p : ptrs_) cudaFree(p);
  }
  void* alloc(std::size_t bytes) {
    void* p = nullptr;
    check_cuda(cudaMalloc(&p, std::max<std::size_t>(bytes, 16)), "cudaMalloc");
    ptrs_.push_back(p);
    bytes_ += bytes;
    return p;
  }
  void release(void* p, std::size_t bytes) {
    auto it = std::find(ptrs_.begin(), ptrs_.end(), p);
    if (it == ptrs_.end()) return;
    cudaFree(p);
    ptrs_.erase(it);
    bytes_ -= bytes;
  }
  unsigned long long bytes() const { return bytes_; }

 private:
  std::vector<void*> ptrs_;
  unsigned long long bytes_ = 0;
};

struct Sizes {
  int n_rot, nx, ny, nr, nz, nzp, nzs, nt, nphi, i0, ra, rb, spa, n_rep, n_ops, n_blocks, mj_max;
  double dt;
  long long n_xy() const { return static_cast<long long>(nx) * ny; }
  long long n_zr() const { return static_cast<long long>(nz) * nr; }
  long long n_psi() const { return n_xy() * n_zr() * n_rot; }
  long long n_chi() const { return static_cast<long long>(nzs) * nr; }
  long long n_expia() const { return static_cast<long long>(nzp) * nr * n_rep * nt * nphi; }
};


// ---------------------------------------------------------------------------------------------
// Launchers of the register-DFT kernels for the sizes they are instantiated for. Each returns
// false for other sizes; the caller then uses the general shared-memory Stockham kernels.
// ---------------------------------------------------------------------------------------------
// Sets a kernel's dynamic shared-memory limit once per device (the attribute is per device context).
template <typename K>
void allow_smem(K kernel, std::size_t bytes, unsigned long long& done_mask, const char* what) {
  int dev = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 64 && (done_mask >> dev & 1ull)) return;
  check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)), what);
  if (dev < 64) done_mask |= 1ull << dev;
}

// The device's largest dynamic shared memory per block (opt-in).
inline std::size_t smem_optin_bytes() {
  int dev = 0, optin = 0;
  check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  check_cuda(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev), "smem attribute");
  return static_cast<std::size_t>(optin);
}

// Blocks of a persistent kernel: the SMs times the blocks that fit on one (looked up once per kernel).
template <typename K>
long long persistent_blocks(K kernel, int threads, std::size_t smem, int& cached) {
  if (cached <= 0) {
    int dev = 0, sms = 0, per_sm = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem), "occupancy");
    cached = std::max(1, sms * per_sm);
  }
  return cached;
}

template <typename T, int N1, int N2, int TB>
bool launch_axis2_tb(const spo::Axis2Args<T>& a, long long outer, cudaStream_t stream) {
  constexpr int NS = N1 > N2 ? N1 : N2;
  constexpr int N = N1 * N2;
  // the tile, then the factors (mixed form: their parts, spo::fmul_t) and the twiddles (mixed form: and their low parts)
  const std::size_t smem =
      sizeof(spo::Vec<T>) * (static_cast<std::size_t>(N) * TB + (sizeof(T) == 4 ? spo::kFactorParts + 2 : 2) * N);
  static unsigned long long configured = 0;
  allow_smem(spo::axis2_kernel<T, N1, N2, TB>, smem, configured, "axis2 smem");
  if (a.persistent && a.window == 0) {
    static unsigned long long configured_p = 0;
    static int blocks_p = 0;
    allow_smem(spo::axis2p_kernel<T, N1, N2, TB>, smem, configured_p, "axis2p smem");
    const long long lane_blocks = (a.inner + TB - 1) / TB;
    const long long n_tiles = outer * lane_blocks;
    const long long grid = std::min(n_tiles, persistent_blocks(spo::axis2p_kernel<T, N1, N2, TB>, TB * NS, smem, blocks_p));
    spo::axis2p_kernel<T, N1, N2, TB><<<static_cast<unsigned>(grid), TB * NS, smem, stream>>>(a, lane_blocks, n_tiles);
    return true;
  }
  if constexpr (N2 == 2 * N1) {
    if (a.balanced && a.window == 0) {
      static unsigned long long configured_b = 0;
      allow_smem(spo::axis2b_kernel<T, N1, N2, TB>, smem, configured_b, "axis2b smem");
      const dim3 grid(static_cast<unsigned>((a.inner + TB - 1) / TB), static_cast<unsigned>(outer));
      spo::axis2b_kernel<T, N1, N2, TB><<<grid, TB * N1, smem, stream>>>(a);
      return true;
    }
  }
  if (a.window > 0) {  // lane windows: groups x ceil(window / TB) blocks
    spo::Axis2Args<T> w = a;
    w.blocks_per_group = static_cast<int>((a.window + TB - 1) / TB);
    const dim3 grid(static_cast<unsigned>(a.groups * w.blocks_per_group), static_cast<unsigned>(outer));
    spo::axis2_kernel<T, N1, N2, TB><<<grid, TB * NS, smem, stream>>>(w);
    return true;
  }
  const dim3 grid(static_cast<unsigned>((a.inner + TB - 1) / TB), static_cast<unsigned>(outer));
  spo::axis2_kernel<T, N1, N2, TB><<<grid, TB * NS, smem, stream>>>(a);
  return true;
}

// Tile width (batch lanes per block): 32 lanes when a line has at most 8 sub-rows; for more sub-rows
// 16 lanes by default, or 8 or 32 lanes as the autotuner chose.
template <typename T, int N1, int N2>
bool launch_axis2_n(const spo::Axis2Args<T>& a, long long outer, cudaStream_t stream) {
  constexpr int NS = N1 > N2 ? N1 : N2;
  if constexpr (NS <= 8) {
    return launch_axis2_tb<T, N1, N2, 32>(a, outer, stream);
  } else {
    if (a.tile == 8) return launch_axis2_tb<T, N1, N2, 8>(a, outer, stream);
    if (a.tile == 32) return launch_axis2_tb<T, N1, N2, 32>(a, outer, stream);
    return launch_axis2_tb<T, N1, N2, 16>(a, outer, stream);
  }
}

// The prime-factor splits N = N1 x N2 (N1, N2 coprime) with an axis2pfa_kernel instantiation; LT threads per
// batch lane (LT >= N1).
inline bool pfa_split(int n, int& n1, int& n2) {
  switch (n) {
    case 24: n1 = 3; n2 = 8; return true;
    case 40: n1 = 5; n2 = 8; return true;
    case 48: n1 = 3; n2 = 16; return true;
    case 56: n1 = 7; n2 = 8; return true;
    case 80: n1 = 5; n2 = 16; return true;
    case 112: n1 = 7; n2 = 16; return true;
    default: return false;
  }
}
// Position k1 + N1 k2 of the prime-factor order holds the factor of momentum index
// k = (N2 u k1 + N1 v k2) mod N, u = N2^-1 mod N1, v = N1^-1 mod N2 (axis2pfa_kernel).
template <typename C>
std::vector<C> pfa_order(const std::vector<C>& f, int n1, int n2) {
  const int n = n1 * n2, u = spo::pfa_inverse(n2 % n1, n1), v = spo::pfa_inverse(n1 % n2, n2);
  std::vector<C> out(f.size());
  for (int k1 = 0; k1 < n1; ++k1)
    for (int k2 = 0; k2 < n2; ++k2) out[k1 + n1 * k2] = f[(static_cast<long long>(n2) * u * k1 + static_cast<long long>(n1) * v * k2) % n];
  return out;
}
template <typename T, int N1, int N2, int LT>
bool launch_axis2_pfa_n(const spo::Axis2Args<T>& a, long long outer, cudaStream_t stream) {
  constexpr int TB = 32, N = N1 * N2;
  const std::size_t smem = sizeof(spo::Vec<T>) * (static_cast<std::size_t>(N) * TB + (sizeof(T) == 4 ? spo::kFactorParts : 1) * N);
  static unsigned long long configured = 0;
  allow_smem(spo::axis2pfa_kernel<T, N1, N2, TB, LT>, smem, configured, "axis2pfa smem");
  spo::Axis2Args<T> w = a;
  unsigned blocks_x;
  if (a.window > 0) {
    w.blocks_per_group = static_cast<int>((a.window + TB - 1) / TB);
    blocks_x = static_cast<unsigned>(a.groups * w.blocks_per_group);
  } else {
    blocks_x = static_cast<unsigned>((a.inner + TB - 1) / TB);
  }
  spo::axis2pfa_kernel<T, N1, N2, TB, LT><<<dim3(blocks_x, static_cast<unsigned>(outer)), TB * LT, smem, stream>>>(w);
  return true;
}
template <typename T>
bool launch_axis2_pfa(int n, const spo::Axis2Args<T>& a, long long outer, cudaStream_t stream) {
  switch (n) {
    case 24: return launch_axis2_pfa_n<T, 3, 8, 4>(a, outer, stream);
    case 40: return launch_axis2_pfa_n<T, 5, 8, 8>(a, outer, stream);
    case 48: return launch_axis2_pfa_n<T, 3, 16, 4>(a, outer, stream);
    case 56: return launch_axis2_pfa_n<T, 7, 8, 8>(a, outer, stream);
    case 80: return launch_axis2_pfa_n<T, 5, 16, 8>(a, outer, stream);
    case 112: return launch_axis2_pfa_n<T, 7, 16, 8>(a, outer, stream);
    default: return false;
  }
}

template <typename T>
bool launch_axis2(int n, const spo::Axis2Args<T>& a, long long outer, cudaStream_t stream) {
  if (a.factor_pfa && !a.persistent) return launch_axis2_pfa<T>(n, a, outer, stream);
  switch (n) {
    // N = N1 N2 with N2 >= N1: the first level, which streams the tile in from HBM, uses every thread.
    case 24: return launch_axis2_n<T, 4, 6>(a, outer, stream);
    case 32: return launch_axis2_n<T, 4, 8>(a, outer, stream);
    case 40: return launch_axis2_n<T, 5, 8>(a, outer, stream);
    case 48: return launch_axis2_n<T, 6, 8>(a, outer, stream);
    case 56: return launch_axis2_n<T, 7, 8>(a, outer, stream);
    case 64: return launch_axis2_n<T, 8, 8>(a, outer, stream);
    case 80: return launch_axis2_n<T, 8, 10>(a, outer, stream);
    case 96: return launch_axis2_n<T, 8, 12>(a, outer, stream);
    case 112: return launch_axis2_n<T, 7, 16>(a, outer, stream);
    case 128: return launch_axis2_n<T, 8, 16>(a, outer, stream);
    case 160: return launch_axis2_n<T, 10, 16>(a, outer, stream);
    case 176: return launch_axis2_n<T, 11, 16>(a, outer, stream);
    case 192: return launch_axis2_n<T, 12, 16>(a, outer, stream);
    case 224: return launch_axis2_n<T, 14, 16>(a, outer, stream);
    case 256: return launch_axis2_n<T, 16, 16>(a, outer, stream);
    default: return false;
  }
}
// Lengths whose register kernel has more than 8 sub-rows, i.e. a choice of tile widths.
inline bool axis2_has_tiles(int n) {
  switch (n) {
    case 80: case 96: case 112: case 128: case 160: case 176: case 192: case 224: case 256: return true;
    default: return false;
  }
}
// Lengths N1 x 2 N1, which have the balanced form (axis2b_kernel).
inline bool axis2_balanced(int n) { return n == 32 || n == 128; }
inline bool axis2_supported(int n) {
  switch (n) {
    case 24: case 32: case 40: case 48: case 56: case 64: case 80: case 96: case 112: case 128: case 160: case 176:
    case 192: case 224: case 256: return true;
    default: return false;
  }
}

inline bool xy2_supported(int n) { return n == 2 || n == 4 || n == 6 || n == 8 || n == 12 || n == 16; }

template <typename T, int NX, int NY, int TB>
void launch_xy2_tb(const spo::XyArgs<T>& a, long long n_zr, cudaStream_t stream) {
  constexpr int NS = NX > NY ? NX : NY;
  const std::size_t smem =
      sizeof(spo::Vec<T>) * (static_cast<std::size_t>(NX * NY) * TB + (sizeof(T) == 4 ? spo::kFactorParts : 1) * NX * NY);
  if (a.persistent) {
    static unsigned long long configured_p = 0;
    static int blocks_p = 0;
    allow_smem(spo::xy2p_kernel<T, NX, NY, TB>, smem, configured_p, "xy2p smem");
    const long long rot_tiles = (a.n_rot + TB - 1) / TB;
    const long long n_tiles = n_zr * rot_tiles;
    const long long grid = std::min(n_tiles, persistent_blocks(spo::xy2p_kernel<T, NX, NY, TB>, TB * NS, smem, blocks_p));
    spo::xy2p_kernel<T, NX, NY, TB><<<static_cast<unsigned>(grid), TB * NS, smem, stream>>>(a, rot_tiles, n_tiles);
    return;
  }
  static unsigned long long configured = 0;
  allow_smem(spo::xy2_kernel<T, NX, NY, TB>, smem, configured, "xy2 smem");
  const dim3 grid(static_cast<unsigned>((a.n_rot + TB - 1) / TB), static_cast<unsigned>(n_zr));
  spo::xy2_kernel<T, NX, NY, TB><<<grid, TB * NS, smem, stream>>>(a);
}

template <typename T, int NX, int NY>
void launch_xy2_n(const spo::XyArgs<T>& a, long long n_zr, cudaStream_t stream) {
  constexpr int NS = NX > NY ? NX : NY;
  if constexpr (NS <= 8) {
    launch_xy2_tb<T, NX, NY, 32>(a, n_zr, stream);
  } else {
    if (a.tile == 8) launch_xy2_tb<T, NX, NY, 8>(a, n_zr, stream);
    else if (a.tile == 32) launch_xy2_tb<T, NX, NY, 32>(a, n_zr, stream);
    else launch_xy2_tb<T, NX, NY, 16>(a, n_zr, stream);
  }
}

template <typename T>
bool launch_xy2(const spo::XyArgs<T>& a, long long n_zr, cudaStream_t stream) {
  if (a.nx != a.ny) return false;
  switch (a.nx) {
    case 2: launch_xy2_n<T, 2, 2>(a, n_zr, stream); return true;
    case 4: launch_xy2_n<T, 4, 4>(a, n_zr, stream); return true;
    case 6: launch_xy2_n<T, 6, 6>(a, n_zr, stream); return true;
    case 8: launch_xy2_n<T, 8, 8>(a, n_zr, stream); return true;
    case 12: launch_xy2_n<T, 12, 12>(a, n_zr, stream); return true;
    case 16: launch_xy2_n<T, 16, 16>(a, n_zr, stream); return true;
    default: return false;
  }
}

// Shared memory of potential2_kernel<T, NPHI, CB>.
template <typename T>
std::size_t pot2_smem(int cb, int n_rot, int nt, int nphi, long long n_xy) {
  return sizeof(spo::Vec<T>) * (static_cast<std::size_t>(cb) * n_rot + static_cast<std::size_t>(cb) * nt * (nphi + 1) +
                                n_xy + 32) +
         (sizeof(T) == 4 ? 2 : 1) * sizeof(T) * static_cast<std::size_t>(nt) * n_rot;  // matrix (+ low parts)
}

template <typename T, int NPHI, int CB>
void launch_pot2_n(const spo::Pot2Args<T>& a, unsigned blocks, std::size_t smem, cudaStream_t stream) {
  // The shared memory depends on the case's sizes, not only on the instantiation: allow the device's
  // maximum, so that every case with this instantiation can launch.
  static unsigned long long configured = 0;
  allow_smem(spo::potential2_kernel<T, NPHI, CB>, smem_optin_bytes(), configured, "potential2 smem");
  spo::potential2_kernel<T, NPHI, CB><<<blocks, 128, smem, stream>>>(a);
}

template <typename T, int NPHI>
void launch_pot2_phi(const spo::Pot2Args<T>& a, unsigned blocks, std::size_t smem, cudaStream_t stream) {
  switch (a.cb) {
    case 32: launch_pot2_n<T, NPHI, 32>(a, blocks, smem, stream); break;
    case 8: launch_pot2_n<T, NPHI, 8>(a, blocks, smem, stream); break;
    default: launch_pot2_n<T, NPHI, 4>(a, blocks, smem, stream); break;
  }
}

template <typename T>
void launch_pot2(int nphi, const spo::Pot2Args<T>& a, unsigned blocks, std::size_t smem, cudaStream_t stream) {
  switch (nphi) {
    case 6: launch_pot2_phi<T, 6>(a, blocks, smem, stream); break;
    case 8: launch_pot2_phi<T, 8>(a, blocks, smem, stream); break;
    case 10: launch_pot2_phi<T, 10>(a, blocks, smem, stream); break;
    case 12: launch_pot2_phi<T, 12>(a, blocks, smem, stream); break;
    case 16: launch_pot2_phi<T, 16>(a, blocks, smem, stream); break;
    case 20: launch_pot2_phi<T, 20>(a, blocks, smem, stream); break;
    case 24: launch_pot2_phi<T, 24>(a, blocks, smem, stream); break;
    case 28: launch_pot2_phi<T, 28>(a, blocks, smem, stream); break;
    case 30: launch_pot2_phi<T, 30>(a, blocks, smem, stream); break;
    case 32: launch_pot2_phi<T, 32>(a, blocks, smem, stream); break;
    default: break;
  }
}
// Shared memory of potential3_kernel<T, NPHI, CB>: F (slot-major, jp values per slot) and D share it.
template <typename T>
std::size_t pot3_smem(int cb, int jp, int nt, int nphi) {
  return sizeof(spo::Vec<T>) * std::max(static_cast<std::size_t>(cb) * (static_cast<std::size_t>(nphi) * jp + 2),
                                        static_cast<std::size_t>(cb) * nt * (nphi + 1));
}

template <typename T, int NPHI, int CB>
void launch_pot3_n(const spo::Pot2Args<T>& a, dim3 grid, unsigned threads, std::size_t smem, cudaStream_t stream) {
  static unsigned long long configured = 0;
  allow_smem(spo::potential3_kernel<T, NPHI, CB>, smem_optin_bytes(), configured, "potential3 smem");
  spo::potential3_kernel<T, NPHI, CB><<<grid, threads, smem, stream>>>(a);
}

template <typename T, int NPHI>
void launch_pot3_phi(const spo::Pot2Args<T>& a, dim3 grid, unsigned threads, std::size_t smem, cudaStream_t stream) {
  if (a.cb == 16) launch_pot3_n<T, NPHI, 16>(a, grid, threads, smem, stream);
  else launch_pot3_n<T, NPHI, 8>(a, grid, threads, smem, stream);
}

template <typename T>
void launch_pot3(int nphi, const spo::Pot2Args<T>& a, dim3 grid, unsigned threads, std::size_t smem,
                 cudaStream_t stream) {
  switch (nphi) {
    case 6: launch_pot3_phi<T, 6>(a, grid, threads, smem, stream); break;
    case 8: launch_pot3_phi<T, 8>(a, grid, threads, smem, stream); break;
    case 10: launch_pot3_phi<T, 10>(a, grid, threads, smem, stream); break;
    case 12: launch_pot3_phi<T, 12>(a, grid, threads, smem, stream); break;
    case 16: launch_pot3_phi<T, 16>(a, grid, threads, smem, stream); break;
    case 20: launch_pot3_phi<T, 20>(a, grid, threads, smem, stream); break;
    case 24: launch_pot3_phi<T, 24>(a, grid, threads, smem, stream); break;
    case 28: launch_pot3_phi<T, 28>(a, grid, threads, smem, stream); break;
    case 30: launch_pot3_phi<T, 30>(a, grid, threads, smem, stream); break;
    case 32: launch_pot3_phi<T, 32>(a, grid, threads, smem, stream); break;
    default: break;
  }
}

// The potential4 instantiation for (nphi, ntheta), or null: ntheta 16, 8 and 4 with 8, 16 and 32 columns
// per chunk, nphi 8, 16 and 32 (and 12 with ntheta 4, a phi grid of the C6v symmetry).
template <typename T>
using Pot4Kernel = void (*)(spo::Pot4Args<T>);
template <typename T>
Pot4Kernel<T> pot4_kernel_for(int nphi, int nt) {
  if (nt == 16 && nphi == 32) return spo::potential4_kernel<T, 32, 16, 8>;
  if (nt == 16 && nphi == 16) return spo::potential4_kernel<T, 16, 16, 8>;
  if (nt == 8 && nphi == 16) return spo::potential4_kernel<T, 16, 8, 16>;
  if (nt == 8 && nphi == 32) return spo::potential4_kernel<T, 32, 8, 16>;
  if (nt == 4 && nphi == 8) return spo::potential4_kernel<T, 8, 4, 32>;
  if (nt == 4 && nphi == 12) return spo::potential4_kernel<T, 12, 4, 32>;  // C6v grids
  return nullptr;
}

// The potential5 instantiation (mixed form only) for (nphi, ntheta), or null.
template <typename T>
using Pot5Kernel = void (*)(spo::Pot4Args<T>, int*);
template <typename T>
Pot5Kernel<T> pot5_kernel_for(int nphi, int nt, bool l2e) {
  if constexpr (sizeof(T) != 4) {
    return nullptr;
  } else {
    if (l2e) {
      if (nt == 16 && nphi == 32) return spo::potential5_kernel<T, 32, 16, 8, true>;
      if (nt == 16 && nphi == 28) return spo::potential5_kernel<T, 28, 16, 8, true>;
      if (nt == 16 && nphi == 24) return spo::potential5_kernel<T, 24, 16, 8, true>;
    }
    if (nt == 16 && nphi == 32) return spo::potential5_kernel<T, 32, 16, 8>;
    if (nt == 16 && nphi == 28) return spo::potential5_kernel<T, 28, 16, 8>;  // JMax 13 (theta 14, padded)
    if (nt == 16 && nphi == 24) return spo::potential5_kernel<T, 24, 16, 8>;  // JMax 11 (theta 12, padded)
    if (nt == 8 && nphi == 16) return spo::potential5_kernel<T, 16, 8, 16>;
    if (nt == 4 && nphi == 8) return spo::potential5_kernel<T, 8, 4, 32>;
    if (nt == 4 && nphi == 12) return spo::potential5_kernel<T, 12, 4, 32>;
    return nullptr;
  }
}

inline bool pot2_phi_supported(int nphi) {
  switch (nphi) {
    case 6: case 8: case 10: case 12: case 16: case 20: case 24: case 28: case 30: case 32: return true;
    default: return false;
  }
}

// Per-kernel CUDA-event timing record.
struct KernelRecord {
  std::string name;
  double ms = 0.0;
  int launches = 0;
  double bytes = 0.0;  // algorithmic bytes of one launch
};

// CUDA events around each launch, resolved after the stream is synchronised.
class Profiler {
 public:
  ~Profiler() {
    for (cudaEvent_t e : pool_) cudaEventDestroy(e);
  }
  void enable(bool on) {
    on_ = on;
    records_.clear();
    pending_.clear();
    used_ = 0;
  }
  bool on() const { return on_; }
  // Returns the index of the pending pair; call end() after the launch.
  void begin(cudaStream_t s) {
    if (!on_) return;
    check_cuda(cudaEventRecord(event(used_), s), "cudaEventRecord");
  }
  void end(cudaStream_t s, const char* name, double bytes) {
    if (!on_) return;
    check_cuda(cudaEventRecord(event(used_ + 1), s), "cudaEventRecord");
    pending_.push_back({name, bytes, used_});
    used_ += 2;
  }
  // After a synchronisation: adds the pending durations to the records.
  void resolve() {
    if (!on_) return;
    for (const Pending& p : pending_) {
      float ms = 0.0f;
      check_cuda(cudaEventElapsedTime(&ms, pool_[p.first], pool_[p.first + 1]), "cudaEventElapsedTime");
      KernelRecord* r = nullptr;
      for (auto& x : records_)
        if (x.name == p.name) r = &x;
      if (!r) {
        records_.push_back({p.name, 0.0, 0, p.bytes});
        r = &records_.back();
      }
      r->ms += ms;
      r->launches += 1;
    }
    pending_.clear();
    used_ = 0;
  }
  const std::vector<KernelRecord>& records() const { return records_; }

 private:
  struct Pending {
    std::string name;
    double bytes;
    std::size_t first;
  };
  cudaEvent_t event(std::size_t i) {
    while (pool_.size() <= i) {
      cudaEvent_t e;
      check_cuda(cudaEventCreate(&e), "cudaEventCreate");
      pool_.push_back(e);
    }
    return pool_[i];
  }
  bool on_ = false;
  std::vector<cudaEvent_t> pool_;
  std::vector<Pending> pending_;
  std::vector<KernelRecord> records_;
  std::size_t used_ = 0;
};

// v rounded to `bits` significant bits (nearest).
inline double round_bits(double v, int bits) {
  if (v == 0.0 || !std::isfinite(v)) return v;
  int e = 0;
  std::frexp(v, &e);
  const double q = std::ldexp(1.0, e - bits);
  return std::nearbyint(v / q) * q;
}

// Rounds a matrix to FP32 row by row so that each row's sum of squares is as close to its FP64 value as
// the roundings allow: every entry takes one of its two FP32 neighbours, chosen by a meet-in-the-middle
// search over the entries' alternatives (rows of up to 24 non-zero entries; longer rows keep the nearest
// rounding). A matrix applied with its transpose at every time step (the theta contractions) then keeps the
// norm of a random state (whose rotational components have independent phases); on a physical wave packet
// the other entries of the Gram matrix still act, which is why potential5 and the small-grid kernels use
// the matrix to ~2^-36 (12-bit high parts with their remainders, or FP64 sums) and only potential4's mixed
// form uses these FP32 rows alone.
inline std::vector<float> norm_preserving_rows(const std::vector<double>& m, int rows, int stride) {
  std::vector<float> out(m.size());
  for (std::size_t i = 0; i < m.size(); ++i) out[i] = static_cast<float>(m[i]);
  for (int r = 0; r < rows; ++r) {
    const std::size_t base = static_cast<std::size_t>(r) * stride;
    double target = 0.0, have = 0.0;
    std::vector<int> idx;
    std::vector<double> delta;  // change of the sum of squares when entry idx[k] takes its other neighbour
    std::vector<float> other;
    for (int c = 0; c < stride; ++c) {
      const double v = m[base + c];
      const float f = out[base + c];
      target += v * v;
      have += static_cast<double>(f) * f;
      if (v == 0.0 || static_cast<double>(f) == v) continue;
      const float g = static_cast<double>(f) < v ? std::nextafter(f, std::numeric_limits<float>::infinity())
                                                 : std::nextafter(f, -std::numeric_limits<float>::infinity());
      idx.push_back(c);
      other.push_back(g);
      delta.push_back(static_cast<double>(g) * g - static_cast<double>(f) * f);
    }
    const int n = static_cast<int>(idx.size());
    if (n == 0 || n > 24) continue;
    const double need = target - have;
    const int na = n / 2, nb = n - na;
    std::vector<std::pair<double, unsigned>> right;
    for (unsigned mask = 0; mask < (1u << nb); ++mask) {
      double sum = 0.0;
      for (int k = 0; k < nb; ++k)
        if (mask >> k & 1u) sum += delta[na + k];
      right.emplace_back(sum, mask);
    }
    std::sort(right.begin(), right.end());
    double best = std::fabs(need);
    unsigned best_a = 0, best_b = 0;
    for (unsigned mask = 0; mask < (1u << na); ++mask) {
      double sum = 0.0;
      for (int k = 0; k < na; ++k)
        if (mask >> k & 1u) sum += delta[k];
      const double want = need - sum;
      auto it = std::lower_bound(right.begin(), right.end(), std::make_pair(want, 0u));
      for (int step = 0; step < 2; ++step, --it) {
        if (it != right.end()) {
          const double err = std::fabs(want - it->first);
          if (err < best) {
            best = err;
            best_a = mask;
            best_b = it->second;
          }
        }
        if (it == right.begin()) break;
      }
    }
    for (int k = 0; k < na; ++k)
      if (best_a >> k & 1u) out[base + idx[k]] = other[k];
    for (int k = 0; k < nb; ++k)
      if (best_b >> k & 1u) out[base + idx[na + k]] = other[na + k];
  }
  return out;
}

class StepBase {
 public:
  virtual ~StepBase() = default;
  virtual void propagate_analysis_step() = 0;
  // Queues one analysis step on the current stream without synchronising (graph capture).
  virtual void enqueue_analysis_step() = 0;
  virtual std::string describe() const = 0;
  virtual void averages(const double* z, const double* zs, const double* r, double vol_scat, double vol_spec,
                        int iz_analysis, int surface_index, double* out) = 0;
  virtual void upload(const double* psi, const double* chi) = 0;
  virtual void download(double* psi, double* chi) = 0;
  virtual void z_plane(int iz, double* out) = 0;
  virtual void block_densities(double* out) = 0;
  virtual void site_column(int ixy, double* out) = 0;
  virtual void apply_stage(int stage, bool half) = 0;
  virtual void analysis_setup(const spo_analysis_desc& d) = 0;
  virtual void bk(double time, bool fixed, int surface_index, bool accumulate, double* out) = 0;
  virtual void s_sums(double* out) = 0;
  virtual unsigned long long bytes() const = 0;
  virtual int launches() const = 0;
  virtual void set_stream(cudaStream_t s) = 0;
  virtual void profile(bool on) = 0;
  virtual void set_wait_test(int poll_limit, unsigned extra_bytes) = 0;
  virtual int norm_budget_setup(const spo_norm_budget_desc& d) = 0;
  virtual bool norm_budget_add(double* out) = 0;
  virtual int norm_budget_absorbers() const = 0;
  virtual const std::vector<KernelRecord>& records() const = 0;
};

template <typename T>
class Step final : public StepBase {
  using V = spo::Vec<T>;

 public:
  Step(const spo_desc& d, const Sizes& s, cudaStream_t stream) : s_(s), stream_(stream), own_stream_(stream) {
    build(d);
  }

  void propagate_analysis_step() override {
    enqueue_analysis_step();
    check_cuda(cudaStreamSynchronize(stream_), "propagate_analysis_step");
    prof_.resolve();
    check_device_error();
  }

  // Failure-detection test: the waits of potential5/6 give up after poll_limit polls (<= 0: the default),
  // and every item's first barrier phase expects extra_bytes more than its copies deliver.
  void set_wait_test(int poll_limit, unsigned extra_bytes) override {
    const int limit = poll_limit > 0 ? poll_limit : spo::pot5::kWaitLimit;
    pot4_args_.poll_limit = pot6_args_.poll_limit = limit;
    pot4_args_.extra_tx = pot6_args_.extra_tx = extra_bytes;
  }

  // A kernel whose bounded wait gave up has set the device flag: report it (and clear it).
  void check_device_error() {
    if (!error_flag_) return;
    int flag = 0;
    check_cuda(cudaMemcpy(&flag, error_flag_, sizeof(int), cudaMemcpyDeviceToHost), "error flag");
    if (flag) {
      check_cuda(cudaMemset(error_flag_, 0, sizeof(int)), "error flag");
      throw SpoError(SPO_ERR_TIMEOUT, std::string(pot_kind_ == 6 ? "potential6" : "potential5") +
                                          ": a bounded wait for an asynchronous copy or tensor-core work gave up");
    }
  }

  void enqueue_analysis_step() override {
    launches_ = 0;
    const int n = s_.spa;
    for (int k = 0; k <= n; ++k) {
      const bool half = k == 0 || k == n;  // T(dt/2) V, (T V) n-1 times, T(dt/2)
      const bool kinetic_only = k == n;
      sub_step(half, kinetic_only);
    }
    check_cuda(cudaGetLastError(), "propagate_analysis_step launch");
  }

  std::string describe() const override {
    auto lanes = [](int tile, bool has_tiles) { return "tb" + std::to_string(!has_tiles ? 32 : tile ? tile : 16); };
    auto axis_name = [&](int n, int tile, bool persistent) {
      if (!(use_v2_ && axis2_supported(n))) return std::string("axis_pass(general)");
      int n1 = 0, n2 = 0;
      if (use_pfa_ && !persistent && pfa_split(n, n1, n2))
        return "axis2pfa<" + std::to_string(n) + "=" + std::to_string(n1) + "x" + std::to_string(n2) + ",tb32>";
      const char* form = zr_window_ > 0 ? "axis2" : persistent ? "axis2p" : balanced_ && axis2_balanced(n) ? "axis2b" : "axis2";
      return form + std::string("<") + std::to_string(n) + "," + lanes(tile, axis2_has_tiles(n)) + ">";
    };
    std::string out = std::string(sizeof(T) == 8 ? "fp64" : "mixed");
    out += " z=" + axis_name(s_.nz, tile_z_, persist_z_);
    out += " r=" + axis_name(s_.nr, tile_r_, persist_r_);
    const bool xy2 = use_v2_ && s_.nx == s_.ny && xy2_supported(s_.nx);
    out += std::string(" xy=") + (xy2 ? std::string(persist_xy_ ? "xy2p<" : "xy2<") + std::to_string(s_.nx) + "," + lanes(tile_xy_, s_.nx > 8) + ">"
                                      : std::string("xy_pass(general)"));
    if (pot_kind_ == 6) {
      out += " potential=potential6<nphi=" + std::to_string(s_.nphi) + ",nt=" + std::to_string(s_.nt) +
             ",tcgen05.tf32x3,tile=64,blocks=" + std::to_string(pot6_blocks_) + ">";
    } else if (pot_kind_ == 5) {
      const int nt_k = (s_.nt == 12 || s_.nt == 14) ? 16 : s_.nt;  // 12 and 14 run on the 16-row tile
      out += " potential=potential5<nphi=" + std::to_string(s_.nphi) + ",nt=" + std::to_string(nt_k) +
             ",cb=" + std::to_string(128 / nt_k) + ",blocks=" + std::to_string(pot5_blocks_) + (pot5_l2e_ ? ",l2e" : "") + ">";
      if (nt_k != s_.nt) out += "(theta " + std::to_string(s_.nt) + " padded)";
    }
    else if (pot_kind_ == 4)
      out += " potential=potential4<nphi=" + std::to_string(s_.nphi) + ",nt=" + std::to_string(s_.nt) +
             ",cb=" + std::to_string(128 / s_.nt) + ",blocks=" + std::to_string(pot4_blocks_) + ">";
    else if (pot_kind_ == 3)
      out += " potential=potential3<nphi=" + std::to_string(s_.nphi) + ",cb=" + std::to_string(pot3_cb_) +
             ",chunks=" + std::to_string(pot3_chunks_) + ">";
    else if (pot_kind_ == 2)
      out += " potential=potential2<nphi=" + std::to_string(s_.nphi) + ",cb=" + std::to_string(pot2_cb_) + ">";
    else
      out += " potential=potential(general)";
    out += std::string(" balanced=") + (balanced_ ? "1" : "0") + " persistent=" + (persist_z_ ? "z" : "") + (persist_r_ ? "r" : "") + (persist_xy_ ? "xy" : "") +
           " zr_window=" + std::to_string(zr_window_) + " rxy_planes=" + std::to_string(rxy_planes_) + " tiles=" + tiles_source_ + " potential_choice=" + pot_source_;
    return out;
  }

  void upload(const double* psi, const double* chi) override {
    if (psi) copy_in(psi, psi_, s_.n_psi());
    if (chi) copy_in(chi, chi_, s_.n_chi());
    check_cuda(cudaStreamSynchronize(stream_), "upload");
  }

  void download(double* psi, double* chi) override {
    if (psi) copy_out(psi_, psi, s_.n_psi());
    if (chi) copy_out(chi_, chi, s_.n_chi());
    check_cuda(cudaStreamSynchronize(stream_), "download");
  }

  void z_plane(int iz, double* out) override {
    require(iz >= 0 && iz < s_.nz, "z_plane: iz out of range");
    const long long plane = s_.n_xy() * s_.nr * s_.n_rot;
    copy_out(psi_ + plane * iz, out, plane);
    check_cuda(cudaStreamSynchronize(stream_), "z_plane");
  }

  void block_densities(double* out) override {
    spo::block_density_kernel<T><<<static_cast<unsigned>(s_.n_zr()), 256, 0, stream_>>>(
        psi_, s_.n_xy() * s_.n_rot, densities_);
    check_cuda(cudaGetLastError(), "block_densities launch");
    check_cuda(cudaMemcpyAsync(out, densities_, sizeof(double) * s_.n_zr(), cudaMemcpyDeviceToHost, stream_),
               "block_densities copy");
    check_cuda(cudaStreamSynchronize(stream_), "block_densities");
  }

  // The norm budget's absorption of every cell of both grids, as NormBudget's constructor
  // (src/analysis/norm_budget.cpp:39-71): absorbers ZOpt, [ZOptLow], ROpt (scattering), ZSpOpt, [ZSpOptLow],
  // ROpt (specular); per cell the window exponent 2 n V_opt dt, the Z absorber and its share of the loss
  // (V_opt,Z / (V_opt,Z + V_opt,r)), the r absorber. Returns the number of absorbers.
  int norm_budget_setup(const spo_norm_budget_desc& d) override {
    int n_abs = 0;
    const int z_opt = n_abs++;
    const int z_opt_low = d.z_low_first >= 0 ? n_abs++ : -1;
    const int r_opt = n_abs++;
    const int zsp_opt = n_abs++;
    const int zsp_opt_low = d.zs_low_first >= 0 ? n_abs++ : -1;
    const int r_opt_spec = n_abs++;
    auto absorption = [&](const std::vector<double>& zf, int z_high, int z_low, int low_first, int low_last,
                          int r_index, spo::BudgetGrid& g, std::vector<double>& exponent, std::vector<double>& share,
                          std::vector<int>& za, std::vector<int>& ra) {
      const std::size_t cells = zf.size() * static_cast<std::size_t>(s_.nr);
      exponent.assign(cells, 0.0);
      share.assign(cells, 0.0);
      za.assign(cells, -1);
      ra.assign(cells, -1);
      for (int iz = 0; iz < static_cast<int>(zf.size()); ++iz)
        for (int ir = 0; ir < s_.nr; ++ir) {
          const double v_z = -std::log(zf[iz]), v_r = -std::log(host_opt_r_[ir]);
          if (v_z == 0.0 && v_r == 0.0) continue;
          const std::size_t k = ir + static_cast<std::size_t>(s_.nr) * iz;
          exponent[k] = 2.0 * s_.spa * (v_z + v_r);
          if (v_z != 0.0) {
            za[k] = (low_first >= 0 && iz >= low_first && iz <= low_last) ? z_low : z_high;
            share[k] = v_z / (v_z + v_r);
          }
          if (v_r != 0.0) ra[k] = r_index;
        }
      g.cells = static_cast<long long>(cells);
    };
    std::vector<double> e0, s0, e1, s1;
    std::vector<int> za0, ra0, za1, ra1;
    absorption(host_opt_z_, z_opt, z_opt_low, d.z_low_first, d.z_low_last, r_opt, budget_scat_, e0, s0, za0, ra0);
    absorption(host_opt_zs_, zsp_opt, zsp_opt_low, d.zs_low_first, d.zs_low_last, r_opt_spec, budget_spec_, e1, s1,
               za1, ra1);
    auto up_d = [&](const std::vector<double>& v) {
      double* p = dev<double>(v.size());
      check_cuda(cudaMemcpy(p, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice), "norm budget tables");
      return p;
    };
    auto up_i = [&](const std::vector<int>& v) {
      int* p = dev<int>(v.size());
      check_cuda(cudaMemcpy(p, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice), "norm budget tables");
      return p;
    };
    budget_scat_.exponent = up_d(e0);
    budget_scat_.z_share = up_d(s0);
    budget_scat_.z_absorber = up_i(za0);
    budget_scat_.r_absorber = up_i(ra0);
    budget_scat_.previous = dev<double>(e0.size());
    budget_spec_.exponent = up_d(e1);
    budget_spec_.z_share = up_d(s1);
    budget_spec_.z_absorber = up_i(za1);
    budget_spec_.r_absorber = up_i(ra1);
    budget_spec_.previous = dev<double>(e1.size());
    budget_out_ = dev<double>(2 * spo::kBudgetMaxAbsorbers + 2);
    budget_abs_ = n_abs;
    budget_vol_scat_ = d.volume_scattering;
    budget_vol_spec_ = d.volume_specular;
    budget_has_previous_ = false;
    return n_abs;
  }

  int norm_budget_absorbers() const override { return budget_abs_; }

  // One window of the norm budget (NormBudget::add, src/analysis/norm_budget.cpp:100-112) from the resident
  // state: out = losses (n_absorbers), loss errors (n_absorbers), norm at the window's start and end. False (out
  // untouched) at the first call, which only records the cells.
  bool norm_budget_add(double* out) override {
    require(budget_abs_ > 0, "spo_norm_budget_add: spo_norm_budget_setup was not called");
    spo::block_density_kernel<T><<<static_cast<unsigned>(s_.n_zr()), 256, 0, stream_>>>(
        psi_, s_.n_xy() * s_.n_rot, densities_);
    spo::norm_budget_kernel<T><<<1, 256, 0, stream_>>>(densities_, budget_vol_scat_, chi_, budget_vol_spec_,
                                                      budget_scat_, budget_spec_, budget_abs_,
                                                      budget_has_previous_ ? 1 : 0, budget_out_);
    check_cuda(cudaGetLastError(), "norm budget launch");
    const bool window = budget_has_previous_;
    if (window)
      check_cuda(cudaMemcpyAsync(out, budget_out_, sizeof(double) * (2 * budget_abs_ + 2), cudaMemcpyDeviceToHost,
                                 stream_), "norm budget copy");
    check_cuda(cudaStreamSynchronize(stream_), "norm budget");
    budget_has_previous_ = true;
    return window;
  }

  void averages(const double* z, const double* zs, const double* r, double vol_scat, double vol_spec, int iz_analysis,
                int surface_index, double* out) override {
    require(z && zs && r && out, "averages: null pointer");
    require(iz_analysis >= -1 && iz_analysis < s_.nzs && surface_index < s_.nzs, "averages: index out of range");
    // The grids and the four results pass through the staging buffer (>= 8M doubles).
    double* g = reinterpret_cast<double*>(staging_);
    const long long ng = static_cast<long long>(s_.nz) + s_.nzs + s_.nr;
    require(ng + 4 <= 2 * staging_elems_, "averages: grids larger than the staging buffer");
    check_cuda(cudaMemcpyAsync(g, z, sizeof(double) * s_.nz, cudaMemcpyHostToDevice, stream_), "averages grids");
    check_cuda(cudaMemcpyAsync(g + s_.nz, zs, sizeof(double) * s_.nzs, cudaMemcpyHostToDevice, stream_), "averages grids");
    check_cuda(cudaMemcpyAsync(g + s_.nz + s_.nzs, r, sizeof(double) * s_.nr, cudaMemcpyHostToDevice, stream_),
               "averages grids");
    spo::block_density_kernel<T><<<static_cast<unsigned>(s_.n_zr()), 256, 0, stream_>>>(
        psi_, s_.n_xy() * s_.n_rot, densities_);
    spo::averages_kernel<T><<<1, 256, 0, stream_>>>(densities_, chi_, g, s_.nz, s_.nr, s_.nzs, iz_analysis,
                                                    surface_index, vol_scat, vol_spec, g + ng);
    check_cuda(cudaGetLastError(), "averages launch");
    check_cuda(cudaMemcpyAsync(out, g + ng, sizeof(double) * 4, cudaMemcpyDeviceToHost, stream_), "averages copy");
    check_cuda(cudaStreamSynchronize(stream_), "averages");
  }

  void site_column(int ixy, double* out) override {
    require(ixy >= 0 && ixy < s_.n_xy(), "site_column: ixy out of range");
    const long long n = s_.n_zr() * s_.n_rot;
    spo::site_column_kernel<T><<<592, 256, 0, stream_>>>(psi_, staging_, s_.n_rot, static_cast<int>(s_.n_xy()),
                                                         s_.n_zr(), ixy);
    check_cuda(cudaGetLastError(), "site_column launch");
    // staging_ holds staging_elems_ complex values; the column is n_zr*n_rot <= that (checked at build).
    check_cuda(cudaMemcpyAsync(out, staging_, sizeof(double2) * n, cudaMemcpyDeviceToHost, stream_),
               "site_column copy");
    check_cuda(cudaStreamSynchronize(stream_), "site_column");
  }

  void apply_stage(int stage, bool half) override {
    launches_ = 0;
    switch (stage) {
      case SPO_STAGE_SPECULAR: specular(half, false); break;
      case SPO_STAGE_SPECULAR_KINETIC: specular(half, true); break;
      case SPO_STAGE_ZR: kinetic_zr(half); break;
      case SPO_STAGE_XY: kinetic_xy(half, false); break;
      case SPO_STAGE_POTENTIAL:
        gas_phase();
        interaction();
        break;
      default: require(false, "unknown stage");
    }
    check_cuda(cudaGetLastError(), "apply_stage launch");
    check_cuda(cudaStreamSynchronize(stream_), "apply_stage");
    prof_.resolve();
  }

  void analysis_setup(const spo_analysis_desc& d) override {
    require(d.n_v > 0 && d.n_rotation > 0 && d.n_diffraction > 0 && d.n_energies >= 0, "analysis sizes invalid");
    require(d.iz_analysis >= 0 && d.iz_analysis < s_.nz, "iz_analysis out of range");
    require(d.initial_state >= 0 && d.initial_state < d.n_rotation * d.n_diffraction, "initial_state out of range");
    require(d.j_in >= 0 && d.j_in <= d.j_max_gas, "j_in out of range");
    an_ = d;
    const std::vector<int> rot = int_array(d.rotation_index, d.n_rotation, "rotation_index");
    const std::vector<int> rj = int_array(d.rotation_j, d.n_rotation, "rotation_j");
    const std::vector<int> cx = int_array(d.channel_ix, d.n_diffraction, "channel_ix");
    const std::vector<int> cy = int_array(d.channel_iy, d.n_diffraction, "channel_iy");
    for (int i = 0; i < d.n_rotation; ++i)
      require(rot[i] >= 0 && rot[i] < s_.n_rot && rj[i] >= 0 && rj[i] <= d.j_max_gas, "analysed rotation out of range");
    for (int i = 0; i < d.n_diffraction; ++i)
      require(cx[i] >= 0 && cx[i] < s_.nx && cy[i] >= 0 && cy[i] < s_.ny, "diffraction channel out of range");
    const std::size_t n_phi = static_cast<std::size_t>(s_.nr) * (d.j_max_gas + 1) * d.n_v;
    an_rot_ = upload_int(rot);
    an_j_ = upload_int(rj);
    an_cx_ = upload_int(cx);
    an_cy_ = upload_int(cy);
    an_phi_ = upload_f64(real_array(d.phi_vj, n_phi, "phi_vj"));
    an_energies_ = upload_f64(d.n_energies > 0 ? real_array(d.energies_hartree, d.n_energies, "energies_hartree")
                                               : std::vector<double>(1, 0.0));
    an_twx_ = upload_c128(twiddles(s_.nx));
    an_twy_ = upload_c128(twiddles(s_.ny));
    an_shift_ = upload_c128(shift_host_);
    const long long n = static_cast<long long>(d.n_rotation) * d.n_diffraction * d.n_v;
    an_bk_ = dev<double2>(n);
    an_sums_ = dev<double2>(std::max<long long>(n * d.n_energies, 1));
    check_cuda(cudaMemsetAsync(an_sums_, 0, sizeof(double2) * std::max<long long>(n * d.n_energies, 1), stream_),
               "zero S sums");
    check_cuda(cudaStreamSynchronize(stream_), "analysis_setup");
    an_ready_ = true;
  }

  void bk(double time, bool fixed, int surface_index, bool accumulate, double* out) override {
    require(an_ready_, "spo_analysis_setup was not called");
    require(!fixed || (surface_index >= 0 && surface_index < s_.nzs), "surface_index out of range");
    spo::BkArgs<T> a{};
    a.psi = psi_;
    a.n_rot = s_.n_rot;
    a.nx = s_.nx;
    a.ny = s_.ny;
    a.nr = s_.nr;
    a.iz_analysis = an_.iz_analysis;
    a.n_v = an_.n_v;
    a.n_rotation = an_.n_rotation;
    a.n_diffraction = an_.n_diffraction;
    a.j_max_gas = an_.j_max_gas;
    a.rotation_index = an_rot_;
    a.rotation_j = an_j_;
    a.channel_ix = an_cx_;
    a.channel_iy = an_cy_;
    a.phi_vj = an_phi_;
    a.shift = an_shift_;
    a.dr = an_.dr;
    a.xy_scale = an_.xy_scale;
    a.px = plan_x_;
    a.py = plan_y_;
    a.twx = an_twx_;
    a.twy = an_twy_;
    a.bk = an_bk_;
    const std::size_t smem = sizeof(double2) * (2 * s_.n_xy() + s_.nx + s_.ny);
    spo::bk_kernel<T><<<an_.n_v * an_.n_rotation, 256, smem, stream_>>>(a);
    const int n_states = an_.n_rotation * an_.n_diffraction;
    if (fixed)
      spo::bk_specular_kernel<T><<<(an_.n_v + 127) / 128, 128, 0, stream_>>>(
          chi_, s_.nr, surface_index, an_phi_, an_.j_max_gas, an_.j_in, an_.n_v, n_states, an_.initial_state, an_.dr,
          an_bk_);
    const int n = n_states * an_.n_v;
    if (accumulate && an_.n_energies > 0)
      spo::s_matrix_add_kernel<<<std::min<long long>((static_cast<long long>(n) * an_.n_energies + 255) / 256, 1184),
                                 256, 0, stream_>>>(an_bk_, n, an_energies_, an_.n_energies, time,
                                                    an_.analysis_time_step, an_sums_);
    check_cuda(cudaGetLastError(), "bk launch");
    if (out)
      check_cuda(cudaMemcpyAsync(out, an_bk_, sizeof(double2) * n, cudaMemcpyDeviceToHost, stream_), "bk copy");
    check_cuda(cudaStreamSynchronize(stream_), "bk");
  }

  void s_sums(double* out) override {
    require(an_ready_, "spo_analysis_setup was not called");
    const long long n = static_cast<long long>(an_.n_rotation) * an_.n_diffraction * an_.n_v * an_.n_energies;
    if (n > 0)
      check_cuda(cudaMemcpyAsync(out, an_sums_, sizeof(double2) * n, cudaMemcpyDeviceToHost, stream_), "S copy");
    check_cuda(cudaStreamSynchronize(stream_), "s_sums");
  }

  unsigned long long bytes() const override { return arena_.bytes(); }
  int launches() const override { return launches_; }
  void set_stream(cudaStream_t s) override { stream_ = s ? s : own_stream_; }
  void profile(bool on) override { prof_.enable(on); }
  const std::vector<KernelRecord>& records() const override { return prof_.records(); }

 private:
  // ------------------------------------------------------------------ one sub-step
  void sub_step(bool half, bool kinetic_only) {
    specular(half, kinetic_only);
    if (rxy_planes_ > 0) {
      kinetic_rxy_slabs(half, !kinetic_only);
    } else {
      kinetic_zr(half);
      kinetic_xy(half, !kinetic_only);  // the gas-phase potential step rides along
    }
    if (!kinetic_only) interaction();
  }

  // T_Z over the whole wave packet, then T_r and T_xy slab by slab of rxy_planes_ Z planes (nr n_xy n_rot
  // values each): T_r and T_xy of a point only involve its own Z plane, and a slab written by the r pass
  // is still in L2 when the xy pass reads it.
  void kinetic_rxy_slabs(bool half, bool with_gas) {
    const double b = 2.0 * sizeof(V) * s_.n_psi();
    axis_psi("kinetic_z", b, 1, plan_z_, tw_z_, s_.n_xy() * s_.nr * s_.n_rot, half ? zk_half_ : zk_full_, tile_z_,
             persist_z_);
    const long long plane = static_cast<long long>(s_.nr) * s_.n_xy() * s_.n_rot;
    for (int iz0 = 0; iz0 < s_.nz; iz0 += rxy_planes_) {
      const int g = std::min(rxy_planes_, s_.nz - iz0);
      spo::Axis2Args<T> r{psi_ + plane * iz0, s_.n_xy() * s_.n_rot, half ? rk_half_ : rk_full_, tw_r_, tile_r_};
      r.factor_pfa = pfa_of(r.factor);
      r.persistent = persist_r_ ? 1 : 0;
      prof_.begin(stream_);
      launch_axis2<T>(plan_r_.n, r, g, stream_);
      prof_.end(stream_, "kinetic_r", 2.0 * sizeof(V) * plane * g);
      ++launches_;
      kinetic_xy(half, with_gas, static_cast<long long>(iz0) * s_.nr, static_cast<long long>(g) * s_.nr);
    }
  }

  // Specular grid: r forward, Z forward * factor * inverse, r inverse (* W factors).
  void specular(bool half, bool kinetic_only) {
    const double b = 2.0 * sizeof(V) * s_.n_chi();
    axis("specular_r", b, chi_, /*outer*/ s_.nzs, plan_r_, tw_r_, /*inner*/ 1, nullptr, spo::kNoFactor, spo::kFwdFactor,
         nullptr);
    axis("specular_z", b, chi_, 1, plan_zs_, tw_zs_, s_.nr, half ? spec_half_ : spec_full_, spo::kFactorAxisInner,
         spo::kFwdFactorInv, nullptr);
    axis("specular_r", b, chi_, s_.nzs, plan_r_, tw_r_, 1, nullptr, spo::kNoFactor, spo::kFactorInv,
         kinetic_only ? nullptr : spec_w_);
  }

  // T_Z and T_r of the scattering wave. With zr_window_ > 0 the two passes run window by window over the
  // (x, y, irot) lanes, Z then r for each window, so that a window written by the Z pass is still in L2
  // when the r pass reads it (nz nr window values per window).
  void kinetic_zr(bool half) {
    const double b = 2.0 * sizeof(V) * s_.n_psi();
    const V* zf = half ? zk_half_ : zk_full_;
    const V* rf = half ? rk_half_ : rk_full_;
    if (zr_window_ == 0) {
      axis_psi("kinetic_z", b, 1, plan_z_, tw_z_, s_.n_xy() * s_.nr * s_.n_rot, zf, tile_z_, persist_z_, balanced_);
      axis_psi("kinetic_r", b, s_.nz, plan_r_, tw_r_, s_.n_xy() * s_.n_rot, rf, tile_r_, persist_r_, balanced_);
      return;
    }
    const long long lanes = s_.n_xy() * s_.n_rot;  // contiguous values per (Z, r) point
    for (long long l0 = 0; l0 < lanes; l0 += zr_window_) {
      const long long w = std::min<long long>(zr_window_, lanes - l0);
      const double bw = b * static_cast<double>(w) / static_cast<double>(lanes);
      spo::Axis2Args<T> z{psi_, 0, zf, tw_z_, tile_z_};
      z.factor_pfa = pfa_of(zf);
      z.groups = s_.nr;  // lanes (ir, l0 + l): groups ir, lanes apart
      z.group_stride = lanes;
      z.lane_offset = l0;
      z.window = w;
      z.line_stride = static_cast<long long>(s_.nr) * lanes;
      z.outer_stride = 0;
      prof_.begin(stream_);
      launch_axis2<T>(plan_z_.n, z, 1, stream_);
      prof_.end(stream_, "kinetic_z", bw);
      ++launches_;
      spo::Axis2Args<T> r{psi_, 0, rf, tw_r_, tile_r_};
      r.factor_pfa = pfa_of(rf);
      r.groups = 1;
      r.group_stride = 0;
      r.lane_offset = l0;
      r.window = w;
      r.line_stride = lanes;
      r.outer_stride = static_cast<long long>(s_.nr) * lanes;  // block y = iz
      prof_.begin(stream_);
      launch_axis2<T>(plan_r_.n, r, s_.nz, stream_);
      prof_.end(stream_, "kinetic_r", bw);
      ++launches_;
    }
  }

  // A kinetic axis pass over psi: the register-DFT kernel for its length when instantiated, else the
  // general Stockham kernel.
  // The prime-factor-order copy of a Z or r factor table (null when that axis has no prime-factor split).
  const V* pfa_of(const V* factor) const {
    if (!use_pfa_ || !use_v2_) return nullptr;
    if (factor == zk_full_) return zk_full_pfa_;
    if (factor == zk_half_) return zk_half_pfa_;
    if (factor == rk_full_) return rk_full_pfa_;
    if (factor == rk_half_) return rk_half_pfa_;
    return nullptr;
  }
  void axis_psi(const char* name, double bytes, long long outer, const spo::FftPlan& plan, const V* tw,
                long long inner, const V* factor, int tile, bool persistent = false, bool balanced = false) {
    if (use_v2_ && axis2_supported(plan.n)) {
      spo::Axis2Args<T> a{psi_, inner, factor, tw, tile};
      a.factor_pfa = pfa_of(factor);
      a.persistent = persistent ? 1 : 0;
      a.balanced = balanced ? 1 : 0;
      prof_.begin(stream_);
      launch_axis2<T>(plan.n, a, outer, stream_);
      prof_.end(stream_, name, bytes);
      ++launches_;
      return;
    }
    axis(name, bytes, psi_, outer, plan, tw, inner, factor, spo::kFactorAxis, spo::kFwdFactorInv, nullptr);
  }

  // T_xy, optionally with the gas-phase potential step fused; over the points izr in [izr_first,
  // izr_first + n_izr) (n_izr < 0: all of them; a range needs the register kernel).
  void kinetic_xy(bool half, bool with_gas, long long izr_first = 0, long long n_izr = -1) {
    spo::XyArgs<T> x{};
    x.psi = psi_;
    x.n_rot = s_.n_rot;
    x.nx = s_.nx;
    x.ny = s_.ny;
    x.px = plan_x_;
    x.py = plan_y_;
    x.twx = tw_x_;
    x.twy = tw_y_;
    x.factor = half ? xyk_half_ : xyk_full_;
    x.shift_f = shift_f_;
    x.shift_b = shift_b_;
    x.tb = xy_tb_;
    x.apply_gas = with_gas ? 1 : 0;
    x.izr_gas_first = static_cast<long long>(s_.nzp) * s_.nr;
    x.nr = s_.nr;
    x.opt_z = opt_z_;
    x.gas_step = gas_step_;
    x.tile = tile_xy_;
    x.persistent = persist_xy_ ? 1 : 0;
    if (n_izr >= 0) {
      x.izr_offset = izr_first;
      prof_.begin(stream_);
      require(launch_xy2<T>(x, n_izr, stream_), "kinetic_xy: a range of points needs the register kernel");
      prof_.end(stream_, "kinetic_xy", 2.0 * sizeof(V) * n_izr * s_.n_xy() * s_.n_rot);
      ++launches_;
      return;
    }
    const dim3 xg((s_.n_rot + xy_tb_ - 1) / xy_tb_, static_cast<unsigned>(s_.n_zr()));
    prof_.begin(stream_);
    if (!(use_v2_ && launch_xy2<T>(x, s_.n_zr(), stream_))) spo::xy_pass_kernel<T><<<xg, 256, xy_smem_, stream_>>>(x);
    prof_.end(stream_, "kinetic_xy", 2.0 * sizeof(V) * s_.n_psi());
    ++launches_;
  }

  void gas_phase() {
    const long long first = static_cast<long long>(s_.nzp) * s_.nr;
    if (first >= s_.n_zr()) return;
    prof_.begin(stream_);
    spo::gas_phase_kernel<T><<<1184, 256, 0, stream_>>>(psi_, first, s_.n_zr(), s_.n_rot, static_cast<int>(s_.n_xy()),
                                                        s_.nr, opt_z_, gas_step_);
    prof_.end(stream_, "gas_phase", 2.0 * sizeof(V) * (s_.n_zr() - first) * s_.n_xy() * s_.n_rot);
    ++launches_;
  }

  void interaction() {
    if (s_.nzp == 0) return;
    prof_.begin(stream_);
    // psi of the interaction region read and written, the exp(i A) table read (the mixed form's entries with
    // their 2-byte modulus corrections)
    const double bytes = sizeof(V) * (2.0 * s_.nzp * s_.nr * s_.n_xy() * s_.n_rot + static_cast<double>(s_.n_expia())) +
                         (sizeof(T) == 4 ? 2.0 * static_cast<double>(s_.n_expia()) : 0.0);
    const unsigned points = static_cast<unsigned>(s_.nzp) * s_.nr;
    if (pot_kind_ >= 3) {
      if (pot_kind_ == 6) {
        pot6_kernel_<<<pot6_blocks_, spo::kPot6Threads, pot6_smem_, stream_>>>(pot6_args_, error_flag_);
      } else if (pot_kind_ == 5) {
        pot5_kernel_<<<pot5_blocks_, 128, pot5_smem_, stream_>>>(pot4_args_, error_flag_);
      } else if (pot_kind_ == 4) {
        pot4_kernel_<<<pot4_blocks_, 128, pot4_smem_, stream_>>>(pot4_args_);
      } else {
        const dim3 grid(static_cast<unsigned>(pot3_chunks_), points);
        launch_pot3<T>(s_.nphi, pot3_args_, grid, static_cast<unsigned>(pot3_cb_ * s_.nt), pot3_smem_, stream_);
      }
      prof_.end(stream_, "potential", bytes);
      ++launches_;
      prof_.begin(stream_);
      spo::projection_finalize_kernel<T><<<points, 128, sizeof(V) * (s_.n_xy() + 1), stream_>>>(
          psi_, chi_, s_.n_rot, static_cast<int>(s_.n_xy()), s_.i0, pot_.sc2sp, pot_.sp2sc);
      prof_.end(stream_, "projection", 2.0 * sizeof(V) * points * s_.n_xy());
      ++launches_;
      return;
    }
    if (pot_kind_ == 2)
      launch_pot2<T>(s_.nphi, pot2_, points, pot2_smem_, stream_);
    else
      spo::potential_kernel<T><<<points, 256, pot_smem_, stream_>>>(pot_);
    prof_.end(stream_, "potential", bytes);
    ++launches_;
  }

  // ------------------------------------------------------------------ tile choice
  // Mean device milliseconds of `launch` over `reps` launches on the handle's stream, after one warm-up.
  template <typename F>
  float time_launches(F&& launch, int reps) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    check_cuda(cudaEventCreate(&e0), "cudaEventCreate");
    check_cuda(cudaEventCreate(&e1), "cudaEventCreate");
    launch();
    check_cuda(cudaEventRecord(e0, stream_), "cudaEventRecord");
    for (int i = 0; i < reps; ++i) launch();
    check_cuda(cudaEventRecord(e1, stream_), "cudaEventRecord");
    check_cuda(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0.0f;
    check_cuda(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_cuda(cudaGetLastError(), "autotune launch");
    return ms / reps;
  }

  // Chooses, per kinetic pass, the tile width (8, 16 or 32 batch lanes per block) of the register kernels
  // with more than 8 sub-rows per line, by timing each on the zero wave packet the handle starts with
  // (a kinetic pass maps zero to zero, so the state is unchanged). All widths compute every line with the
  // same operations in the same order: the choice changes the speed, never the result.
  // SPO_B200_TILES=8|16|32 (every pass) or z,r,xy fixes the choice; SPO_B200_AUTOTUNE=0 keeps the default (16).
  void autotune() {
    tile_z_ = tile_r_ = tile_xy_ = 0;
    zr_window_ = 0;
    rxy_planes_ = 0;
    // The persistent forms are a fixed choice, not a timed one: they agree with the plain kernels to
    // rounding only (the compiler may contract a complex product into FMAs differently in each), and a
    // timed choice could make two runs of one case differ in the last bits. On configuration 3 the
    // persistent xy pass (16 x 16) takes 1.50 ms against 1.66; the persistent Z and r passes are slower
    // (2.17 against 1.43 ms for Z: 127 registers leave one block of 512 threads per SM).
    persist_z_ = persist_r_ = false;
    persist_xy_ = use_v2_ && s_.nx == s_.ny && xy2_supported(s_.nx) && s_.nx >= 12;
    // The balanced axis kernel (lengths N1 x 2 N1: 32 and 128) is a fixed choice for the same reason:
    // Z = 128 on configuration 3 takes 1.38 ms against 1.43 (mixed), 2.69 against 2.71 (FP64). An explicit
    // persistent request takes precedence over it.
    balanced_ = use_v2_;
    tiles_source_ = "default";
    if (!use_v2_) return;
    if (const char* env = std::getenv("SPO_B200_TILES")) {  // one width for every pass, or "z,r,xy"
      std::vector<int> w;
      std::string t(env);
      for (std::size_t k = 0; k <= t.size();) {
        const std::size_t e = std::min(t.find(',', k), t.size());
        const std::string one = t.substr(k, e - k);
        require(one == "8" || one == "16" || one == "32", "SPO_B200_TILES must be 8, 16 or 32, or three of them: z,r,xy");
        w.push_back(std::stoi(one));
        k = e + 1;
      }
      require(w.size() == 1 || w.size() == 3, "SPO_B200_TILES must be 8, 16 or 32, or three of them: z,r,xy");
      tile_z_ = w[0];
      tile_r_ = w.size() == 3 ? w[1] : w[0];
      tile_xy_ = w.size() == 3 ? w[2] : w[0];
      tiles_source_ = "fixed";
    }
    if (const char* env = std::getenv("SPO_B200_ZR_WINDOW")) {  // lanes per Z+r window (0: two full passes)
      zr_window_ = std::max(0ll, std::stoll(env) / 32 * 32);
      tiles_source_ = "fixed";
    }
    if (const char* env = std::getenv("SPO_B200_BALANCED")) {  // 1: the balanced axis kernels (N2 = 2 N1), 0: not
      balanced_ = std::string(env) == "1";
      tiles_source_ = "fixed";
    }
    if (const char* env = std::getenv("SPO_B200_PERSISTENT")) {  // 1: the persistent kinetic kernels, 0: not
      persist_z_ = persist_r_ = persist_xy_ = std::string(env) == "1";
      tiles_source_ = "fixed";
    }
    if (const char* env = std::getenv("SPO_B200_RXY_PLANES")) {  // Z planes per r+xy slab (0: full passes)
      rxy_planes_ = std::max(0, std::stoi(env));
      if (!(axis2_supported(s_.nr) && s_.nx == s_.ny && xy2_supported(s_.nx))) rxy_planes_ = 0;
      tiles_source_ = "fixed";
    }
    if (tiles_source_ == "fixed") return;
    if (const char* env = std::getenv("SPO_B200_AUTOTUNE"))
      if (std::string(env) == "0") return;
    constexpr int reps = 3;
    const double b = 0.0;
    // Each width is timed in two interleaved rounds after one untimed round of all three (the GPU's clock
    // may still be rising when a handle is created), and keeps its faster round.
    auto choose = [&](int& tile, auto&& run) {
      constexpr int widths[3] = {16, 8, 32};
      float ms[3] = {0.0f, 0.0f, 0.0f};
      for (int round = 0; round < 3; ++round)
        for (int k = 0; k < 3; ++k) {
          tile = widths[k];
          const float t = time_launches(run, reps);
          if (round == 1 || (round == 2 && t < ms[k])) ms[k] = t;
        }
      int best = 0;
      for (int k = 1; k < 3; ++k)
        if (ms[k] < 0.98f * ms[best]) best = k;  // another width only when clearly faster
      tile = widths[best];
    };
    const bool was_on = prof_.on();
    prof_.enable(false);
    if (axis2_supported(s_.nz) && axis2_has_tiles(s_.nz))
      choose(tile_z_, [&] { axis_psi("kinetic_z", b, 1, plan_z_, tw_z_, s_.n_xy() * s_.nr * s_.n_rot, zk_full_, tile_z_); });
    if (axis2_supported(s_.nr) && axis2_has_tiles(s_.nr))
      choose(tile_r_, [&] { axis_psi("kinetic_r", b, s_.nz, plan_r_, tw_r_, s_.n_xy() * s_.n_rot, rk_full_, tile_r_); });
    if (s_.nx == s_.ny && xy2_supported(s_.nx) && s_.nx > 8) choose(tile_xy_, [&] { kinetic_xy(false, false); });
    // Z and r through L2: windows whose values (nz nr window) take about 24, 48 or 96 MB, against
    // the two full passes.
    zr_window_ = 0;
    if (axis2_supported(s_.nz) && axis2_supported(s_.nr)) {
      const long long lanes = s_.n_xy() * s_.n_rot;
      float best_ms = time_launches([&] { kinetic_zr(false); }, reps);
      long long best = 0;
      for (const long long mb : {24ll, 48ll, 96ll}) {
        long long w = (mb << 20) / (static_cast<long long>(s_.nz) * s_.nr * static_cast<long long>(sizeof(V)));
        w = (w / 32) * 32;
        if (w < 32 || w >= lanes) continue;
        zr_window_ = w;
        const float ms = time_launches([&] { kinetic_zr(false); }, reps);
        if (ms < 0.98f * best_ms) {
          best = w;
          best_ms = ms;
        }
      }
      zr_window_ = best;
    }
    // T_r and T_xy through L2, slabs of 1, 2 or 4 Z planes, against the full passes.
    rxy_planes_ = 0;
    if (zr_window_ == 0 && axis2_supported(s_.nr) && s_.nx == s_.ny && xy2_supported(s_.nx)) {
      auto run = [&] {
        if (rxy_planes_ > 0) {
          kinetic_rxy_slabs(false, false);
        } else {
          kinetic_zr(false);
          kinetic_xy(false, false);
        }
      };
      float best_ms = time_launches(run, reps);
      int best = 0;
      for (const int g : {1, 2, 4}) {
        if (g >= s_.nz) continue;
        rxy_planes_ = g;
        const float ms = time_launches(run, reps);
        if (ms < 0.98f * best_ms) {
          best = g;
          best_ms = ms;
        }
      }
      rxy_planes_ = best;
    }
    prof_.enable(was_on);
    launches_ = 0;
    tiles_source_ = "autotuned";
  }

  void axis(const char* name, double bytes, V* data, long long outer, const spo::FftPlan& plan, const V* tw,
            long long inner, const V* factor, int factor_mode, int dir, const V* post) {
    spo::AxisArgs<T> a{};
    a.data = data;
    a.inner = inner;
    a.plan = plan;
    a.tw = tw;
    a.factor = factor;
    a.factor_mode = factor_mode;
    a.dir = dir;
    a.post = post;
    a.tb = axis_tile(plan.n, inner);
    const std::size_t smem = sizeof(V) * (2 * static_cast<std::size_t>(plan.n) * a.tb + (sizeof(T) == 4 ? 2 : 1) * plan.n);
    const dim3 grid(static_cast<unsigned>((inner + a.tb - 1) / a.tb), static_cast<unsigned>(outer));
    prof_.begin(stream_);
    spo::axis_pass_kernel<T><<<grid, 256, smem, stream_>>>(a);
    prof_.end(stream_, name, bytes);
    ++launches_;
  }

  // Inner elements per axis-pass tile: a power of two up to 64 (coalesced rows of tb * sizeof(V)
  // bytes), at most ~64 KiB of shared memory for the two ping-pong buffers, at most `inner`.
  static int axis_tile(int n, long long inner) {
    int tb = 64;
    while (tb > 1 && 2ull * n * tb * sizeof(V) > (64u << 10)) tb /= 2;
    while (tb > 1 && tb / 2 >= inner) tb /= 2;
    return tb;
  }

  // ------------------------------------------------------------------ set-up
  template <typename U>
  U* dev(std::size_t n) {
    return static_cast<U*>(arena_.alloc(sizeof(U) * n));
  }

  // A complex table on the device. The mixed form stores each value rounded to FP32 followed by the n
  // roundings of the remainders (value - rounded value): kernels apply the pair as one constant exact to
  // ~2^-48 (spo::cmul2), so that a table applied at every time step does not change the norm
  // systematically through its own rounding.
  V* upload_complex(const std::vector<cplx>& v) {
    const std::size_t n = v.size();
    std::vector<V> h((sizeof(T) == 4 ? 2 : 1) * n);
    for (std::size_t i = 0; i < n; ++i) {
      h[i].x = static_cast<T>(v[i].real());
      h[i].y = static_cast<T>(v[i].imag());
      if constexpr (sizeof(T) == 4) {
        h[n + i].x = static_cast<T>(v[i].real() - static_cast<double>(h[i].x));
        h[n + i].y = static_cast<T>(v[i].imag() - static_cast<double>(h[i].y));
      }
    }
    V* d = dev<V>(h.size());
    check_cuda(cudaMemcpy(d, h.data(), sizeof(V) * h.size(), cudaMemcpyHostToDevice), "upload table");
    return d;
  }
  // A real matrix with, in the mixed form, its low parts: the entries v (as T) followed by the roundings of
  // exact - v; the FP64 form uploads exact.
  // A table of factors s e^{i phi} (s >= 0 real: kinetic and rotation phases with FFT scales or absorbers). The
  // mixed form stores g = e^{i phi} - 1 (n values), the roundings of g's remainders (n values) and, per factor,
  // (s, the rounding of s's remainder) (n pairs): spo::fmul_t applies the factor as s (x + x g), which FP32 rounds
  // without the bias of a near-unity phase product. The FP64 form stores the factors.
  V* upload_factor(const std::vector<cplx>& f) {
    if constexpr (sizeof(T) == 4) {
      const std::size_t n = f.size();
      std::vector<V> h(spo::kFactorParts * n);
      for (std::size_t i = 0; i < n; ++i) {
        const double sc = std::abs(f[i]);
        const cplx g = sc > 0.0 ? cplx(f[i].real() / sc - 1.0, f[i].imag() / sc) : cplx(-1.0, 0.0);
        h[i].x = static_cast<T>(g.real());
        h[i].y = static_cast<T>(g.imag());
        h[n + i].x = static_cast<T>(g.real() - static_cast<double>(h[i].x));
        h[n + i].y = static_cast<T>(g.imag() - static_cast<double>(h[i].y));
        h[2 * n + i].x = static_cast<T>(sc);
        h[2 * n + i].y = static_cast<T>(sc - static_cast<double>(h[2 * n + i].x));
      }
      V* d = dev<V>(h.size());
      check_cuda(cudaMemcpy(d, h.data(), sizeof(V) * h.size(), cudaMemcpyHostToDevice), "upload table");
      return d;
    } else {
      return upload_complex(f);
    }
  }
  T* upload_real_lo(const std::vector<double>& v, const std::vector<double>& exact) {
    if constexpr (sizeof(T) == 4) {
      std::vector<double> both(2 * v.size());
      for (std::size_t i = 0; i < v.size(); ++i) {
        const double hi = static_cast<float>(v[i]);
        both[i] = hi;
        both[v.size() + i] = exact[i] - hi;
      }
      return upload_real(both);
    } else {
      return upload_real(exact);
    }
  }
  T* upload_real(const std::vector<double>& v) {
    std::vector<T> h(v.begin(), v.end());
    T* d = dev<T>(v.size());
    check_cuda(cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice), "upload table");
    return d;
  }
  double* upload_f64(const std::vector<double>& v) {
    double* d = dev<double>(v.size());
    check_cuda(cudaMemcpy(d, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice), "upload table");
    return d;
  }
  double2* upload_c128(const std::vector<cplx>& v) {
    double2* d = dev<double2>(v.size());
    check_cuda(cudaMemcpy(d, v.data(), sizeof(double2) * v.size(), cudaMemcpyHostToDevice), "upload table");
    return d;
  }
  int* upload_int(const std::vector<int>& v) {
    int* d = dev<int>(v.size());
    check_cuda(cudaMemcpy(d, v.data(), sizeof(int) * v.size(), cudaMemcpyHostToDevice), "upload table");
    return d;
  }

  void build(const spo_desc& d) {
    const Sizes& s = s_;
    const long long nxy = s.n_xy();
    plan_z_ = make_plan(s.nz);
    plan_r_ = make_plan(s.nr);
    plan_x_ = make_plan(s.nx);
    plan_y_ = make_plan(s.ny);
    plan_zs_ = make_plan(s.nzs);
    plan_phi_ = make_plan(s.nphi);
    tw_z_ = upload_complex(twiddles(s.nz));
    tw_r_ = upload_complex(twiddles(s.nr));
    tw_x_ = upload_complex(twiddles(s.nx));
    tw_y_ = upload_complex(twiddles(s.ny));
    tw_zs_ = upload_complex(twiddles(s.nzs));
    tw_phi_ = upload_complex(twiddles(s.nphi));

    // Kinetic factors with the FFT scales folded in (the reference applies the forward scale after
    // the forward transform and 1/(n*scale) after the inverse: the product of both is 1/n per axis).
    auto scaled = [](std::vector<cplx> v, double f) {
      for (auto& x : v) x *= f;
      return v;
    };
    zk_full_ = upload_factor(scaled(complex_array(d.z_kinetic_full, s.nz, "z_kinetic_full"), 1.0 / s.nz));
    zk_half_ = upload_factor(scaled(complex_array(d.z_kinetic_half, s.nz, "z_kinetic_half"), 1.0 / s.nz));
    rk_full_ = upload_factor(scaled(complex_array(d.r_kinetic_full, s.nr, "r_kinetic_full"), 1.0 / s.nr));
    rk_half_ = upload_factor(scaled(complex_array(d.r_kinetic_half, s.nr, "r_kinetic_half"), 1.0 / s.nr));
    {  // the same factors in the prime-factor order (axis2pfa_kernel), for axes with such a split
      int n1 = 0, n2 = 0;
      if (pfa_split(s.nz, n1, n2)) {
        zk_full_pfa_ = upload_factor(pfa_order(scaled(complex_array(d.z_kinetic_full, s.nz, "z_kinetic_full"), 1.0 / s.nz), n1, n2));
        zk_half_pfa_ = upload_factor(pfa_order(scaled(complex_array(d.z_kinetic_half, s.nz, "z_kinetic_half"), 1.0 / s.nz), n1, n2));
      }
      if (pfa_split(s.nr, n1, n2)) {
        rk_full_pfa_ = upload_factor(pfa_order(scaled(complex_array(d.r_kinetic_full, s.nr, "r_kinetic_full"), 1.0 / s.nr), n1, n2));
        rk_half_pfa_ = upload_factor(pfa_order(scaled(complex_array(d.r_kinetic_half, s.nr, "r_kinetic_half"), 1.0 / s.nr), n1, n2));
      }
    }
    const double sx = s.nx > 1 ? d.fft_scale_x : 1.0;
    const double sy = s.ny > 1 ? d.fft_scale_y : 1.0;
    const double xy_scale = (sx * sy) * ((1.0 / (s.nx * sx)) * (1.0 / (s.ny * sy)));
    xyk_full_ = upload_factor(scaled(complex_array(d.xy_kinetic_full, nxy, "xy_kinetic_full"), xy_scale));
    xyk_half_ = upload_factor(scaled(complex_array(d.xy_kinetic_half, nxy, "xy_kinetic_half"), xy_scale));
    const double sz = d.fft_scale_z, sr = d.fft_scale_r;
    const double spec_scale = (sz * sr) * ((1.0 / (s.nzs * sz)) * (1.0 / (s.nr * sr)));
    spec_full_ = upload_factor(scaled(complex_array(d.specular_kinetic_full, s.n_chi(), "specular_kinetic_full"), spec_scale));
    spec_half_ = upload_factor(scaled(complex_array(d.specular_kinetic_half, s.n_chi(), "specular_kinetic_half"), spec_scale));

    // Potential-step factors (src/propagation/potential_operator.cpp:15-26) and the specular grid's
    // W factors (src/propagation/specular_operator.cpp:11-19, 58-71), merged in FP64.
    const std::vector<cplx> rot = complex_array(d.rotation_half, static_cast<std::size_t>(s.n_rot) * s.nr, "rotation_half");
    const std::vector<double> opt_r = real_array(d.r_optical, s.nr, "r_optical");
    const std::vector<double> opt_z = real_array(d.z_optical, s.nz, "z_optical");
    const std::vector<double> opt_zs = real_array(d.z_specular_optical, s.nzs, "z_specular_optical");
    host_opt_z_ = opt_z;
    host_opt_r_ = opt_r;
    host_opt_zs_ = opt_zs;
    const std::vector<cplx> gas = complex_array(d.gas_phase, s.nr, "gas_phase");
    std::vector<cplx> before(rot.size()), gas_step(rot.size());
    for (int ir = 0; ir < s.nr; ++ir)
      for (int irot = 0; irot < s.n_rot; ++irot) {
        const cplx r = rot[irot + static_cast<std::size_t>(s.n_rot) * ir];
        const double o = s.nr != 1 ? opt_r[ir] : 1.0;
        before[static_cast<std::size_t>(ir) * s.n_rot + irot] = o * r;
        gas_step[static_cast<std::size_t>(ir) * s.n_rot + irot] = o * r * gas[ir] * r;
      }
    std::vector<cplx> spec_w(s.n_chi());
    for (int iz = 0; iz < s.nzs; ++iz)
      for (int ir = 0; ir < s.nr; ++ir) {
        const cplx r = rot[s.i0 + static_cast<std::size_t>(s.n_rot) * ir];
        cplx f = iz >= s.nzp ? r * gas[ir] * r : cplx(1.0, 0.0);
        f *= opt_zs[iz];
        if (s.nr != 1 && ir >= s.ra && ir <= s.rb) f *= opt_r[ir];
        spec_w[ir + static_cast<std::size_t>(s.nr) * iz] = f;
      }
    rot_half_ = upload_factor([&] {
      std::vector<cplx> v(rot.size());
      for (int ir = 0; ir < s.nr; ++ir)
        for (int irot = 0; irot < s.n_rot; ++irot)
          v[static_cast<std::size_t>(ir) * s.n_rot + irot] = rot[irot + static_cast<std::size_t>(s.n_rot) * ir];
      return v;
    }());
    before_ = upload_factor(before);
    gas_step_ = upload_factor(gas_step);
    spec_w_ = upload_factor(spec_w);
    opt_z_ = upload_real(opt_z);

    const std::vector<cplx> shf = complex_array(d.shift_forward, nxy, "shift_forward");
    shift_host_ = shf;
    const bool shift = std::any_of(shf.begin(), shf.end(), [](const cplx& c) { return c.real() != 1.0 || c.imag() != 0.0; });
    if (shift) {
      shift_f_ = upload_factor(shf);
      shift_b_ = upload_factor(complex_array(d.shift_backward, nxy, "shift_backward"));
    }
    const V* sp2sc = upload_complex(complex_array(d.specular_to_scattering, nxy, "specular_to_scattering"));
    const V* sc2sp = upload_complex(complex_array(d.scattering_to_specular, nxy, "scattering_to_specular"));

    // Angular transform tables.
    const std::vector<int> first = int_array(d.mj_fbr_first, s.n_blocks, "mj_fbr_first");
    const std::vector<int> size = int_array(d.mj_fbr_size, s.n_blocks, "mj_fbr_size");
    const std::vector<int> slot = int_array(d.mj_phi_slot, s.n_blocks, "mj_phi_slot");
    std::vector<int> offset(s.n_blocks), irot_block(s.n_rot, -1);
    int off = 0, total_j = 0;
    for (int b = 0; b < s.n_blocks; ++b) {
      offset[b] = off;
      off += s.nt * size[b];
      total_j += size[b];
      const int m = b - s.mj_max;
      require(slot[b] == (m >= 0 ? m : s.nphi + m), "mj_phi_slot does not follow the mJ order");
      for (int j = 0; j < size[b]; ++j) {
        require(first[b] + j >= 0 && first[b] + j < s.n_rot, "mj block outside the rotational basis");
        irot_block[first[b] + j] = b;
      }
    }
    require(total_j == s.n_rot, "mj blocks do not cover the rotational basis");
    std::vector<double> legendre = real_array(d.legendre, static_cast<std::size_t>(off), "legendre");
    const std::vector<double> legendre64 = legendre;  // the FP64 matrix (the low parts of the mixed form's tables)
    if constexpr (sizeof(T) == 4) {
      // The mixed form's matrix, rounded once for every potential kernel so that each rotational state's
      // sum of squares over theta keeps its FP64 value: the forward and the transposed contraction of a step
      // multiply the state by that sum (times nphi), every step (norm_preserving_rows).
      std::vector<double> by_state(static_cast<std::size_t>(s.n_rot) * s.nt);
      for (int b = 0; b < s.n_blocks; ++b)
        for (int t = 0; t < s.nt; ++t)
          for (int j = 0; j < size[b]; ++j)
            by_state[static_cast<std::size_t>(first[b] + j) * s.nt + t] = legendre[offset[b] + t * size[b] + j];
      const std::vector<float> rounded = norm_preserving_rows(by_state, s.n_rot, s.nt);
      for (int b = 0; b < s.n_blocks; ++b)
        for (int t = 0; t < s.nt; ++t)
          for (int j = 0; j < size[b]; ++j)
            legendre[offset[b] + t * size[b] + j] = rounded[static_cast<std::size_t>(first[b] + j) * s.nt + t];
    }

    // Symmetry maps, expanded to one phi map per (x, y) point.
    const std::vector<int> rep = int_array(d.representative_of, nxy, "representative_of");
    const std::vector<int> op = int_array(d.operation_of, nxy, "operation_of");
    const std::vector<int> phi_index = int_array(d.phi_index, static_cast<std::size_t>(s.n_ops) * s.nphi, "phi_index");
    std::vector<int> phi_map(nxy * s.nphi);
    for (long long ixy = 0; ixy < nxy; ++ixy) {
      require(rep[ixy] >= 0 && rep[ixy] < s.n_rep, "representative_of out of range");
      require(op[ixy] >= 0 && op[ixy] < s.n_ops, "operation_of out of range");
      for (int p = 0; p < s.nphi; ++p) {
        const int q = phi_index[static_cast<std::size_t>(op[ixy]) * s.nphi + p];
        require(q >= 0 && q < s.nphi, "phi_index out of range");
        phi_map[ixy * s.nphi + p] = q;
      }
    }

    // State.
    psi_ = dev<V>(s.n_psi());
    check_cuda(cudaMemsetAsync(psi_, 0, sizeof(V) * s.n_psi(), stream_), "zero psi");
    chi_ = dev<V>(s.n_chi());
    densities_ = dev<double>(s.n_zr());
    staging_elems_ = std::max<long long>(s.n_zr() * s.n_rot, 4ll << 20);
    staging_ = dev<double2>(staging_elems_);
    require(d.chi_initial != nullptr, "chi_initial is null");
    upload(nullptr, d.chi_initial);

    // exp(i A) on the device in FP64, chunk by chunk through the staging buffer.
    const long long n_e = s.n_expia();
    require(d.potential != nullptr || n_e == 0, "potential is null");
    // The mixed form keeps, after the n_e table entries, their n_e modulus corrections (FP16, spo::exp_mul).
    // (from a 16-byte boundary: the kernels read 8 corrections per load and prefetch rows of them into L2)
    const long long n_e_even = (n_e + 1) & ~1ll;
    expia_ = dev<V>(std::max<long long>(n_e_even + (sizeof(T) == 4 ? (n_e + 3) / 4 : 0), 1));
    __half* exp_mod = sizeof(T) == 4 ? reinterpret_cast<__half*>(expia_ + n_e_even) : nullptr;
    double* vstage = reinterpret_cast<double*>(staging_);
    const long long chunk = 2 * staging_elems_;
    for (long long i = 0; i < n_e; i += chunk) {
      const long long m = std::min(chunk, n_e - i);
      check_cuda(cudaMemcpyAsync(vstage, d.potential + i, sizeof(double) * m, cudaMemcpyHostToDevice, stream_),
                 "upload potential");
      spo::exp_potential_kernel<T><<<1184, 256, 0, stream_>>>(vstage, expia_ + i, exp_mod ? exp_mod + i : nullptr, m, s.dt);
      check_cuda(cudaGetLastError(), "exp_potential launch");
      check_cuda(cudaStreamSynchronize(stream_), "exp_potential");
    }

    // Launch shapes and shared memory.
    int smem_optin = 0, dev_id = 0;
    check_cuda(cudaGetDevice(&dev_id), "cudaGetDevice");
    check_cuda(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev_id), "smem attribute");
    check_cuda(cudaFuncSetAttribute(spo::axis_pass_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin),
               "axis smem");
    for (const int n : {s.nz, s.nr, s.nzs}) require(2ull * n * sizeof(V) + n * sizeof(V) <= static_cast<unsigned>(smem_optin),
                                                     "FFT length too long for shared memory");
    xy_tb_ = 1;
    while (xy_tb_ < 32 && xy_tb_ < s.n_rot && 2ull * nxy * (2 * xy_tb_) * sizeof(V) <= (96u << 10)) xy_tb_ *= 2;
    xy_smem_ = sizeof(V) * (2 * nxy * xy_tb_ + (sizeof(T) == 4 ? 2 : 1) * (s.nx + s.ny));
    require(xy_smem_ <= static_cast<std::size_t>(smem_optin), "nx*ny too large for the xy pass");
    check_cuda(cudaFuncSetAttribute(spo::xy_pass_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin),
               "xy smem");

    const int ld = s.nphi + 1;
    auto pot_bytes = [&](int cb) {
      return sizeof(V) * (static_cast<std::size_t>(cb) * s.n_rot + 2ull * cb * s.nt * ld + (sizeof(T) == 4 ? 2 : 1) * s.nphi + nxy + 32) +
             (sizeof(T) == 4 ? 2 : 1) * sizeof(T) * static_cast<std::size_t>(s.nt) * s.n_rot;
    };
    int cb = 1;
    while (cb < 16 && cb < nxy && pot_bytes(cb + 1) <= std::min<std::size_t>(smem_optin, 112u << 10)) ++cb;
    require(pot_bytes(cb) <= static_cast<std::size_t>(smem_optin), "angular grid too large for the potential step");
    pot_smem_ = pot_bytes(cb);
    check_cuda(cudaFuncSetAttribute(spo::potential_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin),
               "potential smem");
    pot_.psi = psi_;
    pot_.chi = chi_;
    pot_.n_rot = s.n_rot;
    pot_.n_xy = static_cast<int>(nxy);
    pot_.nr = s.nr;
    pot_.n_theta = s.nt;
    pot_.n_phi = s.nphi;
    pot_.ld = ld;
    pot_.n_blocks = s.n_blocks;
    pot_.mj_max = s.mj_max;
    pot_.initial_channel = s.i0;
    pot_.n_rep = s.n_rep;
    pot_.cb = cb;
    pot_.pphi = plan_phi_;
    pot_.twphi = tw_phi_;
    pot_.legendre = upload_real_lo(legendre, legendre64);
    pot_.block_first = upload_int(first);
    pot_.block_size = upload_int(size);
    pot_.block_slot = upload_int(slot);
    pot_.block_offset = upload_int(offset);
    pot_.irot_block = upload_int(irot_block);
    pot_.opt_z = opt_z_;
    pot_.before = before_;
    pot_.rot_half = rot_half_;
    pot_.sp2sc = sp2sc;
    pot_.sc2sp = sc2sp;
    pot_.expia = expia_;
    pot_.exp_mod = exp_mod;
    pot_.rep_of = upload_int(rep);
    pot_.phi_map = upload_int(phi_map);

    // The register-phi potential kernel: CB columns per chunk with CB * ntheta lines <= 128 threads and
    // at most ~110 KiB of shared memory (two blocks per SM), when nphi has an instantiation.
    pot2_cb_ = 0;
    if (pot2_phi_supported(s.nphi) && s.nt <= 32) {
      for (const int cb : {32, 8, 4}) {
        if (cb * s.nt > 128 || cb > nxy * 2) continue;
        const std::size_t need = pot2_smem<T>(cb, s.n_rot, s.nt, s.nphi, nxy);
        if (need <= std::min<std::size_t>(smem_optin, 110u << 10) || (cb == 4 && need <= static_cast<std::size_t>(smem_optin))) {
          pot2_cb_ = cb;
          pot2_smem_ = need;
          break;
        }
      }
    }
    if (pot2_cb_ > 0) {
      std::vector<double> leg_t(legendre.size()), leg_t64(legendre.size());
      for (int b = 0; b < s.n_blocks; ++b)
        for (int t = 0; t < s.nt; ++t)
          for (int j = 0; j < size[b]; ++j) {
            leg_t[offset[b] + j * s.nt + t] = legendre[offset[b] + t * size[b] + j];
            leg_t64[offset[b] + j * s.nt + t] = legendre64[offset[b] + t * size[b] + j];
          }
      pot2_.p = pot_;
      pot2_.legendre_t = upload_real_lo(leg_t, leg_t64);
      pot2_.cb = pot2_cb_;
      bool identity = s.n_rep == nxy;
      for (long long ixy = 0; ixy < nxy && identity; ++ixy) {
        identity = rep[ixy] == ixy;
        for (int p = 0; p < s.nphi && identity; ++p) identity = phi_map[ixy * s.nphi + p] == p;
      }
      pot2_.identity_maps = identity ? 1 : 0;
    }
    // The chunked potential kernel: one block per (point, chunk of pot3_cb_ columns), one thread per
    // (column, theta) line, F and D in at most the device's opt-in shared memory.
    pot3_cb_ = 0;
    if (pot2_cb_ > 0 && s.nt <= 16 && 2 * s.mj_max + 1 <= s.nphi) {
      std::vector<int> slot_first(s.nphi, 0), slot_nj(s.nphi, 0);
      int jp = 1;
      for (int b = 0; b < s.n_blocks; ++b) {
        require(slot_nj[slot[b]] == 0, "two mJ blocks share a phi slot");
        slot_first[slot[b]] = first[b];
        slot_nj[slot[b]] = size[b];
        jp = std::max(jp, size[b]);
      }
      const int cb = s.nt <= 4 ? 16 : 8;  // FP64 at cb = 32 spills; 16 columns keep 4+ warps per block
      const std::size_t need = pot3_smem<T>(cb, jp, s.nt, s.nphi);
      if (need <= static_cast<std::size_t>(smem_optin)) {
        std::vector<double> leg_slot(static_cast<std::size_t>(s.nphi) * jp * s.nt, 0.0), leg_slot64(leg_slot);
        for (int b = 0; b < s.n_blocks; ++b)
          for (int j = 0; j < size[b]; ++j)
            for (int t = 0; t < s.nt; ++t) {
              const std::size_t k = (static_cast<std::size_t>(slot[b]) * jp + j) * s.nt + t;
              leg_slot[k] = legendre[offset[b] + t * size[b] + j];
              leg_slot64[k] = legendre64[offset[b] + t * size[b] + j];
            }
        pot3_cb_ = cb;
        pot3_smem_ = need;
        pot3_chunks_ = static_cast<int>((nxy + cb - 1) / cb);
        pot3_args_ = pot2_;
        pot3_args_.cb = cb;
        pot3_args_.slot_first = upload_int(slot_first);
        pot3_args_.slot_nj = upload_int(slot_nj);
        pot3_args_.legendre_slot = upload_real_lo(leg_slot, leg_slot64);
        pot3_args_.jp = jp;
      }
    }
    // The persistent potential kernels with register-tiled contractions: potential4 (ntheta 4, 8, 16;
    // nphi 8, 16, 32) and potential5 (mixed form; ntheta 12 and 14 run on its 16-row tile, the matrix
    // rows of the missing theta zero and their phi lines skipped).
    const bool pot45_ok = pot2_cb_ > 0 && 2 * s.mj_max + 1 <= s.nphi;
    const int nt_k = (s.nt == 12 || s.nt == 14) ? 16 : s.nt;
    pot4_kernel_ = pot45_ok ? pot4_kernel_for<T>(s.nphi, s.nt) : nullptr;
    pot5_l2e_ = nt_k == 16 && !(std::getenv("SPO_B200_POT5_L2E") && std::string(std::getenv("SPO_B200_POT5_L2E")) == "0");
    Pot5Kernel<T> pot5_candidate = pot45_ok && s.n_rot % 2 == 0 ? pot5_kernel_for<T>(s.nphi, nt_k, pot5_l2e_) : nullptr;
    pot5_kernel_ = nullptr;
    if (pot4_kernel_ || pot5_candidate) {
      const int cb = 128 / nt_k;
      // Forward schedule: the slots in (+m, -m) pairs (m = 0 with an empty slot), pairs dealt to the four
      // warps largest first, each to the least loaded warp; half-warp 2w takes the first of each pair
      // of warp w, half-warp 2w + 1 the second.
      std::vector<int> slot_first(s.nphi, 0), slot_nj(s.nphi, 0);
      for (int b = 0; b < s.n_blocks; ++b) {
        slot_first[slot[b]] = first[b];
        slot_nj[slot[b]] = size[b];
      }
      struct Pair { int a, b, cost; };
      std::vector<Pair> pairs;
      std::vector<int> empty;
      for (int p = 0; p < s.nphi; ++p)
        if (slot_nj[p] == 0) empty.push_back(p);
      std::size_t next_empty = 0;
      auto take_empty = [&] { return next_empty < empty.size() ? empty[next_empty++] : -1; };
      for (int m = 0; m <= s.mj_max; ++m) {
        const int pa = m;                          // slot of +m
        const int pb = m == 0 ? take_empty() : s.nphi - m;  // slot of -m
        pairs.push_back({pa, pb, std::max(slot_nj[pa], pb >= 0 ? slot_nj[pb] : 0)});
      }
      while (next_empty < empty.size()) {
        const int pa = take_empty();
        pairs.push_back({pa, take_empty(), 0});
      }
      std::stable_sort(pairs.begin(), pairs.end(), [](const Pair& x, const Pair& y) { return x.cost > y.cost; });
      std::vector<std::vector<Pair>> warp(4);
      std::vector<int> load(4, 0);
      for (const Pair& pr : pairs) {
        const int w = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
        warp[w].push_back(pr);
        load[w] += pr.cost;
      }
      int len = 1;
      for (const auto& w : warp) len = std::max<int>(len, static_cast<int>(w.size()));
      std::vector<int> sched(8 * static_cast<std::size_t>(len), -1);
      for (int w = 0; w < 4; ++w)
        for (std::size_t k = 0; k < warp[w].size(); ++k) {
          sched[(2 * w) * len + k] = warp[w][k].a;
          sched[(2 * w + 1) * len + k] = warp[w][k].b;
        }
      std::vector<double> rows(static_cast<std::size_t>(s.n_rot) * (nt_k + 4), 0.0), rows12(rows), rows_lo(rows);
      std::vector<int> irot_slot(s.n_rot);
      for (int b = 0; b < s.n_blocks; ++b)
        for (int j = 0; j < size[b]; ++j) {
          irot_slot[first[b] + j] = slot[b];
          for (int t = 0; t < s.nt; ++t) {  // theta t >= s.nt (padding) stays zero
            const int quads = nt_k / 4;  // theta t at the position where the forward tiles read it
            const int pos = (t % quads) * 4 + t / quads;
            const std::size_t k = static_cast<std::size_t>(first[b] + j) * (nt_k + 4) + pos;
            rows[k] = legendre[offset[b] + t * size[b] + j];
            const double v = legendre64[offset[b] + t * size[b] + j];
            rows12[k] = round_bits(v, 12);
            rows_lo[k] = v - rows12[k];
          }
        }
      pot4_args_.p = pot2_.p;
      pot4_args_.leg_rows = upload_real(rows);
      pot4_args_.leg_rows12 = sizeof(T) == 4 ? upload_real(rows12) : nullptr;
      pot4_args_.leg_rows_lo = sizeof(T) == 4 ? upload_real(rows_lo) : nullptr;
      pot4_args_.slot_first = upload_int(slot_first);
      pot4_args_.slot_nj = upload_int(slot_nj);
      pot4_args_.irot_slot = upload_int(irot_slot);
      pot4_args_.fwd_sched = upload_int(sched);
      pot4_args_.sched_len = len;
      pot4_args_.chunks = static_cast<int>((nxy + cb - 1) / cb);
      pot4_args_.n_items = static_cast<long long>(s.nzp) * s.nr * pot4_args_.chunks;
      pot4_args_.identity_maps = pot2_.identity_maps;
      pot4_args_.nt_table = s.nt;
      pot4_args_.poll_limit = spo::pot5::kWaitLimit;
      pot4_args_.extra_tx = 0;
      int sms = 0;
      check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id), "SM count");
      const long long items = std::max<long long>(pot4_args_.n_items, 1);
      pot4_smem_ = spo::pot4_smem<T>(s.n_rot, s.nphi, s.nt, cb, len);
      if (pot4_kernel_ && pot4_smem_ <= static_cast<std::size_t>(smem_optin)) {
        check_cuda(cudaFuncSetAttribute(pot4_kernel_, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin),
                   "potential4 smem");
        int per_sm = 0;
        check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pot4_kernel_, 128, pot4_smem_),
                   "potential4 occupancy");
        pot4_blocks_ = static_cast<int>(std::min<long long>(static_cast<long long>(std::max(per_sm, 1)) * sms, items));
      } else {
        pot4_kernel_ = nullptr;
      }
      // potential5: the same tables, the item data by bulk asynchronous copies (columns of n_rot values:
      // 16-byte multiples when n_rot is even)
      pot5_smem_ = spo::pot5_smem<T>(s.n_rot, s.nphi, nt_k, cb, len, pot5_l2e_);
      if (pot5_candidate && pot5_smem_ <= static_cast<std::size_t>(smem_optin)) {
        pot5_kernel_ = pot5_candidate;
        check_cuda(cudaFuncSetAttribute(pot5_kernel_, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin),
                   "potential5 smem");
        check_cuda(cudaFuncSetAttribute(pot5_kernel_, cudaFuncAttributePreferredSharedMemoryCarveout, 100),
                   "potential5 carveout");
        int per_sm = 0;
        check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pot5_kernel_, 128, pot5_smem_),
                   "potential5 occupancy");
        pot5_blocks_per_sm_ = std::max(per_sm, 1);
        pot5_sms_ = sms;
        pot5_blocks_ = static_cast<int>(std::min<long long>(static_cast<long long>(pot5_blocks_per_sm_) * sms, items));
        error_flag_ = dev<int>(1);
        check_cuda(cudaMemset(error_flag_, 0, sizeof(int)), "error flag");
      }
    }
    // potential6 (mixed form): both theta contractions as split-precision TF32 tcgen05 GEMMs over 64-column
    // tiles, for the square heteronuclear basis JMax = MJMax = 15 with ntheta 16 and nphi 32 (configuration
    // 2's angular grid); one block of 256 threads per SM holding all 512 tensor-memory columns.
    pot6_kernel_ = nullptr;
    if constexpr (std::is_same_v<T, float>) {
      using B6 = spo::pot6::Basis<16>;
      bool square = pot2_cb_ > 0 && s.nt == 16 && s.nphi == 32 && s.n_rot == B6::kRot && s.n_blocks == B6::kBlocks;
      for (int b = 0; square && b < s.n_blocks; ++b) square = first[b] == B6::first(b) && size[b] == B6::nj(b);
      const std::size_t need = spo::pot6_smem<16>();
      if (square && need <= static_cast<std::size_t>(smem_optin)) {
        auto tf32 = [](double v) {  // round to TF32 (nearest, ties away from zero), as cvt.rna.tf32.f32
          const float f = static_cast<float>(v);
          uint32_t u;
          std::memcpy(&u, &f, 4);
          u = (u + 0x1000u) & 0xFFFFE000u;
          float r;
          std::memcpy(&r, &u, 4);
          return r;
        };
        // [forward hi | forward lo | transposed hi | transposed lo], canonical K-major layouts (core matrices
        // of 8 rows x 4 values): forward block b: N = theta (16) x K = J (padded to 8 or 16); transposed:
        // N = J (padded to 16) x K = theta (16).
        std::vector<float> tabs(2 * static_cast<std::size_t>(B6::kBfFloats + B6::kBbFloats), 0.0f);
        auto core = [](int n, int k) { return ((k / 4) * 2 + n / 8) * 32 + (n % 8) * 4 + k % 4; };
        for (int b = 0; b < s.n_blocks; ++b)
          for (int t = 0; t < 16; ++t)
            for (int j = 0; j < size[b]; ++j) {
              const double m = legendre[offset[b] + t * size[b] + j];
              const float hi = tf32(m), lo = tf32(m - static_cast<double>(hi));
              const std::size_t f = B6::bf_offset(b) + core(t, j);
              tabs[f] = hi;
              tabs[B6::kBfFloats + f] = lo;
              const std::size_t r = 2 * static_cast<std::size_t>(B6::kBfFloats) + b * 256 + core(j, t);
              tabs[r] = hi;
              tabs[B6::kBbFloats + r] = lo;
            }
        float* dtabs = dev<float>(tabs.size());
        check_cuda(cudaMemcpy(dtabs, tabs.data(), sizeof(float) * tabs.size(), cudaMemcpyHostToDevice), "potential6 tables");
        pot6_args_.p = pot2_.p;
        pot6_args_.bf = dtabs;
        pot6_args_.bb = dtabs + 2 * B6::kBfFloats;
        pot6_args_.tiles = static_cast<int>((nxy + spo::kPot6Tile - 1) / spo::kPot6Tile);
        pot6_args_.n_items = static_cast<long long>(s.nzp) * s.nr * pot6_args_.tiles;
        pot6_args_.identity_maps = pot2_.identity_maps;
        pot6_args_.poll_limit = spo::pot5::kWaitLimit;
        pot6_args_.extra_tx = 0;
        pot6_kernel_ = spo::potential6_kernel<32, 16>;
        pot6_smem_ = need;
        check_cuda(cudaFuncSetAttribute(pot6_kernel_, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(need)),
                   "potential6 smem");
        int sms = 0;
        check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id), "SM count");
        pot6_blocks_ = static_cast<int>(std::min<long long>(sms, std::max<long long>(pot6_args_.n_items, 1)));
        if (!error_flag_) {
          error_flag_ = dev<int>(1);
          check_cuda(cudaMemset(error_flag_, 0, sizeof(int)), "error flag");
        }
      }
    }
    if (pot3_cb_ > 0 || pot4_kernel_ || pot5_kernel_ || pot6_kernel_) {
      require(sizeof(V) * (nxy + 1) <= static_cast<std::size_t>(smem_optin), "nx*ny too large for the projection kernel");
      check_cuda(cudaFuncSetAttribute(spo::projection_finalize_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem_optin), "projection smem");
    }
    // The potential kernel is not chosen by timing: the kernels agree only to rounding (the compiler may
    // contract the products of a complex multiply into FMAs differently in each), and a timing choice
    // could then differ between two runs of the same case. The order is fixed: 5, 4, 3, 2, general.
    pot_kind_ = 1;
    if (use_v2_ && pot2_cb_ > 0) pot_kind_ = 2;
    if (use_v2_ && pot3_cb_ > 0) pot_kind_ = 3;
    if (use_v2_ && pot4_kernel_) pot_kind_ = 4;
    if (use_v2_ && pot5_kernel_) pot_kind_ = 5;
    pot_source_ = "default";
    use_pfa_ = true;
    if (const char* env = std::getenv("SPO_B200_PFA")) use_pfa_ = std::string(env) != "0";
    if (const char* env = std::getenv("SPO_B200_KERNELS")) {
      const std::string k(env);
      require(k == "v1" || k == "v2" || k == "v3" || k == "v4" || k == "v5" || k == "v6",
              "SPO_B200_KERNELS must be v1, v2, v3, v4, v5 or v6");
      use_v2_ = k != "v1";
      const int want = k[1] - '0';
      const bool have = want == 1 || (want == 2 && pot2_cb_ > 0) || (want == 3 && pot3_cb_ > 0) ||
                        (want == 4 && pot4_kernel_ != nullptr) || (want == 5 && pot5_kernel_ != nullptr) ||
                        (want == 6 && pot6_kernel_ != nullptr);
      // an unavailable kernel falls back to the best available one below it
      const bool avail[7] = {false, true, pot2_cb_ > 0, pot3_cb_ > 0, pot4_kernel_ != nullptr, pot5_kernel_ != nullptr,
                             pot6_kernel_ != nullptr};
      pot_kind_ = have ? want : 1;
      if (!have)
        for (int k = want - 1; k >= 2; --k)
          if (use_v2_ && avail[k]) {
            pot_kind_ = k;
            break;
          }
      pot_source_ = "fixed";
    }
    check_cuda(cudaStreamSynchronize(stream_), "set-up");
    autotune();
  }

  // Host FP64 complex -> device T, through the staging buffer.
  void copy_in(const double* src, V* dst, long long n) {
    for (long long i = 0; i < n; i += staging_elems_) {
      const long long m = std::min(staging_elems_, n - i);
      if constexpr (std::is_same_v<T, double>) {
        check_cuda(cudaMemcpyAsync(dst + i, src + 2 * i, sizeof(double2) * m, cudaMemcpyHostToDevice, stream_), "upload");
      } else {
        check_cuda(cudaMemcpyAsync(staging_, src + 2 * i, sizeof(double2) * m, cudaMemcpyHostToDevice, stream_), "upload");
        spo::convert_kernel<T, double><<<1184, 256, 0, stream_>>>(staging_, dst + i, m);
        check_cuda(cudaGetLastError(), "convert launch");
        check_cuda(cudaStreamSynchronize(stream_), "upload");
      }
    }
  }
  void copy_out(const V* src, double* dst, long long n) {
    for (long long i = 0; i < n; i += staging_elems_) {
      const long long m = std::min(staging_elems_, n - i);
      if constexpr (std::is_same_v<T, double>) {
        check_cuda(cudaMemcpyAsync(dst + 2 * i, src + i, sizeof(double2) * m, cudaMemcpyDeviceToHost, stream_), "download");
      } else {
        spo::convert_kernel<double, T><<<1184, 256, 0, stream_>>>(src + i, staging_, m);
        check_cuda(cudaGetLastError(), "convert launch");
        check_cuda(cudaMemcpyAsync(dst + 2 * i, staging_, sizeof(double2) * m, cudaMemcpyDeviceToHost, stream_), "download");
        check_cuda(cudaStreamSynchronize(stream_), "download");
      }
    }
  }

  Sizes s_;
  cudaStream_t stream_;
  cudaStream_t own_stream_;
  DeviceArena arena_;
  Profiler prof_;
  int launches_ = 0;
  spo::FftPlan plan_z_{}, plan_r_{}, plan_x_{}, plan_y_{}, plan_zs_{}, plan_phi_{};
  V *tw_z_ = nullptr, *tw_r_ = nullptr, *tw_x_ = nullptr, *tw_y_ = nullptr, *tw_zs_ = nullptr, *tw_phi_ = nullptr;
  V *zk_full_ = nullptr, *zk_half_ = nullptr, *rk_full_ = nullptr, *rk_half_ = nullptr;
  V *xyk_full_ = nullptr, *xyk_half_ = nullptr, *spec_full_ = nullptr, *spec_half_ = nullptr;
  V *rot_half_ = nullptr, *before_ = nullptr, *gas_step_ = nullptr, *spec_w_ = nullptr;
  V *shift_f_ = nullptr, *shift_b_ = nullptr;
  T* opt_z_ = nullptr;
  V *psi_ = nullptr, *chi_ = nullptr, *expia_ = nullptr;
  double* densities_ = nullptr;
  double2* staging_ = nullptr;
  long long staging_elems_ = 0;
  int xy_tb_ = 1;
  std::size_t xy_smem_ = 0, pot_smem_ = 0;
  spo::PotArgs<T> pot_{};
  spo::Pot2Args<T> pot2_{};
  int pot2_cb_ = 0;
  std::size_t pot2_smem_ = 0;
  bool use_v2_ = true;  // register-DFT kernels where instantiated (SPO_B200_KERNELS=v1: the general kernels)
  // Z and r lengths with a prime-factor split run axis2pfa_kernel (SPO_B200_PFA=0: the kernels with twiddles)
  bool use_pfa_ = true;
  V *zk_full_pfa_ = nullptr, *zk_half_pfa_ = nullptr, *rk_full_pfa_ = nullptr, *rk_half_pfa_ = nullptr;
  spo::Pot2Args<T> pot3_args_{};
  int pot3_cb_ = 0, pot3_chunks_ = 0;
  std::size_t pot3_smem_ = 0;
  Pot4Kernel<T> pot4_kernel_ = nullptr;
  spo::Pot4Args<T> pot4_args_{};
  int pot4_blocks_ = 0;
  std::size_t pot4_smem_ = 0;
  Pot5Kernel<T> pot5_kernel_ = nullptr;
  int pot5_blocks_ = 0, pot5_blocks_per_sm_ = 1, pot5_sms_ = 0;
  std::size_t pot5_smem_ = 0;
  bool pot5_l2e_ = false;  // potential5's L2E form (exp(i A) rows through L2, three blocks per SM)
  int* error_flag_ = nullptr;  // set by a kernel whose bounded wait gave up
  // the norm budget (norm_budget_setup / norm_budget_add) and the FP64 absorber factors it is built from
  std::vector<double> host_opt_z_, host_opt_r_, host_opt_zs_;
  spo::BudgetGrid budget_scat_{}, budget_spec_{};
  double* budget_out_ = nullptr;
  int budget_abs_ = 0;
  double budget_vol_scat_ = 0.0, budget_vol_spec_ = 0.0;
  bool budget_has_previous_ = false;
  int pot_kind_ = 1;  // 1 general, 2 potential2, 3 potential3, 4 potential4, 5 potential5, 6 potential6
  // potential6: both theta contractions on the tensor cores (mixed form, nphi 32, ntheta 16, square basis)
  spo::Pot6Args<float> pot6_args_{};
  void (*pot6_kernel_)(spo::Pot6Args<float>, int*) = nullptr;
  int pot6_blocks_ = 0;
  std::size_t pot6_smem_ = 0;
  std::string pot_source_ = "default";
  int tile_z_ = 0, tile_r_ = 0, tile_xy_ = 0;  // batch lanes per block of the register kinetic kernels (0: default)
  long long zr_window_ = 0;                     // lanes per Z+r window (0: two full passes)
  int rxy_planes_ = 0;                          // Z planes per r+xy slab (0: full passes)
  bool persist_z_ = false, persist_r_ = false, persist_xy_ = false;  // persistent forms of the passes
  bool balanced_ = false;  // balanced axis kernels where N2 = 2 N1
  std::string tiles_source_ = "default";
  // Asymptotic analysis (FP64).
  std::vector<cplx> shift_host_;
  spo_analysis_desc an_{};
  bool an_ready_ = false;
  int *an_rot_ = nullptr, *an_j_ = nullptr, *an_cx_ = nullptr, *an_cy_ = nullptr;
  double *an_phi_ = nullptr, *an_energies_ = nullptr;
  double2 *an_twx_ = nullptr, *an_twy_ = nullptr, *an_shift_ = nullptr, *an_bk_ = nullptr, *an_sums_ = nullptr;
};

inline Sizes sizes_of(const spo_desc& d) {
  Sizes s{};
  s.n_rot = d.n_rot;
  s.nx = d.nx;
  s.ny = d.ny;
  s.nr = d.nr;
  s.nz = d.nz;
  s.nzp = d.nz_potential;
  s.nzs = d.nz_specular;
  s.nt = d.n_theta;
  s.nphi = d.n_phi;
  s.i0 = d.initial_channel;
  s.ra = d.r_absorber_first;
  s.rb = d.r_absorber_last;
  s.spa = d.steps_per_analysis;
  s.n_rep = d.n_rep;
  s.n_ops = d.n_ops;
  s.n_blocks = d.n_mj_blocks;
  s.mj_max = (d.n_mj_blocks - 1) / 2;
  s.dt = d.time_step;
  require(s.n_rot > 0 && s.nx > 0 && s.ny > 0 && s.nr > 1 && s.nz > 0 && s.nzs > 0, "grid sizes must be positive (nR >= 2)");
  require(s.nzp >= 0 && s.nzp <= s.nz && s.nzp <= s.nzs, "nz_potential out of range");
  require(s.nt > 0 && s.nphi > 0 && s.n_blocks % 2 == 1 && s.n_blocks >= 1, "angular grid sizes invalid");
  require(s.nphi >= 2 * s.mj_max + 1, "n_phi < 2*MjMax + 1");
  require(s.i0 >= 0 && s.i0 < s.n_rot, "initial_channel out of range");
  require(s.spa >= 1, "steps_per_analysis must be >= 1");
  require(s.n_rep >= 1 && s.n_rep <= s.n_xy() && s.n_ops >= 1, "symmetry sizes invalid");
  require(s.ra >= 0 && s.rb < s.nr, "r absorber range invalid");
  require(d.precision == SPO_PRECISION_FP64 || d.precision == SPO_PRECISION_MIXED, "unknown precision");
  return s;
}


// The step of one precision form (defined in spo_step_f32.cu / spo_step_f64.cu).
std::unique_ptr<StepBase> make_step_f32(const spo_desc& d, const Sizes& s, cudaStream_t stream);
std::unique_ptr<StepBase> make_step_f64(const spo_desc& d, const Sizes& s, cudaStream_t stream);

}  // namespace spo_host
