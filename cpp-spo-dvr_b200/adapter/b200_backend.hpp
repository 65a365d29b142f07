// The B200 propagation backend as a spodvr::PropagationBackend: the drop-in for the reference's
// CpuBackend / CudaBackend behind its BackendFactory (src/propagation/propagation_backend.hpp:34-74).
// Compiled together with the reference's headers; all device work goes through the C ABI of
// include/spo_b200.h (libspo_b200.so).
#pragma once

#include <complex>
#include <functional>
#include <memory>
#include <span>
#include <vector>

#include "propagation/propagation_backend.hpp"

struct spo_handle;

namespace spodvr::b200 {

enum class Precision { Fp64, Mixed };

class B200Backend final : public PropagationBackend {
 public:
  // Takes over the potential grid (V in hartree; exp(-i V dt) is formed on the device in FP64) and the
  // initial specular wave, as every reference backend does (propagation_backend.hpp:61-62).
  B200Backend(const BackendInput& input, PotentialGrid potential, SpecularWave initial, Precision precision,
              int device);
  ~B200Backend() override;
  B200Backend(const B200Backend&) = delete;
  B200Backend& operator=(const B200Backend&) = delete;

  void read_wave_packet(const std::function<void(WavePacket&)>& read) override;
  [[nodiscard]] const WavePacket& wave_packet_on_host() override;
  void propagate_analysis_step() override;
  [[nodiscard]] const SpecularWave& specular() const override { return specular_; }
  [[nodiscard]] std::span<const std::complex<double>> z_plane(int iz) const override;
  [[nodiscard]] std::vector<double> block_densities() const override;
  void site_column(int ixy, std::span<std::complex<double>> out) const override;

 private:
  void check(int status, const char* what) const;
  WavePacket& host_packet();

  spo_handle* handle_ = nullptr;
  int n_rot_, n_xy_, n_zr_, nr_, nz_specular_;
  SpecularWave specular_;                         // host copy after every analysis step
  mutable std::vector<std::complex<double>> plane_;  // z_plane's buffer (valid until the next call)
  std::unique_ptr<WavePacket> host_;              // full host copy, only for restart and checkpoint
};

// The B200 backend as a BackendFactory (src/app/backend_factory.cpp:22-29 gains this entry).
[[nodiscard]] BackendFactory b200_backend_factory(Precision precision, int device = 0);

}  // namespace spodvr::b200
