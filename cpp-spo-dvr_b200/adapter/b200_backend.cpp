// PropagationBackend over the C ABI of include/spo_b200.h. Every member maps onto one entry point:
//   constructor ............... spo_create (descriptor from BackendInput, PotentialGrid, SpecularWave)
//   read_wave_packet .......... spo_upload_state
//   wave_packet_on_host ....... spo_download_state
//   propagate_analysis_step ... spo_propagate_analysis_step, then spo_get_specular (chi stays on the host
//                               after every analysis step, as the reference's CUDA backend keeps it:
//                               src/cuda/cuda_backend.cpp:175-180)
//   z_plane ................... spo_get_z_plane
//   block_densities ........... spo_block_densities
//   site_column ............... spo_site_column
// A non-zero status becomes an exception of the reference's kinds, so run_program's exit codes stay
// (src/app/run.cpp:596-607): invalid descriptor -> std::invalid_argument, out of device memory ->
// NotSupportedError (as check_device_memory), any other failure -> std::runtime_error.
#include "b200_backend.hpp"

#include <stdexcept>
#include <string>

#include "../../include/spo_b200.h"
#include "core/error.hpp"
#include "propagation/angular_transform.hpp"

namespace spodvr::b200 {

namespace {
using cplx = std::complex<double>;

const double* flat(const std::vector<cplx>& v) { return reinterpret_cast<const double*>(v.data()); }
}  // namespace

void B200Backend::check(int status, const char* what) const {
  if (status == SPO_OK) return;
  const std::string message = std::string("B200 backend, ") + what + ": " + spo_last_error(handle_);
  if (status == SPO_ERR_INVALID) throw std::invalid_argument(message);
  if (status == SPO_ERR_OOM) throw NotSupportedError(message);
  throw std::runtime_error(message);
}

B200Backend::B200Backend(const BackendInput& in, PotentialGrid potential, SpecularWave initial, Precision precision,
                         int device)
    : n_rot_(in.basis.size()),
      n_xy_(in.config.input.nx * in.config.input.ny),
      n_zr_(in.config.input.nr * in.config.input.nz),
      nr_(in.config.input.nr),
      nz_specular_(initial.n_z()),
      specular_(std::move(initial)) {
  const InputParameters& p = in.config.input;
  const PropagationTables& t = in.tables;
  const GridSymmetry& sym = potential.symmetry;
  const AngularTransform transform(in.angular, in.basis, in.fft);

  std::vector<int> first, size, slot;
  for (const AngularTransform::MjBlock& b : transform.mj_blocks()) {
    first.push_back(b.fbr.first);
    size.push_back(b.fbr.size());
    slot.push_back(b.phi_slot);
  }
  std::vector<int> rep, op, phi_index;
  for (int ixy = 0; ixy < sym.n_xy(); ++ixy) {
    rep.push_back(sym.representative_of(ixy));
    op.push_back(sym.operation_of(ixy));
  }
  for (int iop = 0; iop < static_cast<int>(sym.operations().size()); ++iop)
    for (const int i : sym.phi_index(iop)) phi_index.push_back(i);

  spo_desc d{};
  d.n_rot = n_rot_;
  d.nx = p.nx;
  d.ny = p.ny;
  d.nr = p.nr;
  d.nz = p.nz;
  d.nz_potential = in.grids.nz_potential;
  d.nz_specular = nz_specular_;
  d.n_theta = in.angular.n_theta();
  d.n_phi = in.angular.n_phi();
  d.initial_channel = in.basis.initial_index();
  d.r_absorber_first = in.grids.r_optical.first;
  d.r_absorber_last = in.grids.r_optical.last;
  d.steps_per_analysis = in.config.derived.steps_per_analysis;
  d.time_step = p.time_step;
  d.n_mj_blocks = static_cast<int>(first.size());
  d.mj_fbr_first = first.data();
  d.mj_fbr_size = size.data();
  d.mj_phi_slot = slot.data();
  d.legendre = transform.matrix().data();
  d.z_kinetic_full = flat(t.z_kinetic.full);
  d.z_kinetic_half = flat(t.z_kinetic.half);
  d.r_kinetic_full = flat(t.r_kinetic.full);
  d.r_kinetic_half = flat(t.r_kinetic.half);
  d.xy_kinetic_full = flat(t.xy_kinetic.full);
  d.xy_kinetic_half = flat(t.xy_kinetic.half);
  d.specular_kinetic_full = flat(t.specular_kinetic.full);
  d.specular_kinetic_half = flat(t.specular_kinetic.half);
  d.rotation_half = flat(t.rotation.half);
  d.z_optical = t.z_optical.data();
  d.r_optical = t.r_optical.data();
  d.z_specular_optical = t.z_specular_optical.data();
  d.gas_phase = flat(t.gas_phase);
  d.shift_forward = flat(t.shift_forward);
  d.shift_backward = flat(t.shift_backward);
  d.specular_to_scattering = flat(t.specular_to_scattering);
  d.scattering_to_specular = flat(t.scattering_to_specular);
  d.fft_scale_z = t.fft_scale_z;
  d.fft_scale_r = t.fft_scale_r;
  d.fft_scale_x = t.fft_scale_x;
  d.fft_scale_y = t.fft_scale_y;
  d.n_rep = sym.n_representatives();
  d.n_ops = static_cast<int>(sym.operations().size());
  d.potential = potential.values.data();
  d.representative_of = rep.data();
  d.operation_of = op.data();
  d.phi_index = phi_index.data();
  d.chi_initial = reinterpret_cast<const double*>(specular_.values.data());
  d.precision = precision == Precision::Mixed ? SPO_PRECISION_MIXED : SPO_PRECISION_FP64;
  d.device = device;
  check(spo_create(&d, &handle_), "spo_create");
}

B200Backend::~B200Backend() { spo_destroy(handle_); }

WavePacket& B200Backend::host_packet() {
  if (!host_)
    host_ = std::make_unique<WavePacket>(WavePacket{ScatteringWave(n_rot_, n_xy_, n_zr_), SpecularWave(nr_, nz_specular_)});
  return *host_;
}

void B200Backend::read_wave_packet(const std::function<void(WavePacket&)>& read) {
  WavePacket& w = host_packet();
  read(w);
  check(spo_upload_state(handle_, reinterpret_cast<const double*>(w.scattering.values.data()),
                         reinterpret_cast<const double*>(w.specular.values.data())),
        "spo_upload_state");
  specular_.values.assign(w.specular.values.begin(), w.specular.values.end());
}

const WavePacket& B200Backend::wave_packet_on_host() {
  WavePacket& w = host_packet();
  check(spo_download_state(handle_, reinterpret_cast<double*>(w.scattering.values.data()),
                           reinterpret_cast<double*>(w.specular.values.data())),
        "spo_download_state");
  return w;
}

void B200Backend::propagate_analysis_step() {
  check(spo_propagate_analysis_step(handle_), "spo_propagate_analysis_step");
  check(spo_get_specular(handle_, reinterpret_cast<double*>(specular_.values.data())), "spo_get_specular");
}

std::span<const cplx> B200Backend::z_plane(int iz) const {
  plane_.resize(static_cast<std::size_t>(n_rot_) * n_xy_ * nr_);
  check(spo_get_z_plane(handle_, iz, reinterpret_cast<double*>(plane_.data())), "spo_get_z_plane");
  return plane_;
}

std::vector<double> B200Backend::block_densities() const {
  std::vector<double> out(n_zr_);
  check(spo_block_densities(handle_, out.data()), "spo_block_densities");
  return out;
}

void B200Backend::site_column(int ixy, std::span<cplx> out) const {
  if (out.size() < static_cast<std::size_t>(n_zr_) * n_rot_)
    throw std::invalid_argument("B200 backend, site_column: output too small");
  check(spo_site_column(handle_, ixy, reinterpret_cast<double*>(out.data())), "spo_site_column");
}

BackendFactory b200_backend_factory(Precision precision, int device) {
  return [precision, device](const BackendInput& in, PotentialGrid potential, SpecularWave initial) {
    return std::unique_ptr<PropagationBackend>(
        std::make_unique<B200Backend>(in, std::move(potential), std::move(initial), precision, device));
  };
}

}  // namespace spodvr::b200
