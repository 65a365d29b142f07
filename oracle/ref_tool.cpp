// Test infrastructure: the reference's own CPU path driven from its public classes, for the parity
// tests, the golden fixtures and the CPU baseline. Linked against oracle/_ref/libspodvr_ref.so, the
// reference compiled from its sources (oracle/Makefile). Never part of the product.
//
//   spo_ref_tool case INPUT.json OUTDIR [--random SEED] [--analysis-steps K] [--stages] [--no-psi]
//       Sets up a run exactly as the reference program does (src/app/run.cpp:490-560:
//       read_input_file, make_potential, build_config, grids, symmetry, compute_potential_grid,
//       compute_gas_phase) and builds its WavePacketPropagation (src/propagation/propagation.cpp:9-22)
//       with a backend factory that records what crosses the PropagationBackend boundary
//       (BackendInput, PotentialGrid, SpecularWave: src/propagation/propagation_backend.hpp:63-74)
//       into OUTDIR/case/ and then builds the reference CpuBackend. With --random the wave packet is
//       replaced by the reference's 64-bit LCG values (tests/cuda/cuda_test_setup.hpp:53-64). It then
//       runs K analysis steps through PropagationBackend::propagate_analysis_step, after each one
//       recording chi, the BK coefficients of the time loop (src/propagation/propagation.cpp:75-94)
//       and, at the end, psi and the block densities. --stages additionally applies each operator
//       of one full sub-step once to the initial state (specular, T_Zr, T_xy, V) and records the
//       state after each.
//   spo_ref_tool time INPUT.json [--analysis-steps K] [--warmup W] [--random SEED]
//       Times K calls of CpuBackend::propagate_analysis_step after W warm-up calls; prints JSON.
#include <omp.h>

#include <chrono>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <memory>
#include <nlohmann/json.hpp>
#include <optional>
#include <span>
#include <string>
#include <vector>

#include "analysis/analysis_basis.hpp"
#include "analysis/balint_kurti.hpp"
#include "analysis/s_matrix.hpp"
#include "core/loop_schedule.hpp"
#include "fft/fftw_fft.hpp"
#include "gasphase/gas_phase.hpp"
#include "grids/angular_grid.hpp"
#include "grids/rotational_basis.hpp"
#include "grids/spatial_grids.hpp"
#include "input/json_input.hpp"
#include "input/process.hpp"
#include "linalg/symmetric_eigensolver.hpp"
#include "potential/potential_factory.hpp"
#include "potential/potential_grid.hpp"
#include "potential/potential_symmetry.hpp"
#include "propagation/analysis_surface.hpp"
#include "propagation/angular_transform.hpp"
#include "propagation/averages.hpp"
#include "propagation/cpu_backend.hpp"
#include "propagation/kinetic_operators.hpp"
#include "propagation/potential_operator.hpp"
#include "propagation/propagation.hpp"
#include "propagation/specular_operator.hpp"

namespace fs = std::filesystem;
using cplx = std::complex<double>;
using json = nlohmann::json;

namespace {

// The LCG of the reference's GPU tests: values in [-1, 1), real then imaginary part.
void fill_lcg(std::span<cplx> v, std::uint64_t seed) {
  std::uint64_t x = seed;
  auto next = [&x] {
    x = x * 6364136223846793005ULL + 1442695040888963407ULL;
    return double(x >> 11) / double(1ULL << 53) * 2.0 - 1.0;
  };
  for (auto& c : v) {
    const double re = next();
    c = {re, next()};
  }
}

template <typename T>
void write_array(const fs::path& path, std::span<const T> values) {
  std::ofstream out(path, std::ios::binary);
  out.write(reinterpret_cast<const char*>(values.data()), static_cast<std::streamsize>(values.size_bytes()));
  if (!out) throw std::runtime_error("cannot write " + path.string());
}
template <typename T>
void write_vec(const fs::path& path, const std::vector<T>& v) {
  write_array<T>(path, std::span<const T>(v));
}

struct Options {
  std::string mode;
  fs::path input;
  fs::path out;
  std::optional<std::uint64_t> random_seed;
  int analysis_steps = 1;
  int warmup = 1;
  bool stages = false;
  bool dump_psi = true;
};

Options parse(int argc, char** argv) {
  if (argc < 3) throw std::invalid_argument("usage: spo_ref_tool case|time INPUT.json [OUTDIR] [options]");
  Options o;
  o.mode = argv[1];
  o.input = argv[2];
  int i = 3;
  if (o.mode == "case") {
    if (argc < 4) throw std::invalid_argument("case needs OUTDIR");
    o.out = argv[3];
    i = 4;
  }
  for (; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--random" && i + 1 < argc) o.random_seed = std::stoull(argv[++i]);
    else if (a == "--analysis-steps" && i + 1 < argc) o.analysis_steps = std::stoi(argv[++i]);
    else if (a == "--warmup" && i + 1 < argc) o.warmup = std::stoi(argv[++i]);
    else if (a == "--stages") o.stages = true;
    else if (a == "--no-psi") o.dump_psi = false;
    else throw std::invalid_argument("unknown option " + a);
  }
  return o;
}

// Everything the reference sets up before the time loop (src/app/run.cpp:490-560).
struct Setup {
  spodvr::InputParameters input;
  std::unique_ptr<spodvr::Potential> pes;
  std::optional<spodvr::Config> config;
  std::optional<spodvr::AngularGrid> angular;
  std::optional<spodvr::SpatialGrids> grids;
  std::optional<spodvr::PotentialGrid> potential;
  std::optional<spodvr::GasPhase> gas;
  spodvr::FftwFft fft;
  spodvr::LapackEigensolver eigensolver;
  double potential_seconds = 0.0;

  explicit Setup(const fs::path& path) : input(spodvr::read_input_file(path)) {
    spodvr::apply_loop_schedule(spodvr::default_loop_schedule(spodvr::numa_node_count()));
    pes = spodvr::make_potential(input);
    config.emplace(spodvr::build_config(input, *pes));
    angular.emplace(spodvr::make_angular_grid(*config));
    grids.emplace(spodvr::make_spatial_grids(*config));
    spodvr::GridSymmetry symmetry = spodvr::make_grid_symmetry(*config, *angular);
    const spodvr::RotationalBasis basis(*angular, config->input.j_in, config->input.mj_in);
    const spodvr::ScatteringShape shape{basis.size(), config->input.nx, config->input.ny, config->input.nr,
                                        config->input.nz};
    const auto t0 = std::chrono::steady_clock::now();
    potential.emplace(spodvr::compute_potential_grid(*pes, *config, *grids, *angular, std::move(symmetry),
                                                     spodvr::xy_group_points(shape)));
    potential_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    gas.emplace(spodvr::compute_gas_phase(*config, *grids, *angular, potential->asymptotic, fft, eigensolver));
  }
};

// The boundary data of one run: what a PropagationBackend is constructed from.
void write_case(const fs::path& dir, const spodvr::BackendInput& in, const spodvr::PotentialGrid& potential,
                const spodvr::SpecularWave& initial) {
  fs::create_directories(dir);
  const spodvr::InputParameters& p = in.config.input;
  const spodvr::DerivedParameters& d = in.config.derived;
  const spodvr::PropagationTables& t = in.tables;
  const spodvr::GridSymmetry& sym = potential.symmetry;
  const spodvr::AngularTransform transform(in.angular, in.basis, in.fft);

  json m;
  m["n_rot"] = in.basis.size();
  m["nx"] = p.nx;
  m["ny"] = p.ny;
  m["nr"] = p.nr;
  m["nz"] = p.nz;
  m["nz_potential"] = in.grids.nz_potential;
  m["nz_specular"] = in.grids.z_specular.size();
  m["n_theta"] = in.angular.n_theta();
  m["n_phi"] = in.angular.n_phi();
  m["mj_max"] = in.basis.mj_max();
  m["initial_channel"] = in.basis.initial_index();
  m["r_absorber_first"] = in.grids.r_optical.first;
  m["r_absorber_last"] = in.grids.r_optical.last;
  m["steps_per_analysis"] = d.steps_per_analysis;
  m["time_step"] = p.time_step;
  m["n_rep"] = sym.n_representatives();
  m["n_ops"] = static_cast<int>(sym.operations().size());
  m["iz_analysis"] = in.grids.iz_analysis;
  m["dz"] = p.dz;
  m["dr"] = p.dr;
  m["xy_volume_element"] = d.xy_volume_element;
  m["fft_scale_z"] = t.fft_scale_z;
  m["fft_scale_r"] = t.fft_scale_r;
  m["fft_scale_x"] = t.fft_scale_x;
  m["fft_scale_y"] = t.fft_scale_y;
  m["parallel_energy"] = t.parallel_energy;
  m["system"] = p.system_id;
  std::vector<json> blocks;
  for (const auto& b : transform.mj_blocks()) blocks.push_back({b.fbr.first, b.fbr.size(), b.phi_slot});
  m["mj_blocks"] = blocks;
  std::vector<int> j_of, mj_of;
  for (int irot = 0; irot < in.basis.size(); ++irot) {
    j_of.push_back(in.basis.j(irot));
    mj_of.push_back(in.basis.mj(irot));
  }
  m["j"] = j_of;
  m["mj"] = mj_of;
  std::ofstream(dir / "manifest.json") << m.dump(1);
  // The angular DVR nodes (theta, phi), for features of the potential grid's points.
  write_vec(dir / "grid_theta.f64", std::vector<double>(in.angular.thetas().begin(), in.angular.thetas().end()));
  write_vec(dir / "grid_phi.f64", std::vector<double>(in.angular.phis().begin(), in.angular.phis().end()));

  auto c = [&](const char* name, const std::vector<cplx>& v) { write_vec(dir / (std::string(name) + ".c128"), v); };
  auto r = [&](const char* name, const std::vector<double>& v) { write_vec(dir / (std::string(name) + ".f64"), v); };
  c("z_kinetic_full", t.z_kinetic.full);
  c("z_kinetic_half", t.z_kinetic.half);
  c("r_kinetic_full", t.r_kinetic.full);
  c("r_kinetic_half", t.r_kinetic.half);
  c("zr_kinetic_full", t.zr_kinetic.full);
  c("zr_kinetic_half", t.zr_kinetic.half);
  c("xy_kinetic_full", t.xy_kinetic.full);
  c("xy_kinetic_half", t.xy_kinetic.half);
  c("specular_kinetic_full", t.specular_kinetic.full);
  c("specular_kinetic_half", t.specular_kinetic.half);
  c("rotation_full", t.rotation.full);
  c("rotation_half", t.rotation.half);
  r("z_optical", t.z_optical);
  r("r_optical", t.r_optical);
  r("z_specular_optical", t.z_specular_optical);
  c("gas_phase", t.gas_phase);
  c("shift_forward", t.shift_forward);
  c("shift_backward", t.shift_backward);
  c("specular_to_scattering", t.specular_to_scattering);
  c("scattering_to_specular", t.scattering_to_specular);
  r("xy_kinetic_energies", t.xy_kinetic_energies);
  r("rotational_energies", t.rotational_energies);
  r("legendre", transform.matrix());
  write_array<double>(dir / "potential.f64", std::span<const double>(potential.values.data(), potential.values.size()));
  r("asymptotic", potential.asymptotic);
  std::vector<int> rep, op, phi_index;
  for (int ixy = 0; ixy < sym.n_xy(); ++ixy) {
    rep.push_back(sym.representative_of(ixy));
    op.push_back(sym.operation_of(ixy));
  }
  for (int iop = 0; iop < static_cast<int>(sym.operations().size()); ++iop)
    for (const int i : sym.phi_index(iop)) phi_index.push_back(i);
  write_vec(dir / "representative_of.i32", rep);
  write_vec(dir / "operation_of.i32", op);
  write_vec(dir / "phi_index.i32", phi_index);
  write_array<cplx>(dir / "chi_initial.c128", std::span<const cplx>(initial.values.data(), initial.values.size()));
}

// The analysis side of the boundary: what the BK projection and the S-matrix use
// (src/analysis/balint_kurti.cpp:39-84, src/analysis/s_matrix.cpp:49-56).
void write_analysis(const fs::path& dir, const spodvr::Config& config, const spodvr::AnalysisBasis& a,
                    const spodvr::GasPhase& gas, const spodvr::SMatrixAccumulator& s) {
  json m;
  m["n_states"] = a.n_states();
  m["n_v"] = a.n_v();
  m["n_rotation"] = a.n_rotation();
  m["n_diffraction"] = a.n_diffraction();
  m["initial_state"] = a.initial_state();
  m["j_in"] = config.input.j_in;
  m["analysis_time_step"] = config.derived.analysis_time_step;
  m["n_energies"] = s.energies().size();
  m["j_max_gas"] = gas.states.j_max();
  const spodvr::DerivedParameters& d = config.derived;
  m["xy_scale"] = std::sqrt(d.dx * d.dy * std::sin(d.system.skewing_angle) / (config.input.nx * config.input.ny));
  std::vector<int> rot, chan_ix, chan_iy, state_j;
  for (int i = 0; i < a.n_rotation(); ++i) rot.push_back(a.rotation_index(i));
  for (int i = 0; i < a.n_diffraction(); ++i) {
    chan_ix.push_back(a.diffraction_channels()[i].ix);
    chan_iy.push_back(a.diffraction_channels()[i].iy);
  }
  for (int is = 0; is < a.n_states(); ++is) state_j.push_back(a.j(is));
  m["rotation_index"] = rot;
  m["channel_ix"] = chan_ix;
  m["channel_iy"] = chan_iy;
  m["state_j"] = state_j;
  std::ofstream(dir / "analysis.json") << m.dump(1);
  // phi_vj(r) for every analysed v and every j of the basis: (ir, j, v) as RovibrationalStates.
  std::vector<double> phi;
  for (int v = 0; v < a.n_v(); ++v)
    for (int j = 0; j <= gas.states.j_max(); ++j)
      for (const double x : gas.states.wave_function(v, j)) phi.push_back(x);
  write_vec(dir / "phi_vj.f64", phi);
  write_vec(dir / "analysis_energies_hartree.f64", s.energies().total_hartree);
}

void write_bk(const fs::path& path, const std::vector<spodvr::BkCoefficients>& records) {
  std::vector<cplx> all;
  for (const auto& bk : records) all.insert(all.end(), bk.values.begin(), bk.values.end());
  write_vec(path, all);
}

int run_case(const Options& o) {
  Setup s(o.input);
  const spodvr::Config& config = *s.config;
  spodvr::PropagationBackend* backend = nullptr;
  std::optional<spodvr::GridSymmetry> symmetry;
  std::vector<double> potential_values;  // unpremultiplied copy for --stages
  const fs::path case_dir = o.out / "case";
  auto factory = [&](const spodvr::BackendInput& in, spodvr::PotentialGrid potential, spodvr::SpecularWave initial) {
    write_case(case_dir, in, potential, initial);
    symmetry.emplace(potential.symmetry);
    if (o.stages) potential_values.assign(potential.values.begin(), potential.values.end());
    auto b = spodvr::make_cpu_backend(in, std::move(potential), std::move(initial));
    backend = b.get();
    return b;
  };
  spodvr::WavePacketPropagation propagation(config, *s.grids, *s.angular, std::move(*s.potential), *s.gas, s.fft,
                                            factory);
  fs::create_directories(o.out);
  spodvr::AnalysisBasis analysis_basis(config, *s.angular, propagation.rotational_basis(), *s.gas,
                                       propagation.tables().xy_kinetic_energies);
  spodvr::SMatrixAccumulator s_matrix(config, analysis_basis, *s.gas);
  write_analysis(case_dir, config, analysis_basis, *s.gas, s_matrix);

  if (o.random_seed) {
    backend->read_wave_packet([&](spodvr::WavePacket& psi) {
      fill_lcg(psi.scattering.values, *o.random_seed);
      fill_lcg(psi.specular.values, *o.random_seed + 1);
    });
  }
  const spodvr::WavePacket& psi0 = backend->wave_packet_on_host();
  if (o.dump_psi) write_vec(o.out / "psi_initial.c128", std::vector<cplx>(psi0.scattering.values.begin(), psi0.scattering.values.end()));
  write_vec(o.out / "chi_start.c128", std::vector<cplx>(psi0.specular.values.begin(), psi0.specular.values.end()));

  if (o.stages) {
    // One full sub-step, operator by operator, as CpuBackend builds them (src/propagation/cpu_backend.cpp:24-44).
    const spodvr::Config& c = config;
    const spodvr::RotationalBasis& basis = propagation.rotational_basis();
    const spodvr::ScatteringShape shape{basis.size(), c.input.nx, c.input.ny, c.input.nr, c.input.nz};
    const spodvr::AngularTransform transform(
        *s.angular, basis, s.fft,
        spodvr::AngularTransform::columns_per_pass(c.input.nx * c.input.ny, s.angular->n_theta(), s.angular->n_phi()));
    spodvr::premultiply_with_time_step(potential_values, c.input.time_step);
    const spodvr::ScatteringKineticOperator kinetic(shape, propagation.tables(), s.fft);
    const spodvr::PotentialOperator potential_op(shape, s.grids->nz_potential, basis.initial_index(),
                                                 propagation.tables(), transform, potential_values, *symmetry);
    const spodvr::SpecularOperator specular(c.input.nr, s.grids->z_specular.size(), s.grids->nz_potential,
                                            basis.initial_index(), s.grids->r_optical, propagation.tables(), s.fft);
    spodvr::WavePacket w = psi0;
    specular.apply(w.specular, spodvr::TimeStep::Full, false);
    write_vec(o.out / "stage_specular_chi.c128", std::vector<cplx>(w.specular.values.begin(), w.specular.values.end()));
    kinetic.apply_zr(w.scattering, spodvr::TimeStep::Full);
    write_vec(o.out / "stage_zr_psi.c128", std::vector<cplx>(w.scattering.values.begin(), w.scattering.values.end()));
    kinetic.apply_xy(w.scattering, spodvr::TimeStep::Full);
    write_vec(o.out / "stage_xy_psi.c128", std::vector<cplx>(w.scattering.values.begin(), w.scattering.values.end()));
    potential_op.apply(w);
    write_vec(o.out / "stage_potential_psi.c128", std::vector<cplx>(w.scattering.values.begin(), w.scattering.values.end()));
    write_vec(o.out / "stage_potential_chi.c128", std::vector<cplx>(w.specular.values.begin(), w.specular.values.end()));
  }

  // The time loop's per-analysis-step work (src/propagation/propagation.cpp:75-88).
  spodvr::AnalysisSurface surface(config, *s.grids, backend->specular());
  spodvr::BalintKurtiAnalyzer bk(config, *s.grids, analysis_basis, *s.gas, propagation.tables(), s.fft);
  std::vector<spodvr::BkCoefficients> records;
  std::vector<cplx> chis;
  std::vector<int> surface_index;
  std::vector<double> times;
  const spodvr::InputParameters& p = config.input;
  const int n_per_analysis = config.derived.steps_per_analysis;
  const auto t0 = std::chrono::steady_clock::now();
  for (int a = 0; a < o.analysis_steps; ++a) {
    backend->propagate_analysis_step();
    surface.update(backend->specular());
    records.push_back(bk.coefficients(backend->z_plane(s.grids->iz_analysis), backend->specular(), surface));
    const double time = p.t_end + ((a + 1) * n_per_analysis - p.n_steps) * p.time_step;
    s_matrix.add(records.back(), time);
    times.push_back(time);
    const auto& chi = backend->specular().values;
    chis.insert(chis.end(), chi.begin(), chi.end());
    surface_index.push_back(surface.fixed() ? surface.index() : -1 - surface.index());
  }
  const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  write_vec(o.out / "chi_steps.c128", chis);
  write_bk(o.out / "bk_steps.c128", records);
  write_vec(o.out / "surface_index.i32", surface_index);
  write_vec(o.out / "analysis_times.f64", times);
  const spodvr::WavePacket& psi = backend->wave_packet_on_host();
  if (o.dump_psi) write_vec(o.out / "psi_final.c128", std::vector<cplx>(psi.scattering.values.begin(), psi.scattering.values.end()));
  write_vec(o.out / "block_densities.f64", backend->block_densities());
  // The averages of the final wave packet (src/propagation/averages.cpp:37-80) with their inputs.
  {
    const double time = times.empty() ? p.t_end : times.back();
    const spodvr::Averages av = spodvr::compute_averages(time, psi, config, *s.grids, surface.index());
    write_vec(o.out / "averages.f64", std::vector<double>{av.norm, av.z_mean, av.r_mean, av.rest_norm});
    write_vec(o.out / "grid_z.f64", std::vector<double>(s.grids->z_scattering.points().begin(), s.grids->z_scattering.points().end()));
    write_vec(o.out / "grid_z_specular.f64", std::vector<double>(s.grids->z_specular.points().begin(), s.grids->z_specular.points().end()));
    write_vec(o.out / "grid_r.f64", std::vector<double>(s.grids->r.points().begin(), s.grids->r.points().end()));
    json g;
    g["volume_scattering"] = p.dz * p.dr * config.derived.xy_volume_element;
    g["volume_specular"] = p.dz * p.dr;
    g["iz_analysis"] = s.grids->iz_analysis;
    g["surface_index"] = surface.index();
    std::ofstream(o.out / "averages.json") << g.dump(1);
  }
  const spodvr::ScatteringResults results = s_matrix.results(surface.fixed_line());
  std::vector<double> p_reaction;
  for (const auto& e : results.energies) p_reaction.push_back(e.p_reaction);
  write_vec(o.out / "p_reaction.f64", p_reaction);
  json info;
  info["analysis_steps"] = o.analysis_steps;
  info["seconds"] = seconds;
  info["threads"] = omp_get_max_threads();
  info["potential_seconds"] = s.potential_seconds;
  info["random_seed"] = o.random_seed ? json(*o.random_seed) : json(nullptr);
  std::ofstream(o.out / "run.json") << info.dump(1);
  return 0;
}

int run_time(const Options& o) {
  Setup s(o.input);
  const spodvr::Config& config = *s.config;
  spodvr::PropagationBackend* backend = nullptr;
  auto factory = [&](const spodvr::BackendInput& in, spodvr::PotentialGrid potential, spodvr::SpecularWave initial) {
    auto b = spodvr::make_cpu_backend(in, std::move(potential), std::move(initial));
    backend = b.get();
    return b;
  };
  spodvr::WavePacketPropagation propagation(config, *s.grids, *s.angular, std::move(*s.potential), *s.gas, s.fft,
                                            factory);
  if (o.random_seed)
    backend->read_wave_packet([&](spodvr::WavePacket& psi) {
      fill_lcg(psi.scattering.values, *o.random_seed);
      fill_lcg(psi.specular.values, *o.random_seed + 1);
    });
  for (int w = 0; w < o.warmup; ++w) backend->propagate_analysis_step();
  const auto t0 = std::chrono::steady_clock::now();
  for (int a = 0; a < o.analysis_steps; ++a) backend->propagate_analysis_step();
  const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  const spodvr::InputParameters& p = config.input;
  const double n_pts = double(p.nz) * p.nr * p.nx * p.ny * s.angular->n_theta() * s.angular->n_phi();
  const int steps = o.analysis_steps * config.derived.steps_per_analysis;
  json out;
  out["analysis_steps"] = o.analysis_steps;
  out["time_steps"] = steps;
  out["seconds"] = seconds;
  out["threads"] = omp_get_max_threads();
  out["n_points"] = n_pts;
  out["grid_point_steps_per_s"] = n_pts * steps / seconds;
  out["potential_seconds"] = s.potential_seconds;
  std::cout << out.dump() << std::endl;
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    const Options o = parse(argc, argv);
    if (o.mode == "case") return run_case(o);
    if (o.mode == "time") return run_time(o);
    throw std::invalid_argument("unknown mode " + o.mode);
  } catch (const std::exception& e) {
    std::cerr << "spo_ref_tool: " << e.what() << '\n';
    return 1;
  }
}
