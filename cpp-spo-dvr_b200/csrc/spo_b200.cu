// C ABI of include/spo_b200.h over the host side in spo_host.cuh: handles, ensembles and the
// allocation-free block densities.
#include "spo_host.cuh"

using namespace spo_host;

struct spo_handle {
  std::string err;
  int device = 0;
  cudaStream_t stream = nullptr;
  Sizes s{};
  std::unique_ptr<StepBase> impl;
  int ensembles = 0;  // live ensembles whose graphs hold this handle's device pointers
};

namespace {
template <typename F>
int guarded(spo_handle* h, F&& f) {
  if (!h) return SPO_ERR_INVALID;
  try {
    check_cuda(cudaSetDevice(h->device), "cudaSetDevice");
    f();
    return SPO_OK;
  } catch (const SpoError& e) {
    h->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    h->err = e.what();
    return SPO_ERR_DEVICE;
  }
}
}  // namespace

extern "C" {

const char* spo_version(void) { return SPO_B200_VERSION; }

const char* spo_last_error(const spo_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int spo_create(const spo_desc* desc, spo_handle** out) {
  if (!out) return SPO_ERR_INVALID;
  *out = nullptr;
  auto h = std::make_unique<spo_handle>();
  try {
    require(desc != nullptr, "descriptor is null");
    h->s = sizes_of(*desc);
    h->device = desc->device;
    check_cuda(cudaSetDevice(h->device), "cudaSetDevice");
    check_cuda(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    if (desc->precision == SPO_PRECISION_FP64)
      h->impl = make_step_f64(*desc, h->s, h->stream);
    else
      h->impl = make_step_f32(*desc, h->s, h->stream);
  } catch (const SpoError& e) {
    g_create_error = e.what();
    if (h->stream) cudaStreamDestroy(h->stream);
    return e.code;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    if (h->stream) cudaStreamDestroy(h->stream);
    return SPO_ERR_DEVICE;
  }
  *out = h.release();
  return SPO_OK;
}

int spo_destroy(spo_handle* h) {
  if (!h) return SPO_OK;
  if (h->ensembles > 0) {
    h->err = "spo_destroy: the handle is a member of a live ensemble; destroy the ensemble first";
    return SPO_ERR_STATE;
  }
  cudaSetDevice(h->device);
  h->impl.reset();
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return SPO_OK;
}

int spo_propagate_analysis_step(spo_handle* h) {
  return guarded(h, [&] { h->impl->propagate_analysis_step(); });
}

int spo_upload_state(spo_handle* h, const double* psi, const double* chi) {
  return guarded(h, [&] { h->impl->upload(psi, chi); });
}

int spo_download_state(spo_handle* h, double* psi, double* chi) {
  return guarded(h, [&] { h->impl->download(psi, chi); });
}

int spo_get_specular(spo_handle* h, double* chi) {
  return guarded(h, [&] {
    require(chi != nullptr, "chi is null");
    h->impl->download(nullptr, chi);
  });
}

int spo_get_z_plane(spo_handle* h, int iz, double* out) {
  return guarded(h, [&] {
    require(out != nullptr, "out is null");
    h->impl->z_plane(iz, out);
  });
}

int spo_block_densities(spo_handle* h, double* out) {
  return guarded(h, [&] {
    require(out != nullptr, "out is null");
    h->impl->block_densities(out);
  });
}

int spo_site_column(spo_handle* h, int ixy, double* out) {
  return guarded(h, [&] {
    require(out != nullptr, "out is null");
    h->impl->site_column(ixy, out);
  });
}

int spo_analysis_setup(spo_handle* h, const spo_analysis_desc* d) {
  return guarded(h, [&] {
    require(d != nullptr, "analysis descriptor is null");
    h->impl->analysis_setup(*d);
  });
}

int spo_bk_coefficients(spo_handle* h, double time, int surface_fixed, int surface_index, int accumulate,
                        double* bk_out) {
  return guarded(h, [&] { h->impl->bk(time, surface_fixed != 0, surface_index, accumulate != 0, bk_out); });
}

int spo_s_matrix_sums(spo_handle* h, double* out) {
  return guarded(h, [&] {
    require(out != nullptr, "out is null");
    h->impl->s_sums(out);
  });
}

int spo_apply_stage(spo_handle* h, int stage, int half_step) {
  return guarded(h, [&] { h->impl->apply_stage(stage, half_step != 0); });
}

int spo_set_stream(spo_handle* h, void* cuda_stream) {
  return guarded(h, [&] { h->impl->set_stream(static_cast<cudaStream_t>(cuda_stream)); });
}

int spo_profile(spo_handle* h, int enable) {
  return guarded(h, [&] { h->impl->profile(enable != 0); });
}

int spo_profile_count(const spo_handle* h, int* n) {
  if (!h || !n) return SPO_ERR_INVALID;
  *n = static_cast<int>(h->impl->records().size());
  return SPO_OK;
}

int spo_profile_entry(const spo_handle* h, int i, char* name, int name_len, double* total_ms, int* launches,
                      double* bytes_per_launch) {
  if (!h) return SPO_ERR_INVALID;
  const auto& r = h->impl->records();
  if (i < 0 || i >= static_cast<int>(r.size())) return SPO_ERR_INVALID;
  if (name && name_len > 0) {
    std::strncpy(name, r[i].name.c_str(), static_cast<std::size_t>(name_len) - 1);
    name[name_len - 1] = '\0';
  }
  if (total_ms) *total_ms = r[i].ms;
  if (launches) *launches = r[i].launches;
  if (bytes_per_launch) *bytes_per_launch = r[i].bytes;
  return SPO_OK;
}

int spo_norm_budget_setup(spo_handle* h, const spo_norm_budget_desc* d, int* n_absorbers) {
  return guarded(h, [&] {
    require(d != nullptr && n_absorbers != nullptr, "spo_norm_budget_setup: null pointer");
    require(d->volume_scattering > 0.0 && d->volume_specular > 0.0, "spo_norm_budget_setup: volumes must be positive");
    require((d->z_low_first < 0 || (d->z_low_first <= d->z_low_last && d->z_low_last < h->s.nz)) &&
                (d->zs_low_first < 0 || (d->zs_low_first <= d->zs_low_last && d->zs_low_last < h->s.nzs)),
            "spo_norm_budget_setup: low absorber range out of the grid");
    *n_absorbers = h->impl->norm_budget_setup(*d);
  });
}

int spo_norm_budget_add(spo_handle* h, double* loss, double* loss_error, double* norms, int* has_window) {
  return guarded(h, [&] {
    require(loss && loss_error && norms && has_window, "spo_norm_budget_add: null pointer");
    double out[2 * spo::kBudgetMaxAbsorbers + 2];
    *has_window = h->impl->norm_budget_add(out) ? 1 : 0;
    if (!*has_window) return;
    const int n = h->impl->norm_budget_absorbers();
    for (int a = 0; a < n; ++a) {
      loss[a] = out[a];
      loss_error[a] = out[n + a];
    }
    norms[0] = out[2 * n];
    norms[1] = out[2 * n + 1];
  });
}

int spo_test_wait_timeout(spo_handle* h, int poll_limit, int unmatched_bytes) {
  if (h && (unmatched_bytes < 0 || unmatched_bytes % 16 != 0 || unmatched_bytes > 4096)) {
    h->err = "spo_test_wait_timeout: unmatched_bytes must be a multiple of 16 in [0, 4096]";
    return SPO_ERR_INVALID;
  }
  return guarded(h, [&] { h->impl->set_wait_test(poll_limit, static_cast<unsigned>(unmatched_bytes)); });
}

int spo_device_bytes(const spo_handle* h, unsigned long long* bytes) {
  if (!h || !bytes) return SPO_ERR_INVALID;
  *bytes = h->impl->bytes();
  return SPO_OK;
}

int spo_last_launch_count(const spo_handle* h, int* launches) {
  if (!h || !launches) return SPO_ERR_INVALID;
  *launches = h->impl->launches();
  return SPO_OK;
}

int spo_describe(const spo_handle* h, char* out, int out_len) {
  if (!h || !out || out_len <= 0) return SPO_ERR_INVALID;
  const std::string d = h->impl->describe();
  const std::size_t n = std::min<std::size_t>(d.size(), static_cast<std::size_t>(out_len - 1));
  std::memcpy(out, d.data(), n);
  out[n] = '\0';
  return SPO_OK;
}

int spo_averages(spo_handle* h, const double* z, const double* z_specular, const double* r, double volume_scattering,
                 double volume_specular, int iz_analysis, int surface_index, double* out) {
  return guarded(h, [&] {
    h->impl->averages(z, z_specular, r, volume_scattering, volume_specular, iz_analysis, surface_index, out);
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Ensembles: one analysis step of several handles captured as one CUDA graph, one branch per member
// between a fork and a join, so that one graph launch runs every member's kernel sequence and the
// independent members overlap on the GPU. Members whose every pass fills the GPU on its own (256 MiB
// or more of device memory) gain nothing from overlapping and lose L2 locality to it: their branches
// are chained one after another inside the graph (32 members of the configuration-4 sizes: 8.81e10
// grid-point-steps/s chained, 8.45e10 all overlapped).
// ---------------------------------------------------------------------------------------------
struct spo_ensemble {
  std::string err;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
  std::vector<spo_handle*> members;
  ~spo_ensemble() {
    for (spo_handle* m : members) --m->ensembles;
    cudaSetDevice(device);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (stream) cudaStreamDestroy(stream);
  }
};

extern "C" {

const char* spo_ensemble_last_error(const spo_ensemble* e) { return e ? e->err.c_str() : g_create_error.c_str(); }

int spo_ensemble_create(spo_handle* const* members, int n_members, spo_ensemble** out) {
  if (!out) return SPO_ERR_INVALID;
  *out = nullptr;
  auto e = std::make_unique<spo_ensemble>();
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> events;
  bool capturing = false;
  auto release = [&] {
    for (cudaStream_t b : branch) cudaStreamDestroy(b);
    for (cudaEvent_t ev : events) cudaEventDestroy(ev);
    branch.clear();
    events.clear();
  };
  try {
    require(members != nullptr && n_members > 0, "spo_ensemble_create: no members");
    for (int i = 0; i < n_members; ++i) {
      require(members[i] != nullptr, "spo_ensemble_create: null member");
      require(members[i]->device == members[0]->device, "spo_ensemble_create: members on different devices");
      for (int k = 0; k < i; ++k) require(members[k] != members[i], "spo_ensemble_create: a member appears twice");
    }
    e->device = members[0]->device;
    e->members.assign(members, members + n_members);
    for (spo_handle* m : e->members) ++m->ensembles;
    check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
    check_cuda(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    events.resize(n_members + 1, nullptr);
    for (cudaEvent_t& ev : events) check_cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
    branch.resize(n_members, nullptr);
    for (cudaStream_t& b : branch) check_cuda(cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking), "cudaStreamCreate");
    // Kernel profiling records events around each launch; a captured graph replays without them.
    for (spo_handle* m : e->members) m->impl->profile(false);
    check_cuda(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
    capturing = true;
    check_cuda(cudaEventRecord(events[0], e->stream), "cudaEventRecord");
    unsigned long long fills_gpu = 256ull << 20;  // SPO_B200_ENSEMBLE_CHAIN_BYTES overrides it
    if (const char* env = std::getenv("SPO_B200_ENSEMBLE_CHAIN_BYTES")) fills_gpu = std::stoull(env);
    cudaEvent_t chain = events[0];  // the last large member's end
    for (int i = 0; i < n_members; ++i) {
      StepBase& m = *e->members[i]->impl;
      const bool large = m.bytes() >= fills_gpu;
      check_cuda(cudaStreamWaitEvent(branch[i], large ? chain : events[0], 0), "cudaStreamWaitEvent");
      if (large) chain = events[i + 1];
      m.set_stream(branch[i]);
      m.enqueue_analysis_step();
      m.set_stream(nullptr);
      e->launches += m.launches();
      check_cuda(cudaEventRecord(events[i + 1], branch[i]), "cudaEventRecord");
      check_cuda(cudaStreamWaitEvent(e->stream, events[i + 1], 0), "cudaStreamWaitEvent");
    }
    capturing = false;
    check_cuda(cudaStreamEndCapture(e->stream, &e->graph), "cudaStreamEndCapture");
    check_cuda(cudaGraphInstantiate(&e->exec, e->graph, 0), "cudaGraphInstantiate");
  } catch (const std::exception& ex) {
    if (capturing) {
      cudaGraph_t partial = nullptr;
      cudaStreamEndCapture(e->stream, &partial);
      if (partial) cudaGraphDestroy(partial);
    }
    for (spo_handle* m : e->members) m->impl->set_stream(nullptr);
    release();
    g_create_error = ex.what();
    const auto* se = dynamic_cast<const SpoError*>(&ex);
    return se ? se->code : SPO_ERR_DEVICE;
  }
  release();
  *out = e.release();
  return SPO_OK;
}

int spo_ensemble_step(spo_ensemble* e) {
  if (!e) return SPO_ERR_INVALID;
  try {
    check_cuda(cudaSetDevice(e->device), "cudaSetDevice");
    check_cuda(cudaGraphLaunch(e->exec, e->stream), "cudaGraphLaunch");
    check_cuda(cudaStreamSynchronize(e->stream), "spo_ensemble_step");
    return SPO_OK;
  } catch (const SpoError& ex) {
    e->err = ex.what();
    return ex.code;
  } catch (const std::exception& ex) {
    e->err = ex.what();
    return SPO_ERR_DEVICE;
  }
}

int spo_ensemble_launch_count(const spo_ensemble* e, int* launches) {
  if (!e || !launches) return SPO_ERR_INVALID;
  *launches = e->launches;
  return SPO_OK;
}

int spo_ensemble_destroy(spo_ensemble* e) {
  delete e;
  return SPO_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// spo_block_densities_noalloc: the block-density kernel with its per-block sums in a file-scope
// device array instead of a handle's allocation (see include/spo_b200.h for who needs this).
// ---------------------------------------------------------------------------------------------
namespace {

// Per-block sums of every call (SPO_NOALLOC_MAX_BLOCKS doubles, 512 KiB per device). In host code
// this name is only a host-side stand-in for the symbol: its device address comes from
// cudaGetSymbolAddress, looked up once per device.
__device__ __align__(256) double g_noalloc_density_scratch[SPO_NOALLOC_MAX_BLOCKS];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
std::atomic<double*> g_noalloc_ptr[kMaxDevices] = {};

// The array's address on the current device. Only a successful lookup is kept: a lookup that fails
// for a passing reason (memory exhausted while the module loads lazily, an error left by earlier work)
// is tried again by the next call.
double* noalloc_scratch(int device) {
  if (double* p = g_noalloc_ptr[device].load(std::memory_order_acquire)) return p;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (double* p = g_noalloc_ptr[device].load(std::memory_order_acquire)) return p;
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_density_scratch);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();  // clears the lookup's own error if it is not sticky; the next call retries
    check_cuda(e, "cudaGetSymbolAddress(g_noalloc_density_scratch)");
  }
  g_noalloc_ptr[device].store(static_cast<double*>(p), std::memory_order_release);
  return static_cast<double*>(p);
}

}  // namespace

extern "C" int spo_block_densities_noalloc(const void* psi_device, int precision, long long n_blocks,
                                           long long block_size, double* out_host, void* cuda_stream) {
  try {
    require(psi_device != nullptr && out_host != nullptr, "spo_block_densities_noalloc: null pointer");
    require(precision == SPO_PRECISION_FP64 || precision == SPO_PRECISION_MIXED,
            "spo_block_densities_noalloc: unknown precision");
    require(n_blocks > 0 && block_size > 0, "spo_block_densities_noalloc: n_blocks and block_size must be positive");
    require(n_blocks <= SPO_NOALLOC_MAX_BLOCKS,
            "spo_block_densities_noalloc: n_blocks = " + std::to_string(n_blocks) + " exceeds SPO_NOALLOC_MAX_BLOCKS = " +
                std::to_string(SPO_NOALLOC_MAX_BLOCKS));
    int device = 0;
    check_cuda(cudaGetDevice(&device), "cudaGetDevice");
    require(device >= 0 && device < kMaxDevices, "spo_block_densities_noalloc: device ordinal out of range");
    const auto stream = static_cast<cudaStream_t>(cuda_stream);
    // The call ends with a synchronisation and a copy into pageable host memory, which a capturing
    // stream refuses: it cannot be captured, so it refuses a capturing stream up front.
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    check_cuda(cudaStreamIsCapturing(stream, &capture), "cudaStreamIsCapturing");
    if (capture != cudaStreamCaptureStatusNone)
      throw SpoError(SPO_ERR_STATE, "spo_block_densities_noalloc: the stream is capturing; this call cannot be captured");
    // An error left by the caller's earlier work is reported as such (and left pending), not as a
    // failure of this call's launch.
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
      throw SpoError(SPO_ERR_DEVICE, std::string("spo_block_densities_noalloc: a CUDA error from earlier work is "
                                                 "pending on this thread (not cleared): ") +
                                         cudaGetErrorString(pending));
    double* scratch = noalloc_scratch(device);
    if (precision == SPO_PRECISION_FP64)
      spo::block_density_kernel<double><<<static_cast<unsigned>(n_blocks), 256, 0, stream>>>(
          static_cast<const double2*>(psi_device), block_size, scratch);
    else
      spo::block_density_kernel<float><<<static_cast<unsigned>(n_blocks), 256, 0, stream>>>(
          static_cast<const float2*>(psi_device), block_size, scratch);
    check_cuda(cudaGetLastError(), "block_density_kernel launch");
    check_cuda(cudaMemcpyAsync(out_host, scratch, sizeof(double) * n_blocks, cudaMemcpyDeviceToHost, stream),
               "block densities copy");
    check_cuda(cudaStreamSynchronize(stream), "spo_block_densities_noalloc");
    return SPO_OK;
  } catch (const SpoError& e) {
    g_create_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    return SPO_ERR_DEVICE;
  }
}
