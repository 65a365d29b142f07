/*
 * spo_b200.h - C ABI of the B200 (sm_100a) split-operator propagation step.
 *
 * A drop-in for the propagation backend of SPO-DVR: every entry point below replaces one member of
 * the reference's PropagationBackend interface (src/propagation/propagation_backend.hpp:34-59) or
 * of its construction (BackendInput + BackendFactory, propagation_backend.hpp:63-74). The
 * descriptor carries exactly the data a backend is built from there: the grid sizes, the
 * precomputed FP64 factor tables (PropagationTables, src/propagation/propagation_tables.hpp:26-72),
 * the angular transform tables (AngularTransform::mj_blocks/matrix, angular_transform.hpp:67-76),
 * the surface-symmetry maps and the potential grid in hartree (PotentialGrid,
 * src/potential/potential_grid.hpp:21-37) and the initial specular wave.
 *
 * Conventions:
 *   - plain C types only; complex numbers are interleaved (re, im) pairs of double;
 *   - every call returns an int status (SPO_OK = 0); no exception crosses the ABI;
 *     spo_last_error(h) gives the message of the last failure of a handle;
 *   - a handle owns all its device memory and one CUDA stream; it is not thread-safe;
 *     every call is synchronous with respect to the host buffers it is given;
 *   - the host-side layouts are the reference's host layouts (src/propagation/wave_function.hpp):
 *       psi[irot + n_rot*(ixy + nx*ny*izr)], ixy = iy + ny*ix, izr = ir + nr*iz
 *       chi[ir + nr*iz] on the specular Z grid.
 *   - the device layout of psi is the same (irot fastest), so readbacks are plain copies.
 */
#ifndef SPO_B200_H
#define SPO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define SPO_B200_VERSION "0.1.0"

/* Status codes. */
enum spo_status {
  SPO_OK = 0,
  SPO_ERR_INVALID = 1,   /* invalid argument or descriptor (reference: InputError / invalid_argument) */
  SPO_ERR_OOM = 2,       /* device memory exhausted (reference: check_device_memory, NotSupportedError) */
  SPO_ERR_DEVICE = 3,    /* CUDA error (reference: CudaError, src/cuda/cuda_error.hpp:10-23) */
  SPO_ERR_TIMEOUT = 4,   /* a bounded device-side wait gave up */
  SPO_ERR_STATE = 5      /* call not valid in the handle's current state */
};

/* Arithmetic of the step: FP64 (complex128 psi, FP64 FFTs and factors), or mixed (complex64 psi,
 * FP32 FFTs and factors rounded once from the FP64 tables; exp(-iV dt) formed in FP64 on the
 * device, then rounded). */
enum spo_precision { SPO_PRECISION_FP64 = 0, SPO_PRECISION_MIXED = 1 };

/* Everything a propagation backend is built from (BackendInput + PotentialGrid + SpecularWave).
 * All pointers are host pointers, read during spo_create only. */
typedef struct spo_desc {
  /* --- grid sizes ------------------------------------------------------------------------ */
  int n_rot;            /* rotational FBR basis size, RotationalBasis::size() */
  int nx, ny, nr, nz;   /* scattering grid */
  int nz_potential;     /* Z points with Z < zasymp (SpatialGrids::nz_potential) */
  int nz_specular;      /* specular Z grid */
  int n_theta, n_phi;   /* angular DVR grid */
  int initial_channel;  /* RotationalBasis::initial_index() */
  int r_absorber_first, r_absorber_last;  /* SpatialGrids::r_optical (inclusive) */
  int steps_per_analysis;                 /* Config::derived.steps_per_analysis (nanspo) */
  double time_step;                       /* dtStep (hartree^-1 units of the reference) */

  /* --- angular transform (AngularTransform::mj_blocks / matrix) ---------------------------- */
  int n_mj_blocks;             /* 2*MjMax + 1, in the order mJ = -MjMax .. MjMax */
  const int* mj_fbr_first;     /* first FBR index of each block */
  const int* mj_fbr_size;      /* number of J values of each block */
  const int* mj_phi_slot;      /* phi FFT slot of each block's mJ */
  const double* legendre;      /* sqrt(w_t/nphi) P_J^m(theta_t), ordered (block, theta, J) */

  /* --- factor tables (PropagationTables), complex as (re, im) pairs ------------------------ */
  const double* z_kinetic_full;        /* nz  */
  const double* z_kinetic_half;        /* nz  (principal square root of the full step) */
  const double* r_kinetic_full;        /* nr  */
  const double* r_kinetic_half;        /* nr  */
  const double* xy_kinetic_full;       /* nx*ny */
  const double* xy_kinetic_half;       /* nx*ny */
  const double* specular_kinetic_full; /* nr*nz_specular, (ir, iz) */
  const double* specular_kinetic_half; /* nr*nz_specular */
  const double* rotation_half;         /* n_rot*nr, (irot, ir): exp(-i E_rot dt/2) */
  const double* z_optical;             /* nz, real: exp(-V_opt dt) */
  const double* r_optical;             /* nr, real */
  const double* z_specular_optical;    /* nz_specular, real */
  const double* gas_phase;             /* nr: exp(-i vasy(r) dt) */
  const double* shift_forward;         /* nx*ny: exp(-i k0.R) */
  const double* shift_backward;        /* nx*ny */
  const double* specular_to_scattering;  /* nx*ny */
  const double* scattering_to_specular;  /* nx*ny */
  double fft_scale_z, fft_scale_r, fft_scale_x, fft_scale_y;

  /* --- potential on the interaction region (PotentialGrid) --------------------------------- */
  int n_rep;                    /* (x, y) representatives of the surface symmetry */
  int n_ops;                    /* usable symmetry operations */
  const double* potential;      /* V (hartree), (itp, irep, izr), itp = iphi + nphi*itheta, izr < nz_potential*nr */
  const int* representative_of; /* nx*ny */
  const int* operation_of;      /* nx*ny */
  const int* phi_index;         /* n_ops*n_phi */

  /* --- initial state and options ----------------------------------------------------------- */
  const double* chi_initial;    /* nr*nz_specular complex: the initial packet; psi starts at zero */
  int precision;                /* enum spo_precision */
  int device;                   /* CUDA device ordinal */
} spo_desc;

typedef struct spo_handle spo_handle;

/* Library version string. */
const char* spo_version(void);

/* Message of the last failed call on h (or of the last failed spo_create when h is NULL). */
const char* spo_last_error(const spo_handle* h);

/* Builds a backend: uploads the tables, forms exp(-iV dt) on the device in FP64, zeroes psi and
 * sets chi to desc->chi_initial. Replaces the CpuBackend/CudaBackend constructors
 * (src/propagation/cpu_backend.cpp:24-44) behind BackendFactory (propagation_backend.hpp:73-74). */
int spo_create(const spo_desc* desc, spo_handle** out);

/* Frees the handle and all its device memory. Refused with SPO_ERR_STATE while the handle is a
 * member of a live ensemble (whose graph holds its device pointers). */
int spo_destroy(spo_handle* h);

/* [T(dt/2) V(dt) T(dt/2)]^n over one analysis step, n = steps_per_analysis.
 * Replaces PropagationBackend::propagate_analysis_step (propagation_backend.hpp:47). */
int spo_propagate_analysis_step(spo_handle* h);

/* Replaces the wave packet (restart): psi (n_rot*nx*ny*nr*nz complex) and chi (nr*nz_specular
 * complex) in host layout. Replaces PropagationBackend::read_wave_packet (propagation_backend.hpp:40). */
int spo_upload_state(spo_handle* h, const double* psi, const double* chi);

/* Copies the wave packet to the host layout (checkpoint). Either pointer may be NULL.
 * Replaces PropagationBackend::wave_packet_on_host (propagation_backend.hpp:44). */
int spo_download_state(spo_handle* h, double* psi, double* chi);

/* The specular wave chi (nr*nz_specular complex). Replaces PropagationBackend::specular (:50). */
int spo_get_specular(spo_handle* h, double* chi);

/* The nr (Z, r) blocks of Z index iz, layout (irot, ixy, ir): n_rot*nx*ny*nr complex.
 * Replaces PropagationBackend::z_plane (propagation_backend.hpp:52). */
int spo_get_z_plane(spo_handle* h, int iz, double* out);

/* sum |psi|^2 over (irot, ixy) at every izr (nz*nr doubles), summed in a fixed order on the
 * device in FP64. Replaces PropagationBackend::block_densities (propagation_backend.hpp:55). */
int spo_block_densities(spo_handle* h, double* out);

/* The scattering wave at one (x, y) point, layout (izr, irot) with izr fastest (nz*nr*n_rot
 * complex). Replaces PropagationBackend::site_column (propagation_backend.hpp:58). */
int spo_site_column(spo_handle* h, int ixy, double* out);

/* ---------------------------------------------------------------------------------------------
 * Asymptotic analysis on the device, in FP64 whatever the precision form: the Balint-Kurti
 * projection at the analysis line (BalintKurtiAnalyzer::coefficients, src/analysis/balint_kurti.cpp:
 * 39-84) and the on-the-fly S-matrix sums (SMatrixAccumulator::add, src/analysis/s_matrix.cpp:49-56).
 * The data are those of AnalysisBasis, GasPhase and AnalysisEnergies of the reference.
 * --------------------------------------------------------------------------------------------- */
typedef struct spo_analysis_desc {
  int n_v;                    /* vibrational levels analysed (AnalysisBasis::n_v) */
  int n_rotation;             /* analysed rotational states (AnalysisBasis::n_rotation) */
  int n_diffraction;          /* diffraction channels (AnalysisBasis::n_diffraction) */
  const int* rotation_index;  /* n_rotation: index of each analysed state in the propagation basis */
  const int* rotation_j;      /* n_rotation: its J */
  const int* channel_ix;      /* n_diffraction: (x, y) FFT slot of each diffraction channel */
  const int* channel_iy;
  int j_max_gas;              /* phi_vj holds j = 0 .. j_max_gas */
  const double* phi_vj;       /* (ir, j, v): the gas-phase vibrational functions phi_vj(r) */
  int initial_state;          /* is of (JIn, MJIn, n = m = 0) */
  int j_in;
  int iz_analysis;            /* Z index of the analysis line on the scattering grid */
  double dr;                  /* r grid step */
  double xy_scale;            /* sqrt(dx dy sin(skew) / (nx ny)) */
  int n_energies;
  const double* energies_hartree;  /* the analysis energies (total, hartree) */
  double analysis_time_step;       /* steps_per_analysis * dt */
} spo_analysis_desc;

/* Uploads the analysis data; the S-matrix sums start at zero. */
int spo_analysis_setup(spo_handle* h, const spo_analysis_desc* d);

/* BK coefficients of the current wave packet, (is, v) with is = irotana * n_diffraction + idif
 * (n_rotation * n_diffraction * n_v complex) into bk_out (may be NULL). With surface_fixed != 0 the
 * initial state's coefficient comes from the specular wave at surface_index (the fixed specular
 * analysis line). With accumulate != 0 they are also added to the S-matrix sums at `time`. */
int spo_bk_coefficients(spo_handle* h, double time, int surface_fixed, int surface_index, int accumulate,
                        double* bk_out);

/* The S-matrix sums, (is, v, ien): n_rotation * n_diffraction * n_v * n_energies complex. */
int spo_s_matrix_sums(spo_handle* h, double* out);

/* Operators of one sub-step, for stage-by-stage checks (the reference tests its operators one by one:
 * tests/test_propagation.cpp, test_cuda_backend.cpp:161-278). */
enum spo_stage {
  SPO_STAGE_SPECULAR = 0,          /* SpecularOperator::apply, kinetic + gas phase + absorbers (specular_operator.cpp:40-45) */
  SPO_STAGE_SPECULAR_KINETIC = 1,  /* SpecularOperator::apply with kinetic_only (the last half step) */
  SPO_STAGE_ZR = 2,                /* ScatteringKineticOperator::apply_zr (kinetic_operators.cpp:77-111) */
  SPO_STAGE_XY = 3,                /* ScatteringKineticOperator::apply_xy (kinetic_operators.cpp:114-124) */
  SPO_STAGE_POTENTIAL = 4          /* PotentialOperator::apply (potential_operator.cpp:84-94) */
};

/* Applies one operator to the resident state, with the full (half_step = 0) or half (1) step's factors. */
int spo_apply_stage(spo_handle* h, int stage, int half_step);

/* Runs the handle's work on the caller's CUDA stream (a cudaStream_t of the handle's device, passed
 * as void*), e.g. to bracket it with the caller's CUDA events; NULL returns to the handle's own stream. */
int spo_set_stream(spo_handle* h, void* cuda_stream);

/* Per-kernel timing: with enable != 0 every kernel launch of the following calls is bracketed by
 * CUDA events on the launching stream and its duration added to a per-kernel record (reset by
 * each spo_profile call). */
int spo_profile(spo_handle* h, int enable);

/* Number of per-kernel records. */
int spo_profile_count(const spo_handle* h, int* n);

/* Record i: kernel name (NUL-terminated, truncated to name_len), summed duration (ms), launches,
 * and the algorithmic bytes one launch must move (its minimal HBM traffic: state read + written
 * once, plus the exp(iV dt) table read once by the potential kernel). */
int spo_profile_entry(const spo_handle* h, int i, char* name, int name_len, double* total_ms, int* launches,
                      double* bytes_per_launch);

/* Failure-detection test of the bounded device-side waits (no counterpart in the reference, whose kernels
 * do not wait on barriers). With unmatched_bytes > 0 (a multiple of 16, at most 4096) every item of the
 * potential kernels that move their data by bulk asynchronous copies (potential5, potential6) announces that
 * many bytes more on its first barrier than its copies deliver, so the barrier's phase cannot complete;
 * every copy stays valid and lands. Each wait gives up after poll_limit polls (<= 0: the default limit), the
 * block records the failure, waits (bounded) for its work in flight and leaves, and the next
 * spo_propagate_analysis_step returns SPO_ERR_TIMEOUT; the wave packet is then undefined until the next
 * spo_upload_state. spo_test_wait_timeout(h, 0, 0) restores normal operation. */
int spo_test_wait_timeout(spo_handle* h, int poll_limit, int unmatched_bytes);

/* Bytes of device memory the handle holds. */
int spo_device_bytes(const spo_handle* h, unsigned long long* bytes);

/* Number of kernel launches the last spo_propagate_analysis_step issued. */
int spo_last_launch_count(const spo_handle* h, int* launches);

/* The kernels and tile shapes the handle chose (kernel per pass, tile width per kinetic pass, and
 * whether the autotuner or an environment setting chose them), as one NUL-terminated line truncated
 * to out_len bytes. No counterpart in the reference (its CUDA backend has one fixed plan). */
int spo_describe(const spo_handle* h, char* out, int out_len);

/* Norm and position averages of the resident wave packet, computed on the device in FP64:
 * out[0] = norm (scattering plus specular grid), out[1] = <Z>, out[2] = <r>, out[3] = the specular
 * norm between the analysis line iz_analysis (exclusive) and the analysis surface surface_index
 * (inclusive). z (nz), z_specular (nz_specular), r (nr): the grids; volume_scattering = dZ dr times
 * the xy volume element, volume_specular = dZ dr. Replaces compute_averages
 * (src/propagation/averages.hpp:29-30, averages.cpp:37-80) on the backend's block densities and
 * specular wave. */
int spo_averages(spo_handle* h, const double* z, const double* z_specular, const double* r, double volume_scattering,
                 double volume_specular, int iz_analysis, int surface_index, double* out);

/* ---------------------------------------------------------------------------------------------
 * The norm budget on the device, in FP64 whatever the precision form: per analysis window, the probability
 * each absorber removed (NormBudget, src/analysis/norm_budget.hpp:45-84). The absorbers and their cells come
 * from the handle's absorber factors (spo_desc z_optical, r_optical, z_specular_optical) as NormBudget's
 * constructor builds them (norm_budget.cpp:39-71): ZOpt, [ZOptLow], ROpt (scattering grid), ZSpOpt,
 * [ZSpOptLow], ROpt (specular grid), the bracketed ones only when their Z range is given.
 * --------------------------------------------------------------------------------------------- */
typedef struct spo_norm_budget_desc {
  int z_low_first, z_low_last;    /* SpatialGrids::z_optical_low (inclusive), or -1, -1 */
  int zs_low_first, zs_low_last;  /* SpatialGrids::z_specular_optical_low, or -1, -1 */
  double volume_scattering;       /* dZ dr times the (x, y) volume element (cell_probabilities, averages.cpp:85-97) */
  double volume_specular;         /* dZ dr */
} spo_norm_budget_desc;

/* Builds the budget's tables on the device; *n_absorbers receives their number (4 to 6). Replaces the
 * NormBudget constructor (norm_budget.cpp:39-50). */
int spo_norm_budget_setup(spo_handle* h, const spo_norm_budget_desc* d, int* n_absorbers);

/* The window that ends at the resident state and starts at the state of the previous call (NormBudget::add,
 * norm_budget.cpp:100-112): *has_window = 0 at the first call (nothing written); otherwise loss and loss_error
 * (n_absorbers values each, in the absorber order above) and norms[0], norms[1] (the probability on both grids
 * at the window's start and end). Cell sums in a fixed order on the device. */
int spo_norm_budget_add(spo_handle* h, double* loss, double* loss_error, double* norms, int* has_window);

/* ---------------------------------------------------------------------------------------------
 * Ensembles of wave packets (no counterpart in the reference, which propagates one wave packet per
 * run): one analysis step of every member handle, captured once as one CUDA graph with one branch per
 * member, so that one graph launch advances all of them and members of uneven grid sizes overlap on
 * the GPU. Members keep their own state, tables and precision and stay usable one by one (a member's
 * analysis, download, upload between ensemble steps); each ensemble step gives every member exactly
 * the state that spo_propagate_analysis_step on that member alone gives.
 *
 * All members must live on one device; they must outlive the ensemble. spo_ensemble_create switches
 * the members' kernel profiling off and returns them to their own streams.
 * --------------------------------------------------------------------------------------------- */
typedef struct spo_ensemble spo_ensemble;

int spo_ensemble_create(spo_handle* const* members, int n_members, spo_ensemble** out);

/* One analysis step of every member (one graph launch); returns when all are done. */
int spo_ensemble_step(spo_ensemble* e);

/* Kernel launches in one ensemble step (the sum over the members). */
int spo_ensemble_launch_count(const spo_ensemble* e, int* launches);

/* Message of the last failed call on e (of the last failed spo_ensemble_create when e is NULL). */
const char* spo_ensemble_last_error(const spo_ensemble* e);

int spo_ensemble_destroy(spo_ensemble* e);

/* ---------------------------------------------------------------------------------------------
 * Block densities without any device allocation.
 *
 * No counterpart in the reference: an addition for callers that cannot allocate device memory
 * themselves. A host program whose device memory is owned by a pool allocator (a framework's caching
 * allocator, an application arena sized at start-up) must not call cudaMalloc/cudaFree behind the
 * pool's back: a cudaMalloc can fail while the pool holds the free memory, and cudaFree synchronises
 * the whole device. spo_create allocates, so such callers keep the wave packet in their own buffers
 * and call this entry point on it.
 *
 * psi_device: n_blocks consecutive blocks of block_size complex values in device memory (complex128
 * when precision is SPO_PRECISION_FP64, complex64 when SPO_PRECISION_MIXED), i.e. the wave packet
 * in the layout of this library with block_size = n_rot*nx*ny and n_blocks = nz*nr. out_host: n_blocks
 * doubles in host memory, sum |psi|^2 of each block in FP64 with the fixed summation order of
 * spo_block_densities. cuda_stream: a cudaStream_t of the current device (NULL: the legacy default
 * stream); the call returns after the results are in out_host.
 *
 * Limit: n_blocks <= SPO_NOALLOC_MAX_BLOCKS (larger values are refused with SPO_ERR_INVALID). The
 * per-block sums go through a fixed scratch array of SPO_NOALLOC_MAX_BLOCKS doubles (512 KiB) that
 * every GPU which loads the library holds until the process exits. All calls share that array: calls
 * that overlap on the GPU (different streams or threads at the same time) race on it. Every element a
 * call reads is written by the same call first, so nothing needs clearing between calls. The first
 * call on a device looks up the array's device address for that device, with it current; only a
 * successful lookup is kept, so a lookup that failed (for example while memory was exhausted) is tried
 * again by the next call. The call synchronises the stream and copies into pageable host memory, so it
 * cannot run on a capturing stream: it refuses one with SPO_ERR_STATE. A CUDA error left pending by
 * earlier work on the calling thread is reported as such (SPO_ERR_DEVICE) and left pending.
 * Messages of refused calls: spo_last_error(NULL).
 * --------------------------------------------------------------------------------------------- */
#define SPO_NOALLOC_MAX_BLOCKS 65536
int spo_block_densities_noalloc(const void* psi_device, int precision, long long n_blocks, long long block_size,
                                double* out_host, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* SPO_B200_H */
