// Test infrastructure (oracle build only): the LAPACK symbol the reference's eigensolver calls.
//
// src/linalg/lapack_eigensolver.cpp:9-11 declares dsyevd_ (Fortran LAPACK, 32-bit integers). No
// system LAPACK exists here; SciPy's bundled OpenBLAS exports the same routine under the prefixed
// name scipy_dsyevd_ with the same LP64 interface, so this forwards to it. The reference only uses
// it for the gas-phase Fourier-grid Hamiltonian, whose eigenvector signs it fixes itself
// (src/gasphase/fourier_grid_hamiltonian.cpp:47-55), so the LAPACK build does not change results.
#include <cstddef>

extern "C" void scipy_dsyevd_(const char* jobz, const char* uplo, const int* n, double* a, const int* lda, double* w,
                              double* work, const int* lwork, int* iwork, const int* liwork, int* info,
                              std::size_t jobz_len, std::size_t uplo_len);

extern "C" void dsyevd_(const char* jobz, const char* uplo, const int* n, double* a, const int* lda, double* w,
                        double* work, const int* lwork, int* iwork, const int* liwork, int* info, std::size_t jobz_len,
                        std::size_t uplo_len) {
  scipy_dsyevd_(jobz, uplo, n, a, lda, w, work, lwork, iwork, liwork, info, jobz_len, uplo_len);
}
