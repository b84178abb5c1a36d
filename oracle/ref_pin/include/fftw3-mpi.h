/* Stand-in for the FFTW 3 MPI interface the reference's py/fft.cpp calls.
 * TEST INFRASTRUCTURE: compiled only into oracle/_ref to pin the oracle.
 *
 * One rank owns the whole mesh.  Plans record their shape, direction and
 * layout; execution is a separable 3-D DFT evaluated in double and rounded
 * to float (oracle/ref_pin/stubs.cpp), unnormalised both ways as FFTW's.
 * The layouts are FFTW-MPI's: the real mesh is [n0][n1][2(n2/2+1)]; the
 * half spectrum is [n0][n1][n2/2+1], or [n1][n0][n2/2+1] with
 * FFTW_MPI_TRANSPOSED_OUT (forward) / FFTW_MPI_TRANSPOSED_IN (inverse).
 * The inverse transforms x and y first and keeps the real part along z, so
 * the imaginary parts of the kz = 0 and kz = n2/2 bins are ignored, as in
 * FFTW's rdft2.  A test harness may replace the execution with hooks
 * (fs2ref_set_fft_hooks) to capture or inject the arrays around a
 * transform. */
#ifndef FS2REF_FFTW3_MPI_H
#define FS2REF_FFTW3_MPI_H 1

#include <stddef.h>
#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef double fftw_complex[2];
typedef struct fs2ref_plan* fftwf_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MPI_TRANSPOSED_IN (1U << 29)
#define FFTW_MPI_TRANSPOSED_OUT (1U << 30)

ptrdiff_t fftwf_mpi_local_size_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                  MPI_Comm comm, ptrdiff_t* local_n0,
                                  ptrdiff_t* local_0_start);
ptrdiff_t fftwf_mpi_local_size_3d_transposed(
    ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm comm,
    ptrdiff_t* local_n0, ptrdiff_t* local_0_start, ptrdiff_t* local_n1,
    ptrdiff_t* local_1_start);
fftwf_plan fftwf_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                     float* in, fftwf_complex* out,
                                     MPI_Comm comm, unsigned flags);
fftwf_plan fftwf_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2,
                                     fftwf_complex* in, float* out,
                                     MPI_Comm comm, unsigned flags);
void fftwf_mpi_execute_dft_r2c(fftwf_plan p, float* in, fftwf_complex* out);
void fftwf_mpi_execute_dft_c2r(fftwf_plan p, fftwf_complex* in, float* out);
void fftwf_destroy_plan(fftwf_plan p);
void fftwf_mpi_init(void);
void fftwf_mpi_cleanup(void);
void* fftwf_malloc(size_t n);
void fftwf_free(void* p);

#ifdef __cplusplus
}
#endif

#endif
