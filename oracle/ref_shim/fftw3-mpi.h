// Stand-in for the FFTW 3.3 MPI interface that the reference's periodic
// Poisson solver calls (test infrastructure of the oracle only; FFTW itself
// is not in the reference snapshot). One process: the "MPI" layout is the
// whole grid. Plans carry out FFTW's unnormalised DFTs (forward e^{-2 pi i kn/N})
// of the 3-D real <-> half-complex transform with the transposed layout the
// solver asks for (FFTW_MPI_TRANSPOSED_OUT / _IN: spectrum [n1][n0][n2/2+1]),
// by direct summation with long double twiddles; sizes are the small ones
// the parity tests use.
#pragma once
#include <cstddef>
#include <cstdlib>
#include <mpi.h>

typedef double fftw_complex[2];
struct fftw_plan_s;
typedef fftw_plan_s* fftw_plan;
#define FFTW_MEASURE 0U
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MPI_TRANSPOSED_OUT (1U << 29)
#define FFTW_MPI_TRANSPOSED_IN (1U << 30)
#define MPI_THREAD_FUNNELED 1
inline int MPI_Query_thread(int* p) { *p = 3; return 0; }

int fftw_init_threads(void);
void fftw_plan_with_nthreads(int);
void fftw_mpi_init(void);
void fftw_cleanup_threads(void);
void fftw_mpi_cleanup(void);
ptrdiff_t fftw_mpi_local_size_3d_transposed(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm, ptrdiff_t* local_n0,
                                            ptrdiff_t* local_0_start, ptrdiff_t* local_n1, ptrdiff_t* local_1_start);
double* fftw_alloc_real(size_t n);
fftw_complex* fftw_alloc_complex(size_t n);
void fftw_free(void* p);
fftw_plan fftw_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double* in, fftw_complex* out, MPI_Comm,
                                   unsigned flags);
fftw_plan fftw_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex* in, double* out, MPI_Comm,
                                   unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
