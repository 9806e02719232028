// The FFTW stand-in of ref_shim/fftw3-mpi.h: 3-D real <-> half-complex DFTs by
// direct summation (long double twiddles, double accumulation), in FFTW's
// in-place padded layout: real data [n0][n1][2 (n2/2 + 1)], spectrum
// transposed [n1][n0][n2/2 + 1]. Test infrastructure of the oracle only.
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "fftw3-mpi.h"

struct fftw_plan_s {
  ptrdiff_t n0, n1, n2;
  bool r2c;
  double* real;
  fftw_complex* cplx;
};

int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int) {}
void fftw_mpi_init(void) {}
void fftw_cleanup_threads(void) {}
void fftw_mpi_cleanup(void) {}
ptrdiff_t fftw_mpi_local_size_3d_transposed(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, MPI_Comm, ptrdiff_t* local_n0,
                                            ptrdiff_t* local_0_start, ptrdiff_t* local_n1, ptrdiff_t* local_1_start) {
  *local_n0 = n0, *local_0_start = 0, *local_n1 = n1, *local_1_start = 0;
  return n0 * n1 * n2;
}
double* fftw_alloc_real(size_t n) { return static_cast<double*>(std::calloc(n, sizeof(double))); }
fftw_complex* fftw_alloc_complex(size_t n) { return static_cast<fftw_complex*>(std::calloc(n, sizeof(fftw_complex))); }
void fftw_free(void* p) { std::free(p); }
fftw_plan fftw_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double* in, fftw_complex* out, MPI_Comm,
                                   unsigned) {
  return new fftw_plan_s{n0, n1, n2, true, in, out};
}
fftw_plan fftw_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex* in, double* out, MPI_Comm,
                                   unsigned) {
  return new fftw_plan_s{n0, n1, n2, false, out, in};
}
void fftw_destroy_plan(fftw_plan p) { delete p; }

namespace {
using cd = std::complex<double>;
// y[k] = sum_n x[n] e^{sign 2 pi i k n / N}
void dft(const cd* x, cd* y, ptrdiff_t N, ptrdiff_t stride, int sign) {
  std::vector<cd> tw(N);
  for (ptrdiff_t k = 0; k < N; ++k) {
    const long double a = sign * 2.0L * 3.141592653589793238462643383279502884L * k / N;
    tw[k] = cd((double)cosl(a), (double)sinl(a));
  }
  for (ptrdiff_t k = 0; k < N; ++k) {
    cd s = 0;
    for (ptrdiff_t n = 0; n < N; ++n) s += x[n * stride] * tw[(k * n) % N];
    y[k] = s;
  }
}
}  // namespace

void fftw_execute(const fftw_plan p) {
  const ptrdiff_t n0 = p->n0, n1 = p->n1, n2 = p->n2, nh = n2 / 2 + 1, pad = 2 * nh;
  std::vector<cd> A((size_t)n0 * n1 * nh);  // [i0][i1][k2]
  std::vector<cd> line(std::max(n0, std::max(n1, n2))), out(line.size());
  auto at = [&](ptrdiff_t a, ptrdiff_t b, ptrdiff_t c) -> cd& { return A[((size_t)a * n1 + b) * nh + c]; };
  if (p->r2c) {
    for (ptrdiff_t a = 0; a < n0; ++a)
      for (ptrdiff_t b = 0; b < n1; ++b) {
        for (ptrdiff_t c = 0; c < n2; ++c) line[c] = p->real[((size_t)a * n1 + b) * pad + c];
        dft(line.data(), out.data(), n2, 1, -1);
        for (ptrdiff_t c = 0; c < nh; ++c) at(a, b, c) = out[c];
      }
    for (ptrdiff_t a = 0; a < n0; ++a)
      for (ptrdiff_t c = 0; c < nh; ++c) {
        for (ptrdiff_t b = 0; b < n1; ++b) line[b] = at(a, b, c);
        dft(line.data(), out.data(), n1, 1, -1);
        for (ptrdiff_t b = 0; b < n1; ++b) at(a, b, c) = out[b];
      }
    for (ptrdiff_t b = 0; b < n1; ++b)
      for (ptrdiff_t c = 0; c < nh; ++c) {
        for (ptrdiff_t a = 0; a < n0; ++a) line[a] = at(a, b, c);
        dft(line.data(), out.data(), n0, 1, -1);
        for (ptrdiff_t a = 0; a < n0; ++a) at(a, b, c) = out[a];
      }
    // transposed output [i1][i0][k2]
    for (ptrdiff_t b = 0; b < n1; ++b)
      for (ptrdiff_t a = 0; a < n0; ++a)
        for (ptrdiff_t c = 0; c < nh; ++c) {
          const cd v = at(a, b, c);
          p->cplx[((size_t)b * n0 + a) * nh + c][0] = v.real();
          p->cplx[((size_t)b * n0 + a) * nh + c][1] = v.imag();
        }
  } else {
    for (ptrdiff_t b = 0; b < n1; ++b)
      for (ptrdiff_t a = 0; a < n0; ++a)
        for (ptrdiff_t c = 0; c < nh; ++c) {
          const fftw_complex& v = p->cplx[((size_t)b * n0 + a) * nh + c];
          at(a, b, c) = cd(v[0], v[1]);
        }
    for (ptrdiff_t b = 0; b < n1; ++b)
      for (ptrdiff_t c = 0; c < nh; ++c) {
        for (ptrdiff_t a = 0; a < n0; ++a) line[a] = at(a, b, c);
        dft(line.data(), out.data(), n0, 1, +1);
        for (ptrdiff_t a = 0; a < n0; ++a) at(a, b, c) = out[a];
      }
    for (ptrdiff_t a = 0; a < n0; ++a)
      for (ptrdiff_t c = 0; c < nh; ++c) {
        for (ptrdiff_t b = 0; b < n1; ++b) line[b] = at(a, b, c);
        dft(line.data(), out.data(), n1, 1, +1);
        for (ptrdiff_t b = 0; b < n1; ++b) at(a, b, c) = out[b];
      }
    // half-complex -> real along the last axis (Hermitian completion)
    for (ptrdiff_t a = 0; a < n0; ++a)
      for (ptrdiff_t b = 0; b < n1; ++b) {
        for (ptrdiff_t c = 0; c < nh; ++c) line[c] = at(a, b, c);
        for (ptrdiff_t c = nh; c < n2; ++c) line[c] = std::conj(line[n2 - c]);
        dft(line.data(), out.data(), n2, 1, +1);
        for (ptrdiff_t c = 0; c < n2; ++c) p->real[((size_t)a * n1 + b) * pad + c] = out[c].real();
      }
  }
}
