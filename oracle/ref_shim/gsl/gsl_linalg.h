// Stand-in for the GSL LU routines of Obstacle::computeVelocities (oracle test
// infrastructure; GSL is absent here): LU decomposition with partial pivoting
// (Doolittle, row exchanges recorded in the permutation) and the matching
// forward / back substitution, for the small dense systems that path solves.
#pragma once
#include <cmath>
#include <cstddef>
#include <vector>

struct gsl_matrix { size_t size1, size2, tda; double* data; };
struct gsl_vector { size_t size, stride; double* data; std::vector<double> own; };
struct gsl_matrix_view { gsl_matrix matrix; };
struct gsl_vector_view { gsl_vector vector; };
struct gsl_permutation { size_t size; std::vector<size_t> data; };

inline gsl_matrix_view gsl_matrix_view_array(double* base, size_t n1, size_t n2) {
  return gsl_matrix_view{gsl_matrix{n1, n2, n2, base}};
}
inline gsl_vector_view gsl_vector_view_array(double* base, size_t n) {
  gsl_vector_view v;
  v.vector.size = n, v.vector.stride = 1, v.vector.data = base;
  return v;
}
inline gsl_vector* gsl_vector_alloc(size_t n) {
  gsl_vector* v = new gsl_vector();
  v->size = n, v->stride = 1, v->own.assign(n, 0.0), v->data = v->own.data();
  return v;
}
inline void gsl_vector_free(gsl_vector* v) { delete v; }
inline double gsl_vector_get(const gsl_vector* v, size_t i) { return v->data[i * v->stride]; }
inline gsl_permutation* gsl_permutation_alloc(size_t n) {
  gsl_permutation* p = new gsl_permutation();
  p->size = n, p->data.resize(n);
  for (size_t i = 0; i < n; ++i) p->data[i] = i;
  return p;
}
inline void gsl_permutation_free(gsl_permutation* p) { delete p; }

inline int gsl_linalg_LU_decomp(gsl_matrix* A, gsl_permutation* p, int* signum) {
  const size_t n = A->size1;
  auto a = [&](size_t i, size_t j) -> double& { return A->data[i * A->tda + j]; };
  for (size_t i = 0; i < n; ++i) p->data[i] = i;
  *signum = 1;
  for (size_t j = 0; j + 1 < n; ++j) {
    size_t piv = j;
    double mx = std::fabs(a(j, j));
    for (size_t i = j + 1; i < n; ++i)
      if (std::fabs(a(i, j)) > mx) mx = std::fabs(a(i, j)), piv = i;
    if (piv != j) {
      for (size_t k = 0; k < n; ++k) std::swap(a(j, k), a(piv, k));
      std::swap(p->data[j], p->data[piv]);
      *signum = -*signum;
    }
    const double d = a(j, j);
    if (d == 0) continue;
    for (size_t i = j + 1; i < n; ++i) {
      const double l = a(i, j) / d;
      a(i, j) = l;
      for (size_t k = j + 1; k < n; ++k) a(i, k) -= l * a(j, k);
    }
  }
  return 0;
}

inline int gsl_linalg_LU_solve(const gsl_matrix* LU, const gsl_permutation* p, const gsl_vector* b, gsl_vector* x) {
  const size_t n = LU->size1;
  auto a = [&](size_t i, size_t j) { return LU->data[i * LU->tda + j]; };
  std::vector<double> y(n);
  for (size_t i = 0; i < n; ++i) y[i] = b->data[p->data[i] * b->stride];
  for (size_t i = 0; i < n; ++i)
    for (size_t k = 0; k < i; ++k) y[i] -= a(i, k) * y[k];
  for (size_t i = n; i-- > 0;) {
    for (size_t k = i + 1; k < n; ++k) y[i] -= a(i, k) * y[k];
    y[i] /= a(i, i);
  }
  for (size_t i = 0; i < n; ++i) x->data[i * x->stride] = y[i];
  return 0;
}
