/*
 * jqoracle.c — OpenMP C restatement of how the reference executes a compiled
 * statevector plan on the CPU: one full pass over the state per plan entry
 * (jaqsi/simulation.py:400-409, _run), with the three entry kinds of
 * jaqsi/simulation.py:115-199:
 *   dense   k-qubit matrix on `wires` (_apply_gate, :70-112; k <= 2 here)
 *   gather  composed basis permutation, one 2^n index map (_apply_permutation, :150-152)
 *   diag    composed diagonal over its wires (_apply_diagonal, :155-161)
 * and the flat weighted-sum Z-string expectation (measure_state, :777-801).
 *
 * TEST / BASELINE INFRASTRUCTURE ONLY: used by tests/ and by bench.py's
 * CPU-baseline leg; never linked into or called by the product.
 * Built by oracle/Makefile into oracle/_build/libjqoracle.so.
 * Complex numbers are interleaved (re, im); the "f" variants use float.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define DEFINE_KERNELS(T, SFX)                                                                 \
  void jqo_dense##SFX(T* psi, int n, int k, const int* wires, const double* mat) {             \
    const int64_t dim = (int64_t)1 << n;                                                       \
    if (k == 1) {                                                                              \
      const int64_t b = (int64_t)1 << (n - 1 - wires[0]);                                     \
      const T m00r = (T)mat[0], m00i = (T)mat[1], m01r = (T)mat[2], m01i = (T)mat[3];          \
      const T m10r = (T)mat[4], m10i = (T)mat[5], m11r = (T)mat[6], m11i = (T)mat[7];          \
      _Pragma("omp parallel for schedule(static)")                                             \
      for (int64_t g = 0; g < dim / 2; ++g) {                                                  \
        const int64_t i0 = ((g / b) * 2 * b) + (g % b), i1 = i0 + b;                           \
        const T ar = psi[2 * i0], ai = psi[2 * i0 + 1], br = psi[2 * i1], bi = psi[2 * i1 + 1]; \
        psi[2 * i0] = m00r * ar - m00i * ai + m01r * br - m01i * bi;                           \
        psi[2 * i0 + 1] = m00r * ai + m00i * ar + m01r * bi + m01i * br;                       \
        psi[2 * i1] = m10r * ar - m10i * ai + m11r * br - m11i * bi;                           \
        psi[2 * i1 + 1] = m10r * ai + m10i * ar + m11r * bi + m11i * br;                       \
      }                                                                                        \
      return;                                                                                  \
    }                                                                                          \
    /* k == 2 */                                                                               \
    const int64_t b0 = (int64_t)1 << (n - 1 - wires[0]), b1 = (int64_t)1 << (n - 1 - wires[1]); \
    const int64_t lo = b0 < b1 ? b0 : b1, hi = b0 < b1 ? b1 : b0;                              \
    _Pragma("omp parallel for schedule(static)")                                               \
    for (int64_t g = 0; g < dim / 4; ++g) {                                                    \
      int64_t x = g;                                                                           \
      x = ((x / lo) * 2 * lo) + (x % lo);                                                      \
      x = ((x / hi) * 2 * hi) + (x % hi);                                                      \
      int64_t idx[4] = {x, x | b1, x | b0, x | b0 | b1};                                       \
      T vr[4], vi[4];                                                                          \
      for (int j = 0; j < 4; ++j) { vr[j] = psi[2 * idx[j]]; vi[j] = psi[2 * idx[j] + 1]; }    \
      for (int i = 0; i < 4; ++i) {                                                            \
        T sr = 0, si = 0;                                                                      \
        for (int j = 0; j < 4; ++j) {                                                          \
          const T mr = (T)mat[2 * (4 * i + j)], mi = (T)mat[2 * (4 * i + j) + 1];              \
          sr += mr * vr[j] - mi * vi[j];                                                       \
          si += mr * vi[j] + mi * vr[j];                                                       \
        }                                                                                      \
        psi[2 * idx[i]] = sr;                                                                  \
        psi[2 * idx[i] + 1] = si;                                                              \
      }                                                                                        \
    }                                                                                          \
  }                                                                                            \
  void jqo_gather##SFX(T* psi, T* tmp, int n, const int32_t* index) {                          \
    const int64_t dim = (int64_t)1 << n;                                                       \
    _Pragma("omp parallel for schedule(static)")                                               \
    for (int64_t i = 0; i < dim; ++i) {                                                        \
      tmp[2 * i] = psi[2 * (int64_t)index[i]];                                                 \
      tmp[2 * i + 1] = psi[2 * (int64_t)index[i] + 1];                                         \
    }                                                                                          \
    memcpy(psi, tmp, sizeof(T) * 2 * dim);                                                     \
  }                                                                                            \
  void jqo_diag##SFX(T* psi, int n, int k, const int* wires, const double* diag) {             \
    const int64_t dim = (int64_t)1 << n;                                                       \
    _Pragma("omp parallel for schedule(static)")                                               \
    for (int64_t i = 0; i < dim; ++i) {                                                        \
      int a = 0;                                                                               \
      for (int q = 0; q < k; ++q) a = (a << 1) | (int)((i >> (n - 1 - wires[q])) & 1);         \
      const T dr = (T)diag[2 * a], di = (T)diag[2 * a + 1];                                    \
      const T r = psi[2 * i], im = psi[2 * i + 1];                                             \
      psi[2 * i] = dr * r - di * im;                                                           \
      psi[2 * i + 1] = dr * im + di * r;                                                       \
    }                                                                                          \
  }                                                                                            \
  double jqo_expval_z##SFX(const T* psi, int n, uint64_t zmask) {                              \
    const int64_t dim = (int64_t)1 << n;                                                       \
    double acc = 0.0;                                                                          \
    _Pragma("omp parallel for reduction(+ : acc) schedule(static)")                            \
    for (int64_t i = 0; i < dim; ++i) {                                                        \
      const double p = (double)psi[2 * i] * psi[2 * i] + (double)psi[2 * i + 1] * psi[2 * i + 1]; \
      acc += (__builtin_popcountll((uint64_t)i & zmask) & 1) ? -p : p;                         \
    }                                                                                          \
    return acc;                                                                                \
  }                                                                                            \
  void jqo_init_zero##SFX(T* psi, int n) {                                                     \
    const int64_t dim = (int64_t)1 << n;                                                       \
    _Pragma("omp parallel for schedule(static)")                                               \
    for (int64_t i = 0; i < 2 * dim; ++i) psi[i] = 0;                                          \
    psi[0] = 1;                                                                                \
  }

DEFINE_KERNELS(double, )
DEFINE_KERNELS(float, f)

int jqo_max_threads(void) {
#ifdef _OPENMP
  extern int omp_get_max_threads(void);
  return omp_get_max_threads();
#else
  return 1;
#endif
}
