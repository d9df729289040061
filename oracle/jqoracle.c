/*
 * jqoracle.c — OpenMP C restatement of how the reference executes a compiled
 * statevector plan on the CPU: one full pass over the state per plan entry
 * (jaqsi/simulation.py:400-409, _run), with the three entry kinds of
 * jaqsi/simulation.py:115-199:
 *   dense   k-qubit matrix on `wires` (_apply_gate, :70-112; k <= 4 here)
 *   gather  composed basis permutation, one 2^n index map (_apply_permutation, :150-152)
 *   diag    composed diagonal over its wires (_apply_diagonal, :155-161)
 * and the flat weighted-sum Z-string expectation (measure_state, :777-801).
 * A density matrix runs through the same runner as a 2n-wire vector with the
 * fused superoperators of _compile_mixed (:348-381), 4 x 4 and 16 x 16.
 * jqo_compose_perm builds the gather map of a permutation run the way
 * _compose_permutation does (:243-267), one block at a time.
 *
 * TEST / BASELINE INFRASTRUCTURE ONLY: used by tests/ and by bench.py's
 * CPU-baseline leg; never linked into or called by the product.
 * Built by oracle/Makefile into oracle/_build/libjqoracle.so.
 * Complex numbers are interleaved (re, im); the "f" variants use float.
 *
 * Pair indices are formed by inserting zero bits (shift and mask), so a pass
 * costs memory traffic, not integer division.  A gather writes into a second
 * buffer and the two buffers swap roles (as XLA's `take` yields a new array),
 * so no pass copies the state back.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* g with a zero bit inserted at position s */
static inline int64_t ins0(int64_t g, int s) { return ((g >> s) << (s + 1)) | (g & (((int64_t)1 << s) - 1)); }

enum { JQO_DENSE = 0, JQO_GATHER = 1, JQO_DIAG = 2 };
#define JQO_MAXW 32 /* wires of one plan entry (a composed diagonal spans up to n) */

#define JQO_MAXK 4 /* widest dense block: the 16 x 16 superoperator of a two-qubit gate */

#define DEFINE_KERNELS(T, SFX)                                                                 \
  /* dense k-wire block, 2 < k <= JQO_MAXK (the einsum branch of _apply_gate, :92-94) */     \
  static void jqo_dense_wide##SFX(T* psi, int n, int k, const int* wires, const double* mat) { \
    const int64_t dim = (int64_t)1 << n;                                                       \
    const int m = 1 << k;                                                                      \
    int sorted[JQO_MAXK];                                                                      \
    int64_t off[1 << JQO_MAXK];                                                                \
    for (int q = 0; q < k; ++q) sorted[q] = n - 1 - wires[q];                                  \
    for (int a = 0; a < k; ++a)                                                                \
      for (int b = a + 1; b < k; ++b)                                                          \
        if (sorted[b] < sorted[a]) { int t = sorted[a]; sorted[a] = sorted[b]; sorted[b] = t; } \
    for (int j = 0; j < m; ++j) {                                                              \
      int64_t o = 0;                                                                           \
      for (int q = 0; q < k; ++q)                                                              \
        if ((j >> (k - 1 - q)) & 1) o |= (int64_t)1 << (n - 1 - wires[q]);                     \
      off[j] = o;                                                                              \
    }                                                                                          \
    _Pragma("omp parallel for schedule(static)")                                               \
    for (int64_t g = 0; g < (dim >> k); ++g) {                                                 \
      int64_t x = g;                                                                           \
      for (int q = 0; q < k; ++q) x = ins0(x, sorted[q]);                                      \
      T vr[1 << JQO_MAXK], vi[1 << JQO_MAXK];                                                  \
      for (int j = 0; j < m; ++j) { vr[j] = psi[2 * (x | off[j])]; vi[j] = psi[2 * (x | off[j]) + 1]; } \
      for (int i = 0; i < m; ++i) {                                                            \
        T sr = 0, si = 0;                                                                      \
        for (int j = 0; j < m; ++j) {                                                          \
          const T ar = (T)mat[2 * (m * i + j)], ai = (T)mat[2 * (m * i + j) + 1];              \
          sr += ar * vr[j] - ai * vi[j];                                                       \
          si += ar * vi[j] + ai * vr[j];                                                       \
        }                                                                                      \
        psi[2 * (x | off[i])] = sr;                                                            \
        psi[2 * (x | off[i]) + 1] = si;                                                        \
      }                                                                                        \
    }                                                                                          \
  }                                                                                            \
  void jqo_dense##SFX(T* psi, int n, int k, const int* wires, const double* mat) {             \
    const int64_t dim = (int64_t)1 << n;                                                       \
    if (k == 1) {                                                                              \
      const int s = n - 1 - wires[0];                                                          \
      const int64_t b = (int64_t)1 << s;                                                       \
      const T m00r = (T)mat[0], m00i = (T)mat[1], m01r = (T)mat[2], m01i = (T)mat[3];          \
      const T m10r = (T)mat[4], m10i = (T)mat[5], m11r = (T)mat[6], m11i = (T)mat[7];          \
      _Pragma("omp parallel for schedule(static)")                                             \
      for (int64_t g = 0; g < dim / 2; ++g) {                                                  \
        const int64_t i0 = ins0(g, s), i1 = i0 | b;                                            \
        const T ar = psi[2 * i0], ai = psi[2 * i0 + 1], br = psi[2 * i1], bi = psi[2 * i1 + 1]; \
        psi[2 * i0] = m00r * ar - m00i * ai + m01r * br - m01i * bi;                           \
        psi[2 * i0 + 1] = m00r * ai + m00i * ar + m01r * bi + m01i * br;                       \
        psi[2 * i1] = m10r * ar - m10i * ai + m11r * br - m11i * bi;                           \
        psi[2 * i1 + 1] = m10r * ai + m10i * ar + m11r * bi + m11i * br;                       \
      }                                                                                        \
      return;                                                                                  \
    }                                                                                          \
    if (k > 2) {                                                                               \
      jqo_dense_wide##SFX(psi, n, k, wires, mat);                                              \
      return;                                                                                  \
    }                                                                                          \
    /* k == 2: wires[0] is the most significant bit of the matrix index */                    \
    const int s0 = n - 1 - wires[0], s1 = n - 1 - wires[1];                                    \
    const int64_t b0 = (int64_t)1 << s0, b1 = (int64_t)1 << s1;                                \
    const int slo = s0 < s1 ? s0 : s1, shi = s0 < s1 ? s1 : s0;                                \
    T mr[16], mi[16];                                                                          \
    for (int e = 0; e < 16; ++e) { mr[e] = (T)mat[2 * e]; mi[e] = (T)mat[2 * e + 1]; }         \
    _Pragma("omp parallel for schedule(static)")                                               \
    for (int64_t g = 0; g < dim / 4; ++g) {                                                    \
      const int64_t x = ins0(ins0(g, slo), shi);                                               \
      const int64_t idx[4] = {x, x | b1, x | b0, x | b0 | b1};                                 \
      T vr[4], vi[4];                                                                          \
      for (int j = 0; j < 4; ++j) { vr[j] = psi[2 * idx[j]]; vi[j] = psi[2 * idx[j] + 1]; }    \
      for (int i = 0; i < 4; ++i) {                                                            \
        T sr = 0, si = 0;                                                                      \
        for (int j = 0; j < 4; ++j) {                                                          \
          sr += mr[4 * i + j] * vr[j] - mi[4 * i + j] * vi[j];                                 \
          si += mr[4 * i + j] * vi[j] + mi[4 * i + j] * vr[j];                                 \
        }                                                                                      \
        psi[2 * idx[i]] = sr;                                                                  \
        psi[2 * idx[i] + 1] = si;                                                              \
      }                                                                                        \
    }                                                                                          \
  }                                                                                            \
  /* out[i] = in[index[i]] (a new array, as jnp.take returns one) */                          \
  void jqo_gather_to##SFX(const T* in, T* out, int n, const int32_t* index) {                  \
    const int64_t dim = (int64_t)1 << n;                                                       \
    _Pragma("omp parallel for schedule(static)")                                               \
    for (int64_t i = 0; i < dim; ++i) {                                                        \
      const int64_t j = index[i];                                                              \
      out[2 * i] = in[2 * j];                                                                  \
      out[2 * i + 1] = in[2 * j + 1];                                                          \
    }                                                                                          \
  }                                                                                            \
  /* in-place form kept for callers that hold one buffer */                                   \
  void jqo_gather##SFX(T* psi, T* tmp, int n, const int32_t* index) {                          \
    jqo_gather_to##SFX(psi, tmp, n, index);                                                    \
    memcpy(psi, tmp, sizeof(T) * 2 * ((size_t)1 << n));                                       \
  }                                                                                            \
  void jqo_diag##SFX(T* psi, int n, int k, const int* wires, const double* diag) {             \
    const int64_t dim = (int64_t)1 << n;                                                       \
    int sh[JQO_MAXW];                                                                          \
    for (int q = 0; q < k; ++q) sh[q] = n - 1 - wires[q];                                      \
    _Pragma("omp parallel for schedule(static)")                                               \
    for (int64_t i = 0; i < dim; ++i) {                                                        \
      int a = 0;                                                                               \
      for (int q = 0; q < k; ++q) a = (a << 1) | (int)((i >> sh[q]) & 1);                      \
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
  /* sum_j rho[j, j] (-1)^popcount(j & zmask) of a row-major dim x dim density               \
   * (measure_density's diagonal, simulation.py:814-857) */                                   \
  double jqo_expval_z_dm##SFX(const T* rho, int n, uint64_t zmask) {                           \
    const int64_t dim = (int64_t)1 << n;                                                       \
    double acc = 0.0;                                                                          \
    _Pragma("omp parallel for reduction(+ : acc) schedule(static)")                            \
    for (int64_t j = 0; j < dim; ++j) {                                                        \
      const double p = (double)rho[2 * (j * dim + j)];                                         \
      acc += (__builtin_popcountll((uint64_t)j & zmask) & 1) ? -p : p;                         \
    }                                                                                          \
    return acc;                                                                                \
  }                                                                                            \
  void jqo_init_zero##SFX(T* psi, int n) {                                                     \
    const int64_t dim = (int64_t)1 << n;                                                       \
    _Pragma("omp parallel for schedule(static)")                                               \
    for (int64_t i = 0; i < 2 * dim; ++i) psi[i] = 0;                                          \
    psi[0] = 1;                                                                                \
  }                                                                                            \
  /* Run a whole plan (_run, simulation.py:400-409): entry e has kind[e],               \
   * nw[e] wires in wires[32e..], its matrix / diagonal at data[e] (complex128,          \
   * interleaved) or its gather map at index[e].  The result ends in bufs[r] for        \
   * the returned r (0 or 1); bufs[0] holds the initial state. */                       \
  int jqo_run_plan##SFX(T* buf0, T* buf1, int n, int n_entries, const int* kind, const int* nw,      \
                        const int* wires, const double* const* data, const int32_t* const* index) {  \
    T* cur = buf0;                                                                             \
    T* oth = buf1;                                                                             \
    for (int e = 0; e < n_entries; ++e) {                                                      \
      if (kind[e] == JQO_DENSE) {                                                              \
        jqo_dense##SFX(cur, n, nw[e], wires + JQO_MAXW * e, data[e]);                                 \
      } else if (kind[e] == JQO_GATHER) {                                                      \
        jqo_gather_to##SFX(cur, oth, n, index[e]);                                             \
        T* t = cur;                                                                            \
        cur = oth;                                                                             \
        oth = t;                                                                               \
      } else {                                                                                 \
        jqo_diag##SFX(cur, n, nw[e], wires + JQO_MAXW * e, data[e]);                                  \
      }                                                                                        \
    }                                                                                          \
    return cur == buf0 ? 0 : 1;                                                                \
  }

DEFINE_KERNELS(double, )
DEFINE_KERNELS(float, f)

/* One permutation block of a run folded into a gather map
 * (_compose_permutation, simulation.py:243-267): with src(o) the input index
 * that the block sends to output o (o's bits on the block's wires replaced by
 * perm[col(o)]), index_out[o] = index_in[src(o)].  bits[i] is the flat-index
 * bit of the block's i-th wire (first wire = most significant matrix bit). */
void jqo_compose_perm(int n, int k, const int* bits, const int32_t* perm, const int32_t* index_in,
                      int32_t* index_out) {
  const int64_t dim = (int64_t)1 << n;
  int64_t mask = 0;
  for (int i = 0; i < k; ++i) mask |= (int64_t)1 << bits[i];
#pragma omp parallel for schedule(static)
  for (int64_t o = 0; o < dim; ++o) {
    int col = 0;
    for (int i = 0; i < k; ++i) col |= (int)((o >> bits[i]) & 1) << (k - 1 - i);
    const int sc = perm[col];
    int64_t src = o & ~mask;
    for (int i = 0; i < k; ++i) src |= (int64_t)((sc >> (k - 1 - i)) & 1) << bits[i];
    index_out[o] = index_in[src];
  }
}

int jqo_max_threads(void) {
#ifdef _OPENMP
  extern int omp_get_max_threads(void);
  return omp_get_max_threads();
#else
  return 1;
#endif
}
