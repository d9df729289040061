// Pulse-gate unitaries on the GPU: ordered products of matrix exponentials.
//
// jaqsi solves time-dependent gates  dU/dt = -i [sum_i f_i(p_i, t) H_i] U
// lazily and in batches (jaqsi/evolution.py:692-773, resolve_pending; called
// from jaqsi/simulation.py:713).  Its commutator-free Magnus integrators
// (evolution.py:195-264) make every step one or two exponentials of
//   Omega = sum_i w_i A_i,   A_i = -i H_i,
// with complex weights w_i (step size x coefficient values at the quadrature
// nodes x the scheme's node weights).  The host side forms the weights; this
// file computes, for a batch of gates,
//   U = expm(Omega_{M-1}) ... expm(Omega_1) expm(Omega_0)
// and the reverse pass d L / d w from d L / d U (PyTorch's convention for
// complex gradients, d/dRe + i d/dIm).
//
// One CTA per gate.  Thread t owns a contiguous chunk of sub-steps and forms
// its chunk's product in registers; the chunk products are combined by an
// ordered tree product in shared memory.  The matrix exponential is the
// Taylor series on a scaled matrix followed by repeated squaring (Moler and
// Van Loan, "Nineteen dubious ways to compute the exponential of a matrix",
// 2003, method 3): Omega is scaled by 2^-s so that its 1-norm is at most 1/2,
// the series is summed to degree 18 (truncation below 1e-20 relative), and the
// result is squared s times.
//
// The reverse pass uses, for each sub-step m,
//   G_E(m) = L_m^H G_U R_m^H     (L_m, R_m: the products after / before m)
// and the adjoint of the Frechet derivative of expm at Omega applied to G_E,
// read from the upper-right block of expm([[Omega^H, G_E], [0, Omega^H]])
// (Najfeld and Havel 1995; the same rule as torch.linalg.matrix_exp's
// backward), then d L / d w_i = sum_jk conj(A_i[j, k]) G_Omega[j, k].
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "../../include/jqsim.h"

namespace jq {
void set_error(const std::string& msg);
}

namespace {

struct cplx {
  double x, y;
};
__device__ __forceinline__ cplx cfma(cplx a, cplx b, cplx c) {
  return {fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y))};
}
__device__ __forceinline__ cplx cconj(cplx a) { return {a.x, -a.y}; }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return {a.x * s, a.y * s}; }

// Row-major D x D complex matrices in local arrays.
template <int D>
__device__ __forceinline__ void mat_eye(cplx* m) {
#pragma unroll
  for (int i = 0; i < D * D; ++i) m[i] = {(i % (D + 1)) == 0 ? 1.0 : 0.0, 0.0};
}
template <int D>
__device__ __forceinline__ void mat_copy(cplx* d, const cplx* s) {
#pragma unroll
  for (int i = 0; i < D * D; ++i) d[i] = s[i];
}
// c = a b (c must not alias a or b)
template <int D>
__device__ __forceinline__ void mat_mul(cplx* c, const cplx* a, const cplx* b) {
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      cplx s = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < D; ++k) s = cfma(a[i * D + k], b[k * D + j], s);
      c[i * D + j] = s;
    }
}
// c = a^H b
template <int D>
__device__ __forceinline__ void mat_mul_hn(cplx* c, const cplx* a, const cplx* b) {
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      cplx s = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < D; ++k) s = cfma(cconj(a[k * D + i]), b[k * D + j], s);
      c[i * D + j] = s;
    }
}
// c = a b^H
template <int D>
__device__ __forceinline__ void mat_mul_nh(cplx* c, const cplx* a, const cplx* b) {
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      cplx s = {0.0, 0.0};
#pragma unroll
      for (int k = 0; k < D; ++k) s = cfma(a[i * D + k], cconj(b[j * D + k]), s);
      c[i * D + j] = s;
    }
}
template <int D>
__device__ __forceinline__ double norm1(const cplx* m) {
  double best = 0.0;
#pragma unroll
  for (int j = 0; j < D; ++j) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < D; ++i) s += hypot(m[i * D + j].x, m[i * D + j].y);
    best = fmax(best, s);
  }
  return best;
}

// e = expm(a): scaling by 2^-s (|a|_1 2^-s <= 1/2), Taylor series to degree
// 18 by Horner's rule, s squarings.  `t` is scratch of D * D.
template <int D>
__device__ void mat_expm(cplx* e, const cplx* a, cplx* t) {
  const double nrm = norm1<D>(a);
  int s = 0;
  if (nrm > 0.5) s = static_cast<int>(ceil(log2(nrm / 0.5)));
  const double scale = ldexp(1.0, -s);
  // Horner: e = I + x (I + x/2 (I + x/3 (... (I + x/18))))
  constexpr int kDeg = 18;
  mat_eye<D>(e);
  for (int k = kDeg; k >= 1; --k) {
    // t = (scale / k) a e ; e = I + t
    mat_mul<D>(t, a, e);
    const double f = scale / k;
#pragma unroll
    for (int i = 0; i < D * D; ++i) e[i] = cscale(t[i], f);
#pragma unroll
    for (int i = 0; i < D; ++i) e[i * D + i].x += 1.0;
  }
  for (int q = 0; q < s; ++q) {
    mat_mul<D>(t, e, e);
    mat_copy<D>(e, t);
  }
}

}  // namespace

namespace {

constexpr int kMaxChunk = 16;  // sub-steps per thread

template <int D>
constexpr int threads_for() {
  return D <= 4 ? 128 : 32;
}

// Omega_m = sum_i w[m, i] A_i (A cached in shared memory)
template <int D>
__device__ __forceinline__ void form_omega(cplx* om, const cplx* sA, const cplx* w, int nt) {
#pragma unroll
  for (int e = 0; e < D * D; ++e) om[e] = {0.0, 0.0};
  for (int i = 0; i < nt; ++i) {
    const cplx wi = w[i];
#pragma unroll
    for (int e = 0; e < D * D; ++e) om[e] = cfma(wi, sA[i * D * D + e], om[e]);
  }
}

// Ordered product of the per-thread chunk products in `buf` (thread t's
// product is buf[t]; later chunks multiply from the left); the total lands in buf[0].
template <int D>
__device__ void tree_product(cplx* buf, int T) {
  cplx tmp[D * D];
  for (int s = 1; s < T; s *= 2) {
    __syncthreads();
    const int t = threadIdx.x;
    if (t % (2 * s) == 0 && t + s < T) {
      mat_mul<D>(tmp, buf + (t + s) * D * D, buf + t * D * D);
      mat_copy<D>(buf + t * D * D, tmp);
    }
  }
  __syncthreads();
}

template <int D>
__global__ void __launch_bounds__(threads_for<D>()) k_magnus(int M, int nt, const cplx* __restrict__ A,
                                                              int64_t a_stride, const cplx* __restrict__ w,
                                                              cplx* __restrict__ U) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* sA = reinterpret_cast<cplx*>(smem_raw);
  cplx* buf = sA + nt * D * D;
  const int g = blockIdx.x, T = blockDim.x, t = threadIdx.x;
  const cplx* Ag = A + g * a_stride;
  for (int e = t; e < nt * D * D; e += T) sA[e] = Ag[e];
  __syncthreads();
  const int chunk = (M + T - 1) / T;
  const int m0 = min(M, t * chunk), m1 = min(M, m0 + chunk);
  cplx P[D * D], om[D * D], E[D * D], tmp[D * D];
  mat_eye<D>(P);
  for (int m = m0; m < m1; ++m) {
    form_omega<D>(om, sA, w + (static_cast<int64_t>(g) * M + m) * nt, nt);
    mat_expm<D>(E, om, tmp);
    mat_mul<D>(tmp, E, P);
    mat_copy<D>(P, tmp);
  }
  mat_copy<D>(buf + t * D * D, P);
  tree_product<D>(buf, T);
  for (int e = t; e < D * D; e += T) U[static_cast<int64_t>(g) * D * D + e] = buf[e];
}

// Reverse pass: gw[g, m, i] = d L / d w[g, m, i] from gU = d L / d U[g].
template <int D>
__global__ void __launch_bounds__(threads_for<D>()) k_magnus_grad(int M, int nt, const cplx* __restrict__ A,
                                                                   int64_t a_stride, const cplx* __restrict__ w,
                                                                   const cplx* __restrict__ gU,
                                                                   cplx* __restrict__ gw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx* sA = reinterpret_cast<cplx*>(smem_raw);
  const int T = blockDim.x, t = threadIdx.x, g = blockIdx.x;
  cplx* buf = sA + nt * D * D;    // chunk products
  cplx* pre = buf + T * D * D;    // product of the chunks before t
  cplx* suf = pre + T * D * D;    // product of the chunks after t
  const cplx* Ag = A + g * a_stride;
  for (int e = t; e < nt * D * D; e += T) sA[e] = Ag[e];
  __syncthreads();
  const int chunk = (M + T - 1) / T;
  const int m0 = min(M, t * chunk), m1 = min(M, m0 + chunk);
  const int L = m1 - m0;
  // the chunk's exponentials and the running products before each of them
  cplx Eloc[kMaxChunk][D * D];
  cplx Rloc[kMaxChunk][D * D];
  cplx om[D * D], tmp[D * D], P[D * D];
  mat_eye<D>(P);
  for (int k = 0; k < L; ++k) {
    form_omega<D>(om, sA, w + (static_cast<int64_t>(g) * M + m0 + k) * nt, nt);
    mat_expm<D>(Eloc[k], om, tmp);
    mat_copy<D>(Rloc[k], P);  // product of the chunk's steps before k
    mat_mul<D>(tmp, Eloc[k], P);
    mat_copy<D>(P, tmp);
  }
  mat_copy<D>(buf + t * D * D, P);
  __syncthreads();
  if (t == 0) {
    // exclusive prefix / suffix products over the chunks (later ones on the left)
    cplx acc[D * D], nxt[D * D];
    mat_eye<D>(acc);
    for (int q = 0; q < T; ++q) {
      mat_copy<D>(pre + q * D * D, acc);
      mat_mul<D>(nxt, buf + q * D * D, acc);
      mat_copy<D>(acc, nxt);
    }
    mat_eye<D>(acc);
    for (int q = T - 1; q >= 0; --q) {
      mat_copy<D>(suf + q * D * D, acc);
      mat_mul<D>(nxt, acc, buf + q * D * D);
      mat_copy<D>(acc, nxt);
    }
  }
  __syncthreads();
  cplx G[D * D];
  for (int e = 0; e < D * D; ++e) G[e] = gU[static_cast<int64_t>(g) * D * D + e];
  // walk the chunk backwards; Lm = suf_t E_{m1-1} ... E_{m+1}
  cplx Lm[D * D], Rm[D * D], GE[D * D];
  mat_copy<D>(Lm, suf + t * D * D);
  for (int k = L - 1; k >= 0; --k) {
    mat_mul<D>(Rm, Rloc[k], pre + t * D * D);  // E_{m-1} ... E_{m0} pre_t
    // GE = Lm^H G Rm^H
    mat_mul_hn<D>(tmp, Lm, G);
    mat_mul_nh<D>(GE, tmp, Rm);
    // G_Omega: upper-right block of expm([[Omega^H, GE], [0, Omega^H]])
    form_omega<D>(om, sA, w + (static_cast<int64_t>(g) * M + m0 + k) * nt, nt);
    cplx big[4 * D * D], ebig[4 * D * D], tbig[4 * D * D];
    for (int i = 0; i < 2 * D; ++i)
      for (int j = 0; j < 2 * D; ++j) {
        cplx v = {0.0, 0.0};
        if (i < D && j < D) v = cconj(om[j * D + i]);
        else if (i >= D && j >= D) v = cconj(om[(j - D) * D + (i - D)]);
        else if (i < D && j >= D) v = GE[i * D + (j - D)];
        big[i * 2 * D + j] = v;
      }
    mat_expm<2 * D>(ebig, big, tbig);
    cplx* out = gw + (static_cast<int64_t>(g) * M + m0 + k) * nt;
    for (int i = 0; i < nt; ++i) {
      cplx s = {0.0, 0.0};
      for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) s = cfma(cconj(sA[i * D * D + r * D + c]), ebig[r * 2 * D + D + c], s);
      out[i] = s;
    }
    // Lm <- Lm E_m for the next (earlier) step
    mat_mul<D>(tmp, Lm, Eloc[k]);
    mat_copy<D>(Lm, tmp);
  }
}

}  // namespace

namespace {

template <int D>
size_t magnus_smem(int nt, bool grad) {
  return (static_cast<size_t>(nt) + (grad ? 3 : 1) * static_cast<size_t>(threads_for<D>())) * D * D * sizeof(cplx);
}

template <int D>
int magnus_launch(int G, int M, int nt, const double* A, int64_t a_stride, const double* w, const double* gU,
                  double* out, cudaStream_t st) {
  const int T = threads_for<D>();
  if (M > T * kMaxChunk) {
    jq::set_error("jq_magnus: " + std::to_string(M) + " sub-steps exceed the limit of " +
                  std::to_string(T * kMaxChunk) + " for " + std::to_string(D) + "x" + std::to_string(D) + " gates");
    return JQ_EUNSUPPORTED;
  }
  const size_t smem = magnus_smem<D>(nt, gU != nullptr);
  if (smem > 227 * 1024) {
    jq::set_error("jq_magnus: too many Hamiltonian terms for shared memory");
    return JQ_EUNSUPPORTED;
  }
  const cplx* a = reinterpret_cast<const cplx*>(A);
  const cplx* ww = reinterpret_cast<const cplx*>(w);
  cudaError_t e;
  if (gU == nullptr) {
    e = cudaFuncSetAttribute(k_magnus<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e == cudaSuccess) {
      k_magnus<D><<<G, T, smem, st>>>(M, nt, a, a_stride, ww, reinterpret_cast<cplx*>(out));
      e = cudaGetLastError();
    }
  } else {
    e = cudaFuncSetAttribute(k_magnus_grad<D>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e == cudaSuccess) {
      k_magnus_grad<D><<<G, T, smem, st>>>(M, nt, a, a_stride, ww, reinterpret_cast<const cplx*>(gU),
                                           reinterpret_cast<cplx*>(out));
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) {
    jq::set_error(std::string("jq_magnus: ") + cudaGetErrorString(e));
    return JQ_ECUDA;
  }
  return JQ_OK;
}

int magnus_dispatch(int G, int dim, int nt, int M, const double* A, int64_t a_stride, const double* w,
                    const double* gU, double* out, void* stream) {
  if (G < 1 || nt < 1 || M < 1 || !A || !w || !out || a_stride < 0) {
    jq::set_error("jq_magnus: bad arguments");
    return JQ_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  switch (dim) {
    case 2: return magnus_launch<2>(G, M, nt, A, a_stride, w, gU, out, st);
    case 4: return magnus_launch<4>(G, M, nt, A, a_stride, w, gU, out, st);
    case 8: return magnus_launch<8>(G, M, nt, A, a_stride, w, gU, out, st);
    default:
      jq::set_error("jq_magnus: gate dimension " + std::to_string(dim) + " is not 2, 4 or 8");
      return JQ_EUNSUPPORTED;
  }
}

}  // namespace

extern "C" {

int jq_magnus_product(int n_gates, int dim, int n_terms, int n_sub, const double* A, int64_t a_stride,
                      const double* w, double* U, void* stream) {
  return magnus_dispatch(n_gates, dim, n_terms, n_sub, A, a_stride, w, nullptr, U, stream);
}

int jq_magnus_product_grad(int n_gates, int dim, int n_terms, int n_sub, const double* A, int64_t a_stride,
                           const double* w, const double* gU, double* gw, void* stream) {
  if (!gU) {
    jq::set_error("jq_magnus_product_grad: gU is NULL");
    return JQ_EINVAL;
  }
  return magnus_dispatch(n_gates, dim, n_terms, n_sub, A, a_stride, w, gU, gw, stream);
}

}  // extern "C"
