// Device helpers of libjqsim: complex arithmetic, gate-matrix construction in
// float64 and small dense matrix algebra.  Included by jqsim.cu only.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "jq_internal.h"

namespace jq {

template <typename R> struct CplxT;
template <> struct CplxT<float> { using T = float2; };
template <> struct CplxT<double> { using T = double2; };

template <typename C> __device__ __forceinline__ C cmake(double re, double im) {
  C r;
  r.x = static_cast<decltype(r.x)>(re);
  r.y = static_cast<decltype(r.y)>(im);
  return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  C r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.y * b.x - a.x * b.y;
  return r;
}
// acc + a * b with fused multiply-adds
template <typename C> __device__ __forceinline__ C cfma(C a, C b, C acc) {
  C r;
  r.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
  r.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
  return r;
}
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
template <typename C> __device__ __forceinline__ C cscale(C a, double s) {
  a.x = static_cast<decltype(a.x)>(a.x * s);
  a.y = static_cast<decltype(a.y)>(a.y * s);
  return a;
}
__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }

// ---- small dense matrices in float64 (row-major, d x d) --------------------
__device__ inline void m_identity(double2* A, int d) {
  for (int i = 0; i < d * d; ++i) A[i] = make_double2(0.0, 0.0);
  for (int i = 0; i < d; ++i) A[i * d + i] = make_double2(1.0, 0.0);
}
__device__ inline void m_zero(double2* A, int d) {
  for (int i = 0; i < d * d; ++i) A[i] = make_double2(0.0, 0.0);
}
__device__ inline void m_copy(const double2* A, double2* B, int d) {
  for (int i = 0; i < d * d; ++i) B[i] = A[i];
}
// C = A * B
__device__ inline void m_mul(const double2* A, const double2* B, double2* C, int d) {
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) {
      double2 acc = make_double2(0.0, 0.0);
      for (int q = 0; q < d; ++q) acc = cfma(A[i * d + q], B[q * d + j], acc);
      C[i * d + j] = acc;
    }
}
// C = A^dagger * B
__device__ inline void m_mul_ah(const double2* A, const double2* B, double2* C, int d) {
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) {
      double2 acc = make_double2(0.0, 0.0);
      for (int q = 0; q < d; ++q) acc = cfma(cconj(A[q * d + i]), B[q * d + j], acc);
      C[i * d + j] = acc;
    }
}
// C = A * B^dagger
__device__ inline void m_mul_bh(const double2* A, const double2* B, double2* C, int d) {
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) {
      double2 acc = make_double2(0.0, 0.0);
      for (int q = 0; q < d; ++q) acc = cfma(A[i * d + q], cconj(B[j * d + q]), acc);
      C[i * d + j] = acc;
    }
}
// Re <G, X> = Re sum conj(G) X
__device__ inline double m_inner_re(const double2* G, const double2* X, int d) {
  double s = 0.0;
  for (int i = 0; i < d * d; ++i) s += G[i].x * X[i].x + G[i].y * X[i].y;
  return s;
}

// Pauli-rotation block cos(t/2) I - i sin(t/2) P on the inner (target)
// positions of a k-wire matrix whose first nc wires are controls
// (jaqsi/gateset.py:399-405, :764-829).  P|c> = i^ny (-1)^popc(c & pz) |c ^ px>.
// With deriv set, writes d/dt of the matrix instead (zero outside the block).
__device__ inline void m_paulirot(double t, int k, int nc, uint32_t px, uint32_t pz, double2* M, bool deriv) {
  const int d = 1 << k, dt = 1 << (k - nc), base = d - dt;
  if (deriv) m_zero(M, d); else m_identity(M, d);
  double s, c;
  sincos(0.5 * t, &s, &c);
  // inner block = a I + (-i b) P
  const double a = deriv ? -0.5 * s : c;
  const double b = deriv ? 0.5 * c : s;
  for (int r = 0; r < dt; ++r)
    for (int cc = 0; cc < dt; ++cc) M[(base + r) * d + base + cc] = make_double2(r == cc ? a : 0.0, 0.0);
  const int ny = __popc(px & pz) & 3;
  const double2 iy = ny == 0 ? make_double2(1, 0) : ny == 1 ? make_double2(0, 1)
                   : ny == 2 ? make_double2(-1, 0) : make_double2(0, -1);
  for (int cc = 0; cc < dt; ++cc) {
    const int r = cc ^ static_cast<int>(px);
    const double sign = (__popc(static_cast<uint32_t>(cc) & pz) & 1) ? -1.0 : 1.0;
    // (-i b) * (i^ny * sign)
    const double2 ph = make_double2(iy.x * sign, iy.y * sign);
    double2& v = M[(base + r) * d + base + cc];
    v.x += b * ph.y;
    v.y += -b * ph.x;
  }
}

// Full float64 matrix of a parametrised or per-call op (2^k x 2^k).
//   deriv < 0: the matrix; deriv = j >= 0: derivative w.r.t. the op's angle j.
__device__ inline void op_matrix(const DevOp& op, const double* ang, const double2* mats, double2* M,
                                 int deriv, double2* tmp) {
  const int k = op.k, d = 1 << k;
  switch (op.kind) {
    case JQ_K_RX: m_paulirot(ang[op.angle_slot], 1, 0, 1u, 0u, M, deriv >= 0); break;
    case JQ_K_RY: m_paulirot(ang[op.angle_slot], 1, 0, 1u, 1u, M, deriv >= 0); break;
    case JQ_K_RZ: m_paulirot(ang[op.angle_slot], 1, 0, 0u, 1u, M, deriv >= 0); break;
    case JQ_K_PAULIROT: m_paulirot(ang[op.angle_slot], k, op.n_ctrl, op.px, op.pz, M, deriv >= 0); break;
    case JQ_K_ROT: {
      // RZ(omega) @ RY(theta) @ RZ(phi)   (gateset.py:653-657)
      double2 a[4], b[4], c[4], t1[4];
      m_paulirot(ang[op.angle_slot + 0], 1, 0, 0u, 1u, a, deriv == 0);
      m_paulirot(ang[op.angle_slot + 1], 1, 0, 1u, 1u, b, deriv == 1);
      m_paulirot(ang[op.angle_slot + 2], 1, 0, 0u, 1u, c, deriv == 2);
      m_mul(b, a, t1, 2);
      m_mul(c, t1, M, 2);
      break;
    }
    case JQ_K_CPHASE: {
      double s, c;
      sincos(ang[op.angle_slot], &s, &c);
      if (deriv >= 0) {
        m_zero(M, d);
        M[d * d - 1] = make_double2(-s, c);
      } else {
        m_identity(M, d);
        M[d * d - 1] = make_double2(c, s);
      }
      break;
    }
    case JQ_K_MATRIX: {
      if (op.mat_is_diag) {
        m_zero(M, d);
        for (int i = 0; i < d; ++i) M[i * d + i] = mats[op.mat_slot + i];
      } else {
        for (int i = 0; i < d * d; ++i) M[i] = mats[op.mat_slot + i];
      }
      break;
    }
    default: m_identity(M, d); break;
  }
  (void)tmp;
}

// Full float64 matrix of a prim (one factor of a fused block).
//   Pf_U: U; PF_CONJ: conj U; PF_KRON: kron(U, conj U); PF_CONST: pool.
__device__ inline void prim_matrix(const DevPrim& p, const DevOp* ops, const double* ang, const double2* mats,
                                   const double2* cpool, double2* M, int deriv, double2* tmp) {
  const int d = 1 << p.k;
  if (p.form == PF_CONST) {
    for (int i = 0; i < d * d; ++i) M[i] = deriv >= 0 ? make_double2(0, 0) : cpool[p.const_off + i];
    return;
  }
  const DevOp& op = ops[p.op];
  if (p.form == PF_U) { op_matrix(op, ang, mats, M, deriv, tmp); return; }
  if (p.form == PF_CONJ) {
    op_matrix(op, ang, mats, M, deriv, tmp);
    for (int i = 0; i < d * d; ++i) M[i].y = -M[i].y;
    return;
  }
  // PF_KRON of a 1-qubit op: kron(U, conj U); derivative kron(dU, U*) + kron(U, dU*)
  double2 U[4], dU[4];
  op_matrix(op, ang, mats, U, -1, tmp);
  if (deriv >= 0) op_matrix(op, ang, mats, dU, deriv, tmp);
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c)
        for (int e = 0; e < 2; ++e) {
          double2 v;
          if (deriv < 0) {
            v = cmul(U[a * 2 + b], cconj(U[c * 2 + e]));
          } else {
            v = cadd(cmul(dU[a * 2 + b], cconj(U[c * 2 + e])), cmul(U[a * 2 + b], cconj(dU[c * 2 + e])));
          }
          M[(a * 2 + c) * 4 + (b * 2 + e)] = v;
        }
}

}  // namespace jq
