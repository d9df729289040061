// libjqsim: sm_100a kernels and the C ABI of the circuit-execution backend.
//
// The state (a 2^n statevector or a 4^n density matrix seen as a 2n-bit
// vector) lives in caller-owned HBM.  A forward sweep is a short list of tile
// passes: each CTA stages a tile of 2^t amplitudes (t qubits, always including
// the low qubits for coalescing) in shared memory, applies every fused gate
// block of the pass that acts inside the tile, and writes the tile back.  One
// pass therefore replaces the reference's one-XLA-loop-per-entry
// (jaqsi/simulation.py:400-409) for all the blocks it holds.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "jq_internal.h"
#include "kernels.cuh"
#include "jit.h"

namespace jq {
void set_error(const std::string& msg);
extern thread_local std::string g_last_error;
int build_plan(const jq_op* ops, int n_ops, const jq_obs* obs, int n_obs, int n_qubits, int mode, int dtype,
               const jq_tune* tune, jq_plan** out);
}  // namespace jq

namespace jq {
namespace {

constexpr int kRedSlots = 64;  // doubles per warp in the block-reduction scratch
constexpr int kMaxBwdSlots = 32;  // snapshot tiles of the checkpointed reverse pass

// ---------------------------------------------------------------------------
// index helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t pdep64(uint64_t v, uint64_t mask) {
  uint64_t r = 0;
  for (uint64_t bb = 1; mask; bb <<= 1) {
    uint64_t low = mask & (~mask + 1);
    if (v & bb) r |= low;
    mask &= mask - 1;
  }
  return r;
}

// Tile index of group g: zeros inserted at the op's fixed bits (ascending),
// control bits set.  Fully unrolled so the descriptor stays in registers.
__device__ __forceinline__ int group_base(int g, const TileOp& op) {
  uint32_t b = static_cast<uint32_t>(g);
#pragma unroll
  for (int i = 0; i < kMaxBlockWires; ++i) {
    if (i < op.nfix) {
      const uint32_t lm = op.lowmask[i];
      b = ((b & ~lm) << 1) | (b & lm);
    }
  }
  return static_cast<int>(b | op.ctrl_mask);
}

// Tile offset of target combination j (bit kt-1-i of j <-> target i).
__device__ __forceinline__ int target_off(int j, const TileOp& op, int kt) {
  uint32_t o = 0;
#pragma unroll
  for (int i = 0; i < kMaxBlockWires; ++i)
    if (i < kt && ((j >> (kt - 1 - i)) & 1)) o |= op.tmask[i];
  return static_cast<int>(o);
}

// Matrix index of tile element l: its target bits (target 0 most significant).
__device__ __forceinline__ int target_index(int l, const TileOp& op) {
  int a = 0;
#pragma unroll
  for (int i = 0; i < kMaxBlockWires; ++i)
    if (i < op.kt) a = (a << 1) | ((static_cast<uint32_t>(l) & op.tmask[i]) ? 1 : 0);
  return a;
}

// Sum `nv` per-thread doubles over the CTA; thread v < nv receives total v.
// Block-wide sum of NV per-thread values; thread v < NV gets sum v in vals[0].
// NV is a compile-time count so the values stay in registers.
template <int NV>
__device__ __forceinline__ void block_reduce(double (&vals)[NV], double* red) {
  static_assert(NV <= kRedSlots, "reduction scratch too small");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double x = vals[v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    vals[v] = x;
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) red[warp * kRedSlots + v] = vals[v];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[w * kRedSlots + threadIdx.x];
    vals[0] = s;
  }
}

// ---------------------------------------------------------------------------
// block application inside a tile (forward: G, adjoint: G^dagger)
// ---------------------------------------------------------------------------
template <typename C, int KT>
__device__ void tile_dense(C* s, int t, const TileOp& op, const C* __restrict__ M, bool dag) {
  constexpr int D = 1 << KT;
  const int G = 1 << (t - op.nfix);
  int off[D];
#pragma unroll
  for (int j = 0; j < D; ++j) off[j] = target_off(j, op, KT);
  C m[D * D];
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) m[i * D + j] = dag ? cconj(M[j * D + i]) : M[i * D + j];
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const int base = group_base(g, op);
    C v[D];
#pragma unroll
    for (int j = 0; j < D; ++j) v[j] = s[base + off[j]];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      C acc = cmake<C>(0, 0);
#pragma unroll
      for (int j = 0; j < D; ++j) acc = cfma(m[i * D + j], v[j], acc);
      s[base + off[i]] = acc;
    }
  }
}

// Blocks on 3..6 target bits (rare): dynamic loops, group held in local memory.
template <typename C>
__device__ __noinline__ void tile_dense_wide(C* s, int t, const TileOp& op, const C* __restrict__ M, bool dag) {
  const int kt = op.kt, D = 1 << kt;
  const int G = 1 << (t - op.nfix);
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const int base = group_base(g, op);
    C v[64];
#pragma unroll 1
    for (int j = 0; j < D; ++j) v[j] = s[base + target_off(j, op, kt)];
#pragma unroll 1
    for (int i = 0; i < D; ++i) {
      C acc = cmake<C>(0, 0);
#pragma unroll 1
      for (int j = 0; j < D; ++j) acc = cfma(dag ? cconj(M[j * D + i]) : M[i * D + j], v[j], acc);
      s[base + target_off(i, op, kt)] = acc;
    }
  }
}

template <typename C>
__device__ void tile_diag(C* s, int t, const TileOp& op, const C* __restrict__ Dg, bool dag) {
  const uint32_t cm = op.ctrl_mask;
  for (int l = threadIdx.x; l < (1 << t); l += blockDim.x) {
    if ((static_cast<uint32_t>(l) & cm) != cm) continue;
    const C d = dag ? cconj(Dg[target_index(l, op)]) : Dg[target_index(l, op)];
    s[l] = cmul(d, s[l]);
  }
}

template <typename C, int KT>
__device__ void tile_perm(C* s, int t, const TileOp& op, const int* __restrict__ P, bool inv) {
  constexpr int D = 1 << KT;
  const int G = 1 << (t - op.nfix);
  int off[D], p[D];
#pragma unroll
  for (int j = 0; j < D; ++j) {
    off[j] = target_off(j, op, KT);
    p[j] = P[j];
  }
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const int base = group_base(g, op);
    C v[D];
#pragma unroll
    for (int j = 0; j < D; ++j) v[j] = s[base + off[j]];
    if (!inv) {
#pragma unroll
      for (int i = 0; i < D; ++i) s[base + off[i]] = v[p[i]];
    } else {
#pragma unroll
      for (int i = 0; i < D; ++i) s[base + off[p[i]]] = v[i];
    }
  }
}

template <typename C>
__device__ __noinline__ void tile_perm_wide(C* s, int t, const TileOp& op, const int* __restrict__ P, bool inv) {
  const int kt = op.kt, D = 1 << kt;
  const int G = 1 << (t - op.nfix);
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const int base = group_base(g, op);
    C v[64];
#pragma unroll 1
    for (int j = 0; j < D; ++j) v[j] = s[base + target_off(j, op, kt)];
#pragma unroll 1
    for (int i = 0; i < D; ++i) {
      if (!inv) s[base + target_off(i, op, kt)] = v[P[i]];
      else s[base + target_off(P[i], op, kt)] = v[i];
    }
  }
}

template <typename C>
__device__ void tile_apply(C* s, int t, const TileOp& op, const C* bm, const int* perms, bool dag) {
  switch (op.kind) {
    case BK_DENSE:
      switch (op.kt) {
        case 1: tile_dense<C, 1>(s, t, op, bm + op.mat_off, dag); break;
        case 2: tile_dense<C, 2>(s, t, op, bm + op.mat_off, dag); break;
        default: tile_dense_wide<C>(s, t, op, bm + op.mat_off, dag); break;
      }
      break;
    case BK_DIAG: tile_diag<C>(s, t, op, bm + op.mat_off, dag); break;
    default:
      switch (op.kt) {
        case 1: tile_perm<C, 1>(s, t, op, perms + op.perm_off, dag); break;
        case 2: tile_perm<C, 2>(s, t, op, perms + op.perm_off, dag); break;
        default: tile_perm_wide<C>(s, t, op, perms + op.perm_off, dag); break;
      }
      break;
  }
}

// Tile geometry shared by the pass kernels.
struct TileGeo {
  int t, c;
  int64_t tiles_per;
  uint64_t outer_mask;
};

__device__ __forceinline__ void fill_table(uint32_t* tbl, const PassDesc& pd) {
  const int nhi = pd.t - pd.c;
  for (int h = threadIdx.x; h < (1 << nhi); h += blockDim.x) {
    uint32_t o = 0;
    for (int i = 0; i < nhi; ++i)
      if ((h >> i) & 1) o |= 1u << pd.bits[pd.c + i];
    tbl[h] = o;
  }
}

// Tile <-> HBM copies.  Each thread keeps kBatch 16-byte loads in flight
// before writing shared memory, so an SM has tens of KB outstanding (a plain
// element loop leaves one load per warp in flight and is latency-bound).
constexpr int kBatch = 8;
// In the register-stage kernel the copy batch shares registers with the
// stage arrays: 4 vectors (complex64) / 2 (complex128) keep it spill-free.
template <typename C> struct SwzBatch { static constexpr int v = sizeof(C) == 8 ? 4 : 2; };

template <typename C>
__device__ __forceinline__ void tile_load(C* s, const C* g, const uint32_t* tbl, int t, int c) {
  constexpr int V = 16 / sizeof(C);  // amplitudes per 16-byte vector
  const int cm = (1 << c) - 1;
  if (c >= (V == 2 ? 1 : 0)) {
    const int nv = (1 << t) / V;
    for (int v0 = threadIdx.x; v0 < nv; v0 += kBatch * blockDim.x) {
      float4 r[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int v = v0 + u * blockDim.x;
        if (v < nv) {
          const int l = v * V;
          r[u] = __ldcs(reinterpret_cast<const float4*>(g + (tbl[l >> c] | (l & cm))));
        }
      }
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int v = v0 + u * blockDim.x;
        if (v < nv) reinterpret_cast<float4*>(s)[v] = r[u];
      }
    }
  } else {
    for (int l = threadIdx.x; l < (1 << t); l += blockDim.x) s[l] = g[tbl[l >> c] | (l & cm)];
  }
}
template <typename C>
__device__ __forceinline__ void tile_store(const C* s, C* g, const uint32_t* tbl, int t, int c) {
  constexpr int V = 16 / sizeof(C);
  const int cm = (1 << c) - 1;
  if (c >= (V == 2 ? 1 : 0)) {
    const int nv = (1 << t) / V;
    for (int v0 = threadIdx.x; v0 < nv; v0 += kBatch * blockDim.x) {
      float4 r[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int v = v0 + u * blockDim.x;
        if (v < nv) r[u] = reinterpret_cast<const float4*>(s)[v];
      }
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        const int v = v0 + u * blockDim.x;
        if (v < nv) {
          const int l = v * V;
          __stcs(reinterpret_cast<float4*>(g + (tbl[l >> c] | (l & cm))), r[u]);
        }
      }
    }
  } else {
    for (int l = threadIdx.x; l < (1 << t); l += blockDim.x) g[tbl[l >> c] | (l & cm)] = s[l];
  }
}

// ---------------------------------------------------------------------------
// forward tile pass
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(512, 2) k_tile_fwd(typename CplxT<R>::T* __restrict__ state, int nb, int batch,
                                                   PassDesc pd, const TileOp* __restrict__ ops,
                                                   const typename CplxT<R>::T* __restrict__ bmat, int64_t bmat_stride,
                                                   const int* __restrict__ perms) {
  using C = typename CplxT<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  const int t = pd.t, c = pd.c;
  uint32_t* tbl = reinterpret_cast<uint32_t*>(s + (1 << t));
  fill_table(tbl, pd);
  const int64_t tiles_per = 1LL << (nb - t);
  const int64_t ntiles = tiles_per * batch;
  const uint64_t full = (nb >= 64) ? ~0ULL : ((1ULL << nb) - 1);
  const uint64_t outer_mask = full & ~pd.tile_mask;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t inst = tile >> (nb - t);
    const uint64_t ti = static_cast<uint64_t>(tile) & static_cast<uint64_t>(tiles_per - 1);
    C* g = state + (inst << nb) + pdep64(ti, outer_mask);
    const C* bm = bmat + inst * bmat_stride;
    __syncthreads();
    tile_load(s, g, tbl, t, c);
    __syncthreads();
    for (int oi = pd.op_begin; oi < pd.op_end; ++oi) {
      const TileOp op = ops[oi];
      tile_apply<C>(s, t, op, bm, perms, false);
      __syncthreads();
    }
    tile_store(s, g, tbl, t, c);
  }
}

// ---------------------------------------------------------------------------
// register-stage forward pass
// ---------------------------------------------------------------------------
// Shared-memory swizzle: the bank bits of element l are XORed with all its
// higher bits folded onto them (4 bank bits of 8-byte elements for complex64,
// 3 of 16-byte elements for complex128).  Linear over XOR, so a tile offset
// splits into per-bit offsets (Step::ebits / tbits).
template <typename C> __device__ __forceinline__ uint32_t swz(uint32_t l);
template <> __device__ __forceinline__ uint32_t swz<float2>(uint32_t l) {
  return l ^ (((l >> 4) ^ (l >> 8) ^ (l >> 12)) & 15u);
}
template <> __device__ __forceinline__ uint32_t swz<double2>(uint32_t l) {
  return l ^ (((l >> 3) ^ (l >> 6) ^ (l >> 9) ^ (l >> 12)) & 7u);
}

template <typename C>
__device__ __forceinline__ void tile_load_swz(C* s, const C* g, const uint32_t* tbl, int t, int c) {
  constexpr int V = 16 / sizeof(C);
  const int cm = (1 << c) - 1;
  const int nv = (1 << t) / V;
  for (int v0 = threadIdx.x; v0 < nv; v0 += SwzBatch<C>::v * blockDim.x) {
    float4 r[SwzBatch<C>::v];
#pragma unroll
    for (int u = 0; u < SwzBatch<C>::v; ++u) {
      const int v = v0 + u * blockDim.x;
      if (v < nv) {
        const int l = v * V;
        r[u] = __ldcs(reinterpret_cast<const float4*>(g + (tbl[l >> c] | (l & cm))));
      }
    }
#pragma unroll
    for (int u = 0; u < SwzBatch<C>::v; ++u) {
      const int v = v0 + u * blockDim.x;
      if (v < nv) {
        const uint32_t l = static_cast<uint32_t>(v * V);
        if constexpr (V == 2) {
          reinterpret_cast<float2*>(s)[swz<C>(l)] = make_float2(r[u].x, r[u].y);
          reinterpret_cast<float2*>(s)[swz<C>(l + 1)] = make_float2(r[u].z, r[u].w);
        } else {
          reinterpret_cast<float4*>(s)[swz<C>(l)] = r[u];
        }
      }
    }
  }
}

template <typename C>
__device__ __forceinline__ void tile_store_swz(const C* s, C* g, const uint32_t* tbl, int t, int c) {
  constexpr int V = 16 / sizeof(C);
  const int cm = (1 << c) - 1;
  const int nv = (1 << t) / V;
  for (int v0 = threadIdx.x; v0 < nv; v0 += SwzBatch<C>::v * blockDim.x) {
    float4 r[SwzBatch<C>::v];
#pragma unroll
    for (int u = 0; u < SwzBatch<C>::v; ++u) {
      const int v = v0 + u * blockDim.x;
      if (v < nv) {
        const uint32_t l = static_cast<uint32_t>(v * V);
        if constexpr (V == 2) {
          const float2 a = reinterpret_cast<const float2*>(s)[swz<C>(l)];
          const float2 b = reinterpret_cast<const float2*>(s)[swz<C>(l + 1)];
          r[u] = make_float4(a.x, a.y, b.x, b.y);
        } else {
          r[u] = reinterpret_cast<const float4*>(s)[swz<C>(l)];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < SwzBatch<C>::v; ++u) {
      const int v = v0 + u * blockDim.x;
      if (v < nv) {
        const int l = v * V;
        __stcs(reinterpret_cast<float4*>(g + (tbl[l >> c] | (l & cm))), r[u]);
      }
    }
  }
}

// Generic shared-memory op on the swizzled tile (blocks the register forms do
// not cover): a copy of the group loop with swizzled addressing.
template <typename C>
__device__ __noinline__ void swz_apply_generic(C* s, int t, const TileOp& op, const C* __restrict__ bm,
                                               const int* __restrict__ perms) {
  const int kt = op.kt, D = 1 << kt;
  const int G = 1 << (t - op.nfix);
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const int base = group_base(g, op);
    C v[64];
#pragma unroll 1
    for (int j = 0; j < D; ++j) v[j] = s[swz<C>(base + target_off(j, op, kt))];
    if (op.kind == BK_DENSE) {
      const C* M = bm + op.mat_off;
#pragma unroll 1
      for (int i = 0; i < D; ++i) {
        C acc = cmake<C>(0, 0);
#pragma unroll 1
        for (int j = 0; j < D; ++j) acc = cfma(M[i * D + j], v[j], acc);
        s[swz<C>(base + target_off(i, op, kt))] = acc;
      }
    } else if (op.kind == BK_DIAG) {
      const C* Dg = bm + op.mat_off;
#pragma unroll 1
      for (int j = 0; j < D; ++j) s[swz<C>(base + target_off(j, op, kt))] = cmul(Dg[j], v[j]);
    } else {
      const int* P = perms + op.perm_off;
#pragma unroll 1
      for (int i = 0; i < D; ++i) s[swz<C>(base + target_off(i, op, kt))] = v[P[i]];
    }
  }
}

// --- register forms (NR amplitudes per thread, compile-time indices) --------
// Controls that are register bits (crm) select per amplitude group with a
// predicate-free select; CTRL = false is the common uncontrolled path.
template <typename C>
__device__ __forceinline__ C csel(bool p, const C& a, const C& b) {
  C r;
  r.x = p ? a.x : b.x;
  r.y = p ? a.y : b.y;
  return r;
}

template <typename C, int NR, int Q, bool CTRL>
__device__ __forceinline__ void r_dense1(C (&a)[NR], const C* __restrict__ M, uint32_t crm) {
  const C m00 = M[0], m01 = M[1], m10 = M[2], m11 = M[3];
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    if ((j >> Q) & 1) continue;
    const int k = j | (1 << Q);
    const C x = a[j], y = a[k];
    const C nx = cfma(m01, y, cmul(m00, x));
    const C ny = cfma(m11, y, cmul(m10, x));
    if (CTRL) {
      const bool on = (static_cast<uint32_t>(j) & crm) == crm;
      a[j] = csel(on, nx, x);
      a[k] = csel(on, ny, y);
    } else {
      a[j] = nx;
      a[k] = ny;
    }
  }
}

// X on register bit Q, controlled by register bit QC: a pure register rename.
template <typename C, int NR, int Q, int QC>
__device__ __forceinline__ void r_cx(C (&a)[NR]) {
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    if (((j >> Q) & 1) || !((j >> QC) & 1)) continue;
    const int k = j | (1 << Q);
    const C x = a[j];
    a[j] = a[k];
    a[k] = x;
  }
}

template <typename C, int NR, int Q>
__device__ __forceinline__ void r_perm1(C (&a)[NR], uint32_t crm) {
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    if ((j >> Q) & 1) continue;
    const int k = j | (1 << Q);
    const bool on = (static_cast<uint32_t>(j) & crm) == crm;
    const C x = a[j], y = a[k];
    a[j] = csel(on, y, x);
    a[k] = csel(on, x, y);
  }
}

template <typename C, int NR, int Q1, int Q2>
__device__ __forceinline__ void r_dense2(C (&a)[NR], const C* __restrict__ M, uint32_t crm) {
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    if (((j >> Q1) & 1) || ((j >> Q2) & 1)) continue;
    const int i1 = j | (1 << Q2), i2 = j | (1 << Q1), i3 = j | (1 << Q1) | (1 << Q2);
    const C v0 = a[j], v1 = a[i1], v2 = a[i2], v3 = a[i3];
    const bool on = (static_cast<uint32_t>(j) & crm) == crm;
    C o[4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
      o[r] = cfma(M[4 * r + 3], v3, cfma(M[4 * r + 2], v2, cfma(M[4 * r + 1], v1, cmul(M[4 * r], v0))));
    a[j] = csel(on, o[0], v0);
    a[i1] = csel(on, o[1], v1);
    a[i2] = csel(on, o[2], v2);
    a[i3] = csel(on, o[3], v3);
  }
}

template <typename C>
__device__ __forceinline__ C sel4(const C& v0, const C& v1, const C& v2, const C& v3, uint32_t i) {
  return i == 0 ? v0 : i == 1 ? v1 : i == 2 ? v2 : v3;
}

template <typename C, int NR, int Q1, int Q2>
__device__ __forceinline__ void r_perm2(C (&a)[NR], uint32_t perm, uint32_t crm) {
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    if (((j >> Q1) & 1) || ((j >> Q2) & 1)) continue;
    const int i1 = j | (1 << Q2), i2 = j | (1 << Q1), i3 = j | (1 << Q1) | (1 << Q2);
    const C v0 = a[j], v1 = a[i1], v2 = a[i2], v3 = a[i3];
    const bool on = (static_cast<uint32_t>(j) & crm) == crm;
    const uint32_t p = on ? perm : 0xE4u;  // 0xE4 = identity (0,1,2,3)
    a[j] = sel4(v0, v1, v2, v3, p & 3u);
    a[i1] = sel4(v0, v1, v2, v3, (p >> 2) & 3u);
    a[i2] = sel4(v0, v1, v2, v3, (p >> 4) & 3u);
    a[i3] = sel4(v0, v1, v2, v3, (p >> 6) & 3u);
  }
}

template <typename C, int NR>
__device__ __forceinline__ void r_diag(C (&a)[NR], const C* __restrict__ Dg, uint32_t dq, int dk, uint32_t crm) {
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    int idx = 0;
#pragma unroll
    for (int i = 0; i < kMaxRegBits; ++i)
      if (i < dk) idx = (idx << 1) | ((j >> ((dq >> (3 * i)) & 7u)) & 1);
    const bool on = (static_cast<uint32_t>(j) & crm) == crm;
    a[j] = csel(on, cmul(Dg[idx], a[j]), a[j]);
  }
}

#define JQ_Q1(F, ...)                                             \
  switch (q1) {                                                   \
    case 0: F<C, NR, 0 __VA_OPT__(,) __VA_ARGS__); break;         \
    default: break;                                               \
  }

#define JQ_PAIR(F, A, B, ...) case (A) * 8 + (B): F<C, NR, A, B>(a __VA_OPT__(,) __VA_ARGS__); break;
#define JQ_Q2(F, ...)                                                                                    \
  switch (q1 * 8 + q2) {                                                                                 \
    JQ_PAIR(F, 0, 1, __VA_ARGS__) JQ_PAIR(F, 0, 2, __VA_ARGS__) JQ_PAIR(F, 0, 3, __VA_ARGS__)             \
    JQ_PAIR(F, 1, 0, __VA_ARGS__) JQ_PAIR(F, 1, 2, __VA_ARGS__) JQ_PAIR(F, 1, 3, __VA_ARGS__)             \
    JQ_PAIR(F, 2, 0, __VA_ARGS__) JQ_PAIR(F, 2, 1, __VA_ARGS__) JQ_PAIR(F, 2, 3, __VA_ARGS__)             \
    JQ_PAIR(F, 3, 0, __VA_ARGS__) JQ_PAIR(F, 3, 1, __VA_ARGS__) JQ_PAIR(F, 3, 2, __VA_ARGS__)             \
    default:                                                                                              \
      if constexpr (NR > 16) {                                                                            \
        switch (q1 * 8 + q2) {                                                                            \
          JQ_PAIR(F, 0, 4, __VA_ARGS__) JQ_PAIR(F, 1, 4, __VA_ARGS__) JQ_PAIR(F, 2, 4, __VA_ARGS__)       \
          JQ_PAIR(F, 3, 4, __VA_ARGS__) JQ_PAIR(F, 4, 0, __VA_ARGS__) JQ_PAIR(F, 4, 1, __VA_ARGS__)       \
          JQ_PAIR(F, 4, 2, __VA_ARGS__) JQ_PAIR(F, 4, 3, __VA_ARGS__)                                     \
          default: break;                                                                                 \
        }                                                                                                 \
      }                                                                                                   \
      break;                                                                                              \
  }

template <typename C, int NR, int Q>
__device__ __forceinline__ void r_dense1_any(C (&a)[NR], const C* M, uint32_t crm) {
  if (crm == 0) r_dense1<C, NR, Q, false>(a, M, 0);
  else r_dense1<C, NR, Q, true>(a, M, crm);
}

template <typename C, int NR>
__device__ __forceinline__ void reg_apply(C (&a)[NR], uint32_t w0, uint32_t w1, const C* M) {
  const uint32_t ctm = (w1 >> 8) & 0xFFFFu;
  if ((threadIdx.x & ctm) != ctm) return;
  const uint32_t crm = w1 & 0xFFu;
  const int q1 = (w0 >> 4) & 15, q2 = (w0 >> 8) & 15;
  switch (w0 & 15u) {
    case RK_DENSE1:
      switch (q1) {
        case 0: r_dense1_any<C, NR, 0>(a, M, crm); break;
        case 1: r_dense1_any<C, NR, 1>(a, M, crm); break;
        case 2: r_dense1_any<C, NR, 2>(a, M, crm); break;
        case 3: r_dense1_any<C, NR, 3>(a, M, crm); break;
        default: if constexpr (NR > 16) r_dense1_any<C, NR, (NR > 16 ? 4 : 0)>(a, M, crm); break;
      }
      break;
    case RK_PERM1:
      if (crm != 0 && (crm & (crm - 1)) == 0) {
        // single control in a register bit: compile-time rename
        switch (q1 * 8 + (__ffs(crm) - 1)) {
          JQ_PAIR(r_cx, 0, 1) JQ_PAIR(r_cx, 0, 2) JQ_PAIR(r_cx, 0, 3)
          JQ_PAIR(r_cx, 1, 0) JQ_PAIR(r_cx, 1, 2) JQ_PAIR(r_cx, 1, 3)
          JQ_PAIR(r_cx, 2, 0) JQ_PAIR(r_cx, 2, 1) JQ_PAIR(r_cx, 2, 3)
          JQ_PAIR(r_cx, 3, 0) JQ_PAIR(r_cx, 3, 1) JQ_PAIR(r_cx, 3, 2)
          default:
            if constexpr (NR > 16) {
              switch (q1 * 8 + (__ffs(crm) - 1)) {
                JQ_PAIR(r_cx, 0, 4) JQ_PAIR(r_cx, 1, 4) JQ_PAIR(r_cx, 2, 4) JQ_PAIR(r_cx, 3, 4)
                JQ_PAIR(r_cx, 4, 0) JQ_PAIR(r_cx, 4, 1) JQ_PAIR(r_cx, 4, 2) JQ_PAIR(r_cx, 4, 3)
                default: break;
              }
            }
            break;
        }
        break;
      }
      switch (q1) {
        case 0: r_perm1<C, NR, 0>(a, crm); break;
        case 1: r_perm1<C, NR, 1>(a, crm); break;
        case 2: r_perm1<C, NR, 2>(a, crm); break;
        case 3: r_perm1<C, NR, 3>(a, crm); break;
        default: if constexpr (NR > 16) r_perm1<C, NR, (NR > 16 ? 4 : 0)>(a, crm); break;
      }
      break;
    case RK_DIAG: r_diag<C, NR>(a, M, w0 >> 16, (w0 >> 12) & 15, crm); break;
    case RK_DENSE2: JQ_Q2(r_dense2, M, crm) break;
    default: JQ_Q2(r_perm2, w1 >> 24, crm) break;
  }
}

constexpr int kStepWords = sizeof(Step) / 4;

template <typename R, int RB>
__global__ void __launch_bounds__(256, 2) k_tile_fwd2(typename CplxT<R>::T* __restrict__ state, int nb, int batch,
                                                      PassDesc pd, const Step* __restrict__ steps,
                                                      const RegOp* __restrict__ rops, const TileOp* __restrict__ tops,
                                                      const typename CplxT<R>::T* __restrict__ bmat,
                                                      int64_t bmat_stride, const int* __restrict__ perms) {
  using C = typename CplxT<R>::T;
  constexpr int NR = 1 << RB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = pd.t, c = pd.c;
  const int nst = pd.step_end - pd.step_begin, nro = pd.rop_end - pd.rop_begin;
  C* s = reinterpret_cast<C*>(smem_raw);
  C* smat = s + (1 << t);
  uint32_t* tbl = reinterpret_cast<uint32_t*>(smat + ((pd.smat_len + 1) & ~1));
  // every region starts on a 16-byte boundary (sro is read as uint4)
  uint32_t* sst = tbl + (((1 << (t - c)) + 3) & ~3);
  uint4* sro = reinterpret_cast<uint4*>(sst + ((nst * kStepWords + 3) & ~3));
  fill_table(tbl, pd);
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(steps + pd.step_begin);
    for (int i = threadIdx.x; i < nst * kStepWords; i += blockDim.x) sst[i] = src[i];
    for (int i = threadIdx.x; i < nro; i += blockDim.x) {
      const RegOp ro = rops[pd.rop_begin + i];
      sro[i] = make_uint4(ro.w0, ro.w1, ro.w2, ro.w3);
    }
  }
  const int64_t tiles_per = 1LL << (nb - t);
  const int64_t ntiles = tiles_per * batch;
  const uint64_t full = (nb >= 64) ? ~0ULL : ((1ULL << nb) - 1);
  const uint64_t outer_mask = full & ~pd.tile_mask;
  const int nthr_bits = t - RB;
  int64_t last_inst = -1;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t inst = tile >> (nb - t);
    const uint64_t ti = static_cast<uint64_t>(tile) & static_cast<uint64_t>(tiles_per - 1);
    C* g = state + (inst << nb) + pdep64(ti, outer_mask);
    const C* bm = bmat + inst * bmat_stride;
    __syncthreads();
    if (inst != last_inst) {
      // gate matrices of this pass for this instance
      for (int i = 0; i < nro; ++i) {
        const RegOp& ro = rops[pd.rop_begin + i];
        for (int e = threadIdx.x; e < ro.mat_len; e += blockDim.x) smat[ro.w2 + e] = bm[ro.w3 + e];
      }
      last_inst = inst;
    }
    tile_load_swz(s, g, tbl, t, c);
    __syncthreads();
    for (int si = 0; si < nst; ++si) {
      const uint32_t* st = sst + si * kStepWords;
      // Step layout: kind, a, b, ebits[kMaxRegBits], tbits[kMaxThreadBits]
      if (st[0] == 1u) {
        swz_apply_generic<C>(s, t, tops[st[1]], bm, perms);
        __syncthreads();
        continue;
      }
      uint32_t tb = 0;
      for (int i = 0; i < nthr_bits; ++i)
        if ((threadIdx.x >> i) & 1) tb ^= st[3 + kMaxRegBits + i];
      uint32_t e[RB];
#pragma unroll
      for (int q = 0; q < RB; ++q) e[q] = st[3 + q];
      C a[NR];
#pragma unroll
      for (int j = 0; j < NR; ++j) {
        uint32_t o = tb;
#pragma unroll
        for (int q = 0; q < RB; ++q)
          if ((j >> q) & 1) o ^= e[q];
        a[j] = s[o];
      }
      const int ob = static_cast<int>(st[1]) - pd.rop_begin, oe = static_cast<int>(st[2]) - pd.rop_begin;
      for (int oi = ob; oi < oe; ++oi) {
        const uint4 ro = sro[oi];
        reg_apply<C, NR>(a, ro.x, ro.y, smat + ro.z);
      }
#pragma unroll
      for (int j = 0; j < NR; ++j) {
        uint32_t o = tb;
#pragma unroll
        for (int q = 0; q < RB; ++q)
          if ((j >> q) & 1) o ^= e[q];
        s[o] = a[j];
      }
      __syncthreads();
    }
    tile_store_swz(s, g, tbl, t, c);
  }
}

// ---------------------------------------------------------------------------
// adjoint tile pass: psi <- G^dagger psi, grad += lam psi^dagger, lam <- G^dagger lam
// ---------------------------------------------------------------------------
template <typename C, int KT>
__device__ void adj_dense(C* sp, C* sl, int t, const TileOp& op, const C* __restrict__ M, double2* gacc,
                          double* red) {
  constexpr int D = 1 << KT;
  const int G = 1 << (t - op.nfix);
  const bool grad = op.grad_off >= 0;
  int off[D];
#pragma unroll
  for (int j = 0; j < D; ++j) off[j] = target_off(j, op, KT);
  C mh[D * D];  // M^dagger
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) mh[i * D + j] = cconj(M[j * D + i]);
  double2 acc[D * D];
#pragma unroll
  for (int e = 0; e < D * D; ++e) acc[e] = make_double2(0, 0);
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const int base = group_base(g, op);
    C vp[D], vl[D], np[D];
#pragma unroll
    for (int j = 0; j < D; ++j) {
      vp[j] = sp[base + off[j]];
      vl[j] = sl[base + off[j]];
    }
    // psi_{k-1} = G^dagger psi_k
#pragma unroll
    for (int i = 0; i < D; ++i) {
      C a = cmake<C>(0, 0);
#pragma unroll
      for (int j = 0; j < D; ++j) a = cfma(mh[i * D + j], vp[j], a);
      np[i] = a;
      sp[base + off[i]] = a;
    }
    if (grad) {
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const double2 li = to_d2(vl[i]);
#pragma unroll
        for (int j = 0; j < D; ++j) acc[i * D + j] = cfma(li, cconj(to_d2(np[j])), acc[i * D + j]);
      }
    }
#pragma unroll
    for (int i = 0; i < D; ++i) {
      C a = cmake<C>(0, 0);
#pragma unroll
      for (int j = 0; j < D; ++j) a = cfma(mh[i * D + j], vl[j], a);
      sl[base + off[i]] = a;
    }
  }
  if (grad) {
    double vals[2 * D * D];
#pragma unroll
    for (int e = 0; e < D * D; ++e) {
      vals[2 * e] = acc[e].x;
      vals[2 * e + 1] = acc[e].y;
    }
    block_reduce<2 * D * D>(vals, red);
    if (threadIdx.x < 2 * D * D) atomicAdd(reinterpret_cast<double*>(gacc + op.grad_off) + threadIdx.x, vals[0]);
  }
}

// Wide blocks (3..6 target bits): dynamic loops, gradient by direct atomics.
template <typename C>
__device__ __noinline__ void adj_dense_wide(C* sp, C* sl, int t, const TileOp& op, const C* __restrict__ M, double2* gacc) {
  const int kt = op.kt, D = 1 << kt;
  const int G = 1 << (t - op.nfix);
  const bool grad = op.grad_off >= 0;
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const int base = group_base(g, op);
    C vp[64], vl[64], np[64];
#pragma unroll 1
    for (int j = 0; j < D; ++j) {
      vp[j] = sp[base + target_off(j, op, kt)];
      vl[j] = sl[base + target_off(j, op, kt)];
    }
#pragma unroll 1
    for (int i = 0; i < D; ++i) {
      C a = cmake<C>(0, 0), b = cmake<C>(0, 0);
#pragma unroll 1
      for (int j = 0; j < D; ++j) {
        const C mh = cconj(M[j * D + i]);
        a = cfma(mh, vp[j], a);
        b = cfma(mh, vl[j], b);
      }
      np[i] = a;
      sp[base + target_off(i, op, kt)] = a;
      sl[base + target_off(i, op, kt)] = b;
    }
    if (grad) {
#pragma unroll 1
      for (int i = 0; i < D; ++i)
#pragma unroll 1
        for (int j = 0; j < D; ++j) {
          const double2 v = cmul(to_d2(vl[i]), cconj(to_d2(np[j])));
          atomicAdd(&gacc[op.grad_off + i * D + j].x, v.x);
          atomicAdd(&gacc[op.grad_off + i * D + j].y, v.y);
        }
    }
  }
}

template <typename C>
__device__ void adj_diag(C* sp, C* sl, int t, const TileOp& op, const C* __restrict__ Dg, double2* gacc,
                         double* red) {
  const int kt = op.kt, D = 1 << kt;
  const int G = 1 << (t - op.nfix);
  const bool grad = op.grad_off >= 0;
  const int total = G * D;
  double2 acc[4];
  for (int e = 0; e < 4; ++e) acc[e] = make_double2(0, 0);
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int g = e >> kt, j = e & (D - 1);
    const int idx = group_base(g, op) + target_off(j, op, kt);
    const C dc = cconj(Dg[j]);
    const C np = cmul(dc, sp[idx]);
    const C l = sl[idx];
    sp[idx] = np;
    sl[idx] = cmul(dc, l);
    if (grad) {
      const double2 v = cmul(to_d2(l), cconj(to_d2(np)));
      if (kt <= 2) {
        // j < 4: keep in registers
        for (int q = 0; q < 4; ++q)
          if (q == j) acc[q] = cadd(acc[q], v);
      } else {
        atomicAdd(&gacc[op.grad_off + j].x, v.x);
        atomicAdd(&gacc[op.grad_off + j].y, v.y);
      }
    }
  }
  if (grad && kt <= 2) {
    double vals[8];
    for (int q = 0; q < 4; ++q) {
      vals[2 * q] = acc[q].x;
      vals[2 * q + 1] = acc[q].y;
    }
    block_reduce<8>(vals, red);
    if (threadIdx.x < 2 * D) atomicAdd(reinterpret_cast<double*>(gacc + op.grad_off) + threadIdx.x, vals[0]);
  }
}

template <typename C>
__device__ void adj_apply(C* sp, C* sl, int t, const TileOp& op, const C* bm, const int* perms, double2* gacc,
                          double* red) {
  switch (op.kind) {
    case BK_DENSE:
      switch (op.kt) {
        case 1: adj_dense<C, 1>(sp, sl, t, op, bm + op.mat_off, gacc, red); break;
        case 2: adj_dense<C, 2>(sp, sl, t, op, bm + op.mat_off, gacc, red); break;
        default: adj_dense_wide<C>(sp, sl, t, op, bm + op.mat_off, gacc); break;
      }
      break;
    case BK_DIAG: adj_diag<C>(sp, sl, t, op, bm + op.mat_off, gacc, red); break;
    default:
      tile_apply<C>(sp, t, op, bm, perms, true);
      tile_apply<C>(sl, t, op, bm, perms, true);
      break;
  }
}

template <typename R>
__global__ void __launch_bounds__(512, 1) k_tile_adj(typename CplxT<R>::T* __restrict__ psi,
                                                   typename CplxT<R>::T* __restrict__ lam, int nb, int batch,
                                                   PassDesc pd, const TileOp* __restrict__ ops,
                                                   const typename CplxT<R>::T* __restrict__ bmat, int64_t bmat_stride,
                                                   const int* __restrict__ perms, double2* gacc, int64_t grad_stride) {
  using C = typename CplxT<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = pd.t, c = pd.c;
  C* sp = reinterpret_cast<C*>(smem_raw);
  C* sl = sp + (1 << t);
  double* red = reinterpret_cast<double*>(sl + (1 << t));
  uint32_t* tbl = reinterpret_cast<uint32_t*>(red + 32 * kRedSlots);
  fill_table(tbl, pd);
  const int64_t tiles_per = 1LL << (nb - t);
  const int64_t ntiles = tiles_per * batch;
  const uint64_t full = (nb >= 64) ? ~0ULL : ((1ULL << nb) - 1);
  const uint64_t outer_mask = full & ~pd.tile_mask;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t inst = tile >> (nb - t);
    const uint64_t ti = static_cast<uint64_t>(tile) & static_cast<uint64_t>(tiles_per - 1);
    const uint64_t o = (inst << nb) + pdep64(ti, outer_mask);
    const C* bm = bmat + inst * bmat_stride;
    double2* ga = gacc ? gacc + inst * grad_stride : nullptr;
    __syncthreads();
    tile_load(sp, psi + o, tbl, t, c);
    tile_load(sl, lam + o, tbl, t, c);
    __syncthreads();
    for (int oi = pd.op_end - 1; oi >= pd.op_begin; --oi) {
      TileOp op = ops[oi];
      if (!ga) op.grad_off = -1;
      adj_apply<C>(sp, sl, t, op, bm, perms, ga, red);
      __syncthreads();
    }
    tile_store(sp, psi + o, tbl, t, c);
    tile_store(sl, lam + o, tbl, t, c);
  }
}

// ---------------------------------------------------------------------------
// checkpointed reverse step: one block, x is the block's input (kept), lam is
// pulled back through G (lam <- G^dagger lam) and grad += lam x^dagger.
// ---------------------------------------------------------------------------
template <typename C, int KT>
__device__ void bwd_dense(const C* sx, C* sl, int t, const TileOp& op, const C* __restrict__ M, double2* gacc,
                          double* red, double* stage = nullptr) {
  constexpr int D = 1 << KT;
  const int G = 1 << (t - op.nfix);
  const bool grad = op.grad_off >= 0;
  int off[D];
#pragma unroll
  for (int j = 0; j < D; ++j) off[j] = target_off(j, op, KT);
  // G^dagger entries are read from the (L1-cached) block matrix when used
  // rather than held in registers: with the float64 cotangent accumulators
  // they would not fit in a 512-thread CTA's register budget
  double2 acc[D * D];
#pragma unroll
  for (int e = 0; e < D * D; ++e) acc[e] = make_double2(0, 0);
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const int base = group_base(g, op);
    C vx[D], vl[D];
#pragma unroll
    for (int j = 0; j < D; ++j) {
      vx[j] = sx[base + off[j]];
      vl[j] = sl[base + off[j]];
    }
    if (grad) {
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) acc[i * D + j] = cfma(to_d2(vl[i]), cconj(to_d2(vx[j])), acc[i * D + j]);
    }
#pragma unroll
    for (int i = 0; i < D; ++i) {
      C a = cmake<C>(0, 0);
#pragma unroll
      for (int j = 0; j < D; ++j) a = cfma(cconj(__ldg(&M[j * D + i])), vl[j], a);
      sl[base + off[i]] = a;
    }
  }
  if (grad) {
    double vals[2 * D * D];
#pragma unroll
    for (int e = 0; e < D * D; ++e) {
      vals[2 * e] = acc[e].x;
      vals[2 * e + 1] = acc[e].y;
    }
    block_reduce<2 * D * D>(vals, red);
    if (threadIdx.x < 2 * D * D) {
      if (stage) stage[threadIdx.x] += vals[0];  // per-CTA staging, flushed by the caller
      else atomicAdd(reinterpret_cast<double*>(gacc + op.grad_off) + threadIdx.x, vals[0]);
    }
  }
}

template <typename C>
__device__ __noinline__ void bwd_dense_wide(const C* sx, C* sl, int t, const TileOp& op, const C* __restrict__ M,
                               double2* gacc) {
  const int kt = op.kt, D = 1 << kt;
  const int G = 1 << (t - op.nfix);
  const bool grad = op.grad_off >= 0;
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const int base = group_base(g, op);
    C vx[64], vl[64];
#pragma unroll 1
    for (int j = 0; j < D; ++j) {
      vx[j] = sx[base + target_off(j, op, kt)];
      vl[j] = sl[base + target_off(j, op, kt)];
    }
    if (grad) {
#pragma unroll 1
      for (int i = 0; i < D; ++i)
#pragma unroll 1
        for (int j = 0; j < D; ++j) {
          const double2 v = cmul(to_d2(vl[i]), cconj(to_d2(vx[j])));
          atomicAdd(&gacc[op.grad_off + i * D + j].x, v.x);
          atomicAdd(&gacc[op.grad_off + i * D + j].y, v.y);
        }
    }
#pragma unroll 1
    for (int i = 0; i < D; ++i) {
      C a = cmake<C>(0, 0);
#pragma unroll 1
      for (int j = 0; j < D; ++j) a = cfma(cconj(M[j * D + i]), vl[j], a);
      sl[base + target_off(i, op, kt)] = a;
    }
  }
}

template <typename C>
__device__ void bwd_diag(const C* sx, C* sl, int t, const TileOp& op, const C* __restrict__ Dg, double2* gacc,
                         double* red, double* stage = nullptr) {
  const int kt = op.kt, D = 1 << kt;
  const int G = 1 << (t - op.nfix);
  const bool grad = op.grad_off >= 0;
  const int total = G * D;
  double2 acc[4];
  for (int e = 0; e < 4; ++e) acc[e] = make_double2(0, 0);
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int g = e >> kt, j = e & (D - 1);
    const int idx = group_base(g, op) + target_off(j, op, kt);
    const C l = sl[idx];
    sl[idx] = cmul(cconj(Dg[j]), l);
    if (grad) {
      const double2 v = cmul(to_d2(l), cconj(to_d2(sx[idx])));
      if (kt <= 2) {
        for (int q = 0; q < 4; ++q)
          if (q == j) acc[q] = cadd(acc[q], v);
      } else {
        atomicAdd(&gacc[op.grad_off + j].x, v.x);
        atomicAdd(&gacc[op.grad_off + j].y, v.y);
      }
    }
  }
  if (grad && kt <= 2) {
    double vals[8];
    for (int q = 0; q < 4; ++q) {
      vals[2 * q] = acc[q].x;
      vals[2 * q + 1] = acc[q].y;
    }
    block_reduce<8>(vals, red);
    if (threadIdx.x < 2 * D) {
      if (stage) stage[threadIdx.x] += vals[0];
      else atomicAdd(reinterpret_cast<double*>(gacc + op.grad_off) + threadIdx.x, vals[0]);
    }
  }
}

// Warp reduce-scatter of N (power of two, <= 32) per-lane float64 partial
// sums by recursive halving: at the step exchanging with lane ^ O the lanes
// with bit O set keep the upper half of the remaining values.  N - 1 shuffles
// for the halving steps plus one per remaining lane bit; afterwards the lanes
// whose low 5 - log2(N) bits are zero hold value lane >> (5 - log2 N), summed
// over the warp.
template <int O, int N>
struct WarpRSum {
  static __device__ __forceinline__ void run(double* v, unsigned lane) {
    if constexpr (N > 1) {
      constexpr int h = N / 2;
      const bool up = (lane & O) != 0;
#pragma unroll
      for (int i = 0; i < h; ++i) {
        const double send = up ? v[i] : v[i + h];
        const double keep = up ? v[i + h] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, O);
      }
      if constexpr (O > 1) WarpRSum<O / 2, h>::run(v, lane);
    } else {
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], O);
      if constexpr (O > 1) WarpRSum<O / 2, 1>::run(v, lane);
    }
  }
};

// Checkpointed reverse step of one dense block on k = KT bits: x is the
// block's input (kept), lam is pulled back through G (lam <- G^dagger lam)
// and the block cotangent lam x^dagger is added into `stage` (float64, per
// CTA, flushed by the caller): per-lane partial sums, one warp
// reduce-scatter, one shared atomic add per lane that holds a result.
template <typename C, int KT>
__device__ void bwd_dense_rs(const C* sx, C* sl, int t, const TileOp& op, const C* __restrict__ M, double* stage) {
  constexpr int D = 1 << KT;
  constexpr int NV = 2 * D * D;  // 8 or 32 doubles
  const int G = 1 << (t - op.nfix);
  const bool grad = op.grad_off >= 0 && stage != nullptr;
  int off[D];
#pragma unroll
  for (int j = 0; j < D; ++j) off[j] = target_off(j, op, KT);
  double acc[NV];
#pragma unroll
  for (int e = 0; e < NV; ++e) acc[e] = 0.0;
  for (int g = threadIdx.x; g < G; g += blockDim.x) {
    const int base = group_base(g, op);
    C vx[D], vl[D];
#pragma unroll
    for (int j = 0; j < D; ++j) {
      vx[j] = sx[base + off[j]];
      vl[j] = sl[base + off[j]];
    }
    if (grad) {
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
          const double2 p = cfma(to_d2(vl[i]), cconj(to_d2(vx[j])), make_double2(acc[2 * (i * D + j)],
                                                                                acc[2 * (i * D + j) + 1]));
          acc[2 * (i * D + j)] = p.x;
          acc[2 * (i * D + j) + 1] = p.y;
        }
    }
#pragma unroll
    for (int i = 0; i < D; ++i) {
      C a = cmake<C>(0, 0);
#pragma unroll
      for (int j = 0; j < D; ++j) a = cfma(cconj(__ldg(&M[j * D + i])), vl[j], a);
      sl[base + off[i]] = a;
    }
  }
  if (grad) {
    const unsigned lane = threadIdx.x & 31u;
    WarpRSum<16, NV>::run(acc, lane);
    constexpr int lg = NV >= 32 ? 5 : (NV >= 16 ? 4 : 3);
    if ((lane & ((32u >> lg) - 1u)) == 0) atomicAdd(stage + (lane >> (5 - lg)), acc[0]);
  }
}

// Checkpointed reverse pass over one forward pass (density matrices with
// channels, non-unitary pure circuits).  Per tile: x is the state before the
// pass, lam the cotangent after it.  The states before the pass's blocks are
// rebuilt in shared memory without the quadratic recompute:
//  - a forward walk through the pass keeps snapshots of the state before
//    each non-unitary block (slot 0 is the pass input), as many as the
//    shared-memory budget allows (`nslot` tiles);
//  - the reverse walk holds the state before the current block in a work
//    tile; stepping back over a unitary block (a gate, CX halves, two-sided
//    gates) applies its dagger, which undoes it exactly; stepping back over a
//    non-unitary block copies its snapshot, or, for blocks beyond the
//    snapshot budget, re-applies the blocks since the nearest earlier one.
// Block cotangents of 1- and 2-bit dense blocks are staged per CTA (32
// doubles per block) and flushed into the instance's accumulator when the
// CTA moves to another instance.
template <typename R>
__global__ void __launch_bounds__(512, 1) k_tile_bwd(const typename CplxT<R>::T* __restrict__ x,
                                                   typename CplxT<R>::T* __restrict__ lam, int nb, int batch,
                                                   PassDesc pd, const TileOp* __restrict__ ops,
                                                   const typename CplxT<R>::T* __restrict__ bmat, int64_t bmat_stride,
                                                   const int* __restrict__ perms, double2* gacc, int64_t grad_stride,
                                                   int nslot) {
  using C = typename CplxT<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = pd.t, c = pd.c;
  const int T = 1 << t;
  const int nops = pd.op_end - pd.op_begin;
  C* sl = reinterpret_cast<C*>(smem_raw);  // lambda
  C* sw = sl + T;                          // state before the current block
  C* slots = sw + T;                       // snapshots, nslot tiles
  double* red = reinterpret_cast<double*>(slots + static_cast<size_t>(nslot) * T);
  double* stage = red + 32 * kRedSlots;    // 32 doubles per op of the pass
  uint32_t* tbl = reinterpret_cast<uint32_t*>(stage + 32 * nops);
  int* snap_slot = reinterpret_cast<int*>(tbl + (((1 << (t - c)) + 3) & ~3));  // per op: slot of its input, -1
  int* snap_pos = snap_slot + nops;                                             // per slot: op index
  fill_table(tbl, pd);
  for (int e = threadIdx.x; e < 32 * nops; e += blockDim.x) stage[e] = 0.0;
  if (threadIdx.x == 0) {
    // slot 0: the pass input (input of op 0); further slots: inputs of
    // non-unitary ops, evenly spread when there are more than nslot - 1
    int nc = 0;
    for (int k = 1; k < nops; ++k) nc += ops[pd.op_begin + k].inv ? 0 : 1;
    for (int k = 0; k < nops; ++k) snap_slot[k] = -1;
    snap_slot[0] = 0;
    snap_pos[0] = 0;
    int used = 1, seen = 0;
    for (int k = 1; k < nops; ++k) {
      if (ops[pd.op_begin + k].inv) continue;
      // candidate number `seen` of nc is taken when there is room for all of
      // them, else when it is the next of nslot - 1 evenly spaced picks
      if (used < nslot &&
          (nc <= nslot - 1 || seen == static_cast<int>(static_cast<int64_t>(used - 1) * nc / (nslot - 1)))) {
        snap_slot[k] = used;
        snap_pos[used] = k;
        ++used;
      }
      ++seen;
    }
    for (int j = used; j < nslot; ++j) snap_pos[j] = nops;  // unused
  }
  auto stage_slot = [&](const TileOp& op) -> bool { return op.kind == BK_DENSE && op.kt <= 2; };
  auto diag_stage = [&](const TileOp& op) -> bool { return op.kind == BK_DIAG && op.kt <= 2; };
  auto flush = [&](int64_t inst) {
    __syncthreads();
    double* g = reinterpret_cast<double*>(gacc + inst * grad_stride);
    for (int k = 0; k < nops; ++k) {
      const TileOp& op = ops[pd.op_begin + k];
      if (op.grad_off < 0 || !(stage_slot(op) || diag_stage(op))) continue;
      const int nv = op.kind == BK_DENSE ? 2 * (1 << op.kt) * (1 << op.kt) : 2 * (1 << op.kt);
      for (int e = threadIdx.x; e < nv; e += blockDim.x) {
        atomicAdd(g + 2 * op.grad_off + e, stage[32 * k + e]);
        stage[32 * k + e] = 0.0;
      }
    }
    __syncthreads();
  };
  auto copy_tile = [&](C* dst, const C* src) {
    constexpr int V = 16 / sizeof(C);
    for (int v = threadIdx.x; v < T / V; v += blockDim.x)
      reinterpret_cast<float4*>(dst)[v] = reinterpret_cast<const float4*>(src)[v];
  };
  int64_t last_inst = -1;
  const int64_t tiles_per = 1LL << (nb - t);
  const int64_t ntiles = tiles_per * batch;
  const uint64_t full = (nb >= 64) ? ~0ULL : ((1ULL << nb) - 1);
  const uint64_t outer_mask = full & ~pd.tile_mask;
  __syncthreads();
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t inst = tile >> (nb - t);
    const uint64_t ti = static_cast<uint64_t>(tile) & static_cast<uint64_t>(tiles_per - 1);
    const uint64_t o = (inst << nb) + pdep64(ti, outer_mask);
    const C* bm = bmat + inst * bmat_stride;
    double2* ga = gacc ? gacc + inst * grad_stride : nullptr;
    if (gacc && inst != last_inst) {
      if (last_inst >= 0) flush(last_inst);
      last_inst = inst;
    }
    __syncthreads();
    tile_load(slots, x + o, tbl, t, c);
    tile_load(sl, lam + o, tbl, t, c);
    __syncthreads();
    // forward walk: sw <- input of the last op, snapshots on the way
    if (nops > 1) {
      copy_tile(sw, slots);
      __syncthreads();
      for (int k = 0; k + 1 < nops; ++k) {
        if (k > 0 && snap_slot[k] > 0) {
          copy_tile(slots + static_cast<size_t>(snap_slot[k]) * T, sw);
          __syncthreads();
        }
        tile_apply<C>(sw, t, ops[pd.op_begin + k], bm, perms, false);
        __syncthreads();
      }
    }
    // reverse walk
    for (int k = nops - 1; k >= 0; --k) {
      const C* xs = nops > 1 ? sw : slots;
      TileOp op = ops[pd.op_begin + k];
      if (!ga) op.grad_off = -1;
      double* st = stage + 32 * k;
      switch (op.kind) {
        case BK_DENSE:
          switch (op.kt) {
            case 1: bwd_dense_rs<C, 1>(xs, sl, t, op, bm + op.mat_off, ga ? st : nullptr); break;
            case 2: bwd_dense_rs<C, 2>(xs, sl, t, op, bm + op.mat_off, ga ? st : nullptr); break;
            default: bwd_dense_wide<C>(xs, sl, t, op, bm + op.mat_off, ga); break;
          }
          break;
        case BK_DIAG:
          bwd_diag<C>(xs, sl, t, op, bm + op.mat_off, ga, red, op.kt <= 2 ? st : nullptr);
          break;
        default: tile_apply<C>(sl, t, op, bm, perms, true); break;
      }
      __syncthreads();
      if (k == 0 || nops == 1) continue;
      // sw <- input of op k - 1
      const TileOp& prev = ops[pd.op_begin + k - 1];
      if (prev.inv) {
        tile_apply<C>(sw, t, prev, bm, perms, true);
        __syncthreads();
        continue;
      }
      int j = 0;  // the nearest snapshot at or before op k - 1
      for (int q = 1; q < nslot; ++q)
        if (snap_pos[q] <= k - 1) j = q;
      copy_tile(sw, slots + static_cast<size_t>(j) * T);
      __syncthreads();
      for (int q = snap_pos[j]; q < k - 1; ++q) {
        tile_apply<C>(sw, t, ops[pd.op_begin + q], bm, perms, false);
        __syncthreads();
      }
    }
    tile_store(sl, lam + o, tbl, t, c);
  }
  if (gacc && last_inst >= 0) flush(last_inst);
}

// ---------------------------------------------------------------------------
// block matrices: fuse each block's prims in float64, round to the run dtype
// ---------------------------------------------------------------------------
// Inner matrix (or diagonal) of one block of one instance into bm (the
// instance's block matrices); `sc` is the instance's scratch (k > 2 blocks).
template <typename R>
__device__ __noinline__ void prep_block(const DevBlock& blk, const DevPrim* __restrict__ prims, const DevOp* __restrict__ ops,
                           const double* ang, const double2* mt, const double2* __restrict__ cpool,
                           typename CplxT<R>::T* bm, double2* sc) {
  using C = typename CplxT<R>::T;
  if (blk.kind == BK_PERM) return;
  const int d = 1 << blk.k;
  double2 la[16], lb[16], lc[16];
  double2 *acc = la, *pm = lb, *tmp = lc;
  if (blk.k > 2) {
    sc += blk.scratch_off;
    acc = sc;
    pm = sc + d * d;
    tmp = sc + 2 * d * d;
  }
  prim_matrix(prims[blk.prim_begin], ops, ang, mt, cpool, acc, -1, tmp);
  for (int p = blk.prim_begin + 1; p < blk.prim_end; ++p) {
    prim_matrix(prims[p], ops, ang, mt, cpool, pm, -1, tmp);
    m_mul(pm, acc, tmp, d);
    m_copy(tmp, acc, d);
  }
  C* out = bm + blk.mat_off;
  const int base = d - blk.d;
  if (blk.kind == BK_DIAG) {
    for (int i = 0; i < blk.d; ++i) {
      const double2 v = acc[(base + i) * d + base + i];
      out[i] = cmake<C>(v.x, v.y);
    }
  } else {
    for (int i = 0; i < blk.d; ++i)
      for (int j = 0; j < blk.d; ++j) {
        const double2 v = acc[(base + i) * d + base + j];
        out[i * blk.d + j] = cmake<C>(v.x, v.y);
      }
  }
}

template <typename R>
__global__ void k_prep(const DevBlock* __restrict__ blocks, int nblocks, const DevPrim* __restrict__ prims,
                       const DevOp* __restrict__ ops, const double* __restrict__ angles, int n_angles,
                       const double2* __restrict__ mats, int n_mats, const double2* __restrict__ cpool,
                       typename CplxT<R>::T* __restrict__ bmat, int64_t bmat_stride, double2* scratch,
                       int64_t scratch_stride, int batch) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<int64_t>(batch) * nblocks) return;
  const int inst = static_cast<int>(idx / nblocks), b = static_cast<int>(idx % nblocks);
  const DevBlock blk = blocks[b];
  const double* ang = angles ? angles + static_cast<int64_t>(inst) * n_angles : nullptr;
  const double2* mt = mats ? mats + static_cast<int64_t>(inst) * n_mats : nullptr;
  prep_block<R>(blk, prims, ops, ang, mt, cpool, bmat + inst * bmat_stride, scratch + inst * scratch_stride);
}

// ---------------------------------------------------------------------------
// chain rule: block cotangents -> per-prim cotangents -> angles / matrices
// ---------------------------------------------------------------------------
// Chain rule of one block of one instance: block cotangent (gacc: the
// instance's accumulators) -> per-prim cotangents -> angle / matrix gradients
// (ga_out / gm_out: the instance's gradient rows, accumulated atomically).
__device__ __noinline__ void chain_block(const DevBlock& blk, const DevPrim* __restrict__ prims, const DevOp* __restrict__ ops,
                            const double* ang, const double2* mt, const double2* __restrict__ cpool,
                            const double2* gacc, double2* sc, double* ga_out, double2* gm_out) {
  if (blk.grad_off < 0) return;
  const double2* ga = gacc + blk.grad_off;
  const int d = 1 << blk.k;
  double2 l0[16], l1[16], l2[16], l3[16], l4[16], l5[16];
  double2 *Gb = l0, *A = l1, *B = l2, *P = l3, *T = l4, *T2 = l5;
  if (blk.k > 2) {
    sc += blk.scratch_off;
    Gb = sc; A = sc + d * d; B = sc + 2 * d * d; P = sc + 3 * d * d; T = sc + 4 * d * d; T2 = sc + 5 * d * d;
  }
  m_zero(Gb, d);
  const int base = d - blk.d;
  if (blk.kind == BK_DIAG) {
    for (int i = 0; i < blk.d; ++i) Gb[(base + i) * d + base + i] = ga[i];
  } else {
    for (int i = 0; i < blk.d; ++i)
      for (int j = 0; j < blk.d; ++j) Gb[(base + i) * d + base + j] = ga[i * blk.d + j];
  }
  const int m = blk.prim_end - blk.prim_begin;
  for (int i = 0; i < m; ++i) {
    const DevPrim p = prims[blk.prim_begin + i];
    if (p.op < 0 || p.form == PF_CONST) continue;
    const DevOp op = ops[p.op];
    if (!op.grad) continue;
    if (op.kind != JQ_K_MATRIX && op.n_angles == 0) continue;
    // B = P_{i-1} ... P_0
    m_identity(B, d);
    for (int q = 0; q < i; ++q) {
      prim_matrix(prims[blk.prim_begin + q], ops, ang, mt, cpool, P, -1, T2);
      m_mul(P, B, T, d);
      m_copy(T, B, d);
    }
    // A = P_{m-1} ... P_{i+1}
    m_identity(A, d);
    for (int q = i + 1; q < m; ++q) {
      prim_matrix(prims[blk.prim_begin + q], ops, ang, mt, cpool, P, -1, T2);
      m_mul(P, A, T, d);
      m_copy(T, A, d);
    }
    // grad_P = A^dagger Gb B^dagger
    m_mul_ah(A, Gb, T, d);
    m_mul_bh(T, B, A, d);  // A now holds grad_P
    if (op.kind == JQ_K_MATRIX) {
      if (!gm_out) continue;
      double2* gm = gm_out + op.mat_slot;
      const int du = 1 << op.k;
      if (p.form == PF_U || p.form == PF_CONJ) {
        const double sgn = (p.form == PF_CONJ) ? -1.0 : 1.0;
        if (op.mat_is_diag) {
          for (int q = 0; q < du; ++q) {
            atomicAdd(&gm[q].x, A[q * d + q].x);
            atomicAdd(&gm[q].y, sgn * A[q * d + q].y);
          }
        } else {
          for (int q = 0; q < du * du; ++q) {
            atomicAdd(&gm[q].x, A[q].x);
            atomicAdd(&gm[q].y, sgn * A[q].y);
          }
        }
      } else if (p.form == PF_KRON) {
        // S = U (x) conj U: grad_U = X1 + X2 with
        // X1_ab = sum_cd G[ac,bd] U_cd, X2_cd = sum_ab conj(G[ac,bd]) U_ab
        double2 U[4];
        op_matrix(op, ang, mt, U, -1, T2);
        double2 gu[4];
        for (int q = 0; q < 4; ++q) gu[q] = make_double2(0, 0);
        for (int a = 0; a < 2; ++a)
          for (int bb = 0; bb < 2; ++bb)
            for (int c = 0; c < 2; ++c)
              for (int e = 0; e < 2; ++e) {
                const double2 g = A[(a * 2 + c) * 4 + (bb * 2 + e)];
                gu[a * 2 + bb] = cfma(g, U[c * 2 + e], gu[a * 2 + bb]);
                gu[c * 2 + e] = cfma(cconj(g), U[a * 2 + bb], gu[c * 2 + e]);
              }
        if (op.mat_is_diag) {
          atomicAdd(&gm[0].x, gu[0].x); atomicAdd(&gm[0].y, gu[0].y);
          atomicAdd(&gm[1].x, gu[3].x); atomicAdd(&gm[1].y, gu[3].y);
        } else {
          for (int q = 0; q < 4; ++q) { atomicAdd(&gm[q].x, gu[q].x); atomicAdd(&gm[q].y, gu[q].y); }
        }
      }
      continue;
    }
    if (!ga_out) continue;
    for (int j = 0; j < op.n_angles; ++j) {
      prim_matrix(p, ops, ang, mt, cpool, P, j, T2);
      const double g = m_inner_re(A, P, d);
      atomicAdd(&ga_out[op.angle_slot + j], g);
    }
  }
}

__global__ void k_chain(const DevBlock* __restrict__ blocks, int nblocks, const DevPrim* __restrict__ prims,
                        const DevOp* __restrict__ ops, const double* __restrict__ angles, int n_angles,
                        const double2* __restrict__ mats, int n_mats, const double2* __restrict__ cpool,
                        const double2* __restrict__ gacc, int64_t grad_stride, double2* scratch,
                        int64_t scratch_stride, int batch, double* grad_angles, double2* grad_mats) {
  const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= static_cast<int64_t>(batch) * nblocks) return;
  const int inst = static_cast<int>(idx / nblocks), b = static_cast<int>(idx % nblocks);
  const DevBlock blk = blocks[b];
  const double* ang = angles ? angles + static_cast<int64_t>(inst) * n_angles : nullptr;
  const double2* mt = mats ? mats + static_cast<int64_t>(inst) * n_mats : nullptr;
  chain_block(blk, prims, ops, ang, mt, cpool, gacc + inst * grad_stride, scratch + inst * scratch_stride,
              grad_angles ? grad_angles + static_cast<int64_t>(inst) * n_angles : nullptr,
              grad_mats ? grad_mats + static_cast<int64_t>(inst) * n_mats : nullptr);
}

// ---------------------------------------------------------------------------
// state initialisation and measurements
// ---------------------------------------------------------------------------
template <typename R>
__global__ void k_init(typename CplxT<R>::T* state, int64_t elems, int batch, const typename CplxT<R>::T* init,
                       int64_t init_elems, int init_batched, int pure_density) {
  using C = typename CplxT<R>::T;
  const int64_t total = elems * batch;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t inst = i / elems, j = i - inst * elems;
    C v;
    if (!init) {
      v = cmake<C>(j == 0 ? 1.0 : 0.0, 0.0);
    } else {
      const C* src = init + (init_batched ? inst * init_elems : 0);
      if (!pure_density) {
        v = src[j];
      } else {
        // rho = psi psi^dagger (jaqsi/simulation.py:470-471)
        const int64_t r = j / init_elems, c = j - r * init_elems;
        v = cmulc(src[r], src[c]);
      }
    }
    state[i] = v;
  }
}

template <typename R>
__global__ void k_probs_sv(const typename CplxT<R>::T* psi, R* out, int64_t total) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const auto a = psi[i];
    out[i] = a.x * a.x + a.y * a.y;
  }
}

template <typename R>
__global__ void k_probs_dm(const typename CplxT<R>::T* rho, R* out, int64_t dim, int batch) {
  const int64_t total = dim * batch;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t inst = i / dim, j = i - inst * dim;
    out[i] = rho[inst * dim * dim + j * dim + j].x;
  }
}

template <typename R>
__global__ void k_outer(const typename CplxT<R>::T* psi, typename CplxT<R>::T* out, int64_t dim, int batch) {
  const int64_t total = dim * dim * batch;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t inst = i / (dim * dim), e = i - inst * dim * dim;
    const int64_t r = e / dim, c = e - r * dim;
    out[i] = cmulc(psi[inst * dim + r], psi[inst * dim + c]);
  }
}

// i^ny * w, real part
__device__ __forceinline__ double re_iy(int ny, double2 w) {
  switch (ny & 3) {
    case 0: return w.x;
    case 1: return -w.y;
    case 2: return -w.x;
    default: return w.y;
  }
}
__device__ __forceinline__ double2 mul_iy(int ny, double2 w) {
  switch (ny & 3) {
    case 0: return w;
    case 1: return make_double2(-w.y, w.x);
    case 2: return make_double2(-w.x, -w.y);
    default: return make_double2(w.y, -w.x);
  }
}

constexpr int kObsChunk = 16;

// <psi| coeff P |psi> for up to kObsChunk Pauli words, float64 accumulation.
// Z strings only (x_mask == 0 for every word of the chunk), one read of the
// state.  A thread takes 8 consecutive amplitudes j0 + u at a time and forms
// the Walsh sums w[m] = sum_u (-1)^popc(u & m) |psi_{j0+u}|^2 (m < 8) in
// shared memory; word z then adds (-1)^popc((j0 >> 3) & (z >> 3)) w[z & 7].
// The coefficients multiply the reduced sums.  Needs z >> 3 < 2^32.
template <typename C>
__device__ __forceinline__ void probs8(const C* p, double pa[8]);
template <>
__device__ __forceinline__ void probs8<float2>(const float2* p, double pa[8]) {
  const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const float4 v = q[h];
    pa[2 * h] = static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y;
    pa[2 * h + 1] = static_cast<double>(v.z) * v.z + static_cast<double>(v.w) * v.w;
  }
}
template <>
__device__ __forceinline__ void probs8<double2>(const double2* p, double pa[8]) {
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const double2 v = p[u];
    pa[u] = v.x * v.x + v.y * v.y;
  }
}

template <typename R>
__global__ void __launch_bounds__(256, 2) k_expval_zdiag_sv(const typename CplxT<R>::T* psi, int64_t dim,
                                                            const DevObs* obs, int o_begin, int o_cnt, double* out,
                                                            int n_obs) {
  __shared__ double red[8 * kRedSlots];
  __shared__ double sw[8][256];
  __shared__ uint2 sinfo[kObsChunk];
  __shared__ double sc[kObsChunk];
  const int tid = threadIdx.x;
  if (tid < kObsChunk) {
    const bool on = tid < o_cnt;
    const DevObs ob = obs[o_begin + (on ? tid : 0)];
    sinfo[tid] = make_uint2(static_cast<uint32_t>(ob.z_mask >> 3), static_cast<uint32_t>(ob.z_mask & 7));
    sc[tid] = on ? ob.coeff : 0.0;
  }
  __syncthreads();
  const int inst = blockIdx.y;
  const auto* p = psi + static_cast<int64_t>(inst) * dim;
  double acc[kObsChunk];
#pragma unroll
  for (int o = 0; o < kObsChunk; ++o) acc[o] = 0.0;
  const int64_t ng = dim >> 3;
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + tid; g < ng;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double pa[8];
    probs8(p + (g << 3), pa);
    const double a0 = pa[0] + pa[1], a1 = pa[0] - pa[1], a2 = pa[2] + pa[3], a3 = pa[2] - pa[3];
    const double a4 = pa[4] + pa[5], a5 = pa[4] - pa[5], a6 = pa[6] + pa[7], a7 = pa[6] - pa[7];
    const double b0 = a0 + a2, b1 = a1 + a3, b2 = a0 - a2, b3 = a1 - a3;
    const double b4 = a4 + a6, b5 = a5 + a7, b6 = a4 - a6, b7 = a5 - a7;
    sw[0][tid] = b0 + b4;
    sw[1][tid] = b1 + b5;
    sw[2][tid] = b2 + b6;
    sw[3][tid] = b3 + b7;
    sw[4][tid] = b0 - b4;
    sw[5][tid] = b1 - b5;
    sw[6][tid] = b2 - b6;
    sw[7][tid] = b3 - b7;
    const uint32_t gh = static_cast<uint32_t>(g);
#pragma unroll
    for (int o = 0; o < kObsChunk; ++o) {
      if (o < o_cnt) {
        // volatile: re-read per group instead of holding 2 x 16 words in registers
        const volatile uint32_t* vi = reinterpret_cast<const volatile uint32_t*>(sinfo) + 2 * o;
        const uint32_t zx = vi[0], zl = vi[1];
        const double w = sw[zl][tid];
        acc[o] += (__popc(gh & zx) & 1) ? -w : w;
      }
    }
  }
  // fewer than 8 amplitudes (up to two qubits)
  if (dim < 8 && blockIdx.x == 0) {
    for (int64_t j = tid; j < dim; j += blockDim.x) {
      const double2 a = to_d2(p[j]);
      const double pj = a.x * a.x + a.y * a.y;
#pragma unroll
      for (int o = 0; o < kObsChunk; ++o) {
        if (o < o_cnt) {
          const uint64_t z = (static_cast<uint64_t>(sinfo[o].x) << 3) | sinfo[o].y;
          acc[o] += (__popcll(static_cast<uint64_t>(j) & z) & 1) ? -pj : pj;
        }
      }
    }
  }
  block_reduce<kObsChunk>(acc, red);
  if (tid < o_cnt) atomicAdd(&out[static_cast<int64_t>(inst) * n_obs + o_begin + tid], sc[tid] * acc[0]);
}

// Z strings, up to kZMax words in one read of the state (n >= 9).  A warp
// takes 512-amplitude chunks with contiguous 16-byte loads: lane l's k-th
// load is element 32 k + l of the chunk, so a thread's 16 amplitudes vary in
// index bits {0, 6, 7, 8} (complex64, two amplitudes a load) or {5, 6, 7, 8}
// (complex128).  The thread forms the 16 Walsh sums of their probabilities;
// a word's bits on those four positions pick one sum, its parity on the
// thread's other index bits gives the sign.  Float64 sums throughout.
constexpr int kZMax = 32;

template <typename R>
__global__ void __launch_bounds__(256) k_expval_zstr_sv(const typename CplxT<R>::T* psi, int64_t dim,
                                                        const DevObs* obs, int o_begin, int o_cnt, double* out,
                                                        int n_obs) {
  using C = typename CplxT<R>::T;
  constexpr bool F = sizeof(C) == 8;
  __shared__ double red[8 * kRedSlots];
  __shared__ uint64_t sz[kZMax];
  __shared__ int sm[kZMax];
  __shared__ double sc[kZMax];
  __shared__ double sw[16][256];
  const int tid = threadIdx.x;
  if (tid < kZMax) {
    const bool on = tid < o_cnt;
    const uint64_t z = on ? obs[o_begin + tid].z_mask : 0;
    sz[tid] = z;
    sm[tid] = F ? static_cast<int>((z & 1) | ((z >> 5) & 14)) : static_cast<int>((z >> 5) & 15);
    sc[tid] = on ? obs[o_begin + tid].coeff : 0.0;
  }
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5, nw = static_cast<int>(blockDim.x >> 5);
  const int inst = blockIdx.y;
  const C* p = psi + static_cast<int64_t>(inst) * dim;
  double acc[kZMax];
#pragma unroll
  for (int o = 0; o < kZMax; ++o) acc[o] = 0.0;
  const int64_t nchunk = dim >> 9;
  for (int64_t ch = static_cast<int64_t>(blockIdx.x) * nw + warp; ch < nchunk;
       ch += static_cast<int64_t>(gridDim.x) * nw) {
    double w[16];
    if constexpr (F) {
      const float4* q = reinterpret_cast<const float4*>(p + (ch << 9));
      float4 v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = __ldcs(q + 32 * k + lane);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        w[2 * k] = static_cast<double>(v[k].x) * v[k].x + static_cast<double>(v[k].y) * v[k].y;
        w[2 * k + 1] = static_cast<double>(v[k].z) * v[k].z + static_cast<double>(v[k].w) * v[k].w;
      }
    } else {
      const double2* q = reinterpret_cast<const double2*>(p + (ch << 9));
      double2 v[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = __ldcs(q + 32 * k + lane);
#pragma unroll
      for (int k = 0; k < 16; ++k) w[k] = v[k].x * v[k].x + v[k].y * v[k].y;
    }
    // Walsh-Hadamard transform over the 4 group bits: w[m] = sum_j p_j (-1)^popc(j & m)
#pragma unroll
    for (int b = 1; b < 16; b <<= 1)
#pragma unroll
      for (int j = 0; j < 16; ++j)
        if (!(j & b)) {
          const double a = w[j], c = w[j | b];
          w[j] = a + c;
          w[j | b] = a - c;
        }
#pragma unroll
    for (int m = 0; m < 16; ++m) sw[m][tid] = w[m];
    const uint64_t gb = (static_cast<uint64_t>(ch) << 9) | static_cast<uint64_t>(F ? (lane << 1) : lane);
#pragma unroll
    for (int o = 0; o < kZMax; ++o) {
      if (o < o_cnt) {
        const double x = sw[sm[o]][tid];
        acc[o] += (__popcll(gb & sz[o]) & 1) ? -x : x;
      }
    }
  }
  block_reduce<kZMax>(acc, red);
  if (tid < o_cnt) atomicAdd(&out[static_cast<int64_t>(inst) * n_obs + o_begin + tid], sc[tid] * acc[0]);
}

// General Pauli words: <psi| coeff P |psi> = coeff sum_j conj(psi_j) phase(j ^ x) psi_{j ^ x}.
template <typename R>
__global__ void __launch_bounds__(256, 2) k_expval_pauli_sv(const typename CplxT<R>::T* psi, int64_t dim,
                                                            const DevObs* obs, int o_begin, int o_cnt, double* out,
                                                            int n_obs) {
  __shared__ double red[8 * kRedSlots];
  __shared__ uint64_t sx[kObsChunk], sz[kObsChunk];
  __shared__ double sc[kObsChunk];
  __shared__ int sy[kObsChunk];
  if (threadIdx.x < kObsChunk) {
    const bool on = threadIdx.x < o_cnt;
    const DevObs ob = obs[o_begin + (on ? threadIdx.x : 0)];
    sx[threadIdx.x] = ob.x_mask;
    sz[threadIdx.x] = ob.z_mask;
    sc[threadIdx.x] = on ? ob.coeff : 0.0;
    sy[threadIdx.x] = ob.n_y;
  }
  __syncthreads();
  const int inst = blockIdx.y;
  const auto* p = psi + static_cast<int64_t>(inst) * dim;
  double acc[kObsChunk];
#pragma unroll
  for (int o = 0; o < kObsChunk; ++o) acc[o] = 0.0;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < dim;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double2 a = to_d2(p[j]);
    const double pa = a.x * a.x + a.y * a.y;
#pragma unroll
    for (int o = 0; o < kObsChunk; ++o) {
      if (o < o_cnt) {
        const uint64_t x = sx[o];
        const int64_t jx = j ^ static_cast<int64_t>(x);
        const double sign = (__popcll(static_cast<uint64_t>(jx) & sz[o]) & 1) ? -sc[o] : sc[o];
        if (x == 0) {
          acc[o] = fma(sign, pa, acc[o]);
        } else {
          const double2 w = cmul(cconj(a), to_d2(p[jx]));
          acc[o] = fma(sign, re_iy(sy[o], w), acc[o]);
        }
      }
    }
  }
  block_reduce<kObsChunk>(acc, red);
  if (threadIdx.x < o_cnt) atomicAdd(&out[static_cast<int64_t>(inst) * n_obs + o_begin + threadIdx.x], acc[0]);
}

// <psi|O|psi> for one dense Hermitian observable on k wires.
template <typename R>
__global__ void k_expval_dense_sv(const typename CplxT<R>::T* psi, int n, const DevObs* obs, int oi,
                                  const double2* pool, double* out, int n_obs) {
  __shared__ double red[32 * kRedSlots];
  const int inst = blockIdx.y;
  const DevObs ob = obs[oi];
  const int k = ob.k, D = 1 << k;
  const int64_t dim = 1LL << n;
  const auto* p = psi + static_cast<int64_t>(inst) * dim;
  const double2* O = pool + ob.mat_off;
  uint64_t fix = 0;
  for (int i = 0; i < k; ++i) fix |= 1ULL << ob.bits[i];
  const int64_t groups = dim >> k;
  double acc = 0.0;
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < groups;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint64_t base = pdep64(static_cast<uint64_t>(g), ((dim - 1) & ~fix));
    for (int a = 0; a < D; ++a) {
      uint64_t ia = base;
      for (int i = 0; i < k; ++i)
        if ((a >> (k - 1 - i)) & 1) ia |= 1ULL << ob.bits[i];
      const double2 va = to_d2(p[ia]);
      double2 row = make_double2(0, 0);
      for (int bcol = 0; bcol < D; ++bcol) {
        uint64_t ib = base;
        for (int i = 0; i < k; ++i)
          if ((bcol >> (k - 1 - i)) & 1) ib |= 1ULL << ob.bits[i];
        row = cfma(O[a * D + bcol], to_d2(p[ib]), row);
      }
      acc += va.x * row.x + va.y * row.y;
    }
  }
  double accv[1] = {acc};
  block_reduce<1>(accv, red);
  if (threadIdx.x == 0) atomicAdd(&out[static_cast<int64_t>(inst) * n_obs + oi], accv[0]);
}

// Tr(coeff P rho) = coeff sum_k phase(k) rho[k][k ^ x]
template <typename R>
__global__ void k_expval_pauli_dm(const typename CplxT<R>::T* rho, int64_t dim, const DevObs* obs, int o_begin,
                                  int o_cnt, double* out, int n_obs) {
  __shared__ double red[32 * kRedSlots];
  const int inst = blockIdx.y;
  const auto* p = rho + static_cast<int64_t>(inst) * dim * dim;
  double acc[kObsChunk];
#pragma unroll
  for (int o = 0; o < kObsChunk; ++o) acc[o] = 0.0;
  for (int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < dim;
       j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int o = 0; o < kObsChunk; ++o) {
      if (o < o_cnt) {
        const DevObs ob = obs[o_begin + o];
        const int64_t jx = j ^ static_cast<int64_t>(ob.x_mask);
        const double sign = (__popcll(static_cast<uint64_t>(j) & ob.z_mask) & 1) ? -1.0 : 1.0;
        const double2 v = to_d2(p[j * dim + jx]);
        acc[o] += ob.coeff * sign * re_iy(ob.n_y, v);
      }
    }
  }
  block_reduce<kObsChunk>(acc, red);
  if (threadIdx.x < o_cnt) atomicAdd(&out[static_cast<int64_t>(inst) * n_obs + o_begin + threadIdx.x], acc[0]);
}

// Tr(O rho) = sum_ab O_ab sum_rest rho[(b,rest)][(a,rest)]
template <typename R>
__global__ void k_expval_dense_dm(const typename CplxT<R>::T* rho, int n, const DevObs* obs, int oi,
                                  const double2* pool, double* out, int n_obs) {
  __shared__ double red[32 * kRedSlots];
  const int inst = blockIdx.y;
  const DevObs ob = obs[oi];
  const int k = ob.k, D = 1 << k;
  const int64_t dim = 1LL << n;
  const auto* p = rho + static_cast<int64_t>(inst) * dim * dim;
  const double2* O = pool + ob.mat_off;
  uint64_t fix = 0;
  for (int i = 0; i < k; ++i) fix |= 1ULL << ob.bits[i];
  const int64_t groups = dim >> k;
  double acc = 0.0;
  for (int64_t g = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; g < groups;
       g += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const uint64_t base = pdep64(static_cast<uint64_t>(g), ((dim - 1) & ~fix));
    for (int a = 0; a < D; ++a) {
      uint64_t ia = base;
      for (int i = 0; i < k; ++i)
        if ((a >> (k - 1 - i)) & 1) ia |= 1ULL << ob.bits[i];
      for (int bcol = 0; bcol < D; ++bcol) {
        uint64_t ib = base;
        for (int i = 0; i < k; ++i)
          if ((bcol >> (k - 1 - i)) & 1) ib |= 1ULL << ob.bits[i];
        const double2 w = cmul(O[a * D + bcol], to_d2(p[ib * dim + ia]));
        acc += w.x;
      }
    }
  }
  double accv[1] = {acc};
  block_reduce<1>(accv, red);
  if (threadIdx.x == 0) atomicAdd(&out[static_cast<int64_t>(inst) * n_obs + oi], accv[0]);
}

// ---------------------------------------------------------------------------
// seeds of the reverse pass (lam = dL/dRe + i dL/dIm of the final state)
// ---------------------------------------------------------------------------
// statevector expval: lam = 2 sum_o ct_o O_o psi
template <typename R>
__global__ void k_seed_expval_sv(const typename CplxT<R>::T* psi, typename CplxT<R>::T* lam, int n, int batch,
                                 const DevObs* obs, int n_obs, const double2* pool, const double* ct) {
  using C = typename CplxT<R>::T;
  const int64_t dim = 1LL << n;
  const int64_t total = dim * batch;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t inst = i / dim, j = i - inst * dim;
    const C* p = psi + inst * dim;
    double2 acc = make_double2(0, 0);
    for (int o = 0; o < n_obs; ++o) {
      const DevObs ob = obs[o];
      const double w = 2.0 * ct[inst * n_obs + o];
      if (w == 0.0) continue;
      if (ob.kind == JQ_OBS_PAULI) {
        const int64_t jx = j ^ static_cast<int64_t>(ob.x_mask);
        const double sign = (__popcll(static_cast<uint64_t>(jx) & ob.z_mask) & 1) ? -1.0 : 1.0;
        const double2 v = mul_iy(ob.n_y, to_d2(p[jx]));
        acc.x += w * ob.coeff * sign * v.x;
        acc.y += w * ob.coeff * sign * v.y;
      } else {
        const int k = ob.k, D = 1 << k;
        int a = 0;
        uint64_t rest = static_cast<uint64_t>(j);
        for (int q = 0; q < k; ++q) {
          a = (a << 1) | static_cast<int>((j >> ob.bits[q]) & 1);
          rest &= ~(1ULL << ob.bits[q]);
        }
        double2 row = make_double2(0, 0);
        for (int bcol = 0; bcol < D; ++bcol) {
          uint64_t ib = rest;
          for (int q = 0; q < k; ++q)
            if ((bcol >> (k - 1 - q)) & 1) ib |= 1ULL << ob.bits[q];
          row = cfma(pool[ob.mat_off + a * D + bcol], to_d2(p[ib]), row);
        }
        acc.x += w * row.x;
        acc.y += w * row.y;
      }
    }
    lam[i] = cmake<C>(acc.x, acc.y);
  }
}

// statevector probs: lam_j = 2 ct_j psi_j
template <typename R>
__global__ void k_seed_probs_sv(const typename CplxT<R>::T* psi, typename CplxT<R>::T* lam, const R* ct,
                                int64_t total) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const R w = 2 * ct[i];
    auto a = psi[i];
    a.x *= w;
    a.y *= w;
    lam[i] = a;
  }
}

// pure density output rho = psi psi^dagger: lam = (G + G^dagger) psi
template <typename R>
__global__ void k_seed_density_sv(const typename CplxT<R>::T* psi, typename CplxT<R>::T* lam,
                                  const typename CplxT<R>::T* G, int64_t dim, int batch) {
  using C = typename CplxT<R>::T;
  const int64_t total = dim * batch;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t inst = i / dim, r = i - inst * dim;
    const C* g = G + inst * dim * dim;
    const C* p = psi + inst * dim;
    double2 acc = make_double2(0, 0);
    for (int64_t c = 0; c < dim; ++c) {
      const double2 m = cadd(to_d2(g[r * dim + c]), cconj(to_d2(g[c * dim + r])));
      acc = cfma(m, to_d2(p[c]), acc);
    }
    lam[i] = cmake<C>(acc.x, acc.y);
  }
}

// density expval: lam[r][c] = sum_o ct_o O_o[r][c]
template <typename R>
__global__ void k_seed_expval_dm(typename CplxT<R>::T* lam, int n, int batch, const DevObs* obs, int n_obs,
                                 const double2* pool, const double* ct) {
  using C = typename CplxT<R>::T;
  const int64_t dim = 1LL << n, sz = dim * dim;
  const int64_t total = sz * batch;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t inst = i / sz, e = i - inst * sz;
    const uint64_t r = static_cast<uint64_t>(e / dim), c = static_cast<uint64_t>(e - (e / dim) * dim);
    double2 acc = make_double2(0, 0);
    for (int o = 0; o < n_obs; ++o) {
      const DevObs ob = obs[o];
      const double w = ct[inst * n_obs + o];
      if (w == 0.0) continue;
      if (ob.kind == JQ_OBS_PAULI) {
        if ((r ^ c) != ob.x_mask) continue;
        const double sign = (__popcll(c & ob.z_mask) & 1) ? -1.0 : 1.0;
        const double2 v = mul_iy(ob.n_y, make_double2(w * ob.coeff * sign, 0.0));
        acc = cadd(acc, v);
      } else {
        uint64_t fix = 0;
        int a = 0, bcol = 0;
        for (int q = 0; q < ob.k; ++q) {
          fix |= 1ULL << ob.bits[q];
          a = (a << 1) | static_cast<int>((r >> ob.bits[q]) & 1);
          bcol = (bcol << 1) | static_cast<int>((c >> ob.bits[q]) & 1);
        }
        if ((r & ~fix) != (c & ~fix)) continue;
        const double2 v = pool[ob.mat_off + a * (1 << ob.k) + bcol];
        acc.x += w * v.x;
        acc.y += w * v.y;
      }
    }
    lam[i] = cmake<C>(acc.x, acc.y);
  }
}

// density probs: lam = diag(ct)
template <typename R>
__global__ void k_seed_probs_dm(typename CplxT<R>::T* lam, const R* ct, int64_t dim, int batch) {
  using C = typename CplxT<R>::T;
  const int64_t sz = dim * dim, total = sz * batch;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t inst = i / sz, e = i - inst * sz;
    const int64_t r = e / dim, c = e - r * dim;
    lam[i] = cmake<C>(r == c ? static_cast<double>(ct[inst * dim + r]) : 0.0, 0.0);
  }
}

// cotangent of psi0 when rho0 = psi0 psi0^dagger: (L + L^dagger) psi0
template <typename R>
__global__ void k_grad_init_dm(const typename CplxT<R>::T* lam, const typename CplxT<R>::T* init, int init_batched,
                               typename CplxT<R>::T* out, int64_t dim, int batch) {
  using C = typename CplxT<R>::T;
  const int64_t total = dim * batch;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t inst = i / dim, r = i - inst * dim;
    const C* L = lam + inst * dim * dim;
    const C* p = init + (init_batched ? inst * dim : 0);
    double2 acc = make_double2(0, 0);
    for (int64_t c = 0; c < dim; ++c) {
      const double2 m = cadd(to_d2(L[r * dim + c]), cconj(to_d2(L[c * dim + r])));
      acc = cfma(m, to_d2(p[c]), acc);
    }
    out[i] = cmake<C>(acc.x, acc.y);
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
#define JQ_CUDA(expr)                                                                     \
  do {                                                                                    \
    cudaError_t _e = (expr);                                                              \
    if (_e != cudaSuccess) {                                                              \
      set_error(std::string("CUDA error: ") + cudaGetErrorString(_e) + " at " #expr);     \
      return JQ_ECUDA;                                                                    \
    }                                                                                     \
  } while (0)

int g_sm_count = 0;

int sm_count() {
  if (g_sm_count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0) g_sm_count = 148;
  }
  return g_sm_count;
}

std::mutex g_upload_mu;

template <typename T>
int upload(const std::vector<T>& v, T** dst) {
  *dst = nullptr;
  if (v.empty()) return JQ_OK;
  JQ_CUDA(cudaMalloc(reinterpret_cast<void**>(dst), v.size() * sizeof(T)));
  JQ_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return JQ_OK;
}

int device_tables(const jq_plan* cplan, const DeviceTables** out) {
  jq_plan* plan = const_cast<jq_plan*>(cplan);
  int dev = 0;
  JQ_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_upload_mu);
  for (const DeviceTables& t : plan->dev)
    if (t.device == dev) {
      if (t.jit_rc) {
        set_error(t.jit_err);
        return t.jit_rc;
      }
      *out = &t;
      return JQ_OK;
    }
  DeviceTables t;
  t.device = dev;
  int rc;
  if ((rc = upload(plan->ops, &t.ops))) return rc;
  if ((rc = upload(plan->prims, &t.prims))) return rc;
  if ((rc = upload(plan->blocks, &t.blocks))) return rc;
  if ((rc = upload(plan->fwd.ops, &t.fwd_ops))) return rc;
  if ((rc = upload(plan->adj.ops, &t.adj_ops))) return rc;
  if ((rc = upload(plan->const_pool, &t.const_pool))) return rc;
  if ((rc = upload(plan->perm_pool, &t.perm_pool))) return rc;
  if ((rc = upload(plan->obs_pool, &t.obs_pool))) return rc;
  DevObs* od = nullptr;
  if ((rc = upload(plan->obs, &od))) return rc;
  t.obs_desc = od;
  TileOp* bo = nullptr;
  if ((rc = upload(plan->bwd.ops, &bo))) return rc;
  t.bwd_ops = bo;
  if ((rc = upload(plan->fwd.steps, &t.fwd_steps))) return rc;
  if ((rc = upload(plan->fwd.rops, &t.fwd_rops))) return rc;
  if ((rc = upload(plan->bwd.steps, &t.bwd_steps))) return rc;
  if ((rc = upload(plan->bwd.rops, &t.bwd_rops))) return rc;
  if (plan->jit && jit_available()) {
    JitModule* jm = new JitModule();
    if ((rc = jit_build(plan, plan->fwd, jm)) == JQ_OK) {
      t.jit = jm;
    } else {
      jit_free(jm);
      delete jm;
      // automatic mode: the register-stage interpreter kernels run instead;
      // jq_tune.jit = 1: the plan fails on this device (tables kept for jq_plan_free)
      if (plan->jit_required) {
        t.jit_rc = rc;
        t.jit_err = g_last_error;
      }
    }
  } else if (plan->jit_required) {
    t.jit_rc = JQ_EUNSUPPORTED;
    t.jit_err = "jq_tune.jit = 1 but NVRTC or the CUDA driver entry points are not available";
  }
  t.jit_tried = true;
  plan->dev.push_back(t);
  if (t.jit_rc) {
    set_error(t.jit_err);
    return t.jit_rc;
  }
  *out = &plan->dev.back();
  return JQ_OK;
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

struct WsLayout {
  size_t bmat = 0, scratch = 0, lam = 0, psi = 0, gacc = 0, ckpt = 0, seg = 0, work = 0, total = 0;
  int64_t n_ckpt = 0, seg_len = 0;
};

WsLayout layout(const jq_plan* plan, int batch, int mode_grad /*0 fwd, 1 adjoint, 2 ckpt*/) {
  WsLayout L;
  const size_t elem = plan->dtype == JQ_C64 ? 8 : 16;
  const size_t state = static_cast<size_t>(plan->state_elems) * elem * batch;
  size_t off = 0;
  L.bmat = off;
  off += align256(static_cast<size_t>(plan->bmat_stride) * elem * batch);
  L.scratch = off;
  off += align256(static_cast<size_t>(plan->scratch_stride) * 16 * batch);
  if (mode_grad >= 1) {
    L.lam = off;
    off += align256(state);
    L.gacc = off;
    off += align256(static_cast<size_t>(plan->grad_stride) * 16 * batch);
  }
  if (mode_grad == 1) {
    L.psi = off;
    off += align256(state);
  }
  if (mode_grad == 2) {
    const int64_t P = static_cast<int64_t>(plan->fwd.passes.size());
    int64_t S = plan->ckpt_stride > 0 ? plan->ckpt_stride : static_cast<int64_t>(std::ceil(std::sqrt(static_cast<double>(std::max<int64_t>(P, 1)))));
    S = std::max<int64_t>(1, S);
    L.seg_len = S;
    L.n_ckpt = (P + S - 1) / S;
    L.work = off;
    off += align256(state);
    L.ckpt = off;
    off += align256(state) * static_cast<size_t>(std::max<int64_t>(L.n_ckpt, 1));
    L.seg = off;
    off += align256(state) * static_cast<size_t>(S);
  }
  L.total = off;
  return L;
}

// Largest grid.y of a launch (instances of a batch run along y).
constexpr int kMaxGridY = 65535;

int grid_for(int64_t work, int threads) {
  int64_t g = (work + threads - 1) / threads;
  const int64_t cap = static_cast<int64_t>(sm_count()) * 16;
  return static_cast<int>(std::max<int64_t>(1, std::min(g, cap)));
}

template <typename R>
size_t tile_smem(const PassDesc& pd, int n_tiles_in_smem) {
  const size_t elem = sizeof(typename CplxT<R>::T);
  size_t s = (static_cast<size_t>(n_tiles_in_smem) << pd.t) * elem;
  if (n_tiles_in_smem == 2) s += 32 * kRedSlots * sizeof(double);
  s += (static_cast<size_t>(1) << (pd.t - pd.c)) * sizeof(uint32_t);
  return s;
}

template <typename R>
int set_smem_attrs() {
  static bool done = false;
  if (done) return JQ_OK;
  const int max_smem = 227 * 1024;
  JQ_CUDA(cudaFuncSetAttribute(k_tile_fwd<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
  JQ_CUDA(cudaFuncSetAttribute(k_tile_adj<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
  JQ_CUDA(cudaFuncSetAttribute(k_tile_bwd<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem));
  JQ_CUDA(cudaFuncSetAttribute(k_tile_fwd2<R, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               max_smem));
  done = true;
  return JQ_OK;
}

template <typename K>
int ctas_for(K kernel, int threads, size_t smem, int64_t ntiles) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  if (per_sm < 1) per_sm = 1;
  int64_t cap = static_cast<int64_t>(sm_count()) * per_sm;
  return static_cast<int>(std::max<int64_t>(1, std::min(ntiles, cap)));
}

// Run passes [p0, p1) of a schedule over `state` (batch instances).  Passes
// with a register-stage program use k_tile_fwd2, the others k_tile_fwd.
template <typename R>
int run_passes(const jq_plan* plan, const Schedule& sch, const TileOp* dops, const Step* dsteps,
               const RegOp* drops, const DeviceTables* T, typename CplxT<R>::T* state, int batch,
               const typename CplxT<R>::T* bmat, size_t p0, size_t p1, cudaStream_t st,
               const JitModule* jm = nullptr) {
  constexpr int RB = 4;
  for (size_t p = p0; p < p1; ++p) {
    const PassDesc& pd = sch.passes[p];
    if (pd.op_end == pd.op_begin) continue;
    if (jm && p < jm->fn.size() && jm->fn[p]) {
      const int rc = jit_launch(*jm, sch, static_cast<int>(p), plan->n_bits, sm_count(), state, batch, bmat,
                                plan->bmat_stride, static_cast<int>(sizeof(typename CplxT<R>::T)), st);
      if (rc) return rc;
      continue;
    }
    const size_t smem = tile_smem<R>(pd, 1);
    const int64_t ntiles = (1LL << (plan->n_bits - pd.t)) * batch;
    if (pd.step_end > pd.step_begin && sch.reg_bits == RB) {
      const int threads = 1 << (pd.t - RB);
      const size_t elem = sizeof(typename CplxT<R>::T);
      const int nst = pd.step_end - pd.step_begin;
      const size_t smem2 = (static_cast<size_t>(1) << pd.t) * elem + ((pd.smat_len + 1) & ~1) * elem +
                           (((static_cast<size_t>(1) << (pd.t - pd.c)) + 3) & ~static_cast<size_t>(3)) * 4 +
                           ((nst * kStepWords + 3) & ~3) * 4 +
                           static_cast<size_t>(pd.rop_end - pd.rop_begin) * 16;
      const int ctas = ctas_for(k_tile_fwd2<R, RB>, threads, smem2, ntiles);
      k_tile_fwd2<R, RB><<<ctas, threads, smem2, st>>>(state, plan->n_bits, batch, pd, dsteps, drops, dops, bmat,
                                                       plan->bmat_stride, T->perm_pool);
    } else {
      const int ctas = ctas_for(k_tile_fwd<R>, plan->threads, smem, ntiles);
      k_tile_fwd<R><<<ctas, plan->threads, smem, st>>>(state, plan->n_bits, batch, pd, dops, bmat, plan->bmat_stride,
                                                        T->perm_pool);
    }
  }
  JQ_CUDA(cudaGetLastError());
  return JQ_OK;
}

template <typename R>
int prep(const jq_plan* plan, const DeviceTables* T, int batch, const double* angles, const void* mats,
         typename CplxT<R>::T* bmat, double2* scratch, cudaStream_t st) {
  const int nbk = static_cast<int>(plan->blocks.size());
  if (nbk == 0) return JQ_OK;
  const int64_t work = static_cast<int64_t>(nbk) * batch;
  const int threads = 128;
  const int grid = static_cast<int>((work + threads - 1) / threads);
  k_prep<R><<<grid, threads, 0, st>>>(T->blocks, nbk, T->prims, T->ops, angles, plan->n_angles,
                                      reinterpret_cast<const double2*>(mats), plan->n_mats,
                                      reinterpret_cast<const double2*>(T->const_pool), bmat, plan->bmat_stride,
                                      scratch, plan->scratch_stride, batch);
  JQ_CUDA(cudaGetLastError());
  return JQ_OK;
}

template <typename R>
int measure(const jq_plan* plan, const DeviceTables* T, int batch, int out_type, const typename CplxT<R>::T* state,
            void* out, cudaStream_t st) {
  using C = typename CplxT<R>::T;
  const int n = plan->n_qubits;
  const int64_t dim = 1LL << n;
  const bool dm = plan->mode == JQ_DENSITY;
  const int threads = 256;
  if (out_type == JQ_OUT_STATE) return JQ_OK;
  if (out_type == JQ_OUT_PROBS) {
    if (dm) {
      k_probs_dm<R><<<grid_for(dim * batch, threads), threads, 0, st>>>(state, static_cast<R*>(out), dim, batch);
    } else {
      k_probs_sv<R><<<grid_for(dim * batch, threads), threads, 0, st>>>(state, static_cast<R*>(out), dim * batch);
    }
  } else if (out_type == JQ_OUT_DENSITY) {
    if (dm) return JQ_OK;  // the state is the density matrix
    k_outer<R><<<grid_for(dim * dim * batch, threads), threads, 0, st>>>(state, static_cast<C*>(out), dim, batch);
  } else if (out_type == JQ_OUT_EXPVAL) {
    const int n_obs = static_cast<int>(plan->obs.size());
    if (n_obs == 0) return JQ_OK;
    double* o = static_cast<double*>(out);
    JQ_CUDA(cudaMemsetAsync(o, 0, sizeof(double) * n_obs * batch, st));
    const DevObs* od = static_cast<const DevObs*>(T->obs_desc);
    const double2* pool = reinterpret_cast<const double2*>(T->obs_pool);
    // Pauli observables in chunks; dense ones one launch each
    int i = 0;
    while (i < n_obs) {
      if (plan->obs[i].kind == JQ_OBS_PAULI) {
        // runs of Pauli words that are all Z strings (or all not), kObsChunk at
        // most (kZMax for the one-read Z-string kernel, statevectors of n >= 9)
        const bool zdiag = plan->obs[i].x_mask == 0 && (plan->obs[i].z_mask >> 35) == 0;
        const bool zstr = zdiag && !dm && n >= 9;
        const int chunk = zstr ? kZMax : kObsChunk;
        int j = i;
        while (j < n_obs && j - i < chunk && plan->obs[j].kind == JQ_OBS_PAULI &&
               (plan->obs[j].x_mask == 0 && (plan->obs[j].z_mask >> 35) == 0) == zdiag)
          ++j;
        const int gx = std::max(1, std::min<int>(static_cast<int>((dim + threads - 1) / threads),
                                                 std::max(1, 4 * sm_count() / std::max(batch, 1))));
        // instances run along grid.y, at most kMaxGridY per launch
        for (int b0 = 0; b0 < batch; b0 += kMaxGridY) {
          const dim3 grid(gx, std::min(batch - b0, kMaxGridY));
          const C* sb = state + static_cast<int64_t>(b0) * plan->state_elems;
          double* ob = o + static_cast<int64_t>(b0) * n_obs;
          if (dm) k_expval_pauli_dm<R><<<grid, threads, 0, st>>>(sb, dim, od, i, j - i, ob, n_obs);
          else if (zstr) {
            // one warp per 512-amplitude chunk
            const int gz = std::max(1, std::min<int>(static_cast<int>((dim >> 9) / (threads / 32)) + 1,
                                                     std::max(1, 4 * sm_count() / std::max(batch, 1))));
            k_expval_zstr_sv<R><<<dim3(gz, grid.y), threads, 0, st>>>(sb, dim, od, i, j - i, ob, n_obs);
          } else if (zdiag) k_expval_zdiag_sv<R><<<grid, threads, 0, st>>>(sb, dim, od, i, j - i, ob, n_obs);
          else k_expval_pauli_sv<R><<<grid, threads, 0, st>>>(sb, dim, od, i, j - i, ob, n_obs);
        }
        i = j;
      } else {
        const int64_t groups = dim >> plan->obs[i].k;
        const int gx = std::max(1, std::min<int>(static_cast<int>((groups + threads - 1) / threads),
                                                 std::max(1, 4 * sm_count() / std::max(batch, 1))));
        for (int b0 = 0; b0 < batch; b0 += kMaxGridY) {
          const dim3 grid(gx, std::min(batch - b0, kMaxGridY));
          const C* sb = state + static_cast<int64_t>(b0) * plan->state_elems;
          double* ob = o + static_cast<int64_t>(b0) * n_obs;
          if (dm) k_expval_dense_dm<R><<<grid, threads, 0, st>>>(sb, n, od, i, pool, ob, n_obs);
          else k_expval_dense_sv<R><<<grid, threads, 0, st>>>(sb, n, od, i, pool, ob, n_obs);
        }
        ++i;
      }
    }
  } else {
    set_error("unknown out_type");
    return JQ_EINVAL;
  }
  JQ_CUDA(cudaGetLastError());
  return JQ_OK;
}

template <typename R>
int forward_impl(const jq_plan* plan, int batch, const double* angles, const void* mats, const void* init,
                 int init_batched, int out_type, void* state, void* out, void* ws, size_t ws_bytes,
                 cudaStream_t st) {
  using C = typename CplxT<R>::T;
  const DeviceTables* T = nullptr;
  int rc = device_tables(plan, &T);
  if (rc) return rc;
  if ((rc = set_smem_attrs<R>())) return rc;
  WsLayout L = layout(plan, batch, 0);
  if (ws_bytes < L.total || (L.total > 0 && !ws)) {
    set_error("workspace too small: need " + std::to_string(L.total) + " bytes");
    return JQ_ENOMEM;
  }
  char* w = static_cast<char*>(ws);
  C* bmat = reinterpret_cast<C*>(w + L.bmat);
  double2* scratch = reinterpret_cast<double2*>(w + L.scratch);
  if ((rc = prep<R>(plan, T, batch, angles, mats, bmat, scratch, st))) return rc;
  C* S = static_cast<C*>(state);
  const bool dm = plan->mode == JQ_DENSITY;
  const int64_t dim = 1LL << plan->n_qubits;
  const bool init_rho = dm && init && (init_batched & JQ_INIT_DENSITY);  // init is a density matrix
  k_init<R><<<grid_for(plan->state_elems * batch, 256), 256, 0, st>>>(
      S, plan->state_elems, batch, static_cast<const C*>(init), init_rho ? plan->state_elems : dim,
      init_batched & 1, dm && init && !init_rho ? 1 : 0);
  JQ_CUDA(cudaGetLastError());
  if ((rc = run_passes<R>(plan, plan->fwd, T->fwd_ops, T->fwd_steps, T->fwd_rops, T, S, batch, bmat, 0, plan->fwd.passes.size(), st,
                          static_cast<const JitModule*>(T->jit)))) return rc;
  return measure<R>(plan, T, batch, out_type, S, out, st);
}

template <typename R>
int sweep_impl(const jq_plan* plan, int batch, const double* angles, const void* mats, void* state, void* ws,
               size_t ws_bytes, cudaStream_t st) {
  using C = typename CplxT<R>::T;
  const DeviceTables* T = nullptr;
  int rc = device_tables(plan, &T);
  if (rc) return rc;
  if ((rc = set_smem_attrs<R>())) return rc;
  WsLayout L = layout(plan, batch, 0);
  if (ws_bytes < L.total || (L.total > 0 && !ws)) {
    set_error("workspace too small: need " + std::to_string(L.total) + " bytes");
    return JQ_ENOMEM;
  }
  char* w = static_cast<char*>(ws);
  C* bmat = reinterpret_cast<C*>(w + L.bmat);
  double2* scratch = reinterpret_cast<double2*>(w + L.scratch);
  if ((rc = prep<R>(plan, T, batch, angles, mats, bmat, scratch, st))) return rc;
  return run_passes<R>(plan, plan->fwd, T->fwd_ops, T->fwd_steps, T->fwd_rops, T, static_cast<C*>(state), batch, bmat, 0,
                       plan->fwd.passes.size(), st, static_cast<const JitModule*>(T->jit));
}

template <typename R>
int seed_sv(const jq_plan* plan, const DeviceTables* T, int batch, int out_type, const typename CplxT<R>::T* psi,
            const double* ct, const void* ct_state, typename CplxT<R>::T* lam, cudaStream_t st) {
  using C = typename CplxT<R>::T;
  const int64_t dim = 1LL << plan->n_qubits;
  const int threads = 256;
  switch (out_type) {
    case JQ_OUT_EXPVAL:
      k_seed_expval_sv<R><<<grid_for(dim * batch, threads), threads, 0, st>>>(
          psi, lam, plan->n_qubits, batch, static_cast<const DevObs*>(T->obs_desc), static_cast<int>(plan->obs.size()),
          reinterpret_cast<const double2*>(T->obs_pool), ct);
      break;
    case JQ_OUT_STATE:
      JQ_CUDA(cudaMemcpyAsync(lam, ct_state, sizeof(C) * dim * batch, cudaMemcpyDeviceToDevice, st));
      break;
    case JQ_OUT_PROBS:
      k_seed_probs_sv<R><<<grid_for(dim * batch, threads), threads, 0, st>>>(psi, lam, static_cast<const R*>(ct_state),
                                                                             dim * batch);
      break;
    case JQ_OUT_DENSITY:
      k_seed_density_sv<R><<<grid_for(dim * batch, threads), threads, 0, st>>>(psi, lam, static_cast<const C*>(ct_state),
                                                                               dim, batch);
      break;
    default:
      set_error("unknown out_type");
      return JQ_EINVAL;
  }
  JQ_CUDA(cudaGetLastError());
  return JQ_OK;
}

template <typename R>
int seed_dm(const jq_plan* plan, const DeviceTables* T, int batch, int out_type, const double* ct,
            const void* ct_state, typename CplxT<R>::T* lam, cudaStream_t st) {
  using C = typename CplxT<R>::T;
  const int64_t dim = 1LL << plan->n_qubits;
  const int threads = 256;
  switch (out_type) {
    case JQ_OUT_EXPVAL:
      k_seed_expval_dm<R><<<grid_for(dim * dim * batch, threads), threads, 0, st>>>(
          lam, plan->n_qubits, batch, static_cast<const DevObs*>(T->obs_desc), static_cast<int>(plan->obs.size()),
          reinterpret_cast<const double2*>(T->obs_pool), ct);
      break;
    case JQ_OUT_STATE:
    case JQ_OUT_DENSITY:
      JQ_CUDA(cudaMemcpyAsync(lam, ct_state, sizeof(C) * dim * dim * batch, cudaMemcpyDeviceToDevice, st));
      break;
    case JQ_OUT_PROBS:
      k_seed_probs_dm<R><<<grid_for(dim * dim * batch, threads), threads, 0, st>>>(lam, static_cast<const R*>(ct_state),
                                                                                  dim, batch);
      break;
    default:
      set_error("unknown out_type");
      return JQ_EINVAL;
  }
  JQ_CUDA(cudaGetLastError());
  return JQ_OK;
}

template <typename R>
int chain(const jq_plan* plan, const DeviceTables* T, int batch, const double* angles, const void* mats,
          const double2* gacc, double2* scratch, double* grad_angles, void* grad_mats, cudaStream_t st) {
  if (grad_angles && plan->n_angles > 0)
    JQ_CUDA(cudaMemsetAsync(grad_angles, 0, sizeof(double) * plan->n_angles * batch, st));
  if (grad_mats && plan->n_mats > 0)
    JQ_CUDA(cudaMemsetAsync(grad_mats, 0, 16 * static_cast<size_t>(plan->n_mats) * batch, st));
  const int nbk = static_cast<int>(plan->blocks.size());
  if (nbk == 0 || plan->grad_stride == 0) return JQ_OK;
  const int64_t work = static_cast<int64_t>(nbk) * batch;
  const int threads = 64;
  k_chain<<<static_cast<int>((work + threads - 1) / threads), threads, 0, st>>>(
      T->blocks, nbk, T->prims, T->ops, angles, plan->n_angles, reinterpret_cast<const double2*>(mats), plan->n_mats,
      reinterpret_cast<const double2*>(T->const_pool), gacc, plan->grad_stride, scratch, plan->scratch_stride, batch,
      grad_angles, static_cast<double2*>(grad_mats));
  JQ_CUDA(cudaGetLastError());
  return JQ_OK;
}

template <typename R>
int adjoint_impl(const jq_plan* plan, int batch, const double* angles, const void* mats, const void* state,
                 int out_type, const double* ct, const void* ct_state, double* grad_angles, void* grad_mats,
                 void* grad_init, void* ws, size_t ws_bytes, cudaStream_t st) {
  using C = typename CplxT<R>::T;
  if (plan->mode != JQ_STATEVECTOR || !plan->unitary) {
    set_error("jq_adjoint needs a unitary statevector plan; use jq_backward");
    return JQ_EINVAL;
  }
  const DeviceTables* T = nullptr;
  int rc = device_tables(plan, &T);
  if (rc) return rc;
  if ((rc = set_smem_attrs<R>())) return rc;
  WsLayout L = layout(plan, batch, 1);
  if (ws_bytes < L.total || !ws) {
    set_error("workspace too small: need " + std::to_string(L.total) + " bytes");
    return JQ_ENOMEM;
  }
  char* w = static_cast<char*>(ws);
  C* bmat = reinterpret_cast<C*>(w + L.bmat);
  double2* scratch = reinterpret_cast<double2*>(w + L.scratch);
  C* lam = reinterpret_cast<C*>(w + L.lam);
  C* psi = reinterpret_cast<C*>(w + L.psi);
  double2* gacc = reinterpret_cast<double2*>(w + L.gacc);
  const int64_t elems = plan->state_elems;
  if ((rc = prep<R>(plan, T, batch, angles, mats, bmat, scratch, st))) return rc;
  JQ_CUDA(cudaMemcpyAsync(psi, state, sizeof(C) * elems * batch, cudaMemcpyDeviceToDevice, st));
  if ((rc = seed_sv<R>(plan, T, batch, out_type, psi, ct, ct_state, lam, st))) return rc;
  const bool want_grad = (grad_angles || grad_mats) && plan->grad_stride > 0;
  if (want_grad) JQ_CUDA(cudaMemsetAsync(gacc, 0, 16 * static_cast<size_t>(plan->grad_stride) * batch, st));
  // Specialised adjoint: the forward schedule's passes in reverse, each one
  // kernel holding both tiles (psi and lam) in shared memory.
  const JitModule* jm = static_cast<const JitModule*>(T->jit);
  bool use_jit = jm && jm->has_adjoint;
  if (use_jit)
    for (size_t p = 0; p < plan->fwd.passes.size(); ++p)
      if (plan->fwd.passes[p].op_end > plan->fwd.passes[p].op_begin && !jm->afn[p]) use_jit = false;
  if (use_jit) {
    const Schedule& fs = plan->fwd;
    for (size_t pi = fs.passes.size(); pi-- > 0;) {
      if (fs.passes[pi].op_end == fs.passes[pi].op_begin) continue;
      if ((rc = jit_launch_adj(*jm, fs, static_cast<int>(pi), plan->n_bits, sm_count(), psi, lam, batch, bmat,
                               plan->bmat_stride, want_grad ? reinterpret_cast<double*>(gacc) : nullptr,
                               plan->grad_stride, static_cast<int>(sizeof(C)), st)))
        return rc;
    }
  }
  const Schedule& sch = plan->adj;
  for (size_t pi = sch.passes.size(); !use_jit && pi-- > 0;) {
    const PassDesc& pd = sch.passes[pi];
    if (pd.op_end == pd.op_begin) continue;
    const size_t smem = tile_smem<R>(pd, 2);
    const int64_t ntiles = (1LL << (plan->n_bits - pd.t)) * batch;
    const int ctas = ctas_for(k_tile_adj<R>, plan->threads, smem, ntiles);
    k_tile_adj<R><<<ctas, plan->threads, smem, st>>>(psi, lam, plan->n_bits, batch, pd, T->adj_ops, bmat,
                                                      plan->bmat_stride, T->perm_pool, want_grad ? gacc : nullptr,
                                                      plan->grad_stride);
  }
  JQ_CUDA(cudaGetLastError());
  if (grad_init) JQ_CUDA(cudaMemcpyAsync(grad_init, lam, sizeof(C) * elems * batch, cudaMemcpyDeviceToDevice, st));
  if ((grad_angles || grad_mats)) {
    if ((rc = chain<R>(plan, T, batch, angles, mats, gacc, scratch, grad_angles, grad_mats, st))) return rc;
  }
  return JQ_OK;
}

template <typename R>
int backward_impl(const jq_plan* plan, int batch, const double* angles, const void* mats, const void* init,
                  int init_batched, int out_type, const double* ct, const void* ct_state, double* grad_angles,
                  void* grad_mats, void* grad_init, void* ws, size_t ws_bytes, cudaStream_t st) {
  using C = typename CplxT<R>::T;
  const DeviceTables* T = nullptr;
  int rc = device_tables(plan, &T);
  if (rc) return rc;
  if ((rc = set_smem_attrs<R>())) return rc;
  WsLayout L = layout(plan, batch, 2);
  if (ws_bytes < L.total || !ws) {
    set_error("workspace too small: need " + std::to_string(L.total) + " bytes");
    return JQ_ENOMEM;
  }
  char* w = static_cast<char*>(ws);
  C* bmat = reinterpret_cast<C*>(w + L.bmat);
  double2* scratch = reinterpret_cast<double2*>(w + L.scratch);
  C* lam = reinterpret_cast<C*>(w + L.lam);
  C* work = reinterpret_cast<C*>(w + L.work);
  double2* gacc = reinterpret_cast<double2*>(w + L.gacc);
  const int64_t elems = plan->state_elems;
  const size_t sbytes = align256(sizeof(C) * elems * batch);
  auto ckpt = [&](int64_t i) { return reinterpret_cast<C*>(w + L.ckpt + sbytes * i); };
  auto seg = [&](int64_t i) { return reinterpret_cast<C*>(w + L.seg + sbytes * i); };
  if ((rc = prep<R>(plan, T, batch, angles, mats, bmat, scratch, st))) return rc;
  const bool dm = plan->mode == JQ_DENSITY;
  const int64_t dim = 1LL << plan->n_qubits;
  const bool init_rho = dm && init && (init_batched & JQ_INIT_DENSITY);  // init is a density matrix
  k_init<R><<<grid_for(elems * batch, 256), 256, 0, st>>>(work, elems, batch, static_cast<const C*>(init),
                                                          init_rho ? elems : dim, init_batched & 1,
                                                          dm && init && !init_rho ? 1 : 0);
  JQ_CUDA(cudaGetLastError());
  // The reverse walks the fused forward schedule: checkpoints every S passes,
  // recompute of a segment with the (specialised) forward passes, and one
  // k_tile_bwd per pass that recomputes the states between the pass's
  // blocks inside each tile.
  const Schedule& sch = plan->fwd;
  const TileOp* sops = T->fwd_ops;
  const JitModule* jm = static_cast<const JitModule*>(T->jit);
  const int64_t P = static_cast<int64_t>(sch.passes.size());
  const int64_t S = L.seg_len;
  for (int64_t p = 0; p < P; ++p) {
    if (p % S == 0) JQ_CUDA(cudaMemcpyAsync(ckpt(p / S), work, sizeof(C) * elems * batch, cudaMemcpyDeviceToDevice, st));
    if ((rc = run_passes<R>(plan, sch, sops, T->fwd_steps, T->fwd_rops, T, work, batch, bmat, p, p + 1, st, jm))) return rc;
  }
  // seed
  if (dm) rc = seed_dm<R>(plan, T, batch, out_type, ct, ct_state, lam, st);
  else rc = seed_sv<R>(plan, T, batch, out_type, work, ct, ct_state, lam, st);
  if (rc) return rc;
  const bool want_grad = (grad_angles || grad_mats) && plan->grad_stride > 0;
  if (want_grad) JQ_CUDA(cudaMemsetAsync(gacc, 0, 16 * static_cast<size_t>(plan->grad_stride) * batch, st));
  for (int64_t c = L.n_ckpt - 1; c >= 0; --c) {
    const int64_t p0 = c * S, p1 = std::min(P, p0 + S);
    // states before passes p0..p1-1: seg[j] = state before pass p0 + j
    JQ_CUDA(cudaMemcpyAsync(seg(0), ckpt(c), sizeof(C) * elems * batch, cudaMemcpyDeviceToDevice, st));
    for (int64_t j = 0; j + 1 < p1 - p0; ++j) {
      const size_t pj = static_cast<size_t>(p0 + j);
      if (jm && pj < jm->fn.size() && jm->fn[pj]) {
        // the specialised pass reads seg(j) and writes seg(j + 1): no copy
        if ((rc = jit_launch(*jm, sch, static_cast<int>(pj), plan->n_bits, sm_count(), seg(j), batch, bmat,
                             plan->bmat_stride, static_cast<int>(sizeof(C)), st, seg(j + 1))))
          return rc;
        continue;
      }
      JQ_CUDA(cudaMemcpyAsync(seg(j + 1), seg(j), sizeof(C) * elems * batch, cudaMemcpyDeviceToDevice, st));
      if ((rc = run_passes<R>(plan, sch, sops, T->fwd_steps, T->fwd_rops, T, seg(j + 1), batch, bmat, p0 + j, p0 + j + 1, st, jm))) return rc;
    }
    for (int64_t p = p1 - 1; p >= p0; --p) {
      const PassDesc& pd = sch.passes[p];
      if (pd.op_end == pd.op_begin) continue;
      const int nops = pd.op_end - pd.op_begin;
      // lambda + work tile + snapshot slots, reduction scratch, cotangent
      // staging, bit-deposit table, snapshot tables
      const size_t tile = (static_cast<size_t>(1) << pd.t) * sizeof(C);
      const size_t fixed = 2 * tile + 32 * kRedSlots * sizeof(double) + 32 * sizeof(double) * nops +
                           ((static_cast<size_t>(1) << (pd.t - pd.c)) + 3) / 4 * 16 + 8 * (nops + kMaxBwdSlots);
      const size_t budget = 227 * 1024;
      if (fixed + tile > budget) {
        set_error("jq_backward: tile of " + std::to_string(pd.t) + " bits does not fit the reverse pass");
        return JQ_EUNSUPPORTED;
      }
      const int nslot = static_cast<int>(std::min<size_t>({static_cast<size_t>(nops), static_cast<size_t>(kMaxBwdSlots),
                                                           (budget - fixed) / tile}));
      const size_t smem = fixed + static_cast<size_t>(nslot) * tile;
      const int64_t ntiles = (1LL << (plan->n_bits - pd.t)) * batch;
      if (jm && jm->has_backward && jm->bfn[p]) {
        // the pass specialised for this plan (NVRTC)
        if ((rc = jit_launch_bwd(*jm, sch, static_cast<int>(p), plan->n_bits, sm_count(), seg(p - p0), lam, batch,
                                 bmat, plan->bmat_stride, want_grad ? reinterpret_cast<double*>(gacc) : nullptr,
                                 plan->grad_stride, static_cast<int>(sizeof(C)), st)))
          return rc;
        continue;
      }
      const int ctas = ctas_for(k_tile_bwd<R>, plan->threads, smem, ntiles);
      k_tile_bwd<R><<<ctas, plan->threads, smem, st>>>(seg(p - p0), lam, plan->n_bits, batch, pd, sops, bmat,
                                                        plan->bmat_stride, T->perm_pool, want_grad ? gacc : nullptr,
                                                        plan->grad_stride, nslot);
    }
    JQ_CUDA(cudaGetLastError());
  }
  if (grad_init) {
    if (init_rho) {
      // the cotangent of an initial density matrix is lambda itself
      JQ_CUDA(cudaMemcpyAsync(grad_init, lam, sizeof(C) * elems * batch, cudaMemcpyDeviceToDevice, st));
    } else if (dm) {
      if (!init) {
        set_error("grad_init requested without an initial state");
        return JQ_EINVAL;
      }
      k_grad_init_dm<R><<<grid_for(dim * batch, 256), 256, 0, st>>>(lam, static_cast<const C*>(init), init_batched & 1,
                                                                     static_cast<C*>(grad_init), dim, batch);
      JQ_CUDA(cudaGetLastError());
    } else {
      JQ_CUDA(cudaMemcpyAsync(grad_init, lam, sizeof(C) * elems * batch, cudaMemcpyDeviceToDevice, st));
    }
  }
  if (grad_angles || grad_mats) {
    if ((rc = chain<R>(plan, T, batch, angles, mats, gacc, scratch, grad_angles, grad_mats, st))) return rc;
  }
  return JQ_OK;
}

#include "batch.cuh"

size_t sample_ws_bytes(int batch, int64_t dim) {
  const int64_t ntiles = (dim + 1023) / 1024;
  return static_cast<size_t>(batch) * static_cast<size_t>(dim + ntiles) * sizeof(double);
}

#include "sample.cuh"

jq_batch_config batch_default_config(int dtype) {
  jq_batch_config c;
  c.warp_max_qubits = dtype == JQ_C64 ? 9 : 8;
  c.cta_max_qubits = dtype == JQ_C64 ? 13 : 12;
  c.warp_threads = 256;
  c.cta_threads = 512;
  c.cluster_bits = 3;
  return c;
}

bool batch_config_ok(const jq_batch_config& c) {
  return c.warp_max_qubits >= 0 && c.warp_max_qubits <= 12 && c.cta_max_qubits >= 0 && c.cta_max_qubits <= 14 &&
         c.warp_threads >= 32 && c.warp_threads <= 512 && (c.warp_threads % 32) == 0 && c.cta_threads >= 64 &&
         c.cta_threads <= 512 && (c.cta_threads % 32) == 0 && c.cluster_bits >= 0 && c.cluster_bits <= 3;
}

std::vector<jq_batch_config> batch_candidates(const jq_batch* b) {
  std::vector<jq_batch_config> out;
  const bool c64 = b->dtype == JQ_C64;
  const int wmax[] = {5, 7, 8, 9, 10};
  const int cmax_c64[] = {12, 13};
  const int cmax_c128[] = {11, 12};
  for (int wm : wmax) {
    if (!c64 && wm > 9) continue;
    for (int cm : (c64 ? cmax_c64 : cmax_c128))
      for (int wt : {128, 256})
        for (int ct : {256, 512}) {
          jq_batch_config c{wm, cm, wt, ct, 3};
          const int elem = c64 ? 8 : 16;
          if (batch_smem(wm, wt / 32, elem, 0) > 227 * 1024) continue;
          out.push_back(c);
        }
  }
  return out;
}

template <typename R>
int batch_run_graph(jq_batch* b, const double* angles, const double* ct, double* expval, double* grad, void* ws,
                    cudaStream_t st) {
  if (std::getenv("JQ_BATCH_NO_GRAPH")) {
    // the same launches without the CUDA graph (debugging, timing breakdowns)
    if (int rc = set_smem_attrs<R>()) return rc;
    return batch_enqueue<R>(b, angles, ct, expval, grad, static_cast<char*>(ws), st);
  }
  const void* key[7] = {angles, ct, expval, grad, ws, st, nullptr};
  bool same = b->graph != nullptr;
  for (int i = 0; i < 6 && same; ++i) same = key[i] == b->graph_key[i];
  if (!same) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    // everything that allocates or uploads happens before the capture
    if (int rc = set_smem_attrs<R>()) return rc;
    for (const auto& tg : b->tiles) {
      const DeviceTables* T = nullptr;
      if (int rc = device_tables(b->plans[tg.plan], &T)) return rc;
    }
    JQ_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    const int rc = batch_enqueue<R>(b, angles, ct, expval, grad, static_cast<char*>(ws), b->cap);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(b->cap, &g);
    if (rc || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      if (!rc) set_error(std::string("graph capture of the batch failed: ") + cudaGetErrorString(ce));
      return rc ? rc : JQ_ECUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      b->graph = nullptr;
      set_error(std::string("graph instantiation of the batch failed: ") + cudaGetErrorString(ie));
      return JQ_ECUDA;
    }
    for (int i = 0; i < 6; ++i) b->graph_key[i] = key[i];
  }
  JQ_CUDA(cudaGraphLaunch(b->graph, st));
  return JQ_OK;
}

}  // namespace
}  // namespace jq

// ===========================================================================
// C ABI
// ===========================================================================
using namespace jq;

extern "C" {

int jq_plan_build(const jq_op* ops, int n_ops, const jq_obs* obs, int n_obs, int n_qubits, int mode, int dtype,
                  const jq_tune* tune, jq_plan** out) {
  try {
    return build_plan(ops, n_ops, obs, n_obs, n_qubits, mode, dtype, tune, out);
  } catch (const std::exception& e) {
    set_error(std::string("jq_plan_build: ") + e.what());
    return JQ_EINVAL;
  }
}

int jq_plan_free(jq_plan* plan) {
  if (!plan) return JQ_OK;
  int cur = -1;
  cudaGetDevice(&cur);
  for (DeviceTables& t : plan->dev) {
    if (t.device >= 0) cudaSetDevice(t.device);
    cudaFree(t.ops); cudaFree(t.prims); cudaFree(t.blocks); cudaFree(t.fwd_ops); cudaFree(t.adj_ops);
    cudaFree(t.bwd_ops); cudaFree(t.fwd_steps); cudaFree(t.fwd_rops); cudaFree(t.bwd_steps); cudaFree(t.bwd_rops);
    cudaFree(t.const_pool);
    if (t.jit) {
      jit_free(static_cast<JitModule*>(t.jit));
      delete static_cast<JitModule*>(t.jit);
    } cudaFree(t.perm_pool); cudaFree(t.obs_pool); cudaFree(t.obs_desc);
  }
  if (cur >= 0 && !plan->dev.empty()) cudaSetDevice(cur);
  delete plan;
  return JQ_OK;
}

int jq_plan_get_info(const jq_plan* plan, jq_plan_info* info) {
  if (!plan || !info) { set_error("jq_plan_get_info: NULL argument"); return JQ_EINVAL; }
  std::memset(info, 0, sizeof(*info));
  info->n_qubits = plan->n_qubits;
  info->n_bits = plan->n_bits;
  info->mode = plan->mode;
  info->dtype = plan->dtype;
  info->n_ops = static_cast<int32_t>(plan->ops.size());
  info->n_blocks = static_cast<int32_t>(plan->blocks.size());
  info->n_passes_fwd = static_cast<int32_t>(plan->fwd.passes.size());
  info->n_passes_adj = static_cast<int32_t>(plan->adj.passes.size());
  info->n_tile_ops_fwd = static_cast<int32_t>(plan->fwd.ops.size());
  info->tile_bits_fwd = plan->fwd.t;
  info->tile_bits_adj = plan->adj.t;
  info->n_angles = plan->n_angles;
  info->n_mats = plan->n_mats;
  info->n_obs = static_cast<int32_t>(plan->obs.size());
  info->unitary = plan->unitary ? 1 : 0;
  info->state_elems = plan->state_elems;
  for (const Step& st : plan->fwd.steps) {
    if (st.kind == 0) ++info->n_stages_fwd;
    else ++info->n_smem_ops_fwd;
  }
  return JQ_OK;
}

int jq_plan_block_passes(const jq_plan* plan, int which, int32_t* block_pass, int32_t* block_wires, int n) {
  if (!plan || !block_pass || which < 0 || which > 2) { set_error("jq_plan_block_passes: bad argument"); return JQ_EINVAL; }
  if (n < static_cast<int>(plan->blocks.size())) { set_error("jq_plan_block_passes: array too short"); return JQ_EINVAL; }
  const Schedule& s = which == 0 ? plan->fwd : which == 1 ? plan->adj : plan->bwd;
  for (int b = 0; b < n; ++b) block_pass[b] = -1;
  for (size_t p = 0; p < s.passes.size(); ++p)
    for (int o = s.passes[p].op_begin; o < s.passes[p].op_end; ++o) block_pass[s.ops[o].block] = static_cast<int32_t>(p);
  if (block_wires) {
    for (size_t b = 0; b < plan->block_wires.size(); ++b)
      for (int j = 0; j < kMaxBlockWires; ++j) block_wires[b * kMaxBlockWires + j] = plan->block_wires[b][j];
  }
  return JQ_OK;
}

size_t jq_plan_jit_source(const jq_plan* plan, char* buf, size_t n) {
  if (!plan) return 0;
  const std::string src = jit_source(plan, plan->fwd);
  if (buf && n > 0) {
    const size_t k = std::min(n - 1, src.size());
    std::memcpy(buf, src.data(), k);
    buf[k] = '\0';
  }
  return src.size();
}

size_t jq_workspace_bytes(const jq_plan* plan, int batch, int out_type, int with_grad) {
  (void)out_type;
  if (!plan || batch < 1) return 0;
  int mode = 0;
  if (with_grad == 1) mode = 1;       // jq_adjoint
  else if (with_grad == 2) mode = 2;  // jq_backward
  return layout(plan, batch, mode).total;
}

// A plan that absorbed trailing blocks into its Z strings (jq_tune.expval_only)
// is run for expectation values only.
static int check_expval_only(const jq_plan* plan, int out_type, const char* who) {
  if (plan->absorbed > 0 && out_type != JQ_OUT_EXPVAL) {
    set_error(std::string(who) + ": the plan was built with jq_tune.expval_only and absorbed " +
              std::to_string(plan->absorbed) + " trailing blocks into its observables; it measures "
              "expectation values only");
    return JQ_EINVAL;
  }
  return JQ_OK;
}

static int check_common(const jq_plan* plan, int batch, const double* angles, const void* mats) {
  if (!plan) { set_error("NULL plan"); return JQ_EINVAL; }
  if (batch < 1) { set_error("batch must be >= 1"); return JQ_EINVAL; }
  if (plan->n_angles > 0 && !angles) { set_error("plan needs angles but none given"); return JQ_EINVAL; }
  if (plan->n_mats > 0 && !mats) { set_error("plan needs matrices but none given"); return JQ_EINVAL; }
  return JQ_OK;
}

int jq_forward(const jq_plan* plan, int batch, const double* angles, const void* mats, const void* init,
               int init_batched, int out_type, void* state, void* out, void* workspace, size_t workspace_bytes,
               void* stream) {
  int rc = check_common(plan, batch, angles, mats);
  if (rc) return rc;
  if ((rc = check_expval_only(plan, out_type, "jq_forward"))) return rc;
  if (!state) { set_error("jq_forward: state buffer is NULL"); return JQ_EINVAL; }
  if (out_type != JQ_OUT_STATE && !(out_type == JQ_OUT_DENSITY && plan->mode == JQ_DENSITY) && !out &&
      !(out_type == JQ_OUT_EXPVAL && plan->obs.empty())) {
    set_error("jq_forward: out buffer is NULL");
    return JQ_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (plan->dtype == JQ_C64)
    return forward_impl<float>(plan, batch, angles, mats, init, init_batched, out_type, state, out, workspace,
                               workspace_bytes, st);
  return forward_impl<double>(plan, batch, angles, mats, init, init_batched, out_type, state, out, workspace,
                              workspace_bytes, st);
}

int jq_sweep(const jq_plan* plan, int batch, const double* angles, const void* mats, void* state, void* workspace,
             size_t workspace_bytes, void* stream) {
  int rc = check_common(plan, batch, angles, mats);
  if (rc) return rc;
  if (!state) { set_error("jq_sweep: state is NULL"); return JQ_EINVAL; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (plan->dtype == JQ_C64) return sweep_impl<float>(plan, batch, angles, mats, state, workspace, workspace_bytes, st);
  return sweep_impl<double>(plan, batch, angles, mats, state, workspace, workspace_bytes, st);
}

int jq_adjoint(const jq_plan* plan, int batch, const double* angles, const void* mats, const void* state,
               int out_type, const double* ct, const void* ct_state, double* grad_angles, void* grad_mats,
               void* grad_init, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_common(plan, batch, angles, mats);
  if (rc) return rc;
  if ((rc = check_expval_only(plan, out_type, "jq_adjoint"))) return rc;
  if (!state) { set_error("jq_adjoint: state is NULL"); return JQ_EINVAL; }
  if (out_type == JQ_OUT_EXPVAL ? (!ct && !plan->obs.empty()) : !ct_state) {
    set_error("jq_adjoint: missing cotangent");
    return JQ_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (plan->dtype == JQ_C64)
    return adjoint_impl<float>(plan, batch, angles, mats, state, out_type, ct, ct_state, grad_angles, grad_mats,
                               grad_init, workspace, workspace_bytes, st);
  return adjoint_impl<double>(plan, batch, angles, mats, state, out_type, ct, ct_state, grad_angles, grad_mats,
                              grad_init, workspace, workspace_bytes, st);
}

int jq_backward(const jq_plan* plan, int batch, const double* angles, const void* mats, const void* init,
                int init_batched, int out_type, const double* ct, const void* ct_state, double* grad_angles,
                void* grad_mats, void* grad_init, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_common(plan, batch, angles, mats);
  if (rc) return rc;
  if ((rc = check_expval_only(plan, out_type, "jq_backward"))) return rc;
  if (out_type == JQ_OUT_EXPVAL ? (!ct && !plan->obs.empty()) : !ct_state) {
    set_error("jq_backward: missing cotangent");
    return JQ_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (plan->dtype == JQ_C64)
    return backward_impl<float>(plan, batch, angles, mats, init, init_batched, out_type, ct, ct_state, grad_angles,
                                grad_mats, grad_init, workspace, workspace_bytes, st);
  return backward_impl<double>(plan, batch, angles, mats, init, init_batched, out_type, ct, ct_state, grad_angles,
                               grad_mats, grad_init, workspace, workspace_bytes, st);
}

}  // extern "C"

// Workspace of jq_forward_noalloc: a file-scope device array, so that entry
// point performs no allocation.  Host code cannot use the symbol as a device
// address; its address is resolved per device with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_ws[JQ_STATIC_WS_BYTES];

namespace {
std::mutex g_noalloc_mu;
std::vector<std::pair<int, void*>> g_noalloc_ptr;  // (device, address of g_noalloc_ws)
}  // namespace

extern "C" {

int jq_forward_noalloc(const jq_plan* plan, int batch, const double* angles, const void* mats, const void* init,
                       int init_batched, int out_type, void* state, void* out, void* stream) {
  int rc = check_common(plan, batch, angles, mats);
  if (rc) return rc;
  if ((rc = check_expval_only(plan, out_type, "jq_forward_noalloc"))) return rc;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    set_error("jq_forward_noalloc: no current CUDA device");
    return JQ_ECUDA;
  }
  bool resident = false;
  {
    std::lock_guard<std::mutex> lock(g_upload_mu);  // device_tables() appends under this lock
    for (const DeviceTables& t : plan->dev) resident = resident || t.device == dev;
  }
  if (!resident) {
    set_error("jq_forward_noalloc: the plan is not resident on this device; run jq_forward (or another "
              "execution entry point) with it once on this device first");
    return JQ_EINVAL;
  }
  const size_t need = layout(plan, batch, 0).total;
  if (need > JQ_STATIC_WS_BYTES) {
    set_error("jq_forward_noalloc: the plan needs " + std::to_string(need) + " workspace bytes for batch " +
              std::to_string(batch) + ", above the static limit of " + std::to_string(JQ_STATIC_WS_BYTES) +
              " bytes; use jq_forward with a caller-provided workspace");
    return JQ_ENOMEM;
  }
  void* ws = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    for (const auto& e : g_noalloc_ptr)
      if (e.first == dev) ws = e.second;
    if (!ws) {
      // the address is resolved once per device, and not inside a stream
      // capture (the runtime call is not part of what a capture records)
      cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cap) != cudaSuccess ||
          cap != cudaStreamCaptureStatusNone) {
        set_error("jq_forward_noalloc: the first call on a device resolves the static workspace address and "
                  "must not run inside a stream capture; call it once on this device outside the capture first");
        return JQ_EINVAL;
      }
      const cudaError_t e = cudaGetSymbolAddress(&ws, g_noalloc_ws);
      if (e != cudaSuccess || !ws) {
        set_error(std::string("jq_forward_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        return JQ_ECUDA;
      }
      g_noalloc_ptr.emplace_back(dev, ws);
    }
  }
  return jq_forward(plan, batch, angles, mats, init, init_batched, out_type, state, out, ws, JQ_STATIC_WS_BYTES,
                    stream);
}

// ---------------------------------------------------------------------------
// shot sampling
// ---------------------------------------------------------------------------
size_t jq_sample_workspace_bytes(int batch, int64_t dim) {
  if (batch <= 0 || dim <= 0) return 0;
  return sample_ws_bytes(batch, dim);
}

int jq_sample_shots(const double* probs, int batch, int64_t dim, int64_t shots, uint64_t seed, uint32_t* counts,
                    void* workspace, size_t workspace_bytes, void* stream) {
  if (!probs || !counts || batch <= 0 || dim <= 0 || shots < 0 || dim > (int64_t(1) << 34) ||
      shots > 0xFFFFFFFFll) {
    set_error("jq_sample_shots: need probs and counts, batch > 0, 0 < dim <= 2^34, 0 <= shots < 2^32");
    return JQ_EINVAL;
  }
  return sample_impl(probs, batch, dim, shots, seed, workspace, workspace_bytes, counts,
                     static_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------
// batched uneven instances
// ---------------------------------------------------------------------------
int jq_batch_build(jq_plan* const* plans, int n_plans, const int32_t* plan_of, int n_inst,
                   const jq_batch_config* cfg, jq_batch** out) {
  if (!out || !plans || n_plans <= 0 || n_inst <= 0 || !plan_of) {
    set_error("jq_batch_build: need plans, plan_of and n_inst > 0");
    return JQ_EINVAL;
  }
  *out = nullptr;
  std::unique_ptr<jq_batch> b(new jq_batch());
  b->dtype = plans[0]->dtype;
  cudaGetDevice(&b->device);
  b->sm_count = sm_count();
  for (int p = 0; p < n_plans; ++p) {
    const jq_plan* pl = plans[p];
    if (!pl || pl->mode != JQ_STATEVECTOR || !pl->unitary || pl->n_mats > 0 || pl->dtype != b->dtype) {
      set_error("jq_batch_build: plan " + std::to_string(p) +
                " is not a unitary statevector plan without matrix arguments of the batch dtype");
      return JQ_EINVAL;
    }
    b->plans.push_back(pl);
    b->n_of_plan.push_back(pl->n_qubits);
    BPlan bp;
    std::memset(&bp, 0, sizeof(bp));
    bp.n = pl->n_qubits;
    bp.nblocks = static_cast<int32_t>(pl->blocks.size());
    bp.blk_off = static_cast<int32_t>(b->dblk.size());
    bp.n_angles = pl->n_angles;
    bp.obs_off = static_cast<int32_t>(b->obs.size());
    bp.n_obs = static_cast<int32_t>(pl->obs.size());
    bp.bmat_stride = static_cast<int32_t>(pl->bmat_stride);
    bp.grad_stride = static_cast<int32_t>(pl->grad_stride);
    const int32_t prim_base = static_cast<int32_t>(b->prims.size());
    const int32_t op_base = static_cast<int32_t>(b->ops.size());
    const int32_t cpool_base = static_cast<int32_t>(b->cpool.size() / 2);
    for (size_t i = 0; i < pl->blocks.size(); ++i) {
      DevBlock blk = pl->blocks[i];
      BBlock bb;
      std::memset(&bb, 0, sizeof(bb));
      bb.kind = blk.kind;
      bb.nt = blk.k - blk.n_ctrl;
      bb.grad_off = blk.grad_off;
      bb.mat_off = blk.mat_off;
      const auto& wires = pl->block_wires[i];
      for (int c = 0; c < blk.n_ctrl; ++c) bb.cmask |= 1u << (pl->n_bits - 1 - wires[c]);
      bb.tb0 = bb.nt >= 1 ? pl->n_bits - 1 - wires[blk.n_ctrl] : 0;
      bb.tb1 = bb.nt >= 2 ? pl->n_bits - 1 - wires[blk.n_ctrl + 1] : 0;
      if (blk.kind == BK_PERM && bb.nt >= 1 && bb.nt <= 2)
        for (int r = 0; r < (1 << bb.nt); ++r) bb.perm |= (pl->perm_pool[blk.perm_off + r] & 3) << (2 * r);
      b->bblk.push_back(bb);
      blk.prim_begin += prim_base;
      blk.prim_end += prim_base;
      b->dblk.push_back(blk);
    }
    for (DevPrim pr : pl->prims) {
      if (pr.op >= 0) pr.op += op_base;
      if (pr.form == PF_CONST) pr.const_off += cpool_base;
      b->prims.push_back(pr);
    }
    for (const DevOp& o : pl->ops) b->ops.push_back(o);
    b->cpool.insert(b->cpool.end(), pl->const_pool.begin(), pl->const_pool.end());
    // pair consecutive uncontrolled one-target dense blocks on different bits
    // (greedy from the front; a paired block is never the first of another pair)
    for (int i = 0; i + 1 < bp.nblocks; ++i) {
      BBlock& x = b->bblk[bp.blk_off + i];
      const BBlock& y = b->bblk[bp.blk_off + i + 1];
      auto single = [](const BBlock& q) { return q.kind == BK_DENSE && q.nt == 1 && q.cmask == 0; };
      if (single(x) && single(y) && x.tb0 != y.tb0) {
        x.pair = 1;
        ++i;
      }
    }
    for (const DevObs& o : pl->obs) b->obs.push_back(o);
    b->bplans.push_back(bp);
  }
  int64_t ang = 0, outs = 0;
  for (int i = 0; i < n_inst; ++i) {
    const int p = plan_of[i];
    if (p < 0 || p >= n_plans) {
      set_error("jq_batch_build: plan_of[" + std::to_string(i) + "] out of range");
      return JQ_EINVAL;
    }
    BInst bi;
    std::memset(&bi, 0, sizeof(bi));
    bi.plan = p;
    bi.angle_off = ang;
    bi.out_off = outs;
    ang += b->plans[p]->n_angles;
    outs += static_cast<int64_t>(b->plans[p]->obs.size());
    b->inst.push_back(bi);
  }
  b->n_inst = n_inst;
  b->n_angles_total = ang;
  b->n_obs_total = outs;
  b->cfg = cfg ? *cfg : batch_default_config(b->dtype);
  if (!batch_config_ok(b->cfg)) {
    set_error("jq_batch_build: configuration out of range");
    return JQ_EINVAL;
  }
  auto up = [](const void* src, size_t bytes, void** dst) -> int {
    if (bytes == 0) bytes = 16;
    if (cudaMalloc(dst, bytes) != cudaSuccess) return JQ_ECUDA;
    if (src && cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return JQ_ECUDA;
    return JQ_OK;
  };
  if (b->cpool.empty()) b->cpool.assign(2, 0.0);
  if (up(b->bplans.data(), b->bplans.size() * sizeof(BPlan), &b->d_plans) ||
      up(b->inst.data(), b->inst.size() * sizeof(BInst), &b->d_inst) ||
      up(b->bblk.data(), b->bblk.size() * sizeof(BBlock), &b->d_bblk) ||
      up(b->dblk.data(), b->dblk.size() * sizeof(DevBlock), &b->d_dblk) ||
      up(b->prims.data(), b->prims.size() * sizeof(DevPrim), &b->d_prims) ||
      up(b->ops.data(), b->ops.size() * sizeof(DevOp), &b->d_ops) ||
      up(b->cpool.data(), b->cpool.size() * sizeof(double), &b->d_cpool) ||
      up(b->obs.data(), b->obs.size() * sizeof(DevObs), &b->d_obs)) {
    set_error("jq_batch_build: upload of the batch tables failed");
    return JQ_ECUDA;
  }
  for (int i = 0; i < 5; ++i)
    if (cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking) != cudaSuccess) return JQ_ECUDA;
  if (cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess) return JQ_ECUDA;
  for (int i = 0; i < 6; ++i)
    if (cudaEventCreateWithFlags(&b->ev[i], cudaEventDisableTiming) != cudaSuccess) return JQ_ECUDA;
  if (int rc = batch_classify(b.get())) return rc;
  *out = b.release();
  return JQ_OK;
}

int jq_batch_free(jq_batch* b) {
  if (!b) return JQ_OK;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  void* bufs[] = {b->d_plans, b->d_inst, b->d_bblk, b->d_dblk, b->d_prims, b->d_ops, b->d_cpool, b->d_obs,
                  b->d_order, b->d_tile_off, b->d_rstg, b->d_rop};
  for (void* p : bufs)
    if (p) cudaFree(p);
  for (int i = 0; i < 5; ++i)
    if (b->side[i]) cudaStreamDestroy(b->side[i]);
  if (b->cap) cudaStreamDestroy(b->cap);
  for (int i = 0; i < 6; ++i)
    if (b->ev[i]) cudaEventDestroy(b->ev[i]);
  delete b;
  return JQ_OK;
}

int jq_batch_info(const jq_batch* b, int64_t* n_angles, int64_t* n_obs, int32_t* n_class, jq_batch_config* cfg) {
  if (!b) {
    set_error("jq_batch_info: NULL batch");
    return JQ_EINVAL;
  }
  if (n_angles) *n_angles = b->n_angles_total;
  if (n_obs) *n_obs = b->n_obs_total;
  if (n_class) {
    n_class[0] = static_cast<int32_t>(b->order_warp.size());
    n_class[1] = static_cast<int32_t>(b->order_cta.size());
    int32_t t = 0;
    for (const auto& tg : b->tiles) t += static_cast<int32_t>(tg.members.size());
    n_class[2] = t;
    n_class[3] = static_cast<int32_t>(b->order_cl[0].size() + b->order_cl[1].size() + b->order_cl[2].size());
  }
  if (cfg) *cfg = b->cfg;
  return JQ_OK;
}

size_t jq_batch_workspace_bytes(const jq_batch* cb) {
  if (!cb) return 0;
  jq_batch* b = const_cast<jq_batch*>(cb);
  size_t need = batch_ws_for(b, b->cfg);
  for (const jq_batch_config& c : batch_candidates(b)) need = std::max(need, batch_ws_for(b, c));
  return need;
}

int jq_batch_set_config(jq_batch* b, const jq_batch_config* cfg) {
  if (!b || !cfg || !batch_config_ok(*cfg)) {
    set_error("jq_batch_set_config: configuration out of range");
    return JQ_EINVAL;
  }
  const jq_batch_config keep = b->cfg;
  b->cfg = *cfg;
  if (int rc = batch_classify(b)) {
    b->cfg = keep;
    batch_classify(b);
    return rc;
  }
  return JQ_OK;
}

int jq_batch_run(jq_batch* b, const double* angles, const double* ct, double* expval, double* grad, void* ws,
                 size_t ws_bytes, void* stream) {
  if (!b || (!angles && b->n_angles_total > 0) || !expval || (!grad && b->n_angles_total > 0)) {
    set_error("jq_batch_run: need a batch, angles, expval and grad buffers");
    return JQ_EINVAL;
  }
  if (ws_bytes < b->ws_total || !ws) {
    set_error("workspace too small: need " + std::to_string(b->ws_total) + " bytes");
    return JQ_ENOMEM;
  }
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != b->device) {
    set_error("jq_batch_run: the batch was built on device " + std::to_string(b->device));
    return JQ_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (b->dtype == JQ_C64) return batch_run_graph<float>(b, angles, ct, expval, grad, ws, st);
  return batch_run_graph<double>(b, angles, ct, expval, grad, ws, st);
}

int jq_batch_autotune(jq_batch* b, const double* angles, double* expval, double* grad, void* ws, size_t ws_bytes,
                      void* stream, jq_batch_config* chosen) {
  if (!b) {
    set_error("jq_batch_autotune: NULL batch");
    return JQ_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaEvent_t e0, e1;
  JQ_CUDA(cudaEventCreate(&e0));
  JQ_CUDA(cudaEventCreate(&e1));
  const jq_batch_config start = b->cfg;
  jq_batch_config best = start;
  float best_ms = -1.0f;
  std::vector<jq_batch_config> cands = batch_candidates(b);
  cands.insert(cands.begin(), start);
  int rc = JQ_OK;
  for (const jq_batch_config& c : cands) {
    if (batch_ws_for(b, c) > ws_bytes) continue;
    if ((rc = jq_batch_set_config(b, &c))) continue;
    // one warm-up run (captures the graph), then one timed replay
    if ((rc = jq_batch_run(b, angles, nullptr, expval, grad, ws, ws_bytes, stream))) continue;
    cudaEventRecord(e0, st);
    if ((rc = jq_batch_run(b, angles, nullptr, expval, grad, ws, ws_bytes, stream))) continue;
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = JQ_ECUDA;
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (best_ms < 0.0f || ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best_ms < 0.0f) {
    if (!rc) set_error("jq_batch_autotune: no candidate fits the workspace");
    jq_batch_set_config(b, &start);
    return rc ? rc : JQ_ENOMEM;
  }
  if ((rc = jq_batch_set_config(b, &best))) return rc;
  if (chosen) *chosen = best;
  return JQ_OK;
}

const char* jq_last_error(void) { return g_last_error.c_str(); }

const char* jq_version(void) { return "jqsim 0.1.0 (sm_100a)"; }

}  // extern "C"
