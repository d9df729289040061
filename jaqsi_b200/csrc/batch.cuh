// Batched uneven instances: many independent circuits (different qubit
// counts, depths and parameters) run forward + adjoint in one persistent
// launch, captured with the rest of the batch in one CUDA graph.
//
// Instance classes (chosen per plan by qubit count; the thresholds are the
// autotuned configuration):
//   warp   n <= warp_max: one warp runs one instance; psi and lambda live in
//          that warp's slice of shared memory (CTA = several instances)
//   cta    n <= cta_max:  one CTA runs one instance, psi and lambda in its
//          shared memory
//   tile   larger:        instances of the same plan run as one batched
//          jq_forward + jq_adjoint (tile passes through HBM / L2)
// The warp and cta kernels take instances from a global work counter in
// descending cost order (largest first), so the persistent grid balances
// uneven instances by itself.
//
// Included by jqsim.cu inside namespace jq::(anonymous).

// One block applied to the whole in-shared-memory state.
struct BBlock {
  int32_t kind;      // BK_DENSE / BK_DIAG / BK_PERM
  int32_t nt;        // target bits: 1 or 2
  uint32_t cmask;    // flat bits of the controls (all must be 1)
  int32_t tb0, tb1;  // flat bit of target 0 (matrix MSB) and of target 1
  int32_t perm;      // BK_PERM: output row r takes input row (perm >> 2r) & 3
  int32_t grad_off;  // complex128 offset of the block cotangent, -1 if none
  int32_t mat_off;   // run-dtype complex offset of the inner matrix / diagonal
  int32_t pair;      // 1: this block and the next are uncontrolled one-target dense
                     // blocks on different bits, applied in one sweep (greedy,
                     // non-overlapping, so the reverse walk finds the same pairs)
};

struct BPlan {
  int32_t n, nblocks, blk_off;     // BBlock and DevBlock rows [blk_off, blk_off + nblocks)
  int32_t n_angles, obs_off, n_obs;
  int32_t bmat_stride, grad_stride;
  int32_t cls;                     // 0 warp, 1 cta, 2 tile, 3 cluster
  int32_t stg_off, n_stg;          // register-stage program (cluster class): RStage rows
};

// Register-stage program of a cluster-class instance (complex64, 16
// amplitudes a thread).  A stage loads, for every thread, the 16 amplitudes
// whose 4 register bits vary and whose other index bits are the thread's
// index T (over the whole cluster) deposited at tpos[], applies its ops in
// registers and stores them back; one shared-memory sweep per stage instead
// of one per block.
enum { RO_DENSE1 = 0, RO_DENSE2 = 1, RO_DIAG = 2, RO_PERM1 = 3, RO_PERM2 = 4 };

struct alignas(16) RStage {
  int32_t op_begin, op_end;  // RPacked rows
  int32_t dist;              // a register bit is a rank bit: the stage reads other CTAs' slices
  uint32_t rpos;             // byte q: flat index bit of register bit q
  uint32_t tpos[5];          // byte i: flat index bit of thread-index bit i (n - 4 used)
  int32_t pad[3];
};

// One op of a stage as the device reads it (16 bytes, one vector load):
// w0 = kind | nt << 3 | q0 << 5 | q1 << 7 | crm << 9 | perm << 13 | iperm << 21
struct alignas(16) RPacked {
  uint32_t w0, ctm;
  int32_t mat_off, grad_off;
};

// Decoded op.
struct ROp {
  int32_t kind, nt;
  int32_t q0, q1;            // register bits of target 0 (matrix MSB) and target 1
  uint32_t crm;              // controls on register bits (mask over register bits)
  uint32_t ctm;              // controls on thread bits (mask over flat index bits)
  int32_t mat_off, grad_off;
  int32_t perm, iperm;       // RO_PERM*: output row r takes input row (perm >> 2r) & 3; iperm inverts it
};

__host__ __device__ inline RPacked rs_pack(const ROp& r) {
  RPacked p;
  p.w0 = static_cast<uint32_t>(r.kind) | static_cast<uint32_t>(r.nt) << 3 | static_cast<uint32_t>(r.q0) << 5 |
         static_cast<uint32_t>(r.q1) << 7 | r.crm << 9 | static_cast<uint32_t>(r.perm & 255) << 13 |
         static_cast<uint32_t>(r.iperm & 255) << 21;
  p.ctm = r.ctm;
  p.mat_off = r.mat_off;
  p.grad_off = r.grad_off;
  return p;
}

__host__ __device__ inline ROp rs_unpack(RPacked p) {
  ROp r;
  r.kind = static_cast<int32_t>(p.w0 & 7u);
  r.nt = static_cast<int32_t>((p.w0 >> 3) & 3u);
  r.q0 = static_cast<int32_t>((p.w0 >> 5) & 3u);
  r.q1 = static_cast<int32_t>((p.w0 >> 7) & 3u);
  r.crm = (p.w0 >> 9) & 15u;
  r.perm = static_cast<int32_t>((p.w0 >> 13) & 255u);
  r.iperm = static_cast<int32_t>((p.w0 >> 21) & 255u);
  r.ctm = p.ctm;
  r.mat_off = p.mat_off;
  r.grad_off = p.grad_off;
  return r;
}

struct BInst {
  int32_t plan;
  int32_t pad;
  int64_t angle_off;  // first angle (and gradient entry) of the instance
  int64_t out_off;    // first expectation value of the instance
};

struct BatchArgs {
  const BPlan* plans;
  const BInst* inst;
  const int32_t* order;  // instances of this class, largest first
  int n_order;
  int nmax;              // largest qubit count of the class (shared memory sizing)
  const BBlock* bblk;
  const DevBlock* dblk;
  const DevPrim* prims;
  const DevOp* ops;
  const double2* cpool;
  const DevObs* obs;
  const double* angles;
  const double* ct;      // per (instance, observable) cotangent; NULL: all ones
  double* expval;
  double* grad;
  double2* gacc_ws;      // per group slot: gacc_slot complex128
  int64_t bmat_slot;     // run-dtype complex of the block matrices per group (shared memory)
  int64_t gacc_slot;
  int* counter;
};

__device__ __forceinline__ int ins0(int g, int q) { return ((g >> q) << (q + 1)) | (g & ((1 << q) - 1)); }

// Group = one warp (WARP) or the whole CTA.
template <bool WARP>
__device__ __forceinline__ void gsync() {
  if (WARP) __syncwarp();
  else __syncthreads();
}

// Sum over the group; the result is returned to every thread of the group.
template <bool WARP>
__device__ __forceinline__ double gsum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (WARP) return v;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < nw; ++w) s += red[w];
  return s;
}

// Warp reduce-scatter of N (power of two, <= 32) per-lane values by recursive
// halving: at the step exchanging with lane ^ O the lanes with bit O set keep
// the upper half.  Afterwards the top log2(N) lane bits index the value a lane
// holds (summed over the lanes that differ only in the low bits).
template <int O, int N, typename F>
struct WarpRS {
  static __device__ __forceinline__ void run(F* v, unsigned lane) {
    if constexpr (N > 1) {
      constexpr int h = N / 2;
      const bool up = (lane & O) != 0;
#pragma unroll
      for (int i = 0; i < h; ++i) {
        const F send = up ? v[i] : v[i + h];
        const F keep = up ? v[i + h] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, O);
      }
      if constexpr (O > 1) WarpRS<O / 2, h, F>::run(v, lane);
    } else {
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], O);
      if constexpr (O > 1) WarpRS<O / 2, 1, F>::run(v, lane);
    }
  }
};

// Gradient partial sums: float for complex64 runs, double for complex128.
template <typename C> struct AccT { using T = double; };
template <> struct AccT<float2> { using T = float; };

// Add the group's partial block cotangent (NV doubles per thread) into dst.
template <bool WARP, int NV>
__device__ __forceinline__ void gacc_add(double (&v)[NV], double* dst) {
  WarpRS<16, NV, double>::run(v, threadIdx.x & 31u);
  constexpr int lg = (NV >= 32) ? 5 : (NV >= 16) ? 4 : (NV >= 8) ? 3 : (NV >= 4) ? 2 : (NV >= 2) ? 1 : 0;
  const unsigned lane = threadIdx.x & 31u;
  if ((lane & ((32u >> lg) - 1u)) == 0) {
    if (WARP) dst[lane >> (5 - lg)] += v[0];
    else atomicAdd(dst + (lane >> (5 - lg)), v[0]);
  }
}

// acc += l * conj(p), in the accumulator type A
template <typename A, typename C>
__device__ __forceinline__ void acc_lconjp(A& re, A& im, C l, C p) {
  re += static_cast<A>(l.x) * static_cast<A>(p.x) + static_cast<A>(l.y) * static_cast<A>(p.y);
  im += static_cast<A>(l.y) * static_cast<A>(p.x) - static_cast<A>(l.x) * static_cast<A>(p.y);
}

template <bool WARP, int NV, typename A>
__device__ __forceinline__ void gacc_add_acc(A (&v)[NV], double* dst) {
  double d[NV];
#pragma unroll
  for (int e = 0; e < NV; ++e) d[e] = static_cast<double>(v[e]);
  gacc_add<WARP, NV>(d, dst);
}

// Forward application of one block to the n-qubit state s.
// gbase: global index bits above the n local ones (a cluster CTA's rank
// bits; 0 for a state held whole); controls and diagonal rows may sit there.
template <typename C>
__device__ void bapply(C* s, int n, const BBlock& B, const C* bm, int lt, int gs, uint32_t gbase = 0) {
  const int dim = 1 << n;
  const C* M = bm + B.mat_off;
  if (B.kind == BK_DIAG) {
    for (int j = lt; j < dim; j += gs) {
      const uint32_t gj = gbase | static_cast<uint32_t>(j);
      if ((gj & B.cmask) != B.cmask) continue;
      const int r = (B.nt == 1) ? ((gj >> B.tb0) & 1) : ((((gj >> B.tb0) & 1) << 1) | ((gj >> B.tb1) & 1));
      s[j] = cmul(M[r], s[j]);
    }
    return;
  }
  if (B.nt == 1) {
    const int q = B.tb0, half = dim >> 1;
    if (B.kind == BK_PERM && !(B.perm & 1)) return;
    const C m0 = M[0], m1 = M[1], m2 = M[2], m3 = M[3];
    // 4 pairs per thread at a time: every load before any store
    for (int g0 = lt; g0 < half; g0 += 4 * gs) {
      C x[4], y[4];
      int i0[4];
      bool ok[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int g = g0 + u * gs;
        i0[u] = ins0(g, q);
        ok[u] = g < half && ((gbase | static_cast<uint32_t>(i0[u])) & B.cmask) == B.cmask;
        if (ok[u]) {
          x[u] = s[i0[u]];
          y[u] = s[i0[u] | (1 << q)];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (!ok[u]) continue;
        if (B.kind == BK_PERM) {
          s[i0[u]] = y[u];
          s[i0[u] | (1 << q)] = x[u];
        } else {
          s[i0[u]] = cfma(m1, y[u], cmul(m0, x[u]));
          s[i0[u] | (1 << q)] = cfma(m3, y[u], cmul(m2, x[u]));
        }
      }
    }
    return;
  }
  const int lo = min(B.tb0, B.tb1), hi = max(B.tb0, B.tb1);
  for (int g = lt; g < (dim >> 2); g += gs) {
    const int i = ins0(ins0(g, lo), hi);
    if (((gbase | static_cast<uint32_t>(i)) & B.cmask) != B.cmask) continue;
    const int id[4] = {i, i | (1 << B.tb1), i | (1 << B.tb0), i | (1 << B.tb0) | (1 << B.tb1)};
    C a[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) a[r] = s[id[r]];
    if (B.kind == BK_PERM) {
#pragma unroll
      for (int r = 0; r < 4; ++r) s[id[r]] = a[(B.perm >> (2 * r)) & 3];
    } else {
#pragma unroll
      for (int r = 0; r < 4; ++r)
        s[id[r]] = cfma(M[4 * r + 3], a[3], cfma(M[4 * r + 2], a[2], cfma(M[4 * r + 1], a[1], cmul(M[4 * r], a[0]))));
    }
  }
}

// Two uncontrolled one-target dense blocks A (bit qa) then B (bit qb) in one
// sweep: each thread takes groups of 4 amplitudes {i, i|b, i|a, i|a|b}.
template <typename C>
__device__ void bapply2(C* s, int n, const BBlock& A, const BBlock& B, const C* bm, int lt, int gs) {
  const int dim = 1 << n, qa = A.tb0, qb = B.tb0;
  const int lo = min(qa, qb), hi = max(qa, qb);
  const C* MA = bm + A.mat_off;
  const C* MB = bm + B.mat_off;
  const C a0 = MA[0], a1 = MA[1], a2 = MA[2], a3 = MA[3];
  const C b0 = MB[0], b1 = MB[1], b2 = MB[2], b3 = MB[3];
  for (int g = lt; g < (dim >> 2); g += gs) {
    const int i = ins0(ins0(g, lo), hi);
    const int ia = i | (1 << qa), ib = i | (1 << qb), iab = ia | (1 << qb);
    C x00 = s[i], x01 = s[ib], x10 = s[ia], x11 = s[iab];
    // A on qa: pairs (x00, x10), (x01, x11)
    C y00 = cfma(a1, x10, cmul(a0, x00)), y10 = cfma(a3, x10, cmul(a2, x00));
    C y01 = cfma(a1, x11, cmul(a0, x01)), y11 = cfma(a3, x11, cmul(a2, x01));
    // B on qb: pairs (y00, y01), (y10, y11)
    s[i] = cfma(b1, y01, cmul(b0, y00));
    s[ib] = cfma(b3, y01, cmul(b2, y00));
    s[ia] = cfma(b1, y11, cmul(b0, y10));
    s[iab] = cfma(b3, y11, cmul(b2, y10));
  }
}

// Reverse of bapply2: un-apply B then A, each with its cotangent.
template <typename C, bool WARP>
__device__ void badjoint2(C* sp, C* sl, int n, const BBlock& A, const BBlock& B, const C* bm, double* ga, int lt,
                          int gs) {
  using Acc = typename AccT<C>::T;
  const int dim = 1 << n, qa = A.tb0, qb = B.tb0;
  const int lo = min(qa, qb), hi = max(qa, qb);
  const C* MA = bm + A.mat_off;
  const C* MB = bm + B.mat_off;
  // G^dagger = [[conj m00, conj m10], [conj m01, conj m11]]
  const C ha00 = cconj(MA[0]), ha01 = cconj(MA[2]), ha10 = cconj(MA[1]), ha11 = cconj(MA[3]);
  const C hb00 = cconj(MB[0]), hb01 = cconj(MB[2]), hb10 = cconj(MB[1]), hb11 = cconj(MB[3]);
  const bool gA = ga && A.grad_off >= 0, gB = ga && B.grad_off >= 0;
  Acc g[16];
#pragma unroll
  for (int e = 0; e < 16; ++e) g[e] = Acc(0);
  for (int gi = lt; gi < (dim >> 2); gi += gs) {
    const int i = ins0(ins0(gi, lo), hi);
    const int ia = i | (1 << qa), ib = i | (1 << qb), iab = ia | (1 << qb);
    C p00 = sp[i], p01 = sp[ib], p10 = sp[ia], p11 = sp[iab];
    C l00 = sl[i], l01 = sl[ib], l10 = sl[ia], l11 = sl[iab];
    // un-apply B on qb: pairs (00, 01), (10, 11)
    {
      const C q00 = cfma(hb01, p01, cmul(hb00, p00)), q01 = cfma(hb11, p01, cmul(hb10, p00));
      const C q10 = cfma(hb01, p11, cmul(hb00, p10)), q11 = cfma(hb11, p11, cmul(hb10, p10));
      acc_lconjp(g[8], g[9], l00, q00);
      acc_lconjp(g[10], g[11], l00, q01);
      acc_lconjp(g[12], g[13], l01, q00);
      acc_lconjp(g[14], g[15], l01, q01);
      acc_lconjp(g[8], g[9], l10, q10);
      acc_lconjp(g[10], g[11], l10, q11);
      acc_lconjp(g[12], g[13], l11, q10);
      acc_lconjp(g[14], g[15], l11, q11);
      const C m00 = cfma(hb01, l01, cmul(hb00, l00)), m01 = cfma(hb11, l01, cmul(hb10, l00));
      const C m10 = cfma(hb01, l11, cmul(hb00, l10)), m11 = cfma(hb11, l11, cmul(hb10, l10));
      p00 = q00; p01 = q01; p10 = q10; p11 = q11;
      l00 = m00; l01 = m01; l10 = m10; l11 = m11;
    }
    // un-apply A on qa: pairs (00, 10), (01, 11)
    {
      const C q00 = cfma(ha01, p10, cmul(ha00, p00)), q10 = cfma(ha11, p10, cmul(ha10, p00));
      const C q01 = cfma(ha01, p11, cmul(ha00, p01)), q11 = cfma(ha11, p11, cmul(ha10, p01));
      acc_lconjp(g[0], g[1], l00, q00);
      acc_lconjp(g[2], g[3], l00, q10);
      acc_lconjp(g[4], g[5], l10, q00);
      acc_lconjp(g[6], g[7], l10, q10);
      acc_lconjp(g[0], g[1], l01, q01);
      acc_lconjp(g[2], g[3], l01, q11);
      acc_lconjp(g[4], g[5], l11, q01);
      acc_lconjp(g[6], g[7], l11, q11);
      sp[i] = q00; sp[ib] = q01; sp[ia] = q10; sp[iab] = q11;
      sl[i] = cfma(ha01, l10, cmul(ha00, l00));
      sl[ia] = cfma(ha11, l10, cmul(ha10, l00));
      sl[ib] = cfma(ha01, l11, cmul(ha00, l01));
      sl[iab] = cfma(ha11, l11, cmul(ha10, l01));
    }
  }
  // g[0..7]: A's cotangent, g[8..15]: B's (every lane takes part in both reductions)
  Acc gav[8], gbv[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    gav[e] = g[e];
    gbv[e] = g[8 + e];
  }
  if (ga && (A.grad_off >= 0 || B.grad_off >= 0)) {
    if (gA) gacc_add_acc<WARP, 8>(gav, ga + 2 * A.grad_off);
    if (gB) gacc_add_acc<WARP, 8>(gbv, ga + 2 * B.grad_off);
  }
}

// Adjoint of one block: psi <- G^dagger psi, cotangent += lam psi^dagger
// (psi after the un-apply), lam <- G^dagger lam.
template <typename C, bool WARP>
__device__ void badjoint(C* sp, C* sl, int n, const BBlock& B, const C* bm, double* ga, int lt, int gs,
                         uint32_t gbase = 0) {
  const int dim = 1 << n;
  const C* M = bm + B.mat_off;
  const bool grad = ga && B.grad_off >= 0;
  double* gdst = grad ? ga + 2 * B.grad_off : nullptr;
  using A = typename AccT<C>::T;
  if (B.kind == BK_DIAG) {
    A g[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) g[e] = A(0);
    for (int j = lt; j < dim; j += gs) {
      const uint32_t gj = gbase | static_cast<uint32_t>(j);
      if ((gj & B.cmask) != B.cmask) continue;
      const int r = (B.nt == 1) ? ((gj >> B.tb0) & 1) : ((((gj >> B.tb0) & 1) << 1) | ((gj >> B.tb1) & 1));
      const C d = cconj(M[r]);
      const C p = cmul(d, sp[j]);
      const C l = sl[j];
      sp[j] = p;
      sl[j] = cmul(d, l);
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (q == r) acc_lconjp(g[2 * q], g[2 * q + 1], l, p);
    }
    if (grad) gacc_add_acc<WARP, 8>(g, gdst);
    return;
  }
  if (B.nt == 1) {
    const int q = B.tb0;
    A g[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) g[e] = A(0);
    for (int gi = lt; gi < (dim >> 1); gi += gs) {
      const int i0 = ins0(gi, q);
      if (((gbase | static_cast<uint32_t>(i0)) & B.cmask) != B.cmask) continue;
      const int i1 = i0 | (1 << q);
      const C x = sp[i0], y = sp[i1], u = sl[i0], w = sl[i1];
      if (B.kind == BK_PERM) {
        if (B.perm & 1) { sp[i0] = y; sp[i1] = x; sl[i0] = w; sl[i1] = u; }
        continue;
      }
      // G^dagger = [[conj m00, conj m10], [conj m01, conj m11]]
      const C h00 = cconj(M[0]), h01 = cconj(M[2]), h10 = cconj(M[1]), h11 = cconj(M[3]);
      const C p0 = cfma(h01, y, cmul(h00, x)), p1 = cfma(h11, y, cmul(h10, x));
      sp[i0] = p0;
      sp[i1] = p1;
      acc_lconjp(g[0], g[1], u, p0);
      acc_lconjp(g[2], g[3], u, p1);
      acc_lconjp(g[4], g[5], w, p0);
      acc_lconjp(g[6], g[7], w, p1);
      sl[i0] = cfma(h01, w, cmul(h00, u));
      sl[i1] = cfma(h11, w, cmul(h10, u));
    }
    if (grad) gacc_add_acc<WARP, 8>(g, gdst);
    return;
  }
  const int lo = min(B.tb0, B.tb1), hi = max(B.tb0, B.tb1);
  A g[32];
#pragma unroll
  for (int e = 0; e < 32; ++e) g[e] = A(0);
  for (int gi = lt; gi < (dim >> 2); gi += gs) {
    const int i = ins0(ins0(gi, lo), hi);
    if (((gbase | static_cast<uint32_t>(i)) & B.cmask) != B.cmask) continue;
    const int id[4] = {i, i | (1 << B.tb1), i | (1 << B.tb0), i | (1 << B.tb0) | (1 << B.tb1)};
    C a[4], b[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) { a[r] = sp[id[r]]; b[r] = sl[id[r]]; }
    if (B.kind == BK_PERM) {
      // inverse: new[p[r]] = old[r]
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        sp[id[(B.perm >> (2 * r)) & 3]] = a[r];
        sl[id[(B.perm >> (2 * r)) & 3]] = b[r];
      }
      continue;
    }
    C p[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      C acc = cmul(cconj(M[r]), a[0]);
#pragma unroll
      for (int q = 1; q < 4; ++q) acc = cfma(cconj(M[4 * q + r]), a[q], acc);
      p[r] = acc;
      sp[id[r]] = acc;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc_lconjp(g[2 * (4 * r + q)], g[2 * (4 * r + q) + 1], b[r], p[q]);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      C acc = cmul(cconj(M[r]), b[0]);
#pragma unroll
      for (int q = 1; q < 4; ++q) acc = cfma(cconj(M[4 * q + r]), b[q], acc);
      sl[id[r]] = acc;
    }
  }
  if (grad) gacc_add_acc<WARP, 32>(g, gdst);
}

template <typename R, bool WARP>
__global__ void __launch_bounds__(512, 1) k_batch(BatchArgs a) {
  using C = typename CplxT<R>::T;
  extern __shared__ __align__(16) unsigned char smem[];
  const int gs = WARP ? 32 : static_cast<int>(blockDim.x);
  const int ngroups = WARP ? static_cast<int>(blockDim.x >> 5) : 1;
  const int gid = WARP ? static_cast<int>(threadIdx.x >> 5) : 0;
  const int lt = WARP ? static_cast<int>(threadIdx.x & 31) : static_cast<int>(threadIdx.x);
  const int dmax = 1 << a.nmax;
  // shared memory: psi and lambda of every group, then the block matrices
  // of every group's current instance, then reduction scratch
  C* sp = reinterpret_cast<C*>(smem) + static_cast<int64_t>(gid) * 2 * dmax;
  C* sl = sp + dmax;
  C* bm = reinterpret_cast<C*>(smem) + static_cast<int64_t>(ngroups) * 2 * dmax + gid * a.bmat_slot;
  double* red =
      reinterpret_cast<double*>(reinterpret_cast<C*>(smem) + static_cast<int64_t>(ngroups) * (2 * dmax + a.bmat_slot));
  int* snext = reinterpret_cast<int*>(red + 64);
  const int64_t slot = static_cast<int64_t>(blockIdx.x) * ngroups + gid;
  double2* gacc = a.gacc_ws + slot * a.gacc_slot;
  for (;;) {
    int k;
    if (WARP) {
      if (lt == 0) k = atomicAdd(a.counter, 1);
      k = __shfl_sync(0xffffffffu, k, 0);
    } else {
      if (threadIdx.x == 0) snext[0] = atomicAdd(a.counter, 1);
      __syncthreads();
      k = snext[0];
      __syncthreads();
    }
    if (k >= a.n_order) break;
    const BInst I = a.inst[a.order[k]];
    const BPlan P = a.plans[I.plan];
    const double* ang = a.angles + I.angle_off;
    const int n = P.n, dim = 1 << n;
    const BBlock* BB = a.bblk + P.blk_off;
    // block matrices of this instance, zeroed cotangents, |0...0>
    for (int b = lt; b < P.nblocks; b += gs)
      prep_block<R>(a.dblk[P.blk_off + b], a.prims, a.ops, ang, nullptr, a.cpool, bm, nullptr);
    for (int e = lt; e < P.grad_stride; e += gs) gacc[e] = make_double2(0.0, 0.0);
    for (int j = lt; j < dim; j += gs) sp[j] = cmake<C>(j == 0 ? 1.0 : 0.0, 0.0);
    gsync<WARP>();
    for (int b = 0; b < P.nblocks;) {
      if (BB[b].pair) {
        bapply2<C>(sp, n, BB[b], BB[b + 1], bm, lt, gs);
        b += 2;
      } else {
        bapply<C>(sp, n, BB[b], bm, lt, gs);
        b += 1;
      }
      gsync<WARP>();
    }
    // expectation values; lambda = 2 sum_o ct_o coeff_o P_o psi
    for (int j = lt; j < dim; j += gs) sl[j] = cmake<C>(0.0, 0.0);
    for (int o = 0; o < P.n_obs; ++o) {
      const DevObs ob = a.obs[P.obs_off + o];
      const double w = 2.0 * (a.ct ? a.ct[I.out_off + o] : 1.0) * ob.coeff;
      double part = 0.0;
      for (int j = lt; j < dim; j += gs) {
        const int jx = j ^ static_cast<int>(ob.x_mask);
        const double sign = (__popc(static_cast<uint32_t>(jx) & static_cast<uint32_t>(ob.z_mask)) & 1) ? -1.0 : 1.0;
        const double2 v = mul_iy(ob.n_y, to_d2(sp[jx]));  // (P psi)_j = sign * i^ny * psi_{j^x}
        const double2 pj = to_d2(sp[j]);
        part += sign * (pj.x * v.x + pj.y * v.y);
        const double2 l = to_d2(sl[j]);
        sl[j] = cmake<C>(l.x + w * sign * v.x, l.y + w * sign * v.y);
      }
      const double tot = gsum<WARP>(part, red);
      if (lt == 0) a.expval[I.out_off + o] = ob.coeff * tot;
    }
    gsync<WARP>();
    for (int b = P.nblocks - 1; b >= 0;) {
      if (b >= 1 && BB[b - 1].pair) {
        badjoint2<C, WARP>(sp, sl, n, BB[b - 1], BB[b], bm, reinterpret_cast<double*>(gacc), lt, gs);
        b -= 2;
      } else {
        badjoint<C, WARP>(sp, sl, n, BB[b], bm, reinterpret_cast<double*>(gacc), lt, gs);
        b -= 1;
      }
      gsync<WARP>();
    }
    for (int b = lt; b < P.nblocks; b += gs)
      chain_block(a.dblk[P.blk_off + b], a.prims, a.ops, ang, nullptr, a.cpool, gacc, nullptr, a.grad + I.angle_off,
                  nullptr);
    gsync<WARP>();
  }
}

// ---------------------------------------------------------------------------
// cluster class: one instance on a cluster of CL CTAs; CTA `rank` holds the
// amplitudes whose top log2(CL) index bits equal rank (its local slice of
// 2^L, L = n - log2 CL, for psi and for lambda).  Blocks whose targets are
// local bits run as in the single-CTA kernel (controls and diagonal rows
// may use the rank bits); a dense or permutation block with a target among
// the rank bits reads its sibling amplitudes from the other CTAs' shared
// memory (distributed shared memory), computes this CTA's new values into
// a global scratch slice, waits for the cluster, then writes them back.
// ---------------------------------------------------------------------------
struct ClusterArgs {
  BatchArgs a;
  int lbits;          // L: local index bits per CTA
  void* xs_ws;        // per CTA: 2 * 2^L run-dtype complex exchange scratch
  const RStage* stg;  // register-stage programs (k_batch_rs)
  const RPacked* rop;
};

__device__ __forceinline__ bool bdist(const BBlock& B, int lbits) {
  return B.kind != BK_DIAG && (B.tb0 >= lbits || (B.nt == 2 && B.tb1 >= lbits));
}

// Global index of sibling c (target bits set to c) of global index g.
__device__ __forceinline__ uint32_t bsib(const BBlock& B, uint32_t g, int c) {
  if (B.nt == 1) return (g & ~(1u << B.tb0)) | (static_cast<uint32_t>(c & 1) << B.tb0);
  g &= ~((1u << B.tb0) | (1u << B.tb1));
  return g | (static_cast<uint32_t>((c >> 1) & 1) << B.tb0) | (static_cast<uint32_t>(c & 1) << B.tb1);
}

__device__ __forceinline__ int brow(const BBlock& B, uint32_t g) {
  return B.nt == 1 ? static_cast<int>((g >> B.tb0) & 1) : static_cast<int>((((g >> B.tb0) & 1) << 1) | ((g >> B.tb1) & 1));
}

// Adjoint of a block with a target among the rank bits (NT targets): new
// psi and lambda of this CTA's rows into xs (psi) and xs + 2^L (lambda), the
// block cotangent into gacc.  Every sibling row is read from the CTA that
// holds it; the caller syncs the cluster before and after.
template <typename C, int NT, int CL>
__device__ __forceinline__ void cl_adj_dist(cooperative_groups::cluster_group& cluster, const BBlock& B, const C* bm,
                                            C* sp, C* sl, C* xs, double2* gacc, int lb, uint32_t gbase, int lt,
                                            int gs) {
  using A = typename AccT<C>::T;
  constexpr int ND = 1 << NT;
  const int nloc = 1 << lb;
  const C* M = bm + B.mat_off;
  const bool grad = B.grad_off >= 0;
  A gs2[2 * ND * ND];
#pragma unroll
  for (int e = 0; e < 2 * ND * ND; ++e) gs2[e] = A(0);
  for (int j = lt; j < nloc; j += gs) {
    const uint32_t g = gbase | static_cast<uint32_t>(j);
    if ((g & B.cmask) != B.cmask) continue;
    const int r = brow(B, g);
    C vp[ND], vl[ND];
#pragma unroll
    for (int c = 0; c < ND; ++c) {
      const uint32_t gc = bsib(B, g, c);
      vp[c] = cluster.map_shared_rank(sp, gc >> lb)[gc & (nloc - 1)];
      vl[c] = cluster.map_shared_rank(sl, gc >> lb)[gc & (nloc - 1)];
    }
    if (B.kind == BK_PERM) {
      // inverse permutation: new[p[r']] = old[r'] (exactly one r' has p[r'] = r)
      C op = vp[0], ol = vl[0];
#pragma unroll
      for (int c = 1; c < ND; ++c)
        if (((B.perm >> (2 * c)) & 3) == r) { op = vp[c]; ol = vl[c]; }
      xs[j] = op;
      xs[nloc + j] = ol;
      continue;
    }
    // psi' = G^dagger psi on every row of the group (rows other CTAs own too)
    C np[ND];
#pragma unroll
    for (int c = 0; c < ND; ++c) {
      C acc = cmul(cconj(M[c]), vp[0]);
#pragma unroll
      for (int c2 = 1; c2 < ND; ++c2) acc = cfma(cconj(M[c2 * ND + c]), vp[c2], acc);
      np[c] = acc;
    }
    C nl = cmul(cconj(M[r]), vl[0]);
#pragma unroll
    for (int c2 = 1; c2 < ND; ++c2) nl = cfma(cconj(M[c2 * ND + r]), vl[c2], nl);
    C mine = np[0], lr = vl[0];
#pragma unroll
    for (int c = 1; c < ND; ++c)
      if (c == r) { mine = np[c]; lr = vl[c]; }
    xs[j] = mine;
    xs[nloc + j] = nl;
    if (grad) {
#pragma unroll
      for (int rr = 0; rr < ND; ++rr) {
        if (rr != r) continue;
#pragma unroll
        for (int c = 0; c < ND; ++c) {
          // lambda_r conj(psi'_c)
          gs2[2 * (rr * ND + c)] += static_cast<A>(lr.x) * np[c].x + static_cast<A>(lr.y) * np[c].y;
          gs2[2 * (rr * ND + c) + 1] += static_cast<A>(lr.y) * np[c].x - static_cast<A>(lr.x) * np[c].y;
        }
      }
    }
  }
  if (grad) {
    double gd[2 * ND * ND];
#pragma unroll
    for (int e = 0; e < 2 * ND * ND; ++e) gd[e] = static_cast<double>(gs2[e]);
    gacc_add<false, 2 * ND * ND>(gd, reinterpret_cast<double*>(gacc) + 2 * B.grad_off);
  }
}

// Fast path of a one-target block on a rank bit (complex64, 16 amplitudes
// per thread): the partner CTA's amplitudes at this thread's own local
// indices are the only ones needed, so they move as 8 independent 16-byte
// DSMEM loads per vector into registers between the two cluster barriers.
template <int CL>
__device__ __forceinline__ void cl_fwd_fast(cooperative_groups::cluster_group& cluster, const BBlock& B,
                                            const float2* M, float2* sp, int lb, uint32_t rank, int lt, int gs) {
  const uint32_t pr = rank ^ (1u << (B.tb0 - lb));
  const int mybit = static_cast<int>((rank >> (B.tb0 - lb)) & 1);
  const uint32_t gbase = rank << lb;
  const float4* rsp = reinterpret_cast<const float4*>(cluster.map_shared_rank(sp, pr));
  float4* own = reinterpret_cast<float4*>(sp);
  float4 pv[8];
  cluster.sync();  // partner values final
#pragma unroll
  for (int k = 0; k < 8; ++k) pv[k] = rsp[lt + k * gs];
  cluster.sync();  // every CTA holds what it needs
  const bool perm = B.kind == BK_PERM;
  const bool swap = perm && (B.perm & 1);
  const float2 a = mybit ? M[3] : M[0], b = mybit ? M[2] : M[1];  // new own = a own + b partner
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int idx = lt + k * gs;
    float4 o = own[idx];
    const float4 q = pv[k];
    float2 x0 = make_float2(o.x, o.y), x1 = make_float2(o.z, o.w);
    const float2 y0 = make_float2(q.x, q.y), y1 = make_float2(q.z, q.w);
    const uint32_t g0 = gbase | static_cast<uint32_t>(2 * idx);
    const bool c0 = (g0 & B.cmask) == B.cmask, c1 = ((g0 | 1u) & B.cmask) == B.cmask;
    if (perm) {
      if (swap && c0) x0 = y0;
      if (swap && c1) x1 = y1;
    } else {
      if (c0) x0 = cfma(b, y0, cmul(a, x0));
      if (c1) x1 = cfma(b, y1, cmul(a, x1));
    }
    own[idx] = make_float4(x0.x, x0.y, x1.x, x1.y);
  }
  __syncthreads();
}

template <int CL>
__device__ __forceinline__ void cl_adj_fast(cooperative_groups::cluster_group& cluster, const BBlock& B,
                                            const float2* M, float2* sp, float2* sl, double2* gacc, int lb,
                                            uint32_t rank, int lt, int gs) {
  const uint32_t pr = rank ^ (1u << (B.tb0 - lb));
  const int mybit = static_cast<int>((rank >> (B.tb0 - lb)) & 1);
  const uint32_t gbase = rank << lb;
  const float4* rsp = reinterpret_cast<const float4*>(cluster.map_shared_rank(sp, pr));
  const float4* rsl = reinterpret_cast<const float4*>(cluster.map_shared_rank(sl, pr));
  float4* ownp = reinterpret_cast<float4*>(sp);
  float4* ownl = reinterpret_cast<float4*>(sl);
  float4 pp[8], pl[8];
  cluster.sync();
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    pp[k] = rsp[lt + k * gs];
    pl[k] = rsl[lt + k * gs];
  }
  cluster.sync();
  const bool perm = B.kind == BK_PERM;
  const bool swap = perm && (B.perm & 1);
  const bool grad = !perm && B.grad_off >= 0;
  // rows: b = mybit (own), 1 - b (partner).  G^dagger[c][c2] = conj(M[c2][c]).
  const int bo = mybit, bp = 1 - mybit;
  float g[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) g[e] = 0.0f;
  auto step = [&](float2& xo, float2 xp, float2& lo, float2 lp) {
    if (perm) {
      if (swap) { xo = xp; lo = lp; }
      return;
    }
    // psi_c for c = bo (own) and bp (partner); psi'_c = sum_c2 conj(M[c2][c]) psi_c2
    float2 ps[2], ls[2];
    ps[bo] = xo; ps[bp] = xp;
    ls[bo] = lo; ls[bp] = lp;
    const float2 n0 = cfma(cconj(M[2]), ps[1], cmul(cconj(M[0]), ps[0]));
    const float2 n1 = cfma(cconj(M[3]), ps[1], cmul(cconj(M[1]), ps[0]));
    const float2 lnew = bo ? cfma(cconj(M[3]), ls[1], cmul(cconj(M[1]), ls[0]))
                           : cfma(cconj(M[2]), ls[1], cmul(cconj(M[0]), ls[0]));
    if (grad) {
      // lambda_bo conj(psi'_c)
      const float2 l = lo;
      g[4 * bo + 0] += l.x * n0.x + l.y * n0.y;
      g[4 * bo + 1] += l.y * n0.x - l.x * n0.y;
      g[4 * bo + 2] += l.x * n1.x + l.y * n1.y;
      g[4 * bo + 3] += l.y * n1.x - l.x * n1.y;
    }
    xo = bo ? n1 : n0;
    lo = lnew;
  };
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int idx = lt + k * gs;
    const float4 op = ownp[idx], ol = ownl[idx], qp = pp[k], ql = pl[k];
    float2 x0 = make_float2(op.x, op.y), x1 = make_float2(op.z, op.w);
    float2 l0 = make_float2(ol.x, ol.y), l1 = make_float2(ol.z, ol.w);
    const uint32_t g0 = gbase | static_cast<uint32_t>(2 * idx);
    if ((g0 & B.cmask) == B.cmask) step(x0, make_float2(qp.x, qp.y), l0, make_float2(ql.x, ql.y));
    if (((g0 | 1u) & B.cmask) == B.cmask) step(x1, make_float2(qp.z, qp.w), l1, make_float2(ql.z, ql.w));
    ownp[idx] = make_float4(x0.x, x0.y, x1.x, x1.y);
    ownl[idx] = make_float4(l0.x, l0.y, l1.x, l1.y);
  }
  if (grad) gacc_add_acc<false, 8>(g, reinterpret_cast<double*>(gacc) + 2 * B.grad_off);
  __syncthreads();
}

template <typename R, int CL>
__global__ void __launch_bounds__(512, 1) k_batch_cluster(ClusterArgs ca) {
  using C = typename CplxT<R>::T;
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const BatchArgs& a = ca.a;
  extern __shared__ __align__(16) unsigned char smem[];
  const int lb = ca.lbits, nloc = 1 << lb;
  const int gs = static_cast<int>(blockDim.x), lt = static_cast<int>(threadIdx.x);
  const uint32_t rank = cluster.block_rank();
  C* sp = reinterpret_cast<C*>(smem);
  C* sl = sp + nloc;
  C* bm = sl + nloc;                                    // block matrices of the instance
  double* red = reinterpret_cast<double*>(bm + a.bmat_slot);  // 32 doubles
  double* spart = red + 32;                            // 32 per-observable partial sums
  int* snext = reinterpret_cast<int*>(spart + 32);
  C* rp[CL];
  C* rl[CL];
#pragma unroll
  for (int r = 0; r < CL; ++r) {
    rp[r] = cluster.map_shared_rank(sp, r);
    rl[r] = cluster.map_shared_rank(sl, r);
  }
  const int64_t cid = blockIdx.x / CL;
  double2* gacc = a.gacc_ws + cid * a.gacc_slot;
  C* xs = static_cast<C*>(ca.xs_ws) + static_cast<int64_t>(blockIdx.x) * 2 * nloc;
  const uint32_t gbase = rank << lb;
  for (;;) {
    if (rank == 0 && lt == 0) snext[0] = atomicAdd(a.counter, 1);
    cluster.sync();
    const int k = *cluster.map_shared_rank(snext, 0);
    cluster.sync();
    if (k >= a.n_order) break;
    const BInst I = a.inst[a.order[k]];
    const BPlan P = a.plans[I.plan];
    const double* ang = a.angles + I.angle_off;
    const BBlock* BB = a.bblk + P.blk_off;
    for (int b = lt; b < P.nblocks; b += gs)
      prep_block<R>(a.dblk[P.blk_off + b], a.prims, a.ops, ang, nullptr, a.cpool, bm, nullptr);
    if (rank == 0)
      for (int e = lt; e < P.grad_stride; e += gs) gacc[e] = make_double2(0.0, 0.0);
    for (int j = lt; j < nloc; j += gs) sp[j] = cmake<C>((gbase | static_cast<uint32_t>(j)) == 0 ? 1.0 : 0.0, 0.0);
    cluster.sync();
    // forward
    for (int b = 0; b < P.nblocks; ++b) {
      const BBlock B = BB[b];
      if (B.pair && B.tb0 < lb && BB[b + 1].tb0 < lb) {
        bapply2<C>(sp, lb, B, BB[b + 1], bm, lt, gs);
        __syncthreads();
        ++b;
        continue;
      }
      if (!bdist(B, lb)) {
        bapply<C>(sp, lb, B, bm, lt, gs, gbase);
        __syncthreads();
        continue;
      }
      if constexpr (sizeof(C) == 8) {
        if (B.nt == 1 && nloc == 16 * gs) {
          cl_fwd_fast<CL>(cluster, B, bm + B.mat_off, sp, lb, rank, lt, gs);
          continue;
        }
      }
      cluster.sync();  // every CTA's earlier writes are final
      const C* M = bm + B.mat_off;
      const int nd = 1 << B.nt;
      // U elements per thread at a time: all sibling loads (local or remote)
      // issue before any use; the new values go to the lambda slice, which
      // the forward sweep does not use yet
      constexpr int U = 2;
      for (int j0 = lt; j0 < nloc; j0 += U * gs) {
        C v[U][4];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int j = j0 + u * gs;
          const uint32_t g = gbase | static_cast<uint32_t>(j);
          if (j < nloc && (g & B.cmask) == B.cmask) {
#pragma unroll
            for (int c = 0; c < 4; ++c)
              if (c < nd) {
                const uint32_t gc = bsib(B, g, c);
                v[u][c] = cluster.map_shared_rank(sp, gc >> lb)[gc & (nloc - 1)];
              }
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int j = j0 + u * gs;
          const uint32_t g = gbase | static_cast<uint32_t>(j);
          if (j >= nloc || (g & B.cmask) != B.cmask) continue;
          const int r = brow(B, g);
          C out;
          if (B.kind == BK_PERM) {
            const int src = (B.perm >> (2 * r)) & 3;
            out = v[u][0];
#pragma unroll
            for (int c = 1; c < 4; ++c)
              if (c == src) out = v[u][c];
          } else {
            out = cmul(M[r * nd], v[u][0]);
#pragma unroll
            for (int c = 1; c < 4; ++c)
              if (c < nd) out = cfma(M[r * nd + c], v[u][c], out);
          }
          sl[j] = out;
        }
      }
      cluster.sync();  // every read of the old values is done
      for (int j = lt; j < nloc; j += gs)
        if (((gbase | static_cast<uint32_t>(j)) & B.cmask) == B.cmask) sp[j] = sl[j];
      __syncthreads();
    }
    cluster.sync();
    // expectation values (partial sums per CTA, added by rank 0) and lambda
    for (int j = lt; j < nloc; j += gs) sl[j] = cmake<C>(0.0, 0.0);
    for (int o = 0; o < P.n_obs; ++o) {
      const DevObs ob = a.obs[P.obs_off + o];
      const double w = 2.0 * (a.ct ? a.ct[I.out_off + o] : 1.0) * ob.coeff;
      double part = 0.0;
      for (int j = lt; j < nloc; j += gs) {
        const uint32_t g = gbase | static_cast<uint32_t>(j);
        const uint32_t gx = g ^ static_cast<uint32_t>(ob.x_mask);
        const double sign = (__popc(gx & static_cast<uint32_t>(ob.z_mask)) & 1) ? -1.0 : 1.0;
        const double2 v = mul_iy(ob.n_y, to_d2(rp[gx >> lb][gx & (nloc - 1)]));
        const double2 pj = to_d2(sp[j]);
        part += sign * (pj.x * v.x + pj.y * v.y);
        const double2 l = to_d2(sl[j]);
        sl[j] = cmake<C>(l.x + w * sign * v.x, l.y + w * sign * v.y);
      }
      const double tot = gsum<false>(part, red);
      if (lt == 0) spart[o] = tot;
    }
    cluster.sync();
    if (rank == 0 && lt < P.n_obs) {
      double tot = 0.0;
      for (int r = 0; r < CL; ++r) tot += *cluster.map_shared_rank(spart + lt, r);
      a.expval[I.out_off + lt] = a.obs[P.obs_off + lt].coeff * tot;
    }
    // adjoint
    for (int b = P.nblocks - 1; b >= 0; --b) {
      const BBlock B = BB[b];
      if (b >= 1 && BB[b - 1].pair && BB[b - 1].tb0 < lb && B.tb0 < lb) {
        badjoint2<C, false>(sp, sl, lb, BB[b - 1], B, bm, reinterpret_cast<double*>(gacc), lt, gs);
        __syncthreads();
        --b;
        continue;
      }
      if (!bdist(B, lb)) {
        badjoint<C, false>(sp, sl, lb, B, bm, reinterpret_cast<double*>(gacc), lt, gs, gbase);
        __syncthreads();
        continue;
      }
      if constexpr (sizeof(C) == 8) {
        if (B.nt == 1 && nloc == 16 * gs) {
          cl_adj_fast<CL>(cluster, B, bm + B.mat_off, sp, sl, gacc, lb, rank, lt, gs);
          continue;
        }
      }
      cluster.sync();
      if (B.nt == 1) cl_adj_dist<C, 1, CL>(cluster, B, bm, sp, sl, xs, gacc, lb, gbase, lt, gs);
      else cl_adj_dist<C, 2, CL>(cluster, B, bm, sp, sl, xs, gacc, lb, gbase, lt, gs);
      cluster.sync();
      for (int j = lt; j < nloc; j += gs)
        if (((gbase | static_cast<uint32_t>(j)) & B.cmask) == B.cmask) {
          sp[j] = xs[j];
          sl[j] = xs[nloc + j];
        }
      __syncthreads();
    }
    cluster.sync();  // every cotangent contribution is in
    for (int b = static_cast<int>(rank) * gs + lt; b < P.nblocks; b += CL * gs)
      chain_block(a.dblk[P.blk_off + b], a.prims, a.ops, ang, nullptr, a.cpool, gacc, nullptr, a.grad + I.angle_off,
                  nullptr);
    cluster.sync();  // the cotangent slot and block matrices are free again
  }
}

// ---------------------------------------------------------------------------
// register-stage cluster class (complex64): the same instances as
// k_batch_cluster, one shared-memory sweep per stage of up to 4 register
// bits (RStage) instead of one per block.  psi and lambda slices are stored
// under rs_swz (an XOR-linear involution of the local offset that folds the
// higher bits into the four bank-group bits), so the 16 lanes of a
// shared-memory wavefront, which the stage builder places on local bits of
// distinct residues mod 4, hit distinct banks.  A thread owns its 16
// amplitudes for the whole stage, so a stage updates them in place; a stage
// with a rank bit among its register bits reads and writes other CTAs'
// slices through distributed shared memory between two cluster barriers.
// Block cotangents are reduced per op: a warp reduce-scatter, then float
// atomics into this CTA's shared accumulator, summed over the cluster once
// per instance.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t rs_swz(uint32_t a) { return a ^ (((a >> 4) ^ (a >> 8) ^ (a >> 12)) & 15u); }

// Packed complex64 products in the two-accumulator form: with broadcast
// pairs mr = (re, re), mi = (im, im) of each matrix entry, p = sum mr * x and
// q = sum mi * x, the product is (p.x - q.y, p.y + q.x) (conj entries:
// (p.x + q.y, p.y - q.x)).
__device__ __forceinline__ void rs_coef(float2 m, float2& r, float2& i) {
  r = make_float2(m.x, m.x);
  i = make_float2(m.y, m.y);
}
__device__ __forceinline__ float2 rs_fin(float2 p, float2 q) { return make_float2(p.x - q.y, p.y + q.x); }
__device__ __forceinline__ float2 rs_finc(float2 p, float2 q) { return make_float2(p.x + q.y, p.y - q.x); }
// m x + n y
__device__ __forceinline__ float2 rs_dot(float2 mr, float2 mi, float2 nr, float2 ni, float2 x, float2 y) {
  return rs_fin(__ffma2_rn(nr, y, __fmul2_rn(mr, x)), __ffma2_rn(ni, y, __fmul2_rn(mi, x)));
}
// conj(m) x + conj(n) y
__device__ __forceinline__ float2 rs_dotc(float2 mr, float2 mi, float2 nr, float2 ni, float2 x, float2 y) {
  return rs_finc(__ffma2_rn(nr, y, __fmul2_rn(mr, x)), __ffma2_rn(ni, y, __fmul2_rn(mi, x)));
}

// Reduce 8 per-thread float partials over the warp and add them to dst[0..7].
__device__ __forceinline__ void rs_flush8(float (&g)[8], float* dst, unsigned lane) {
  WarpRS<16, 8, float>::run(g, lane);
  if ((lane & 3u) == 0) atomicAdd(dst + (lane >> 2), g[0]);
}

__device__ __forceinline__ float2 rs_sel4(float2 a0, float2 a1, float2 a2, float2 a3, int k) {
  const float2 lo = (k & 1) ? a1 : a0, hi = (k & 1) ? a3 : a2;
  return (k & 2) ? hi : lo;
}

// forward one-target dense block on register bit Q
template <int Q, bool CTRL>
__device__ __forceinline__ void rs_d1(float2 (&v)[16], const float2* M, uint32_t crm, bool tp) {
  float2 ar, ai, br, bi, cr, ci, dr, di;
  rs_coef(M[0], ar, ai);
  rs_coef(M[1], br, bi);
  rs_coef(M[2], cr, ci);
  rs_coef(M[3], dr, di);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (j & (1 << Q)) continue;
    const int k = j | (1 << Q);
    const float2 x = v[j], y = v[k];
    const float2 nx = rs_dot(ar, ai, br, bi, x, y);
    const float2 ny = rs_dot(cr, ci, dr, di, x, y);
    if (CTRL) {
      const bool on = tp && ((static_cast<uint32_t>(j) & crm) == crm);
      v[j] = on ? nx : x;
      v[k] = on ? ny : y;
    } else {
      v[j] = nx;
      v[k] = ny;
    }
  }
}

// reverse one-target dense block: psi <- G^dagger psi, cotangent += lam psi^dagger,
// lam <- G^dagger lam
template <int Q, bool CTRL>
__device__ __forceinline__ void rs_d1_adj(float2 (&vp)[16], float2 (&vl)[16], const float2* M, uint32_t crm, bool tp,
                                          float* dst, unsigned lane) {
  // G^dagger = [[conj m00, conj m10], [conj m01, conj m11]]; three sweeps over
  // the pairs (psi, cotangent, lambda) keep few values live at a time
  float2 ar, ai, br, bi, cr, ci, dr, di;
  rs_coef(M[0], ar, ai);
  rs_coef(M[2], br, bi);
  rs_coef(M[1], cr, ci);
  rs_coef(M[3], dr, di);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (j & (1 << Q)) continue;
    const int k = j | (1 << Q);
    if (CTRL && !(tp && ((static_cast<uint32_t>(j) & crm) == crm))) continue;
    const float2 x = vp[j], y = vp[k];
    vp[j] = rs_dotc(ar, ai, br, bi, x, y);
    vp[k] = rs_dotc(cr, ci, dr, di, x, y);
  }
  if (dst) {
    float g[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) g[e] = 0.f;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      if (j & (1 << Q)) continue;
      const int k = j | (1 << Q);
      if (CTRL && !(tp && ((static_cast<uint32_t>(j) & crm) == crm))) continue;
      acc_lconjp(g[0], g[1], vl[j], vp[j]);
      acc_lconjp(g[2], g[3], vl[j], vp[k]);
      acc_lconjp(g[4], g[5], vl[k], vp[j]);
      acc_lconjp(g[6], g[7], vl[k], vp[k]);
    }
    rs_flush8(g, dst, lane);
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (j & (1 << Q)) continue;
    const int k = j | (1 << Q);
    if (CTRL && !(tp && ((static_cast<uint32_t>(j) & crm) == crm))) continue;
    const float2 u = vl[j], w = vl[k];
    vl[j] = rs_dotc(ar, ai, br, bi, u, w);
    vl[k] = rs_dotc(cr, ci, dr, di, u, w);
  }
}

// forward two-target dense block on register bits (Q0 = matrix MSB, Q1)
template <int Q0, int Q1>
__device__ __forceinline__ void rs_d2(float2 (&v)[16], const float2* M, uint32_t crm, bool tp) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if ((j >> Q0) & 1 || (j >> Q1) & 1) continue;
    if (!(tp && ((static_cast<uint32_t>(j) & crm) == crm))) continue;
    const int id[4] = {j, j | (1 << Q1), j | (1 << Q0), j | (1 << Q0) | (1 << Q1)};
    float2 a[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) a[c] = v[id[c]];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      float2 mr, mi;
      rs_coef(M[4 * r], mr, mi);
      float2 p = __fmul2_rn(mr, a[0]), q = __fmul2_rn(mi, a[0]);
#pragma unroll
      for (int c = 1; c < 4; ++c) {
        rs_coef(M[4 * r + c], mr, mi);
        p = __ffma2_rn(mr, a[c], p);
        q = __ffma2_rn(mi, a[c], q);
      }
      v[id[r]] = rs_fin(p, q);
    }
  }
}

// G^dagger applied to the group of v at base j (rows r = sum_q conj M[4q + r] a_q)
template <int Q0, int Q1>
__device__ __forceinline__ void rs_d2h(float2 (&v)[16], const float2* M, int j) {
  const int id[4] = {j, j | (1 << Q1), j | (1 << Q0), j | (1 << Q0) | (1 << Q1)};
  float2 a[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) a[c] = v[id[c]];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    float2 mr, mi;
    rs_coef(M[r], mr, mi);
    float2 p = __fmul2_rn(mr, a[0]), q = __fmul2_rn(mi, a[0]);
#pragma unroll
    for (int c = 1; c < 4; ++c) {
      rs_coef(M[4 * c + r], mr, mi);
      p = __ffma2_rn(mr, a[c], p);
      q = __ffma2_rn(mi, a[c], q);
    }
    v[id[r]] = rs_finc(p, q);
  }
}

template <int Q0, int Q1>
__device__ __forceinline__ void rs_d2_adj(float2 (&vp)[16], float2 (&vl)[16], const float2* M, uint32_t crm, bool tp,
                                          float* dst, unsigned lane) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if ((j >> Q0) & 1 || (j >> Q1) & 1) continue;
    if (tp && ((static_cast<uint32_t>(j) & crm) == crm)) rs_d2h<Q0, Q1>(vp, M, j);
  }
  if (dst) {
    // cotangent row r: lam_r (before its update) times conj of the new psi
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      float g[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) g[e] = 0.f;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        if ((j >> Q0) & 1 || (j >> Q1) & 1) continue;
        if (!(tp && ((static_cast<uint32_t>(j) & crm) == crm))) continue;
        const int id[4] = {j, j | (1 << Q1), j | (1 << Q0), j | (1 << Q0) | (1 << Q1)};
#pragma unroll
        for (int q = 0; q < 4; ++q) acc_lconjp(g[2 * q], g[2 * q + 1], vl[id[r]], vp[id[q]]);
      }
      rs_flush8(g, dst + 8 * r, lane);
    }
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if ((j >> Q0) & 1 || (j >> Q1) & 1) continue;
    if (tp && ((static_cast<uint32_t>(j) & crm) == crm)) rs_d2h<Q0, Q1>(vl, M, j);
  }
}

__device__ __forceinline__ int rs_drow(int j, const ROp& op) {
  return op.nt == 1 ? ((j >> op.q0) & 1) : ((((j >> op.q0) & 1) << 1) | ((j >> op.q1) & 1));
}

__device__ __forceinline__ void rs_diag(float2 (&v)[16], const float2* M, const ROp& op, bool tp) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (!(tp && ((static_cast<uint32_t>(j) & op.crm) == op.crm))) continue;
    float2 mr, mi;
    rs_coef(M[rs_drow(j, op)], mr, mi);
    v[j] = rs_fin(__fmul2_rn(mr, v[j]), __fmul2_rn(mi, v[j]));
  }
}

__device__ __forceinline__ void rs_diag_adj(float2 (&vp)[16], float2 (&vl)[16], const float2* M, const ROp& op,
                                            bool tp, float* dst, unsigned lane) {
  float g[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) g[e] = 0.f;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (!(tp && ((static_cast<uint32_t>(j) & op.crm) == op.crm))) continue;
    const int r = rs_drow(j, op);
    float2 mr, mi;
    rs_coef(M[r], mr, mi);
    const float2 p = rs_finc(__fmul2_rn(mr, vp[j]), __fmul2_rn(mi, vp[j]));
    const float2 l = vl[j];
    vp[j] = p;
    vl[j] = rs_finc(__fmul2_rn(mr, l), __fmul2_rn(mi, l));
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (q == r) acc_lconjp(g[2 * q], g[2 * q + 1], l, p);
  }
  if (dst) rs_flush8(g, dst, lane);
}

// one-target permutation (X on register bit Q); its own inverse
template <int Q>
__device__ __forceinline__ void rs_p1(float2 (&v)[16], uint32_t crm, bool tp) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (j & (1 << Q)) continue;
    const int k = j | (1 << Q);
    const bool on = tp && ((static_cast<uint32_t>(j) & crm) == crm);
    const float2 x = v[j], y = v[k];
    v[j] = on ? y : x;
    v[k] = on ? x : y;
  }
}

// two-target permutation: output row r takes input row (perm >> 2r) & 3
template <int Q0, int Q1>
__device__ __forceinline__ void rs_p2(float2 (&v)[16], int perm, uint32_t crm, bool tp) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if ((j >> Q0) & 1 || (j >> Q1) & 1) continue;
    if (!(tp && ((static_cast<uint32_t>(j) & crm) == crm))) continue;
    const int id[4] = {j, j | (1 << Q1), j | (1 << Q0), j | (1 << Q0) | (1 << Q1)};
    const float2 a0 = v[id[0]], a1 = v[id[1]], a2 = v[id[2]], a3 = v[id[3]];
#pragma unroll
    for (int r = 0; r < 4; ++r) v[id[r]] = rs_sel4(a0, a1, a2, a3, (perm >> (2 * r)) & 3);
  }
}

// Dispatch over the (Q0, Q1) pairs of distinct register bits.
#define JQ_RS_PAIRS(F, ...)                                     \
  switch (op.q0 * 4 + op.q1) {                                  \
    case 1: F<0, 1>(__VA_ARGS__); break;                        \
    case 2: F<0, 2>(__VA_ARGS__); break;                        \
    case 3: F<0, 3>(__VA_ARGS__); break;                        \
    case 4: F<1, 0>(__VA_ARGS__); break;                        \
    case 6: F<1, 2>(__VA_ARGS__); break;                        \
    case 7: F<1, 3>(__VA_ARGS__); break;                        \
    case 8: F<2, 0>(__VA_ARGS__); break;                        \
    case 9: F<2, 1>(__VA_ARGS__); break;                        \
    case 11: F<2, 3>(__VA_ARGS__); break;                       \
    case 12: F<3, 0>(__VA_ARGS__); break;                       \
    case 13: F<3, 1>(__VA_ARGS__); break;                       \
    case 14: F<3, 2>(__VA_ARGS__); break;                       \
    default: break;                                             \
  }
#define JQ_RS_ONE(F, ...)                                       \
  switch (op.q0) {                                              \
    case 0: F<0>(__VA_ARGS__); break;                           \
    case 1: F<1>(__VA_ARGS__); break;                           \
    case 2: F<2>(__VA_ARGS__); break;                           \
    default: F<3>(__VA_ARGS__); break;                          \
  }

__device__ __forceinline__ void rs_fwd_op(float2 (&v)[16], const ROp& op, const float2* bm, uint32_t g0) {
  const bool tp = (g0 & op.ctm) == op.ctm;
  const float2* M = bm + op.mat_off;
  const uint32_t crm = op.crm;
  switch (op.kind) {
    case RO_DENSE1:
      if (crm == 0 && op.ctm == 0) {
        switch (op.q0) {
          case 0: rs_d1<0, false>(v, M, crm, tp); break;
          case 1: rs_d1<1, false>(v, M, crm, tp); break;
          case 2: rs_d1<2, false>(v, M, crm, tp); break;
          default: rs_d1<3, false>(v, M, crm, tp); break;
        }
      } else {
        switch (op.q0) {
          case 0: rs_d1<0, true>(v, M, crm, tp); break;
          case 1: rs_d1<1, true>(v, M, crm, tp); break;
          case 2: rs_d1<2, true>(v, M, crm, tp); break;
          default: rs_d1<3, true>(v, M, crm, tp); break;
        }
      }
      break;
    case RO_DENSE2: JQ_RS_PAIRS(rs_d2, v, M, crm, tp) break;
    case RO_DIAG: rs_diag(v, M, op, tp); break;
    case RO_PERM1: JQ_RS_ONE(rs_p1, v, crm, tp) break;
    default: JQ_RS_PAIRS(rs_p2, v, op.perm, crm, tp) break;
  }
}

__device__ __forceinline__ void rs_adj_op(float2 (&vp)[16], float2 (&vl)[16], const ROp& op, const float2* bm,
                                          uint32_t g0, float* acc, unsigned lane) {
  const bool tp = (g0 & op.ctm) == op.ctm;
  const float2* M = bm + op.mat_off;
  const uint32_t crm = op.crm;
  float* dst = op.grad_off >= 0 ? acc + 2 * op.grad_off : nullptr;
  switch (op.kind) {
    case RO_DENSE1:
      if (crm == 0 && op.ctm == 0) {
        switch (op.q0) {
          case 0: rs_d1_adj<0, false>(vp, vl, M, crm, tp, dst, lane); break;
          case 1: rs_d1_adj<1, false>(vp, vl, M, crm, tp, dst, lane); break;
          case 2: rs_d1_adj<2, false>(vp, vl, M, crm, tp, dst, lane); break;
          default: rs_d1_adj<3, false>(vp, vl, M, crm, tp, dst, lane); break;
        }
      } else {
        switch (op.q0) {
          case 0: rs_d1_adj<0, true>(vp, vl, M, crm, tp, dst, lane); break;
          case 1: rs_d1_adj<1, true>(vp, vl, M, crm, tp, dst, lane); break;
          case 2: rs_d1_adj<2, true>(vp, vl, M, crm, tp, dst, lane); break;
          default: rs_d1_adj<3, true>(vp, vl, M, crm, tp, dst, lane); break;
        }
      }
      break;
    case RO_DENSE2: JQ_RS_PAIRS(rs_d2_adj, vp, vl, M, crm, tp, dst, lane) break;
    case RO_DIAG: rs_diag_adj(vp, vl, M, op, tp, dst, lane); break;
    case RO_PERM1:
      JQ_RS_ONE(rs_p1, vp, crm, tp)
      JQ_RS_ONE(rs_p1, vl, crm, tp)
      break;
    default:
      JQ_RS_PAIRS(rs_p2, vp, op.iperm, crm, tp)
      JQ_RS_PAIRS(rs_p2, vl, op.iperm, crm, tp)
      break;
  }
}

// Thread base index of a stage: thread-index bit i at flat bit (byte i of tpos).
__device__ __forceinline__ uint32_t rs_base(const uint32_t (&tw)[5], uint32_t T, int ntb) {
  uint32_t g = 0;
#pragma unroll
  for (int i = 0; i < 20; ++i)
    if (i < ntb) g |= ((T >> i) & 1u) << ((tw[i >> 2] >> (8 * (i & 3))) & 31u);
  return g;
}

template <int J>
__device__ __forceinline__ uint32_t rs_sel(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
  return ((J & 1) ? r0 : 0u) ^ ((J & 2) ? r1 : 0u) ^ ((J & 4) ? r2 : 0u) ^ ((J & 8) ? r3 : 0u);
}

// Distributed shared memory by address: the 32-bit shared::cluster address
// of offset `a` (a shared::cta address) in the CTA of cluster rank r, and
// 8-byte loads / stores through it.
__device__ __forceinline__ uint32_t rs_mapa(uint32_t a, uint32_t r) {
  uint32_t out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(a), "r"(r));
  return out;
}
__device__ __forceinline__ float2 rs_ldc(uint32_t a) {
  float2 v;
  asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ void rs_stc(uint32_t a, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}

// Load / store the 16 amplitudes of a stage.  A local stage addresses this
// CTA's slice: offset = swz(base) ^ swz(register bits), both XOR-linear.  A
// distributed one splits every index the same way into a local offset and a
// CTA rank (rank bits of the base XOR the rank bits of the register part).
template <bool STORE, int J = 0>
__device__ __forceinline__ void rs_move_local(float2 (&v)[16], float2* buf, uint32_t base, uint32_t s0, uint32_t s1,
                                              uint32_t s2, uint32_t s3) {
  if constexpr (J < 16) {
    const uint32_t off = base ^ rs_sel<J>(s0, s1, s2, s3);
    if (STORE) buf[off] = v[J];
    else v[J] = buf[off];
    rs_move_local<STORE, J + 1>(v, buf, base, s0, s1, s2, s3);
  }
}

template <bool STORE, int J = 0>
__device__ __forceinline__ void rs_move_dist(float2 (&v)[16], uint32_t buf, uint32_t base, uint32_t c0, uint32_t s0,
                                             uint32_t s1, uint32_t s2, uint32_t s3, uint32_t k0, uint32_t k1,
                                             uint32_t k2, uint32_t k3) {
  if constexpr (J < 16) {
    const uint32_t a = rs_mapa(buf + 8u * (base ^ rs_sel<J>(s0, s1, s2, s3)), c0 ^ rs_sel<J>(k0, k1, k2, k3));
    if (STORE) rs_stc(a, v[J]);
    else v[J] = rs_ldc(a);
    rs_move_dist<STORE, J + 1>(v, buf, base, c0, s0, s1, s2, s3, k0, k1, k2, k3);
  }
}

// Per-thread addressing of one stage.
struct RSAddr {
  uint32_t g0;              // thread base index
  uint32_t base, c0;        // swz(local part of g0), rank part of g0
  uint32_t s[4], k[4];      // per register bit: swz(local part), rank part
};

__device__ __forceinline__ RSAddr rs_addr(const RStage* S, uint32_t T, int ntb, int lb, int& dist, int& ob, int& oe) {
  const int4 h = *reinterpret_cast<const int4*>(S);
  const int4 t0 = *(reinterpret_cast<const int4*>(S) + 1);
  const int4 t1 = *(reinterpret_cast<const int4*>(S) + 2);
  ob = h.x;
  oe = h.y;
  dist = h.z;
  const uint32_t tw[5] = {static_cast<uint32_t>(t0.x), static_cast<uint32_t>(t0.y), static_cast<uint32_t>(t0.z),
                          static_cast<uint32_t>(t0.w), static_cast<uint32_t>(t1.x)};
  RSAddr A;
  const uint32_t lmask = (1u << lb) - 1u;
  A.g0 = rs_base(tw, T, ntb);
  A.base = rs_swz(A.g0 & lmask);
  A.c0 = A.g0 >> lb;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t r = 1u << ((static_cast<uint32_t>(h.w) >> (8 * q)) & 31u);
    A.s[q] = rs_swz(r & lmask);
    A.k[q] = r >> lb;
  }
  return A;
}

template <int CL>
__global__ void __launch_bounds__(512, 1) k_batch_rs(ClusterArgs ca) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const BatchArgs& a = ca.a;
  extern __shared__ __align__(16) unsigned char smem[];
  const int lb = ca.lbits, nloc = 1 << lb;
  const uint32_t lmask = static_cast<uint32_t>(nloc) - 1u;
  const int gs = static_cast<int>(blockDim.x), lt = static_cast<int>(threadIdx.x);
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t rank = cluster.block_rank();
  const uint32_t T = rank * static_cast<uint32_t>(gs) + static_cast<uint32_t>(lt);
  float2* sp = reinterpret_cast<float2*>(smem);
  float2* sl = sp + nloc;
  const uint32_t sp_s = static_cast<uint32_t>(__cvta_generic_to_shared(sp));
  const uint32_t sl_s = static_cast<uint32_t>(__cvta_generic_to_shared(sl));
  float2* bm = sl + nloc;                                    // block matrices of the instance
  float* acc = reinterpret_cast<float*>(bm + a.bmat_slot);   // this CTA's block cotangents
  double* red = reinterpret_cast<double*>(acc + 2 * a.gacc_slot);
  double* spart = red + 32;
  int* snext = reinterpret_cast<int*>(spart + 32);
  const int64_t cid = blockIdx.x / CL;
  double2* gacc = a.gacc_ws + cid * a.gacc_slot;
  const uint32_t gbase = rank << lb;
  for (;;) {
    if (rank == 0 && lt == 0) snext[0] = atomicAdd(a.counter, 1);
    cluster.sync();
    const int k = *cluster.map_shared_rank(snext, 0);
    cluster.sync();
    if (k >= a.n_order) break;
    const BInst I = a.inst[a.order[k]];
    const BPlan P = a.plans[I.plan];
    const double* ang = a.angles + I.angle_off;
    for (int b = lt; b < P.nblocks; b += gs)
      prep_block<float>(a.dblk[P.blk_off + b], a.prims, a.ops, ang, nullptr, a.cpool, bm, nullptr);
    for (int e = lt; e < 2 * P.grad_stride; e += gs) acc[e] = 0.f;
    for (int j = lt; j < nloc; j += gs) sp[j] = make_float2((gbase | static_cast<uint32_t>(j)) == 0 ? 1.f : 0.f, 0.f);
    cluster.sync();
    const RStage* SS = ca.stg + P.stg_off;
    const RPacked* OPS = ca.rop;
    const int ntb = P.n - 4;
    // forward; a distributed stage needs a cluster barrier before it (unless
    // the stage before it was distributed too) and after it
    bool prev_dist = false;
    for (int s = 0; s < P.n_stg; ++s) {
      int dist, ob, oe;
      const RSAddr A = rs_addr(SS + s, T, ntb, lb, dist, ob, oe);
      float2 v[16];
      if (dist) {
        if (!prev_dist) cluster.sync();
        rs_move_dist<false>(v, sp_s, A.base, A.c0, A.s[0], A.s[1], A.s[2], A.s[3], A.k[0], A.k[1], A.k[2], A.k[3]);
      } else {
        rs_move_local<false>(v, sp, A.base, A.s[0], A.s[1], A.s[2], A.s[3]);
      }
      if (ob < oe) {
        RPacked nx = OPS[ob];
        for (int o = ob; o < oe; ++o) {
          const RPacked cur = nx;
          if (o + 1 < oe) nx = OPS[o + 1];
          rs_fwd_op(v, rs_unpack(cur), bm, A.g0);
        }
      }
      if (dist) {
        rs_move_dist<true>(v, sp_s, A.base, A.c0, A.s[0], A.s[1], A.s[2], A.s[3], A.k[0], A.k[1], A.k[2], A.k[3]);
        cluster.sync();
      } else {
        rs_move_local<true>(v, sp, A.base, A.s[0], A.s[1], A.s[2], A.s[3]);
        __syncthreads();
      }
      prev_dist = dist != 0;
    }
    cluster.sync();
    // expectation values (partial sums per CTA, added by rank 0) and the seed of lambda
    for (int j = lt; j < nloc; j += gs) sl[j] = make_float2(0.f, 0.f);
    for (int o = 0; o < P.n_obs; ++o) {
      const DevObs ob = a.obs[P.obs_off + o];
      const double w = 2.0 * (a.ct ? a.ct[I.out_off + o] : 1.0) * ob.coeff;
      double part = 0.0;
      for (int j = lt; j < nloc; j += gs) {
        const uint32_t g = gbase | rs_swz(static_cast<uint32_t>(j));
        const uint32_t gx = g ^ static_cast<uint32_t>(ob.x_mask);
        const double sign = (__popc(gx & static_cast<uint32_t>(ob.z_mask)) & 1) ? -1.0 : 1.0;
        const double2 v = mul_iy(ob.n_y, to_d2(*cluster.map_shared_rank(sp + rs_swz(gx & lmask), gx >> lb)));
        const double2 pj = to_d2(sp[j]);
        part += sign * (pj.x * v.x + pj.y * v.y);
        const double2 l = to_d2(sl[j]);
        sl[j] = make_float2(static_cast<float>(l.x + w * sign * v.x), static_cast<float>(l.y + w * sign * v.y));
      }
      const double tot = gsum<false>(part, red);
      if (lt == 0) spart[o] = tot;
    }
    cluster.sync();
    if (rank == 0 && lt < P.n_obs) {
      double tot = 0.0;
      for (int r = 0; r < CL; ++r) tot += *cluster.map_shared_rank(spart + lt, r);
      a.expval[I.out_off + lt] = a.obs[P.obs_off + lt].coeff * tot;
    }
    // adjoint: stages in reverse, each stage's ops in reverse
    prev_dist = true;  // the barrier after the expectation values
    for (int s = P.n_stg - 1; s >= 0; --s) {
      int dist, ob, oe;
      const RSAddr A = rs_addr(SS + s, T, ntb, lb, dist, ob, oe);
      float2 vp[16], vl[16];
      if (dist) {
        if (!prev_dist) cluster.sync();
        rs_move_dist<false>(vp, sp_s, A.base, A.c0, A.s[0], A.s[1], A.s[2], A.s[3], A.k[0], A.k[1], A.k[2], A.k[3]);
        rs_move_dist<false>(vl, sl_s, A.base, A.c0, A.s[0], A.s[1], A.s[2], A.s[3], A.k[0], A.k[1], A.k[2], A.k[3]);
      } else {
        rs_move_local<false>(vp, sp, A.base, A.s[0], A.s[1], A.s[2], A.s[3]);
        rs_move_local<false>(vl, sl, A.base, A.s[0], A.s[1], A.s[2], A.s[3]);
      }
      if (ob < oe) {
        RPacked nx = OPS[oe - 1];
        for (int o = oe - 1; o >= ob; --o) {
          const RPacked cur = nx;
          if (o > ob) nx = OPS[o - 1];
          rs_adj_op(vp, vl, rs_unpack(cur), bm, A.g0, acc, lane);
        }
      }
      if (dist) {
        rs_move_dist<true>(vp, sp_s, A.base, A.c0, A.s[0], A.s[1], A.s[2], A.s[3], A.k[0], A.k[1], A.k[2], A.k[3]);
        rs_move_dist<true>(vl, sl_s, A.base, A.c0, A.s[0], A.s[1], A.s[2], A.s[3], A.k[0], A.k[1], A.k[2], A.k[3]);
        cluster.sync();
      } else {
        rs_move_local<true>(vp, sp, A.base, A.s[0], A.s[1], A.s[2], A.s[3]);
        rs_move_local<true>(vl, sl, A.base, A.s[0], A.s[1], A.s[2], A.s[3]);
        __syncthreads();
      }
      prev_dist = dist != 0;
    }
    cluster.sync();  // every CTA's cotangent contributions are in
    for (int e = static_cast<int>(rank) * gs + lt; e < P.grad_stride; e += CL * gs) {
      double re = 0.0, im = 0.0;
      for (int r = 0; r < CL; ++r) {
        const float2 c = *reinterpret_cast<const float2*>(cluster.map_shared_rank(acc + 2 * e, r));
        re += c.x;
        im += c.y;
      }
      gacc[e] = make_double2(re, im);
    }
    cluster.sync();
    for (int b = static_cast<int>(rank) * gs + lt; b < P.nblocks; b += CL * gs)
      chain_block(a.dblk[P.blk_off + b], a.prims, a.ops, ang, nullptr, a.cpool, gacc, nullptr, a.grad + I.angle_off,
                  nullptr);
    cluster.sync();  // the cotangent slots and block matrices are free again
  }
}

// gather / scatter between the batch's instance layout and a plan group's
// dense (instance, entry) layout
__global__ void k_gather_rows(const double* src, const int64_t* src_off, int rows, int width, double* dst) {
  const int64_t total = static_cast<int64_t>(rows) * width;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / width, c = i - r * width;
    dst[i] = src ? src[src_off[r] + c] : 1.0;
  }
}
__global__ void k_scatter_rows(const double* src, const int64_t* dst_off, int rows, int width, double* dst) {
  const int64_t total = static_cast<int64_t>(rows) * width;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = i / width, c = i - r * width;
    dst[dst_off[r] + c] = src[i];
  }
}

}  // namespace
}  // namespace jq

// ---------------------------------------------------------------------------
// host side of the batch
// ---------------------------------------------------------------------------
struct jq_batch {
  int dtype = 0;
  int device = -1;
  int n_inst = 0;
  int64_t n_angles_total = 0, n_obs_total = 0;
  std::vector<const jq_plan*> plans;
  std::vector<jq::BPlan> bplans;
  std::vector<jq::BInst> inst;
  std::vector<jq::BBlock> bblk;
  std::vector<jq::DevBlock> dblk;
  std::vector<jq::DevPrim> prims;
  std::vector<jq::DevOp> ops;
  std::vector<double> cpool;
  std::vector<jq::DevObs> obs;
  std::vector<jq::RStage> rstg;  // register-stage programs of the cluster-class plans
  std::vector<jq::RPacked> rop;
  std::vector<int> n_of_plan;   // qubit count per plan
  // configuration (autotuned)
  jq_batch_config cfg{};
  // device copies
  void* d_plans = nullptr;
  void* d_inst = nullptr;
  void* d_bblk = nullptr;
  void* d_dblk = nullptr;
  void* d_prims = nullptr;
  void* d_ops = nullptr;
  void* d_cpool = nullptr;
  void* d_obs = nullptr;
  void* d_rstg = nullptr;
  void* d_rop = nullptr;
  void* d_order = nullptr;     // warp-class order then cta-class order
  void* d_tile_off = nullptr;  // per tile group: angle offsets then output offsets of its instances
  // classes under the current configuration
  std::vector<int32_t> order_warp, order_cta;
  std::vector<int32_t> order_cl[3];   // cluster class, clusters of 2, 4, 8 CTAs
  struct TileGroup {
    int plan;
    std::vector<int32_t> members;
    int64_t off_angles = 0, off_outs = 0;  // offsets into d_tile_off (int64 entries)
  };
  std::vector<TileGroup> tiles;
  int nmax_warp = 0, nmax_cta = 0;
  int64_t bmat_slot = 0, gacc_slot = 0, slots_warp = 0;
  int64_t bs_warp = 0, bs_cta = 0, bs_cl = 0;  // block-matrix elements per group in shared memory
  // workspace layout
  size_t ws_total = 0, ws_counter = 0, ws_gacc = 0, ws_cl_xs = 0;
  std::vector<size_t> ws_tile;  // per tile group: angles, ct, outs, grads, state, fwd ws, adj ws
  std::vector<size_t> ws_tile_fwd, ws_tile_adj;
  // side streams and the captured graph
  cudaStream_t side[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaStream_t cap = nullptr;   // the graph is captured on this stream
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaGraphExec_t graph = nullptr;
  const void* graph_key[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int sm_count = 0;
};

namespace jq {
namespace {

// Shared memory of a warp / cta / cluster kernel: per group psi, lambda
// (2^nmax each) and the block matrices (bs run-dtype complex, even).
size_t batch_smem(int nmax, int groups, int elem, int64_t bs) {
  return static_cast<size_t>(groups) * (2 * (static_cast<size_t>(1) << nmax) + static_cast<size_t>(bs)) * elem +
         64 * 8 + 16;
}

int64_t even(int64_t x) { return (x + 1) & ~static_cast<int64_t>(1); }

int64_t plan_cost(const jq_batch* b, int p) {
  return (static_cast<int64_t>(1) << b->n_of_plan[p]) * std::max(1, b->bplans[p].nblocks);
}

// Register-stage program of one cluster-class plan (n qubits, lb local bits,
// 16 amplitudes a thread).  Blocks join the current stage greedily in
// program order while their targets fit in 4 register bits; a block that
// does not fit, or that shares a bit (target or control) with a block
// already deferred, is deferred, so every block still follows the blocks it
// does not commute with.  Free register slots take the highest free local
// bits.  Thread-index bits: the four lowest take local positions of distinct
// residues mod 4 (a 16-lane wavefront then hits 16 bank groups under
// rs_swz), the other lane bits the next local positions, the CTA-rank bits
// of the thread index what is left, rank positions last (a stage without a
// rank register bit therefore stays inside each CTA's slice).
void build_rstages(const BBlock* bb, int nblocks, int n, int lb, std::vector<RStage>* stg,
                   std::vector<RPacked>* rops) {
  std::vector<int> rem(nblocks);
  for (int i = 0; i < nblocks; ++i) rem[i] = i;
  while (!rem.empty()) {
    uint32_t R = 0, blocked = 0;
    std::vector<int> members;
    for (int o : rem) {
      const BBlock& B = bb[o];
      uint32_t tg = 1u << B.tb0;
      if (B.nt == 2) tg |= 1u << B.tb1;
      const uint32_t all = tg | B.cmask;
      if (all & blocked) {
        blocked |= all;
        continue;
      }
      if (__builtin_popcount(R | tg) <= 4) {
        R |= tg;
        members.push_back(o);
      } else {
        blocked |= all;
      }
    }
    for (int pos = lb - 1; pos >= 0 && __builtin_popcount(R) < 4; --pos) R |= 1u << pos;
    RStage st;
    std::memset(&st, 0, sizeof(st));
    int rix[32];
    int nr = 0;
    for (int pos = 0; pos < 32; ++pos) rix[pos] = -1;
    for (int pos = 0; pos < n; ++pos)
      if (R >> pos & 1u) {
        st.rpos |= static_cast<uint32_t>(pos) << (8 * nr);
        rix[pos] = nr++;
      }
    std::vector<int> first, rest;
    uint32_t classes = 0;
    for (int pos = 0; pos < lb; ++pos) {
      if (R >> pos & 1u) continue;
      const uint32_t cb = 1u << (pos % 4);
      if (first.size() < 4 && !(classes & cb)) {
        classes |= cb;
        first.push_back(pos);
      } else {
        rest.push_back(pos);
      }
    }
    first.insert(first.end(), rest.begin(), rest.end());
    for (int pos = lb; pos < n; ++pos)
      if (!(R >> pos & 1u)) first.push_back(pos);
    for (size_t i = 0; i < first.size(); ++i) st.tpos[i / 4] |= static_cast<uint32_t>(first[i]) << (8 * (i % 4));
    st.dist = (R >> lb) != 0 ? 1 : 0;
    st.op_begin = static_cast<int32_t>(rops->size());
    for (int o : members) {
      const BBlock& B = bb[o];
      if (B.kind == BK_PERM && B.nt == 1 && (B.perm & 3) == 0) continue;  // identity
      ROp r;
      std::memset(&r, 0, sizeof(r));
      r.nt = B.nt;
      if (B.kind == BK_DENSE) r.kind = B.nt == 1 ? RO_DENSE1 : RO_DENSE2;
      else if (B.kind == BK_DIAG) r.kind = RO_DIAG;
      else r.kind = B.nt == 1 ? RO_PERM1 : RO_PERM2;
      r.q0 = rix[B.tb0];
      r.q1 = B.nt == 2 ? rix[B.tb1] : 0;
      for (int pos = 0; pos < n; ++pos) {
        if (!(B.cmask >> pos & 1u)) continue;
        if (rix[pos] >= 0) r.crm |= 1u << rix[pos];
        else r.ctm |= 1u << pos;
      }
      r.mat_off = B.mat_off;
      r.grad_off = B.grad_off;
      r.perm = B.perm;
      if (B.nt == 2)
        for (int q = 0; q < 4; ++q) r.iperm |= q << (2 * ((B.perm >> (2 * q)) & 3));
      rops->push_back(rs_pack(r));
    }
    st.op_end = static_cast<int32_t>(rops->size());
    stg->push_back(st);
    std::vector<int> left;
    for (int o : rem)
      if (std::find(members.begin(), members.end(), o) == members.end()) left.push_back(o);
    rem.swap(left);
  }
}

// The register-stage cluster kernel runs a cluster launch when the batch is
// complex64, a CTA holds 16 amplitudes a thread (cta_threads = 2^(L - 4)),
// its shared memory also takes the per-CTA cotangent accumulators, and
// JQ_BATCH_RS is not 0.
bool batch_rs_ok(const jq_batch* b, int elem) {
  if (const char* e = std::getenv("JQ_BATCH_RS"))
    if (std::atoi(e) == 0) return false;
  const int lb = b->cfg.cta_max_qubits;
  if (elem != 8 || lb < 8 || lb > 16 || b->cfg.cta_threads != (1 << (lb - 4))) return false;
  return batch_smem(lb, 1, elem, b->bs_cl) + static_cast<size_t>(b->gacc_slot) * 8 <= 227 * 1024;
}

// Which class each plan runs in under the configuration.
int plan_class(const jq_batch* b, int p, const jq_batch_config& c) {
  const jq_plan* pl = b->plans[p];
  const int n = pl->n_qubits;
  bool smem_ok = true;
  for (const DevBlock& blk : pl->blocks) {
    const int nt = blk.k - blk.n_ctrl;
    if (nt < 1 || nt > 2) smem_ok = false;
    if (blk.kind != BK_PERM && blk.k > 2) smem_ok = false;
  }
  for (const DevObs& o : pl->obs)
    if (o.kind != JQ_OBS_PAULI) smem_ok = false;
  if (!smem_ok) return 2;
  const int elem = b->dtype == JQ_C64 ? 8 : 16;
  const int64_t bs = even(pl->bmat_stride);
  const size_t budget = 227 * 1024;
  if (n <= c.warp_max_qubits && batch_smem(c.warp_max_qubits, c.warp_threads / 32, elem, bs) <= budget) return 0;
  if (n <= c.cta_max_qubits && batch_smem(c.cta_max_qubits, 1, elem, bs) <= budget) return 1;
  if (n > c.cta_max_qubits && n <= c.cta_max_qubits + std::min(c.cluster_bits, 3) && pl->obs.size() <= 32 &&
      n <= 31 && batch_smem(c.cta_max_qubits, 1, elem, bs) <= budget)
    return 3;
  return 2;
}

// Clusters per SM slot of the cluster class (one 2^L slice per CTA).
int cluster_index(int n, int cta_max) { return n - cta_max - 1; }  // 0: 2 CTAs, 1: 4, 2: 8


int batch_classify(jq_batch* b, bool dry = false);

// Workspace bytes the batch needs under configuration c: classified on a
// copy, so the batch itself (class lists, offset tables, graph) is untouched.
size_t batch_ws_for(const jq_batch* b, const jq_batch_config& c) {
  jq_batch tmp;
  tmp.dtype = b->dtype;
  tmp.n_inst = b->n_inst;
  tmp.plans = b->plans;
  tmp.bplans = b->bplans;
  tmp.inst = b->inst;
  tmp.n_of_plan = b->n_of_plan;
  tmp.sm_count = b->sm_count;
  tmp.cfg = c;
  return batch_classify(&tmp, true) == JQ_OK ? tmp.ws_total : 0;
}

int batch_classify(jq_batch* b, bool dry) {
  const jq_batch_config& c = b->cfg;
  b->order_warp.clear();
  b->order_cta.clear();
  for (auto& v : b->order_cl) v.clear();
  b->tiles.clear();
  b->nmax_warp = b->nmax_cta = 0;
  std::vector<int> cls(b->plans.size());
  for (size_t p = 0; p < b->plans.size(); ++p) {
    cls[p] = plan_class(b, static_cast<int>(p), c);
    b->bplans[p].cls = cls[p];
  }
  std::vector<int> tile_of(b->plans.size(), -1);
  for (int i = 0; i < b->n_inst; ++i) {
    const int p = b->inst[i].plan;
    if (cls[p] == 0) {
      b->order_warp.push_back(i);
      b->nmax_warp = std::max(b->nmax_warp, b->n_of_plan[p]);
    } else if (cls[p] == 1) {
      b->order_cta.push_back(i);
      b->nmax_cta = std::max(b->nmax_cta, b->n_of_plan[p]);
    } else if (cls[p] == 3) {
      b->order_cl[cluster_index(b->n_of_plan[p], c.cta_max_qubits)].push_back(i);
    } else {
      if (tile_of[p] < 0) {
        tile_of[p] = static_cast<int>(b->tiles.size());
        b->tiles.push_back(jq_batch::TileGroup{p, {}, 0, 0});
      }
      b->tiles[tile_of[p]].members.push_back(i);
    }
  }
  auto by_cost = [&](int32_t x, int32_t y) {
    const int64_t cx = plan_cost(b, b->inst[x].plan), cy = plan_cost(b, b->inst[y].plan);
    return cx != cy ? cx > cy : x < y;
  };
  std::sort(b->order_warp.begin(), b->order_warp.end(), by_cost);
  std::sort(b->order_cta.begin(), b->order_cta.end(), by_cost);
  for (auto& v : b->order_cl) std::sort(v.begin(), v.end(), by_cost);
  b->bs_warp = b->bs_cta = b->bs_cl = 0;
  for (size_t p = 0; p < b->plans.size(); ++p) {
    const int64_t bs = even(b->plans[p]->bmat_stride);
    if (cls[p] == 0) b->bs_warp = std::max(b->bs_warp, bs);
    if (cls[p] == 1) b->bs_cta = std::max(b->bs_cta, bs);
    if (cls[p] == 3) b->bs_cl = std::max(b->bs_cl, bs);
  }
  const int elem = b->dtype == JQ_C64 ? 8 : 16;
  const int wgroups = c.warp_threads / 32;

  if (dry) {
    // workspace size only (same arithmetic as below)
    int64_t bs = 1, gsl = 1;
    for (size_t p = 0; p < b->plans.size(); ++p) {
      if (cls[p] == 2) continue;
      bs = std::max<int64_t>(bs, b->plans[p]->bmat_stride);
      gsl = std::max<int64_t>(gsl, b->plans[p]->grad_stride);
    }
    const int64_t slots = static_cast<int64_t>(b->sm_count) * (16 * (std::max(1, wgroups) + 1) + 3);
    size_t off = 256 + align256(static_cast<size_t>(slots) * gsl * 16);
    (void)bs;
    off += align256(static_cast<size_t>(3) * b->sm_count * 2 * (static_cast<size_t>(1) << c.cta_max_qubits) * elem);
    for (auto& tg : b->tiles) {
      const jq_plan* pl = b->plans[tg.plan];
      const int nb = static_cast<int>(tg.members.size());
      const size_t na = static_cast<size_t>(std::max(pl->n_angles, 1)) * nb * 8;
      const size_t no = static_cast<size_t>(std::max<size_t>(pl->obs.size(), 1)) * nb * 8;
      const size_t st = static_cast<size_t>(pl->state_elems) * elem * nb;
      off += align256(na) * 2 + align256(no) * 2 + align256(st);
      off += align256(std::max<size_t>(layout(pl, nb, 0).total, 1)) + align256(std::max<size_t>(layout(pl, nb, 1).total, 1));
    }
    b->ws_total = off;
    return JQ_OK;
  }
  // order table and tile-group offset table
  std::vector<int32_t> order(b->order_warp);
  order.insert(order.end(), b->order_cta.begin(), b->order_cta.end());
  for (auto& v : b->order_cl) order.insert(order.end(), v.begin(), v.end());
  if (order.empty()) order.push_back(0);
  std::vector<int64_t> toff;
  for (auto& tg : b->tiles) {
    tg.off_angles = static_cast<int64_t>(toff.size());
    for (int32_t i : tg.members) toff.push_back(b->inst[i].angle_off);
    tg.off_outs = static_cast<int64_t>(toff.size());
    for (int32_t i : tg.members) toff.push_back(b->inst[i].out_off);
  }
  if (toff.empty()) toff.push_back(0);
  if (b->d_order) cudaFree(b->d_order);
  if (b->d_tile_off) cudaFree(b->d_tile_off);
  b->d_order = b->d_tile_off = nullptr;
  JQ_CUDA(cudaMalloc(&b->d_order, order.size() * sizeof(int32_t)));
  JQ_CUDA(cudaMemcpy(b->d_order, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  JQ_CUDA(cudaMalloc(&b->d_tile_off, toff.size() * sizeof(int64_t)));
  JQ_CUDA(cudaMemcpy(b->d_tile_off, toff.data(), toff.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  // register-stage programs of the cluster class (they depend on the local bits L)
  b->rstg.clear();
  b->rop.clear();
  for (size_t p = 0; p < b->plans.size(); ++p) {
    BPlan& bp = b->bplans[p];
    bp.stg_off = bp.n_stg = 0;
    if (cls[p] != 3) continue;
    bp.stg_off = static_cast<int32_t>(b->rstg.size());
    build_rstages(b->bblk.data() + bp.blk_off, bp.nblocks, b->n_of_plan[p], c.cta_max_qubits, &b->rstg, &b->rop);
    bp.n_stg = static_cast<int32_t>(b->rstg.size()) - bp.stg_off;
  }
  if (b->d_rstg) cudaFree(b->d_rstg);
  if (b->d_rop) cudaFree(b->d_rop);
  b->d_rstg = b->d_rop = nullptr;
  JQ_CUDA(cudaMalloc(&b->d_rstg, std::max<size_t>(1, b->rstg.size()) * sizeof(RStage)));
  JQ_CUDA(cudaMalloc(&b->d_rop, std::max<size_t>(1, b->rop.size()) * sizeof(RPacked)));
  if (!b->rstg.empty())
    JQ_CUDA(cudaMemcpy(b->d_rstg, b->rstg.data(), b->rstg.size() * sizeof(RStage), cudaMemcpyHostToDevice));
  if (!b->rop.empty())
    JQ_CUDA(cudaMemcpy(b->d_rop, b->rop.data(), b->rop.size() * sizeof(RPacked), cudaMemcpyHostToDevice));
  JQ_CUDA(cudaMemcpy(b->d_plans, b->bplans.data(), b->bplans.size() * sizeof(BPlan), cudaMemcpyHostToDevice));
  // workspace: counters, per-slot block matrices and cotangents, tile groups
  int64_t bs = 1, gsl = 1;
  for (size_t p = 0; p < b->plans.size(); ++p) {
    if (cls[p] == 2) continue;
    bs = std::max<int64_t>(bs, b->plans[p]->bmat_stride);
    gsl = std::max<int64_t>(gsl, b->plans[p]->grad_stride);
  }
  b->bmat_slot = bs;
  b->gacc_slot = gsl;
  // the two shared-memory kernels run concurrently: warp-class slots first,
  // then one slot per CTA of the cta-class kernel
  b->slots_warp = static_cast<int64_t>(b->sm_count) * 16 * std::max(1, wgroups);
  // then one slot per CTA of the cta-class kernel, then 3 x sm_count for the
  // three cluster launches (at most one cluster-class CTA per SM each)
  const int64_t slots = b->slots_warp + static_cast<int64_t>(b->sm_count) * 16 + 3LL * b->sm_count;
  size_t off = 0;
  b->ws_counter = off;
  off += 256;
  b->ws_gacc = off;
  off += align256(static_cast<size_t>(slots) * gsl * 16);
  b->ws_cl_xs = off;
  off += align256(static_cast<size_t>(3) * b->sm_count * 2 * (static_cast<size_t>(1) << c.cta_max_qubits) * elem);
  b->ws_tile.clear();
  b->ws_tile_fwd.clear();
  b->ws_tile_adj.clear();
  for (auto& tg : b->tiles) {
    const jq_plan* pl = b->plans[tg.plan];
    const int nb = static_cast<int>(tg.members.size());
    const size_t na = static_cast<size_t>(std::max(pl->n_angles, 1)) * nb * 8;
    const size_t no = static_cast<size_t>(std::max<size_t>(pl->obs.size(), 1)) * nb * 8;
    const size_t st = static_cast<size_t>(pl->state_elems) * elem * nb;
    const size_t wf = layout(pl, nb, 0).total, wa = layout(pl, nb, 1).total;
    b->ws_tile.push_back(off);  // angles, ct, outs, grads, state, fwd ws, adj ws
    off += align256(na) * 2 + align256(no) * 2 + align256(st);
    b->ws_tile_fwd.push_back(off);
    off += align256(std::max<size_t>(wf, 1));
    b->ws_tile_adj.push_back(off);
    off += align256(std::max<size_t>(wa, 1));
  }
  b->ws_total = off;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return JQ_OK;
}

template <typename R>
int batch_launch_smem(jq_batch* b, bool warp, const double* angles, const double* ct, double* expval, double* grad,
                      char* w, cudaStream_t st) {
  const std::vector<int32_t>& ord = warp ? b->order_warp : b->order_cta;
  if (ord.empty()) return JQ_OK;
  const int elem = static_cast<int>(sizeof(typename CplxT<R>::T));
  BatchArgs a;
  a.plans = static_cast<const BPlan*>(b->d_plans);
  a.inst = static_cast<const BInst*>(b->d_inst);
  a.order = static_cast<const int32_t*>(b->d_order) + (warp ? 0 : b->order_warp.size());
  a.n_order = static_cast<int>(ord.size());
  a.nmax = warp ? b->nmax_warp : b->nmax_cta;
  a.bblk = static_cast<const BBlock*>(b->d_bblk);
  a.dblk = static_cast<const DevBlock*>(b->d_dblk);
  a.prims = static_cast<const DevPrim*>(b->d_prims);
  a.ops = static_cast<const DevOp*>(b->d_ops);
  a.cpool = static_cast<const double2*>(b->d_cpool);
  a.obs = static_cast<const DevObs*>(b->d_obs);
  a.angles = angles;
  a.ct = ct;
  a.expval = expval;
  a.grad = grad;
  const int64_t slot0 = warp ? 0 : b->slots_warp;
  a.gacc_ws = reinterpret_cast<double2*>(w + b->ws_gacc) + slot0 * b->gacc_slot;
  a.bmat_slot = warp ? b->bs_warp : b->bs_cta;
  a.gacc_slot = b->gacc_slot;
  a.counter = reinterpret_cast<int*>(w + b->ws_counter) + (warp ? 0 : 1);
  const int threads = warp ? b->cfg.warp_threads : b->cfg.cta_threads;
  const int groups = warp ? threads / 32 : 1;
  const size_t smem = batch_smem(a.nmax, groups, elem, a.bmat_slot);
  auto kern = warp ? k_batch<R, true> : k_batch<R, false>;
  JQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int per_sm = 0;
  JQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
  if (per_sm < 1) {
    set_error("batch kernel does not fit on an SM with this configuration");
    return JQ_EINVAL;
  }
  per_sm = std::min(per_sm, 16);
  const int64_t need = (static_cast<int64_t>(ord.size()) + groups - 1) / groups;
  const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(need, static_cast<int64_t>(b->sm_count) * per_sm)));
  kern<<<grid, threads, smem, st>>>(a);
  JQ_CUDA(cudaGetLastError());
  return JQ_OK;
}

template <typename R, int CL>
int batch_launch_cluster(jq_batch* b, int ci, const double* angles, const double* ct, double* expval, double* grad,
                         char* w, cudaStream_t st) {
  const std::vector<int32_t>& ord = b->order_cl[ci];
  if (ord.empty()) return JQ_OK;
  const int elem = static_cast<int>(sizeof(typename CplxT<R>::T));
  const int lbits = b->cfg.cta_max_qubits;
  ClusterArgs ca;
  BatchArgs& a = ca.a;
  size_t before = b->order_warp.size() + b->order_cta.size();
  for (int i = 0; i < ci; ++i) before += b->order_cl[i].size();
  a.plans = static_cast<const BPlan*>(b->d_plans);
  a.inst = static_cast<const BInst*>(b->d_inst);
  a.order = static_cast<const int32_t*>(b->d_order) + before;
  a.n_order = static_cast<int>(ord.size());
  a.nmax = lbits;
  a.bblk = static_cast<const BBlock*>(b->d_bblk);
  a.dblk = static_cast<const DevBlock*>(b->d_dblk);
  a.prims = static_cast<const DevPrim*>(b->d_prims);
  a.ops = static_cast<const DevOp*>(b->d_ops);
  a.cpool = static_cast<const double2*>(b->d_cpool);
  a.obs = static_cast<const DevObs*>(b->d_obs);
  a.angles = angles;
  a.ct = ct;
  a.expval = expval;
  a.grad = grad;
  // CTA slots (block matrices) and cluster slots (cotangents) after the
  // warp- and cta-class slots; sm_count of each per cluster launch
  const int64_t slot0 = b->slots_warp + static_cast<int64_t>(b->sm_count) * 16 + static_cast<int64_t>(ci) * b->sm_count;
  a.gacc_ws = reinterpret_cast<double2*>(w + b->ws_gacc) + slot0 * b->gacc_slot;
  a.bmat_slot = b->bs_cl;
  a.gacc_slot = b->gacc_slot;
  a.counter = reinterpret_cast<int*>(w + b->ws_counter) + 2 + ci;
  ca.lbits = lbits;
  ca.xs_ws = w + b->ws_cl_xs + static_cast<size_t>(ci) * b->sm_count * 2 * (static_cast<size_t>(1) << lbits) * elem;
  ca.stg = static_cast<const RStage*>(b->d_rstg);
  ca.rop = static_cast<const RPacked*>(b->d_rop);
  const int threads = b->cfg.cta_threads;
  size_t smem = batch_smem(lbits, 1, elem, a.bmat_slot);
  auto kern = k_batch_cluster<R, CL>;
  if constexpr (std::is_same<R, float>::value) {
    if (batch_rs_ok(b, elem)) {
      kern = k_batch_rs<CL>;
      smem += static_cast<size_t>(a.gacc_slot) * 8;
    }
  }
  JQ_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(CL * 16, 1, 1);
  int max_clusters = 0;
  JQ_CUDA(cudaOccupancyMaxActiveClusters(&max_clusters, kern, &cfg));
  if (max_clusters < 1) {
    set_error("batch cluster kernel does not fit with this configuration");
    return JQ_EINVAL;
  }
  const int64_t cap = std::max<int64_t>(1, std::min<int64_t>(max_clusters, b->sm_count / CL));
  const int64_t nclusters = std::max<int64_t>(1, std::min<int64_t>(static_cast<int64_t>(ord.size()), cap));
  cfg.gridDim = dim3(static_cast<unsigned>(nclusters * CL), 1, 1);
  JQ_CUDA(cudaLaunchKernelEx(&cfg, kern, ca));
  return JQ_OK;
}

template <typename R>
int batch_tile_group(jq_batch* b, size_t g, const double* angles, const double* ct, double* expval, double* grad,
                     char* w, cudaStream_t st) {
  const jq_batch::TileGroup& tg = b->tiles[g];
  const jq_plan* pl = b->plans[tg.plan];
  const int nb = static_cast<int>(tg.members.size());
  const int elem = static_cast<int>(sizeof(typename CplxT<R>::T));
  const int na = pl->n_angles, no = static_cast<int>(pl->obs.size());
  char* base = w + b->ws_tile[g];
  double* g_ang = reinterpret_cast<double*>(base);
  const size_t sa = align256(static_cast<size_t>(std::max(na, 1)) * nb * 8);
  const size_t so = align256(static_cast<size_t>(std::max(no, 1)) * nb * 8);
  double* g_grad = reinterpret_cast<double*>(base + sa);
  double* g_ct = reinterpret_cast<double*>(base + 2 * sa);
  double* g_out = reinterpret_cast<double*>(base + 2 * sa + so);
  void* g_state = base + 2 * sa + 2 * so;
  const int64_t* toff = static_cast<const int64_t*>(b->d_tile_off);
  const int threads = 256;
  auto grid_of = [&](int64_t total) {
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((total + threads - 1) / threads, 4096)));
  };
  if (na > 0) {
    k_gather_rows<<<grid_of(static_cast<int64_t>(na) * nb), threads, 0, st>>>(angles, toff + tg.off_angles, nb, na,
                                                                               g_ang);
  }
  if (no > 0) {
    k_gather_rows<<<grid_of(static_cast<int64_t>(no) * nb), threads, 0, st>>>(ct, toff + tg.off_outs, nb, no, g_ct);
  }
  JQ_CUDA(cudaGetLastError());
  int rc = forward_impl<R>(pl, nb, na ? g_ang : nullptr, nullptr, nullptr, 0, JQ_OUT_EXPVAL, g_state, g_out,
                           w + b->ws_tile_fwd[g], layout(pl, nb, 0).total, st);
  if (rc) return rc;
  if (na > 0) JQ_CUDA(cudaMemsetAsync(g_grad, 0, static_cast<size_t>(na) * nb * 8, st));
  rc = adjoint_impl<R>(pl, nb, na ? g_ang : nullptr, nullptr, g_state, JQ_OUT_EXPVAL, g_ct, nullptr,
                       na ? g_grad : nullptr, nullptr, nullptr, w + b->ws_tile_adj[g], layout(pl, nb, 1).total, st);
  if (rc) return rc;
  if (no > 0)
    k_scatter_rows<<<grid_of(static_cast<int64_t>(no) * nb), threads, 0, st>>>(g_out, toff + tg.off_outs, nb, no,
                                                                                expval);
  if (na > 0)
    k_scatter_rows<<<grid_of(static_cast<int64_t>(na) * nb), threads, 0, st>>>(g_grad, toff + tg.off_angles, nb, na,
                                                                                grad);
  JQ_CUDA(cudaGetLastError());
  (void)elem;
  return JQ_OK;
}

// Everything of one run on `st` (with the side streams forked and joined):
// the host enqueues only, so the same sequence is captured into the graph.
template <typename R>
int batch_enqueue(jq_batch* b, const double* angles, const double* ct, double* expval, double* grad, char* w,
                  cudaStream_t st) {
  JQ_CUDA(cudaMemsetAsync(w + b->ws_counter, 0, 256, st));
  if (b->n_angles_total > 0) JQ_CUDA(cudaMemsetAsync(grad, 0, static_cast<size_t>(b->n_angles_total) * 8, st));
  JQ_CUDA(cudaEventRecord(b->ev[0], st));
  for (int i = 0; i < 5; ++i) JQ_CUDA(cudaStreamWaitEvent(b->side[i], b->ev[0], 0));
  int rc;
  // largest work first: clusters of 8, 4, 2 CTAs on side streams 2..4, tile
  // groups on side stream 0, warp class on side stream 1, cta class on st
  if ((rc = batch_launch_cluster<R, 8>(b, 2, angles, ct, expval, grad, w, b->side[2]))) return rc;
  if ((rc = batch_launch_cluster<R, 4>(b, 1, angles, ct, expval, grad, w, b->side[3]))) return rc;
  if ((rc = batch_launch_cluster<R, 2>(b, 0, angles, ct, expval, grad, w, b->side[4]))) return rc;
  for (size_t g = 0; g < b->tiles.size(); ++g)
    if ((rc = batch_tile_group<R>(b, g, angles, ct, expval, grad, w, b->side[0]))) return rc;
  if ((rc = batch_launch_smem<R>(b, true, angles, ct, expval, grad, w, b->side[1]))) return rc;
  if ((rc = batch_launch_smem<R>(b, false, angles, ct, expval, grad, w, st))) return rc;
  for (int i = 0; i < 5; ++i) {
    JQ_CUDA(cudaEventRecord(b->ev[1 + i], b->side[i]));
    JQ_CUDA(cudaStreamWaitEvent(st, b->ev[1 + i], 0));
  }
  return JQ_OK;
}

}  // namespace
}  // namespace jq

namespace jq {
namespace {
