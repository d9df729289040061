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
};

struct BPlan {
  int32_t n, nblocks, blk_off;     // BBlock and DevBlock rows [blk_off, blk_off + nblocks)
  int32_t n_angles, obs_off, n_obs;
  int32_t bmat_stride, grad_stride;
  int32_t cls;                     // 0 warp, 1 cta, 2 tile
};

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
  void* bmat_ws;         // per group slot: bmat_slot run-dtype complex
  double2* gacc_ws;      // per group slot: gacc_slot complex128
  int64_t bmat_slot, gacc_slot;
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

// Forward application of one block to the n-qubit state s.
template <typename C>
__device__ void bapply(C* s, int n, const BBlock& B, const C* bm, int lt, int gs) {
  const int dim = 1 << n;
  const C* M = bm + B.mat_off;
  if (B.kind == BK_DIAG) {
    for (int j = lt; j < dim; j += gs) {
      if ((static_cast<uint32_t>(j) & B.cmask) != B.cmask) continue;
      const int r = (B.nt == 1) ? ((j >> B.tb0) & 1) : ((((j >> B.tb0) & 1) << 1) | ((j >> B.tb1) & 1));
      s[j] = cmul(M[r], s[j]);
    }
    return;
  }
  if (B.nt == 1) {
    const int q = B.tb0;
    for (int g = lt; g < (dim >> 1); g += gs) {
      const int i0 = ins0(g, q);
      if ((static_cast<uint32_t>(i0) & B.cmask) != B.cmask) continue;
      const int i1 = i0 | (1 << q);
      const C x = s[i0], y = s[i1];
      if (B.kind == BK_PERM) {
        if (B.perm & 1) { s[i0] = y; s[i1] = x; }
      } else {
        s[i0] = cfma(M[1], y, cmul(M[0], x));
        s[i1] = cfma(M[3], y, cmul(M[2], x));
      }
    }
    return;
  }
  const int lo = min(B.tb0, B.tb1), hi = max(B.tb0, B.tb1);
  for (int g = lt; g < (dim >> 2); g += gs) {
    const int i = ins0(ins0(g, lo), hi);
    if ((static_cast<uint32_t>(i) & B.cmask) != B.cmask) continue;
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

// Adjoint of one block: psi <- G^dagger psi, cotangent += lam psi^dagger
// (psi after the un-apply), lam <- G^dagger lam.
template <typename C, bool WARP>
__device__ void badjoint(C* sp, C* sl, int n, const BBlock& B, const C* bm, double* ga, int lt, int gs) {
  const int dim = 1 << n;
  const C* M = bm + B.mat_off;
  const bool grad = ga && B.grad_off >= 0;
  double* gdst = grad ? ga + 2 * B.grad_off : nullptr;
  if (B.kind == BK_DIAG) {
    double g[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) g[e] = 0.0;
    for (int j = lt; j < dim; j += gs) {
      if ((static_cast<uint32_t>(j) & B.cmask) != B.cmask) continue;
      const int r = (B.nt == 1) ? ((j >> B.tb0) & 1) : ((((j >> B.tb0) & 1) << 1) | ((j >> B.tb1) & 1));
      const C d = cconj(M[r]);
      const C p = cmul(d, sp[j]);
      const C l = sl[j];
      sp[j] = p;
      sl[j] = cmul(d, l);
      const double2 v = cmul(to_d2(l), cconj(to_d2(p)));
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (q == r) { g[2 * q] += v.x; g[2 * q + 1] += v.y; }
    }
    if (grad) gacc_add<WARP, 8>(g, gdst);
    return;
  }
  if (B.nt == 1) {
    const int q = B.tb0;
    double g[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) g[e] = 0.0;
    for (int gi = lt; gi < (dim >> 1); gi += gs) {
      const int i0 = ins0(gi, q);
      if ((static_cast<uint32_t>(i0) & B.cmask) != B.cmask) continue;
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
      const double2 du = to_d2(u), dw = to_d2(w), d0 = cconj(to_d2(p0)), d1 = cconj(to_d2(p1));
      const double2 g00 = cmul(du, d0), g01 = cmul(du, d1), g10 = cmul(dw, d0), g11 = cmul(dw, d1);
      g[0] += g00.x; g[1] += g00.y; g[2] += g01.x; g[3] += g01.y;
      g[4] += g10.x; g[5] += g10.y; g[6] += g11.x; g[7] += g11.y;
      sl[i0] = cfma(h01, w, cmul(h00, u));
      sl[i1] = cfma(h11, w, cmul(h10, u));
    }
    if (grad) gacc_add<WARP, 8>(g, gdst);
    return;
  }
  const int lo = min(B.tb0, B.tb1), hi = max(B.tb0, B.tb1);
  double g[32];
#pragma unroll
  for (int e = 0; e < 32; ++e) g[e] = 0.0;
  for (int gi = lt; gi < (dim >> 2); gi += gs) {
    const int i = ins0(ins0(gi, lo), hi);
    if ((static_cast<uint32_t>(i) & B.cmask) != B.cmask) continue;
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
    for (int r = 0; r < 4; ++r) {
      const double2 lr = to_d2(b[r]);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double2 v = cmul(lr, cconj(to_d2(p[q])));
        g[2 * (4 * r + q)] += v.x;
        g[2 * (4 * r + q) + 1] += v.y;
      }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      C acc = cmul(cconj(M[r]), b[0]);
#pragma unroll
      for (int q = 1; q < 4; ++q) acc = cfma(cconj(M[4 * q + r]), b[q], acc);
      sl[id[r]] = acc;
    }
  }
  if (grad) gacc_add<WARP, 32>(g, gdst);
}

template <typename R, bool WARP>
__global__ void __launch_bounds__(512) k_batch(BatchArgs a) {
  using C = typename CplxT<R>::T;
  extern __shared__ __align__(16) unsigned char smem[];
  const int gs = WARP ? 32 : static_cast<int>(blockDim.x);
  const int ngroups = WARP ? static_cast<int>(blockDim.x >> 5) : 1;
  const int gid = WARP ? static_cast<int>(threadIdx.x >> 5) : 0;
  const int lt = WARP ? static_cast<int>(threadIdx.x & 31) : static_cast<int>(threadIdx.x);
  const int dmax = 1 << a.nmax;
  C* sp = reinterpret_cast<C*>(smem) + static_cast<int64_t>(gid) * 2 * dmax;
  C* sl = sp + dmax;
  double* red = reinterpret_cast<double*>(reinterpret_cast<C*>(smem) + static_cast<int64_t>(ngroups) * 2 * dmax);
  int* snext = reinterpret_cast<int*>(red + 32);
  const int64_t slot = static_cast<int64_t>(blockIdx.x) * ngroups + gid;
  C* bm = static_cast<C*>(a.bmat_ws) + slot * a.bmat_slot;
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
    for (int b = 0; b < P.nblocks; ++b) {
      bapply<C>(sp, n, BB[b], bm, lt, gs);
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
    for (int b = P.nblocks - 1; b >= 0; --b) {
      badjoint<C, WARP>(sp, sl, n, BB[b], bm, reinterpret_cast<double*>(gacc), lt, gs);
      gsync<WARP>();
    }
    for (int b = lt; b < P.nblocks; b += gs)
      chain_block(a.dblk[P.blk_off + b], a.prims, a.ops, ang, nullptr, a.cpool, gacc, nullptr, a.grad + I.angle_off,
                  nullptr);
    gsync<WARP>();
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
  void* d_order = nullptr;     // warp-class order then cta-class order
  void* d_tile_off = nullptr;  // per tile group: angle offsets then output offsets of its instances
  // classes under the current configuration
  std::vector<int32_t> order_warp, order_cta;
  struct TileGroup {
    int plan;
    std::vector<int32_t> members;
    int64_t off_angles = 0, off_outs = 0;  // offsets into d_tile_off (int64 entries)
  };
  std::vector<TileGroup> tiles;
  int nmax_warp = 0, nmax_cta = 0;
  int64_t bmat_slot = 0, gacc_slot = 0, slots_warp = 0;
  // workspace layout
  size_t ws_total = 0, ws_counter = 0, ws_bmat = 0, ws_gacc = 0;
  std::vector<size_t> ws_tile;  // per tile group: angles, ct, outs, grads, state, fwd ws, adj ws
  std::vector<size_t> ws_tile_fwd, ws_tile_adj;
  // side streams and the captured graph
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaStream_t cap = nullptr;   // the graph is captured on this stream
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaGraphExec_t graph = nullptr;
  const void* graph_key[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int sm_count = 0;
};

namespace jq {
namespace {

int64_t plan_cost(const jq_batch* b, int p) {
  return (static_cast<int64_t>(1) << b->n_of_plan[p]) * std::max(1, b->bplans[p].nblocks);
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
  if (n <= c.warp_max_qubits) return 0;
  if (n <= c.cta_max_qubits) return 1;
  return 2;
}

size_t batch_smem(int nmax, int groups, int elem) {
  return static_cast<size_t>(groups) * 2 * (static_cast<size_t>(1) << nmax) * elem + 32 * 8 + 16;
}

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
  const int elem = b->dtype == JQ_C64 ? 8 : 16;
  const int wgroups = c.warp_threads / 32;
  if (!b->order_warp.empty() && batch_smem(b->nmax_warp, wgroups, elem) > 227 * 1024) {
    set_error("warp-class shared memory above 227 KB: lower warp_max_qubits or warp_threads");
    return JQ_EINVAL;
  }
  if (!b->order_cta.empty() && batch_smem(b->nmax_cta, 1, elem) > 227 * 1024) {
    set_error("cta-class shared memory above 227 KB: lower cta_max_qubits");
    return JQ_EINVAL;
  }
  if (dry) {
    // workspace size only (same arithmetic as below)
    int64_t bs = 1, gsl = 1;
    for (size_t p = 0; p < b->plans.size(); ++p) {
      if (cls[p] == 2) continue;
      bs = std::max<int64_t>(bs, b->plans[p]->bmat_stride);
      gsl = std::max<int64_t>(gsl, b->plans[p]->grad_stride);
    }
    const int64_t slots = static_cast<int64_t>(b->sm_count) * 16 * (std::max(1, wgroups) + 1);
    size_t off = 256 + align256(static_cast<size_t>(slots) * bs * elem) + align256(static_cast<size_t>(slots) * gsl * 16);
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
  const int64_t slots = b->slots_warp + static_cast<int64_t>(b->sm_count) * 16;
  size_t off = 0;
  b->ws_counter = off;
  off += 256;
  b->ws_bmat = off;
  off += align256(static_cast<size_t>(slots) * bs * elem);
  b->ws_gacc = off;
  off += align256(static_cast<size_t>(slots) * gsl * 16);
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
  a.bmat_ws = w + b->ws_bmat + static_cast<size_t>(slot0 * b->bmat_slot) * elem;
  a.gacc_ws = reinterpret_cast<double2*>(w + b->ws_gacc) + slot0 * b->gacc_slot;
  a.bmat_slot = b->bmat_slot;
  a.gacc_slot = b->gacc_slot;
  a.counter = reinterpret_cast<int*>(w + b->ws_counter) + (warp ? 0 : 1);
  const int threads = warp ? b->cfg.warp_threads : b->cfg.cta_threads;
  const int groups = warp ? threads / 32 : 1;
  const size_t smem = batch_smem(a.nmax, groups, elem);
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
  JQ_CUDA(cudaStreamWaitEvent(b->side[0], b->ev[0], 0));
  JQ_CUDA(cudaStreamWaitEvent(b->side[1], b->ev[0], 0));
  int rc;
  // tile groups on side stream 0, warp class on side stream 1, cta class on st
  for (size_t g = 0; g < b->tiles.size(); ++g)
    if ((rc = batch_tile_group<R>(b, g, angles, ct, expval, grad, w, b->side[0]))) return rc;
  if ((rc = batch_launch_smem<R>(b, true, angles, ct, expval, grad, w, b->side[1]))) return rc;
  if ((rc = batch_launch_smem<R>(b, false, angles, ct, expval, grad, w, st))) return rc;
  JQ_CUDA(cudaEventRecord(b->ev[1], b->side[0]));
  JQ_CUDA(cudaEventRecord(b->ev[2], b->side[1]));
  JQ_CUDA(cudaStreamWaitEvent(st, b->ev[1], 0));
  JQ_CUDA(cudaStreamWaitEvent(st, b->ev[2], 0));
  return JQ_OK;
}

}  // namespace
}  // namespace jq

namespace jq {
namespace {
