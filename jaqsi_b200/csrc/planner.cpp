// Host planner of libjqsim: lowers a recorded tape into prims on the
// (2n-)bit vector, fuses them into blocks and schedules the blocks into tile
// passes.  No CUDA call is made here, so plans can be built and inspected on
// a machine without a GPU.
//
// Reference behaviour restated (jaqsi/simulation.py):
//   _fuse             :214-240  same-wire fusion rule (kept exactly, plus a cap
//                               on the run length)
//   _fused_structure  :202-211  structure of a fused product
//   _compile_mixed    :348-381  gates and channels as superoperators on the
//                               (ket, bra) axes of the density tensor
// The pass scheduler has no reference counterpart: the reference runs one
// XLA pass per fused entry, here one pass applies every block whose bits fit
// in the pass's tile.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "jq_internal.h"

namespace jq {

using cd = std::complex<double>;

thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

namespace {

struct HostPrim {
  int op = -1;
  int form = PF_U;
  std::vector<int> wires;      // wires on the bit vector (n or 2n wires)
  Structure st;
  std::vector<cd> cmat;        // PF_CONST: full matrix
};

struct HostBlock {
  std::vector<int> wires;
  Structure st;
  std::vector<int> prims;
  bool unitary = true;  // every prim is a unitary gate: the block is undone exactly by its dagger
};

std::vector<cd> read_matrix(const double* p, int dim) {
  std::vector<cd> m(static_cast<size_t>(dim) * dim);
  for (size_t i = 0; i < m.size(); ++i) m[i] = cd(p[2 * i], p[2 * i + 1]);
  return m;
}

std::vector<cd> kron(const std::vector<cd>& a, int da, const std::vector<cd>& b, int db) {
  int d = da * db;
  std::vector<cd> r(static_cast<size_t>(d) * d);
  for (int i = 0; i < da; ++i)
    for (int j = 0; j < da; ++j)
      for (int p = 0; p < db; ++p)
        for (int q = 0; q < db; ++q)
          r[static_cast<size_t>(i * db + p) * d + (j * db + q)] = a[i * da + j] * b[p * db + q];
  return r;
}

std::vector<cd> conj_of(const std::vector<cd>& a) {
  std::vector<cd> r(a.size());
  for (size_t i = 0; i < a.size(); ++i) r[i] = std::conj(a[i]);
  return r;
}

// Structure read off the values of a constant matrix: diagonal, permutation
// (exact 0/1 entries) and leading controls (identity on every index whose
// control bits are not all one).
Structure detect_structure(const std::vector<cd>& m, int k) {
  Structure st;
  int d = 1 << k;
  bool diag = true, perm = true;
  std::vector<int32_t> p(d, -1);
  for (int i = 0; i < d; ++i) {
    int ones = 0;
    for (int j = 0; j < d; ++j) {
      cd v = m[static_cast<size_t>(i) * d + j];
      if (i != j && v != cd(0, 0)) diag = false;
      if (v == cd(1, 0)) {
        ++ones;
        p[i] = j;
      } else if (v != cd(0, 0)) {
        perm = false;
      }
    }
    if (ones != 1) perm = false;
  }
  if (perm) {
    std::vector<int> seen(d, 0);
    for (int i = 0; i < d; ++i) {
      if (p[i] < 0 || seen[p[i]]) { perm = false; break; }
      seen[p[i]] = 1;
    }
  }
  st.diagonal = diag;
  if (perm) st.perm = p;
  // controls: largest c such that m = I (+) inner with inner 2^(k-c) square
  for (int c = k - 1; c >= 1; --c) {
    int inner = 1 << (k - c);
    int base = d - inner;
    bool ok = true;
    for (int i = 0; i < d && ok; ++i)
      for (int j = 0; j < d && ok; ++j) {
        if (i >= base && j >= base) continue;
        cd want = (i == j) ? cd(1, 0) : cd(0, 0);
        if (m[static_cast<size_t>(i) * d + j] != want) ok = false;
      }
    if (ok) { st.controls = c; break; }
  }
  return st;
}

// GateStructure of a product right @ left on identical wires
// (jaqsi/simulation.py:202-211).
Structure fused_structure(const Structure& left, const Structure& right) {
  Structure st;
  if (!left.perm.empty() && !right.perm.empty()) {
    st.perm.resize(right.perm.size());
    for (size_t i = 0; i < right.perm.size(); ++i) st.perm[i] = left.perm[right.perm[i]];
  }
  st.diagonal = left.diagonal && right.diagonal;
  st.controls = std::min(left.controls, right.controls);
  return st;
}

int popcount64(uint64_t x) { return __builtin_popcountll(x); }

bool validate_perm(const std::vector<int32_t>& p, int d) {
  if (static_cast<int>(p.size()) != d) return false;
  std::vector<int> seen(d, 0);
  for (int v : p) {
    if (v < 0 || v >= d || seen[v]) return false;
    seen[v] = 1;
  }
  return true;
}

// Greedy tile-pass scheduler.  Walks the blocks in program order; a block
// joins the current pass when none of its bits is blocked and the pass's bit
// set stays within t bits; otherwise its bits become blocked for the rest of
// the pass (a later block on those bits must follow it).  Members of a pass
// therefore never depend on a deferred block, and program order is kept.
Schedule schedule(const std::vector<HostBlock>& blocks, const std::vector<DevBlock>& dblocks,
                  int nb, int t_max, int c_seed, bool one_per_pass) {
  Schedule s;
  s.t = t_max;
  int nblk = static_cast<int>(blocks.size());
  std::vector<char> done(nblk, 0);
  int cursor = 0;
  const uint64_t all_bits = (nb >= 64) ? ~0ULL : ((1ULL << nb) - 1);
  auto block_bits = [&](int b) {
    uint64_t m = 0;
    for (int w : blocks[b].wires) m |= 1ULL << (nb - 1 - w);
    return m;
  };
  while (cursor < nblk) {
    uint64_t S = (c_seed >= 64) ? ~0ULL : ((1ULL << c_seed) - 1);
    uint64_t blocked = 0;
    std::vector<int> members;
    for (int b = cursor; b < nblk; ++b) {
      if (done[b]) continue;
      uint64_t bb = block_bits(b);
      if (bb & blocked) { blocked |= bb; continue; }
      if (popcount64(S | bb) <= t_max && !(one_per_pass && !members.empty())) {
        S |= bb;
        members.push_back(b);
        done[b] = 1;
      } else {
        blocked |= bb;
      }
      if ((blocked | 0) == all_bits) break;
    }
    while (cursor < nblk && done[cursor]) ++cursor;
    // Fill the tile up to t_max with the lowest free bits: the same ops then
    // run on fewer, larger tiles (longer contiguous runs, fewer per-tile
    // reductions), which matters most for one-block passes.
    for (int bit = 0; bit < nb && popcount64(S) < t_max; ++bit) S |= 1ULL << bit;
    PassDesc pd;
    std::memset(&pd, 0, sizeof(pd));
    int t = 0;
    for (int bit = 0; bit < nb; ++bit)
      if (S >> bit & 1ULL) pd.bits[t++] = static_cast<int8_t>(bit);
    pd.t = t;
    pd.tile_mask = S;
    int c = 0;
    while (c < t && pd.bits[c] == c) ++c;
    pd.c = c;
    pd.op_begin = static_cast<int32_t>(s.ops.size());
    int rank[64];
    for (int i = 0; i < 64; ++i) rank[i] = -1;
    for (int i = 0; i < t; ++i) rank[pd.bits[i]] = i;
    for (int b : members) {
      const DevBlock& db = dblocks[b];
      TileOp op;
      std::memset(&op, 0, sizeof(op));
      op.block = b;
      op.kind = db.kind;
      op.kt = db.k - db.n_ctrl;
      op.nfix = db.k;
      op.ctrl_mask = 0;
      int pos[kMaxBlockWires];
      for (int i = 0; i < db.k; ++i) {
        int bit = nb - 1 - blocks[b].wires[i];
        pos[i] = rank[bit];
        if (i < db.n_ctrl) op.ctrl_mask |= 1u << pos[i];
        else op.tmask[i - db.n_ctrl] = 1u << pos[i];
      }
      std::sort(pos, pos + db.k);
      for (int i = 0; i < db.k; ++i) op.lowmask[i] = (1u << pos[i]) - 1u;
      op.mat_off = db.mat_off;
      op.perm_off = db.perm_off;
      op.grad_off = db.grad_off;
      op.inv = blocks[b].unitary ? 1 : 0;
      s.ops.push_back(op);
    }
    pd.op_end = static_cast<int32_t>(s.ops.size());
    s.passes.push_back(pd);
  }
  return s;
}

// Swizzled shared-memory offset of tile bit `pos` (linear over XOR): bank
// bits are folded from all higher bits so that any 4 (c64) / 3 (c128) lane
// bits with distinct residues hit distinct banks.
uint32_t swz_bit(int pos, int dtype) {
  const int nbank = (dtype == JQ_C64) ? 4 : 3;
  uint32_t v = 1u << pos;
  if (pos >= nbank) v |= 1u << (pos % nbank);
  return v;
}

// Register-stage program of every pass of `s` (see Step in jq_internal.h).
// Ops join the current stage greedily in program order while their targets
// fit in r register bits; an op that does not fit, or that touches a bit of a
// deferred op, is deferred to a later stage.  Ops with more targets than the
// register forms cover run as generic shared-memory steps.
void build_steps(Schedule& s, const std::vector<int32_t>& perm_pool, int dtype, const std::vector<uint8_t>& su2) {
  // register bits per stage (amplitudes per thread = 2^r); JQ_REG_BITS=3
  // selects 8 amplitudes per thread (more threads, more stages)
  int r = 4;
  if (const char* e = std::getenv("JQ_REG_BITS")) r = std::max(3, std::min(5, std::atoi(e)));
  s.reg_bits = r;
  for (PassDesc& pd : s.passes) {
    pd.step_begin = pd.step_end = static_cast<int32_t>(s.steps.size());
    pd.rop_begin = pd.rop_end = static_cast<int32_t>(s.rops.size());
    pd.smat_len = 0;
    int smat = 0;
    const int t = pd.t;
    if (t < r + 5 || t > r + 8) continue;  // 32..256 threads per CTA, else generic kernel
    std::vector<int> rem;
    for (int o = pd.op_begin; o < pd.op_end; ++o) rem.push_back(o);
    auto targets_of = [&](const TileOp& op) {
      uint32_t m = 0;
      for (int i = 0; i < op.kt; ++i) m |= op.tmask[i];
      return m;
    };
    auto reg_ok = [&](const TileOp& op) {
      if (op.kind == BK_DENSE) return op.kt <= 2;
      if (op.kind == BK_DIAG) return op.kt <= r;
      if (op.kind == BK_PERM) {
        if (op.kt == 2) return true;
        if (op.kt == 1) return perm_pool[op.perm_off] == 1 || perm_pool[op.perm_off] == 0;
        return false;
      }
      return false;
    };
    while (!rem.empty()) {
      uint32_t R = 0, blocked = 0;
      std::vector<int> members;
      int smem_op = -1;
      for (int o : rem) {
        const TileOp& op = s.ops[o];
        const uint32_t tg = targets_of(op), all = tg | op.ctrl_mask;
        if (all & blocked) { blocked |= all; continue; }
        if (!reg_ok(op)) {
          if (members.empty()) { smem_op = o; break; }
          blocked |= all;
          continue;
        }
        if (__builtin_popcount(R | tg) <= r) {
          R |= tg;
          members.push_back(o);
        } else {
          blocked |= all;
        }
      }
      Step st;
      std::memset(&st, 0, sizeof(st));
      if (smem_op >= 0) {
        st.kind = 1;
        st.a = smem_op;
        st.b = smem_op + 1;
        s.steps.push_back(st);
        rem.erase(std::find(rem.begin(), rem.end(), smem_op));
        continue;
      }
      // fill the register set with the highest free tile bits (lanes then
      // map to the lowest bits, which keeps shared memory conflict-free)
      for (int pos = t - 1; pos >= 0 && __builtin_popcount(R) < r; --pos) R |= 1u << pos;
      int rank_r[32], rank_t[32];
      int nr = 0, nt = 0;
      // Thread-bit order: the lowest lane bits (the lanes of one shared-memory
      // wavefront: 16 for 8-byte, 8 for 16-byte amplitudes) take positions of
      // distinct swizzle classes pos % nbank, so a stage access hits distinct
      // bank groups; the other thread bits follow in ascending order.
      const int nbank = (dtype == JQ_C64) ? 4 : 3;
      std::vector<int> tpos, first, rest;
      for (int pos = 0; pos < t; ++pos)
        if (!(R >> pos & 1u)) tpos.push_back(pos);
      uint32_t classes = 0;
      for (int pos : tpos) {
        const uint32_t cb = 1u << (pos % nbank);
        if (static_cast<int>(first.size()) < nbank && !(classes & cb)) {
          classes |= cb;
          first.push_back(pos);
        } else {
          rest.push_back(pos);
        }
      }
      first.insert(first.end(), rest.begin(), rest.end());
      for (int pos = 0; pos < t; ++pos) {
        rank_r[pos] = rank_t[pos] = -1;
        if (R >> pos & 1u) {
          st.ebits[nr] = swz_bit(pos, dtype);
          rank_r[pos] = nr++;
        }
      }
      for (int pos : first) {
        st.tbits[nt] = swz_bit(pos, dtype);
        rank_t[pos] = nt++;
      }
      st.kind = 0;
      st.a = static_cast<int32_t>(s.rops.size());
      for (int o : members) {
        const TileOp& op = s.ops[o];
        RegOp ro;
        std::memset(&ro, 0, sizeof(ro));
        auto qpos = [&](uint32_t mask) { return static_cast<uint32_t>(rank_r[__builtin_ctz(mask)]); };
        uint32_t crm = 0, ctm = 0;
        for (int pos = 0; pos < t; ++pos) {
          if (!(op.ctrl_mask >> pos & 1u)) continue;
          if (rank_r[pos] >= 0) crm |= 1u << rank_r[pos];
          else ctm |= 1u << rank_t[pos];
        }
        uint32_t kind = 0, q1 = 0, q2 = 0, dk = 0, dq = 0, perm = 0;
        int mat_len = 0;
        if (op.kind == BK_DENSE) {
          kind = op.kt == 1 ? RK_DENSE1 : RK_DENSE2;
          q1 = qpos(op.tmask[0]);
          q2 = op.kt == 2 ? qpos(op.tmask[1]) : 0;
          mat_len = (1 << op.kt) * (1 << op.kt);
          // pad[0]: the inner matrix is in SU(2) (m11 = conj m00, m10 = -conj m01)
          if (op.kt == 1 && op.block >= 0 && op.block < static_cast<int32_t>(su2.size()) && su2[op.block])
            ro.pad[0] = 1;
        } else if (op.kind == BK_DIAG) {
          kind = RK_DIAG;
          dk = static_cast<uint32_t>(op.kt);
          for (int i = 0; i < op.kt; ++i) dq |= qpos(op.tmask[i]) << (3 * i);
          mat_len = 1 << op.kt;
        } else if (op.kt == 1) {
          if (perm_pool[op.perm_off] == 0) continue;  // identity
          kind = RK_PERM1;
          q1 = qpos(op.tmask[0]);
        } else {
          kind = RK_PERM2;
          q1 = qpos(op.tmask[0]);
          q2 = qpos(op.tmask[1]);
          for (int i = 0; i < 4; ++i) perm |= static_cast<uint32_t>(perm_pool[op.perm_off + i]) << (2 * i);
        }
        ro.w0 = kind | (q1 << 4) | (q2 << 8) | (dk << 12) | (dq << 16);
        ro.w1 = crm | (ctm << 8) | (perm << 24);
        ro.w2 = static_cast<uint32_t>(smat);
        ro.w3 = static_cast<uint32_t>(op.mat_off < 0 ? 0 : op.mat_off);
        ro.mat_len = mat_len;
        ro.grad_off = (kind == RK_PERM1 || kind == RK_PERM2) ? -1 : op.grad_off;
        smat += mat_len;
        s.rops.push_back(ro);
      }
      st.b = static_cast<int32_t>(s.rops.size());
      s.steps.push_back(st);
      std::vector<int> left;
      for (int o : rem)
        if (std::find(members.begin(), members.end(), o) == members.end()) left.push_back(o);
      rem.swap(left);
    }
    pd.step_end = static_cast<int32_t>(s.steps.size());
    pd.rop_end = static_cast<int32_t>(s.rops.size());
    pd.smat_len = smat;
  }
}

int default_tile_bits(int nb, int dtype, int maxk, int c_seed, bool adjoint, bool density, bool grad) {
  // 16 amplitudes per thread, 128 threads per tile: small tiles leave
  // several CTAs per SM to hide shared-memory and barrier latency
  int t = 11;
  if (adjoint) t = 11;
  // Density matrices: the checkpointed reverse step keeps one tile per
  // register stage in shared memory, so smaller tiles fit more CTAs an SM.
  // Measured on the 12-qubit noisy circuit (forward + gradient per set):
  // complex64 51.7 / 48.3 / 63.9 ms at 11 / 10 / 9 bits (forward alone also
  // fastest at 10), complex128 98.4 / 93.4 / 89.2 ms (forward 13.7 / 14.1 /
  // 14.9 ms).
  if (density) t = (dtype == JQ_C128 && grad) ? 9 : 10;
  // keep at least ~256 tiles per state when the state is large enough
  int floor_t = std::max(std::min(t, 10), maxk + c_seed);
  if (nb - 8 < t) t = std::max(nb - 8, floor_t);
  t = std::max(t, maxk + c_seed);
  if (t > nb) t = nb;
  return t;
}

}  // namespace

int build_plan(const jq_op* ops, int n_ops, const jq_obs* obs, int n_obs, int n_qubits, int mode,
               int dtype, const jq_tune* tune, jq_plan** out) {
  if (!out) { set_error("jq_plan_build: out is NULL"); return JQ_EINVAL; }
  *out = nullptr;
  if (mode != JQ_STATEVECTOR && mode != JQ_DENSITY) { set_error("jq_plan_build: bad mode"); return JQ_EINVAL; }
  if (dtype != JQ_C64 && dtype != JQ_C128) { set_error("jq_plan_build: bad dtype"); return JQ_EINVAL; }
  if (n_qubits < 1 || n_qubits > JQ_MAX_QUBITS || (mode == JQ_DENSITY && n_qubits > JQ_MAX_QUBITS / 2)) {
    set_error("jq_plan_build: n_qubits out of range (" + std::to_string(n_qubits) + ")");
    return JQ_EINVAL;
  }
  if (n_ops < 0 || (n_ops > 0 && !ops) || n_obs < 0 || (n_obs > 0 && !obs)) {
    set_error("jq_plan_build: bad op / observable arrays");
    return JQ_EINVAL;
  }
  jq_plan* plan = new (std::nothrow) jq_plan();
  if (!plan) { set_error("jq_plan_build: out of host memory"); return JQ_ENOMEM; }
  plan->n_qubits = n_qubits;
  plan->mode = mode;
  plan->dtype = dtype;
  const int n = n_qubits;
  const int nb = (mode == JQ_DENSITY) ? 2 * n : n;
  plan->n_bits = nb;
  plan->state_elems = 1LL << nb;

  std::vector<HostPrim> prims;
  auto fail = [&](const std::string& msg) {
    set_error(msg);
    delete plan;
    return JQ_EINVAL;
  };

  // ---- ops -> DevOp + prims ------------------------------------------------
  for (int i = 0; i < n_ops; ++i) {
    const jq_op& o = ops[i];
    int k = o.n_wires;
    if (k < 1 || k > JQ_MAX_OP_WIRES) return fail("op " + std::to_string(i) + ": wire count out of range");
    for (int a = 0; a < k; ++a) {
      if (o.wires[a] < 0 || o.wires[a] >= n)
        return fail("op " + std::to_string(i) + ": wire " + std::to_string(o.wires[a]) + " outside 0.." + std::to_string(n - 1));
      for (int b = 0; b < a; ++b)
        if (o.wires[a] == o.wires[b]) return fail("op " + std::to_string(i) + ": duplicate wires");
    }
    DevOp d;
    std::memset(&d, 0, sizeof(d));
    d.kind = o.kind;
    d.k = k;
    d.n_ctrl = o.n_controls;
    d.angle_slot = o.angle_slot;
    d.mat_slot = o.mat_slot;
    d.mat_is_diag = o.mat_is_diag;
    d.px = o.pauli_x;
    d.pz = o.pauli_z;
    d.grad = o.grad;
    switch (o.kind) {
      case JQ_K_CONST: case JQ_K_MATRIX: case JQ_K_CHANNEL: d.n_angles = 0; break;
      case JQ_K_RX: case JQ_K_RY: case JQ_K_RZ: case JQ_K_CPHASE: case JQ_K_PAULIROT: d.n_angles = 1; break;
      case JQ_K_ROT: d.n_angles = 3; break;
      default: return fail("op " + std::to_string(i) + ": unknown kind " + std::to_string(o.kind));
    }
    if ((o.kind == JQ_K_RX || o.kind == JQ_K_RY || o.kind == JQ_K_RZ || o.kind == JQ_K_ROT) && k != 1)
      return fail("op " + std::to_string(i) + ": single-qubit rotation on " + std::to_string(k) + " wires");
    if (o.kind == JQ_K_PAULIROT && (o.n_controls < 0 || o.n_controls >= k))
      return fail("op " + std::to_string(i) + ": bad control count");
    if (d.n_angles > 0) {
      if (o.angle_slot < 0) return fail("op " + std::to_string(i) + ": negative angle slot");
      plan->n_angles = std::max(plan->n_angles, o.angle_slot + d.n_angles);
    }
    if (o.kind == JQ_K_MATRIX) {
      if (o.mat_slot < 0) return fail("op " + std::to_string(i) + ": negative matrix slot");
      int len = o.mat_is_diag ? (1 << k) : (1 << (2 * k));
      plan->n_mats = std::max(plan->n_mats, o.mat_slot + len);
    }
    if (!o.unitary) plan->unitary = false;
    if (o.kind == JQ_K_CHANNEL) plan->unitary = false;
    if (o.grad && (d.n_angles > 0 || o.kind == JQ_K_MATRIX)) plan->any_grad = true;
    plan->ops.push_back(d);

    // declared structure of the op
    Structure st;
    int dim = 1 << k;
    if (o.has_perm) {
      st.perm.assign(o.perm, o.perm + dim);
      if (!validate_perm(st.perm, dim)) return fail("op " + std::to_string(i) + ": invalid permutation");
    }
    st.diagonal = o.diagonal != 0;
    st.controls = std::max(0, std::min(o.n_controls, k - 1));
    if (o.kind == JQ_K_MATRIX && o.mat_is_diag) { st.diagonal = true; st.perm.clear(); }

    std::vector<int> ket(o.wires, o.wires + k);
    std::vector<int> bra(k);
    for (int a = 0; a < k; ++a) bra[a] = o.wires[a] + n;

    if (o.kind == JQ_K_CHANNEL) {
      if (mode != JQ_DENSITY)
        return fail("op " + std::to_string(i) + ": a noise channel cannot be applied to a pure statevector");
      if (2 * k > kMaxBlockWires) return fail("op " + std::to_string(i) + ": channel on more than 3 wires");
      if (o.n_kraus < 1 || !o.const_mat) return fail("op " + std::to_string(i) + ": channel without Kraus matrices");
      int dd = dim * dim;
      std::vector<cd> sup(static_cast<size_t>(dd) * dd, cd(0, 0));
      for (int q = 0; q < o.n_kraus; ++q) {
        std::vector<cd> K = read_matrix(o.const_mat + 2 * static_cast<size_t>(q) * dim * dim, dim);
        std::vector<cd> kk = kron(K, dim, conj_of(K), dim);
        for (size_t e = 0; e < sup.size(); ++e) sup[e] += kk[e];
      }
      HostPrim p;
      p.op = i;
      p.form = PF_CONST;
      p.wires = ket;
      p.wires.insert(p.wires.end(), bra.begin(), bra.end());
      p.st = detect_structure(sup, 2 * k);
      p.cmat = std::move(sup);
      prims.push_back(std::move(p));
      continue;
    }
    if (o.kind == JQ_K_CONST && !o.const_mat) return fail("op " + std::to_string(i) + ": constant op without matrix");

    if (mode == JQ_STATEVECTOR) {
      HostPrim p;
      p.op = i;
      p.wires = ket;
      if (o.kind == JQ_K_CONST) {
        p.form = PF_CONST;
        p.cmat = read_matrix(o.const_mat, dim);
        p.st = detect_structure(p.cmat, k);
      } else {
        p.form = PF_U;
        p.st = st;
      }
      prims.push_back(std::move(p));
    } else if (k == 1) {
      // 1-qubit gate on a density matrix: superoperator kron(U, conj U) on the
      // (ket, bra) wires, so it fuses with the channels on the same wire.
      HostPrim p;
      p.op = i;
      p.wires = {ket[0], bra[0]};
      if (o.kind == JQ_K_CONST) {
        std::vector<cd> U = read_matrix(o.const_mat, 2);
        p.form = PF_CONST;
        p.cmat = kron(U, 2, conj_of(U), 2);
        p.st = detect_structure(p.cmat, 2);
      } else {
        p.form = PF_KRON;
        p.st.diagonal = st.diagonal;
        p.st.controls = 0;
        if (!st.perm.empty()) {
          p.st.perm.resize(4);
          for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) p.st.perm[a * 2 + b] = st.perm[a] * 2 + st.perm[b];
        }
      }
      prims.push_back(std::move(p));
    } else {
      // wider gate on a density matrix: U on the ket wires, conj(U) on the bra
      // wires, each keeping its structure.
      HostPrim pk, pb;
      pk.op = pb.op = i;
      pk.wires = ket;
      pb.wires = bra;
      if (o.kind == JQ_K_CONST) {
        std::vector<cd> U = read_matrix(o.const_mat, dim);
        pk.form = pb.form = PF_CONST;
        pk.cmat = U;
        pb.cmat = conj_of(U);
        pk.st = detect_structure(pk.cmat, k);
        pb.st = detect_structure(pb.cmat, k);
      } else {
        pk.form = PF_U;
        pb.form = PF_CONJ;
        pk.st = pb.st = st;
      }
      prims.push_back(std::move(pk));
      prims.push_back(std::move(pb));
    }
  }

  // ---- same-wire fusion (jaqsi _fuse, simulation.py:214-240) ----------------
  const bool no_fuse = tune && tune->no_fuse;
  std::vector<HostBlock> blocks;
  {
    std::vector<int> last(nb, -1);
    for (int pi = 0; pi < static_cast<int>(prims.size()); ++pi) {
      const HostPrim& p = prims[pi];
      int bi = last[p.wires[0]];
      bool merge = !no_fuse && bi >= 0 && blocks[bi].wires == p.wires &&
                   static_cast<int>(blocks[bi].prims.size()) < kMaxFusePrims;
      if (merge)
        for (int w : p.wires)
          if (last[w] != bi) { merge = false; break; }
      // per-call matrices are not trusted to be exactly unitary (the caller's data)
      const bool pu = p.op >= 0 && ops[p.op].unitary && ops[p.op].kind != JQ_K_CHANNEL &&
                      ops[p.op].kind != JQ_K_MATRIX;
      if (merge) {
        blocks[bi].st = fused_structure(blocks[bi].st, p.st);
        blocks[bi].prims.push_back(pi);
        blocks[bi].unitary = blocks[bi].unitary && pu;
        continue;
      }
      HostBlock b;
      b.wires = p.wires;
      b.st = p.st;
      b.prims.push_back(pi);
      b.unitary = pu;
      blocks.push_back(std::move(b));
      for (int w : p.wires) last[w] = static_cast<int>(blocks.size()) - 1;
    }
  }

  // ---- trailing blocks absorbed into Z-string observables -------------------
  // (jq_tune.expval_only, statevector, every observable a Z string).  From the
  // end of the circuit: a constant diagonal unitary commutes with every Z
  // string and is dropped; a constant permutation that is affine over the
  // index bits, P(i) = A i ^ b, is dropped after each word z becomes A^T z
  // with the sign (-1)^popc(z & b).  Blocks with parameters stop the walk.
  std::vector<uint64_t> zt;
  std::vector<double> zsign;
  if (tune && tune->expval_only && mode == JQ_STATEVECTOR && n_obs > 0) {
    bool all_z = true;
    for (int i = 0; i < n_obs; ++i)
      if (obs[i].kind != JQ_OBS_PAULI || obs[i].x_mask != 0) all_z = false;
    if (all_z) {
      zt.resize(n_obs);
      zsign.assign(n_obs, 1.0);
      for (int i = 0; i < n_obs; ++i) zt[i] = obs[i].z_mask;
      while (!blocks.empty()) {
        const HostBlock& hb = blocks.back();
        const int k = static_cast<int>(hb.wires.size()), dim = 1 << k;
        bool constant = hb.unitary;
        for (int pi : hb.prims) {
          const int op = prims[pi].op;
          if (op >= 0 && (plan->ops[op].n_angles > 0 || plan->ops[op].kind == JQ_K_MATRIX ||
                          plan->ops[op].kind == JQ_K_CHANNEL))
            constant = false;
        }
        if (!constant) break;
        if (!hb.st.diagonal) {
          if (static_cast<int>(hb.st.perm.size()) != dim) break;
          // P(i): the row that takes input row i (out[r] = in[perm[r]])
          std::vector<int> inv(dim);
          for (int r = 0; r < dim; ++r) inv[hb.st.perm[r]] = r;
          const int b0 = inv[0];
          std::vector<int> col(k);
          for (int m = 0; m < k; ++m) col[m] = inv[1 << m] ^ b0;
          bool affine = true;
          for (int x = 0; x < dim && affine; ++x) {
            int v = b0;
            for (int m = 0; m < k; ++m)
              if (x >> m & 1) v ^= col[m];
            affine = v == inv[x];
          }
          if (!affine) break;
          // local bit m is wire wires[k - 1 - m], flat bit nb - 1 - that wire
          auto gbit = [&](int m) { return nb - 1 - hb.wires[k - 1 - m]; };
          for (int i = 0; i < n_obs; ++i) {
            uint32_t zl = 0;
            for (int m = 0; m < k; ++m) zl |= static_cast<uint32_t>((zt[i] >> gbit(m)) & 1ULL) << m;
            if (__builtin_popcount(zl & static_cast<uint32_t>(b0)) & 1) zsign[i] = -zsign[i];
            uint64_t z = zt[i];
            for (int m = 0; m < k; ++m) {
              const uint64_t bit = 1ULL << gbit(m);
              z = (__builtin_popcount(zl & static_cast<uint32_t>(col[m])) & 1) ? (z | bit) : (z & ~bit);
            }
            zt[i] = z;
          }
        }
        blocks.pop_back();
        ++plan->absorbed;
      }
    }
  }

  // ---- device prims / blocks -----------------------------------------------
  int maxk = 1;
  for (const HostBlock& b : blocks) maxk = std::max(maxk, static_cast<int>(b.wires.size()));
  std::vector<int> prim_order;
  int64_t bmat = 0, grad = 0, scratch = 0;
  for (const HostBlock& hb : blocks) {
    DevBlock db;
    std::memset(&db, 0, sizeof(db));
    int k = static_cast<int>(hb.wires.size());
    int dim = 1 << k;
    db.k = k;
    db.prim_begin = static_cast<int32_t>(plan->prims.size());
    bool needs_grad = false;
    for (int pi : hb.prims) {
      const HostPrim& p = prims[pi];
      DevPrim dp;
      dp.op = p.op;
      dp.form = p.form;
      dp.k = static_cast<int32_t>(p.wires.size());
      dp.const_off = -1;
      if (p.form == PF_CONST) {
        dp.const_off = static_cast<int32_t>(plan->const_pool.size() / 2);
        for (const cd& v : p.cmat) {
          plan->const_pool.push_back(v.real());
          plan->const_pool.push_back(v.imag());
        }
      } else if (p.op >= 0) {
        const DevOp& o = plan->ops[p.op];
        if (o.grad && (o.n_angles > 0 || o.kind == JQ_K_MATRIX)) needs_grad = true;
      }
      plan->prims.push_back(dp);
    }
    db.prim_end = static_cast<int32_t>(plan->prims.size());
    Structure st = hb.st;
    int c = std::max(0, std::min(st.controls, k - 1));
    if (!st.perm.empty()) {
      // inner permutation of the controlled part
      int d = 1 << (k - c), base = dim - d;
      bool ok = true;
      for (int i = 0; i < base && ok; ++i) ok = st.perm[i] == i;
      for (int i = 0; i < d && ok; ++i) ok = st.perm[base + i] >= base;
      if (!ok) { c = 0; d = dim; base = 0; }
      db.kind = BK_PERM;
      db.n_ctrl = c;
      db.d = d;
      db.perm_off = static_cast<int32_t>(plan->perm_pool.size());
      for (int i = 0; i < d; ++i) plan->perm_pool.push_back(st.perm[base + i] - base);
      db.mat_off = -1;
      db.grad_off = -1;
    } else {
      db.kind = st.diagonal ? BK_DIAG : BK_DENSE;
      db.n_ctrl = c;
      db.d = 1 << (k - c);
      db.perm_off = -1;
      db.mat_off = static_cast<int32_t>(bmat);
      bmat += (db.kind == BK_DIAG) ? db.d : static_cast<int64_t>(db.d) * db.d;
      if (needs_grad) {
        db.grad_off = static_cast<int32_t>(grad);
        grad += (db.kind == BK_DIAG) ? db.d : static_cast<int64_t>(db.d) * db.d;
      } else {
        db.grad_off = -1;
      }
    }
    if (k > 2) {
      db.scratch_off = static_cast<int32_t>(scratch);
      scratch += 8LL * dim * dim;
    } else {
      db.scratch_off = -1;
    }
    plan->blocks.push_back(db);
    std::array<int32_t, kMaxBlockWires> bw;
    bw.fill(-1);
    for (int i = 0; i < k; ++i) bw[i] = hb.wires[i];
    plan->block_wires.push_back(bw);
  }
  plan->bmat_stride = bmat;
  plan->grad_stride = grad;
  plan->scratch_stride = scratch;

  // ---- schedules ---------------------------------------------------------------
  // low index bits every tile holds (contiguous runs of 2^c amplitudes:
  // 128 bytes complex64, 128 bytes complex128); JQ_TILE_LOW overrides
  int c_seed = std::min(nb, dtype == JQ_C64 ? 4 : 3);
  if (const char* e = std::getenv("JQ_TILE_LOW")) c_seed = std::min(nb, std::max(2, std::min(6, std::atoi(e))));
  const bool dens = mode == JQ_DENSITY;
  int tf = (tune && tune->tile_bits > 0) ? tune->tile_bits
                                         : default_tile_bits(nb, dtype, maxk, c_seed, false, dens, plan->any_grad);
  int ta = (tune && tune->tile_bits_adj > 0) ? tune->tile_bits_adj
                                             : default_tile_bits(nb, dtype, maxk, c_seed, true, dens, plan->any_grad);
  tf = std::min(std::min(tf, nb), kMaxTileBits);
  ta = std::min(std::min(ta, nb), kMaxTileBits);
  if (tf < std::min(nb, maxk + c_seed) || ta < std::min(nb, maxk + c_seed)) {
    return fail("jq_plan_build: tile too small for a " + std::to_string(maxk) + "-wire block");
  }
  int max_t = (dtype == JQ_C64) ? 14 : 13;
  if (tf > max_t || ta > max_t - 1) return fail("jq_plan_build: tile_bits too large for shared memory");
  plan->fwd = schedule(blocks, plan->blocks, nb, tf, c_seed, no_fuse);
  plan->adj = schedule(blocks, plan->blocks, nb, ta, c_seed, no_fuse);
  plan->bwd = schedule(blocks, plan->blocks, nb, ta, c_seed, true);
  // one-wire blocks fused from rotations only (RX, RY, RZ, Rot and their
  // conjugates) are SU(2) matrices: their passes read half the matrix
  std::vector<uint8_t> su2(plan->blocks.size(), 0);
  for (size_t b = 0; b < plan->blocks.size(); ++b) {
    const DevBlock& blk = plan->blocks[b];
    if (blk.kind != BK_DENSE || blk.k != 1 || blk.n_ctrl != 0 || blk.prim_end <= blk.prim_begin) continue;
    bool ok = true;
    for (int pi = blk.prim_begin; pi < blk.prim_end && ok; ++pi) {
      const DevPrim& pr = plan->prims[pi];
      if (pr.op < 0 || (pr.form != PF_U && pr.form != PF_CONJ) || pr.k != 1) { ok = false; break; }
      const DevOp& dop = plan->ops[pr.op];
      ok = dop.k == 1 && (dop.kind == JQ_K_RX || dop.kind == JQ_K_RY || dop.kind == JQ_K_RZ || dop.kind == JQ_K_ROT);
    }
    su2[b] = ok ? 1 : 0;
  }
  build_steps(plan->fwd, plan->perm_pool, dtype, su2);
  build_steps(plan->bwd, plan->perm_pool, dtype, su2);
  plan->threads = (tune && tune->threads > 0) ? tune->threads : 512;
  if (plan->threads % 32 || plan->threads < 64 || plan->threads > 1024)
    return fail("jq_plan_build: threads must be a multiple of 32 in 64..1024");
  plan->ckpt_stride = (tune && tune->ckpt_stride > 0) ? tune->ckpt_stride : 0;
  {
    const int mode_jit = tune ? tune->jit : 0;
    const char* env = std::getenv("JQ_NO_JIT");
    const bool env_off = env && env[0] && env[0] != '0';
    plan->jit = !env_off && (mode_jit > 0 || (mode_jit == 0 && nb >= 16));
    plan->jit_required = !env_off && mode_jit > 0;
  }

  // ---- observables -----------------------------------------------------------------
  for (int i = 0; i < n_obs; ++i) {
    const jq_obs& o = obs[i];
    DevObs d;
    std::memset(&d, 0, sizeof(d));
    d.kind = o.kind;
    d.k = o.n_wires;
    if (o.kind == JQ_OBS_PAULI) {
      uint64_t lim = (n >= 64) ? ~0ULL : ((1ULL << n) - 1);
      if ((o.x_mask | o.z_mask) & ~lim) return fail("observable " + std::to_string(i) + ": Pauli mask outside the register");
      d.x_mask = o.x_mask;
      d.z_mask = zt.empty() ? o.z_mask : zt[i];
      d.n_y = o.n_y;
      d.coeff = zt.empty() ? o.coeff : o.coeff * zsign[i];
    } else if (o.kind == JQ_OBS_DENSE) {
      int k = o.n_wires;
      if (k < 1 || k > JQ_MAX_OP_WIRES || !o.mat) return fail("observable " + std::to_string(i) + ": bad dense observable");
      for (int a = 0; a < k; ++a) {
        if (o.wires[a] < 0 || o.wires[a] >= n) return fail("observable " + std::to_string(i) + ": wire out of range");
        for (int b = 0; b < a; ++b)
          if (o.wires[a] == o.wires[b]) return fail("observable " + std::to_string(i) + ": duplicate wires");
        d.bits[a] = static_cast<int8_t>(n - 1 - o.wires[a]);
      }
      d.mat_off = static_cast<int32_t>(plan->obs_pool.size() / 2);
      int dim = 1 << k;
      for (int e = 0; e < 2 * dim * dim; ++e) plan->obs_pool.push_back(o.mat[e]);
      d.coeff = 1.0;
    } else {
      return fail("observable " + std::to_string(i) + ": unknown kind");
    }
    plan->obs.push_back(d);
  }
  *out = plan;
  return JQ_OK;
}

}  // namespace jq
