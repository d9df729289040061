// Internal data model shared by the host planner (planner.cpp) and the device
// kernels (kernels.cu).  Nothing here crosses the C ABI.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <deque>
#include <vector>

#include "../../include/jqsim.h"

namespace jq {

constexpr int kMaxBlockWires = 6;   // widest fused block on the (2n-)bit vector
constexpr int kMaxTileBits = 15;    // tile = 2^t amplitudes held by one CTA
constexpr int kMaxFusePrims = 16;   // longest same-wire fusion run

// How a block is applied inside a tile.
enum BlockKind : int32_t { BK_DENSE = 0, BK_DIAG = 1, BK_PERM = 2 };

// How a prim's full matrix is obtained from its op.
enum PrimForm : int32_t {
  PF_U = 0,     // the op's matrix U
  PF_CONJ = 1,  // conj(U)           (bra side of a wide gate on a density matrix)
  PF_KRON = 2,  // kron(U, conj(U))  (superoperator of a 1-qubit gate)
  PF_CONST = 3  // constant matrix from the plan's constant pool
};

// Static guarantees of a matrix (jaqsi GateStructure, operations.py:176-185).
struct Structure {
  std::vector<int32_t> perm;  // empty: no permutation guarantee
  bool diagonal = false;
  int32_t controls = 0;
};

// Device descriptor of a recorded op (matrix construction).
struct DevOp {
  int32_t kind;        // jq_op_kind
  int32_t k;           // op wires
  int32_t n_ctrl;      // PAULIROT controls
  int32_t angle_slot;
  int32_t mat_slot;
  int32_t mat_is_diag;
  uint32_t px, pz;     // PAULIROT word masks over target positions
  int32_t grad;
  int32_t n_angles;    // parameters of the op
};

// Device descriptor of a prim (one factor of a fused block).
struct DevPrim {
  int32_t op;          // DevOp index, -1 for constants without an op
  int32_t form;        // PrimForm
  int32_t k;           // wires of the prim on the bit vector
  int32_t const_off;   // PF_CONST: complex128 offset in the constant pool
};

// Device descriptor of a fused block.
struct DevBlock {
  int32_t kind;        // BlockKind
  int32_t k;           // wires
  int32_t n_ctrl;      // leading control wires
  int32_t d;           // inner dimension 2^(k - n_ctrl)
  int32_t prim_begin, prim_end;
  int32_t mat_off;     // run-dtype complex offset of the inner matrix / diagonal
  int32_t perm_off;    // BK_PERM: offset of the inner permutation in the perm pool
  int32_t grad_off;    // complex128 offset of the cotangent accumulator, -1 if none
  int32_t scratch_off; // complex128 offset of per-instance scratch (k > 2), -1 if none
};

// One block application inside a tile pass (tile-local bit positions).
struct TileOp {
  int32_t block;
  int32_t kind;
  int32_t kt;          // target bits
  int32_t nfix;        // target + control bits
  uint32_t ctrl_mask;  // tile-local mask of the control bits (all must be 1)
  uint32_t lowmask[kMaxBlockWires];  // (1 << f) - 1 for each fixed bit f, ascending
  uint32_t tmask[kMaxBlockWires];    // 1 << target bit; tmask[0] = most significant matrix bit
  int32_t mat_off, perm_off, grad_off;
  int32_t inv;         // 1: the block is unitary (its dagger undoes it exactly)
};

// One HBM pass: a tile covers the bits of `tile_mask`.
struct PassDesc {
  int32_t t;           // tile bits
  int32_t c;           // tile bits 0..c-1 are global bits 0..c-1
  uint64_t tile_mask;  // global bits held in the tile
  int32_t op_begin, op_end;
  int32_t step_begin, step_end;  // register-stage program (empty: generic kernel)
  int32_t rop_begin, rop_end;    // register ops of the program
  int32_t smat_len;              // complex elements of the shared-memory matrix area
  int8_t bits[kMaxTileBits];  // global bit of each tile bit, ascending
};

// Register-stage program of a pass.  Each thread holds 2^r amplitudes of the
// tile in registers (r "register bits" of the tile); a stage loads them from
// shared memory, applies every op whose targets are register bits, and
// stores them back.  Shared memory is XOR-swizzled (see swz_* in jqsim.cu);
// ebits / tbits hold the swizzled offset of each register / thread bit.
enum RegKind : int32_t { RK_DENSE1 = 0, RK_PERM1 = 1, RK_DIAG = 2, RK_DENSE2 = 3, RK_PERM2 = 4 };

struct RegOp {
  // w0: kind | q1 << 4 | q2 << 8 | dk << 12 | dq << 16 (dq: register bit of
  //     DIAG target i at bits 3i..3i+2)
  // w1: crm (control bits that are register bits, over j) | ctm << 8 (control
  //     bits that are thread bits, over the thread index) | perm << 24
  //     (PERM2 inner permutation, 2 bits per entry)
  // w2: matrix offset in the pass's shared-memory matrix area
  // w3: matrix offset in the block-matrix buffer (complex elements)
  uint32_t w0, w1, w2, w3;
  int32_t mat_len;     // complex elements of the matrix / diagonal (0: none)
  int32_t grad_off;    // block cotangent accumulator (complex128 offset), -1 if none
  int32_t pad[2];
};

constexpr int kMaxRegBits = 5;
constexpr int kMaxThreadBits = kMaxTileBits - 4;

struct Step {
  int32_t kind;        // 0: register stage over rops[a, b); 1: generic shared-memory op tops[a]
  int32_t a, b;
  uint32_t ebits[kMaxRegBits];
  uint32_t tbits[kMaxThreadBits];
};

struct Schedule {
  int32_t t = 0;
  int32_t reg_bits = 0;  // r of the register-stage program (0: none)
  std::vector<PassDesc> passes;
  std::vector<TileOp> ops;
  std::vector<Step> steps;
  std::vector<RegOp> rops;
};

// Device copies of a plan's tables on one GPU.
struct DeviceTables {
  int device = -1;
  DevOp* ops = nullptr;
  DevPrim* prims = nullptr;
  DevBlock* blocks = nullptr;
  TileOp* fwd_ops = nullptr;
  TileOp* adj_ops = nullptr;
  TileOp* bwd_ops = nullptr;
  Step* fwd_steps = nullptr;
  RegOp* fwd_rops = nullptr;
  Step* bwd_steps = nullptr;
  RegOp* bwd_rops = nullptr;
  double* const_pool = nullptr;   // complex128 (re, im) pairs
  int32_t* perm_pool = nullptr;
  double* obs_pool = nullptr;     // dense observables, complex128
  void* obs_desc = nullptr;       // DevObs array
  void* jit = nullptr;            // JitModule of the forward schedule (or nullptr)
  bool jit_tried = false;
  int jit_rc = 0;                 // nonzero: the required specialisation failed
  std::string jit_err;            // (its error text, returned by every later call)
};

struct DevObs {
  int32_t kind;        // jq_obs_kind
  int32_t k;
  uint64_t x_mask, z_mask;  // PAULI, flat-index bits
  int32_t n_y;
  double coeff;
  int32_t mat_off;     // DENSE: complex128 offset in obs_pool
  int8_t bits[JQ_MAX_OP_WIRES];  // DENSE: flat-index bit of each wire (wire 0 = MSB of matrix)
};

}  // namespace jq

struct jq_plan {
  int n_qubits = 0;
  int n_bits = 0;
  int mode = 0, dtype = 0;
  int n_angles = 0, n_mats = 0;
  bool unitary = true;
  bool any_grad = false;
  int64_t state_elems = 0;
  std::vector<jq::DevOp> ops;
  std::vector<jq::DevPrim> prims;
  std::vector<jq::DevBlock> blocks;
  std::vector<std::array<int32_t, jq::kMaxBlockWires>> block_wires;  // wires per block, -1 padded
  std::vector<double> const_pool;
  std::vector<int32_t> perm_pool;
  std::vector<jq::DevObs> obs;
  std::vector<double> obs_pool;
  jq::Schedule fwd, adj, bwd;  // bwd: one block per pass (the unfused order; diagnostics)
  int64_t bmat_stride = 0;     // run-dtype complex elements per instance
  int64_t grad_stride = 0;     // complex128 elements per instance
  int64_t scratch_stride = 0;  // complex128 elements per instance (k > 2 blocks)
  int threads = 512;
  int ckpt_stride = 0;
  bool jit = false;             // specialise the forward passes with NVRTC
  bool jit_required = false;    // jq_tune.jit = 1: a failed specialisation is an error
  int absorbed = 0;             // trailing blocks absorbed into the Z strings (jq_tune.expval_only)
  std::deque<jq::DeviceTables> dev;  // per-device uploads (a deque: references stay valid as devices are added)
};
