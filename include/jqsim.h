/*
 * jqsim.h — C ABI of libjqsim.so, the B200 (sm_100a) execution backend for
 * jaqsi's circuit-simulation hot path.
 *
 * The reference runs this path as Python over JAX/XLA (jaqsi/simulation.py).
 * Each entry point below replaces one reference function; the citation names
 * the reference file:line of the interface it stands in for.
 *
 * Conventions (identical to the reference):
 *   - wire 0 is the most significant bit of the flat amplitude index
 *     (jaqsi/simulation.py:406, :796);
 *   - in a k-wire matrix the first listed wire is the most significant bit of
 *     the row/column index (jaqsi/simulation.py:177, :259);
 *   - a density matrix is a row-major (dim, dim) array; seen as a 2n-wire
 *     vector its ket wires are 0..n-1 and its bra wires n..2n-1
 *     (jaqsi/simulation.py:349-353, :466-473).
 *
 * Ownership: the caller owns every device buffer (angles, matrices, states,
 * outputs, workspace) and passes raw device pointers.  A plan is built on the
 * host without touching the GPU; its constant tables are uploaded to the
 * current device on first use.  No entry point allocates device memory except
 * jq_plan_* (device copies of the plan's constant tables).
 *
 * Errors: every call returns JQ_OK (0) or a negative status; the message of
 * the last failure on the calling thread is available from jq_last_error().
 * No C++ exception crosses this boundary.
 */
#ifndef JQSIM_H
#define JQSIM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define JQ_API __attribute__((visibility("default")))
#else
#define JQ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define JQ_OK 0
#define JQ_EINVAL (-1)       /* bad argument or plan                          */
#define JQ_ENOMEM (-2)       /* workspace too small / allocation failed       */
#define JQ_ECUDA (-3)        /* a CUDA runtime call failed                    */
#define JQ_ETIMEOUT (-4)     /* a bounded device wait ran out                 */
#define JQ_EABORT (-5)       /* the host abort flag was raised                */
#define JQ_EUNSUPPORTED (-6) /* valid input outside what this build supports */

/* init_batched flag of a density plan: `init` holds density matrices. */
#define JQ_INIT_DENSITY 2

/* ---- limits -------------------------------------------------------------- */
#define JQ_MAX_OP_WIRES 6 /* widest gate / observable (matrix 64 x 64)      */
#define JQ_MAX_QUBITS 30  /* statevector; density matrices up to 15 qubits  */

/* ---- enums --------------------------------------------------------------- */
enum jq_dtype { JQ_C64 = 0, JQ_C128 = 1 };
enum jq_mode { JQ_STATEVECTOR = 0, JQ_DENSITY = 1 };
enum jq_out_type {
  JQ_OUT_STATE = 0,   /* final statevector / density matrix only          */
  JQ_OUT_PROBS = 1,   /* |psi|^2 or diag(rho), real                       */
  JQ_OUT_EXPVAL = 2,  /* one real value per observable (float64)          */
  JQ_OUT_DENSITY = 3  /* |psi><psi| (pure) or rho (mixed)                  */
};

/* How the device builds an op's matrix (all in float64, then rounded to the
 * run dtype).  Parameter conventions follow jaqsi/gateset.py. */
enum jq_op_kind {
  JQ_K_CONST = 0,     /* constant 2^k x 2^k matrix, host copy in const_mat   */
  JQ_K_MATRIX = 1,    /* per-call matrix in the mats buffer at mat_slot       */
  JQ_K_RX = 2,        /* cos(t/2) I - i sin(t/2) X          gateset.py:399    */
  JQ_K_RY = 3,
  JQ_K_RZ = 4,
  JQ_K_ROT = 5,       /* RZ(omega) RY(theta) RZ(phi), angles phi,theta,omega
                         gateset.py:653-657                                   */
  JQ_K_CPHASE = 6,    /* diag(1,..,1, e^{i phi}) on the last index            */
  JQ_K_PAULIROT = 7,  /* cos(t/2) I - i sin(t/2) P(word), optionally with
                         n_controls leading control wires (gateset.py:670-829) */
  JQ_K_CHANNEL = 8    /* Kraus channel, n_kraus host matrices in const_mat    */
};

/* One recorded tape entry (an Operation of jaqsi/operations.py:188). */
typedef struct jq_op {
  int32_t kind;                     /* enum jq_op_kind                        */
  int32_t n_wires;                  /* k, 1..JQ_MAX_OP_WIRES                  */
  int32_t wires[JQ_MAX_OP_WIRES];   /* first = most significant matrix bit    */
  /* GateStructure (operations.py:176-185): static guarantees of the matrix. */
  int32_t n_controls;               /* leading control wires                  */
  int32_t diagonal;                 /* nonzero: matrix is diagonal            */
  int32_t has_perm;                 /* nonzero: perm[] holds a permutation    */
  int32_t perm[1 << JQ_MAX_OP_WIRES]; /* output row i takes input column perm[i] */
  int32_t angle_slot;               /* first angle of the op in the angles row */
  int32_t mat_slot;                 /* JQ_K_MATRIX: element offset in mats row */
  int32_t mat_is_diag;              /* JQ_K_MATRIX: mats holds only 2^k diagonal */
  uint32_t pauli_x;                 /* JQ_K_PAULIROT: X/Y positions (bit k-1-i = wire i) */
  uint32_t pauli_z;                 /* JQ_K_PAULIROT: Z/Y positions           */
  int32_t n_kraus;                  /* JQ_K_CHANNEL: number of Kraus matrices */
  int32_t grad;                     /* nonzero: parameters need gradients     */
  int32_t unitary;                  /* operations.py:223 is_unitary           */
  const double* const_mat;          /* CONST / CHANNEL: host complex128 data,
                                       read only during jq_plan_build         */
} jq_op;

enum jq_obs_kind {
  JQ_OBS_PAULI = 0, /* tensor product of I/X/Y/Z, given as masks           */
  JQ_OBS_DENSE = 1  /* Hermitian 2^k x 2^k on `wires`                       */
};

/* One observable of an "expval" measurement (simulation.py:735-857). */
typedef struct jq_obs {
  int32_t kind;
  int32_t n_wires;
  int32_t wires[JQ_MAX_OP_WIRES];
  uint64_t x_mask;     /* PAULI: flat-index bits carrying X or Y             */
  uint64_t z_mask;     /* PAULI: flat-index bits carrying Z or Y             */
  int32_t n_y;         /* PAULI: number of Y factors (phase i^n_y)           */
  double coeff;        /* PAULI: real prefactor (1.0 for a plain Pauli word) */
  const double* mat;   /* DENSE: host complex128 2^k x 2^k, read at build    */
} jq_obs;

/* Tuning knobs (0 = choose automatically). */
typedef struct jq_tune {
  int32_t tile_bits;     /* qubits held per CTA in a forward tile pass        */
  int32_t tile_bits_adj; /* qubits held per CTA in an adjoint tile pass       */
  int32_t threads;       /* threads per CTA of the tile kernels               */
  int32_t no_fuse;       /* nonzero: one pass per gate block (unfused baseline) */
  int32_t ckpt_stride;   /* passes between checkpoints of the checkpointed
                            reverse pass (0: ceil(sqrt(passes)))             */
  int32_t jit;           /* forward passes specialised per plan with NVRTC:
                            0 auto (states of >= 2^16 amplitudes; if the
                            specialisation fails the register-stage
                            interpreter runs), 1 on (a failed specialisation
                            fails every call on that device with its error
                            text), -1 off (register-stage interpreter only)    */
  int32_t expval_only;   /* nonzero: the plan is run for expectation values
                            only (jq_forward / jq_adjoint / jq_backward with
                            JQ_OUT_EXPVAL).  When every observable is a Z
                            string (Pauli, no X or Y) of a statevector plan,
                            trailing blocks that are affine permutations of
                            the index bits (X, CX, SWAP and their fusions) or
                            constant diagonal unitaries are absorbed into the
                            words (P psi with P(i) = A i ^ b gives
                            <Z_z> = (-1)^popc(z & b) <Z_{A^T z}> before P)
                            and not run; the state buffers then hold the
                            state before them (jq_sweep applies the passes
                            the plan keeps), and other out types fail with
                            JQ_EINVAL.                                         */
} jq_tune;

/* Plan summary. */
typedef struct jq_plan_info {
  int32_t n_qubits;
  int32_t n_bits;          /* qubits (statevector) or 2 x qubits (density)   */
  int32_t mode, dtype;
  int32_t n_ops;           /* recorded ops (barriers removed by the caller)  */
  int32_t n_blocks;        /* after same-wire fusion (jaqsi _fuse)           */
  int32_t n_passes_fwd;    /* HBM passes of the forward sweep                */
  int32_t n_passes_adj;    /* passes of one adjoint sweep                    */
  int32_t n_tile_ops_fwd;  /* gate applications inside the forward passes    */
  int32_t tile_bits_fwd, tile_bits_adj;
  int32_t n_angles;        /* length of one angles row                       */
  int32_t n_mats;          /* complex128 elements of one mats row            */
  int32_t n_obs;
  int32_t unitary;         /* every op unitary (adjoint allowed)             */
  int64_t state_elems;     /* complex elements of one state (2^n or 4^n)     */
  int32_t n_stages_fwd;    /* register stages over all forward passes        */
  int32_t n_smem_ops_fwd;  /* generic shared-memory steps of the forward     */
} jq_plan_info;

typedef struct jq_plan jq_plan;

/* Compile a recorded tape into an execution plan.
 * Replaces jaqsi/simulation.py:338-345 (_compile) and :348-381
 * (_compile_mixed): same-wire fusion with the reference's rule (:214-240),
 * then a B200 pass schedule (many gate blocks per HBM pass).
 * Host only: no CUDA call is made. */
JQ_API int jq_plan_build(const jq_op* ops, int n_ops, const jq_obs* obs, int n_obs,
                  int n_qubits, int mode, int dtype, const jq_tune* tune,
                  jq_plan** out);
JQ_API int jq_plan_free(jq_plan* plan);
JQ_API int jq_plan_get_info(const jq_plan* plan, jq_plan_info* info);

/* Schedule of a plan: pass index of every fused block (which = 0 forward,
 * also walked backwards by jq_backward; 1 adjoint interpreter; 2 one block
 * per pass, the unfused order) into block_pass[0..n-1], and the wires
 * of each block into block_wires[6 * b ..] (-1 padded) when non-NULL.
 * Diagnostic; no reference counterpart (the reference runs one pass per
 * entry of its plan, jaqsi/simulation.py:400-409). */
JQ_API int jq_plan_block_passes(const jq_plan* plan, int which, int32_t* block_pass,
                                int32_t* block_wires, int n);

/* CUDA C++ source of the plan's per-plan specialised forward passes (see
 * jq_tune.jit), written to buf (NUL-terminated, truncated to n bytes);
 * returns the full length.  Diagnostic; no reference counterpart. */
JQ_API size_t jq_plan_jit_source(const jq_plan* plan, char* buf, size_t n);

/* Device workspace (bytes) for `batch` instances: with_grad 0 sizes
 * jq_forward, 1 sizes jq_adjoint, 2 sizes jq_backward. */
JQ_API size_t jq_workspace_bytes(const jq_plan* plan, int batch, int out_type,
                          int with_grad);

/* Forward simulation and measurement of `batch` instances of one plan.
 * Replaces jaqsi/simulation.py:658-732 (simulate_and_measure) with
 * :412-440 (simulate_pure), :443-473 (simulate_mixed), :735-811
 * (measure_state) and :814-857 (measure_density).
 *   angles   float64 [batch, n_angles] (device) or NULL if n_angles == 0
 *   mats     complex128 [batch, n_mats] (device) or NULL if n_mats == 0
 *   init     NULL (|0..0>) or complex (run dtype) statevector(s):
 *            [2^n] broadcast when init_batched bit 0 is clear, else
 *            [batch, 2^n]; for a density plan with init_batched bit 1
 *            (JQ_INIT_DENSITY) set, density matrices [2^n, 2^n] (or
 *            [batch, 2^n, 2^n]) instead, copied as the initial state (the
 *            reverse pass then returns the cotangent of that matrix)
 *   state    complex (run dtype) [batch, state_elems]: receives psi or rho
 *   out      EXPVAL: float64 [batch, n_obs]; PROBS: real run dtype
 *            [batch, 2^n]; DENSITY (pure): complex [batch, 4^n];
 *            ignored for STATE and for DENSITY of a mixed plan (= state).
 *   stream   cudaStream_t (NULL = legacy default stream) */
JQ_API int jq_forward(const jq_plan* plan, int batch, const double* angles,
               const void* mats, const void* init, int init_batched,
               int out_type, void* state, void* out, void* workspace,
               size_t workspace_bytes, void* stream);

/* Forward gate sweep of a statevector / density plan applied in place to a
 * resident state (no initialisation, no measurement): the state after
 * jq_sweep equals simulate_pure's result for `state` as initial state.
 * Replaces jaqsi/simulation.py:400-409 (_run) for a caller that keeps the
 * state on the device between circuit segments. */
JQ_API int jq_sweep(const jq_plan* plan, int batch, const double* angles,
                    const void* mats, void* state, void* workspace,
                    size_t workspace_bytes, void* stream);

/* jq_forward without any device allocation, for callers that cannot
 * allocate device memory: hosts that bind this C ABI holding only raw device
 * pointers and no allocator (an FFI host whose memory belongs to another
 * runtime), and services running under a fixed device-memory budget that must
 * not grow at run time.  No counterpart in the reference (jaqsi allocates
 * through XLA).
 *
 * The workspace is a file-scope static device array of JQ_STATIC_WS_BYTES
 * (4 MiB) that every GPU loading the library holds until exit; plans whose
 * forward workspace for `batch` instances exceeds it are rejected with
 * JQ_ENOMEM.  The plan's tables must already be resident on the current device
 * (one prior jq_forward / jq_adjoint / jq_backward / jq_sweep on that device),
 * otherwise JQ_EINVAL.  The first call on a device resolves the array's
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture (a first call made while `stream` is capturing returns JQ_EINVAL
 * and does nothing).  All calls share the array and it keeps the last call's contents,
 * so calls that overlap on the GPU (other streams, other threads) race:
 * serialise them.  Arguments and results are those of jq_forward. */
#define JQ_STATIC_WS_BYTES (4u << 20)
JQ_API int jq_forward_noalloc(const jq_plan* plan, int batch, const double* angles,
                              const void* mats, const void* init, int init_batched,
                              int out_type, void* state, void* out, void* stream);

/* Adjoint-method gradient of the expectation values of a unitary pure-state
 * plan, O(1) extra statevectors.  Replaces jaqsi/simulation.py:546-655
 * (_adjoint_expval).  `state` holds the forward result (it is left intact).
 * The seed cotangent is ct (float64 [batch, n_obs]) for out_type EXPVAL, or
 * ct_state for STATE (complex [batch, 2^n]), PROBS (real [batch, 2^n]) and
 * DENSITY (complex [batch, 4^n]), in the run dtype.
 * Gradients follow PyTorch's convention (d/dRe + i d/dIm for complex).
 *   grad_angles  float64 [batch, n_angles] (written, may be NULL)
 *   grad_mats    complex128 [batch, n_mats] (written, may be NULL)
 *   grad_init    complex (run dtype) [batch, 2^n] (written, may be NULL) */
JQ_API int jq_adjoint(const jq_plan* plan, int batch, const double* angles,
               const void* mats, const void* state, int out_type,
               const double* ct, const void* ct_state, double* grad_angles,
               void* grad_mats, void* grad_init, void* workspace,
               size_t workspace_bytes, void* stream);

/* Checkpointed reverse pass for any plan (density matrices with Kraus
 * channels, non-unitary pure circuits): the forward is recomputed from
 * ceil(sqrt(P)) checkpoints.  Replaces the plain-autodiff fallback of
 * jaqsi/simulation.py:715-720 (noisy) and :540-543 (non-unitary).
 *   out_type EXPVAL: ct float64 [batch, n_obs]
 *   out_type STATE / DENSITY / PROBS: ct_state is the cotangent of the
 *   returned state / density / probabilities (run dtype layout of `out`). */
JQ_API int jq_backward(const jq_plan* plan, int batch, const double* angles,
                const void* mats, const void* init, int init_batched,
                int out_type, const double* ct, const void* ct_state,
                double* grad_angles, void* grad_mats, void* grad_init,
                void* workspace, size_t workspace_bytes, void* stream);

/* Shot sampling: `shots` basis-state draws per row from the probabilities
 * probs float64 [batch, dim] (device; negative rounding noise counts as 0,
 * rows need not be normalised), histogram into counts uint32 [batch, dim]
 * (device, overwritten).  Inverse CDF over a float64 prefix sum; the
 * random stream is a counter-based generator of (seed, row, shot), so a
 * seed reproduces the counts exactly.  Replaces jax.random.choice + the
 * histogram of jaqsi/simulation.py:860-917 (same distribution, not JAX's
 * stream).  workspace: jq_sample_workspace_bytes(batch, dim) bytes. */
JQ_API size_t jq_sample_workspace_bytes(int batch, int64_t dim);
JQ_API int jq_sample_shots(const double* probs, int batch, int64_t dim, int64_t shots, uint64_t seed,
                           uint32_t* counts, void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------
 * Batched uneven instances: forward + adjoint of many independent circuits
 * of different qubit counts, depths and parameters in one CUDA-graph launch.
 * Replaces the reference's batched trace of _single_execute under vmap /
 * shard_map (jaqsi/script.py:426-434, :87-125) for gradient workloads.
 *
 * Instance i runs plans[plan_of[i]]; every plan is a unitary statevector
 * plan of one dtype with Pauli or dense observables and no matrix
 * arguments.  Angles and gradients are concatenated per instance in order
 * (instance i owns n_angles(plan) entries), expectation values likewise
 * (n_obs(plan) entries).
 * ---------------------------------------------------------------------- */
typedef struct jq_batch jq_batch;

typedef struct jq_batch_config {
  int32_t warp_max_qubits; /* n <= this: one warp per instance, state in shared memory */
  int32_t cta_max_qubits;  /* n <= this: one CTA per instance, state in shared memory  */
  int32_t warp_threads;    /* threads per CTA of the warp-per-instance kernel (32..512) */
  int32_t cta_threads;     /* threads per CTA of the CTA-per-instance and cluster kernels (64..512) */
  int32_t cluster_bits;    /* n <= cta_max_qubits + cluster_bits (at most 3): one cluster of
                              2^(n - cta_max_qubits) CTAs per instance, the state split over
                              their shared memory; larger: batched tile passes             */
} jq_batch_config;

/* cfg NULL: defaults (complex64 9 / 13 qubits, complex128 8 / 12; 256 / 512 threads;
 * cluster_bits 3). */
JQ_API int jq_batch_build(jq_plan* const* plans, int n_plans, const int32_t* plan_of, int n_inst,
                          const jq_batch_config* cfg, jq_batch** out);
JQ_API int jq_batch_free(jq_batch* batch);
/* totals: angles (= gradient entries) and expectation values over all
 * instances; n_class[4] = instances in the warp, cta, tile and cluster classes. */
JQ_API int jq_batch_info(const jq_batch* batch, int64_t* n_angles, int64_t* n_obs, int32_t* n_class,
                         jq_batch_config* cfg);
/* Workspace for jq_batch_run under the current configuration and under
 * every configuration jq_batch_autotune tries (the maximum). */
JQ_API size_t jq_batch_workspace_bytes(const jq_batch* batch);
JQ_API int jq_batch_set_config(jq_batch* batch, const jq_batch_config* cfg);
/* Expectation values and d(sum_o ct_o <O_o>)/d angles of every instance
 * (ct: float64 [n_obs total] or NULL for all ones); device pointers.  The
 * first call with a set of pointers captures a CUDA graph, later calls with
 * the same pointers replay it. */
JQ_API int jq_batch_run(jq_batch* batch, const double* angles, const double* ct, double* expval, double* grad,
                        void* workspace, size_t workspace_bytes, void* stream);
/* Time candidate configurations on these inputs, keep the fastest (also
 * returned in *chosen when non-NULL).  Synchronises the stream. */
JQ_API int jq_batch_autotune(jq_batch* batch, const double* angles, double* expval, double* grad,
                             void* workspace, size_t workspace_bytes, void* stream, jq_batch_config* chosen);

/* ------------------------------------------------------------------------
 * Pulse-gate unitaries: ordered products of matrix exponentials, the form
 * of every step of jaqsi's commutator-free Magnus integrators
 * (jaqsi/evolution.py:195-264) that resolve_pending solves in batches for
 * the pulse gates of a tape (jaqsi/evolution.py:730-773, called from
 * jaqsi/simulation.py:713).  For gate g:
 *   U[g] = expm(Om[g, M-1]) ... expm(Om[g, 0]),  Om[g, m] = sum_i w[g, m, i] A[g, i]
 *   A      complex128 [n_gates][n_terms][dim][dim] (A_i = -i H_i), gate g at
 *          A + 2 * g * a_stride doubles (a_stride complex elements; 0: shared)
 *   w      complex128 [n_gates][n_sub][n_terms]
 *   U      complex128 [n_gates][dim][dim] (written)
 * dim is 2, 4 or 8; n_sub at most 2048 (dim <= 4) or 512 (dim 8).  Device
 * pointers; no workspace.
 * jq_magnus_product_grad: gw[g, m, i] = dL/dw[g, m, i] (complex128, written)
 * from gU = dL/dU (complex128 [n_gates][dim][dim]), PyTorch's convention
 * for complex gradients (d/dRe + i d/dIm). */
JQ_API int jq_magnus_product(int n_gates, int dim, int n_terms, int n_sub, const double* A, int64_t a_stride,
                             const double* w, double* U, void* stream);
JQ_API int jq_magnus_product_grad(int n_gates, int dim, int n_terms, int n_sub, const double* A, int64_t a_stride,
                                  const double* w, const double* gU, double* gw, void* stream);

/* Message of the last failed call on this thread ("" if none). */
JQ_API const char* jq_last_error(void);

/* Library version string. */
JQ_API const char* jq_version(void);

#ifdef __cplusplus
}
#endif
#endif /* JQSIM_H */
