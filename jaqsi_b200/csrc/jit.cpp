// Per-plan specialisation of the forward tile passes.
//
// The register-stage interpreter (k_tile_fwd2 in jqsim.cu) decodes every op
// at run time; for a plan that will be executed many times the pass programs
// are instead emitted as straight-line CUDA C++ (literal shared-memory
// offsets, gate bodies unrolled over named registers, basis permutations such
// as CX folded into register renames at generation time) and compiled once
// per plan and device with NVRTC for sm_100a.  Gate matrices stay run-time
// data (staged in shared memory per tile), so one compiled plan serves every
// parameter set of the same circuit structure, like the reference caches one
// compiled executable per circuit signature (jaqsi/script.py:695-725).
//
// NVRTC and the driver entry points are resolved at run time (dlopen /
// cudaGetDriverEntryPoint); without them the interpreter kernel runs instead.
#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "jit.h"

namespace jq {
void set_error(const std::string& msg);

namespace {

// ---- run-time bindings ------------------------------------------------------
struct Nvrtc {
  bool ok = false;
  nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*, const char* const*);
  nvrtcResult (*compile)(nvrtcProgram, int, const char* const*);
  nvrtcResult (*log_size)(nvrtcProgram, size_t*);
  nvrtcResult (*log)(nvrtcProgram, char*);
  nvrtcResult (*cubin_size)(nvrtcProgram, size_t*);
  nvrtcResult (*cubin)(nvrtcProgram, char*);
  nvrtcResult (*destroy)(nvrtcProgram*);
};

struct Driver {
  bool ok = false;
  CUresult (*module_load)(CUmodule*, const void*);
  CUresult (*module_unload)(CUmodule);
  CUresult (*get_function)(CUfunction*, CUmodule, const char*);
  CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                     void**, void**);
  CUresult (*set_attr)(CUfunction, CUfunction_attribute, int);
  CUresult (*occupancy)(int*, CUfunction, int, size_t);
  CUresult (*launch_ex)(const CUlaunchConfig*, CUfunction, void**, void**) = nullptr;  // optional
};

std::once_flag g_once;
Nvrtc g_nvrtc;
Driver g_drv;

template <typename F>
bool sym(void* h, const char* name, F* out) {
  *out = reinterpret_cast<F>(dlsym(h, name));
  return *out != nullptr;
}

template <typename F>
bool entry(const char* name, F* out) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    return false;
  *out = reinterpret_cast<F>(p);
  return true;
}

void init_bindings() {
  const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
  void* h = nullptr;
  for (const char* n : names)
    if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
  if (h) {
    g_nvrtc.ok = sym(h, "nvrtcCreateProgram", &g_nvrtc.create) && sym(h, "nvrtcCompileProgram", &g_nvrtc.compile) &&
                 sym(h, "nvrtcGetProgramLogSize", &g_nvrtc.log_size) && sym(h, "nvrtcGetProgramLog", &g_nvrtc.log) &&
                 sym(h, "nvrtcGetCUBINSize", &g_nvrtc.cubin_size) && sym(h, "nvrtcGetCUBIN", &g_nvrtc.cubin) &&
                 sym(h, "nvrtcDestroyProgram", &g_nvrtc.destroy);
  }
  g_drv.ok = entry("cuModuleLoadData", &g_drv.module_load) && entry("cuModuleUnload", &g_drv.module_unload) &&
             entry("cuModuleGetFunction", &g_drv.get_function) && entry("cuLaunchKernel", &g_drv.launch) &&
             entry("cuFuncSetAttribute", &g_drv.set_attr) &&
             entry("cuOccupancyMaxActiveBlocksPerMultiprocessor", &g_drv.occupancy);
  if (!entry("cuLaunchKernelEx", &g_drv.launch_ex)) g_drv.launch_ex = nullptr;
}

// Generated passes start with griddepcontrol.launch_dependents and wait
// (griddepcontrol.wait) for the preceding kernel of the stream before their
// first global access, so back-to-back passes launched with programmatic
// stream serialisation overlap the next pass's launch and prologue with the
// previous pass's last tiles; the wait returns at once for a plain launch.
// JQ_PDL is a bit mask of the pass kinds launched that way: 1 forward,
// 2 adjoint, 4 checkpointed reverse (default 1).
enum { kPdlFwd = 1, kPdlAdj = 2, kPdlBwd = 4 };
int pdl_mask() {
  static const int m = [] {
    const char* e = std::getenv("JQ_PDL");
    return e ? std::atoi(e) : int(kPdlFwd);
  }();
  return m;
}

CUresult launch_pass(CUfunction f, unsigned grid, unsigned threads, unsigned smem, cudaStream_t st, void** args,
                     int kind) {
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (g_drv.launch_ex && (pdl_mask() & kind) && cudaStreamIsCapturing(st, &cap) == cudaSuccess &&
      cap == cudaStreamCaptureStatusNone) {
    CUlaunchAttribute attr[1];
    std::memset(attr, 0, sizeof(attr));
    attr[0].id = CU_LAUNCH_ATTRIBUTE_PROGRAMMATIC_STREAM_SERIALIZATION;
    attr[0].value.programmaticStreamSerializationAllowed = 1;
    CUlaunchConfig cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDimX = grid;
    cfg.gridDimY = cfg.gridDimZ = 1;
    cfg.blockDimX = threads;
    cfg.blockDimY = cfg.blockDimZ = 1;
    cfg.sharedMemBytes = smem;
    cfg.hStream = reinterpret_cast<CUstream>(st);
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return g_drv.launch_ex(&cfg, f, args, nullptr);
  }
  return g_drv.launch(f, grid, 1, 1, threads, 1, 1, smem, reinterpret_cast<CUstream>(st), args, nullptr);
}
const char* kPdlTrigger = "  asm volatile(\"griddepcontrol.launch_dependents;\");\n";
const char* kPdlWait = "  asm volatile(\"griddepcontrol.wait;\" ::: \"memory\");\n";

// ---- device prelude shared by every generated kernel --------------------------
const char* kPrelude = R"JQ(
typedef unsigned int u32;
typedef unsigned long long u64;
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename C> __device__ __forceinline__ C cfma(C a, C b, C acc) {
  C r; r.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x)); r.y = fma(a.x, b.y, fma(a.y, b.x, acc.y)); return r;
}
__device__ __forceinline__ u64 pdep64(u64 v, u64 mask) {
  u64 r = 0;
  for (u64 bb = 1; mask; bb <<= 1) { u64 low = mask & (~mask + 1); if (v & bb) r |= low; mask &= mask - 1; }
  return r;
}
__device__ __forceinline__ void cp_async8(void* s, const void* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async16(void* s, const void* g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_waitn() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ u32 swz8(u32 l) { return l ^ (((l >> 4) ^ (l >> 8) ^ (l >> 12)) & 15u); }
__device__ __forceinline__ u32 swz16(u32 l) { return l ^ (((l >> 3) ^ (l >> 6) ^ (l >> 9) ^ (l >> 12)) & 7u); }
// Asynchronous tile load (global -> swizzled shared memory, no registers):
// one 8-byte (complex64) or 16-byte (complex128) copy per amplitude.
__device__ __forceinline__ void prefetch8(float2* s, const float2* g, const u32* tbl, int t, int c) {
  const int cm = (1 << c) - 1, nv = 1 << t;
  for (int l = threadIdx.x; l < nv; l += blockDim.x) cp_async8(s + swz8(l), g + (tbl[l >> c] | (l & cm)));
}
__device__ __forceinline__ void prefetch16(double2* s, const double2* g, const u32* tbl, int t, int c) {
  const int cm = (1 << c) - 1, nv = 1 << t;
  for (int l = threadIdx.x; l < nv; l += blockDim.x) cp_async16(s + swz16(l), g + (tbl[l >> c] | (l & cm)));
}
// Tile copies with the thread count (2^LT), tile bits TB and contiguous low
// bits CB known at compile time.  Amplitude l = tid | (i << LT); the swizzle
// is XOR-linear, so swz(l) = swz(tid) ^ swz(i << LT) with the second term a
// constant; likewise l >> CB = (tid >> CB) | ((i << LT) >> CB) and
// l & cm = (tid & cm) | ((i << LT) & cm) split into a per-thread and a constant part.
template <int LT, int TB, int CB>
__device__ __forceinline__ void prefetch8t(float2* s, const float2* g, const u32* tbl) {
  constexpr u32 cm = (1u << CB) - 1u;
  const u32 tid = threadIdx.x, st = swz8(tid), lo = tid & cm;
  const u32* tb = tbl + (tid >> CB);
#pragma unroll
  for (int i = 0; i < (1 << (TB - LT)); ++i) {
    const u32 hi = (u32)i << LT;
    cp_async8(s + (st ^ swz8(hi)), g + (tb[hi >> CB] | lo | (hi & cm)));
  }
}
template <int LT, int TB, int CB>
__device__ __forceinline__ void prefetch16t(double2* s, const double2* g, const u32* tbl) {
  constexpr u32 cm = (1u << CB) - 1u;
  const u32 tid = threadIdx.x, st = swz16(tid), lo = tid & cm;
  const u32* tb = tbl + (tid >> CB);
#pragma unroll
  for (int i = 0; i < (1 << (TB - LT)); ++i) {
    const u32 hi = (u32)i << LT;
    cp_async16(s + (st ^ swz16(hi)), g + (tb[hi >> CB] | lo | (hi & cm)));
  }
}
// complex64 store: pairs (2v, 2v + 1), v = tid | (i << LT), one 16-byte store
// each (CB >= 1: the pair is contiguous in global memory)
template <int LT, int TB, int CB>
__device__ __forceinline__ void store8t(const float2* s, float2* g, const u32* tbl) {
  static_assert(CB >= 1, "complex64 pairs need one contiguous low bit");
  constexpr u32 cm = (1u << CB) - 1u;
  const u32 tid = threadIdx.x, l0 = 2 * tid, s0 = swz8(l0), s1 = swz8(l0 + 1), lo = l0 & cm;
  const u32* tb = tbl + (l0 >> CB);
#pragma unroll
  for (int i = 0; i < (1 << (TB - 1 - LT)); ++i) {
    const u32 hi = (u32)i << (LT + 1);
    const u32 k = swz8(hi);
    const float2 a = s[s0 ^ k], b = s[s1 ^ k];
    __stcs((float4*)(g + (tb[hi >> CB] | lo | (hi & cm))), make_float4(a.x, a.y, b.x, b.y));
  }
}
template <int LT, int TB, int CB>
__device__ __forceinline__ void store16t(const double2* s, double2* g, const u32* tbl) {
  constexpr u32 cm = (1u << CB) - 1u;
  const u32 tid = threadIdx.x, st = swz16(tid), lo = tid & cm;
  const u32* tb = tbl + (tid >> CB);
#pragma unroll
  for (int i = 0; i < (1 << (TB - LT)); ++i) {
    const u32 hi = (u32)i << LT;
    __stcs(g + (tb[hi >> CB] | lo | (hi & cm)), s[st ^ swz16(hi)]);
  }
}
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
template <int B>
__device__ __forceinline__ void load8(float2* s, const float2* g, const u32* tbl, int t, int c) {
  const int cm = (1 << c) - 1, nv = (1 << t) / 2;
  for (int v0 = threadIdx.x; v0 < nv; v0 += B * blockDim.x) {
    float4 r[B];
#pragma unroll
    for (int u = 0; u < B; ++u) { const int v = v0 + u * blockDim.x; if (v < nv) { const int l = 2 * v; r[u] = __ldcs((const float4*)(g + (tbl[l >> c] | (l & cm)))); } }
#pragma unroll
    for (int u = 0; u < B; ++u) { const int v = v0 + u * blockDim.x; if (v < nv) { const u32 l = 2 * v; s[swz8(l)] = make_float2(r[u].x, r[u].y); s[swz8(l + 1)] = make_float2(r[u].z, r[u].w); } }
  }
}
template <int B>
__device__ __forceinline__ void store8(const float2* s, float2* g, const u32* tbl, int t, int c) {
  const int cm = (1 << c) - 1, nv = (1 << t) / 2;
  for (int v0 = threadIdx.x; v0 < nv; v0 += B * blockDim.x) {
    float4 r[B];
#pragma unroll
    for (int u = 0; u < B; ++u) { const int v = v0 + u * blockDim.x; if (v < nv) { const u32 l = 2 * v; const float2 a = s[swz8(l)], b = s[swz8(l + 1)]; r[u] = make_float4(a.x, a.y, b.x, b.y); } }
#pragma unroll
    for (int u = 0; u < B; ++u) { const int v = v0 + u * blockDim.x; if (v < nv) { const int l = 2 * v; __stcs((float4*)(g + (tbl[l >> c] | (l & cm))), r[u]); } }
  }
}
template <int B>
__device__ __forceinline__ void load16(double2* s, const double2* g, const u32* tbl, int t, int c) {
  const int cm = (1 << c) - 1, nv = 1 << t;
  for (int v0 = threadIdx.x; v0 < nv; v0 += B * blockDim.x) {
    double2 r[B];
#pragma unroll
    for (int u = 0; u < B; ++u) { const int v = v0 + u * blockDim.x; if (v < nv) r[u] = __ldcs(g + (tbl[v >> c] | (v & cm))); }
#pragma unroll
    for (int u = 0; u < B; ++u) { const int v = v0 + u * blockDim.x; if (v < nv) s[swz16(v)] = r[u]; }
  }
}
template <int B>
__device__ __forceinline__ void store16(const double2* s, double2* g, const u32* tbl, int t, int c) {
  const int cm = (1 << c) - 1, nv = 1 << t;
  for (int v0 = threadIdx.x; v0 < nv; v0 += B * blockDim.x) {
    double2 r[B];
#pragma unroll
    for (int u = 0; u < B; ++u) { const int v = v0 + u * blockDim.x; if (v < nv) r[u] = s[swz16(v)]; }
#pragma unroll
    for (int u = 0; u < B; ++u) { const int v = v0 + u * blockDim.x; if (v < nv) __stcs(g + (tbl[v >> c] | (v & cm)), r[u]); }
  }
}
// Warp reduce-scatter of N (power of two, <= 32) per-lane partial sums by
// recursive halving: at the step exchanging with lane ^ o the lanes with bit o
// set keep the upper half of the remaining values.  N - 1 shuffles for the
// halving steps plus one per remaining lane bit; afterwards the top log2(N)
// lane bits index the value a lane holds and the lanes whose low bits are zero
// add it into dst[index] (float64 shared accumulators).
template <int O, int N, typename F> struct WarpRS {
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
template <int N, typename F> __device__ __forceinline__ void warp_rs_add(F (&v)[N], double* dst) {
  const unsigned lane = threadIdx.x & 31u;
  WarpRS<16, N, F>::run(v, lane);
  constexpr int lg = (N >= 32) ? 5 : (N >= 16) ? 4 : (N >= 8) ? 3 : (N >= 4) ? 2 : (N >= 2) ? 1 : 0;
  if ((lane & ((32u >> lg) - 1u)) == 0) atomicAdd(dst + (lane >> (5 - lg)), (double)v[0]);
}
// Packed-float32 complex dot products (sm_100 two-lane FMA): with the matrix
// entries staged as broadcast pairs (re, re) and (im, im),
//   p = sum_q Re(m_q) (x_q.re, x_q.im),  s = sum_q Im(m_q) (x_q.re, x_q.im),
//   sum_q m_q x_q = (p.re - s.im, p.im + s.re).
__device__ __forceinline__ float2 cdot2(float2 ar, float2 ai, float2 br, float2 bi, float2 x, float2 y) {
  float2 p = __fmul2_rn(ar, x), q = __fmul2_rn(ai, x);
  p = __ffma2_rn(br, y, p);
  q = __ffma2_rn(bi, y, q);
  return make_float2(p.x - q.y, p.y + q.x);
}
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }
// mb: one float4 (re, re, im, im) per matrix entry (one 16-byte shared load each)
__device__ __forceinline__ float2 cdot4(const float4* mb, float2 a0, float2 a1, float2 a2, float2 a3) {
  const float4 m0 = mb[0], m1 = mb[1], m2 = mb[2], m3 = mb[3];
  float2 p = __fmul2_rn(lo2(m0), a0), q = __fmul2_rn(hi2(m0), a0);
  p = __ffma2_rn(lo2(m1), a1, p);
  q = __ffma2_rn(hi2(m1), a1, q);
  p = __ffma2_rn(lo2(m2), a2, p);
  q = __ffma2_rn(hi2(m2), a2, q);
  p = __ffma2_rn(lo2(m3), a3, p);
  q = __ffma2_rn(hi2(m3), a3, q);
  return make_float2(p.x - q.y, p.y + q.x);
}
// sum_q conj(m_q) x_q from the same broadcast pairs
__device__ __forceinline__ float2 cdot2c(float2 ar, float2 ai, float2 br, float2 bi, float2 x, float2 y) {
  float2 p = __fmul2_rn(ar, x), q = __fmul2_rn(ai, x);
  p = __ffma2_rn(br, y, p);
  q = __ffma2_rn(bi, y, q);
  return make_float2(p.x + q.y, p.y - q.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
)JQ";

std::string hex(uint64_t v) {
  char b[32];
  std::snprintf(b, sizeof(b), "0x%llxull", static_cast<unsigned long long>(v));
  return b;
}

// Straight-line bit deposit of `v` into the set bits of `mask`: one
// shift-and-mask term per contiguous run of mask bits.
std::string pdep_expr(const std::string& v, uint64_t mask) {
  std::string e;
  int src = 0;
  for (int b = 0; b < 64;) {
    if (!((mask >> b) & 1)) { ++b; continue; }
    int len = 0;
    while (b + len < 64 && ((mask >> (b + len)) & 1)) ++len;
    const uint64_t lm = (len >= 64) ? ~0ULL : ((1ULL << len) - 1);
    std::string term = "(((" + v + ") >> " + std::to_string(src) + ") & " + hex(lm) + ")";
    if (b) term = "(" + term + " << " + std::to_string(b) + ")";
    e += (e.empty() ? "" : " | ") + term;
    src += len;
    b += len;
  }
  return e.empty() ? std::string("0ull") : "(" + e + ")";
}

// Split-complex form of a complex64 register stage.  Amplitudes are held in
// pairs (v, v ^ sp) as R = (re_v, re_{v^sp}) and I = (im_v, im_{v^sp}), so a
// one-qubit gate costs four packed FMAs per amplitude instead of six (no
// re/im cross terms to recombine).  Valid when every gate and swap of the
// stage maps the pairing onto itself: for each of its variable pairs (x, y)
// the pair (x ^ sp, y ^ sp) is one of its pairs too, in the same roles, and x,
// y sit in the same lane (the lane of v is the parity of v & lane_sel).
struct SplitStage {
  bool ok = false;
  uint32_t sp = 0, lane_sel = 0;
};

static int parity32(uint32_t v) { return __builtin_popcount(v) & 1; }

// rops [ri0, rb_end) of a stage with nr register slots; `dense_min` one-qubit
// gates at least (the pack / unpack moves must pay off).
static SplitStage plan_split(const Schedule& s, int ri0, int rb_end, int nr, int dense_min) {
  SplitStage res;
  std::vector<int> var(nr);
  for (int j = 0; j < nr; ++j) var[j] = j;
  std::vector<std::vector<std::pair<int, int>>> lists;  // ordered (x, y) pairs per gate / swap
  std::vector<bool> ordered;
  int ndense = 0;
  for (int ri = ri0; ri < rb_end; ++ri) {
    const RegOp& ro = s.rops[ri];
    const uint32_t kind = ro.w0 & 15u, q1 = (ro.w0 >> 4) & 15u;
    const uint32_t crm = ro.w1 & 0xFFu, ctm = (ro.w1 >> 8) & 0xFFFFu;
    if (kind != RK_DENSE1 && kind != RK_PERM1) return res;
    std::vector<std::pair<int, int>> pr;
    for (int j = 0; j < nr; ++j) {
      if ((j >> q1) & 1) continue;
      if ((static_cast<uint32_t>(j) & crm) != crm) continue;
      const int k = j | (1 << q1);
      if (kind == RK_PERM1 && ctm == 0) std::swap(var[j], var[k]);
      else pr.emplace_back(var[j], var[k]);
    }
    if (kind == RK_DENSE1) ++ndense;
    if (!pr.empty()) {
      lists.push_back(std::move(pr));
      ordered.push_back(kind == RK_DENSE1);
    }
  }
  if (ndense < dense_min) return res;
  for (uint32_t sp = 1; sp < static_cast<uint32_t>(nr); ++sp) {
    for (uint32_t ls = 1; ls < static_cast<uint32_t>(nr); ++ls) {
      if (!parity32(ls & sp)) continue;
      bool good = true;
      for (size_t li = 0; li < lists.size() && good; ++li) {
        const auto& L = lists[li];
        for (const auto& xy : L) {
          const uint32_t x = xy.first, y = xy.second;
          if (parity32(ls & (x ^ y))) { good = false; break; }
          bool found = false;
          for (const auto& uv : L) {
            const uint32_t u = uv.first, v = uv.second;
            if ((u == (x ^ sp) && v == (y ^ sp)) || (!ordered[li] && u == (y ^ sp) && v == (x ^ sp))) {
              found = true;
              break;
            }
          }
          if (!found) { good = false; break; }
        }
      }
      if (good) {
        res.ok = true;
        res.sp = sp;
        res.lane_sel = ls;
        return res;
      }
    }
  }
  return res;
}

}  // namespace

// Tile buffers of a forward pass (2: double buffering; JQ_JIT_BUFS=3 or 4
// keeps more tiles in flight per CTA).
int jit_bufs() {
  static const int n = [] {
    const char* e = std::getenv("JQ_JIT_BUFS");
    return e ? std::max(2, std::min(4, std::atoi(e))) : 2;
  }();
  return n;
}

// Tile load with literal offsets: amplitude l = tid | (i << lt) goes to
// shared offset swz(tid) ^ swz(i << lt) from global offset gdep(tid) ^
// gdep(i << lt) (both maps XOR-linear); `sw` and `gd` are those maps.
template <typename SW, typename GD>
std::string tile_load_literal(bool c64, int t, int lt, bool wide, SW sw, GD gd, const std::string& sdst,
                              const std::string& gsrc) {
  std::ostringstream o;
  const char* OT = wide ? "u64" : "u32";
  const char* L = wide ? "ull" : "u";
  o << "    { const u32 tst = " << (c64 ? "swz8" : "swz16") << "(tid); " << OT << " tgo = 0;";
  for (int i = 0; i < lt; ++i) o << " if (tid & " << (1u << i) << "u) tgo ^= " << gd(1ULL << i) << L << ";";
  o << "\n";
  for (int i = 0; i < (1 << (t - lt)); ++i) {
    const uint64_t hi = static_cast<uint64_t>(i) << lt;
    o << "      " << (c64 ? "cp_async8" : "cp_async16") << "(" << sdst << " + (tst ^ " << sw(hi) << "u), " << gsrc
      << " + (tgo ^ " << gd(hi) << L << "));\n";
  }
  o << "    }\n";
  return o.str();
}

// JQ_JIT_PFTBL=1: tile loads through the shared-memory deposit table
bool pf_table_env() {
  static const bool on = [] {
    const char* e = std::getenv("JQ_JIT_PFTBL");
    return e && std::atoi(e) == 1;
  }();
  return on;
}

// One-qubit dense blocks of forward passes read their matrix as two 16-byte
// (re, im) loads instead of four broadcast-pair loads (JQ_JIT_COMPACT=0: the
// broadcast pairs).
bool compact_mats() {
  static const bool on = [] {
    const char* e = std::getenv("JQ_JIT_COMPACT");
    return !(e && std::atoi(e) == 0);
  }();
  return on;
}

// Broadcast pairs (re, re), (im, im) of a complex64 one-qubit matrix at
// smat[M..M+3] (m00, m01, m10, m11) as ar..di: a b / c d are the rows of G,
// or of G^dagger (a = conj-free m00, b = m10, c = m01, d = m11; the
// conjugation is in cdot2c).
std::string dense1_coefs(uint32_t M, bool dagger, const std::string& ind, bool su2) {
  if (su2 && compact_mats() && M % 2 == 0) {
    // SU(2): one 16-byte load of (m00, m01); m10 = -conj m01, m11 = conj m00
    const std::string b = dagger ? "-m01.z" : "m01.z", bi = dagger ? "m01.w" : "m01.w";
    const std::string c = dagger ? "m01.z" : "-m01.z", ci = dagger ? "m01.w" : "m01.w";
    return ind + "const float4 m01 = *(const float4*)(smat + " + std::to_string(M) + ");\n" + ind +
           "const float2 ar = make_float2(m01.x, m01.x), ai = make_float2(m01.y, m01.y), br = make_float2(" + b + ", " +
           b + "), bi = make_float2(" + bi + ", " + bi + "), cr = make_float2(" + c + ", " + c + "), ci = make_float2(" +
           ci + ", " + ci + "), dr = make_float2(m01.x, m01.x), di = make_float2(-m01.y, -m01.y);\n";
  }
  if (compact_mats() && M % 2 == 0) {
    const char* b = dagger ? "m23.x" : "m01.z";
    const char* bi = dagger ? "m23.y" : "m01.w";
    const char* c = dagger ? "m01.z" : "m23.x";
    const char* ci = dagger ? "m01.w" : "m23.y";
    return ind + "const float4 m01 = *(const float4*)(smat + " + std::to_string(M) + "), m23 = *(const float4*)(smat + " +
           std::to_string(M + 2) + ");\n" + ind +
           "const float2 ar = make_float2(m01.x, m01.x), ai = make_float2(m01.y, m01.y), br = make_float2(" + b + ", " +
           b + "), bi = make_float2(" + bi + ", " + bi + "), cr = make_float2(" + c + ", " + c + "), ci = make_float2(" +
           ci + ", " + ci + "), dr = make_float2(m23.z, m23.z), di = make_float2(m23.w, m23.w);\n";
  }
  return ind + "const float4* mq = (const float4*)smatb + " + std::to_string(M) + ";\n" + ind +
         (dagger ? "const float4 A = mq[0], Bq = mq[2], Cq = mq[1], Dq = mq[3];\n"
                 : "const float4 A = mq[0], Bq = mq[1], Cq = mq[2], Dq = mq[3];\n") +
         ind + "const float2 ar = lo2(A), ai = hi2(A), br = lo2(Bq), bi = hi2(Bq), cr = lo2(Cq), ci = hi2(Cq), "
               "dr = lo2(Dq), di = hi2(Dq);\n";
}

// Tile order of consecutive forward passes: alternately ascending and
// descending, so that each pass starts on the tiles the pass before it wrote
// last (24-qubit sweep: -1% a step); JQ_JIT_REV=0 keeps every pass ascending.
bool alternate_tile_order() {
  static const bool on = [] {
    const char* e = std::getenv("JQ_JIT_REV");
    return !(e && std::atoi(e) == 0);
  }();
  return on;
}

namespace {

// Consecutive register stages a then b with the warp-index thread bits
// (above the 5 lane bits) on the same tile positions: every warp reads in b
// exactly the amplitudes it wrote in a, so a warp barrier orders them.
bool warp_owned(const Step& a, const Step& b, int nthb) {
  if (a.kind != 0 || b.kind != 0 || nthb <= 5) return false;
  for (int i = 5; i < nthb; ++i)
    if (a.tbits[i] != b.tbits[i]) return false;
  return true;
}

// Emit the kernel of pass p (register-stage program only).
void emit_pass(std::ostringstream& o, const jq_plan* plan, const Schedule& s, int p, bool c64, int rb) {
  const PassDesc& pd = s.passes[p];
  const char* T = c64 ? "float2" : "double2";
  const int t = pd.t, c = pd.c, nb = plan->n_bits;
  const int nthr = 1 << (t - rb);
  const int nr = 1 << rb;
  // register budget: 16 complex64 amplitudes fit about 100 registers (5
  // CTAs of 128 threads an SM: 4.29 -> 4.21 ms for the 24-qubit sweep against
  // 4 CTAs at 128 registers); complex128 needs about 168
  int minb = std::max(1, std::min(8, 65536 / (nthr * (c64 ? 100 : 168))));
  if (const char* e = std::getenv("JQ_JIT_MINB")) minb = std::max(1, std::min(16, std::atoi(e)));
  // complex64 dense blocks use packed two-lane FMA unless JQ_JIT_SCALAR=1
  const bool packed = c64 && !(std::getenv("JQ_JIT_SCALAR") && std::atoi(std::getenv("JQ_JIT_SCALAR")) == 1);
  // split-complex stages (see plan_split) with JQ_JIT_SPLIT=1
  const bool split_on = packed && std::getenv("JQ_JIT_SPLIT") && std::atoi(std::getenv("JQ_JIT_SPLIT")) == 1;
  const uint64_t full = (nb >= 64) ? ~0ULL : ((1ULL << nb) - 1);
  const uint64_t outer = full & ~pd.tile_mask;
  const int smat_pad = (pd.smat_len + 1) & ~1;
  int nmc = 0;
  for (int ri = pd.rop_begin; ri < pd.rop_end; ++ri) nmc += s.rops[ri].mat_len > 0;
  // the pass reads `state` and writes `out` (the same buffer for an
  // in-place pass, another one for the checkpointed reverse pass's recompute)
  o << "extern \"C\" __global__ void __launch_bounds__(" << nthr << ", " << minb << ") @KERNEL@(" << T
    << "* state, int batch, const " << T << "* __restrict__ bmat, long long bstride, "
    << "const int* __restrict__ mc, " << T << "* out, int rev) {\n";
  // nbuf tile buffers: the next nbuf - 1 tiles stream in (cp.async) while
  // this one is computed
  const int nbuf = jit_bufs();
  o << "  extern __shared__ __align__(16) unsigned char smem[];\n";
  o << "  " << T << "* s0 = (" << T << "*)smem;\n";
  o << "  " << T << "* smat = s0 + " << nbuf * (1 << t) << ";\n";
  if (c64) {
    // broadcast copies (re, re), (im, im) of every staged matrix entry
    o << "  float2* smatb = smat + " << smat_pad << ";\n";
    o << "  u32* tbl = (u32*)(smatb + " << 2 * smat_pad << ");\n";
  } else {
    o << "  u32* tbl = (u32*)(smat + " << smat_pad << ");\n";
  }
  o << "  const u32 tid = threadIdx.x;\n";
  o << kPdlTrigger;
  // bit-deposit table of the tile's high bits
  o << "  { const u32 hb[] = {";
  for (int i = c; i < t; ++i) o << (i > c ? ", " : "") << (1u << pd.bits[i]);
  if (t == c) o << "0u";
  o << "};\n    for (int h = tid; h < " << (1 << (t - c)) << "; h += blockDim.x) { u32 v = 0;";
  o << " for (int i = 0; i < " << (t - c) << "; ++i) if ((h >> i) & 1) v |= hb[i]; tbl[h] = v; } }\n";
  // per-stage thread bases (tile independent)
  int nstage = 0;
  for (int si = pd.step_begin; si < pd.step_end; ++si) {
    const Step& st = s.steps[si];
    o << "  u32 tb" << nstage << " = 0;";
    for (int i = 0; i < t - rb; ++i) o << " if (tid & " << (1u << i) << "u) tb" << nstage << " ^= " << st.tbits[i] << "u;";
    o << "\n";
    ++nstage;
  }
  // The last stage stores its registers straight to global memory (skipping
  // the shared-memory write-back and the tile copy-out) when its lowest lane
  // bits hold the lowest tile bits, so that every 32-byte sector is written
  // whole by one warp instruction: lanes 0-3 (complex64) or lanes 0-1
  // (complex128) on tile bits 0-1 / 0, which are contiguous in global memory.
  // The tile's logical index of a shared-memory offset is its swizzle (an
  // XOR-linear involution) and the global offset of a logical index is the
  // deposit of its bits (also XOR-linear), so the global offset of register
  // slot j is a per-thread base XOR a compile-time constant.
  const Step& last = s.steps[pd.step_end - 1];
  bool direct = t - rb >= 2 && c >= 2 &&
                (c64 ? (last.tbits[0] == 1u && last.tbits[1] == 2u) : last.tbits[0] == 1u);
  if (const char* e = std::getenv("JQ_JIT_DIRECT_STORE")) direct = direct && std::atoi(e) != 0;
  const bool wide = nb > 31;
  const char* OT = wide ? "u64" : "u32";
  auto unswz = [&](uint64_t a) -> uint64_t {  // swz8 / swz16 of the device prelude (involutions)
    if (c64) return a ^ (((a >> 4) ^ (a >> 8) ^ (a >> 12)) & 15u);
    return a ^ (((a >> 3) ^ (a >> 6) ^ (a >> 9) ^ (a >> 12)) & 7u);
  };
  auto gdep = [&](uint64_t logical) -> uint64_t {  // global offset of a tile-local index
    uint64_t g = 0;
    for (int i = 0; i < t; ++i)
      if ((logical >> i) & 1) g |= 1ULL << pd.bits[i];
    return g;
  };
  if (direct) {
    o << "  " << OT << " gt = 0;";
    for (int i = 0; i < t - rb; ++i)
      o << " if (tid & " << (1u << i) << "u) gt ^= " << gdep(unswz(last.tbits[i])) << (wide ? "ull;" : "u;");
    o << "\n";
  }
  const std::string tpl = "<" + std::to_string(t - rb) + ", " + std::to_string(t) + ", " + std::to_string(c) + ">";
  // Tile loads: amplitude l = tid | hi (hi = i << LT) goes to shared offset
  // swz(tid) ^ swz(hi) from global offset gdep(tid) ^ gdep(hi), both
  // XOR-linear, so every copy is a per-thread base XOR a literal (no table
  // lookups; JQ_JIT_PFTBL=1 keeps the table-driven copy)
  const bool pf_table = std::getenv("JQ_JIT_PFTBL") && std::atoi(std::getenv("JQ_JIT_PFTBL")) == 1;
  std::string pf = (c64 ? "prefetch8t" : "prefetch16t") + tpl;
  const char* PFEND = pf_table ? ", tbl)" : ")";
  if (!pf_table) {
    const int lt = t - rb;
    o << "  // tile copy: " << t << " tile bits, the lowest " << c << " contiguous\n";
    o << "  const u32 pst = " << (c64 ? "swz8" : "swz16") << "(tid);\n";
    o << "  " << OT << " pgo = 0;";
    for (int i = 0; i < lt; ++i) o << " if (tid & " << (1u << i) << "u) pgo ^= " << gdep(1ULL << i) << (wide ? "ull;" : "u;");
    o << "\n";
    if (c64 && !direct) {  // copy-out base of the pair (2 tid, 2 tid + 1)
      o << "  const u32 pso0 = swz8(2u * tid), pso1 = swz8(2u * tid + 1u);\n";
      o << "  " << OT << " pgo2 = 0;";
      for (int i = 0; i < lt; ++i)
        o << " if (tid & " << (1u << i) << "u) pgo2 ^= " << gdep(2ULL << i) << (wide ? "ull;" : "u;");
      o << "\n";
    }
    o << "  auto pfx = [&](" << T << "* sd, const " << T << "* gs) {\n";
    for (int i = 0; i < (1 << (t - lt)); ++i) {
      const uint64_t hi = static_cast<uint64_t>(i) << lt;
      o << "    " << (c64 ? "cp_async8" : "cp_async16") << "(sd + (pst ^ " << unswz(hi) << "u), gs + (pgo ^ " << gdep(hi)
        << (wide ? "ull" : "u") << "));\n";
    }
    o << "  };\n";
    pf = "pfx";
  }
  o << "  const long long tiles_per = 1ll << " << (nb - t) << ";\n";
  o << "  const long long ntiles = tiles_per * batch;\n";
  // rev != 0 walks an instance's tiles in descending order (tile index bits
  // complemented), so a pass that follows an ascending one starts on the
  // amplitudes written last, which are still in L2
  o << "  const u64 rmask = rev ? (u64)(tiles_per - 1) : 0ull;\n";
  o << "  auto gaddr = [&](long long tl) { const u64 ti = ((u64)tl & (u64)(tiles_per - 1)) ^ rmask; return state + ((tl >> "
    << (nb - t) << ") << " << nb << ") + " << pdep_expr("ti", outer) << "; };\n";
  o << "  __syncthreads();\n";
  o << kPdlWait;  // the state is read (and written) only after the previous pass completed
  for (int j = 0; j + 1 < nbuf; ++j) {
    o << "  if ((long long)blockIdx.x + " << j << "ll * gridDim.x < ntiles) " << pf << "(s0 + " << j * (1 << t)
      << ", gaddr(blockIdx.x + " << j << "ll * gridDim.x)" << PFEND << ";\n";
    o << "  cp_commit();\n";
  }
  o << "  long long last_inst = -1;\n";
  o << "  int cur = 0;\n";
  o << "  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {\n";
  o << "    " << T << "* s = s0 + cur * " << (1 << t) << ";\n";
  o << "    { const int nx = cur == 0 ? " << nbuf - 1 << " : cur - 1;  // the buffer computed last\n";
  o << "      const long long ahead = tile + " << nbuf - 1 << "ll * gridDim.x;\n";
  o << "      if (ahead < ntiles) " << pf << "(s0 + nx * " << (1 << t) << ", gaddr(ahead)" << PFEND << "; }\n";
  o << "    cur = cur + 1 == " << nbuf << " ? 0 : cur + 1;\n";
  o << "    cp_commit();\n";
  o << "    const long long inst = tile >> " << (nb - t) << ";\n";
  o << "    " << T << "* g = out + (gaddr(tile) - state);\n";
  // gate matrices of this pass: mc holds (smem offset, block-matrix offset,
  // length) per matrix, so passes that differ only in their gates share code
  o << "    if (inst != last_inst) {\n      const " << T << "* bm = bmat + inst * bstride;\n";
  o << "      for (int i = 0; i < " << nmc << "; ++i) { const int d = mc[3 * i], a = mc[3 * i + 1], n = mc[3 * i + 2];\n";
  if (c64)
    o << "        for (int e = tid; e < n; e += blockDim.x) { const float2 v = bm[a + e]; smat[d + e] = v; "
         "smatb[2 * (d + e)] = make_float2(v.x, v.x); smatb[2 * (d + e) + 1] = make_float2(v.y, v.y); } }\n";
  else
    o << "        for (int e = tid; e < n; e += blockDim.x) smat[d + e] = bm[a + e]; }\n";
  o << "      (void)bm; last_inst = inst;\n    }\n";
  o << "    cp_waitn<" << nbuf - 1 << ">();\n";
  o << "    __syncthreads();\n";
  nstage = 0;
  for (int si = pd.step_begin; si < pd.step_end; ++si) {
    const Step& st = s.steps[si];
    // address of register slot j
    std::vector<uint32_t> off(nr);
    for (int j = 0; j < nr; ++j) {
      uint32_t a = 0;
      for (int q = 0; q < rb; ++q)
        if ((j >> q) & 1) a ^= st.ebits[q];
      off[j] = a;
    }
    std::vector<int> var(nr);  // var[j]: variable holding amplitude j of the register block
    for (int j = 0; j < nr; ++j) var[j] = j;
    o << "    {\n";
    // Thread-controlled swaps of whole register halves (a permutation whose
    // control is a thread bit and whose target is a register bit, with no
    // register-bit control) at the head of the stage become part of the load
    // address: slot j of a controlled thread loads slot j ^ 2^q1, i.e. the
    // base offset moves by the offset of register bit q1.  The stores keep the
    // unmoved base.
    int ri0 = st.a;
    std::string lbase = "tb" + std::to_string(nstage);
    while (ri0 < st.b) {
      const RegOp& ro = s.rops[ri0];
      const uint32_t kind = ro.w0 & 15u, q1 = (ro.w0 >> 4) & 15u;
      const uint32_t crm = ro.w1 & 0xFFu, ctm = (ro.w1 >> 8) & 0xFFFFu;
      if (kind != RK_PERM1 || ctm == 0 || crm != 0) break;
      if (ri0 == st.a) o << "      u32 tl = " << lbase << ";\n";
      o << "      if ((tid & " << ctm << "u) == " << ctm << "u) tl ^= " << st.ebits[q1] << "u;\n";
      lbase = "tl";
      ++ri0;
    }
    for (int j = 0; j < nr; ++j) o << "      " << T << " v" << j << " = s[" << lbase << " ^ " << off[j] << "u];\n";
    const SplitStage sps = split_on ? plan_split(s, ri0, st.b, nr, 2) : SplitStage{};
    auto is_lead = [&](int v) { return !parity32(sps.lane_sel & static_cast<uint32_t>(v)); };
    std::vector<int> lead(nr);  // lane-0 variable of the pack holding variable v
    if (sps.ok) {
      for (int v = 0; v < nr; ++v) lead[v] = is_lead(v) ? v : (v ^ static_cast<int>(sps.sp));
      for (int l = 0; l < nr; ++l)
        if (is_lead(l))
          o << "      float2 R" << l << " = make_float2(v" << l << ".x, v" << (l ^ sps.sp) << ".x), I" << l
            << " = make_float2(v" << l << ".y, v" << (l ^ sps.sp) << ".y);\n";
    }
    // final value of register slot j
    auto outv = [&](int j) -> std::string {
      if (!sps.ok) return "v" + std::to_string(var[j]);
      const int v = var[j], l = lead[v];
      const std::string ln = (v == l) ? ".x" : ".y";
      return "make_float2(R" + std::to_string(l) + ln + ", I" + std::to_string(l) + ln + ")";
    };
    for (int ri = ri0; ri < st.b; ++ri) {
      const RegOp& ro = s.rops[ri];
      const uint32_t kind = ro.w0 & 15u, q1 = (ro.w0 >> 4) & 15u, q2 = (ro.w0 >> 8) & 15u;
      const uint32_t dk = (ro.w0 >> 12) & 15u, dq = ro.w0 >> 16;
      const uint32_t crm = ro.w1 & 0xFFu, ctm = (ro.w1 >> 8) & 0xFFFFu, perm = ro.w1 >> 24;
      const uint32_t M = ro.w2;
      const bool guard = ctm != 0;
      if (sps.ok) {  // plan_split admitted only one-qubit gates and swaps
        if (guard) o << "      if ((tid & " << ctm << "u) == " << ctm << "u) {\n";
        else o << "      {\n";
        if (kind == RK_DENSE1) {
          o << "        const float4* mq = (const float4*)smatb + " << M << ";\n";
          o << "        const float4 A = mq[0], Bq = mq[1], Cq = mq[2], Dq = mq[3];\n";
          o << "        const float2 ar = lo2(A), ai = hi2(A), br = lo2(Bq), bi = hi2(Bq), cr = lo2(Cq), ci = hi2(Cq), "
               "dr = lo2(Dq), di = hi2(Dq);\n";
          o << "        const float2 nai = make_float2(-ai.x, -ai.y), nbi = make_float2(-bi.x, -bi.y), "
               "nci = make_float2(-ci.x, -ci.y), ndi = make_float2(-di.x, -di.y);\n";
        }
        for (int j = 0; j < nr; ++j) {
          if ((j >> q1) & 1) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int k = j | (1 << q1);
          if (kind == RK_PERM1 && !guard) {
            std::swap(var[j], var[k]);
            continue;
          }
          const int x = var[j], y = var[k];
          if (!is_lead(x)) continue;  // its pack is handled through the lane-0 pair
          const std::string Rx = "R" + std::to_string(x), Ix = "I" + std::to_string(x);
          const std::string Ry = "R" + std::to_string(y), Iy = "I" + std::to_string(y);
          if (kind == RK_PERM1) {
            o << "        { const float2 r = " << Rx << ", i = " << Ix << "; " << Rx << " = " << Ry << "; " << Ix << " = "
              << Iy << "; " << Ry << " = r; " << Iy << " = i; }\n";
            continue;
          }
          o << "        { const float2 rx = " << Rx << ", ix = " << Ix << ", ry = " << Ry << ", iy = " << Iy << ";\n";
          o << "          " << Rx << " = __ffma2_rn(nbi, iy, __ffma2_rn(br, ry, __ffma2_rn(nai, ix, __fmul2_rn(ar, rx))));\n";
          o << "          " << Ix << " = __ffma2_rn(bi, ry, __ffma2_rn(br, iy, __ffma2_rn(ai, rx, __fmul2_rn(ar, ix))));\n";
          o << "          " << Ry << " = __ffma2_rn(ndi, iy, __ffma2_rn(dr, ry, __ffma2_rn(nci, ix, __fmul2_rn(cr, rx))));\n";
          o << "          " << Iy << " = __ffma2_rn(di, ry, __ffma2_rn(dr, iy, __ffma2_rn(ci, rx, __fmul2_rn(cr, ix)))); }\n";
        }
        o << "      }\n";
        continue;
      }
      if (guard) o << "      if ((tid & " << ctm << "u) == " << ctm << "u) {\n";
      else o << "      {\n";
      auto V = [&](int j) { return std::string("v") + std::to_string(var[j]); };
      if (kind == RK_DENSE1 && packed) {
        if (compact_mats() && M % 2 == 0) {
          o << dense1_coefs(M, false, "        ", ro.pad[0] != 0);
        } else {
          o << "        const float4* mq = (const float4*)smatb + " << M << ";\n";
          o << "        const float4 A = mq[0], Bq = mq[1], Cq = mq[2], Dq = mq[3];\n";
          o << "        const float2 ar = lo2(A), ai = hi2(A), br = lo2(Bq), bi = hi2(Bq), cr = lo2(Cq), ci = hi2(Cq), "
               "dr = lo2(Dq), di = hi2(Dq);\n";
        }
        for (int j = 0; j < nr; ++j) {
          if ((j >> q1) & 1) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int k = j | (1 << q1);
          o << "        { const float2 x = " << V(j) << ", y = " << V(k) << "; " << V(j)
            << " = cdot2(ar, ai, br, bi, x, y); " << V(k) << " = cdot2(cr, ci, dr, di, x, y); }\n";
        }
      } else if (kind == RK_DENSE1) {
        o << "        const " << T << " m00 = smat[" << M << "], m01 = smat[" << M + 1 << "], m10 = smat[" << M + 2
          << "], m11 = smat[" << M + 3 << "];\n";
        for (int j = 0; j < nr; ++j) {
          if ((j >> q1) & 1) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int k = j | (1 << q1);
          o << "        { const " << T << " x = " << V(j) << ", y = " << V(k) << "; " << V(j)
            << " = cfma(m01, y, cmul(m00, x)); " << V(k) << " = cfma(m11, y, cmul(m10, x)); }\n";
        }
      } else if (kind == RK_PERM1) {
        for (int j = 0; j < nr; ++j) {
          if ((j >> q1) & 1) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int k = j | (1 << q1);
          if (!guard) {
            std::swap(var[j], var[k]);  // free: a rename
          } else {
            o << "        { const " << T << " x = " << V(j) << "; " << V(j) << " = " << V(k) << "; " << V(k)
              << " = x; }\n";
          }
        }
      } else if (kind == RK_DIAG) {
        for (int j = 0; j < nr; ++j) {
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          int idx = 0;
          for (uint32_t i = 0; i < dk; ++i) idx = (idx << 1) | ((j >> ((dq >> (3 * i)) & 7u)) & 1);
          o << "        " << V(j) << " = cmul(smat[" << M + idx << "], " << V(j) << ");\n";
        }
      } else if (kind == RK_DENSE2 && packed) {
        for (int j = 0; j < nr; ++j) {
          if (((j >> q1) & 1) || ((j >> q2) & 1)) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int id[4] = {j, j | (1 << q2), j | (1 << q1), j | (1 << q1) | (1 << q2)};
          o << "        { const float2 a0 = " << V(id[0]) << ", a1 = " << V(id[1]) << ", a2 = " << V(id[2])
            << ", a3 = " << V(id[3]) << ";\n";
          for (int r = 0; r < 4; ++r)
            o << "          " << V(id[r]) << " = cdot4((const float4*)smatb + " << M + 4 * r << ", a0, a1, a2, a3);\n";
          o << "        }\n";
        }
      } else if (kind == RK_DENSE2) {
        o << "        " << T << " mm[16];\n        for (int e = 0; e < 16; ++e) mm[e] = smat[" << M << " + e];\n";
        for (int j = 0; j < nr; ++j) {
          if (((j >> q1) & 1) || ((j >> q2) & 1)) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int id[4] = {j, j | (1 << q2), j | (1 << q1), j | (1 << q1) | (1 << q2)};
          o << "        { const " << T << " a0 = " << V(id[0]) << ", a1 = " << V(id[1]) << ", a2 = " << V(id[2])
            << ", a3 = " << V(id[3]) << ";\n";
          for (int r = 0; r < 4; ++r)
            o << "          " << V(id[r]) << " = cfma(mm[" << 4 * r + 3 << "], a3, cfma(mm[" << 4 * r + 2
              << "], a2, cfma(mm[" << 4 * r + 1 << "], a1, cmul(mm[" << 4 * r << "], a0))));\n";
          o << "        }\n";
        }
      } else {  // RK_PERM2: output row r takes input column p[r]
        for (int j = 0; j < nr; ++j) {
          if (((j >> q1) & 1) || ((j >> q2) & 1)) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int id[4] = {j, j | (1 << q2), j | (1 << q1), j | (1 << q1) | (1 << q2)};
          int pv[4];
          for (int r = 0; r < 4; ++r) pv[r] = (perm >> (2 * r)) & 3u;
          if (!guard) {
            int nv[4];
            for (int r = 0; r < 4; ++r) nv[r] = var[id[pv[r]]];
            for (int r = 0; r < 4; ++r) var[id[r]] = nv[r];
          } else {
            o << "        { const " << T << " a0 = " << V(id[0]) << ", a1 = " << V(id[1]) << ", a2 = " << V(id[2])
              << ", a3 = " << V(id[3]) << ";";
            for (int r = 0; r < 4; ++r) o << " " << V(id[r]) << " = a" << pv[r] << ";";
            o << " }\n";
          }
        }
      }
      o << "      }\n";
    }
    if (direct && si == pd.step_end - 1) {
      for (int j = 0; j < nr; ++j) {
        uint64_t gj = gdep(unswz(off[j]));
        o << "      __stcs(g + (gt ^ " << gj << (wide ? "ull" : "u") << "), " << outv(j) << ");\n";
      }
      o << "    }\n";
    } else {
      for (int j = 0; j < nr; ++j) o << "      s[tb" << nstage << " ^ " << off[j] << "u] = " << outv(j) << ";\n";
      o << "    }\n    " << (si + 1 < pd.step_end && warp_owned(st, s.steps[si + 1], t - rb) ? "__syncwarp()" : "__syncthreads()")
        << ";\n";
    }
    ++nstage;
  }
  // (direct: the barrier below keeps the next prefetch out of this buffer
  // until every warp has loaded its last stage)
  if (!direct && !pf_table) {
    // tile copy-out with the same per-thread base / literal split as the
    // loads (complex64: one 16-byte store of the pair (2 tid | hi, 2 tid | hi | 1))
    const int lt = t - rb;
    o << "    {\n";
    if (c64) {
      for (int i = 0; i < (1 << (t - 1 - lt)); ++i) {
        const uint64_t hi = static_cast<uint64_t>(i) << (lt + 1);
        o << "      { const float2 a = s[pso0 ^ " << unswz(hi) << "u], b = s[pso1 ^ " << unswz(hi)
          << "u]; __stcs((float4*)(g + (pgo2 ^ " << gdep(hi) << (wide ? "ull" : "u")
          << ")), make_float4(a.x, a.y, b.x, b.y)); }\n";
      }
    } else {
      for (int i = 0; i < (1 << (t - lt)); ++i) {
        const uint64_t hi = static_cast<uint64_t>(i) << lt;
        o << "      __stcs(g + (pgo ^ " << gdep(hi) << (wide ? "ull" : "u") << "), s[pst ^ " << unswz(hi) << "u]);\n";
      }
    }
    o << "    }\n";
  } else if (!direct) {
    o << "    " << (c64 ? "store8t" : "store16t") << tpl << "(s, g, tbl);\n";
  }
  o << "    __syncthreads();\n";
  o << "  }\n}\n";
}

// Emit the adjoint kernel of pass p: the pass's register stages in reverse,
// psi <- G^dagger psi, block cotangent += lam psi^dagger (float64 shared
// accumulators, flushed to the global accumulator per instance), lam <- G^dagger lam.
void emit_adj_pass(std::ostringstream& o, const jq_plan* plan, const Schedule& s, int p, bool c64, int rb) {
  const PassDesc& pd = s.passes[p];
  const char* T = c64 ? "float2" : "double2";
  const int t = pd.t, c = pd.c, nb = plan->n_bits;
  const int nthr = 1 << (t - rb);
  const int nr = 1 << rb;
  // both tiles' register blocks are live: allow up to 255 registers a thread
  int minb = std::max(1, std::min(8, 65536 / (nthr * 256)));
  if (const char* e = std::getenv("JQ_JIT_AMINB")) minb = std::max(1, std::min(16, std::atoi(e)));
  const uint64_t full = (nb >= 64) ? ~0ULL : ((1ULL << nb) - 1);
  const uint64_t outer = full & ~pd.tile_mask;
  const int smat_pad = (pd.smat_len + 1) & ~1;
  const char* F = c64 ? "float" : "double";
  int nmc = 0, ngt = 0, nacc = 0;
  std::vector<int> acc_off(pd.rop_end - pd.rop_begin, -1);
  for (int ri = pd.rop_begin; ri < pd.rop_end; ++ri) {
    const RegOp& ro = s.rops[ri];
    nmc += ro.mat_len > 0;
    if (ro.grad_off >= 0) {
      acc_off[ri - pd.rop_begin] = nacc;
      nacc += 2 * ro.mat_len;  // re/im of each entry of the inner matrix / diagonal
      ++ngt;
    }
  }
  const int nacc_pad = (nacc + 1) & ~1;
  o << "extern \"C\" __global__ void __launch_bounds__(" << nthr << ", " << minb << ") @KERNEL@(" << T
    << "* __restrict__ psi, " << T << "* __restrict__ lam, int batch, const " << T
    << "* __restrict__ bmat, long long bstride, const int* __restrict__ mc, double* __restrict__ gacc, "
    << "long long gstride, const int* __restrict__ gt) {\n";
  o << "  extern __shared__ __align__(16) unsigned char smem[];\n";
  o << "  " << T << "* sp = (" << T << "*)smem;\n";
  o << "  " << T << "* sl = sp + " << (1 << t) << ";\n";
  o << "  " << T << "* smat = sl + " << (1 << t) << ";\n";
  if (c64) {
    o << "  float2* smatb = smat + " << smat_pad << ";\n";
    o << "  double* sacc = (double*)(smatb + " << 2 * smat_pad << ");\n";
  } else {
    o << "  double* sacc = (double*)(smat + " << smat_pad << ");\n";
  }
  o << "  u32* tbl = (u32*)(sacc + " << nacc_pad << ");\n";
  o << "  const u32 tid = threadIdx.x;\n";
  o << kPdlTrigger << kPdlWait;
  o << "  { const u32 hb[] = {";
  for (int i = c; i < t; ++i) o << (i > c ? ", " : "") << (1u << pd.bits[i]);
  if (t == c) o << "0u";
  o << "};\n    for (int h = tid; h < " << (1 << (t - c)) << "; h += blockDim.x) { u32 v = 0;";
  o << " for (int i = 0; i < " << (t - c) << "; ++i) if ((h >> i) & 1) v |= hb[i]; tbl[h] = v; } }\n";
  o << "  for (int e = tid; e < " << nacc_pad << "; e += blockDim.x) sacc[e] = 0.0;\n";
  int nstage = 0;
  for (int si = pd.step_begin; si < pd.step_end; ++si) {
    const Step& st = s.steps[si];
    o << "  u32 tb" << nstage << " = 0;";
    for (int i = 0; i < t - rb; ++i) o << " if (tid & " << (1u << i) << "u) tb" << nstage << " ^= " << st.tbits[i] << "u;";
    o << "\n";
    ++nstage;
  }
  // The stage run last (the pass's first step) stores psi and lambda straight
  // to global memory under the same condition as the forward pass's last
  // stage; the barrier at the top of the next tile keeps the next loads out
  // of the tiles until every warp has read them.
  const Step& fin = s.steps[pd.step_begin];
  bool direct = t - rb >= 2 && c >= 2 &&
                (c64 ? (fin.tbits[0] == 1u && fin.tbits[1] == 2u) : fin.tbits[0] == 1u);
  if (const char* e = std::getenv("JQ_JIT_DIRECT_STORE")) direct = direct && std::atoi(e) != 0;
  const bool wide = nb > 31;
  auto unswz = [&](uint64_t v) -> uint64_t {
    if (c64) return v ^ (((v >> 4) ^ (v >> 8) ^ (v >> 12)) & 15u);
    return v ^ (((v >> 3) ^ (v >> 6) ^ (v >> 9) ^ (v >> 12)) & 7u);
  };
  auto gdep = [&](uint64_t logical) -> uint64_t {
    uint64_t g = 0;
    for (int i = 0; i < t; ++i)
      if ((logical >> i) & 1) g |= 1ULL << pd.bits[i];
    return g;
  };
  if (direct) {
    o << "  " << (wide ? "u64" : "u32") << " gpos = 0;";
    for (int i = 0; i < t - rb; ++i)
      o << " if (tid & " << (1u << i) << "u) gpos ^= " << gdep(unswz(fin.tbits[i])) << (wide ? "ull;" : "u;");
    o << "\n";
  }
  // flush of the shared accumulators into the instance's global accumulator
  // (skipped when the caller wants no parameter gradient: gacc is NULL)
  auto flush_for = [&](const std::string& inst) {
    return "      if (gacc) for (int i = 0; i < " + std::to_string(ngt) +
           "; ++i) { const int so = gt[3 * i], go = gt[3 * i + 1], n = gt[3 * i + 2];\n"
           "        for (int e = tid; e < n; e += blockDim.x) atomicAdd(&gacc[" + inst +
           " * gstride * 2 + 2 * go + e], sacc[so + e]); }\n";
  };
  o << "  const long long tiles_per = 1ll << " << (nb - t) << ";\n";
  o << "  const long long ntiles = tiles_per * batch;\n";
  o << "  long long last_inst = -1;\n";
  o << "  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {\n";
  o << "    const long long inst = tile >> " << (nb - t) << ";\n";
  o << "    const u64 ti = (u64)tile & (u64)(tiles_per - 1);\n";
  o << "    const long long goff = (inst << " << nb << ") + (long long)" << pdep_expr("ti", outer) << ";\n";
  o << "    __syncthreads();\n";
  o << "    if (inst != last_inst) {\n";
  o << "      if (last_inst >= 0) {\n" << flush_for("last_inst") << "        __syncthreads();\n";
  o << "        for (int e = tid; e < " << nacc_pad << "; e += blockDim.x) sacc[e] = 0.0;\n      }\n";
  o << "      const " << T << "* bm = bmat + inst * bstride;\n";
  o << "      for (int i = 0; i < " << nmc << "; ++i) { const int d = mc[3 * i], a = mc[3 * i + 1], n = mc[3 * i + 2];\n";
  if (c64)
    o << "        for (int e = tid; e < n; e += blockDim.x) { const float2 v = bm[a + e]; smat[d + e] = v; "
         "smatb[2 * (d + e)] = make_float2(v.x, v.x); smatb[2 * (d + e) + 1] = make_float2(v.y, v.y); } }\n";
  else
    o << "        for (int e = tid; e < n; e += blockDim.x) smat[d + e] = bm[a + e]; }\n";
  o << "      (void)bm; last_inst = inst;\n      __syncthreads();\n    }\n";
  const std::string tpl = "<" + std::to_string(t - rb) + ", " + std::to_string(t) + ", " + std::to_string(c) + ">";
  if (pf_table_env()) {
    o << "    " << (c64 ? "prefetch8t" : "prefetch16t") << tpl << "(sp, psi + goff, tbl);\n";
    o << "    " << (c64 ? "prefetch8t" : "prefetch16t") << tpl << "(sl, lam + goff, tbl);\n";
  } else {
    o << "    // tile copy: " << t << " tile bits, the lowest " << c << " contiguous\n";
    o << tile_load_literal(c64, t, t - rb, wide, unswz, gdep, "sp", "psi + goff");
    o << tile_load_literal(c64, t, t - rb, wide, unswz, gdep, "sl", "lam + goff");
  }
  o << "    cp_commit();\n    cp_wait0();\n";
  o << "    __syncthreads();\n";
  for (int si = pd.step_end - 1; si >= pd.step_begin; --si) {
    const int k = si - pd.step_begin;
    const Step& st = s.steps[si];
    std::vector<uint32_t> off(nr);
    for (int j = 0; j < nr; ++j) {
      uint32_t a = 0;
      for (int q = 0; q < rb; ++q)
        if ((j >> q) & 1) a ^= st.ebits[q];
      off[j] = a;
    }
    std::vector<int> var(nr);
    for (int j = 0; j < nr; ++j) var[j] = j;
    o << "    {\n";
    for (int j = 0; j < nr; ++j) {
      o << "      " << T << " p" << j << " = sp[tb" << k << " ^ " << off[j] << "u];";
      o << " " << T << " l" << j << " = sl[tb" << k << " ^ " << off[j] << "u];\n";
    }
    for (int ri = st.b - 1; ri >= st.a; --ri) {
      const RegOp& ro = s.rops[ri];
      const uint32_t kind = ro.w0 & 15u, q1 = (ro.w0 >> 4) & 15u, q2 = (ro.w0 >> 8) & 15u;
      const uint32_t dk = (ro.w0 >> 12) & 15u, dq = ro.w0 >> 16;
      const uint32_t crm = ro.w1 & 0xFFu, ctm = (ro.w1 >> 8) & 0xFFFFu, perm = ro.w1 >> 24;
      const uint32_t M = ro.w2;
      const bool guard = ctm != 0;
      const bool grad = ro.grad_off >= 0;
      const int ao = acc_off[ri - pd.rop_begin];
      auto P = [&](int j) { return std::string("p") + std::to_string(var[j]); };
      auto Lm = [&](int j) { return std::string("l") + std::to_string(var[j]); };
      o << "      {\n";
      int ng = 0;
      if (grad) {
        ng = (kind == RK_DIAG) ? (1 << dk) : (kind == RK_DENSE1 ? 4 : 16);
        o << "        " << T << " g[" << ng << "];\n        for (int e = 0; e < " << ng
          << "; ++e) { g[e].x = 0; g[e].y = 0; }\n";
      }
      if (guard) o << "        if ((tid & " << ctm << "u) == " << ctm << "u) {\n";
      else o << "        {\n";
      auto B = [&](uint32_t e, int part) { return "smatb[" + std::to_string(2 * (M + e) + part) + "]"; };
      if (kind == RK_DENSE1) {
        // G^dagger = [[conj m00, conj m10], [conj m01, conj m11]]
        if (c64)
          o << dense1_coefs(M, true, "          ", ro.pad[0] != 0);
        else
          o << "          const " << T << " h00 = cconj(smat[" << M << "]), h01 = cconj(smat[" << M + 2
            << "]), h10 = cconj(smat[" << M + 1 << "]), h11 = cconj(smat[" << M + 3 << "]);\n";
        auto upd = [&](const std::string& a, const std::string& b) {
          if (c64)
            return a + " = cdot2c(ar, ai, br, bi, x, y); " + b + " = cdot2c(cr, ci, dr, di, x, y);";
          return a + " = cfma(h01, y, cmul(h00, x)); " + b + " = cfma(h11, y, cmul(h10, x));";
        };
        for (int j = 0; j < nr; ++j) {
          if ((j >> q1) & 1) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int kk = j | (1 << q1);
          o << "          { " << T << " x = " << P(j) << ", y = " << P(kk) << "; " << upd(P(j), P(kk)) << "\n";
          if (grad)
            o << "            g[0] = cadd(g[0], cmulc(" << Lm(j) << ", " << P(j) << ")); g[1] = cadd(g[1], cmulc(" << Lm(j)
              << ", " << P(kk) << ")); g[2] = cadd(g[2], cmulc(" << Lm(kk) << ", " << P(j)
              << ")); g[3] = cadd(g[3], cmulc(" << Lm(kk) << ", " << P(kk) << "));\n";
          o << "            x = " << Lm(j) << "; y = " << Lm(kk) << "; " << upd(Lm(j), Lm(kk)) << " }\n";
        }
      } else if (kind == RK_PERM1) {
        for (int j = 0; j < nr; ++j) {
          if ((j >> q1) & 1) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int kk = j | (1 << q1);
          if (!guard) {
            std::swap(var[j], var[kk]);
          } else {
            o << "          { " << T << " x = " << P(j) << "; " << P(j) << " = " << P(kk) << "; " << P(kk)
              << " = x; x = " << Lm(j) << "; " << Lm(j) << " = " << Lm(kk) << "; " << Lm(kk) << " = x; }\n";
          }
        }
      } else if (kind == RK_DIAG) {
        for (int j = 0; j < nr; ++j) {
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          int idx = 0;
          for (uint32_t i = 0; i < dk; ++i) idx = (idx << 1) | ((j >> ((dq >> (3 * i)) & 7u)) & 1);
          o << "          { const " << T << " d = cconj(smat[" << M + idx << "]); " << P(j) << " = cmul(d, " << P(j)
            << ");";
          if (grad) o << " g[" << idx << "] = cadd(g[" << idx << "], cmulc(" << Lm(j) << ", " << P(j) << "));";
          o << " " << Lm(j) << " = cmul(d, " << Lm(j) << "); }\n";
        }
      } else if (kind == RK_DENSE2) {
        for (int j = 0; j < nr; ++j) {
          if (((j >> q1) & 1) || ((j >> q2) & 1)) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int id[4] = {j, j | (1 << q2), j | (1 << q1), j | (1 << q1) | (1 << q2)};
          o << "          { const " << T << " a0 = " << P(id[0]) << ", a1 = " << P(id[1]) << ", a2 = " << P(id[2])
            << ", a3 = " << P(id[3]) << ";\n";
          // (G^dagger)[r][q] = conj(G[q][r]), read from shared memory each time
          auto H = [&](int r, int q) { return "cconj(smat[" + std::to_string(M + 4 * q + r) + "])"; };
          // complex64: sum_q conj(G[q][r]) a_q from the broadcast pairs
          auto HC = [&](const std::string& dst, int r, const char* a) {
            std::string e = "{ float2 p = __fmul2_rn(" + B(r, 0) + ", " + a + "0), q = __fmul2_rn(" + B(r, 1) + ", " +
                            a + "0);";
            for (int q = 1; q < 4; ++q)
              e += " p = __ffma2_rn(" + B(4 * q + r, 0) + ", " + a + std::to_string(q) + ", p); q = __ffma2_rn(" +
                   B(4 * q + r, 1) + ", " + a + std::to_string(q) + ", q);";
            return e + " " + dst + " = make_float2(p.x + q.y, p.y - q.x); }";
          };
          for (int r = 0; r < 4; ++r) {
            if (c64) {
              o << "            " << HC(P(id[r]), r, "a") << "\n";
              continue;
            }
            o << "            " << P(id[r]) << " = cfma(" << H(r, 3) << ", a3, cfma(" << H(r, 2) << ", a2, cfma("
              << H(r, 1) << ", a1, cmul(" << H(r, 0) << ", a0))));\n";
          }
          if (grad)
            for (int r = 0; r < 4; ++r)
              for (int q = 0; q < 4; ++q)
                o << "            g[" << 4 * r + q << "] = cadd(g[" << 4 * r + q << "], cmulc(" << Lm(id[r]) << ", "
                  << P(id[q]) << "));\n";
          o << "            const " << T << " b0 = " << Lm(id[0]) << ", b1 = " << Lm(id[1]) << ", b2 = " << Lm(id[2])
            << ", b3 = " << Lm(id[3]) << ";\n";
          for (int r = 0; r < 4; ++r) {
            if (c64) {
              o << "            " << HC(Lm(id[r]), r, "b") << "\n";
              continue;
            }
            o << "            " << Lm(id[r]) << " = cfma(" << H(r, 3) << ", b3, cfma(" << H(r, 2) << ", b2, cfma("
              << H(r, 1) << ", b1, cmul(" << H(r, 0) << ", b0))));\n";
          }
          o << "          }\n";
        }
      } else {  // RK_PERM2, inverse: new[p[r]] = old[r]
        for (int j = 0; j < nr; ++j) {
          if (((j >> q1) & 1) || ((j >> q2) & 1)) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int id[4] = {j, j | (1 << q2), j | (1 << q1), j | (1 << q1) | (1 << q2)};
          int pv[4];
          for (int r = 0; r < 4; ++r) pv[r] = (perm >> (2 * r)) & 3u;
          if (!guard) {
            int nv[4];
            for (int r = 0; r < 4; ++r) nv[pv[r]] = var[id[r]];
            for (int r = 0; r < 4; ++r) var[id[r]] = nv[r];
          } else {
            o << "          { const " << T << " a0 = " << P(id[0]) << ", a1 = " << P(id[1]) << ", a2 = " << P(id[2])
              << ", a3 = " << P(id[3]) << ";";
            for (int r = 0; r < 4; ++r) o << " " << P(id[pv[r]]) << " = a" << r << ";";
            o << " }\n";
            o << "          { const " << T << " a0 = " << Lm(id[0]) << ", a1 = " << Lm(id[1]) << ", a2 = " << Lm(id[2])
              << ", a3 = " << Lm(id[3]) << ";";
            for (int r = 0; r < 4; ++r) o << " " << Lm(id[pv[r]]) << " = a" << r << ";";
            o << " }\n";
          }
        }
      }
      o << "        }\n";
      if (grad) {
        // reduce the warp's partial cotangent, 32 values at a time
        const int nv = 2 * ng;
        for (int c0 = 0; c0 < nv; c0 += 32) {
          const int cn = std::min(32, nv - c0);
          o << "        { " << F << " vv[" << cn << "] = {";
          for (int e = 0; e < cn; ++e)
            o << (e ? ", " : "") << "g[" << (c0 + e) / 2 << "]." << (((c0 + e) & 1) ? "y" : "x");
          o << "}; warp_rs_add<" << cn << ">(vv, &sacc[" << ao + c0 << "]); }\n";
        }
      }
      o << "      }\n";
    }
    if (direct && si == pd.step_begin) {
      for (int j = 0; j < nr; ++j) {
        const std::string gj = std::to_string(gdep(unswz(off[j]))) + (wide ? "ull" : "u");
        o << "      __stcs(psi + goff + (gpos ^ " << gj << "), p" << var[j] << "); __stcs(lam + goff + (gpos ^ " << gj
          << "), l" << var[j] << ");\n";
      }
      o << "    }\n";
    } else {
      for (int j = 0; j < nr; ++j)
        o << "      sp[tb" << k << " ^ " << off[j] << "u] = p" << var[j] << "; sl[tb" << k << " ^ " << off[j]
          << "u] = l" << var[j] << ";\n";
      o << "    }\n    "
        << (si > pd.step_begin && warp_owned(st, s.steps[si - 1], t - rb) ? "__syncwarp()" : "__syncthreads()")
        << ";\n";
    }
  }
  if (!direct) {
    o << "    " << (c64 ? "store8t" : "store16t") << tpl << "(sp, psi + goff, tbl);\n";
    o << "    " << (c64 ? "store8t" : "store16t") << tpl << "(sl, lam + goff, tbl);\n";
  }
  o << "  }\n  __syncthreads();\n  if (last_inst >= 0) {\n" << flush_for("last_inst") << "  }\n}\n";
}

// Forward application of register op `ro` to the registers arr<var[j]>
// (j = register slot): the non-split forms of emit_pass.  Unguarded
// permutations rename `var` at generation time.
void emit_fwd_rop(std::ostringstream& o, const RegOp& ro, bool c64, const std::string& arr, std::vector<int>& var,
                  int nr) {
  const char* T = c64 ? "float2" : "double2";
  const uint32_t kind = ro.w0 & 15u, q1 = (ro.w0 >> 4) & 15u, q2 = (ro.w0 >> 8) & 15u;
  const uint32_t dk = (ro.w0 >> 12) & 15u, dq = ro.w0 >> 16;
  const uint32_t crm = ro.w1 & 0xFFu, ctm = (ro.w1 >> 8) & 0xFFFFu, perm = ro.w1 >> 24;
  const uint32_t M = ro.w2;
  const bool guard = ctm != 0;
  auto V = [&](int j) { return arr + std::to_string(var[j]); };
  if (guard) o << "      if ((tid & " << ctm << "u) == " << ctm << "u) {\n";
  else o << "      {\n";
  if (kind == RK_DENSE1) {
    if (c64) {
      o << dense1_coefs(M, false, "        ", ro.pad[0] != 0);
    } else {
      o << "        const double2 m00 = smat[" << M << "], m01 = smat[" << M + 1 << "], m10 = smat[" << M + 2
        << "], m11 = smat[" << M + 3 << "];\n";
    }
    for (int j = 0; j < nr; ++j) {
      if ((j >> q1) & 1) continue;
      if ((static_cast<uint32_t>(j) & crm) != crm) continue;
      const int k = j | (1 << q1);
      if (c64)
        o << "        { const float2 x = " << V(j) << ", y = " << V(k) << "; " << V(j) << " = cdot2(ar, ai, br, bi, x, y); "
          << V(k) << " = cdot2(cr, ci, dr, di, x, y); }\n";
      else
        o << "        { const double2 x = " << V(j) << ", y = " << V(k) << "; " << V(j) << " = cfma(m01, y, cmul(m00, x)); "
          << V(k) << " = cfma(m11, y, cmul(m10, x)); }\n";
    }
  } else if (kind == RK_PERM1) {
    for (int j = 0; j < nr; ++j) {
      if ((j >> q1) & 1) continue;
      if ((static_cast<uint32_t>(j) & crm) != crm) continue;
      const int k = j | (1 << q1);
      if (!guard) std::swap(var[j], var[k]);
      else o << "        { const " << T << " x = " << V(j) << "; " << V(j) << " = " << V(k) << "; " << V(k) << " = x; }\n";
    }
  } else if (kind == RK_DIAG) {
    for (int j = 0; j < nr; ++j) {
      if ((static_cast<uint32_t>(j) & crm) != crm) continue;
      int idx = 0;
      for (uint32_t i = 0; i < dk; ++i) idx = (idx << 1) | ((j >> ((dq >> (3 * i)) & 7u)) & 1);
      o << "        " << V(j) << " = cmul(smat[" << M + idx << "], " << V(j) << ");\n";
    }
  } else if (kind == RK_DENSE2) {
    for (int j = 0; j < nr; ++j) {
      if (((j >> q1) & 1) || ((j >> q2) & 1)) continue;
      if ((static_cast<uint32_t>(j) & crm) != crm) continue;
      const int id[4] = {j, j | (1 << q2), j | (1 << q1), j | (1 << q1) | (1 << q2)};
      o << "        { const " << T << " a0 = " << V(id[0]) << ", a1 = " << V(id[1]) << ", a2 = " << V(id[2])
        << ", a3 = " << V(id[3]) << ";\n";
      for (int r = 0; r < 4; ++r) {
        if (c64)
          o << "          " << V(id[r]) << " = cdot4((const float4*)smatb + " << M + 4 * r << ", a0, a1, a2, a3);\n";
        else
          o << "          " << V(id[r]) << " = cfma(smat[" << M + 4 * r + 3 << "], a3, cfma(smat[" << M + 4 * r + 2
            << "], a2, cfma(smat[" << M + 4 * r + 1 << "], a1, cmul(smat[" << M + 4 * r << "], a0))));\n";
      }
      o << "        }\n";
    }
  } else {  // RK_PERM2: output row r takes input column p[r]
    for (int j = 0; j < nr; ++j) {
      if (((j >> q1) & 1) || ((j >> q2) & 1)) continue;
      if ((static_cast<uint32_t>(j) & crm) != crm) continue;
      const int id[4] = {j, j | (1 << q2), j | (1 << q1), j | (1 << q1) | (1 << q2)};
      int pv[4];
      for (int r = 0; r < 4; ++r) pv[r] = (perm >> (2 * r)) & 3u;
      if (!guard) {
        int nv[4];
        for (int r = 0; r < 4; ++r) nv[r] = var[id[pv[r]]];
        for (int r = 0; r < 4; ++r) var[id[r]] = nv[r];
      } else {
        o << "        { const " << T << " a0 = " << V(id[0]) << ", a1 = " << V(id[1]) << ", a2 = " << V(id[2])
          << ", a3 = " << V(id[3]) << ";";
        for (int r = 0; r < 4; ++r) o << " " << V(id[r]) << " = a" << pv[r] << ";";
        o << " }\n";
      }
    }
  }
  o << "      }\n";
}

// Shared memory of a checkpointed reverse pass: the input tile of every
// register stage, the lambda tile, staged matrices, float64 cotangent
// accumulators and the bit-deposit table.
size_t bwd_smem_bytes(const Schedule& s, int p, int elem) {
  const PassDesc& pd = s.passes[p];
  int nacc = 0;
  for (int ri = pd.rop_begin; ri < pd.rop_end; ++ri)
    if (s.rops[ri].grad_off >= 0) nacc += 2 * s.rops[ri].mat_len;
  const size_t smat_pad = static_cast<size_t>((pd.smat_len + 1) & ~1);
  const size_t nst = static_cast<size_t>(pd.step_end - pd.step_begin);
  return (nst + 1) * (static_cast<size_t>(1) << pd.t) * elem + smat_pad * elem + (elem == 8 ? 2 * smat_pad * elem : 0) +
         static_cast<size_t>((nacc + 1) & ~1) * 8 + (static_cast<size_t>(1) << (pd.t - pd.c)) * 4;
}

// Emit the checkpointed reverse kernel of pass p (density matrices with
// channels, non-unitary pure circuits).  Per tile: the pass input x and the
// cotangent lam after the pass are loaded; a forward walk runs the register
// stages, each writing its output into a fresh shared-memory tile, so the
// input of every stage is kept; then the stages run in reverse.  Inside a
// stage the state before each gate block is recomputed in registers from the
// stage input (the stage's earlier blocks, a handful), the block cotangent
// lam x^dagger is accumulated (warp reduce-scatter into float64 shared
// accumulators, flushed per instance) and lam <- G^dagger lam.  Unguarded
// permutations stay register renames in both directions.
void emit_bwd_pass(std::ostringstream& o, const jq_plan* plan, const Schedule& s, int p, bool c64, int rb) {
  const PassDesc& pd = s.passes[p];
  const char* T = c64 ? "float2" : "double2";
  const char* F = c64 ? "float" : "double";
  const int t = pd.t, c = pd.c, nb = plan->n_bits;
  const int nthr = 1 << (t - rb);
  const int nr = 1 << rb;
  const int nst = pd.step_end - pd.step_begin;
  const uint64_t full = (nb >= 64) ? ~0ULL : ((1ULL << nb) - 1);
  const uint64_t outer = full & ~pd.tile_mask;
  const int smat_pad = (pd.smat_len + 1) & ~1;
  int nmc = 0, ngt = 0, nacc = 0;
  std::vector<int> acc_off(pd.rop_end - pd.rop_begin, -1);
  for (int ri = pd.rop_begin; ri < pd.rop_end; ++ri) {
    const RegOp& ro = s.rops[ri];
    nmc += ro.mat_len > 0;
    if (ro.grad_off >= 0) {
      acc_off[ri - pd.rop_begin] = nacc;
      nacc += 2 * ro.mat_len;
      ++ngt;
    }
  }
  const int nacc_pad = (nacc + 1) & ~1;
  o << "extern \"C\" __global__ void __launch_bounds__(" << nthr << ", 1) @KERNEL@(" << T
    << "* __restrict__ xin, " << T << "* __restrict__ lam, int batch, const " << T
    << "* __restrict__ bmat, long long bstride, const int* __restrict__ mc, double* __restrict__ gacc, "
    << "long long gstride, const int* __restrict__ gt) {\n";
  o << "  extern __shared__ __align__(16) unsigned char smem[];\n";
  o << "  " << T << "* sx = (" << T << "*)smem;  // stage inputs, " << nst << " tiles\n";
  o << "  " << T << "* sl = sx + " << nst * (1 << t) << ";\n";
  o << "  " << T << "* smat = sl + " << (1 << t) << ";\n";
  if (c64) {
    o << "  float2* smatb = smat + " << smat_pad << ";\n";
    o << "  double* sacc = (double*)(smatb + " << 2 * smat_pad << ");\n";
  } else {
    o << "  double* sacc = (double*)(smat + " << smat_pad << ");\n";
  }
  o << "  u32* tbl = (u32*)(sacc + " << nacc_pad << ");\n";
  o << "  const u32 tid = threadIdx.x;\n";
  o << kPdlTrigger << kPdlWait;
  o << "  { const u32 hb[] = {";
  for (int i = c; i < t; ++i) o << (i > c ? ", " : "") << (1u << pd.bits[i]);
  if (t == c) o << "0u";
  o << "};\n    for (int h = tid; h < " << (1 << (t - c)) << "; h += blockDim.x) { u32 v = 0;";
  o << " for (int i = 0; i < " << (t - c) << "; ++i) if ((h >> i) & 1) v |= hb[i]; tbl[h] = v; } }\n";
  o << "  for (int e = tid; e < " << nacc_pad << "; e += blockDim.x) sacc[e] = 0.0;\n";
  std::vector<std::vector<uint32_t>> offs(nst);
  for (int k = 0; k < nst; ++k) {
    const Step& st = s.steps[pd.step_begin + k];
    o << "  u32 tb" << k << " = 0;";
    for (int i = 0; i < t - rb; ++i) o << " if (tid & " << (1u << i) << "u) tb" << k << " ^= " << st.tbits[i] << "u;";
    o << "\n";
    offs[k].resize(nr);
    for (int j = 0; j < nr; ++j) {
      uint32_t a = 0;
      for (int q = 0; q < rb; ++q)
        if ((j >> q) & 1) a ^= st.ebits[q];
      offs[k][j] = a;
    }
  }
  // lambda leaves the last reverse stage (the pass's first) straight to
  // global memory under the forward pass's direct-store condition
  const Step& fin = s.steps[pd.step_begin];
  bool direct = t - rb >= 2 && c >= 2 && (c64 ? (fin.tbits[0] == 1u && fin.tbits[1] == 2u) : fin.tbits[0] == 1u);
  if (const char* e = std::getenv("JQ_JIT_DIRECT_STORE")) direct = direct && std::atoi(e) != 0;
  const bool wide = nb > 31;
  auto unswz = [&](uint64_t v) -> uint64_t {
    if (c64) return v ^ (((v >> 4) ^ (v >> 8) ^ (v >> 12)) & 15u);
    return v ^ (((v >> 3) ^ (v >> 6) ^ (v >> 9) ^ (v >> 12)) & 7u);
  };
  auto gdep = [&](uint64_t logical) -> uint64_t {
    uint64_t g = 0;
    for (int i = 0; i < t; ++i)
      if ((logical >> i) & 1) g |= 1ULL << pd.bits[i];
    return g;
  };
  if (direct) {
    o << "  " << (wide ? "u64" : "u32") << " gpos = 0;";
    for (int i = 0; i < t - rb; ++i)
      o << " if (tid & " << (1u << i) << "u) gpos ^= " << gdep(unswz(fin.tbits[i])) << (wide ? "ull;" : "u;");
    o << "\n";
  }
  auto flush_for = [&](const std::string& inst) {
    return "      if (gacc) for (int i = 0; i < " + std::to_string(ngt) +
           "; ++i) { const int so = gt[3 * i], go = gt[3 * i + 1], n = gt[3 * i + 2];\n"
           "        for (int e = tid; e < n; e += blockDim.x) atomicAdd(&gacc[" + inst +
           " * gstride * 2 + 2 * go + e], sacc[so + e]); }\n";
  };
  o << "  const long long tiles_per = 1ll << " << (nb - t) << ";\n";
  o << "  const long long ntiles = tiles_per * batch;\n";
  o << "  long long last_inst = -1;\n";
  o << "  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {\n";
  o << "    const long long inst = tile >> " << (nb - t) << ";\n";
  o << "    const u64 ti = (u64)tile & (u64)(tiles_per - 1);\n";
  o << "    const long long goff = (inst << " << nb << ") + (long long)" << pdep_expr("ti", outer) << ";\n";
  o << "    __syncthreads();\n";
  o << "    if (inst != last_inst) {\n";
  o << "      if (last_inst >= 0) {\n" << flush_for("last_inst") << "        __syncthreads();\n";
  o << "        for (int e = tid; e < " << nacc_pad << "; e += blockDim.x) sacc[e] = 0.0;\n      }\n";
  o << "      const " << T << "* bm = bmat + inst * bstride;\n";
  o << "      for (int i = 0; i < " << nmc << "; ++i) { const int d = mc[3 * i], a = mc[3 * i + 1], n = mc[3 * i + 2];\n";
  if (c64)
    o << "        for (int e = tid; e < n; e += blockDim.x) { const float2 v = bm[a + e]; smat[d + e] = v; "
         "smatb[2 * (d + e)] = make_float2(v.x, v.x); smatb[2 * (d + e) + 1] = make_float2(v.y, v.y); } }\n";
  else
    o << "        for (int e = tid; e < n; e += blockDim.x) smat[d + e] = bm[a + e]; }\n";
  o << "      (void)bm; last_inst = inst;\n      __syncthreads();\n    }\n";
  const std::string tpl = "<" + std::to_string(t - rb) + ", " + std::to_string(t) + ", " + std::to_string(c) + ">";
  if (pf_table_env()) {
    o << "    " << (c64 ? "prefetch8t" : "prefetch16t") << tpl << "(sx, xin + goff, tbl);\n";
    o << "    " << (c64 ? "prefetch8t" : "prefetch16t") << tpl << "(sl, lam + goff, tbl);\n";
  } else {
    o << "    // tile copy: " << t << " tile bits, the lowest " << c << " contiguous\n";
    o << tile_load_literal(c64, t, t - rb, wide, unswz, gdep, "sx", "xin + goff");
    o << tile_load_literal(c64, t, t - rb, wide, unswz, gdep, "sl", "lam + goff");
  }
  o << "    cp_commit();\n    cp_wait0();\n";
  o << "    __syncthreads();\n";
  // forward walk: stage k reads tile k and writes tile k + 1
  for (int k = 0; k + 1 < nst; ++k) {
    const Step& st = s.steps[pd.step_begin + k];
    std::vector<int> var(nr);
    for (int j = 0; j < nr; ++j) var[j] = j;
    o << "    {\n      const " << T << "* src = sx + " << k * (1 << t) << ";\n      " << T << "* dst = sx + "
      << (k + 1) * (1 << t) << ";\n";
    for (int j = 0; j < nr; ++j) o << "      " << T << " v" << j << " = src[tb" << k << " ^ " << offs[k][j] << "u];\n";
    for (int ri = st.a; ri < st.b; ++ri) emit_fwd_rop(o, s.rops[ri], c64, "v", var, nr);
    for (int j = 0; j < nr; ++j) o << "      dst[tb" << k << " ^ " << offs[k][j] << "u] = v" << var[j] << ";\n";
    o << "    }\n    "
      << (k + 1 < nst && warp_owned(st, s.steps[pd.step_begin + k + 1], t - rb) ? "__syncwarp()" : "__syncthreads()")
      << ";\n";
  }
  // reverse walk over the stages
  for (int k = nst - 1; k >= 0; --k) {
    const Step& st = s.steps[pd.step_begin + k];
    std::vector<int> lvar(nr);
    for (int j = 0; j < nr; ++j) lvar[j] = j;
    o << "    {\n      const " << T << "* src = sx + " << k * (1 << t) << ";\n";
    for (int j = 0; j < nr; ++j) o << "      " << T << " l" << j << " = sl[tb" << k << " ^ " << offs[k][j] << "u];\n";
    for (int ri = st.b - 1; ri >= st.a; --ri) {
      const RegOp& ro = s.rops[ri];
      const uint32_t kind = ro.w0 & 15u, q1 = (ro.w0 >> 4) & 15u, q2 = (ro.w0 >> 8) & 15u;
      const uint32_t dk = (ro.w0 >> 12) & 15u, dq = ro.w0 >> 16;
      const uint32_t crm = ro.w1 & 0xFFu, ctm = (ro.w1 >> 8) & 0xFFFFu, perm = ro.w1 >> 24;
      const uint32_t M = ro.w2;
      const bool guard = ctm != 0;
      const bool grad = ro.grad_off >= 0;
      const int ao = acc_off[ri - pd.rop_begin];
      auto Lm = [&](int j) { return std::string("l") + std::to_string(lvar[j]); };
      if (kind == RK_PERM1 || kind == RK_PERM2) {
        // lam <- P^-1 lam: renames, or explicit moves under a thread-bit control
        if (guard) o << "      if ((tid & " << ctm << "u) == " << ctm << "u) {\n";
        for (int j = 0; j < nr; ++j) {
          if (kind == RK_PERM1) {
            if ((j >> q1) & 1) continue;
            if ((static_cast<uint32_t>(j) & crm) != crm) continue;
            const int kk = j | (1 << q1);
            if (!guard) std::swap(lvar[j], lvar[kk]);
            else o << "        { const " << T << " x = " << Lm(j) << "; " << Lm(j) << " = " << Lm(kk) << "; " << Lm(kk) << " = x; }\n";
          } else {
            if (((j >> q1) & 1) || ((j >> q2) & 1)) continue;
            if ((static_cast<uint32_t>(j) & crm) != crm) continue;
            const int id[4] = {j, j | (1 << q2), j | (1 << q1), j | (1 << q1) | (1 << q2)};
            int pv[4];
            for (int r = 0; r < 4; ++r) pv[r] = (perm >> (2 * r)) & 3u;
            if (!guard) {
              int nv[4];
              for (int r = 0; r < 4; ++r) nv[pv[r]] = lvar[id[r]];
              for (int r = 0; r < 4; ++r) lvar[id[r]] = nv[r];
            } else {
              o << "        { const " << T << " a0 = " << Lm(id[0]) << ", a1 = " << Lm(id[1]) << ", a2 = " << Lm(id[2])
                << ", a3 = " << Lm(id[3]) << ";";
              for (int r = 0; r < 4; ++r) o << " " << Lm(id[pv[r]]) << " = a" << r << ";";
              o << " }\n";
            }
          }
        }
        if (guard) o << "      }\n";
        continue;
      }
      // the state before this block: the stage input with the stage's
      // earlier blocks applied (registers y*)
      std::vector<int> yvar(nr);
      for (int j = 0; j < nr; ++j) yvar[j] = j;
      o << "      {\n";
      for (int j = 0; j < nr; ++j) o << "      " << T << " y" << j << " = src[tb" << k << " ^ " << offs[k][j] << "u];\n";
      for (int rj = st.a; rj < ri; ++rj) emit_fwd_rop(o, s.rops[rj], c64, "y", yvar, nr);
      auto Y = [&](int j) { return std::string("y") + std::to_string(yvar[j]); };
      int ng = 0;
      if (grad) {
        ng = (kind == RK_DIAG) ? (1 << dk) : (kind == RK_DENSE1 ? 4 : 16);
        o << "        " << T << " g[" << ng << "];\n        for (int e = 0; e < " << ng
          << "; ++e) { g[e].x = 0; g[e].y = 0; }\n";
      }
      if (guard) o << "        if ((tid & " << ctm << "u) == " << ctm << "u) {\n";
      else o << "        {\n";
      if (kind == RK_DENSE1) {
        if (c64)
          o << dense1_coefs(M, true, "          ", ro.pad[0] != 0);
        else
          o << "          const double2 h00 = cconj(smat[" << M << "]), h01 = cconj(smat[" << M + 2
            << "]), h10 = cconj(smat[" << M + 1 << "]), h11 = cconj(smat[" << M + 3 << "]);\n";
        for (int j = 0; j < nr; ++j) {
          if ((j >> q1) & 1) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int kk = j | (1 << q1);
          if (grad)
            o << "          g[0] = cadd(g[0], cmulc(" << Lm(j) << ", " << Y(j) << ")); g[1] = cadd(g[1], cmulc(" << Lm(j)
              << ", " << Y(kk) << ")); g[2] = cadd(g[2], cmulc(" << Lm(kk) << ", " << Y(j)
              << ")); g[3] = cadd(g[3], cmulc(" << Lm(kk) << ", " << Y(kk) << "));\n";
          if (c64)
            o << "          { const float2 x = " << Lm(j) << ", y = " << Lm(kk) << "; " << Lm(j)
              << " = cdot2c(ar, ai, br, bi, x, y); " << Lm(kk) << " = cdot2c(cr, ci, dr, di, x, y); }\n";
          else
            o << "          { const double2 x = " << Lm(j) << ", y = " << Lm(kk) << "; " << Lm(j)
              << " = cfma(h01, y, cmul(h00, x)); " << Lm(kk) << " = cfma(h11, y, cmul(h10, x)); }\n";
        }
      } else if (kind == RK_DIAG) {
        for (int j = 0; j < nr; ++j) {
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          int idx = 0;
          for (uint32_t i = 0; i < dk; ++i) idx = (idx << 1) | ((j >> ((dq >> (3 * i)) & 7u)) & 1);
          o << "          {";
          if (grad) o << " g[" << idx << "] = cadd(g[" << idx << "], cmulc(" << Lm(j) << ", " << Y(j) << "));";
          o << " " << Lm(j) << " = cmul(cconj(smat[" << M + idx << "]), " << Lm(j) << "); }\n";
        }
      } else {  // RK_DENSE2
        auto B = [&](uint32_t e, int part) { return "smatb[" + std::to_string(2 * (M + e) + part) + "]"; };
        auto H = [&](int r, int q) { return "cconj(smat[" + std::to_string(M + 4 * q + r) + "])"; };
        auto HC = [&](const std::string& dst, int r) {
          std::string e = "{ float2 p = __fmul2_rn(" + B(r, 0) + ", b0), q = __fmul2_rn(" + B(r, 1) + ", b0);";
          for (int q = 1; q < 4; ++q)
            e += " p = __ffma2_rn(" + B(4 * q + r, 0) + ", b" + std::to_string(q) + ", p); q = __ffma2_rn(" +
                 B(4 * q + r, 1) + ", b" + std::to_string(q) + ", q);";
          return e + " " + dst + " = make_float2(p.x + q.y, p.y - q.x); }";
        };
        for (int j = 0; j < nr; ++j) {
          if (((j >> q1) & 1) || ((j >> q2) & 1)) continue;
          if ((static_cast<uint32_t>(j) & crm) != crm) continue;
          const int id[4] = {j, j | (1 << q2), j | (1 << q1), j | (1 << q1) | (1 << q2)};
          o << "          {\n";
          if (grad)
            for (int r = 0; r < 4; ++r)
              for (int q = 0; q < 4; ++q)
                o << "            g[" << 4 * r + q << "] = cadd(g[" << 4 * r + q << "], cmulc(" << Lm(id[r]) << ", "
                  << Y(id[q]) << "));\n";
          o << "            const " << T << " b0 = " << Lm(id[0]) << ", b1 = " << Lm(id[1]) << ", b2 = " << Lm(id[2])
            << ", b3 = " << Lm(id[3]) << ";\n";
          for (int r = 0; r < 4; ++r) {
            if (c64) o << "            " << HC(Lm(id[r]), r) << "\n";
            else
              o << "            " << Lm(id[r]) << " = cfma(" << H(r, 3) << ", b3, cfma(" << H(r, 2) << ", b2, cfma("
                << H(r, 1) << ", b1, cmul(" << H(r, 0) << ", b0))));\n";
          }
          o << "          }\n";
        }
      }
      o << "        }\n";
      if (grad) {
        const int nv = 2 * ng;
        for (int c0 = 0; c0 < nv; c0 += 32) {
          const int cn = std::min(32, nv - c0);
          o << "        { " << F << " vv[" << cn << "] = {";
          for (int e = 0; e < cn; ++e)
            o << (e ? ", " : "") << "g[" << (c0 + e) / 2 << "]." << (((c0 + e) & 1) ? "y" : "x");
          o << "}; warp_rs_add<" << cn << ">(vv, &sacc[" << ao + c0 << "]); }\n";
        }
      }
      o << "      }\n";
    }
    if (direct && k == 0) {
      for (int j = 0; j < nr; ++j)
        o << "      __stcs(lam + goff + (gpos ^ " << gdep(unswz(offs[k][j])) << (wide ? "ull" : "u") << "), l"
          << lvar[j] << ");\n";
      o << "    }\n";
    } else {
      for (int j = 0; j < nr; ++j) o << "      sl[tb" << k << " ^ " << offs[k][j] << "u] = l" << lvar[j] << ";\n";
      o << "    }\n    "
        << (k > 0 && warp_owned(st, s.steps[pd.step_begin + k - 1], t - rb) ? "__syncwarp()" : "__syncthreads()")
        << ";\n";
    }
  }
  if (!direct) o << "    " << (c64 ? "store8t" : "store16t") << tpl << "(sl, lam + goff, tbl);\n";
  o << "  }\n  __syncthreads();\n  if (last_inst >= 0) {\n" << flush_for("last_inst") << "  }\n}\n";
}

}  // namespace

bool jit_available() {
  std::call_once(g_once, init_bindings);
  return g_nvrtc.ok && g_drv.ok;
}

bool jit_pass_eligible(const Schedule& s, int p) {
  const PassDesc& pd = s.passes[p];
  if (pd.step_end == pd.step_begin) return false;
  for (int si = pd.step_begin; si < pd.step_end; ++si)
    if (s.steps[si].kind != 0) return false;
  return true;
}

// Kernel text of every eligible pass (forward, or adjoint when `adjoint`);
// identical texts share one kernel.  Appends to `all`, names kernels prefix + k.
// mode 0: forward passes, 1: adjoint passes (unitary statevector plans),
// 2: checkpointed reverse passes (every other plan; passes whose stage inputs
// do not fit in shared memory keep the generic kernel).
void emit_kernels(const jq_plan* plan, const Schedule& s, int mode, const char* prefix, std::ostringstream& all,
                  std::vector<int>* kernel_of, std::vector<std::string>* names,
                  std::vector<std::string>* bodies = nullptr) {
  kernel_of->assign(s.passes.size(), -1);
  std::vector<std::string> texts;
  const int elem = plan->dtype == JQ_C64 ? 8 : 16;
  for (int p = 0; p < static_cast<int>(s.passes.size()); ++p) {
    if (!jit_pass_eligible(s, p)) continue;
    if (mode == 2 && bwd_smem_bytes(s, p, elem) > 227 * 1024) continue;
    std::ostringstream o;
    if (mode == 1) emit_adj_pass(o, plan, s, p, plan->dtype == JQ_C64, s.reg_bits);
    else if (mode == 2) emit_bwd_pass(o, plan, s, p, plan->dtype == JQ_C64, s.reg_bits);
    else emit_pass(o, plan, s, p, plan->dtype == JQ_C64, s.reg_bits);
    const std::string text = o.str();
    int k = -1;
    for (size_t i = 0; i < texts.size(); ++i)
      if (texts[i] == text) { k = static_cast<int>(i); break; }
    if (k < 0) {
      k = static_cast<int>(texts.size());
      texts.push_back(text);
      const std::string name = prefix + std::to_string(k);
      names->push_back(name);
      std::string body = text;
      body.replace(body.find("@KERNEL@"), 8, name);
      all << body;
      if (bodies) bodies->push_back(body);
    }
    (*kernel_of)[p] = k;
  }
}

// The adjoint kernels are specialised too when the plan can run jq_adjoint
// (a unitary statevector plan).
bool plan_wants_adjoint(const jq_plan* plan) { return plan->mode == JQ_STATEVECTOR && plan->unitary; }
// The checkpointed reverse passes are specialised for every other plan that
// has parameters to differentiate.
bool plan_wants_backward(const jq_plan* plan) { return !plan_wants_adjoint(plan) && plan->any_grad; }

std::string jit_source(const jq_plan* plan, const Schedule& s) {
  std::ostringstream all;
  all << kPrelude;
  std::vector<int> kernel_of;
  std::vector<std::string> names;
  emit_kernels(plan, s, 0, "jqk", all, &kernel_of, &names);
  if (plan_wants_adjoint(plan)) emit_kernels(plan, s, 1, "jqa", all, &kernel_of, &names);
  if (plan_wants_backward(plan)) emit_kernels(plan, s, 2, "jqb", all, &kernel_of, &names);
  return all.str();
}

int jit_build(const jq_plan* plan, const Schedule& s, JitModule* out) {
  if (!jit_available()) {
    set_error("NVRTC or the CUDA driver entry points are not available");
    return JQ_EUNSUPPORTED;
  }
  std::ostringstream all;
  std::vector<int> kernel_of, akernel_of, bkernel_of;
  std::vector<std::string> names, anames, bnames, bodies;
  emit_kernels(plan, s, 0, "jqk", all, &kernel_of, &names, &bodies);
  const bool adj = plan_wants_adjoint(plan);
  if (adj) emit_kernels(plan, s, 1, "jqa", all, &akernel_of, &anames, &bodies);
  const bool bwd = plan_wants_backward(plan);
  if (bwd) emit_kernels(plan, s, 2, "jqb", all, &bkernel_of, &bnames, &bodies);
  out->fn.assign(s.passes.size(), nullptr);
  out->afn.assign(s.passes.size(), nullptr);
  out->bfn.assign(s.passes.size(), nullptr);
  out->modules.clear();
  out->mc = nullptr;
  out->gt = nullptr;
  out->mc_off.assign(s.passes.size(), 0);
  out->gt_off.assign(s.passes.size(), 0);
  if (names.empty()) return JQ_OK;
  // The kernels compile as independent NVRTC programs on parallel host
  // threads (a large plan has hundreds of straight-line kernels); each
  // chunk is loaded as its own module.
  const int nk = static_cast<int>(bodies.size());
  int hw = static_cast<int>(std::thread::hardware_concurrency());
  if (hw <= 0) hw = 4;
  const int nchunk = std::max(1, std::min(std::min(hw, 32), (nk + 1) / 2));
  std::vector<std::string> srcs(nchunk, std::string(kPrelude));
  std::vector<int> chunk_of(nk);
  for (int k = 0; k < nk; ++k) {
    chunk_of[k] = k % nchunk;
    srcs[k % nchunk] += bodies[k];
  }
  std::vector<std::vector<char>> bins(nchunk);
  std::vector<std::string> errs(nchunk);
  auto compile = [&](int c) {
    nvrtcProgram prog;
    if (g_nvrtc.create(&prog, srcs[c].c_str(), "jq_plan.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
      errs[c] = "nvrtcCreateProgram failed";
      return;
    }
    const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device"};
    if (g_nvrtc.compile(prog, 3, opts) != NVRTC_SUCCESS) {
      size_t n = 0;
      g_nvrtc.log_size(prog, &n);
      std::string log(n, '\0');
      g_nvrtc.log(prog, &log[0]);
      errs[c] = "NVRTC compile of the plan failed: " + log.substr(0, 2000);
      g_nvrtc.destroy(&prog);
      return;
    }
    size_t nbin = 0;
    g_nvrtc.cubin_size(prog, &nbin);
    bins[c].resize(nbin);
    g_nvrtc.cubin(prog, bins[c].data());
    g_nvrtc.destroy(&prog);
  };
  {
    std::vector<std::thread> th;
    for (int c = 1; c < nchunk; ++c) th.emplace_back(compile, c);
    compile(0);
    for (auto& t : th) t.join();
  }
  for (int c = 0; c < nchunk; ++c)
    if (!errs[c].empty()) {
      set_error(errs[c]);
      return JQ_EUNSUPPORTED;
    }
  for (int c = 0; c < nchunk; ++c) {
    CUmodule mod;
    if (g_drv.module_load(&mod, bins[c].data()) != CUDA_SUCCESS) {
      set_error("cuModuleLoadData failed for the specialised plan");
      return JQ_ECUDA;
    }
    out->modules.push_back(mod);
  }
  // kernel k of the forward list is body k; adjoint kernel k is body |names| + k
  auto lookup = [&](const std::vector<std::string>& nm, int base, std::vector<void*>* fk) -> int {
    fk->assign(nm.size(), nullptr);
    for (size_t k = 0; k < nm.size(); ++k) {
      CUfunction f;
      CUmodule mod = static_cast<CUmodule>(out->modules[chunk_of[base + static_cast<int>(k)]]);
      if (g_drv.get_function(&f, mod, nm[k].c_str()) != CUDA_SUCCESS) {
        set_error("cuModuleGetFunction failed for " + nm[k]);
        return JQ_ECUDA;
      }
      g_drv.set_attr(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, 227 * 1024);
      (*fk)[k] = f;
    }
    return JQ_OK;
  };
  std::vector<void*> fk, ak, bk;
  if (lookup(names, 0, &fk) || lookup(anames, static_cast<int>(names.size()), &ak) ||
      lookup(bnames, static_cast<int>(names.size() + anames.size()), &bk))
    return JQ_ECUDA;
  // per-pass matrix staging tables
  std::vector<int32_t> mc;
  // per-pass gradient flush tables: (shared accumulator offset, block
  // cotangent offset in complex128 units, number of doubles)
  std::vector<int32_t> gt;
  for (int p = 0; p < static_cast<int>(s.passes.size()); ++p) {
    if (kernel_of[p] < 0) continue;
    out->fn[p] = fk[kernel_of[p]];
    if (adj && akernel_of[p] >= 0) out->afn[p] = ak[akernel_of[p]];
    if (bwd && bkernel_of[p] >= 0) out->bfn[p] = bk[bkernel_of[p]];
    out->mc_off[p] = static_cast<int64_t>(mc.size());
    out->gt_off[p] = static_cast<int64_t>(gt.size());
    const PassDesc& pd = s.passes[p];
    int acc = 0;
    for (int ri = pd.rop_begin; ri < pd.rop_end; ++ri) {
      const RegOp& ro = s.rops[ri];
      if (ro.grad_off >= 0) {
        gt.push_back(acc);
        gt.push_back(ro.grad_off);
        gt.push_back(2 * ro.mat_len);
        acc += 2 * ro.mat_len;
      }
      if (ro.mat_len <= 0) continue;
      mc.push_back(static_cast<int32_t>(ro.w2));
      mc.push_back(static_cast<int32_t>(ro.w3));
      mc.push_back(ro.mat_len);
    }
  }
  if (mc.empty()) mc.push_back(0);
  if (gt.empty()) gt.push_back(0);
  if (cudaMalloc(&out->mc, mc.size() * sizeof(int32_t)) != cudaSuccess ||
      cudaMemcpy(out->mc, mc.data(), mc.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMalloc(&out->gt, gt.size() * sizeof(int32_t)) != cudaSuccess ||
      cudaMemcpy(out->gt, gt.data(), gt.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_error("upload of the matrix staging tables failed");
    return JQ_ECUDA;
  }
  out->has_adjoint = adj && !anames.empty();
  out->has_backward = bwd && !bnames.empty();
  out->n_kernels = static_cast<int>(names.size());
  return JQ_OK;
}

void jit_free(JitModule* m) {
  if (m && g_drv.ok)
    for (void* mod : m->modules) g_drv.module_unload(static_cast<CUmodule>(mod));
  if (m && m->mc) cudaFree(m->mc);
  if (m && m->gt) cudaFree(m->gt);
  if (m) {
    m->mc = nullptr;
    m->gt = nullptr;
    m->afn.clear();
    m->bfn.clear();
    m->modules.clear();
    m->fn.clear();
  }
}

size_t jit_smem(const Schedule& s, int p, int elem) {
  const PassDesc& pd = s.passes[p];
  const size_t smat_pad = static_cast<size_t>((pd.smat_len + 1) & ~1);
  return jit_bufs() * (static_cast<size_t>(1) << pd.t) * elem + smat_pad * elem + (elem == 8 ? 2 * smat_pad * elem : 0) +
         (static_cast<size_t>(1) << (pd.t - pd.c)) * 4;
}

int jit_launch(const JitModule& m, const Schedule& s, int p, int n_bits, int sm_count, void* state, int batch,
               const void* bmat, int64_t bstride, int elem, cudaStream_t st, void* out) {
  if (!out) out = state;
  CUfunction f = static_cast<CUfunction>(m.fn[p]);
  const PassDesc& pd = s.passes[p];
  const int threads = 1 << (pd.t - s.reg_bits);
  const size_t smem = jit_smem(s, p, elem);
  int per_sm = 0;
  g_drv.occupancy(&per_sm, f, threads, smem);
  if (per_sm < 1) per_sm = 1;
  const int64_t ntiles = (1LL << (n_bits - pd.t)) * batch;
  const int64_t cap = static_cast<int64_t>(sm_count) * per_sm;
  const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min(ntiles, cap)));
  long long bs = bstride;
  const int32_t* mc = static_cast<const int32_t*>(m.mc) + m.mc_off[p];
  int rev = alternate_tile_order() ? (p & 1) : 0;
  void* args[] = {&state, &batch, const_cast<void**>(&bmat), &bs, &mc, &out, &rev};
  if (launch_pass(f, grid, static_cast<unsigned>(threads), static_cast<unsigned>(smem), st, args, kPdlFwd) !=
      CUDA_SUCCESS) {
    set_error("cuLaunchKernel failed for a specialised pass");
    return JQ_ECUDA;
  }
  return JQ_OK;
}

}  // namespace jq

namespace jq {

size_t jit_adj_smem(const Schedule& s, int p, int elem) {
  const PassDesc& pd = s.passes[p];
  int nacc = 0;
  for (int ri = pd.rop_begin; ri < pd.rop_end; ++ri)
    if (s.rops[ri].grad_off >= 0) nacc += 2 * s.rops[ri].mat_len;
  const size_t smat_pad = static_cast<size_t>((pd.smat_len + 1) & ~1);
  return 2 * (static_cast<size_t>(1) << pd.t) * elem + smat_pad * elem + (elem == 8 ? 2 * smat_pad * elem : 0) +
         static_cast<size_t>((nacc + 1) & ~1) * 8 + (static_cast<size_t>(1) << (pd.t - pd.c)) * 4;
}

int jit_launch_adj(const JitModule& m, const Schedule& s, int p, int n_bits, int sm_count, void* psi, void* lam,
                   int batch, const void* bmat, int64_t bstride, double* gacc, int64_t gstride, int elem,
                   cudaStream_t st) {
  CUfunction f = static_cast<CUfunction>(m.afn[p]);
  const PassDesc& pd = s.passes[p];
  const int threads = 1 << (pd.t - s.reg_bits);
  const size_t smem = jit_adj_smem(s, p, elem);
  int per_sm = 0;
  g_drv.occupancy(&per_sm, f, threads, smem);
  if (per_sm < 1) per_sm = 1;
  const int64_t ntiles = (1LL << (n_bits - pd.t)) * batch;
  const int64_t cap = static_cast<int64_t>(sm_count) * per_sm;
  const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min(ntiles, cap)));
  long long bs = bstride, gs = gstride;
  const int32_t* mc = static_cast<const int32_t*>(m.mc) + m.mc_off[p];
  const int32_t* gt = static_cast<const int32_t*>(m.gt) + m.gt_off[p];
  void* args[] = {&psi, &lam, &batch, const_cast<void**>(&bmat), &bs, &mc, &gacc, &gs, &gt};
  if (launch_pass(f, grid, static_cast<unsigned>(threads), static_cast<unsigned>(smem), st, args, kPdlAdj) !=
      CUDA_SUCCESS) {
    set_error("cuLaunchKernel failed for a specialised adjoint pass");
    return JQ_ECUDA;
  }
  return JQ_OK;
}

int jit_launch_bwd(const JitModule& m, const Schedule& s, int p, int n_bits, int sm_count, const void* xin, void* lam,
                   int batch, const void* bmat, int64_t bstride, double* gacc, int64_t gstride, int elem,
                   cudaStream_t st) {
  CUfunction f = static_cast<CUfunction>(m.bfn[p]);
  const PassDesc& pd = s.passes[p];
  const int threads = 1 << (pd.t - s.reg_bits);
  const size_t smem = bwd_smem_bytes(s, p, elem);
  int per_sm = 0;
  g_drv.occupancy(&per_sm, f, threads, smem);
  if (per_sm < 1) per_sm = 1;
  const int64_t ntiles = (1LL << (n_bits - pd.t)) * batch;
  const int64_t cap = static_cast<int64_t>(sm_count) * per_sm;
  const unsigned grid = static_cast<unsigned>(std::max<int64_t>(1, std::min(ntiles, cap)));
  long long bs = bstride, gs = gstride;
  const int32_t* mc = static_cast<const int32_t*>(m.mc) + m.mc_off[p];
  const int32_t* gt = static_cast<const int32_t*>(m.gt) + m.gt_off[p];
  void* xp = const_cast<void*>(xin);
  void* args[] = {&xp, &lam, &batch, const_cast<void**>(&bmat), &bs, &mc, &gacc, &gs, &gt};
  if (launch_pass(f, grid, static_cast<unsigned>(threads), static_cast<unsigned>(smem), st, args, kPdlBwd) !=
      CUDA_SUCCESS) {
    set_error("cuLaunchKernel failed for a specialised reverse pass");
    return JQ_ECUDA;
  }
  return JQ_OK;
}

}  // namespace jq
