// Per-plan specialised forward passes compiled with NVRTC (see jit.cpp).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "jq_internal.h"

namespace jq {

struct JitModule {
  std::vector<void*> modules;   // CUmodule per NVRTC program (kernels compile in parallel chunks)
  std::vector<void*> fn;        // CUfunction per pass (nullptr: interpreter)
  std::vector<void*> afn;       // adjoint CUfunction per pass (unitary statevector plans)
  std::vector<void*> bfn;       // checkpointed reverse CUfunction per pass (other plans)
  void* mc = nullptr;           // device int32 matrix staging tables
  void* gt = nullptr;           // device int32 gradient flush tables (adjoint and reverse passes)
  std::vector<int64_t> mc_off;  // per pass offset into mc
  std::vector<int64_t> gt_off;  // per pass offset into gt
  int n_kernels = 0;            // distinct kernels after sharing identical passes
  bool has_adjoint = false;
  bool has_backward = false;
};

bool jit_available();
std::string jit_source(const jq_plan* plan, const Schedule& s);
bool jit_pass_eligible(const Schedule& s, int p);
int jit_build(const jq_plan* plan, const Schedule& s, JitModule* out);
void jit_free(JitModule* m);
size_t jit_smem(const Schedule& s, int p, int elem);
int jit_bufs();
// One forward pass reading `state` and writing `out` (NULL: in place).
int jit_launch(const JitModule& m, const Schedule& s, int p, int n_bits, int sm_count, void* state, int batch,
               const void* bmat, int64_t bstride, int elem, cudaStream_t st, void* out = nullptr);

size_t jit_adj_smem(const Schedule& s, int p, int elem);
// One checkpointed reverse pass: xin is the state before the pass (read
// only), lam the cotangent after it (overwritten by the cotangent before it);
// block cotangents into gacc as for jit_launch_adj.
int jit_launch_bwd(const JitModule& m, const Schedule& s, int p, int n_bits, int sm_count, const void* xin, void* lam,
                   int batch, const void* bmat, int64_t bstride, double* gacc, int64_t gstride, int elem,
                   cudaStream_t st);
// One adjoint pass: psi <- G^dagger psi, lam <- G^dagger lam over the pass's
// blocks in reverse; block cotangents into gacc (instance stride gstride
// complex128 entries), none when gacc is NULL.
int jit_launch_adj(const JitModule& m, const Schedule& s, int p, int n_bits, int sm_count, void* psi, void* lam,
                   int batch, const void* bmat, int64_t bstride, double* gacc, int64_t gstride, int elem,
                   cudaStream_t st);

}  // namespace jq
