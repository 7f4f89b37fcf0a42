// The fused block-row step of the left-looking chunk catch-up (rowsolve.cu).
#pragma once

#include "common.cuh"

namespace lub {

// Rows of the widest block row one launch solves (its L_tt panels fill
// 135 KB of shared memory).
constexpr int kRowSolveMaxRows = 256;

struct RowSolveArgs {
  float* r = nullptr;        // block row: in rows x nc columns, column-major
  int64_t ldr = 0;
  const float* l = nullptr;  // L_tt: in x in, unit lower part used
  int64_t ldl = 0;
  const void* la = nullptr;  // L_{t,t-1}: in rows x kl, row r at la + r * lda_k
  int64_t lda_k = 0;
  const void* xb = nullptr;  // X_{t-1}: kl x nc, column c at xb + c * ldx
  void* xo = nullptr;        // X_t copy: in x nc, column c at xo + c * ldx
  int64_t ldx = 0;
  int64_t nc = 0;
  int in = 0;
  int kl = 0;                // 0: no product to subtract (the first step)
  const float* part = nullptr;  // early products: ns split-K slabs, slab s,
  int64_t slab = 0, ldp = 0;    //   column c, row i at part[s * slab + c * ldp + i],
  int ns = 0;                   //   summed in slab order and subtracted first
  bool r_vec = false;        // set by the launcher: 16-byte paths usable
  bool l_vec = false;
};

// Whether a block row of `in` rows with a previous step of kl columns fits
// the fused kernel (in a multiple of 32 up to kRowSolveMaxRows, kl a
// multiple of 32, the operand copies' leading dimension a multiple of 8).
bool rowsolve_supported(int64_t in, int64_t kl, int64_t ldk);
size_t rowsolve_smem_bytes(int in);
// R -= sum of the slabs; R -= L_{t,t-1} X_{t-1}; X_t = L_tt^{-1} R in
// place; X_t's fp16 (bf16 if bf16) copy to xo.  The operand pointers la, xb
// and xo are 16-byte aligned, part too with slab and ldp multiples of 4.
lu_status launch_ll_rowsolve(cudaStream_t st, bool bf16, const RowSolveArgs& a);

}  // namespace lub
