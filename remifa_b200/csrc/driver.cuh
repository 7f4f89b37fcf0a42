// Factorization drivers (host C++) shared by the C-ABI layer.
#pragma once

#include "common.cuh"

namespace lub {

// Left-looking outer blocks wider than this are factored as sub-blocks of
// this width (the one-CTA Crout diagonal kernel's limit).
constexpr int64_t kLlSub = 128;

// Everything a factorization call needs to know before enqueueing work.
struct Plan {
  int64_t n = 0;
  int64_t nb = 256;
  int diag_w = 128;
  lu_compute inner = LU_COMPUTE_FP32;
  lu_compute outer = LU_COMPUTE_FP32;
  lu_variant variant = LU_RIGHT_LOOKING;
  bool lookahead = true;
  lu_dtype dtype = LU_F32;
  bool panel_fp32 = false;  // fp16 storage: block update kept in fp32
  int bulk_group = 1;       // outer steps per bulk trailing-update pass (1..4)
  bool bulk_pair = false;   // bulk_group >= 2 (the host entry's catch-up pairs steps)
  // workspace layout (byte offsets into one device allocation)
  size_t off_status = 0;    // int first_bad
  size_t off_lcopy = 0;     // low-precision L21 copy (row-major)
  size_t off_ucopy = 0;     // low-precision U12 copy (column-major)
  size_t off_scales = 0;    // int per-tile scales (fp8)
  size_t off_shadow = 0;    // fp16 storage: fp32 copy of the current block
  int64_t ld_shadow = 0;    //   column and row, where the panel is factored
  size_t off_part = 0;      // left-looking tensor-core updates: split-K
  size_t part_bytes = 0;    //   partial slabs, block column then block row
  size_t lcopy_bytes = 0, ucopy_bytes = 0, scale_bytes = 0;
  size_t ws_bytes = 0;
};

lu_status check_device();
lu_status make_plan(const lu_opts& o, int64_t m, int64_t n, lu_dtype dtype,
                    Plan* p);
lu_status factorize(const lu_opts& o, cudaStream_t st, int64_t m, int64_t n,
                    void* d_a, lu_dtype dtype_a, int64_t lda, int* d_info,
                    void* d_a_lowp, int64_t ld_lowp, void* workspace,
                    size_t ws_bytes);
lu_status factorize_host(const lu_opts& o, cudaStream_t st, int64_t n, float* h_a,
                         int64_t lda, float* d_a, int64_t ldda, int* d_info,
                         void* workspace, size_t ws_bytes);
lu_status gemm_update(lu_compute compute, cudaStream_t st, int64_t m, int64_t n,
                      int64_t k, double alpha, const float* a, int64_t lda,
                      const float* b, int64_t ldb, double beta, float* c,
                      int64_t ldc, void* workspace, size_t ws_bytes);
lu_status gemm_update_ex(lu_compute compute, cudaStream_t st, int64_t m, int64_t n,
                         int64_t k, double alpha, const void* a, lu_dtype ta, int64_t lda,
                         const void* b, lu_dtype tb, int64_t ldb, double beta, void* c,
                         lu_dtype tc, int64_t ldc, void* workspace, size_t ws_bytes);

// A block row's early products as split-K partial slabs (slab s, column q,
// row i at part[s * slab + q * ldp + i]), summed in slab order and
// subtracted before anything else; ns = 0: none.
struct EarlyPart {
  const float* part = nullptr;
  int64_t slab = 0, ldp = 0;
  int ns = 0;
};

// One block row of the host entry's left-looking chunk catch-up: on the
// block whose factored in x in diagonal block sits at blk, the block row
// coff columns right of it (in x nc) gets R -= La Xb (K = kl, fp16 / bf16
// operands: La row i at la[i * lda_k], Xb column q at xb[q * ldx]), then the
// unit-lower solve in place, whose fp16 / bf16 copy goes to xo[q * ldx + i];
// with ep, R first loses the sum of its early partial products.  fused: one
// launch; otherwise the unfused kernels (split-K finish, tensor-core update,
// U-panel solves of diag_w rows, rank-8 updates between them).
lu_status catchup_row_step(cudaStream_t st, bool fused, bool bf16, float* blk, int64_t lda,
                           int64_t in, int64_t coff, int64_t nc, int64_t kl, const void* la,
                           int64_t lda_k, const void* xb, void* xo, int64_t ldx, int diag_w,
                           int* err, const EarlyPart& ep = EarlyPart());

}  // namespace lub
