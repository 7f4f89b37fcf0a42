// Internal launchers shared between the kernel files and the drivers.
#pragma once

#include "common.cuh"

namespace lub {

// panel.cu
size_t diag_smem_bytes(int w);
lu_status launch_diag_factor(cudaStream_t st, float* a, int64_t lda, int w,
                             int64_t col0, int* first_bad);
// Low-precision K-major copies a panel launch also writes (fp16 or bf16:
// the tensor-core operands of the trailing update).  L row r of the launch
// (counted from its first item) goes to pa[(row0 + r) * ldk + k0 + c],
// c < w; U column q to pb[(col0 + q) * ldk + k0 + i], i < w.  Rows and
// columns whose packed index is negative lie inside the outer block and are
// not copied.
struct LuPack {
  void* pa = nullptr;
  void* pb = nullptr;
  int64_t ldk = 0;
  int64_t row0 = 0, col0 = 0;
  int k0 = 0;
  int bf16 = 0;
  // a second copy of the L rows (row r at pa2[(row02 + r) * ldk2 + k02 + c]),
  // every row of the launch
  void* pa2 = nullptr;
  int64_t ldk2 = 0, row02 = 0;
  int k02 = 0;
};

// L rows (M of them, below) and U columns (N, right) of the w x w factored
// diagonal block dg, one launch.  left: left-looking (Crout) update order.
// offL / offU: the first L row / U column handled is that many rows below /
// columns right of the block's edge.  pack: also write the finished rows /
// columns as low-precision operand copies.
lu_status launch_lupanel(cudaStream_t st, float* dg, int64_t lda, int w,
                         int64_t M, int64_t N, bool left = false, int64_t offL = 0,
                         int64_t offU = 0, const LuPack* pack = nullptr);
// Left-looking (Crout) factorization of a w x w (w <= 128) diagonal block.
lu_status launch_diag_crout(cudaStream_t st, float* a, int64_t lda, int w,
                            int64_t col0, int* first_bad);
lu_status launch_ref_panel(cudaStream_t st, int64_t m, int n, const float* d,
                           int64_t ldd, float* l, int64_t ldl, float* u,
                           int64_t ldu, int* stat);
// The same with fp16 storage and IEEE fp16 arithmetic (lu_nopiv_panel<half,8>).
lu_status launch_ref_panel_f16(cudaStream_t st, int64_t m, int n, const __half* d,
                               int64_t ldd, __half* l, int64_t ldl, __half* u,
                               int64_t ldu, int* stat);

// gemm_simt.cu
lu_status launch_sgemm_update(cudaStream_t st, int64_t M, int64_t N, int64_t K,
                              float alpha, const float* A, int64_t lda,
                              const float* B, int64_t ldb, float beta, float* C,
                              int64_t ldc, bool chunk8);

// Two independent rank-8-chunked updates C -= A * B in one launch (either
// region may be empty).
lu_status launch_sgemm_chunk8_2(cudaStream_t st, int64_t M0, int64_t N0,
                                int64_t K0, const float* A0, int64_t lda0,
                                const float* B0, int64_t ldb0, float* C0,
                                int64_t ldc0, int64_t M1, int64_t N1, int64_t K1,
                                const float* A1, int64_t lda1, const float* B1,
                                int64_t ldb1, float* C1, int64_t ldc1);

// convert.cu
lu_status launch_convert(cudaStream_t st, int64_t m, int64_t n, const void* a,
                         lu_dtype ta, int64_t lda, void* out, lu_dtype tout,
                         int64_t ldout, int scale_log2);

// gen.cu
lu_status launch_gen_matrix(cudaStream_t st, int64_t n, float* a, int64_t lda,
                            uint64_t seed, int kind, double alpha, int kscale,
                            double gamma_bits);

lu_status launch_gen_batch(cudaStream_t st, int64_t batch, float* const* ptrs,
                           const int32_t* ns, const int32_t* ldas, uint64_t seed,
                           int kind, double alpha);

// misc.cu
lu_status launch_fill_int(cudaStream_t st, int* p, int v, int64_t count);
lu_status launch_finalize_info(cudaStream_t st, const int* first_bad,
                               const int* err, int* info);

// Set the dynamic shared-memory limit of `func` for the current device.
cudaError_t set_smem_limit(const void* func, size_t bytes);

}  // namespace lub
