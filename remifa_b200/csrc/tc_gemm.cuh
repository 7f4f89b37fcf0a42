// Tensor-core update and operand packing (internal interface).
#pragma once

#include "common.cuh"

namespace lub {

enum class TcOperand { F16 = 0, BF16 = 1, E4M3 = 2 };

inline int tc_operand_bytes(TcOperand k) { return k == TcOperand::E4M3 ? 1 : 2; }

// C[M x N] (fp32, column-major, ldc) += alpha * A * B, A row-major (lda_p),
// B column-major (ldb_p), both of type `kind`.  scale_a / scale_b (log2 per
// 128-row tile of A / 128-column tile of B) are divided out of the product.
// err: device int set non-zero if a bounded wait in the kernel gave up.
// tiles_per_cta = 0 launches one persistent CTA per SM (max_ctas caps it);
// > 0 gives every CTA that many consecutive 128 x 256 tiles, so SMs free up
// while the update runs and concurrent (higher-priority) work can start.
lu_status launch_tc_update(cudaStream_t st, TcOperand kind, int64_t M,
                           int64_t N, int64_t K, float alpha, const void* A,
                           int64_t lda_p, const void* B, int64_t ldb_p, float* C,
                           int64_t ldc, const int* scale_a, const int* scale_b,
                           int* err, int max_ctas = 0, int tiles_per_cta = 0);

// Largest power-of-two scale per 128-row tile of the fp32 column-major
// src (M x K) / per 128-column tile of src (K x N) such that amax * 2^s <=
// 448 (e4m3 max).  `tmp` needs one int per tile.
lu_status launch_scale_rowtiles(cudaStream_t st, int64_t M, int64_t K,
                                const float* src, int64_t lds, int* scale,
                                int* tmp);
lu_status launch_scale_coltiles(cudaStream_t st, int64_t K, int64_t N,
                                const float* src, int64_t lds, int* scale,
                                int* tmp);

// A operand: dst[i*ldd + k] = round(src[i + k*lds] * 2^scale[i/128]).
lu_status launch_pack_a(cudaStream_t st, TcOperand kind, int64_t M, int64_t K,
                        const float* src, int64_t lds, void* dst, int64_t ldd,
                        const int* scale);
// B operand: dst[k + j*ldd] = round(src[k + j*lds] * 2^scale[j/128]).
lu_status launch_pack_b(cudaStream_t st, TcOperand kind, int64_t K, int64_t N,
                        const float* src, int64_t lds, void* dst, int64_t ldd,
                        const int* scale);

}  // namespace lub
