// Tensor-core update and operand packing (internal interface).
#pragma once

#include "common.cuh"

namespace lub {

// SPLIT16: compensated fp16, x * 2^s = hi + lo (both fp16); the copies hold
// three K segments, A: [hi | hi | lo], B: [hi ; lo ; hi], so one fp16 product
// of the concatenated operands is hi*hi + hi*lo + lo*hi.
enum class TcOperand { F16 = 0, BF16 = 1, E4M3 = 2, SPLIT16 = 3 };

inline int tc_operand_bytes(TcOperand k) { return k == TcOperand::E4M3 ? 1 : 2; }

// Kinds whose copies carry one power-of-two scale per 128-row / 128-column
// tile, and the bound the scaled tile maximum is brought under.
inline bool tc_scaled(TcOperand k) { return k == TcOperand::E4M3 || k == TcOperand::SPLIT16; }
inline float tc_scale_bound(TcOperand k) { return k == TcOperand::E4M3 ? 448.0f : 32768.0f; }

// Length of one packed row / column along K (segments padded to 16).
inline int64_t tc_packed_k(TcOperand k, int64_t K) {
  const int64_t kp = (K + 15) / 16 * 16;
  return k == TcOperand::SPLIT16 ? 3 * kp : kp;
}

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

// C -= A B + A2 B2 in one pass over C: two K-major operand sets (unscaled
// fp16 or bf16, the same leading dimension ld_p, K and K2 columns) summed
// in one fp32 accumulator, so C is read and written once for two outer
// steps' updates (c - (acc1 + acc2), one rounding).
lu_status launch_tc_update2(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                            int64_t K, const void* A, const void* B, int64_t K2,
                            const void* A2, const void* B2, int64_t ld_p, float* C,
                            int64_t ldc, int* err, int max_ctas = 0, int tiles_per_cta = 0);

// C -= sum_q A[q] B[q] in one pass over C: up to eight K-major operand sets
// (unscaled fp16 or bf16, the same leading dimension ld_p, K[q] columns
// each) summed in one fp32 accumulator, so C is read and written once for
// several outer steps' updates.  Persistent launches (tiles_per_cta = 0) of
// at least 296 tiles of 128 x 256 with K >= 512 in all and a C that TMA can
// address run as CTA pairs (tcgen05 cta_group::2, 256 x 256 tiles); every
// element's sum runs over K in the same order either way.
lu_status launch_tc_update_sets(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                                int nsets, const int64_t* K, const void* const* A,
                                const void* const* B, int64_t ld_p, float* C, int64_t ldc,
                                int* err, int max_ctas = 0, int tiles_per_cta = 0);

// The same update with C stored in fp16 (C = rn16(C + alpha * acc), the sum
// in fp32): the left-looking factorization of an fp16 matrix.
lu_status launch_tc_update_h(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                             int64_t K, float alpha, const void* A, int64_t lda_p,
                             const void* B, int64_t ldb_p, __half* C, int64_t ldc,
                             int* err);

// Split-K form of the update (unscaled fp16 / bf16 operands): the K blocks
// are cut into ksplit near-equal ranges, each tile x range a work unit (one
// CTA each, so concurrent launches share the SMs unit by unit) whose raw
// fp32 product goes to its own slab of `part` (ksplit x round4(M) x N
// floats); a second kernel adds the slabs in split order and stores
// C = rn(C + alpha * sum) (fp16 when c_half), and the stored value widened
// to fp32 into `shadow` (ld lds) when given.  The same result for every
// run, whatever the scheduling.
lu_status launch_tc_update_split(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                                 int64_t K, float alpha, const void* A, int64_t lda_p,
                                 const void* B, int64_t ldb_p, void* C, bool c_half,
                                 int64_t ldc, float* shadow, int64_t lds, int ksplit,
                                 float* part, int* err);

// The two halves of the split-K update, for callers that compute some K
// ranges ahead of others: launch_tc_partials writes the raw products of the
// K ranges of (A, B) cut into ksplit near-equal parts to slabs slab0,
// slab0 + 1, ... of `part` (each splitk_slab_floats(M, N) floats) and
// returns their number; launch_splitk_finish adds slabs 0 .. S-1 in order
// and stores C = rn(C + alpha * sum) (and the fp32 shadow when given).
int64_t splitk_slab_floats(int64_t M, int64_t N);
lu_status launch_tc_partials(cudaStream_t st, TcOperand kind, int64_t M, int64_t N,
                             int64_t K, const void* A, int64_t lda_p, const void* B,
                             int64_t ldb_p, int ksplit, float* part, int slab0, int* nslabs,
                             int* err);
lu_status launch_splitk_finish(cudaStream_t st, int64_t M, int64_t N, int S, const float* part,
                               float alpha, void* C, bool c_half, int64_t ldc, float* shadow,
                               int64_t lds);

// Number of K splits (1..smax, at least K = 256 fp16 per split) that
// minimises waves x K blocks per split for `tiles` 128 x 256 tiles on `sms`
// SMs (tiles: all the tiles launched at the same time).
int tc_split_choice(int64_t tiles, int64_t K, int esize, int sms, int smax);

// Self-test of the give-up path: the same fp16 update with the TMA producer
// issuing no loads and every barrier wait bounded by wait_cycles, so each
// consumer wait runs out; the kernel records its code in *err, unwinds,
// frees its TMEM and returns (tiles_per_cta > 2 selects the streaming-C
// epilogue, otherwise the reduce-add one).
lu_status launch_tc_update_withheld(cudaStream_t st, int64_t M, int64_t N, int64_t K,
                                    const void* A, int64_t lda_p, const void* B,
                                    int64_t ldb_p, float* C, int64_t ldc, int* err,
                                    long long wait_cycles, int tiles_per_cta);

// Largest power-of-two scale per 128-row tile of the fp32 column-major
// src (M x K) / per 128-column tile of src (K x N) such that amax * 2^s <=
// bound (448: e4m3 max; 32768 for split fp16).  `tmp` needs one int per tile.
lu_status launch_scale_rowtiles(cudaStream_t st, int64_t M, int64_t K,
                                const float* src, int64_t lds, int* scale,
                                int* tmp, float bound = 448.0f);
lu_status launch_scale_coltiles(cudaStream_t st, int64_t K, int64_t N,
                                const float* src, int64_t lds, int* scale,
                                int* tmp, float bound = 448.0f);

// A operand: dst[i*ldd + k] = round(src[i + k*lds] * 2^scale[i/128])
// (SPLIT16: the three segments, each round16(K) long, zero padded).
lu_status launch_pack_a(cudaStream_t st, TcOperand kind, int64_t M, int64_t K,
                        const float* src, int64_t lds, void* dst, int64_t ldd,
                        const int* scale);
// The same copies of fp16 sources (F16 kind, no scales): A transposed into
// the row-major copy, B into the compact column-major copy.
lu_status launch_pack_a_f16(cudaStream_t st, int64_t M, int64_t K, const __half* src,
                            int64_t lds, __half* dst, int64_t ldd);
lu_status launch_pack_b_f16(cudaStream_t st, int64_t K, int64_t N, const __half* src,
                            int64_t lds, __half* dst, int64_t ldd);
// B operand: dst[k + j*ldd] = round(src[k + j*lds] * 2^scale[j/128]).
lu_status launch_pack_b(cudaStream_t st, TcOperand kind, int64_t K, int64_t N,
                        const float* src, int64_t lds, void* dst, int64_t ldd,
                        const int* scale);

}  // namespace lub
