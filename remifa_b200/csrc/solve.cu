// Triangular solves with the in-place L\U factors and the FP64 residual of
// iterative refinement.
//
// The reference solves on the host with LAPACK getrs and identity pivots
// (tests/testing_lu_gpu.hxx:1309-1313); its GPU solve is referenced but not
// shipped (tests/testing_lu_gpu.hxx:1353-1359).  Here the solves run on the
// device: the factors stay fp32 (4 bytes per element read per solve, the
// bandwidth that bounds a triangular solve), the right-hand sides and all
// arithmetic are fp64, so the solve adds no fp32 rounding on top of the
// factorization error -- what iterative refinement in fp64 needs.
//
// op(T) x = b with T = L (unit lower) or U (upper), op = identity or
// transpose, is solved blockwise (block NBS = 256) in the order the
// triangle dictates: a one-CTA kernel solves the diagonal block (in 32-row
// chunks, a warp substituting each chunk with shuffles), then a wide kernel
// subtracts that block's contribution from all later rows.  Transposed
// solves read the factor along rows, so their kernels assign a warp per row
// and reduce with shuffles to keep the loads coalesced.
#include "common.cuh"
#include "kernels.cuh"
#include "solve.cuh"

namespace lub {
namespace {

constexpr int NBS = 256;   // block of the blocked solve
constexpr int CH = 32;     // chunk solved by one warp
constexpr int kT = 256;    // threads per CTA

// element (i, k) of op(T) inside the stored factor `lu`
__device__ __forceinline__ double opT(const float* lu, int64_t ld, int64_t i,
                                      int64_t k, bool trans) {
  return (double)(trans ? lu[k + i * ld] : lu[i + k * ld]);
}

// Solve the diagonal block rows [b0, b0+nbk) of op(T) for RHS column
// blockIdx.x of X (ld ldx).  forward: lower-triangular op(T) (L, or U^T);
// unit: unit diagonal (L or L^T).
__global__ void __launch_bounds__(kT)
trsm_diag_kernel(const float* __restrict__ lu, int64_t ld, int64_t b0, int nbk,
                 double* __restrict__ X, int64_t ldx, bool trans, bool forward,
                 bool unit) {
  __shared__ double xs[NBS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* x = X + (int64_t)blockIdx.x * ldx + b0;
  for (int i = tid; i < nbk; i += kT) xs[i] = x[i];
  __syncthreads();
  const int nch = (nbk + CH - 1) / CH;
  for (int cc = 0; cc < nch; ++cc) {
    const int c = forward ? cc : nch - 1 - cc;
    const int c0 = c * CH;
    const int cw = min(CH, nbk - c0);
    if (warp == 0) {
      // lane i holds row c0+i of the chunk triangle
      double tri[CH];
      const bool live = lane < cw;
#pragma unroll
      for (int k = 0; k < CH; ++k)
        tri[k] = (live && k < cw) ? opT(lu, ld, b0 + c0 + lane, b0 + c0 + k, trans) : 0.0;
      double xi = live ? xs[c0 + lane] : 0.0;
      if (forward) {
#pragma unroll
        for (int k = 0; k < CH; ++k) {
          if (k < cw) {
            if (!unit && lane == k) xi = xi / tri[k];
            const double xk = __shfl_sync(0xffffffffu, xi, k);
            if (lane > k && live) xi = fma(-tri[k], xk, xi);
          }
        }
      } else {
#pragma unroll
        for (int kk = 0; kk < CH; ++kk) {
          const int k = CH - 1 - kk;
          if (k < cw) {
            if (!unit && lane == k) xi = xi / tri[k];
            const double xk = __shfl_sync(0xffffffffu, xi, k);
            if (lane < k && live) xi = fma(-tri[k], xk, xi);
          }
        }
      }
      if (live) xs[c0 + lane] = xi;
    }
    __syncthreads();
    // rows of the block still to solve receive this chunk's contribution
    const int r_lo = forward ? c0 + cw : 0;
    const int r_hi = forward ? nbk : c0;
    if (!trans) {
      for (int r = r_lo + tid; r < r_hi; r += kT) {
        double acc = 0.0;
        for (int k = 0; k < cw; ++k)
          acc = fma(opT(lu, ld, b0 + r, b0 + c0 + k, false), xs[c0 + k], acc);
        xs[r] -= acc;
      }
    } else {
      for (int r = r_lo + warp; r < r_hi; r += kT / 32) {
        double p = lane < cw ? opT(lu, ld, b0 + r, b0 + c0 + lane, true) * xs[c0 + lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        if (lane == 0) xs[r] -= p;
      }
    }
    __syncthreads();
  }
  for (int i = tid; i < nbk; i += kT) x[i] = xs[i];
}

// X[rows, :] -= op(T)[rows, blk] * X[blk, :] for the rows [r0, r1) outside
// the block; blockIdx.y = RHS column.  Non-transposed: thread per row,
// loads coalesced along the column of T.
__global__ void __launch_bounds__(kT)
trsm_update_n_kernel(const float* __restrict__ lu, int64_t ld, int64_t b0,
                     int nbk, int64_t r0, int64_t r1, double* __restrict__ X,
                     int64_t ldx) {
  __shared__ double xb[NBS];
  double* x = X + (int64_t)blockIdx.y * ldx;
  for (int k = threadIdx.x; k < nbk; k += kT) xb[k] = x[b0 + k];
  __syncthreads();
  const int64_t r = r0 + (int64_t)blockIdx.x * kT + threadIdx.x;
  if (r >= r1) return;
  const float* col = lu + r + b0 * ld;
  double acc = 0.0;
#pragma unroll 8
  for (int k = 0; k < nbk; ++k) acc = fma((double)col[k * ld], xb[k], acc);
  x[r] -= acc;
}

// Transposed: op(T)[r, k] = lu[k + r*ld] is contiguous in k; a warp per row.
__global__ void __launch_bounds__(kT)
trsm_update_t_kernel(const float* __restrict__ lu, int64_t ld, int64_t b0,
                     int nbk, int64_t r0, int64_t r1, double* __restrict__ X,
                     int64_t ldx) {
  __shared__ double xb[NBS];
  double* x = X + (int64_t)blockIdx.y * ldx;
  for (int k = threadIdx.x; k < nbk; k += kT) xb[k] = x[b0 + k];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t r = r0 + ((int64_t)blockIdx.x * kT + threadIdx.x) / 32;
  if (r >= r1) return;
  const float* row = lu + b0 + r * ld;
  double p = 0.0;
  for (int k = lane; k < nbk; k += 32) p = fma((double)row[k], xb[k], p);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
  if (lane == 0) x[r] -= p;
}

// ---- residual r = b - A x (fp32 A, fp64 b, x, r) -------------------------
// Column chunks of kRC columns give partial dot products P[chunk][row]; a
// second pass adds them in chunk order, so the result does not depend on
// scheduling.
constexpr int kRC = 256;

__global__ void __launch_bounds__(kT)
residual_partial_kernel(int64_t n, const float* __restrict__ A, int64_t lda,
                        const double* __restrict__ x, double* __restrict__ P) {
  __shared__ double xs[kRC];
  const int64_t c0 = (int64_t)blockIdx.y * kRC;
  const int cn = (int)((n - c0) < kRC ? (n - c0) : kRC);
  for (int k = threadIdx.x; k < cn; k += kT) xs[k] = x[c0 + k];
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
  if (i >= n) return;
  const float* col = A + i + c0 * lda;
  double acc = 0.0;
#pragma unroll 8
  for (int k = 0; k < cn; ++k) acc = fma((double)col[k * lda], xs[k], acc);
  P[(int64_t)blockIdx.y * n + i] = acc;
}

// r = b - sum_chunks P; also the row sums |A| once (rowsum != null) and the
// maxima needed for the backward error (atomicMax on non-negative doubles
// through their bit patterns).
__global__ void __launch_bounds__(kT)
residual_final_kernel(int64_t n, int nchunks, const double* __restrict__ P,
                      const double* __restrict__ b, const double* __restrict__ x,
                      double* __restrict__ r, unsigned long long* __restrict__ maxes) {
  const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
  double ri = 0.0, xi = 0.0, bi = 0.0;
  if (i < n) {
    double s = 0.0;
    for (int c = 0; c < nchunks; ++c) s += P[(int64_t)c * n + i];
    bi = b[i];
    ri = bi - s;
    r[i] = ri;
    xi = x[i];
  }
  // maxes[0] = max |r|, [1] = max |x|, [2] = max |b|
  double v[3] = {fabs(ri), fabs(xi), fabs(bi)};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double m = v[q];
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&maxes[q], (unsigned long long)__double_as_longlong(m));
  }
}

// max_i sum_j |a_ij| (the infinity norm), same chunked scheme.
__global__ void __launch_bounds__(kT)
rowsum_partial_kernel(int64_t n, const float* __restrict__ A, int64_t lda,
                      double* __restrict__ P) {
  const int64_t c0 = (int64_t)blockIdx.y * kRC;
  const int cn = (int)((n - c0) < kRC ? (n - c0) : kRC);
  const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
  if (i >= n) return;
  const float* col = A + i + c0 * lda;
  double acc = 0.0;
  for (int k = 0; k < cn; ++k) acc += fabs((double)col[k * lda]);
  P[(int64_t)blockIdx.y * n + i] = acc;
}

__global__ void __launch_bounds__(kT)
rowsum_final_kernel(int64_t n, int nchunks, const double* __restrict__ P,
                    unsigned long long* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * kT + threadIdx.x;
  double s = 0.0;
  if (i < n)
    for (int c = 0; c < nchunks; ++c) s += P[(int64_t)c * n + i];
  for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(s));
}

__global__ void axpy_kernel(int64_t n, const double* __restrict__ d,
                            double* __restrict__ x) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += d[i];
}

}  // namespace

lu_status launch_trsm(cudaStream_t st, int64_t n, const float* lu, int64_t ld,
                      double* X, int64_t ldx, int64_t nrhs, bool upper,
                      bool trans) {
  if (n <= 0 || nrhs <= 0) return LU_SUCCESS;
  if (nrhs > 65535) return LU_ERR_INVALID_ARG;
  // op(T) is lower (forward substitution) for L and for U^T
  const bool forward = (upper == trans);
  const bool unit = !upper;
  const int64_t nblk = ceil_div(n, NBS);
  for (int64_t bb = 0; bb < nblk; ++bb) {
    const int64_t blk = forward ? bb : nblk - 1 - bb;
    const int64_t b0 = blk * NBS;
    const int nbk = (int)std::min<int64_t>(NBS, n - b0);
    trsm_diag_kernel<<<(unsigned)nrhs, kT, 0, st>>>(lu, ld, b0, nbk, X, ldx,
                                                    trans, forward, unit);
    LUB_LAUNCH_CHECK();
    const int64_t r0 = forward ? b0 + nbk : 0;
    const int64_t r1 = forward ? n : b0;
    if (r1 > r0) {
      if (!trans) {
        dim3 g((unsigned)ceil_div(r1 - r0, kT), (unsigned)nrhs);
        trsm_update_n_kernel<<<g, kT, 0, st>>>(lu, ld, b0, nbk, r0, r1, X, ldx);
      } else {
        dim3 g((unsigned)ceil_div((r1 - r0) * 32, kT), (unsigned)nrhs);
        trsm_update_t_kernel<<<g, kT, 0, st>>>(lu, ld, b0, nbk, r0, r1, X, ldx);
      }
      LUB_LAUNCH_CHECK();
    }
  }
  return LU_SUCCESS;
}

size_t residual_ws_bytes(int64_t n) {
  return align_up((size_t)ceil_div(n, kRC) * n * sizeof(double), 256) + 256;
}

lu_status launch_residual(cudaStream_t st, int64_t n, const float* A,
                          int64_t lda, const double* b, const double* x,
                          double* r, void* ws, unsigned long long* maxes) {
  const int nch = (int)ceil_div(n, kRC);
  double* P = static_cast<double*>(ws);
  LUB_CUDA_TRY(cudaMemsetAsync(maxes, 0, 3 * sizeof(unsigned long long), st));
  dim3 g((unsigned)ceil_div(n, kT), (unsigned)nch);
  residual_partial_kernel<<<g, kT, 0, st>>>(n, A, lda, x, P);
  LUB_LAUNCH_CHECK();
  residual_final_kernel<<<(unsigned)ceil_div(n, kT), kT, 0, st>>>(n, nch, P, b, x, r, maxes);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_norm_inf(cudaStream_t st, int64_t n, const float* A,
                          int64_t lda, void* ws, unsigned long long* out) {
  const int nch = (int)ceil_div(n, kRC);
  double* P = static_cast<double*>(ws);
  LUB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(unsigned long long), st));
  dim3 g((unsigned)ceil_div(n, kT), (unsigned)nch);
  rowsum_partial_kernel<<<g, kT, 0, st>>>(n, A, lda, P);
  LUB_LAUNCH_CHECK();
  rowsum_final_kernel<<<(unsigned)ceil_div(n, kT), kT, 0, st>>>(n, nch, P, out);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

lu_status launch_axpy(cudaStream_t st, int64_t n, const double* d, double* x) {
  axpy_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(n, d, x);
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace lub
