// One step of the left-looking catch-up of a column chunk, fused into one
// launch: for block row t of the chunk (rows [ofs, ofs + in), the chunk's
// columns)
//   R -= sum_s P_s              the products with the solved rows of steps
//                               < t-1, as split-K partial slabs computed
//                               beforehand, summed in slab order (the
//                               split-K finish's arithmetic)
//   R -= L_{t,t-1} X_{t-1}      fp16 / bf16 operands, fp32 accumulation
//                               (mma.sync m16n8k16; K = the previous step's
//                               width), one rounding of the sum as in a
//                               tensor-core trailing update
//   X_t = L_tt^{-1} R           unit-lower forward substitution in fp32,
//                               in place
// and X_t's low-precision copy, the B operand of the later block rows and of
// the chunk's rows below.
//
// The solve applies the reference's operation order for the U part of a
// panel (src/lu_nopiv.cu:304-316 inside a tile of 8 rows; one K = 8 update
// per earlier tile, src/lu_nopiv_inner_rl.hxx:155-190): for element x_p of
// tile P, first, per earlier tile T in order, acc = sum over the tile's 8
// rows k of fma(x_k, L[p][k]) and x_p -= acc; then x_p = fma(-L[p][k], x_k,
// x_p) for the rows k < p of its own tile.  That is exactly what the blocked
// U-panel kernel and the rank-8-chunked update between its diagonal
// sub-blocks give, so X_t is bit-identical to the unfused solve for the
// same R.
//
// CTA = 32 columns, 16 warps.  Shared memory: the block row (column c at
// S[c * ls + p]) and the strictly-lower part of L_tt by panels of 8 columns
// (panel T: rows [8T, in) of columns 8T..8T+7, column-major), fp32 --
// 135 KB at in = 256.  Per tile T, after one barrier, warp 0 (one lane per
// column) applies tile T to tile T+1 and eliminates tile T+1 (look-ahead),
// while warps 1-15 apply tile T to the rows below tile T+1 in register
// micro-tiles of 2 columns x 8 rows (16 warps rather than 8 with 4 x 8
// tiles: more warps to cover the dependent chains; 31.1 -> 29.1 us per step
// at 256 x 4096 x K 256).
#include <type_traits>

#include "kernels.cuh"
#include "rowsolve.cuh"

namespace lub {
namespace {

constexpr int kRsCols = 32;   // columns per CTA
constexpr int kRsT = 512;     // threads
constexpr int kRsW = kRsT / 32;  // warps

__device__ __forceinline__ void rs_ld8(const float* p, float (&v)[8]) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  const float4 b = *reinterpret_cast<const float4*>(p + 4);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void rs_st8(float* p, const float (&v)[8]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  *reinterpret_cast<float4*>(p + 4) = make_float4(v[4], v[5], v[6], v[7]);
}

// First float of panel T (8 columns of in - 8T rows each) in the packed
// lower-triangle layout.
__host__ __device__ constexpr int rs_panel_off(int in, int T) {
  return 8 * T * in - 32 * T * (T - 1);
}

template <typename E>
__device__ __forceinline__ void rs_mma(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                       uint32_t a3, uint32_t b0, uint32_t b1) {
  if constexpr (std::is_same<E, __half>::value) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
  } else {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
  }
}

template <typename E>
__device__ __forceinline__ uint32_t rs_pack2(float x, float y) {
  if constexpr (std::is_same<E, __half>::value) {
    const __half2 h = __floats2half2_rn(x, y);
    return *reinterpret_cast<const uint32_t*>(&h);
  } else {
    const __nv_bfloat162 h = __floats2bfloat162_rn(x, y);
    return *reinterpret_cast<const uint32_t*>(&h);
  }
}

template <typename E>
__global__ void __launch_bounds__(kRsT)
ll_rowsolve_kernel(RowSolveArgs g) {
  extern __shared__ __align__(16) float smem[];
  const int in = g.in, nt = in / 8, ls = in + 4;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t col0 = (int64_t)blockIdx.x * kRsCols;
  const int64_t left = g.nc - col0;
  const int ncols = left < kRsCols ? (int)left : kRsCols;
  float* S = smem;                       // kRsCols x ls
  float* Fp = smem + kRsCols * ls;       // packed panels of L_tt

  // 1. the block row (group 0), then the panels of L_tt (group 1); with
  // early partial products the row is read directly and loses their sum
  // (slab order, then one fused subtraction: fma(-1, sum, r))
  {
    const float* R = g.r + col0 * g.ldr;
    // warp w: columns w and w + 16; its lanes stride down the column
    for (int c = warp; c < kRsCols; c += kRsW)
    for (int p = 4 * lane; p < in; p += 128) {
      float* d = S + c * ls + p;
      if (c >= ncols) {
        *reinterpret_cast<float4*>(d) = make_float4(0.f, 0.f, 0.f, 0.f);
      } else if (g.ns > 0) {
        const float* q = g.part + (col0 + c) * g.ldp + p;
        float4 t = __ldg(reinterpret_cast<const float4*>(q));
        for (int sl = 1; sl < g.ns; ++sl) {
          const float4 u = __ldg(reinterpret_cast<const float4*>(q + sl * g.slab));
          t.x = __fadd_rn(t.x, u.x);
          t.y = __fadd_rn(t.y, u.y);
          t.z = __fadd_rn(t.z, u.z);
          t.w = __fadd_rn(t.w, u.w);
        }
        const float* rp = R + p + (int64_t)c * g.ldr;
        float4 v;
        if (g.r_vec) {
          v = *reinterpret_cast<const float4*>(rp);
        } else {
          v.x = rp[0]; v.y = rp[1]; v.z = rp[2]; v.w = rp[3];
        }
        v.x = __fmaf_rn(-1.0f, t.x, v.x);
        v.y = __fmaf_rn(-1.0f, t.y, v.y);
        v.z = __fmaf_rn(-1.0f, t.z, v.z);
        v.w = __fmaf_rn(-1.0f, t.w, v.w);
        *reinterpret_cast<float4*>(d) = v;
      } else if (g.r_vec) {
        cp_async16(d, R + p + (int64_t)c * g.ldr);
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) cp_async4(d + e, R + p + e + (int64_t)c * g.ldr);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    // panel T, column k = warp % 8: rows [8T, in) down the lanes, the two
    // halves of the warps on alternate 128-row stretches
    for (int T = 0; T < nt; ++T) {
      const int rows = in - 8 * T, k = warp & 7;
      float* dst = Fp + rs_panel_off(in, T) + k * rows;
      const float* src = g.l + 8 * T + (int64_t)(8 * T + k) * g.ldl;
      for (int p = 4 * lane + 128 * (warp >> 3); p < rows; p += 256) {
        if (g.l_vec) {
          cp_async16(dst + p, src + p);
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e) cp_async4(dst + p + e, src + p + e);
        }
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 1;" ::: "memory");
    __syncthreads();
  }

  // 2. R -= L_{t,t-1} X_{t-1}: warp w owns the 16-row tile w (and w + 16) and
  // all four 8-column tiles.  Each lane loads 8 consecutive k of its A row
  // and B column per 32-k slab and feeds them to two MMAs (k permuted the
  // same way in A and B, so the products pair up).
  if (g.kl > 0) {
    const int gid = lane >> 2, tig = lane & 3;
    const int mt = in / 16;
    const E* A = static_cast<const E*>(g.la);
    const E* B = static_cast<const E*>(g.xb);
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0f;
    const bool has0 = warp < mt, has1 = warp + kRsW < mt;
#pragma unroll 2
    for (int kc = 0; kc < g.kl; kc += 32) {
      uint4 a[2][2], b[4];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int m = (warp + kRsW * i) * 16 + gid;
        const bool h = i == 0 ? has0 : has1;
#pragma unroll
        for (int r = 0; r < 2; ++r)
          a[i][r] = h ? __ldg(reinterpret_cast<const uint4*>(A + (int64_t)(m + 8 * r) * g.lda_k +
                                                             kc + 8 * tig))
                      : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = 8 * j + gid;
        b[j] = c < ncols ? __ldg(reinterpret_cast<const uint4*>(B + (col0 + c) * g.ldx + kc +
                                                                8 * tig))
                         : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        if (i == 0 ? !has0 : !has1) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          rs_mma<E>(acc[i][j], a[i][0].x, a[i][1].x, a[i][0].y, a[i][1].y, b[j].x, b[j].y);
          rs_mma<E>(acc[i][j], a[i][0].z, a[i][1].z, a[i][0].w, a[i][1].w, b[j].z, b[j].w);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      if (i == 0 ? !has0 : !has1) continue;
      const int m = (warp + kRsW * i) * 16 + gid;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = 8 * j + 2 * tig;
        float* s0 = S + c * ls + m;
        float* s1 = s0 + ls;
        s0[0] = __fsub_rn(s0[0], acc[i][j][0]);
        s1[0] = __fsub_rn(s1[0], acc[i][j][1]);
        s0[8] = __fsub_rn(s0[8], acc[i][j][2]);
        s1[8] = __fsub_rn(s1[8], acc[i][j][3]);
      }
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();

  // 3. X = L_tt^{-1} R in place
  if (warp == 0) {  // tile 0
    float x[8];
    float* xr = S + lane * ls;
    rs_ld8(xr, x);
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      float f[8];
      rs_ld8(Fp + k * in, f);  // L[c][k], c = 0..7
#pragma unroll
      for (int c = k + 1; c < 8; ++c) x[c] = __fmaf_rn(-f[c], x[k], x[c]);
    }
    rs_st8(xr, x);
  }
  __syncthreads();
  for (int T = 0; T + 1 < nt; ++T) {
    const int t0 = 8 * T, p0 = t0 + 8, rows = in - t0;
    const float* FT = Fp + rs_panel_off(in, T);  // L[p][t0 + k] at FT[k * rows + p - t0]
    if (warp == 0) {
      float* xr = S + lane * ls;
      float xv[8], x[8], acc[8];
      rs_ld8(xr + t0, xv);
      rs_ld8(xr + p0, x);
#pragma unroll
      for (int b = 0; b < 8; ++b) acc[b] = 0.0f;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        float f[8];
        rs_ld8(FT + k * rows + 8, f);  // L[p0 + b][t0 + k]
#pragma unroll
        for (int b = 0; b < 8; ++b) acc[b] = __fmaf_rn(xv[k], f[b], acc[b]);
      }
#pragma unroll
      for (int b = 0; b < 8; ++b) x[b] = __fsub_rn(x[b], acc[b]);
      const float* F1 = Fp + rs_panel_off(in, T + 1);
      const int rows1 = rows - 8;
#pragma unroll
      for (int k = 0; k < 7; ++k) {
        float f[8];
        rs_ld8(F1 + k * rows1, f);  // L[p0 + c][p0 + k]
#pragma unroll
        for (int c = k + 1; c < 8; ++c) x[c] = __fmaf_rn(-f[c], x[k], x[c]);
      }
      rs_st8(xr + p0, x);
    } else {
      const int q0 = p0 + 8;
      const int npos = (in - q0) / 8;
      for (int m = tid - 32; m < npos * 16; m += kRsT - 32) {
        const int ig = m & 15, pp = q0 + 8 * (m >> 4);
        float xv[2][8], acc[2][8];
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          rs_ld8(S + (ig + 16 * a) * ls + t0, xv[a]);
#pragma unroll
          for (int b = 0; b < 8; ++b) acc[a][b] = 0.0f;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          float f[8];
          rs_ld8(FT + k * rows + (pp - t0), f);  // L[pp + b][t0 + k]
#pragma unroll
          for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) acc[a][b] = __fmaf_rn(xv[a][k], f[b], acc[a][b]);
        }
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          float* row = S + (ig + 16 * a) * ls + pp;
          float c[8];
          rs_ld8(row, c);
#pragma unroll
          for (int b = 0; b < 8; ++b) c[b] = __fsub_rn(c[b], acc[a][b]);
          rs_st8(row, c);
        }
      }
    }
    __syncthreads();
  }

  // 4. X back in place, and its low-precision copy (column c, row p at
  // xo[(col0 + c) * ldx + p])
  {
    float* R = g.r + col0 * g.ldr;
    for (int c = warp; c < ncols; c += kRsW)
    for (int p = 4 * lane; p < in; p += 128) {
      const float4 v = *reinterpret_cast<const float4*>(S + c * ls + p);
      float* d = R + p + (int64_t)c * g.ldr;
      if (g.r_vec) {
        *reinterpret_cast<float4*>(d) = v;
      } else {
        d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
      }
    }
    E* xo = static_cast<E*>(g.xo);
    for (int c = warp; c < ncols; c += kRsW)
    for (int p = 8 * lane; p < in; p += 256) {
      float v[8];
      rs_ld8(S + c * ls + p, v);
      uint4 o;
      o.x = rs_pack2<E>(v[0], v[1]);
      o.y = rs_pack2<E>(v[2], v[3]);
      o.z = rs_pack2<E>(v[4], v[5]);
      o.w = rs_pack2<E>(v[6], v[7]);
      *reinterpret_cast<uint4*>(xo + (col0 + c) * g.ldx + p) = o;
    }
  }
}

}  // namespace

size_t rowsolve_smem_bytes(int in) {
  const int nt = in / 8;
  return sizeof(float) * ((size_t)kRsCols * (in + 4) + (size_t)rs_panel_off(in, nt));
}

bool rowsolve_supported(int64_t in, int64_t kl, int64_t ldk) {
  return in > 0 && in <= kRowSolveMaxRows && in % 32 == 0 && kl >= 0 && kl % 32 == 0 &&
         ldk % 8 == 0;
}

lu_status launch_ll_rowsolve(cudaStream_t st, bool bf16, const RowSolveArgs& a) {
  if (a.nc <= 0 || a.in <= 0) return LU_SUCCESS;
  if (!rowsolve_supported(a.in, a.kl, a.ldx) || a.ldx < a.in || a.ldx < a.kl ||
      (a.kl > 0 && a.lda_k % 8 != 0))
    return LU_ERR_INVALID_ARG;
  const auto al16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  if (!al16(a.xo) || (a.kl > 0 && (!al16(a.la) || !al16(a.xb)))) return LU_ERR_INVALID_ARG;
  if (a.ns > 0 && (!a.part || !al16(a.part) || a.slab % 4 != 0 || a.ldp % 4 != 0 ||
                   a.ldp < a.in || a.slab < a.ldp * a.nc))
    return LU_ERR_INVALID_ARG;
  RowSolveArgs g = a;
  g.r_vec = al16(a.r) && a.ldr % 4 == 0;
  g.l_vec = al16(a.l) && a.ldl % 4 == 0;
  const size_t sm = rowsolve_smem_bytes(a.in);
  const unsigned grid = (unsigned)ceil_div(a.nc, kRsCols);
  if (bf16) {
    LUB_CUDA_TRY(set_smem_limit((const void*)ll_rowsolve_kernel<__nv_bfloat16>, sm));
    ll_rowsolve_kernel<__nv_bfloat16><<<grid, kRsT, sm, st>>>(g);
  } else {
    LUB_CUDA_TRY(set_smem_limit((const void*)ll_rowsolve_kernel<__half>, sm));
    ll_rowsolve_kernel<__half><<<grid, kRsT, sm, st>>>(g);
  }
  LUB_LAUNCH_CHECK();
  return LU_SUCCESS;
}

}  // namespace lub
