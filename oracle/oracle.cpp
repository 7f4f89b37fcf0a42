// TEST INFRASTRUCTURE ONLY -- CPU oracle for the no-pivot LU hot path.
// See oracle.h for the contract.  Loaded only by tests/, the smoke check and
// bench.py's CPU-baseline leg; never by the product library.
//
// Each function cites the reference (flipflapflop/remifa) file:line whose
// behaviour it restates.  Nothing is copied: the loops below are written
// from the algorithm, with the floating-point order made explicit so the
// GPU's FP32 path can be compared bit for bit.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include <omp.h>

namespace {

inline float& at(float* a, int64_t lda, int64_t i, int64_t j) {
  return a[i + j * lda];
}
inline float at(const float* a, int64_t lda, int64_t i, int64_t j) {
  return a[i + j * lda];
}

// splitmix64 finaliser (Steele, Lea, Flood 2014) -- a published mixing
// function; the device generator in the library uses the same one.
inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

inline uint64_t key_hash(uint64_t seed, uint64_t i, uint64_t j) {
  return mix64(((i << 32) | (j & 0xffffffffull)) ^ mix64(seed));
}

// Integer sample for entry (i, j): kind 0 -> q in [-2^23, 2^23) (value
// q * 2^-23); kind 1 -> Irwin-Hall sum of twelve 21-bit uniforms, centred,
// |q| < 6 * 2^21 (value q * 2^-21 ~ N(0,1)).
inline int32_t sample_q(uint64_t seed, uint64_t i, uint64_t j, int kind) {
  uint64_t h = key_hash(seed, i, j);
  if (kind == 0) return (int32_t)(h >> 40) - (1 << 23);
  int64_t s = 0;
  for (int w = 0; w < 4; ++w) {
    s += (int64_t)(h & 0x1fffff);
    s += (int64_t)((h >> 21) & 0x1fffff);
    s += (int64_t)((h >> 42) & 0x1fffff);
    h = mix64(h);
  }
  const int32_t q = (int32_t)(s - 6ll * (1ll << 21));
  return kind == 2 ? (q < 0 ? q : -q) : q;  // kind 2: -|kind 1|
}

// Round a finite value to a binary format with p significant bits, minimum
// normal exponent emin and largest finite value maxf; ties to even.
double round_format(double v, int p, int emin, double maxf, bool saturate) {
  if (v == 0.0 || !std::isfinite(v)) return v;
  double a = std::fabs(v);
  int e2;
  std::frexp(a, &e2);  // a = f * 2^e2, f in [0.5, 1)
  int e = std::max(e2 - 1, emin);
  double quantum = std::ldexp(1.0, e - (p - 1));
  double r = std::nearbyint(a / quantum) * quantum;  // default mode: RN-even
  if (r > maxf) r = saturate ? maxf : INFINITY;
  return std::copysign(r, v);
}

float round_fmt(float x, int fmt) {
  switch (fmt) {
    case 1:  // binary16
      return (float)round_format(x, 11, -14, 65504.0, false);
    case 2:  // bfloat16
      return (float)round_format(x, 8, -126, 3.3895313892515355e38, false);
    case 3:  // e4m3 (OCP FP8), saturating like cvt.rn.satfinite
      if (std::isnan(x)) return x;
      return (float)round_format(x, 4, -6, 448.0, true);
    default:
      return x;
  }
}

// Largest power of two 2^s with amax * 2^s <= fmax (the per-tile scale of the
// fp8 copies); 0 for an all-zero tile.
int pow2_scale(float amax, double fmax) {
  if (!(amax > 0.0f) || !std::isfinite(amax)) return 0;
  int e2;
  std::frexp((double)amax, &e2);  // amax in [2^(e2-1), 2^e2)
  int s = 0;
  double lim = fmax;
  // want amax * 2^s <= fmax
  s = (int)std::floor(std::log2(lim)) - e2;
  while (std::ldexp((double)amax, s + 1) <= lim) ++s;
  while (std::ldexp((double)amax, s) > lim) --s;
  return s;
}

}  // namespace

extern "C" {

int orc_num_threads(void) { return omp_get_max_threads(); }

// ---------------------------------------------------------------- generators

// reference tests/genmat.hxx:69-102
void orc_gen_diagdom_f32(int64_t m, int64_t n, float* a, int64_t lda) {
  std::default_random_engine generator;
  std::uniform_real_distribution<float> distribution(-1.0f, 1.0f);
  for (int64_t i = 0; i < m; ++i) {
    for (int64_t j = 0; j < n; ++j) at(a, lda, i, j) = distribution(generator);
    at(a, lda, i, i) = (float)m;
  }
}

// reference tests/common.hxx:298-319
void orc_gen_randmat_f32(int64_t m, int64_t n, float* a, int64_t lda,
                         uint32_t seed) {
  std::default_random_engine generator(seed);
  std::uniform_real_distribution<float> distribution(-1.0f, 1.0f);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t i = 0; i < m; ++i) at(a, lda, i, j) = distribution(generator);
}

void orc_gen_matrix_f32(int64_t n, float* a, int64_t lda, uint64_t seed,
                        int kind, double alpha, int kscale, double gamma_bits) {
  const float scale =
      kind == 0 ? std::ldexp(1.0f, -23)
                : (float)(std::ldexp(1.0, -21) / std::sqrt((double)n));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int64_t rowsum = 0;
    int shift = 0;
    if (gamma_bits != 0.0 && n > 1)
      shift = -(int)std::llrint(gamma_bits * (double)i / (double)(n - 1));
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      int32_t q = sample_q(seed, (uint64_t)i, (uint64_t)j, kind);
      rowsum += q < 0 ? -(int64_t)q : (int64_t)q;
      float v = (float)q * scale;
      at(a, lda, i, j) = std::ldexp(std::ldexp(v, kscale), shift);
    }
    float d = (float)(alpha * (double)rowsum * (double)scale);
    at(a, lda, i, i) = std::ldexp(std::ldexp(d, kscale), shift);
  }
}

void orc_gen_vector_f64(int64_t n, double* x, uint64_t seed, int kind) {
  for (int64_t i = 0; i < n; ++i) {
    int32_t q = sample_q(seed, (uint64_t)i, 0xffffffffull, kind);
    x[i] = kind == 0 ? std::ldexp((double)q, -23) : std::ldexp((double)q, -21);
  }
}

// reference tests/common.hxx:744-756 (b = A x); BLAS order is unspecified
// there, so this version accumulates in fp64 and rounds once.
void orc_gen_rhs_f32(int64_t m, const float* a, int64_t lda, const float* x,
                     float* b) {
  std::vector<double> acc(m, 0.0);
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = 0; i < m; ++i)
      acc[i] += (double)at(a, lda, i, j) * (double)x[j];
  for (int64_t i = 0; i < m; ++i) b[i] = (float)acc[i];
}

// ---------------------------------------------------------------- rounding

float orc_round_fmt(float x, int fmt, int scale_log2) {
  return round_fmt(std::ldexp(x, scale_log2), fmt);
}

// reference src/convert.cu:99-101 (fp32 -> fp16, round to nearest even)
void orc_convert(int64_t m, int64_t n, const float* a, int64_t lda, float* out,
                 int64_t ldo, int fmt, int scale_log2) {
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < n; ++j)
    for (int64_t i = 0; i < m; ++i)
      out[i + j * ldo] = orc_round_fmt(at(a, lda, i, j), fmt, scale_log2);
}

// ---------------------------------------------------------------- panel

// reference src/lu_nopiv.cu:105-180 (dev_lu_nopiv_block), :256-326
// (dev_lu_nopiv_br_block), launcher :364-400.  The diagonal tile is factored
// from the copy d (src/lu_nopiv_inner_rl.hxx:117-122 makes that copy); the L
// rows use 1/d then a multiply (src/lu_nopiv.cu:134,141-152), the rank-1
// updates are fused a - b*c (src/lu_nopiv.cu:156-168, :304-316).
void orc_panel_f32(int64_t m, int64_t n, const float* d, int64_t ldd, float* l,
                   int64_t ldl, float* u, int64_t ldu) {
  float T[8][8];  // T[row][col]
  float inv[8];
  for (int r = 0; r < 8; ++r)
    for (int c = 0; c < 8; ++c)
      T[r][c] = (r < n && c < n) ? d[r + c * ldd] : 0.0f;
  for (int k = 0; k < n; ++k) {
    inv[k] = 1.0f / T[k][k];
    for (int r = k + 1; r < n; ++r) T[r][k] = T[r][k] * inv[k];
    for (int c = k + 1; c < n; ++c)
      for (int r = k + 1; r < 8; ++r)
        T[r][c] = std::fma(-T[r][k], T[k][c], T[r][c]);
  }
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < n; ++r) l[r + c * ldl] = T[r][c];
  // L rows below the tile (independent of each other)
#pragma omp parallel for schedule(static) if (m - n > 4096)
  for (int64_t r = n; r < m; ++r) {
    float row[8];
    for (int c = 0; c < n; ++c) row[c] = l[r + c * ldl];
    for (int k = 0; k < n; ++k) {
      row[k] = row[k] * inv[k];
      for (int c = k + 1; c < n; ++c) row[c] = std::fma(-row[k], T[k][c], row[c]);
    }
    for (int c = 0; c < n; ++c) l[r + c * ldl] = row[c];
  }
  // U columns right of the tile (the block row runs to column m: the
  // reference assumes a square trailing matrix, src/lu_nopiv.cu:364-372)
#pragma omp parallel for schedule(static) if (m - n > 4096)
  for (int64_t c = n; c < m; ++c) {
    float col[8];
    for (int r = 0; r < n; ++r) col[r] = u[r + c * ldu];
    for (int k = 0; k < n; ++k)
      for (int r = k + 1; r < n; ++r) col[r] = std::fma(-T[r][k], col[k], col[r]);
    for (int r = 0; r < n; ++r) u[r + c * ldu] = col[r];
  }
}

// reference src/lu_nopiv.cu:105-326 instantiated for half (lu_nopiv_panel
// <half,8>): the same loops in fp16 arithmetic -- the reciprocal 1/d and the
// scaling each rounded to fp16, and a -= l * u, which nvcc contracts into an
// fp16 fused multiply-add (the reference's outputs agree only with the fused
// form), rounded once.  Values are held in floats (each an fp16 number).
// 1/d and l * (1/d): computed in fp32 and rounded once to fp16, which is the
// correctly rounded fp16 result (exact products; 24 >= 2 * 11 + 2 bits for
// the quotient).  a - l * u: the product is exact in fp64, the difference is
// formed exactly as a double-double (two-sum), and the sum rounded to fp16
// with the low part breaking a tie of the high part.
static float rn16(float x) { return round_fmt(x, 1); }

static double rn16d(double v) { return round_format(v, 11, -14, 65504.0, false); }

static float fma16(float a, float l, float u) {
  const double p = (double)l * (double)u;  // exact (22 bits)
  const double s = (double)a - p;
  const double bb = s - (double)a;         // two-sum: a - p = s + e exactly
  const double e = ((double)a - (s - bb)) + (-p - bb);
  double r = rn16d(s);
  if (e != 0.0 && std::isfinite(r)) {
    // s differs from the exact value by less than half a double ulp, so only
    // a tie (s exactly halfway between two fp16 numbers r and r2) can round
    // differently: then the exact value lies on e's side of s
    const double r2 = 2.0 * s - r;
    if (r2 != r && rn16d(r2) == r2) r = e > 0.0 ? std::max(r, r2) : std::min(r, r2);
  }
  return (float)r;
}

void orc_panel_f16(int64_t m, int64_t n, const float* d, int64_t ldd, float* l,
                   int64_t ldl, float* u, int64_t ldu) {
  float T[8][8];
  float inv[8];
  for (int r = 0; r < 8; ++r)
    for (int c = 0; c < 8; ++c) T[r][c] = (r < n && c < n) ? d[r + c * ldd] : 0.0f;
  auto sub_mul = [](float a, float x, float y) { return fma16(a, x, y); };
  for (int k = 0; k < n; ++k) {
    inv[k] = rn16(1.0f / T[k][k]);
    for (int r = k + 1; r < n; ++r) T[r][k] = rn16(T[r][k] * inv[k]);
    for (int c = k + 1; c < n; ++c)
      for (int r = k + 1; r < n; ++r) T[r][c] = sub_mul(T[r][c], T[r][k], T[k][c]);
  }
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < n; ++r) l[r + c * ldl] = T[r][c];
  for (int64_t r = n; r < m; ++r) {
    float row[8];
    for (int c = 0; c < n; ++c) row[c] = l[r + c * ldl];
    for (int k = 0; k < n; ++k) {
      row[k] = rn16(row[k] * inv[k]);
      for (int c = k + 1; c < n; ++c) row[c] = sub_mul(row[c], row[k], T[k][c]);
    }
    for (int c = 0; c < n; ++c) l[r + c * ldl] = row[c];
  }
  for (int64_t c = n; c < m; ++c) {
    float col[8];
    for (int r = 0; r < n; ++r) col[r] = u[r + c * ldu];
    for (int k = 0; k < n; ++k)
      for (int r = k + 1; r < n; ++r) col[r] = sub_mul(col[r], T[r][k], col[k]);
    for (int r = 0; r < n; ++r) u[r + c * ldu] = col[r];
  }
}

// reference src/gemm.cu:17-35 (gemmex -> cublasSgemm, alpha=-1, beta=1)
void orc_gemm_sub_f32(int64_t m, int64_t n, int64_t k, const float* a,
                      int64_t lda, const float* b, int64_t ldb, float* c,
                      int64_t ldc) {
  if (m <= 0 || n <= 0 || k <= 0) return;
  const int64_t IB = 512;
#pragma omp parallel
  {
    std::vector<float> acc(IB);
#pragma omp for schedule(dynamic, 4) collapse(2)
    for (int64_t j = 0; j < n; ++j)
      for (int64_t i0 = 0; i0 < m; i0 += IB) {
        const int64_t ie = std::min(m, i0 + IB);
        const int64_t len = ie - i0;
        float* acp = acc.data();
        for (int64_t i = 0; i < len; ++i) acp[i] = 0.0f;
        for (int64_t t = 0; t < k; ++t) {
          const float bt = b[t + j * ldb];
          const float* ap = a + i0 + t * lda;
          for (int64_t i = 0; i < len; ++i) acp[i] = std::fma(ap[i], bt, acp[i]);
        }
        float* cp = c + i0 + j * ldc;
        for (int64_t i = 0; i < len; ++i) cp[i] = cp[i] - acp[i];
      }
  }
}

namespace {

// reference src/lu_nopiv_inner_rl.hxx:104-196 (ib = 8); a points at the
// outer block's diagonal, m = remaining rows, n = outer block width, nb =
// nominal outer block size (column offset of the block row beyond it).
void inner_rl(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda) {
  const int64_t ib = 8;
  const int64_t inc = (n - 1) / ib + 1;
  float d[64];
  for (int64_t k = 0; k < inc; ++k) {
    const int64_t iofs = k * ib;
    const int64_t cblkm = m - iofs;
    const int64_t cblkn = std::min(n - iofs, ib);
    const int64_t iofst = (k + 1) * ib;
    const int64_t tblkm = m - iofst;
    const int64_t tblkn = n - iofst;
    for (int64_t c = 0; c < cblkn; ++c)
      for (int64_t r = 0; r < cblkn; ++r)
        d[r + c * 8] = at(a, lda, iofs + r, iofs + c);
    float* t = a + iofs + iofs * lda;
    orc_panel_f32(cblkm, cblkn, d, 8, t, lda, t, lda);
    if (tblkn > 0) {
      orc_gemm_sub_f32(tblkm, tblkn, ib, a + iofst + iofs * lda, lda,
                       a + iofs + iofst * lda, lda, a + iofst + iofst * lda,
                       lda);
      if (tblkm > tblkn)
        orc_gemm_sub_f32(tblkn, tblkm - tblkn, ib, a + iofst + iofs * lda, lda,
                         a + iofs + nb * lda, lda, a + iofst + nb * lda, lda);
    }
  }
}

// Copy a (rows x cols) block into `out` rounded to fmt, with one
// power-of-two scale per `tile` rows (by_rows) or per `tile` columns.
void round_copy(int64_t rows, int64_t cols, const float* a, int64_t lda,
                float* out, int64_t ldo, int fmt, bool by_rows, int64_t tile,
                std::vector<int>& scales) {
  const int64_t ntile = ((by_rows ? rows : cols) + tile - 1) / tile;
  scales.assign(ntile, 0);
  for (int64_t t = 0; t < ntile; ++t) {
    int64_t r0 = by_rows ? t * tile : 0, r1 = by_rows ? std::min(rows, r0 + tile) : rows;
    int64_t c0 = by_rows ? 0 : t * tile, c1 = by_rows ? cols : std::min(cols, c0 + tile);
    int s = 0;
    if (fmt == 3) {
      float amax = 0.0f;
      for (int64_t j = c0; j < c1; ++j)
        for (int64_t i = r0; i < r1; ++i)
          amax = std::max(amax, std::fabs(at(a, lda, i, j)));
      s = pow2_scale(amax, 448.0);
    }
    scales[t] = s;
    for (int64_t j = c0; j < c1; ++j)
      for (int64_t i = r0; i < r1; ++i)
        out[i + j * ldo] = orc_round_fmt(at(a, lda, i, j), fmt, s);
  }
}

// Split fp16 copies (hi and lo parts) with per-tile scales bound 32768.
void split_copy(int64_t rows, int64_t cols, const float* a, int64_t lda, float* hi,
                float* lo, int64_t ldo, bool by_rows, int64_t tile,
                std::vector<int>& scales) {
  const int64_t ntile = ((by_rows ? rows : cols) + tile - 1) / tile;
  scales.assign(ntile, 0);
  for (int64_t t = 0; t < ntile; ++t) {
    int64_t r0 = by_rows ? t * tile : 0, r1 = by_rows ? std::min(rows, r0 + tile) : rows;
    int64_t c0 = by_rows ? 0 : t * tile, c1 = by_rows ? cols : std::min(cols, c0 + tile);
    float amax = 0.0f;
    for (int64_t j = c0; j < c1; ++j)
      for (int64_t i = r0; i < r1; ++i) amax = std::max(amax, std::fabs(at(a, lda, i, j)));
    const int s = pow2_scale(amax, 32768.0);
    scales[t] = s;
    for (int64_t j = c0; j < c1; ++j)
      for (int64_t i = r0; i < r1; ++i) {
        const float x = std::ldexp(at(a, lda, i, j), s);
        const float h = round_fmt(x, 1);
        hi[i + j * ldo] = h;
        lo[i + j * ldo] = round_fmt(x - h, 1);
      }
  }
}

}  // namespace

// reference src/lu_nopiv.hxx:130-197
void orc_lu_rl_f32(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda,
                   int outer_fmt, int threads) {
  orc_lu_rl_f32_range(m, n, nb, a, lda, outer_fmt, threads, 0, -1);
}

void orc_lu_rl_f32_range(int64_t m, int64_t n, int64_t nb, float* a,
                         int64_t lda, int outer_fmt, int threads, int64_t kk0,
                         int64_t kk1) {
  const int saved = omp_get_max_threads();
  if (threads > 0) omp_set_num_threads(threads);
  const int64_t nc = (n - 1) / nb + 1;
  if (kk1 < 0 || kk1 > nc) kk1 = nc;
  std::vector<float> lc, uc;
  std::vector<int> ls, us;
  for (int64_t kk = kk0; kk < kk1; ++kk) {
    const int64_t ofs = kk * nb;
    const int64_t ofst = (kk + 1) * nb;
    const int64_t in = std::min(n - ofs, nb);
    const int64_t updm = m - ofs;
    inner_rl(updm, in, nb, a + ofs + ofs * lda, lda);
    const int64_t tm = m - ofst, tn = n - ofst;
    if (tn <= 0) continue;
    if (outer_fmt == 0) {
      orc_gemm_sub_f32(tm, tn, nb, a + ofst + ofs * lda, lda,
                       a + ofs + ofst * lda, lda, a + ofst + ofst * lda, lda);
    } else if (outer_fmt == 4) {
      // Split fp16 (new; no reference counterpart): per 128-row tile of L21
      // / 128-column tile of U12 a power-of-two scale bringing the tile max
      // under 32768, x * 2^s = hi + lo with hi = rn16(x * 2^s) and lo =
      // rn16(x * 2^s - hi); the product is taken over the concatenated K
      // segments [hi|hi|lo] x [hi;lo;hi] (all hi*hi terms, then hi*lo, then
      // lo*hi) accumulated in fp32, then the two scales are removed.
      const int64_t T = 128;
      std::vector<float> lh((size_t)tm * nb), ll((size_t)tm * nb);
      std::vector<float> uh((size_t)nb * tn), ul((size_t)nb * tn);
      split_copy(tm, nb, a + ofst + ofs * lda, lda, lh.data(), ll.data(), tm, true, T, ls);
      split_copy(nb, tn, a + ofs + ofst * lda, lda, uh.data(), ul.data(), nb, false, T, us);
#pragma omp parallel for schedule(dynamic, 4)
      for (int64_t j = 0; j < tn; ++j) {
        std::vector<float> acc(tm, 0.0f);
        const float* seg_a[3] = {lh.data(), lh.data(), ll.data()};
        const float* seg_b[3] = {uh.data(), ul.data(), uh.data()};
        for (int sg = 0; sg < 3; ++sg)
          for (int64_t t = 0; t < nb; ++t) {
            const float bt = seg_b[sg][t + j * nb];
            const float* ap = seg_a[sg] + t * tm;
            for (int64_t i = 0; i < tm; ++i) acc[i] = std::fma(ap[i], bt, acc[i]);
          }
        const int su = us[j / T];
        float* cp = a + ofst + (ofst + j) * lda;
        for (int64_t i = 0; i < tm; ++i)
          cp[i] = cp[i] - std::ldexp(acc[i], -(ls[i / T] + su));
      }
    } else {
      // TC32 with W = fp32 (src/lu_nopiv.hxx:155-183): the update multiplies
      // low-precision copies of L21 and U12 with fp32 accumulation.  For e4m3
      // each 128-row tile of L21 / 128-column tile of U12 carries a
      // power-of-two scale that the product removes again.
      const int64_t T = 128;
      lc.resize((size_t)tm * nb);
      uc.resize((size_t)nb * tn);
      round_copy(tm, nb, a + ofst + ofs * lda, lda, lc.data(), tm, outer_fmt,
                 true, T, ls);
      round_copy(nb, tn, a + ofs + ofst * lda, lda, uc.data(), nb, outer_fmt,
                 false, T, us);
#pragma omp parallel for schedule(dynamic, 4)
      for (int64_t j = 0; j < tn; ++j) {
        std::vector<float> acc(tm, 0.0f);
        for (int64_t t = 0; t < nb; ++t) {
          const float bt = uc[t + j * nb];
          const float* ap = lc.data() + t * tm;
          for (int64_t i = 0; i < tm; ++i) acc[i] = std::fma(ap[i], bt, acc[i]);
        }
        const int su = us[j / T];
        float* cp = a + ofst + (ofst + j) * lda;
        for (int64_t i = 0; i < tm; ++i)
          cp[i] = cp[i] - std::ldexp(acc[i], -(ls[i / T] + su));
      }
    }
  }
  omp_set_num_threads(saved);
}

// reference src/lu_nopiv_inner_ll.hxx:197-370 (T = P = F = float, ib = 8):
// m rows, n = outer block width; l and u point at the outer block's
// diagonal (the same matrix for W = fp32).
static void inner_ll(int64_t m, int64_t n, float* a, int64_t lda) {
  const int64_t ib = 8;
  const int64_t inc = (n - 1) / ib + 1;
  float d[64];
  for (int64_t k = 0; k < inc; ++k) {
    const int64_t iofs = k * ib;
    const int64_t cblkm = m - iofs;
    const int64_t cblkn = std::min(n - iofs, ib);
    const int64_t iofst = (k + 1) * ib;
    if (iofs > 0) {
      // L inner panel (src/lu_nopiv_inner_ll.hxx:225-246)
      orc_gemm_sub_f32(cblkm, cblkn, iofs, a + iofs, lda, a + iofs * lda, lda,
                       a + iofs + iofs * lda, lda);
      // U inner panel (src/lu_nopiv_inner_ll.hxx:249-300)
      if (cblkm > cblkn)
        orc_gemm_sub_f32(cblkn, cblkm - cblkn, iofs, a + iofs, lda,
                         a + iofst * lda, lda, a + iofs + iofst * lda, lda);
    }
    for (int64_t c = 0; c < cblkn; ++c)
      for (int64_t r = 0; r < cblkn; ++r) d[r + c * 8] = at(a, lda, iofs + r, iofs + c);
    float* t = a + iofs + iofs * lda;
    orc_panel_f32(cblkm, cblkn, d, 8, t, lda, t, lda);
  }
}

// The product library's inside of a left-looking outer block wider than
// its one-CTA Crout kernel (sub columns): sub-block c first receives the
// K = c update from the block's own earlier columns (column below, row to
// the right), then inner_ll.  For n <= sub this is inner_ll itself.
static void inner_ll_blocked(int64_t m, int64_t n, float* a, int64_t lda, int64_t sub) {
  for (int64_t c = 0; c < n; c += sub) {
    const int64_t w = std::min(sub, n - c);
    if (c > 0) {
      orc_gemm_sub_f32(m - c, w, c, a + c, lda, a + c * lda, lda, a + c + c * lda, lda);
      if (m - c > w)
        orc_gemm_sub_f32(w, m - c - w, c, a + c, lda, a + (c + w) * lda, lda,
                         a + c + (c + w) * lda, lda);
    }
    inner_ll(m - c, w, a + c + c * lda, lda);
  }
}

// reference src/lu_nopiv_ll.hxx:208-575 for W = OP = OF = float, I = O = FP32
// (the lu_nopiv_ll_f32 wrapper, src/lu_nopiv_ll.cxx:14-29); outer blocks
// wider than `sub` factored as inner_ll_blocked
void orc_lu_ll_f32_sub(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda,
                       int threads, int64_t sub) {
  const int saved = omp_get_max_threads();
  if (threads > 0) omp_set_num_threads(threads);
  const int64_t nc = (n - 1) / nb + 1;
  for (int64_t kk = 0; kk < nc; ++kk) {
    const int64_t ofs = kk * nb;
    const int64_t in = std::min(n - ofs, nb);
    const int64_t updm = m - ofs;
    if (ofs > 0) {
      orc_gemm_sub_f32(updm, in, ofs, a + ofs, lda, a + ofs * lda, lda,
                       a + ofs + ofs * lda, lda);
      if (updm > in)
        orc_gemm_sub_f32(in, updm - in, ofs, a + ofs, lda, a + (ofs + in) * lda,
                         lda, a + ofs + (ofs + in) * lda, lda);
    }
    inner_ll_blocked(updm, in, a + ofs + ofs * lda, lda, sub);
  }
  omp_set_num_threads(saved);
}

// reference src/lu_nopiv_ll.hxx:208-575 for W = OP = OF = float, I = O = FP32
// (the lu_nopiv_ll_f32 wrapper, src/lu_nopiv_ll.cxx:14-29)
void orc_lu_ll_f32(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda,
                   int threads) {
  const int saved = omp_get_max_threads();
  if (threads > 0) omp_set_num_threads(threads);
  const int64_t nc = (n - 1) / nb + 1;
  for (int64_t kk = 0; kk < nc; ++kk) {
    const int64_t ofs = kk * nb;
    const int64_t in = std::min(n - ofs, nb);
    const int64_t updm = m - ofs;
    if (ofs > 0) {
      // block column (src/lu_nopiv_ll.hxx:239-250) and block row (:311-339)
      orc_gemm_sub_f32(updm, in, ofs, a + ofs, lda, a + ofs * lda, lda,
                       a + ofs + ofs * lda, lda);
      if (updm > in)
        orc_gemm_sub_f32(in, updm - in, ofs, a + ofs, lda, a + (ofs + in) * lda,
                         lda, a + ofs + (ofs + in) * lda, lda);
    }
    inner_ll(updm, in, a + ofs + ofs * lda, lda);
  }
  omp_set_num_threads(saved);
}

// Left-looking factorization of an fp16 matrix (values held in fp32, every
// one fp16-representable): reference src/lu_nopiv_ll.hxx:208-575 with
// W = fp16, O = TC32 -- the K = ofs products of fp16 values accumulated in
// fp32 and the updated block column / row rounded to fp16 once -- and the
// inner Crout elimination in fp32 with its results rounded to fp16 (the
// product library's fp16 variant; the reference's fp16 wrappers factor the
// panel in fp16 arithmetic instead).
// panel_fp32 = 1 (the reference's OP = OF = fp32 wrappers,
// src/lu_nopiv_ll.hxx:172-201): the updated block column / row is not
// rounded to fp16 before its elimination.  Outer blocks wider than `sub` are
// factored as inner_ll_blocked.
void orc_lu_ll_f16_ex(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda,
                      int threads, int64_t sub, int panel_fp32) {
  const int saved = omp_get_max_threads();
  if (threads > 0) omp_set_num_threads(threads);
  auto round_block = [&](int64_t rows, int64_t cols, float* p) {
    for (int64_t j = 0; j < cols; ++j)
      for (int64_t i = 0; i < rows; ++i) p[i + j * lda] = round_fmt(p[i + j * lda], 1);
  };
  const int64_t nc = (n - 1) / nb + 1;
  for (int64_t kk = 0; kk < nc; ++kk) {
    const int64_t ofs = kk * nb;
    const int64_t in = std::min(n - ofs, nb);
    const int64_t updm = m - ofs;
    float* blk = a + ofs + ofs * lda;
    if (ofs > 0) {
      orc_gemm_sub_f32(updm, in, ofs, a + ofs, lda, a + ofs * lda, lda, blk, lda);
      if (!panel_fp32) round_block(updm, in, blk);
      if (updm > in) {
        orc_gemm_sub_f32(in, updm - in, ofs, a + ofs, lda, a + (ofs + in) * lda, lda,
                         blk + in * lda, lda);
        if (!panel_fp32) round_block(in, updm - in, blk + in * lda);
      }
    }
    inner_ll_blocked(updm, in, blk, lda, sub);
    round_block(updm, in, blk);
    if (updm > in) round_block(in, updm - in, blk + in * lda);
  }
  omp_set_num_threads(saved);
}

void orc_lu_ll_f16(int64_t m, int64_t n, int64_t nb, float* a, int64_t lda,
                   int threads) {
  const int saved = omp_get_max_threads();
  if (threads > 0) omp_set_num_threads(threads);
  auto round_block = [&](int64_t rows, int64_t cols, float* p) {
    for (int64_t j = 0; j < cols; ++j)
      for (int64_t i = 0; i < rows; ++i) p[i + j * lda] = round_fmt(p[i + j * lda], 1);
  };
  const int64_t nc = (n - 1) / nb + 1;
  for (int64_t kk = 0; kk < nc; ++kk) {
    const int64_t ofs = kk * nb;
    const int64_t in = std::min(n - ofs, nb);
    const int64_t updm = m - ofs;
    float* blk = a + ofs + ofs * lda;
    if (ofs > 0) {
      orc_gemm_sub_f32(updm, in, ofs, a + ofs, lda, a + ofs * lda, lda, blk, lda);
      round_block(updm, in, blk);
      if (updm > in) {
        orc_gemm_sub_f32(in, updm - in, ofs, a + ofs, lda, a + (ofs + in) * lda, lda,
                         blk + in * lda, lda);
        round_block(in, updm - in, blk + in * lda);
      }
    }
    inner_ll(updm, in, blk, lda);
    round_block(updm, in, blk);
    if (updm > in) round_block(in, updm - in, blk + in * lda);
  }
  omp_set_num_threads(saved);
}

// ---------------------------------------------------------------- FP64

void orc_lu_f64(int64_t n, double* a, int64_t lda) {
  const int64_t nb = 64;
  for (int64_t k0 = 0; k0 < n; k0 += nb) {
    const int64_t k1 = std::min(n, k0 + nb);
    // unblocked on the panel columns k0..k1, rows k0..n
    for (int64_t k = k0; k < k1; ++k) {
      const double piv = a[k + k * lda];
      for (int64_t i = k + 1; i < n; ++i) a[i + k * lda] /= piv;
      for (int64_t j = k + 1; j < k1; ++j) {
        const double ukj = a[k + j * lda];
        for (int64_t i = k + 1; i < n; ++i) a[i + j * lda] -= a[i + k * lda] * ukj;
      }
    }
    // U12 = L11^-1 A12
#pragma omp parallel for schedule(static)
    for (int64_t j = k1; j < n; ++j)
      for (int64_t k = k0; k < k1; ++k) {
        const double ukj = a[k + j * lda];
        for (int64_t i = k + 1; i < k1; ++i) a[i + j * lda] -= a[i + k * lda] * ukj;
      }
    // A22 -= L21 U12
#pragma omp parallel for schedule(static)
    for (int64_t j = k1; j < n; ++j)
      for (int64_t k = k0; k < k1; ++k) {
        const double ukj = a[k + j * lda];
        for (int64_t i = k1; i < n; ++i) a[i + j * lda] -= a[i + k * lda] * ukj;
      }
  }
}

void orc_lu_solve_f64(int64_t n, const double* lu, int64_t ld, double* b) {
  for (int64_t j = 0; j < n; ++j) {
    const double bj = b[j];
    for (int64_t i = j + 1; i < n; ++i) b[i] -= lu[i + j * ld] * bj;
  }
  for (int64_t j = n - 1; j >= 0; --j) {
    b[j] /= lu[j + j * ld];
    const double bj = b[j];
    for (int64_t i = 0; i < j; ++i) b[i] -= lu[i + j * ld] * bj;
  }
}

void orc_lu_solve_f32f64(int64_t n, const float* lu, int64_t ld, double* b) {
  for (int64_t j = 0; j < n; ++j) {
    const double bj = b[j];
    for (int64_t i = j + 1; i < n; ++i) b[i] -= (double)lu[i + j * ld] * bj;
  }
  for (int64_t j = n - 1; j >= 0; --j) {
    b[j] /= (double)lu[j + j * ld];
    const double bj = b[j];
    for (int64_t i = 0; i < j; ++i) b[i] -= (double)lu[i + j * ld] * bj;
  }
}

// reference tests/testing_lu_gpu.hxx:1309-1313 (host getrs with ipiv = 1..m,
// in the working precision)
void orc_lu_solve_f32(int64_t n, const float* lu, int64_t ld, float* b) {
  for (int64_t j = 0; j < n; ++j) {
    const float bj = b[j];
    for (int64_t i = j + 1; i < n; ++i) b[i] = std::fma(-lu[i + j * ld], bj, b[i]);
  }
  for (int64_t j = n - 1; j >= 0; --j) {
    b[j] = b[j] / lu[j + j * ld];
    const float bj = b[j];
    for (int64_t i = 0; i < j; ++i) b[i] = std::fma(-lu[i + j * ld], bj, b[i]);
  }
}

// ---------------------------------------------------------------- errors

// reference tests/errors.hxx:187-249 (unsym_backward_error, "nwerr")
double orc_nwerr_f32(int64_t m, const float* a, int64_t lda, const float* b,
                     const float* x) {
  double anorm = 0.0;
  for (int64_t j = 0; j < m; ++j) {
    double s = 0.0;
    for (int64_t i = 0; i < m; ++i) s += std::fabs((double)at(a, lda, i, j));
    anorm = std::max(anorm, s);
  }
  std::vector<double> r(m);
  for (int64_t i = 0; i < m; ++i) r[i] = (double)b[i];
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = 0; i < m; ++i) r[i] -= (double)at(a, lda, i, j) * (double)x[j];
  double rn = 0.0, bn = 0.0, xn = 0.0;
  bool nan = false;
  for (int64_t i = 0; i < m; ++i) {
    rn = std::max(rn, std::fabs(r[i]));
    bn = std::max(bn, std::fabs((double)b[i]));
    xn = std::max(xn, std::fabs((double)x[i]));
    if (std::isnan(r[i])) nan = true;
  }
  if (nan) return NAN;
  return rn / (anorm * xn + bn);
}

// reference tests/errors.hxx:23-182 (unsym_compwise_error, "cwerr")
double orc_cwerr_f32(int64_t m, const float* a, int64_t lda, const float* b,
                     const float* x, const float* lu, int64_t ldlu) {
  std::vector<double> r(m), ax(m, 0.0), ux(m, 0.0), lux(m, 0.0), xa(m);
  for (int64_t i = 0; i < m; ++i) {
    r[i] = (double)b[i];
    xa[i] = std::fabs((double)x[i]);
  }
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = 0; i < m; ++i) {
      const double aij = (double)at(a, lda, i, j);
      r[i] -= aij * (double)x[j];
      ax[i] += std::fabs(aij) * xa[j];
    }
  // |U||x|
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = 0; i <= j; ++i) ux[i] += std::fabs((double)lu[i + j * ldlu]) * xa[j];
  // |L|(|U||x|), unit diagonal
  for (int64_t i = 0; i < m; ++i) lux[i] = ux[i];
  for (int64_t j = 0; j < m; ++j)
    for (int64_t i = j + 1; i < m; ++i) lux[i] += std::fabs((double)lu[i + j * ldlu]) * ux[j];
  double cw = 0.0;
  for (int64_t i = 0; i < m; ++i) {
    double ri = std::fabs(r[i]);
    double den = ax[i] + lux[i];
    if (den > 0.0) ri = ri / den;
    cw = std::max(cw, ri);
  }
  return cw;
}

double orc_factor_error_f32(int64_t n, const float* a, int64_t lda,
                            const float* lu, int64_t ldlu) {
  double num = 0.0, den = 0.0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : num, den)
  for (int64_t j = 0; j < n; ++j) {
    std::vector<double> col(n, 0.0);
    // (L U)(:, j) = sum_{k <= j} L(:, k) U(k, j)
    for (int64_t k = 0; k <= j; ++k) {
      const double ukj = (double)lu[k + j * ldlu];
      col[k] += ukj;  // unit diagonal of L
      for (int64_t i = k + 1; i < n; ++i) col[i] += (double)lu[i + k * ldlu] * ukj;
    }
    for (int64_t i = 0; i < n; ++i) {
      const double aij = (double)at(a, lda, i, j);
      num += (aij - col[i]) * (aij - col[i]);
      den += aij * aij;
    }
  }
  return std::sqrt(num / den);
}

double orc_backward_error_f64(int64_t n, const float* a, int64_t lda,
                              const double* b, const double* x) {
  std::vector<double> r(b, b + n), rows(n, 0.0);
  for (int64_t j = 0; j < n; ++j)
    for (int64_t i = 0; i < n; ++i) {
      const double aij = (double)at(a, lda, i, j);
      r[i] -= aij * x[j];
      rows[i] += std::fabs(aij);
    }
  double rn = 0.0, an = 0.0, xn = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    rn = std::max(rn, std::fabs(r[i]));
    an = std::max(an, rows[i]);
    xn = std::max(xn, std::fabs(x[i]));
  }
  return rn / (an * xn);
}

}  // extern "C"
