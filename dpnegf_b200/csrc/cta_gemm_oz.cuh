// CTA-wide complex GEMM on the int8 tensor cores (tcgen05.mma, kind::i8)
// with exact integer slice products: FP64-class complex products from the
// int8 pipe (the Ozaki scheme).
//
//   acc = op(A) * op(B),   epi(m, n, acc) for every in-range element
//
// Same operands (complex128 in global memory), operand transforms, GemmArgs
// and epilogue functors as the FP64 tile GEMM (cta_gemm.cuh) and the 3xTF32
// GEMM (cta_gemm_tc.cuh).
//
// Method (error-free splitting of Ozaki, Ogita, Oishi and Rump, Numer.
// Algorithms 59 (2012) 95-118, in the integer form of Ootomo, Ozaki and
// Yokota, Int. J. High Perform. Comput. Appl. 38 (2024)).  Row m of op(A) gets
// the exponent ea_m with max_k |op(A)_mk| < 2^ea_m (maximum over real and
// imaginary parts), column n of op(B) the exponent eb_n.  A real entry x of
// row m is cut into S int8 digits,
//   x = 2^ea_m sum_{i<S} a_i 2^-7(i+1) + r,   |r| < 2^(ea_m - 7S),
// the base-128 digits of the two's-complement integer Y = trunc(x 2^(7S - ea_m))
// (|Y| < 2^7S): a_0 = Y >> 7(S-1) in [-128, 127] carries the sign and the
// others are the unsigned 7-bit fields in [0, 127].  Digit planes
// multiply exactly in int32, and the pairs with i + j = l share one accumulator
// acc_l (l < S; the pairs with i + j >= S are dropped), so
//   C_mn = 2^(ea_m + eb_n - 14) sum_{l<S} 2^-7l acc_l,
// accurate to about 2 K S 2^-7S 2^(ea_m + eb_n) (a normwise bound: the error
// is relative to the largest entries of the row and the column).  S = 8
// (56-bit digits) matches FP64 products; S = 6 gives about 42 bits.
//
// Complex products without a negate: with A' = [Ar | Ai] (M x 2K) and
// B' = [[Br, Bi], [-Bi, Br]] (2K x 2N), A' B' = [Cr | Ci], one real product of
// doubled K.  Real and imaginary parts of a row (or column) share its exponent.
// Bound on one accumulator: S pairs x 2K x 128^2 < 2^31 for K <= 1024.
//
// Tiles.  One CTA (8 warps) walks tiles of 128 complex rows x 32 complex
// columns; the MMA is M = 128, N = 64 (the re and im halves of the 32
// columns), K = 32 int8 = one slab of 16 complex k.  The S level accumulators
// take 64 int32 columns each of the CTA's 512 tensor-memory columns (S <= 8).
// Before the first slab the CTA makes one pass over op(A) and op(B) for the
// exponents.  Raw FP64 slabs are copied into shared memory with cp.async two
// slabs ahead; the CTA cuts the current slab into S digit planes per operand
// in the canonical K-major no-swizzle layout ([k/16][row][16 bytes]: core
// matrices of 8 rows x 16 bytes, leading-byte offset = rows x 16 B,
// stride-byte offset = 128 B), and thread 0 issues the slab's S(S+1)/2 MMAs
// and commits them to the plane stage's mbarrier.  A plane stage is rewritten
// only after its mbarrier reports the MMAs that read it complete.  Every
// mbarrier wait is bounded (tc_err, as in the 3xTF32 GEMM).
//
// Non-finite inputs: a row or column holding Inf or NaN gets the exponent
// OZ_BAD, its digits are zero and its outputs are NaN, so an item's
// non-finite status still surfaces.
#pragma once
#include "cta_gemm_tc.cuh"

namespace negf {

constexpr int OZ_M = 128, OZ_NC = 32, OZ_N = 2 * OZ_NC, OZ_KC = 16;
constexpr int OZ_MAXMN = 512;                      // largest M and N (NEGF_MAX_BLOCK)
constexpr int OZ_PLANE_A = OZ_M * 32;              // bytes of one A digit plane (128 rows x 32 int8)
constexpr int OZ_PLANE_B = OZ_N * 32;              // bytes of one B digit plane (64 rows x 32 int8)
constexpr int OZ_PITCH = OZ_KC + 1;                // complex pitch of raw slabs stored with k innermost
constexpr int OZ_RAW_A = OZ_M * OZ_PITCH * 16;     // raw A slab (either orientation fits)
constexpr int OZ_RAW_B = OZ_NC * OZ_PITCH * 16;    // raw B slab
constexpr int OZ_RAW_BYTES = OZ_RAW_A + OZ_RAW_B;
constexpr int OZ_EPI_PITCH = 17;                   // complex entries per transposed row (epilogue)
constexpr int OZ_EPI_BYTES = 8 * 32 * OZ_EPI_PITCH * 16;
constexpr int OZ_BAD = 1 << 20;                    // exponent marking a non-finite row / column
constexpr int OZ_EMIN = -960;                      // exponents are clamped here (2^(7S - e) stays normal)

template <int S>
struct OzLayout {
  static_assert(S >= 2 && S <= 8, "S digit planes, 2..8 (S accumulators of 64 columns in 512)");
  static constexpr int PLANES = S * (OZ_PLANE_A + OZ_PLANE_B);
  // a stage also hosts half of the epilogue's transpose buffers
  static constexpr int STAGE = PLANES > OZ_EPI_BYTES / 2 ? PLANES : OZ_EPI_BYTES / 2;
  static constexpr int RAW_OFF = 2 * STAGE;
  static constexpr int EXP_OFF = RAW_OFF + 2 * OZ_RAW_BYTES;
  static constexpr int SMEM = EXP_OFF + 2 * OZ_MAXMN * 4;
  static constexpr int MMAS = S * (S + 1) / 2;
};
static_assert(OZ_RAW_A % 16 == 0 && OZ_RAW_B % 16 == 0, "raw slabs keep 16-byte alignment");

NEGF_DEV void tc_mma_i8(uint32_t d_tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

// 16 consecutive int32 accumulator columns of this warp's 32 lanes.
NEGF_DEV void tc_ld16i(uint32_t taddr, int* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = static_cast<int>(r[j]);
}

// Exponent e with max < 2^e; OZ_BAD for a non-finite maximum.
NEGF_DEV int oz_exponent(double mx) {
  if (!(mx <= 1.7976931348623157e308)) return OZ_BAD;  // Inf or NaN
  if (mx == 0.0) return OZ_EMIN;
  int e;
  frexp(mx, &e);  // mx = f 2^e, f in [0.5, 1)
  return e < OZ_EMIN ? OZ_EMIN : e;
}

NEGF_DEV double cmax_abs(cplx v) { return fmax(fabs(v.x), fabs(v.y)); }

// Row exponents of op(A) (ea[0..M)) and column exponents of op(B) (eb[0..N));
// entries up to OZ_MAXMN beyond M / N are set to OZ_EMIN.  Whole CTA; ends
// with __syncthreads().
template <int OPA, int OPB>
NEGF_DEV void oz_exponents(const GemmArgs& g, int* ea, int* eb) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (OPA == OP_C) {  // stored K x M: one column of storage per thread, coalesced over m
    for (int m = tid; m < g.M; m += CTA_THREADS) {
      double mx = 0.0;
#pragma unroll 4
      for (int k = 0; k < g.K; ++k) mx = fmax(mx, cmax_abs(g.A[(int64_t)k * g.lda + m]));
      ea[m] = oz_exponent(mx);
    }
  } else {  // stored M x K: one warp per row
    for (int m = warp; m < g.M; m += CTA_THREADS / 32) {
      double mx = 0.0;
      for (int k = lane; k < g.K; k += 32) mx = fmax(mx, cmax_abs(g.A[(int64_t)m * g.lda + k]));
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
      if (lane == 0) ea[m] = oz_exponent(mx);
    }
  }
  if (OPB == OP_C) {  // stored N x K: one warp per column of op(B)
    for (int n = warp; n < g.N; n += CTA_THREADS / 32) {
      double mx = 0.0;
      for (int k = lane; k < g.K; k += 32) mx = fmax(mx, cmax_abs(g.B[(int64_t)n * g.ldb + k]));
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
      if (lane == 0) eb[n] = oz_exponent(mx);
    }
  } else {  // stored K x N: coalesced over n
    for (int n = tid; n < g.N; n += CTA_THREADS) {
      double mx = 0.0;
#pragma unroll 4
      for (int k = 0; k < g.K; ++k) mx = fmax(mx, cmax_abs(g.B[(int64_t)k * g.ldb + n]));
      eb[n] = oz_exponent(mx);
    }
  }
  for (int m = g.M + tid; m < OZ_MAXMN; m += CTA_THREADS) ea[m] = OZ_EMIN;
  for (int n = g.N + tid; n < OZ_MAXMN; n += CTA_THREADS) eb[n] = OZ_EMIN;
  __syncthreads();
}

// 2^(7S - e) for a clamped exponent (a normal double), 0 for OZ_BAD.
template <int S>
NEGF_DEV double oz_factor(int e) {
  if (e == OZ_BAD) return 0.0;
  return __longlong_as_double((long long)(1023 + 7 * S - e) << 52);
}

// Bits sh..sh+31 of the 64-bit two's-complement value (hi:lo).
template <int SH>
NEGF_DEV uint32_t oz_window(uint32_t lo, uint32_t hi) {
  if constexpr (SH < 32) return __funnelshift_r(lo, hi, SH);
  else return hi >> (SH - 32);
}

// Digit I (most significant first) of four values Y_j = (hi_j:lo_j), packed
// as four int8 in one word: the low byte of Y >> 7(S-1-I), masked to 7 bits
// below the top digit.
template <int S, int I>
NEGF_DEV uint32_t oz_digit4(const uint32_t* lo, const uint32_t* hi) {
  constexpr int SH = 7 * (S - 1 - I);
  const uint32_t w01 = __byte_perm(oz_window<SH>(lo[0], hi[0]), oz_window<SH>(lo[1], hi[1]), 0x0040);
  const uint32_t w23 = __byte_perm(oz_window<SH>(lo[2], hi[2]), oz_window<SH>(lo[3], hi[3]), 0x0040);
  const uint32_t w = __byte_perm(w01, w23, 0x5410);
  return I == 0 ? w : (w & 0x7F7F7F7Fu);
}

// Y = trunc(x f) split into 32-bit halves.
NEGF_DEV void oz_int(double x, double f, uint32_t& lo, uint32_t& hi) {
  const long long y = (long long)(x * f);
  lo = static_cast<uint32_t>(y);
  hi = static_cast<uint32_t>(y >> 32);
}

template <int S, int I = 0>
NEGF_DEV void oz_store_a(char* dst, const uint32_t* lo, const uint32_t* hi) {
  if constexpr (I < S) {
    uint4 w;
    w.x = oz_digit4<S, I>(lo + 0, hi + 0);
    w.y = oz_digit4<S, I>(lo + 4, hi + 4);
    w.z = oz_digit4<S, I>(lo + 8, hi + 8);
    w.w = oz_digit4<S, I>(lo + 12, hi + 12);
    *reinterpret_cast<uint4*>(dst + I * OZ_PLANE_A) = w;
    oz_store_a<S, I + 1>(dst, lo, hi);
  }
}

template <int S, int I = 0>
NEGF_DEV void oz_store_b(char* dst, int off, const uint32_t* lo, const uint32_t* hi) {
  if constexpr (I < S) {
    *reinterpret_cast<uint32_t*>(dst + I * OZ_PLANE_B + off) = oz_digit4<S, I>(lo, hi);
    oz_store_b<S, I + 1>(dst, off, lo, hi);
  }
}

// Raw slab staging (cp.async, zero fill outside the matrix), keeping the
// operand's contiguous dimension innermost so the copies coalesce:
//   op(A) N/K: raw [128 m][16 k] (pitch 17)    op(A) C: raw [16 k][128 m]
//   op(B) N/K: raw [16 k][32 n]                op(B) C: raw [32 n][16 k] (pitch 17)
template <int OPA>
NEGF_DEV void oz_fetch_a(cplx* raw, const GemmArgs& g, int m0, int k0, int tid) {
#pragma unroll
  for (int i = 0; i < (OZ_M * OZ_KC) / CTA_THREADS; ++i) {
    const int e = tid + CTA_THREADS * i;
    if (OPA == OP_C) {
      const int k = e >> 7, m = e & 127, kg = k0 + k, mg = m0 + m;
      const bool v = kg < g.K && mg < g.M;
      cp_async16(raw + e, v ? g.A + (int64_t)kg * g.lda + mg : g.A, v);
    } else {
      const int m = e >> 4, k = e & 15, kg = k0 + k, mg = m0 + m;
      const bool v = kg < g.K && mg < g.M;
      cp_async16(raw + m * OZ_PITCH + k, v ? g.A + (int64_t)mg * g.lda + kg : g.A, v);
    }
  }
}

template <int OPB>
NEGF_DEV void oz_fetch_b(cplx* raw, const GemmArgs& g, int k0, int n0, int tid) {
#pragma unroll
  for (int i = 0; i < (OZ_NC * OZ_KC) / CTA_THREADS; ++i) {
    const int e = tid + CTA_THREADS * i;
    if (OPB == OP_C) {
      const int n = e >> 4, k = e & 15, kg = k0 + k, ng = n0 + n;
      const bool v = kg < g.K && ng < g.N;
      cp_async16(raw + n * OZ_PITCH + k, v ? g.B + (int64_t)ng * g.ldb + kg : g.B, v);
    } else {
      const int k = e >> 5, n = e & 31, kg = k0 + k, ng = n0 + n;
      const bool v = kg < g.K && ng < g.N;
      cp_async16(raw + e, v ? g.B + (int64_t)kg * g.ldb + ng : g.B, v);
    }
  }
}

// Cut the raw slabs of one stage into the S digit planes of A' and B'.
//   A plane i: [kgroup (0 re, 1 im)][128 rows][16 bytes]
//   B plane j: [kgroup][64 rows][16 bytes]; rows 0..31 are the re-half
//   columns ([Br | -Bi] along K'), rows 32..63 the im-half ([Bi | Br]).
template <int S, int OPA, int OPB>
NEGF_DEV void oz_slice(char* pl, const cplx* rawA, const cplx* rawB, const int* ea, const int* eb, int tid) {
  constexpr bool CA = OPA != OP_N, CB = OPB != OP_N;
  {  // A: one (row, part) per thread, 16 values
    const int r = tid >> 1, part = tid & 1;
    const double f = oz_factor<S>(ea[r]);
    uint32_t lo[16], hi[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const cplx v = OPA == OP_C ? rawA[c * OZ_M + r] : rawA[r * OZ_PITCH + c];
      oz_int(part ? (CA ? -v.y : v.y) : v.x, f, lo[c], hi[c]);
    }
    oz_store_a<S>(pl + part * (OZ_M * 16) + r * 16, lo, hi);
  }
  {  // B: one (column, part, k quarter) per thread, 4 values
    const int n = tid & 31, part = (tid >> 5) & 1, kq = tid >> 6;
    const double f = oz_factor<S>(eb[n]);
    uint32_t lo[4], hi[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = kq * 4 + j;
      const cplx v = OPB == OP_C ? rawB[n * OZ_PITCH + k] : rawB[k * OZ_NC + n];
      oz_int(part ? (CB ? -v.y : v.y) : v.x, f, lo[j], hi[j]);
    }
    char* bp = pl + S * OZ_PLANE_A + kq * 4;
    // re part: row n kgroup 0 and row 32+n kgroup 1 take d(Br);
    // im part: row 32+n kgroup 0 takes d(Bi), row n kgroup 1 takes d(-Bi)
    if (part == 0) {
      oz_store_b<S>(bp, n * 16, lo, hi);
      oz_store_b<S>(bp, (OZ_NC + n) * 16 + OZ_N * 16, lo, hi);
    } else {
      oz_store_b<S>(bp, (OZ_NC + n) * 16, lo, hi);
#pragma unroll
      for (int j = 0; j < 4; ++j) {  // -Y in two's complement
        const unsigned long long y = ~((unsigned long long)hi[j] << 32 | lo[j]) + 1ull;
        lo[j] = static_cast<uint32_t>(y);
        hi[j] = static_cast<uint32_t>(y >> 32);
      }
      oz_store_b<S>(bp, n * 16 + OZ_N * 16, lo, hi);
    }
  }
}

// The S(S+1)/2 MMAs of one slab (thread 0): acc_l += A_i B_j for i + j = l.
// first: the slab starts a tile.
template <int S>
NEGF_DEV void oz_issue_slab(const char* pl, uint32_t tmem, bool first) {
  const uint32_t a0 = smem_addr(pl), b0 = smem_addr(pl + S * OZ_PLANE_A);
  const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OZ_N >> 3) << 17) |
                         ((uint32_t)(OZ_M >> 4) << 24);  // S32 += S8 x S8, K-major, M 128, N 64
#pragma unroll
  for (int l = 0; l < S; ++l) {
#pragma unroll
    for (int i = 0; i <= l; ++i) {
      const uint64_t da = tc_desc(a0 + i * OZ_PLANE_A, OZ_M * 16, 128);
      const uint64_t db = tc_desc(b0 + (l - i) * OZ_PLANE_B, OZ_N * 16, 128);
      tc_mma_i8(tmem + l * OZ_N, da, db, idesc, (first && i == 0) ? 0u : 1u);
    }
  }
}

// acc = op(A) op(B) over the whole M x N output (M, N <= 512); epi(m, n, acc)
// once per in-range element.  The output must not alias A or B.  Ends with
// __syncthreads().  Requires tc_tmem_alloc() earlier in the kernel.
template <int S, int OPA, int OPB, class Epi>
__device__ __noinline__ void cta_gemm_oz_epi(const GemmArgs g, char* smem, const Epi epi) {
  typedef OzLayout<S> LY;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nk = (g.K + OZ_KC - 1) / OZ_KC;
  const int tiles_n = (g.N + OZ_NC - 1) / OZ_NC, tiles = ((g.M + OZ_M - 1) / OZ_M) * tiles_n;
  if (nk == 0) {  // empty sum
    for (int e = tid; e < g.M * g.N; e += CTA_THREADS) epi(e / g.N, e % g.N, cmk(0.0, 0.0));
    __syncthreads();
    return;
  }
  if (g.M > OZ_MAXMN || g.N > OZ_MAXMN) {  // outside the exponent tables: report, touch nothing
    if (tid == 0) tc_err = 1;
    __syncthreads();
    return;
  }
  int* ea = reinterpret_cast<int*>(smem + LY::EXP_OFF);
  int* eb = ea + OZ_MAXMN;
  oz_exponents<OPA, OPB>(g, ea, eb);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(&tc_bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(&tc_bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  __syncthreads();
  const uint32_t bar[2] = {smem_addr(&tc_bar[0]), smem_addr(&tc_bar[1])};
  uint32_t uses[2] = {0u, 0u}, seen[2] = {0u, 0u};
  const uint32_t tmem = tc_tmem;
  bool ok = tc_err == 0;
  const int NS = tiles * nk;
  auto plane = [&](int b) { return smem + b * LY::STAGE; };
  auto rawA = [&](int b) { return reinterpret_cast<cplx*>(smem + LY::RAW_OFF + b * OZ_RAW_BYTES); };
  auto rawB = [&](int b) { return reinterpret_cast<cplx*>(smem + LY::RAW_OFF + b * OZ_RAW_BYTES + OZ_RAW_A); };
  auto tile_of = [&](int t, int& m0, int& n0) {
    m0 = (t / tiles_n) * OZ_M;
    n0 = (t % tiles_n) * OZ_NC;
  };
  auto fetch = [&](int s) {
    if (s < NS) {
      int m0, n0;
      tile_of(s / nk, m0, n0);
      const int k0 = (s % nk) * OZ_KC;
      oz_fetch_a<OPA>(rawA(s & 1), g, m0, k0, tid);
      oz_fetch_b<OPB>(rawB(s & 1), g, k0, n0, tid);
    }
    cp_async_commit();
  };
  auto drain = [&](int b) {
    if (seen[b] < uses[b]) {
      if (ok && !tc_bar_wait(bar[b], (uses[b] - 1u) & 1u)) ok = false;
      seen[b] = uses[b];
    }
  };

  fetch(0);
  fetch(1);
  for (int s = 0; s < NS; ++s) {
    const int b = s & 1, kc = s % nk;
    int m0, n0;
    tile_of(s / nk, m0, n0);
    cp_async_wait<1>();
    __syncthreads();  // raw slab s is visible to every thread
    drain(b);         // the MMAs of slab s-2 no longer read planes b
    oz_slice<S, OPA, OPB>(plane(b), rawA(b), rawB(b), ea + m0, eb + n0, tid);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    ok = __syncthreads_and(ok) != 0;  // planes visible to the tensor core; raw b consumed; `ok` uniform
    fetch(s + 2);
    if (tid == 0 && ok) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      oz_issue_slab<S>(plane(b), tmem, kc == 0);
      tc_commit(bar[b]);
    }
    ++uses[b];
    if (kc != nk - 1) continue;

    // ---- tile complete: epilogue.  Warp w reads lanes 32 (w % 4).. and the
    // complex columns 16 (w / 4).. (re at column c, im at column 32 + c of
    // every level), combines the levels in FP64 and writes through a
    // transpose in the planes area.
    drain(0);
    drain(1);
    ok = __syncthreads_and(ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const int lq = warp & 3, ch = warp >> 2;
    const int row = lq * 32 + lane, c0 = ch * 16;
    cplx* tb = reinterpret_cast<cplx*>(smem) + warp * 32 * OZ_EPI_PITCH;
    double vr[16], vi[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) vr[j] = vi[j] = 0.0;
    if (ok) {
      const uint32_t ta = tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)c0;
#pragma unroll 1
      for (int l = S - 1; l >= 0; --l) {
        int ar[16], ai[16];
        tc_ld16i(ta + l * OZ_N, ar);
        tc_ld16i(ta + l * OZ_N + OZ_NC, ai);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          vr[j] = fma(vr[j], 0.0078125, (double)ar[j]);  // v 2^-7 + acc_l
          vi[j] = fma(vi[j], 0.0078125, (double)ai[j]);
        }
      }
    }
    const int em = ea[m0 + row];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int en = eb[n0 + c0 + j];
      cplx o;
      if (em == OZ_BAD || en == OZ_BAD) {
        o = cmk(__longlong_as_double(0x7ff8000000000000LL), __longlong_as_double(0x7ff8000000000000LL));
      } else {
        const int sc = em + en - 14;
        o = cmk(scalbn(vr[j], sc), scalbn(vi[j], sc));
      }
      tb[lane * OZ_EPI_PITCH + j] = o;
    }
    __syncwarp();
    const int n = n0 + c0 + (lane & 15);
#pragma unroll 4
    for (int r = lane >> 4; r < 32; r += 2) {
      const int m = m0 + lq * 32 + r;
      if (m < g.M && n < g.N) epi(m, n, tb[r * OZ_EPI_PITCH + (lane & 15)]);
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();  // accumulators and the planes area are free again
  }
  cp_async_wait<0>();
  if (tid == 0) {
    if (!ok) tc_err = 1;
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(bar[0]));
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(bar[1]));
  }
  __syncthreads();
}

// C = alpha op(A) op(B) + beta D on the int8 slice path (D may alias C).
template <int S, int OPA, int OPB>
NEGF_DEV void cta_gemm_oz(const GemmArgs& g, char* smem) {
  cta_gemm_oz_epi<S, OPA, OPB>(g, smem, EpiStore{g});
}

}  // namespace negf
