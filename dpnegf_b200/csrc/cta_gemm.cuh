// CTA-wide complex128 GEMM on FP64 tensor cores (DMMA m8n8k4), 3M products.
//
//   C[M x N] = alpha * op(A) * op(B) + beta * D        (D may alias C)
//
// One CTA of 256 threads (8 warps) walks the 64x64 output tiles of C; each
// tile streams 16-wide k-slabs of op(A) and op(B) into padded shared-memory
// tiles with cp.async (3-stage ring).  Each warp owns a 32x16 sub-tile and
// forms every complex product with three real DMMA m16n8k8 (Gauss/3M):
//   T1 = Ar*Br, T2 = Ai*Bi, T3 = (Ar+Ai)*(Br+Bi);  Re = T1-T2, Im = T3-T1-T2.
// Shared-memory pitches are chosen so the DMMA fragment reads (one 16-byte
// complex per lane) are bank-conflict free for every operand orientation.
#pragma once
#include <type_traits>
#include "negf_common.cuh"

namespace negf {

#ifndef NEGF_GT_K
#define NEGF_GT_K 16
#endif
constexpr int GT_M = 64, GT_N = 64, GT_K = NEGF_GT_K;
static_assert(GT_K == 16 || GT_K == 32, "k slab of 16 or 32");
constexpr int PITCH_MK = GT_K + 4;  // [64 rows][GT_K k] tiles (pitch = 4 mod 8)
constexpr int PITCH_KN = GT_N + 2;  // [GT_K k][64 cols] tiles (pitch = 2 mod 8)
constexpr int GT_LOADS = GT_M * GT_K / 256;  // 16-byte copies per thread per operand tile
constexpr int GT_TILE = (GT_M * PITCH_MK > GT_K * PITCH_KN) ? GT_M * PITCH_MK : GT_K * PITCH_KN;
#ifndef NEGF_GT_STAGES
#define NEGF_GT_STAGES 3
#endif
// Depth of the cp.async k-slab ring; one value for the whole library (the host-side shared-memory
// sizes of every kernel derive from it).  4 stages measured 4 % slower on the 256^3 product and
// the sweep (LU solves 2 % faster).
constexpr int GT_STAGES = NEGF_GT_STAGES;
static_assert(GT_STAGES == 3 || GT_STAGES == 4, "3- or 4-stage ring");
constexpr int GEMM_SMEM_BYTES = 2 * GT_STAGES * GT_TILE * (int)sizeof(cplx);  // stages x (A,B)
constexpr int CTA_THREADS = 256;

struct GemmArgs {
  int M, N, K;
  const cplx* A;
  int64_t lda;
  const cplx* B;
  int64_t ldb;
  cplx* C;
  int64_t ldc;
  const cplx* D;  // addend, read only when use_d
  int64_t ldd;
  cplx alpha, beta;
  bool use_d;
};

NEGF_DEV GemmArgs gemm_args(int M, int N, int K, const cplx* A, int64_t lda, const cplx* B, int64_t ldb,
                            cplx* C, int64_t ldc) {
  GemmArgs g;
  g.M = M; g.N = N; g.K = K;
  g.A = A; g.lda = lda; g.B = B; g.ldb = ldb; g.C = C; g.ldc = ldc;
  g.D = nullptr; g.ldd = 0;
  g.alpha = cmk(1.0, 0.0); g.beta = cmk(0.0, 0.0); g.use_d = false;
  return g;
}

// op(A) tile element (m, k) -> shared-memory index
template <int OP>
NEGF_DEV int a_idx(int m, int k) { return OP == OP_C ? k * PITCH_KN + m : m * PITCH_MK + k; }
// op(B) tile element (k, n) -> shared-memory index
template <int OP>
NEGF_DEV int b_idx(int k, int n) { return OP == OP_C ? n * PITCH_MK + k : k * PITCH_KN + n; }

// Stage the (m0,k0) tile of op(A) into sA.
template <int OP>
NEGF_DEV void load_a_tile(cplx* sA, const GemmArgs& g, int m0, int k0, int tid) {
#pragma unroll
  for (int s = 0; s < GT_LOADS; ++s) {
    int e = tid + s * CTA_THREADS;
    if (OP == OP_C) {  // stored X is K x M: tile rows k, cols m
      int r = e >> 6, c = e & 63;
      int k = k0 + r, m = m0 + c;
      bool v = (k < g.K) && (m < g.M);
      const cplx* src = v ? g.A + (int64_t)k * g.lda + m : g.A;
      cp_async16(sA + r * PITCH_KN + c, src, v);
    } else {  // stored A is M x K: tile rows m, cols k
      int r = e / GT_K, c = e % GT_K;
      int m = m0 + r, k = k0 + c;
      bool v = (m < g.M) && (k < g.K);
      const cplx* src = v ? g.A + (int64_t)m * g.lda + k : g.A;
      cp_async16(sA + r * PITCH_MK + c, src, v);
    }
  }
}

// Stage the (k0,n0) tile of op(B) into sB.
template <int OP>
NEGF_DEV void load_b_tile(cplx* sB, const GemmArgs& g, int k0, int n0, int tid) {
#pragma unroll
  for (int s = 0; s < GT_LOADS; ++s) {
    int e = tid + s * CTA_THREADS;
    if (OP == OP_C) {  // stored X is N x K: tile rows n, cols k
      int r = e / GT_K, c = e % GT_K;
      int n = n0 + r, k = k0 + c;
      bool v = (n < g.N) && (k < g.K);
      const cplx* src = v ? g.B + (int64_t)n * g.ldb + k : g.B;
      cp_async16(sB + r * PITCH_MK + c, src, v);
    } else {  // stored B is K x N: tile rows k, cols n
      int r = e >> 6, c = e & 63;
      int k = k0 + r, n = n0 + c;
      bool v = (k < g.K) && (n < g.N);
      const cplx* src = v ? g.B + (int64_t)k * g.ldb + n : g.B;
      cp_async16(sB + r * PITCH_KN + c, src, v);
    }
  }
}

struct Acc3M {
  double t1[2][2][4], t2[2][2][4], t3[2][2][4];  // [m16 frag][n8 frag][c0..c3]
  NEGF_DEV void zero() {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) t1[i][j][e] = t2[i][j][e] = t3[i][j][e] = 0.0;
  }
};

// Position in the warp's 32x16 sub-tile of accumulator element (i, j, e).
NEGF_DEV int acc_row(int i, int e, int wm, int lane) { return wm + 16 * i + (lane >> 2) + ((e & 2) ? 8 : 0); }
NEGF_DEV int acc_col(int j, int e, int wn, int lane) { return wn + 8 * j + 2 * (lane & 3) + (e & 1); }

// One warp: ksteps x (k=8) slabs of its 32x16 sub-tile (2 x 2 DMMA m16n8k8
// fragments per real plane).  Fragment reads go through the index functors
// so the same loop serves the GEMM tiles and the Gauss-Jordan panel update.
// G3 selects the complex product: Gauss/3M (three real MMAs, t1..t3) or the
// conventional 4M form (four real MMAs into t1 = Re, t2 = Im), whose
// componentwise error bound is tighter -- used where an iteration amplifies
// rounding (the lead decimation).
template <bool CONJ_A, bool CONJ_B, bool G3 = true, class AIdx, class BIdx>
NEGF_DEV void warp_mma_3m(Acc3M& acc, const cplx* sA, const cplx* sB, int ksteps, int wm, int wn, int lane,
                          AIdx aidx, BIdx bidx) {
  const int gr = lane >> 2, gc = lane & 3;
  for (int ks = 0; ks < ksteps; ++ks) {
    const int k0 = ks * 8 + gc;
    double ar[2][4], ai[2][4], as[2][4], br[2][2], bi[2][2], bs[2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int r = wm + 16 * i + gr;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        cplx a = sA[aidx(r + ((e & 1) ? 8 : 0), k0 + ((e & 2) ? 4 : 0))];
        ar[i][e] = a.x;
        ai[i][e] = CONJ_A ? -a.y : a.y;
        as[i][e] = ar[i][e] + ai[i][e];
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int c = wn + 8 * j + gr;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        cplx b = sB[bidx(k0 + 4 * e, c)];
        br[j][e] = b.x;
        bi[j][e] = CONJ_B ? -b.y : b.y;
        bs[j][e] = br[j][e] + bi[j][e];
      }
    }
    if (G3) {
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          dmma1688(acc.t1[i][j], ar[i], br[j]);
          dmma1688(acc.t2[i][j], ai[i], bi[j]);
          dmma1688(acc.t3[i][j], as[i], bs[j]);
        }
    } else {
      double an[2][4];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int e = 0; e < 4; ++e) an[i][e] = -ai[i][e];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          dmma1688(acc.t1[i][j], ar[i], br[j]);
          dmma1688(acc.t1[i][j], an[i], bi[j]);
          dmma1688(acc.t2[i][j], ar[i], bi[j]);
          dmma1688(acc.t2[i][j], ai[i], br[j]);
        }
    }
  }
}

// Complex value of accumulator element (i, j, e).
template <bool G3>
NEGF_DEV cplx acc_value(const Acc3M& acc, int i, int j, int e) {
  const double t1 = acc.t1[i][j][e], t2 = acc.t2[i][j][e];
  if (G3) return cmk(t1 - t2, acc.t3[i][j][e] - t1 - t2);
  return cmk(t1, t2);
}

// Visit every accumulator element of this warp: f(row, col, value).
template <bool G3, class F>
NEGF_DEV void acc_foreach(const Acc3M& acc, int wm, int wn, int lane, F f) {
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) f(acc_row(i, e, wm, lane), acc_col(j, e, wn, lane), acc_value<G3>(acc, i, j, e));
}

struct AIdxOp0 { NEGF_DEV int operator()(int m, int k) const { return a_idx<OP_N>(m, k); } };
struct AIdxOpC { NEGF_DEV int operator()(int m, int k) const { return a_idx<OP_C>(m, k); } };
struct BIdxOp0 { NEGF_DEV int operator()(int k, int n) const { return b_idx<OP_N>(k, n); } };
struct BIdxOpC { NEGF_DEV int operator()(int k, int n) const { return b_idx<OP_C>(k, n); } };

// Default epilogue: C = alpha * acc + beta * D.
struct EpiStore {
  GemmArgs g;
  NEGF_DEV void operator()(int m, int n, cplx v) const {
    cplx o = cmul(g.alpha, v);
    if (g.use_d) o = cfma(g.beta, g.D[(int64_t)m * g.ldd + n], o);
    g.C[(int64_t)m * g.ldc + n] = o;
  }
};

// acc = op(A) op(B) over the whole M x N output by the whole CTA; epi(m, n, acc)
// is called once for every in-range element.  The output must not alias A or
// B.  Ends with __syncthreads(), so whatever epi wrote to global memory is
// visible to every thread of the CTA on return.  k-slabs flow through a
// GT_STAGES-deep cp.async ring (one barrier per slab).
// With SKIP, a warp whose 32 x 16 sub-tile lies wholly outside the product
// skips its MMAs (ragged sizes then execute ~1.07x the useful products instead
// of up to 16x at n = 16); off by default because the extra live predicate
// raises register spills in the RGF sweep, which sits at the 255-register cap.
template <int OPA, int OPB, bool G3, class Epi, bool SKIP = false>
__device__ __noinline__ void cta_gemm_epi(const GemmArgs g, cplx* smem, const Epi epi) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 2) * 32, wn = (warp & 3) * 16;
  const int nk = (g.K + GT_K - 1) / GT_K;
  typedef typename std::conditional<OPA == OP_C, AIdxOpC, AIdxOp0>::type AI;
  typedef typename std::conditional<OPB == OP_C, BIdxOpC, BIdxOp0>::type BI;
  constexpr bool CA = (OPA != OP_N), CB = (OPB != OP_N);
  auto sA = [&](int s) { return smem + (2 * s) * GT_TILE; };
  auto sB = [&](int s) { return smem + (2 * s + 1) * GT_TILE; };

  for (int m0 = 0; m0 < g.M; m0 += GT_M) {
    for (int n0 = 0; n0 < g.N; n0 += GT_N) {
      __syncthreads();  // the previous tile's last slab is no longer being read
#pragma unroll
      for (int s = 0; s < GT_STAGES - 1; ++s) {
        if (s < nk) {
          load_a_tile<OPA>(sA(s), g, m0, s * GT_K, tid);
          load_b_tile<OPB>(sB(s), g, s * GT_K, n0, tid);
        }
        cp_async_commit();
      }
      Acc3M acc;
      acc.zero();
      const bool live = !SKIP || (m0 + wm < g.M && n0 + wn < g.N);
      for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<GT_STAGES - 2>();
        __syncthreads();
        const int nx = kt + GT_STAGES - 1;
        if (nx < nk) {
          load_a_tile<OPA>(sA(nx % GT_STAGES), g, m0, nx * GT_K, tid);
          load_b_tile<OPB>(sB(nx % GT_STAGES), g, nx * GT_K, n0, tid);
        }
        cp_async_commit();
        if (live) warp_mma_3m<CA, CB, G3>(acc, sA(kt % GT_STAGES), sB(kt % GT_STAGES), GT_K / 8, wm, wn, lane, AI(), BI());
      }
      acc_foreach<G3>(acc, wm, wn, lane, [&](int r, int c, cplx v) {
        int m = m0 + r, n = n0 + c;
        if (m < g.M && n < g.N) epi(m, n, v);
      });
    }
  }
  cp_async_wait<0>();
  __syncthreads();
}

// C = alpha op(A) op(B) + beta D (D may alias C; C must not alias A or B).
template <int OPA, int OPB, bool G3 = true, bool SKIP = false>
NEGF_DEV void cta_gemm(const GemmArgs& g, cplx* smem) {
  cta_gemm_epi<OPA, OPB, G3, EpiStore, SKIP>(g, smem, EpiStore{g});
}

}  // namespace negf
