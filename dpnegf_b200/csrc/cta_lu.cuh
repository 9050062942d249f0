// CTA-wide complex128 linear solve X = A^-1 B by LU factorisation with partial
// pivoting, as LAPACK's zgetrf + zgetrs (what numpy.linalg.solve and
// numpy.linalg.inv run).
//
// The lead decimation solves (zS - eps) [Xa Xb] = [alpha beta] at every
// doubling step, and its convergence test on g_s = (zS - eps_s)^-1 is a right
// residual.  An explicit Gauss-Jordan inverse followed by a product has a
// right residual up to cond(A) times larger than a backward-stable solve, which
// measured 100-1000x above the reference's at well-conditioned energies; the
// LU solve is backward stable (|A X - B| <= c u |L||U||X|) and does less work
// (n^3/3 for the factorisation + n^2 nb for the two triangular solves, against
// n^3 + n^2 nb for inverse-then-multiply).
//
// Recursive blocking (the order of LAPACK's zgetrf2), so every update is a
// CTA GEMM of depth up to n/2:
//   LU([A11 A12; A21 A22]):  LU of the left half [A11; A21] (recursively, down to
//   panels of NB columns factorised in shared memory), its row swaps applied to
//   the right half, A12 <- L11^-1 A12, A22 <- A22 - L21 A12, LU of A22, its row
//   swaps applied back to A21.
// The right-hand sides are then written in the pivoted row order by the caller
// (one gather, instead of swapping their rows one pivot at a time) and
// B <- L^-1 B, B <- U^-1 B run as recursive triangular solves whose diagonal
// blocks of at most 16 are solved column by column in registers.
// W (n x n) is destroyed (it holds L and U); B (n x nb) is overwritten by X.
#pragma once
#include "cta_inverse.cuh"  // pivot search helpers, the CTA GEMM

namespace negf {

// 1/a as conj(a) / |a|^2 (one division; pivots here are far from the
// over/underflow range of |a|^2).
NEGF_DEV cplx crcp_fast(cplx a) {
  const double r = 1.0 / fma(a.x, a.x, a.y * a.y);
  return cmk(a.x * r, -a.y * r);
}

constexpr int LU_TB = 16;  // diagonal blocks of the triangular solves (register columns)

template <int NB>
struct LuLayout {
  static constexpr int PP = NB + 1;  // panel pitch (complex entries)
  __host__ __device__ static size_t panel_bytes(int n) { return (size_t)n * PP * sizeof(double2); }
  // the small arrays sit above both the panel and the GEMM ring (the GEMM reuses the panel area)
  __host__ __device__ static size_t small_offset(int n) {
    size_t a = panel_bytes(n), g = (size_t)GEMM_SMEM_BYTES;
    return ((a > g ? a : g) + 255) & ~(size_t)255;
  }
  __host__ __device__ static size_t bytes(int n) {
    return small_offset(n) + LU_TB * sizeof(double2) + 8 * sizeof(double) + (8 + 4) * sizeof(int) +
           2 * (size_t)n * sizeof(int);
  }
};

inline size_t lu_smem_bytes_host(int max_n) {
  size_t a = LuLayout<32>::bytes(max_n < 256 ? max_n : 256);
  if (max_n > 256) {
    const size_t b = LuLayout<16>::bytes(max_n);
    if (b > a) a = b;
  }
  return a;
}

struct LuCtx {
  cplx* W;
  int64_t ldw;
  int n;
  char* smem;
  cplx* rdiag;    // [LU_TB] reciprocal diagonal of the current upper block
  long long* red_v;  // [8] pivot candidates (keys, see pivot_key)
  int* red_i;     // [8]
  int* flag;      // [1] zero / non-finite pivot met
  int* ipiv;      // [n] row swapped with row k at step k (LAPACK order)
  int* perm;      // [n] the swaps composed: row k of P A is row perm[k] of A
  PhaseClock* pc; // optional per-phase cycle counters (null: off)
  NEGF_DEV void mark(int ph) const {
    if (pc) pc->mark(ph);
  }
};

NEGF_DEV void lu_gemm_sub(const LuCtx& c, int M, int N, int K, const cplx* A, int64_t lda, const cplx* B,
                          int64_t ldb, cplx* C, int64_t ldc) {
  GemmArgs g = gemm_args(M, N, K, A, lda, B, ldb, C, ldc);
  g.alpha = cmk(-1.0, 0.0);
  g.D = C; g.ldd = ldc; g.beta = cmk(1.0, 0.0); g.use_d = true;
  cta_gemm<OP_N, OP_N, false, true>(g, reinterpret_cast<cplx*>(c.smem));  // 4M products (see lopez_sancho.cu)
  c.mark(PH_INV_UPDATE);
}

// Row swaps ipiv[ka..kb) applied in order to the ncols columns starting at col (row stride ld).
// Each thread owns whole columns; ends with __syncthreads().
NEGF_DEV void lu_laswp(const LuCtx& c, cplx* col0, int64_t ld, int ncols, int ka, int kb) {
  for (int j = threadIdx.x; j < ncols; j += CTA_THREADS) {
    cplx* col = col0 + j;
    for (int k = ka; k < kb; ++k) {
      const int p = c.ipiv[k];
      if (p != k) {
        const cplx t = col[(int64_t)k * ld];
        col[(int64_t)k * ld] = col[(int64_t)p * ld];
        col[(int64_t)p * ld] = t;
      }
    }
  }
  __syncthreads();
  c.mark(PH_INV_STAGE);
}

// Unblocked LU with row swaps of rows r0..n-1, columns r0..r0+w-1 (w <= NB) in shared memory.
template <int NB>
NEGF_DEV void lu_panel(const LuCtx& c, int r0, int w) {
  constexpr int PP = LuLayout<NB>::PP;
  constexpr int NWARP = CTA_THREADS / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m = c.n - r0;
  cplx* P = reinterpret_cast<cplx*>(c.smem);
  cplx* Wp = c.W + (int64_t)r0 * c.ldw + r0;
  for (int e = tid; e < m * NB; e += CTA_THREADS) {
    const int r = e / NB, k = e % NB;
    P[r * PP + k] = k < w ? Wp[(int64_t)r * c.ldw + k] : cmk(0.0, 0.0);
  }
  __syncthreads();
  for (int j = 0; j < w; ++j) {
    long long bv = -1;
    int bi = m;
    for (int r = j + tid; r < m; r += CTA_THREADS) argmax_merge_key(bv, bi, pivot_key(P[r * PP + j]), r);
    warp_argmax_key(bv, bi);
    if (lane == 0) { c.red_v[warp] = bv; c.red_i[warp] = bi; }
    __syncthreads();
    bv = c.red_v[0];
    bi = c.red_i[0];
#pragma unroll
    for (int k = 1; k < NWARP; ++k) argmax_merge_key(bv, bi, c.red_v[k], c.red_i[k]);
    if (bi != j)
      for (int k = tid; k < NB; k += CTA_THREADS) {
        const cplx t = P[j * PP + k];
        P[j * PP + k] = P[bi * PP + k];
        P[bi * PP + k] = t;
      }
    if (tid == 0) {
      c.ipiv[r0 + j] = r0 + bi;
      if (pivot_key_singular(bv)) *c.flag = 1;
    }
    __syncthreads();
    const cplx d = crcp_fast(P[j * PP + j]);
    for (int r = j + 1 + tid; r < m; r += CTA_THREADS) {
      const cplx l = cmul(P[r * PP + j], d);
      P[r * PP + j] = l;
      for (int k = j + 1; k < w; ++k) P[r * PP + k] = csub(P[r * PP + k], cmul(l, P[j * PP + k]));
    }
    __syncthreads();
  }
  for (int e = tid; e < m * w; e += CTA_THREADS) {
    const int r = e / w, k = e % w;
    Wp[(int64_t)r * c.ldw + k] = P[r * PP + k];
  }
  __syncthreads();
  c.mark(PH_INV_PANEL);
}

// C (h x N, row stride ldc) <- L^-1 C with L the unit-lower triangle of W at (r0, r0), h <= LU_TB:
// L staged in shared memory, each thread solves whole columns in registers.
NEGF_DEV void lu_trsm_lower_leaf(const LuCtx& c, int r0, int h, cplx* C, int64_t ldc, int N) {
  constexpr int TP = LU_TB + 1;
  cplx* Ls = reinterpret_cast<cplx*>(c.smem);
  for (int e = threadIdx.x; e < h * h; e += CTA_THREADS) {
    const int i = e / h, j = e % h;
    Ls[i * TP + j] = c.W[(int64_t)(r0 + i) * c.ldw + r0 + j];
  }
  __syncthreads();
  for (int col = threadIdx.x; col < N; col += CTA_THREADS) {
    cplx* p = C + col;
    cplx x[LU_TB];
#pragma unroll
    for (int j = 0; j < LU_TB; ++j) x[j] = j < h ? p[(int64_t)j * ldc] : cmk(0.0, 0.0);
#pragma unroll
    for (int j = 1; j < LU_TB; ++j) {
      if (j < h) {
#pragma unroll
        for (int i = 0; i < j; ++i) x[j] = csub(x[j], cmul(Ls[j * TP + i], x[i]));
      }
    }
#pragma unroll
    for (int j = 1; j < LU_TB; ++j)
      if (j < h) p[(int64_t)j * ldc] = x[j];
  }
  __syncthreads();
  c.mark(PH_INV_GATHER);
}

// C <- U^-1 C with U the upper triangle (non-unit) of W at (r0, r0), h <= LU_TB.
NEGF_DEV void lu_trsm_upper_leaf(const LuCtx& c, int r0, int h, cplx* C, int64_t ldc, int N) {
  constexpr int TP = LU_TB + 1;
  cplx* Us = reinterpret_cast<cplx*>(c.smem);
  for (int e = threadIdx.x; e < h * h; e += CTA_THREADS) {
    const int i = e / h, j = e % h;
    Us[i * TP + j] = c.W[(int64_t)(r0 + i) * c.ldw + r0 + j];
  }
  __syncthreads();
  if (threadIdx.x < h) c.rdiag[threadIdx.x] = crcp_fast(Us[threadIdx.x * TP + threadIdx.x]);
  __syncthreads();
  for (int col = threadIdx.x; col < N; col += CTA_THREADS) {
    cplx* p = C + col;
    cplx x[LU_TB];
#pragma unroll
    for (int j = 0; j < LU_TB; ++j) x[j] = j < h ? p[(int64_t)j * ldc] : cmk(0.0, 0.0);
#pragma unroll
    for (int j = LU_TB - 1; j >= 0; --j) {
      if (j < h) {
#pragma unroll
        for (int i = j + 1; i < LU_TB; ++i)
          if (i < h) x[j] = csub(x[j], cmul(Us[j * TP + i], x[i]));
        x[j] = cmul(x[j], c.rdiag[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < LU_TB; ++j)
      if (j < h) p[(int64_t)j * ldc] = x[j];
  }
  __syncthreads();
  c.mark(PH_INV_GATHER);
}

NEGF_DEV int lu_split(int h, int unit) { return ((h / 2 + unit - 1) / unit) * unit; }

// C <- L^-1 C, L the unit-lower triangle of W at (r0, r0) of size h: halves down to LU_TB.
template <int LV>
__device__ __noinline__ void lu_trsm_lower(const LuCtx c, int r0, int h, cplx* C, int64_t ldc, int N) {
  if constexpr (LV == 0) {
    lu_trsm_lower_leaf(c, r0, h, C, ldc, N);
  } else {
    if (h <= LU_TB) { lu_trsm_lower_leaf(c, r0, h, C, ldc, N); return; }
    const int h1 = lu_split(h, LU_TB);
    lu_trsm_lower<LV - 1>(c, r0, h1, C, ldc, N);
    lu_gemm_sub(c, h - h1, N, h1, c.W + (int64_t)(r0 + h1) * c.ldw + r0, c.ldw, C, ldc, C + (int64_t)h1 * ldc, ldc);
    lu_trsm_lower<LV - 1>(c, r0 + h1, h - h1, C + (int64_t)h1 * ldc, ldc, N);
  }
}

// C <- U^-1 C, U the upper triangle of W at (r0, r0) of size h.
template <int LV>
__device__ __noinline__ void lu_trsm_upper(const LuCtx c, int r0, int h, cplx* C, int64_t ldc, int N) {
  if constexpr (LV == 0) {
    lu_trsm_upper_leaf(c, r0, h, C, ldc, N);
  } else {
    if (h <= LU_TB) { lu_trsm_upper_leaf(c, r0, h, C, ldc, N); return; }
    const int h1 = lu_split(h, LU_TB);
    lu_trsm_upper<LV - 1>(c, r0 + h1, h - h1, C + (int64_t)h1 * ldc, ldc, N);
    lu_gemm_sub(c, h1, N, h - h1, c.W + (int64_t)r0 * c.ldw + r0 + h1, c.ldw, C + (int64_t)h1 * ldc, ldc, C, ldc);
    lu_trsm_upper<LV - 1>(c, r0, h1, C, ldc, N);
  }
}

// LU with partial pivoting of rows r0..n-1 x columns r0..r0+w-1 (zgetrf2's recursion).
template <int NB, int LV>
__device__ __noinline__ void lu_rec(const LuCtx c, int r0, int w) {
  if constexpr (LV == 0) {
    lu_panel<NB>(c, r0, w);
  } else {
    if (w <= NB) { lu_panel<NB>(c, r0, w); return; }
    const int h = lu_split(w, NB), w2 = w - h;
    cplx* W = c.W;
    const int64_t ld = c.ldw;
    lu_rec<NB, LV - 1>(c, r0, h);
    lu_laswp(c, W + r0 + h, ld, w2, r0, r0 + h);                               // swaps -> A12, A22
    lu_trsm_lower<LV>(c, r0, h, W + (int64_t)r0 * ld + r0 + h, ld, w2);        // A12 <- L11^-1 A12
    lu_gemm_sub(c, c.n - r0 - h, w2, h, W + (int64_t)(r0 + h) * ld + r0, ld,   // A22 -= L21 A12
                W + (int64_t)r0 * ld + r0 + h, ld, W + (int64_t)(r0 + h) * ld + r0 + h, ld);
    lu_rec<NB, LV - 1>(c, r0 + h, w2);
    lu_laswp(c, W + r0, ld, h, r0 + h, r0 + w);                                // swaps of A22 -> L21
  }
}

template <int NB>
NEGF_DEV LuCtx lu_ctx(cplx* W, int64_t ldw, int n, char* smem_raw, PhaseClock* pc) {
  char* sm = smem_raw + LuLayout<NB>::small_offset(n);
  LuCtx c;
  c.W = W; c.ldw = ldw; c.n = n; c.smem = smem_raw;
  c.rdiag = reinterpret_cast<cplx*>(sm);
  c.red_v = reinterpret_cast<long long*>(c.rdiag + LU_TB);
  c.red_i = reinterpret_cast<int*>(c.red_v + 8);
  c.flag = c.red_i + 8;
  c.ipiv = c.flag + 4;
  c.perm = c.ipiv + n;
  c.pc = pc;
  return c;
}

// P A = L U in place (W holds L below the diagonal, U on and above); the permutation is left in
// shared memory for cta_lu_perm / cta_lu_trsolve.  Returns 0, or 1 if a zero or non-finite pivot
// was met.  Uniform across the CTA; ends with __syncthreads().
template <int NB>
__device__ __noinline__ int cta_lu_factor_nb(cplx* W, int64_t ldw, int n, char* smem_raw, PhaseClock* pc) {
  const LuCtx c = lu_ctx<NB>(W, ldw, n, smem_raw, pc);
  if (threadIdx.x == 0) *c.flag = 0;
  __syncthreads();
  lu_rec<NB, 6>(c, 0, n);
  if (threadIdx.x == 0) {  // compose the swaps into a row permutation
    for (int k = 0; k < n; ++k) c.perm[k] = k;
    for (int k = 0; k < n; ++k) {
      const int p = c.ipiv[k];
      const int t = c.perm[k];
      c.perm[k] = c.perm[p];
      c.perm[p] = t;
    }
  }
  __syncthreads();
  const int f = *c.flag;
  __syncthreads();
  return f;
}

// B <- U^-1 L^-1 B for B already in the pivoted row order (row k = row perm[k] of the original).
template <int NB>
__device__ __noinline__ void cta_lu_trsolve_nb(cplx* W, int64_t ldw, int n, cplx* B, int64_t ldb, int nb,
                                               char* smem_raw, PhaseClock* pc) {
  const LuCtx c = lu_ctx<NB>(W, ldw, n, smem_raw, pc);
  lu_trsm_lower<6>(c, 0, n, B, ldb, nb);
  lu_trsm_upper<6>(c, 0, n, B, ldb, nb);
}

// The factorisation of A (n <= 512) for X = A^-1 B, in three steps: cta_lu_factor, then the
// right-hand sides written in the pivoted row order (row k from row cta_lu_perm()[k]), then
// cta_lu_trsolve.  pc: optional phase counters (panel / row swaps / GEMM updates / register
// triangular solves).
NEGF_DEV int cta_lu_factor(cplx* W, int64_t ldw, int n, char* smem_raw, PhaseClock* pc = nullptr) {
  if (n <= 256) return cta_lu_factor_nb<32>(W, ldw, n, smem_raw, pc);
  return cta_lu_factor_nb<16>(W, ldw, n, smem_raw, pc);
}
// The row permutation of the last cta_lu_factor of an n-row matrix (shared memory; valid until the
// next factorisation).
NEGF_DEV const int* cta_lu_perm(const char* smem_raw, int n) {
  const LuCtx c = n <= 256 ? lu_ctx<32>(nullptr, 0, n, const_cast<char*>(smem_raw), nullptr)
                           : lu_ctx<16>(nullptr, 0, n, const_cast<char*>(smem_raw), nullptr);
  return c.perm;
}
NEGF_DEV void cta_lu_trsolve(cplx* W, int64_t ldw, int n, cplx* B, int64_t ldb, int nb, char* smem_raw,
                             PhaseClock* pc = nullptr) {
  if (n <= 256) cta_lu_trsolve_nb<32>(W, ldw, n, B, ldb, nb, smem_raw, pc);
  else cta_lu_trsolve_nb<16>(W, ldw, n, B, ldb, nb, smem_raw, pc);
}

}  // namespace negf
