// CTA-wide complex128 linear solve X = A^-1 B by LU factorisation with partial
// pivoting, in the order of LAPACK's zgetrf + zgetrs (what numpy.linalg.solve
// and numpy.linalg.inv run).
//
// The lead decimation solves (zS - eps) [Xa Xb] = [alpha beta] at every
// doubling step, and its convergence test on g_s = (zS - eps_s)^-1 is a right
// residual.  An explicit Gauss-Jordan inverse followed by a product has a
// right residual up to cond(A) times larger than a backward-stable solve, which
// measured 100-1000x above the reference's at well-conditioned energies; the
// LU solve below is backward stable (|A X - B| <= c u |L||U||X|) and also does
// less work (n^3/3 for the factorisation + n^2 nb for the two triangular
// solves, against n^3 + n^2 nb for inverse-then-multiply).
//
// Blocking: panels of NB columns (32 for n <= 256, 16 above) are factorised in
// shared memory with physical row swaps; the panel's swaps are then applied to
// the columns on its right and to B (laswp), its unit-lower triangle is solved
// against those rows (trsm), and the trailing rows of A and of B are updated
// with one CTA GEMM each.  Back substitution walks the same blocks from the
// bottom: one GEMM for the rows already solved, then the block's upper
// triangle column by column.  W (n x n) is destroyed; B (n x nb) is overwritten
// by X.
#pragma once
#include "cta_inverse.cuh"  // pivot search helpers, the CTA GEMM

namespace negf {

// 1/a as conj(a) / |a|^2 (one division; pivots here are far from the
// over/underflow range of |a|^2).
NEGF_DEV cplx crcp_fast(cplx a) {
  const double r = 1.0 / fma(a.x, a.x, a.y * a.y);
  return cmk(a.x * r, -a.y * r);
}

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
    return small_offset(n) + NB * sizeof(double2) + 8 * sizeof(double) + (8 + NB + 4) * sizeof(int);
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

// Returns 0 on success, 1 if a zero or non-finite pivot was met (the result is then
// not usable).  Uniform across the CTA; ends with __syncthreads().
template <int NB, bool G3, bool SKIP>
__device__ __noinline__ int cta_lu_solve_nb(cplx* W, int64_t ldw, int n, cplx* B, int64_t ldb, int nb,
                                            char* smem_raw) {
  constexpr int PP = LuLayout<NB>::PP;
  constexpr int NWARP = CTA_THREADS / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  cplx* P = reinterpret_cast<cplx*>(smem_raw);
  char* sm = smem_raw + LuLayout<NB>::small_offset(n);
  cplx* rdiag = reinterpret_cast<cplx*>(sm);             // [NB]
  double* red_v = reinterpret_cast<double*>(rdiag + NB);  // [NWARP]
  int* red_i = reinterpret_cast<int*>(red_v + NWARP);     // [NWARP]
  int* ipiv = red_i + NWARP;                              // [NB]
  int* flag = ipiv + NB;                                  // [1]
  const cplx MONE = cmk(-1.0, 0.0);
  if (tid == 0) *flag = 0;

  for (int k0 = 0; k0 < n; k0 += NB) {
    const int w = min(NB, n - k0), m = n - k0;
    // ---- stage the panel: rows k0..n-1, columns k0..k0+w-1
    for (int e = tid; e < m * NB; e += CTA_THREADS) {
      const int r = e / NB, c = e % NB;
      P[r * PP + c] = c < w ? W[(int64_t)(k0 + r) * ldw + k0 + c] : cmk(0.0, 0.0);
    }
    __syncthreads();
    // ---- unblocked LU of the panel with row swaps (local row indices)
    for (int j = 0; j < w; ++j) {
      double bv = -1.0;
      int bi = m;
      for (int r = j + tid; r < m; r += CTA_THREADS) argmax_merge(bv, bi, pivot_measure(P[r * PP + j]), r);
      warp_argmax(bv, bi);
      if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
      __syncthreads();
      bv = red_v[0];
      bi = red_i[0];
#pragma unroll
      for (int k = 1; k < NWARP; ++k) argmax_merge(bv, bi, red_v[k], red_i[k]);
      if (bi != j)
        for (int c = tid; c < NB; c += CTA_THREADS) {
          const cplx t = P[j * PP + c];
          P[j * PP + c] = P[bi * PP + c];
          P[bi * PP + c] = t;
        }
      if (tid == 0) {
        ipiv[j] = bi;
        if (!(bv > 0.0) || !isfinite(bv)) *flag = 1;
      }
      __syncthreads();
      const cplx d = crcp_fast(P[j * PP + j]);
      for (int r = j + 1 + tid; r < m; r += CTA_THREADS) {
        const cplx l = cmul(P[r * PP + j], d);
        P[r * PP + j] = l;
        for (int c = j + 1; c < w; ++c) P[r * PP + c] = csub(P[r * PP + c], cmul(l, P[j * PP + c]));
      }
      __syncthreads();
    }
    // ---- the factorised panel back to W
    for (int e = tid; e < m * w; e += CTA_THREADS) {
      const int r = e / w, c = e % w;
      W[(int64_t)(k0 + r) * ldw + k0 + c] = P[r * PP + c];
    }
    // ---- the panel's swaps on the columns right of it and on B, then the unit-lower solve of
    //      the panel rows there: each thread owns whole columns, so neither needs a barrier
    const int ncw = n - k0 - w;
    for (int c = tid; c < ncw + nb; c += CTA_THREADS) {
      cplx* col = c < ncw ? W + (int64_t)k0 * ldw + k0 + w + c : B + (int64_t)k0 * ldb + (c - ncw);
      const int64_t ld = c < ncw ? ldw : ldb;
      for (int j = 0; j < w; ++j) {
        const int p = ipiv[j];
        if (p != j) {
          const cplx t = col[(int64_t)j * ld];
          col[(int64_t)j * ld] = col[(int64_t)p * ld];
          col[(int64_t)p * ld] = t;
        }
      }
      cplx x[NB];
#pragma unroll
      for (int j = 0; j < NB; ++j) x[j] = j < w ? col[(int64_t)j * ld] : cmk(0.0, 0.0);
#pragma unroll
      for (int j = 1; j < NB; ++j) {
#pragma unroll
        for (int i = 0; i < j; ++i) x[j] = csub(x[j], cmul(P[j * PP + i], x[i]));
      }
#pragma unroll
      for (int j = 1; j < NB; ++j)
        if (j < w) col[(int64_t)j * ld] = x[j];
    }
    __syncthreads();
    // ---- trailing rows: A22 -= L21 U12, B2 -= L21 B1
    if (ncw > 0) {
      const cplx* L21 = W + (int64_t)(k0 + w) * ldw + k0;
      GemmArgs g = gemm_args(ncw, ncw, w, L21, ldw, W + (int64_t)k0 * ldw + k0 + w, ldw,
                             W + (int64_t)(k0 + w) * ldw + k0 + w, ldw);
      g.alpha = MONE; g.D = g.C; g.ldd = g.ldc; g.beta = cmk(1.0, 0.0); g.use_d = true;
      cta_gemm<OP_N, OP_N, G3, SKIP>(g, P);
      g = gemm_args(ncw, nb, w, L21, ldw, B + (int64_t)k0 * ldb, ldb, B + (int64_t)(k0 + w) * ldb, ldb);
      g.alpha = MONE; g.D = g.C; g.ldd = g.ldc; g.beta = cmk(1.0, 0.0); g.use_d = true;
      cta_gemm<OP_N, OP_N, G3, SKIP>(g, P);
    }
  }

  // ---- back substitution, last block first: B_r -= U_{r,>r} X_{>r}; X_r = U_rr^-1 B_r
  for (int r0 = ((n - 1) / NB) * NB; r0 >= 0; r0 -= NB) {
    const int w = min(NB, n - r0), r1 = r0 + w;
    if (r1 < n) {
      GemmArgs g = gemm_args(w, nb, n - r1, W + (int64_t)r0 * ldw + r1, ldw, B + (int64_t)r1 * ldb, ldb,
                             B + (int64_t)r0 * ldb, ldb);
      g.alpha = MONE; g.D = g.C; g.ldd = g.ldc; g.beta = cmk(1.0, 0.0); g.use_d = true;
      cta_gemm<OP_N, OP_N, G3, SKIP>(g, P);
    }
    for (int e = tid; e < w * w; e += CTA_THREADS) {
      const int i = e / w, j = e % w;
      P[i * PP + j] = W[(int64_t)(r0 + i) * ldw + r0 + j];
    }
    __syncthreads();
    if (tid < w) rdiag[tid] = crcp_fast(P[tid * PP + tid]);
    __syncthreads();
    for (int c = tid; c < nb; c += CTA_THREADS) {
      cplx* col = B + (int64_t)r0 * ldb + c;
      cplx x[NB];
#pragma unroll
      for (int j = 0; j < NB; ++j) x[j] = j < w ? col[(int64_t)j * ldb] : cmk(0.0, 0.0);
#pragma unroll
      for (int j = NB - 1; j >= 0; --j) {
        if (j < w) {
#pragma unroll
          for (int i = j + 1; i < NB; ++i)
            if (i < w) x[j] = csub(x[j], cmul(P[j * PP + i], x[i]));
          x[j] = cmul(x[j], rdiag[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < NB; ++j)
        if (j < w) col[(int64_t)j * ldb] = x[j];
    }
    __syncthreads();
  }
  const int f = *flag;
  __syncthreads();
  return f;
}

// X = A^-1 B (n <= 512), see above.  G3 / SKIP select the GEMM's complex product form
// (Gauss/3M or 4M) and the skipping of warps outside ragged products.
template <bool G3 = false, bool SKIP = true>
NEGF_DEV int cta_lu_solve(cplx* W, int64_t ldw, int n, cplx* B, int64_t ldb, int nb, char* smem_raw) {
  if (n <= 256) return cta_lu_solve_nb<32, G3, SKIP>(W, ldw, n, B, ldb, nb, smem_raw);
  return cta_lu_solve_nb<16, G3, SKIP>(W, ldw, n, B, ldb, nb, smem_raw);
}

}  // namespace negf
