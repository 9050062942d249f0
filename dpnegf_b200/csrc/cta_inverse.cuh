// CTA-wide complex128 matrix inverse: blocked Gauss-Jordan with partial
// pivoting, rank-NB updates on FP64 tensor cores.
//
// The matrix W (n x n, row stride ldw) is a work buffer in global memory and
// is destroyed; the inverse is written to G.  Pivoting is implicit: rows never
// move in memory.  For logical column c the pivot is the unused physical row
// p(c) of largest |re|+|im| (LAPACK's izamax measure).  The sweep leaves the
// accumulated row transform T (T A = the pivot-row permutation of I) stored
// in place: column c of W holds column p(c) of T.  Since row i of A^-1 is row
// p(i) of T, the inverse is recovered by the gather
//     G[i][j] = W[p(i)][p^-1(j)],
// fused into the final store.  Each panel of NB columns is factorised in
// shared memory (one warp row-group per row, one lane per column, warp-level
// argmax for the pivot) and then applied to every other column as
//     W[:, c] <- P * W[pivots, c] + (W[:, c] with the pivot rows zeroed),
// a GEMM with k = NB whose A operand (the factorised panel P) already sits in
// shared memory.  Work: n^3 complex multiply-adds, as for an explicit inverse
// by LU.
#pragma once
#include "cta_gemm.cuh"

namespace negf {

template <int NB>
struct InvLayout {
  static constexpr int PP = NB + 4;  // panel pitch (= 4 mod 8: conflict-free A fragments)
  static constexpr int RP = GT_N + 2;
  NEGF_DEV static int rows(int n) { return (n + GT_M - 1) / GT_M * GT_M; }
  NEGF_DEV static size_t bytes(int n) {
    size_t b = (size_t)rows(n) * PP * sizeof(cplx) + (size_t)NB * RP * sizeof(cplx);
    b += (size_t)(2 * n + 64) * sizeof(int) + 16 * sizeof(double);
    return b;
  }
};

inline size_t inv_smem_bytes_host(int n) {
  const int NB = n <= 256 ? 32 : 16;
  const int rows = (n + GT_M - 1) / GT_M * GT_M;
  size_t b = (size_t)rows * (NB + 4) * sizeof(double2) + (size_t)NB * (GT_N + 2) * sizeof(double2);
  b += (size_t)(2 * n + 64) * sizeof(int) + 16 * sizeof(double);
  return b;
}

struct PanelIdx {
  int pitch;
  NEGF_DEV int operator()(int m, int k) const { return m * pitch + k; }
};
struct RIdx {
  NEGF_DEV int operator()(int k, int n) const { return k * (GT_N + 2) + n; }
};

// Returns 0 on success, 1 if a zero or non-finite pivot was met.  Uniform
// across the CTA; ends with __syncthreads().
template <int NB>
NEGF_DEV int cta_inverse_nb(cplx* W, int64_t ldw, int n, cplx* G, int64_t ldg, char* smem_raw) {
  constexpr int PP = InvLayout<NB>::PP;
  constexpr int RP = InvLayout<NB>::RP;
  constexpr int NWARP = CTA_THREADS / 32;
  constexpr int ROWS_PER_PASS = CTA_THREADS / NB;  // rows updated concurrently
  cplx* P = reinterpret_cast<cplx*>(smem_raw);
  const int n_pad = InvLayout<NB>::rows(n);  // panel rows padded to the 64-row tiles
  cplx* R = P + (size_t)n_pad * PP;
  int* piv = reinterpret_cast<int*>(R + NB * RP);  // logical column -> physical row
  int* pinv = piv + n;                             // physical row -> logical column (-1: unused)
  int* red_i = pinv + n;                           // [NWARP]
  int* s_misc = red_i + NWARP;                     // [0]: pivot row, [1]: singular flag
  double* red_v = reinterpret_cast<double*>(s_misc + 56);  // [NWARP], 8-byte aligned
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int my_col = tid % NB, my_rg = tid / NB;

  for (int i = tid; i < n; i += CTA_THREADS) pinv[i] = -1;
  if (tid == 0) s_misc[1] = 0;
  __syncthreads();

  for (int p0 = 0; p0 < n; p0 += NB) {
    const int w = min(NB, n - p0);
    // ---- stage the panel W[:, p0:p0+w) (zero padded to NB columns, n_pad rows)
    for (int e = tid; e < n_pad * NB; e += CTA_THREADS) {
      int i = e / NB, jj = e % NB;
      P[i * PP + jj] = (jj < w && i < n) ? W[(int64_t)i * ldw + p0 + jj] : cmk(0.0, 0.0);
    }
    __syncthreads();

    // ---- unblocked Gauss-Jordan on the panel
    for (int jj = 0; jj < w; ++jj) {
      const int c = p0 + jj;
      // pivot search over unused rows
      double best = -1.0;
      int bidx = n;
      for (int i = tid; i < n; i += CTA_THREADS) {
        if (pinv[i] < 0) {
          double v = cabs1(P[i * PP + jj]);
          if (!(v == v)) v = INFINITY;  // NaN pivots are taken (and flagged) first
          if (v > best || (v == best && i < bidx)) { best = v; bidx = i; }
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        double ov = __shfl_down_sync(0xffffffffu, best, off);
        int oi = __shfl_down_sync(0xffffffffu, bidx, off);
        if (ov > best || (ov == best && oi < bidx)) { best = ov; bidx = oi; }
      }
      if (lane == 0) { red_v[warp] = best; red_i[warp] = bidx; }
      __syncthreads();
      if (tid == 0) {
        double bv = red_v[0];
        int bi = red_i[0];
        for (int k = 1; k < NWARP; ++k)
          if (red_v[k] > bv || (red_v[k] == bv && red_i[k] < bi)) { bv = red_v[k]; bi = red_i[k]; }
        if (!(bv > 0.0) || !isfinite(bv)) s_misc[1] = 1;
        piv[c] = bi;
        pinv[bi] = c;
        s_misc[0] = bi;
      }
      __syncthreads();
      const int p = s_misc[0];
      const cplx d = crcp(P[p * PP + jj]);
      const cplx pd = cmul(P[p * PP + my_col], d);  // scaled pivot row, my column
      __syncthreads();  // pivot row / column jj are rewritten below
      // warp-uniform trip count: every lane reaches each __syncwarp
      for (int base = 0; base < n; base += ROWS_PER_PASS) {
        const int i = base + my_rg;
        const bool act = i < n;
        const cplx f = act ? P[i * PP + jj] : cmk(0.0, 0.0);
        const cplx x = act ? P[i * PP + my_col] : cmk(0.0, 0.0);
        __syncwarp();
        if (act && my_col < w) {
          cplx o;
          if (i == p) o = (my_col == jj) ? d : pd;
          else o = (my_col == jj) ? cneg(cmul(f, d)) : csub(x, cmul(f, pd));
          P[i * PP + my_col] = o;
        }
        __syncwarp();
      }
      __syncthreads();
    }

    // ---- apply the panel to every other column, one 64-wide column tile at a time
    const int wm = (warp >> 2) * 32, wn = (warp & 3) * 16;
    for (int c0 = 0; c0 < n; c0 += GT_N) {
      const int c1 = min(c0 + GT_N, n);
      if (c0 >= p0 && c1 <= p0 + w) continue;  // tile lies inside the panel
      for (int e = tid; e < NB * GT_N; e += CTA_THREADS) {
        int kk = e / GT_N, cc = e % GT_N;
        cplx v = cmk(0.0, 0.0);
        if (kk < w && c0 + cc < n) v = W[(int64_t)piv[p0 + kk] * ldw + c0 + cc];
        R[kk * RP + cc] = v;
      }
      __syncthreads();
      for (int r0 = 0; r0 < n; r0 += GT_M) {
        Acc3M acc;
        acc.zero();
        warp_mma_3m<false, false>(acc, P + (size_t)r0 * PP, R, NB / 4, wm, wn, lane, PanelIdx{PP}, RIdx());
        acc_foreach(acc, wm, wn, lane, [&](int r, int cc, cplx v) {
          int i = r0 + r, col = c0 + cc;
          if (i < n && col < n && (col < p0 || col >= p0 + w)) {
            int lc = pinv[i];
            bool is_piv = (lc >= p0 && lc < p0 + w);
            cplx* dst = W + (int64_t)i * ldw + col;
            *dst = is_piv ? v : cadd(*dst, v);
          }
        });
      }
      __syncthreads();
    }
    // ---- write the factorised panel back
    for (int e = tid; e < n * NB; e += CTA_THREADS) {
      int i = e / NB, jj = e % NB;
      if (jj < w) W[(int64_t)i * ldw + p0 + jj] = P[i * PP + jj];
    }
    __syncthreads();
  }

  // ---- undo the implicit pivoting while storing: G[i][j] = W[p(i)][p^-1(j)]
  for (int e = tid; e < n * n; e += CTA_THREADS) {
    int i = e / n, j = e % n;
    G[(int64_t)i * ldg + j] = W[(int64_t)piv[i] * ldw + pinv[j]];
  }
  const int flag = s_misc[1];
  __syncthreads();
  return flag;
}

// Shared-memory bytes cta_inverse needs for an n x n matrix.
NEGF_DEV size_t inv_smem_bytes(int n) {
  return n <= 256 ? InvLayout<32>::bytes(n) : InvLayout<16>::bytes(n);
}

NEGF_DEV int cta_inverse(cplx* W, int64_t ldw, int n, cplx* G, int64_t ldg, char* smem_raw) {
  if (n <= 256) return cta_inverse_nb<32>(W, ldw, n, G, ldg, smem_raw);
  return cta_inverse_nb<16>(W, ldw, n, G, ldg, smem_raw);
}

}  // namespace negf
