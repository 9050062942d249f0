// CTA-wide complex128 matrix inverse: two-level blocked Gauss-Jordan with
// partial pivoting on FP64 tensor cores.
//
// The matrix W (n x n, row stride ldw) is a work buffer in global memory and
// is destroyed; the inverse is written to G.  Pivoting is implicit: rows never
// move in memory.  For logical column c the pivot is the unused physical row
// p(c) of largest |re|+|im| (LAPACK's izamax measure).  The sweep leaves the
// accumulated row transform T (T A = the pivot-row permutation of I) stored
// in place: column c of W holds column p(c) of T.  Since row i of A^-1 is row
// p(i) of T, the inverse is recovered by the gather
//     G[i][j] = W[p(i)][p^-1(j)],
// fused into the final store.
//
// Blocking.  Columns are taken in outer blocks of OB = 128 (the whole matrix
// when n <= 128).  Inside a block, panels of NB columns are factorised in
// shared memory and applied to the block's other columns only (rank-NB
// updates, k = NB).  The finished block transform is then applied to every
// column outside the block with one GEMM of depth k = OB at full tile-GEMM
// efficiency:
//     W[:, c] <- W[:, block] * W[block pivots, c] + (W[:, c] with the block's pivot rows zeroed),
// reading the block's pivot rows from a snapshot (they are overwritten by the
// same update).  Work: n^3 complex multiply-adds, as for an explicit inverse
// by LU.
//
// Panel factorisation in registers: every thread holds whole panel rows
// (row tid + 256 r, NB complex entries), so a column step is one broadcast of
// the scaled pivot row through shared memory and register-only updates; the
// pivot search for the next column uses the entries each thread just
// produced.  Two barriers per column.
#pragma once
#include "cta_gemm_tc.cuh"

namespace negf {

#ifndef NEGF_INV_SMALL_NB
#define NEGF_INV_SMALL_NB 8
#endif
// Panel width of the Gauss-Jordan inverse for blocks of n <= 64 (the block inverse's leaves).
// Measured against 16-wide panels (every SM inverting its own matrices): 4-9 % faster for
// n = 32..64, 2-3 % for the block inverse of n = 128..192, equal at n = 256 and n = 16.
constexpr int INV_SMALL_NB = NEGF_INV_SMALL_NB;
static_assert(INV_SMALL_NB == 8 || INV_SMALL_NB == 16, "8- or 16-wide panels for small blocks");
constexpr int INV_OB = 128;      // default outer block (columns) of the two-level Gauss-Jordan
constexpr int INV_OB_MAX = 512;  // widest outer block (one block: no outer update for n <= 512)

// Shared memory: panel, R tiles, pivot row and multiplier columns, then the
// integer maps (piv, pinv, reductions).  The maps start above the outer
// update's GEMM staging area (the DMMA ring, or the tcgen05 planes with TC),
// which that GEMM overwrites while the update epilogue still reads pinv.
template <int NB>
struct InvLayout {
  static constexpr int PP = NB + 4;  // panel pitch (= 4 mod 8: conflict-free A fragments)
  static constexpr int RP = GT_N + 2;
  __host__ __device__ static int rows(int n) { return (n + GT_M - 1) / GT_M * GT_M; }
  __host__ __device__ static size_t panel_bytes(int n) {
    size_t b = (size_t)rows(n) * PP * sizeof(double2) + 2 * (size_t)NB * RP * sizeof(double2);
    return b + 2 * (size_t)rows(n) * sizeof(double2) + NB * sizeof(double2);  // multiplier columns, spare row
  }
  __host__ __device__ static size_t maps_offset(int n, bool tc) {
    const size_t b = panel_bytes(n), g = tc ? (size_t)TC_SMEM_BYTES : (size_t)GEMM_SMEM_BYTES;
    return b < g ? g : b;
  }
  __host__ __device__ static size_t bytes(int n, bool tc) {
    return maps_offset(n, tc) + (size_t)(2 * n + 64) * sizeof(int) + 16 * sizeof(double);
  }
};

// Largest footprint over every block size up to max_n: blocks of 65..256 use
// 32-wide panels, the others 16-wide panels, and a device may mix both.
inline size_t inv_smem_bytes_host(int max_n, bool tc = false) {
  size_t a = InvLayout<32>::bytes(max_n < 256 ? max_n : 256, tc);
  const size_t s = InvLayout<INV_SMALL_NB>::bytes(max_n < 64 ? max_n : 64, tc);
  if (s > a) a = s;
  if (max_n > 256) {
    const size_t b = InvLayout<16>::bytes(max_n, tc);
    if (b > a) a = b;
  }
  size_t g = tc ? (size_t)TC_SMEM_BYTES : (size_t)GEMM_SMEM_BYTES;  // the outer update runs a CTA GEMM
  return a > g ? a : g;
}

// Complex elements of the pivot-row snapshot the inverse needs (INV_OB x n).
__host__ __device__ inline size_t inv_snapshot_elems(int n) { return (size_t)INV_OB * n; }

struct PanelIdx {
  int pitch;
  NEGF_DEV int operator()(int m, int k) const { return m * pitch + k; }
};
struct RIdx {
  NEGF_DEV int operator()(int k, int n) const { return k * (GT_N + 2) + n; }
};

// argmax over (value, index) pairs: larger value wins, ties go to the lower index
NEGF_DEV void argmax_merge(double& v, int& i, double ov, int oi) {
  if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
}
NEGF_DEV void warp_argmax(double& v, int& i) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    double ov = __shfl_xor_sync(0xffffffffu, v, off);
    int oi = __shfl_xor_sync(0xffffffffu, i, off);
    argmax_merge(v, i, ov, oi);
  }
}
NEGF_DEV double pivot_measure(cplx a) {
  double v = cabs1(a);
  return (v == v) ? v : INFINITY;  // NaN pivots are taken (and flagged) first
}

// The same search on integer keys: a pivot measure is >= 0 or +inf, and for such doubles the
// order of the IEEE bit patterns read as signed 64-bit integers is the numeric order, so the
// winner (ties to the lower index) is the one the double comparison picks, while the compares
// and shuffles stay on the integer pipes instead of the long-latency FP64 ones.  -1 is "no
// candidate"; a key <= 0 (zero pivot) or >= PIVOT_KEY_INF (infinite or NaN) is singular.
constexpr long long PIVOT_KEY_INF = 0x7ff0000000000000LL;
NEGF_DEV long long pivot_key(cplx a) { return __double_as_longlong(pivot_measure(a)); }
NEGF_DEV void argmax_merge_key(long long& v, int& i, long long ov, int oi) {
  if (ov > v || (ov == v && oi < i)) { v = ov; i = oi; }
}
NEGF_DEV void warp_argmax_key(long long& v, int& i) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    const long long ov = __shfl_xor_sync(0xffffffffu, v, off);
    const int oi = __shfl_xor_sync(0xffffffffu, i, off);
    argmax_merge_key(v, i, ov, oi);
  }
}
NEGF_DEV bool pivot_key_singular(long long k) { return k <= 0 || k >= PIVOT_KEY_INF; }

// Outer-update epilogue: pivot rows of the block take the product, the other
// rows add it to their current value.
struct EpiGJ {
  cplx* W;
  int64_t ldw;
  const int* pinv;
  int c_lo, c_hi, col0;
  NEGF_DEV void operator()(int m, int n, cplx v) const {
    cplx* dst = W + (int64_t)m * ldw + col0 + n;
    const int lc = pinv[m];
    *dst = (lc >= c_lo && lc < c_hi) ? v : cadd(*dst, v);
  }
};

// Returns 0 on success, 1 if a zero or non-finite pivot was met.  Uniform
// across the CTA; ends with __syncthreads().  `snap` is global scratch of
// inv_snapshot_elems(n) complex elements (unused when n <= INV_OB).  TC runs
// the outer update on the tcgen05 3xTF32 GEMM (FP32-accurate products).
template <int NB, int RT, bool G3, bool TC>
__device__ __noinline__ int cta_inverse_nb(cplx* W, int64_t ldw, int n, cplx* G, int64_t ldg, char* smem_raw,
                                           PhaseClock* pc, cplx* snap, int ob_max) {
  constexpr int PP = InvLayout<NB>::PP;
  constexpr int RP = InvLayout<NB>::RP;
  constexpr int NWARP = CTA_THREADS / 32;
  static_assert(NB * RT <= 32, "a thread holds RT panel rows of NB complex entries (n <= 256 RT)");
  const int n_pad = InvLayout<NB>::rows(n);
  cplx* P = reinterpret_cast<cplx*>(smem_raw);
  cplx* Rb[2] = {P + (size_t)n_pad * PP, P + (size_t)n_pad * PP + NB * RP};
  cplx* qrow = Rb[1] + NB * RP;  // [NB] published pivot row of the current column
  int* piv = reinterpret_cast<int*>(smem_raw + InvLayout<NB>::maps_offset(n, TC));  // logical column -> physical row
  int* pinv = piv + n;                           // physical row -> logical column (-1: unused)
  int* red_i = pinv + n;                         // [2][NWARP] pivot candidates (double buffered)
  int* s_misc = red_i + 2 * NWARP;               // [1]: singular flag
  long long* red_v = reinterpret_cast<long long*>(s_misc + 48);  // [2][NWARP] pivot keys
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp >> 2) * 32, wn = (warp & 3) * 16;
  // Panel rows owned by this thread: tid + 256 r, r < RT (n <= 256 RT).
  // Bit r of `used` is set once that row has served as a pivot.
  unsigned used = 0u;
  int par = 0;

  for (int i = tid; i < n; i += CTA_THREADS) pinv[i] = -1;
  if (tid == 0) s_misc[1] = 0;
  __syncthreads();

  // Every thread merges the per-warp candidates (one barrier per pivot) and
  // marks the winner as used; thread 0 records it for the updates and gather.
  auto choose_pivot = [&](long long v, int i, int c) -> int {
    warp_argmax_key(v, i);
    if (lane == 0) { red_v[par * NWARP + warp] = v; red_i[par * NWARP + warp] = i; }
    __syncthreads();
    long long bv = red_v[par * NWARP];
    int bi = red_i[par * NWARP];
#pragma unroll
    for (int k = 1; k < NWARP; ++k) argmax_merge_key(bv, bi, red_v[par * NWARP + k], red_i[par * NWARP + k]);
    par ^= 1;
    if (tid == 0) {
      if (pivot_key_singular(bv)) s_misc[1] = 1;
      piv[c] = bi;
      pinv[bi] = c;
    }
    if (bi % CTA_THREADS == tid) used |= 1u << (bi / CTA_THREADS);
    return bi;
  };

  const int ob = n <= ob_max ? n : ob_max;
  for (int c_lo = 0; c_lo < n; c_lo += ob) {
    const int c_hi = min(c_lo + ob, n);
    for (int p0 = c_lo; p0 < c_hi; p0 += NB) {
      const int w = min(NB, c_hi - p0);
      // ---- stage the panel W[:, p0:p0+w) (zero padded to NB columns, n_pad rows)
      for (int e = tid; e < n_pad * NB; e += CTA_THREADS) {
        int i = e / NB, jj = e % NB;
        bool v = (jj < w && i < n);
        cp_async16(P + i * PP + jj, v ? W + (int64_t)i * ldw + p0 + jj : W, v);
      }
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
      // each thread takes its rows (tid + 256 r) of the panel into registers
      cplx row[RT][NB];
      cplx mm[RT];  // the rows' entries in the column being eliminated
      long long bv = -1;
      int bi = n;
#pragma unroll
      for (int r = 0; r < RT; ++r) {
        const int i = tid + CTA_THREADS * r;
#pragma unroll
        for (int k = 0; k < NB; ++k) row[r][k] = (i < n) ? P[i * PP + k] : cmk(0.0, 0.0);
        mm[r] = row[r][0];
        if (i < n && !((used >> r) & 1u)) argmax_merge_key(bv, bi, pivot_key(mm[r]), i);
      }
      int p = choose_pivot(bv, bi, p0);
      pc->mark(PH_INV_STAGE);

      // ---- unblocked Gauss-Jordan on the panel, in registers.  Column jj:
      // the pivot row's owner publishes q_k = P[p][k]/P[p][jj] (q_jj = 1/P[p][jj])
      // and keeps it as its row; every other row i does
      //     P[i][k] <- (k == jj ? 0 : P[i][k]) - m_i q_k,   m_i = P[i][jj],
      // and hands the next column's entry to the pivot search.
      for (int jj = 0; jj < w; ++jj) {
#pragma unroll
        for (int r = 0; r < RT; ++r) {
          if (tid + CTA_THREADS * r == p) {
            const cplx d = crcp(mm[r]);
#pragma unroll
            for (int k = 0; k < NB; ++k) {
              const cplx q = (k == jj) ? d : cmul(row[r][k], d);
              row[r][k] = q;
              qrow[k] = q;
            }
          }
        }
        __syncthreads();
        const int nxt = jj + 1;
        bv = -1;
        bi = n;
#pragma unroll
        for (int r = 0; r < RT; ++r) {
          const int i = tid + CTA_THREADS * r;
          cplx mnext = cmk(0.0, 0.0);
          if (i < n) {
            if (i != p) {
              const cplx m = mm[r];
#pragma unroll
              for (int k = 0; k < NB; ++k) {
                const cplx q = qrow[k];
                const cplx x = (k == jj) ? cmk(0.0, 0.0) : row[r][k];
                const cplx o = csub(x, cmul(m, q));
                row[r][k] = o;
                if (k == nxt) mnext = o;
              }
            } else {
#pragma unroll
              for (int k = 0; k < NB; ++k)
                if (k == nxt) mnext = row[r][k];
            }
            if (nxt < w && i != p && !((used >> r) & 1u)) argmax_merge_key(bv, bi, pivot_key(mnext), i);
          }
          mm[r] = mnext;
        }
        if (nxt < w) p = choose_pivot(bv, bi, p0 + nxt);
        else __syncthreads();  // qrow is rewritten by the next panel's first column
      }
      // the factorised panel goes back to shared memory as the update's A operand
#pragma unroll
      for (int r = 0; r < RT; ++r) {
        const int i = tid + CTA_THREADS * r;
        if (i < n_pad) {
#pragma unroll
          for (int k = 0; k < NB; ++k) P[i * PP + k] = row[r][k];
        }
      }
      __syncthreads();
      pc->mark(PH_INV_PANEL);

      // ---- apply the panel to the block's other columns, one 64-wide tile at a time
      auto load_r = [&](cplx* Rt, int c0) {
        for (int e = tid; e < NB * GT_N; e += CTA_THREADS) {
          int kk = e / GT_N, cc = e % GT_N;
          bool v = (kk < w && c0 + cc < c_hi);
          const cplx* src = v ? W + (int64_t)piv[p0 + kk] * ldw + c0 + cc : W;
          cp_async16(Rt + kk * RP + cc, src, v);
        }
        cp_async_commit();
      };
      int tiles[INV_OB_MAX / GT_N + 1];
      int ntile = 0;
      for (int c0 = c_lo; c0 < c_hi; c0 += GT_N) {
        const int c1 = min(c0 + GT_N, c_hi);
        if (!(c0 >= p0 && c1 <= p0 + w)) tiles[ntile++] = c0;
      }
      if (ntile > 0) load_r(Rb[0], tiles[0]);
      for (int t = 0; t < ntile; ++t) {
        const int c0 = tiles[t];
        cplx* Rt = Rb[t & 1];
        if (t + 1 < ntile) load_r(Rb[(t + 1) & 1], tiles[t + 1]);
        else cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        for (int r0 = 0; r0 < n; r0 += GT_M) {
          // fetch this warp's slice of W (the addend) ahead of the tensor-core work
          cplx old[2][2][4];
#pragma unroll
          for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                int row = r0 + acc_row(i, e, wm, lane), col = c0 + acc_col(j, e, wn, lane);
                old[i][j][e] = cmk(0.0, 0.0);
                if (row < n && col < c_hi) old[i][j][e] = ldg_early(W + (int64_t)row * ldw + col);
              }
          Acc3M acc;
          acc.zero();
          warp_mma_3m<false, false, G3>(acc, P + (size_t)r0 * PP, Rt, NB / 8, wm, wn, lane, PanelIdx{PP}, RIdx());
#pragma unroll
          for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
              for (int e = 0; e < 4; ++e) {
                int row = r0 + acc_row(i, e, wm, lane), col = c0 + acc_col(j, e, wn, lane);
                if (row < n && col < c_hi && (col < p0 || col >= p0 + w)) {
                  cplx v = acc_value<G3>(acc, i, j, e);
                  int lc = pinv[row];
                  bool is_piv = (lc >= p0 && lc < p0 + w);
                  W[(int64_t)row * ldw + col] = is_piv ? v : cadd(old[i][j][e], v);
                }
              }
        }
        __syncthreads();  // R[t & 1] is refilled two tiles later
      }
      cp_async_wait<0>();
      // ---- write the factorised panel back
      for (int e = tid; e < n * NB; e += CTA_THREADS) {
        int i = e / NB, jj = e % NB;
        if (jj < w) W[(int64_t)i * ldw + p0 + jj] = P[i * PP + jj];
      }
      __syncthreads();
      pc->mark(PH_INV_UPDATE);
    }

    // ---- apply the block transform to the columns outside the block (k = block width)
    if (ob < n) {
      const int kb = c_hi - c_lo;
#pragma unroll 4
      for (int e = tid; e < kb * n; e += CTA_THREADS) {
        int kk = e / n, c = e % n;
        snap[e] = W[(int64_t)piv[c_lo + kk] * ldw + c];
      }
      __syncthreads();
      if (c_lo > 0) {
        GemmArgs g = gemm_args(n, c_lo, kb, W + c_lo, ldw, snap, n, W, ldw);
        if constexpr (TC) cta_gemm_tc_epi<OP_N, OP_N>(g, smem_raw, EpiGJ{W, ldw, pinv, c_lo, c_hi, 0});
        else cta_gemm_epi<OP_N, OP_N, G3>(g, reinterpret_cast<cplx*>(smem_raw), EpiGJ{W, ldw, pinv, c_lo, c_hi, 0});
      }
      if (c_hi < n) {
        GemmArgs g = gemm_args(n, n - c_hi, kb, W + c_lo, ldw, snap + c_hi, n, W + c_hi, ldw);
        if constexpr (TC) cta_gemm_tc_epi<OP_N, OP_N>(g, smem_raw, EpiGJ{W, ldw, pinv, c_lo, c_hi, c_hi});
        else cta_gemm_epi<OP_N, OP_N, G3>(g, reinterpret_cast<cplx*>(smem_raw), EpiGJ{W, ldw, pinv, c_lo, c_hi, c_hi});
      }
      pc->mark(PH_INV_UPDATE);
    }
  }

  // ---- undo the implicit pivoting while storing: G[i][j] = W[p(i)][p^-1(j)]
#pragma unroll 4
  for (int e = tid; e < n * n; e += CTA_THREADS) {
    int i = e / n, j = e % n;
    G[(int64_t)i * ldg + j] = W[(int64_t)piv[i] * ldw + pinv[j]];
  }
  const int flag = s_misc[1];
  __syncthreads();
  pc->mark(PH_INV_GATHER);
  return flag;
}

// G3: complex products of the rank updates (Gauss/3M or conventional 4M);
// TC: outer update on the tensor-core 3xTF32 GEMM.  ob: outer block width,
// a multiple of 32 up to INV_OB_MAX (narrower blocks move work from the
// panels' rank-NB updates to the outer GEMM; ob >= n leaves no outer update).
// With ob < n the snapshot needs ob x n complex elements.
template <bool G3 = true, bool TC = false>
NEGF_DEV int cta_inverse(cplx* W, int64_t ldw, int n, cplx* G, int64_t ldg, char* smem_raw, PhaseClock* pc,
                         cplx* snap, int ob = INV_OB) {
  // Narrow panels for small blocks (the block inverse's 64-wide leaves): a column step's
  // latency chain is shorter (16-wide measured 22 % faster than 32-wide at n = 64, 8 % at
  // n = 128, where the rank-16 updates start to cost more; 8-wide another 4-9 % for n <= 64).
  // One register row per thread up to n = 256.
  if (n > 64 && n <= 256) return cta_inverse_nb<32, 1, G3, TC>(W, ldw, n, G, ldg, smem_raw, pc, snap, ob);
  if (n <= 64) return cta_inverse_nb<INV_SMALL_NB, 1, G3, TC>(W, ldw, n, G, ldg, smem_raw, pc, snap, ob);
  return cta_inverse_nb<16, 2, G3, TC>(W, ldw, n, G, ldg, smem_raw, pc, snap, ob);
}

}  // namespace negf
