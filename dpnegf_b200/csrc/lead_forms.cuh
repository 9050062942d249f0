// CTA helpers shared by the lead kernels (lopez_sancho.cu, products.cu): the
// energy-shifted lead blocks, a CTA max reduction, the conventional-4M tile GEMM
// the lead iterations use, and an explicit inverse from the pivoted LU.
#pragma once
#include "cta_lu.cuh"
#include "cta_stream.cuh"

namespace negf {

// out[i][j] = conj(X[j][i]) - z conj(Y[j][i])   (n x n), i.e. X^H - z Y^H
NEGF_DEV void form_herm_shift(cplx* out, const cplx* X, const cplx* Y, cplx z, int n) {
#pragma unroll 4
  for (int e = threadIdx.x; e < n * n; e += CTA_THREADS) {
    int i = e / n, j = e % n;
    cplx x = cconj(X[(int64_t)j * n + i]), y = cconj(Y[(int64_t)j * n + i]);
    out[e] = csub(x, cmul(z, y));
  }
  __syncthreads();
}

// out[i][j] = z conj(S[j][i]) - conj(H[j][i])   for an (rows x cols) H/S pair
// stored (cols x rows): E S^H - H^H.
NEGF_DEV void form_eS_minus_h_herm(cplx* out, const cplx* H, const cplx* S, cplx z, int rows, int cols) {
  for (int e = threadIdx.x; e < rows * cols; e += CTA_THREADS) {
    int i = e / cols, j = e % cols;
    cplx h = cconj(H[(int64_t)j * rows + i]), s = cconj(S[(int64_t)j * rows + i]);
    out[e] = csub(cmul(z, s), h);
  }
  __syncthreads();
}

// Max of v over the CTA (NaN-free inputs); begins and ends with a barrier.
NEGF_DEV double cta_max(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double m = red[0];
  for (int w = 1; w < CTA_THREADS / 32; ++w) m = fmax(m, red[w]);
  __syncthreads();
  return m;
}

// C = alpha op(A) op(B) (+ beta D when D is given).  By default conventional 4M complex products
// (see warp_mma_3m): the decimation squares and accumulates products, which amplifies the looser
// componentwise error of Gauss/3M products; G3 = true selects Gauss/3M where no iteration feeds
// rounding back into the result.  Lead blocks come in every size, so warps outside the product
// skip their MMAs.
template <int OPA, int OPB, bool G3 = false>
NEGF_DEV void gemm_ls(cplx* smem, int M, int N, int K, const cplx* A, int64_t lda, const cplx* B, int64_t ldb,
                      cplx* C, int64_t ldc, const cplx* D = nullptr, int64_t ldd = 0,
                      cplx alpha = cmk(1.0, 0.0), cplx beta = cmk(1.0, 0.0)) {
  GemmArgs g = gemm_args(M, N, K, A, lda, B, ldb, C, ldc);
  g.alpha = alpha;
  if (D) { g.D = D; g.ldd = ldd; g.beta = beta; g.use_d = true; }
  cta_gemm<OPA, OPB, G3, true>(g, smem);
}

// out = W^-1 (n x n, row stride n) by the LU solve against I (numpy.linalg.inv's route); W is
// destroyed.  Returns 1 on a zero or non-finite pivot.
NEGF_DEV int cta_lu_inverse(cplx* W, cplx* out, int n, char* smem_raw) {
  const int64_t n2 = (int64_t)n * n;
  const int f = cta_lu_factor(W, n, n, smem_raw);
  const int* perm = cta_lu_perm(smem_raw, n);
  for (int64_t e = threadIdx.x; e < n2; e += CTA_THREADS) out[e] = cmk(perm[e / n] == e % n ? 1.0 : 0.0, 0.0);
  __syncthreads();
  cta_lu_trsolve(W, n, n, out, n, n, smem_raw);
  return f;
}

// Shared memory of a lead kernel: the GEMM ring, the LU workspace and the streaming forms.
inline size_t lead_smem_bytes(int max_n) {
  size_t a = GEMM_SMEM_BYTES, b = lu_smem_bytes_host(max_n), c = STREAM_SMEM_BYTES;
  size_t m = a > b ? a : b;
  return m > c ? m : c;
}

}  // namespace negf
