// Batched block-tridiagonal recursive Green's function (RGF) sweep, sm_100a.
//
// Persistent kernel: one CTA per work slot pulls (device, energy) items from
// an atomic queue and runs the whole sweep for that item -- forward
// left-connected inverses, backward retarded blocks, optional lesser blocks,
// and the T(E) / per-orbital DOS reductions -- keeping its intermediates in a
// private scratch slot.  All contractions go through the CTA tile GEMM and the
// blocked Gauss-Jordan inverse on FP64 tensor cores (cta_gemm.cuh,
// cta_inverse.cuh); the mixed-precision variant (NEGF_MIXED) runs every block
// product, including the inverse's outer update, on the tcgen05 3xTF32 GEMM
// (cta_gemm_tc.cuh) and keeps pivoting, panels and storage in FP64.  Its
// T(E) can be refined (NEGF_REFINE): one step of iterative refinement of the
// column X = G_{:,N} with an FP64 residual, see rgf_item.
//
// Follows negf/recursive_green_cal.py (dpnegf):
//   forward   g_0 = (-D_0)^-1,  g_q = (-D_q - L_{q-1} g_{q-1} U_{q-1})^-1     :88-94
//   backward  gU = g_q U_q;  G_{q+1,q} = G_{q+1,q+1} L_q g_q;
//             G_{q,q+1} = gU G_{q+1,q+1};  G_qq = g_q + gU G_{q+1,q};
//             G_{q,N} = gU G_{q+1,N}                                           :98-114
//   lesser    gin_0 = g_0 s_0 g_0^H;  gin_{q+1} = g_{q+1}(s_{q+1} + L gin_q U) g_{q+1}^H
//             gnl_q = G_{q+1,q+1} L gin_q + gnd_{q+1} L g_q^H
//             gnd_q = gin_q + g_q U gnd_{q+1} L g_q^H + gin_q U G_{q,q+1}^H
//                     + G_{q,q+1} L gin_q;  gnu_q = gnl_q^H                      :121-140
//   greater   gip_0 = g_0 s'_0 g_0^*;  gip_{q+1} = g_{q+1}(s'_{q+1} + L gip_q U^*) g_{q+1}^*
//             gpl_q = G_{q+1,q+1} L gip_q + gpd_{q+1} L^* g_q^*
//             gpd_q = gip_q + g_q U gpd_{q+1} L^* g_q^* + gip_q U^* G_{q+1,q}^*
//                     + G_{q,q+1} L gip_q;  gpu_q = gpl_q^H                      :143-161
//             (^* is the elementwise conjugate, exactly as the reference writes it)
// with D = H + Sigma - zS, L = hl - z sl, U = hu - z su (:75-78), and the
// reductions of negf/device_property.py: T = Re Tr[G_L G_1N G_R G_1N^H]
// (:374-406) and -Im diag(G_qq S_qq + G_{q,q+1} S_{q+1,q} + G_{q,q-1} S_{q-1,q})/pi
// per orbital (:408-470).
#pragma once
#include <cstdio>
#include "../../include/negf_b200.h"
#include "cta_inverse.cuh"
#include "cta_stream.cuh"

namespace negf {

constexpr int RGF_NBUF = 18;  // per-slot max_n^2 work buffers (see SlotBufs)

struct SlotBufs {
  cplx* gslab;    // g_q storage when gr_left is not an output
  cplx* ginslab;  // lesser gin_q storage when gin_left is not an output
  cplx* grdslab;  // adjoint: G_qq of every block (when grd is not an output)
  cplx* colslab;  // adjoint / refinement: G_qN of every block (when gr_lc is not an output)
  cplx* yslab;    // refinement: forward-substituted residual y_q of every block
  cplx* gipslab;  // greater gip_q storage when gip_left is not an output
  cplx* Pd;       // greater: gpd_{q+1} when gpd is not an output
  cplx* gdslab;   // density gradient: z-tangent dg_q/dz of every block
  cplx *D0, *D1;  // density gradient: dG_qq/dz of the current / next block
  cplx *W, *T1, *Lz, *Uz, *gU, *Gd, *Gl, *Gu, *Gt0, *Gt1, *tA, *tB, *tC, *tD;
  cplx *Nd, *Nl, *Nu, *tE;  // lesser work
};

// Elements of the g slab (and of the z-tangent slab): every g_q, or with sqrt(K) checkpointing
// (NEGF_ADJOINT, ckpt = s > 0) the checkpoints g_0, g_s, ... plus one segment of s blocks.
__host__ __device__ inline size_t rgf_g_elems(const NegfRgfProblem& p) {
  const size_t mn2 = (size_t)p.max_n * p.max_n;
  if ((p.flags & NEGF_ADJOINT) && p.ckpt > 0)
    return ((size_t)(p.ckpt_blocks + p.ckpt - 1) / p.ckpt + p.ckpt) * mn2;
  return (size_t)p.max_g_slab;
}

__host__ __device__ inline size_t rgf_slot_elems(const NegfRgfProblem& p) {
  size_t mn2 = (size_t)p.max_n * p.max_n;
  size_t e = RGF_NBUF * mn2;
  if (!(p.flags & NEGF_OUT_GR_LEFT)) e += rgf_g_elems(p);
  if (p.flags & NEGF_LESSER) e += (size_t)p.max_g_slab;
  if (p.flags & NEGF_ADJOINT) e += (size_t)p.max_g_slab;
  if (p.flags & (NEGF_ADJOINT | NEGF_REFINE)) e += (size_t)p.col_slab;
  if (p.flags & NEGF_REFINE) e += (size_t)p.col_slab;
  if (p.flags & NEGF_GREATER) e += (size_t)p.max_g_slab + mn2;
  if ((p.flags & NEGF_ADJOINT) && (p.flags & NEGF_ADJ_DOS)) e += rgf_g_elems(p) + 2 * mn2;
  return (e + 15) & ~(size_t)15;  // keep slots 256-byte aligned
}
constexpr size_t RGF_SCRATCH_HEADER = 256;  // work-queue counter
constexpr double REFINE_TOL = 1e-10;        // relative correction of G_1N that ends the refinement

NEGF_DEV SlotBufs slot_bufs(const NegfRgfProblem& p, int slot) {
  cplx* base = reinterpret_cast<cplx*>(reinterpret_cast<char*>(p.scratch) + RGF_SCRATCH_HEADER) +
               (size_t)slot * rgf_slot_elems(p);
  size_t mn2 = (size_t)p.max_n * p.max_n;
  SlotBufs s;
  cplx* b = base;
  cplx** bufs[RGF_NBUF] = {&s.W, &s.T1, &s.Lz, &s.Uz, &s.gU, &s.Gd, &s.Gl, &s.Gu, &s.Gt0,
                           &s.Gt1, &s.tA, &s.tB, &s.tC, &s.tD, &s.Nd, &s.Nl, &s.Nu, &s.tE};
  for (int i = 0; i < RGF_NBUF; ++i) { *bufs[i] = b; b += mn2; }
  s.gslab = nullptr;
  s.ginslab = nullptr;
  s.grdslab = nullptr;
  s.colslab = nullptr;
  s.yslab = nullptr;
  s.gipslab = nullptr;
  s.Pd = nullptr;
  s.gdslab = s.D0 = s.D1 = nullptr;
  if (!(p.flags & NEGF_OUT_GR_LEFT)) { s.gslab = b; b += rgf_g_elems(p); }
  if (p.flags & NEGF_LESSER) { s.ginslab = b; b += p.max_g_slab; }
  if (p.flags & NEGF_ADJOINT) { s.grdslab = b; b += p.max_g_slab; }
  if (p.flags & (NEGF_ADJOINT | NEGF_REFINE)) { s.colslab = b; b += p.col_slab; }
  if (p.flags & NEGF_REFINE) { s.yslab = b; b += p.col_slab; }
  if (p.flags & NEGF_GREATER) {
    s.gipslab = b; b += p.max_g_slab;
    s.Pd = b; b += mn2;
  }
  if ((p.flags & NEGF_ADJOINT) && (p.flags & NEGF_ADJ_DOS)) {
    s.gdslab = b; b += rgf_g_elems(p);
    s.D0 = b; b += mn2;
    s.D1 = b; b += mn2;
  }
  return s;
}

// Out = X - z Y  ([m x n]); a missing X or Y (offset -1) is a zero block.
NEGF_DEV void form_shift(cplx* out, const cplx* hs, int64_t ox, int64_t oy, cplx z, int m, int n, cplx* smem) {
  cta_shift_form(out, ox >= 0 ? hs + ox : nullptr, oy >= 0 ? hs + oy : nullptr, z, cmk(1.0, 0.0), m * n, smem);
}

// W = z S - H - (Sigma_L in the top-left corner) - (Sigma_R in the bottom-right
// corner); the corner rule is recursive_green_cal.py:411-428.
NEGF_DEV void form_a0(cplx* W, const cplx* hs, const NegfBlock& b, cplx z, const cplx* seL, int nsl,
                      const cplx* seR, int nsr, cplx* smem) {
  const int n = b.n, tid = threadIdx.x;
  cta_shift_form(W, hs + b.hd, hs + b.sd, z, cmk(-1.0, 0.0), n * n, smem);
  const int cl = seL ? min(n, nsl) : 0;
  const int cr = seR ? min(n, nsr) : 0;
  for (int e = tid; e < cl * cl; e += CTA_THREADS) {
    int i = e / cl, j = e % cl;
    W[(int64_t)i * n + j] = csub(W[(int64_t)i * n + j], seL[(int64_t)i * nsl + j]);
  }
  __syncthreads();  // a block can carry both corners (K = 1)
  for (int e = tid; e < cr * cr; e += CTA_THREADS) {
    int i = e / cr, j = e % cr;
    int64_t w = (int64_t)(n - cr + i) * n + (n - cr + j);
    W[w] = csub(W[w], seR[(int64_t)(nsr - cr + i) * nsr + (nsr - cr + j)]);
  }
  __syncthreads();
}

NEGF_DEV void copy_mat(cplx* dst, const cplx* src, int m, int n, cplx* smem) {
  cta_shift_form(dst, src, nullptr, cmk(0.0, 0.0), cmk(1.0, 0.0), m * n, smem);
}

// dst[i] (+)= -Im( sum_j A[i][j] BT[i][j] ) / pi  = -Im diag(A B)_i / pi, with
// BT = B^T stored row-major (A and BT both rows x inner).  dst may be null;
// the row values are also summed into dsum (lane 0 of each warp).
NEGF_DEV void diag_im_acc(double* dst, double& dsum, const cplx* A, const cplx* BT, int rows, int inner,
                          bool init) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = warp; i < rows; i += CTA_THREADS / 32) {
    double acc = 0.0;
#pragma unroll 4
    for (int j = lane; j < inner; j += 32) {
      cplx a = A[(int64_t)i * inner + j], b = BT[(int64_t)i * inner + j];
      acc += a.x * b.y + a.y * b.x;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) {
      double v = -acc * 0.31830988618379067154;  // 1/pi
      dsum += v;
      if (dst) dst[i] = init ? v : dst[i] + v;
    }
  }
}

// Gamma = i (Sigma - Sigma^H) on the c x c corner of Sigma (ns x ns) at (r0, r0).
NEGF_DEV void form_gamma(cplx* out, const cplx* se, int ns, int r0, int c) {
  for (int e = threadIdx.x; e < c * c; e += CTA_THREADS) {
    int i = e / c, k = e % c;
    cplx a = se[(int64_t)(r0 + i) * ns + r0 + k], b = se[(int64_t)(r0 + k) * ns + r0 + i];
    cplx d = csub(a, cconj(b));
    out[e] = cmk(-d.y, d.x);
  }
}

NEGF_DEV double cta_max(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, off));
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = red[0];
  for (int w = 1; w < CTA_THREADS / 32; ++w) s = fmax(s, red[w]);
  __syncthreads();
  return s;
}

NEGF_DEV double cta_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < CTA_THREADS / 32; ++w) s += red[w];
  __syncthreads();
  return s;
}

// C = alpha op(A) op(B) (+ beta D) on the FP64 DMMA GEMM, or on the tcgen05
// 3xTF32 GEMM when MX.
template <int OPA, int OPB, bool MX>
NEGF_DEV void gemm(cplx* smem, int M, int N, int K, const cplx* A, int64_t lda, const cplx* B, int64_t ldb,
                   cplx* C, int64_t ldc, cplx alpha = cmk(1.0, 0.0), const cplx* D = nullptr,
                   int64_t ldd = 0, cplx beta = cmk(1.0, 0.0)) {
  GemmArgs g = gemm_args(M, N, K, A, lda, B, ldb, C, ldc);
  g.alpha = alpha;
  if (D) { g.D = D; g.ldd = ldd; g.beta = beta; g.use_d = true; }
  if constexpr (MX) cta_gemm_tc<OPA, OPB>(g, reinterpret_cast<char*>(smem));
  else cta_gemm<OPA, OPB>(g, smem);
}

template <int OPA, int OPB, bool MX, class Epi>
NEGF_DEV void gemm_epi(const GemmArgs& g, cplx* smem, const Epi& e) {
  if constexpr (MX) cta_gemm_tc_epi<OPA, OPB>(g, reinterpret_cast<char*>(smem), e);
  else cta_gemm_epi<OPA, OPB, true>(g, smem, e);
}

// Recursive 2x2 block inverse (inv_mode 1): G = W^-1, W destroyed.  With
// W = [[A11, A12], [A21, A22]] split at h:
//   X = A11^-1,  U = A21 X,  S = A22 - U A12,  Y = S^-1,  T = X A12,
//   G = [[X + T Y U, -T Y], [-Y U, Y]]
// X and Y recursively down to INVB_LEAF-wide leaves, which the pivoted
// Gauss-Jordan inverse handles; every other operation is a CTA GEMM, in place
// in W and G (U in G21, S in W22, T in W11 once A11 is consumed, -Y U via W21).
// Pivoting stays inside the leaves, so the leading blocks must be nonsingular:
// true for the retarded problem with eta > 0, whose matrices have a
// positive-definite imaginary part (so have all their leading blocks and
// Schur complements).  Work n^3 complex MACs, as for Gauss-Jordan.
constexpr int INVB_LEAF = 64;
template <int LV, bool MX>
__device__ __noinline__ int cta_inverse_blk(cplx* W, int64_t ldw, int n, cplx* G, int64_t ldg, cplx* smem,
                                           PhaseClock& pc, cplx* snap) {
  if constexpr (LV == 0) {
    return cta_inverse<true, MX>(W, ldw, n, G, ldg, reinterpret_cast<char*>(smem), &pc, snap, INV_OB_MAX);
  } else {
    if (n <= INVB_LEAF)
      return cta_inverse<true, MX>(W, ldw, n, G, ldg, reinterpret_cast<char*>(smem), &pc, snap, INV_OB_MAX);
    const int h = ((n + 1) / 2 + 7) & ~7, m = n - h;
    cplx *W11 = W, *W12 = W + h, *W21 = W + (int64_t)h * ldw, *W22 = W21 + h;
    cplx *G11 = G, *G12 = G + h, *G21 = G + (int64_t)h * ldg, *G22 = G21 + h;
    const cplx ONE = cmk(1.0, 0.0), MONE = cmk(-1.0, 0.0);
    int bad = cta_inverse_blk<LV - 1, MX>(W11, ldw, h, G11, ldg, smem, pc, snap);             // X
    gemm<OP_N, OP_N, MX>(smem, m, h, h, W21, ldw, G11, ldg, G21, ldg);                         // U = A21 X
    gemm<OP_N, OP_N, MX>(smem, m, m, h, G21, ldg, W12, ldw, W22, ldw, MONE, W22, ldw);         // S
    pc.mark(PH_INV_UPDATE);
    bad |= cta_inverse_blk<LV - 1, MX>(W22, ldw, m, G22, ldg, smem, pc, snap);               // Y
    gemm<OP_N, OP_N, MX>(smem, h, m, h, G11, ldg, W12, ldw, W11, ldw);                         // T = X A12
    gemm<OP_N, OP_N, MX>(smem, h, m, m, W11, ldw, G22, ldg, G12, ldg, MONE);                  // G12 = -T Y
    gemm<OP_N, OP_N, MX>(smem, h, h, m, G12, ldg, G21, ldg, G11, ldg, MONE, G11, ldg);       // X + T Y U
    gemm<OP_N, OP_N, MX>(smem, m, h, m, G22, ldg, G21, ldg, W21, ldw, MONE);                  // -Y U
    for (int e = threadIdx.x; e < m * h; e += CTA_THREADS) {
      const int i = e / h, j = e % h;
      G21[(int64_t)i * ldg + j] = W21[(int64_t)i * ldw + j];
    }
    __syncthreads();
    pc.mark(PH_INV_UPDATE);
    (void)ONE;
    return bad;
  }
}

// Residual probe of an inverse G of A (n x n, row stride n): with a fixed
// sign vector v (entries +-1 +-i from a hash of the index), y = G v and
// r = A y - v; true when max|r| <= tol n max|A| max|y| (a backward-stable
// inverse leaves about n u there) and everything is finite.  Whole CTA (the
// decision is uniform); y lives in smem.
NEGF_DEV bool inv_probe(const cplx* A, const cplx* G, int n, double tol, cplx* smem, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  auto v = [](int j) {
    const unsigned h = (unsigned)(j + 1) * 2654435761u;
    return cmk((h & 0x10000u) ? 1.0 : -1.0, (h & 0x20000u) ? 1.0 : -1.0);
  };
  cplx* y = smem;
  for (int i = warp; i < n; i += CTA_THREADS / 32) {
    cplx acc = cmk(0.0, 0.0);
    for (int j = lane; j < n; j += 32) acc = cfma(G[(int64_t)i * n + j], v(j), acc);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
    }
    if (lane == 0) y[i] = acc;
  }
  __syncthreads();
  double rmax = 0.0, amax = 0.0, ymax = 0.0;
  for (int i = warp; i < n; i += CTA_THREADS / 32) {
    cplx acc = cmk(0.0, 0.0);
    double am = 0.0;
    for (int j = lane; j < n; j += 32) {
      const cplx a = A[(int64_t)i * n + j];
      acc = cfma(a, y[j], acc);
      am = fmax(am, cabs1(a));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
      am = fmax(am, __shfl_xor_sync(0xffffffffu, am, off));
    }
    const double r = cabs1(csub(acc, v(i)));
    rmax = (r == r) ? fmax(rmax, r) : INFINITY;
    amax = fmax(amax, am);
    ymax = fmax(ymax, cabs1(y[i]));
  }
  rmax = cta_max(rmax, red);
  amax = cta_max(amax, red);
  ymax = cta_max(ymax, red);
  return rmax <= tol * (double)n * amax * ymax;
}

// Adjoint epilogue: W (rows of block q x cols of block p) contributes
// dL/dX_pq = 2c W^H to the H accumulator and -2c conj(z) W^H to the S one
// (X = H + Sigma - zS); the lead corners of the edge blocks also feed the
// self-energy gradients.
struct EpiGrad {
  cplx* gH;
  cplx* gS;
  int ldT;       // columns of the gradient block (= rows of W)
  double c2;     // 2 c
  cplx zc;       // conj(z)
  cplx* gseL;    // corner targets (null unless this W is the first / last diagonal block)
  int cl, nsl;
  cplx* gseR;
  int cr, nsr, r0;  // r0 = n_N - cr
  NEGF_DEV void operator()(int m, int n, cplx v) const {
    const cplx h = cscale(cconj(v), c2);
    const int64_t t = (int64_t)n * ldT + m;
    gH[t] = cadd(gH[t], h);
    gS[t] = csub(gS[t], cmul(zc, h));
    if (gseL && m < cl && n < cl) {
      cplx* d = gseL + (int64_t)n * nsl + m;
      *d = cadd(*d, h);
    }
    if (gseR && m >= r0 && n >= r0) {
      cplx* d = gseR + (int64_t)(nsr - cr + n - r0) * nsr + (nsr - cr + m - r0);
      *d = cadd(*d, h);
    }
  }
};

// One forward step of an item: g_q = (-D_q - L_{q-1} g_{q-1} U_{q-1})^-1 into gq from gprev
// (null for q = 0), and with dgq its z-tangent dg_q from dgprev.  Uses the slot's W, T1, Lz, Uz
// and tA..tE; leaves L_{q-1}, U_{q-1} in Lz, Uz and L_{q-1} g_{q-1} in T1 for the lesser and
// greater steps.  Inlined into the sweep; the checkpointed adjoint recomputes its segments
// through the non-inlined copy below.  Returns the singular-pivot flag.
template <bool MX>
NEGF_DEV int forward_block_body(const NegfRgfProblem& P, const NegfItem& it, const SlotBufs& sb,
                                char* smem_raw, double* red, PhaseClock& pc, int q,
                                const cplx* gprev, cplx* gq, const cplx* dgprev, cplx* dgq) {
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);
  const NegfDevice dv = P.devices[it.dev];
  const NegfBlock* blk = P.blocks + dv.blk0;
  const int K = dv.n_blocks;
  const cplx z = cmk(it.z_re, it.z_im);
  const cplx* hs = reinterpret_cast<const cplx*>(P.hs);
  const cplx* seL = reinterpret_cast<const cplx*>(it.se_l);
  const cplx* seR = reinterpret_cast<const cplx*>(it.se_r);
  const cplx ONE = cmk(1.0, 0.0), MONE = cmk(-1.0, 0.0);
  int bad = 0;
  const NegfBlock& b = blk[q];
  const int nq = b.n;
  form_a0(sb.W, hs, b, z, q == 0 ? seL : nullptr, it.nse_l, q == K - 1 ? seR : nullptr, it.nse_r, smem);
  if (q > 0) {
    const NegfBlock& bp = blk[q - 1];
    const int np = bp.n;
    form_shift(sb.Lz, hs, bp.hl, bp.sl, z, nq, np, smem);  // L_{q-1}: n_q x n_{q-1}
    form_shift(sb.Uz, hs, bp.hu, bp.su, z, np, nq, smem);  // U_{q-1}: n_{q-1} x n_q
    __syncthreads();
    pc.mark(PH_FORM);
    gemm<OP_N, OP_N, MX>(smem, nq, np, np, sb.Lz, np, gprev, np, sb.T1, np);
    gemm<OP_N, OP_N, MX>(smem, nq, nq, np, sb.T1, np, sb.Uz, nq, sb.W, nq, MONE, sb.W, nq);
    pc.mark(PH_GEMM_FWD);
  } else {
    __syncthreads();
    pc.mark(PH_FORM);
  }
  bool gj = P.inv_mode != 1;
  if (!gj) {
    // block inverse on a copy of W; a failed residual probe (or a singular leaf) falls
    // back to the pivoted Gauss-Jordan on the saved W
    copy_mat(sb.tD, sb.W, nq, nq, smem);
    const int bb = cta_inverse_blk<3, MX>(sb.W, nq, nq, gq, nq, smem, pc, sb.tE);
    if (bb || !inv_probe(sb.tD, gq, nq, MX ? 1e-4 : 1e-10, smem, red)) {
      copy_mat(sb.W, sb.tD, nq, nq, smem);
      gj = true;
    }
    pc.mark(PH_INV_GATHER);
  }
  if (gj)
    bad |= cta_inverse<true, MX>(sb.W, nq, nq, gq, nq, smem_raw, &pc, sb.tE,  // tE: pivot-row snapshot
                                 P.inv_ob > 0 ? P.inv_ob : INV_OB);
  if (dgq) {
    // dg_q/dz = -g_q Kd g_q with Kd = S_q - (L dg_{q-1} - sl g_{q-1}) U + (L g_{q-1}) su
    // (d/dz of g_q^-1 = zS_q - H_q - Sigma - L g U, dL/dz = -sl, dU/dz = -su; sb.T1 = L g_{q-1})
    const cplx* Kd = hs + b.sd;
    if (q > 0) {
      const NegfBlock& bp = blk[q - 1];
      const int np = bp.n;
      gemm<OP_N, OP_N, MX>(smem, nq, np, np, sb.Lz, np, dgprev, np, sb.tA, np);
      if (bp.sl >= 0) gemm<OP_N, OP_N, MX>(smem, nq, np, np, hs + bp.sl, np, gprev, np, sb.tA, np, MONE, sb.tA, np);
      gemm<OP_N, OP_N, MX>(smem, nq, nq, np, sb.tA, np, sb.Uz, nq, sb.tB, nq, MONE, hs + b.sd, nq);
      if (bp.su >= 0) gemm<OP_N, OP_N, MX>(smem, nq, nq, np, sb.T1, np, hs + bp.su, nq, sb.tB, nq, ONE, sb.tB, nq);
      Kd = sb.tB;
    }
    gemm<OP_N, OP_N, MX>(smem, nq, nq, nq, gq, nq, Kd, nq, sb.tC, nq);
    gemm<OP_N, OP_N, MX>(smem, nq, nq, nq, sb.tC, nq, gq, nq, dgq, nq, MONE);
    pc.mark(PH_GEMM_FWD);
  }
  return bad;
}

template <bool MX>
__device__ __noinline__ int rgf_forward_block(const NegfRgfProblem& P, const NegfItem& it, const SlotBufs& sb,
                                              char* smem_raw, double* red, PhaseClock& pc, int q,
                                              const cplx* gprev, cplx* gq, const cplx* dgprev, cplx* dgq) {
  return forward_block_body<MX>(P, it, sb, smem_raw, red, pc, q, gprev, gq, dgprev, dgq);
}

// Feature sets compiled into separate kernels, so a launch carries only the live state of
// the paths it can take (the T / DOS / block-output sweep sits at the 255-register cap).
enum RgfFeat : int {
  FEAT_RETARDED = 0,  // retarded blocks, T(E), DOS and per-orbital reductions, refinement
  FEAT_LESSER = 1,    // + lesser and greater sweeps
  FEAT_ADJOINT = 2    // + adjoint and density-gradient passes, checkpointing
};

template <bool MX, int FEAT>
NEGF_DEV void rgf_item(const NegfRgfProblem& P, const NegfItem& it, const SlotBufs& sb, char* smem_raw,
                       double* red, PhaseClock& pc) {
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);
  const NegfDevice dv = P.devices[it.dev];
  const NegfBlock* blk = P.blocks + dv.blk0;
  const int K = dv.n_blocks;
  const int row = it.row;
  const uint32_t fl = P.flags;
  const cplx z = cmk(it.z_re, it.z_im);
  const cplx* hs = reinterpret_cast<const cplx*>(P.hs);
  const cplx* sin = reinterpret_cast<const cplx*>(P.s_in);
  const cplx* sout = reinterpret_cast<const cplx*>(P.s_out);
  cplx* out = reinterpret_cast<cplx*>(P.out);
  const cplx* seL = reinterpret_cast<const cplx*>(it.se_l);
  const cplx* seR = reinterpret_cast<const cplx*>(it.se_r);
  const cplx ONE = cmk(1.0, 0.0), MONE = cmk(-1.0, 0.0);
  const bool lesser = FEAT >= FEAT_LESSER && (fl & NEGF_LESSER) != 0;
  const bool greater = FEAT >= FEAT_LESSER && (fl & NEGF_GREATER) != 0;
  const bool adj = FEAT >= FEAT_ADJOINT && (fl & NEGF_ADJOINT) != 0;
  // density gradient of this item: the z-tangent sweep (forward after each inverse,
  // backward beside the retarded blocks) and the elementwise accumulation below
  const bool dosg = adj && (fl & NEGF_ADJ_DOS) && it.w_d != 0.0;
  int bad = 0;
  cplx *gHd = nullptr, *gSd = nullptr, *gHu = nullptr, *gSu = nullptr, *gHl = nullptr, *gSl = nullptr;
  if (adj) {
    const int64_t u_slab = (P.grad_slab - 2 * dv.g_slab) / 4;
    cplx* gslot = reinterpret_cast<cplx*>(P.grad) + (size_t)blockIdx.x * P.grad_slab;
    gHd = gslot;
    gSd = gslot + dv.g_slab;
    gHu = gslot + 2 * dv.g_slab;
    gSu = gHu + u_slab;
    gHl = gSu + u_slab;
    gSl = gHl + u_slab;
    // the per-item self-energy gradients are sums of the T and density terms
    cplx* gl = reinterpret_cast<cplx*>(it.gse_l);
    cplx* gr = reinterpret_cast<cplx*>(it.gse_r);
    if (gl) for (int e = threadIdx.x; e < it.nse_l * it.nse_l; e += CTA_THREADS) gl[e] = cmk(0.0, 0.0);
    if (gr) for (int e = threadIdx.x; e < it.nse_r * it.nse_r; e += CTA_THREADS) gr[e] = cmk(0.0, 0.0);
    __syncthreads();
  }
  // Density-gradient weight: DOS = -(2/pi) Im Tr[G S], and with Y = G S G = -dG/dz the
  // torch-convention gradients of w_d DOS are i c conj(Y_qp)^T for H and Sigma and
  // i c (-conj(z) conj(Y_qp) + conj(G_qp))^T for S, c = -(2/pi) w_d.
  const double cd = -0.63661977236758134308 * it.w_d;
  const cplx zc_d = cconj(z);
  // gradient block [r x s] += from the tangent Yd = dG/dz and G, both stored [s x r]
  auto acc_hs = [&](cplx* gH, cplx* gS, const cplx* Yd, const cplx* Gm, int r, int s_) {
    for (int e = threadIdx.x; e < r * s_; e += CTA_THREADS) {
      const int i = e / s_, j = e % s_;
      const cplx y = cconj(Yd[(int64_t)j * r + i]), gg = cconj(Gm[(int64_t)j * r + i]);
      gH[e] = cadd(gH[e], cmk(cd * y.y, -cd * y.x));  // -i c y
      const cplx t = cadd(cmul(zc_d, y), gg);
      gS[e] = cadd(gS[e], cmk(-cd * t.y, cd * t.x));  // i c (conj(z) y + g)
    }
  };
  // self-energy corner [c x c] at (os, os) of gse (ns x ns) from Yd (n x n) at (oy, oy)
  auto acc_se = [&](double* gse_raw, int ns, int os, const cplx* Yd, int n, int oy, int c) {
    cplx* gse = reinterpret_cast<cplx*>(gse_raw);
    for (int e = threadIdx.x; e < c * c; e += CTA_THREADS) {
      const int i = e / c, j = e % c;
      const cplx y = cconj(Yd[(int64_t)(oy + j) * n + oy + i]);
      cplx* d = gse + (int64_t)(os + i) * ns + os + j;
      *d = cadd(*d, cmk(cd * y.y, -cd * y.x));
    }
  };

  auto sq = [&](int q) { return (int64_t)blk[q].n * blk[q].n; };
  // sqrt(K) checkpointing (adjoint only): g_q of q = 0, ck, 2ck, ... in nck checkpoint blocks,
  // the others in a segment of ck blocks that is recomputed from its checkpoint when needed
  const int ck = (adj && P.ckpt > 0) ? P.ckpt : 0;
  const int nck = ck ? (K + ck - 1) / ck : 0;
  const size_t mn2 = (size_t)P.max_n * P.max_n;
  const int ckd = ck ? ck : 1;  // divisor for the checkpoint layout (unused when ck == 0)
  auto slab_ptr = [&](cplx* slab, int q) -> cplx* {
    if (!ck) return slab + blk[q].g;
    return slab + (size_t)(q % ckd == 0 ? q / ckd : nck + q % ckd) * mn2;
  };
  auto gptr = [&](int q) -> cplx* {
    return (fl & NEGF_OUT_GR_LEFT) ? out + blk[q].o_grleft + row * sq(q) : slab_ptr(sb.gslab, q);
  };
  auto dgptr = [&](int q) -> cplx* { return slab_ptr(sb.gdslab, q); };
  auto ginptr = [&](int q) -> cplx* {
    return blk[q].o_ginleft >= 0 ? out + blk[q].o_ginleft + row * sq(q) : sb.ginslab + blk[q].g;
  };
  auto sinptr = [&](int q) -> const cplx* {
    return blk[q].s_in >= 0 ? sin + blk[q].s_in + row * sq(q) : nullptr;
  };
  auto gipptr = [&](int q) -> cplx* {
    return blk[q].o_gipleft >= 0 ? out + blk[q].o_gipleft + row * sq(q) : sb.gipslab + blk[q].g;
  };
  auto soutptr = [&](int q) -> const cplx* {
    return blk[q].s_out >= 0 ? sout + blk[q].s_out + row * sq(q) : nullptr;
  };

  // ------------------------------------------------------------ forward sweep
  for (int q = 0; q < K; ++q) {
    bad |= forward_block_body<MX>(P, it, sb, smem_raw, red, pc, q, q > 0 ? gptr(q - 1) : nullptr, gptr(q),
                                  dosg && q > 0 ? dgptr(q - 1) : nullptr, dosg ? dgptr(q) : nullptr);
    const NegfBlock& b = blk[q];
    const int nq = b.n;
    if (lesser) {
      // gin_q = g_q (s_q + L gin_{q-1} U) g_q^H
      const cplx* s = sinptr(q);
      if (q > 0) {
        const int np = blk[q - 1].n;
        gemm<OP_N, OP_N, MX>(smem, nq, np, np, sb.Lz, np, ginptr(q - 1), np, sb.T1, np);
        if (s) gemm<OP_N, OP_N, MX>(smem, nq, nq, np, sb.T1, np, sb.Uz, nq, sb.tA, nq, ONE, s, nq);
        else gemm<OP_N, OP_N, MX>(smem, nq, nq, np, sb.T1, np, sb.Uz, nq, sb.tA, nq);
      } else {
        if (s) copy_mat(sb.tA, s, nq, nq, smem);
        else for (int e = threadIdx.x; e < nq * nq; e += CTA_THREADS) sb.tA[e] = cmk(0.0, 0.0);
        __syncthreads();
      }
      gemm<OP_N, OP_N, MX>(smem, nq, nq, nq, gptr(q), nq, sb.tA, nq, sb.tB, nq);
      gemm<OP_N, OP_C, MX>(smem, nq, nq, nq, sb.tB, nq, gptr(q), nq, ginptr(q), nq);
      pc.mark(PH_LESSER);
    }
    if (greater) {
      // gip_q = g_q (s'_q + L gip_{q-1} U^*) g_q^*   (elementwise conjugates)
      const cplx* s = soutptr(q);
      if (q > 0) {
        const int np = blk[q - 1].n;
        gemm<OP_N, OP_N, MX>(smem, nq, np, np, sb.Lz, np, gipptr(q - 1), np, sb.T1, np);
        if (s) gemm<OP_N, OP_K, MX>(smem, nq, nq, np, sb.T1, np, sb.Uz, nq, sb.tA, nq, ONE, s, nq);
        else gemm<OP_N, OP_K, MX>(smem, nq, nq, np, sb.T1, np, sb.Uz, nq, sb.tA, nq);
      } else {
        if (s) copy_mat(sb.tA, s, nq, nq, smem);
        else for (int e = threadIdx.x; e < nq * nq; e += CTA_THREADS) sb.tA[e] = cmk(0.0, 0.0);
        __syncthreads();
      }
      gemm<OP_N, OP_N, MX>(smem, nq, nq, nq, gptr(q), nq, sb.tA, nq, sb.tB, nq);
      gemm<OP_N, OP_K, MX>(smem, nq, nq, nq, sb.tB, nq, gptr(q), nq, gipptr(q), nq);
      pc.mark(PH_LESSER);
    }
  }

  // ----------------------------------------------------------- backward sweep
  const int nN = blk[K - 1].n;
  const bool need_gt = (fl & (NEGF_OUT_GTRANS | NEGF_OUT_GR_LC | NEGF_TRANS | NEGF_ORB_AR | NEGF_ADJOINT)) != 0;
  cplx* orbg = (fl & NEGF_ORB_GDIAG) ? reinterpret_cast<cplx*>(P.orb_g) + it.orb : nullptr;
  double* orbar = ((fl & NEGF_ORB_AR) && seR) ? P.orb_ar + it.orb : nullptr;
  const int crA = seR ? min(nN, it.nse_r) : 0;
  // diag(G_qN Gamma_R G_qN^H) of block q from gt = G_qN (nq x nN); Gamma_R corner in sb.Nu
  auto spectral_diag = [&](double* dst, const cplx* gtq, int nq) {
    gemm<OP_N, OP_N, MX>(smem, nq, crA, crA, gtq + (nN - crA), nN, sb.Nu, crA, sb.W, crA);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = warp; i < nq; i += CTA_THREADS / 32) {
      double acc = 0.0;
      for (int l = lane; l < crA; l += 32) {
        cplx y = sb.W[(int64_t)i * crA + l], g = gtq[(int64_t)i * nN + (nN - crA) + l];
        acc += y.x * g.x + y.y * g.y;  // Re(y conj(g))
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      if (lane == 0) dst[i] = acc;
    }
    __syncthreads();
  };
  auto gdiag = [&](cplx* dst, const cplx* G, int nq) {
    for (int i = threadIdx.x; i < nq; i += CTA_THREADS) dst[i] = G[(int64_t)i * nq + i];
  };
  const bool want_dos = (fl & (NEGF_ORB_DOS | NEGF_DOS)) != 0;
  double* orb = (fl & NEGF_ORB_DOS) ? P.orb_dos + it.orb : nullptr;
  double dsum = 0.0;  // per-thread partial of sum_i -Im diag(GS)_i / pi

  const cplx* Gnext = gptr(K - 1);
  if (fl & NEGF_OUT_GRD) {
    cplx* d = out + blk[K - 1].o_grd + row * sq(K - 1);
    copy_mat(d, gptr(K - 1), nN, nN, smem);
    Gnext = d;
  }
  const cplx* gt = gptr(K - 1);
  if (fl & NEGF_OUT_GR_LC) {
    cplx* d = out + blk[K - 1].o_grlc + row * sq(K - 1);
    copy_mat(d, gptr(K - 1), nN, nN, smem);
    gt = d;
  }
  const cplx* Nnext = nullptr;  // gnd_{q+1}
  if (lesser) {
    Nnext = ginptr(K - 1);
    if (blk[K - 1].o_gnd >= 0) {
      cplx* d = out + blk[K - 1].o_gnd + row * sq(K - 1);
      copy_mat(d, ginptr(K - 1), nN, nN, smem);
      Nnext = d;
    }
  }
  const cplx* Pnext = nullptr;  // gpd_{q+1}
  if (greater) {
    Pnext = gipptr(K - 1);
    if (blk[K - 1].o_gpd >= 0) {
      cplx* d = out + blk[K - 1].o_gpd + row * sq(K - 1);
      copy_mat(d, gipptr(K - 1), nN, nN, smem);
      Pnext = d;
    }
  }
  __syncthreads();
  pc.mark(PH_FORM);
  if (want_dos) {
    diag_im_acc(orb ? orb + blk[K - 1].orb0 : nullptr, dsum, gptr(K - 1), hs + blk[K - 1].sdT, nN, nN, true);
    __syncthreads();
    pc.mark(PH_DOS);
  }
  if (orbg) gdiag(orbg + blk[K - 1].orb0, gptr(K - 1), nN);
  if (orbar) {
    form_gamma(sb.Nu, seR, it.nse_r, it.nse_r - crA, crA);
    __syncthreads();
    spectral_diag(orbar + blk[K - 1].orb0, gt, nN);
  }
  const cplx* Dnext = nullptr;  // dG_{q+1,q+1}/dz
  int dtog = 0;
  if (dosg) {
    Dnext = dgptr(K - 1);
    acc_hs(gHd + blk[K - 1].g, gSd + blk[K - 1].g, Dnext, gptr(K - 1), nN, nN);
    if (seR && it.gse_r) {
      const int crd = min(nN, it.nse_r);
      acc_se(it.gse_r, it.nse_r, it.nse_r - crd, Dnext, nN, nN - crd, crd);
    }
    __syncthreads();
  }
  int tog = 0;
  int seg_lo = ck ? ((K - 1) / ck) * ck : 0;  // checkpoint of the segment whose g_q are in the slab
  // with checkpointing: bring the segment [c, c + ck) into the slab, recomputed from g_c
  auto load_segment = [&](int c, bool want_dg) {
    for (int r = c + 1; r < c + ck && r < K; ++r)
      bad |= rgf_forward_block<MX>(P, it, sb, smem_raw, red, pc, r, gptr(r - 1), gptr(r),
                                   want_dg ? dgptr(r - 1) : nullptr, want_dg ? dgptr(r) : nullptr);
    seg_lo = c;
  };
  for (int q = K - 2; q >= 0; --q) {
    if (ck && q < seg_lo) load_segment(seg_lo - ck, dosg);
    const NegfBlock& b = blk[q];
    const int nq = b.n, nn = b.n_next;
    const int64_t szu = (int64_t)nq * nn;
    form_shift(sb.Lz, hs, b.hl, b.sl, z, nn, nq, smem);  // L_q: n_{q+1} x n_q
    form_shift(sb.Uz, hs, b.hu, b.su, z, nq, nn, smem);  // U_q: n_q x n_{q+1}
    __syncthreads();
    pc.mark(PH_FORM);
    const cplx* g = gptr(q);
    cplx* grl = (fl & NEGF_OUT_GRL) ? out + b.o_grl + row * szu : sb.Gl;
    cplx* gru = (fl & NEGF_OUT_GRU) ? out + b.o_gru + row * szu : sb.Gu;
    cplx* grd = (fl & NEGF_OUT_GRD) ? out + b.o_grd + row * sq(q) : (adj ? sb.grdslab + b.g : sb.Gd);
    gemm<OP_N, OP_N, MX>(smem, nq, nn, nq, g, nq, sb.Uz, nn, sb.gU, nn);         // gU = g U
    gemm<OP_N, OP_N, MX>(smem, nn, nq, nn, Gnext, nn, sb.Lz, nq, sb.T1, nq);     // G_{q+1,q+1} L
    gemm<OP_N, OP_N, MX>(smem, nn, nq, nq, sb.T1, nq, g, nq, grl, nq);           // grl
    gemm<OP_N, OP_N, MX>(smem, nq, nn, nn, sb.gU, nn, Gnext, nn, gru, nn);       // gru
    gemm<OP_N, OP_N, MX>(smem, nq, nq, nn, sb.gU, nn, grl, nq, grd, nq, ONE, g, nq);  // grd
    if (need_gt) {
      cplx* gtn = (fl & NEGF_OUT_GR_LC) ? out + b.o_grlc + row * (int64_t)nq * nN
                                          : (sb.colslab ? sb.colslab + b.gc : (tog ? sb.Gt1 : sb.Gt0));
      gemm<OP_N, OP_N, MX>(smem, nq, nN, nn, sb.gU, nn, gt, nN, gtn, nN);
      gt = gtn;
      tog ^= 1;
    }
    if (dosg) {
      // z-tangents of the retarded blocks (Gnext = G_{q+1,q+1}, sb.T1 = Gnext L, sb.gU = g U):
      //   gUd = dg U - g su;  T1d = Dnext L - Gnext sl;  dgrl = T1d g + T1 dg;
      //   dgru = gUd Gnext + gU Dnext;  dgrd = dg + gUd grl + gU dgrl
      const cplx* dg = dgptr(q);
      cplx* Dcur = dtog ? sb.D1 : sb.D0;
      gemm<OP_N, OP_N, MX>(smem, nq, nn, nq, dg, nq, sb.Uz, nn, sb.tA, nn);
      if (b.su >= 0) gemm<OP_N, OP_N, MX>(smem, nq, nn, nq, g, nq, hs + b.su, nn, sb.tA, nn, MONE, sb.tA, nn);
      gemm<OP_N, OP_N, MX>(smem, nn, nq, nn, Dnext, nn, sb.Lz, nq, sb.tB, nq);
      if (b.sl >= 0) gemm<OP_N, OP_N, MX>(smem, nn, nq, nn, Gnext, nn, hs + b.sl, nq, sb.tB, nq, MONE, sb.tB, nq);
      gemm<OP_N, OP_N, MX>(smem, nn, nq, nq, sb.tB, nq, g, nq, sb.tC, nq);
      gemm<OP_N, OP_N, MX>(smem, nn, nq, nq, sb.T1, nq, dg, nq, sb.tC, nq, ONE, sb.tC, nq);
      gemm<OP_N, OP_N, MX>(smem, nq, nn, nn, sb.tA, nn, Gnext, nn, sb.tD, nn);
      gemm<OP_N, OP_N, MX>(smem, nq, nn, nn, sb.gU, nn, Dnext, nn, sb.tD, nn, ONE, sb.tD, nn);
      gemm<OP_N, OP_N, MX>(smem, nq, nq, nn, sb.tA, nn, grl, nq, Dcur, nq, ONE, dg, nq);
      gemm<OP_N, OP_N, MX>(smem, nq, nq, nn, sb.gU, nn, sb.tC, nq, Dcur, nq, ONE, Dcur, nq);
      acc_hs(gHd + b.g, gSd + b.g, Dcur, grd, nq, nq);         // (q, q)
      acc_hs(gHu + b.gu, gSu + b.gu, sb.tC, grl, nq, nn);      // (q, q+1): Y_{q+1,q}, G_{q+1,q}
      acc_hs(gHl + b.gu, gSl + b.gu, sb.tD, gru, nn, nq);      // (q+1, q): Y_{q,q+1}, G_{q,q+1}
      __syncthreads();
      Dnext = Dcur;
      dtog ^= 1;
    }
    pc.mark(PH_GEMM_BWD);
    if (orbg) gdiag(orbg + b.orb0, grd, nq);
    if (orbar) spectral_diag(orbar + b.orb0, gt, nq);
    if (lesser) {
      const cplx* gin = ginptr(q);
      cplx* gnl = b.o_gnl >= 0 ? out + b.o_gnl + row * szu : sb.Nl;
      cplx* gnd = b.o_gnd >= 0 ? out + b.o_gnd + row * sq(q) : sb.Nd;
      // gLmH = L g^H  (n_{q+1} x n_q)
      gemm<OP_N, OP_C, MX>(smem, nn, nq, nq, sb.Lz, nq, g, nq, sb.tA, nq);
      // gnl = G_{q+1,q+1} L gin + gnd_{q+1} gLmH ; sb.T1 still holds G_{q+1,q+1} L
      gemm<OP_N, OP_N, MX>(smem, nn, nq, nn, Nnext, nn, sb.tA, nq, sb.tB, nq);
      gemm<OP_N, OP_N, MX>(smem, nn, nq, nq, sb.T1, nq, gin, nq, gnl, nq, ONE, sb.tB, nq);
      // gnd = gin + (g U) gnd_{q+1} gLmH + gin U gru^H + gru L gin
      gemm<OP_N, OP_N, MX>(smem, nq, nq, nn, sb.gU, nn, sb.tB, nq, sb.tC, nq, ONE, gin, nq);
      gemm<OP_N, OP_N, MX>(smem, nq, nn, nq, gin, nq, sb.Uz, nn, sb.tD, nn);
      gemm<OP_N, OP_C, MX>(smem, nq, nq, nn, sb.tD, nn, gru, nn, sb.tC, nq, ONE, sb.tC, nq);
      gemm<OP_N, OP_N, MX>(smem, nq, nq, nn, gru, nn, sb.Lz, nq, sb.tE, nq);
      gemm<OP_N, OP_N, MX>(smem, nq, nq, nq, sb.tE, nq, gin, nq, gnd, nq, ONE, sb.tC, nq);
      if (b.o_gnu >= 0) {
        cplx* gnu = out + b.o_gnu + row * szu;
        for (int e = threadIdx.x; e < nq * nn; e += CTA_THREADS) {
          int i = e / nn, j = e % nn;  // gnu[i][j] = conj(gnl[j][i])
          gnu[e] = cconj(gnl[(int64_t)j * nq + i]);
        }
      }
      __syncthreads();
      Nnext = gnd;
      pc.mark(PH_LESSER);
    }
    if (greater) {
      const cplx* gip = gipptr(q);
      cplx* gpl = b.o_gpl >= 0 ? out + b.o_gpl + row * szu : sb.Nl;
      cplx* gpd = b.o_gpd >= 0 ? out + b.o_gpd + row * sq(q) : sb.Pd;
      // lcgc = L^* g^*  (n_{q+1} x n_q)
      gemm<OP_K, OP_K, MX>(smem, nn, nq, nq, sb.Lz, nq, g, nq, sb.tA, nq);
      // gpl = G_{q+1,q+1} L gip + gpd_{q+1} lcgc ; sb.T1 still holds G_{q+1,q+1} L
      gemm<OP_N, OP_N, MX>(smem, nn, nq, nn, Pnext, nn, sb.tA, nq, sb.tB, nq);
      gemm<OP_N, OP_N, MX>(smem, nn, nq, nq, sb.T1, nq, gip, nq, gpl, nq, ONE, sb.tB, nq);
      // gpd = gip + (g U) gpd_{q+1} lcgc + gip U^* grl^* + gru L gip
      gemm<OP_N, OP_N, MX>(smem, nq, nq, nn, sb.gU, nn, sb.tB, nq, sb.tC, nq, ONE, gip, nq);
      gemm<OP_N, OP_K, MX>(smem, nq, nn, nq, gip, nq, sb.Uz, nn, sb.tD, nn);
      gemm<OP_N, OP_K, MX>(smem, nq, nq, nn, sb.tD, nn, grl, nq, sb.tC, nq, ONE, sb.tC, nq);
      gemm<OP_N, OP_N, MX>(smem, nq, nq, nn, gru, nn, sb.Lz, nq, sb.tE, nq);
      gemm<OP_N, OP_N, MX>(smem, nq, nq, nq, sb.tE, nq, gip, nq, gpd, nq, ONE, sb.tC, nq);
      if (b.o_gpu >= 0) {
        cplx* gpu = out + b.o_gpu + row * szu;
        for (int e = threadIdx.x; e < nq * nn; e += CTA_THREADS) {
          int i = e / nn, j = e % nn;  // gpu[i][j] = conj(gpl[j][i])
          gpu[e] = cconj(gpl[(int64_t)j * nq + i]);
        }
      }
      __syncthreads();
      Pnext = gpd;
      pc.mark(PH_LESSER);
    }
    if (want_dos) {
      diag_im_acc(orb ? orb + b.orb0 : nullptr, dsum, grd, hs + b.sdT, nq, nq, true);
      __syncthreads();
      if (b.slT >= 0) {
        diag_im_acc(orb ? orb + b.orb0 : nullptr, dsum, gru, hs + b.slT, nq, nn, false);
        __syncthreads();
      }
      if (b.suT >= 0) {
        diag_im_acc(orb ? orb + blk[q + 1].orb0 : nullptr, dsum, grl, hs + b.suT, nn, nq, false);
        __syncthreads();
      }
      pc.mark(PH_DOS);
    }
    Gnext = grd;
  }
  if (dosg && seL && it.gse_l) {  // Dnext = dG_11/dz
    acc_se(it.gse_l, it.nse_l, 0, Dnext, blk[0].n, 0, min(blk[0].n, it.nse_l));
    __syncthreads();
  }
  if (fl & NEGF_OUT_GTRANS) {
    cplx* d = out + dv.o_gtrans + row * (int64_t)blk[0].n * nN;
    copy_mat(d, gt, blk[0].n, nN, smem);
    __syncthreads();
  }
  double dos_total = 0.0;
  if (fl & NEGF_DOS) dos_total = 2.0 * cta_sum(dsum, red);
  pc.mark(PH_DOS);

  // ------------------------------------------------------------ refinement
  // Iterative refinement of the column X = G_{:,N} (X_q = G_qN), per step:
  //   R_q  = delta_qN I - A_qq X_q + L_{q-1} X_{q-1} + U_q X_{q+1}   (FP64 tensor cores)
  //   y_0 = R_0,  y_q = R_q + L_{q-1} g_{q-1} y_{q-1}
  //   dX_N = g_N y_N,  dX_q = g_q (y_q + U_q dX_{q+1}),  X_q += dX_q  (sweep's product path)
  // with A = zS - H - Sigma (A_{q,q-1} = -L_{q-1}, A_{q,q+1} = -U_q, the same
  // sign convention as the forward sweep) and the stored left-connected g_q.
  // Each step multiplies the error of X by the contraction of the approximate
  // solve (about the relative error of the unrefined sweep, which grows with
  // the number of blocks).  The item stops after refine_steps steps, or
  // earlier once max|dX_0| <= REFINE_TOL max|X_0|.
  if ((fl & NEGF_REFINE) && (fl & NEGF_TRANS) && seL && seR) {
    const int steps = P.refine_steps > 0 ? P.refine_steps : 1;
    auto colx = [&](int q) -> cplx* {
      return (fl & NEGF_OUT_GR_LC) ? out + blk[q].o_grlc + row * (int64_t)blk[q].n * nN : sb.colslab + blk[q].gc;
    };
    if (!(fl & NEGF_OUT_GR_LC)) copy_mat(colx(K - 1), gptr(K - 1), nN, nN, smem);  // X_N apart from g_N
    auto add_into = [&](cplx* x, const cplx* d, int64_t cnt) {
      for (int64_t e = threadIdx.x; e < cnt; e += CTA_THREADS) x[e] = cadd(x[e], d[e]);
      __syncthreads();
    };
    for (int step = 0; step < steps; ++step) {
      for (int q = 0; q < K; ++q) {
        const NegfBlock& b = blk[q];
        const int nq = b.n;
        cplx* yq = sb.yslab + b.gc;
        form_a0(sb.W, hs, b, z, q == 0 ? seL : nullptr, it.nse_l, q == K - 1 ? seR : nullptr, it.nse_r, smem);
        gemm<OP_N, OP_N, false>(smem, nq, nN, nq, sb.W, nq, colx(q), nN, yq, nN, MONE);  // -A_qq X_q
        if (q == K - 1) {
          for (int i = threadIdx.x; i < nN; i += CTA_THREADS) yq[(int64_t)i * nN + i].x += 1.0;
          __syncthreads();
        }
        if (q > 0) {
          const int np = blk[q - 1].n;
          form_shift(sb.Lz, hs, blk[q - 1].hl, blk[q - 1].sl, z, nq, np, smem);
          gemm<OP_N, OP_N, false>(smem, nq, nN, np, sb.Lz, np, colx(q - 1), nN, yq, nN, ONE, yq, nN);
        }
        if (q < K - 1) {
          const int nn = b.n_next;
          form_shift(sb.Uz, hs, b.hu, b.su, z, nq, nn, smem);
          gemm<OP_N, OP_N, false>(smem, nq, nN, nn, sb.Uz, nn, colx(q + 1), nN, yq, nN, ONE, yq, nN);
        }
        if (q > 0) {
          const int np = blk[q - 1].n;
          gemm<OP_N, OP_N, MX>(smem, np, nN, np, gptr(q - 1), np, sb.yslab + blk[q - 1].gc, nN, sb.T1, nN);
          gemm<OP_N, OP_N, MX>(smem, nq, nN, np, sb.Lz, np, sb.T1, nN, yq, nN, ONE, yq, nN);
        }
      }
      cplx* dx = sb.Gt0;
      cplx* dn = sb.Gt1;
      gemm<OP_N, OP_N, MX>(smem, nN, nN, nN, gptr(K - 1), nN, sb.yslab + blk[K - 1].gc, nN, dx, nN);
      add_into(colx(K - 1), dx, (int64_t)nN * nN);
      for (int q = K - 2; q >= 0; --q) {
        const NegfBlock& b = blk[q];
        const int nq = b.n, nn = b.n_next;
        form_shift(sb.Uz, hs, b.hu, b.su, z, nq, nn, smem);
        gemm<OP_N, OP_N, MX>(smem, nq, nN, nn, sb.Uz, nn, dx, nN, sb.T1, nN, ONE, sb.yslab + b.gc, nN);
        gemm<OP_N, OP_N, MX>(smem, nq, nN, nq, gptr(q), nq, sb.T1, nN, dn, nN);
        add_into(colx(q), dn, (int64_t)nq * nN);
        cplx* t = dx; dx = dn; dn = t;
      }
      if (step + 1 < steps) {  // dx holds dX_0
        const cplx* x0 = colx(0);
        double dmax = 0.0, xmax = 0.0;
        for (int64_t e = threadIdx.x; e < (int64_t)blk[0].n * nN; e += CTA_THREADS) {
          dmax = fmax(dmax, cabs1(dx[e]));
          xmax = fmax(xmax, cabs1(x0[e]));
        }
        dmax = cta_max(dmax, red);
        xmax = cta_max(xmax, red);
        if (!(dmax > REFINE_TOL * xmax)) break;  // uniform: every thread sees the same maxima
      }
    }
    gt = colx(0);
    pc.mark(PH_REFINE);
  }

  // ------------------------------------------------------------ T(E)
  double tval = 0.0;
  if ((fl & NEGF_TRANS) && seL && seR) {
    const int n0 = blk[0].n;
    const int cl = min(n0, it.nse_l), cr = min(nN, it.nse_r);
    const cplx* Gc = gt + (nN - cr);  // G_1N[0:cl, nN-cr:nN], row stride nN
    form_gamma(sb.tA, seL, it.nse_l, 0, cl);
    form_gamma(sb.tB, seR, it.nse_r, it.nse_r - cr, cr);
    __syncthreads();
    // FP64 on both paths: per energy (not per block), and the mixed path's
    // refined G_1N must not meet FP32-level products here
    gemm<OP_N, OP_N, false>(smem, cl, cr, cl, sb.tA, cl, Gc, nN, sb.tC, cr);   // Gamma_L G
    gemm<OP_N, OP_N, false>(smem, cl, cr, cr, sb.tC, cr, sb.tB, cr, sb.tD, cr);  // ... Gamma_R
    double part = 0.0;
    for (int e = threadIdx.x; e < cl * cr; e += CTA_THREADS) {
      int i = e / cr, l = e % cr;
      cplx a = sb.tD[e], gg = Gc[(int64_t)i * nN + l];
      part += a.x * gg.x + a.y * gg.y;  // Re(a conj(g))
    }
    tval = cta_sum(part, red);
  }
  // ------------------------------------------------------------ adjoint
  // d(c T)/dX_pq = 2c W_qp^H with W_qp = G_qN M G_1p, M = Gamma_R G_1N^H Gamma_L
  // restricted to the lead corners: W_qp = R_q (M_c F_p), R_q = G_qN[:, nN-cr:],
  // F_p = G_1p[0:cl, :] = P_p G_pp, P_{p+1} = P_p g_p U_p, P_0 = I (rows 0..cl).
  if (adj && seL && seR && it.w_t != 0.0) {
    const int n0 = blk[0].n;
    const int cl = min(n0, it.nse_l), cr = min(nN, it.nse_r);
    const double c2 = 2.0 * it.w_t;
    const cplx zc = cconj(z);
    const cplx* Gc = gt + (nN - cr);  // G_1N[0:cl, nN-cr:], row stride nN
    cplx* Mc = sb.Nu;                 // cr x cl (a buffer the forward step leaves alone)
    gemm<OP_N, OP_C, MX>(smem, cr, cl, cr, sb.tB, cr, Gc, nN, sb.T1, cl);   // Gamma_R Gc^H
    gemm<OP_N, OP_N, MX>(smem, cr, cl, cl, sb.T1, cl, sb.tA, cl, Mc, cl);   // ... Gamma_L
    // explicit Gamma terms: dT/dSigma_L = -2i K, K = Gc Gamma_R Gc^H; dT/dSigma_R = -2i Gc^H Gamma_L Gc
    cplx* gseL = reinterpret_cast<cplx*>(it.gse_l);
    cplx* gseR = reinterpret_cast<cplx*>(it.gse_r);
    if (gseL) {
      gemm<OP_N, OP_N, MX>(smem, cl, cl, cr, Gc, nN, sb.T1, cl, sb.Nd, cl);
      const int ns = it.nse_l;
      for (int e = threadIdx.x; e < ns * ns; e += CTA_THREADS) {
        int i = e / ns, j = e % ns;
        cplx v = cmk(0.0, 0.0);
        if (i < cl && j < cl) {
          cplx k = sb.Nd[(int64_t)i * cl + j];
          v = cmk(c2 * k.y, -c2 * k.x);  // -2ic k
        }
        gseL[e] = cadd(gseL[e], v);
      }
    }
    if (gseR) {
      gemm<OP_C, OP_N, MX>(smem, cr, cr, cl, Gc, nN, sb.tC, cr, sb.Nl, cr);  // Gc^H (Gamma_L Gc)
      const int ns = it.nse_r, o = ns - cr;
      for (int e = threadIdx.x; e < ns * ns; e += CTA_THREADS) {
        int i = e / ns, j = e % ns;
        cplx v = cmk(0.0, 0.0);
        if (i >= o && j >= o) {
          cplx k = sb.Nl[(int64_t)(i - o) * cr + (j - o)];
          v = cmk(c2 * k.y, -c2 * k.x);
        }
        gseR[e] = cadd(gseR[e], v);
      }
    }
    __syncthreads();
    auto colp = [&](int q) -> const cplx* {
      if (q == K - 1) return gptr(K - 1);
      return (fl & NEGF_OUT_GR_LC) ? out + blk[q].o_grlc + row * (int64_t)blk[q].n * nN : sb.colslab + blk[q].gc;
    };
    auto gpp = [&](int q) -> const cplx* {
      if (q == K - 1) return gptr(K - 1);
      return (fl & NEGF_OUT_GRD) ? out + blk[q].o_grd + row * sq(q) : sb.grdslab + blk[q].g;
    };
    cplx* Pc = sb.Gl;   // cl x n_p
    cplx* Pn = sb.Gu;
    cplx* Ycur = sb.Gd; // cr x n_p
    for (int p = 0; p < K; ++p) {
      if (ck && p % ck == 0 && p != seg_lo) load_segment(p, false);
      const int np = blk[p].n;
      const cplx* F;
      int ldF;
      if (p == 0) { F = gpp(0); ldF = np; }
      else {
        gemm<OP_N, OP_N, MX>(smem, cl, np, np, Pc, np, gpp(p), np, sb.Lz, np);
        F = sb.Lz; ldF = np;
      }
      gemm<OP_N, OP_N, MX>(smem, cr, np, cl, Mc, cl, F, ldF, Ycur, np);       // Y_p = M_c F_p
      const cplx* Rp = colp(p) + (nN - cr);
      {
        GemmArgs g = gemm_args(np, np, cr, Rp, nN, Ycur, np, nullptr, 0);
        EpiGrad e{gHd + blk[p].g, gSd + blk[p].g, np, c2, zc, p == 0 ? gseL : nullptr, cl, it.nse_l,
                  p == K - 1 ? gseR : nullptr, cr, it.nse_r, nN - cr};
        gemm_epi<OP_N, OP_N, MX>(g, smem, e);                        // W_pp
      }
      if (p > 0) {  // W_{p-1,p} -> d/d(hl_{p-1}, sl_{p-1})  [n_p x n_{p-1}]
        const int nm = blk[p - 1].n;
        GemmArgs g = gemm_args(nm, np, cr, colp(p - 1) + (nN - cr), nN, Ycur, np, nullptr, 0);
        EpiGrad e{gHl + blk[p - 1].gu, gSl + blk[p - 1].gu, nm, c2, zc, nullptr, 0, 0, nullptr, 0, 0, 0};
        gemm_epi<OP_N, OP_N, MX>(g, smem, e);
      }
      if (p < K - 1) {
        const int nn = blk[p].n_next;
        {  // W_{p+1,p} -> d/d(hu_p, su_p)  [n_p x n_{p+1}]
          GemmArgs g = gemm_args(nn, np, cr, colp(p + 1) + (nN - cr), nN, Ycur, np, nullptr, 0);
          EpiGrad e{gHu + blk[p].gu, gSu + blk[p].gu, nn, c2, zc, nullptr, 0, 0, nullptr, 0, 0, 0};
          gemm_epi<OP_N, OP_N, MX>(g, smem, e);
        }
        // P_{p+1} = P_p g_p U_p
        form_shift(sb.Uz, hs, blk[p].hu, blk[p].su, z, np, nn, smem);
        gemm<OP_N, OP_N, MX>(smem, np, nn, np, gptr(p), np, sb.Uz, nn, sb.gU, nn);
        if (p == 0) copy_mat(Pn, sb.gU, cl, nn, smem);
        else gemm<OP_N, OP_N, MX>(smem, cl, nn, np, Pc, np, sb.gU, nn, Pn, nn);
        cplx* t = Pc; Pc = Pn; Pn = t;
      }
    }
    pc.mark(PH_GEMM_BWD);
  }

  if (threadIdx.x == 0) {
    if (fl & NEGF_TRANS) P.trans[it.out] = tval;
    if (fl & NEGF_DOS) P.dos[it.out] = dos_total;
    int st = NEGF_OK;
    if (bad) st = NEGF_ERR_SINGULAR;
    else if (MX && tc_err) st = NEGF_ERR_TIMEOUT;
    else if (!isfinite(tval) || !isfinite(dos_total)) st = NEGF_ERR_NONFINITE;
    P.status[it.out] = st;
  }
  __syncthreads();
  pc.mark(PH_TRANS);
}

template <bool MX, int FEAT>
__global__ void __launch_bounds__(CTA_THREADS, 1) rgf_kernel(const NegfRgfProblem P) {
  extern __shared__ __align__(1024) char smem[];
  __shared__ int s_item;
  __shared__ double red[CTA_THREADS / 32];
  unsigned* queue = reinterpret_cast<unsigned*>(P.scratch);
  const SlotBufs sb = slot_bufs(P, blockIdx.x);
  PhaseClock pc;
  pc.start(P.phase_cycles != nullptr);
  if constexpr (MX) tc_tmem_alloc();
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int idx = s_item;
    __syncthreads();
    pc.mark(PH_OTHER);
    if (idx >= P.n_items) break;
    const NegfItem it = P.items[idx];
    rgf_item<MX, FEAT>(P, it, sb, smem, red, pc);
  }
  if constexpr (MX) tc_tmem_free();
  if (pc.on)
    for (int i = 0; i < NPH; ++i) P.phase_cycles[(size_t)blockIdx.x * NPH + i] = pc.c[i];
}

// Dynamic shared memory: the union of the GEMM ring, the inverse panel and the
// streaming buffers (they are used one after another).
inline size_t rgf_smem_bytes(int max_n, bool mixed) {
  size_t a = mixed ? TC_SMEM_BYTES : GEMM_SMEM_BYTES, b = inv_smem_bytes_host(max_n, mixed), c = STREAM_SMEM_BYTES;
  size_t m = a > b ? a : b;
  return m > c ? m : c;
}
static_assert(CTA_THREADS == 256, "cta_stream.cuh assumes 256-thread CTAs");


// Set the shared-memory limit of one instantiation and launch it (grid CTAs).  The FP64 sweep
// is compiled per feature set (rgf.cu); the mixed-precision sweep is one instantiation with
// every feature (rgf_mx.cu).
template <bool MX, int FEAT>
inline int rgf_launch_impl(const NegfRgfProblem& p, size_t smem, int grid, cudaStream_t s) {
  auto kern = rgf_kernel<MX, FEAT>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return NEGF_ERR_CUDA;
  kern<<<grid, CTA_THREADS, smem, s>>>(p);
  return cudaGetLastError() == cudaSuccess ? NEGF_OK : NEGF_ERR_CUDA;
}
int rgf_launch_fp64(int feat, const NegfRgfProblem& p, size_t smem, int grid, cudaStream_t s);  // rgf.cu
int rgf_launch_mx(const NegfRgfProblem& p, size_t smem, int grid, cudaStream_t s);                // rgf_mx.cu

}  // namespace negf
