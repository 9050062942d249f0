// Product chains around the sweep and the decimation (sm_100a, FP64 tensor cores):
//
//   negf_gamma_sum_run      out = sum_i w_i Re(G_i[:, c0:c0+k] Gamma_i G_i[:, c0:c0+k]^H)
//                           the non-equilibrium density matrix of Ozaki.integrate
//                           (negf/density.py:183-195, DM_neq = sum w (G Gamma_R G^H).real (f_R - f_L))
//   negf_lead_adjoint_run   dL/d(H, H01, S, S01, H_DL, S_DL) of a lead's self-energies through the
//                           converged decimation fixed point (the implicit-function adjoint of
//                           g_s = (zS - H - tau g_s tau')^-1, the relation the reference's residual
//                           check tests, negf/surface_green.py:142-145)
//
// Both are batched over energies and use the CTA tile GEMM of the sweep (DMMA, Gauss/3M complex
// products, as the sweep: no iteration here feeds rounding back) and the pivoted LU of the
// decimation.  Sums over energies run in a fixed order, so
// results are bitwise reproducible.
#include "../../include/negf_b200.h"
#include "lead_forms.cuh"

namespace negf {

// ---------------------------------------------------------------------------------------------
// Weighted G Gamma G^H sum.  Stage 1 (one CTA per energy): T_i = w_i G_i[:, c0:] Gamma_i and a
// copy of G_i[:, c0:], side by side as the column blocks of two n x (n_items k) matrices.
// Stage 2: out = Re(T_stack G_stack^H), one GEMM over every energy.  Its k-loop is split into
// up to GS_MAX_SPLIT contiguous ranges so that the output tiles times the splits fill the GPU
// (a 256 x 256 output is only 16 tiles); each (tile, range) CTA writes the real part of its
// partial product, and stage 3 sums the ranges in range order, so the result does not depend
// on scheduling.

constexpr size_t PROD_ALIGN = 256;
constexpr int GS_MAX_SPLIT = 16;

inline size_t round_up(size_t b) { return (b + PROD_ALIGN - 1) & ~(PROD_ALIGN - 1); }

inline size_t gamma_stack_bytes(const NegfGammaSum& p) {
  return round_up((size_t)p.n * (size_t)p.n_items * (size_t)p.k * sizeof(cplx));
}

inline size_t gamma_part_bytes(const NegfGammaSum& p) {
  return round_up((size_t)GS_MAX_SPLIT * p.n * p.n * sizeof(double));
}

// k-range length of stage 2 for `split` ranges: a multiple of the 16-deep k slab.
inline int64_t gamma_split_len(int64_t K, int split) { return ((K + split - 1) / split + 15) / 16 * 16; }

__global__ void __launch_bounds__(CTA_THREADS, 1) gamma_stack_kernel(const NegfGammaSum P, cplx* Tst, cplx* Gst) {
  extern __shared__ __align__(16) char smem_raw[];
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);
  const int64_t K = (int64_t)P.n_items * P.k;
  for (int i = blockIdx.x; i < P.n_items; i += gridDim.x) {
    const cplx* G = reinterpret_cast<const cplx*>(P.g) + (int64_t)i * P.g_stride + P.c0;
    const cplx* Gam = reinterpret_cast<const cplx*>(P.gamma) + (int64_t)i * P.gamma_stride;
    gemm_ls<OP_N, OP_N, true>(smem, P.n, P.k, P.k, G, P.ldg, Gam, P.ldgam, Tst + (int64_t)i * P.k, K, nullptr, 0,
                        cmk(P.w[i], 0.0));
    for (int64_t e = threadIdx.x; e < (int64_t)P.n * P.k; e += CTA_THREADS) {
      const int64_t r = e / P.k, c = e % P.k;
      Gst[r * K + (int64_t)i * P.k + c] = G[r * P.ldg + c];
    }
    __syncthreads();
  }
}

struct EpiRealOut {
  double* out;
  int64_t ld;
  int m0, n0;
  NEGF_DEV void operator()(int m, int n, cplx v) const { out[(int64_t)(m0 + m) * ld + n0 + n] = v.x; }
};

// Stage 2: CTA (x, y, z) multiplies output tile (y, x) over k-range z into part[z].
__global__ void __launch_bounds__(CTA_THREADS, 1) gamma_reduce_kernel(const NegfGammaSum P, const cplx* Tst,
                                                                      const cplx* Gst, double* part,
                                                                      int64_t klen) {
  extern __shared__ __align__(16) char smem_raw[];
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);
  const int64_t K = (int64_t)P.n_items * P.k;
  const int m0 = blockIdx.y * GT_M, n0 = blockIdx.x * GT_N;
  const int64_t k0 = (int64_t)blockIdx.z * klen;
  const int M = min(GT_M, P.n - m0), N = min(GT_N, P.n - n0);
  const int Kz = (int)(k0 < K ? (K - k0 < klen ? K - k0 : klen) : 0);
  double* out = part + (size_t)blockIdx.z * P.n * P.n;
  if (Kz == 0) {  // an empty range still writes its (zero) partial tile
    for (int e = threadIdx.x; e < M * N; e += CTA_THREADS) out[(int64_t)(m0 + e / N) * P.n + n0 + e % N] = 0.0;
    return;
  }
  GemmArgs g = gemm_args(M, N, Kz, Tst + (int64_t)m0 * K + k0, K, Gst + (int64_t)n0 * K + k0, K, nullptr, 0);
  cta_gemm_epi<OP_N, OP_C, true, EpiRealOut, true>(g, smem, EpiRealOut{out, P.n, m0, n0});
}

// Stage 3: out = sum of the partial outputs in range order.
__global__ void gamma_sum_parts_kernel(double* out, const double* part, int64_t n2, int split) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n2; e += (int64_t)gridDim.x * blockDim.x) {
    double s = part[e];
    for (int z = 1; z < split; ++z) s += part[(size_t)z * n2 + e];
    out[e] = s;
  }
}

// ---------------------------------------------------------------------------------------------
// Lead adjoint.  Per energy (z = E + i eta, tau = z S01 - H01, tau' = z S01^H - H01^H, g = g_s):
//   V = dL/dg from Sigma(g):  form 0  Sigma = L g[:b,:b] R,  L = E S_DL - H_DL, R = E S_DL^H - H_DL^H
//                                      V[:b,:b] = L^H Gs R^H,  dL/dL = Gs R^H g_b^H,  dL/dR = g_b^H L^H Gs
//                             form 1  Sigma = g^-1:           V = -g^-H Gs g^-H
//                             form 2  Sigma = E S - H - g^-1: V = +g^-H Gs g^-H, dS += conj(E) Gs, dH -= Gs
//   Lambda = V + P^H Lambda Q^H with P = g tau, Q = tau' g, by doubling
//            (Lambda += P^H Lambda Q^H, P <- P^2, Q <- Q^2 until max|P| max|Q| < tol)
//   F = (zS - H - tau g tau')^-1, dW = -F^H Lambda F^H
//   dS += conj(z) dW, dH -= dW, dtau = -dW (g tau')^H, dtau' = -(tau g)^H dW,
//   dS01 += conj(z) dtau + z dtau'^H, dH01 -= dtau + dtau'^H
// (PyTorch's convention: the gradient of a real loss w.r.t. a complex tensor is dL/d conj(x)).
// Energies go to the CTAs round-robin; each CTA sums its energies' contributions in its own slot,
// and a second kernel sums the slots in slot order.

constexpr int LA_NACC = 6, LA_NWORK = 12;

__host__ __device__ inline int la_max_n(const NegfLead& ld) { return ld.nc > ld.n ? ld.nc : ld.n; }

__host__ __device__ inline size_t la_slot_elems(const NegfLeadAdjProblem& p) {
  const size_t mn = (size_t)la_max_n(p.lead);
  return ((LA_NACC + LA_NWORK) * mn * mn + 15) & ~(size_t)15;
}

__host__ __device__ inline int64_t la_grad_elems(const NegfLeadAdjProblem& p) {
  const int64_t n = p.lead.n, ncb = p.form == 0 ? (int64_t)p.lead.nc * p.lead.b : 0;
  return 4 * n * n + 2 * ncb;
}

NEGF_DEV void la_item(const NegfLeadAdjProblem& P, int idx, cplx* slot, char* smem_raw, double* red) {
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);
  const NegfLead ld = P.lead;
  const int n = ld.n;
  const int64_t n2 = (int64_t)n * n;
  const size_t mn = (size_t)la_max_n(ld), mn2 = mn * mn;
  const NegfLeadAdjItem it = P.items[idx];
  const cplx* ar = reinterpret_cast<const cplx*>(P.arena);
  const cplx *H = ar + ld.h, *S = ar + ld.s, *H01 = ar + ld.h01, *S01 = ar + ld.s01;
  const cplx* g = reinterpret_cast<const cplx*>(it.gs);
  const cplx* Gs = reinterpret_cast<const cplx*>(it.gsig);
  const cplx E = cmk(it.e_re, it.e_im);
  const cplx z = cmk(it.e_re, it.e_im + P.eta);
  const cplx ONE = cmk(1.0, 0.0), MONE = cmk(-1.0, 0.0);
  cplx* acc[LA_NACC];
  for (int r = 0; r < LA_NACC; ++r) acc[r] = slot + r * mn2;
  cplx* w_[LA_NWORK];
  for (int r = 0; r < LA_NWORK; ++r) w_[r] = slot + (LA_NACC + r) * mn2;
  cplx *lam = w_[0], *Pm = w_[1], *Qm = w_[2], *P2 = w_[3], *Q2 = w_[4], *T1 = w_[5];
  cplx *tau = w_[6], *taup = w_[7], *Y1 = w_[8], *W = w_[9], *F = w_[10], *gW = w_[11];
  int bad = 0;

  // ---- V = dL/dg into lam
  for (int64_t e = threadIdx.x; e < n2; e += CTA_THREADS) lam[e] = cmk(0.0, 0.0);
  __syncthreads();
  if (P.form == 0) {
    const int nc = ld.nc, b = ld.b;
    const cplx *hdl = ar + ld.hdl, *sdl = ar + ld.sdl;
    cplx *Lm = Pm, *Rm = Qm, *T2 = P2, *gL = Q2, *gR = Y1;
    for (int e = threadIdx.x; e < nc * b; e += CTA_THREADS) Lm[e] = csub(cmul(E, sdl[e]), hdl[e]);
    __syncthreads();
    form_eS_minus_h_herm(Rm, hdl, sdl, E, b, nc);                       // b x nc
    gemm_ls<OP_C, OP_N, true>(smem, b, nc, nc, Lm, b, Gs, nc, T1, nc);        // L^H Gs       (b x nc)
    gemm_ls<OP_N, OP_C, true>(smem, b, b, nc, T1, nc, Rm, nc, lam, n);        // V[:b,:b]
    gemm_ls<OP_N, OP_C, true>(smem, nc, b, nc, Gs, nc, Rm, nc, T2, b);        // Gs R^H       (nc x b)
    gemm_ls<OP_N, OP_C, true>(smem, nc, b, b, T2, b, g, n, gL, b);            // dL/dL        (nc x b)
    gemm_ls<OP_C, OP_N, true>(smem, b, nc, b, g, n, T1, nc, gR, nc);          // dL/dR        (b x nc)
    const cplx Ec = cconj(E);
    for (int e = threadIdx.x; e < nc * b; e += CTA_THREADS) {
      const int i = e / b, j = e % b;
      const cplx l = gL[e], rH = cconj(gR[(int64_t)j * nc + i]);
      acc[4][e] = csub(acc[4][e], cadd(l, rH));                          // H_DL
      acc[5][e] = cadd(acc[5][e], cadd(cmul(Ec, l), cmul(E, rH)));      // S_DL
    }
    __syncthreads();
  } else {
    for (int64_t e = threadIdx.x; e < n2; e += CTA_THREADS) F[e] = g[e];
    __syncthreads();
    bad |= cta_lu_inverse(F, W, n, smem_raw);                           // W = g^-1
    gemm_ls<OP_C, OP_N, true>(smem, n, n, n, W, n, Gs, n, T1, n);             // g^-H Gs
    gemm_ls<OP_N, OP_C, true>(smem, n, n, n, T1, n, W, n, lam, n, nullptr, 0, P.form == 1 ? MONE : ONE);
    if (P.form == 2) {
      const cplx Ec = cconj(E);
      for (int64_t e = threadIdx.x; e < n2; e += CTA_THREADS) {
        acc[0][e] = csub(acc[0][e], Gs[e]);
        acc[2][e] = cadd(acc[2][e], cmul(Ec, Gs[e]));
      }
      __syncthreads();
    }
  }

  // ---- Lambda by doubling
  cta_shift_form(tau, H01, S01, z, MONE, (int)n2, smem);                // z S01 - H01
  form_eS_minus_h_herm(taup, H01, S01, z, n, n);                        // z S01^H - H01^H
  gemm_ls<OP_N, OP_N, true>(smem, n, n, n, g, n, tau, n, Pm, n);              // P = g tau
  gemm_ls<OP_N, OP_N, true>(smem, n, n, n, taup, n, g, n, Qm, n);             // Q = tau' g
  int steps = 0;
  bool finite = true;
  for (int s = 0; s < P.max_iter; ++s) {
    steps = s + 1;
    gemm_ls<OP_C, OP_N, true>(smem, n, n, n, Pm, n, lam, n, T1, n);           // P^H Lambda
    gemm_ls<OP_N, OP_C, true>(smem, n, n, n, T1, n, Qm, n, lam, n, lam, n);   // Lambda += ... Q^H
    gemm_ls<OP_N, OP_N, true>(smem, n, n, n, Pm, n, Pm, n, P2, n);
    gemm_ls<OP_N, OP_N, true>(smem, n, n, n, Qm, n, Qm, n, Q2, n);
    cplx* t = Pm; Pm = P2; P2 = t;
    t = Qm; Qm = Q2; Q2 = t;
    double mp = 0.0, mq = 0.0;
    for (int64_t e = threadIdx.x; e < n2; e += CTA_THREADS) {
      const double a = hypot(Pm[e].x, Pm[e].y), c = hypot(Qm[e].x, Qm[e].y);
      mp = (a == a) ? fmax(mp, a) : INFINITY;
      mq = (c == c) ? fmax(mq, c) : INFINITY;
    }
    mp = cta_max(mp, red);
    mq = cta_max(mq, red);
    if (!isfinite(mp) || !isfinite(mq)) { finite = false; break; }
    if (mp * mq < P.tol) break;
  }

  // ---- F = (zS - H - tau g tau')^-1 and the parameter gradients
  gemm_ls<OP_N, OP_N, true>(smem, n, n, n, g, n, taup, n, Y1, n);             // g tau'
  gemm_ls<OP_N, OP_N, true>(smem, n, n, n, tau, n, Y1, n, W, n);              // tau g tau'
  for (int64_t e = threadIdx.x; e < n2; e += CTA_THREADS) W[e] = csub(csub(cmul(z, S[e]), H[e]), W[e]);
  __syncthreads();
  bad |= cta_lu_inverse(W, F, n, smem_raw);
  gemm_ls<OP_C, OP_N, true>(smem, n, n, n, F, n, lam, n, T1, n);              // F^H Lambda
  gemm_ls<OP_N, OP_C, true>(smem, n, n, n, T1, n, F, n, gW, n, nullptr, 0, MONE);  // dW
  gemm_ls<OP_N, OP_C, true>(smem, n, n, n, gW, n, Y1, n, T1, n, nullptr, 0, MONE);  // dtau = -dW (g tau')^H
  gemm_ls<OP_N, OP_N, true>(smem, n, n, n, tau, n, g, n, Pm, n);              // tau g
  gemm_ls<OP_C, OP_N, true>(smem, n, n, n, Pm, n, gW, n, Qm, n, nullptr, 0, MONE);  // dtau' = -(tau g)^H dW
  const cplx zc = cconj(z);
  for (int64_t e = threadIdx.x; e < n2; e += CTA_THREADS) {
    const int64_t i = e / n, j = e % n;
    const cplx dw = gW[e], dt = T1[e], dtpH = cconj(Qm[j * n + i]);
    acc[0][e] = csub(acc[0][e], dw);                                      // H
    acc[2][e] = cadd(acc[2][e], cmul(zc, dw));                            // S
    acc[1][e] = csub(acc[1][e], cadd(dt, dtpH));                          // H01
    acc[3][e] = cadd(acc[3][e], cadd(cmul(zc, dt), cmul(z, dtpH)));       // S01
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    P.status[idx] = bad ? NEGF_ERR_SINGULAR : (finite ? NEGF_OK : NEGF_ERR_NONFINITE);
    if (P.iters) P.iters[idx] = steps;
  }
}

__global__ void __launch_bounds__(CTA_THREADS, 1) lead_adjoint_kernel(const NegfLeadAdjProblem P) {
  extern __shared__ __align__(16) char smem[];
  __shared__ double red[CTA_THREADS / 32];
  cplx* slot = reinterpret_cast<cplx*>(P.scratch) + (size_t)blockIdx.x * la_slot_elems(P);
  const size_t mn = (size_t)la_max_n(P.lead);
  for (size_t e = threadIdx.x; e < LA_NACC * mn * mn; e += CTA_THREADS) slot[e] = cmk(0.0, 0.0);
  __syncthreads();
  for (int i = blockIdx.x; i < P.n_items; i += gridDim.x) la_item(P, i, slot, smem, red);
}

// grad[e] = sum over slots, in slot order, of the slots' accumulators.
__global__ void lead_adjoint_sum_kernel(const NegfLeadAdjProblem P, int slots) {
  const int64_t n2 = (int64_t)P.lead.n * P.lead.n;
  const int64_t total = la_grad_elems(P);
  const size_t mn = (size_t)la_max_n(P.lead), mn2 = mn * mn;
  const cplx* base = reinterpret_cast<const cplx*>(P.scratch);
  cplx* out = reinterpret_cast<cplx*>(P.grad);
  const size_t stride = la_slot_elems(P);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    int r;
    int64_t off;
    if (e < 4 * n2) { r = (int)(e / n2); off = e % n2; }
    else { const int64_t ncb = (int64_t)P.lead.nc * P.lead.b; r = 4 + (int)((e - 4 * n2) / ncb); off = (e - 4 * n2) % ncb; }
    cplx s = cmk(0.0, 0.0);
    for (int k = 0; k < slots; ++k) s = cadd(s, base[(size_t)k * stride + r * mn2 + off]);
    out[e] = s;
  }
}

static int sm_count_or(int fallback) {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fallback;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return fallback;
  return n > 0 ? n : fallback;
}

}  // namespace negf

extern "C" {

size_t negf_gamma_sum_scratch_bytes(const NegfGammaSum* p) {
  if (!p || p->n <= 0 || p->k <= 0 || p->n_items <= 0) return 0;
  return 2 * negf::gamma_stack_bytes(*p) + negf::gamma_part_bytes(*p);
}

int negf_gamma_sum_run(const NegfGammaSum* p, void* stream) {
  if (!p || !p->g || !p->gamma || !p->w || !p->out) return NEGF_ERR_ARGUMENT;
  if (p->n <= 0 || p->k <= 0 || p->n_items < 0 || p->c0 < 0 || p->ldg < p->c0 + p->k || p->ldgam < p->k)
    return NEGF_ERR_ARGUMENT;
  if ((int64_t)p->n_items * p->k > 0x7fffffff) return NEGF_ERR_UNSUPPORTED;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (p->n_items == 0)
    return cudaMemsetAsync(p->out, 0, (size_t)p->n * p->n * sizeof(double), s) == cudaSuccess ? NEGF_OK : NEGF_ERR_CUDA;
  if (!p->scratch || p->scratch_bytes < negf_gamma_sum_scratch_bytes(p)) return NEGF_ERR_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(p->scratch) & 255) != 0) return NEGF_ERR_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(p->g) & 15) || (reinterpret_cast<uintptr_t>(p->gamma) & 15)) return NEGF_ERR_ARGUMENT;
  negf::cplx* Tst = reinterpret_cast<negf::cplx*>(p->scratch);
  negf::cplx* Gst = reinterpret_cast<negf::cplx*>(reinterpret_cast<char*>(p->scratch) + negf::gamma_stack_bytes(*p));
  const int smem = negf::GEMM_SMEM_BYTES;
  if (cudaFuncSetAttribute(negf::gamma_stack_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
      cudaFuncSetAttribute(negf::gamma_reduce_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
    return NEGF_ERR_CUDA;
  const int sms = negf::sm_count_or(148);
  const int grid1 = p->n_items < sms ? p->n_items : sms;
  negf::gamma_stack_kernel<<<grid1, negf::CTA_THREADS, smem, s>>>(*p, Tst, Gst);
  double* part = reinterpret_cast<double*>(reinterpret_cast<char*>(p->scratch) + 2 * negf::gamma_stack_bytes(*p));
  const int tiles = (p->n + negf::GT_M - 1) / negf::GT_M;
  const int64_t K = (int64_t)p->n_items * p->k;
  int split = (2 * sms + tiles * tiles - 1) / (tiles * tiles);  // about two CTAs per SM
  if (split > negf::GS_MAX_SPLIT) split = negf::GS_MAX_SPLIT;
  if ((int64_t)split > (K + 255) / 256) split = (int)((K + 255) / 256);  // keep ranges >= 256 deep
  if (split < 1) split = 1;
  const int64_t klen = negf::gamma_split_len(K, split);
  negf::gamma_reduce_kernel<<<dim3(tiles, tiles, split), negf::CTA_THREADS, smem, s>>>(*p, Tst, Gst, part, klen);
  const int64_t n2 = (int64_t)p->n * p->n;
  const int rgrid = (int)((n2 + 255) / 256 < 1024 ? (n2 + 255) / 256 : 1024);
  negf::gamma_sum_parts_kernel<<<rgrid, 256, 0, s>>>(p->out, part, n2, split);
  return cudaGetLastError() == cudaSuccess ? NEGF_OK : NEGF_ERR_CUDA;
}

size_t negf_lead_adjoint_scratch_bytes(const NegfLeadAdjProblem* p) {
  if (!p || p->n_slots <= 0 || p->lead.n <= 0) return 0;
  return (size_t)p->n_slots * negf::la_slot_elems(*p) * sizeof(double2);
}

int negf_lead_adjoint_run(const NegfLeadAdjProblem* p, void* stream) {
  if (!p || !p->arena || !p->items || !p->grad || !p->status || !p->scratch) return NEGF_ERR_ARGUMENT;
  const NegfLead& ld = p->lead;
  if (ld.n <= 0 || p->n_slots <= 0 || p->max_iter < 0 || p->form < 0 || p->form > 2) return NEGF_ERR_ARGUMENT;
  if (ld.n > NEGF_MAX_BLOCK || ld.nc > NEGF_MAX_BLOCK) return NEGF_ERR_UNSUPPORTED;
  if (p->form == 0 && (ld.nc <= 0 || ld.b <= 0 || ld.b > ld.n || ld.hdl < 0 || ld.sdl < 0)) return NEGF_ERR_ARGUMENT;
  if (p->scratch_bytes < negf_lead_adjoint_scratch_bytes(p)) return NEGF_ERR_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(p->scratch) & 255) != 0) return NEGF_ERR_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (p->n_items <= 0)
    return cudaMemsetAsync(p->grad, 0, (size_t)negf::la_grad_elems(*p) * sizeof(double2), s) == cudaSuccess
               ? NEGF_OK : NEGF_ERR_CUDA;
  const size_t smem = negf::lead_smem_bytes(negf::la_max_n(ld));
  if (cudaFuncSetAttribute(negf::lead_adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return NEGF_ERR_CUDA;
  const int grid = p->n_slots < p->n_items ? p->n_slots : p->n_items;
  negf::lead_adjoint_kernel<<<grid, negf::CTA_THREADS, smem, s>>>(*p);
  const int64_t total = negf::la_grad_elems(*p);
  const int rgrid = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
  negf::lead_adjoint_sum_kernel<<<rgrid, 256, 0, s>>>(*p, grid);
  return cudaGetLastError() == cudaSuccess ? NEGF_OK : NEGF_ERR_CUDA;
}

}  // extern "C"
