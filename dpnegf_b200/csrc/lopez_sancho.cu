// Batched Lopez-Sancho decimation for lead surface Green's functions and
// self-energies (sm_100a, FP64 tensor cores).
//
// Persistent kernel: one CTA per work slot pulls (lead, energy) items from an
// atomic queue and runs the whole decimation for that item in a private
// scratch slot, with the same CTA tile GEMM and blocked Gauss-Jordan inverse
// as the RGF sweep.  Follows _surface_green_numba_core
// (negf/surface_green.py:102-159) step for step:
//   alpha = h10 - z s10,  beta = h01 - z s01,  eps = eps_s = H
//   repeat (at most max_iter + 1 times):
//     [Xa Xb] = (zS - eps)^-1 [alpha beta]      (one LU solve, as the reference's
//                                                np.linalg.solve with stacked right-hand sides)
//     eps += alpha Xb + beta Xa;  eps_s += beta Xa
//     alpha <- alpha Xa;  beta <- beta Xb
//     stop when max(|alpha| + |beta|) < tol
//   g_s = (zS - eps_s)^-1, accepted when
//     max |(zS - H - (z s01 - h01) g_s (z s10 - h10)) g_s - I| < 3e-5
//     (warning status above 1e-8)
// The four products of a step are one GEMM of the stacked [alpha; beta] with
// [Xa Xb].  Complex products use the conventional 4M form: the doubling iteration
// amplifies the looser componentwise error of Gauss/3M products to ~1e-9 on
// g_s at ill-conditioned energies.
// and the self-energy product of selfEnergy (:73-86):
//   Sigma = (E S_DL - H_DL) g_s[:b,:b] (E S_DL^H - H_DL^H),   E without i*eta,
// or the bulk form Sigma = (E S - H) - g_s^-1 when the lead has no H_DL.
#include <cstdio>
#include "../../include/negf_b200.h"
#include "lead_forms.cuh"

namespace negf {

constexpr int LS_NBUF = 14;  // max_n^2 buffers per slot (see ls_item)
constexpr size_t LS_SCRATCH_HEADER = 256;

__host__ __device__ inline size_t ls_slot_elems(const NegfLsProblem& p) {
  size_t mn2 = (size_t)p.max_n * p.max_n;
  size_t e = LS_NBUF * mn2;
  return (e + 15) & ~(size_t)15;
}

NEGF_DEV void ls_item(const NegfLsProblem& P, const NegfLsItem& it, cplx* slot, char* smem_raw, double* red) {
  cplx* smem = reinterpret_cast<cplx*>(smem_raw);
  const NegfLead ld = P.leads[it.lead];
  // every slot buffer holds max_n^2 elements: refuse a lead that would not fit (H_DL products are
  // nc x b and nc x nc) before touching any memory.  The coupling product alone reads g from the
  // caller's memory and uses only nc x b and b x nc slot buffers.
  const bool sig_only = it.mode == NEGF_LS_SIGMA_FROM_GS;
  const bool bad_mode = it.mode != NEGF_LS_DECIMATE && !sig_only;
  const bool bad_size = sig_only ? (ld.nc <= 0 || ld.nc > P.max_n || ld.b > P.max_n)
                                 : (ld.n > P.max_n || ld.nc < 0 || ld.nc > P.max_n);
  if (bad_mode || bad_size || ld.n <= 0 || (ld.nc > 0 && (ld.b <= 0 || ld.b > ld.n))) {
    if (threadIdx.x == 0) {
      P.status[it.out] = NEGF_ERR_ARGUMENT;
      if (P.iters) P.iters[it.out] = 0;
      if (P.resid) P.resid[it.out] = INFINITY;
    }
    __syncthreads();
    return;
  }
  const int n = ld.n;
  const int64_t n2 = (int64_t)n * n;
  const size_t mn2 = (size_t)P.max_n * P.max_n;
  const cplx* ar = reinterpret_cast<const cplx*>(P.arena);
  const cplx* H = ar + ld.h;
  const cplx* S = ar + ld.s;
  const cplx* h01 = ar + ld.h01;
  const cplx* s01 = ar + ld.s01;
  const cplx E = cmk(it.e_re, it.e_im);
  const cplx z = cmk(it.e_re, it.e_im + it.eta);
  const cplx ONE = cmk(1.0, 0.0);
  cplx* b_[LS_NBUF];
  for (int i = 0; i < LS_NBUF; ++i) b_[i] = slot + i * mn2;
  // [alpha; beta] stacked (2n x n, row stride n) in the pair b_[2..3]; the next step's in b_[4..5]
  cplx *eps = b_[0], *epss = b_[1], *AB = b_[2], *AB2 = b_[4];
  // Xab = [Xa Xb] (n x 2n, row stride 2n) spans b_[8..9]; Pm = [alpha; beta][Xa Xb] (2n x 2n) spans
  // b_[10..13], whose blocks serve as T, gsb, t1, t2 once the doubling is done
  cplx *A = b_[6], *Xab = b_[8], *Pm = b_[10], *T = b_[10], *gsb = b_[11], *t1 = b_[12], *t2 = b_[13];
  cplx *Ya = b_[8], *Yb = b_[9];  // separate n x n work blocks once the doubling is done
  const int n2c = 2 * n;
  int bad = 0;
  auto lu_inverse = [&](cplx* W, cplx* out) { return cta_lu_inverse(W, out, n, smem_raw); };
  // Sigma = (E S_DL - H_DL) g[:b,:b] (E S_DL^H - H_DL^H) (selfEnergy, negf/surface_green.py:73-86)
  auto coupling_sigma = [&](const cplx* g, cplx* sig) {
    const int nc = ld.nc, b = ld.b;
    const cplx* hdl = ar + ld.hdl;
    const cplx* sdl = ar + ld.sdl;
    // t1 = E S_DL - H_DL  (nc x b)
    for (int e = threadIdx.x; e < nc * b; e += CTA_THREADS) t1[e] = csub(cmul(E, sdl[e]), hdl[e]);
    __syncthreads();
    // t2 = E S_DL^H - H_DL^H (b x nc)
    form_eS_minus_h_herm(t2, hdl, sdl, E, b, nc);
    gemm_ls<OP_N, OP_N>(smem, nc, b, b, t1, b, g, n, Ya, b);   // (E S_DL - H_DL) g[:b,:b]
    gemm_ls<OP_N, OP_N>(smem, nc, nc, b, Ya, b, t2, nc, sig, nc);
  };

  if (sig_only) {
    // the coupling product alone, on a surface Green's function the caller supplies (Bloch-unfolded
    // leads build g from the decimations of the folded cell)
    int st = NEGF_OK;
    if (it.gs && it.sigma) coupling_sigma(reinterpret_cast<const cplx*>(it.gs), reinterpret_cast<cplx*>(it.sigma));
    else st = NEGF_ERR_ARGUMENT;
    if (threadIdx.x == 0) {
      P.status[it.out] = st;
      if (P.iters) P.iters[it.out] = 0;
      if (P.resid) P.resid[it.out] = 0.0;
    }
    __syncthreads();
    return;
  }

  // alpha = h10 - z s10 = h01^H - z s01^H ; beta = h01 - z s01 ; eps = eps_s = H
  form_herm_shift(AB, h01, s01, z, n);
  cta_shift_form(AB + n2, h01, s01, z, ONE, (int)n2, smem);
  cta_shift_form(eps, H, nullptr, cmk(0.0, 0.0), ONE, (int)n2, smem);
  cta_shift_form(epss, H, nullptr, cmk(0.0, 0.0), ONE, (int)n2, smem);

  int it_n = 0;
  bool converged = false;
  for (int iter = 1; iter <= P.max_iter + 1; ++iter) {
    it_n = iter;
    // A = zS - eps;  [Xa Xb] = A^-1 [alpha beta]
    cta_shift_form(A, eps, S, z, cmk(-1.0, 0.0), (int)n2, smem);
    bad |= cta_lu_factor(A, n, n, smem_raw);
    {  // the right-hand sides [alpha beta] in the pivoted row order
      const int* perm = cta_lu_perm(smem_raw, n);
      for (int e = threadIdx.x; e < n2; e += CTA_THREADS) {
        const int i = e / n, j = e % n;
        const int64_t src = (int64_t)perm[i] * n + j;
        Xab[(int64_t)i * n2c + j] = AB[src];
        Xab[(int64_t)i * n2c + n + j] = AB[n2 + src];
      }
      __syncthreads();
    }
    cta_lu_trsolve(A, n, n, Xab, n2c, n2c, smem_raw);
    // the four products of the step in one GEMM: [alpha; beta] [Xa Xb] = [[aXa, aXb], [bXa, bXb]]
    gemm_ls<OP_N, OP_N>(smem, n2c, n2c, n, AB, n, Xab, n2c, Pm, n2c);
    // eps = eps + alpha Xb + beta Xa;  eps_s += beta Xa;  alpha <- alpha Xa;  beta <- beta Xb
    double m = 0.0;
    for (int e = threadIdx.x; e < n2; e += CTA_THREADS) {
      const int64_t i = e / n, j = e % n;
      const cplx aXa = Pm[i * n2c + j], aXb = Pm[i * n2c + n + j];
      const cplx bXa = Pm[(n + i) * n2c + j], bXb = Pm[(n + i) * n2c + n + j];
      eps[e] = cadd(cadd(eps[e], aXb), bXa);
      epss[e] = cadd(epss[e], bXa);
      AB2[e] = aXa;
      AB2[n2 + e] = bXb;
      const double v = cabs1(aXa) + cabs1(bXb);  // bounds |aXa| + |bXb| within a factor sqrt(2)
      m = (v == v) ? fmax(m, v) : INFINITY;
    }
    cplx* t = AB; AB = AB2; AB2 = t;
    m = cta_max(m, red);  // begins with a barrier: the pass above is complete
    // The reference's test is max(|alpha| + |beta|) < tol with complex moduli.  Since
    // cabs1(z) / sqrt(2) <= |z| <= cabs1(z), the bound m decides it (with 8 ulp of slack for the
    // rounding of both sums) unless m lies within a factor sqrt(2) of tol; only then are the
    // moduli summed, so the decision and the step count are those of the moduli.
    constexpr double SLACK = 8.0 * 2.220446049250313e-16, RSQRT2 = 0.70710678118654752440;
    bool conv = false;
    if (isfinite(m) && m * (1.0 + SLACK) < P.tol) {
      conv = true;
    } else if (isfinite(m) && m * (1.0 - SLACK) * RSQRT2 < P.tol) {
      double x = 0.0;
      for (int e = threadIdx.x; e < n2; e += CTA_THREADS) {
        const double v = hypot(AB[e].x, AB[e].y) + hypot(AB[n2 + e].x, AB[n2 + e].y);
        x = (v == v) ? fmax(x, v) : INFINITY;
      }
      m = cta_max(x, red);
      conv = m < P.tol;
    }
    if (conv) { converged = true; break; }
    if (!isfinite(m)) break;
  }

  int st = NEGF_OK;
  double res = INFINITY;
  if (!converged) {
    st = NEGF_ERR_LS_NOT_CONVERGED;
  } else {
    cplx* gs = it.gs ? reinterpret_cast<cplx*>(it.gs) : gsb;
    // g_s = (zS - eps_s)^-1
    cta_shift_form(A, epss, S, z, cmk(-1.0, 0.0), (int)n2, smem);
    bad |= lu_inverse(A, gs);
    // residual: (zS - H - (z s01 - h01) g_s (z s10 - h10)) g_s - I
    // z s01 - h01
#pragma unroll 4
    for (int e = threadIdx.x; e < n2; e += CTA_THREADS) t1[e] = csub(cmul(z, s01[e]), h01[e]);
    __syncthreads();
    // z s10 - h10 = z s01^H - h01^H
    form_eS_minus_h_herm(t2, h01, s01, z, n, n);
    gemm_ls<OP_N, OP_N>(smem, n, n, n, t1, n, gs, n, Ya, n);  // (z s01 - h01) g_s
    gemm_ls<OP_N, OP_N>(smem, n, n, n, Ya, n, t2, n, Yb, n);  // ... (z s10 - h10)
    // test = zS - H - Yb
#pragma unroll 4
    for (int e = threadIdx.x; e < n2; e += CTA_THREADS) T[e] = csub(csub(cmul(z, S[e]), H[e]), Yb[e]);
    __syncthreads();
    gemm_ls<OP_N, OP_N>(smem, n, n, n, T, n, gs, n, Ya, n);  // test g_s
    double m = 0.0;
    for (int e = threadIdx.x; e < n2; e += CTA_THREADS) {
      cplx v = Ya[e];
      if (e / n == e % n) v.x -= 1.0;
      double a = hypot(v.x, v.y);
      m = (a == a) ? fmax(m, a) : INFINITY;
    }
    res = cta_max(m, red);
    if (!(res < 3.0e-5)) st = NEGF_ERR_LS_RESIDUAL;
    else if (res > 1.0e-8) st = NEGF_WARN_LS_CONVERGENCE;

    if (it.sigma && st != NEGF_ERR_LS_RESIDUAL) {
      cplx* sig = reinterpret_cast<cplx*>(it.sigma);
      if (ld.nc > 0) {
        coupling_sigma(gs, sig);
      } else {
        // bulk form: Sigma = (E S - H) - g_s^-1
        cta_shift_form(A, gs, nullptr, cmk(0.0, 0.0), ONE, (int)n2, smem);
        bad |= lu_inverse(A, Ya);
#pragma unroll 4
        for (int e = threadIdx.x; e < n2; e += CTA_THREADS) sig[e] = csub(csub(cmul(E, S[e]), H[e]), Ya[e]);
        __syncthreads();
      }
    }
  }
  if (bad && st == NEGF_OK) st = NEGF_ERR_SINGULAR;
  if (threadIdx.x == 0) {
    P.status[it.out] = st;
    if (P.iters) P.iters[it.out] = it_n;
    if (P.resid) P.resid[it.out] = res;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(CTA_THREADS, 1) ls_kernel(const NegfLsProblem P) {
  extern __shared__ __align__(16) char smem[];
  __shared__ int s_item;
  __shared__ double red[CTA_THREADS / 32];
  unsigned* queue = reinterpret_cast<unsigned*>(P.scratch);
  cplx* slot = reinterpret_cast<cplx*>(reinterpret_cast<char*>(P.scratch) + LS_SCRATCH_HEADER) +
               (size_t)blockIdx.x * ls_slot_elems(P);
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(queue, 1u);
    __syncthreads();
    const int idx = s_item;
    __syncthreads();
    if (idx >= P.n_items) break;
    const NegfLsItem it = P.items[idx];
    ls_item(P, it, slot, smem, red);
  }
}

size_t ls_smem_bytes(int max_n) { return lead_smem_bytes(max_n); }

}  // namespace negf

extern "C" {

size_t negf_lopez_sancho_scratch_bytes(const NegfLsProblem* p) {
  if (!p || p->n_slots <= 0 || p->max_n <= 0) return 0;
  return negf::LS_SCRATCH_HEADER + (size_t)p->n_slots * negf::ls_slot_elems(*p) * sizeof(double2);
}

int negf_lopez_sancho_run(const NegfLsProblem* p, void* stream) {
  if (!p || !p->leads || !p->items || !p->arena || !p->status || !p->scratch) return NEGF_ERR_ARGUMENT;
  if (p->n_items <= 0) return NEGF_OK;
  if (p->max_n <= 0 || p->n_slots <= 0 || p->max_iter < 0) return NEGF_ERR_ARGUMENT;
  if (p->max_n > NEGF_MAX_BLOCK) return NEGF_ERR_UNSUPPORTED;
  if (p->scratch_bytes < negf_lopez_sancho_scratch_bytes(p)) return NEGF_ERR_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(p->scratch) & 255) != 0) return NEGF_ERR_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const size_t smem = negf::ls_smem_bytes(p->max_n);
  if (cudaFuncSetAttribute(negf::ls_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return NEGF_ERR_CUDA;
  if (cudaMemsetAsync(p->scratch, 0, negf::LS_SCRATCH_HEADER, s) != cudaSuccess) return NEGF_ERR_CUDA;
  const int grid = p->n_slots < p->n_items ? p->n_slots : p->n_items;
  negf::ls_kernel<<<grid, negf::CTA_THREADS, smem, s>>>(*p);
  return cudaGetLastError() == cudaSuccess ? NEGF_OK : NEGF_ERR_CUDA;
}

}  // extern "C"
