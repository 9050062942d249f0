/*
 * negf_b200.h -- C ABI of the B200-native NEGF transport core.
 *
 * Every entry point takes plain pointers and sizes.  All array pointers in the
 * problem descriptors are DEVICE pointers (cudaMalloc'd or torch-owned CUDA
 * memory) unless a field says otherwise; complex numbers are complex128
 * stored interleaved (re, im) -- the layout of torch.complex128 / numpy
 * complex128, so caller tensors are passed without conversion.  Calls are
 * asynchronous on the given stream and allocate no device memory: scratch is
 * supplied by the caller (size from the matching *_scratch_bytes query).
 *
 * Offsets named "offset" count complex elements (16 bytes), not bytes.
 *
 * Reference interfaces replaced (dpnegf, paths relative to its source tree):
 *   negf_rgf_run           negf/recursive_green_cal.py:4-296  recursive_gf_cal
 *                          (called by recursive_gf :324-477), fused with the
 *                          T(E) / DOS / LDOS reductions of
 *                          negf/device_property.py:374-470
 *   negf_lopez_sancho_run  negf/surface_green.py:102-159  _surface_green_numba_core
 *                          + the self-energy product of selfEnergy :9-91
 */
#ifndef NEGF_B200_H
#define NEGF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (per call and per work item) ------------------------- */
#define NEGF_OK 0
#define NEGF_WARN_LS_CONVERGENCE 1 /* Lopez-Sancho residual in (1e-8, 3e-5): surface_green.py:149-150 */
#define NEGF_ERR_LS_NOT_CONVERGED 2 /* > 100 decimation steps: surface_green.py:156-157 (RuntimeError) */
#define NEGF_ERR_LS_RESIDUAL 3      /* residual >= 3e-5: surface_green.py:154 (ArithmeticError) */
#define NEGF_ERR_SINGULAR 4         /* zero / non-finite pivot (torch.linalg.solve raises) */
#define NEGF_ERR_NONFINITE 5        /* non-finite result */
#define NEGF_ERR_TIMEOUT 6          /* a bounded tensor-core completion wait expired (NEGF_MIXED) */
#define NEGF_ERR_ARGUMENT -1        /* malformed descriptor (call-level) */
#define NEGF_ERR_UNSUPPORTED -2     /* block size above the compiled maximum (call-level) */
#define NEGF_ERR_CUDA -3            /* CUDA launch / attribute error (call-level) */
#define NEGF_ERR_SCRATCH_LIMIT -4   /* negf_rgf_run_static: one work slot needs more than the static array */

#define NEGF_MAX_BLOCK 512 /* largest diagonal block the kernels accept */

/* ---- RGF output selection (NegfRgfProblem.flags) ------------------------ */
#define NEGF_OUT_GTRANS (1u << 0)  /* g_trans = G_{1N}           [n_0 x n_{K-1}] */
#define NEGF_OUT_GR_LC (1u << 1)   /* gr_lc[q] = G_{q,N}         [n_q x n_{K-1}] */
#define NEGF_OUT_GRD (1u << 2)     /* grd[q]  = G_{q,q}          [n_q x n_q]     */
#define NEGF_OUT_GRL (1u << 3)     /* grl[q]  = G_{q+1,q}        [n_{q+1} x n_q] */
#define NEGF_OUT_GRU (1u << 4)     /* gru[q]  = G_{q,q+1}        [n_q x n_{q+1}] */
#define NEGF_OUT_GR_LEFT (1u << 5) /* gr_left[q] = g_q (left-connected) [n_q x n_q] */
#define NEGF_TRANS (1u << 6)       /* T(E) = Re Tr[G_L G_1N G_R G_1N^H] -> trans[]  */
#define NEGF_ORB_DOS (1u << 7)     /* -Im diag(G S)_i / pi per orbital -> orb_dos[] */
#define NEGF_LESSER (1u << 8)      /* lesser sweep: gin_left, gnd, gnl, gnu          */
#define NEGF_DOS (1u << 9)         /* DOS = 2 sum_i (-Im diag(G S)_i / pi) -> dos[]  */
#define NEGF_ORB_GDIAG (1u << 10)  /* diag(G_qq) per orbital (complex128)  -> orb_g[] */
#define NEGF_ORB_AR (1u << 11)     /* diag(G_qN Gamma_R G_qN^H) per orbital -> orb_ar[] */
#define NEGF_ADJOINT (1u << 12)    /* accumulate d(sum_items w_T T)/d(H, S) and dT/dSigma (single device) */
#define NEGF_MIXED (1u << 13)      /* mixed precision: every block product on tcgen05 3xTF32 (FP32-accurate
                                      products, FP32 accumulation); pivots, panels and storage stay FP64 */
#define NEGF_REFINE (1u << 14)     /* with NEGF_TRANS: refine_steps iterative-refinement steps of the column
                                      G_{:,N} before T(E) -- FP64 residual E_N - (zS - H - Sigma) G_{:,N} on
                                      FP64 tensor cores, correction solved with the stored g_q (needs
                                      col_slab); gr_lc outputs carry the refined column */
#define NEGF_ADJ_DOS (1u << 16)    /* with NEGF_ADJOINT: also accumulate the gradient of sum_items w_d DOS(E)
                                      (the summed onsite density over the items' energies, DOS as in
                                      NEGF_DOS) by a z-tangent sweep: Tr[G S] = d/dz log det(zS - H - Sigma),
                                      so the gradient needs the BTD blocks of G S G = -dG/dz */
#define NEGF_GREATER (1u << 15)    /* greater sweep from s_out: gip_left, gpd, gpl, gpu
                                      (recursive_green_cal.py:143-161, :267-289) */

/* Phase indices of NegfRgfProblem.phase_cycles (clock64 cycles per slot). */
#define NEGF_PHASES 12 /* form, gemm_fwd, inv_stage, inv_panel, inv_update, inv_gather,
                          gemm_bwd, lesser, dos, trans, other, refine */

/* One diagonal block q of a block-tridiagonal device. */
typedef struct NegfBlock {
  int32_t n;      /* n_q */
  int32_t n_next; /* n_{q+1}; 0 for the last block */
  int64_t hd, sd; /* offsets of H_qq, S_qq in hs */
  int64_t hu, su; /* offsets of H_{q,q+1}, S_{q,q+1} [n_q x n_{q+1}]; -1 = zero block */
  int64_t hl, sl; /* offsets of H_{q+1,q}, S_{q+1,q} [n_{q+1} x n_q]; -1 = zero block */
  int64_t sdT, suT, slT; /* transposed copies S_qq^T, S_{q,q+1}^T, S_{q+1,q}^T (row-major) used by
                            the DOS diagonals; -1 = zero block */
  int64_t orb0;   /* first orbital of block q within its device */
  int64_t g;      /* offset of g_q inside one item's g slab (prefix sum of n^2) */
  int64_t gc;     /* NEGF_ADJOINT: offset of G_qN in the per-slot column slab (prefix of n_q n_N) */
  int64_t gu;     /* NEGF_ADJOINT: offset of the coupling gradients of block q (prefix of n_q n_{q+1}) */
  /* block outputs: offset of batch row 0 in out; row b adds b * (block size).
     -1 when not produced. */
  int64_t o_grd, o_grl, o_gru, o_grlc, o_grleft;
  int64_t o_gnd, o_gnl, o_gnu, o_ginleft;
  int64_t s_in; /* lesser input Sigma^in_q for batch row 0 in s_in; -1 = zero */
  int64_t o_gpd, o_gpl, o_gpu, o_gipleft; /* NEGF_GREATER block outputs (same row rule); -1 = not produced */
  int64_t s_out; /* greater input Sigma^out_q for batch row 0 in s_out; -1 = zero */
} NegfBlock;

/* One device (k-point / realisation): a run of n_blocks NegfBlock entries. */
typedef struct NegfDevice {
  int32_t n_blocks; /* K */
  int32_t blk0;     /* index of block 0 in the block table */
  int32_t n_orb;    /* sum of n_q */
  int32_t pad;
  int64_t o_gtrans; /* g_trans for batch row 0 in out; -1 when not produced */
  int64_t g_slab;   /* elements of one item's g slab (sum of n_q^2) */
} NegfDevice;

/* One work item: a device at one complex energy. */
typedef struct NegfItem {
  int32_t dev;     /* device index */
  int32_t row;     /* batch row of this energy within the device's outputs */
  double z_re;     /* z = E + E_ref + i*eta (recursive_green_cal.py:75,:378) */
  double z_im;
  const double* se_l; /* Sigma_L [nse_l x nse_l] complex128 (device memory); NULL = none */
  const double* se_r; /* Sigma_R [nse_r x nse_r] complex128 (device memory); NULL = none */
  int32_t nse_l, nse_r;
  int64_t out;     /* index into trans[] and status[] */
  int64_t orb;     /* offset (doubles) of this item's n_orb entries in orb_dos[] */
  double w_t;      /* NEGF_ADJOINT: weight of this item's T(E) in the loss */
  double* gse_l;   /* NEGF_ADJOINT: d loss / d Sigma_L [nse_l x nse_l] (torch convention); NULL = skip */
  double* gse_r;   /* NEGF_ADJOINT: d loss / d Sigma_R [nse_r x nse_r]; NULL = skip */
  double w_d;      /* NEGF_ADJ_DOS: weight of this item's DOS(E) in the loss */
} NegfItem;

typedef struct NegfRgfProblem {
  const NegfBlock* blocks;  /* device memory */
  const NegfDevice* devices; /* device memory */
  const NegfItem* items;    /* device memory, processed in this order */
  int32_t n_items;
  int32_t max_n;            /* largest n_q over all devices (<= NEGF_MAX_BLOCK); with max_g_slab and
                               col_slab it sizes every slot, and the kernel trusts the tables to fit */
  int64_t max_g_slab;       /* largest g slab over all devices */
  const double* hs;         /* complex128 arena of H/S blocks */
  const double* s_in;       /* complex128 arena of Sigma^in blocks (NEGF_LESSER) */
  double* out;              /* complex128 arena of block outputs */
  double* trans;            /* [n_items] T(E) (NEGF_TRANS) */
  double* orb_dos;          /* per-orbital -Im diag(GS)/pi (NEGF_ORB_DOS) */
  double* dos;              /* [n_items] DOS with spin factor 2 (NEGF_DOS) */
  double* orb_g;            /* complex128 per-orbital diag(G_qq), item offset = NegfItem.orb (NEGF_ORB_GDIAG) */
  double* orb_ar;           /* per-orbital diag(G_qN Gamma_R G_qN^H), offset NegfItem.orb (NEGF_ORB_AR) */
  int32_t* status;          /* [n_items] per-item status (always written) */
  uint32_t flags;
  int32_t n_slots;          /* concurrent work slots = CTAs launched */
  void* scratch;            /* >= negf_rgf_scratch_bytes(problem) bytes, 256-aligned */
  size_t scratch_bytes;
  unsigned long long* phase_cycles; /* optional [n_slots x NEGF_PHASES] SM-cycle counters; NULL = off */
  /* NEGF_ADJOINT: per-slot gradient accumulators, complex128, [n_slots x grad_slab]; the caller
     zeroes them and sums over slots.  Within a slot: d/dhd, d/dsd at g offsets (g_slab each),
     then d/dhu, d/dsu, d/dhl, d/dsl at gu offsets (u_slab = sum n_q n_{q+1} each).
     Gradients follow torch's convention for complex inputs: dL/dRe + i dL/dIm. */
  double* grad;
  int64_t grad_slab;        /* complex elements per slot: 2 g_slab + 4 u_slab */
  int64_t col_slab;         /* NEGF_ADJOINT / NEGF_REFINE: sum_q n_q n_N (last-column slab per slot) */
  int32_t refine_steps;     /* NEGF_REFINE: at most this many refinement steps (<= 0 means 1); an item
                               stops early once the correction to G_1N is below 1e-10 relative */
  int32_t inv_ob;           /* Gauss-Jordan outer block width: 32, 64, 128, 256 or 512 columns (0 = 128);
                               results agree to rounding, the speed depends on block size and precision */
  const double* s_out;      /* complex128 arena of Sigma^out blocks (NEGF_GREATER) */
  int32_t inv_mode;         /* 0: Gauss-Jordan with partial pivoting over the whole block (inv_ob);
                               1: recursive 2x2 block inverse, pivoting only inside 64-wide leaves and
                               every update a CTA GEMM.  Mode 1 needs nonsingular leading sub-blocks,
                               which the retarded problem guarantees for eta > 0 (zS - H - Sigma - L g U
                               has a positive-definite imaginary part when H is Hermitian, S positive
                               definite and Im Sigma <= 0) */
  int32_t ckpt;             /* NEGF_ADJOINT: 0 keeps every left-connected g_q (and, with NEGF_ADJ_DOS, its
                               z-tangent) for the whole item; s > 0 keeps only g_q for q = 0, s, 2s, ...
                               plus one segment of s blocks, and recomputes each segment from its
                               checkpoint when the backward sweep and the adjoint pass reach it (sqrt(K)
                               checkpointing: g storage (ceil(K/s) + s) max_n^2 instead of sum n_q^2, at
                               the cost of up to two extra forward sweeps).  Not with gr_left outputs,
                               lesser, greater or refinement */
  int32_t ckpt_blocks;      /* with ckpt > 0: the device's block count K (sizes the checkpoint area) */
} NegfRgfProblem;

/* ---- Lopez-Sancho lead decimation ------------------------------------ */

/* One lead principal layer (energy independent).  Offsets into `arena`. */
typedef struct NegfLead {
  int32_t n;   /* principal-layer size */
  int32_t nc;  /* rows of H_DL (device side of the coupling); 0 = bulk form Sigma = (ES - H) - g_s^-1 */
  int32_t b;   /* columns of H_DL (leading block of g_s used), <= n */
  int32_t pad;
  int64_t h, s, h01, s01; /* H, S, H_01, S_01 [n x n] (H_01 couples the surface layer to the next) */
  int64_t hdl, sdl;       /* H_DL, S_DL [nc x b]; -1 when nc == 0 */
} NegfLead;

/* One decimation: a lead at one energy. */
/* NegfLsItem.mode */
#define NEGF_LS_DECIMATE 0       /* decimation, g_s, residual check, Sigma */
#define NEGF_LS_SIGMA_FROM_GS 1  /* Sigma = (E S_DL - H_DL) g[:b,:b] (E S_DL^H - H_DL^H) from the item's gs as INPUT
                                    (lead.n x lead.n, row stride lead.n) with no decimation; needs lead.nc > 0.
                                    The Bloch-unfolded self-energy of LeadProperty.self_energy
                                    (negf/lead_property.py:330-379) builds g from the folded cell's decimations */

typedef struct NegfLsItem {
  int32_t lead;
  int32_t mode;      /* NEGF_LS_DECIMATE or NEGF_LS_SIGMA_FROM_GS */
  double e_re, e_im; /* E = energy + E_ref (may be complex, e.g. Ozaki poles) */
  double eta;        /* decimation runs at z = E + i eta (surface_green.py:65-70, :83) */
  double* sigma;     /* complex128 [nc x nc] (or [n x n] bulk form) output; NULL = not wanted */
  double* gs;        /* complex128 [n x n] surface Green's function output; NULL = not wanted */
  int64_t out;       /* index into status[], iters[], resid[] */
} NegfLsItem;

typedef struct NegfLsProblem {
  const NegfLead* leads;    /* device memory */
  const NegfLsItem* items;  /* device memory */
  int32_t n_items;
  int32_t max_n;            /* largest of n and nc over all leads (sizes the slot buffers; an item whose
                               lead exceeds it gets NEGF_ERR_ARGUMENT as its status and is skipped) */
  const double* arena;      /* complex128 lead blocks */
  int32_t* status;          /* [n_items]: NEGF_OK, NEGF_WARN_LS_CONVERGENCE, NEGF_ERR_LS_* , NEGF_ERR_SINGULAR */
  int32_t* iters;           /* [n_items] decimation steps taken */
  double* resid;            /* [n_items] max |(ES - H - (zs01-h01) g_s (zs10-h10)) g_s - I| */
  double tol;               /* convergence threshold on max(|alpha|+|beta|) (1e-40 in the reference) */
  int32_t max_iter;         /* 100 in the reference: the step after it raises */
  int32_t n_slots;
  void* scratch;
  size_t scratch_bytes;
} NegfLsProblem;

/* Bytes of scratch negf_lopez_sancho_run needs for p->n_slots and p->max_n. */
size_t negf_lopez_sancho_scratch_bytes(const NegfLsProblem* p);

/* Batched Lopez-Sancho decimation over (lead, energy) items, one CTA per item.
 * Replaces _surface_green_numba_core (negf/surface_green.py:102-159) and the
 * self-energy product of selfEnergy (:9-91):
 *   alpha = h10 - z s10, beta = h01 - z s01, eps = eps_s = H;
 *   [Xa Xb] = (zS - eps)^-1 [alpha beta]; eps += alpha Xb + beta Xa;
 *   eps_s += beta Xa; alpha <- alpha Xa; beta <- beta Xb
 * until max(|alpha| + |beta|) < tol; g_s = (zS - eps_s)^-1 with the residual
 * check of :142-155; Sigma = (E S_DL - H_DL) g_s[:b,:b] (E S_DL^H - H_DL^H). */
int negf_lopez_sancho_run(const NegfLsProblem* p, void* cuda_stream);

/* Weighted sum of G Gamma G^H products over energies:
 *   out = sum_i w_i Re(G_i[:, c0:c0+k] Gamma_i G_i[:, c0:c0+k]^H)      (real n x n, row stride n)
 * the non-equilibrium density matrix of Ozaki.integrate (negf/density.py:183-195:
 * DM_neq = sum_i wlg_i (G_i Gamma_R,i G_i^H).real (f_R - f_L)(x_i), Gamma_R in the corner of G). */
typedef struct NegfGammaSum {
  const double* g;       /* complex128; item i's G at g + i * g_stride (complex elements), n rows of stride ldg */
  int64_t g_stride;
  const double* gamma;   /* complex128; item i's Gamma (k x k, row stride ldgam) at gamma + i * gamma_stride */
  int64_t gamma_stride;
  const double* w;       /* [n_items] real weights (device memory) */
  double* out;           /* [n x n] real output (device memory) */
  int32_t n_items;
  int32_t n;             /* rows of G and of out */
  int32_t ldg;           /* >= c0 + k */
  int32_t c0;            /* first column of G that Gamma couples to */
  int32_t k;             /* size of Gamma */
  int32_t ldgam;         /* >= k */
  void* scratch;         /* 256-byte aligned, negf_gamma_sum_scratch_bytes */
  size_t scratch_bytes;
} NegfGammaSum;

size_t negf_gamma_sum_scratch_bytes(const NegfGammaSum* p);
/* Two launches on the stream: per-energy products, then one GEMM over all energies in order
 * (bitwise reproducible).  Returns NEGF_OK or a call-level error. */
int negf_gamma_sum_run(const NegfGammaSum* p, void* cuda_stream);

/* Gradient of a loss through one lead's self-energies at many energies, by implicit
 * differentiation of the converged decimation: g_s is the fixed point of
 * f(g) = (zS - H - tau g tau')^-1, tau = z S01 - H01, tau' = z S01^H - H01^H (the relation
 * the reference's residual check tests, negf/surface_green.py:142-145).  With V = dL/dg_s from
 * Sigma(g_s), Lambda = V + (g_s tau)^H Lambda (tau' g_s)^H is solved by doubling and
 * dL/dtheta = Lambda-weighted derivative of f at the fixed point, plus Sigma's explicit terms.
 * No reference counterpart: the reference differentiates through its decimation loop with
 * torch autograd. */
typedef struct NegfLeadAdjItem {
  double e_re, e_im;     /* E = energy + E_ref (Sigma uses E; g_s was computed at z = E + i eta) */
  const double* gs;      /* complex128 [n x n] converged g_s */
  const double* gsig;    /* complex128 dL/dSigma (PyTorch convention): [nc x nc] for form 0, else [n x n] */
} NegfLeadAdjItem;

typedef struct NegfLeadAdjProblem {
  NegfLead lead;                /* blocks as offsets into arena; hdl/sdl used by form 0 */
  const double* arena;          /* complex128 lead blocks */
  const NegfLeadAdjItem* items; /* device memory */
  int32_t n_items;
  int32_t form;                 /* 0: Sigma = (E S_DL - H_DL) g_s[:b,:b] (E S_DL^H - H_DL^H);
                                   1: Sigma = g_s^-1; 2: Sigma = E S - H - g_s^-1 */
  double eta;
  double tol;                   /* doubling stops once max|P| max|Q| < tol */
  int32_t max_iter;             /* doubling steps at most */
  int32_t n_slots;              /* CTAs; energies go to them round-robin */
  double* grad;                 /* complex128 out: dL/dH, dL/dH01, dL/dS, dL/dS01 [n x n] each, then
                                   dL/dH_DL, dL/dS_DL [nc x b] each for form 0; summed over energies */
  int32_t* status;              /* [n_items] NEGF_OK, NEGF_ERR_SINGULAR, NEGF_ERR_NONFINITE */
  int32_t* iters;               /* [n_items] doubling steps (may be NULL) */
  void* scratch;                /* 256-byte aligned, negf_lead_adjoint_scratch_bytes */
  size_t scratch_bytes;
} NegfLeadAdjProblem;

size_t negf_lead_adjoint_scratch_bytes(const NegfLeadAdjProblem* p);
int negf_lead_adjoint_run(const NegfLeadAdjProblem* p, void* cuda_stream);

/* Bytes of scratch negf_rgf_run needs for p->n_slots, p->max_n, p->max_g_slab, p->flags. */
size_t negf_rgf_scratch_bytes(const NegfRgfProblem* p);

/* Batched RGF sweep over p->n_items (device, energy) items.  Replaces
 * recursive_gf_cal (negf/recursive_green_cal.py:4-296): forward left-connected
 * g_q = (-D_q - L_{q-1} g_{q-1} U_{q-1})^-1 with D = H + Sigma - zS, L = hl - z sl,
 * U = hu - z su; backward G_qq, G_{q+1,q}, G_{q,q+1}, G_{q,N}; optional lesser
 * sweep (:121-140) and greater sweep (:143-161).  T(E) (device_property.py:374-406) and the per-orbital DOS
 * diagonal (:408-470) are reduced inside the sweep.  Returns a call-level
 * status; per-item status in p->status. */
int negf_rgf_run(const NegfRgfProblem* p, void* cuda_stream);

/* negf_rgf_run for callers that cannot allocate device memory (no counterpart
 * in the reference, which allocates through torch on every call).  A host code
 * that embeds the sweep in its own solver loop often owns the GPU through its
 * own memory pool or receives only input/output buffers, and cudaMalloc would
 * synchronise the device or fail there.  This entry point takes its scratch
 * from a 64 MiB array inside the library (one per GPU, kept until exit)
 * instead of p->scratch / p->scratch_bytes, which are ignored, and allocates
 * nothing.  Inputs and outputs are still the caller's.  The slot count is
 * lowered to what fits; a problem whose single slot does not fit returns
 * NEGF_ERR_SCRATCH_LIMIT.  All calls on a GPU share the array (the work-queue
 * counter is cleared on entry; overlapping calls on the GPU race), and the
 * first call on a device resolves the array's address, so make it before any
 * stream capture. */
int negf_rgf_run_static(const NegfRgfProblem* p, void* cuda_stream);

/* Work slots negf_rgf_run_static will run for this problem: p->n_slots lowered to what fits in
 * the static array (>= 1), or NEGF_ERR_SCRATCH_LIMIT / NEGF_ERR_ARGUMENT / NEGF_ERR_UNSUPPORTED.
 * Host-only arithmetic, no device access.  The array's address is looked up once per device and
 * kept for the life of the process, so no negf_rgf_run_static call may follow a cudaDeviceReset. */
int negf_rgf_static_slots(const NegfRgfProblem* p);

/* Size in bytes of the static scratch array used by negf_rgf_run_static. */
size_t negf_rgf_static_scratch_bytes(void);

/* Number of SMs of the current CUDA device (grid sizing helper). */
int negf_sm_count(void);

/* Library version string. */
const char* negf_version(void);

/* sizeof of the ABI structs (0 NegfBlock, 1 NegfDevice, 2 NegfItem,
 * 3 NegfRgfProblem, 4 NegfLead, 5 NegfLsItem, 6 NegfLsProblem, 7 NegfGammaSum,
 * 8 NegfLeadAdjItem, 9 NegfLeadAdjProblem) so bindings
 * can verify their mirrors; 0 if unknown. */
size_t negf_abi_struct_size(int which);

#ifdef __cplusplus
}
#endif
#endif /* NEGF_B200_H */
