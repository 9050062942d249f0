// The C ABI of the RGF sweep (include/negf_b200.h) and its FP64 kernels; the sweep itself is
// in rgf_sweep.cuh, the mixed-precision kernel in rgf_mx.cu.
#include "rgf_sweep.cuh"

namespace negf {

int rgf_launch_fp64(int feat, const NegfRgfProblem& p, size_t smem, int grid, cudaStream_t s) {
  if (feat == FEAT_ADJOINT) return rgf_launch_impl<false, FEAT_ADJOINT>(p, smem, grid, s);
  if (feat == FEAT_LESSER) return rgf_launch_impl<false, FEAT_LESSER>(p, smem, grid, s);
  return rgf_launch_impl<false, FEAT_RETARDED>(p, smem, grid, s);
}

}  // namespace negf

extern "C" {

size_t negf_rgf_scratch_bytes(const NegfRgfProblem* p) {
  if (!p || p->n_slots <= 0 || p->max_n <= 0) return 0;
  return negf::RGF_SCRATCH_HEADER + (size_t)p->n_slots * negf::rgf_slot_elems(*p) * sizeof(double2);
}

int negf_rgf_run(const NegfRgfProblem* p, void* stream) {
  if (!p || !p->blocks || !p->devices || !p->items || !p->hs || !p->status || !p->scratch) return NEGF_ERR_ARGUMENT;
  if (p->n_items <= 0) return NEGF_OK;
  if (p->max_n <= 0 || p->n_slots <= 0) return NEGF_ERR_ARGUMENT;
  if (p->max_n > NEGF_MAX_BLOCK) return NEGF_ERR_UNSUPPORTED;
  if (p->scratch_bytes < negf_rgf_scratch_bytes(p)) return NEGF_ERR_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(p->scratch) & 255) != 0) return NEGF_ERR_ARGUMENT;
  if ((p->flags & NEGF_TRANS) && !p->trans) return NEGF_ERR_ARGUMENT;
  if ((p->flags & NEGF_ORB_DOS) && !p->orb_dos) return NEGF_ERR_ARGUMENT;
  if ((p->flags & NEGF_DOS) && !p->dos) return NEGF_ERR_ARGUMENT;
  if ((p->flags & NEGF_ORB_GDIAG) && !p->orb_g) return NEGF_ERR_ARGUMENT;
  if ((p->flags & NEGF_ORB_AR) && !p->orb_ar) return NEGF_ERR_ARGUMENT;
  if ((p->flags & NEGF_ADJOINT) &&
      (!p->grad || p->grad_slab <= 0 || p->col_slab <= 0 || !(p->flags & NEGF_TRANS)))
    return NEGF_ERR_ARGUMENT;
  if ((p->flags & NEGF_REFINE) && (p->col_slab <= 0 || !(p->flags & NEGF_TRANS))) return NEGF_ERR_ARGUMENT;
  if ((p->flags & NEGF_ADJ_DOS) && !(p->flags & NEGF_ADJOINT)) return NEGF_ERR_ARGUMENT;
  if (p->ckpt < 0) return NEGF_ERR_ARGUMENT;
  if (p->ckpt > 0 && (p->flags & NEGF_ADJOINT) &&
      ((p->flags & (NEGF_OUT_GR_LEFT | NEGF_LESSER | NEGF_GREATER | NEGF_REFINE)) || p->ckpt_blocks <= 0))
    return NEGF_ERR_ARGUMENT;
  if (p->inv_mode != 0 && p->inv_mode != 1) return NEGF_ERR_ARGUMENT;
  if (p->inv_ob != 0 && p->inv_ob != 32 && p->inv_ob != 64 && p->inv_ob != 128 && p->inv_ob != 256 &&
      p->inv_ob != 512)
    return NEGF_ERR_ARGUMENT;
  const uint32_t blockouts = NEGF_OUT_GTRANS | NEGF_OUT_GR_LC | NEGF_OUT_GRD | NEGF_OUT_GRL | NEGF_OUT_GRU |
                             NEGF_OUT_GR_LEFT | NEGF_LESSER | NEGF_GREATER;
  if ((p->flags & blockouts) && !p->out) return NEGF_ERR_ARGUMENT;
  if ((p->flags & NEGF_LESSER) && !p->s_in) return NEGF_ERR_ARGUMENT;
  if ((p->flags & NEGF_GREATER) && !p->s_out) return NEGF_ERR_ARGUMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const bool mixed = (p->flags & NEGF_MIXED) != 0;
  const size_t smem = negf::rgf_smem_bytes(p->max_n, mixed);
  const int feat = (p->flags & NEGF_ADJOINT) ? negf::FEAT_ADJOINT
                   : (p->flags & (NEGF_LESSER | NEGF_GREATER)) ? negf::FEAT_LESSER : negf::FEAT_RETARDED;
  if (cudaMemsetAsync(p->scratch, 0, negf::RGF_SCRATCH_HEADER, s) != cudaSuccess) return NEGF_ERR_CUDA;
  const int grid = p->n_slots < p->n_items ? p->n_slots : p->n_items;
  if (!mixed) return negf::rgf_launch_fp64(feat, *p, smem, grid, s);
  return negf::rgf_launch_mx(*p, smem, grid, s);  // one mixed instantiation with every feature
}

int negf_sm_count(void) {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  return n;
}

const char* negf_version(void) { return "negf_b200 0.1.0 (sm_100a)"; }

size_t negf_abi_struct_size(int which) {
  switch (which) {
    case 0: return sizeof(NegfBlock);
    case 1: return sizeof(NegfDevice);
    case 2: return sizeof(NegfItem);
    case 3: return sizeof(NegfRgfProblem);
    case 4: return sizeof(NegfLead);
    case 5: return sizeof(NegfLsItem);
    case 6: return sizeof(NegfLsProblem);
    case 7: return sizeof(NegfGammaSum);
    case 8: return sizeof(NegfLeadAdjItem);
    case 9: return sizeof(NegfLeadAdjProblem);
    default: return 0;
  }
}

}  // extern "C"
