// Shared device primitives for the NEGF kernels (sm_100a).
//
// Complex numbers are complex128 stored interleaved (re, im) as double2, the
// same layout torch.complex128 uses, so host tensors are passed through
// without conversion.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define NEGF_DEV __device__ __forceinline__

namespace negf {

typedef double2 cplx;

NEGF_DEV cplx cmk(double r, double i) { return make_double2(r, i); }
NEGF_DEV cplx cadd(cplx a, cplx b) { return cmk(a.x + b.x, a.y + b.y); }
NEGF_DEV cplx csub(cplx a, cplx b) { return cmk(a.x - b.x, a.y - b.y); }
NEGF_DEV cplx cmul(cplx a, cplx b) { return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
NEGF_DEV cplx cconj(cplx a) { return cmk(a.x, -a.y); }
NEGF_DEV cplx cneg(cplx a) { return cmk(-a.x, -a.y); }
NEGF_DEV cplx cscale(cplx a, double s) { return cmk(a.x * s, a.y * s); }
// a*b + c
NEGF_DEV cplx cfma(cplx a, cplx b, cplx c) {
  return cmk(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
// Reciprocal by Smith's scaling (avoids overflow in |a|^2).
NEGF_DEV cplx crcp(cplx a) {
  if (fabs(a.x) >= fabs(a.y)) {
    double r = a.y / a.x, den = a.x + a.y * r;
    return cmk(1.0 / den, -r / den);
  } else {
    double r = a.x / a.y, den = a.x * r + a.y;
    return cmk(r / den, -1.0 / den);
  }
}
NEGF_DEV double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }
NEGF_DEV bool cfinite(cplx a) { return isfinite(a.x) && isfinite(a.y); }

// ---------------------------------------------------------------------------
// cp.async (16-byte, L2-only) with zero fill when the source is out of range.
NEGF_DEV void cp_async16(void* smem_dst, const void* gmem_src, bool valid) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem_src), "r"(n));
}
// Global load that the compiler may not sink below later volatile asm (the
// DMMAs): used to put a read-modify-write's reads in flight before the math.
NEGF_DEV cplx ldg_early(const cplx* p) {
  cplx v;
  asm volatile("ld.global.cg.v2.f64 {%0,%1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
NEGF_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
NEGF_DEV void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ---------------------------------------------------------------------------
// FP64 tensor-core MMA, D(8x8) += A(8x4, row) * B(4x8, col).
// Fragment ownership for lane l: A[l/4][l%4], B[l%4][l/4],
// C[l/4][2*(l%4) + {0,1}].
NEGF_DEV void dmma884(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// FP64 tensor-core MMA, D(16x8) += A(16x8, row) * B(8x8, col).
// Fragment ownership for lane l (g = l/4, t = l%4):
//   A: a0 (g, t), a1 (g+8, t), a2 (g, t+4), a3 (g+8, t+4)
//   B: b0 (t, g), b1 (t+4, g)
//   C: c0 (g, 2t), c1 (g, 2t+1), c2 (g+8, 2t), c3 (g+8, 2t+1)
NEGF_DEV void dmma1688(double* c, const double* a, const double* b) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
               : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
               : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Operand transforms for the tile GEMM.
enum Op : int { OP_N = 0, OP_C = 1 /* conjugate transpose */, OP_K = 2 /* conjugate */ };

// Per-CTA phase clocks (thread 0): the cycles since the previous mark are
// charged to the phase that just ended.  Every mark follows a __syncthreads.
enum Phase {
  PH_FORM = 0, PH_GEMM_FWD, PH_INV_STAGE, PH_INV_PANEL, PH_INV_UPDATE, PH_INV_GATHER,
  PH_GEMM_BWD, PH_LESSER, PH_DOS, PH_TRANS, PH_OTHER, PH_REFINE, NPH
};
struct PhaseClock {
  unsigned long long c[NPH];
  long long t0;
  bool on;
  NEGF_DEV void start(bool enable) {
    on = enable && threadIdx.x == 0;
    for (int i = 0; i < NPH; ++i) c[i] = 0;
    t0 = on ? clock64() : 0;
  }
  NEGF_DEV void mark(int ph) {
    if (on) {
      long long t = clock64();
      c[ph] += (unsigned long long)(t - t0);
      t0 = t;
    }
  }
};

}  // namespace negf
