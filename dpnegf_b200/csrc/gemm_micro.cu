// gemm_micro: check and time the CTA-level complex GEMMs of the sweep.
//
//   gemm_micro [n] [reps]
//
// Correctness: every GEMM against a CPU complex128 product for every operand
// transform pair on ragged and multi-tile sizes (the DMMA GEMM to 1e-12
// relative, the 3xTF32 tensor-core GEMM to 2e-6 relative of sum |a||b|, the
// int8 slice GEMM with 8 / 6 digit planes to 1e-13 / 1e-10 of sum |a||b|).
// Timing: every SM runs one CTA that multiplies its own n x n complex
// operands `reps` times (operands larger than L2 in total), CUDA events.
// Exit code 0 only when every check passed.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "cta_gemm_oz.cuh"

using namespace negf;
typedef std::complex<double> zc;

// KIND: 0 DMMA FP64, 1 tcgen05 3xTF32, 6 / 8 tcgen05 int8 slices (S = 6 / 8)
template <int KIND>
struct Kind {
  static constexpr bool TC = KIND != 0;
  static constexpr int SMEM = KIND == 0 ? GEMM_SMEM_BYTES
                            : KIND == 1 ? TC_SMEM_BYTES
                                        : OzLayout<(KIND >= 2 ? KIND : 2)>::SMEM;
  static constexpr double TOL = KIND == 0 ? 1e-12 : KIND == 1 ? 2e-6 : KIND == 8 ? 1e-13 : 1e-10;
  static const char* name() {
    return KIND == 0 ? "dmma" : KIND == 1 ? "tf32x3" : KIND == 8 ? "int8x8" : KIND == 6 ? "int8x6"
         : KIND == 4 ? "int8x4" : "int8x2";
  }
};

template <int OPA, int OPB, int KIND>
__global__ void __launch_bounds__(CTA_THREADS, 1) k_gemm(GemmArgs g, int reps, int64_t stride) {
  extern __shared__ __align__(1024) char smem[];
  constexpr bool TC = Kind<KIND>::TC;
  if (TC) tc_tmem_alloc();
  GemmArgs h = g;
  h.A += blockIdx.x * stride;
  h.B += blockIdx.x * stride;
  h.C += blockIdx.x * stride;
  if (h.use_d) h.D = h.C;
  for (int r = 0; r < reps; ++r) {
    if constexpr (KIND == 1) cta_gemm_tc<OPA, OPB>(h, smem);
    else if constexpr (KIND >= 2) cta_gemm_oz<KIND, OPA, OPB>(h, smem);
    else cta_gemm<OPA, OPB>(h, reinterpret_cast<cplx*>(smem));
  }
  if (TC) {
    if (threadIdx.x == 0 && tc_err) printf("gemm_micro: tensor-core wait expired in block %d\n", blockIdx.x);
    tc_tmem_free();
  }
}

static zc op_a(int op, const std::vector<zc>& A, int lda, int m, int k) {
  if (op == OP_C) return std::conj(A[(size_t)k * lda + m]);
  if (op == OP_K) return std::conj(A[(size_t)m * lda + k]);
  return A[(size_t)m * lda + k];
}
static zc op_b(int op, const std::vector<zc>& B, int ldb, int k, int n) {
  if (op == OP_C) return std::conj(B[(size_t)n * ldb + k]);
  if (op == OP_K) return std::conj(B[(size_t)k * ldb + n]);
  return B[(size_t)k * ldb + n];
}

static GemmArgs host_args(int M, int N, int K, const cplx* A, int64_t lda, const cplx* B, int64_t ldb, cplx* C,
                          int64_t ldc) {
  GemmArgs g;
  g.M = M; g.N = N; g.K = K;
  g.A = A; g.lda = lda; g.B = B; g.ldb = ldb; g.C = C; g.ldc = ldc;
  g.D = nullptr; g.ldd = 0;
  g.alpha = make_double2(1.0, 0.0); g.beta = make_double2(0.0, 0.0); g.use_d = false;
  return g;
}

#define CK(x)                                                                          \
  do {                                                                                 \
    cudaError_t e_ = (x);                                                              \
    if (e_ != cudaSuccess) {                                                           \
      fprintf(stderr, "gemm_micro: %s: %s\n", #x, cudaGetErrorString(e_));            \
      exit(2);                                                                         \
    }                                                                                  \
  } while (0)

template <int OPA, int OPB, int KIND>
static bool check(int M, int N, int K, bool use_d, zc alpha, zc beta) {
  const int lda = OPA == OP_C ? M + 3 : K + 1, ldb = OPB == OP_C ? K + 2 : N + 5, ldc = N + 1;
  const size_t na = (size_t)lda * (OPA == OP_C ? K : M), nb = (size_t)ldb * (OPB == OP_C ? N : K);
  const size_t nc = (size_t)ldc * M;
  std::vector<zc> A(na), B(nb), C(nc), R(nc), H(nc);
  srand(M * 131 + N * 7 + K);
  auto rnd = []() { return (double)rand() / RAND_MAX - 0.5; };
  for (auto& x : A) x = zc(rnd(), rnd());
  for (auto& x : B) x = zc(rnd(), rnd());
  for (auto& x : C) x = zc(rnd(), rnd());
  double scale = 0.0;
  for (int m = 0; m < M; ++m)
    for (int n = 0; n < N; ++n) {
      zc s = 0.0;
      double sa = 0.0;
      for (int k = 0; k < K; ++k) {
        zc p = op_a(OPA, A, lda, m, k) * op_b(OPB, B, ldb, k, n);
        s += p;
        sa += std::abs(p);
      }
      R[(size_t)m * ldc + n] = alpha * s + (use_d ? beta * C[(size_t)m * ldc + n] : zc(0.0));
      scale = std::max(scale, sa * std::abs(alpha));
    }
  cplx *dA, *dB, *dC;
  CK(cudaMalloc(&dA, na * 16));
  CK(cudaMalloc(&dB, nb * 16));
  CK(cudaMalloc(&dC, nc * 16));
  CK(cudaMemcpy(dA, A.data(), na * 16, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dB, B.data(), nb * 16, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dC, C.data(), nc * 16, cudaMemcpyHostToDevice));
  GemmArgs g = host_args(M, N, K, dA, lda, dB, ldb, dC, ldc);
  g.alpha = make_double2(alpha.real(), alpha.imag());
  g.beta = make_double2(beta.real(), beta.imag());
  g.use_d = use_d;
  g.D = dC;
  g.ldd = ldc;
  const int smem = Kind<KIND>::SMEM;
  CK(cudaFuncSetAttribute(k_gemm<OPA, OPB, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k_gemm<OPA, OPB, KIND><<<1, CTA_THREADS, smem>>>(g, 1, 0);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(H.data(), dC, nc * 16, cudaMemcpyDeviceToHost));
  double err = 0.0;
  int untouched = 0;
  for (int m = 0; m < M; ++m)
    for (int n = 0; n < ldc; ++n) {
      const size_t i = (size_t)m * ldc + n;
      if (n < N) err = std::max(err, std::abs(H[i] - R[i]));
      else if (H[i] != C[i]) ++untouched;  // the padding column must stay untouched
    }
  const double rel = err / scale, tol = Kind<KIND>::TOL;
  const bool ok = rel < tol && untouched == 0;
  printf("%-8s op(%d,%d) M=%d N=%d K=%d d=%d: rel err %.2e %s\n", Kind<KIND>::name(), OPA, OPB, M, N, K,
         (int)use_d, rel, ok ? "ok" : "FAIL");
  CK(cudaFree(dA));
  CK(cudaFree(dB));
  CK(cudaFree(dC));
  return ok;
}

template <int KIND>
static void timeit(int n, int reps, int sms) {
  const size_t per = (size_t)n * n;
  cplx *dA, *dB, *dC;
  CK(cudaMalloc(&dA, per * sms * 16));
  CK(cudaMalloc(&dB, per * sms * 16));
  CK(cudaMalloc(&dC, per * sms * 16));
  CK(cudaMemset(dA, 0, per * sms * 16));
  CK(cudaMemset(dB, 0, per * sms * 16));
  GemmArgs g = host_args(n, n, n, dA, n, dB, n, dC, n);
  const int smem = Kind<KIND>::SMEM;
  CK(cudaFuncSetAttribute(k_gemm<OP_N, OP_N, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k_gemm<OP_N, OP_N, KIND><<<sms, CTA_THREADS, smem>>>(g, 2, (int64_t)per);
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  CK(cudaEventRecord(a));
  k_gemm<OP_N, OP_N, KIND><<<sms, CTA_THREADS, smem>>>(g, reps, (int64_t)per);
  CK(cudaEventRecord(b));
  CK(cudaDeviceSynchronize());
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, a, b));
  const double flop = 8.0 * n * (double)n * n * reps * sms;
  printf("%-8s n=%d reps=%d CTAs=%d: %.1f us per GEMM per CTA, %.2f TFLOP/s (8 n^3 complex count)\n",
         Kind<KIND>::name(), n, reps, sms, ms * 1e3 / reps, flop / (ms * 1e-3) / 1e12);
  CK(cudaFree(dA));
  CK(cudaFree(dB));
  CK(cudaFree(dC));
}

int main(int argc, char** argv) {
  const int n = argc > 1 ? atoi(argv[1]) : 256;
  const int reps = argc > 2 ? atoi(argv[2]) : 20;
  if (n <= 0 || n > 1024 || reps <= 0) {
    fprintf(stderr, "usage: gemm_micro [n <= 1024] [reps]\n");
    return 2;
  }
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  bool ok = true;
  const bool only_oz = argc > 3 && atoi(argv[3]) != 0;  // third argument 1: int8 slice GEMM only
  if (!only_oz) {
    ok &= check<OP_N, OP_N, 0>(100, 72, 37, true, zc(-1, 0), zc(1, 0));
    ok &= check<OP_N, OP_C, 0>(130, 96, 200, false, zc(1, 0), zc(0, 0));
    ok &= check<OP_N, OP_N, 1>(256, 256, 256, false, zc(1, 0), zc(0, 0));
    ok &= check<OP_N, OP_N, 1>(100, 72, 37, true, zc(-1, 0), zc(1, 0));
    ok &= check<OP_N, OP_N, 1>(8, 8, 8, false, zc(0.5, 0.25), zc(0, 0));
    ok &= check<OP_N, OP_N, 1>(300, 520, 64, true, zc(1, 0), zc(0.5, -1));
    ok &= check<OP_N, OP_C, 1>(130, 96, 200, false, zc(1, 0), zc(0, 0));
    ok &= check<OP_C, OP_N, 1>(96, 130, 77, true, zc(1, 0), zc(1, 0));
    ok &= check<OP_C, OP_C, 1>(64, 48, 33, false, zc(1, 0), zc(0, 0));
    ok &= check<OP_K, OP_N, 1>(50, 60, 70, false, zc(1, 0), zc(0, 0));
    ok &= check<OP_N, OP_K, 1>(50, 60, 70, false, zc(1, 0), zc(0, 0));
  }
  ok &= check<OP_N, OP_N, 8>(8, 8, 8, false, zc(1, 0), zc(0, 0));
  ok &= check<OP_N, OP_N, 8>(256, 256, 256, false, zc(1, 0), zc(0, 0));
  ok &= check<OP_N, OP_N, 8>(100, 72, 37, true, zc(-1, 0), zc(1, 0));
  ok &= check<OP_N, OP_N, 8>(300, 500, 64, true, zc(1, 0), zc(0.5, -1));
  ok &= check<OP_N, OP_N, 8>(512, 512, 512, false, zc(1, 0), zc(0, 0));
  ok &= check<OP_N, OP_C, 8>(130, 96, 200, false, zc(1, 0), zc(0, 0));
  ok &= check<OP_C, OP_N, 8>(96, 130, 77, true, zc(1, 0), zc(1, 0));
  ok &= check<OP_C, OP_C, 8>(64, 48, 33, false, zc(1, 0), zc(0, 0));
  ok &= check<OP_K, OP_N, 8>(50, 60, 70, false, zc(1, 0), zc(0, 0));
  ok &= check<OP_N, OP_K, 8>(50, 60, 70, false, zc(1, 0), zc(0, 0));
  ok &= check<OP_K, OP_K, 8>(40, 33, 90, false, zc(1, 0), zc(0, 0));
  ok &= check<OP_N, OP_N, 6>(256, 256, 256, false, zc(1, 0), zc(0, 0));
  ok &= check<OP_C, OP_K, 6>(100, 72, 37, true, zc(-1, 0), zc(1, 0));
  if (!ok) {
    printf("gemm_micro: correctness FAILED\n");
    return 1;
  }
  if (!only_oz) {
    timeit<0>(n, reps, sms);
    timeit<1>(n, reps, sms);
  }
  timeit<8>(n, reps, sms);
  timeit<6>(n, reps, sms);
  if (only_oz) {  // fewer digit planes: how the time splits between fixed and per-plane work
    timeit<4>(n, reps, sms);
    timeit<2>(n, reps, sms);
  }
  return 0;
}
