// CTA-wide complex GEMM on the fifth-generation tensor cores (tcgen05.mma,
// kind::tf32) with 3xTF32 split products and FP32 accumulation in tensor
// memory: the bulk product of the mixed-precision sweep.
//
//   acc = op(A) * op(B),   epi(m, n, acc) for every in-range element
//
// Same operands (complex128 in global memory), operand transforms, GemmArgs
// and epilogue functors as the FP64 tile GEMM (cta_gemm.cuh), so a sweep
// switches between the two with a template flag.
//
// Split products.  Every real operand x is split into two TF32 numbers,
// hi = tf32(x) and lo = tf32(x - hi); a real product is formed as
// A_hi B_hi + A_hi B_lo + A_lo B_hi (the lo*lo term is below FP32 rounding),
// which gives products accurate to FP32 level at TF32 tensor throughput.
// A complex product takes four real planes per operand (re/im x hi/lo):
//   C_re += Ar Br - Ai Bi,   C_im += Ar Bi + Ai Br
// i.e. 12 MMAs of 128 x N x 8 per k = 8 step; the minus sign is the B-negate
// bit of the instruction descriptor.
//
// Tiles.  One CTA (8 warps) walks 128 x 256 output tiles.  C_re and C_im of
// a tile are two FP32 accumulators of 256 columns each in tensor memory (the
// CTA holds all 512 columns, allocated once per kernel by tc_tmem_alloc).
// k advances in slabs of 8 complex entries.  Raw FP64 slabs of op(A) and
// op(B) are copied into shared memory with cp.async two slabs ahead; the CTA
// splits the current slab into eight K-major TF32 planes in the canonical
// no-swizzle layout (core matrices of 8 rows x 16 bytes; planes are
// [k/4][row][4], so the leading-byte offset is the plane's row count x 16 B
// and the stride-byte offset 128 B), and thread 0 issues the slab's 12 MMAs
// and commits them to that plane stage's mbarrier.  A plane stage is
// rewritten only after its mbarrier reports the MMAs that read it complete.
// Every mbarrier wait is bounded; on expiry the CTA records tc_err and skips
// the remaining tensor-core work (the caller turns tc_err into an item status).
//
// Epilogue.  Each warp reads its 32-lane quarter of the accumulators with
// tcgen05.ld (32 rows x 16 columns at a time), transposes the block through
// shared memory and calls epi with consecutive columns on consecutive lanes,
// so row-major outputs are written in 256-byte runs.
#pragma once
#include "cta_gemm.cuh"

namespace negf {

constexpr int TC_M = 128, TC_N = 256, TC_KC = 8;
constexpr int TC_PLANE_A = TC_M * TC_KC * 4;                   // bytes of one A plane
constexpr int TC_PLANE_B = TC_N * TC_KC * 4;                   // bytes of one B plane
constexpr int TC_LBO_A = TC_M * 16, TC_LBO_B = TC_N * 16;      // k/4 group pitch
constexpr int TC_STAGE_BYTES = 4 * TC_PLANE_A + 4 * TC_PLANE_B;  // also the raw FP64 slab pair
constexpr int TC_SMEM_BYTES = 4 * TC_STAGE_BYTES;
constexpr int TC_TMEM_COLS = 512;
constexpr int TC_EPI_PITCH = 17;                               // complex entries per transposed row
constexpr long long TC_WAIT_CYCLES = 4000000000LL;             // about two seconds
static_assert(CTA_THREADS == 256, "the tensor-core GEMM assumes 256-thread CTAs");
static_assert(8 * 32 * TC_EPI_PITCH * 16 <= 2 * TC_STAGE_BYTES, "epilogue transpose buffers fit in the planes area");
static_assert(TC_M * TC_KC * 16 + TC_N * TC_KC * 16 == TC_STAGE_BYTES, "a raw slab pair fills one stage");

static __shared__ uint32_t tc_tmem;                            // tensor-memory base address of this CTA
static __shared__ __align__(8) unsigned long long tc_bar[2];   // per-stage MMA completion
static __shared__ int tc_err;                                  // a bounded wait expired

NEGF_DEV uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Whole CTA; warp 0 owns the allocation.  Call once per kernel before the
// first tensor-core GEMM, and tc_tmem_free before the kernel returns.
NEGF_DEV void tc_tmem_alloc() {
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(&tc_tmem)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (threadIdx.x == 0) tc_err = 0;
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
}

NEGF_DEV void tc_tmem_free() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tc_tmem), "r"(TC_TMEM_COLS));
  }
}

NEGF_DEV bool tc_bar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the given phase parity; false when the limit expired.
NEGF_DEV bool tc_bar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!tc_bar_try(bar, parity))
    if (clock64() - t0 > TC_WAIT_CYCLES) return false;
  return true;
}

NEGF_DEV uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

// x ~ hi + lo with hi, lo TF32 (bit patterns in 32-bit containers)
NEGF_DEV void tf32_split(double x, uint32_t& hi, uint32_t& lo) {
  const float f = static_cast<float>(x);
  hi = tf32_rna(f);
  lo = tf32_rna(f - __uint_as_float(hi));  // exact in FP32: hi is f with its low mantissa bits rounded off
}

// Shared-memory matrix descriptor, K-major, no swizzle (sm_100 version 1).
NEGF_DEV uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

NEGF_DEV void tc_mma(uint32_t d_tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

NEGF_DEV void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}

// 16 consecutive FP32 accumulator columns of this warp's 32 lanes.
NEGF_DEV void tc_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// Store the split of 4 consecutive-k complex entries of one row into the
// four planes (re hi, re lo, im hi, im lo) at byte offset `off`.
NEGF_DEV void tc_put4(char* st, int plane_bytes, int off, const cplx* v, bool conj) {
  uint4 rh, rl, ih, il;
  tf32_split(v[0].x, rh.x, rl.x); tf32_split(conj ? -v[0].y : v[0].y, ih.x, il.x);
  tf32_split(v[1].x, rh.y, rl.y); tf32_split(conj ? -v[1].y : v[1].y, ih.y, il.y);
  tf32_split(v[2].x, rh.z, rl.z); tf32_split(conj ? -v[2].y : v[2].y, ih.z, il.z);
  tf32_split(v[3].x, rh.w, rl.w); tf32_split(conj ? -v[3].y : v[3].y, ih.w, il.w);
  *reinterpret_cast<uint4*>(st + off) = rh;
  *reinterpret_cast<uint4*>(st + plane_bytes + off) = rl;
  *reinterpret_cast<uint4*>(st + 2 * plane_bytes + off) = ih;
  *reinterpret_cast<uint4*>(st + 3 * plane_bytes + off) = il;
}

// Raw slab staging (cp.async, zero fill outside the matrix).  The raw copy
// keeps the orientation of the operand in global memory (its contiguous
// dimension innermost), so the copies are coalesced.
//   op(A) N/K: raw [128 m][8 k]      op(A) C: raw [8 k][128 m]
//   op(B) N/K: raw [8 k][256 n]      op(B) C: raw [256 n][8 k]
template <int OPA>
NEGF_DEV void tc_fetch_a(cplx* raw, const GemmArgs& g, int m0, int k0, int tid) {
#pragma unroll
  for (int i = 0; i < (TC_M * TC_KC) / CTA_THREADS; ++i) {
    const int e = tid + CTA_THREADS * i;
    if (OPA == OP_C) {
      const int k = e >> 7, m = e & 127, kg = k0 + k, mg = m0 + m;
      const bool v = kg < g.K && mg < g.M;
      cp_async16(raw + e, v ? g.A + (int64_t)kg * g.lda + mg : g.A, v);
    } else {
      const int m = e >> 3, k = e & 7, kg = k0 + k, mg = m0 + m;
      const bool v = kg < g.K && mg < g.M;
      cp_async16(raw + e, v ? g.A + (int64_t)mg * g.lda + kg : g.A, v);
    }
  }
}

template <int OPB>
NEGF_DEV void tc_fetch_b(cplx* raw, const GemmArgs& g, int k0, int n0, int tn, int tid) {
#pragma unroll
  for (int i = 0; i < (TC_N * TC_KC) / CTA_THREADS; ++i) {
    const int e = tid + CTA_THREADS * i;
    if (OPB == OP_C) {
      const int n = e >> 3, k = e & 7, kg = k0 + k, ng = n0 + n;
      const bool v = kg < g.K && ng < g.N;
      if (n < tn) cp_async16(raw + e, v ? g.B + (int64_t)ng * g.ldb + kg : g.B, v);
    } else {
      const int k = e >> 8, n = e & 255, kg = k0 + k, ng = n0 + n;
      const bool v = kg < g.K && ng < g.N;
      if (n < tn) cp_async16(raw + e, v ? g.B + (int64_t)kg * g.ldb + ng : g.B, v);
    }
  }
}

// Split the raw slabs of one stage into the eight TF32 planes.
template <int OPA, int OPB>
NEGF_DEV void tc_split(char* pl, const cplx* rawA, const cplx* rawB, int tn, int tid) {
  cplx v[4];
  {  // A: one (row, k group) per thread
    const int m = OPA == OP_C ? (tid & 127) : (tid >> 1), kg = OPA == OP_C ? (tid >> 7) : (tid & 1);
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = OPA == OP_C ? rawA[(4 * kg + j) * TC_M + m] : rawA[m * TC_KC + 4 * kg + j];
    tc_put4(pl, TC_PLANE_A, kg * TC_LBO_A + m * 16, v, OPA != OP_N);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {  // B: two (row, k group) per thread
    const int p = tid + CTA_THREADS * i;
    const int n = OPB == OP_C ? (p >> 1) : (p & 255), kg = OPB == OP_C ? (p & 1) : (p >> 8);
    if (n < tn) {
#pragma unroll
      for (int j = 0; j < 4; ++j) v[j] = OPB == OP_C ? rawB[n * TC_KC + 4 * kg + j] : rawB[(4 * kg + j) * TC_N + n];
      tc_put4(pl + 4 * TC_PLANE_A, TC_PLANE_B, kg * TC_LBO_B + n * 16, v, OPB != OP_N);
    }
  }
}

// The 12 MMAs of one k = 8 slab (thread 0).  first: the slab starts the tile.
NEGF_DEV void tc_issue_slab(const char* pl, uint32_t tmem, uint32_t idesc, bool first) {
  const uint32_t a0 = smem_addr(pl), b0 = smem_addr(pl + 4 * TC_PLANE_A);
  const uint32_t idn = idesc | (1u << 14);  // negate B
  const uint32_t c_re = tmem, c_im = tmem + 256;
  auto A = [&](int plane) { return tc_desc(a0 + plane * TC_PLANE_A, TC_LBO_A, 128); };
  auto B = [&](int plane) { return tc_desc(b0 + plane * TC_PLANE_B, TC_LBO_B, 128); };
  const uint32_t acc = first ? 0u : 1u;
  // planes: 0 re hi, 1 re lo, 2 im hi, 3 im lo
  tc_mma(c_re, A(0), B(0), idesc, acc);
  tc_mma(c_re, A(0), B(1), idesc, 1u);
  tc_mma(c_re, A(1), B(0), idesc, 1u);
  tc_mma(c_re, A(2), B(2), idn, 1u);
  tc_mma(c_re, A(2), B(3), idn, 1u);
  tc_mma(c_re, A(3), B(2), idn, 1u);
  tc_mma(c_im, A(0), B(2), idesc, acc);
  tc_mma(c_im, A(0), B(3), idesc, 1u);
  tc_mma(c_im, A(1), B(2), idesc, 1u);
  tc_mma(c_im, A(2), B(0), idesc, 1u);
  tc_mma(c_im, A(2), B(1), idesc, 1u);
  tc_mma(c_im, A(3), B(0), idesc, 1u);
}

// acc = op(A) op(B) over the whole M x N output; epi(m, n, acc) once per
// in-range element.  The output must not alias A or B.  Ends with
// __syncthreads().  Requires tc_tmem_alloc() earlier in the kernel.
//
// Shared memory: [planes 0][planes 1][raw 0][raw 1], 48 KB each.  The k
// slabs of all tiles form one sequence s = 0..S-1; slab s+2 is fetched
// while slab s is split and multiplied, across tile boundaries too.
template <int OPA, int OPB, class Epi>
__device__ __noinline__ void cta_gemm_tc_epi(const GemmArgs g, char* smem, const Epi epi) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nk = (g.K + TC_KC - 1) / TC_KC;
  const int tiles_n = (g.N + TC_N - 1) / TC_N, tiles = ((g.M + TC_M - 1) / TC_M) * tiles_n;
  if (nk == 0) {  // empty sum
    for (int e = tid; e < g.M * g.N; e += CTA_THREADS) epi(e / g.N, e % g.N, cmk(0.0, 0.0));
    __syncthreads();
    return;
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(&tc_bar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(&tc_bar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  __syncthreads();
  const uint32_t bar[2] = {smem_addr(&tc_bar[0]), smem_addr(&tc_bar[1])};
  uint32_t uses[2] = {0u, 0u}, seen[2] = {0u, 0u};  // commits issued / completions observed per stage
  const uint32_t tmem = tc_tmem;
  bool ok = tc_err == 0;
  const int S = tiles * nk;
  auto plane = [&](int b) { return smem + b * TC_STAGE_BYTES; };
  auto rawA = [&](int b) { return reinterpret_cast<cplx*>(smem + 2 * TC_STAGE_BYTES + b * TC_STAGE_BYTES); };
  auto rawB = [&](int b) { return rawA(b) + TC_M * TC_KC; };
  auto tile_of = [&](int t, int& m0, int& n0, int& tn) {
    m0 = (t / tiles_n) * TC_M;
    n0 = (t % tiles_n) * TC_N;
    tn = min(TC_N, (g.N - n0 + 15) & ~15);
  };
  auto fetch = [&](int s) {
    if (s < S) {
      int m0, n0, tn;
      tile_of(s / nk, m0, n0, tn);
      const int k0 = (s % nk) * TC_KC;
      tc_fetch_a<OPA>(rawA(s & 1), g, m0, k0, tid);
      tc_fetch_b<OPB>(rawB(s & 1), g, k0, n0, tn, tid);
    }
    cp_async_commit();
  };
  auto drain = [&](int b) {  // wait until every commit issued on stage b has completed
    if (seen[b] < uses[b]) {
      if (ok && !tc_bar_wait(bar[b], (uses[b] - 1u) & 1u)) ok = false;
      seen[b] = uses[b];
    }
  };

  fetch(0);
  fetch(1);
  for (int s = 0; s < S; ++s) {
    const int b = s & 1, kc = s % nk;
    int m0, n0, tn;
    tile_of(s / nk, m0, n0, tn);
    cp_async_wait<1>();
    __syncthreads();  // raw slab s is visible to every thread
    drain(b);         // the MMAs of slab s-2 no longer read planes b
    tc_split<OPA, OPB>(plane(b), rawA(b), rawB(b), tn, tid);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    ok = __syncthreads_and(ok) != 0;  // planes visible to the tensor core; raw b consumed; `ok` uniform
    fetch(s + 2);
    if (tid == 0 && ok) {
      const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(tn >> 3) << 17) |
                             ((uint32_t)(TC_M >> 4) << 24);
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      tc_issue_slab(plane(b), tmem, idesc, kc == 0);
      tc_commit(bar[b]);
    }
    ++uses[b];
    if (kc != nk - 1) continue;

    // ---- tile complete: epilogue.  Warp w reads lanes 32 (w % 4).. and
    // columns 128 (w / 4).. in blocks of 16, transposed through the planes area.
    drain(0);
    drain(1);
    ok = __syncthreads_and(ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    const int lq = warp & 3, ch = warp >> 2;
    cplx* tb = reinterpret_cast<cplx*>(smem) + warp * 32 * TC_EPI_PITCH;
    for (int c0 = ch * 128; c0 < ch * 128 + 128 && c0 < tn; c0 += 16) {
      float re[16], im[16];
      if (ok) {
        const uint32_t ta = tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)c0;
        tc_ld16(ta, re);
        tc_ld16(ta + 256, im);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) re[j] = im[j] = 0.0f;
      }
#pragma unroll
      for (int j = 0; j < 16; ++j) tb[lane * TC_EPI_PITCH + j] = cmk((double)re[j], (double)im[j]);
      __syncwarp();
      const int n = n0 + c0 + (lane & 15);
#pragma unroll 4
      for (int r = lane >> 4; r < 32; r += 2) {
        const int m = m0 + lq * 32 + r;
        if (m < g.M && n < g.N) epi(m, n, tb[r * TC_EPI_PITCH + (lane & 15)]);
      }
      __syncwarp();
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();  // accumulators and the planes area are free again
  }
  cp_async_wait<0>();
  if (tid == 0) {
    if (!ok) tc_err = 1;
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(bar[0]));
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(bar[1]));
  }
  __syncthreads();
}

// C = alpha op(A) op(B) + beta D on the tensor-core path (D may alias C).
template <int OPA, int OPB>
NEGF_DEV void cta_gemm_tc(const GemmArgs& g, char* smem) {
  cta_gemm_tc_epi<OPA, OPB>(g, smem, EpiStore{g});
}

}  // namespace negf
