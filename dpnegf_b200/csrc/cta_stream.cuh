// CTA-wide elementwise passes streamed through shared memory.
//
// Plain per-thread global loads leave too few bytes in flight per SM (the
// form passes of the first kernel version were load-latency bound at
// ~25 GB/s per SM).  Here every thread stages its elements of 2048-element
// chunks with cp.async, two chunks in flight (128 KB per SM), and consumes
// exactly the elements it staged, so no barrier is needed inside the loop.
#pragma once
#include "negf_common.cuh"

namespace negf {

constexpr int STREAM_CHUNK = 2048;
constexpr int STREAM_SMEM_BYTES = 4 * STREAM_CHUNK * (int)sizeof(cplx);

// out[e] = alpha * (X[e] - z * Y[e]) for e < count; a null X or Y is zero.
// Ends with __syncthreads().
NEGF_DEV void cta_shift_form(cplx* out, const cplx* X, const cplx* Y, cplx z, cplx alpha, int count,
                             cplx* smem) {
  const int tid = threadIdx.x;
  cplx* sx[2] = {smem, smem + STREAM_CHUNK};
  cplx* sy[2] = {smem + 2 * STREAM_CHUNK, smem + 3 * STREAM_CHUNK};
  const int nch = (count + STREAM_CHUNK - 1) / STREAM_CHUNK;
  auto issue = [&](int c) {
    const int base = c * STREAM_CHUNK;
#pragma unroll
    for (int s = 0; s < STREAM_CHUNK / 256; ++s) {
      const int k = tid + s * 256, e = base + k;
      const bool v = e < count;
      if (X) cp_async16(sx[c & 1] + k, v ? X + e : X, v);
      if (Y) cp_async16(sy[c & 1] + k, v ? Y + e : Y, v);
    }
    cp_async_commit();
  };
  if (nch > 0) issue(0);
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) issue(c + 1);
    else cp_async_commit();
    cp_async_wait<1>();
    const int base = c * STREAM_CHUNK;
#pragma unroll
    for (int s = 0; s < STREAM_CHUNK / 256; ++s) {
      const int k = tid + s * 256, e = base + k;
      if (e < count) {
        cplx x = X ? sx[c & 1][k] : cmk(0.0, 0.0);
        cplx y = Y ? sy[c & 1][k] : cmk(0.0, 0.0);
        out[e] = cmul(alpha, csub(x, cmul(z, y)));
      }
    }
  }
  cp_async_wait<0>();
  __syncthreads();
}

}  // namespace negf
