// RGF sweep whose scratch lives in a fixed, library-owned device array.
//
// negf_rgf_run needs the caller to supply scratch memory sized by
// negf_rgf_scratch_bytes.  Some callers cannot allocate device memory at the
// point where they want to run the sweep: a host NEGF code that embeds this
// library inside its own solver loop usually owns the GPU through its own
// memory pool (a C or Fortran transport code, or a plugin host that only
// hands over input and output buffers), and cudaMalloc both synchronises the
// whole device and can fail once that pool has taken the memory.  For them,
// negf_rgf_run_static takes its scratch from the file-scope array below
// instead.  The caller still passes every input and output buffer; this entry
// point calls no cudaMalloc, cudaFree or other allocating routine.
//
// Limits and sharing:
//   * the array is NEGF_RGF_STATIC_SCRATCH_BYTES (64 MiB) on every GPU that
//     loads the library, held until the process exits;
//   * problems whose scratch for even one work slot exceeds it are rejected
//     with NEGF_ERR_SCRATCH_LIMIT; otherwise the slot count is reduced to what
//     fits (fewer concurrent energies, same results);
//   * all calls on a device share the one array and it keeps the previous
//     call's contents: the work-queue counter is cleared at the start of every
//     call (the only state that must start at zero), and calls that overlap
//     on the GPU (different streams, or different host threads without
//     ordering) race on it;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current), so
//     make that first call before any stream capture begins;
//   * that address is kept for the life of the process: after a
//     cudaDeviceReset the module is loaded again and the array may move, so
//     no call may follow a device reset;
//   * negf_rgf_static_slots reports how many work slots a call will run, so a
//     caller can see when the slot count was lowered to fit.
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/negf_b200.h"

namespace {

constexpr size_t kStaticScratchBytes = (size_t)64 << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_rgf_static_scratch[kStaticScratchBytes];

void* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of g_rgf_static_scratch on the current device (looked up once).
int static_scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return NEGF_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return NEGF_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_rgf_static_scratch) != cudaSuccess || p == nullptr) return NEGF_ERR_CUDA;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return NEGF_OK;
}

}  // namespace

extern "C" {

size_t negf_rgf_static_scratch_bytes(void) { return kStaticScratchBytes; }

int negf_rgf_static_slots(const NegfRgfProblem* p) {
  if (!p || p->n_slots <= 0 || p->max_n <= 0) return NEGF_ERR_ARGUMENT;
  if (p->max_n > NEGF_MAX_BLOCK) return NEGF_ERR_UNSUPPORTED;
  NegfRgfProblem q = *p;
  q.n_slots = 1;
  const size_t one = negf_rgf_scratch_bytes(&q);
  if (one == 0) return NEGF_ERR_ARGUMENT;
  if (one > kStaticScratchBytes) return NEGF_ERR_SCRATCH_LIMIT;
  q.n_slots = 2;
  const size_t per_slot = negf_rgf_scratch_bytes(&q) - one;
  size_t fit = per_slot ? 1 + (kStaticScratchBytes - one) / per_slot : (size_t)p->n_slots;
  return (int)(fit < (size_t)p->n_slots ? fit : (size_t)p->n_slots);
}

int negf_rgf_run_static(const NegfRgfProblem* p, void* stream) {
  if (!p) return NEGF_ERR_ARGUMENT;
  if (p->n_items <= 0) return NEGF_OK;
  const int slots = negf_rgf_static_slots(p);
  if (slots <= 0) return slots;
  NegfRgfProblem q = *p;
  q.n_slots = slots;
  void* addr = nullptr;
  const int st = static_scratch_address(&addr);
  if (st != NEGF_OK) return st;
  q.scratch = addr;
  q.scratch_bytes = kStaticScratchBytes;
  return negf_rgf_run(&q, stream);
}

}  // extern "C"
