// temf_solve_noalloc: the triangular solve for callers that cannot let a
// library allocate GPU memory.
//
// Some callers cannot call cudaMalloc (or let a library call it) at the point
// where they solve: an application that reserves all device memory for its own
// pool up front, a driver that must not call into the allocator while another
// thread is capturing CUDA work, or a time loop with a fixed memory budget.
// temf_solve allocates staging and scratch buffers on first use; this entry
// point does not.  Its scratch lives in one file-scope __device__ array of
// kNoAllocScratchBytes (32 MiB), which every GPU that loads the library holds
// until the process exits.  The caller passes the right-hand side and the
// solution in device memory.
#include <mutex>

#include "../../include/temf_b200.h"
#include "common.h"
#include "ctx.h"
#include "solve.h"

namespace temf {

const int* ctx_perm_device(temf_ctx* c);  // capi.cu

constexpr size_t kNoAllocScratchBytes = 32u << 20;

// Scratch of the allocation-free solve.  Host code must not use this symbol as
// an address: it is a host-side stand-in.  The device address comes from
// cudaGetSymbolAddress (scratch_base below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_lock;
void* g_base[64] = {nullptr};

// Device address of the scratch array on the current device; looked up once
// per device, with that device current.
unsigned char* scratch_base(int device) {
  if (device < 0 || device >= 64) throw ArgError("device index out of range for the allocation-free solve");
  std::lock_guard<std::mutex> g(g_lock);
  if (!g_base[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw CudaError(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_base[device] = p;
  }
  return static_cast<unsigned char*>(g_base[device]);
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

__global__ void k_na_set_ptr(double** dst, double* v) { *dst = v; }

__global__ void k_na_gather(int n, const int* __restrict__ perm, const double* __restrict__ b,
                            double* __restrict__ w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w[i] = b[perm[i]];
}

__global__ void k_na_scatter(int n, const int* __restrict__ perm, const double* __restrict__ w,
                             double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[perm[i]] = w[i];
}

}  // namespace
}  // namespace temf

using namespace temf;

extern "C" int temf_solve_noalloc(temf_ctx* c, int slot, const double* b_dev, double* x_dev) {
  if (!c) return TEMF_EARG;
  try {
    TEMF_CUDA(cudaSetDevice(c->device));
    c->err.clear();
    if (slot != 1 && slot != 2) throw ArgError("slot must be 1 or 2");
    if (!c->slots[slot - 1].valid) throw StateError("temf_solve_noalloc: the slot holds no valid factor");
    if (c->slots[slot - 1].indefinite)
      throw StateError("temf_solve_noalloc: the slot holds an indefinite factor (refined solves: use temf_solve)");
    if (!b_dev || !x_dev) throw ArgError("temf_solve_noalloc: NULL device pointer");
    const SolvePlan& P = c->splan;
    const int n = c->n_edges;
    // scratch layout: [factor pointer | error word] [work vector] [sync words] [partial sums]
    const size_t off_work = 256;
    const size_t off_sync = align256(off_work + (size_t)n * sizeof(double));
    const size_t off_part = align256(off_sync + (4 * (size_t)P.nsn + 4) * sizeof(int));
    const size_t need = off_part + (size_t)std::max<int64_t>(P.part_len, 1) * sizeof(double);
    if (need > kNoAllocScratchBytes)
      throw ArgError("temf_solve_noalloc: this factor needs " + std::to_string(need) +
                     " bytes of scratch; the allocation-free solve holds at most " +
                     std::to_string(kNoAllocScratchBytes) + " bytes (use temf_solve)");
    unsigned char* base = scratch_base(c->device);
    double** lbase = reinterpret_cast<double**>(base);
    int* err = reinterpret_cast<int*>(base + 64);
    double* work = reinterpret_cast<double*>(base + off_work);
    int* sync = reinterpret_cast<int*>(base + off_sync);
    double* part = reinterpret_cast<double*>(base + off_part);
    cudaStream_t st = c->stream;
    TEMF_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    k_na_set_ptr<<<1, 1, 0, st>>>(lbase, c->slots[slot - 1].L.p);
    k_na_gather<<<ceil_div(n, 256), 256, 0, st>>>(n, ctx_perm_device(c), b_dev, work);
    TEMF_CHECK_LAUNCH();
    launch_solve_scratch(*c, lbase, work, sync, part, err, st);
    k_na_scatter<<<ceil_div(n, 256), 256, 0, st>>>(n, ctx_perm_device(c), work, x_dev);
    TEMF_CHECK_LAUNCH();
    int flag = 0;
    TEMF_CUDA(cudaMemcpyAsync(&flag, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    TEMF_CUDA(cudaStreamSynchronize(st));
    if (flag) throw StateError("temf_solve_noalloc: a triangular-solve wait timed out (code " + std::to_string(flag) + ")");
    return TEMF_OK;
  } catch (const ArgError& e) {
    c->err = e.what();
    return TEMF_EARG;
  } catch (const StateError& e) {
    c->err = e.what();
    return TEMF_ESTATE;
  } catch (const CudaError& e) {
    c->err = e.what();
    return TEMF_ECUDA;
  } catch (const std::exception& e) {
    c->err = e.what();
    return TEMF_EINTERNAL;
  }
}
