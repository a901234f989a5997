// Allocation-free variant of the lu_gpu_par.h triangular solve.
//
// trisolve_par_kernel needs n ints and 2n doubles of scratch (the inverse row
// permutation, P b and the intermediate y), which the regular entry point
// takes from the caller.  Some callers cannot provide or allocate device
// memory at solve time: a circuit simulator's time-step loop that sizes all
// device memory when the netlist is loaded and must not call cudaMalloc in
// the middle of a run (the call synchronizes the whole device, stalling the
// other streams, and an out-of-memory failure there loses the run), or host
// code that owns every device byte through its own arena.  For them the
// scratch lives in the file-scope arrays below, sized for n <= LUSP_NOALLOC_MAX_N,
// which every GPU that loads this library holds until the process exits
// (1.25 MiB per device).
#include <cuda_runtime.h>

#include <mutex>

#include "lu_gpu_par.h"
#include "luspice_b200.h"
#include "engine_internal.h"

static __device__ __align__(256) int g_noalloc_work_i[LUSP_NOALLOC_MAX_N];
static __device__ __align__(256) double g_noalloc_work_d[2 * LUSP_NOALLOC_MAX_N];

namespace {

constexpr int kMaxDevices = 64;

struct NoallocScratch {
    int* work_i = nullptr;
    double* work_d = nullptr;
};

std::mutex g_mu;
NoallocScratch g_scratch[kMaxDevices];

// Device addresses of the scratch arrays for the current device, looked up
// once per device (the names are host-side stand-ins, not device addresses).
int scratch_for_current_device(NoallocScratch* out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return lusp::cuda_fail(e, "trisolve_par_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) {
        lusp::set_error("trisolve_par_noalloc: device ordinal %d above %d", dev, kMaxDevices - 1);
        return LUSP_EARG;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    NoallocScratch& s = g_scratch[dev];
    if (!s.work_i) {
        void* pi = nullptr;
        void* pd = nullptr;
        e = cudaGetSymbolAddress(&pi, g_noalloc_work_i);
        if (e != cudaSuccess) return lusp::cuda_fail(e, "trisolve_par_noalloc: cudaGetSymbolAddress(work_i)");
        e = cudaGetSymbolAddress(&pd, g_noalloc_work_d);
        if (e != cudaSuccess) return lusp::cuda_fail(e, "trisolve_par_noalloc: cudaGetSymbolAddress(work_d)");
        s.work_i = static_cast<int*>(pi);
        s.work_d = static_cast<double*>(pd);
    }
    *out = s;
    return LUSP_OK;
}

}  // namespace

extern "C" int lusp_trisolve_par_noalloc(int n, const int* Lp, const int* Li, const double* Lx,
                                         const int* Up, const int* Ui, const double* Ux,
                                         const int* pinv, const int* q, const double* b, double* x,
                                         void* stream) {
    if (n <= 0 || !Lp || !Li || !Lx || !Up || !Ui || !Ux || !pinv || !b || !x) {
        lusp::set_error("trisolve_par_noalloc: bad arguments");
        return LUSP_EARG;
    }
    if (n > LUSP_NOALLOC_MAX_N) {
        lusp::set_error("trisolve_par_noalloc: n = %d exceeds LUSP_NOALLOC_MAX_N = %d; use "
                        "lusp_trisolve_par_launch with caller-provided work arrays",
                        n, LUSP_NOALLOC_MAX_N);
        return LUSP_EARG;
    }
    NoallocScratch s;
    int rc = scratch_for_current_device(&s);
    if (rc != LUSP_OK) return rc;
    // Nothing in the scratch has to start at zero: the kernel writes every
    // work_i / work_d entry it reads (rowat, P b, y) before reading it.
    trisolve_par_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(n, Lp, Li, Lx, Up, Ui, Ux, pinv, q, b,
                                                            x, s.work_i, s.work_d);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LUSP_OK : lusp::cuda_fail(e, "trisolve_par_noalloc: launch");
}
