// snn_noalloc.cu -- score one greedy step without allocating device memory.
//
// Some callers cannot call cudaMalloc: code that runs while another runtime
// owns the device memory (a framework's caching allocator or a fixed memory
// budget that must not grow), real-time or embedded hosts that forbid
// allocation after start-up, and code paths that must not synchronise the
// device (cudaMalloc/cudaFree can).  For them this entry point takes
// caller-owned device buffers for all inputs and outputs and keeps its own
// scratch -- the per-(candidate, k, row) kNN predictions, the device-side
// step state and copies of the small index arrays -- in one file-scope
// static __device__ array of fixed size.  It calls no cudaMalloc, cudaFree or
// allocating library routine.
//
// The array is device memory of the library's own module: the CUDA runtime
// places it on a GPU when it loads this library's kernels there (with lazy
// loading, the CUDA 12 default, at the first launch or symbol lookup of the
// library on that GPU -- the first call of this or any other entry point),
// and it stays there until the process exits.  A caller with a strict
// no-allocation window should make one call (or any library call) on each GPU
// before the window opens.  All calls share the array and it keeps the last
// call's contents, so calls whose GPU work overlaps (two host threads, or two
// streams, with work in flight at the same time) race on it; run them one
// after another.
#include <float.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "../../include/speedynn_b200.h"
#include "snn_internal.h"

namespace {

constexpr size_t kStateFloats = 64;     // snn::State, padded to 256 bytes
constexpr size_t kKvFloats = 256;       // k values
constexpr size_t kCandFloats = 1024;    // candidate feature ids
constexpr size_t kPredFloats = size_t(1) << 22;  // predictions: n_cand * num_k_vals * n_rows <= 4,194,304
constexpr size_t kScratchFloats = kStateFloats + kKvFloats + kCandFloats + kPredFloats;  // ~16 MB

static_assert(sizeof(snn::State) <= kStateFloats * sizeof(float), "state must fit its slot");

// The scratch.  Host code must not use this name as an address: on the host it
// is only a stand-in, so the device address is looked up per device below.
static __device__ __align__(256) float g_step_scratch[kScratchFloats];

// Device address of the scratch on the current device.  Looked up on every
// call (a cheap runtime query) rather than cached: after a device reset the
// module is loaded again and the array may sit at another address.
int scratch_address(float **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_step_scratch);
    if (e != cudaSuccess || !p) {
        char msg[256];
        snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the step scratch failed: %s", cudaGetErrorString(e));
        cudaGetLastError();
        return snn::record_error(SNN_ERR_CUDA, msg);
    }
    *out = static_cast<float *>(p);
    return SNN_OK;
}

int err(int code, const char *msg) { return snn::record_error(code, msg); }

int cuda_err(cudaError_t e, const char *what)
{
    char msg[256];
    snprintf(msg, sizeof msg, "%s failed: %s", what, cudaGetErrorString(e));
    cudaGetLastError();
    return snn::record_error(SNN_ERR_CUDA, msg);
}

}  // namespace

extern "C" SNN_API int snn_score_step_noalloc(const float *D, int ld, const float *XT, const float *XV, int ldr,
                                              const float *y_train, const float *y_val, int n_rows, int n_cols, int p,
                                              const int *cands, int n_cand, const int *k_vals, int num_k_vals,
                                              int backward, float *errors, double *errors64, void *stream)
{
    snn::clear_error();
    if (!D || !XT || !XV || !y_train || !y_val || !cands || !k_vals || !errors || !errors64)
        return err(SNN_ERR_ARG, "snn_score_step_noalloc: null pointer argument");
    if (n_rows <= 0 || n_cols <= 0 || p <= 0 || n_cand <= 0 || num_k_vals <= 0)
        return err(SNN_ERR_ARG, "snn_score_step_noalloc: sizes must be positive");
    if (ld < n_cols || ld % snn::kPadCols != 0 || ldr < n_rows)
        return err(SNN_ERR_ARG, "snn_score_step_noalloc: ld must be a multiple of 64 and >= n_train, ldr >= n_rows");
    if ((size_t)num_k_vals > kKvFloats || (size_t)n_cand > kCandFloats)
        return err(SNN_ERR_ARG, "snn_score_step_noalloc: at most 256 k values and 1024 candidates");
    if ((size_t)n_cand * (size_t)num_k_vals * (size_t)n_rows > kPredFloats)
        return err(SNN_ERR_ARG,
                   "snn_score_step_noalloc: n_cand * num_k_vals * n_rows exceeds the fixed scratch of 4,194,304 predictions");
    int kmax = 0;
    for (int m = 0; m < num_k_vals; ++m) {
        if (k_vals[m] <= 0) return err(SNN_ERR_ARG, "snn_score_step_noalloc: k values must be >= 1");
        kmax = std::max(kmax, k_vals[m]);
    }
    for (int c = 0; c < n_cand; ++c)
        if (cands[c] < 0 || cands[c] >= p) return err(SNN_ERR_ARG, "snn_score_step_noalloc: candidate id outside [0, p)");
    if ((reinterpret_cast<uintptr_t>(D) | reinterpret_cast<uintptr_t>(XT)) & 15u)
        return err(SNN_ERR_ARG, "snn_score_step_noalloc: D and XT must be 16-byte aligned (they are read by TMA copies)");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
    float *base = nullptr;
    if (int rc = scratch_address(&base)) return rc;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const snn::ScorePlan plan = snn::plan_score(kmax, n_cand, max_smem);
    if (plan.cc == 0) return err(SNN_ERR_UNSUPPORTED, "snn_score_step_noalloc: k_max above 256");

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    snn::State *st = reinterpret_cast<snn::State *>(base);
    int *kv = reinterpret_cast<int *>(base + kStateFloats);
    int *cd = reinterpret_cast<int *>(base + kStateFloats + kKvFloats);
    float *pred = base + kStateFloats + kKvFloats + kCandFloats;

    // the state must start at zero (not done, no error) on every call
    if ((e = cudaMemsetAsync(st, 0, sizeof(snn::State), s)) != cudaSuccess) return cuda_err(e, "cudaMemsetAsync");
    if ((e = cudaMemcpyAsync(kv, k_vals, sizeof(int) * num_k_vals, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_err(e, "cudaMemcpyAsync");
    if ((e = cudaMemcpyAsync(cd, cands, sizeof(int) * n_cand, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return cuda_err(e, "cudaMemcpyAsync");

    snn::Bufs b;
    memset(&b, 0, sizeof b);
    b.XT = XT;
    b.XV = XV;
    b.ldc = ld;
    b.ldr = ldr;
    b.yc = y_train;
    b.yr = y_val;
    b.D = const_cast<float *>(D);  // read only here
    b.n_rows = n_rows;
    b.n_cols = n_cols;
    b.p = p;
    b.kvals = kv;
    b.nk = num_k_vals;
    b.kmax = kmax;
    b.pred = pred;
    b.rmse32 = errors;
    b.rmse64 = errors64;
    b.cands = cd;
    b.st = st;

    if (snn::score_tma_supported(kmax)) e = snn::launch_score_tma(b, n_cand, backward, s);
    else e = snn::launch_score(b, n_cand, plan, backward, s);
    if (e != cudaSuccess) return cuda_err(e, "scoring kernel launch");
    if ((e = snn::launch_reduce(b, n_cand, s)) != cudaSuccess) return cuda_err(e, "error reduction launch");

    snn::State hs;
    if ((e = cudaMemcpyAsync(&hs, st, sizeof hs, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return cuda_err(e, "cudaMemcpyAsync");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_err(e, "cudaStreamSynchronize");
    if (hs.error == snn::kErrTimeout) return err(SNN_ERR_TIMEOUT, "snn_score_step_noalloc: a device pipeline wait timed out");
    return SNN_OK;
}
