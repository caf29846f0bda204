// noalloc.cu -- local energy of a built H_VV that allocates no device memory.
//
// Some callers may not allocate device memory themselves: an XLA custom call
// (JAX FFI handler) runs inside XLA's own memory plan, and an embedding
// application may hand this library a fixed memory budget up front.  For
// them dnq_ham_local_energy_noalloc computes the same result as
// dnq_ham_local_energy without cudaMalloc, cudaMallocAsync, cudaFree or any
// allocating library routine.  Its scratch -- the FP32 copy of x and the
// per-block partial sums of the reduction -- lives in the file-scope array
// below, which every GPU that loads this library holds until the process
// exits (4 MiB + 74 KiB).
//
// Rules of use:
//   * x and eloc must be device memory of the handle's GPU and must not
//     overlap: eloc first receives H.x while x is still being gathered, then
//     y_i / x_i;
//   * out2 may be device memory of the handle's GPU (the call then only
//     enqueues work on the stream and returns) or host memory (the call
//     copies the pair back and waits for the stream);
//   * n_V <= kNoAllocMaxDets (larger handles are rejected, nothing is run);
//   * precision DNQ_F32 needs the handle's FP32 values to exist already
//     (one earlier dnq_ham_spmv / dnq_ham_local_energy call with DNQ_F32);
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.  The address is cached per device ordinal
//     for the life of the process and is not valid after cudaDeviceReset;
//   * all calls share one array: calls that overlap on the GPU (different
//     streams, or another process thread) race on it and must be serialised
//     by the caller.  Every call overwrites what it reads, so nothing needs
//     clearing between calls.
#include <mutex>

#include "ham.cuh"

namespace dnq {

void spmv_block(const dnq_ham_s* h, const Csr& m, const double* x, double* y,
                const double* yadd, int precision, cudaStream_t s, float* x32,
                const double* diag);
void to_f32(const double* x, i64 n, float* o, cudaStream_t s);
void energy_reduce_into(const double* x, const double* y, i64 n, double* eloc, double* part,
                        int nb, double* out2_dev, cudaStream_t s);

namespace {

constexpr i64 kNoAllocMaxDets = 1 << 20;        // FP32 copy of x: 4 MiB
constexpr int kNoAllocBlocks = 592;             // reduction partials: 4 per block
constexpr size_t kX32Doubles = kNoAllocMaxDets / 2;
constexpr size_t kScratchDoubles = kX32Doubles + 4 * kNoAllocBlocks + 2;

// File-scope scratch: [x32 as floats | partials | result pair].  In host
// code this name is only a stand-in; the device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

double* scratch_for(int device) {
    require(device >= 0 && device < kMaxDevices, DNQ_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
        int cur = -1;
        DNQ_CUDA(cudaGetDevice(&cur));
        require(cur == device, DNQ_ERR_INVALID, "scratch set-up needs the handle's device current");
        void* p = nullptr;
        DNQ_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_addr[device] = static_cast<double*>(p);
    }
    return g_addr[device];
}

}  // namespace
}  // namespace dnq

using namespace dnq;

extern "C" {

int dnq_ham_local_energy_noalloc(dnq_ham_t h, const double* x, double* eloc, double* out2,
                                 int precision, void* stream) {
    DNQ_API_BEGIN
    require(h && x && eloc && out2, DNQ_ERR_INVALID, "null argument");
    require(precision == DNQ_F64 || precision == DNQ_F32, DNQ_ERR_INVALID, "invalid precision");
    const i64 n = h->n_v;
    require(n <= kNoAllocMaxDets, DNQ_ERR_INVALID,
            "n_V exceeds the no-allocation scratch capacity (1048576 determinants)");
    require(is_device_ptr(x) && is_device_ptr(eloc), DNQ_ERR_INVALID,
            "x and eloc must be device memory for the no-allocation entry point");
    require_on_device(x, h->device, "x");
    require_on_device(eloc, h->device, "eloc");
    {
        const char* xb = reinterpret_cast<const char*>(x);
        const char* eb = reinterpret_cast<const char*>(eloc);
        const size_t len = (size_t)n * sizeof(double);
        require(n == 0 || xb + len <= eb || eb + len <= xb, DNQ_ERR_INVALID,
                "x and eloc must not overlap: eloc receives H x while x is read");
    }
    if (precision == DNQ_F32)
        require(h->vv.f32_ready() && h->diag_op.n == (size_t)h->n_v,
                DNQ_ERR_INVALID,
                "FP32 values not prepared: run one FP32 dnq_ham_spmv or "
                "dnq_ham_local_energy on this handle first");
    const bool dev_out = is_device_ptr(out2);
    if (dev_out) require_on_device(out2, h->device, "out2");
    DeviceGuard g(h->device);
    cudaStream_t s = (cudaStream_t)stream;
    double* base = scratch_for(h->device);
    float* x32 = reinterpret_cast<float*>(base);
    double* part = base + kX32Doubles;
    double* res = dev_out ? out2 : part + 4 * kNoAllocBlocks;
    if (n == 0) {
        if (dev_out) {
            DNQ_CUDA(cudaMemsetAsync(out2, 0, 2 * sizeof(double), s));   // +0.0 bits
        } else {
            out2[0] = 0.0;
            out2[1] = 0.0;
        }
        return DNQ_OK;
    }
    // y = H x goes into eloc, then eloc <- y / x in place by the reduction.
    if (precision == DNQ_F32) {
        to_f32(x, n, x32, s);
        spmv_block(h, h->vv, x, eloc, nullptr, DNQ_F32, s, x32, h->diag_op.p);
    } else {
        spmv_block(h, h->vv, x, eloc, nullptr, DNQ_F64, s, nullptr, nullptr);
    }
    energy_reduce_into(x, eloc, n, eloc, part, kNoAllocBlocks, res, s);
    if (!dev_out) {
        DNQ_CUDA(cudaMemcpyAsync(out2, res, 2 * sizeof(double), cudaMemcpyDefault, s));
        DNQ_CUDA(cudaStreamSynchronize(s));
    }
    DNQ_API_END
}

}  // extern "C"
