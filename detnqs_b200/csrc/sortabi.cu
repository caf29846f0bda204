// sortabi.cu -- the build's radix sort behind a C entry point, so that its
// order can be checked from outside (tests compare it with a stable host
// sort).  No counterpart in the reference.
#include "prim.cuh"

using namespace dnq;

extern "C" {

int dnq_sort_order(const uint64_t* keys, int64_t n, int words, const int* bits,
                   uint32_t* order, int device, void* stream) {
    DNQ_API_BEGIN
    require(keys && bits && order, DNQ_ERR_INVALID, "null argument");
    require(words == 1 || words == 2, DNQ_ERR_INVALID, "words must be 1 or 2");
    require(n >= 0 && n < (int64_t)0xffffffffll, DNQ_ERR_INVALID, "n out of range");
    for (int w = 0; w < words; ++w)
        require(bits[w] >= 0 && bits[w] <= 64, DNQ_ERR_INVALID, "bits must be in [0, 64]");
    DeviceGuard g(device);
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) return DNQ_OK;
    DIn<u64> kd(keys, (size_t)n * words, s);
    DBuf<u32> od(n, s);
    if (words == 1) {
        DBuf<u64> ks(n, s);
        prim::radix_sort<u64, u32>(kd.p, ks.p, nullptr, od.p, n, bits, s);
    } else {
        DBuf<ulonglong2> ks(n, s);
        prim::radix_sort<ulonglong2, u32>(reinterpret_cast<const ulonglong2*>(kd.p), ks.p,
                                          nullptr, od.p, n, bits, s);
    }
    copy_out(order, od.p, n, s);
    DNQ_CUDA(cudaStreamSynchronize(s));
    DNQ_API_END
}

}  // extern "C"
