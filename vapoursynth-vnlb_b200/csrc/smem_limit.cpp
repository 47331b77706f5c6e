// Dynamic shared-memory limits of the kernels, raised and never lowered.
//
// A kernel's cudaFuncAttributeMaxDynamicSharedMemorySize is one value per
// function and device, while sessions on different host threads launch the
// same kernels with different amounts (a gray clip's match beside a YUV
// clip's, one rank's filter beside another's).  Setting the exact amount
// before each launch would let another thread lower the limit between this
// thread's set and its launch, which then fails with an invalid argument.
// The limit only ever grows here, under a lock, so every launch that asked
// for at most the recorded limit stays valid.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

namespace vnlbgpu {

cudaError_t raise_smem_limit(const void* kernel, size_t bytes) {
    static std::mutex lock;
    static std::map<std::pair<int, const void*>, size_t> limits;
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return err;
    std::lock_guard<std::mutex> guard(lock);
    size_t& current = limits[{device, kernel}];
    if (bytes <= current) return cudaSuccess;
    err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (err == cudaSuccess) current = bytes;
    return err;
}

}  // namespace vnlbgpu
