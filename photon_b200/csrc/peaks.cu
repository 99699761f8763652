// L2 read-bandwidth probe: the denominator for kernels whose working set (the BVH, the triangles)
// stays in the 126 MB L2, so that their algorithmic bytes can be read against L2 as well as HBM.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_scene.h"
#include "peaks.h"

namespace ptw {
namespace {

// Every thread reads its grid-strided 16-byte words `reps` times with ld.global.cg (cached in L2,
// not L1), so each load is an L2 access. The XOR keeps the loads live; the store never happens for
// the zero-filled buffer the host passes.
__global__ void __launch_bounds__(256) k_l2_read(const uint4* __restrict__ buf, size_t words, int reps, uint32_t* sink) {
    uint32_t acc = 0;
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    for (int r = 0; r < reps; r++) {
        for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < words; i += stride) {
            uint4 v = __ldcg(buf + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    }
    if (acc == 0x9e3779b9u) sink[0] = acc;
}

}  // namespace

double measure_l2_read_gbs(int device, size_t bytes, int reps) {
    if (bytes < (1u << 20) || bytes > (size_t(64) << 20) || reps < 1 || reps > 1000)
        throw Error{PT_ERR_INVALID, "L2 probe: bytes must be 1..64 MiB and reps 1..1000"};
    PTW_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop{};
    PTW_CUDA(cudaGetDeviceProperties(&prop, device));
    int per_sm = 0;
    PTW_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_l2_read, 256, 0));
    const int grid = prop.multiProcessorCount * (per_sm > 0 ? per_sm : 1);
    const size_t words = bytes / sizeof(uint4);
    DeviceBuffer<uint4> buf;
    DeviceBuffer<uint32_t> sink;
    buf.allocate(words);
    sink.allocate(1);
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double best = 0.0;
    cudaError_t err = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    if (err == cudaSuccess) err = cudaMemsetAsync(buf.ptr, 0, words * sizeof(uint4), s);
    if (err == cudaSuccess) {
        k_l2_read<<<grid, 256, 0, s>>>(buf.ptr, words, reps, sink.ptr);  // warm-up: brings the buffer into L2
        err = cudaGetLastError();
    }
    for (int k = 0; k < 5 && err == cudaSuccess; k++) {
        err = cudaEventRecord(e0, s);
        k_l2_read<<<grid, 256, 0, s>>>(buf.ptr, words, reps, sink.ptr);
        if (err == cudaSuccess) err = cudaGetLastError();
        if (err == cudaSuccess) err = cudaEventRecord(e1, s);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (err == cudaSuccess && ms > 0.0f) {
            double gbs = double(words * sizeof(uint4)) * double(reps) / (double(ms) * 1e-3) / 1e9;
            if (gbs > best) best = gbs;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    PTW_CUDA(err);
    return best;
}

}  // namespace ptw
