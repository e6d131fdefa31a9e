// The ALU issue-rate probe that gives the noise and shaping kernels their roofline denominator:
// those kernels are bound by integer and FP32 lane operations, not by HBM or the tensor cores, so
// their peak is the rate the SMs retire a mix of IMAD and FFMA, measured on the device at hand.
//
// Every counted operation must really execute. An affine integer recurrence (a = a * m + c with
// constants) unrolled 16 times is one affine map the compiler may fold into a single multiply-add,
// so the integer chains are quadratic (a = a * a + seed, one IMAD that no rewriting shortens) and
// the float chains are FFMAs, which IEEE rounding keeps from being combined. The count is 8 lane
// operations per iteration and thread: 4 IMAD and 4 FFMA, plus loop overhead the count leaves
// out, so the rate is a floor of the issue rate, which is at most 128 lane instructions per SM
// per clock.
#include "kernels.h"

namespace tgb {
namespace {

constexpr int kIterations = 8192;
constexpr int kChains = 8;  // 4 IMAD + 4 FFMA chains per thread, independent of one another
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) alu_probe_kernel(uint32_t* sink, uint32_t seed) {
    uint32_t a0 = threadIdx.x ^ seed, a1 = a0 * 3u + 1u, a2 = a0 * 5u + 3u, a3 = a0 * 7u + 5u;
    float f0 = float(threadIdx.x) * 1e-3f, f1 = f0 + 0.25f, f2 = f0 + 0.5f, f3 = f0 + 0.75f;
#pragma unroll 16
    for (int i = 0; i < kIterations; ++i) {
        a0 = a0 * a0 + seed;
        f0 = fmaf(f0, 0.999f, 0.001f);
        a1 = a1 * a1 + seed;
        f1 = fmaf(f1, 0.999f, 0.001f);
        a2 = a2 * a2 + seed;
        f2 = fmaf(f2, 0.999f, 0.001f);
        a3 = a3 * a3 + seed;
        f3 = fmaf(f3, 0.999f, 0.001f);
    }
    const uint32_t r = (a0 ^ a1 ^ a2 ^ a3) + __float_as_uint(f0 + f1 + f2 + f3);
    if (r == 0x12345678u) {
        sink[blockIdx.x & 4095u] = r;
    }
}

}  // namespace

cudaError_t launch_alu_probe(uint32_t* sink, uint64_t* laneOps, cudaStream_t stream) {
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const uint32_t blocks = uint32_t(sms) * 16u;
    alu_probe_kernel<<<blocks, kThreads, 0, stream>>>(sink, 7u);
    *laneOps = uint64_t(blocks) * kThreads * kIterations * kChains;
    return cudaGetLastError();
}

}  // namespace tgb
