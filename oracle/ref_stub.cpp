// Link stub for building the reference TerrainGen CPU path offline (test infrastructure only).
//
// The reference's CMake build generates a few files and fetches Vulkan's loader (volk); none of
// that is available offline. This file supplies, in our own words, the pieces the CPU path links
// against:
//   - VulkanCompute, which always reports itself unavailable (src/gpu/vulkan.h:35-66 declares it);
//   - CompiledKernel<> forms for the four Slang kernels (cmake/Kernel.cpp.in generates these
//     in the reference build), as tags: with the reference's own CUDA device they are never run
//     (the CPU build reports no CUDA kernels), and the product's drop-in device recognises them;
//   - GetBuildInfo (src/util/build_info.cpp.in).
// Nothing here computes terrain; the reference's own sources do.
#include "gpu/vulkan.h"

#include "terraingen/layers/kernels/craters.h"
#include "terraingen/layers/kernels/noise_layer.h"
#include "terraingen/util/build_info.h"

#include <stdexcept>

namespace terraingen {

struct VulkanCompute::State {};

VulkanCompute::VulkanCompute(std::unique_ptr<State> state) : m_state(std::move(state)) {}
VulkanCompute::~VulkanCompute() = default;

const std::string& VulkanCompute::DeviceName() const {
    static const std::string name = "none";
    return name;
}

bool VulkanCompute::CanRun(const KernelProgram&) const {
    return false;
}

void VulkanCompute::Run(const KernelProgram&, Span<const DeviceBuffer>, Span<const std::byte>,
                        const Dispatch&) {
    throw std::runtime_error("Vulkan is not part of the oracle build");
}

std::unique_ptr<VulkanCompute> VulkanCompute::Open() {
    throw std::runtime_error("Vulkan is not part of the oracle build");
}

std::optional<std::size_t> PickDevice(Span<const DeviceKind>) {
    return std::nullopt;
}

std::string VulkanInstallHint() {
    return "Vulkan is not part of the oracle build";
}

// Each kernel's "compiled form" is a distinct tag string: nothing reads it as PTX, but a CUDA
// device told apart by its address (the product's drop-in CudaCompute) can recognise the kernel.
namespace {
const char kNoiseTag[] = "noise_layer";
const char kCraterTag[] = "craters";
const char kDatumTag[] = "crater_datums";
const char kBodyDatumTag[] = "crater_body_datums";

KernelProgram Tagged(const char* tag, std::size_t size) {
    KernelProgram program;
    program.ptx = {tag, size};
    return program;
}
}  // namespace

template <> KernelProgram CompiledKernel<NoiseLayerKernel>() {
    return Tagged(kNoiseTag, sizeof(kNoiseTag));
}
template <> KernelProgram CompiledKernel<CraterShapeKernel>() {
    return Tagged(kCraterTag, sizeof(kCraterTag));
}
template <> KernelProgram CompiledKernel<CraterDatumKernel>() {
    return Tagged(kDatumTag, sizeof(kDatumTag));
}
template <> KernelProgram CompiledKernel<CraterBodyDatumKernel>() {
    return Tagged(kBodyDatumTag, sizeof(kBodyDatumTag));
}

BuildInfo GetBuildInfo() {
    return BuildInfo{"oracle", false, "offline"};
}

}  // namespace terraingen
