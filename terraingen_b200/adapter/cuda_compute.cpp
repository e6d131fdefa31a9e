// TerrainGen's CUDA device on libtgb200: a drop-in replacement for the reference's
// src/gpu/cuda.cpp, implementing the same `CudaCompute` (src/gpu/cuda.h) over the C ABI in
// include/tgb200.h.
//
// Built inside a TerrainGen tree in place of src/gpu/cuda.cpp, with src/gpu/backend.cpp
// compiled with TERRAINGEN_HAS_CUDA_KERNELS=1 and linked to libtgb200.so, it makes
// Backend::Cuda run the noise-layer and crater kernels on the B200 kernels of libtgb200 instead of
// JIT-compiled Slang PTX: RunKernel (src/gpu/kernel.cpp) binds the same buffers and push
// constants, and this device maps them onto tg_noise_layer_rows, tg_craters_apply_lists and
// tg_crater_datums.
// Programs are told apart by their compiled form's address, so the generated CompiledKernel<>
// definitions (cmake/Kernel.cpp.in) are used as they are; PTX is not read.
#include "gpu/cuda.h"

#include "terraingen/layers/kernels/craters.h"
#include "terraingen/layers/kernels/noise_layer.h"
#include "tgb200.h"

#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

namespace terraingen {

namespace {

/// The push constants RunKernel passes (src/gpu/kernel.cpp:34-40).
struct Params {
    std::uint32_t width;
    std::uint32_t rows;
    std::uint32_t noData;
    float noDataValue;
    std::uint32_t firstRow;
};

enum class Program { None, NoiseLayer, Craters, Datums, BodyDatums };

/// Whether `program` is the compiled form of kernel `Kernel`.
template <typename Kernel> bool Is(const KernelProgram& program) {
    const KernelProgram compiled = CompiledKernel<Kernel>();
    return program.ptx.data() == compiled.ptx.data() &&
           program.spirv.data() == compiled.spirv.data();
}

Program Identify(const KernelProgram& program) {
    if (Is<NoiseLayerKernel>(program)) {
        return Program::NoiseLayer;
    }
    if (Is<CraterShapeKernel>(program)) {
        return Program::Craters;
    }
    if (Is<CraterDatumKernel>(program)) {
        return Program::Datums;
    }
    if (Is<CraterBodyDatumKernel>(program)) {
        return Program::BodyDatums;
    }
    return Program::None;
}

[[noreturn]] void Throw(const char* what) {
    throw std::runtime_error(std::string("tgb200 ") + what + ": " + tg_last_error());
}

template <typename T> const T* As(const DeviceBuffer& buffer) {
    return reinterpret_cast<const T*>(buffer.bytes.data());
}

template <typename T> std::uint32_t Count(const DeviceBuffer& buffer) {
    return static_cast<std::uint32_t>(buffer.bytes.size() / sizeof(T));
}

}  // namespace

struct CudaCompute::State {
    tg_device* device = nullptr;
    std::string name;
};

CudaCompute::CudaCompute(std::unique_ptr<State> state) : m_state(std::move(state)) {}

CudaCompute::~CudaCompute() {
    if (m_state && m_state->device != nullptr) {
        tg_close(m_state->device);
    }
}

std::unique_ptr<CudaCompute> CudaCompute::Open() {
    auto state = std::make_unique<State>();
    if (tg_open(0, &state->device) != TG_OK) {
        throw std::runtime_error(std::string("tgb200: ") + tg_last_error());
    }
    char name[256] = {};
    tg_device_name(state->device, name, sizeof(name));
    state->name = std::string(name) + " (tgb200)";
    return std::unique_ptr<CudaCompute>(new CudaCompute(std::move(state)));
}

const std::string& CudaCompute::DeviceName() const {
    return m_state->name;
}

bool CudaCompute::CanRun(const KernelProgram& program) const {
    return Identify(program) != Program::None;
}

void CudaCompute::Run(const KernelProgram& program, Span<const DeviceBuffer> buffers,
                      Span<const std::byte> pushConstants, const Dispatch& /*dispatch*/) {
    if (pushConstants.size() < sizeof(Params)) {
        throw std::runtime_error("tgb200: push constants are not RunKernel's");
    }
    Params params;
    std::memcpy(&params, pushConstants.data(), sizeof(params));
    const tg_nodata nodata{params.noData, params.noDataValue};
    const Program kind = Identify(program);
    if (kind == Program::NoiseLayer && buffers.size() >= 4) {
        // heights, xs, ys, NoiseLayerKernel (src/layers/kernels/noise_layer.slang)
        float* heights = reinterpret_cast<float*>(buffers[0].output);
        if (tg_noise_layer_rows(m_state->device, buffers[3].bytes.data(), buffers[3].bytes.size(),
                                As<float>(buffers[1]), As<float>(buffers[2]), params.width,
                                params.rows, heights, nodata, TG_MEMORY_HOST,
                                nullptr) != TG_OK) {
            Throw("noise layer");
        }
        return;
    }
    if (kind == Program::Craters && buffers.size() >= 11) {
        // heights, xs, ys, CraterShapeKernel, records, data, tiles, entries, frames, points,
        // lows (src/layers/kernels/craters.slang, bound by ShapeTilesOnGpu, apply.cpp:174-196)
        float* heights = reinterpret_cast<float*>(buffers[0].output);
        const std::uint32_t* tiles = As<std::uint32_t>(buffers[6]);
        if (Count<std::uint32_t>(buffers[6]) >= 3 && tiles[2] != 0u) {
            // On a body: the craters' frames and the strip's cells as split points
            // (ShapeCratersOnBody, craters.slang's body branch).
            if (tg_craters_apply_body(
                    m_state->device, buffers[3].bytes.data(), buffers[3].bytes.size(),
                    buffers[4].bytes.data(), Count<CraterRecord>(buffers[4]),
                    As<float>(buffers[5]), Count<float>(buffers[5]), buffers[8].bytes.data(),
                    tiles, Count<std::uint32_t>(buffers[6]), As<std::uint32_t>(buffers[7]),
                    Count<std::uint32_t>(buffers[7]), buffers[9].bytes.data(), params.width,
                    params.rows, params.firstRow, heights, nodata, TG_MEMORY_HOST,
                    nullptr) != TG_OK) {
                Throw("craters on a body");
            }
            return;
        }
        const float* lows = As<float>(buffers[10]);
        if (tg_craters_apply_lists(
                m_state->device, buffers[3].bytes.data(), buffers[3].bytes.size(),
                buffers[4].bytes.data(), Count<CraterRecord>(buffers[4]), As<float>(buffers[5]),
                Count<float>(buffers[5]), As<std::uint32_t>(buffers[6]),
                Count<std::uint32_t>(buffers[6]), As<std::uint32_t>(buffers[7]),
                Count<std::uint32_t>(buffers[7]), As<float>(buffers[1]), lows,
                As<float>(buffers[2]), lows + params.width, params.width, params.rows,
                params.firstRow, heights, nodata, TG_MEMORY_HOST, nullptr) != TG_OK) {
            Throw("craters");
        }
        return;
    }
    if (kind == Program::Datums && buffers.size() >= 11) {
        // heights, xs, ys, CraterDatumKernel, records, data, band floats, band cells, cells,
        // entries, targets (src/layers/kernels/crater_datums.slang, bound by AddDatumRelief,
        // datum_fit.cpp:303-328)
        float* heights = reinterpret_cast<float*>(buffers[0].output);
        if (tg_crater_datums(m_state->device, buffers[3].bytes.data(), buffers[3].bytes.size(),
                             buffers[4].bytes.data(), Count<CraterRecord>(buffers[4]),
                             As<float>(buffers[5]), Count<float>(buffers[5]),
                             As<float>(buffers[6]), Count<float>(buffers[6]),
                             As<std::uint32_t>(buffers[7]), Count<std::uint32_t>(buffers[7]),
                             As<std::uint32_t>(buffers[8]), Count<std::uint32_t>(buffers[8]),
                             As<std::uint32_t>(buffers[9]), Count<std::uint32_t>(buffers[9]),
                             As<std::uint32_t>(buffers[10]), Count<std::uint32_t>(buffers[10]),
                             params.width, params.rows, params.firstRow, heights, TG_MEMORY_HOST,
                             nullptr) != TG_OK) {
            Throw("crater datums");
        }
        return;
    }
    if (kind == Program::BodyDatums && buffers.size() >= 11) {
        // heights, xs, ys, CraterBodyDatumKernel, records, data, frames, bounds, lists, entries,
        // positions (src/layers/kernels/crater_body_datums.slang, bound by FitBodyDatumsOnGpu)
        float* heights = reinterpret_cast<float*>(buffers[0].output);
        if (tg_crater_body_datums(m_state->device, buffers[3].bytes.data(),
                                  buffers[3].bytes.size(), buffers[4].bytes.data(),
                                  Count<CraterRecord>(buffers[4]), As<float>(buffers[5]),
                                  Count<float>(buffers[5]), buffers[6].bytes.data(),
                                  As<float>(buffers[7]), As<std::uint32_t>(buffers[8]),
                                  Count<std::uint32_t>(buffers[8]), As<std::uint32_t>(buffers[9]),
                                  Count<std::uint32_t>(buffers[9]), buffers[10].bytes.data(),
                                  params.width, params.rows, params.firstRow, heights, nodata,
                                  TG_MEMORY_HOST, nullptr) != TG_OK) {
            Throw("crater datums on a body");
        }
        return;
    }
    throw std::runtime_error("tgb200: no form of this kernel");
}

}  // namespace terraingen
