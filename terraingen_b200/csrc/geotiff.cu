// GeoTIFF heightmap output (WriteGeoTiff, src/raster/geotiff/geotiff_write.cpp) with the tile
// encoding on the device.
//
// The reference writes a tiled, little-endian float32 GeoTIFF: every band's tiles in order (band,
// tile row, tile column), each `tile` x `tile` pixels padded with the no-data value (or 0), and,
// compressed, first run through TIFF's floating-point predictor (3) and then LZW or Deflate;
// tiles at even offsets after an 8-byte (16 for BigTIFF) header, the IFD after the last tile.
// Here:
//   1. tiles_kernel lays every tile out in device memory, with the predictor when compressed:
//      each predicted byte is a byte plane's difference from the byte before it in the row, so
//      every output byte is computed independently (one thread per sample, 4 planes);
//   2. LZW: lzw_kernel encodes each tile with one warp, the whole warp staging the tile's bytes
//      through shared memory and clearing the string table, one lane running the encoder (the
//      reference's code stream exactly: greedy longest match, 9- to 12-bit MSB-first codes with
//      the early width change, Clear when the next code reaches 4094); the compressed tiles are
//      packed on the device at their file offsets and copied out in one piece;
//      Deflate: the predicted tiles are copied out and compressed with zlib at level 6 on host
//      threads (the reference uses miniz at level 6: the same decoded data, not the same bytes);
//   3. the header, the tiles and the IFD (the reference's tags, in tag order, values of more
//      than one word after the table at even offsets) are written to the file.
// With compression None or LZW the file is the reference's byte for byte.
#include <cuda_runtime.h>
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tgb200.h"
#include "api_internal.h"
#include "kernels.h"

using namespace tgb;
using namespace tgb::api;

namespace {

constexpr uint32_t kNone = 0, kLzw = 1, kPackBits = 2, kDeflate = 3;  // TiffCompression's order

// --- 1. tiles ----------------------------------------------------------------------------------

struct TileSource {
    const float* const* bands;  // device pointers, row-major width x height
    uint32_t width, height, tile;
    uint32_t across, down;      // tiles per band
    float fill;
    bool predictor;
};

// One block per (tile, row of the tile), threads over its samples. Without the predictor a row
// is its samples' little-endian bytes; with it the bytes are regrouped into planes (the most
// significant byte of every sample first) and each replaced by its difference from the byte
// before it in the row (EncodeFloatPredictor, tiff_codecs.cpp:354, stride 1).
__global__ void tiles_kernel(const TileSource s, uint8_t* __restrict__ out) {
    const uint32_t tileIndex = blockIdx.x / s.tile, y = blockIdx.x % s.tile;
    const uint32_t perBand = s.across * s.down;
    const uint32_t band = tileIndex / perBand, t = tileIndex % perBand;
    const uint32_t ty = t / s.across, tx = t % s.across;
    const uint32_t row = ty * s.tile + y;
    const float* src = s.bands[band];
    uint8_t* dst = out + (size_t(tileIndex) * s.tile + y) * s.tile * 4;
    auto sample = [&](uint32_t x) -> uint32_t {
        const uint32_t col = tx * s.tile + x;
        const float v = col < s.width && row < s.height ? src[size_t(row) * s.width + col] : s.fill;
        return __float_as_uint(v);
    };
    for (uint32_t x = threadIdx.x; x < s.tile; x += blockDim.x) {
        const uint32_t v = sample(x);
        if (!s.predictor) {
            reinterpret_cast<uint32_t*>(dst)[x] = v;
            continue;
        }
        // Plane p holds byte 3 - p of each sample; the byte before plane p's first is the last
        // sample's byte of plane p - 1.
        const uint32_t before = x > 0 ? sample(x - 1) : sample(s.tile - 1);
        for (uint32_t p = 0; p < 4; ++p) {
            const uint32_t b = (v >> (8 * (3 - p))) & 0xffu;
            uint32_t prev;
            if (x > 0) {
                prev = (before >> (8 * (3 - p))) & 0xffu;
            } else {
                prev = p > 0 ? (before >> (8 * (4 - p))) & 0xffu : 0u;
            }
            dst[size_t(p) * s.tile + x] = uint8_t(b - prev);
        }
    }
}

// --- 2. LZW ------------------------------------------------------------------------------------

constexpr int kClear = 256, kEndOfInfo = 257, kFirstCode = 258, kMaxCode = 4096;
constexpr uint32_t kLzwSlots = 8192;       // open-addressed string table, at most 47 % full
constexpr uint32_t kLzwChunk = 1024;       // bytes staged at a time (a tile is a multiple)
constexpr int kLzwLoads = kLzwChunk / 16 / 32;  // 16-byte loads per lane per chunk

struct LzwTiles {
    const uint8_t* in;     // the predicted tiles, `tileBytes` each
    size_t tileBytes;
    uint32_t tiles;
    uint8_t* out;          // `capacity` bytes per tile
    size_t capacity;
    uint32_t* sizes;       // compressed bytes per tile
    uint32_t* overflow;    // set when a tile would pass its capacity
};

// The MSB-first code writer, in 32-bit words stored big-end first.
struct BitSink {
    uint8_t* out;
    size_t capacity, at;
    uint64_t bits;
    int count;
    bool over;
    __device__ void put(int code, int width) {
        bits = (bits << width) | uint64_t(code);
        count += width;
        if (count >= 32) {
            count -= 32;
            const uint32_t word = uint32_t(bits >> count);
            if (at + 4 <= capacity) {
                *reinterpret_cast<uint32_t*>(out + at) = __byte_perm(word, 0, 0x0123);
            } else {
                over = true;
            }
            at += 4;
        }
    }
    // The last partial byte padded with zeros; the compressed size in bytes.
    __device__ size_t finish() {
        while (count >= 8) {
            count -= 8;
            if (at < capacity) out[at] = uint8_t(bits >> count);
            else over = true;
            ++at;
        }
        if (count > 0) {
            if (at < capacity) out[at] = uint8_t(bits << (8 - count));
            else over = true;
            ++at;
            count = 0;
        }
        return at;
    }
};

__device__ __forceinline__ uint32_t lzw_slot(uint32_t key) {
    return (key * 2654435761u) >> (32 - 13);
}

__device__ __forceinline__ int lzw_next_width(int codes, int width) {
    return codes >= (1 << width) && width < 12 ? width + 1 : width;
}

// One warp per tile (blocks loop over the tiles). Table entries are key << 12 | code (key =
// prefix code << 8 | byte, 20 bits), 0 for an empty slot.
__global__ void __launch_bounds__(32) lzw_kernel(const LzwTiles p) {
    __shared__ uint32_t table[kLzwSlots];
    __shared__ uint4 stage[kLzwChunk / 16];
    const uint32_t lane = threadIdx.x;
    const uint32_t chunks = uint32_t(p.tileBytes / kLzwChunk);
    for (uint32_t tile = blockIdx.x; tile < p.tiles; tile += gridDim.x) {
        const uint4* src = reinterpret_cast<const uint4*>(p.in + size_t(tile) * p.tileBytes);
        for (uint32_t i = lane; i < kLzwSlots; i += 32) {
            table[i] = 0u;
        }
        uint4 ahead[kLzwLoads];
#pragma unroll
        for (int j = 0; j < kLzwLoads; ++j) {
            ahead[j] = src[j * 32 + lane];
        }
        BitSink sink{p.out + size_t(tile) * p.capacity, p.capacity, 0, 0, 0, false};
        int cur = -1, next = kFirstCode, width = 9;
        if (lane == 0) {
            sink.put(kClear, width);
        }
        for (uint32_t c = 0; c < chunks; ++c) {
            __syncwarp();
#pragma unroll
            for (int j = 0; j < kLzwLoads; ++j) {
                stage[j * 32 + lane] = ahead[j];
            }
            if (c + 1 < chunks) {
#pragma unroll
                for (int j = 0; j < kLzwLoads; ++j) {
                    ahead[j] = src[size_t(c + 1) * (kLzwChunk / 16) + j * 32 + lane];
                }
            }
            __syncwarp();
            const uint8_t* bytes = reinterpret_cast<const uint8_t*>(stage);
            uint32_t i = 0;
            while (true) {
                // Lane 0 runs the encoder until the chunk ends or the table must be cleared.
                int clear = 0;
                if (lane == 0) {
                    for (; i < kLzwChunk; ++i) {
                        const int b = bytes[i];
                        if (cur < 0) {
                            cur = b;
                            continue;
                        }
                        const uint32_t key = (uint32_t(cur) << 8) | uint32_t(b);
                        uint32_t slot = lzw_slot(key);
                        uint32_t e;
                        while ((e = table[slot]) != 0u && (e >> 12) != key) {
                            slot = (slot + 1) & (kLzwSlots - 1);
                        }
                        if (e != 0u) {
                            cur = int(e & 0xfffu);
                            continue;
                        }
                        table[slot] = (key << 12) | uint32_t(next);
                        sink.put(cur, width);
                        ++next;
                        width = lzw_next_width(next, width);
                        cur = b;
                        if (next >= kMaxCode - 2) {
                            sink.put(kClear, width);
                            width = 9;
                            next = kFirstCode;
                            clear = 1;
                            ++i;
                            break;
                        }
                    }
                }
                clear = __shfl_sync(0xffffffffu, clear, 0);
                if (!clear) {
                    break;
                }
                __syncwarp();
                for (uint32_t k = lane; k < kLzwSlots; k += 32) {
                    table[k] = 0u;
                }
                __syncwarp();
            }
        }
        if (lane == 0) {
            if (cur >= 0) {
                sink.put(cur, width);
                ++next;
                width = lzw_next_width(next, width);
            }
            sink.put(kEndOfInfo, width);
            const size_t size = sink.finish();
            p.sizes[tile] = uint32_t(std::min<size_t>(size, 0xffffffffu));
            if (sink.over) {
                atomicOr(p.overflow, 1u);
            }
        }
        __syncwarp();
    }
}

// The compressed tiles packed back to back at their offsets in the file's tile stream, each
// followed by a 0 byte when its size is odd.
__global__ void pack_tiles_kernel(const uint8_t* __restrict__ in, size_t capacity,
                                  const uint32_t* __restrict__ sizes,
                                  const uint64_t* __restrict__ offsets, uint32_t tiles,
                                  uint8_t* __restrict__ out) {
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint8_t* src = in + size_t(t) * capacity;
        uint8_t* dst = out + offsets[t];
        const uint32_t n = sizes[t];
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            dst[i] = src[i];
        }
        if ((n & 1u) != 0u && threadIdx.x == 0) {
            dst[n] = 0;
        }
    }
}

}  // namespace

// --- 3. the file -------------------------------------------------------------------------------

namespace {

// TIFF tags and field types written (tiff_format.h).
enum : uint16_t {
    kImageWidth = 256, kImageLength = 257, kBitsPerSample = 258, kCompression = 259,
    kPhotometric = 262, kSamplesPerPixel = 277, kPlanarConfiguration = 284, kPredictor = 317,
    kTileWidth = 322, kTileLength = 323, kTileOffsets = 324, kTileByteCounts = 325,
    kExtraSamples = 338, kSampleFormat = 339, kModelPixelScale = 33550, kModelTiepoint = 33922,
    kModelTransformation = 34264, kGeoKeyDirectory = 34735, kGeoDoubleParams = 34736,
    kGeoAsciiParams = 34737, kGdalNoData = 42113,
};
enum : uint16_t { kAscii = 2, kShort = 3, kLong = 4, kDouble = 12, kLong8 = 16 };
constexpr uint16_t kRasterTypeKey = 1025, kPixelIsPoint = 2;

// An IFD of values inline or after the table (IfdWriter, geotiff_write.cpp:23): entries in tag
// order, each value of more than one word at an even offset after the table.
class Ifd {
  public:
    explicit Ifd(bool big) : countSize_(big ? 8 : 2), word_(big ? 8 : 4) {}

    template <typename T>
    void add(uint16_t tag, uint16_t type, const std::vector<T>& values) {
        Entry e{type, values.size(), std::vector<uint8_t>(values.size() * sizeof(T))};
        if (!values.empty()) {
            std::memcpy(e.bytes.data(), values.data(), e.bytes.size());
        }
        entries_[tag] = std::move(e);
    }

    void ascii(uint16_t tag, const std::string& text) {
        std::vector<uint8_t> bytes(text.begin(), text.end());
        bytes.push_back(0);
        entries_[tag] = Entry{kAscii, bytes.size(), std::move(bytes)};
    }

    std::vector<uint8_t> serialize(uint64_t offset) const {
        const size_t entrySize = 4 + 2 * word_;
        const size_t tableSize = countSize_ + entries_.size() * entrySize + word_;
        std::vector<uint8_t> table(tableSize, 0), extra;
        auto put = [&table](size_t at, uint64_t value, size_t size) {
            std::memcpy(table.data() + at, &value, size);
        };
        put(0, entries_.size(), countSize_);
        size_t at = countSize_;
        for (const auto& [tag, e] : entries_) {
            put(at, tag, 2);
            put(at + 2, e.type, 2);
            put(at + 4, e.count, word_);
            const size_t valueAt = at + 4 + word_;
            if (e.bytes.size() <= word_) {
                std::memcpy(table.data() + valueAt, e.bytes.data(), e.bytes.size());
            } else {
                if (extra.size() % 2 != 0) {
                    extra.push_back(0);
                }
                put(valueAt, offset + tableSize + extra.size(), word_);
                extra.insert(extra.end(), e.bytes.begin(), e.bytes.end());
            }
            at += entrySize;
        }
        table.insert(table.end(), extra.begin(), extra.end());
        return table;
    }

  private:
    struct Entry {
        uint16_t type = 0;
        uint64_t count = 0;
        std::vector<uint8_t> bytes;
    };
    size_t countSize_, word_;
    std::map<uint16_t, Entry> entries_;
};

// GTRasterTypeGeoKey is PixelIsPoint (ShortGeoKey, geotiff.cpp:52).
bool pixel_is_point(const tg_geokeys* keys) {
    if (keys == nullptr || keys->directory == nullptr || keys->directory_count < 4) {
        return false;
    }
    const uint16_t* d = keys->directory;
    const size_t count = d[3];
    for (size_t k = 0; k < count && 4 + 4 * k + 3 < keys->directory_count; ++k) {
        const size_t at = 4 + 4 * k;
        if (d[at] == kRasterTypeKey && d[at + 1] == 0) {
            return d[at + 3] == kPixelIsPoint;
        }
    }
    return false;
}

// The image, sample and tile tags (AddImageTags, geotiff_write.cpp:190) and the georeferencing,
// keys and no-data (AddGeoTags, geotiff_write.cpp:229).
void add_tags(Ifd& ifd, const tg_grid& g, uint32_t bands, uint32_t compression, uint32_t tile,
              const std::vector<uint64_t>& offsets, const std::vector<uint64_t>& counts,
              bool big, const tg_geokeys* keys, const tg_nodata& nodata) {
    const auto nb = uint16_t(bands);
    ifd.add<uint32_t>(kImageWidth, kLong, {g.width});
    ifd.add<uint32_t>(kImageLength, kLong, {g.height});
    ifd.add<uint16_t>(kBitsPerSample, kShort, std::vector<uint16_t>(nb, 32));
    const uint16_t code = compression == kLzw ? 5 : compression == kDeflate ? 8 : 1;
    ifd.add<uint16_t>(kCompression, kShort, {code});
    ifd.add<uint16_t>(kPhotometric, kShort, {1});
    ifd.add<uint16_t>(kSamplesPerPixel, kShort, {nb});
    ifd.add<uint16_t>(kPlanarConfiguration, kShort, {uint16_t(nb == 1 ? 1 : 2)});
    if (compression != kNone) {
        ifd.add<uint16_t>(kPredictor, kShort, {3});
    }
    ifd.add<uint32_t>(kTileWidth, kLong, {tile});
    ifd.add<uint32_t>(kTileLength, kLong, {tile});
    if (big) {
        ifd.add<uint64_t>(kTileOffsets, kLong8, offsets);
        ifd.add<uint64_t>(kTileByteCounts, kLong8, counts);
    } else {
        ifd.add<uint32_t>(kTileOffsets, kLong,
                          std::vector<uint32_t>(offsets.begin(), offsets.end()));
        ifd.add<uint32_t>(kTileByteCounts, kLong,
                          std::vector<uint32_t>(counts.begin(), counts.end()));
    }
    if (nb > 1) {
        ifd.add<uint16_t>(kExtraSamples, kShort, std::vector<uint16_t>(nb - 1u, 0));
    }
    ifd.add<uint16_t>(kSampleFormat, kShort, std::vector<uint16_t>(nb, 3));
    const bool hasKeys = keys != nullptr && keys->directory_count > 0;
    const bool identity = g.origin_x == 0.0 && g.pixel_width == 1.0 && g.row_rotation == 0.0 &&
                          g.origin_y == 0.0 && g.col_rotation == 0.0 && g.pixel_height == 1.0;
    if (hasKeys || !identity) {
        // EncodeTransform (tiff_format.cpp:73): PixelIsPoint stores the transform half a pixel on.
        double ox = g.origin_x, oy = g.origin_y;
        if (pixel_is_point(keys)) {
            ox += 0.5 * (g.pixel_width + g.row_rotation);
            oy += 0.5 * (g.col_rotation + g.pixel_height);
        }
        if (g.row_rotation == 0.0 && g.col_rotation == 0.0) {
            ifd.add<double>(kModelPixelScale, kDouble, {g.pixel_width, -g.pixel_height, 0.0});
            ifd.add<double>(kModelTiepoint, kDouble, {0.0, 0.0, 0.0, ox, oy, 0.0});
        } else {
            ifd.add<double>(kModelTransformation, kDouble,
                            {g.pixel_width, g.row_rotation, 0.0, ox, g.col_rotation,
                             g.pixel_height, 0.0, oy, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0});
        }
    }
    if (hasKeys) {
        ifd.add<uint16_t>(kGeoKeyDirectory, kShort,
                          std::vector<uint16_t>(keys->directory,
                                                keys->directory + keys->directory_count));
        if (keys->double_count > 0 && keys->double_params != nullptr) {
            ifd.add<double>(kGeoDoubleParams, kDouble,
                            std::vector<double>(keys->double_params,
                                                keys->double_params + keys->double_count));
        }
        if (keys->ascii_params != nullptr && keys->ascii_params[0] != '\0') {
            ifd.ascii(kGeoAsciiParams, keys->ascii_params);
        }
    }
    if (nodata.mode != 0u) {
        const double v = nodata.mode == 1u ? double(std::numeric_limits<float>::quiet_NaN())
                                           : double(nodata.value);
        char text[40];
        std::snprintf(text, sizeof(text), "%.*g", 9, v);  // FormatNumber(value, 9)
        ifd.ascii(kGdalNoData, text);
    }
}

// A device allocation freed with its scope.
struct DeviceBytes {
    void* ptr = nullptr;
    DeviceBytes() = default;
    DeviceBytes(const DeviceBytes&) = delete;
    DeviceBytes& operator=(const DeviceBytes&) = delete;
    ~DeviceBytes() {
        if (ptr != nullptr) {
            cudaFree(ptr);
        }
    }
    cudaError_t allocate(size_t bytes) {
        return cudaMalloc(&ptr, std::max<size_t>(bytes, 16));
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
};

}  // namespace

extern "C" {

int tg_geotiff_write(tg_device* d, const char* path, const float* const* bands,
                     uint32_t band_count, const tg_grid* grid, tg_nodata nodata,
                     const tg_geokeys* keys, const tg_geotiff_options* options, int memory,
                     void* stream) {
    if (int st = check_device(d)) {
        return st;
    }
    std::lock_guard<std::mutex> lock(d->mutex);
    if (int st = check_memory(memory)) {
        return st;
    }
    if (path == nullptr || bands == nullptr || grid == nullptr || options == nullptr) {
        return fail(TG_ERROR_ARGUMENT, "path, bands, grid and options are required");
    }
    const tg_grid& g = *grid;
    if (band_count == 0 || g.width == 0 || g.height == 0) {
        return fail(TG_ERROR_ARGUMENT, "cannot write an empty raster");
    }
    if (band_count > 65535u) {
        return fail(TG_ERROR_ARGUMENT, "a GeoTIFF holds at most 65535 bands");
    }
    const uint32_t compression = options->compression;
    if (compression == kPackBits) {
        return fail(TG_ERROR_ARGUMENT, "writing PackBits is not supported; use None, Lzw or "
                                       "Deflate");
    }
    if (compression != kNone && compression != kLzw && compression != kDeflate) {
        return fail(TG_ERROR_ARGUMENT, "compression must be 0 (none), 1 (LZW) or 3 (Deflate)");
    }
    const uint32_t tile = options->tile_size;
    if (tile == 0 || tile % 16 != 0) {
        return fail(TG_ERROR_ARGUMENT, "the tile size must be a positive multiple of 16");
    }
    if (nodata.mode > 2u) {
        return fail(TG_ERROR_ARGUMENT, "nodata mode must be 0, 1 or 2");
    }
    for (uint32_t b = 0; b < band_count; ++b) {
        if (bands[b] == nullptr) {
            return fail(TG_ERROR_ARGUMENT, "band %u is null", b);
        }
    }
    const uint32_t across = (g.width + tile - 1) / tile, down = (g.height + tile - 1) / tile;
    const uint64_t total = uint64_t(across) * down * band_count;
    const size_t tileBytes = size_t(tile) * tile * 4;
    if (total * tile >= 0x7fffffffull || total >= 0xffffffffull) {
        return fail(TG_ERROR_UNSUPPORTED, "too many tiles; use a larger tile size");
    }
    // NeedsBigTiff (geotiff_write.cpp:117): uncompressed tiles that could pass 4 GiB.
    const bool big = options->big_tiff != 0u ||
                     total * tileBytes + (uint64_t(1) << 20) >= (uint64_t(1) << 32);
    const uint64_t start = big ? 16 : 8;  // the header, the first IFD's offset at its end
    const cudaStream_t s = memory == TG_MEMORY_DEVICE && stream != nullptr
                               ? static_cast<cudaStream_t>(stream)
                               : d->stream;
    const size_t cells = size_t(g.width) * g.height;
    // The bands on the device.
    std::vector<DeviceBytes> copies(memory == TG_MEMORY_HOST ? band_count : 0);
    std::vector<const float*> devBands(band_count);
    for (uint32_t b = 0; b < band_count; ++b) {
        if (memory == TG_MEMORY_HOST) {
            TG_CUDA(copies[b].allocate(cells * 4), "allocation");
            TG_CUDA(cudaMemcpyAsync(copies[b].ptr, bands[b], cells * 4, cudaMemcpyHostToDevice,
                                    s),
                    "copy");
            devBands[b] = copies[b].as<const float>();
        } else {
            devBands[b] = bands[b];
        }
    }
    DeviceBytes bandTable, tiles;
    TG_CUDA(bandTable.allocate(band_count * sizeof(float*)), "allocation");
    TG_CUDA(cudaMemcpyAsync(bandTable.ptr, devBands.data(), band_count * sizeof(float*),
                            cudaMemcpyHostToDevice, s),
            "copy");
    TG_CUDA(tiles.allocate(total * tileBytes), "allocation");
    const float fill = nodata.mode == 1u   ? std::numeric_limits<float>::quiet_NaN()
                       : nodata.mode == 2u ? nodata.value
                                           : 0.0f;
    TileSource src{bandTable.as<const float* const>(), g.width, g.height, tile, across, down,
                   fill, compression != kNone};
    tiles_kernel<<<uint32_t(total * tile), std::min<uint32_t>(tile, 256), 0, s>>>(
        src, tiles.as<uint8_t>());
    TG_CUDA(cudaGetLastError(), "tiles launch");
    // The tile stream from `start`: each tile at an even offset (WriteTiles,
    // geotiff_write.cpp:145).
    std::vector<uint64_t> offsets(total), counts(total);
    std::vector<uint8_t> stream_;
    if (compression == kNone) {
        stream_.resize(total * tileBytes);
        TG_CUDA(cudaMemcpyAsync(stream_.data(), tiles.ptr, stream_.size(), cudaMemcpyDeviceToHost,
                                s),
                "copy to host");
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");
        for (uint64_t t = 0; t < total; ++t) {
            offsets[t] = start + t * tileBytes;
            counts[t] = tileBytes;
        }
    } else if (compression == kLzw) {
        // At most one 12-bit code per byte, a Clear every 3836 codes, Clear and EndOfInfo.
        const size_t capacity = (tileBytes + tileBytes / 2 + 64 + 15) / 16 * 16;
        DeviceBytes coded, sizes, flag, devOffsets;
        TG_CUDA(coded.allocate(total * capacity), "allocation");
        TG_CUDA(sizes.allocate(total * 4), "allocation");
        TG_CUDA(flag.allocate(4), "allocation");
        TG_CUDA(cudaMemsetAsync(flag.ptr, 0, 4, s), "memset");
        int sms = 0, perSm = 0;
        TG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->ordinal),
                "attribute");
        TG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, lzw_kernel, 32, 0),
                "occupancy");
        LzwTiles lz{tiles.as<const uint8_t>(), tileBytes, uint32_t(total), coded.as<uint8_t>(),
                    capacity, sizes.as<uint32_t>(), flag.as<uint32_t>()};
        const uint64_t blocks = std::min<uint64_t>(total, uint64_t(std::max(perSm, 1)) * sms);
        lzw_kernel<<<uint32_t(blocks), 32, 0, s>>>(lz);
        TG_CUDA(cudaGetLastError(), "lzw launch");
        std::vector<uint32_t> sz(total);
        uint32_t over = 0;
        TG_CUDA(cudaMemcpyAsync(sz.data(), sizes.ptr, total * 4, cudaMemcpyDeviceToHost, s),
                "copy to host");
        TG_CUDA(cudaMemcpyAsync(&over, flag.ptr, 4, cudaMemcpyDeviceToHost, s), "copy to host");
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");
        if (over != 0u) {
            return fail(TG_ERROR_CUDA, "an LZW tile passed its capacity");
        }
        std::vector<uint64_t> local(total);
        uint64_t at = 0;
        for (uint64_t t = 0; t < total; ++t) {
            local[t] = at;
            offsets[t] = start + at;
            counts[t] = sz[t];
            at += sz[t] + (sz[t] & 1u);
        }
        DeviceBytes packed;
        TG_CUDA(devOffsets.allocate(total * 8), "allocation");
        TG_CUDA(packed.allocate(at), "allocation");
        TG_CUDA(cudaMemcpyAsync(devOffsets.ptr, local.data(), total * 8, cudaMemcpyHostToDevice, s),
                "copy");
        pack_tiles_kernel<<<uint32_t(std::min<uint64_t>(total, 65535)), 256, 0, s>>>(
            coded.as<const uint8_t>(), capacity, sizes.as<const uint32_t>(),
            devOffsets.as<const uint64_t>(), uint32_t(total), packed.as<uint8_t>());
        TG_CUDA(cudaGetLastError(), "pack launch");
        stream_.resize(at);
        TG_CUDA(cudaMemcpyAsync(stream_.data(), packed.ptr, at, cudaMemcpyDeviceToHost, s),
                "copy to host");
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");
    } else {
        // Deflate on host threads, from the predicted tiles.
        std::vector<uint8_t> raw(total * tileBytes);
        TG_CUDA(cudaMemcpyAsync(raw.data(), tiles.ptr, raw.size(), cudaMemcpyDeviceToHost, s),
                "copy to host");
        TG_CUDA(cudaStreamSynchronize(s), "synchronize");
        std::vector<std::vector<uint8_t>> coded(total);
        std::vector<int> status(total, Z_OK);
        const unsigned threads = std::max(1u, std::min(std::thread::hardware_concurrency(), 64u));
        std::vector<std::thread> pool;
        for (unsigned w = 0; w < threads; ++w) {
            pool.emplace_back([&, w]() {
                for (uint64_t t = w; t < total; t += threads) {
                    uLongf n = compressBound(uLong(tileBytes));
                    coded[t].resize(n);
                    status[t] = compress2(coded[t].data(), &n, raw.data() + t * tileBytes,
                                          uLong(tileBytes), 6);
                    coded[t].resize(n);
                }
            });
        }
        for (std::thread& th : pool) {
            th.join();
        }
        uint64_t at = 0;
        for (uint64_t t = 0; t < total; ++t) {
            if (status[t] != Z_OK) {
                return fail(TG_ERROR_CUDA, "Deflate compression failed");
            }
            offsets[t] = start + at;
            counts[t] = coded[t].size();
            at += coded[t].size() + (coded[t].size() & 1u);
        }
        stream_.resize(at, 0);
        for (uint64_t t = 0; t < total; ++t) {
            std::memcpy(stream_.data() + (offsets[t] - start), coded[t].data(), coded[t].size());
        }
    }
    const uint64_t end = start + stream_.size();
    if (!big && end >= (uint64_t(1) << 32) - (uint64_t(1) << 20)) {
        return fail(TG_ERROR_ARGUMENT, "data too large for classic TIFF; set big_tiff");
    }
    Ifd ifd(big);
    add_tags(ifd, g, band_count, compression, tile, offsets, counts, big, keys, nodata);
    const std::vector<uint8_t> table = ifd.serialize(end);
    // The header (WriteHeader, geotiff_write.cpp:176) with the IFD's offset.
    std::vector<uint8_t> header = {'I', 'I', uint8_t(big ? 43 : 42), 0};
    if (big) {
        header.insert(header.end(), {8, 0, 0, 0});
    }
    const size_t word = big ? 8 : 4;
    header.resize(header.size() + word, 0);
    std::memcpy(header.data() + header.size() - word, &end, word);
    std::ofstream file(path, std::ios::binary);
    if (!file) {
        return fail(TG_ERROR_ARGUMENT, "cannot open %s for writing", path);
    }
    file.write(reinterpret_cast<const char*>(header.data()), std::streamsize(header.size()));
    file.write(reinterpret_cast<const char*>(stream_.data()), std::streamsize(stream_.size()));
    file.write(reinterpret_cast<const char*>(table.data()), std::streamsize(table.size()));
    if (!file) {
        return fail(TG_ERROR_ARGUMENT, "write error on %s", path);
    }
    return TG_OK;
}

}  // extern "C"
