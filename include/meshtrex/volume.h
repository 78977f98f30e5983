// Volume and loadVolume of the C++ drop-in facade (meshtrex: src/volume.h:8-43),
// and the PushConstants of src/common.h:29-34 as meshtrex's main fills them
// (src/meshtrex.cpp:76-84).
#pragma once

#include <cstdint>
#include <fstream>
#include <string>
#include <vector>

#include "meshtrex/context.h"

namespace meshtrex {

struct uvec3 {
    uint32_t x = 0, y = 0, z = 0;
};

// Host voxels, x fastest.  volume_type is "uint8", "uint16" or "float32".
struct Volume {
    uvec3 volume_dims;
    std::string volume_type;
    std::vector<uint8_t> volume_data;
};

inline uint32_t volumeDtype(const std::string &type) {
    if (type == "uint8") return MTX_DTYPE_U8;
    if (type == "uint16") return MTX_DTYPE_U16;
    if (type == "float32" || type == "float") return MTX_DTYPE_F32;
    throw Error(MTX_ERR_UNSUPPORTED, "unsupported volume type " + type);
}

// Reads "<name>_<X>x<Y>x<Z>_<type>.raw" into host memory.  meshtrex treats
// every type other than uint8 as 16-bit and prints (does not throw) on a
// short file; here float32 is a type of its own and a short or missing file
// throws.  mtx_volume_load streams such a file straight to the device.
inline Volume loadVolume(const char *path) {
    uint32_t dims[3], dtype;
    check(mtx_parse_volume_name(path, dims, &dtype), nullptr, "loadVolume: unrecognized raw volume naming scheme");
    Volume v;
    v.volume_dims = {dims[0], dims[1], dims[2]};
    v.volume_type = dtype == MTX_DTYPE_U8 ? "uint8" : dtype == MTX_DTYPE_U16 ? "uint16" : "float32";
    const size_t esz = dtype == MTX_DTYPE_U8 ? 1 : dtype == MTX_DTYPE_U16 ? 2 : 4;
    v.volume_data.resize((size_t)dims[0] * dims[1] * dims[2] * esz);
    std::ifstream in(path, std::ios::binary);
    if (!in || !in.read(reinterpret_cast<char *>(v.volume_data.data()), (std::streamsize)v.volume_data.size()))
        throw Error(MTX_ERR_INVALID_ARG, std::string("loadVolume: cannot read ") + path);
    return v;
}

using PushConstants = mtx_push_constants;

inline PushConstants makePushConstants(const uvec3 &dims, uint32_t blockEdge, float isovalue) {
    PushConstants pc;
    const uint32_t d[3] = {dims.x, dims.y, dims.z};
    check(mtx_push_constants_init(d, blockEdge, isovalue, &pc), nullptr, "mtx_push_constants_init");
    return pc;
}

}  // namespace meshtrex
