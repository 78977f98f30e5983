// The no-allocation compaction entry point (mtx_filter_active_blocks_noalloc)
// in more than one CUDA context.  Its scratch array has one device address
// per context, so the program calls it in the device's primary context, then
// in a second context made with the driver API on the same device (device
// memory of one context is not mapped in the other), then in the primary
// context again.  All device memory here comes from the driver API; the
// entry point itself allocates nothing.  Each call compacts the same
// {min,max} keys; the program prints one JSON line with each call's status,
// active count and FNV-1a hashes of the id list and the rank map.
//
//   noalloc_contexts <keys.bin> <dtype> <isovalue>
#include <cuda.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "meshtrex/mtx.h"

static unsigned long long fnv1a(const void *p, size_t n) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    unsigned long long h = 1469598103934665603ull;
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

#define CU(x)                                                             \
    do {                                                                  \
        CUresult r_ = (x);                                                \
        if (r_ != CUDA_SUCCESS) {                                         \
            std::fprintf(stderr, "%s failed: %d\n", #x, (int)r_);         \
            std::exit(3);                                                 \
        }                                                                 \
    } while (0)

struct Result {
    int status;
    uint32_t count;
    uint32_t device_status;
    unsigned long long ids_hash;
    unsigned long long rank_hash;
};

// One call in the current context: copy the keys in, compact, copy back.
static Result run_once(const std::vector<uint32_t> &keys, uint32_t dtype, float iso) {
    const uint64_t nblocks = keys.size() / 2;
    CUdeviceptr d_keys, d_ids, d_rank, d_count, d_status;
    CU(cuMemAlloc(&d_keys, keys.size() * 4));
    CU(cuMemAlloc(&d_ids, nblocks * 4));
    CU(cuMemAlloc(&d_rank, nblocks * 4));
    CU(cuMemAlloc(&d_count, 4));
    CU(cuMemAlloc(&d_status, 16));
    CU(cuMemcpyHtoD(d_keys, keys.data(), keys.size() * 4));
    CU(cuMemsetD32(d_ids, 0xdeadbeefu, nblocks));
    Result r{};
    r.status = (int)mtx_filter_active_blocks_noalloc(
        reinterpret_cast<const uint32_t *>(d_keys), nblocks, dtype, iso, reinterpret_cast<uint32_t *>(d_ids),
        reinterpret_cast<uint32_t *>(d_rank), reinterpret_cast<uint32_t *>(d_count),
        reinterpret_cast<uint32_t *>(d_status), nullptr);
    CU(cuCtxSynchronize());
    if (r.status == MTX_OK) {
        uint32_t st[4];
        CU(cuMemcpyDtoH(&r.count, d_count, 4));
        CU(cuMemcpyDtoH(st, d_status, 16));
        r.device_status = st[0];
        std::vector<uint32_t> ids(r.count <= nblocks ? r.count : 0), rank(nblocks);
        if (!ids.empty()) CU(cuMemcpyDtoH(ids.data(), d_ids, ids.size() * 4));
        CU(cuMemcpyDtoH(rank.data(), d_rank, nblocks * 4));
        r.ids_hash = fnv1a(ids.data(), ids.size() * 4);
        r.rank_hash = fnv1a(rank.data(), rank.size() * 4);
    }
    CU(cuMemFree(d_keys));
    CU(cuMemFree(d_ids));
    CU(cuMemFree(d_rank));
    CU(cuMemFree(d_count));
    CU(cuMemFree(d_status));
    return r;
}

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <keys.bin> <dtype> <isovalue>\n", argv[0]);
        return 2;
    }
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    std::vector<uint32_t> keys;
    uint32_t w;
    while (std::fread(&w, 4, 1, f) == 1) keys.push_back(w);
    std::fclose(f);
    const uint32_t dtype = (uint32_t)std::atoi(argv[2]);
    const float iso = (float)std::atof(argv[3]);

    CU(cuInit(0));
    CUdevice dev;
    CU(cuDeviceGet(&dev, 0));
    CUcontext primary, second;
    CU(cuDevicePrimaryCtxRetain(&primary, dev));
    CU(cuCtxSetCurrent(primary));
    Result a = run_once(keys, dtype, iso);
    CU(cuCtxCreate(&second, 0, dev));  // made current by cuCtxCreate
    Result b = run_once(keys, dtype, iso);
    CU(cuCtxDestroy(second));
    CU(cuCtxSetCurrent(primary));
    Result c = run_once(keys, dtype, iso);
    CU(cuDevicePrimaryCtxRelease(dev));

    std::string out = "{\"calls\": [";
    const Result *rs[3] = {&a, &b, &c};
    for (int i = 0; i < 3; ++i) {
        char buf[256];
        std::snprintf(buf, sizeof buf,
                      "%s{\"status\": %d, \"count\": %u, \"device_status\": %u, \"ids\": \"%016llx\", "
                      "\"rank\": \"%016llx\"}",
                      i ? ", " : "", rs[i]->status, rs[i]->count, rs[i]->device_status, rs[i]->ids_hash,
                      rs[i]->rank_hash);
        out += buf;
    }
    out += "]}";
    std::printf("%s\n", out.c_str());
    return 0;
}
