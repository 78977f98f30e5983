// meshtrex's main sequence (src/meshtrex.cpp:100-141) through the C++ facade:
// loadVolume -> computeMinMaxMip -> filterActiveBlocks -> readActiveBlockCount
// -> extractMeshletDescriptors (-> writeGPUExtractionToOBJ), then one JSON line
// with the counts and FNV-1a hashes of the vertex and index bytes.
//
//   drop_in_main <name>_<X>x<Y>x<Z>_<type>.raw <block edge> <isovalue> [out.obj]
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "meshtrex/meshtrex.hpp"

static unsigned long long fnv1a(const std::vector<uint8_t> &b) {
    unsigned long long h = 1469598103934665603ull;
    for (uint8_t c : b) h = (h ^ c) * 1099511628211ull;
    return h;
}

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <name>_<X>x<Y>x<Z>_<type>.raw <block edge> <isovalue> [out.obj]\n", argv[0]);
        return 2;
    }
    try {
        meshtrex::Context context(0);
        meshtrex::GPUProfiler profiler(context);
        meshtrex::Volume volume = meshtrex::loadVolume(argv[1]);
        meshtrex::PushConstants pc =
            meshtrex::makePushConstants(volume.volume_dims, (uint32_t)std::atoi(argv[2]), (float)std::atof(argv[3]));
        profiler.beginFrame();
        meshtrex::MinMaxOutput mm = meshtrex::computeMinMaxMip(context, volume, pc, nullptr, &profiler);
        meshtrex::FilteringOutput f = meshtrex::filterActiveBlocks(context, mm, pc, nullptr, &profiler);
        meshtrex::readActiveBlockCount(context, f);
        meshtrex::ExtractionOutput x = meshtrex::extractMeshletDescriptors(context, mm, f, pc, nullptr, &profiler);
        context.synchronize();
        profiler.endFrame();
        std::vector<uint8_t> vb(x.vertexBuffer.size), ib(x.indexBuffer.size);
        meshtrex::check(mtx_read_buffer(context.handle(), &x.raw.vertexBuffer, 0, vb.data(), vb.size()),
                        context.handle(), "read vertices");
        meshtrex::check(mtx_read_buffer(context.handle(), &x.raw.indexBuffer, 0, ib.data(), ib.size()),
                        context.handle(), "read indices");
        mtx_obj_stats st{};
        if (argc > 4) st = meshtrex::writeGPUExtractionToOBJ(context, x, argv[4]);
        std::printf(
            "{\"activeBlocks\": %u, \"meshlets\": %u, \"vertices\": %u, \"indices\": %u, \"mipLevels\": %u, "
            "\"vertexHash\": \"%016llx\", \"indexHash\": \"%016llx\", \"uniqueVertices\": %u, "
            "\"degenerateTriangles\": %u, \"leafMs\": %.5f}\n",
            f.activeBlockCount, x.meshletCount, x.vertexCount, x.indexCount, mm.mipLevels, fnv1a(vb), fnv1a(ib),
            st.uniqueVertexCount, st.degenerateTriangleCount, profiler.lastMs("MinMax_Leaf_Pass"));
    } catch (const meshtrex::Error &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
