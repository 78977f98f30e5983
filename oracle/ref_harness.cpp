// Reference harness -- TEST INFRASTRUCTURE ONLY.
//
// Runs meshtrex's own CPU code for the parts of the path that compile on
// their own, so the oracle can be pinned against the reference itself:
//   computeMinMaxFromFile + computeActiveBlockCountCPU (src/testMinMax.h:28-242)
//   MarchingCubes::triTable / edgeTable               (src/mc_tables.h:17-308)
// The reference headers are included from the read-only reference tree at
// build time (oracle/Makefile, target "ref"); nothing of them is copied here.
//
//   ref_harness minmax <volume_256x256x256_uint8.raw> <out.bin>
//       out.bin = uint32 {min,max} per 4^3 block (64^3 blocks, x fastest)
//   ref_harness count  <volume.raw> <iso>       prints the active-block count
//   ref_harness tables <out.bin>
//       out.bin = int32 triTable[256][16] then int32 edgeTable[256]
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "testMinMax.h"
#include "mc_tables.h"

static int usage() {
    std::fprintf(stderr, "usage: ref_harness minmax <raw> <out> | count <raw> <iso> | tables <out>\n");
    return 2;
}

int main(int argc, char **argv) {
    if (argc < 3) return usage();
    std::string cmd = argv[1];
    // the reference narrates on stdout; keep our own output on stdout clean
    std::stringstream sink;
    std::streambuf *old = std::cout.rdbuf(sink.rdbuf());
    int rc = 0;
    try {
        if (cmd == "minmax" && argc == 4) {
            std::vector<MinMaxResult> r = computeMinMaxFromFile(argv[2]);
            std::FILE *f = std::fopen(argv[3], "wb");
            if (!f) throw std::runtime_error("cannot open output");
            std::fwrite(r.data(), sizeof(MinMaxResult), r.size(), f);
            std::fclose(f);
        } else if (cmd == "count" && argc == 4) {
            std::vector<MinMaxResult> r = computeMinMaxFromFile(argv[2]);
            uint32_t n = computeActiveBlockCountCPU(r, std::strtof(argv[3], nullptr));
            std::cout.rdbuf(old);
            std::printf("%u\n", n);
            return 0;
        } else if (cmd == "tables" && argc == 3) {
            std::FILE *f = std::fopen(argv[2], "wb");
            if (!f) throw std::runtime_error("cannot open output");
            std::fwrite(MarchingCubes::triTable, sizeof(int), 256 * 16, f);
            std::fwrite(MarchingCubes::edgeTable, sizeof(int), 256, f);
            std::fclose(f);
        } else {
            rc = usage();
        }
    } catch (const std::exception &e) {
        std::cout.rdbuf(old);
        std::fprintf(stderr, "ref_harness: %s\n", e.what());
        return 1;
    }
    std::cout.rdbuf(old);
    return rc;
}
