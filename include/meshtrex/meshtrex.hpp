// The C++ drop-in facade: meshtrex's manager functions and output structs under
// their own names, over the C ABI of meshtrex/mtx.h.
//
//   meshtrex::Context context;
//   meshtrex::Volume volume = meshtrex::loadVolume(path);
//   meshtrex::PushConstants pc = meshtrex::makePushConstants(volume.volume_dims, 8, iso);
//   auto mm = meshtrex::computeMinMaxMip(context, volume, pc);
//   auto f = meshtrex::filterActiveBlocks(context, mm, pc);
//   meshtrex::readActiveBlockCount(context, f);
//   auto x = meshtrex::extractMeshletDescriptors(context, mm, f, pc);
#pragma once

#include "meshtrex/context.h"
#include "meshtrex/extractionManager.h"
#include "meshtrex/extractionOutput.h"
#include "meshtrex/filteringManager.h"
#include "meshtrex/filteringOutput.h"
#include "meshtrex/minMaxManager.h"
#include "meshtrex/minMaxOutput.h"
#include "meshtrex/volume.h"
