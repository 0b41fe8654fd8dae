// fyzz::WorldBackend over the B200 C ABI (include/fyzz_b200.h).
//
// The reference SDK's World owns one WorldBackend (include/fyzzxyzzy/
// world.h:226-394, World(std::unique_ptr<WorldBackend>) at world.h:400) and
// validates every argument before forwarding it (src/world.cpp:25-69).  This
// backend forwards each member the B200 step implements to its C-ABI entry
// point and maps the status codes back to the reference's exception types
// (1 invalid_argument, 2 logic_error, 3 overflow_error, 4 runtime_error).
// Members outside the B200 step (static boxes and spheres, aggregates, scene
// queries, shape detaching and flags, forces, per-body dynamics) keep the
// base class's explicit std::logic_error rejection, as the reference asks
// of additional backends.
//
// Build: compile this file inside the reference SDK's build (it includes
// fyzzxyzzy/world.h and fyzzxyzzy/convex.h) and link libfyzz_b200.so.
#pragma once

#include "fyzzxyzzy/world.h"

#include <memory>

namespace fyzz {

// A backend on CUDA device `device`; options.contact_notifications is
// honoured, the other WorldOptions fields select reference behaviour the
// B200 step always has (PCM manifolds) or does not model.
std::unique_ptr<WorldBackend> create_b200_world_backend(int device = 0, WorldOptions options = {});

// World{create_b200_world_backend(device, options)}: the counterpart of
// create_native_gpu_world (include/fyzzxyzzy/native_gpu_world.h:90-138).
World create_b200_world(int device = 0, WorldOptions options = {});

}  // namespace fyzz
