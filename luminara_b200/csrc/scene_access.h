// scene_access.h -- internal hooks for entry points defined outside host.cpp.
#pragma once

#include <cuda_runtime.h>

#include "../../include/luminara_gpu.h"
#include "device_scene.h"

namespace lum {

// Sets lum_last_error() for the calling thread; returns code.
lum_status set_error(lum_status code, const char* msg);

// Validates params, makes the scene's device current and returns its device view, the
// launch description of the render and the scene's stream.
lum_status prepare_render(lum_scene* s, const lum_render_params* params, SceneDev& dev, RenderDev& R,
                          cudaStream_t& stream);

// Device view, owning device ordinal and render description of a scene for `params`
// (validated), without touching the scene's stream.
lum_status scene_view(lum_scene* s, const lum_render_params* params, SceneDev& dev, RenderDev& R, int& device);
// Largest LUM_MAT_* kind among the scene's materials (0 when it has none).
int scene_max_material_kind(const lum_scene* s);

}  // namespace lum
