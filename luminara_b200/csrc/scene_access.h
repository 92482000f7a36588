// scene_access.h -- internal hooks for entry points defined outside host.cpp.
#pragma once

#include <cuda_runtime.h>

#include <mutex>

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
// The mutex that serialises calls on one scene handle (held by every entry point that reads
// the scene's device buffers).
std::mutex& scene_mutex(lum_scene* s);
// Looks up the allocation-free render's device array on the current device (kernels.cu), so
// that the module holding it is loaded while the caller can still allocate.  Best effort: a
// failure is reported by lum_render_noalloc itself.
void noalloc_preload();

}  // namespace lum
