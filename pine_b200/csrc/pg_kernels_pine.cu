// The wavefront kernels of the pine math mode, compiled apart from the other mode so that the
// two build in parallel.
#include "pg_launch.cuh"

namespace pg {

cudaError_t ConfigureKernelsPine() {
    return ConfigureKernelsM<kPine>();
}

void DispatchRegenPine(const LaunchEnv& env, Wave& w, LaunchTimer* timer, RenderResult* res) {
    DispatchRegenM<kPine>(env, w, timer, res);
}

void DispatchBodyPine(const LaunchEnv& env, Wave& w, int n, bool persistent, LaunchTimer* timer,
                      RenderResult* res) {
    DispatchBodyM<kPine>(env, w, n, persistent, timer, res);
}

}  // namespace pg
