// The wavefront kernels of the fast math mode, compiled apart from the other mode so that the
// two build in parallel.
#include "pg_launch.cuh"

namespace pg {

cudaError_t ConfigureKernelsFast() {
    return ConfigureKernelsM<kFast>();
}

void DispatchRegenFast(const LaunchEnv& env, Wave& w, LaunchTimer* timer, RenderResult* res) {
    DispatchRegenM<kFast>(env, w, timer, res);
}

void DispatchBodyFast(const LaunchEnv& env, Wave& w, int n, bool persistent, LaunchTimer* timer,
                      RenderResult* res) {
    DispatchBodyM<kFast>(env, w, n, persistent, timer, res);
}

}  // namespace pg
