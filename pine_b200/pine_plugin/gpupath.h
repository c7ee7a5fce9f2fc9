// GpuPathIntegrator: the B200 path tracer as one of pine's integrators.  Added to pine's
// sources with one line in CreateIntegrator (src/core/integrator.cpp:20-37),
//     CASE("GpuPath") return new GpuPathIntegrator(params, scene);
// it is selected by a scene file's `Integrator: GpuPath{ ... }` and rendered by pine's own
// command line, `pine scene.txt` (src/cli/main.cpp:6-29).
//
// It derives from pine's Integrator (src/core/integrator.h:15-30), not RayIntegrator, so pine
// builds no BVH of its own (RayIntegrator's constructor runs accel->Initialize,
// integrator.cpp:52-56).  Render() loads the scene file into libpinegpu, whose loader
// restates pine's grammar and factories, renders it and hands the per-pixel means to pine's
// Film, which writes its image as for any other integrator (tonemap, gamma, BMP).
//
// Parameters (besides the Path integrator's maxDepth, sampler{samplesPerPixel} and
// lightSampler, which the library reads from the scene file):
//   mathMode: pine | fast   pine's pstd numerics on the device, or CUDA's (default fast)
//   seed: int               random stream key (default 0)
//   device: int             CUDA device (default 0)
//   linearFile: name        also write the linear film (mean, variance, sample count) to
//                           this file in the scene's directory (see WriteLinearFilm)
#ifndef PINE_B200_GPUPATH_H
#define PINE_B200_GPUPATH_H

#include <core/integrator.h>

#include <pine_gpu.h>

namespace pine {

class GpuPathIntegrator : public Integrator {
  public:
    GpuPathIntegrator(const Parameters& params, Scene* scene);
    void Render() override;

  private:
    int mathMode;
    uint64_t seed;
    int device;
    pstd::string linearFile;
};

}  // namespace pine

#endif  // PINE_B200_GPUPATH_H
