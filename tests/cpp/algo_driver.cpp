// Drives the C++ RenderingAlgo adapter (include/toytrace_gpu_algo.hpp) the way toytrace's
// main does (toytrace.cxx:174-221): construct, set the callback, Run on this thread,
// request an interrupt from another thread, and generate images from the callback.
#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>

#include "toytrace_gpu_algo.hpp"

int main() {
  // A floor quad lit by a downward-facing square area light.
  std::vector<float> v = {0, 0, 0, 0, 0, 1, 1, 0, 1, 1, 0, 0,
                          0.4f, 0.99f, 0.4f, 0.6f, 0.99f, 0.4f, 0.6f, 0.99f, 0.6f, 0.4f, 0.99f, 0.6f};
  std::vector<uint32_t> idx = {0, 1, 2, 0, 2, 3, 4, 5, 6, 4, 6, 7};
  std::vector<uint32_t> mat = {0, 0, 1, 1};
  tt_material m[2] = {};
  m[0].shader = TT_SHADER_DIFFUSE;
  m[1].shader = TT_SHADER_DIFFUSE;
  m[1].emissive = 1;
  for (int b = 0; b < TT_NBINS; ++b) { m[0].reflectance[b] = 0.7f; m[1].emission[b] = 10.f; }
  tt_scene_desc d = {};
  d.num_vertices = 8; d.vertices = v.data();
  d.num_triangles = 4; d.indices = idx.data(); d.material_ids = mat.data();
  d.num_materials = 2; d.materials = m;
  d.camera.kind = TT_CAMERA_PINHOLE;
  float pos[3] = {0.5f, 0.5f, -1.2f}, dir[3] = {0, -0.3f, 1}, up[3] = {0, 1, 0};
  for (int k = 0; k < 3; ++k) { d.camera.pos[k] = pos[k]; d.camera.dir[k] = dir[k]; d.camera.up[k] = up[k]; }
  d.camera.fov_deg = 50; d.camera.xres = 64; d.camera.yres = 48;
  tt_params p = {};
  p.max_ray_depth = 8; p.pt_sample_mode = TT_SAMPLE_BOTH; p.max_samples_per_pixel = 7;
  int complete = 0, incomplete = 0;
  double mean = 0;
  {
    toytrace_gpu::GpuPathTracer algo(d, p);
    algo.SetInterruptCallback([&](bool is_complete) {
      (is_complete ? complete : incomplete)++;
      auto img = algo.GenerateImage();
      double s = 0;
      for (uint8_t c : img->rgb) s += c;
      mean = s / img->rgb.size();
    });
    std::thread t([&] { algo.RequestInterrupt(); });
    t.join();
    algo.Run();
    auto img = algo.GenerateImage();
    std::FILE* f = std::fopen("algo_driver_image.ppm", "wb");
    if (f) {
      std::fprintf(f, "P6\n%d %d\n255\n", img->width, img->height);
      std::fwrite(img->rgb.data(), 1, img->rgb.size(), f);
      std::fclose(f);
    }
  }
  // Bad input surfaces as an exception from the constructor.
  bool threw = false;
  try {
    mat[0] = 9;
    toytrace_gpu::GpuPathTracer bad(d, p);
  } catch (const toytrace_gpu::Error& e) {
    threw = e.status == TT_ERR_INVALID;
  }
  std::printf("complete=%d incomplete=%d mean=%.2f threw=%d\n", complete, incomplete, mean, threw ? 1 : 0);
  return (complete == 3 && incomplete == 1 && mean > 1.0 && threw) ? 0 : 1;
}
