// toytrace_gpu_algo.hpp -- C++ host adapter: ToyTrace's RenderingAlgo interface on top of
// the C ABI of toytrace_gpu.h.
//
// RenderingAlgo (src/renderingalgorithms_interface.hxx:13-30) is the plugin boundary every
// ToyTrace renderer implements.  Inside the reference tree GpuPathTracer would derive from
// ::RenderingAlgo directly (its factory, RenderAlgorithmFactory in
// src/renderingalgorithms.cxx:27-42, would construct it for a new algorithm name);
// standalone, RenderingAlgoInterface below declares the same members with the same contracts:
//  - the interrupt callback runs on the thread that called Run();
//  - RequestInterrupt / RequestFullStop may come from any thread, also before Run();
//  - GenerateImage may be called from inside the callback or after Run() returned.
// The pass loop follows SimplePixelByPixelRenderingAlgo::Run
// (renderingalgorithms_simplebase.hxx:125-157) with SamplesPerPixelSchedule (:34-62).
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "toytrace_gpu.h"

namespace toytrace_gpu {

using InterruptCallback = std::function<void(bool)>;

// 8-bit RGB image, row 0 at the top (the reference's Image, image.hxx:16-92).
struct Image8 {
  int width = 0, height = 0;
  std::vector<uint8_t> rgb;
};

class RenderingAlgoInterface {
  InterruptCallback irq_cb;

 public:
  virtual ~RenderingAlgoInterface() noexcept(false) {}
  void SetInterruptCallback(InterruptCallback cb) { irq_cb = std::move(cb); }
  virtual void InitializeScene() {}
  virtual void Run() = 0;
  virtual void RequestInterrupt() = 0;
  virtual void RequestFullStop() = 0;
  virtual std::unique_ptr<Image8> GenerateImage() = 0;

 protected:
  void CallInterruptCb(bool is_complete_pass) {
    if (irq_cb) irq_cb(is_complete_pass);
  }
};

// Parse/config errors surface as std::runtime_error, as in the reference
// (parse_yaml_scene.cxx:137-146); the C ABI underneath never throws.
class Error : public std::runtime_error {
 public:
  Error(tt_status s, const std::string& what) : std::runtime_error(what), status(s) {}
  tt_status status;
};

class GpuPathTracer : public RenderingAlgoInterface {
 public:
  // The scene description is copied by tt_create; it need not outlive the constructor.
  GpuPathTracer(const tt_scene_desc& scene, const tt_params& params, bool linear_output = false,
                uint64_t seed = 1)
      : params_(params), linear_output_(linear_output), seed_(seed) {
    tt_status st = tt_create(&scene, &params, &ctx_);
    if (st != TT_OK) throw Error(st, "tt_create: " + LastError(nullptr));
    xres_ = scene.camera.xres;
    yres_ = scene.camera.yres;
  }
  ~GpuPathTracer() noexcept(false) override { tt_destroy(ctx_); }
  GpuPathTracer(const GpuPathTracer&) = delete;
  GpuPathTracer& operator=(const GpuPathTracer&) = delete;

  void InitializeScene() override {
    if (!initialized_) {
      Check(tt_upload_scene(ctx_), "tt_upload_scene");
      initialized_ = true;
    }
  }

  void Run() override {
    InitializeScene();
    int spp = 1, total = 0;
    const int max_spp = params_.max_samples_per_pixel;
    while (!tt_stop_requested(ctx_) && spp > 0) {
      const tt_status st = tt_render_pass(ctx_, spp, seed_);
      if (st == TT_ERR_INTERRUPTED) break;
      Check(st, "tt_render_pass");
      if (tt_poll_interrupt(ctx_)) CallInterruptCb(false);
      CallInterruptCb(true);
      // SamplesPerPixelSchedule::UpdateForNextPass.
      total += spp;
      if (spp < 1024) spp *= 2;
      if (max_spp > 0 && total + spp > max_spp) spp = max_spp - total;
    }
  }

  void RequestInterrupt() override { tt_request_interrupt(ctx_); }
  void RequestFullStop() override { tt_request_stop(ctx_); }

  std::unique_ptr<Image8> GenerateImage() override {
    auto img = std::make_unique<Image8>();
    img->width = xres_;
    img->height = yres_;
    img->rgb.resize((size_t)xres_ * yres_ * 3);
    Check(tt_generate_image(ctx_, linear_output_ ? 1 : 0, img->rgb.data()), "tt_generate_image");
    return img;
  }

  // Linear float RGB (unit order, row 0 at the bottom) for HDR output.
  std::vector<float> LinearFramebuffer() {
    std::vector<float> out((size_t)xres_ * yres_ * 3);
    Check(tt_read_framebuffer(ctx_, out.data(), nullptr), "tt_read_framebuffer");
    return out;
  }

  tt_ctx* handle() { return ctx_; }

 private:
  static std::string LastError(tt_ctx* c) {
    char buf[1024];
    tt_last_error(c, buf, sizeof(buf));
    return buf;
  }
  void Check(tt_status st, const char* what) {
    if (st != TT_OK) throw Error(st, std::string(what) + ": " + LastError(ctx_));
  }

  tt_ctx* ctx_ = nullptr;
  tt_params params_;
  bool linear_output_;
  uint64_t seed_;
  int xres_ = 0, yres_ = 0;
  bool initialized_ = false;
};

}  // namespace toytrace_gpu
