// beams_mapper.hpp — C++ host adapter over the C ABI, mirroring the reference's
// beams::rendering::MapperLightedVolume (beams/rendering/MapperLightedVolume.h:16-62).
//
// A reference scene's Ready() (beams/rendering/SpheresScene.cxx:181-211) keeps
// its calls: SetShadowMapSize, SetUseShadowMap, ClearLights, AddLight,
// SetSampleDistance, SetCompositeBackground, SetActiveColorTable, then
// RenderCells. VTK-m types are replaced by plain arrays (VTK-m is not a
// dependency of this library); errors raise beams::Error, where the reference
// raises vtkm::cont::ErrorBadValue.
#pragma once

#include <algorithm>
#include <array>
#include <chrono>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "beams_b200.h"

namespace beams {

struct Error : std::runtime_error {
  beams_status status;
  Error(beams_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(beams_status s, const beams_renderer* r) {
  if (s != BEAMS_OK) throw Error(s, beams_last_error(r));
}

// Camera in the reference's terms: position, look-at, view-up, vertical field of view.
struct Camera {
  std::array<double, 3> position{0.5, 0.5, 2.0};
  std::array<double, 3> look_at{0.5, 0.5, 0.5};
  std::array<double, 3> up{0.0, 1.0, 0.0};
  double fov_y_deg = 30.0;
};

// Uniform point (or cell) field on a structured grid; data on the host unless on_device.
struct Field {
  const float* data = nullptr;
  std::array<int, 3> point_dims{2, 2, 2};
  std::array<double, 3> origin{0, 0, 0};
  std::array<double, 3> spacing{1, 1, 1};
  bool cell_associated = false;
  bool on_device = false;
};

// The reference's profiler (beams/Profiler.h:12-60, Profiler.cxx): a tree of
// named frames, each keeping its elapsed times. StartFrame/EndFrame time host
// code; a MapperLightedVolume given the profiler adds every render's frames
// ("Render" > "Phase 1", "Phase 4", "Phase 5", CUDA-event times) under the frame
// open at that moment. Collect() is local here (one process; the reference
// reduces over MPI ranks), PrintSummary writes "name: Min = a ms, Max = b ms,
// Avg = c ms" per frame, two spaces of indent per level, as the reference does.
class Profiler {
 public:
  struct Frame {
    std::string name;
    std::vector<double> ms;
    std::vector<std::unique_ptr<Frame>> sub;
    std::chrono::steady_clock::time_point start{};
    Frame* child(const std::string& n) {
      for (auto& f : sub)
        if (f->name == n) return f.get();
      sub.push_back(std::unique_ptr<Frame>(new Frame{n, {}, {}, {}}));
      return sub.back().get();
    }
  };

  explicit Profiler(const std::string& name) : root_(new Frame{name, {}, {}, {}}) {
    stack_.push_back(root_.get());
    root_->start = std::chrono::steady_clock::now();
  }
  void StartFrame(const std::string& name) {
    Frame* f = stack_.empty() ? root_.get() : stack_.back()->child(name);
    stack_.push_back(f);
    f->start = std::chrono::steady_clock::now();
  }
  void EndFrame() {
    if (stack_.empty()) return;
    Frame* f = stack_.back();
    stack_.pop_back();
    f->ms.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - f->start).count());
  }
  // A frame timed elsewhere: depth 0 under the frame open now, depth d under the
  // last frame recorded at depth d - 1.
  void Record(const std::string& name, int depth, double ms) {
    Frame* parent = depth <= 0 || (size_t)depth > last_.size() ? (stack_.empty() ? root_.get() : stack_.back())
                                                                : last_[(size_t)depth - 1];
    Frame* f = parent->child(name);
    f->ms.push_back(ms);
    last_.resize((size_t)std::max(depth, 0) + 1);
    last_[(size_t)std::max(depth, 0)] = f;
  }
  void Collect() {}
  void PrintSummary(std::ostream& os) const { print(os, *root_, 0); }
  const Frame& Root() const { return *root_; }

 private:
  static void print(std::ostream& os, const Frame& f, int level) {
    double mn = 0.0, mx = 0.0, sum = 0.0;
    if (!f.ms.empty()) {
      mn = *std::min_element(f.ms.begin(), f.ms.end());
      mx = *std::max_element(f.ms.begin(), f.ms.end());
      for (double v : f.ms) sum += v;
    }
    os << std::string((size_t)level * 2, ' ') << f.name << ": Min = " << mn << " ms, Max = " << mx
       << " ms, Avg = " << (f.ms.empty() ? 0.0 : sum / (double)f.ms.size()) << " ms\n";
    for (const auto& c : f.sub) print(os, *c, level + 1);
  }
  std::unique_ptr<Frame> root_;
  std::vector<Frame*> stack_;
  std::vector<Frame*> last_;
};

class MapperLightedVolume {
 public:
  explicit MapperLightedVolume(int device = 0, void* cuda_stream = nullptr) {
    check(beams_create(&r_, device, cuda_stream), nullptr);
  }
  ~MapperLightedVolume() { beams_destroy(r_); }
  MapperLightedVolume(const MapperLightedVolume&) = delete;
  MapperLightedVolume& operator=(const MapperLightedVolume&) = delete;

  // SetCanvas (MapperLightedVolume.cxx:54-69): the canvas is a width x height RGBA buffer.
  void SetCanvas(int width, int height) {
    if (width < 1 || height < 1) throw Error(BEAMS_ERR_INVALID_ARG, "Ray Tracer: bad canvas size");
    width_ = width;
    height_ = height;
  }
  void SetShadowMapSize(std::array<int, 3> m) { check(beams_set_shadow_map_size(r_, m[0], m[1], m[2]), r_); }
  void SetUseShadowMap(bool on) { check(beams_set_use_shadow_map(r_, on ? 1 : 0), r_); }
  void ClearLights() { check(beams_clear_lights(r_), r_); }
  // AddLight with a PointLight{Position, Color, Intensity} (PointLight.h:16-30).
  void AddLight(const std::array<double, 3>& position, const std::array<float, 3>& color, float intensity) {
    check(beams_add_point_light(r_, position.data(), color.data(), intensity), r_);
  }
  // The reference stores the value and forwards it at render time unless it is
  // DEFAULT_SAMPLE_DISTANCE (-1) (MapperLightedVolume.cxx:155-158).
  void SetSampleDistance(float d) { sample_distance_ = d; }
  void SetCompositeBackground(bool on, std::array<float, 4> rgba = {1, 1, 1, 1}) {
    check(beams_set_background(r_, on ? 1 : 0, rgba.data()), r_);
  }
  // The canvas depth buffer MapCanvasToRays reads (MapperLightedVolume.cxx:151-152):
  // OpenGL window depth in [0, 1] with the camera's near/far planes, row 0 at the
  // bottom; an empty vector removes it.
  void SetCanvasDepth(const std::vector<float>& depth, int width, int height, double near_plane, double far_plane) {
    if (depth.empty()) {
      check(beams_set_depth_buffer(r_, nullptr, 0, 0, 0, 0.0, 0.0, 0), r_);
      return;
    }
    if (depth.size() != (size_t)width * height) throw Error(BEAMS_ERR_INVALID_ARG, "depth buffer size");
    check(beams_set_depth_buffer(r_, depth.data(), width, height, BEAMS_DEPTH_WINDOW, near_plane, far_plane, 0), r_);
  }
  void SetDensityScale(float s) { check(beams_set_density_scale(r_, s), r_); }  // stored, never read (as in the reference)
  // Extension: build only the map vertices the frame's view rays read (same
  // image); keep_marks keeps the marked cells while the view is unchanged.
  void SetLazyShadowMap(bool on, bool keep_marks = false) {
    check(beams_set_lazy_shadow_map(r_, on ? (keep_marks ? 2 : 1) : 0), r_);
  }
  // SetProfiler (MapperLightedVolume.cxx:305-309): every RenderCells adds its frames to p.
  void SetProfiler(std::shared_ptr<Profiler> p) {
    check(beams_set_profiler(r_, p ? &MapperLightedVolume::record : nullptr, p.get()), r_);
    profiler_ = std::move(p);
  }
  // SetActiveColorTable: the colour table already sampled to RGBA entries.
  void SetActiveColorTable(const std::vector<float>& rgba) {
    if (rgba.empty() || rgba.size() % 4 != 0) throw Error(BEAMS_ERR_INVALID_ARG, "colour table must be RGBA");
    color_map_ = rgba;
  }

  // RenderCells (MapperLightedVolume.cxx:114-193): returns premultiplied RGBA,
  // width*height*4 floats, row 0 at the bottom.
  std::vector<float> RenderCells(const Field& f, const std::array<double, 2>& scalar_range, const Camera& cam,
                                 beams_timings* timings = nullptr) {
    if (width_ < 1) throw Error(BEAMS_ERR_STATE, "Ray Tracer: no canvas set");
    if (color_map_.empty()) throw Error(BEAMS_ERR_STATE, "no active colour table");
    if (sample_distance_ != -1.f) check(beams_set_sample_distance(r_, sample_distance_), r_);
    beams_volume v{};
    v.data = f.data;
    v.dtype = BEAMS_F32;
    for (int d = 0; d < 3; ++d) {
      v.dims[d] = f.point_dims[d];
      v.origin[d] = f.origin[d];
      v.spacing[d] = f.spacing[d];
    }
    v.range[0] = scalar_range[0];
    v.range[1] = scalar_range[1];
    v.assoc = f.cell_associated ? BEAMS_ASSOC_CELLS : BEAMS_ASSOC_POINTS;
    v.on_device = f.on_device ? 1 : 0;
    check(beams_set_volume(r_, &v), r_);
    check(beams_set_color_map(r_, color_map_.data(), (int)(color_map_.size() / 4)), r_);
    beams_camera c{};
    for (int d = 0; d < 3; ++d) {
      c.position[d] = cam.position[d];
      c.look_at[d] = cam.look_at[d];
      c.up[d] = cam.up[d];
    }
    c.fov_y_deg = cam.fov_y_deg;
    c.width = width_;
    c.height = height_;
    std::vector<float> rgba((size_t)width_ * height_ * 4);
    check(beams_render(r_, &c, rgba.data(), 0, timings), r_);
    return rgba;
  }

  beams_renderer* handle() { return r_; }

 private:
  static void record(void* user, const char* frame, int depth, double ms) {
    static_cast<Profiler*>(user)->Record(frame, depth, ms);
  }
  beams_renderer* r_ = nullptr;
  std::shared_ptr<Profiler> profiler_;
  int width_ = 0, height_ = 0;
  float sample_distance_ = -1.f;
  std::vector<float> color_map_;
};

}  // namespace beams
