// The reference-side call sequence of the integration notes, compiled against
// include/beams_mapper.hpp and linked with libbeams_b200.so the way a caller of
// beams::rendering::MapperLightedVolume would (MapperLightedVolume.h:16-62;
// SpheresScene.cxx:181-211 sets the mapper up, Beams.cxx:258-266 renders).
//
// Test program: reads a float32 point field and a 256-entry RGBA colour table,
// renders one frame through the adapter and writes the premultiplied RGBA image.
//   mapper_snippet <dir> nx ny nz m lx ly lz cx cy cz ux uy uz fov w h sd
// <dir>/field.bin (nz*ny*nx floats, x fastest), <dir>/tf.bin (256*4 floats)
// -> <dir>/rgba.bin (h*w*4 floats); prints the lit-sample count.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "beams_mapper.hpp"

static std::vector<float> read_floats(const std::string& path, size_t n) {
  std::vector<float> v(n);
  std::ifstream f(path, std::ios::binary);
  if (!f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(float))))
    throw std::runtime_error("cannot read " + path);
  return v;
}

int main(int argc, char** argv) {
  if (argc != 19) {
    std::fprintf(stderr, "usage: mapper_snippet dir nx ny nz m lx ly lz cx cy cz ux uy uz fov w h sd\n");
    return 2;
  }
  const std::string dir = argv[1];
  const int nx = std::atoi(argv[2]), ny = std::atoi(argv[3]), nz = std::atoi(argv[4]), m = std::atoi(argv[5]);
  const double light[3] = {std::atof(argv[6]), std::atof(argv[7]), std::atof(argv[8])};
  beams::Camera camera;
  camera.position = {std::atof(argv[9]), std::atof(argv[10]), std::atof(argv[11])};
  camera.up = {std::atof(argv[12]), std::atof(argv[13]), std::atof(argv[14])};
  camera.fov_y_deg = std::atof(argv[15]);
  const int width = std::atoi(argv[16]), height = std::atoi(argv[17]);
  const float sd = (float)std::atof(argv[18]);
  try {
    const std::vector<float> field = read_floats(dir + "/field.bin", (size_t)nx * ny * nz);
    const std::vector<float> sampled_rgba = read_floats(dir + "/tf.bin", 256 * 4);

    // --- the integration notes' snippet ---------------------------------------
    beams::MapperLightedVolume mapper(/*device=*/0);
    mapper.SetCanvas(width, height);
    mapper.SetShadowMapSize({m, m, m});
    mapper.SetUseShadowMap(true);
    mapper.ClearLights();
    mapper.AddLight({light[0], light[1], light[2]}, {1.0f, 1.0f, 1.0f}, 2.0f);
    mapper.SetActiveColorTable(sampled_rgba);
    mapper.SetSampleDistance(sd);
    mapper.SetDensityScale(1.0f);
    beams::Field f;
    f.data = field.data();
    f.point_dims = {nx, ny, nz};
    f.origin = {0.0, 0.0, 0.0};
    f.spacing = {1.0 / (nx - 1), 1.0 / (ny - 1), 1.0 / (nz - 1)};
    auto profiler = std::make_shared<beams::Profiler>("Beams");
    mapper.SetProfiler(profiler);
    beams_timings t{};
    std::vector<float> rgba = mapper.RenderCells(f, {0.0, 1.0}, camera, &t);
    // ---------------------------------------------------------------------------
    profiler->StartFrame("Second render");
    mapper.RenderCells(f, {0.0, 1.0}, camera);
    profiler->EndFrame();
    // the lazy map extension gives the same image bit for bit
    mapper.SetLazyShadowMap(true);
    const std::vector<float> lazy = mapper.RenderCells(f, {0.0, 1.0}, camera);
    mapper.SetLazyShadowMap(false);
    if (lazy != rgba) return 5;
    profiler->Collect();
    profiler->PrintSummary(std::cerr);  // the reference prints to a stream as well

    std::ofstream out(dir + "/rgba.bin", std::ios::binary);
    out.write(reinterpret_cast<const char*>(rgba.data()), (std::streamsize)(rgba.size() * sizeof(float)));
    std::printf("%llu\n", (unsigned long long)t.lit_samples);
    // an error surfaces as beams::Error, as the reference raises ErrorBadValue
    try {
      mapper.SetCanvas(0, 0);
      return 3;
    } catch (const beams::Error& e) {
      if (e.status != BEAMS_ERR_INVALID_ARG) return 4;
    }
  } catch (const beams::Error& e) {
    std::fprintf(stderr, "beams error %d: %s\n", (int)e.status, e.what());
    return 1;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  return 0;
}
