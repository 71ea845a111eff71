// beams_run — the reference's driver loop (beams/main.cxx:27-44, Beams.cxx:52-105,
// :233-290) on top of the C ABI: read the stage TOML, build the scene, orbit the
// light around the volume in 5-degree steps, render each frame, print its
// timings as one JSON line and optionally save it as a PNG named like the
// reference's canvases (<scene>_<rank>_<NNN>.png, Beams.cxx:292-301).
//
//   beams_run --base-dir=<dir> | --config=<file.toml> [--frames=N] [--out=<dir>] [--device=D]
//
// --base-dir reads <dir>/stage.toml as the reference does; --frames defaults to
// the reference's full orbit (phi from 0 to 2 pi inclusive in 5-degree steps).
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "beams_b200.h"

namespace {

uint32_t crc32(const unsigned char* p, size_t n, uint32_t c = 0xffffffffu) {
  for (size_t i = 0; i < n; ++i) {
    c ^= p[i];
    for (int k = 0; k < 8; ++k) c = (c >> 1) ^ (0xedb88320u & (0u - (c & 1u)));
  }
  return c;
}

void put32(std::vector<unsigned char>& v, uint32_t x) {
  for (int s = 24; s >= 0; s -= 8) v.push_back((unsigned char)(x >> s));
}

void chunk(FILE* f, const char* type, const std::vector<unsigned char>& data) {
  std::vector<unsigned char> b;
  put32(b, (uint32_t)data.size());
  b.insert(b.end(), type, type + 4);
  b.insert(b.end(), data.begin(), data.end());
  const uint32_t c = crc32(b.data() + 4, b.size() - 4) ^ 0xffffffffu;
  put32(b, c);
  fwrite(b.data(), 1, b.size(), f);
}

// 8-bit RGBA PNG with stored (uncompressed) deflate blocks; rows top to bottom.
bool write_png(const char* path, const std::vector<unsigned char>& rgba, int w, int h) {
  FILE* f = std::fopen(path, "wb");
  if (!f) return false;
  static const unsigned char sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  fwrite(sig, 1, 8, f);
  std::vector<unsigned char> ihdr;
  put32(ihdr, (uint32_t)w);
  put32(ihdr, (uint32_t)h);
  ihdr.insert(ihdr.end(), {8, 6, 0, 0, 0});
  chunk(f, "IHDR", ihdr);
  std::vector<unsigned char> raw;
  raw.reserve((size_t)h * (4 * w + 1));
  for (int y = 0; y < h; ++y) {
    raw.push_back(0);  // filter: none
    raw.insert(raw.end(), rgba.begin() + (size_t)y * 4 * w, rgba.begin() + (size_t)(y + 1) * 4 * w);
  }
  std::vector<unsigned char> z = {0x78, 0x01};
  uint32_t a = 1, b = 0;
  for (unsigned char c : raw) {
    a = (a + c) % 65521u;
    b = (b + a) % 65521u;
  }
  for (size_t off = 0; off < raw.size() || off == 0;) {
    const size_t n = std::min<size_t>(65535, raw.size() - off);
    const bool last = off + n >= raw.size();
    z.push_back(last ? 1 : 0);
    z.push_back((unsigned char)(n & 0xff));
    z.push_back((unsigned char)(n >> 8));
    z.push_back((unsigned char)(~n & 0xff));
    z.push_back((unsigned char)((~n >> 8) & 0xff));
    z.insert(z.end(), raw.begin() + off, raw.begin() + off + n);
    off += n;
    if (last) break;
  }
  put32(z, (b << 16) | a);
  chunk(f, "IDAT", z);
  chunk(f, "IEND", {});
  return std::fclose(f) == 0;
}

bool arg(const char* a, const char* name, std::string& out) {
  const size_t n = std::strlen(name);
  if (std::strncmp(a, name, n) == 0 && a[n] == '=') {
    out = a + n + 1;
    return true;
  }
  return false;
}

}  // namespace

int main(int argc, char** argv) {
  std::string base, config, out, frames_s, dev_s;
  bool lazy = false;
  for (int i = 1; i < argc; ++i) {
    std::string preset;
    if (std::strcmp(argv[i], "--lazy-shadow-map") == 0) {
      lazy = true;  // build only the map vertices the view reads, marking once for the fixed camera
      continue;
    }
    if (!arg(argv[i], "--base-dir", base) && !arg(argv[i], "--config", config) && !arg(argv[i], "--out", out) &&
        !arg(argv[i], "--frames", frames_s) && !arg(argv[i], "--device", dev_s) &&
        !arg(argv[i], "--preset", preset)) {
      std::fprintf(stderr,
                   "usage: %s --base-dir=<dir> | --config=<file.toml> [--frames=N] [--out=<dir>] [--device=D] "
                   "[--lazy-shadow-map]\n",
                   argv[0]);
      return 2;
    }
  }
  if (config.empty()) {
    if (base.empty()) {
      std::fprintf(stderr, "beams_run: --base-dir or --config is required\n");
      return 2;
    }
    config = base + "/stage.toml";
  }
  beams_scene_desc d;
  char err[512];
  if (beams_load_config_toml(config.c_str(), &d, err, sizeof(err)) != BEAMS_OK) {
    std::fprintf(stderr, "beams_run: %s: %s\n", config.c_str(), err);
    return 1;
  }
  const int device = dev_s.empty() ? 0 : std::atoi(dev_s.c_str());
  // the reference's loop: phi = 0, 5, ..., 360 degrees (Beams.cxx:239-286)
  const int frames = frames_s.empty() ? 73 : std::atoi(frames_s.c_str());
  beams_renderer* r = nullptr;
  if (beams_create(&r, device, nullptr) != BEAMS_OK) {
    std::fprintf(stderr, "beams_run: %s\n", beams_last_error(nullptr));
    return 1;
  }
  beams_camera cam;
  if (beams_apply_scene(r, &d, &cam) != BEAMS_OK) {
    std::fprintf(stderr, "beams_run: scene: %s\n", beams_last_error(r));
    beams_destroy(r);
    return 1;
  }
  if (lazy && beams_set_lazy_shadow_map(r, 2) != BEAMS_OK) {
    std::fprintf(stderr, "beams_run: %s\n", beams_last_error(r));
    beams_destroy(r);
    return 1;
  }
  std::vector<float> img((size_t)cam.width * cam.height * 4);
  std::vector<unsigned char> px(img.size());
  int rc = 0;
  for (int k = 0; k < frames; ++k) {
    beams_timings t;
    if (beams_orbit_light(r, &d, k) != BEAMS_OK || beams_render(r, &cam, img.data(), 0, &t) != BEAMS_OK) {
      std::fprintf(stderr, "beams_run: frame %d: %s\n", k, beams_last_error(r));
      rc = 1;
      break;
    }
    std::printf("{\"scene\": \"%s\", \"frame\": %d, \"map_build_ms\": %.4f, \"view_march_ms\": %.4f, "
                "\"copy_ms\": %.4f, \"total_ms\": %.4f, \"light_samples\": %llu, \"lit_samples\": %llu, "
                "\"rays_hit\": %llu}\n",
                d.provider_name, k, t.map_build_ms, t.view_march_ms, t.composite_ms, t.total_ms,
                (unsigned long long)t.light_samples, (unsigned long long)t.lit_samples,
                (unsigned long long)t.rays_hit);
    std::fflush(stdout);
    if (!out.empty()) {
      // rows are stored bottom-up (row 0 at the bottom of the canvas); PNG is top-down
      for (int y = 0; y < cam.height; ++y)
        for (int x = 0; x < cam.width * 4; ++x) {
          float v = img[(size_t)(cam.height - 1 - y) * cam.width * 4 + x];
          v = v < 0.f ? 0.f : (v > 1.f ? 1.f : v);
          px[(size_t)y * cam.width * 4 + x] = (unsigned char)(v * 255.f + 0.5f);
        }
      char name[1024];
      std::snprintf(name, sizeof(name), "%s/%s_0_%03d.png", out.c_str(), d.provider_name, k);
      if (!write_png(name, px, cam.width, cam.height)) {
        std::fprintf(stderr, "beams_run: cannot write %s\n", name);
        rc = 1;
        break;
      }
    }
  }
  beams_destroy(r);
  return rc;
}
