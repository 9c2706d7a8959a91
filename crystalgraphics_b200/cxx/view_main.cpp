// view_main.cpp — a headless counterpart of the reference's CLI loop
// (main.cpp:61-84): EnvInit, LoadScene(path), View() frames, then the film is
// written to a file instead of being presented in a window: a binary PPM of
// the sRGB RGBA8 film, or, for a name ending in ".pfm", a little-endian PFM
// of the linear-sRGB RGB32F film (rows bottom first, as PFM stores them).
//
//   cg_view <scene.gltf> <out.ppm|out.pfm> [width height spp depth frames]
//           [px py pz dx dy dz vx vy]
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "CrystalGraphics/graphics.h"

using namespace crystal::graphics;

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s scene.gltf out.ppm|out.pfm [w h spp depth frames] [camera x8]\n", argv[0]);
    return 2;
  }
  PathTraceConf conf;
  int frames = 1;
  if (argc >= 8) {
    conf.render_width = std::atoi(argv[3]);
    conf.render_height = std::atoi(argv[4]);
    conf.sample_count = std::atoi(argv[5]);
    conf.trace_depth = std::atoi(argv[6]);
    frames = std::atoi(argv[7]);
  }
  Camera cam;
  if (argc >= 16) {
    cam.position = {std::strtof(argv[8], nullptr), std::strtof(argv[9], nullptr),
                    std::strtof(argv[10], nullptr)};
    cam.direction = {std::strtof(argv[11], nullptr), std::strtof(argv[12], nullptr),
                     std::strtof(argv[13], nullptr)};
    cam.viewport = {std::strtof(argv[14], nullptr), std::strtof(argv[15], nullptr)};
  }
  if (auto r = EnvInit(conf); !r) {
    std::fprintf(stderr, "EnvInit: %s\n", r.error().c_str());
    return 1;
  }
  auto scene = LoadScene(argv[1]);
  if (!scene) {
    std::fprintf(stderr, "LoadScene: %s\n", scene.error().c_str());
    return 1;
  }
  for (int f = 0; f < frames; ++f) {
    if (auto r = View(*scene, cam); !r) {
      std::fprintf(stderr, "View: %s\n", r.error().c_str());
      return 1;
    }
  }
  const std::string out = argv[2];
  const bool pfm = out.size() >= 4 && out.compare(out.size() - 4, 4, ".pfm") == 0;
  const size_t w = conf.render_width, h = conf.render_height;
  std::vector<unsigned char> rgba(pfm ? 0 : w * h * 4);
  std::vector<float> rgb(pfm ? w * h * 3 : 0);
  auto read = pfm ? ReadFilm(rgb.data(), rgb.size() * sizeof(float), FilmFormat::kRgb32f)
                  : ReadFilm(rgba.data(), rgba.size(), FilmFormat::kRgba8);
  if (!read) {
    std::fprintf(stderr, "ReadFilm: %s\n", read.error().c_str());
    return 1;
  }
  FILE* f = std::fopen(out.c_str(), "wb");
  if (!f) {
    std::fprintf(stderr, "cannot write %s\n", out.c_str());
    return 1;
  }
  bool ok = true;
  if (pfm) {
    // little-endian floats (every CUDA host is), hence the negative scale
    std::fprintf(f, "PF\n%zu %zu\n-1.0\n", w, h);
    for (size_t y = h; y-- > 0;) ok = ok && std::fwrite(&rgb[y * w * 3], sizeof(float), w * 3, f) == w * 3;
  } else {
    std::fprintf(f, "P6\n%zu %zu\n255\n", w, h);
    for (size_t i = 0; i < rgba.size(); i += 4) ok = ok && std::fwrite(&rgba[i], 1, 3, f) == 3;
  }
  ok = std::fclose(f) == 0 && ok;
  if (!ok) {
    std::fprintf(stderr, "cannot write %s\n", out.c_str());
    return 1;
  }
  (void)EnvTerm();
  return 0;
}
