// view_main.cpp — a headless counterpart of the reference's CLI loop
// (main.cpp:61-84): EnvInit, LoadScene(path), View() frames, then the film is
// written as a binary PPM instead of being presented in a window.
//
//   cg_view <scene.gltf> <out.ppm> [width height spp depth frames]
//           [px py pz dx dy dz vx vy]
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "CrystalGraphics/graphics.h"

using namespace crystal::graphics;

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s scene.gltf out.ppm [w h spp depth frames] [camera x8]\n", argv[0]);
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
  std::vector<unsigned char> rgba(size_t(conf.render_width) * conf.render_height * 4);
  if (auto r = ReadFilm(rgba.data(), rgba.size(), FilmFormat::kRgba8); !r) {
    std::fprintf(stderr, "ReadFilm: %s\n", r.error().c_str());
    return 1;
  }
  FILE* f = std::fopen(argv[2], "wb");
  if (!f) return 1;
  std::fprintf(f, "P6\n%u %u\n255\n", conf.render_width, conf.render_height);
  for (size_t i = 0; i < rgba.size(); i += 4) std::fwrite(&rgba[i], 1, 3, f);
  std::fclose(f);
  (void)EnvTerm();
  return 0;
}
