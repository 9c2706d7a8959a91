// crystal_graphics.cpp — the reference's public C++23 API
// (include/CrystalGraphics/*.h of ray847/CrystalGraphics) over the C ABI of
// libcg_cuda.so.  Signatures, argument meaning and error strings follow the
// reference: every call returns std::expected<..., Error> and View() without
// an environment fails with "Environment not initialized." (src/view.cpp:13).
#include <cstring>
#include <expected>
#include <filesystem>
#include <string>
#include <utility>

#include "CrystalGraphics/graphics.h"
#include "cg_cuda.h"

namespace crystal::graphics {
namespace {

std::unexpected<Error> lastError() { return std::unexpected(Error{cg_last_error()}); }

cg_camera toC(const Camera& c) {
  cg_camera out{};
  out.position[0] = c.position.x;
  out.position[1] = c.position.y;
  out.position[2] = c.position.z;
  out.direction[0] = c.direction.x;
  out.direction[1] = c.direction.y;
  out.direction[2] = c.direction.z;
  out.viewport[0] = c.viewport.x;
  out.viewport[1] = c.viewport.y;
  return out;
}

}  // namespace

// ---- environment (environment.h:20-24) -------------------------------------------
std::expected<void, Error> EnvInit(PathTraceConf conf) {
  cg_conf c{conf.window_width, conf.window_height, conf.render_width, conf.render_height,
            conf.sample_count, conf.trace_depth, conf.max_transport_sample_count,
            conf.max_diffuse_sample_count, conf.max_rough_sample_count,
            conf.max_emission_sample_count};
  if (cg_init(&c, 0) != CG_OK) return lastError();
  return {};
}

std::expected<void, Error> EnvTerm() {
  if (cg_term() != CG_OK) return lastError();
  return {};
}

// Headless: no window to poll and no swap chain to present.
std::expected<void, Error> EnvPoll() {
  if (!cg_status()) return std::unexpected(Error{"Environment not initialized."});
  return {};
}
std::expected<void, Error> EnvPresent() {
  if (!cg_status()) return std::unexpected(Error{"Environment not initialized."});
  return {};
}

bool EnvStatus() { return cg_status() == 1; }

// ---- scenes (scene.h) ------------------------------------------------------------------
Scene::Scene(const std::filesystem::path& filepath, void* handle)
    : filepath_(filepath), handle_(handle) {}

Scene::Scene(Scene&& other) noexcept
    : filepath_(other.filepath_), handle_(std::exchange(other.handle_, nullptr)) {}

Scene::~Scene() {
  if (handle_) cg_scene_destroy(static_cast<cg_scene_t>(handle_));
}

std::expected<Scene, Error> LoadScene(std::filesystem::path file) {
  cg_scene_t h = nullptr;
  if (cg_scene_load_gltf(file.string().c_str(), &h) != CG_OK) return lastError();
  return Scene(file, h);
}

std::expected<Scene, Error> LoadScene(const cg_scene_desc& desc) {
  cg_scene_t h = nullptr;
  if (cg_scene_create(&desc, &h) != CG_OK) return lastError();
  return Scene(std::filesystem::path{}, h);
}

// ---- View (api.h:13) -----------------------------------------------------------------------
std::expected<void, Error> View(const Scene& scene, const Camera& camera) {
  if (!cg_status()) return std::unexpected(Error{"Environment not initialized."});
  cg_camera c = toC(camera);
  if (cg_view(static_cast<cg_scene_t>(scene.Handle()), &c) != CG_OK) return lastError();
  return {};
}

std::expected<void, Error> ReadFilm(void* host, std::size_t bytes, FilmFormat format) {
  if (cg_film_read(host, bytes, static_cast<int>(format)) != CG_OK) return lastError();
  return {};
}

}  // namespace crystal::graphics
