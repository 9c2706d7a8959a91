// crystal::graphics::Scene — move-only handle of an uploaded scene, as in the
// reference (include/CrystalGraphics/scene.h:12-37).  LoadScene(path) reads a
// glTF 2.0 file; LoadScene(desc) uploads an in-memory description (the
// cg_scene_desc of cg_cuda.h).
#ifndef CRYSTALGRAPHICS_SCENE_H_
#define CRYSTALGRAPHICS_SCENE_H_

#include <cstdint>
#include <expected>
#include <filesystem>
#include <memory>

#include "error.h"

struct cg_scene_desc;

namespace crystal::graphics {

class Scene {
 public:
  const auto& FilePath() const { return filepath_; }
  ~Scene();
  Scene(Scene&& other) noexcept;
  Scene& operator=(Scene&&) = delete;
  Scene(const Scene&) = delete;

  // Backend handle (cg_scene_t) for the C ABI.
  void* Handle() const { return handle_; }

 private:
  const std::filesystem::path filepath_;
  void* handle_ = nullptr;

  Scene(const std::filesystem::path& filepath, void* handle);
  friend std::expected<Scene, Error> LoadScene(std::filesystem::path file);
  friend std::expected<Scene, Error> LoadScene(const cg_scene_desc& desc);
};

std::expected<Scene, Error> LoadScene(std::filesystem::path file);
std::expected<Scene, Error> LoadScene(const cg_scene_desc& desc);

}  // namespace crystal::graphics

#endif
