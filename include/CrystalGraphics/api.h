// View() — the hot path (include/CrystalGraphics/api.h:13), plus the
// headless film readback that replaces presentation.
#ifndef CRYSTALGRAPHICS_API_H_
#define CRYSTALGRAPHICS_API_H_

#include <cstddef>
#include <expected>

#include "camera.h"
#include "error.h"
#include "scene.h"

namespace crystal::graphics {

std::expected<void, Error> View(const Scene& scene, const Camera& camera = {});

enum class FilmFormat : int { kXyz32f = 0, kRgba8 = 1, kRgb32f = 2 };
// Copies the film (row-major, render_width x render_height) into `host`.
std::expected<void, Error> ReadFilm(void* host, std::size_t bytes,
                                    FilmFormat format = FilmFormat::kRgba8);

}  // namespace crystal::graphics

#endif
