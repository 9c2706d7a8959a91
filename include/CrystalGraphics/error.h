// crystal::graphics::Error — same definition as the reference
// (include/CrystalGraphics/error.h:8): errors are strings.
#ifndef CRYSTALGRAPHICS_ERROR_H_
#define CRYSTALGRAPHICS_ERROR_H_

#include <string>

namespace crystal::graphics {

using Error = std::string;

}  // namespace crystal::graphics

#endif
