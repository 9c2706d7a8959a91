// size32_t, as in the reference (include/CrystalGraphics/public.h:11).
#ifndef CRYSTALGRAPHICS_PUBLIC_H_
#define CRYSTALGRAPHICS_PUBLIC_H_

#include <cstdint>

namespace crystal::graphics {

using size32_t = uint32_t;

}  // namespace crystal::graphics

#endif
