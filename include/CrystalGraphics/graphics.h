#ifndef CRYSTALGRAPHICS_GRAPHICS_H_
#define CRYSTALGRAPHICS_GRAPHICS_H_

#include "api.h"
#include "environment.h"
#include "error.h"
#include "scene.h"

#endif
