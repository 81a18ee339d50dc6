// handler.cpp - RayTracer::set_intersection_handler (src/lib.rs:291-295).
// The handler source is kept on the tracer and copied into every pipeline created from it; the
// default handler (src/default_intersection_handler.wesl) always reports a miss.
#include <string>

#include "scene.h"
#include "tracer.h"

namespace lam {

int set_intersection_handler(lam_tracer* t, const char* src) {
    t->intersection_handler = src ? std::string(src) : std::string();
    return LAM_OK;
}

}  // namespace lam
