// Temporary: spatial and geometry entry points are filled in by spatial.cu and geometry.cu.
#include <string>
#include "rawengine_b200.h"
extern "C" {
re_status re_guided_filter(const float*, size_t, float*, size_t, uint32_t, uint32_t, uint32_t, double, uint32_t, void*) { return RE_INVALID_ARGUMENT; }
re_status re_local_statistics(const float*, size_t, uint32_t, uint32_t, uint32_t, float*, float*, uint32_t*, void*) { return RE_INVALID_ARGUMENT; }
re_status re_cubic_resize(const float*, size_t, uint32_t, uint32_t, uint32_t, uint32_t, re_rect, uint32_t, float*, size_t, void*) { return RE_INVALID_ARGUMENT; }
re_status re_rotate(const float*, size_t, uint32_t, uint32_t, double, re_rect, uint32_t, float*, size_t, void*) { return RE_INVALID_ARGUMENT; }
re_status re_cubic_axis(uint32_t, uint32_t, uint32_t, uint32_t*, uint32_t*, double*, uint32_t*) { return RE_INVALID_ARGUMENT; }
re_status re_rotation_coefficients(double, double*, double*) { return RE_INVALID_ARGUMENT; }
}
