/* Error reporting shared by the host-side parts of the engine. */
#ifndef VGPU_UTIL_H
#define VGPU_UTIL_H

#include <cstdarg>
#include <cstdio>
#include <string>

namespace vgpu {

/* thread-local "last error" text behind virg_gpu_last_error() */
void set_error(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
const char *last_error();
void clear_error();

}  // namespace vgpu

/* record an error and return VIRG_FAIL (0) from the enclosing function */
#define VGPU_FAIL(...) do { ::vgpu::set_error(__VA_ARGS__); return 0; } while (0)
#define VGPU_CHECK(cond, ...) do { if (!(cond)) VGPU_FAIL(__VA_ARGS__); } while (0)

#endif
