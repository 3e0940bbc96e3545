// Error state and ABI metadata of the C interface.
#include <stdarg.h>
#include <stdio.h>

#include "common.cuh"

namespace lakde {

static thread_local char g_last_error[512] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

void clear_error() { g_last_error[0] = '\0'; }

int check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: kernel launch failed: %s", what, cudaGetErrorString(e));
    return LAKDE_ECUDA;
  }
  return LAKDE_OK;
}

int bind_device(const char *what, std::initializer_list<const void *> ptrs) {
  int dev = -1;
  for (const void *p : ptrs) {
    if (!p) continue;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error("%s: cannot query pointer %p: %s", what, p, cudaGetErrorString(e));
      return LAKDE_EINVAL;
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) {
      set_error("%s: pointer %p is not device memory", what, p);
      return LAKDE_EINVAL;
    }
    if (dev < 0) {
      dev = a.device;
    } else if (a.device != dev) {
      set_error("%s: buffers live on different devices (%d and %d)", what, dev, a.device);
      return LAKDE_EINVAL;
    }
  }
  if (dev >= 0) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != dev) {
      cudaError_t e = cudaSetDevice(dev);
      if (e != cudaSuccess) {
        set_error("%s: cudaSetDevice(%d): %s", what, dev, cudaGetErrorString(e));
        return LAKDE_ECUDA;
      }
    }
  }
  return LAKDE_OK;
}

}  // namespace lakde

extern "C" const char *lakde_last_error(void) { return lakde::g_last_error; }

extern "C" int lakde_abi_version(void) { return 5; }

extern "C" int lakde_max_dim(void) { return lakde::kMaxDim; }
