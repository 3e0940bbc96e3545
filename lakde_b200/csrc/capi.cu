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

// Launch choices set by an autotuner, per knob and class of D (D <= 16, 32,
// 48, 64); process-wide, read at every launch.
static int g_tuning[LAKDE_TUNE_KNOBS][4] = {};

static int d_class(int64_t D) { return D <= 16 ? 0 : D <= 32 ? 1 : D <= 48 ? 2 : 3; }

int tuning(int knob, int64_t D) {
  return (knob >= 0 && knob < LAKDE_TUNE_KNOBS && D >= 1 && D <= kMaxDim) ? g_tuning[knob][d_class(D)] : 0;
}

}  // namespace lakde

extern "C" int lakde_tuning_set(int knob, int64_t D, int value) {
  lakde::clear_error();
  static const int kChoices[LAKDE_TUNE_KNOBS] = {2, 2, 2};
  if (knob < 0 || knob >= LAKDE_TUNE_KNOBS || D < 1 || D > lakde::kMaxDim || value < 0 || value >= kChoices[knob]) {
    lakde::set_error("tuning_set: knob %d at D=%lld has no choice %d", knob, (long long)D, value);
    return LAKDE_EINVAL;
  }
  lakde::g_tuning[knob][lakde::d_class(D)] = value;
  return LAKDE_OK;
}

extern "C" int lakde_tuning_get(int knob, int64_t D) { return lakde::tuning(knob, D); }

extern "C" const char *lakde_last_error(void) { return lakde::g_last_error; }

extern "C" int lakde_abi_version(void) { return 6; }

extern "C" int lakde_max_dim(void) { return lakde::kMaxDim; }
