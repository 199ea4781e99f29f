// Host-side helpers shared by the C-ABI translation units (capi.cu, batch_capi.cu): the
// thread-local error message, launch accounting and optional per-stage event timing.
#pragma once

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "layout.h"

namespace omnigs {

extern thread_local std::string g_last_error;

// Sets the message of omnigs_last_error() and returns `code`.
int fail(int code, const char* msg);
// OMNIGS_ERR_CUDA with the pending CUDA error's text, or OMNIGS_OK.
int check_launch(const char* what);

// Argument checks shared by the single-view and batched entry points (error texts are the
// reference's where it has one).
int validate_common(int P, int D, int M, int W, int H, const void* shs, const float* colors,
                    const float* scales, const float* rotations, const float* cov3D,
                    const float* means3D, const float* viewmatrix, const float* campos);

// OMNIGS_ERR_INVALID_ARGUMENT unless every given workspace buffer (NULL: not given) is 16-byte
// aligned: the kernels move their records with 16-byte loads and stores.
int check_aligned(const void* a, const void* b = nullptr, const void* c = nullptr);

template <class T>
T* at(void* base, size_t off) {
  return reinterpret_cast<T*>(static_cast<unsigned char*>(base) + off);
}
template <class T>
const T* at(const void* base, size_t off) {
  return reinterpret_cast<const T*>(static_cast<const unsigned char*>(base) + off);
}

struct TimedLaunch {
  int stage;
  int kernels;
  cudaEvent_t start, stop;
};
extern std::atomic<uint64_t> g_launches;
extern std::atomic<bool> g_timing;
extern std::mutex g_timing_mu;
extern std::vector<TimedLaunch> g_timed;
cudaEvent_t take_event();

// Runs `launch` (which enqueues `kernels` kernels on `s`) and accounts for it: counts the launches
// and, while timing is enabled, brackets them with events recorded on `s`.
template <class F>
void staged(int stage, int kernels, cudaStream_t s, F&& launch) {
  g_launches.fetch_add((uint64_t)kernels, std::memory_order_relaxed);
  if (!g_timing.load(std::memory_order_relaxed)) {
    launch();
    return;
  }
  std::lock_guard<std::mutex> lock(g_timing_mu);
  TimedLaunch t{stage, kernels, take_event(), take_event()};
  cudaEventRecord(t.start, s);
  launch();
  cudaEventRecord(t.stop, s);
  g_timed.push_back(t);
}

// Blend staging batch size per direction (0 forward, 1 backward), see blend_batch_size.
extern std::atomic<int> g_blend_batch[2];

// Clears the per-pass state in the header (status capacity bits, counters) and copies the
// instance total into num_rendered; one thread.
void launch_begin_render(GeomHeader* hdr, cudaStream_t s);

}  // namespace omnigs
