// Host utilities that callers of the CUDA-ORB API use alongside it
// (cuda_utils.h of the reference): the exit-on-error CHECK convention, size
// helpers, device selection and a CUDA-event timer.
#pragma once
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>

#define H_PI 1.5707963267948966f
#define CHECK(err) orb_utils_check((err), __FILE__, __LINE__)
#define CheckMsg(msg) orb_utils_check_msg((msg), __FILE__, __LINE__)

// Print the CUDA error and exit(-1), as every reference call site does.
inline void orb_utils_check(cudaError_t err, const char* file, int line) {
  if (err != cudaSuccess) {
    std::fprintf(stderr, "CHECK() Runtime API error in file <%s>, line %i : %s.\n", file, line,
                 cudaGetErrorString(err));
    std::exit(-1);
  }
}

inline void orb_utils_check_msg(const char* msg, const char* file, int line) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    std::fprintf(stderr, "CheckMsg() CUDA error: %s in file <%s>, line %i : %s.\n", msg, file, line,
                 cudaGetErrorString(err));
    std::exit(-1);
  }
}

// Select device `dev` (clamped to the available range) and print its name.
inline bool initDevice(int dev) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    std::fprintf(stderr, "CUDA error: no devices supporting CUDA.\n");
    return false;
  }
  dev = dev < 0 ? 0 : (dev >= n ? n - 1 : dev);
  cudaDeviceProp prop;
  CHECK(cudaGetDeviceProperties(&prop, dev));
  CHECK(cudaSetDevice(dev));
  int drv = 0, rt = 0;
  CHECK(cudaDriverGetVersion(&drv));
  CHECK(cudaRuntimeGetVersion(&rt));
  std::fprintf(stderr, "Using Device %d: %s, CUDA Driver Version: %d.%d, Runtime Version: %d.%d\n", dev, prop.name,
               drv / 1000, drv % 1000, rt / 1000, rt % 1000);
  return true;
}

// Microseconds since the epoch.
inline long long cpuTimer() {
  return std::chrono::duration_cast<std::chrono::microseconds>(
             std::chrono::system_clock::now().time_since_epoch())
      .count();
}

// Milliseconds elapsed on `stream` since construction, measured with CUDA events.
class GpuTimer {
 public:
  explicit GpuTimer(cudaStream_t stream = 0) : stream_(stream) {
    cudaEventCreate(&start_);
    cudaEventCreate(&stop_);
    cudaEventRecord(start_, stream_);
  }
  ~GpuTimer() {
    cudaEventDestroy(start_);
    cudaEventDestroy(stop_);
  }
  float read() {
    cudaEventRecord(stop_, stream_);
    cudaEventSynchronize(stop_);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, start_, stop_);
    return ms;
  }

 private:
  cudaEvent_t start_, stop_;
  cudaStream_t stream_;
};

inline int iAlignUp(const int a, const int b) { return (a % b != 0) ? (a - a % b + b) : a; }
inline int iDivUp(int a, int b) { return (a % b != 0) ? (a / b + 1) : (a / b); }
inline int iExp2UpP(const int a) {
  int p = 0, v = 1;
  while (v < a) {
    v <<= 1;
    p++;
  }
  return p;
}
