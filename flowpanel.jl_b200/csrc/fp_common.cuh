// Shared definitions of the B200 panel-method library (sm_100a).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/flowpanel_b200.h"

namespace fpb {

constexpr double kPi = 3.14159265358979323846;
constexpr double kFourPi = 4.0 * kPi;   // Julia's 4*pi (one rounding of the product)

// Packed panel record in HBM: up to 4 nodes (x,y,z) + node count. 16 doubles
// (128 bytes) so that a warp loads whole records with aligned vector loads.
struct __align__(16) PanelRec {
  double p[12];   // node k at p[3k..3k+2]
  double nn;      // node count (3 or 4)
  double pad[3];
};

// Error reporting: every entry point returns an FP_* status; the text of the
// last failure is kept per context.
struct ErrorSink {
  std::string msg;
  int set(int code, const std::string& m) {
    msg = m;
    return code;
  }
};

#define FP_CUDA_TRY(sink, expr)                                                      \
  do {                                                                               \
    cudaError_t _e = (expr);                                                         \
    if (_e != cudaSuccess) {                                                         \
      return (sink).set(FP_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    }                                                                                \
  } while (0)

// Programmatic dependent launch: hold this grid until the grids it depends
// on have completed and their memory is visible (a no-op for a grid launched
// without the programmatic attribute).
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the stream's next grid (launched with the programmatic attribute) begin
// its launch: that grid still waits in griddep_wait() for this one to finish.
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

inline int64_t round_up(int64_t a, int64_t b) { return (a + b - 1) / b * b; }
__host__ __device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }

// Device-side status bits written by kernels that can give up (bounded waits)
// or detect numerical trouble; read back by the host after the stream sync.
enum DevStatus : int {
  DEV_OK = 0,
  DEV_TIMEOUT = 1,      // a bounded spin-wait ran out
  DEV_ZERO_PIVOT = 2,   // exact zero pivot
};

}  // namespace fpb
