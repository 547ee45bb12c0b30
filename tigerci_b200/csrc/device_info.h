// Device properties the launch code sizes its grids by.
#pragma once
#include <cuda_runtime.h>

namespace tci_dev {

// Streaming multiprocessors of the current device (cached per device; 148 on a B200, the value used when the
// query fails): grid-stride kernels launch a small multiple of it, persistent kernels one CTA per SM.
inline unsigned device_sms() {
  static int cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cached[dev] = v;
  }
  return (unsigned)cached[dev];
}

}  // namespace tci_dev
