// Host interface of the tcgen05 grouped GEMM (gemm_tc.cu): the mixed-precision
// form of the plan's GEMM steps.
#pragma once
#include <cuda_runtime.h>

#include "gemm_tables.h"

namespace tci_gtc_host {

int tile_m();  // rows of C per CTA tile (problem tables must be tiled with tile_m x tile_n)
int tile_n();
cudaError_t prepare();  // raises the kernel's dynamic shared-memory limit (once per process)
// kblock: k elements per FP64 promotion block, a multiple of 32.
cudaError_t launch(const tci_dev::DGemmProblem* probs, int nprob, const tci_dev::DGemmSeg* segs, long long ntiles,
                   int* status, int kblock, cudaStream_t st);

}  // namespace tci_gtc_host
