// Mixed-precision chi contraction: split-BF16 operands on the sm_100a tensor
// cores (tcgen05.mma, accumulators in TMEM), FP32 partial sums per
// transition block, FP64 accumulation of the partials.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "pmx_chi.hpp"

namespace pmx {
namespace dev {

// Workspace the mixed contraction needs for T transitions (bytes).
size_t mixed_workspace_bytes(const ContractArgs& a, long long T);
// Same contract as launch_contract_f64 (writes a.acc); nlaunch receives the
// number of kernels launched, mmas (optional) the number of tcgen05 MMA
// instructions (M 128, N 256, K 16, BF16) the contraction issues.
cudaError_t launch_contract_mixed(const ContractArgs& a, long long T, void* ws, int& nlaunch, cudaStream_t st,
                                  long long* mmas = nullptr);

}  // namespace dev
}  // namespace pmx
