// Mixed-precision chi contraction (split-BF16 tcgen05). See pmx_mixed.hpp.
#include "pmx_mixed.hpp"

namespace pmx {
namespace dev {

size_t mixed_workspace_bytes(const ContractArgs&, long long) { return 0; }

cudaError_t launch_contract_mixed(const ContractArgs&, long long, void*, int& nlaunch, cudaStream_t) {
  nlaunch = 0;
  return cudaErrorNotSupported;
}

}  // namespace dev
}  // namespace pmx
