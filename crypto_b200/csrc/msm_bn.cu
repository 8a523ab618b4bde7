// BN254 G1 instantiation of the MSM kernels.
#include "msm_kernels.cuh"

namespace kb200 {
const MsmLaunchers& msm_launchers_bn() {
    static const MsmLaunchers L = MsmLaunchImpl<G1BN>::table();
    return L;
}
}  // namespace kb200
