// BLS12-381 G1 instantiation of the MSM kernels.
#include "msm_kernels.cuh"

namespace kb200 {
const MsmLaunchers& msm_launchers_bls() {
    static const MsmLaunchers L = MsmLaunchImpl<G1BLS>::table();
    return L;
}
}  // namespace kb200
