// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "fro_fused".
#include "cl_registry.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<4, RQR<4>>, Frame<4, RGALI<true>>, NoFrame, 2, 1, 2, 3>(r, a, A, s, i, m);
}
const Registrar R0("s3d4p0|k4:QR4|k4:GALI,SALI|", L0, minb_mask<1, 2, 3>());

}  // namespace
}  // namespace cl
