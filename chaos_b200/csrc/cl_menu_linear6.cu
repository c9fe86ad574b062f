// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "linear6".
#include "cl_registry.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysLinear<6>, double, Frame<6, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R0("s5d6p0|k6:QR2|", L0, minb_mask<1>());

cudaError_t L1(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysLinear<6>, double, Frame<6, RQR<4>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R1("s5d6p0|k6:QR4|", L1, minb_mask<1>());

cudaError_t L2(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysLinear<6>, double, Frame<6, RGALI<false>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R2("s5d6p0|k6:GALI|", L2, minb_mask<1>());

}  // namespace
}  // namespace cl
