// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "std_mixed".
#include "cl_registry.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysStandard, float, Frame<2, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R0("s1d2p1|k2:QR2|", L0, minb_mask<1>());

cudaError_t L1(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysStandard, float, Frame<2, RQR<4>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R1("s1d2p1|k2:QR4|", L1, minb_mask<1>());

cudaError_t L2(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysStandard, float, Frame<2, RQR<6>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R2("s1d2p1|k2:QR6|", L2, minb_mask<1>());

cudaError_t L3(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysStandard, float, Frame<1, RBenettin>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R3("s1d2p1|k1:BEN|", L3, minb_mask<1>());

}  // namespace
}  // namespace cl
