// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "wchain5".
#include "cl_registry.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedChain<5>, double, Frame<8, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R0("s9d10p0|k8:QR2|", L0, minb_mask<1>());

cudaError_t L1(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedChain<5>, double, Frame<8, RQR<4>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R1("s9d10p0|k8:QR4|", L1, minb_mask<1>());

cudaError_t L2(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedChain<5>, double, Frame<8, RGALI<false>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R2("s9d10p0|k8:GALI|", L2, minb_mask<1>());

cudaError_t L3(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedChain<5>, float, Frame<8, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R3("s9d10p1|k8:QR2|", L3, minb_mask<1>());

cudaError_t L4(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedChain<5>, float, Frame<8, RQR<4>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R4("s9d10p1|k8:QR4|", L4, minb_mask<1>());

cudaError_t L5(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedChain<5>, float, Frame<8, RGALI<false>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R5("s9d10p1|k8:GALI|", L5, minb_mask<1>());

cudaError_t L6(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedChain<5>, double, Frame<2, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R6("s9d10p0|k2:QR2|", L6, minb_mask<1>());

cudaError_t L7(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedChain<5>, double, Frame<2, RSALI>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R7("s9d10p0|k2:SALI|", L7, minb_mask<1>());

cudaError_t L8(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedChain<5>, double, Frame<2, RMEGNO<true>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R8("s9d10p0|k2:MEGNO1|", L8, minb_mask<1>());

cudaError_t L9(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedChain<5>, double, Frame<1, RBenettin>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R9("s9d10p0|k1:BEN|", L9, minb_mask<1>());

}  // namespace
}  // namespace cl
