// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "fro_mixed".
#include "cl_registry.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i) {
    return launch_instance<SysFroeschle, float, Frame<4, RQR<4>>, Frame<4, RGALI<true>>, NoFrame, 2>(r, a, A, s, i);
}
const Registrar R0("s3d4p1|k4:QR4|k4:GALI,SALI|", L0);

cudaError_t L1(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i) {
    return launch_instance<SysFroeschle, float, Frame<4, RQR<4>>, NoFrame, NoFrame, 1>(r, a, A, s, i);
}
const Registrar R1("s3d4p1|k4:QR4|", L1);

cudaError_t L2(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i) {
    return launch_instance<SysFroeschle, float, Frame<4, RQR<2>>, NoFrame, NoFrame, 1>(r, a, A, s, i);
}
const Registrar R2("s3d4p1|k4:QR2|", L2);

cudaError_t L3(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i) {
    return launch_instance<SysFroeschle, float, Frame<4, RGALI<true>>, NoFrame, NoFrame, 1>(r, a, A, s, i);
}
const Registrar R3("s3d4p1|k4:GALI,SALI|", L3);

cudaError_t L4(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i) {
    return launch_instance<SysFroeschle, float, Frame<4, RGALI<false>>, NoFrame, NoFrame, 1>(r, a, A, s, i);
}
const Registrar R4("s3d4p1|k4:GALI|", L4);

cudaError_t L5(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i) {
    return launch_instance<SysFroeschle, float, Frame<2, RQR<2>>, NoFrame, NoFrame, 1>(r, a, A, s, i);
}
const Registrar R5("s3d4p1|k2:QR2|", L5);

cudaError_t L6(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i) {
    return launch_instance<SysFroeschle, float, Frame<2, RSALI>, NoFrame, NoFrame, 1>(r, a, A, s, i);
}
const Registrar R6("s3d4p1|k2:SALI|", L6);

cudaError_t L7(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i) {
    return launch_instance<SysFroeschle, float, Frame<2, RMEGNO<true>>, NoFrame, NoFrame, 1>(r, a, A, s, i);
}
const Registrar R7("s3d4p1|k2:MEGNO1|", L7);

}  // namespace
}  // namespace cl
