// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "fro4".
#include "cl_registry.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<3, RQR<1>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R0("s3d4p0|k3:QR1|", L0, minb_mask<1>());

cudaError_t L1(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<3, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R1("s3d4p0|k3:QR2|", L1, minb_mask<1>());

cudaError_t L2(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<3, RQR<3>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R2("s3d4p0|k3:QR3|", L2, minb_mask<1>());

cudaError_t L3(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<3, RQR<4>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R3("s3d4p0|k3:QR4|", L3, minb_mask<1>());

cudaError_t L4(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<3, RQR<5>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R4("s3d4p0|k3:QR5|", L4, minb_mask<1>());

cudaError_t L5(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<3, RQR<6>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R5("s3d4p0|k3:QR6|", L5, minb_mask<1>());

cudaError_t L6(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<3, RGALI<false>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R6("s3d4p0|k3:GALI|", L6, minb_mask<1>());

cudaError_t L7(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<4, RQR<1>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R7("s3d4p0|k4:QR1|", L7, minb_mask<1>());

cudaError_t L8(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<4, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R8("s3d4p0|k4:QR2|", L8, minb_mask<1>());

cudaError_t L9(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<4, RQR<3>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R9("s3d4p0|k4:QR3|", L9, minb_mask<1>());

cudaError_t L10(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<4, RQR<4>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R10("s3d4p0|k4:QR4|", L10, minb_mask<1>());

cudaError_t L11(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<4, RQR<5>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R11("s3d4p0|k4:QR5|", L11, minb_mask<1>());

cudaError_t L12(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<4, RQR<6>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R12("s3d4p0|k4:QR6|", L12, minb_mask<1>());

cudaError_t L13(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<4, RGALI<false>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R13("s3d4p0|k4:GALI|", L13, minb_mask<1>());

cudaError_t L14(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<4, RGALI<true>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R14("s3d4p0|k4:GALI,SALI|", L14, minb_mask<1>());

}  // namespace
}  // namespace cl
