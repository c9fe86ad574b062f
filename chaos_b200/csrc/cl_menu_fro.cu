// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "fro".
#include "cl_registry.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<1, RBenettin>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R0("s3d4p0|k1:BEN|", L0, minb_mask<1>());

cudaError_t L1(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<1, RQR<1>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R1("s3d4p0|k1:QR1|", L1, minb_mask<1>());

cudaError_t L2(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<1, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R2("s3d4p0|k1:QR2|", L2, minb_mask<1>());

cudaError_t L3(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<1, RQR<3>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R3("s3d4p0|k1:QR3|", L3, minb_mask<1>());

cudaError_t L4(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<1, RQR<4>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R4("s3d4p0|k1:QR4|", L4, minb_mask<1>());

cudaError_t L5(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<1, RQR<5>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R5("s3d4p0|k1:QR5|", L5, minb_mask<1>());

cudaError_t L6(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<1, RQR<6>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R6("s3d4p0|k1:QR6|", L6, minb_mask<1>());

cudaError_t L7(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RQR<1>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R7("s3d4p0|k2:QR1|", L7, minb_mask<1>());

cudaError_t L8(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R8("s3d4p0|k2:QR2|", L8, minb_mask<1>());

cudaError_t L9(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RQR<3>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R9("s3d4p0|k2:QR3|", L9, minb_mask<1>());

cudaError_t L10(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RQR<4>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R10("s3d4p0|k2:QR4|", L10, minb_mask<1>());

cudaError_t L11(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RQR<5>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R11("s3d4p0|k2:QR5|", L11, minb_mask<1>());

cudaError_t L12(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RQR<6>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R12("s3d4p0|k2:QR6|", L12, minb_mask<1>());

cudaError_t L13(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RSALI>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R13("s3d4p0|k2:SALI|", L13, minb_mask<1>());

cudaError_t L14(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RGALI<false>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R14("s3d4p0|k2:GALI|", L14, minb_mask<1>());

cudaError_t L15(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RMEGNO<true>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R15("s3d4p0|k2:MEGNO1|", L15, minb_mask<1>());

cudaError_t L16(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RFLI<true>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R16("s3d4p0|k2:FLI1|", L16, minb_mask<1>());

cudaError_t L17(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RMEGNO<false>, RFLI<false>, RQR<6>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R17("s3d4p0|k2:MEGNO0,FLI0,QR6|", L17, minb_mask<1>());

cudaError_t L18(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RMEGNO<false>, RSALI>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R18("s3d4p0|k2:MEGNO0,SALI|", L18, minb_mask<1>());

cudaError_t L19(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RFLI<false>, RSALI>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R19("s3d4p0|k2:FLI0,SALI|", L19, minb_mask<1>());

cudaError_t L20(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2, RMEGNO<false>, RFLI<false>, RSALI>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R20("s3d4p0|k2:MEGNO0,FLI0,SALI|", L20, minb_mask<1>());

cudaError_t L21(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, double, Frame<2>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R21("s3d4p0|k2:|", L21, minb_mask<1>());

}  // namespace
}  // namespace cl
