// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "wfro".
#include "cl_registry.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<1, RBenettin>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R0("s8d4p0|k1:BEN|", L0, minb_mask<1>());

cudaError_t L1(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<1, RQR<1>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R1("s8d4p0|k1:QR1|", L1, minb_mask<1>());

cudaError_t L2(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<1, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R2("s8d4p0|k1:QR2|", L2, minb_mask<1>());

cudaError_t L3(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<2, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R3("s8d4p0|k2:QR2|", L3, minb_mask<1>());

cudaError_t L4(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<2, RQR<6>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R4("s8d4p0|k2:QR6|", L4, minb_mask<1>());

cudaError_t L5(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<2, RSALI>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R5("s8d4p0|k2:SALI|", L5, minb_mask<1>());

cudaError_t L6(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<2, RMEGNO<true>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R6("s8d4p0|k2:MEGNO1|", L6, minb_mask<1>());

cudaError_t L7(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<2, RFLI<true>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R7("s8d4p0|k2:FLI1|", L7, minb_mask<1>());

cudaError_t L8(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<2, RMEGNO<false>, RFLI<false>, RQR<6>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R8("s8d4p0|k2:MEGNO0,FLI0,QR6|", L8, minb_mask<1>());

cudaError_t L9(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<2, RMEGNO<false>, RSALI>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R9("s8d4p0|k2:MEGNO0,SALI|", L9, minb_mask<1>());

cudaError_t L10(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<4, RQR<4>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R10("s8d4p0|k4:QR4|", L10, minb_mask<1>());

cudaError_t L11(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<4, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R11("s8d4p0|k4:QR2|", L11, minb_mask<1>());

cudaError_t L12(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<4, RGALI<false>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R12("s8d4p0|k4:GALI|", L12, minb_mask<1>());

cudaError_t L13(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<4, RGALI<true>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R13("s8d4p0|k4:GALI,SALI|", L13, minb_mask<1>());

cudaError_t L14(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysWrappedFroeschle, double, Frame<4, RQR<4>>, Frame<4, RGALI<true>>, NoFrame, 2, 1, 2, 3>(r, a, A, s, i, m);
}
const Registrar R14("s8d4p0|k4:QR4|k4:GALI,SALI|", L14, minb_mask<1, 2, 3>());

}  // namespace
}  // namespace cl
