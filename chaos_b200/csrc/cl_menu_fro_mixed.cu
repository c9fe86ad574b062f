// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "fro_mixed".
#include "cl_registry.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, float, Frame<4, RQR<4>>, Frame<4, RGALI<true>>, NoFrame, 2, 1, 2, 3, 4>(r, a, A, s, i, m);
}
const Registrar R0("s3d4p1|k4:QR4|k4:GALI,SALI|", L0, minb_mask<1, 2, 3, 4>());

cudaError_t L1(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, float, Frame<4, RQR<4>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R1("s3d4p1|k4:QR4|", L1, minb_mask<1>());

cudaError_t L2(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, float, Frame<4, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R2("s3d4p1|k4:QR2|", L2, minb_mask<1>());

cudaError_t L3(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, float, Frame<4, RGALI<true>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R3("s3d4p1|k4:GALI,SALI|", L3, minb_mask<1>());

cudaError_t L4(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, float, Frame<4, RGALI<false>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R4("s3d4p1|k4:GALI|", L4, minb_mask<1>());

cudaError_t L5(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, float, Frame<2, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R5("s3d4p1|k2:QR2|", L5, minb_mask<1>());

cudaError_t L6(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, float, Frame<2, RSALI>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R6("s3d4p1|k2:SALI|", L6, minb_mask<1>());

cudaError_t L7(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, float, Frame<2, RMEGNO<true>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R7("s3d4p1|k2:MEGNO1|", L7, minb_mask<1>());

cudaError_t L8(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysFroeschle, float, Frame<2, RMEGNO<false>, RSALI>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R8("s3d4p1|k2:MEGNO0,SALI|", L8, minb_mask<1>());

}  // namespace
}  // namespace cl
