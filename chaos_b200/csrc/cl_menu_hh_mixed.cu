// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "hh_mixed".
#include "cl_registry.cuh"
#include "cl_gauss.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysGauss3HH, float, Frame<2, RMEGNO<false>, RFLI<false>, RQR<6>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R0("s6d4p1|k2:MEGNO0,FLI0,QR6|", L0, minb_mask<1>());

cudaError_t L1(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysGauss3HH, float, Frame<2, RQR<2>>, NoFrame, NoFrame, 1, 1>(r, a, A, s, i, m);
}
const Registrar R1("s6d4p1|k2:QR2|", L1, minb_mask<1>());

}  // namespace
}  // namespace cl
