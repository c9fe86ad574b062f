// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "split_mixed".
#include "cl_registry.cuh"
#include "cl_split.cuh"

namespace cl {
namespace {

cudaError_t L0(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysSplitHH, float, Frame<2, RMEGNO<false>, RFLI<false>, RQR<6>>, NoFrame, NoFrame, 1, 1, 2, 3, 4>(r, a, A, s, i, m);
}
const Registrar R0("s7d4p1|k2:MEGNO0,FLI0,QR6|", L0, minb_mask<1, 2, 3, 4>());

cudaError_t L1(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysSplitHH, float, Frame<2, RQR<2>>, NoFrame, NoFrame, 1, 1, 2, 3, 4>(r, a, A, s, i, m);
}
const Registrar R1("s7d4p1|k2:QR2|", L1, minb_mask<1, 2, 3, 4>());

cudaError_t L2(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysSplitHH, float, Frame<4, RQR<4>>, NoFrame, NoFrame, 1, 1, 2, 3, 4>(r, a, A, s, i, m);
}
const Registrar R2("s7d4p1|k4:QR4|", L2, minb_mask<1, 2, 3, 4>());

cudaError_t L3(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {
    return launch_instance<SysSplitHH, float, Frame<4, RGALI<false>>, NoFrame, NoFrame, 1, 1, 2, 3, 4>(r, a, A, s, i, m);
}
const Registrar R3("s7d4p1|k4:GALI|", L3, minb_mask<1, 2, 3, 4>());

}  // namespace
}  // namespace cl
