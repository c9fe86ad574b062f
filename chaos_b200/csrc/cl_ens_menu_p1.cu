// Generated by chaos_b200/csrc/gen_menu.py (do not edit): ensemble kernel instances.
#include "cl_coop.cuh"

namespace cl {
namespace {
cudaError_t E0(const cl_run& r, const EArgs& a, int g, const ETune& t, cudaStream_t s, LaunchInfo* i) {
    return launch_ensemble_any<SysStandard, float, Frame<2, RQR<4>>, 5>(r, a, g, t, s, i);
}
const ERegistrar R0("s1d2p1|k2:QR4|", E0);
cudaError_t E1(const cl_run& r, const EArgs& a, int g, const ETune& t, cudaStream_t s, LaunchInfo* i) {
    return launch_ensemble_any<SysChain<2>, float, Frame<4, RQR<4>>, 10>(r, a, g, t, s, i);
}
const ERegistrar R1("s4d4p1|k4:QR4|", E1);
cudaError_t E2(const cl_run& r, const EArgs& a, int g, const ETune& t, cudaStream_t s, LaunchInfo* i) {
    return launch_ensemble_any<SysChain<4>, float, Frame<8, RQR<4>>, 10>(r, a, g, t, s, i);
}
const ERegistrar R2("s4d8p1|k8:QR4|", E2);
cudaError_t E3(const cl_run& r, const EArgs& a, int g, const ETune& t, cudaStream_t s, LaunchInfo* i) {
    return launch_ensemble_any<SysChain<8>, float, Frame<8, RQR<4>>, 20>(r, a, g, t, s, i);
}
const ERegistrar R3("s4d16p1|k8:QR4|", E3);
}  // namespace
}  // namespace cl
