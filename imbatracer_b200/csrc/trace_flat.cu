// The persistent traversal kernels for scenes whose top level is one identity instance
// (configs with a single mesh): the launch shapes of trace.cu with the instance entry and
// exit compiled out, in their own unit so that they build in parallel with the others.
#include "trace_launch.cuh"

namespace imbart {

LaunchSpec persistent_kernel_spec_flat(bool stats, int variant, bool any, bool masked, int count, int device,
                                       float share, TraceParams& p) {
    return stats ? persistent_kernel_spec<true, 8, true>(variant, any, masked, count, device, share, p)
                 : persistent_kernel_spec<false, 8, true>(variant, any, masked, count, device, share, p);
}

}  // namespace imbart
