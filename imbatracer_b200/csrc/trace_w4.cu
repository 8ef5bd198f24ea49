// The persistent traversal kernels for 4-wide scenes (imbart_set_node_width(4)): the launch
// shapes of trace.cu with the 4-slot node test, compiled in their own unit so that the two
// sets of instantiations build in parallel.
#include "trace_launch.cuh"

namespace imbart {

LaunchSpec persistent_kernel_spec_w4(bool stats, int variant, bool any, bool masked, int count, int device,
                                     float share, TraceParams& p) {
    return stats ? persistent_kernel_spec<true, 4>(variant, any, masked, count, device, share, p)
                 : persistent_kernel_spec<false, 4>(variant, any, masked, count, device, share, p);
}

}  // namespace imbart
