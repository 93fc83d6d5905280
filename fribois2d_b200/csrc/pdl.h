// Programmatic dependent launch: kernels of one stream launched with the
// programmatic-stream-serialization attribute may be scheduled while the
// kernel before them drains; each such kernel starts with FB_GRID_WAIT, which
// returns once the preceding grid has completed and its writes are visible.
// Every kernel that this header launches waits before its first access to
// global memory that earlier kernels write (grouped kernels first stage their
// case's view, which only the host writes), so ordering is the stream's as
// without the attribute.
#pragma once

#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <utility>

// After its wait, every block lets the next kernel of the stream launch: that
// kernel's blocks take free SM slots while this grid's last blocks run and
// wait in their own FB_GRID_WAIT, so the launch latency is hidden.  Since a
// block triggers only once it is running, the next grid launches after all of
// this grid's blocks have started: a waiting grid never holds slots that this
// one still needs.
#define FB_GRID_WAIT() asm volatile("griddepcontrol.wait;\n\tgriddepcontrol.launch_dependents;" ::: "memory")

namespace fb {

inline bool pdl_enabled() {
    static const bool on = [] {
        const char *v = std::getenv("FRIBOIS2D_PDL");
        return !(v && std::strcmp(v, "0") == 0);
    }();
    return on;
}

template <typename... KArgs, typename... Args>
inline void pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args &&...args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

}  // namespace fb
