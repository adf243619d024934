// Mixed-precision two-body commutator (tcgen05) hooks used by engine.cu.
#pragma once

#include <cuda_runtime.h>
#include <string>

#include "fp64_kernels.cuh"

namespace g12 {

struct MixedState {
    int ready = 0;
};

inline int mixed_init(MixedState &m, const Dev &, int, std::string *err)
{
    m.ready = 0;
    if (err) *err = "mixed-precision path not built in this library";
    return -1;
}
inline void mixed_free(MixedState &) {}
inline int mixed_on_state(MixedState &, const Dev &, cudaStream_t) { return -1; }
inline void mixed_enqueue_stage(MixedState &, const Dev &, int, int, cudaStream_t) {}
inline int mixed_launches_per_stage(const MixedState &) { return 0; }
inline int mixed_kernel_kinds(const MixedState &) { return 0; }
inline const char *mixed_kernel_name(const MixedState &, int) { return ""; }
inline void mixed_enqueue_kind(MixedState &, const Dev &, int, int, int, cudaStream_t) {}

}  // namespace g12
