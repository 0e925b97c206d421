// mlp_les.h -- the closure network's forward pass fused with the LES mode's
// checks and blend (les.cuh): the output layer's epilogue blends each point
// into the subgrid stresses instead of storing the network's outputs.
#pragma once
#include "chanflow.h"
#include "les.cuh"

namespace cfd {
// y = network(b.F[pt]) for pt < n, blended into b.S (LesBlend); T is the
// storage precision of the stresses.  CFG_OK or a cfg error code.
template <typename T>
int mlp_forward_blend(cfg_mlp* m, long long n, const LesBlend<T>& b, void* stream);
}  // namespace cfd
