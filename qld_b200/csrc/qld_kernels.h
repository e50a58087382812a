// qld_kernels.h -- host-side view of the counts kernels (internal to libqld_cuda).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "qld_device.cuh"

namespace qld {

// Geometry a launcher needs from a kernel: output tile, and the TMA box
// (box_words words along K by box_rows rows) its tensor maps must use.
struct KernelShape {
    int bm, bn;       // A rows x B rows per output tile
    int box_words;    // K words per TMA box (one stage)
    int box_rows;     // rows per TMA box
};

extern const KernelShape kPopcShape;

// Variant (a): tiles_b tile rows starting at p.tb0; p.nk = ceil(K / box_words).
cudaError_t launch_popc(const CUtensorMap &tmA, const CUtensorMap &tmB, const LdParams &p,
                        int tiles_b, int r2_mode, cudaStream_t st);

}  // namespace qld
