// GPU planner for one native GEMM call: block tile shape and split-K.
//
// Replaces the reference's CPU planner (core/matrix_matrix/planner.zig):
// desiredThreadCount :88 / rowTaskCount :170 / runPlannedTasks :296 split C
// into at most 64 disjoint column/row tasks for host threads.  On the GPU the
// equivalent decision is how many CTAs cover C (tile shape) and, when C has
// too few tiles to fill the 148 SMs, how far to split K.
#include <algorithm>

#include "kernels.h"

namespace zb {

GemmPlan plan_native_gemm(int m, int n, int k, int elem_bytes, int sm_count) {
    GemmPlan p;
    // n == 1 or m == 1: matrix-vector kernels, K split only while the outputs
    // alone leave SMs idle.
    if (n == 1 || m == 1) {
        p.tile = TILE_GEMV;
        p.splits = gemv_split_count(n == 1 ? m : n, k);
        return p;
    }
    // At most 16 columns (rows) of C: 128 x 16 (16 x 128) FP64 tiles or the
    // FP32 narrow kernel, K split while the output tiles leave SMs idle.
    if ((n <= 16 && m >= 512) || (m <= 16 && n >= 512)) {
        p.tile = n <= 16 ? TILE_NARROW_N : TILE_NARROW_M;
        p.splits = narrow_split_count(m, n, k, sm_count);
        return p;
    }
    // FP64 with fewer 128 x 128 tiles than half the SMs and a short K (<= 1024,
    // too short for split-K to fill the machine with 256-deep slices): 64 x 64
    // tiles (4 warps), K split into slices down to 64 deep until about two CTAs
    // per SM are resident (small products, the coupling GEMMs of blocked TRSM;
    // one CTA per SM measured 5-20 % slower at 512-1024 x 512 x 512-1024, three
    // or four no better than two).  Longer K keeps the 128 x 128 tiles and
    // their split-K below.
    if (elem_bytes == 8 && k <= 1024 && 2L * ((m + 127) / 128) * ((n + 127) / 128) < sm_count) {
        p.tile = TILE_64x64;
        const long tiles = (long)((m + 63) / 64) * ((n + 63) / 64);
        if (tiles < 2L * sm_count && k >= 128) {
            long s = 2L * sm_count / std::max<long>(tiles, 1);
            s = std::min<long>(s, k / 64);
            s = std::min<long>(s, 64);
            if (s >= 2) p.splits = (int)s;
        }
        return p;
    }
    // Narrow-N, tall-M shapes (e.g. 131072 x 64 x 64) are HBM-bound: a 64-wide
    // tile avoids computing (and staging) a half-empty 128-wide tile.
    if (elem_bytes == 8 && n <= 64 && m >= 1024) p.tile = TILE_128x64;
    const int bn = (p.tile == TILE_128x64) ? 64 : 128;
    const long tiles = (long)((m + 127) / 128) * ((n + bn - 1) / bn);
    // Fewer tiles than SMs: split K (each slice at least 256 deep) so that
    // about one wave of CTAs covers the machine; the partials cost one
    // (splits + 2) m n element pass.
    p.splits = 1;
    if (tiles < sm_count && k >= 512) {
        long s = sm_count / std::max<long>(tiles, 1);
        s = std::min<long>(s, k / 256);
        s = std::min<long>(s, 64);
        if (s >= 2) p.splits = (int)s;
    }
    return p;
}

}  // namespace zb
