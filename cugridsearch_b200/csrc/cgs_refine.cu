// cgs_refine.cu -- coarse-to-fine search: the reference driver's loop of grid searches, each on
// the previous grid shrunk about its argmin (src/gpu/cudaGridSearch_main_mi.cu:312-363).
#include <cmath>
#include <string>

#include "cgs_internal.h"

extern "C" {

cgs_status cgs_search_refine(const cgs_image *mov, const cgs_image *fix, const cgs_grid *grid,
                             const cgs_options *options, int32_t depth, cgs_argmin *levels, cgs_grid *final_grid,
                             cgs_stream_t stream) {
    using namespace cgs;
    cgs_status s = check_grid(grid);
    if (s != CGS_SUCCESS) return s;
    if (depth < 1 || depth > 64) return fail(CGS_ERROR_INVALID_VALUE, "depth must be 1..64");
    cgs_grid g = *grid;
    cgs_argmin r{};
    for (int32_t lv = 0; lv < depth; lv++) {
        if ((s = cgs_search_sync(mov, fix, &g, options, nullptr, &r, stream)) != CGS_SUCCESS) return s;
        if (levels) levels[lv] = r;
        if (!r.valid) {
            // no finite cost on this level: the remaining levels have nothing to centre on
            for (int32_t k = lv + 1; levels && k < depth; k++) levels[k] = r;
            break;
        }
        if (lv + 1 == depth) break;
        // the reference's update, in float: start' = p - (end - start) / 4, then
        // end' = p + (end - start') / 4 with the updated start (:354-355); the counts are set
        // again from the first level's (:300-308, :319)
        for (int a = 0; a < g.dims; a++) {
            const float p = r.params[a];
            g.start[a] = p - (g.end[a] - g.start[a]) / 4;
            g.end[a] = p + (g.end[a] - g.start[a]) / 4;
            g.count[a] = grid->count[a];
        }
        // the setters' update() (cudaGridSearch.cuh:198-215): the last one sees the final rows
        if ((s = cgs_grid_update(&g, -1)) != CGS_SUCCESS) return s;
    }
    if (final_grid) *final_grid = g;
    return CGS_SUCCESS;
}

}  // extern "C"
