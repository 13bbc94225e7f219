// The build's host entry points inside the library (shared by the C ABI in
// build.cu and the request server in server.cu).
#pragma once

#include "common.cuh"

#include <cstdint>
#include <vector>

namespace d3g {

/// Device-resident result of one build of one or more sets.
struct DeviceResult {
    DevBuf<int4> cells;          // finite cells of every set, set by set, canonical order
    DevBuf<int4> all;            // single set only: all cells
    DevBuf<int64_t> inc_off;     // single set only: incident CSR
    DevBuf<int32_t> inc;
    int64_t n_cells = 0, n_all = 0, n_vertices = 0, n_inc = 0;
    std::vector<int64_t> cell_off;   // per set: [cell_off[s], cell_off[s+1]) of `cells`
    std::vector<int64_t> set_nv;     // per set: distinct points
    d3g_build_stats stats{};
    void reset() {
        cells.release();
        all.release();
        inc_off.release();
        inc.release();
        n_cells = n_all = n_vertices = n_inc = 0;
        cell_off.clear();
        set_nv.clear();
        stats = d3g_build_stats{};
    }
};

/// Builds the sets [h_off[s], h_off[s+1]) of the device points d_xyz on stream
/// `s` (the legacy stream is replaced by the calling thread's internal stream).
/// Synchronises the stream it ran on before returning.
int build_on_stream(const double* d_xyz, const int64_t* h_off, int nsets, const d3g_options& opt,
                    cudaStream_t s, DeviceResult& R);

}  // namespace d3g
