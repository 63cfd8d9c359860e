// ORACLE -- test infrastructure only. C entry points over the reference's
// own 3D launchers (compiled in place from the reference sources by
// oracle/Makefile into oracle/_ref/libref3d.so), so the GPU tests can run the
// reference kernels and ours on byte-identical device buffers. The records
// of include/pfb200_3d.h are checked against the reference's here.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdio>

#include "../include/pfb200_3d.h"
#include "pf3d/kernels.cuh"

static_assert(sizeof(pf3d::CellState3D) == sizeof(pfb_cell3d), "CellState3D");
static_assert(offsetof(pf3d::CellState3D, V) == offsetof(pfb_cell3d, V), "CellState3D.V");
static_assert(offsetof(pf3d::CellState3D, storage_edge) == offsetof(pfb_cell3d, storage_edge),
              "CellState3D.storage_edge");
static_assert(sizeof(pf3d::SLayout3D) == sizeof(pfb_layout3d), "SLayout3D");
static_assert(sizeof(pf3d::MeasureArgs3D) == sizeof(pfb_measure_args3d), "MeasureArgs3D");
static_assert(offsetof(pf3d::MeasureArgs3D, apply_tumble) ==
                  offsetof(pfb_measure_args3d, apply_tumble),
              "MeasureArgs3D.apply_tumble");
static_assert(offsetof(pf3d::MeasureArgs3D, storage) == offsetof(pfb_measure_args3d, storage),
              "MeasureArgs3D.storage");
static_assert(sizeof(pf3d::UpdateArgs3D) == sizeof(pfb_update_args3d), "UpdateArgs3D");
static_assert(offsetof(pf3d::UpdateArgs3D, tile_pass) == offsetof(pfb_update_args3d, tile_pass),
              "UpdateArgs3D.tile_pass");
static_assert(offsetof(pf3d::UpdateArgs3D, storage) == offsetof(pfb_update_args3d, storage),
              "UpdateArgs3D.storage");
static_assert(sizeof(pf3d::InitArgs3D) == sizeof(pfb_init_args3d), "InitArgs3D");
static_assert(sizeof(pf3d::ScatterArgs3D) == sizeof(pfb_scatter_args3d), "ScatterArgs3D");
static_assert(sizeof(pf3d::MomentPartial3D) == sizeof(pfb_moment_partial3d), "MomentPartial3D");

namespace {
int status(bool ok, const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (!ok || e != cudaSuccess) {
        std::fprintf(stderr, "%s: %s\n", what, ok ? cudaGetErrorString(e) : "launch refused");
        return -1;
    }
    return 0;
}
const pf3d::MeasureArgs3D& M(const void* a) { return *static_cast<const pf3d::MeasureArgs3D*>(a); }
const pf3d::UpdateArgs3D& U(const void* a) { return *static_cast<const pf3d::UpdateArgs3D*>(a); }
cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }
}  // namespace

extern "C" {

int ref3d_measure_cells_only(const void* a, void* s) {
    return status(pf3d::launch_measure_cells_only(M(a), S(s)), "measure");
}
int ref3d_apply_cell_motion(const void* a, void* s) {
    pf3d::launch_apply_cell_motion(M(a), S(s));
    return status(true, "motion");
}
int ref3d_update_periodic(const void* a, void* s) {
    return status(pf3d::detail::launch_update_periodic_slab_walk_fast(U(a), S(s)), "slab walk");
}
// grid: persistent CTAs of the work-queue update (the host uses occupancy)
int ref3d_update_tiled(const void* a, int grid, void* s) {
    return status(pf3d::detail::launch_update_tiled_fast(U(a), grid, S(s)), "tiled update");
}
int ref3d_clear_S(uint32_t* S_, const void* layout, void* s) {
    pf3d::launch_clear_S(S_, *static_cast<const pf3d::SLayout3D*>(layout), S(s));
    return status(true, "clear");
}
int ref3d_repair_after_fatal(const void* a, void* s) {
    pf3d::launch_repair_after_fatal(U(a), S(s));
    return status(true, "repair");
}
int ref3d_finalize_origins(void* cells, int N, uint32_t* g, void* s) {
    pf3d::launch_finalize_origins(static_cast<pf3d::CellState3D*>(cells), N, g, S(s));
    return status(true, "finalize");
}
int ref3d_restore_cells_after_fatal(void* cells, const void* acc, int N, const uint32_t* g,
                                    void* s) {
    pf3d::launch_restore_cells_after_fatal(static_cast<pf3d::CellState3D*>(cells),
                                           static_cast<const pf3d::CellState3D*>(acc), N, g,
                                           nullptr, S(s));
    return status(true, "restore");
}
int ref3d_advance_step(uint64_t* step, const uint32_t* g, void* s) {
    pf3d::launch_advance_step(step, g, S(s));
    return status(true, "advance");
}
int ref3d_initialize_spheres(const void* a, void* s) {
    pf3d::launch_initialize_spheres(*static_cast<const pf3d::InitArgs3D*>(a), S(s));
    return status(true, "initialize");
}
int ref3d_scatter_current(const void* a, void* s) {
    pf3d::launch_scatter_current(*static_cast<const pf3d::ScatterArgs3D*>(a), S(s));
    return status(true, "scatter");
}

}  // extern "C"
