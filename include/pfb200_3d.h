/* pfb200_3d.h — C ABI of the B200 3D cell update (sm_100a).
 *
 * Drop-in for the three-dimensional launch interface of the reference
 * (pf3d_core, reference include/pf3d/kernels.cuh:255-542): the argument
 * records below are byte-identical to pf3d::CellState3D, SLayout3D,
 * MeasureArgs3D, UpdateArgs3D, InitArgs3D and ScatterArgs3D, so a host that
 * fills the reference's records passes them here unchanged (cast the
 * pointer). Every launcher enqueues on the caller's stream, allocates
 * nothing, and returns PFB_OK or a negative status (see pfb200.h) where the
 * reference launcher returns false or silently declines.
 *
 * Supported: cubic cell storage (storage.z_cap == 0), all three boundary
 * geometries (periodic XYZ, substrate slab, hard-wall channel), cell
 * selections, the whole-brick tile pass. Cells with a promoted support
 * (storage_edge != 0) are skipped by the base-brick kernels, as in the
 * reference. Compact storage, promoted-cell launchers, the in-place update
 * and the spatially sharded launchers have no counterpart here.
 */
#ifndef PFB200_3D_H
#define PFB200_3D_H

#include <stddef.h>
#include <stdint.h>

#include "pfb200.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__) || defined(__CUDACC__)
#define PFB3D_ALIGNED(n) __attribute__((aligned(n)))
#else
#define PFB3D_ALIGNED(n)
#endif

/* Boundary flags (reference include/pf3d/params.cuh:24-33). */
#define PFB3D_BOUNDARY_PERIODIC_XYZ 0x7u
#define PFB3D_BOUNDARY_SUBSTRATE_SLAB 0x3u
#define PFB3D_BOUNDARY_HARD_WALL_CHANNEL 0xBu

/* Sticky flag indices (reference include/pf3d/kernels.cuh:55-68). The cell
 * record holds them as bits, global_flags as one u32 counter each. */
enum {
    PFB3D_FLAG_S_OVERFLOW = 0,
    PFB3D_FLAG_Q_CLAMP = 1,
    PFB3D_FLAG_S_NEGATIVE = 2,
    PFB3D_FLAG_NONFINITE = 3,
    PFB3D_FLAG_V_NONPOSITIVE = 4,
    PFB3D_FLAG_SUPPORT_EXHAUSTED = 5,
    PFB3D_FLAG_SUPPORT_EDGE = 6,
    PFB3D_FLAG_DESTINATION_CLIP = 7,
    PFB3D_FLAG_INVALID_GEOMETRY = 8,
    PFB3D_FLAG_SLAB_TOP_CONTACT = 9,
    PFB3D_FLAG_COUNT = 10
};
/* All flags but SUPPORT_EDGE stop advancement (kernels.cuh:73-87). */
#define PFB3D_FATAL_MASK 0x3BFu

/* pf3d::CellState3D (kernels.cuh:98-137), 256 bytes, 64-byte aligned. */
typedef struct pfb_cell3d {
    int64_t global_id;
    int64_t origin_x, origin_y, origin_z;
    float polarity_x, polarity_y, polarity_z;
    float velocity_x, velocity_y, velocity_z;
    float gamma, v_A, R_tgt;
    float phi_max;
    uint32_t shift_ctr;
    uint32_t tumble_ctr;
    uint32_t flags;
    uint32_t pad0;
    int32_t bb_lo_x, bb_hi_x;
    int32_t bb_lo_y, bb_hi_y;
    int32_t bb_lo_z, bb_hi_z;
    int32_t pending_shift_x, pending_shift_y, pending_shift_z;
    uint32_t pad1;
    double V;
    double Cx, Cy, Cz;
    double surface;
    double Ix, Iy, Iz;
    uint32_t storage_edge;
    uint32_t pad2;
    double wall_overlap;
    double outside_slit_volume;
    uint32_t reserved[10];
} PFB3D_ALIGNED(64) pfb_cell3d;

/* pf3d::SLayout3D (kernels.cuh:153-176): dense u32 aggregate, x fastest,
 * pitch_x words per row, ny rows per plane. */
typedef struct pfb_layout3d {
    int nx, ny, nz;
    int pitch_x;
    uint32_t boundary_flags;
} pfb_layout3d;

/* pf3d::WeightedWallField3D (kernels.cuh:191-194): kappa_w/kappa psi_w(z)^2
 * per world plane, channel geometry only. */
typedef struct pfb_wall3d {
    const float* values;
    int planes;
} pfb_wall3d;

/* pf3d::CellSelection3D (kernels.cuh:219-229): null ids selects all N. */
typedef struct pfb_selection3d {
    const int* ids;
    int count;
} pfb_selection3d;

/* pf3d::CellFieldStorage3D (phase_storage.hpp:25-27); only z_cap = 0. */
typedef struct pfb_storage3d {
    int z_cap;
} pfb_storage3d;

/* pf3d::MomentPartial3D (kernels.cuh:244-252), 96 bytes. */
typedef struct pfb_moment_partial3d {
    double V, Cx, Cy, Cz;
    double surface;
    double Ix, Iy, Iz;
    int lo_x, hi_x, lo_y, hi_y, lo_z, hi_z;
    unsigned int phi_max_bits;
    unsigned int padding;
} PFB3D_ALIGNED(16) pfb_moment_partial3d;

/* pf3d::MeasureArgs3D (kernels.cuh:254-283), 168 bytes. `partials` and
 * `shards` are accepted and ignored: one cluster per cell reduces on chip. */
typedef struct pfb_measure_args3d {
    const float* phi;
    const uint32_t* S;
    pfb_wall3d wall;
    pfb_cell3d* cells;
    uint32_t* global_flags;
    const uint64_t* step;
    pfb_layout3d layout;
    int N;
    int B;
    pfb_moment_partial3d* partials;
    int shards;
    uint64_t polarity_stream;
    uint64_t aging_steps;
    double p_tumble;
    float motility_coeff;
    int max_shift;
    int support_margin;
    uint8_t apply_tumble;
    uint8_t compute_surface;
    pfb_selection3d selection;
    pfb_storage3d storage;
} pfb_measure_args3d;

/* pf3d::UpdateTilePass3D and TileExchangeRegion3D (tile_partition.cuh:9-18). */
enum { PFB3D_TILE_PASS_ALL = 0, PFB3D_TILE_PASS_BOUNDARY = 1, PFB3D_TILE_PASS_INTERIOR = 2 };
typedef struct pfb_exchange_region3d {
    int y_lo[4];
    int y_hi[4];
    int y_count;
    int z_lo;
    int z_hi;
} pfb_exchange_region3d;

/* pf3d::UpdateArgs3D (kernels.cuh:285-314), 208 bytes. `work_cursor` is
 * not used (the grid is static). */
typedef struct pfb_update_args3d {
    float* phi_in;
    float* phi_out;
    const uint32_t* S_in;
    uint32_t* S_out;
    pfb_wall3d wall;
    pfb_cell3d* cells;
    uint32_t* global_flags;
    unsigned long long* work_cursor;
    pfb_layout3d layout;
    int N;
    int B;
    float dt;
    double V0;
    double volume_scale;
    float bulk_scale;
    float interaction_coeff;
    uint8_t compute_surface;
    pfb_selection3d selection;
    int tile_pass;
    pfb_exchange_region3d exchange_region;
    pfb_storage3d storage;
} pfb_update_args3d;

typedef struct pfb_vec3 {
    double x, y, z;
} pfb_vec3;

/* pf3d::InitArgs3D (kernels.cuh:200-213), 72 bytes. */
typedef struct pfb_init_args3d {
    float* phi_even;
    float* phi_odd;
    pfb_cell3d* cells;
    const pfb_vec3* centres;
    int N;
    int B;
    pfb_layout3d layout;
    float lambda;
    float seed_radius;
    pfb_storage3d storage;
} pfb_init_args3d;

/* pf3d::ScatterArgs3D (kernels.cuh:231-240), 88 bytes. */
typedef struct pfb_scatter_args3d {
    const float* phi;
    pfb_cell3d* cells;
    uint32_t* S;
    uint32_t* global_flags;
    pfb_layout3d layout;
    int N;
    int B;
    pfb_selection3d selection;
    pfb_storage3d storage;
} pfb_scatter_args3d;

/* ---- launchers (reference include/pf3d/kernels.cuh:398-542) ------------- */

/* Measurement of V, centroid, interaction integral, support box, phi_max and
 * (optionally) surface from phi and S, then the recentring plan and the
 * support check; replaces launch_measure_cells_only (kernels.cu:2747). */
int pfb3d_measure_cells_only(const pfb_measure_args3d* args, void* stream);
/* Tumble and velocity of every selected cell; replaces
 * launch_apply_cell_motion (kernels.cu:1739-1788). */
int pfb3d_apply_cell_motion(const pfb_measure_args3d* args, void* stream);
/* Both, in order; replaces launch_measure_cells (kernels.cu:2780). */
int pfb3d_measure_cells(const pfb_measure_args3d* args, void* stream);

/* Moment-free explicit Euler update with recentring and Q5.27 scatter into
 * S_out (when not null). One entry point for all geometries: replaces
 * detail::launch_update_periodic_slab_walk_fast (periodic) and
 * detail::launch_update_tiled_fast (slab and channel). Bit-identical phi
 * and S to those kernels on the same inputs. Requires phi_in != phi_out,
 * S_in != S_out, compute_surface = 0 and tile_pass = ALL. */
int pfb3d_update(const pfb_update_args3d* args, void* stream);

/* The step's measurement, motion and update in one launch (one thread-block
 * cluster per cell holds the brick in shared memory, so each brick is read
 * from HBM once); replaces launch_measure_cells followed by the update
 * launcher of the geometry (reference Sim3D::begin_step/finish_step,
 * src/pf3d/sim.cu:1460-1651). The caller clears update->S_out first. Both
 * records must describe the same system (phi == phi_in, S == S_in, cells,
 * flags, layout, wall and selection). The committed records, phi and S of a
 * step without fatal flags equal those of pfb3d_measure_cells +
 * pfb3d_update; on a step that raises a fatal flag the cells updated before
 * it was raised update normally, so after the repair and restore only the
 * step's global flag counts can differ. PFB_E_CONFIG when the brick edge
 * does not fit (pfb3d_step_cluster returns 0). */
int pfb3d_step_fused(const pfb_measure_args3d* measure, const pfb_update_args3d* update,
                     void* stream);

/* ---- adaptive bricks (reference include/pf3d/brick_classes.hpp,
 * src/pf3d/adaptive_storage.cu, launchers of src/pf3d/kernels.cu) ----------
 * A promoted cell (storage_edge E > B, E a multiple of 8 and at most
 * promoted_edge) lives in its own E^3 cube, promoted_phi[n] (promoted_phi_in
 * and _out for the update); promoted_ids lists the promoted_count promoted
 * cells. The base launchers skip such cells. Per-voxel arithmetic is the base
 * kernels'. */

/* Next tier of a cube of edge `current`: 32 more planes rounded up to a
 * multiple of 16, at most the largest multiple of 8 below `maximum`; 0 when
 * none is larger (reference next_brick_edge). */
int pfb3d_next_brick_edge(int current, int maximum);
/* Smallest centred crop of a cube of edge `current`, not below `minimum`,
 * that keeps 16 spare planes beyond the support box lo3..hi3 on every face,
 * rounded up to a multiple of 16; `current` when none (reference
 * shrink_brick_edge). */
int pfb3d_shrink_brick_edge(int current, int minimum, const int* lo3, const int* hi3);
/* Measurement (moments, support box, recentring plan) of the promoted cubes;
 * replaces launch_measure_promoted (kernels.cu:1413-1427). */
int pfb3d_measure_promoted(const pfb_measure_args3d* args, float* const* promoted_phi,
                           const int* promoted_ids, int promoted_count, int promoted_edge,
                           void* stream);
/* Update of the promoted cubes with their planned shifts and the Q5.27
 * scatter into args->S_out; replaces launch_update_promoted and
 * launch_update_promoted_sharded_fast (kernels.cu:1888-1925). The base pools
 * of args are not used. */
int pfb3d_update_promoted(const pfb_update_args3d* args, float* const* promoted_phi_in,
                          float* const* promoted_phi_out, const int* promoted_ids,
                          int promoted_count, int promoted_edge, void* stream);
/* Q5.27 scatter of the promoted cubes into args->S (k_scatter_promoted). */
int pfb3d_scatter_promoted(const pfb_scatter_args3d* args, float* const* promoted_phi,
                           const int* promoted_ids, int promoted_count, int promoted_edge,
                           void* stream);
/* On a step holding a fatal counter: each promoted cube keeps its accepted
 * field (copied into the output cube and scattered into args->S_out) and its
 * planned shift is dropped (launch_repair_promoted_after_fatal). */
int pfb3d_repair_promoted_after_fatal(const pfb_update_args3d* args,
                                      float* const* promoted_phi_in,
                                      float* const* promoted_phi_out, const int* promoted_ids,
                                      int promoted_count, int promoted_edge, void* stream);
/* rejected[n] |= 1 unless cube n may be cropped to candidate_edges[n]
 * (0: no candidate): every voxel finite and every voxel outside the retained
 * cube's inner 8-plane guard band an exact zero (k_check_promoted_crops). */
int pfb3d_check_promoted_crops(float* const* promoted_phi, const pfb_cell3d* cells,
                               const int* candidate_edges, uint32_t* rejected, int N,
                               int base_edge, void* stream);
/* Cluster size (CTAs per cell) of the fused step for brick edge B, 0 when
 * the brick does not fit it. The measurement launchers use the same cluster
 * size, so both paths sum the moments in the same grouping. */
int pfb3d_step_cluster(int B);
/* Status bits of the 3D kernels' bounded waits since the last clear: bit 0
 * measurement plane wait, bit 1 measurement fold, bit 2 update plane wait,
 * bit 4 fused-step plane wait, bit 5 fused-step fold, bit 6 fused-step
 * broadcast. 0 on a healthy device. */
int pfb3d_device_status(unsigned* out, int clear);

/* launch_clear_S (kernels.cu:2704). */
int pfb3d_clear_S(uint32_t* S, const pfb_layout3d* layout, void* stream);
/* launch_repair_after_fatal: restores phi_out and rebuilds S_out from phi_in
 * when a fatal global flag is set; otherwise returns at once. */
int pfb3d_repair_after_fatal(const pfb_update_args3d* args, void* stream);
/* launch_finalize_origins: origin += pending shift for cells without a fatal
 * bit. */
int pfb3d_finalize_origins(pfb_cell3d* cells, int N, uint32_t* global_flags, void* stream);
/* launch_restore_cells_after_fatal. */
int pfb3d_restore_cells_after_fatal(pfb_cell3d* cells, const pfb_cell3d* accepted, int N,
                                    const uint32_t* global_flags, uint32_t* support_requests,
                                    void* stream);
/* launch_advance_step: ++*step unless a fatal flag is set. */
int pfb3d_advance_step(uint64_t* step, const uint32_t* global_flags, void* stream);
/* launch_initialize_spheres (kernels.cu:1071-1122). */
int pfb3d_initialize_spheres(const pfb_init_args3d* args, void* stream);
/* launch_scatter_current: S += q(phi) of every selected cell. */
int pfb3d_scatter_current(const pfb_scatter_args3d* args, void* stream);

/* ---- host helpers -------------------------------------------------------- */

/* Bisection for the tanh-sphere seed radius whose discrete sum of phi^2 in a
 * centred brick equals 4/3 pi R^3 (reference include/pf3d/reference.hpp:
 * 712-745). Writes the radius; returns PFB_OK or PFB_E_ARG. */
int pfb3d_calibrate_seed_radius(double radius, double lambda, int brick_edge,
                                double* seed_radius, double* measured_volume);
/* Smallest multiple of 8 covering the diffuse sphere plus the safety margin
 * (reference include/pf3d/params.cuh:130-166). */
int pfb3d_automatic_brick_edge(double radius, double lambda);
/* Initial polarity on the unit sphere (planar != 0: in the substrate plane)
 * from the POLI Philox domain (reference include/pf3d/rng.cuh:41-60). */
void pfb3d_initial_polarity(int64_t global_id, uint64_t stream, int planar, double* out3);
/* Lognormal active speed from the VALO domain (rng.cuh:65-78). */
double pfb3d_initial_active_speed(int64_t global_id, uint64_t seed, double median,
                                  double sigma);
/* Soft identities (reference include/pf3d/initializer.hpp:17-95,
 * soft_id_membership): out[i] = 1 for the round(fraction n) ids a
 * Philox-driven Fisher-Yates shuffle of 0..n-1 puts first (domain "SFT3",
 * bounded draws by rejection), 0 otherwise. Independent of placement. */
int pfb3d_soft_membership(int n, double fraction, uint64_t seed, uint8_t* out);
/* Tumble draw of step `step` (rng.cuh:80-150): returns 1 on an event and
 * writes the new polarity, else 0. */
int pfb3d_tumble(uint64_t step, int64_t global_id, uint64_t stream, double probability,
                 int planar, double* out3);

/* ---- host driver ---------------------------------------------------------- */

/* Model and run parameters of the 3D driver (the subset of the reference's
 * SimParams3D, include/pf3d/params.cuh:257-330, that the update reads). */
typedef struct pfb_params3d {
    int Nx, Ny, Nz;
    uint32_t boundary_flags;
    int num_cells;
    int B; /* 0: automatic brick edge */
    double dt;
    double lambda;
    double target_radius;
    double kappa;
    double mu;
    double xi;
    double tau;
    double v_A;
    double gamma;
    double v_A_sigma;
    double aging_time;
    double wall_kappa; /* channel only */
    double wall_width; /* channel only */
    int channel_height; /* channel only */
    int channel_padding; /* channel only */
    uint64_t seed;
    uint64_t polarity_seed;
    int full_moment_every;
    /* soft cells (reference gamma_cancer / cancer_fraction): round(
     * soft_fraction N) identities drawn without replacement take gamma_soft */
    double gamma_soft;
    double soft_fraction;
    /* storage of the base phi pools: 0 binary32 (the reference's layout),
     * 1 binary16, 2 bfloat16, both with binary32 arithmetic and stochastic
     * rounding of every stored value (seeded by `seed`); promoted cubes stay
     * binary32, and fields are read and written as binary32 */
    int phi_storage;
} pfb_params3d;

typedef struct pfb_sim3d pfb_sim3d;

/* Fresh start from cell centres (world coordinates, substrate centres at
 * z = -0.5 as in the reference; channel centres in slit coordinates, moved
 * to array coordinates as z + padding - 1/2 in binary32 as the reference
 * does); N = p->num_cells entries. */
pfb_sim3d* pfb_sim3d_create(const pfb_params3d* p, const pfb_vec3* centres, int device);

/* Storage modes (reference StorageMode3D, --memory-mode): throughput keeps
 * two phi pools and two aggregates; balanced one pool, two aggregates and
 * scratch bricks the update writes before committing each healthy cell;
 * compact one pool and one aggregate rebuilt after every update. Fields,
 * aggregates and flags are the same in every mode. AUTO takes throughput when
 * it fits in 90 % of the free device memory, else balanced, else compact. */
enum {
    PFB3D_MEMORY_AUTO = -1,
    PFB3D_MEMORY_THROUGHPUT = 0,
    PFB3D_MEMORY_BALANCED = 1,
    PFB3D_MEMORY_COMPACT = 2
};
/* pfb_sim3d_create / _create_from_state with a storage mode and a number of
 * scratch bricks (0: two per SM, at most N). The plain functions use AUTO. */
pfb_sim3d* pfb_sim3d_create_ex(const pfb_params3d* p, const pfb_vec3* centres, int device,
                               int memory_mode, int scratch_slots);
pfb_sim3d* pfb_sim3d_create_from_state_ex(const pfb_params3d* p, const pfb_cell3d* cells,
                                          const float* phi, long long step, int device,
                                          int memory_mode, int scratch_slots);
int pfb_sim3d_memory_mode(const pfb_sim3d* s);
int pfb_sim3d_scratch_slots(const pfb_sim3d* s);
/* The in-place update of the balanced and compact modes (reference
 * launch_update_inplace / launch_update_inplace_fast): the selected cells,
 * scratch_slots at a time, update from the single pool args->phi_in into the
 * scratch bricks (scratch_slots * B^3 floats), then each cell without a fatal
 * flag is copied back (with one, its field stays and its planned shift is
 * dropped). args->phi_out is ignored; args->S_out may be null. */
int pfb3d_update_inplace(const pfb_update_args3d* args, float* scratch, int scratch_slots,
                         void* stream);
/* Restart from cell records and fields (x fastest) of step `step`, as the
 * reference's Sim3D::init_checkpoint does (src/pf3d/sim.cu:794-885): the
 * records and fields become the current state, the aggregate is rebuilt and
 * the cells are measured once (surface included, no tumble). Ids must be
 * 0..N-1. phi packs each cell's field in cell order: B^3 values for a base
 * cell (storage_edge 0 or B), E^3 for a cell on a promoted cube of edge
 * E = storage_edge > B (N * B^3 when no cell is promoted). */
pfb_sim3d* pfb_sim3d_create_from_state(const pfb_params3d* p, const pfb_cell3d* cells,
                                       const float* phi, long long step, int device);
void pfb_sim3d_destroy(pfb_sim3d* s);
/* Measure the current state (moments, surface, support, recentring plan)
 * and set velocities without a tumble, as the reference does before output
 * and before writing a checkpoint (Sim3D::ensure_measurements ->
 * refresh_measurements(false, true), src/pf3d/sim.cu:1301-1377, 2045-2047). */
int pfb_sim3d_measure_current(pfb_sim3d* s);
/* Advance by `steps` accepted steps (the reference's begin_step/finish_step
 * sequence per step, synchronising at the end and at every multiple of 1024
 * accepted steps). A step on which a cell's support reaches its brick is
 * rolled back and the cell's brick grows to the next tier (reference
 * Sim3D::recover_support_exhaustion, src/pf3d/sim.cu:1653-1727), then the
 * step is retried; promoted cubes are cropped back where their support
 * allows at every multiple of 1024 accepted steps
 * (Sim3D::compact_promoted_fields). Returns early, with the flags set, at any
 * other fatal flag or when no larger cube fits the domain. */
int pfb_sim3d_advance(pfb_sim3d* s, int steps);
/* 1: one fused launch per step (pfb3d_step_fused), 0 (default): the
 * separate measurement, motion and update launches. */
int pfb_sim3d_set_fused(pfb_sim3d* s, int fused);
int pfb_sim3d_fused(const pfb_sim3d* s);
/* Replay pairs of steps without a surface pass from a CUDA graph (default
 * 1). */
int pfb_sim3d_set_graph(pfb_sim3d* s, int use_graph);
/* Visit order of the cells in every launch: 1 (default) the Morton order of
 * the brick centres, refreshed every 4096 steps, so that clusters in flight
 * share aggregate words in L2; 0 the slot order. Results do not depend on
 * it. */
int pfb_sim3d_set_order(pfb_sim3d* s, int morton);
int pfb_sim3d_sync(pfb_sim3d* s);
int pfb_sim3d_brick(const pfb_sim3d* s);
long long pfb_sim3d_step(const pfb_sim3d* s);
int pfb_sim3d_get_cells(pfb_sim3d* s, pfb_cell3d* out);
/* N * B^3 floats of the base pool's current field (the slot of a promoted
 * cell is not its field: pfb_sim3d_get_packed). */
int pfb_sim3d_get_phi(pfb_sim3d* s, float* out);
/* Length and values of the current fields packed in cell order, each cell on
 * its own cube (B^3 or E^3 values), as the PF3D checkpoint stores them. */
int pfb_sim3d_packed_words(pfb_sim3d* s, unsigned long long* words);
int pfb_sim3d_get_packed(pfb_sim3d* s, float* out);
/* Adaptive bricks: cells currently on promoted cubes, the largest cube edge
 * the domain allows, and the support-exhaustion recoveries so far. */
int pfb_sim3d_promoted_count(const pfb_sim3d* s);
int pfb_sim3d_max_edge(const pfb_sim3d* s);
long long pfb_sim3d_recoveries(const pfb_sim3d* s);
/* nz * ny * pitch_x words of the current aggregate. */
int pfb_sim3d_get_S(pfb_sim3d* s, uint32_t* out);
int pfb_sim3d_get_flags(pfb_sim3d* s, uint32_t* out10);
int pfb_sim3d_layout(const pfb_sim3d* s, pfb_layout3d* out);
/* Device pointers and coefficients of the current step, as the reference's
 * Sim3D would pass them (for callers that drive the launchers directly). */
int pfb_sim3d_update_args(pfb_sim3d* s, pfb_update_args3d* out);
int pfb_sim3d_measure_args(pfb_sim3d* s, pfb_measure_args3d* out);
void* pfb_sim3d_stream(const pfb_sim3d* s);
/* Device time of `steps` steps after `warmup`, in ms (CUDA events). */
int pfb_sim3d_bench(pfb_sim3d* s, int warmup, int steps, double* ms);

/* Channel wall diagnostics of the current field (reference
 * k_measure_wall_diagnostics, src/pf3d/kernels.cu): sets each cell's
 * wall_overlap = sum of phi^2 psi_w^2(z) and outside_slit_volume = sum of
 * phi^2 outside the slit over its in-domain voxels, psi_w^2 the binary32
 * wall profile. Hard-wall channel only. */
int pfb_sim3d_measure_wall(pfb_sim3d* s);

/* Invariant check (reference Sim3D::verify, src/pf3d/sim.cu:2078-2137, the
 * --strict cadence): measures the current state, then per cell recomputes
 * V from the in-domain voxels and counts support voxels (|phi| > 1e-5) on a
 * brick face, outside the domain or on the slab's top plane.
 * *max_rel_V = max |V recomputed - V of the record| / max(1, V recomputed),
 * *edge_voxels = their total, *max_S = the largest aggregate word.
 * Returns PFB_E_STATE for a non-finite sample. */
int pfb_sim3d_verify(pfb_sim3d* s, double* max_rel_V, uint32_t* max_S,
                     unsigned long long* edge_voxels);

/* PFB3D boundary recorder (reference src/pf3d/boundary_output.cu, file
 * layout common/boundary_format_3d.h): creates a NEW file at `path` with its
 * 128-byte header. Each capture appends a frame of the current step: per
 * cell a 64-byte record and the 2x2 squares that phi = 1/2 crosses in the
 * cell's (B+2)^2 projected plane (zero ring around the x/y faces), binary32
 * corners in ascending plane order. The projection is the maximum over the
 * brick's in-domain z planes (PFB3D_PROJECTION_MAXIMUM) or the plane on the
 * substrate (PFB3D_PROJECTION_BASAL, substrate slab only). Close with
 * `complete` != 0 writes the end record; a file closed otherwise (or by
 * pfb_sim3d_destroy) stays unterminated, marking an incomplete run.
 * `compress` (zstd) is refused: this build has no zstd. */
#define PFB3D_PROJECTION_BASAL 1
#define PFB3D_PROJECTION_MAXIMUM 2
int pfb_sim3d_boundary_open(pfb_sim3d* s, const char* path, int projection, long long interval,
                            int compress);
int pfb_sim3d_boundary_capture(pfb_sim3d* s);
int pfb_sim3d_boundary_close(pfb_sim3d* s, int complete);

#ifdef __cplusplus
}
#endif

#endif /* PFB200_3D_H */
