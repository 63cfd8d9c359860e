/*
 * pfb200.h -- C ABI of the B200-native active multi-phase-field cell update.
 *
 * Every entry point takes plain pointers and sizes. The two records below are
 * byte-for-byte the records the reference passes between its host driver and
 * its 2D step kernel, so a caller that already owns those buffers (the
 * reference's `Sim`, or a checkpoint loader) can hand them over unchanged:
 *
 *   pfb_cell2d       == pf::CellState   (reference include/kernels.cuh:27-57)
 *   pfb_step_args2d  == pf::StepArgs    (reference include/kernels.cuh:74-116)
 *
 * Conventions (reference include/kernels.cuh:219-225, src/sim.cu:207-230):
 *   - the caller owns every device buffer; no launcher allocates;
 *   - launchers return 0 on success and a negative PFB_E* code when the launch
 *     contract is violated (the reference 3D launchers return false in the same
 *     situations, src/pf3d/kernels.cu:2747-2787);
 *   - numerical failures never abort a kernel: they raise the sticky u32
 *     counters of the `flags` array (PFB_FLAG_*), exactly as the reference does
 *     (include/params.cuh:433-495);
 *   - all work is issued on the caller's stream; nothing synchronises.
 */
#ifndef PFB200_H
#define PFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define PFB_OK 0
#define PFB_E_ARG (-1)        /* null pointer, bad size or alignment       */
#define PFB_E_CUDA (-2)       /* a CUDA runtime call failed                */
#define PFB_E_CONFIG (-3)     /* unsupported configuration (e.g. cluster)  */
#define PFB_E_STATE (-4)      /* object used in the wrong state            */
#define PFB_E_NOMEM (-5)      /* host or device allocation failed          */

/* ---- sticky device flags (indices into the u32 flags[8] array) -------
 * reference include/params.cuh:434-445. All but SUPPORT_CLIP are fatal. */
#define PFB_FLAG_S_OVERFLOW 0
#define PFB_FLAG_Q_CLAMP 1
#define PFB_FLAG_SUPPORT_CLIP 2
#define PFB_FLAG_CLASS_EXHAUSTED 3
#define PFB_FLAG_S_NEGATIVE 4
#define PFB_FLAG_NONFINITE 5
#define PFB_FLAG_V_NONPOS 6
#define PFB_FLAG_CLASS_UNSUPPORTED 7
#define PFB_FLAG_COUNT 8

/* ---- fixed 2D tile geometry (reference include/params.cuh:121-147) ---- */
#define PFB_TILE_PITCH 288
#define PFB_TILE_AREA (288 * 288)
#define PFB_NUM_CLASSES 6

/* Runtime velocity-observer accumulator carried inside the cell record
 * (reference common/velocity_moments.h:24-27): time integrals of the active
 * velocity (q[0..1]), the interaction velocity (q[2..3]) and the rounding of
 * the stored binary32 velocity (q[4..5]), and the observed step count.
 * Updated by the observed steps only. */
typedef struct pfb_advection_accum {
    double q[6];
    unsigned long long count;
} pfb_advection_accum;

/* Per-cell spatial-observer state, 240 B (reference
 * common/velocity_moments.h:29-40, pf::velocity::MomentAccum): q[12] are
 * the PFVMOM4 integral channels (active, interaction, interfacial,
 * overlap, area, advection correction; x/y pairs), held[] the interfacial
 * and overlap rates of the last spatial sample then the normalised
 * same-cell neighbour overlaps, and the sampling bookkeeping. */
typedef struct pfb_moment_accum2d {
    double q[12];
    unsigned long long count;
    double held[6];
    unsigned long long spatial_count;
    unsigned long long last_sample;
    unsigned long long last_interval;
    double last_totals[4];
    double correction[4];
} pfb_moment_accum2d;

/* Velocity observation of a step (reference include/kernels.cuh:216,
 * pf::VelocityStep). */
#define PFB_VELOCITY_DISABLED 0
#define PFB_VELOCITY_ADVECTION 1 /* advection accumulators in the cells   */
#define PFB_VELOCITY_SPATIAL 2   /* + spatial rates into args->moments    */

/* Per-cell state, 192 B, 64-B aligned (reference include/kernels.cuh:27-57). */
typedef struct pfb_cell2d {
    int32_t gx0, gy0;          /* global coords of window pixel (0,0)   */
    uint8_t cls;               /* shape class of the field to be read   */
    uint8_t cls_written[2];    /* class last written into phi[parity]   */
    uint8_t pad0;
    int32_t global_id;         /* Philox key; stable across reordering  */
    float gamma, v_A, R_tgt;
    float theta;               /* polarity angle                        */
    double V;                  /* sum phi^2 of the field to be read     */
    double Cx, Cy;             /* sum phi^2 x, sum phi^2 y (window)     */
    double perim;              /* full-moment steps only                */
    int32_t bb_lo_x, bb_hi_x, bb_lo_y, bb_hi_y;
    float vx, vy;
    double Ix, Iy;             /* interaction integral                  */
    uint32_t promote_ctr;
    uint32_t shift_ctr;
    uint32_t tumble_ctr;
    float phi_max;
    uint32_t reserved[2];      /* [0] fallback used, [1] no-margin steps */
    pfb_advection_accum advection;
    uint32_t reserved_unused;
    float M_pf;                /* passive Allen-Cahn mobility           */
}
#if defined(__GNUC__) || defined(__CUDACC__)
__attribute__((aligned(64)))
#endif
pfb_cell2d;

/* Arguments of one 2D step launch (reference include/kernels.cuh:74-116).
 * Step counters and cursors are device-resident so a captured CUDA graph can
 * be replayed; `perm` may be null (identity order); `moments` (an array of
 * N pfb_moment_accum2d) is read only by pfb_step2d_launch_observed with
 * PFB_VELOCITY_SPATIAL and must be null otherwise. */
typedef struct pfb_step_args2d {
    const float* phi_in;
    float* phi_out;
    const uint32_t* S_rd;
    uint32_t* S_sc;
    uint32_t* S_cl;
    pfb_cell2d* cell;
    uint8_t* cell_cls;
    const uint32_t* perm;
    unsigned long long* cursor_use;
    unsigned long long* cursor_clear;
    const unsigned long long* step_rd;
    unsigned long long* step_wr;
    uint32_t* flags;
    void* moments;
    double physical_dt;
    int N;
    int L;
    int P;
    int parity_out;
    float dt;
    double A0;
    double vol_scale;
    float bulk_scale;
    float rep_coeff;
    float mot_coeff;
    unsigned long long seed;
    unsigned long long polarity_seed;
    double p_tumble;
    int full_moment_every;
    unsigned long long clear_ahead_words;
} pfb_step_args2d;

/* Simulation parameters (reference include/params.cuh:499-530, SimParams),
 * as plain C. Only the fields the update consumes are carried. */
typedef struct pfb_params2d {
    int L;                        /* domain side (Nx == Ny)                */
    int num_cells;
    double dt;
    double lambda;
    double target_radius;
    double kappa;
    double mu;
    double xi;
    double tau;
    double v_A;
    double gamma_normal;
    double gamma_cancer;
    double cancer_fraction;
    double v_A_sigma;
    double phase_field_mobility;
    unsigned long long seed;
    unsigned long long polarity_seed; /* 0 follows seed                  */
    int full_moment_every;
    /* phi pool storage of the host driver: 0 binary32 (the reference's),
     * 1 binary16, 2 bfloat16 (binary32 arithmetic, stochastic rounding on
     * store; classes 0-3 only) -- no reference counterpart */
    int phi_storage;
} pfb_params2d;

/* Compact trajectory record (reference include/kernels.cuh:60-70). */
typedef struct pfb_traj_cell2d {
    int32_t global_id;
    int32_t cls;
    float cx, cy;
    float vx, vy;
    float theta;
    float volume;
    float perim;
    float gamma, v_A;
    float phi_max;
} pfb_traj_cell2d;

/* ======================================================================
 * Library information
 * ==================================================================== */

/* Version string of this library. */
const char* pfb_version(void);
/* Text of the last error raised on the calling host thread ("" if none). */
const char* pfb_last_error(void);
/* sizeof() of the ABI records, for binding-layer layout checks:
 * which = 0 cell2d, 1 step_args2d, 2 params2d, 3 traj_cell2d. */
size_t pfb_sizeof(int which);

/* ======================================================================
 * 2D step -- replaces pf::launch_step / configure_k_step_smem / k_step_grid
 * (reference include/kernels.cuh:219-225, src/kernels.cu:1304-1363)
 * ==================================================================== */

/* Configure the dynamic shared-memory opt-in of every step kernel on the
 * current device. Idempotent; called implicitly by pfb_step2d_launch. */
int pfb_step2d_configure(void);

/* Number of CTAs the step launch uses for N cells with `cluster` CTAs per
 * cell (cluster = 0 selects the default 2). Replaces k_step_grid(). */
int pfb_step2d_grid(int num_cells, int cluster);

/* One full step for every cell: tumble, interaction integral, Euler update,
 * recentring store, Q5.27 scatter into S_sc, FP64 moments, and clearing of
 * S_cl (clear_ahead_words words). `cluster` is the number of CTAs of the
 * thread-block cluster that cooperates on one cell (2, 4 or 8; 0 = default
 * 2).
 * Returns PFB_E_ARG for a null buffer, a phi pool or S slot not 16-byte
 * aligned, L not larger than 286, or a non-null `moments`. */
int pfb_step2d_launch(const pfb_step_args2d* args, int cluster, void* stream);

/* As pfb_step2d_launch with an explicit kernel variant (0 = default, 1 = one
 * thread-block cluster per cell, the only variant of this version). */
int pfb_step2d_launch_ex(const pfb_step_args2d* args, int cluster, int variant,
                         void* stream);

/* The step with a velocity observer fused in (reference launch_step's
 * VelocityStep argument, include/kernels.cuh:216-225, and the observer
 * specialisations of include/fused_moments.cuh): PFB_VELOCITY_ADVECTION
 * integrates the active, interaction and rounding velocities into each
 * cell's `advection` record; PFB_VELOCITY_SPATIAL additionally closes the
 * held-rate interval of args->moments and measures new interfacial and
 * overlap rates (FP64) from the same pass over phi^n. The field and every
 * other cell field come out bit-identical to the unobserved step. binary32
 * pools only. */
int pfb_step2d_launch_observed(const pfb_step_args2d* args, int cluster, int observation,
                               void* stream);

/* Independent dense observer (reference src/velocity_moments.cu,
 * launch_velocity_moments): adds physical_dt times the twelve velocity
 * channels of the field args->phi_in to out[n].q and counts the step. One
 * CTA per cell; shares no reduction with the step. */
int pfb_velocity_moments2d(const pfb_step_args2d* args, pfb_moment_accum2d* out,
                           double physical_dt, void* stream);

/* Library status word kept in device memory: bit 0 is set when a CTA of the
 * step gave up waiting for its staged band, bit 1 when a step cluster gave up
 * waiting for a reduction, bit 2 when a set-up pass (initial moments,
 * invariant check) gave up waiting for its cluster fold (bounded waits that
 * are never expected to run out). `clear` != 0 resets it after reading. */
int pfb_device_status(unsigned* out, int clear);

/* ======================================================================
 * 2D initialisation and diagnostics -- replace k_init_tiles,
 * k_init_moments, k_scatter_all, k_zero_u32, k_verify_cells, k_verify_S,
 * k_pack_traj (reference include/kernels.cuh:185-207)
 * ==================================================================== */

/* Seed tanh disks into the class window of each tile of both pools and set
 * gx0/gy0/cls/cls_written (reference src/kernels.cu:1050-1094). */
int pfb_init_tiles2d(float* phi_a, float* phi_b, pfb_cell2d* cell,
                     const uint8_t* cls, int N, int L, const float* seed_cx,
                     const float* seed_cy, float radius_eff, float kappa_iface,
                     void* stream);
/* V, Cx, Cy, support box and phi_max of each cell's window (reference
 * src/kernels.cu:1098-1165). */
int pfb_init_moments2d(pfb_cell2d* cell, const uint8_t* cls, const float* phi,
                       int N, void* stream);
/* Build the Q5.27 aggregate S from a phi pool (reference
 * src/kernels.cu:1167-1190). S must be cleared first. */
int pfb_scatter_all2d(const float* phi, const pfb_cell2d* cell,
                      const uint8_t* cls, uint32_t* S, int N, int L, int P,
                      uint32_t* flags, void* stream);
/* Clear n words. */
int pfb_zero_u32(uint32_t* p, size_t n, void* stream);
/* Recompute each cell's V and the largest |phi| outside its window
 * (reference src/kernels.cu:1193-1232). */
int pfb_verify_cells2d(const float* phi, const pfb_cell2d* cell,
                       const uint8_t* cls, int N, double* out_V,
                       float* out_outside_max, void* stream);
/* max over an S buffer into *out_max (must be zeroed by the caller). */
int pfb_verify_S(const uint32_t* S, size_t n, uint32_t* out_max, void* stream);
/* Pack per-cell observables (reference src/kernels.cu:1242-1265). */
int pfb_pack_traj2d(const pfb_cell2d* cell, const uint8_t* cls,
                    pfb_traj_cell2d* out, int N, int L, void* stream);

/* ======================================================================
 * Host-side helpers shared with the reference's initialisers
 * ==================================================================== */

/* Philox4x32-10 (reference common/philox.cuh:32-59). out[4]. */
void pfb_philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                       uint32_t k0, uint32_t k1, uint32_t* out);
/* 53-bit uniform from two words (reference common/philox.cuh:62-67). */
double pfb_philox_uniform53(uint32_t a, uint32_t b);
/* Q5.27 encoding of phi^2 (reference include/params.cuh:103-111). */
uint32_t pfb_q_of(float phi);
/* Sequential periodic placement with minimum separation `min_sep`
 * (reference include/palmieri_initializer.hpp:66-103). Returns 0 or
 * PFB_E_ARG; x, y receive n binary32 centres. */
int pfb_palmieri_centres(int n, double side, double min_sep,
                         unsigned long long seed, float* x, float* y);
/* Default grid-and-jitter centres (reference src/sim.cu:107-129). */
int pfb_grid_jitter_centres(int n, int side, unsigned long long seed, float* x,
                            float* y);
/* Initial polarity angle (reference include/kernels.cuh:153-158). */
float pfb_ic_theta(int32_t gid, unsigned long long stream);
/* Lognormal per-cell speed (reference include/kernels.cuh:161-172). */
double pfb_ic_v_A(int32_t gid, unsigned long long seed, double v_A,
                  double sigma);
/* Domain side for n cells of radius R at packing rho
 * (reference include/params.cuh:568-574). */
int pfb_domain_side_for(int n, double radius, double rho);
/* Step arguments' coefficients from params (reference src/sim.cu:605-616):
 * fills dt, A0, vol_scale, bulk_scale, rep_coeff, mot_coeff, seed,
 * polarity_seed, p_tumble, full_moment_every, physical_dt. */
int pfb_fill_coefficients2d(const pfb_params2d* p, pfb_step_args2d* a);

/* ======================================================================
 * Host driver -- the reference's `Sim` (reference include/sim.cuh:58-152)
 * behind an opaque handle. Owns its device buffers.
 * ==================================================================== */
typedef struct pfb_sim2d pfb_sim2d;

/* Allocate device state for params on `device`; centres x/y (n floats) seed
 * the tanh disks. Returns null on failure (see pfb_last_error). */
pfb_sim2d* pfb_sim2d_create(const pfb_params2d* p, const float* cx,
                            const float* cy, int device);
/* Build from an existing host state (checkpoint-style): cells (N records),
 * phi (N * 288 * 288 floats holding phi^step), at step `step`. S is rebuilt
 * on the device. */
pfb_sim2d* pfb_sim2d_create_from_state(const pfb_params2d* p,
                                       const pfb_cell2d* cells,
                                       const float* phi, long long step,
                                       int device);
void pfb_sim2d_destroy(pfb_sim2d* s);
/* Tuning knobs: cluster CTAs per cell (2/4/8), kernel variant and CUDA-graph
 * use. Variants: 0 (default) and 1 scatter the Q5.27 aggregate with
 * non-returning adds on the common path and detect S_overflow exactly through
 * per-bin bounds the driver keeps (recounting only a bin whose bound reaches
 * 2^32); 2 uses returning adds that test every add (pfb_step2d_launch's
 * scatter). Results, flags included, are identical. */
int pfb_sim2d_set_cluster(pfb_sim2d* s, int cluster);
int pfb_sim2d_set_variant(pfb_sim2d* s, int variant);
/* Bins recounted exactly so far by variants 0/1 (bins whose bound reached
 * 2^32; normally none). No reference counterpart: a diagnostic. */
int pfb_sim2d_scatter_recounts(pfb_sim2d* s, unsigned int* out);
int pfb_sim2d_set_graph(pfb_sim2d* s, int use_graph);
/* Cell visit order (reference src/main.cu:491-492 --morton, src/sim.cu:
 * 284-296, 649-653). PFB_VISIT_MORTON orders the clusters by the Z-order
 * index of each cell's centroid pixel, re-sorted on the device every sixth
 * step; it changes no result. One CTA sorts the keys in shared memory, so
 * N is limited (PFB_E_CONFIG above it; the order is then left unchanged).
 * pfb_sim2d_visit_order copies the current order (N indices) to `out`. */
#define PFB_VISIT_LAUNCH 0
#define PFB_VISIT_MORTON 1
int pfb_sim2d_set_visit_order(pfb_sim2d* s, int order);
int pfb_sim2d_visit_order(pfb_sim2d* s, uint32_t* out);
/* Advance `steps` steps on the simulator's stream (asynchronous). */
int pfb_sim2d_advance(pfb_sim2d* s, long long steps);
/* Wait for the simulator's stream. */
int pfb_sim2d_sync(pfb_sim2d* s);
long long pfb_sim2d_step(const pfb_sim2d* s);
int pfb_sim2d_side(const pfb_sim2d* s);
int pfb_sim2d_pitch(const pfb_sim2d* s);
int pfb_sim2d_num_cells(const pfb_sim2d* s);
/* Copies (synchronous) of the current state to host memory. */
int pfb_sim2d_get_cells(pfb_sim2d* s, pfb_cell2d* out);
int pfb_sim2d_get_phi(pfb_sim2d* s, float* out);      /* N*288*288 floats */
int pfb_sim2d_get_S(pfb_sim2d* s, uint32_t* out);     /* L*P words       */
int pfb_sim2d_get_flags(pfb_sim2d* s, uint32_t* out); /* 8 words         */
/* Replace the whole state from host memory (pinned or pageable) on the
 * simulator's stream; S is rebuilt from phi. */
int pfb_sim2d_set_state(pfb_sim2d* s, const pfb_cell2d* cells,
                        const float* phi, long long step);
/* Pack the per-cell trajectory record into host memory `out` (N records). */
int pfb_sim2d_pack_traj(pfb_sim2d* s, pfb_traj_cell2d* out);
/* Advance `steps` steps and, after every `every`-th step of this call, pack
 * the trajectory records (as pfb_sim2d_pack_traj) and copy them to frame
 * k % frames of `ring` (frames x N records), k = 0, 1, ... counting this
 * call's records: the driver loop of the reference's trajectory output
 * (src/sim.cu:864-930, --trajectory-interval) without a host wait per record.
 * Returns once the work is queued on the simulator's stream; the ring holds
 * the frames after pfb_sim2d_sync. `ring` should be page-locked host memory
 * for the copies to run asynchronously. Six-step graphs replace single
 * launches where no record falls inside the six steps. PFB_E_ARG for a null
 * ring, every < 1, frames < 1 or steps < 0. */
int pfb_sim2d_advance_record(pfb_sim2d* s, long long steps, int every, pfb_traj_cell2d* ring,
                             int frames);
/* In-memory device checkpoint (no reference counterpart): save copies the
 * current pool, cells, aggregate and flags into buffers of the system
 * (allocated on the first save); restore returns to that step exactly as a
 * set_state of the saved state would. */
int pfb_sim2d_save(pfb_sim2d* s);
int pfb_sim2d_restore(pfb_sim2d* s);
/* Timed benchmark in the manner of Sim::bench (reference src/sim.cu:1006):
 * `warmup` untimed steps, then `steps` steps timed with CUDA events on the
 * simulator's stream. Writes ms per step. */
int pfb_sim2d_bench(pfb_sim2d* s, int warmup, int steps, double* ms_per_step);
/* Device pointers for callers that drive kernels themselves. */
int pfb_sim2d_step_args(pfb_sim2d* s, pfb_step_args2d* out);

/* PFVMOM4 velocity-component recorder (reference src/velocity_output.cu,
 * include/velocity_sampling.hpp; file layout common/velocity_format.h):
 * opens a NEW file at `path` (an existing one is refused) and writes the
 * 56-byte header and the frame of the current step. While open, every step
 * taken by pfb_sim2d_advance is observed: spatially on the first step, on
 * the `dense_start` steps that follow the open and on steps that are
 * multiples of `spatial_stride` (1..1000), by advection otherwise; with
 * `reference` != 0 the dense independent observer runs before every step
 * instead. Steps are launched one by one while a recorder is open. */
int pfb_sim2d_velocity_open(pfb_sim2d* s, const char* path, int spatial_stride,
                            long long dense_start, int reference);
/* Append the frame of the current step (int64 step, N x 26 float64). */
int pfb_sim2d_velocity_capture(pfb_sim2d* s);
/* Step of the last frame written, -1 when none is open. */
long long pfb_sim2d_velocity_last_frame(const pfb_sim2d* s);
int pfb_sim2d_velocity_close(pfb_sim2d* s);

/* Invariant check of the current state (reference Sim::verify,
 * src/sim.cu:817-850, the --strict cadence): *max_rel_V = max over cells of
 * |V recomputed from phi - V of the record| / max(1e-12, |V|), *max_outside =
 * max |phi| of a tile outside its class window, *max_S = the largest word of
 * the current aggregate. binary32 pools only. */
int pfb_sim2d_verify(pfb_sim2d* s, double* max_rel_V, float* max_outside, uint32_t* max_S);

/* PFB boundary recorder (reference src/boundary.cu, common/boundary_format.h):
 * creates a NEW file at `path` and writes its 72-byte header (level 1/2,
 * the frame `interval` stored for readers). Each capture appends a frame of
 * the current step: per cell a 40-byte record (id, tile origin, periodic
 * centroid, gamma, mobility, active speed, target radius, square count) and
 * the 2x2 squares of its tile that phi = 1/2 crosses, binary32 corners, in
 * ascending tile order. Frames are written by a background thread; close
 * writes the end record. `compress` (zstd) is refused: this build has no
 * zstd. binary32 pools only. */
int pfb_sim2d_boundary_open(pfb_sim2d* s, const char* path, long long interval, int compress);
int pfb_sim2d_boundary_capture(pfb_sim2d* s);
int pfb_sim2d_boundary_close(pfb_sim2d* s);
void* pfb_sim2d_stream(pfb_sim2d* s);

/* ---- batched ensemble (no reference counterpart) --------------------------
 * R independent 2D systems, each with its own lattice side, cell count,
 * seeds and buffers, advanced together by ONE kernel launch per step
 * (k_step2d_batch: system r is served by its own contiguous range of
 * clusters), six steps per CUDA graph. Each system evolves exactly as it
 * would alone: the per-cell code is the same kernel body. */
typedef struct pfb_ens2d pfb_ens2d;

/* params[r], cx[r], cy[r] (params[r].num_cells centres each) describe
 * system r; every system gets a fresh start as pfb_sim2d_create. All systems
 * must share one phi_storage (one launch serves them all); 16-bit pools
 * limit the cluster to 2 or 4 CTAs per cell. */
pfb_ens2d* pfb_ens2d_create(int R, const pfb_params2d* params, const float* const* cx,
                            const float* const* cy, int device);
void pfb_ens2d_destroy(pfb_ens2d* e);
int pfb_ens2d_num_systems(const pfb_ens2d* e);
int pfb_ens2d_set_cluster(pfb_ens2d* e, int cluster);
/* Times `steps` steps with clusters of 2, 4 and 8 CTAs per cell (2 and 4 with
 * 16-bit pools) and keeps the fastest (the ensemble's autotuner; the timed
 * steps advance the systems). */
int pfb_ens2d_autotune(pfb_ens2d* e, int steps, int* chosen);
int pfb_ens2d_advance(pfb_ens2d* e, int steps);
/* pfb_sim2d_advance_record for every system at once: frame k of `ring`
 * (frames x total records) holds system 0's records, then system 1's, and so
 * on, packed by one launch for all systems after every `every`-th step. */
int pfb_ens2d_advance_record(pfb_ens2d* e, long long steps, int every, pfb_traj_cell2d* ring,
                             int frames);
/* The same steps launched one system at a time (the baseline the batched
 * launch is measured against). */
int pfb_ens2d_advance_serial(pfb_ens2d* e, int steps);
int pfb_ens2d_sync(pfb_ens2d* e);
/* The ensemble's CUDA stream (cudaStream_t), on which its steps and
 * recordings are queued. */
void* pfb_ens2d_stream(pfb_ens2d* e);
long long pfb_ens2d_step(const pfb_ens2d* e);
/* System r as a pfb_sim2d handle owned by the ensemble (after finishing the
 * ensemble's queued work): use pfb_sim2d_get_* on it; do not destroy it. */
pfb_sim2d* pfb_ens2d_system(pfb_ens2d* e, int r);
int pfb_ens2d_bench(pfb_ens2d* e, int warmup, int steps, int serial, double* ms_per_step);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* PFB200_H */
