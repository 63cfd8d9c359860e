// Internal declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include "../../include/pfb200.h"
#include "../../include/pfb200_3d.h"

namespace pfb {

// Record an error message for pfb_last_error() and return `code`.
int set_error(int code, const char* fmt, ...);
void clear_error();

// step2d.cu
int step2d_configure_device();
int step2d_launch(const pfb_step_args2d* a, int cluster, cudaStream_t stream);
// CTAs per cell when a caller passes cluster = 0: pairs of CTAs measured
// fastest on B200 for the class-0 windows (two resident clusters per SM).
constexpr int kDefaultCluster = 2;

int step2d_smem_bytes(int cluster);
// Systems r = 0..R-1 in one launch: d_args[r] (device) is served by CTAs
// [d_block_start[r], d_block_start[r+1]) (R+1 entries, multiples of cluster).
int step2d_launch_batch(const pfb_step_args2d* d_args, const int* d_block_start, int R,
                        int total_blocks, int cluster, int storage, cudaStream_t stream);
int step2d_read_status(unsigned* out, int clear);
int init2d_read_status(unsigned* out, int clear);
// variant: 0 = default, 1 = one thread-block cluster per cell
int step2d_launch_variant(const pfb_step_args2d* a, int cluster, int variant,
                          cudaStream_t stream);
// storage: 0 binary32 pools, 1 binary16, 2 bfloat16 (16-bit pools hold 2-byte
// values at the same tile positions; clusters of 2 or 4)
int step2d_launch_storage(const pfb_step_args2d* a, int cluster, int variant, int storage,
                          cudaStream_t stream);
// Device buffers of the 2D step's exact overflow detection for non-returning
// scatters: two alternating sets of per-bin bounds over 16 x 16 lattice bins
// and two alternating sets of the cells' committed window geometry
// (gx0, gy0, class, 0). All zero when first handed to a launch.
constexpr int kBinShift = 4;
struct BinArgs {
    unsigned long long* bound;  // 2 sets of nbx * nby bounds
    int4* geo;                  // 2 sets of N window geometries
    unsigned int* recounts;     // bins recounted exactly so far (diagnostic)
    int nbx, nby;               // bins per lattice row and column
};
// The step with the identity path's scatter non-returning, overflow exact
// through B (binary32 or 16-bit pools, no observer).
int step2d_launch_binned(const pfb_step_args2d* a, int cluster, int storage, const BinArgs& B,
                         cudaStream_t stream);
// Settles the bounds of the launch that ran at `step` (the last one issued):
// recounts every bin whose bound reached 2^32 from the field it wrote (`phi`,
// storage 0/1/2) and raises S_overflow when some pixel total reaches 2^32.
int step2d_settle_bins(const BinArgs& B, const void* phi, int storage, int N, int L,
                       unsigned long long step, uint32_t* flags, cudaStream_t stream);
// The step with a velocity observer (PFB_VELOCITY_*), binary32 pools.
int step2d_launch_observed(const pfb_step_args2d* a, int cluster, int observation,
                           cudaStream_t stream);

// Velocity observation (velocity2d.cu): the dense observer and the PFVMOM4
// recorder a pfb_sim2d drives.
int velocity2d_observe(const pfb_step_args2d& A, pfb_moment_accum2d* out, double dt,
                       cudaStream_t stream);
struct Velocity2D;
Velocity2D* velocity2d_create(const char* path, int N, double dt, int stride, long long dense,
                              int reference);
void velocity2d_destroy(Velocity2D* v);
int velocity2d_open(Velocity2D* v, const pfb_step_args2d& A, long long step, cudaStream_t stream);
// Observation of the step about to run from `step`: sets *observation and
// A->moments (and runs the dense observer first in the reference mode).
int velocity2d_prepare(Velocity2D* v, pfb_step_args2d* A, long long step, cudaStream_t stream,
                       int* observation);
void velocity2d_advanced(Velocity2D* v);
int velocity2d_capture(Velocity2D* v, const pfb_step_args2d& A, long long step, cudaStream_t stream);
long long velocity2d_last_frame(const Velocity2D* v);
int velocity2d_close(Velocity2D* v);

// PFB boundary recorder (boundary2d.cu).
struct Boundary2D;
Boundary2D* boundary2d_open(const char* path, int N, int side, double dt, double tau,
                            long long interval, int compress);
int boundary2d_capture(Boundary2D* b, const float* phi, const pfb_cell2d* cells,
                       cudaStream_t stream, long long step, double time);
// Finish the file (end record) and free the recorder.
int boundary2d_close(Boundary2D* b);

// Morton visit order of the 2D cells (order2d.cu): the largest N one sorting
// CTA holds, the shared-memory opt-in (outside stream capture), the sort.
int visit_order2d_capacity();
cudaError_t visit_order2d_prepare(int N);
cudaError_t visit_order2d_launch(const pfb_cell2d* cell, uint32_t* perm, int N, int L, cudaStream_t stream);

// PFB3D boundary recorder (boundary3d.cu); projection 1 basal, 2 maximum.
struct Boundary3D;
Boundary3D* boundary3d_open(const char* path, const pfb_params3d& p, int projection,
                            long long interval, int compress);
int boundary3d_capture(Boundary3D* b, const float* phi, float* const* cubes, const pfb_cell3d* cells,
                       int B, cudaStream_t stream, long long step, double time);
// complete != 0 writes the end record; the recorder is freed either way.
int boundary3d_close(Boundary3D* b, int complete);

// init2d.cu
int init_tiles2d(float* phi_a, float* phi_b, pfb_cell2d* cell, const uint8_t* cls, int N, int L,
                 const float* cx, const float* cy, float radius_eff, float kappa_iface,
                 cudaStream_t s);
int init_moments2d(pfb_cell2d* cell, const uint8_t* cls, const float* phi, int N,
                   cudaStream_t s);
int scatter_all2d(const float* phi, const pfb_cell2d* cell, const uint8_t* cls, uint32_t* S,
                  int N, int L, int P, uint32_t* flags, cudaStream_t s);
int zero_u32(uint32_t* p, size_t n, cudaStream_t s);
// binary32 <-> 16-bit pool conversion (round to nearest), storage 1 or 2
int narrow_pool(const float* in, void* out, size_t n, int storage, cudaStream_t s);
int widen_pool(const void* in, float* out, size_t n, int storage, cudaStream_t s);
int verify_cells2d(const float* phi, const pfb_cell2d* cell, const uint8_t* cls, int N,
                   double* out_V, float* out_outside, cudaStream_t s);
int verify_S(const uint32_t* S, size_t n, uint32_t* out_max, cudaStream_t s);
int pack_traj2d(const pfb_cell2d* cell, const uint8_t* cls, pfb_traj_cell2d* out, int N, int L,
                cudaStream_t s);
// A ring of trajectory frames in page-locked host memory (device-visible
// address), filled by pack_traj2d_ring: frame k goes to base + (k % frames) * N.
struct TrajRing2D {
    pfb_traj_cell2d* base;
    unsigned long long k;     // frames packed so far in this call
    int frames;
    unsigned int arrived;     // CTAs of the running pack that are done
};
int ring_begin2d(TrajRing2D* ring, pfb_traj_cell2d* base, int frames, cudaStream_t s);
// One system of a batched pack: its records go to positions off .. off+N-1
// of each frame.
struct TrajSource2D {
    const pfb_cell2d* cell;
    const uint8_t* cls;
    int L;
    int off;
};
int pack_traj2d_ring_batch(const TrajSource2D* src, int R, int total, TrajRing2D* ring, cudaStream_t s);
int pack_traj2d_ring(const pfb_cell2d* cell, const uint8_t* cls, TrajRing2D* ring, int N, int L,
                     cudaStream_t s);

// sim2d.cu: device-side view of a pfb_sim2d for the relaxation tools
struct Sim2DView {
    float* phi_cur;            // pool of the current step (binary32 pools)
    float* phi_prev;           // the other pool (the previous step after a step)
    pfb_cell2d* cells;
    const pfb_cell2d* cells_prev;  // records saved by sim2d_step_keep_prev
    uint8_t* cls;
    uint32_t* S_cur;           // aggregate of the current step
    int N, L, P;
    double dt;
    int storage;
    cudaStream_t stream;
    long long step;
    int device;
};
int sim2d_view(pfb_sim2d* s, Sim2DView* v);
int sim2d_rebuild(pfb_sim2d* s);
int sim2d_step_keep_prev(pfb_sim2d* s);
// relax2d.cu: crops of the current state (network input, origins) and the
// insertion of predicted increments (followed by a rebuild)
int relax_extract(pfb_sim2d* s, void* x0, float* phi_crop, int* origins, const int* origins_in,
                  const float* prev, float hist_scale);
int relax_insert(pfb_sim2d* s, const int* origins, const float* dphi);

// conv2d_tc.cu: 3x3 same convolutions on padded-NHWC bfloat16 activations
int conv3x3_fwd(const void* x, void* y, float* yf, const void* wp, const float* bias,
                const void* gate, int B, int H, int W, int cin, int cout, int relu,
                cudaStream_t s);
size_t conv3x3_wgrad_workspace(int B, int H, int W, int cx, int cy);
int conv3x3_wgrad(const void* x, const void* dy, float* workspace, size_t workspace_bytes,
                  float* dw, float* db, int B, int H, int W, int cx, int cy, cudaStream_t s);
int conv3x3_pack(const float* w, void* packed, int cin, int cout, int transpose, cudaStream_t s);
int conv_read_status(unsigned* out, int clear);

namespace p3 {
// measure3d.cu / update3d.cu / misc3d.cu (pfb200_3d.h records)
int measure3d_launch(const pfb_measure_args3d* a, cudaStream_t stream);
int measure3d_launch_pool(const pfb_measure_args3d* a, int storage, cudaStream_t stream);
int motion3d_launch(const pfb_measure_args3d* a, cudaStream_t stream);
int update3d_launch(const pfb_update_args3d* a, cudaStream_t stream);
// in-place modes: update into `slots` scratch bricks, then commit (reference
// launch_update_inplace); a->phi_out is ignored
int update3d_inplace_launch(const pfb_update_args3d* a, float* scratch, int slots, cudaStream_t stream);
// the same two updates on pools of storage type `storage` (PhiStorage; the
// pointers of `a` then address 16-bit pools), rounding stream of (*step, seed)
int update3d_launch_pool(const pfb_update_args3d* a, int storage, const uint64_t* step, uint64_t seed,
                         cudaStream_t stream);
int update3d_inplace_launch_pool(const pfb_update_args3d* a, void* scratch, int slots, int storage,
                                 const uint64_t* step, uint64_t seed, cudaStream_t stream);
// clears S; with a non-null guard only when a fatal global flag is set
int clear3d_launch(uint32_t* S, const pfb_layout3d* L, const uint32_t* guard,
                   cudaStream_t stream);
int repair3d_launch(const pfb_update_args3d* a, cudaStream_t stream);
int repair3d_launch_pool(const pfb_update_args3d* a, int storage, cudaStream_t stream);
int init3d_launch(const pfb_init_args3d* a, cudaStream_t stream);
int scatter3d_launch(const pfb_scatter_args3d* a, cudaStream_t stream);
int scatter3d_launch_pool(const pfb_scatter_args3d* a, int storage, cudaStream_t stream);
int measure3d_read_status(unsigned* out, int clear);
int update3d_read_status(unsigned* out, int clear);
int check_measure(const pfb_measure_args3d* a);
// pools = false: the base phi pools are not needed (promoted-cube launches)
int check_update(const pfb_update_args3d* a, bool pools = true);
// cluster size of the measurement (the fused step's where it applies)
int measure3d_cluster(int B);
// step3d.cu: fused measure + motion + update; cluster size 0 when the brick
// does not fit the fused kernel's shared memory
int step3d_cluster(int B);
size_t step3d_smem(int B);
int step3d_launch(const pfb_measure_args3d* m, const pfb_update_args3d* u, cudaStream_t stream);
int step3d_read_status(unsigned* out, int clear);
// promote3d.cu: cells in their own cubes (storage_edge > B)
int next_brick_edge3(int current, int maximum);
int shrink_brick_edge3(int current, int minimum, const int* lo, const int* hi);
int measure3d_promoted_launch(const pfb_measure_args3d* a, float* const* cubes, const int* ids,
                              int count, int max_edge, cudaStream_t stream);
int update3d_promoted_launch(const pfb_update_args3d* a, float* const* in, float* const* out,
                             const int* ids, int count, int max_edge, cudaStream_t stream);
int scatter3d_promoted_launch(const pfb_scatter_args3d* a, float* const* cubes, const int* ids,
                              int count, int max_edge, int guard_fatal, cudaStream_t stream);
int repair3d_promoted_launch(const pfb_update_args3d* a, float* const* in, float* const* out,
                             const int* ids, int count, int max_edge, cudaStream_t stream);
int copy_centred3d_launch(const float* src, int Es, float* dst, int Ed, cudaStream_t stream);
int check_crops3d_launch(float* const* cubes, const pfb_cell3d* cells, const int* candidate,
                         uint32_t* rejected, int N, int B, cudaStream_t stream);
int promote3d_read_status(unsigned* out, int clear);
}  // namespace p3

}  // namespace pfb
