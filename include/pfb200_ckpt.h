/* pfb200_ckpt.h -- the reference's 2D checkpoint file (PF "CELL" schema 1).
 *
 * Replaces pf::checkpoint_read / pf::checkpoint_write and the record layout of
 * the reference (common/checkpoint_format.h:1-149, src/checkpoint.cu:348-615,
 * 823-1011): a file written here restarts the reference's cell_gh200
 * (`-c file`), and a file written by cell_gh200 restarts a pfb_sim2d.
 *
 * Layout (little-endian, packed): a 44-byte prefix (magic 'CELL', schema 1,
 * step, time, cell count, save interval, zero, trajectory samples, four zero
 * flag bytes, parameter-record size), the 192-byte parameter record below,
 * the int32 tile pitch 288, a 12-byte rank trailer (1 rank, rank 0, cell
 * count), then per cell a 96-byte header and its 288^2 binary32 tile, then the
 * per-cell sidecars polarity (POLR), gamma (GAMA), active speed (VA_A),
 * target radius (RADI) and phase-field mobility (MOBI, optional on read: 0.5
 * when absent), each an 8-byte header (magic, count) and count binary32
 * values, in any order on read.
 *
 * Return values: PFB_OK or PFB_E_ARG (bad argument), PFB_E_FORMAT (a file
 * the reference would reject, with the reason in pfb_last_error()),
 * PFB_E_IO (open, read, write or rename failed). */
#ifndef PFB200_CKPT_H
#define PFB200_CKPT_H

#include <stddef.h>
#include <stdint.h>

#include "pfb200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PFB_E_FORMAT (-6) /* checkpoint contents rejected               */
#define PFB_E_IO (-7)     /* file could not be opened, read or written  */

/* The checkpoint's parameter record, byte for byte the reference's
 * CheckpointParamsRecord (common/checkpoint_format.h:79-106), 192 bytes. */
#pragma pack(push, 1)
typedef struct pfb_ckpt2d_params {
    int32_t Nx, Ny;             /*   0 */
    double dx, dy;              /*   8 */
    double dt;                  /*  24 */
    double t_end;               /*  32 */
    double rho;                 /*  40 requested packing fraction          */
    double lambda;              /*  48 */
    double gamma_normal;        /*  56 */
    double gamma_soft;          /*  64 (pfb_params2d.gamma_cancer)         */
    double soft_fraction;       /*  72 (pfb_params2d.cancer_fraction)      */
    double kappa;               /*  80 */
    double target_radius;       /*  88 */
    double mu;                  /*  96 */
    double v_A;                 /* 104 */
    double v_A_sigma;           /* 112 */
    double xi;                  /* 120 */
    double tau;                 /* 128 */
    uint64_t seed;              /* 136 */
    uint64_t polarity_seed;     /* 144 resolved tumble stream              */
    uint64_t initialization_hash; /* 152 */
    int32_t print_interval;     /* 160 */
    int32_t full_moment_every;  /* 164 */
    int32_t verify_every;       /* 168 */
    int32_t save_interval;      /* 172 */
    int32_t trajectory_samples; /* 176 */
    int32_t reserved;           /* 180 zero                                */
    int64_t trajectory_interval; /* 184 */
} pfb_ckpt2d_params;
#pragma pack(pop)

/* What a checkpoint holds besides its cells and tiles. */
typedef struct pfb_ckpt2d_info {
    long long step;
    double time;
    int num_cells;
    int L;
    int had_mobility; /* the file carried a MOBI sidecar */
} pfb_ckpt2d_info;

/* Parameter record of a run with parameters p, the run options at the
 * reference's defaults (dx = dy = 1, t_end = 100, print interval 100, verify
 * every 4096, save interval 0, 100 trajectory samples, trajectory interval 0,
 * initialization hash 0) and rho = the realised packing fraction
 * num_cells * pi * R^2 / L^2; the polarity stream resolved (0 -> seed). */
int pfb_ckpt2d_params_from(const pfb_params2d* p, pfb_ckpt2d_params* out);

/* Simulation parameters of a record (phase_field_mobility 0.5; the per-cell
 * mobilities of the file are in the cell records). */
int pfb_ckpt2d_params_to(const pfb_ckpt2d_params* rec, int num_cells, pfb_params2d* out);

/* Read and validate `path` as the reference does. With cells and phi null
 * only the info and the record are returned (the file is still validated in
 * full); otherwise cells[num_cells] receive the records as the reference's
 * restart builds them (window origin = tile origin + class offset, moments,
 * support, class, demotion counter, velocity and the five per-cell
 * sidecars; counters and accumulators zero) and phi[num_cells * 288^2] the
 * tiles. */
int pfb_ckpt2d_read(const char* path, pfb_ckpt2d_info* info, pfb_ckpt2d_params* rec,
                    pfb_cell2d* cells, float* phi);

/* Write cells and tiles as a checkpoint at `step` (time = step * rec->dt) to
 * path (through path.tmp and a rename, so a failed write leaves no partial
 * file). Refuses, as the reference does, non-canonical ids, non-finite or
 * out-of-range state, a class that disagrees with cls_written[step & 1] and
 * support outside the class window. */
int pfb_ckpt2d_write(const char* path, const pfb_ckpt2d_params* rec, long long step,
                     int num_cells, const pfb_cell2d* cells, const float* phi);

/* The current state of `s` written as a checkpoint (binary32 pools). */
int pfb_sim2d_write_checkpoint(pfb_sim2d* s, const char* path, const pfb_ckpt2d_params* rec);

/* A system restarted from a checkpoint: parameters from its record, state
 * and step from its cells and tiles (the aggregate is rebuilt by the scatter,
 * the moments are taken from the file). device as pfb_sim2d_create. */
pfb_sim2d* pfb_sim2d_create_from_checkpoint(const char* path, int device);

#ifdef __cplusplus
}
#endif

#endif /* PFB200_CKPT_H */
