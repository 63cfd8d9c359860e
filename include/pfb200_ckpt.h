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
#include "pfb200_3d.h"

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

/* ======================================================================
 * 3D checkpoint file (PF3D schema 1) -- replaces pf3d::checkpoint_probe_3d /
 * checkpoint_load_3d / checkpoint_write_3d (common/checkpoint_format_3d.h,
 * src/pf3d/checkpoint.cu:116-420, 599-1235). A 96-byte header (magic
 * "PF3D", schema 1, record sizes, endian marker, 3 dimensions, binary32,
 * flags CRC + variable storage, step, time, cell count, B, x-fastest order,
 * B^3 values and bytes per cell, the file's CRC-64/ECMA-182 computed with
 * this field zero, base measurement CTAs per cell), the 288-byte parameter
 * record below, then per cell a 256-byte record and its storage_edge^3
 * binary32 brick. This library writes and reads base bricks only
 * (storage_edge = B); files with promoted (larger) bricks are rejected with
 * PFB_E_CONFIG.
 * ==================================================================== */
#pragma pack(push, 1)
/* The reference's ParamsRecord3D (common/checkpoint_format_3d.h:167-227). */
typedef struct pfb_ckpt3d_params {
    int64_t Nx, Ny, Nz;                /*   0 */
    double dx, dy, dz;                 /*  24 */
    uint32_t brick_edge;               /*  48 */
    uint32_t boundary_flags;           /*  52 */
    double dt, t_end, lambda;          /*  56 */
    double gamma_normal, gamma_soft, soft_fraction;
    double kappa, target_radius, mu, v_A, v_A_sigma, xi, tau;
    double volume_fraction;            /* rho_V; rho_A for a slab          */
    uint64_t seed;                     /* 168 */
    uint64_t polarity_seed;            /* 176 resolved                      */
    int64_t print_interval, full_moment_every, verify_every;
    uint32_t integrator_id;            /* 208: 1 explicit Euler             */
    uint32_t stencil_id;               /* 2: 27-point                       */
    uint32_t rng_id;                   /* 1: Philox4x32-10                  */
    uint32_t trajectory_interval;      /* 220 */
    uint64_t initialization_hash;      /* 224 */
    double aging_time;                 /* 232 */
    uint64_t promoted_measure_policy;  /* 240: 0 one CTA, 1..64, ~0 auto  */
    uint64_t promoted_measure_auto_wave_ctas;
    int64_t channel_height, channel_padding;
    double wall_kappa, wall_width;     /* 272 */
} pfb_ckpt3d_params;
#pragma pack(pop)

typedef struct pfb_ckpt3d_info {
    long long step;
    double time;
    int num_cells;
    int brick_edge;
    int base_measure_shards; /* stored CTAs per cell of the base measurement */
    uint64_t crc64;
} pfb_ckpt3d_info;

/* CRC-64/ECMA-182 (polynomial 0x42F0E1EBA9EA3693, MSB first, initial value
 * and final xor 0) of n bytes, continuing from crc (0 to start). */
uint64_t pfb_crc64_ecma(uint64_t crc, const void* data, size_t n);

/* Record of a run with parameters p and brick edge B (0: the automatic
 * edge): volume fraction realised from the cell count and the domain
 * (areal coverage for a slab, the accessible slit for a channel), t_end 100,
 * print interval 100, verify every 4096, the reference's integrator, stencil
 * and RNG ids, one-CTA promoted-measurement policy. */
int pfb_ckpt3d_params_from(const pfb_params3d* p, int brick, pfb_ckpt3d_params* out);
int pfb_ckpt3d_params_to(const pfb_ckpt3d_params* rec, int num_cells, pfb_params3d* out);

/* Read and validate (header, parameters, file size, every record, CRC) as
 * the reference does. With cells and phi null only info and rec are filled
 * (the CRC is still verified over the whole file); otherwise cells[N]
 * (storage_edge 0 for a base cell, E for a cell stored on a promoted cube of
 * edge E > B; derived wall fields zero) and phi: each cell's field packed in
 * cell order, B^3 values for a base cell and E^3 for a promoted one
 * (pfb_ckpt3d_payload_words gives the length; N * B^3 when no cell is
 * promoted). */
int pfb_ckpt3d_read(const char* path, pfb_ckpt3d_info* info, pfb_ckpt3d_params* rec,
                    pfb_cell3d* cells, float* phi);
/* Packed field length (values) of the PF3D file at path, after the same
 * validation as pfb_ckpt3d_read. */
int pfb_ckpt3d_payload_words(const char* path, unsigned long long* words);

/* Write cells and their packed fields (as pfb_ckpt3d_read returns them) at
 * `step` (time = step * dt) through path.tmp and a rename; base_measure_shards in 1..64 is stored as the measurement
 * grouping the continuation should use. Refuses records the reader would
 * reject. */
int pfb_ckpt3d_write(const char* path, const pfb_ckpt3d_params* rec, long long step, int num_cells,
                     const pfb_cell3d* cells, const float* phi, int base_measure_shards);

/* The current state of `s` (its brick edge, 4 measurement CTAs per cell),
 * measured first (pfb_sim3d_measure_current) as the reference does. */
int pfb_sim3d_write_checkpoint(pfb_sim3d* s, const char* path, const pfb_ckpt3d_params* rec);
pfb_sim3d* pfb_sim3d_create_from_checkpoint(const char* path, int device);
/* The same with a storage mode and scratch bricks (pfb_sim3d_create_ex). */
pfb_sim3d* pfb_sim3d_create_from_checkpoint_ex(const char* path, int device, int memory_mode,
                                               int scratch_slots);

#ifdef __cplusplus
}
#endif

#endif /* PFB200_CKPT_H */
