// The reference's 3D checkpoint file (PF3D schema 1): reader and writer with
// the reference's acceptance rules (common/checkpoint_format_3d.h:1-398;
// src/pf3d/checkpoint.cu:116-152 header, 241-285 parameters, 382-420 cell
// records, 599-751 metadata and layout, 841-996 load with the CRC, 1009-1235
// write; parameter checks of include/pf3d/params.cuh:373-473). The byte
// layout has to be the reference's, so the records below keep its field order
// and sizes; the code is this library's own. Each cell record is followed by
// the cell's own cube: B^3 values on the base brick, E^3 on a promoted cube
// of edge E = storage_edge (reference src/pf3d/checkpoint.cu:655-751).
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "pfb_internal.h"
#include "pfb200_ckpt.h"

using namespace pfb;

namespace {

constexpr uint32_t kMagic3 = 0x44334650u;  // "PF3D"
constexpr uint16_t kSchema3 = 1;
constexpr uint32_t kEndian = 0x01020304u;
constexpr uint32_t kFlags3 = 3u;          // payload CRC-64 | variable cell storage
constexpr uint32_t kPeriodic = 0x7u, kSlab = 0x3u, kChannel = 0xBu;
constexpr uint32_t kKnownFlagMask = (1u << PFB3D_FLAG_COUNT) - 1u;
constexpr double kLapBound3 = 256.0 / 30.0;  // 27-point Laplacian row-sum bound
constexpr double kPolarityTol = 2.0e-5;
constexpr uint64_t kAutoPolicy = ~0ull;

#pragma pack(push, 1)
struct Header3 {
    uint32_t magic;
    uint16_t schema, header_bytes;
    uint32_t endian, dims, scalar, flags;
    int64_t step;
    double time;
    uint64_t cells;
    uint32_t params_bytes, record_bytes, brick, order;
    uint64_t values_per_cell, bytes_per_cell, crc, base_shards;
};
struct Record3 {
    int64_t id, ox, oy, oz;
    float px, py, pz, vx, vy, vz, gamma, v_A, R, phi_max;
    double V, Cx, Cy, Cz, surface, Ix, Iy, Iz;
    uint32_t shift_ctr, tumble_ctr, flags;
    int32_t bb[6];
    int32_t shift[3];
    uint32_t storage_edge, zero32;
    uint64_t zero64[8];
};
#pragma pack(pop)
static_assert(sizeof(Header3) == 96 && sizeof(pfb_ckpt3d_params) == 288 && sizeof(Record3) == 256,
              "PF3D record sizes");
static_assert(offsetof(Header3, crc) == 80 && offsetof(pfb_ckpt3d_params, seed) == 168 &&
                  offsetof(pfb_ckpt3d_params, integrator_id) == 208 &&
                  offsetof(pfb_ckpt3d_params, wall_kappa) == 272 && offsetof(Record3, V) == 72 &&
                  offsetof(Record3, bb) == 148 && offsetof(Record3, storage_edge) == 184,
              "PF3D field offsets");

struct FileCloser {
    void operator()(std::FILE* f) const {
        if (f) std::fclose(f);
    }
};
using File = std::unique_ptr<std::FILE, FileCloser>;

// CRC-64/ECMA-182, byte-wise with a 256-entry table built from the
// polynomial (MSB first, no reflection, initial value and final xor zero).
struct Crc64 {
    uint64_t t[256];
    Crc64() {
        for (int i = 0; i < 256; ++i) {
            uint64_t v = (uint64_t)i << 56;
            for (int b = 0; b < 8; ++b) v = (v >> 63) ? (v << 1) ^ 0x42F0E1EBA9EA3693ull : v << 1;
            t[i] = v;
        }
    }
    uint64_t update(uint64_t crc, const void* p, size_t n) const {
        const uint8_t* b = static_cast<const uint8_t*>(p);
        for (size_t i = 0; i < n; ++i) crc = t[(uint8_t)((crc >> 56) ^ b[i])] ^ (crc << 8);
        return crc;
    }
};
const Crc64& crc_table() {
    static const Crc64 c;
    return c;
}

bool get(std::FILE* f, void* dst, size_t n) { return n == 0 || std::fread(dst, 1, n, f) == n; }

long long steps_of(double t, double dt) {
    const double s = t / dt + 0.5;
    return std::isfinite(s) && s >= 0.0 && s <= 9.0e18 ? (long long)s : -1;
}

int min_domain_edge(const pfb_ckpt3d_params& r) {
    const int64_t xy = std::min(r.Nx, r.Ny);
    return (int)(r.boundary_flags == kChannel ? xy : std::min(xy, r.Nz));
}

int bad(const char* why) { return set_error(PFB_E_FORMAT, "PF3D checkpoint: %s", why); }

// Header rules (format, record sizes, flags, shard count, step and time,
// cell count, brick edge and payload sizes).
int check_header(const Header3& h) {
    if (h.magic != kMagic3) return bad("not a PF3D checkpoint");
    if (h.schema != kSchema3) return bad("unsupported PF3D schema");
    if (h.header_bytes != sizeof(Header3) || h.params_bytes != sizeof(pfb_ckpt3d_params) ||
        h.record_bytes != sizeof(Record3))
        return bad("record-size fields do not match");
    if (h.endian != kEndian || h.dims != 3 || h.scalar != 1 || h.order != 1)
        return bad("incompatible scalar, dimension, endian or phase order");
    if (h.flags != kFlags3) return bad("missing required checksum flag");
    if (h.base_shards > 64) return bad("base measurement shard count is outside 0..64");
    if (h.step < 0 || !std::isfinite(h.time) || h.time < 0.0) return bad("negative step/time or non-finite time");
    if (h.cells == 0 || h.cells > 2147483647ull) return bad("cell count is outside the supported range");
    if (h.brick < 3 || h.brick > 4096 || h.brick % 8 != 0) return bad("brick edge is outside the corruption guard");
    const uint64_t v = (uint64_t)h.brick * h.brick * h.brick;
    if (h.values_per_cell != v || h.bytes_per_cell != 4 * v)
        return bad("phase payload size is inconsistent with B^3 float32");
    return PFB_OK;
}

// Parameter-record rules and the reference's parameter validation.
int check_params(const pfb_ckpt3d_params& p, const Header3& h) {
    if (p.Nx <= 0 || p.Ny <= 0 || p.Nz <= 0 || p.Nx > 2147483647 || p.Ny > 2147483647 || p.Nz > 2147483647)
        return bad("domain dimensions are outside the supported range");
    const bool geo = (p.boundary_flags == kPeriodic && p.Nx == p.Ny && p.Nx == p.Nz) ||
                     ((p.boundary_flags == kSlab || p.boundary_flags == kChannel) && p.Nx == p.Ny);
    if (!geo) return bad("boundary flags and dimensions do not describe a supported geometry");
    const double scal[] = {p.dx, p.dy, p.dz, p.dt, p.t_end, p.lambda, p.gamma_normal, p.gamma_soft,
                           p.soft_fraction, p.kappa, p.target_radius, p.mu, p.v_A, p.v_A_sigma, p.xi,
                           p.tau, p.volume_fraction, p.aging_time};
    for (double v : scal)
        if (!std::isfinite(v)) return bad("a parameter is not finite");
    if (p.brick_edge != h.brick || (int64_t)p.brick_edge >= min_domain_edge(p))
        return bad("parameter and header brick edges disagree");
    if (p.integrator_id != 1 || p.stencil_id != 2 || p.rng_id != 1)
        return bad("integrator, stencil or RNG contract is incompatible");
    if (p.print_interval < 0 || p.print_interval > 2147483647 || p.full_moment_every < 0 ||
        p.full_moment_every > 2147483647 || p.verify_every < 0 || p.verify_every > 2147483647)
        return bad("stored output or verification cadence is out of range");
    const bool policy_ok = p.promoted_measure_policy == kAutoPolicy
                               ? p.promoted_measure_auto_wave_ctas > 0 &&
                                     p.promoted_measure_auto_wave_ctas <= 2147483647ull
                               : p.promoted_measure_policy <= 64 && p.promoted_measure_auto_wave_ctas == 0;
    if (!policy_ok) return bad("invalid promoted-measurement reduction contract");
    if (p.channel_height < 0 || p.channel_height > 2147483647 || p.channel_padding < 0 ||
        p.channel_padding > 2147483647)
        return bad("invalid resolved-wall parameters");
    // the reference's validate(SimParams3D)
    if (!(p.dx == 1.0 && p.dy == 1.0 && p.dz == 1.0)) return bad("dx, dy and dz must all equal 1");
    if (p.boundary_flags == kChannel) {
        if (p.channel_height <= 0 || p.channel_padding <= 0 || !(p.wall_width > 0.0) || !(p.wall_kappa > 0.0))
            return bad("resolved channel wall parameters must be positive");
        if (!(p.kappa > 0.0)) return bad("repulsive channel walls require positive kappa");
        const float ratio = (float)(p.wall_kappa / p.kappa);
        if (!std::isfinite(ratio) || !(ratio > 0.0f)) return bad("wall_kappa / kappa is not representable");
        if (p.wall_width > 2147483647.0 / 3.0 || p.channel_padding < (int64_t)std::ceil(3.0 * p.wall_width))
            return bad("channel padding must be at least ceil(3 wall_width)");
        if (p.channel_height + 2 * p.channel_padding != p.Nz) return bad("channel Nz must equal H + 2 padding");
        if ((double)p.channel_height < std::ceil(2.0 * p.target_radius))
            return bad("accessible channel height is smaller than one cell diameter");
    } else if (p.channel_height != 0 || p.channel_padding != 0 || p.wall_kappa != 0.0 || p.wall_width != 0.0) {
        return bad("wall parameters require the hard-wall channel geometry");
    }
    if (!(p.volume_fraction > 0.0 && p.volume_fraction < 1.0)) return bad("rho must lie in (0, 1)");
    if (!(p.dt > 0.0) || !(p.t_end >= 0.0) || steps_of(p.t_end, p.dt) < 0)
        return bad("dt and t_end do not define a valid step count");
    if (!(p.aging_time >= 0.0) || steps_of(p.aging_time, p.dt) < 0)
        return bad("aging_time does not define a valid step count");
    if (!(p.lambda > 0.0) || !(p.target_radius > 0.0)) return bad("lambda and radius must be positive");
    if (p.kappa < 0.0 || p.mu < 0.0 || !(p.xi > 0.0)) return bad("kappa and mu must be non-negative, xi positive");
    if (!(p.tau > 0.0) || p.v_A < 0.0 || p.v_A_sigma < 0.0)
        return bad("tau must be positive and motility parameters non-negative");
    if (!(p.gamma_normal > 0.0) || !(p.gamma_soft > 0.0) || !(p.soft_fraction >= 0.0 && p.soft_fraction <= 1.0))
        return bad("gamma values and soft fraction are invalid");
    const int edge = pfb3d_automatic_brick_edge(p.target_radius, p.lambda);
    if (edge <= 0 || min_domain_edge(p) <= edge) return bad("the automatic brick must fit inside the domain");
    const double gmax = std::max(p.gamma_normal, p.gamma_soft);
    const double bulk = 30.0 / (p.lambda * p.lambda);
    const double wall = 60.0 * p.wall_kappa / (p.lambda * p.lambda);
    if (p.dt * gmax * kLapBound3 >= 1.0) return bad("explicit-Euler Laplacian stability bound is violated");
    if (p.dt * gmax * bulk >= 1.0) return bad("explicit-Euler bulk-reaction bound is violated");
    if (p.dt * wall >= 1.0) return bad("explicit-Euler wall-repulsion bound is violated");
    if (p.dt * 2.0 * p.mu >= 1.0) return bad("explicit-Euler volume-restoring bound is violated");
    const double fast = p.v_A_sigma == 0.0 ? p.v_A : p.v_A * std::exp(6.0 * p.v_A_sigma);
    if (!std::isfinite(fast) || p.dt * fast >= 1.0) return bad("active-speed bound is violated");
    // the stored brick: at least the automatic edge, aligned, inside the domain
    if ((int)h.brick < edge || (int)h.brick >= min_domain_edge(p))
        return bad("stored brick edge is incompatible with these parameters");
    return PFB_OK;
}

// One cell record against the reference's rules, on a base brick of edge B.
int check_record(const Record3& r, int index, int B, const pfb_ckpt3d_params& p) {
    if (r.id != index) return set_error(PFB_E_FORMAT, "PF3D cell slot %d carries id %lld", index, (long long)r.id);
    if (r.zero32 != 0) return set_error(PFB_E_FORMAT, "PF3D cell %d: reserved field is not zero", index);
    for (uint64_t z : r.zero64)
        if (z != 0) return set_error(PFB_E_FORMAT, "PF3D cell %d: reserved field is not zero", index);
    const int dom = min_domain_edge(p);
    if (r.storage_edge < (uint32_t)B || r.storage_edge > 4096 || r.storage_edge % 8 != 0 ||
        (int64_t)r.storage_edge >= dom)
        return set_error(PFB_E_FORMAT, "PF3D cell %d has an invalid storage edge", index);
    // the cell's own cube: the base brick or a promoted one
    const int e = (int)r.storage_edge;
    bool ok = std::isfinite(r.vx) && std::isfinite(r.vy) && std::isfinite(r.vz);
    if (p.boundary_flags == kPeriodic || p.boundary_flags == kChannel) {
        const double n2 = (double)r.px * r.px + (double)r.py * r.py + (double)r.pz * r.pz;
        ok = ok && std::isfinite(n2) && std::fabs(n2 - 1.0) <= kPolarityTol;
    } else {
        const double n2 = (double)r.px * r.px + (double)r.py * r.py;
        ok = ok && r.pz == 0.0f && r.vz == 0.0f && std::isfinite(n2) && std::fabs(n2 - 1.0) <= kPolarityTol;
    }
    if (p.boundary_flags != kPeriodic)
        ok = ok && r.bb[4] >= 0 && r.bb[4] <= r.bb[5] && r.oz >= -(int64_t)r.bb[4] && r.oz < p.Nz - (int64_t)r.bb[5];
    ok = ok && std::isfinite(r.V) && r.V > 0.0 && std::isfinite(r.Cx) && std::isfinite(r.Cy) &&
         std::isfinite(r.Cz) && std::isfinite(r.surface) && r.surface >= 0.0 && std::isfinite(r.Ix) &&
         std::isfinite(r.Iy) && std::isfinite(r.Iz) && std::isfinite(r.gamma) && r.gamma > 0.0f &&
         std::isfinite(r.v_A) && r.v_A >= 0.0f && std::isfinite(r.R) && r.R > 0.0f &&
         std::isfinite(r.phi_max) && r.phi_max >= 0.0f && (r.flags & ~kKnownFlagMask) == 0 &&
         (r.flags & PFB3D_FATAL_MASK) == 0;
    for (int d = 0; d < 3; ++d)
        ok = ok && r.bb[2 * d] >= 0 && r.bb[2 * d] <= r.bb[2 * d + 1] && r.bb[2 * d + 1] < e &&
             r.shift[d] >= -e && r.shift[d] <= e;
    if (!ok) return set_error(PFB_E_FORMAT, "PF3D cell record %d is invalid", index);
    return PFB_OK;
}

Record3 record_of(const pfb_cell3d& c, int B) {
    // a base cell stores the base edge; a promoted one its cube's edge
    Record3 r;
    std::memset(&r, 0, sizeof(r));
    r.id = c.global_id;
    r.ox = c.origin_x;
    r.oy = c.origin_y;
    r.oz = c.origin_z;
    r.px = c.polarity_x;
    r.py = c.polarity_y;
    r.pz = c.polarity_z;
    r.vx = c.velocity_x;
    r.vy = c.velocity_y;
    r.vz = c.velocity_z;
    r.gamma = c.gamma;
    r.v_A = c.v_A;
    r.R = c.R_tgt;
    r.phi_max = c.phi_max;
    r.V = c.V;
    r.Cx = c.Cx;
    r.Cy = c.Cy;
    r.Cz = c.Cz;
    r.surface = c.surface;
    r.Ix = c.Ix;
    r.Iy = c.Iy;
    r.Iz = c.Iz;
    r.shift_ctr = c.shift_ctr;
    r.tumble_ctr = c.tumble_ctr;
    r.flags = c.flags;
    const int32_t bb[6] = {c.bb_lo_x, c.bb_hi_x, c.bb_lo_y, c.bb_hi_y, c.bb_lo_z, c.bb_hi_z};
    std::memcpy(r.bb, bb, sizeof(bb));
    r.shift[0] = c.pending_shift_x;
    r.shift[1] = c.pending_shift_y;
    r.shift[2] = c.pending_shift_z;
    r.storage_edge = c.storage_edge > (uint32_t)B ? c.storage_edge : (uint32_t)B;
    return r;
}

void cell_of(const Record3& r, int B, pfb_cell3d* c) {
    std::memset(c, 0, sizeof(*c));
    c->global_id = r.id;
    c->origin_x = r.ox;
    c->origin_y = r.oy;
    c->origin_z = r.oz;
    c->polarity_x = r.px;
    c->polarity_y = r.py;
    c->polarity_z = r.pz;
    c->velocity_x = r.vx;
    c->velocity_y = r.vy;
    c->velocity_z = r.vz;
    c->gamma = r.gamma;
    c->v_A = r.v_A;
    c->R_tgt = r.R;
    c->phi_max = r.phi_max;
    c->V = r.V;
    c->Cx = r.Cx;
    c->Cy = r.Cy;
    c->Cz = r.Cz;
    c->surface = r.surface;
    c->Ix = r.Ix;
    c->Iy = r.Iy;
    c->Iz = r.Iz;
    c->shift_ctr = r.shift_ctr;
    c->tumble_ctr = r.tumble_ctr;
    c->flags = r.flags;
    c->bb_lo_x = r.bb[0];
    c->bb_hi_x = r.bb[1];
    c->bb_lo_y = r.bb[2];
    c->bb_hi_y = r.bb[3];
    c->bb_lo_z = r.bb[4];
    c->bb_hi_z = r.bb[5];
    c->pending_shift_x = r.shift[0];
    c->pending_shift_y = r.shift[1];
    c->pending_shift_z = r.shift[2];
    c->storage_edge = r.storage_edge == (uint32_t)B ? 0u : r.storage_edge;  // 0: base brick
}

// Read (and verify) a PF3D file. phi receives each cell's field packed in cell
// order (B^3 values for a base cell, E^3 for a cell stored on a promoted cube
// of edge E); *words the packed length. With cells and phi null the file is
// only verified.
int read3(const char* path, pfb_ckpt3d_info* info, pfb_ckpt3d_params* rec_out, pfb_cell3d* cells, float* phi,
          unsigned long long* words_out = nullptr) {
    File f(std::fopen(path, "rb"));
    if (!f) return set_error(PFB_E_IO, "cannot open %s: %s", path, std::strerror(errno));
    Header3 h;
    pfb_ckpt3d_params p;
    if (!get(f.get(), &h, sizeof(h))) return bad("short read of the header");
    int rc = check_header(h);
    if (rc) return rc;
    if (!get(f.get(), &p, sizeof(p))) return bad("short read of the parameter record");
    if ((rc = check_params(p, h))) return rc;
    const double t_expect = (double)h.step * p.dt;
    if (!std::isfinite(t_expect) || std::fabs(h.time - t_expect) > 1e-12 * std::max(1.0, std::fabs(t_expect)))
        return bad("time does not match step * dt");
    if (std::fseek(f.get(), 0, SEEK_END) != 0) return set_error(PFB_E_IO, "cannot seek %s", path);
    const long long size = std::ftell(f.get());
    const int N = (int)h.cells, B = (int)h.brick;
    // every cell at least a record and a base brick
    const unsigned long long prefix = sizeof(Header3) + sizeof(pfb_ckpt3d_params);
    const unsigned long long least = prefix + (sizeof(Record3) + h.bytes_per_cell) * (unsigned long long)N;
    if (size < 0 || (unsigned long long)size < least)
        return set_error(PFB_E_FORMAT, "PF3D file has %lld bytes; its cell records need at least %llu", size,
                         least);
    if (std::fseek(f.get(), (long)prefix, SEEK_SET) != 0) return set_error(PFB_E_IO, "cannot seek %s", path);
    const Crc64& crc = crc_table();
    Header3 canon = h;
    canon.crc = 0;
    uint64_t c = crc.update(0, &canon, sizeof(canon));
    c = crc.update(c, &p, sizeof(p));
    unsigned long long pos = prefix, packed = 0;
    std::vector<float> tmp;
    for (int i = 0; i < N; ++i) {
        Record3 r;
        if (pos + sizeof(r) > (unsigned long long)size) return bad("the file truncates a cell record");
        if (!get(f.get(), &r, sizeof(r))) return bad("short read of a cell record");
        if ((rc = check_record(r, i, B, p))) return rc;
        c = crc.update(c, &r, sizeof(r));
        const size_t words = (size_t)r.storage_edge * r.storage_edge * r.storage_edge;
        pos += sizeof(r) + words * sizeof(float);
        if (pos > (unsigned long long)size) return bad("the file truncates a phase payload");
        float* dst = phi ? phi + packed : nullptr;
        if (!dst) {
            tmp.resize(words);
            dst = tmp.data();
        }
        if (!get(f.get(), dst, words * sizeof(float))) return bad("short read of a phase payload");
        c = crc.update(c, dst, words * sizeof(float));
        packed += words;
        if (cells) cell_of(r, B, cells + i);
    }
    if (pos != (unsigned long long)size)
        return set_error(PFB_E_FORMAT, "PF3D file has %lld bytes; its cell records require %llu", size, pos);
    if (c != h.crc) return bad("file CRC-64/ECMA mismatch");
    if (info) {
        info->step = h.step;
        info->time = h.time;
        info->num_cells = N;
        info->brick_edge = B;
        info->base_measure_shards = (int)h.base_shards;
        info->crc64 = h.crc;
    }
    if (rec_out) *rec_out = p;
    if (words_out) *words_out = packed;
    return PFB_OK;
}

int write3(const char* path, const pfb_ckpt3d_params* rec, long long step, int N, const pfb_cell3d* cells,
           const float* phi, int shards) {
    if (!path || !rec || !cells || !phi || N <= 0) return set_error(PFB_E_ARG, "PF3D write: bad argument");
    if (shards < 1 || shards > 64) return set_error(PFB_E_ARG, "PF3D write: base measurement shards must be 1..64");
    if (step < 0) return set_error(PFB_E_ARG, "PF3D write: negative step");
    Header3 h;
    std::memset(&h, 0, sizeof(h));
    h.magic = kMagic3;
    h.schema = kSchema3;
    h.header_bytes = (uint16_t)sizeof(Header3);
    h.endian = kEndian;
    h.dims = 3;
    h.scalar = 1;
    h.flags = kFlags3;
    h.step = step;
    h.time = (double)step * rec->dt;
    h.cells = (uint64_t)N;
    h.params_bytes = (uint32_t)sizeof(pfb_ckpt3d_params);
    h.record_bytes = (uint32_t)sizeof(Record3);
    h.brick = rec->brick_edge;
    h.order = 1;
    h.values_per_cell = (uint64_t)h.brick * h.brick * h.brick;
    h.bytes_per_cell = 4 * h.values_per_cell;
    h.base_shards = (uint64_t)shards;
    int rc = check_header(h);
    if (!rc) rc = check_params(*rec, h);
    if (rc) {
        const std::string why = pfb_last_error();
        return set_error(PFB_E_ARG, "PF3D write refused: %s", why.c_str());
    }
    const int B = (int)h.brick;
    std::vector<Record3> recs((size_t)N);
    std::vector<size_t> offs((size_t)N + 1, 0);
    for (int i = 0; i < N; ++i) {
        recs[(size_t)i] = record_of(cells[i], B);
        const size_t e = recs[(size_t)i].storage_edge;
        offs[(size_t)i + 1] = offs[(size_t)i] + e * e * e;
        if ((rc = check_record(recs[(size_t)i], i, B, *rec))) {
            const std::string why = pfb_last_error();
            return set_error(PFB_E_ARG, "PF3D write refused: %s", why.c_str());
        }
    }
    // the CRC covers the header (CRC field zero), the record, cells and bricks
    const Crc64& crc = crc_table();
    uint64_t c = crc.update(0, &h, sizeof(h));
    c = crc.update(c, rec, sizeof(*rec));
    for (int i = 0; i < N; ++i) {
        c = crc.update(c, &recs[(size_t)i], sizeof(Record3));
        c = crc.update(c, phi + offs[(size_t)i], (offs[(size_t)i + 1] - offs[(size_t)i]) * sizeof(float));
    }
    h.crc = c;
    const std::string tmp = std::string(path) + ".tmp";
    std::FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return set_error(PFB_E_IO, "cannot open %s: %s", tmp.c_str(), std::strerror(errno));
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 && std::fwrite(rec, sizeof(*rec), 1, f) == 1;
    for (int i = 0; ok && i < N; ++i) {
        const size_t words = offs[(size_t)i + 1] - offs[(size_t)i];
        ok = std::fwrite(&recs[(size_t)i], sizeof(Record3), 1, f) == 1 &&
             std::fwrite(phi + offs[(size_t)i], sizeof(float), words, f) == words;
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        std::remove(tmp.c_str());
        return set_error(PFB_E_IO, "writing %s failed", tmp.c_str());
    }
    if (std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        return set_error(PFB_E_IO, "rename to %s failed: %s", path, std::strerror(errno));
    }
    return PFB_OK;
}

}  // namespace

extern "C" {

uint64_t pfb_crc64_ecma(uint64_t crc, const void* data, size_t n) {
    return data ? crc_table().update(crc, data, n) : crc;
}

int pfb_ckpt3d_params_from(const pfb_params3d* p, int brick, pfb_ckpt3d_params* out) {
    clear_error();
    if (!p || !out) return set_error(PFB_E_ARG, "params_from: null argument");
    std::memset(out, 0, sizeof(*out));
    out->Nx = p->Nx;
    out->Ny = p->Ny;
    out->Nz = p->Nz;
    out->dx = out->dy = out->dz = 1.0;
    const int B = brick > 0 ? brick : (p->B > 0 ? p->B : pfb3d_automatic_brick_edge(p->target_radius, p->lambda));
    out->brick_edge = (uint32_t)B;
    out->boundary_flags = p->boundary_flags;
    out->dt = p->dt;
    out->t_end = 100.0;
    out->lambda = p->lambda;
    out->gamma_normal = p->gamma;
    out->gamma_soft = p->gamma_soft > 0.0 ? p->gamma_soft : p->gamma;
    out->soft_fraction = p->soft_fraction;
    out->kappa = p->kappa;
    out->target_radius = p->target_radius;
    out->mu = p->mu;
    out->v_A = p->v_A;
    out->v_A_sigma = p->v_A_sigma;
    out->xi = p->xi;
    out->tau = p->tau;
    const double R = p->target_radius, pi = 3.14159265358979323846;
    const double sphere = 4.0 * pi * R * R * R / 3.0;
    const double n = (double)p->num_cells;
    if (p->boundary_flags == kSlab)
        out->volume_fraction = n * pi * R * R / ((double)p->Nx * p->Ny);
    else if (p->boundary_flags == kChannel)
        out->volume_fraction = n * sphere / ((double)p->Nx * p->Ny * p->channel_height);
    else
        out->volume_fraction = n * sphere / ((double)p->Nx * p->Ny * p->Nz);
    out->seed = p->seed;
    out->polarity_seed = p->polarity_seed ? p->polarity_seed : p->seed;
    out->print_interval = 100;
    out->full_moment_every = p->full_moment_every;
    out->verify_every = 4096;
    out->integrator_id = 1;
    out->stencil_id = 2;
    out->rng_id = 1;
    out->aging_time = p->aging_time;
    out->channel_height = p->boundary_flags == kChannel ? p->channel_height : 0;
    out->channel_padding = p->boundary_flags == kChannel ? p->channel_padding : 0;
    out->wall_kappa = p->boundary_flags == kChannel ? p->wall_kappa : 0.0;
    out->wall_width = p->boundary_flags == kChannel ? p->wall_width : 0.0;
    return PFB_OK;
}

int pfb_ckpt3d_params_to(const pfb_ckpt3d_params* r, int num_cells, pfb_params3d* out) {
    clear_error();
    if (!r || !out || num_cells <= 0) return set_error(PFB_E_ARG, "params_to: bad argument");
    std::memset(out, 0, sizeof(*out));
    out->Nx = (int)r->Nx;
    out->Ny = (int)r->Ny;
    out->Nz = (int)r->Nz;
    out->boundary_flags = r->boundary_flags;
    out->num_cells = num_cells;
    out->B = (int)r->brick_edge;
    out->dt = r->dt;
    out->lambda = r->lambda;
    out->target_radius = r->target_radius;
    out->kappa = r->kappa;
    out->mu = r->mu;
    out->xi = r->xi;
    out->tau = r->tau;
    out->v_A = r->v_A;
    out->gamma = r->gamma_normal;
    out->gamma_soft = r->gamma_soft;
    out->soft_fraction = r->soft_fraction;
    out->v_A_sigma = r->v_A_sigma;
    out->aging_time = r->aging_time;
    out->wall_kappa = r->wall_kappa;
    out->wall_width = r->wall_width;
    out->channel_height = (int)r->channel_height;
    out->channel_padding = (int)r->channel_padding;
    out->seed = r->seed;
    out->polarity_seed = r->polarity_seed;
    out->full_moment_every = (int)r->full_moment_every;
    return PFB_OK;
}

int pfb_ckpt3d_read(const char* path, pfb_ckpt3d_info* info, pfb_ckpt3d_params* rec, pfb_cell3d* cells,
                    float* phi) {
    clear_error();
    if (!path) return set_error(PFB_E_ARG, "PF3D read: null path");
    if ((cells == nullptr) != (phi == nullptr)) return set_error(PFB_E_ARG, "PF3D read: cells and phi go together");
    return read3(path, info, rec, cells, phi);
}

int pfb_ckpt3d_write(const char* path, const pfb_ckpt3d_params* rec, long long step, int num_cells,
                     const pfb_cell3d* cells, const float* phi, int base_measure_shards) {
    clear_error();
    return write3(path, rec, step, num_cells, cells, phi, base_measure_shards);
}

int pfb_ckpt3d_payload_words(const char* path, unsigned long long* words) {
    clear_error();
    if (!path || !words) return set_error(PFB_E_ARG, "PF3D payload: null argument");
    return read3(path, nullptr, nullptr, nullptr, nullptr, words);
}

int pfb_sim3d_write_checkpoint(pfb_sim3d* s, const char* path, const pfb_ckpt3d_params* rec) {
    clear_error();
    if (!s || !path || !rec) return set_error(PFB_E_ARG, "write_checkpoint: null argument");
    pfb_layout3d lay;
    int rc = pfb_sim3d_layout(s, &lay);
    if (rc) return rc;
    const int B = pfb_sim3d_brick(s);
    if ((int)rec->brick_edge != B) return set_error(PFB_E_ARG, "record brick edge %u differs from the system's %d",
                                                    rec->brick_edge, B);
    const long long step = pfb_sim3d_step(s);
    // the cell count is the record-independent size of the system
    int N = 0;
    {
        pfb_measure_args3d m;
        rc = pfb_sim3d_measure_args(s, &m);
        if (rc) return rc;
        N = m.N;
    }
    // the reference measures the current state before it writes
    rc = pfb_sim3d_measure_current(s);
    if (rc) return rc;
    unsigned long long words = 0;
    rc = pfb_sim3d_packed_words(s, &words);
    if (rc) return rc;
    std::vector<pfb_cell3d> cells((size_t)N);
    std::vector<float> phi((size_t)words);
    rc = pfb_sim3d_get_cells(s, cells.data());
    if (!rc) rc = pfb_sim3d_get_packed(s, phi.data());
    if (rc) return rc;
    // the base measurement here reduces each cell over a cluster of 4 CTAs
    return write3(path, rec, step, N, cells.data(), phi.data(), 4);
}

pfb_sim3d* pfb_sim3d_create_from_checkpoint(const char* path, int device) {
    return pfb_sim3d_create_from_checkpoint_ex(path, device, PFB3D_MEMORY_AUTO, 0);
}

pfb_sim3d* pfb_sim3d_create_from_checkpoint_ex(const char* path, int device, int memory_mode,
                                               int scratch_slots) {
    clear_error();
    pfb_ckpt3d_info info;
    pfb_ckpt3d_params rec;
    unsigned long long words = 0;
    if (read3(path, &info, &rec, nullptr, nullptr, &words)) return nullptr;
    std::vector<pfb_cell3d> cells((size_t)info.num_cells);
    std::vector<float> phi((size_t)words);
    if (read3(path, &info, &rec, cells.data(), phi.data())) return nullptr;
    pfb_params3d p;
    if (pfb_ckpt3d_params_to(&rec, info.num_cells, &p)) return nullptr;
    return pfb_sim3d_create_from_state_ex(&p, cells.data(), phi.data(), info.step, device, memory_mode,
                                          scratch_slots);
}

}  // extern "C"
