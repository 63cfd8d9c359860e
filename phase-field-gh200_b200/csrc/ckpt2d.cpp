// The reference's 2D checkpoint file (PF "CELL" schema 1): reader and writer
// with the reference's acceptance rules (common/checkpoint_format.h:1-149,
// src/checkpoint.cu:27-45 (helpers), 117-141 (tile extents), 145-241
// (sidecars), 348-615 (reader), 823-1011 (writer); parameter checks of
// include/params.cuh:596-788). The byte layout has to be the reference's, so
// the on-disk records below keep its field order and sizes; everything else
// is this library's own code.
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

#include "pfb_common.cuh"
#include "pfb_internal.h"
#include "pfb200_ckpt.h"

using namespace pfb;

namespace {

constexpr uint32_t kMagicCell = 0x43454C4Cu;  // 'CELL'
constexpr uint32_t kSchema = 1u;
constexpr int32_t kPitch = 288;
constexpr uint32_t kPOLR = 0x504F4C52u, kGAMA = 0x47414D41u, kVA_A = 0x56415F41u,
                   kRADI = 0x52414449u, kMOBI = 0x4D4F4249u;
constexpr double kMobility0 = 0.5;                 // default phase-field mobility
constexpr double kLapBound = 40.0 / 6.0;           // 9-point Laplacian row-sum bound
constexpr int kMaxCells = 4000000;

#pragma pack(push, 1)
struct Prefix {
    uint32_t magic, schema;
    int32_t step;
    double time;
    int32_t cells, save_interval, zero, traj_samples;
    uint8_t flags[4];
    uint32_t record_bytes;
};
struct Ranks {
    int32_t ranks, rank, cells;
};
struct CellHeader {
    int32_t id, tile_x, tile_y, cls;
    uint32_t promote, zero0;
    float cx, cy, vx, vy;
    double V, Mx, My, perim;
    int32_t lo_x, hi_x, lo_y, hi_y;
    float phi_max;
    uint32_t zero1;
};
struct Sidecar {
    uint32_t magic;
    int32_t count;
};
#pragma pack(pop)
static_assert(sizeof(Prefix) == 44 && sizeof(Ranks) == 12 && sizeof(CellHeader) == 96 &&
                  sizeof(Sidecar) == 8 && sizeof(pfb_ckpt2d_params) == 192,
              "checkpoint record sizes");
static_assert(offsetof(pfb_ckpt2d_params, seed) == 136 &&
                  offsetof(pfb_ckpt2d_params, trajectory_interval) == 184 &&
                  offsetof(CellHeader, V) == 40 && offsetof(CellHeader, phi_max) == 88,
              "checkpoint field offsets");

struct FileCloser {
    void operator()(std::FILE* f) const {
        if (f) std::fclose(f);
    }
};
using File = std::unique_ptr<std::FILE, FileCloser>;

int wrap_i(long long v, int L) {
    v %= L;
    return (int)(v < 0 ? v + L : v);
}
double wrap_d(double v, double L) {
    const double m = std::fmod(v, L);
    return m < 0.0 ? m + L : m;
}

bool get(std::FILE* f, void* dst, size_t n) { return n == 0 || std::fread(dst, 1, n, f) == n; }

// The reference's startup validation of a parameter set whose per-cell
// mobilities are resolved (a checkpoint): the checks that decide acceptance.
int check_params(const pfb_ckpt2d_params& r, int N) {
    auto bad = [](const char* why) { return set_error(PFB_E_FORMAT, "checkpoint parameters: %s", why); };
    if (!(r.dx == 1.0 && r.dy == 1.0)) return bad("dx and dy must both be 1");
    if (r.Nx != r.Ny) return bad("Nx must equal Ny");
    if (r.Nx <= 286) return bad("domain side must exceed the largest window (286)");
    if (r.Nx > (1 << 30)) return bad("domain side too large");
    if (N <= 0) return bad("num_cells must be positive");
    if (!std::isfinite(r.lambda) || !(r.lambda > 0.0)) return bad("lambda must be finite and positive");
    if (!std::isfinite(r.target_radius) || !(r.target_radius > 0.0)) return bad("radius must be finite and positive");
    if (!std::isfinite(r.dt) || !(r.dt > 0.0)) return bad("dt must be finite and positive");
    if (!std::isfinite(r.t_end) || r.t_end < 0.0) return bad("t_end must be finite and non-negative");
    if (r.t_end / r.dt >= 9.0e18) return bad("t_end / dt does not fit a 64-bit step count");
    if (!std::isfinite(r.xi) || !(r.xi > 0.0)) return bad("xi must be finite and positive");
    if (!std::isfinite(r.tau) || !(r.tau > 0.0)) return bad("tau must be finite and positive");
    if (!std::isfinite(r.kappa) || r.kappa < 0.0) return bad("kappa must be finite and non-negative");
    if (!std::isfinite(r.mu) || r.mu < 0.0) return bad("mu must be finite and non-negative");
    if (!std::isfinite(r.v_A) || r.v_A < 0.0 || !std::isfinite(r.v_A_sigma) || r.v_A_sigma < 0.0)
        return bad("v_A and v_A_sigma must be finite and non-negative");
    if (!std::isfinite(r.gamma_normal) || !std::isfinite(r.gamma_soft) || !(r.gamma_normal > 0.0) ||
        !(r.gamma_soft > 0.0))
        return bad("both gamma values must be finite and positive");
    if (!std::isfinite(r.soft_fraction) || !(r.soft_fraction >= 0.0 && r.soft_fraction <= 1.0))
        return bad("cancer fraction must lie in [0, 1]");
    if (!std::isfinite(r.rho) || !(r.rho > 0.0 && r.rho < 1.0)) return bad("rho must lie in (0, 1)");
    if (r.print_interval < 0 || r.full_moment_every < 0 || r.verify_every < 0)
        return bad("output and verification intervals must be non-negative");
    return PFB_OK;
}

// Explicit-Euler bound over the resolved per-cell pairs (gamma_i, M_i):
// dt * max_i (M_i / M0) gamma_i * (Laplacian row-sum bound) must stay below 1.
int check_stiffness(double dt, const std::vector<float>& gamma, const std::vector<float>& mob) {
    double gmax = 0.0;
    for (size_t i = 0; i < gamma.size(); ++i) {
        const double g = gamma[i], m = mob[i];
        if (!(g > 0.0) || !std::isfinite(g) || !(m > 0.0) || !std::isfinite(m))
            return set_error(PFB_E_FORMAT, "cell %zu has gamma %.9g, mobility %.9g: both must be "
                             "positive and finite", i, g, m);
        gmax = std::fmax(gmax, (m / kMobility0) * g);
    }
    if (dt * gmax * kLapBound >= 1.0)
        return set_error(PFB_E_FORMAT, "dt * max (M_i / M0) gamma_i * laplacian bound = %.4f >= 1",
                         dt * gmax * kLapBound);
    return PFB_OK;
}

// Bounding boxes of a tile: values above the support threshold and nonzero
// values, in tile coordinates; false when nothing exceeds the threshold.
bool extents(const float* t, int sup[4], int nz[4]) {
    sup[0] = sup[2] = nz[0] = nz[2] = kPitch;
    sup[1] = sup[3] = nz[1] = nz[3] = -1;
    for (int y = 0; y < kPitch; ++y)
        for (int x = 0; x < kPitch; ++x) {
            const float v = t[(size_t)y * kPitch + x];
            if (v == 0.0f) continue;
            nz[0] = std::min(nz[0], x), nz[1] = std::max(nz[1], x);
            nz[2] = std::min(nz[2], y), nz[3] = std::max(nz[3], y);
            if (v <= kSupportEps) continue;
            sup[0] = std::min(sup[0], x), sup[1] = std::max(sup[1], x);
            sup[2] = std::min(sup[2], y), sup[3] = std::max(sup[3], y);
        }
    return sup[1] >= 0;
}

int read_file(const char* path, pfb_ckpt2d_info* info, pfb_ckpt2d_params* rec_out, pfb_cell2d* cells,
              float* phi) {
    File f(std::fopen(path, "rb"));
    if (!f) return set_error(PFB_E_IO, "cannot open %s: %s", path, std::strerror(errno));
    Prefix pre;
    if (!get(f.get(), &pre, sizeof(pre))) return set_error(PFB_E_FORMAT, "short read of the prefix");
    if (pre.magic != kMagicCell)
        return set_error(PFB_E_FORMAT, "%s is not a cell checkpoint (magic 0x%08X)", path, pre.magic);
    if (pre.schema != kSchema)
        return set_error(PFB_E_FORMAT, "unsupported 2D checkpoint schema %u (expected 1)", pre.schema);
    if (pre.step < 0 || pre.zero != 0 || pre.save_interval < 0 || pre.traj_samples < 0 ||
        pre.flags[0] || pre.flags[1] || pre.flags[2] || pre.flags[3])
        return set_error(PFB_E_FORMAT, "fixed checkpoint metadata is invalid or unsupported");
    if (pre.record_bytes != sizeof(pfb_ckpt2d_params))
        return set_error(PFB_E_FORMAT, "parameter record is %u B (expected 192)", pre.record_bytes);
    if (pre.cells <= 0 || pre.cells > kMaxCells)
        return set_error(PFB_E_FORMAT, "implausible cell count %d", pre.cells);
    pfb_ckpt2d_params rec;
    if (!get(f.get(), &rec, sizeof(rec))) return set_error(PFB_E_FORMAT, "short read of the parameter record");
    if (rec.reserved != 0 || rec.save_interval != pre.save_interval ||
        rec.trajectory_samples != pre.traj_samples || rec.trajectory_samples <= 0 ||
        rec.trajectory_interval < 0)
        return set_error(PFB_E_FORMAT, "parameter metadata is internally inconsistent");
    int32_t pitch = 0;
    if (!get(f.get(), &pitch, sizeof(pitch))) return set_error(PFB_E_FORMAT, "short read of the tile pitch");
    if (pitch != kPitch) return set_error(PFB_E_FORMAT, "tile pitch %d (expected 288)", pitch);
    Ranks rk;
    if (!get(f.get(), &rk, sizeof(rk))) return set_error(PFB_E_FORMAT, "short read of the rank trailer");
    if (rk.ranks != 1 || rk.rank != 0 || rk.cells != pre.cells)
        return set_error(PFB_E_FORMAT, "not a complete single-GPU checkpoint");
    const int N = pre.cells;
    const double t_expect = (double)pre.step * rec.dt;
    if (!std::isfinite(pre.time) || !std::isfinite(t_expect) ||
        std::fabs(pre.time - t_expect) > 1e-12 * std::fmax(1.0, std::fabs(t_expect)))
        return set_error(PFB_E_FORMAT, "checkpoint time does not match step * dt");
    int rc = check_params(rec, N);
    if (rc) return rc;
    const int L = rec.Nx;

    std::vector<float> tile((size_t)kPitch * kPitch);
    std::vector<pfb_cell2d> tmp;
    if (cells) std::memset(cells, 0, (size_t)N * sizeof(pfb_cell2d));
    for (int i = 0; i < N; ++i) {
        CellHeader h;
        if (!get(f.get(), &h, sizeof(h)) || !get(f.get(), tile.data(), tile.size() * sizeof(float)))
            return set_error(PFB_E_FORMAT, "short read of cell %d", i);
        if (h.id != i) return set_error(PFB_E_FORMAT, "cell slot %d carries id %d (ids must be 0..N-1)", i, h.id);
        if (h.cls < 0 || h.cls >= kNumClasses || h.promote >= (uint32_t)kDemoteDwell || h.zero0 ||
            h.zero1 || h.tile_x < 0 || h.tile_x >= L || h.tile_y < 0 || h.tile_y >= L ||
            !std::isfinite(h.cx) || !std::isfinite(h.cy) || !std::isfinite(h.vx) ||
            !std::isfinite(h.vy) || !std::isfinite(h.V) || !(h.V > 0.0) || !std::isfinite(h.Mx) ||
            !std::isfinite(h.My) || !std::isfinite(h.perim) || h.perim < 0.0 ||
            !std::isfinite(h.phi_max) || h.phi_max < 0.0f)
            return set_error(PFB_E_FORMAT, "cell %d has invalid state metadata", i);
        const Window w = window_of(h.cls);
        if (h.lo_x < 0 || h.hi_x < h.lo_x || h.hi_x >= w.wx || h.lo_y < 0 || h.hi_y < h.lo_y ||
            h.hi_y >= w.wy)
            return set_error(PFB_E_FORMAT, "cell %d support does not fit class %d", i, h.cls);
        float vmax = 0.0f;
        for (float v : tile) {
            if (!std::isfinite(v)) return set_error(PFB_E_FORMAT, "cell %d phase field is not finite", i);
            vmax = std::fmax(vmax, std::fabs(v));
        }
        int sup[4], nz[4];
        if (!extents(tile.data(), sup, nz))
            return set_error(PFB_E_FORMAT, "cell %d has no phase-field support", i);
        if (sup[0] != w.tx0 + h.lo_x || sup[1] != w.tx0 + h.hi_x || sup[2] != w.ty0 + h.lo_y ||
            sup[3] != w.ty0 + h.hi_y || nz[0] < w.tx0 || nz[1] >= w.tx0 + w.wx || nz[2] < w.ty0 ||
            nz[3] >= w.ty0 + w.wy || vmax != h.phi_max)
            return set_error(PFB_E_FORMAT, "cell %d phase field disagrees with its class or moments", i);
        const float ecx = (float)wrap_d((double)h.tile_x + w.tx0 + h.Mx / h.V, (double)L);
        const float ecy = (float)wrap_d((double)h.tile_y + w.ty0 + h.My / h.V, (double)L);
        if (h.cx != ecx || h.cy != ecy)
            return set_error(PFB_E_FORMAT, "cell %d centroid is internally inconsistent", i);
        if (cells) {
            pfb_cell2d& c = cells[i];
            c.global_id = h.id;
            c.gx0 = wrap_i((long long)h.tile_x + w.tx0, L);
            c.gy0 = wrap_i((long long)h.tile_y + w.ty0, L);
            c.cls = (uint8_t)h.cls;
            c.cls_written[0] = c.cls_written[1] = (uint8_t)h.cls;
            c.vx = h.vx;
            c.vy = h.vy;
            c.V = h.V;
            c.Cx = h.Mx;
            c.Cy = h.My;
            c.perim = h.perim;
            c.bb_lo_x = h.lo_x;
            c.bb_hi_x = h.hi_x;
            c.bb_lo_y = h.lo_y;
            c.bb_hi_y = h.hi_y;
            c.promote_ctr = h.promote;
            c.phi_max = h.phi_max;
            c.M_pf = (float)kMobility0;
        }
        if (phi) std::memcpy(phi + (size_t)i * kTileArea, tile.data(), tile.size() * sizeof(float));
    }

    // sidecars: each of POLR, GAMA, VA_A, RADI exactly once, MOBI at most once
    std::vector<float> vals, gamma((size_t)N), mob((size_t)N, (float)kMobility0);
    bool seen_polr = false, seen_gama = false, seen_va = false, seen_radi = false, seen_mobi = false;
    for (;;) {
        Sidecar sc;
        const size_t got = std::fread(&sc, 1, sizeof(sc), f.get());
        if (got == 0) break;
        if (got != sizeof(sc)) return set_error(PFB_E_FORMAT, "truncated sidecar header");
        bool* seen = sc.magic == kPOLR   ? &seen_polr
                     : sc.magic == kGAMA ? &seen_gama
                     : sc.magic == kVA_A ? &seen_va
                     : sc.magic == kRADI ? &seen_radi
                     : sc.magic == kMOBI ? &seen_mobi
                                         : nullptr;
        if (!seen) return set_error(PFB_E_FORMAT, "unsupported sidecar 0x%08X", sc.magic);
        if (sc.count != N)
            return set_error(PFB_E_FORMAT, "sidecar 0x%08X has %d entries (expected %d)", sc.magic, sc.count, N);
        if (*seen) return set_error(PFB_E_FORMAT, "duplicate sidecar 0x%08X", sc.magic);
        *seen = true;
        vals.assign((size_t)N, 0.0f);
        if (!get(f.get(), vals.data(), vals.size() * sizeof(float)))
            return set_error(PFB_E_FORMAT, "short read of sidecar 0x%08X", sc.magic);
        for (int i = 0; i < N; ++i) {
            const float v = vals[(size_t)i];
            const bool ok = std::isfinite(v) &&
                            (sc.magic == kPOLR || (sc.magic == kVA_A ? v >= 0.0f : v > 0.0f));
            if (!ok) return set_error(PFB_E_FORMAT, "sidecar 0x%08X has an invalid value at cell %d", sc.magic, i);
        }
        if (sc.magic == kGAMA) gamma = vals;
        if (sc.magic == kMOBI) mob = vals;
        if (cells)
            for (int i = 0; i < N; ++i) {
                const float v = vals[(size_t)i];
                pfb_cell2d& c = cells[i];
                if (sc.magic == kPOLR) c.theta = v;
                else if (sc.magic == kGAMA) c.gamma = v;
                else if (sc.magic == kVA_A) c.v_A = v;
                else if (sc.magic == kRADI) c.R_tgt = v;
                else c.M_pf = v;
            }
    }
    if (!seen_polr || !seen_gama || !seen_va || !seen_radi)
        return set_error(PFB_E_FORMAT, "checkpoint is missing required sidecars:%s%s%s%s",
                         seen_polr ? "" : " POLR", seen_gama ? "" : " GAMA", seen_va ? "" : " VA_A",
                         seen_radi ? "" : " RADI");
    rc = check_stiffness(rec.dt, gamma, mob);
    if (rc) return rc;
    if (info) {
        info->step = pre.step;
        info->time = pre.time;
        info->num_cells = N;
        info->L = L;
        info->had_mobility = seen_mobi ? 1 : 0;
    }
    if (rec_out) *rec_out = rec;
    return PFB_OK;
}

// Writes go to path.tmp; the rename happens only after a clean close.
class TmpFile {
public:
    explicit TmpFile(const char* path) : final_(path), tmp_(std::string(path) + ".tmp") {
        f_ = std::fopen(tmp_.c_str(), "wb");
    }
    ~TmpFile() {
        if (f_) {
            std::fclose(f_);
            std::remove(tmp_.c_str());
        }
    }
    bool ok() const { return f_ != nullptr; }
    bool put(const void* p, size_t n) { return n == 0 || std::fwrite(p, 1, n, f_) == n; }
    int commit() {
        const int c = std::fclose(f_);
        f_ = nullptr;
        if (c != 0) {
            std::remove(tmp_.c_str());
            return set_error(PFB_E_IO, "closing %s failed: %s", tmp_.c_str(), std::strerror(errno));
        }
        if (std::rename(tmp_.c_str(), final_.c_str()) != 0) {
            std::remove(tmp_.c_str());
            return set_error(PFB_E_IO, "rename to %s failed: %s", final_.c_str(), std::strerror(errno));
        }
        return PFB_OK;
    }
    const std::string& tmp() const { return tmp_; }

private:
    std::string final_, tmp_;
    std::FILE* f_ = nullptr;
};

int write_file(const char* path, const pfb_ckpt2d_params* rec, long long step, int N,
               const pfb_cell2d* cells, const float* phi) {
    if (!path || !rec || !cells || !phi || N <= 0) return set_error(PFB_E_ARG, "checkpoint write: bad argument");
    if (rec->trajectory_samples <= 0 || rec->trajectory_interval < 0 || rec->save_interval < 0 ||
        rec->reserved != 0)
        return set_error(PFB_E_ARG, "checkpoint write: invalid output schedule metadata");
    int rc = check_params(*rec, N);
    if (rc) return rc;
    if (step < 0 || step > 2147483647LL)
        return set_error(PFB_E_ARG, "step %lld does not fit the checkpoint's int32 field", step);
    const int L = rec->Nx;
    std::vector<float> gamma((size_t)N), mob((size_t)N);
    for (int i = 0; i < N; ++i) {
        gamma[(size_t)i] = cells[i].gamma;
        mob[(size_t)i] = cells[i].M_pf;
    }
    rc = check_stiffness(rec->dt, gamma, mob);
    if (rc) return rc;
    // validate every cell before anything is written
    for (int i = 0; i < N; ++i) {
        const pfb_cell2d& c = cells[i];
        if (c.global_id != i) return set_error(PFB_E_ARG, "cell slot %d carries id %d", i, c.global_id);
        if (!std::isfinite(c.gamma) || !(c.gamma > 0.0f) || !std::isfinite(c.v_A) || c.v_A < 0.0f ||
            !std::isfinite(c.R_tgt) || !(c.R_tgt > 0.0f) || !std::isfinite(c.theta) ||
            !std::isfinite(c.vx) || !std::isfinite(c.vy) || !std::isfinite(c.V) || !(c.V > 0.0) ||
            !std::isfinite(c.Cx) || !std::isfinite(c.Cy) || !std::isfinite(c.perim) || c.perim < 0.0 ||
            !std::isfinite(c.phi_max) || c.phi_max < 0.0f || c.gx0 < 0 || c.gx0 >= L || c.gy0 < 0 ||
            c.gy0 >= L || c.promote_ctr >= (uint32_t)kDemoteDwell)
            return set_error(PFB_E_ARG, "cell %d has invalid state; checkpoint not written", i);
        if (c.cls >= kNumClasses || c.cls_written[step & 1] != c.cls)
            return set_error(PFB_E_ARG, "cell %d class %d disagrees with its written class", i, c.cls);
        const Window w = window_of(c.cls);
        if (c.bb_lo_x < 0 || c.bb_hi_x < c.bb_lo_x || c.bb_hi_x >= w.wx || c.bb_lo_y < 0 ||
            c.bb_hi_y < c.bb_lo_y || c.bb_hi_y >= w.wy)
            return set_error(PFB_E_ARG, "cell %d support bounds are invalid", i);
    }
    TmpFile out(path);
    if (!out.ok()) return set_error(PFB_E_IO, "cannot open %s: %s", out.tmp().c_str(), std::strerror(errno));
    Prefix pre;
    std::memset(&pre, 0, sizeof(pre));
    pre.magic = kMagicCell;
    pre.schema = kSchema;
    pre.step = (int32_t)step;
    pre.time = (double)step * rec->dt;
    pre.cells = N;
    pre.save_interval = rec->save_interval;
    pre.traj_samples = rec->trajectory_samples;
    pre.record_bytes = (uint32_t)sizeof(pfb_ckpt2d_params);
    const int32_t pitch = kPitch;
    const Ranks rk{1, 0, N};
    bool ok = out.put(&pre, sizeof(pre)) && out.put(rec, sizeof(*rec)) && out.put(&pitch, sizeof(pitch)) &&
              out.put(&rk, sizeof(rk));
    for (int i = 0; ok && i < N; ++i) {
        const pfb_cell2d& c = cells[i];
        const Window w = window_of(c.cls);
        CellHeader h;
        std::memset(&h, 0, sizeof(h));
        h.id = c.global_id;
        h.tile_x = wrap_i((long long)c.gx0 - w.tx0, L);
        h.tile_y = wrap_i((long long)c.gy0 - w.ty0, L);
        h.cls = c.cls;
        h.promote = c.promote_ctr;
        const double inv = 1.0 / c.V;  // the reference's writer multiplies by 1/V
        h.cx = (float)wrap_d((double)c.gx0 + c.Cx * inv, (double)L);
        h.cy = (float)wrap_d((double)c.gy0 + c.Cy * inv, (double)L);
        h.vx = c.vx;
        h.vy = c.vy;
        h.V = c.V;
        h.Mx = c.Cx;
        h.My = c.Cy;
        h.perim = c.perim;
        h.lo_x = c.bb_lo_x;
        h.hi_x = c.bb_hi_x;
        h.lo_y = c.bb_lo_y;
        h.hi_y = c.bb_hi_y;
        h.phi_max = c.phi_max;
        ok = out.put(&h, sizeof(h)) && out.put(phi + (size_t)i * kTileArea, (size_t)kTileArea * sizeof(float));
    }
    std::vector<float> col((size_t)N);
    const uint32_t order[5] = {kPOLR, kGAMA, kVA_A, kRADI, kMOBI};
    for (int k = 0; ok && k < 5; ++k) {
        for (int i = 0; i < N; ++i) {
            const pfb_cell2d& c = cells[i];
            col[(size_t)i] = order[k] == kPOLR ? c.theta
                             : order[k] == kGAMA ? c.gamma
                             : order[k] == kVA_A ? c.v_A
                             : order[k] == kRADI ? c.R_tgt
                                                 : c.M_pf;
        }
        const Sidecar sc{order[k], N};
        ok = out.put(&sc, sizeof(sc)) && out.put(col.data(), col.size() * sizeof(float));
    }
    if (!ok) return set_error(PFB_E_IO, "short write to %s", out.tmp().c_str());
    return out.commit();
}

}  // namespace

extern "C" {

int pfb_ckpt2d_params_from(const pfb_params2d* p, pfb_ckpt2d_params* out) {
    clear_error();
    if (!p || !out) return set_error(PFB_E_ARG, "params_from: null argument");
    std::memset(out, 0, sizeof(*out));
    out->Nx = out->Ny = p->L;
    out->dx = out->dy = 1.0;
    out->dt = p->dt;
    out->t_end = 100.0;
    const double area = 3.14159265358979323846 * p->target_radius * p->target_radius;
    out->rho = (double)p->num_cells * area / ((double)p->L * (double)p->L);
    out->lambda = p->lambda;
    out->gamma_normal = p->gamma_normal;
    out->gamma_soft = p->gamma_cancer;
    out->soft_fraction = p->cancer_fraction;
    out->kappa = p->kappa;
    out->target_radius = p->target_radius;
    out->mu = p->mu;
    out->v_A = p->v_A;
    out->v_A_sigma = p->v_A_sigma;
    out->xi = p->xi;
    out->tau = p->tau;
    out->seed = p->seed;
    out->polarity_seed = p->polarity_seed ? p->polarity_seed : p->seed;
    out->initialization_hash = 0;
    out->print_interval = 100;
    out->full_moment_every = p->full_moment_every;
    out->verify_every = 4096;
    out->save_interval = 0;
    out->trajectory_samples = 100;
    out->reserved = 0;
    out->trajectory_interval = 0;
    return PFB_OK;
}

int pfb_ckpt2d_params_to(const pfb_ckpt2d_params* r, int num_cells, pfb_params2d* out) {
    clear_error();
    if (!r || !out || num_cells <= 0) return set_error(PFB_E_ARG, "params_to: bad argument");
    std::memset(out, 0, sizeof(*out));
    out->L = r->Nx;
    out->num_cells = num_cells;
    out->dt = r->dt;
    out->lambda = r->lambda;
    out->target_radius = r->target_radius;
    out->kappa = r->kappa;
    out->mu = r->mu;
    out->xi = r->xi;
    out->tau = r->tau;
    out->v_A = r->v_A;
    out->gamma_normal = r->gamma_normal;
    out->gamma_cancer = r->gamma_soft;
    out->cancer_fraction = r->soft_fraction;
    out->v_A_sigma = r->v_A_sigma;
    out->phase_field_mobility = kMobility0;
    out->seed = r->seed;
    out->polarity_seed = r->polarity_seed;
    out->full_moment_every = r->full_moment_every;
    out->phi_storage = 0;
    return PFB_OK;
}

int pfb_ckpt2d_read(const char* path, pfb_ckpt2d_info* info, pfb_ckpt2d_params* rec, pfb_cell2d* cells,
                    float* phi) {
    clear_error();
    if (!path) return set_error(PFB_E_ARG, "checkpoint read: null path");
    if ((cells == nullptr) != (phi == nullptr))
        return set_error(PFB_E_ARG, "checkpoint read: cells and phi go together");
    return read_file(path, info, rec, cells, phi);
}

int pfb_ckpt2d_write(const char* path, const pfb_ckpt2d_params* rec, long long step, int num_cells,
                     const pfb_cell2d* cells, const float* phi) {
    clear_error();
    return write_file(path, rec, step, num_cells, cells, phi);
}

int pfb_sim2d_write_checkpoint(pfb_sim2d* s, const char* path, const pfb_ckpt2d_params* rec) {
    clear_error();
    if (!s || !path || !rec) return set_error(PFB_E_ARG, "write_checkpoint: null argument");
    const int N = pfb_sim2d_num_cells(s);
    if (N <= 0) return set_error(PFB_E_ARG, "write_checkpoint: empty system");
    std::vector<pfb_cell2d> cells((size_t)N);
    std::vector<float> phi((size_t)N * kTileArea);
    int rc = pfb_sim2d_get_cells(s, cells.data());
    if (!rc) rc = pfb_sim2d_get_phi(s, phi.data());
    if (rc) return rc;
    return write_file(path, rec, pfb_sim2d_step(s), N, cells.data(), phi.data());
}

pfb_sim2d* pfb_sim2d_create_from_checkpoint(const char* path, int device) {
    clear_error();
    pfb_ckpt2d_info info;
    pfb_ckpt2d_params rec;
    if (read_file(path, &info, &rec, nullptr, nullptr)) return nullptr;
    std::vector<pfb_cell2d> cells((size_t)info.num_cells);
    std::vector<float> phi((size_t)info.num_cells * kTileArea);
    if (read_file(path, &info, &rec, cells.data(), phi.data())) return nullptr;
    pfb_params2d p;
    if (pfb_ckpt2d_params_to(&rec, info.num_cells, &p)) return nullptr;
    return pfb_sim2d_create_from_state(&p, cells.data(), phi.data(), info.step, device);
}

}  // extern "C"
