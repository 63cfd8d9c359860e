// pfb_cell_3d: the command line of the 3D run, with the reference's options,
// fresh placement, files and cadences (reference src/pf3d/main.cu:136-1000
// options and their ranges, geometry resolution, resume contract;
// src/pf3d/sim.cu:900-1135 fresh centres, 1183-1218 trajectory cadence,
// 1782-2036 trajectory file, 2142-2270 run loop;
// include/pf3d/palmieri_initializer.hpp:56-125 and 349-410 sequential
// placements; include/pf3d/initializer.hpp:97-124 centre-table hash;
// include/pf3d/trajectory_header.hpp metadata line). Everything goes through
// the library's C ABI.
//
// The PFB3D boundary recorder (--boundary-out; reference
// src/pf3d/boundary_output.cu) writes its opening frame at initialisation,
// frames on the grid of --boundary-interval and a closing frame after the
// final checkpoint. --initial-centres reads the reference's centre tables
// (periodic x,y,z; relaxed x,y for the slab and the one-layer channel;
// channel x,y,z). Soft cells (--cancer-fraction, --gamma-cancer) take
// their identities from the reference's Philox shuffle. Cells whose support
// reaches their brick grow into larger cubes (adaptive bricks), and
// --memory-mode / --scratch-slots select the storage, as in the reference.
// Not part of this build (exit status 2 with a message): the peer device and
// measurement groupings other than this build's (--measure-shards 4,
// --promoted-measure-shards 0), which the trajectory header and checkpoints
// state.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <random>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "centres_csv.hpp"
#include "pfb200.h"
#include "pfb200_3d.h"
#include "pfb200_ckpt.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMeasureShards = 4;
constexpr long long kNever = std::numeric_limits<long long>::max();
volatile std::sig_atomic_t g_stop = 0;
void on_signal(int) { g_stop = 1; }

enum Geometry { kPeriodic, kSlab, kChannel };

struct Options {
    pfb_params3d p{};
    Geometry geometry = kPeriodic;
    double rho = 0.90, t_end = 100.0, gamma_soft = 0.35, soft_fraction = 0.0;
    int slab_height = 0, channel_height = 0, wall_padding = 0;
    long long brick = 0, device = 0, bench = 0, print_interval = 100, verify_every = 4096;
    int mem_mode = PFB3D_MEMORY_AUTO, scratch_slots = 0;
    long long traj_samples = 100, traj_interval = 0, ckpt_interval = 0, save_interval = 0;
    bool final_ckpt = true;
    // which options the command line supplied
    bool model_given = false, t_end_given = false, print_given = false, samples_given = false,
         interval_given = false, ckpt_dir_given = false, schedule_given = false, slab_h_given = false,
         channel_h_given = false, wall_k_given = false, wall_w_given = false, pad_given = false;
    std::string ckpt_in, ckpt_dir, out_path;
    std::string bnd_path;
    long long bnd_interval = 0;
    int bnd_projection = PFB3D_PROJECTION_MAXIMUM;
    bool bnd_compress = false, bnd_given = false;
    std::string centres_path;  // --initial-centres
    bool strict = false;
};

bool parse_real(const char* flag, const char* s, double lo, double hi, double* v) {
    char* e = nullptr;
    errno = 0;
    const double x = std::strtod(s, &e);
    if (errno == ERANGE || e == s || *e != '\0' || !std::isfinite(x) || x < lo || x > hi) {
        std::fprintf(stderr, "[3d] %s expects a finite number in [%.9g, %.9g], got '%s'\n", flag, lo, hi, s);
        return false;
    }
    *v = x;
    return true;
}
bool parse_int(const char* flag, const char* s, long long lo, long long hi, long long* v) {
    char* e = nullptr;
    errno = 0;
    const long long x = std::strtoll(s, &e, 10);
    if (errno == ERANGE || e == s || *e != '\0' || x < lo || x > hi) {
        std::fprintf(stderr, "[3d] %s expects an integer in [%lld, %lld], got '%s'\n", flag, lo, hi, s);
        return false;
    }
    *v = x;
    return true;
}
bool parse_u64(const char* flag, const char* s, uint64_t* v) {
    char* e = nullptr;
    errno = 0;
    const unsigned long long x = s[0] == '-' ? 0 : std::strtoull(s, &e, 10);
    if (s[0] == '-' || errno == ERANGE || e == s || *e != '\0') {
        std::fprintf(stderr, "[3d] %s expects an unsigned integer, got '%s'\n", flag, s);
        return false;
    }
    *v = x;
    return true;
}

// [0, 1) from the top 53 bits of a 64-bit draw.
double u53(std::mt19937_64& g) { return (double)(g() >> 11) * 0x1.0p-53; }
double min_image(double d, double side) { return d - side * std::floor(d / side + 0.5); }

// Sequential placement in the periodic box: cell 0 at the centre, then
// candidates x, y, z drawn from mt19937_64(seed) and accepted at periodic
// distance >= r from every accepted centre, stored binary32 before later
// tests.
void periodic_centres(int n, double side, double r, uint64_t seed, std::vector<float>& x,
                      std::vector<float>& y, std::vector<float>& z) {
    x.assign(1, (float)(0.5 * side));
    y.assign(1, (float)(0.5 * side));
    z.assign(1, (float)(0.5 * side));
    std::mt19937_64 g(seed);
    const double r2 = r * r;
    while ((int)x.size() < n) {
        const double cx = side * u53(g), cy = side * u53(g), cz = side * u53(g);
        bool ok = true;
        for (size_t j = 0; j < x.size() && ok; ++j) {
            const double dx = min_image(cx - x[j], side), dy = min_image(cy - y[j], side),
                         dz = min_image(cz - z[j], side);
            ok = !(dx * dx + dy * dy + dz * dz < r2);
        }
        if (!ok) continue;
        x.push_back((float)cx);
        y.push_back((float)cy);
        z.push_back((float)cz);
    }
}

// The channel variant in slit coordinates: z uniform in [r, H - r], not
// periodic; candidates are rounded to binary32 before the distance test.
void channel_centres(int n, double side, int H, double r, uint64_t seed, std::vector<float>& x,
                     std::vector<float>& y, std::vector<float>& z) {
    x.assign(1, (float)(0.5 * side));
    y.assign(1, (float)(0.5 * side));
    z.assign(1, (float)(0.5 * H));
    std::mt19937_64 g(seed);
    const double lo = r, hi = (double)H - r, r2 = r * r;
    while ((int)x.size() < n) {
        const float cx = (float)(side * u53(g)), cy = (float)(side * u53(g));
        const float cz = (float)(lo + (hi - lo) * u53(g));
        bool ok = true;
        for (size_t j = 0; j < x.size() && ok; ++j) {
            const double dx = min_image((double)cx - x[j], side), dy = min_image((double)cy - y[j], side),
                         dz = (double)cz - z[j];
            ok = !(dx * dx + dy * dy + dz * dz < r2);
        }
        if (!ok) continue;
        x.push_back(cx);
        y.push_back(cy);
        z.push_back(cz);
    }
}

// FNV-1a 64 over each row's int64 id and binary32 x, y, z (little endian).
uint64_t table_hash(const std::vector<float>& x, const std::vector<float>& y, const std::vector<float>& z) {
    uint64_t h = 0xcbf29ce484222325ull;
    auto byte = [&h](uint8_t b) {
        h ^= b;
        h *= 0x00000100000001b3ull;
    };
    for (size_t i = 0; i < x.size(); ++i) {
        const uint64_t id = (uint64_t)i;
        for (int s = 0; s < 64; s += 8) byte((uint8_t)(id >> s));
        for (float f : {x[i], y[i], z[i]}) {
            uint32_t b;
            std::memcpy(&b, &f, 4);
            for (int s = 0; s < 32; s += 8) byte((uint8_t)(b >> s));
        }
    }
    return h;
}

bool mkdirs(const std::string& dir) {
    std::string acc;
    for (size_t i = 0; i <= dir.size(); ++i) {
        if (i == dir.size() || dir[i] == '/')
            if (!acc.empty() && ::mkdir(acc.c_str(), 0777) != 0 && errno != EEXIST) return false;
        if (i < dir.size()) acc.push_back(dir[i]);
    }
    return true;
}
std::string parent_of(const std::string& path) {
    const size_t slash = path.rfind('/');
    return slash == std::string::npos ? std::string() : path.substr(0, slash == 0 ? 1 : slash);
}

double sphere_volume(double R) { return 4.0 * kPi * R * R * R / 3.0; }
double footprint_area(double R) { return kPi * R * R; }

double realized_rho(const pfb_params3d& p) {
    const double lateral = (double)p.Nx * p.Ny;
    if (p.boundary_flags == PFB3D_BOUNDARY_SUBSTRATE_SLAB)
        return (double)p.num_cells * footprint_area(p.target_radius) / lateral;
    const int h = p.boundary_flags == PFB3D_BOUNDARY_HARD_WALL_CHANNEL ? p.channel_height : p.Nz;
    return (double)p.num_cells * sphere_volume(p.target_radius) / (lateral * (double)h);
}

// The metadata line of the trajectory (hexadecimal floats): the
// continuation contract an appending run must match exactly.
std::string header(const pfb_params3d& p, const Options& o, int B, uint64_t hash, long long every) {
    char t[1536];
    const unsigned long long ps = p.polarity_seed ? p.polarity_seed : p.seed;
    const std::string tail =
        "tau=%a v_A=%a v_A_sigma=%a gamma_normal=%a gamma_soft=%a "
        "soft_fraction=%a seed=%llu polarity_stream=%llu init_hash=%016llx "
        "promoted_measure_reduction=one-cta promoted_measure_policy=0 "
        "promoted_measure_auto_wave_ctas=0 base_measure_shards=%d trajectory_interval=%llu";
    if (p.boundary_flags == PFB3D_BOUNDARY_HARD_WALL_CHANNEL) {
        const std::string fmt =
            "# phase_field_gh200 trajectory schema=1 dim=3 geometry=resolved-wall-channel "
            "boundary=periodic-xy outer_array_boundary=homogeneous-neumann-z N=%d "
            "Nx=%d Ny=%d allocated_Nz=%d H=%d padding=%d B=%d "
            "z_coordinate=height-above-lower-wall lower_wall_z=0 upper_wall_z=%d "
            "wall_profile=tanh-union kappa_w=%a lambda_w=%a translation=three-dimensional "
            "dx=%a dt=%a aging_time=%a rho_V_target=%a rho_V_realized=%a "
            "R=%a lambda=%a kappa=%a mu=%a xi=%a " + tail;
        std::snprintf(t, sizeof(t), fmt.c_str(), p.num_cells, p.Nx, p.Ny, p.Nz, p.channel_height,
                      p.channel_padding, B, p.channel_height, p.wall_kappa, p.wall_width, 1.0, p.dt,
                      p.aging_time, o.rho, realized_rho(p), p.target_radius, p.lambda, p.kappa, p.mu, p.xi,
                      p.tau, p.v_A, p.v_A_sigma, p.gamma, o.gamma_soft, o.soft_fraction,
                      (unsigned long long)p.seed, ps, (unsigned long long)hash, kMeasureShards,
                      (unsigned long long)every);
    } else if (p.boundary_flags == PFB3D_BOUNDARY_SUBSTRATE_SLAB) {
        const std::string fmt =
            "# phase_field_gh200 trajectory schema=1 dim=3 geometry=substrate-slab "
            "boundary=periodic-xy N=%d Nx=%d Ny=%d Nz=%d B=%d "
            "z_coordinate=height-above-substrate substrate_z=0 "
            "lattice_substrate_face=%a top=dirichlet-zero top_z=%d translation=planar "
            "dx=%a dt=%a aging_time=%a rho_A_target=%a rho_A_realized=%a "
            "R=%a lambda=%a kappa=%a mu=%a xi=%a " + tail;
        std::snprintf(t, sizeof(t), fmt.c_str(), p.num_cells, p.Nx, p.Ny, p.Nz, B, -0.5, p.Nz, 1.0, p.dt,
                      p.aging_time, o.rho, realized_rho(p), p.target_radius, p.lambda, p.kappa, p.mu, p.xi, p.tau,
                      p.v_A, p.v_A_sigma, p.gamma, o.gamma_soft, o.soft_fraction, (unsigned long long)p.seed, ps,
                      (unsigned long long)hash, kMeasureShards, (unsigned long long)every);
    } else {
        const std::string fmt =
            "# phase_field_gh200 trajectory schema=1 dim=3 geometry=periodic-xyz "
            "N=%d L=%d B=%d "
            "dx=%a dt=%a aging_time=%a rho_V_target=%a rho_V_realized=%a "
            "R=%a lambda=%a kappa=%a mu=%a xi=%a " + tail;
        std::snprintf(t, sizeof(t), fmt.c_str(), p.num_cells, p.Nx, B, 1.0, p.dt, p.aging_time, o.rho,
                      realized_rho(p), p.target_radius, p.lambda, p.kappa, p.mu, p.xi, p.tau, p.v_A, p.v_A_sigma,
                      p.gamma, o.gamma_soft, o.soft_fraction, (unsigned long long)p.seed, ps,
                      (unsigned long long)hash, kMeasureShards, (unsigned long long)every);
    }
    return t;
}
const char* kColsPeriodic =
    "# columns: time cell_id x y z vx vy vz px py pz gamma v_A surface sphericity volume phi_max";
const char* kColsSlab =
    "# columns: time cell_id x y height vx vy vz px py pz gamma v_A "
    "free_interface_proxy hemisphere_normalized_free_surface_compactness volume phi_max";
const char* kColsChannel =
    "# columns: time cell_id x y height vx vy vz px py pz gamma v_A "
    "interface_measure sphericity_proxy volume phi_max wall_overlap wall_overlap_fraction "
    "outside_slit_volume physical_penetration_fraction";

// Open for append. A new (empty) file gets the two header lines and
// *last_step = -1; an existing one must carry this run's header and whole
// frames of canonically ordered rows with strictly increasing times, the
// last of which lies at a step not beyond `step` (returned in *last_step).
bool open_traj(const std::string& path, const std::string& head, const char* cols, int N, double dt,
               long long step, bool channel, std::FILE** out, long long* last_step) {
    const std::string dir = parent_of(path);
    if (!dir.empty() && !mkdirs(dir)) {
        std::fprintf(stderr, "[3d] cannot create trajectory directory\n");
        return false;
    }
    std::FILE* f = std::fopen(path.c_str(), "a+");
    if (!f) {
        std::fprintf(stderr, "[3d] cannot open trajectory %s\n", path.c_str());
        return false;
    }
    auto fail = [f](const char* why) {
        std::fprintf(stderr, "[3d] %s\n", why);
        std::fclose(f);
        return false;
    };
    std::rewind(f);
    if (std::fgetc(f) == EOF) {
        if (std::ferror(f)) return fail("cannot read trajectory");
        std::clearerr(f);
        std::fseek(f, 0, SEEK_END);
        if (std::fprintf(f, "%s\n%s\n", head.c_str(), cols) < 0 || std::fflush(f) != 0)
            return fail("cannot write trajectory header");
        *out = f;
        *last_step = -1;
        return true;
    }
    std::rewind(f);
    std::vector<char> line(2048);
    bool long_line = false;
    auto next = [&]() {
        if (!std::fgets(line.data(), (int)line.size(), f)) return false;
        size_t n = std::strlen(line.data());
        if (n && line[n - 1] == '\n') {
            line[--n] = '\0';
            if (n && line[n - 1] == '\r') line[--n] = '\0';
        } else if (!std::feof(f)) {
            long_line = true;
            return false;
        }
        return true;
    };
    if (!next()) return fail("refusing to append: trajectory metadata does not match this run");
    const std::string first = line.data();
    if (!next() || first != head || std::strcmp(cols, line.data()) != 0)
        return fail("refusing to append: trajectory metadata does not match this run");
    unsigned long long rows = 0;
    double frame_t = 0.0, prev_t = -1.0;
    while (next()) {
        if (line[0] == '\0') return fail("blank line in trajectory payload");
        double v[20];
        long long id = 0;
        char extra = 0;
        // 16 values after the id, 20 with the channel's wall columns
        const int got = std::sscanf(line.data(),
                                    "%lf %lld %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf "
                                    "%lf %lf %lf %lf %c",
                                    &v[0], &id, &v[1], &v[2], &v[3], &v[4], &v[5], &v[6], &v[7], &v[8], &v[9],
                                    &v[10], &v[11], &v[12], &v[13], &v[14], &v[15], &v[16], &v[17], &v[18],
                                    &v[19], &extra);
        const int values = channel ? 20 : 16;
        bool finite = got == values + 1;
        for (int k = 0; finite && k < values; ++k) finite = std::isfinite(v[k]);
        if (!finite) {
            std::fprintf(stderr, "[3d] malformed trajectory row %llu\n", rows + 1);
            std::fclose(f);
            return false;
        }
        const unsigned long long within = rows % (unsigned long long)N;
        if (within == 0) {
            frame_t = v[0];
            if (rows != 0 && !(frame_t > prev_t)) return fail("trajectory frame times are not strictly increasing");
        } else if (v[0] != frame_t) {
            return fail("trajectory contains a frame with mixed times");
        }
        if (id != (long long)within) return fail("trajectory cells are not in canonical ID order");
        if (++rows % (unsigned long long)N == 0) prev_t = frame_t;
    }
    if (long_line || std::ferror(f) || rows % (unsigned long long)N)
        return fail("refusing to append to a partial trajectory frame");
    *last_step = -1;
    if (rows > 0) {
        const double s = prev_t / dt;
        if (!std::isfinite(s) || s < 0.0 || s > 9.0e18) return fail("trajectory time is outside step range");
        const long long last = std::llround(s);
        if (std::fabs((double)last * dt - prev_t) > 1.0e-10 * std::max(1.0, std::fabs(prev_t)) || last > step)
            return fail("trajectory extends beyond the initialized state");
        *last_step = last;
    }
    std::clearerr(f);
    std::fseek(f, 0, SEEK_END);
    *out = f;
    return true;
}

// One frame: positions are the window origin plus the centroid (as the
// device forms it, one fused multiply-add), heights above the lower face for
// the slab, then the shape measure of the geometry.
bool write_frame(std::FILE* f, pfb_sim3d* s, const pfb_params3d& p) {
    const bool channel = p.boundary_flags == PFB3D_BOUNDARY_HARD_WALL_CHANNEL;
    if (pfb_sim3d_measure_current(s) != PFB_OK) return false;
    if (channel && pfb_sim3d_measure_wall(s) != PFB_OK) return false;
    std::vector<pfb_cell3d> c((size_t)p.num_cells);
    if (pfb_sim3d_get_cells(s, c.data()) != PFB_OK) return false;
    const double t = (double)pfb_sim3d_step(s) * p.dt;
    const bool slab = p.boundary_flags == PFB3D_BOUNDARY_SUBSTRATE_SLAB;
    const double hemi = 2.0 * kPi * std::pow(3.0 / (2.0 * kPi), 2.0 / 3.0);
    for (const pfb_cell3d& k : c) {
        const double inv = k.V > 0.0 ? 1.0 / k.V : 0.0;
        const double x = std::fma(k.Cx, inv, (double)k.origin_x);
        const double y = std::fma(k.Cy, inv, (double)k.origin_y);
        double z = std::fma(k.Cz, inv, (double)k.origin_z);
        if (slab) z += 0.5;
        if (channel) z += 0.5 - (double)p.channel_padding;
        double shape = 0.0;
        if (k.V > 0.0 && k.surface > 0.0)
            shape = slab ? hemi * std::pow(k.V, 2.0 / 3.0) / k.surface
                         : std::cbrt(kPi) * std::pow(6.0 * k.V, 2.0 / 3.0) / k.surface;
        if (std::fprintf(f,
                         "%.17g %lld %.17g %.17g %.17g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.17g %.17g %.17g "
                         "%.9g",
                         t, (long long)k.global_id, x, y, z, (double)k.velocity_x, (double)k.velocity_y,
                         (double)k.velocity_z, (double)k.polarity_x, (double)k.polarity_y, (double)k.polarity_z,
                         (double)k.gamma, (double)k.v_A, k.surface, shape, k.V, (double)k.phi_max) < 0 ||
            (channel ? std::fprintf(f, " %.17g %.17g %.17g %.17g\n", k.wall_overlap,
                                    k.V > 0.0 ? k.wall_overlap / k.V : 0.0, k.outside_slit_volume,
                                    k.V > 0.0 ? k.outside_slit_volume / k.V : 0.0)
                     : std::fputc('\n', f)) < 0) {
            std::fprintf(stderr, "[3d] failed to write trajectory frame\n");
            return false;
        }
    }
    return std::fflush(f) == 0 && !std::ferror(f);
}

void usage() {
    std::printf(
        "usage: pfb_cell_3d [options]\n"
        "  geometry: --geometry periodic|slab|channel, --slab-height, --channel-height,\n"
        "            --wall-kappa, --wall-width, --wall-padding\n"
        "  model:    --N --radius --rho --lambda --kappa --mu --xi --tau --v-A --v-A-sigma\n"
        "            --gamma --gamma-cancer --cancer-fraction --dt --aging-time\n"
        "            --seed --polarity-seed --full-moment --verify-every\n"
        "  run:      --t-end --brick-edge --device --bench --print-interval --initial-centres CSV\n"
        "            --strict (invariants every --verify-every steps)\n"
        "  output:   --out --trajectory-samples --trajectory-interval\n"
        "  restart:  -c|--checkpoint FILE --checkpoint-interval --save-interval\n"
        "            --checkpoint-dir --no-final-checkpoint\n"
        "  boundary: --boundary-out FILE --boundary-interval N\n"
        "            --boundary-projection maximum|basal --boundary-compression none|zstd\n");
}

struct RealOpt {
    const char* name;
    double lo, hi;
    double* dst;
    bool* given;
};
struct IntOpt {
    const char* name;
    long long lo, hi;
    long long* dst;
    bool* given;
};

// 0 ready, 1 help, 2 usage error.
int parse(int argc, char** argv, Options* o) {
    pfb_params3d& p = o->p;
    p.num_cells = 288;
    p.dt = 0.01;
    p.lambda = 7.0;
    p.target_radius = 49.0;
    p.kappa = 10.0;
    p.mu = 1.0;
    p.xi = 1500.0;
    p.tau = 1.0e4;
    p.v_A = 1.0e-2;
    p.gamma = 1.0;
    p.seed = 1234;
    p.full_moment_every = 100;
    p.boundary_flags = PFB3D_BOUNDARY_PERIODIC_XYZ;
    long long n_cells = p.num_cells, full_moment = p.full_moment_every;
    long long slab_h = 0, channel_h = 0, pad = 0;
    bool scratch = false;
    const RealOpt reals[] = {
        {"--radius", 1.0e-6, 1.0e6, &p.target_radius, &o->model_given},
        {"--rho", 1.0e-9, 0.999999999, &o->rho, &o->model_given},
        {"--lambda", 1.0e-6, 1.0e6, &p.lambda, &o->model_given},
        {"--kappa", 0.0, 1.0e12, &p.kappa, &o->model_given},
        {"--mu", 0.0, 1.0e12, &p.mu, &o->model_given},
        {"--xi", 1.0e-12, 1.0e15, &p.xi, &o->model_given},
        {"--tau", 1.0e-12, 1.0e15, &p.tau, &o->model_given},
        {"--v-A", 0.0, 1.0e9, &p.v_A, &o->model_given},
        {"--v-A-sigma", 0.0, 10.0, &p.v_A_sigma, &o->model_given},
        {"--gamma", 1.0e-12, 1.0e9, &p.gamma, &o->model_given},
        {"--gamma-cancer", 1.0e-12, 1.0e9, &o->gamma_soft, &o->model_given},
        {"--cancer-fraction", 0.0, 1.0, &o->soft_fraction, &o->model_given},
        {"--dt", 1.0e-12, 1.0e6, &p.dt, &o->model_given},
        {"--aging-time", 0.0, 1.0e15, &p.aging_time, &o->model_given},
        {"--wall-kappa", 1.0e-12, 1.0e12, &p.wall_kappa, &o->wall_k_given},
        {"--wall-width", 1.0e-6, 1.0e6, &p.wall_width, &o->wall_w_given},
        {"--t-end", 0.0, 1.0e15, &o->t_end, &o->t_end_given},
    };
    const IntOpt ints[] = {
        {"--N", 1, 4000000, &n_cells, &o->model_given},
        {"--full-moment", 0, 1000000000, &full_moment, &o->model_given},
        {"--verify-every", 0, 1000000000, &o->verify_every, &o->model_given},
        {"--slab-height", 1, 2147483647, &slab_h, &o->slab_h_given},
        {"--channel-height", 1, 2147483647, &channel_h, &o->channel_h_given},
        {"--wall-padding", 1, 2147483647, &pad, &o->pad_given},
        {"--brick-edge", 0, 4096, &o->brick, &scratch},
        {"--device", 0, 63, &o->device, &scratch},
        {"--bench", 1, 100000000, &o->bench, &scratch},
        {"--print-interval", 0, 1000000000, &o->print_interval, &o->print_given},
        {"--trajectory-samples", 1, 1000000000, &o->traj_samples, &o->samples_given},
        {"--trajectory-interval", 1, 4294967295LL, &o->traj_interval, &o->interval_given},
        {"--checkpoint-interval", 1, 1000000000000LL, &o->ckpt_interval, &o->schedule_given},
        {"--save-interval", 1, 1000000000000LL, &o->save_interval, &o->schedule_given},
        {"--boundary-interval", 1, 1000000000000LL, &o->bnd_interval, &o->bnd_given},
    };
    for (int i = 1; i < argc; ++i) {
        const char* a = argv[i];
        auto value = [&]() -> const char* {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "[3d] %s requires a value\n", a);
                return nullptr;
            }
            return argv[++i];
        };
        if (!std::strcmp(a, "-h") || !std::strcmp(a, "--help")) {
            usage();
            return 1;
        }
        bool done = false;
        for (const RealOpt& r : reals)
            if (!std::strcmp(a, r.name)) {
                const char* v = value();
                if (!v || !parse_real(a, v, r.lo, r.hi, r.dst)) return 2;
                *r.given = done = true;
            }
        for (const IntOpt& r : ints)
            if (!done && !std::strcmp(a, r.name)) {
                const char* v = value();
                if (!v || !parse_int(a, v, r.lo, r.hi, r.dst)) return 2;
                *r.given = done = true;
            }
        if (done) {
            if (o->slab_h_given || o->channel_h_given || o->pad_given || o->wall_k_given || o->wall_w_given)
                o->model_given = true;
            continue;
        }
        if (!std::strcmp(a, "--geometry")) {
            const char* v = value();
            if (!v) return 2;
            if (!std::strcmp(v, "periodic")) o->geometry = kPeriodic;
            else if (!std::strcmp(v, "slab")) o->geometry = kSlab;
            else if (!std::strcmp(v, "channel")) o->geometry = kChannel;
            else {
                std::fprintf(stderr, "[3d] --geometry expects periodic, slab, or channel, got '%s'\n", v);
                return 2;
            }
            o->model_given = true;
        } else if (!std::strcmp(a, "--seed") || !std::strcmp(a, "--polarity-seed")) {
            const char* v = value();
            if (!v || !parse_u64(a, v, !std::strcmp(a, "--seed") ? &p.seed : &p.polarity_seed)) return 2;
            o->model_given = true;
        } else if (!std::strcmp(a, "--out") || !std::strcmp(a, "-c") || !std::strcmp(a, "--checkpoint") ||
                   !std::strcmp(a, "--checkpoint-dir")) {
            const char* v = value();
            if (!v || !v[0]) return 2;
            if (!std::strcmp(a, "--out")) {
                o->out_path = v;
            } else if (!std::strcmp(a, "--checkpoint-dir")) {
                o->ckpt_dir = v;
                o->ckpt_dir_given = true;
            } else {
                o->ckpt_in = v;
            }
        } else if (!std::strcmp(a, "--no-final-checkpoint")) {
            o->final_ckpt = false;
        } else if (!std::strcmp(a, "--strict")) {
            o->strict = true;
        } else if (!std::strcmp(a, "--initial-centres")) {
            const char* v = value();
            if (!v || !v[0]) return 2;
            o->centres_path = v;
        } else if (!std::strcmp(a, "--memory-mode")) {
            const char* v = value();
            if (!v) return 2;
            if (!std::strcmp(v, "auto")) o->mem_mode = PFB3D_MEMORY_AUTO;
            else if (!std::strcmp(v, "throughput")) o->mem_mode = PFB3D_MEMORY_THROUGHPUT;
            else if (!std::strcmp(v, "balanced")) o->mem_mode = PFB3D_MEMORY_BALANCED;
            else if (!std::strcmp(v, "compact")) o->mem_mode = PFB3D_MEMORY_COMPACT;
            else {
                std::fprintf(stderr, "[3d] --memory-mode expects auto, throughput, balanced, or compact\n");
                return 2;
            }
        } else if (!std::strcmp(a, "--scratch-slots")) {
            const char* v = value();
            long long k = 0;
            if (!v || !parse_int(a, v, 0, 1 << 20, &k)) return 2;
            o->scratch_slots = (int)k;
        } else if (!std::strcmp(a, "--measure-shards") || !std::strcmp(a, "--promoted-measure-shards")) {
            // the measurement groupings are fixed: 4 CTAs per base cell, the
            // one-CTA promoted policy (as the trajectory header states)
            const char* v = value();
            long long k = 0;
            if (!v || !parse_int(a, v, -1, 1024, &k)) return 2;
            const bool base = !std::strcmp(a, "--measure-shards");
            if (k != (base ? kMeasureShards : 0)) {
                std::fprintf(stderr, "[3d] %s %lld: this build measures with %s only\n", a, k,
                             base ? "--measure-shards 4" : "--promoted-measure-shards 0");
                return 2;
            }
        } else if (!std::strcmp(a, "--boundary-out") || !std::strcmp(a, "--boundary-projection") ||
                   !std::strcmp(a, "--boundary-compression")) {
            const char* v = value();
            if (!v) return 2;
            o->bnd_given = true;
            if (!std::strcmp(a, "--boundary-out")) {
                o->bnd_path = v;
            } else if (!std::strcmp(a, "--boundary-projection")) {
                if (!std::strcmp(v, "maximum")) o->bnd_projection = PFB3D_PROJECTION_MAXIMUM;
                else if (!std::strcmp(v, "basal")) o->bnd_projection = PFB3D_PROJECTION_BASAL;
                else {
                    std::fprintf(stderr, "[3d] --boundary-projection expects maximum or basal\n");
                    return 2;
                }
            } else {
                if (!std::strcmp(v, "none")) o->bnd_compress = false;
                else if (!std::strcmp(v, "zstd")) o->bnd_compress = true;
                else {
                    std::fprintf(stderr, "[3d] --boundary-compression expects none or zstd\n");
                    return 2;
                }
            }
        } else {
            std::fprintf(stderr, "[3d] unknown option '%s' or one this build does not provide (try --help)\n", a);
            return 2;
        }
    }
    if (o->bnd_given && (o->bnd_path.empty() || o->bnd_interval <= 0)) {
        std::fprintf(stderr, "[3d] boundary output requires --boundary-out and --boundary-interval\n");
        return 2;
    }
    if (o->bnd_given && o->bench > 0) {
        std::fprintf(stderr, "[3d] boundary output cannot be combined with --bench\n");
        return 2;
    }
    p.num_cells = (int)n_cells;
    p.full_moment_every = (int)full_moment;
    o->slab_height = (int)slab_h;
    o->channel_height = (int)channel_h;
    o->wall_padding = (int)pad;
    return 0;
}

// Domain, heights and wall padding of a fresh run; false on a usage error.
bool resolve_geometry(Options* o) {
    pfb_params3d& p = o->p;
    const bool slab = o->geometry == kSlab, channel = o->geometry == kChannel;
    const char* bad = nullptr;
    if (o->slab_h_given && !slab) bad = "--slab-height requires --geometry slab";
    if (o->channel_h_given && !channel) bad = "--channel-height requires --geometry channel";
    if ((o->wall_k_given || o->wall_w_given) && !channel) bad = "--wall-kappa/--wall-width require --geometry channel";
    if (o->pad_given && !channel) bad = "--wall-padding requires --geometry channel";
    if (bad) {
        std::fprintf(stderr, "[3d] %s\n", bad);
        return false;
    }
    const double R = p.target_radius;
    p.boundary_flags = slab ? PFB3D_BOUNDARY_SUBSTRATE_SLAB
                       : channel ? PFB3D_BOUNDARY_HARD_WALL_CHANNEL
                                 : PFB3D_BOUNDARY_PERIODIC_XYZ;
    int H = 0;
    double side = 0.0;
    if (channel) {
        if (!o->wall_k_given) p.wall_kappa = p.kappa;
        if (!o->wall_w_given) p.wall_width = p.lambda;
        const double diameter = std::ceil(2.0 * R);
        H = o->channel_h_given ? o->channel_height : (int)diameter;
        if (H < (int)diameter) {
            std::fprintf(stderr, "[3d] channel height %d is smaller than the one-diameter minimum %d\n", H,
                         (int)diameter);
            return false;
        }
        side = std::ceil(std::sqrt((double)p.num_cells * sphere_volume(R) / (o->rho * (double)H)));
    } else if (slab) {
        side = std::ceil(std::sqrt((double)p.num_cells * footprint_area(R) / o->rho));
    } else {
        side = std::ceil(std::cbrt((double)p.num_cells * sphere_volume(R) / o->rho));
    }
    if (!(side >= 1.0 && side <= 2147483647.0)) {
        std::fprintf(stderr, "[3d] could not derive a finite domain\n");
        return false;
    }
    p.Nx = p.Ny = p.Nz = (int)side;
    if (slab) {
        const int autoB = pfb3d_automatic_brick_edge(R, p.lambda);
        p.Nz = o->slab_h_given ? o->slab_height : 2 * autoB;
        if (autoB <= 0 || p.Nz <= autoB) {
            std::fprintf(stderr, "[3d] slab height %d must exceed automatic brick edge %d\n", p.Nz, autoB);
            return false;
        }
    } else if (channel) {
        const double minpad = std::ceil(3.0 * p.wall_width);
        const int pad = o->pad_given ? o->wall_padding : (int)minpad;
        if (pad < (int)minpad) {
            std::fprintf(stderr, "[3d] --wall-padding %d is smaller than the minimum %d\n", pad, (int)minpad);
            return false;
        }
        p.channel_height = H;
        p.channel_padding = pad;
        p.Nz = H + 2 * pad;
    }
    return true;
}

long long steps_of(double t_end, double dt) {
    const double s = t_end / dt + 0.5;
    return std::isfinite(s) && s >= 0.0 && s <= 9.0e18 ? (long long)s : -1;
}
long long after(long long cur, long long every) { return every <= 0 ? kNever : cur + every; }
long long grid_after(long long cur, long long every) {
    if (every <= 0) return kNever;
    const long long r = cur % every;
    return cur + (r == 0 ? every : every - r);
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    const int parsed = parse(argc, argv, &o);
    if (parsed == 1) return 0;
    if (parsed) return 2;
    pfb_params3d& p = o.p;
    const bool resumed = !o.ckpt_in.empty();
    uint64_t hash = 0;
    pfb_ckpt3d_params rec{};
    std::vector<pfb_vec3> centres;
    if (resumed) {
        if (o.model_given || !o.centres_path.empty()) {
            std::fprintf(stderr, "[3d] checkpoint continuation preserves its model and initialized state; only "
                                 "--t-end and run/output options may change\n");
            return 2;
        }
        pfb_ckpt3d_info info{};
        if (pfb_ckpt3d_read(o.ckpt_in.c_str(), &info, &rec, nullptr, nullptr) != PFB_OK ||
            pfb_ckpt3d_params_to(&rec, info.num_cells, &p) != PFB_OK) {
            std::fprintf(stderr, "[3d] %s\n", pfb_last_error());
            return 1;
        }
        hash = rec.initialization_hash;
        o.soft_fraction = rec.soft_fraction;
        o.rho = rec.volume_fraction;
        o.gamma_soft = rec.gamma_soft;
        o.verify_every = rec.verify_every;
        if (!o.print_given) o.print_interval = rec.print_interval;
        if (!o.samples_given && !o.interval_given && rec.trajectory_interval > 0)
            o.traj_interval = rec.trajectory_interval;
        if (!o.t_end_given) o.t_end = rec.t_end;
        if (steps_of(o.t_end, p.dt) < info.step) {
            std::fprintf(stderr, "[3d] --t-end precedes checkpoint step %lld\n", info.step);
            return 2;
        }
        o.geometry = p.boundary_flags == PFB3D_BOUNDARY_SUBSTRATE_SLAB       ? kSlab
                     : p.boundary_flags == PFB3D_BOUNDARY_HARD_WALL_CHANNEL ? kChannel
                                                                            : kPeriodic;
    } else {
        if (!resolve_geometry(&o)) return 2;
        p.B = (int)o.brick;
        p.gamma_soft = o.gamma_soft;
        p.soft_fraction = o.soft_fraction;
        const double R = p.target_radius;
        std::vector<float> x, y, z;
        std::string err;
        bool read_ok = true;
        if (!o.centres_path.empty()) {
            // the reference's tables (src/pf3d/sim.cu:900-1096)
            std::vector<int64_t> ids;
            if (o.geometry == kSlab) {
                read_ok = pfb_csv::read_relaxed2(o.centres_path, p.num_cells, (double)p.Nx, false, ids, x, y, &err);
                z.assign(x.size(), -0.5f);
            } else if (o.geometry == kChannel && pfb_csv::first_line(o.centres_path) == "global_id,x,y") {
                const int one_layer = (int)std::ceil(2.0 * R);
                if (p.channel_height != one_layer) {
                    std::fprintf(stderr, "[3d] a 2D relaxed x/y table is accepted only for the one-layer "
                                         "channel H=ceil(2R)=%d\n", one_layer);
                    return 1;
                }
                read_ok = pfb_csv::read_relaxed2(o.centres_path, p.num_cells, (double)p.Nx, true, ids, x, y, &err);
                z.assign(x.size(), (float)(0.5 * one_layer));
            } else if (o.geometry == kChannel) {
                read_ok = pfb_csv::read_channel3(o.centres_path, p.num_cells, (double)p.Nx, p.channel_height, R,
                                                 x, y, z, &err);
            } else {
                read_ok = pfb_csv::read_table3(o.centres_path, p.num_cells, (double)p.Nx, R, x, y, z, &err);
            }
            if (!read_ok) {
                std::fprintf(stderr, "[3d] %s\n", err.c_str());
                return 1;
            }
        } else if (o.geometry == kSlab) {
            x.resize((size_t)p.num_cells);
            y.resize((size_t)p.num_cells);
            if (pfb_palmieri_centres(p.num_cells, (double)p.Nx, R, p.seed, x.data(), y.data()) != PFB_OK) {
                std::fprintf(stderr, "[3d] slab initializer failed: %s\n", pfb_last_error());
                return 1;
            }
            z.assign(x.size(), -0.5f);
        } else if (o.geometry == kChannel) {
            channel_centres(p.num_cells, (double)p.Nx, p.channel_height, R, p.seed, x, y, z);
        } else {
            periodic_centres(p.num_cells, (double)p.Nx, R, p.seed, x, y, z);
        }
        hash = table_hash(x, y, z);
        std::printf("  centres: %d placed, table hash %016llx\n", p.num_cells, (unsigned long long)hash);
        std::fflush(stdout);
        // channel centres stay in slit coordinates: pfb_sim3d_create moves
        // them to array coordinates (z + padding - 1/2 in binary32)
        for (size_t i = 0; i < x.size(); ++i) centres.push_back(pfb_vec3{x[i], y[i], z[i]});
    }
    if (!o.ckpt_dir_given && o.schedule_given) {
        o.ckpt_dir = parent_of(o.out_path);
        if (o.ckpt_dir.empty()) o.ckpt_dir = parent_of(o.ckpt_in);
        if (o.ckpt_dir.empty()) o.ckpt_dir = ".";
    }
    const long long total = steps_of(o.t_end, p.dt);
    if (total < 0) {
        std::fprintf(stderr, "[3d] dt and t_end do not define a valid step count\n");
        return 2;
    }
    if (!o.bnd_path.empty() && o.bnd_projection == PFB3D_PROJECTION_BASAL && o.geometry != kSlab) {
        std::fprintf(stderr, "[3d] basal boundary output requires --geometry slab\n");
        return 2;
    }

    pfb_sim3d* s = resumed ? pfb_sim3d_create_from_checkpoint_ex(o.ckpt_in.c_str(), (int)o.device, o.mem_mode,
                                                                 o.scratch_slots)
                           : pfb_sim3d_create_ex(&p, centres.data(), (int)o.device, o.mem_mode,
                                                 o.scratch_slots);
    if (!s) {
        std::fprintf(stderr, "[3d] initialisation failed: %s\n", pfb_last_error());
        return 1;
    }
    const int B = pfb_sim3d_brick(s);
    std::printf("pfb_cell_3d: %s  N=%d  domain=%dx%dx%d  B=%d  steps %lld -> %lld  table hash %016llx\n",
                resumed ? "resume" : "fresh", p.num_cells, p.Nx, p.Ny, p.Nz, B, pfb_sim3d_step(s), total,
                (unsigned long long)hash);
    if (o.bench > 0) {
        double ms = 0.0;
        const int rc = pfb_sim3d_bench(s, 2, (int)o.bench, &ms);
        if (rc == PFB_OK) std::printf("bench: %lld steps, %.6f ms/step\n", o.bench, ms);
        pfb_sim3d_destroy(s);
        return rc == PFB_OK ? 0 : 1;
    }

    const long long traj_every =
        o.traj_interval > 0 ? o.traj_interval : std::max<long long>(1, total / std::max<long long>(1, o.traj_samples));
    if (!o.ckpt_dir.empty() && traj_every > 4294967295LL) {
        std::fprintf(stderr, "[3d] resolved trajectory interval exceeds the checkpoint limit\n");
        pfb_sim3d_destroy(s);
        return 1;
    }
    pfb_params3d rp = p;
    rp.B = B;
    pfb_ckpt3d_params_from(&rp, B, &rec);
    rec.t_end = o.t_end;
    rec.volume_fraction = o.rho;
    rec.gamma_soft = o.gamma_soft;
    rec.soft_fraction = o.soft_fraction;
    rec.initialization_hash = hash;
    rec.print_interval = o.print_interval;
    rec.verify_every = o.verify_every;
    rec.trajectory_interval = (uint32_t)traj_every;

    bool ok = true;
    std::FILE* traj = nullptr;
    long long step = pfb_sim3d_step(s), last_frame = -1;
    if (!o.out_path.empty()) {
        const char* cols = o.geometry == kSlab ? kColsSlab : o.geometry == kChannel ? kColsChannel : kColsPeriodic;
        ok = open_traj(o.out_path, header(p, o, B, hash, traj_every), cols, p.num_cells, p.dt, step,
                       o.geometry == kChannel, &traj, &last_frame);
        // a new file starts at the initialized state
        if (ok && last_frame < 0) {
            ok = write_frame(traj, s, p);
            last_frame = step;
        }
    }
    long long last_bnd = -1;
    if (ok && !o.bnd_path.empty()) {
        // refuse a boundary file that would collide with the trajectory or a checkpoint
        const size_t slash = o.bnd_path.rfind('/');
        const std::string name = slash == std::string::npos ? o.bnd_path : o.bnd_path.substr(slash + 1);
        const bool ckpt_name = name == "checkpoint.pf3d" ||
                               (name.rfind("checkpoint_", 0) == 0 && name.size() > 5 &&
                                name.compare(name.size() - 5, 5, ".pf3d") == 0);
        if (o.bnd_path == o.out_path) {
            std::fprintf(stderr, "[3d] boundary output and trajectory paths must differ\n");
            ok = false;
        } else if (!o.ckpt_dir.empty() && ckpt_name &&
                   (parent_of(o.bnd_path).empty() ? std::string(".") : parent_of(o.bnd_path)) == o.ckpt_dir) {
            std::fprintf(stderr, "[3d] boundary output must not use a checkpoint filename\n");
            ok = false;
        } else if (pfb_sim3d_boundary_open(s, o.bnd_path.c_str(), o.bnd_projection, o.bnd_interval,
                                           o.bnd_compress ? 1 : 0) != PFB_OK ||
                   pfb_sim3d_boundary_capture(s) != PFB_OK) {
            std::fprintf(stderr, "[3d] %s\n", pfb_last_error());
            ok = false;
        } else {
            last_bnd = step;
        }
    }
    const bool ckpt_on = !o.ckpt_dir.empty();
    if (ok && ckpt_on && !mkdirs(o.ckpt_dir)) {
        std::fprintf(stderr, "[3d] cannot create checkpoint directory %s\n", o.ckpt_dir.c_str());
        ok = false;
    }
    auto save = [&](const std::string& path) {
        if (pfb_sim3d_write_checkpoint(s, path.c_str(), &rec) == PFB_OK) return true;
        std::fprintf(stderr, "[3d] %s\n", pfb_last_error());
        return false;
    };
    std::signal(SIGINT, on_signal);
    std::signal(SIGTERM, on_signal);
    long long next_traj = traj ? grid_after(step, traj_every) : kNever;
    long long next_ckpt = ckpt_on ? after(step, o.ckpt_interval) : kNever;
    long long next_save = ckpt_on ? after(step, o.save_interval) : kNever;
    long long next_print = after(step, o.print_interval);
    long long next_bnd = o.bnd_path.empty() ? kNever : grid_after(step, o.bnd_interval);
    // --strict: invariants at multiples of verify_every (reference src/pf3d/sim.cu:2167-2214)
    const long long verify_every = o.strict ? o.verify_every : 0;
    long long next_verify = verify_every > 0 ? after(step, verify_every - step % verify_every) : kNever;
    constexpr long long kPollEvery = 256;
    uint32_t flags[PFB3D_FLAG_COUNT];
    while (ok && step < total && !g_stop) {
        const long long stop =
            std::min({total, next_traj, next_ckpt, next_save, next_print, next_bnd, next_verify,
                      step + kPollEvery});
        if (pfb_sim3d_advance(s, (int)(stop - step)) != PFB_OK || pfb_sim3d_get_flags(s, flags) != PFB_OK) {
            std::fprintf(stderr, "[3d] step failed: %s\n", pfb_last_error());
            ok = false;
            break;
        }
        step = pfb_sim3d_step(s);
        for (int i = 0; i < PFB3D_FLAG_COUNT; ++i)
            if (((PFB3D_FATAL_MASK >> i) & 1u) && flags[i]) {
                std::fprintf(stderr, "[3d] fatal flag %d raised by step %lld; the last rolling checkpoint was not "
                                     "replaced\n", i, step);
                ok = false;
            }
        if (!ok) break;
        if (step >= next_print) {
            std::printf("[3d] step %lld  t %.6g\n", step, (double)step * p.dt);
            std::fflush(stdout);
            next_print = after(next_print, o.print_interval);
        }
        if (traj && step >= next_traj) {
            ok = write_frame(traj, s, p);
            last_frame = step;
            next_traj = after(next_traj, traj_every);
        }
        if (ok && step >= next_verify) {
            double rel = 0.0;
            uint32_t maxS = 0;
            unsigned long long edges = 0;
            if (pfb_sim3d_verify(s, &rel, &maxS, &edges) != PFB_OK || rel > 1.0e-12 || edges != 0) {
                std::fprintf(stderr, "[3d] strict verification failed: relV %.3e, edge voxels %llu\n", rel, edges);
                ok = false;
            }
            next_verify = after(next_verify, verify_every);
        }
        if (ok && step >= next_bnd) {
            if (pfb_sim3d_boundary_capture(s) != PFB_OK) {
                std::fprintf(stderr, "[3d] %s\n", pfb_last_error());
                ok = false;
            }
            last_bnd = step;
            next_bnd = after(next_bnd, o.bnd_interval);
        }
        if (ok && step >= next_ckpt) {
            ok = save(o.ckpt_dir + "/checkpoint.pf3d");
            next_ckpt = after(next_ckpt, o.ckpt_interval);
        }
        if (ok && step >= next_save) {
            char name[64];
            std::snprintf(name, sizeof(name), "/checkpoint_%012lld.pf3d", step);
            ok = save(o.ckpt_dir + name);
            next_save = after(next_save, o.save_interval);
        }
    }
    if (ok && traj && last_frame != step) ok = write_frame(traj, s, p);
    if (traj) std::fclose(traj);
    if (ok && ckpt_on && o.final_ckpt) ok = save(o.ckpt_dir + "/checkpoint.pf3d");
    if (ok && !o.bnd_path.empty()) {
        if (last_bnd != step && pfb_sim3d_boundary_capture(s) != PFB_OK) ok = false;
        if (pfb_sim3d_boundary_close(s, ok ? 1 : 0) != PFB_OK) ok = false;
        if (!ok) std::fprintf(stderr, "[3d] %s\n", pfb_last_error());
    }
    if (ok && g_stop) std::printf("[3d] termination requested; stopped at accepted step %lld\n", step);
    pfb_sim3d_destroy(s);
    return ok ? 0 : 1;
}
