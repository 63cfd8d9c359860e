// pfb_cell: the command line of the 2D run, with the reference's options,
// files and cadences (reference src/main.cu:22-720, src/sim.cu:95-135 fresh
// centres, 851-1004 run loop, 1095-1140 trajectory rows; src/trajectory.cpp
// metadata and append rules). Everything goes through the library's C ABI.
//
// Supported: the model and run options, resume from a CELL checkpoint (-c),
// rolling / tagged / final checkpoints, the plain-text trajectory (--out),
// the PFVMOM4 velocity-moment recorder (--velocity-moments; reference
// src/velocity_output.cu), the PFB boundary recorder (--boundary-out;
// src/boundary.cu), --strict (the reference's invariant report on the
// verify cadence), the per-cell mobility map (--phase-field-mobility-map;
// reference src/checkpoint.cu:663-820: uniform mobility then listed
// overrides on a fresh start, listed overrides of the stored values on
// resume), --bench, --morton (the Morton visit order, re-sorted every sixth
// step) and --no-l2 (accepted: this build sets no L2 persistence window for
// S) and --self-test (host checks of this build's stencil, coefficients,
// force sign, tumble draws and windows; exit status 4 when one fails). Not
// part of this build (they exit with status 2 and a message): velocity
// observation under --bench, and, on
// resume, overrides of model parameters other than the output cadences and
// t_end. zstd boundary compression is refused at open (no zstd here).
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pfb_common.cuh"
#include <sys/stat.h>
#include <utility>
#include <vector>

#include "centres_csv.hpp"
#include "pfb200.h"
#include "pfb200_ckpt.h"

namespace {

volatile std::sig_atomic_t g_stop = 0;
void on_signal(int) { g_stop = 1; }

struct Options {
    pfb_params2d p{};
    double rho = 0.90, t_end = 100.0;
    int print_interval = 100, verify_every = 4096;
    std::string ckpt_in, ckpt_dir, out_path;
    long long ckpt_interval = 0, save_interval = 0;
    bool final_ckpt = true;
    int traj_samples = 100;
    long long traj_interval = 0;
    bool traj_samples_set = false, traj_interval_set = false;
    bool t_end_set = false, print_set = false, verify_set = false;
    int device = 0;
    long long bench = 0;
    bool graph = true;
    bool model_override = false;  // a model option given on the command line
    bool n_or_rho = false;
    std::string vel_path;
    int vel_stride = 100;
    long long vel_dense = 10000;
    bool vel_reference = false, vel_given = false;
    std::string bnd_path;
    long long bnd_interval = 0;
    bool bnd_compress = false;
    std::string centres_path;  // --initial-centres
    bool strict = false;
    bool morton = false;
    bool self_test = false;
    std::string mobility_map;  // --phase-field-mobility-map
};

// Read a mobility map: one "global_id value" pair per line, blank lines and
// '#' comments skipped; ids in int32, unique; values finite and positive as
// binary32 (reference src/checkpoint.cu:663-728).
bool read_mobility_map(const std::string& path, std::vector<std::pair<int32_t, float>>* out, std::string* err) {
    out->clear();
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return *err = "cannot open " + path + ": " + std::strerror(errno), false;
    char line[256];
    int lineno = 0;
    std::vector<int32_t> seen;
    bool ok = true;
    auto fail = [&](const char* what) {
        *err = path + ":" + std::to_string(lineno) + ": " + what;
        ok = false;
    };
    while (ok && std::fgets(line, sizeof(line), f)) {
        ++lineno;
        const size_t len = std::strlen(line);
        if (len + 1 == sizeof(line) && line[len - 1] != '\n') {
            fail("line exceeds 254 characters");
            break;
        }
        const char* s = line;
        while (*s && std::isspace((unsigned char)*s)) ++s;
        if (*s == '\0' || *s == '#') continue;
        char* end = nullptr;
        errno = 0;
        const long long id = std::strtoll(s, &end, 10);
        if (end == s || !std::isspace((unsigned char)*end)) {
            fail("malformed global id");
            break;
        }
        if (errno == ERANGE || id < 0 || id > 2147483647LL) {
            fail("global id out of the int32 range or negative");
            break;
        }
        s = end;
        while (*s && std::isspace((unsigned char)*s)) ++s;
        const double v = std::strtod(s, &end);
        if (end == s) {
            fail("malformed mobility value");
            break;
        }
        s = end;
        while (*s && std::isspace((unsigned char)*s)) ++s;
        if (*s != '\0') {
            fail("trailing characters after the value");
            break;
        }
        const float mv = (float)v;
        if (!std::isfinite(v) || !std::isfinite(mv) || !(mv > 0.0f)) {
            fail("mobility must be finite and positive as binary32");
            break;
        }
        if (std::find(seen.begin(), seen.end(), (int32_t)id) != seen.end()) {
            fail("duplicate global id");
            break;
        }
        seen.push_back((int32_t)id);
        out->emplace_back((int32_t)id, mv);
    }
    const bool read_error = std::ferror(f) != 0;
    std::fclose(f);
    if (!ok) return false;
    if (read_error) return *err = "read error on " + path, false;
    if (out->empty()) return *err = path + ": contains no 'global_id value' entries", false;
    return true;
}

// Explicit-Euler bound over the resolved per-cell pairs (gamma_i, M_i), the
// reference's validate_effective_stiffness (include/params.cuh:729-775):
// dt * max_i (M_i / M0) gamma_i * 40/6 must stay below 1 (fatal, with its
// message), with warnings when a margin falls under 2x.
bool effective_stiffness_ok(const pfb_params2d& p, const std::vector<pfb_cell2d>& cells) {
    constexpr double kM0 = 0.5, kLapRowSum = 40.0 / 6.0;
    double geff_max = 0.0, mrel_max = 0.0;
    for (size_t i = 0; i < cells.size(); ++i) {
        const double g = (double)cells[i].gamma, m = (double)cells[i].M_pf;
        if (!(g > 0.0) || !std::isfinite(g) || !(m > 0.0) || !std::isfinite(m)) {
            std::fprintf(stderr,
                         "[fatal] cell %d has gamma = %.9g, phase-field mobility = %.9g; both must be "
                         "positive and finite.\n",
                         (int)i, g, m);
            return false;
        }
        geff_max = std::fmax(geff_max, (m / kM0) * g);
        mrel_max = std::fmax(mrel_max, m / kM0);
    }
    const double cfl = p.dt * geff_max * kLapRowSum;
    if (cfl >= 1.0) {
        std::fprintf(stderr,
                     "[fatal] max_i[(M_i/M0)*gamma_i] = %.6g gives dt*coeff*laplacian_bound = %.4f; the "
                     "configured safety limit is 1. Reduce dt below %.5g.\n",
                     geff_max, cfl, 1.0 / (geff_max * kLapRowSum));
        return false;
    }
    if (cfl > 0.5)
        std::fprintf(stderr,
                     "[warn] max_i[(M_i/M0)*gamma_i] = %.6g; dt*coeff*laplacian_bound = %.4f leaves under "
                     "2x margin to the safety limit.\n",
                     geff_max, cfl);
    const double rep = 60.0 * p.kappa / (p.lambda * p.lambda);
    const double rep_cfl = p.dt * mrel_max * rep;
    if (rep_cfl > 0.5)
        std::fprintf(stderr,
                     "[warn] dt*max_i(M_i/M0)*rep_coeff = %.4f; the overlap-repulsion term has under 2x "
                     "explicit-Euler margin at S_other ~ 1. Consider reducing dt (it is not changed "
                     "automatically).\n",
                     rep_cfl);
    const double vol_cfl = p.dt * mrel_max * 2.0 * p.mu;
    if (vol_cfl > 0.5)
        std::fprintf(stderr,
                     "[warn] dt*max_i(M_i/M0)*2*mu = %.4f; the area-constraint term has under 2x "
                     "explicit-Euler margin.\n",
                     vol_cfl);
    return true;
}

// Host-side check of the resolved per-cell pairs before any device work, as
// the reference validates the host initial condition before opening a GPU
// context (src/sim.cu:308-317, :390-399): a fresh start resolves gamma from
// the soft fraction and the mobility from the uniform value and the map; a
// resume reads the checkpoint's records and overlays the map. Unknown map ids
// are left to apply_mobility_map's message.
bool precheck_stiffness(const pfb_params2d& p, const std::string& ckpt_in,
                        const std::vector<std::pair<int32_t, float>>& map) {
    std::vector<pfb_cell2d> cells((size_t)p.num_cells);
    if (ckpt_in.empty()) {
        const long long soft = std::llround(p.cancer_fraction * (double)p.num_cells);
        for (int i = 0; i < p.num_cells; ++i) {
            cells[(size_t)i].global_id = i;
            cells[(size_t)i].gamma = (float)(i < soft ? p.gamma_cancer : p.gamma_normal);
            cells[(size_t)i].M_pf = (float)p.phase_field_mobility;
        }
    } else {
        std::vector<float> phi((size_t)p.num_cells * PFB_TILE_AREA);
        pfb_ckpt2d_info info{};
        pfb_ckpt2d_params rec{};
        if (pfb_ckpt2d_read(ckpt_in.c_str(), &info, &rec, cells.data(), phi.data()) != PFB_OK)
            return true;  // the resume path reports the reader's error
    }
    for (const auto& e : map)
        for (auto& c : cells)
            if (c.global_id == e.first) c.M_pf = e.second;
    return effective_stiffness_ok(p, cells);
}

// Overlay the map on the system's cell records (every listed id must exist);
// the resolved records must pass the explicit-Euler bound before the first
// step, on a fresh start and on a resume alike.
bool apply_mobility_map(pfb_sim2d* s, const pfb_params2d& p,
                        const std::vector<std::pair<int32_t, float>>& map, std::string* err) {
    const int N = pfb_sim2d_num_cells(s);
    std::vector<pfb_cell2d> cells((size_t)N);
    std::vector<float> phi((size_t)N * PFB_TILE_AREA);
    if (pfb_sim2d_get_cells(s, cells.data()) != PFB_OK || pfb_sim2d_get_phi(s, phi.data()) != PFB_OK)
        return *err = pfb_last_error(), false;
    for (const auto& e : map) {
        int hit = -1;
        for (int i = 0; i < N; ++i)
            if (cells[(size_t)i].global_id == e.first) hit = i;
        if (hit < 0)
            return *err = "map id " + std::to_string(e.first) + " does not exist among the " + std::to_string(N) +
                          " simulated global cell ids",
                   false;
        cells[(size_t)hit].M_pf = e.second;
    }
    if (!effective_stiffness_ok(p, cells))
        return *err = "the resolved per-cell mobilities break the explicit-Euler bound", false;
    if (pfb_sim2d_set_state(s, cells.data(), phi.data(), pfb_sim2d_step(s)) != PFB_OK)
        return *err = pfb_last_error(), false;
    return true;
}

constexpr double kPi = 3.14159265358979323846;

void usage() {
    std::printf(
        "usage: pfb_cell [options]\n"
        "  --N <int> --radius <f> --rho <f> --lambda <f> --kappa <f> --mu <f> --xi <f>\n"
        "  --tau <f> --v-A <f> --v-A-sigma <f> --gamma <f> --gamma-cancer <f>\n"
        "  --cancer-fraction <f> --phase-field-mobility <f> --dt <f> --t-end <f>\n"
        "  --seed <u64> --polarity-seed <u64> --full-moment <int> --verify-every <int>\n"
        "  --print-interval <int>  --initial-centres <csv>  -c|--checkpoint <path>\n"
        "  --checkpoint-interval <n>  --strict\n"
        "  --save-interval <n>  --checkpoint-dir <path>  --no-final-checkpoint\n"
        "  --trajectory-samples <n>  --trajectory-interval <n>  --out <path>\n"
        "  --device <int>  --bench <steps>  --no-graph  --morton  --no-l2\n"
        "  --velocity-moments <path>  --velocity-spatial-stride <1..1000>\n"
        "  --velocity-dense-start <int>  --velocity-moments-reference\n"
        "  --boundary-out <path>  --boundary-interval <int>  --boundary-compression <none|zstd>\n");
}

bool num(const char* s, double* v) {
    char* e = nullptr;
    errno = 0;
    *v = std::strtod(s, &e);
    return e != s && *e == '\0' && errno == 0 && std::isfinite(*v);
}
bool num(const char* s, long long* v) {
    char* e = nullptr;
    errno = 0;
    *v = std::strtoll(s, &e, 10);
    return e != s && *e == '\0' && errno == 0;
}
bool num(const char* s, unsigned long long* v) {
    char* e = nullptr;
    errno = 0;
    *v = std::strtoull(s, &e, 10);
    return e != s && *e == '\0' && errno == 0;
}

// FNV-1a 64 over the little-endian bytes of x0, y0, x1, y1, ... (binary32),
// the reference's centre-table fingerprint (include/palmieri_initializer.hpp:104-121).
uint64_t table_fnv1a64(const std::vector<float>& x, const std::vector<float>& y) {
    uint64_t h = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < x.size(); ++i)
        for (float f : {x[i], y[i]}) {
            uint32_t b;
            std::memcpy(&b, &f, 4);
            for (int k = 0; k < 4; ++k) {
                h ^= (b >> (8 * k)) & 0xffu;
                h *= 0x00000100000001b3ull;
            }
        }
    return h;
}

long long next_boundary(long long cur, long long every) {
    if (cur < 0 || every <= 0) return (1LL << 62);
    const long long r = cur % every;
    return cur + (r == 0 ? every : every - r);
}

bool mkdirs(const std::string& dir) {
    std::string acc;
    for (size_t i = 0; i <= dir.size(); ++i) {
        if (i == dir.size() || dir[i] == '/') {
            if (!acc.empty() && ::mkdir(acc.c_str(), 0777) != 0 && errno != EEXIST) return false;
        }
        if (i < dir.size()) acc.push_back(dir[i]);
    }
    return true;
}

// ---- trajectory text (reference src/trajectory.cpp, src/sim.cu:1104-1140) ----
std::string metadata(const pfb_params2d& p, double rho, uint64_t hash, long long every) {
    char line[2048];
    const double area0 = kPi * p.target_radius * p.target_radius;
    const double realized = (double)p.num_cells * area0 / ((double)p.L * p.L);
    const unsigned long long pstream = p.polarity_seed ? p.polarity_seed : p.seed;
    std::snprintf(line, sizeof(line),
                  "# trajectory_schema=1 dim=2 model=run_tumble N=%d Lx=%d Ly=%d "
                  "dx=%.17g dy=%.17g dt=%.17g rho_target=%.17g "
                  "rho_realized=%.17g lambda=%.17g R=%.17g kappa=%.17g mu=%.17g "
                  "xi=%.17g tau=%.17g v_A=%.17g v_A_sigma=%.17g "
                  "gamma_normal=%.17g gamma_soft=%.17g soft_fraction=%.17g "
                  "soft_assignment=lowest_global_ids seed=%llu polarity_seed=%llu "
                  "initialization_hash=%016llx full_moment=%d perim_offset=%.17g "
                  "trajectory_interval=%lld",
                  p.num_cells, p.L, p.L, 1.0, 1.0, p.dt, rho, realized, p.lambda, p.target_radius,
                  p.kappa, p.mu, p.xi, p.tau, p.v_A, p.v_A_sigma, p.gamma_normal, p.gamma_cancer,
                  p.cancer_fraction, (unsigned long long)p.seed, pstream, (unsigned long long)hash,
                  p.full_moment_every, kPi / (2.7386127875258306 / p.lambda), every);
    return line;
}
const char* kTitle = "# Trajectory data";
const char* kColumns = "# Format: time cell_id x y vx vy px py theta v_A_i L_n volume";

// Open for append: an empty file gets the three header lines; a non-empty one
// must carry this run's header and whole frames, in canonical id order, with
// strictly increasing times that end at or before the current step.
std::FILE* open_trajectory(const std::string& path, const std::string& meta, int N, double dt, long long step) {
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos && !mkdirs(path.substr(0, slash))) return nullptr;
    std::FILE* f = std::fopen(path.c_str(), "a+");
    if (!f) return nullptr;
    std::rewind(f);
    const int c0 = std::fgetc(f);
    if (c0 == EOF) {
        std::clearerr(f);
        std::fseek(f, 0, SEEK_END);
        std::fprintf(f, "%s\n%s\n%s\n", kTitle, kColumns, meta.c_str());
        std::fflush(f);
        return f;
    }
    std::rewind(f);
    std::vector<char> line(1 << 16);
    auto next = [&]() -> bool {
        if (!std::fgets(line.data(), (int)line.size(), f)) return false;
        size_t n = std::strlen(line.data());
        if (n && line[n - 1] == '\n') line[--n] = '\0';
        if (n && line[n - 1] == '\r') line[--n] = '\0';
        return true;
    };
    for (const std::string& want : {std::string(kTitle), std::string(kColumns), meta}) {
        if (!next() || want != line.data()) {
            std::fprintf(stderr, "[error] refusing to append: trajectory metadata does not match this run\n");
            std::fclose(f);
            return nullptr;
        }
    }
    unsigned long long rows = 0;
    double frame_t = 0.0, prev_t = -1.0;
    while (next()) {
        double v[11];
        long long id = 0;
        char extra = 0;
        const int got = std::sscanf(line.data(), "%lf %lld %lf %lf %lf %lf %lf %lf %lf %lf %lf %lf %c", &v[0], &id,
                                    &v[1], &v[2], &v[3], &v[4], &v[5], &v[6], &v[7], &v[8], &v[9], &v[10], &extra);
        bool ok = got == 12;
        for (double x : v) ok = ok && std::isfinite(x);
        const long long within = (long long)(rows % (unsigned long long)N);
        if (ok && within == 0) {
            frame_t = v[0];
            ok = rows == 0 || frame_t > prev_t;
        } else if (ok) {
            ok = v[0] == frame_t;
        }
        ok = ok && id == within;
        if (!ok) {
            std::fprintf(stderr, "[error] trajectory row %llu is malformed or out of order\n", rows + 1);
            std::fclose(f);
            return nullptr;
        }
        ++rows;
        if (rows % (unsigned long long)N == 0) prev_t = frame_t;
    }
    if (rows % (unsigned long long)N != 0) {
        std::fprintf(stderr, "[error] refusing to append to a partial trajectory frame\n");
        std::fclose(f);
        return nullptr;
    }
    if (rows > 0) {
        const long long last = std::llround(prev_t / dt);
        if (std::fabs((double)last * dt - prev_t) > 1e-10 * std::max(1.0, std::fabs(prev_t)) || last > step) {
            std::fprintf(stderr, "[error] trajectory extends beyond the initialized state\n");
            std::fclose(f);
            return nullptr;
        }
    }
    std::clearerr(f);
    std::fseek(f, 0, SEEK_END);
    return f;
}

bool write_frame(std::FILE* f, pfb_sim2d* s, const pfb_params2d& p, long long step,
                 std::vector<pfb_traj_cell2d>& t) {
    if (pfb_sim2d_pack_traj(s, t.data()) != PFB_OK) return false;
    const double Lw = (double)p.L;
    auto wrap = [Lw](double v) {
        double m = std::fmod(v, Lw);
        return m < 0.0 ? m + Lw : m;
    };
    for (const pfb_traj_cell2d& c : t) {
        const double th = (double)c.theta;
        if (std::fprintf(f, "%.17g %d %.6f %.6f %.6f %.6f %.6f %.6f %.6f %.6f %.6f %.6f\n", (double)step * p.dt,
                         c.global_id, wrap((double)c.cx), wrap((double)c.cy), (double)c.vx, (double)c.vy,
                         std::cos(th), std::sin(th), th, (double)c.v_A,
                         (double)c.perim / (2.0 * kPi * p.target_radius), (double)c.volume) < 0)
            return false;
    }
    return std::fflush(f) == 0;
}

bool fatal(const uint32_t* flags) {
    for (int i = 0; i < PFB_FLAG_COUNT; ++i)
        if (i != PFB_FLAG_SUPPORT_CLIP && flags[i]) return true;
    return false;
}

int parse(int argc, char** argv, Options* o) {
    pfb_params2d& p = o->p;
    p.num_cells = 288;
    p.dt = 0.01;
    p.lambda = 7.0;
    p.target_radius = 49.0;
    p.kappa = 10.0;
    p.mu = 1.0;
    p.xi = 1500.0;
    p.tau = 1.0e4;
    p.v_A = 1.0e-2;
    p.gamma_normal = 1.0;
    p.gamma_cancer = 0.35;
    p.cancer_fraction = 0.0;
    p.v_A_sigma = 0.0;
    p.phase_field_mobility = 0.5;
    p.seed = 1234;
    p.polarity_seed = 0;
    p.full_moment_every = 100;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&](void) -> const char* {
            if (i + 1 >= argc) return nullptr;
            return argv[++i];
        };
        double d;
        long long n;
        unsigned long long u;
        const char* v = nullptr;
        auto need_d = [&](double* dst, bool model) {
            v = val();
            if (!v || !num(v, &d)) return false;
            *dst = d;
            o->model_override = o->model_override || model;
            return true;
        };
        if (a == "-h" || a == "--help") {
            usage();
            std::exit(0);
        } else if (a == "--N") {
            if (!(v = val()) || !num(v, &n) || n <= 0 || n > 4000000) return 2;
            p.num_cells = (int)n;
            o->n_or_rho = true;
        } else if (a == "--radius") {
            if (!need_d(&p.target_radius, true)) return 2;
        } else if (a == "--rho") {
            if (!need_d(&o->rho, false)) return 2;
            o->n_or_rho = true;
        } else if (a == "--lambda") {
            if (!need_d(&p.lambda, true)) return 2;
        } else if (a == "--kappa") {
            if (!need_d(&p.kappa, true)) return 2;
        } else if (a == "--mu") {
            if (!need_d(&p.mu, true)) return 2;
        } else if (a == "--xi") {
            if (!need_d(&p.xi, true)) return 2;
        } else if (a == "--tau") {
            if (!need_d(&p.tau, true)) return 2;
        } else if (a == "--v-A") {
            if (!need_d(&p.v_A, true)) return 2;
        } else if (a == "--v-A-sigma") {
            if (!need_d(&p.v_A_sigma, true)) return 2;
        } else if (a == "--gamma") {
            if (!need_d(&p.gamma_normal, true)) return 2;
        } else if (a == "--gamma-cancer") {
            if (!need_d(&p.gamma_cancer, true)) return 2;
        } else if (a == "--cancer-fraction") {
            if (!need_d(&p.cancer_fraction, true)) return 2;
        } else if (a == "--phase-field-mobility") {
            if (!need_d(&p.phase_field_mobility, true)) return 2;
        } else if (a == "--dt") {
            if (!need_d(&p.dt, true)) return 2;
        } else if (a == "--t-end") {
            if (!need_d(&o->t_end, false)) return 2;
            o->t_end_set = true;
        } else if (a == "--seed") {
            if (!(v = val()) || !num(v, &u)) return 2;
            p.seed = u;
            o->model_override = true;
        } else if (a == "--polarity-seed") {
            if (!(v = val()) || !num(v, &u)) return 2;
            p.polarity_seed = u;
            o->model_override = true;
        } else if (a == "--full-moment") {
            if (!(v = val()) || !num(v, &n) || n < 0) return 2;
            p.full_moment_every = (int)n;
        } else if (a == "--verify-every") {
            if (!(v = val()) || !num(v, &n) || n < 0) return 2;
            o->verify_every = (int)n;
            o->verify_set = true;
        } else if (a == "--print-interval") {
            if (!(v = val()) || !num(v, &n) || n < 0) return 2;
            o->print_interval = (int)n;
            o->print_set = true;
        } else if (a == "-c" || a == "--checkpoint") {
            if (!(v = val())) return 2;
            o->ckpt_in = v;
        } else if (a == "--checkpoint-interval") {
            if (!(v = val()) || !num(v, &n) || n < 0) return 2;
            o->ckpt_interval = n;
        } else if (a == "--save-interval") {
            if (!(v = val()) || !num(v, &n) || n < 0) return 2;
            o->save_interval = n;
        } else if (a == "--checkpoint-dir") {
            if (!(v = val())) return 2;
            o->ckpt_dir = v;
        } else if (a == "--no-final-checkpoint") {
            o->final_ckpt = false;
        } else if (a == "--trajectory-samples") {
            if (!(v = val()) || !num(v, &n) || n <= 0) return 2;
            o->traj_samples = (int)n;
            o->traj_samples_set = true;
        } else if (a == "--trajectory-interval") {
            if (!(v = val()) || !num(v, &n) || n < 0) return 2;
            o->traj_interval = n;
            o->traj_interval_set = true;
        } else if (a == "--out") {
            if (!(v = val())) return 2;
            o->out_path = v;
        } else if (a == "--device") {
            if (!(v = val()) || !num(v, &n) || n < 0) return 2;
            o->device = (int)n;
        } else if (a == "--bench") {
            if (!(v = val()) || !num(v, &n) || n <= 0) return 2;
            o->bench = n;
        } else if (a == "--no-graph") {
            o->graph = false;
        } else if (a == "--velocity-moments") {
            if (!(v = val())) return 2;
            o->vel_path = v;
            o->vel_given = true;
        } else if (a == "--velocity-spatial-stride") {
            if (!(v = val()) || !num(v, &n) || n < 1 || n > 1000) return 2;
            o->vel_stride = (int)n;
            o->vel_given = true;
        } else if (a == "--velocity-dense-start") {
            if (!(v = val()) || !num(v, &n) || n < 0 || n > 1000000000) return 2;
            o->vel_dense = n;
            o->vel_given = true;
        } else if (a == "--velocity-moments-reference") {
            o->vel_reference = true;
            o->vel_given = true;
        } else if (a == "--boundary-out") {
            if (!(v = val()) || !v[0]) return 2;
            o->bnd_path = v;
        } else if (a == "--boundary-interval") {
            if (!(v = val()) || !num(v, &n) || n < 1 || n > 1000000000000LL) return 2;
            o->bnd_interval = n;
        } else if (a == "--boundary-compression") {
            if (!(v = val())) return 2;
            if (!std::strcmp(v, "none"))
                o->bnd_compress = false;
            else if (!std::strcmp(v, "zstd"))
                o->bnd_compress = true;
            else
                return 2;
        } else if (a == "--initial-centres") {
            if (!(v = val())) return 2;
            if (!v[0]) {
                std::fprintf(stderr, "[fatal] --initial-centres requires a non-empty path\n");
                return 2;
            }
            o->centres_path = v;
        } else if (a == "--strict") {
            o->strict = true;
        } else if (a == "--phase-field-mobility-map") {
            if (!(v = val()) || !v[0]) {
                std::fprintf(stderr, "[fatal] --phase-field-mobility-map requires a non-empty path\n");
                return 2;
            }
            o->mobility_map = v;
        } else if (a == "--morton") {
            o->morton = true;
        } else if (a == "--no-l2") {
            // S is never pinned in an L2 persisting carve-out here
        } else if (a == "--self-test") {
            o->self_test = true;
        } else {
            std::fprintf(stderr, "[fatal] unknown option '%s' (try --help)\n", a.c_str());
            return 2;
        }
    }
    return 0;
}

long long total_steps(double t_end, double dt) {
    const double n = t_end / dt + 0.5;
    return (n >= 0.0 && n <= 9.0e18) ? (long long)n : -1;
}

}  // namespace

// --self-test (reference src/main.cu:144-321): host checks of the nine-point
// stencil, the model coefficients the library derives, the sign of the
// repulsive velocity between two overlapping disks, the tumble probability
// and the uniformity of the Philox stream, and the class windows against the
// interface width. Returns the number of failed checks.
static int self_test(const pfb_params2d& p) {
    std::printf("--- self-test checks ---\n");
    int bad = 0;
    auto mark = [&](bool ok) {
        bad += ok ? 0 : 1;
        return ok ? "PASS" : "FAIL";
    };
    {
        const float lap = pfb::lap9(1, 0, 1, 1, 0, 1, 1, 0, 1);  // f = x^2 around x = 0
        const float flat = pfb::lap9(1, 1, 1, 1, 1, 1, 1, 1, 1);
        std::printf("  [%s] Laplacian stencil: lap(x^2) = %.9g (expected 2), lap(1) = %.9g\n",
                    mark(lap == 2.0f && flat == 0.0f), lap, flat);
    }
    pfb_step_args2d a;
    std::memset(&a, 0, sizeof(a));
    pfb_fill_coefficients2d(&p, &a);
    {
        const double bulk = pfb::coeff_bulk(p.lambda), rep = pfb::coeff_interaction(p.kappa, p.lambda);
        const double ratio = (double)a.rep_coeff / (double)a.mot_coeff;
        const bool ok = std::fabs(rep - 2.0 * p.kappa * bulk) <= 1e-12 * rep &&
                        std::fabs((double)a.rep_coeff - rep) <= 1e-6 * rep &&
                        std::fabs(ratio - p.xi) <= 1e-6 * p.xi;
        std::printf("  [%s] coefficients: 30/l^2 = %.9g  60k/l^2 = %.9g (library %.9g)  "
                    "60k/(xi l^2) = %.9g  ratio = %.9g (want xi = %.9g)\n",
                    mark(ok), bulk, rep, (double)a.rep_coeff, (double)a.mot_coeff, ratio, p.xi);
    }
    {
        // cell n left of cell m: phi_n falls to the right inside their overlap,
        // so the interaction integral, and n's velocity, point away from m
        const int L = 192;
        const double R = 20.0, k = pfb::iface_k(p.lambda);
        std::vector<double> pn((size_t)L * L), pm((size_t)L * L);
        for (int sep = 26; sep <= 38; sep += 4) {
            const double xn = 0.5 * (L - sep), xm = 0.5 * (L + sep);
            for (int y = 0; y < L; ++y)
                for (int x = 0; x < L; ++x) {
                    const double dy = y - 0.5 * L;
                    pn[(size_t)y * L + x] = 0.5 * (1.0 - std::tanh(k * (std::hypot(x - xn, dy) - R)));
                    pm[(size_t)y * L + x] = 0.5 * (1.0 - std::tanh(k * (std::hypot(x - xm, dy) - R)));
                }
            double Ix = 0.0;
            for (int y = 0; y < L; ++y)
                for (int x = 1; x < L - 1; ++x) {
                    const size_t i = (size_t)y * L + x;
                    Ix += pn[i] * 0.5 * (pn[i + 1] - pn[i - 1]) * pm[i] * pm[i];
                }
            std::printf("  [%s] repulsive sign at separation %d: Ix = %+.6e  vx = %+.6e (n moves away from m)\n",
                        mark(Ix < 0.0), sep, Ix, (double)a.mot_coeff * Ix);
        }
    }
    {
        const double tau_eff = -p.dt / std::log1p(-a.p_tumble);
        std::printf("  [%s] tumble probability %.9e per step -> tau_eff = %.6f (tau %.6f)\n",
                    mark(std::fabs(tau_eff - p.tau) <= 1e-9 * p.tau), a.p_tumble, tau_eff, p.tau);
        const double tau_s = 10.0, ps = -std::expm1(-p.dt / tau_s);
        const long long trials = 5000000;
        long long hits = 0;
        for (long long i = 0; i < trials; ++i) {
            const pfb::Words4 r = pfb::philox10((uint32_t)i, (uint32_t)(i >> 32), 7u, 0xA5A5A5A5u,
                                                (uint32_t)p.seed, 0u);
            hits += pfb::u53(r.w[0], r.w[1]) < ps;
        }
        const double ph = (double)hits / (double)trials, tau_m = -p.dt / std::log1p(-ph);
        const double sigma = std::sqrt(ps * (1.0 - ps) / (double)trials) / ps;
        std::printf("  [%s] Philox draws: %lld at p = %.6e, tau_eff = %.3f (want %.1f +- %.3f at 5 sigma)\n",
                    mark(std::fabs(tau_m - tau_s) <= 5.0 * sigma * tau_s), trials, ps, tau_m, tau_s,
                    5.0 * sigma * tau_s);
    }
    {
        // a relaxed hexagon's circumradius plus the distance at which phi^2
        // falls below half a Q5.27 quantum, plus one pixel, on each axis
        const double k = pfb::iface_k(p.lambda), A0 = kPi * p.target_radius * p.target_radius;
        const double need = std::sqrt(A0 / (1.5 * std::sqrt(3.0))) + std::log(2.0 / pfb::kQInvD) / (4.0 * k) + 1.0;
        for (int c = 0; c < pfb::kNumClasses; ++c) {
            const pfb::Window w = pfb::window_of(c);
            const int half = std::min(w.wx, w.wy) / 2;
            std::printf("  [%s] class %d window %d x %d: half-width %d, required %.2f\n",
                        mark((double)half >= need), c, w.wx, w.wy, half, need);
        }
    }
    std::printf("--- %s ---\n", bad ? "SELF-TEST FAILED" : "self-test passed");
    return bad;
}

int main(int argc, char** argv) {
    Options o;
    if (parse(argc, argv, &o)) {
        std::fprintf(stderr, "[fatal] invalid or missing option value (try --help)\n");
        return 2;
    }
    if (o.vel_given && (o.vel_path.empty() || (o.out_path.empty() && o.bench == 0))) {
        std::fprintf(stderr, "[fatal] velocity recording requires --velocity-moments and --out\n");
        return 2;
    }
    if (o.vel_given && o.bench > 0) {
        std::fprintf(stderr, "[fatal] velocity observation under --bench is not part of this build\n");
        return 2;
    }
    if (o.bnd_path.empty() != (o.bnd_interval == 0) || (o.bnd_compress && o.bnd_path.empty()) ||
        (!o.bnd_path.empty() && o.bench > 0)) {
        std::fprintf(stderr, "[fatal] boundary output requires a path and interval, and cannot be used "
                             "with --bench\n");
        return 2;
    }
    if ((!o.bnd_path.empty() && (o.bnd_path == o.out_path || o.bnd_path == o.vel_path)) ||
        (!o.vel_path.empty() && o.vel_path == o.out_path)) {
        std::fprintf(stderr, "[fatal] output files must use distinct paths\n");
        return 2;
    }
    std::vector<std::pair<int32_t, float>> mobility;
    if (!o.mobility_map.empty()) {
        std::string err;
        if (!read_mobility_map(o.mobility_map, &mobility, &err)) {
            std::fprintf(stderr, "[fatal] phase-field mobility map: %s\n", err.c_str());
            return 2;
        }
    }
    pfb_params2d p = o.p;
    uint64_t hash = 0;
    pfb_sim2d* s = nullptr;
    pfb_ckpt2d_params rec{};
    if (!o.ckpt_in.empty()) {
        if (!o.centres_path.empty()) {
            std::fprintf(stderr, "[fatal] --initial-centres is valid only for a fresh start; a checkpoint "
                                 "already holds the initialised state\n");
            return 2;
        }
        if (o.n_or_rho) {
            std::fprintf(stderr, "[fatal] --N and --rho cannot be overridden on resume\n");
            return 2;
        }
        if (o.model_override) {
            std::fprintf(stderr, "[fatal] this build resumes with the checkpoint's model parameters; "
                                 "drop the model options\n");
            return 2;
        }
        pfb_ckpt2d_info info{};
        if (pfb_ckpt2d_read(o.ckpt_in.c_str(), &info, &rec, nullptr, nullptr) != PFB_OK) {
            std::fprintf(stderr, "[ckpt] %s\n", pfb_last_error());
            return 8;
        }
        if (pfb_ckpt2d_params_to(&rec, info.num_cells, &p) != PFB_OK) return 8;
        hash = rec.initialization_hash;
        o.rho = rec.rho;
        if (!o.traj_samples_set && !o.traj_interval_set) {
            o.traj_samples = rec.trajectory_samples;
            o.traj_interval = rec.trajectory_interval;
        }
        if (!o.t_end_set) o.t_end = rec.t_end;
        if (!o.print_set) o.print_interval = rec.print_interval;
        if (!o.verify_set) o.verify_every = rec.verify_every;
        if (o.self_test && self_test(p)) return 4;
        if (!mobility.empty() && !precheck_stiffness(p, o.ckpt_in, mobility)) return 5;
        s = pfb_sim2d_create_from_checkpoint(o.ckpt_in.c_str(), o.device);
    } else {
        p.L = pfb_domain_side_for(p.num_cells, p.target_radius, o.rho);
        if (p.L <= 286) {
            std::fprintf(stderr, "[fatal] domain side %d must exceed 286\n", p.L);
            return 3;
        }
        std::vector<float> x((size_t)p.num_cells), y((size_t)p.num_cells);
        if (!o.centres_path.empty()) {
            // a validated table (reference src/sim.cu:90-106)
            std::string err;
            if (!pfb_csv::read_table2(o.centres_path, p.num_cells, (double)p.L, p.target_radius, x, y, &err)) {
                std::fprintf(stderr, "[fatal] invalid --initial-centres '%s': %s\n", o.centres_path.c_str(),
                             err.c_str());
                return 5;
            }
        } else if (pfb_grid_jitter_centres(p.num_cells, p.L, p.seed, x.data(), y.data()) != PFB_OK) {
            return 3;
        }
        hash = table_fnv1a64(x, y);
        std::printf("  centres: %d, table hash %016llx\n", p.num_cells, (unsigned long long)hash);
        std::fflush(stdout);
        if (o.self_test && self_test(p)) return 4;
        if (!mobility.empty() && !precheck_stiffness(p, "", mobility)) return 5;
        s = pfb_sim2d_create(&p, x.data(), y.data(), o.device);
    }
    if (!s) {
        std::fprintf(stderr, "[fatal] initialisation failed: %s\n", pfb_last_error());
        return 5;
    }
    if (!mobility.empty()) {
        std::string err;
        if (!apply_mobility_map(s, p, mobility, &err)) {
            std::fprintf(stderr, "[fatal] phase-field mobility: %s\n", err.c_str());
            pfb_sim2d_destroy(s);
            return 5;
        }
    }
    pfb_sim2d_set_graph(s, o.graph ? 1 : 0);
    if (o.morton) {
        const int rc = pfb_sim2d_set_visit_order(s, PFB_VISIT_MORTON);
        if (rc == PFB_E_CONFIG) {
            std::fprintf(stderr, "[warn] %s. Falling back to launch order.\n", pfb_last_error());
        } else if (rc) {
            std::fprintf(stderr, "[fatal] visit order: %s\n", pfb_last_error());
            pfb_sim2d_destroy(s);
            return 5;
        } else {
            std::printf("  visit order: Morton, re-sorted every six steps\n");
        }
    }
    const long long total = total_steps(o.t_end, p.dt);
    if (total < pfb_sim2d_step(s)) {
        std::fprintf(stderr, "[fatal] t_end ends at step %lld, before the state's step %lld\n", total,
                     pfb_sim2d_step(s));
        pfb_sim2d_destroy(s);
        return 3;
    }
    std::printf("pfb_cell: N %d  L %d  dt %g  steps %lld -> %lld  centre table %016llx\n", p.num_cells, p.L, p.dt,
                pfb_sim2d_step(s), total, (unsigned long long)hash);

    if (o.bench > 0) {
        double ms = 0.0;
        if (pfb_sim2d_bench(s, 30, (int)o.bench, &ms) != PFB_OK) {
            std::fprintf(stderr, "[fatal] bench failed: %s\n", pfb_last_error());
            pfb_sim2d_destroy(s);
            return 6;
        }
        std::printf("bench: %lld steps -> %.6f ms/step\n", o.bench, ms);
        pfb_sim2d_destroy(s);
        return 0;
    }

    // checkpoint record of this run
    pfb_ckpt2d_params_from(&p, &rec);
    rec.t_end = o.t_end;
    rec.rho = o.rho;
    rec.initialization_hash = hash;
    rec.print_interval = o.print_interval;
    rec.verify_every = o.verify_every;
    rec.save_interval = (int32_t)o.save_interval;
    rec.trajectory_samples = o.traj_samples;
    const long long traj_every = o.traj_interval > 0 ? o.traj_interval
                                                     : std::max<long long>(1, total / std::max(1, o.traj_samples));
    rec.trajectory_interval = traj_every;
    const bool ckpt_on = !o.ckpt_dir.empty() || o.ckpt_interval > 0 || o.save_interval > 0 || !o.ckpt_in.empty();
    std::string dir = o.ckpt_dir;
    if (ckpt_on && dir.empty()) {
        const std::string src = !o.out_path.empty() ? o.out_path : o.ckpt_in;
        const size_t slash = src.rfind('/');
        dir = slash == std::string::npos ? "." : src.substr(0, slash);
    }
    if (ckpt_on && !mkdirs(dir)) {
        std::fprintf(stderr, "[fatal] cannot create checkpoint directory %s\n", dir.c_str());
        pfb_sim2d_destroy(s);
        return 2;
    }
    std::FILE* traj = nullptr;
    std::vector<pfb_traj_cell2d> rows((size_t)p.num_cells);
    if (!o.out_path.empty()) {
        traj = open_trajectory(o.out_path, metadata(p, o.rho, hash, traj_every), p.num_cells, p.dt,
                               pfb_sim2d_step(s));
        if (!traj) {
            pfb_sim2d_destroy(s);
            return 9;
        }
    }
    if (!o.vel_path.empty() &&
        pfb_sim2d_velocity_open(s, o.vel_path.c_str(), o.vel_stride, o.vel_dense, o.vel_reference ? 1 : 0) !=
            PFB_OK) {
        std::fprintf(stderr, "[velocity] %s\n", pfb_last_error());
        if (traj) std::fclose(traj);
        pfb_sim2d_destroy(s);
        return 9;
    }
    long long last_boundary = -1;
    if (!o.bnd_path.empty()) {
        if (pfb_sim2d_boundary_open(s, o.bnd_path.c_str(), o.bnd_interval, o.bnd_compress ? 1 : 0) != PFB_OK ||
            pfb_sim2d_boundary_capture(s) != PFB_OK) {
            std::fprintf(stderr, "[boundary] %s\n", pfb_last_error());
            if (traj) std::fclose(traj);
            pfb_sim2d_destroy(s);
            return 9;
        }
        last_boundary = pfb_sim2d_step(s);
    }
    std::signal(SIGINT, on_signal);
    std::signal(SIGTERM, on_signal);

    auto save = [&](const std::string& path) {
        if (pfb_sim2d_write_checkpoint(s, path.c_str(), &rec) != PFB_OK) {
            std::fprintf(stderr, "[ckpt] %s\n", pfb_last_error());
            return false;
        }
        std::printf("[ckpt] saved step %lld -> %s\n", pfb_sim2d_step(s), path.c_str());
        return true;
    };
    const long long pi = o.print_interval > 0 ? o.print_interval : total;
    long long step = pfb_sim2d_step(s);
    long long next_traj = traj ? next_boundary(step, traj_every) : total + 1;
    long long next_ckpt = ckpt_on && o.ckpt_interval > 0 ? step + o.ckpt_interval : total + 1;
    long long next_save = ckpt_on && o.save_interval > 0 ? step + o.save_interval : total + 1;
    constexpr long long kFatalPoll = 1000;
    long long next_poll = step + kFatalPoll;
    long long next_bnd = o.bnd_path.empty() ? total + 1 : step + o.bnd_interval;
    // --strict: invariant report at multiples of verify_every (reference src/sim.cu:860-973)
    long long next_verify = o.strict && o.verify_every > 0 ? next_boundary(step, o.verify_every) : total + 1;
    bool failed = false;
    uint32_t flags[PFB_FLAG_COUNT];
    while (step < total && !failed) {
        const long long stop =
            std::min({total, (step / pi + 1) * pi, next_traj, next_ckpt, next_save, next_poll, next_bnd,
                      next_verify});
        if (pfb_sim2d_advance(s, stop - step) != PFB_OK) {
            std::fprintf(stderr, "[fatal] %s\n", pfb_last_error());
            failed = true;
            break;
        }
        step = stop;
        if (pfb_sim2d_get_flags(s, flags) != PFB_OK || fatal(flags)) {
            std::fprintf(stderr, "[fatal] a fatal flag was raised by step %lld\n", step);
            failed = true;
            break;
        }
        if (step >= next_poll) next_poll = step + kFatalPoll;
        if (step % pi == 0 || step >= total)
            std::printf("step %8lld  t %10.3f\n", step, (double)step * p.dt);
        if (traj && step >= next_traj) {
            if (!write_frame(traj, s, p, step, rows)) {
                std::fprintf(stderr, "[error] trajectory write failed at step %lld\n", step);
                failed = true;
                break;
            }
            next_traj = next_boundary(step, traj_every);
            // a velocity frame rides with every trajectory frame
            if (!o.vel_path.empty() && pfb_sim2d_velocity_capture(s) != PFB_OK) {
                std::fprintf(stderr, "[velocity] %s\n", pfb_last_error());
                failed = true;
                break;
            }
        }
        if (step >= next_bnd) {
            if (pfb_sim2d_boundary_capture(s) != PFB_OK) {
                std::fprintf(stderr, "[boundary] %s\n", pfb_last_error());
                failed = true;
                break;
            }
            last_boundary = step;
            next_bnd = step + o.bnd_interval;
        }
        if (step >= next_ckpt) {
            if (!save(dir + "/checkpoint.bin")) failed = true;
            next_ckpt = step + o.ckpt_interval;
        }
        if (step >= next_save) {
            char name[64];
            std::snprintf(name, sizeof(name), "/checkpoint_%08lld.bin", step);
            if (!save(dir + name)) failed = true;
            next_save = step + o.save_interval;
        }
        if (step >= next_verify) {
            double mr = 0.0;
            float mo = 0.0f;
            uint32_t ms = 0;
            if (pfb_sim2d_verify(s, &mr, &mo, &ms) == PFB_OK)
                std::printf("  [verify] step %lld  max rel V error %.3e   max|phi| outside window %.3e   "
                            "max S %.6f\n",
                            step, mr, (double)mo, (double)ms * 7.45058059692382812e-09);
            next_verify = step + o.verify_every;
        }
        if (g_stop) {
            std::printf("[signal] termination requested at step %lld\n", step);
            break;
        }
    }
    if (traj) std::fclose(traj);
    if (!o.vel_path.empty()) {
        // a closing frame of a valid state, then close the file
        if (!failed && pfb_sim2d_velocity_last_frame(s) != step && pfb_sim2d_velocity_capture(s) != PFB_OK) {
            std::fprintf(stderr, "[velocity] %s\n", pfb_last_error());
            failed = true;
        }
        if (pfb_sim2d_velocity_close(s) != PFB_OK) failed = true;
    }
    if (!o.bnd_path.empty()) {
        if (!failed && last_boundary != step && pfb_sim2d_boundary_capture(s) != PFB_OK) {
            std::fprintf(stderr, "[boundary] %s\n", pfb_last_error());
            failed = true;
        }
        if (pfb_sim2d_boundary_close(s) != PFB_OK) {
            std::fprintf(stderr, "[boundary] %s\n", pfb_last_error());
            failed = true;
        }
    }
    if (ckpt_on && (o.final_ckpt || failed)) {
        if (!save(dir + (failed ? "/checkpoint_failed.bin" : "/checkpoint.bin"))) failed = true;
    }
    pfb_sim2d_destroy(s);
    return failed ? 9 : 0;
}
