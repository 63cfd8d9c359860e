// Centre tables accepted by --initial-centres (host only, used by the command
// lines). Formats and acceptance rules follow the reference so that a table
// it accepts is accepted here with the same binary32 values:
//   * read_table2: "global_id,x,y" then N rows "id,x,y" (LF only); ordered ids
//     0..N-1; cell 0 exactly at the box centre; every centre in [0, L); no two
//     centres closer than `radius` (periodic) (include/palmieri_initializer.hpp:
//     122-175, 245-306);
//   * read_relaxed2: the relaxed 2D table of a substrate or one-layer channel:
//     a byte-order mark and CR line ends tolerated, "global_id,x,y", an
//     optional "# source_L=<L>" line that must equal the box side (required
//     with `need_source_side`), N rows of int64 id, x, y in [0, L), no
//     separation rule (include/relaxed_centres.hpp:30-183);
//   * read_table3 / read_channel3: "global_id,x,y,z" then N rows; the periodic
//     table as read_table2 in three dimensions; the channel table with cell 0
//     at (L/2, L/2, H/2), z in [radius, H - radius] and the separation taken
//     periodically in x, y only (include/pf3d/palmieri_initializer.hpp:
//     134-194, 270-347, 411-543).
// Numbers are parsed with std::from_chars (general format) directly to
// binary32. Each reader returns false with a message in `err`.
#pragma once

#include <charconv>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <limits>
#include <string>
#include <system_error>
#include <vector>

namespace pfb_csv {

inline bool parse_int(const char* a, const char* b, int* v) {
    const auto r = std::from_chars(a, b, *v, 10);
    return r.ec == std::errc{} && r.ptr == b;
}
inline bool parse_i64(const char* a, const char* b, int64_t* v) {
    const auto r = std::from_chars(a, b, *v, 10);
    return r.ec == std::errc{} && r.ptr == b;
}
inline bool parse_f32(const char* a, const char* b, float* v) {
    const auto r = std::from_chars(a, b, *v, std::chars_format::general);
    return r.ec == std::errc{} && r.ptr == b;
}
inline double min_image(double d, double side) { return d - side * std::floor(d / side + 0.5); }

// Split a row into exactly `n` comma-separated fields [begin, end).
inline bool split(const std::string& line, int n, const char** b, const char** e) {
    size_t start = 0;
    for (int k = 0; k < n; ++k) {
        const size_t c = line.find(',', start);
        const bool last = k == n - 1;
        if (last ? c != std::string::npos : c == std::string::npos) return false;
        const size_t stop = last ? line.size() : c;
        b[k] = line.data() + start;
        e[k] = line.data() + stop;
        start = stop + 1;
    }
    return true;
}

// Shared body of the strict 2D and 3D tables: header, N ordered rows of
// `dims` binary32 coordinates, no extra row.
inline bool read_strict(const std::string& path, int n, int dims, const char* header,
                        std::vector<float>* out, std::string* err) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return *err = "cannot open centre CSV: " + path, false;
    std::string line;
    if (!std::getline(in, line) || line != header)
        return *err = std::string("CSV header must be exactly ") + header + " with LF line endings", false;
    for (int d = 0; d < dims; ++d) out[d].clear();
    for (int id = 0; id < n; ++id) {
        if (!std::getline(in, line)) return *err = "centre CSV ended before expected N rows", false;
        const char* b[4];
        const char* e[4];
        if (!split(line, dims + 1, b, e))
            return *err = dims == 2 ? "centre CSV row must contain exactly three fields"
                                    : "centre CSV row must contain exactly four fields",
                   false;
        int got = -1;
        float v[3] = {0.0f, 0.0f, 0.0f};
        bool ok = parse_int(b[0], e[0], &got);
        for (int d = 0; ok && d < dims; ++d) ok = parse_f32(b[d + 1], e[d + 1], &v[d]);
        if (!ok) return *err = "centre CSV contains a malformed field", false;
        if (got != id) return *err = "global_id must be the ordered sequence 0..N-1", false;
        for (int d = 0; d < dims; ++d) out[d].push_back(v[d]);
    }
    if (std::getline(in, line)) return *err = "centre CSV contains more than expected N rows", false;
    if (in.bad()) return *err = "I/O failure while reading centre CSV", false;
    return true;
}

// Cell 0 at the centre, every centre in [0, side) and the separation rule,
// periodically in the first `periodic` coordinates.
inline bool validate(const std::vector<float>* c, int dims, int periodic, double side,
                     const float* centre, const double* lo, const double* hi, double radius,
                     std::string* err) {
    const size_t n = c[0].size();
    for (int d = 0; d < dims; ++d)
        if (c[d][0] != centre[d]) return *err = "global_id 0 is not exactly at the box centre", false;
    for (size_t i = 0; i < n; ++i)
        for (int d = 0; d < dims; ++d) {
            const float v = c[d][i];
            if (!std::isfinite(v) || !(v >= lo[d] && v < hi[d]))
                return *err = "centre is non-finite or outside its box", false;
        }
    const double r2 = radius * radius;
    for (size_t i = 1; i < n; ++i)
        for (size_t j = 0; j < i; ++j) {
            double d2 = 0.0;
            for (int d = 0; d < dims; ++d) {
                double x = (double)c[d][i] - (double)c[d][j];
                if (d < periodic) x = min_image(x, side);
                d2 += x * x;
            }
            if (d2 < r2) return *err = "centre table violates the minimum-separation rule", false;
        }
    return true;
}

inline bool read_table2(const std::string& path, int n, double side, double radius,
                        std::vector<float>& x, std::vector<float>& y, std::string* err) {
    std::vector<float> c[2];
    if (!read_strict(path, n, 2, "global_id,x,y", c, err)) return false;
    const float mid = (float)(0.5 * side);
    const float centre[2] = {mid, mid};
    const double lo[2] = {0.0, 0.0}, hi[2] = {side, side};
    if (!validate(c, 2, 2, side, centre, lo, hi, radius, err)) return false;
    x = c[0];
    y = c[1];
    return true;
}

inline bool read_table3(const std::string& path, int n, double side, double radius,
                        std::vector<float>& x, std::vector<float>& y, std::vector<float>& z,
                        std::string* err) {
    std::vector<float> c[3];
    if (!read_strict(path, n, 3, "global_id,x,y,z", c, err)) return false;
    const float mid = (float)(0.5 * side);
    const float centre[3] = {mid, mid, mid};
    const double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {side, side, side};
    if (!validate(c, 3, 3, side, centre, lo, hi, radius, err)) return false;
    x = c[0];
    y = c[1];
    z = c[2];
    return true;
}

// z must lie in [radius, H - radius] (both ends included).
inline bool read_channel3(const std::string& path, int n, double side, int H, double radius,
                          std::vector<float>& x, std::vector<float>& y, std::vector<float>& z,
                          std::string* err) {
    std::vector<float> c[3];
    if (!read_strict(path, n, 3, "global_id,x,y,z", c, err)) return false;
    if ((double)H - radius < radius) return *err = "channel height is smaller than one cell diameter", false;
    const float mid = (float)(0.5 * side);
    const float centre[3] = {mid, mid, (float)(0.5 * H)};
    const size_t cnt = c[0].size();
    for (int d = 0; d < 3; ++d)
        if (c[d][0] != centre[d]) return *err = "global_id 0 is not exactly at the channel centre", false;
    for (size_t i = 0; i < cnt; ++i) {
        const float xv = c[0][i], yv = c[1][i], zv = c[2][i];
        if (!std::isfinite(xv) || !std::isfinite(yv) || !std::isfinite(zv) || xv < 0.0f || xv >= side ||
            yv < 0.0f || yv >= side || zv < radius || zv > (double)H - radius)
            return *err = "channel centre is non-finite, outside x/y, or lacks wall clearance", false;
    }
    const double lo[3] = {0.0, 0.0, -1e300}, hi[3] = {side, side, 1e300};
    if (!validate(c, 3, 2, side, centre, lo, hi, radius, err)) return false;
    x = c[0];
    y = c[1];
    z = c[2];
    return true;
}

inline void normalise(std::string* line, bool first) {
    if (!line->empty() && line->back() == '\r') line->pop_back();
    if (first && line->size() >= 3 && (unsigned char)(*line)[0] == 0xEF &&
        (unsigned char)(*line)[1] == 0xBB && (unsigned char)(*line)[2] == 0xBF)
        line->erase(0, 3);
}

// The header line of a table (normalised), empty if unreadable.
inline std::string first_line(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    std::string line;
    if (!in || !std::getline(in, line)) return std::string();
    normalise(&line, true);
    return line;
}

inline bool read_relaxed2(const std::string& path, int n, double side, bool need_source_side,
                          std::vector<int64_t>& ids, std::vector<float>& x, std::vector<float>& y,
                          std::string* err) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return *err = "cannot open relaxed-centre CSV: " + path, false;
    std::string line;
    if (!std::getline(in, line)) return *err = "centre CSV is empty", false;
    normalise(&line, true);
    if (line != "global_id,x,y") return *err = "CSV header must be exactly global_id,x,y", false;
    if (!std::getline(in, line)) return *err = "centre CSV has no data rows", false;
    normalise(&line, false);
    bool pending = true;  // `line` holds the first data row
    static const std::string kSide = "# source_L=";
    if (line.compare(0, kSide.size(), kSide) == 0) {
        int64_t s = 0;
        if (!parse_i64(line.data() + kSide.size(), line.data() + line.size(), &s) || s <= 0 ||
            s > std::numeric_limits<int>::max())
            return *err = "centre CSV has an invalid source_L", false;
        if ((double)s != side) return *err = "centre CSV source_L does not match the target box", false;
        pending = false;
    } else if (need_source_side) {
        return *err = "one-layer channel centre CSV requires # source_L=L", false;
    }
    ids.clear();
    x.clear();
    y.clear();
    for (int row = 0; row < n; ++row) {
        if ((!pending || row != 0) && !std::getline(in, line))
            return *err = "centre CSV ended before expected N rows", false;
        normalise(&line, false);
        const char* b[3];
        const char* e[3];
        if (!split(line, 3, b, e)) return *err = "centre CSV row must contain exactly three fields", false;
        int64_t id = 0;
        float xv = 0.0f, yv = 0.0f;
        if (!parse_i64(b[0], e[0], &id) || !parse_f32(b[1], e[1], &xv) || !parse_f32(b[2], e[2], &yv))
            return *err = "centre CSV contains a malformed field", false;
        if (id != (int64_t)row) return *err = "centre CSV rows must have global_id 0..N-1 in order", false;
        if (!std::isfinite(xv) || !std::isfinite(yv) || !(xv >= 0.0f && xv < side) || !(yv >= 0.0f && yv < side))
            return *err = "centre is non-finite or outside the target [0,L) box", false;
        ids.push_back(id);
        x.push_back(xv);
        y.push_back(yv);
    }
    if (std::getline(in, line)) return *err = "centre CSV contains more than expected N rows", false;
    if (in.bad()) return *err = "I/O failure while reading centre CSV", false;
    return true;
}

}  // namespace pfb_csv
