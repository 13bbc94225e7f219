// Input readers: the point and mesh formats the reference's viewer reads
// (viewer/mesh_io.h:26-60, implemented in viewer/mesh_io.cpp) - Wavefront OBJ,
// OFF, ASCII and binary little-endian PLY, ASCII and binary STL, "x y z" text -
// plus weld and drop_non_finite, the "x y z" stream reader of
// examples/simple.cpp:17-23, and a loader that reads many files on host threads
// straight into the back-to-back layout of a batched build.
//
// A file is read into memory in one call and parsed in place by a cursor that
// applies the extraction rules of a C++ input stream in the "C" locale (what
// the reference's readers use): whitespace is ' ', \t, \n, \v, \f, \r; a
// number is an optional sign, digits with at most one decimal point and an
// exponent only after a digit, converted with correct rounding and rejected
// when incomplete ("1e", "."), on overflow, or when it starts with neither a
// sign, a digit nor a point ("nan" and "inf" are not numbers); a failed
// extraction leaves the cursor failed, so every later read fails too.  The
// vertices, faces and error texts are then the reference's for the same bytes.
//
// Deliberate differences, where the reference's behaviour is undefined, a
// crash or a near-endless loop: a NaN coordinate never merges in weld (the
// reference orders vertices with operator<, which NaN breaks); element counts
// in headers reserve no memory up front, so a corrupt count cannot abort the
// process; a binary PLY element without properties is skipped instead of
// walking its claimed item count (its items occupy no bytes).
#include "../../include/del3d_b200.h"
#include "../../include/del3d/mesh_io.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <charconv>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <string_view>
#include <thread>
#include <new>
#include <unordered_map>
#include <vector>

#include <sys/stat.h>

namespace d3g {
void set_error(const std::string& msg);
void* host_result_alloc(size_t bytes);
void host_result_free(void* p);
}  // namespace d3g

namespace {

using std::string_view;

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }
bool is_digit(char c) { return c >= '0' && c <= '9'; }

std::string lower(string_view s) {
    std::string r(s);
    for (char& c : r)
        if (c >= 'A' && c <= 'Z') c = char(c - 'A' + 'a');
    return r;
}

/// Decimal digits to a long as strtol does (base 10): optional sign, saturating
/// at LONG_MAX / LONG_MIN; `any` tells whether there was a digit.
long digits_to_long(const char*& p, const char* e, bool& any, bool& overflow) {
    bool neg = false;
    if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
    const unsigned long long lim = neg ? 9223372036854775808ull : 9223372036854775807ull;
    unsigned long long acc = 0;
    any = overflow = false;
    for (; p < e && is_digit(*p); ++p) {
        any = true;
        if (!overflow) {
            const unsigned d = unsigned(*p - '0');
            if (acc > (lim - d) / 10) overflow = true;
            else acc = acc * 10 + d;
        }
    }
    if (!any) return 0;
    if (overflow) return neg ? LONG_MIN : LONG_MAX;
    return neg ? (acc == 9223372036854775808ull ? LONG_MIN : -(long)acc) : (long)acc;
}

/// strtol(token, nullptr, 10) for a token without whitespace.
long token_to_long(string_view t) {
    const char* p = t.data();
    bool any, over;
    return digits_to_long(p, t.data() + t.size(), any, over);
}

/// A read position in a byte range with an input stream's fail state.
class Cursor {
public:
    Cursor() = default;
    explicit Cursor(string_view s) { reset(s); }
    void reset(string_view s) {
        b_ = p_ = s.data();
        e_ = s.data() + s.size();
        failed_ = false;
    }
    bool good() const { return !failed_; }
    size_t size() const { return size_t(e_ - b_); }
    const char* base() const { return b_; }
    void seek(size_t off) {
        failed_ = false;
        p_ = b_ + std::min(off, size());
    }

    /// std::getline: up to '\n' (consumed, not returned); fails when nothing,
    /// not even a '\n', is left.
    bool line(string_view& out) {
        if (failed_ || p_ >= e_) return fail();
        const char* nl = static_cast<const char*>(std::memchr(p_, '\n', size_t(e_ - p_)));
        const char* end = nl ? nl : e_;
        out = string_view(p_, size_t(end - p_));
        p_ = nl ? nl + 1 : e_;
        return true;
    }

    /// `>> std::string`.
    bool word(string_view& out) {
        if (!skip()) return false;
        const char* s = p_;
        while (p_ < e_ && !is_space(*p_)) ++p_;
        out = string_view(s, size_t(p_ - s));
        return true;
    }

    /// `>> double`.  On a malformed number the value becomes 0, on overflow
    /// +-DBL_MAX, and the cursor fails; at the end it fails with `v` unchanged.
    bool number(double& v) {
        if (!skip()) return false;
        const char* s = p_;
        if (*p_ == '+' || *p_ == '-') ++p_;
        bool mant = false, point = false, expo = false;
        while (p_ < e_) {
            const char c = *p_;
            if (is_digit(c)) {
                if (!expo) mant = true;
                ++p_;
            } else if (c == '.' && !point && !expo) {
                point = true;
                ++p_;
            } else if ((c == 'e' || c == 'E') && !expo && mant) {
                expo = true;
                ++p_;
                if (p_ < e_ && (*p_ == '+' || *p_ == '-')) ++p_;
            } else {
                break;
            }
        }
        const char* t = s + (s < p_ && *s == '+' ? 1 : 0);
        double r = 0.0;
        const auto res = std::from_chars(t, p_, r, std::chars_format::general);
        if (res.ec == std::errc() && res.ptr == p_ && (t == s || (*t != '-' && *t != '+'))) {
            v = r;
            return true;
        }
        if (res.ec == std::errc::result_out_of_range && res.ptr == p_) {
            // Overflow fails; underflow gives what strtod gives (0 or a subnormal).
            const std::string tok(s, p_);
            const double d = std::strtod(tok.c_str(), nullptr);
            if (std::isinf(d)) {
                v = d > 0 ? DBL_MAX : -DBL_MAX;
                return fail();
            }
            v = d;
            return true;
        }
        v = 0.0;
        return fail();
    }

    /// `>> long`: value 0 without digits, LONG_MAX / LONG_MIN on overflow, both failing.
    bool number(long& v) {
        if (!skip()) return false;
        bool any, over;
        v = digits_to_long(p_, e_, any, over);
        if (!any || over) return fail();
        return true;
    }

    /// istream::read.
    bool bytes(void* dst, size_t n) {
        if (failed_) return false;
        if (size_t(e_ - p_) < n) {
            p_ = e_;
            return fail();
        }
        std::memcpy(dst, p_, n);
        p_ += n;
        return true;
    }

private:
    bool fail() {
        failed_ = true;
        return false;
    }
    /// The sentry of a formatted extraction: skips whitespace, fails at the end.
    bool skip() {
        if (failed_) return false;
        while (p_ < e_ && is_space(*p_)) ++p_;
        if (p_ >= e_) return fail();
        return true;
    }

    const char* b_ = nullptr;
    const char* p_ = nullptr;
    const char* e_ = nullptr;
    bool failed_ = false;
};

struct Mesh {
    std::vector<double> v;      // x y z per vertex
    std::vector<int32_t> f;     // 3 indices per face
    size_t nv() const { return v.size() / 3; }
    void vertex(double x, double y, double z) {
        v.push_back(x);
        v.push_back(y);
        v.push_back(z);
    }
    void face(int a, int b, int c) {
        f.push_back(a);
        f.push_back(b);
        f.push_back(c);
    }
    /// A polygon as a fan of triangles from its first corner.
    void polygon(const std::vector<int>& p) {
        for (size_t k = 2; k < p.size(); ++k) face(p[0], p[k - 1], p[k]);
    }
};

// ---- OBJ (viewer/mesh_io.cpp:42-71) ------------------------------------------------

void read_obj(Cursor& in, Mesh& m, std::string& err) {
    string_view ln, tag, tok;
    std::vector<int> poly;
    Cursor ls;
    while (in.line(ln)) {
        if (ln.empty() || ln[0] == '#') continue;
        ls.reset(ln);
        if (!ls.word(tag)) continue;
        if (tag == "v") {
            double x, y, z;
            if (ls.number(x) && ls.number(y) && ls.number(z)) m.vertex(x, y, z);
        } else if (tag == "f") {
            poly.clear();
            while (ls.word(tok)) {
                const size_t slash = tok.find('/');       // v, v/vt, v//vn, v/vt/vn
                if (slash != string_view::npos) tok = tok.substr(0, slash);
                if (tok.empty()) continue;
                long idx = token_to_long(tok);
                idx = idx < 0 ? long(m.nv()) + idx : idx - 1;   // relative or 1-based
                if (idx >= 0 && idx < long(m.nv())) poly.push_back(int(idx));
            }
            if (poly.size() >= 3) m.polygon(poly);
        }
    }
    if (m.v.empty()) err = "no vertices in the OBJ";
}

// ---- OFF (viewer/mesh_io.cpp:76-134) -----------------------------------------------

void read_off(Cursor& in, Mesh& m, std::string& err) {
    Cursor ls;
    // The next line with something on it, comments ('#' to the end) removed.
    auto next_tokens = [&in, &ls]() -> bool {
        string_view ln;
        while (in.line(ln)) {
            const size_t hash = ln.find('#');
            if (hash != string_view::npos) ln = ln.substr(0, hash);
            if (ln.find_first_not_of(" \t\r\n") == string_view::npos) continue;
            ls.reset(ln);
            return true;
        }
        return false;
    };
    if (!next_tokens()) {
        err = "empty OFF";
        return;
    }
    string_view magic;
    if (!ls.word(magic)) magic = string_view();
    if (lower(magic).find("off") == std::string::npos) {
        err = "not an OFF file";
        return;
    }
    long nv = 0, nf = 0, ne = 0;
    if (!(ls.number(nv) && ls.number(nf) && ls.number(ne))) {   // or on the next line
        if (!next_tokens() || !(ls.number(nv) && ls.number(nf) && ls.number(ne))) {
            err = "malformed OFF header";
            return;
        }
    }
    string_view rest;
    for (long i = 0; i < nv; ++i) {
        double x, y, z;
        if (!(in.number(x) && in.number(y) && in.number(z))) {
            err = "OFF ended inside the vertex list";
            return;
        }
        m.vertex(x, y, z);
        in.line(rest);                                  // colour or normal
    }
    std::vector<int> poly;
    for (long i = 0; i < nf; ++i) {
        long n = 0;
        if (!in.number(n)) break;
        poly.clear();
        for (long k = 0; k < n; ++k) {
            long idx = 0;
            if (!in.number(idx)) break;
            if (idx >= 0 && idx < long(m.nv())) poly.push_back(int(idx));
        }
        if (poly.size() >= 3) m.polygon(poly);
        in.line(rest);                                  // colour
    }
}

// ---- PLY (viewer/mesh_io.cpp:139-315) ----------------------------------------------

/// A PLY scalar type: bytes (0 if the name is unknown), float, signed.
struct PlyType {
    int size = 0;
    bool flt = false, sgn = false;
};

struct PlyProp {
    std::string name, type, count_type;   // type: scalar type or a list's item type
    bool list = false;
    PlyType t, ct;                        // resolved once the header is read
};

struct PlyElement {
    std::string name;
    long count = 0;
    std::vector<PlyProp> props;
};

/// The PLY scalar type named `t`.
PlyType ply_type(const std::string& t) {
    struct T {
        const char* name;
        int size;
        bool flt, sgn;
    };
    static const T table[] = {{"char", 1, false, true},    {"int8", 1, false, true},   {"uchar", 1, false, false},
                              {"uint8", 1, false, false},  {"short", 2, false, true},  {"int16", 2, false, true},
                              {"ushort", 2, false, false}, {"uint16", 2, false, false}, {"int", 4, false, true},
                              {"int32", 4, false, true},   {"uint", 4, false, false},  {"uint32", 4, false, false},
                              {"float", 4, true, false},   {"float32", 4, true, false}, {"double", 8, true, false},
                              {"float64", 8, true, false}};
    PlyType r;
    for (const T& e : table)
        if (t == e.name) {
            r.size = e.size;
            r.flt = e.flt;
            r.sgn = e.sgn;
        }
    return r;
}

/// One little-endian binary value of type `t`, widened to double.
bool ply_binary(Cursor& in, const PlyType& t, double& out) {
    const int n = t.size;
    unsigned char b[8];
    if (n == 0 || !in.bytes(b, size_t(n))) return false;
    uint64_t raw = 0;
    for (int i = n - 1; i >= 0; --i) raw = (raw << 8) | b[i];
    if (t.flt && n == 4) {
        const uint32_t r = uint32_t(raw);
        float f;
        std::memcpy(&f, &r, 4);
        out = double(f);
    } else if (t.flt) {
        std::memcpy(&out, &raw, 8);
    } else if (t.sgn) {
        const int sh = 64 - 8 * n;
        out = double(int64_t(raw << sh) >> sh);
    } else {
        out = double(raw);
    }
    return true;
}

/// A list count or face index read as a double, converted as x86-64 converts
/// an out-of-range double (to the most negative value).
long to_long(double d) { return (d >= -9223372036854775808.0 && d < 9223372036854775808.0) ? long(d) : LONG_MIN; }
int to_int(double d) { return (d > -2147483649.0 && d < 2147483648.0) ? int(d) : INT_MIN; }

void read_ply(Cursor& in, Mesh& m, std::string& err) {
    string_view ln;
    if (!in.line(ln) || lower(ln.substr(0, 3)) != "ply") {
        err = "not a PLY file";
        return;
    }
    std::string format = "ascii";
    std::vector<PlyElement> elements;
    Cursor ls;
    string_view w;
    while (in.line(ln)) {
        if (!ln.empty() && ln.back() == '\r') ln.remove_suffix(1);
        ls.reset(ln);
        string_view tag;
        if (!ls.word(tag)) tag = string_view();
        if (tag == "comment" || tag == "obj_info") continue;
        if (tag == "format") {
            if (ls.word(w)) format = std::string(w);
            continue;
        }
        if (tag == "element") {
            PlyElement e;
            if (ls.word(w)) {
                e.name = std::string(w);
                ls.number(e.count);
            }
            elements.push_back(std::move(e));
            continue;
        }
        if (tag == "property") {
            if (elements.empty()) continue;
            PlyProp p;
            string_view t;
            if (!ls.word(t)) t = string_view();
            if (t == "list") {
                p.list = true;
                if (ls.word(w)) p.count_type = std::string(w);
                if (ls.word(w)) p.type = std::string(w);
                if (ls.word(w)) p.name = std::string(w);
            } else {
                p.type = std::string(t);
                if (ls.word(w)) p.name = std::string(w);
            }
            elements.back().props.push_back(std::move(p));
            continue;
        }
        if (tag == "end_header") break;
    }
    if (format != "ascii" && format != "binary_little_endian") {
        err = "unsupported PLY format '" + format + "' (ascii and binary_little_endian are read)";
        return;
    }
    const bool ascii = format == "ascii";
    for (PlyElement& e : elements)
        for (PlyProp& p : e.props) {
            p.t = ply_type(p.type);
            p.ct = ply_type(p.count_type);
        }
    std::vector<double> scalars;
    std::vector<int> poly, clean;
    Cursor as;
    for (const PlyElement& e : elements) {
        const bool is_vertex = e.name == "vertex", is_face = e.name == "face";
        int ix = -1, iy = -1, iz = -1;
        for (size_t i = 0; i < e.props.size(); ++i) {
            if (e.props[i].name == "x") ix = int(i);
            if (e.props[i].name == "y") iy = int(i);
            if (e.props[i].name == "z") iz = int(i);
        }
        if (is_vertex && (ix < 0 || iy < 0 || iz < 0)) {
            err = "PLY vertex element has no x/y/z";
            return;
        }
        // A binary element without properties occupies no bytes: its items change
        // nothing, however many the header claims (the reference walks them all).
        if (!ascii && e.props.empty()) continue;
        for (long n = 0; n < e.count; ++n) {
            scalars.assign(e.props.size(), 0.0);
            poly.clear();
            if (ascii) {
                if (!in.line(ln)) {
                    err = "PLY ended early";
                    return;
                }
                as.reset(ln);
            }
            for (size_t p = 0; p < e.props.size(); ++p) {
                const PlyProp& pr = e.props[p];
                if (pr.list) {
                    double cnt = 0;
                    if (ascii) {
                        if (!as.number(cnt)) break;
                    } else if (!ply_binary(in, pr.ct, cnt)) {
                        err = "PLY ended inside a list";
                        return;
                    }
                    const long c = to_long(cnt);
                    for (long k = 0; k < c; ++k) {
                        double v = 0;
                        if (ascii) {
                            if (!as.number(v)) break;
                        } else if (!ply_binary(in, pr.t, v)) {
                            err = "PLY ended inside a list";
                            return;
                        }
                        if (is_face) poly.push_back(to_int(v));
                    }
                } else {
                    double v = 0;
                    if (ascii) {
                        if (!as.number(v)) break;
                    } else if (!ply_binary(in, pr.t, v)) {
                        err = "PLY ended inside an element";
                        return;
                    }
                    scalars[p] = v;
                }
            }
            if (is_vertex) m.vertex(scalars[size_t(ix)], scalars[size_t(iy)], scalars[size_t(iz)]);
            if (is_face) {
                clean.clear();
                for (int idx : poly)
                    if (idx >= 0 && idx < int(m.nv())) clean.push_back(idx);
                if (clean.size() >= 3) m.polygon(clean);
            }
        }
    }
    if (m.v.empty() && err.empty()) err = "no vertices in the PLY";
}

// ---- STL (viewer/mesh_io.cpp:320-397) ----------------------------------------------

/// Binary unless the file starts with "solid" and its first 511 bytes hold
/// "facet"; when neither decides, binary iff the size is exactly 84 + 50 n.
bool stl_binary(const Cursor& in) {
    const size_t size = in.size();
    const std::string head = lower(string_view(in.base(), std::min<size_t>(size, 511)));
    if (head.compare(0, 5, "solid") != 0 || head.size() < 5) return true;
    if (head.find("facet") != std::string::npos) return false;
    if (size >= 84) {
        uint32_t n = 0;
        std::memcpy(&n, in.base() + 80, 4);
        if (uint64_t(84) + uint64_t(n) * 50 == size) return true;
    }
    return false;
}

void read_stl_binary(Cursor& in, Mesh& m, std::string& err) {
    in.seek(80);
    uint32_t n = 0;
    if (!in.bytes(&n, 4)) {
        err = "truncated STL header";
        return;
    }
    for (uint32_t i = 0; i < n; ++i) {
        float t[12];
        uint16_t attr = 0;
        if (!in.bytes(t, 48) || !in.bytes(&attr, 2)) break;   // a cut-off tail is dropped
        const int base = int(m.nv());
        for (int k = 1; k <= 3; ++k) m.vertex(double(t[3 * k]), double(t[3 * k + 1]), double(t[3 * k + 2]));
        m.face(base, base + 1, base + 2);
    }
    if (m.v.empty()) err = "no triangles in the STL";
}

void read_stl_ascii(Cursor& in, Mesh& m, std::string& err) {
    string_view ln, tag;
    Cursor ls;
    int corner[3], nc = 0;
    while (in.line(ln)) {
        ls.reset(ln);
        if (!ls.word(tag) || lower(tag) != "vertex") continue;
        double x, y, z;
        if (!(ls.number(x) && ls.number(y) && ls.number(z))) continue;
        corner[nc++] = int(m.nv());
        m.vertex(x, y, z);
        if (nc == 3) {
            m.face(corner[0], corner[1], corner[2]);
            nc = 0;
        }
    }
    if (m.v.empty()) err = "no vertices in the STL";
}

// ---- "x y z" text (viewer/mesh_io.cpp:402-413) -------------------------------------

void xyz_lines(string_view text, std::vector<double>& v) {
    Cursor in(text), ls;
    string_view ln;
    while (in.line(ln)) {
        if (ln.empty() || ln[0] == '#') continue;
        ls.reset(ln);
        double x, y, z;
        if (ls.number(x) && ls.number(y) && ls.number(z)) {
            v.push_back(x);
            v.push_back(y);
            v.push_back(z);
        }
    }
}

/// Lines are read independently, so a large file is cut at line starts into
/// one piece per thread and the pieces' points are joined in order: the same
/// points as one pass.
void read_xyz_lines(string_view text, Mesh& m, std::string& err, int threads) {
    constexpr size_t kMinPiece = size_t(2) << 20;
    const int nt = int(std::min<size_t>(size_t(std::max(threads, 1)), text.size() / kMinPiece + 1));
    if (nt <= 1) {
        xyz_lines(text, m.v);
    } else {
        std::vector<size_t> cut(size_t(nt) + 1, text.size());
        cut[0] = 0;
        for (int t = 1; t < nt; ++t) {
            size_t pos = std::max(cut[size_t(t) - 1], text.size() / size_t(nt) * size_t(t));
            const size_t nl = text.find('\n', pos);
            cut[size_t(t)] = nl == string_view::npos ? text.size() : nl + 1;
        }
        std::vector<std::vector<double>> part(static_cast<size_t>(nt));
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t)
            pool.emplace_back([&, t] { xyz_lines(text.substr(cut[size_t(t)], cut[size_t(t) + 1] - cut[size_t(t)]), part[size_t(t)]); });
        xyz_lines(text.substr(0, cut[1]), part[0]);
        for (std::thread& th : pool) th.join();
        size_t total = 0;
        for (const auto& p : part) total += p.size();
        m.v.reserve(total);
        for (const auto& p : part) m.v.insert(m.v.end(), p.begin(), p.end());
    }
    if (m.v.empty()) err = "no points in the file";
}

// ---- weld / drop_non_finite (viewer/mesh_io.cpp:417-478) ---------------------------

struct CoordKey {
    double x, y, z;
    bool operator==(const CoordKey& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct CoordHash {
    size_t operator()(const CoordKey& k) const {
        auto bits = [](double d) {
            uint64_t u;
            d = d == 0.0 ? 0.0 : d;                    // -0.0 and 0.0 are one vertex
            std::memcpy(&u, &d, 8);
            return u;
        };
        uint64_t h = bits(k.x) * 0x9E3779B97F4A7C15ull;
        h ^= bits(k.y) + 0x7F4A7C159E3779B9ull + (h << 6) + (h >> 2);
        h ^= bits(k.z) + 0x94D049BB133111EBull + (h << 6) + (h >> 2);
        return size_t(h ^ (h >> 31));
    }
};

/// Merges vertices with equal coordinates (first occurrence kept, faces
/// remapped, faces whose corners merged dropped); nothing changes when no two
/// vertices are equal.  Works in place; returns the new counts.
void weld_arrays(double* v, int64_t& nv, int32_t* f, int64_t& nf) {
    std::unordered_map<CoordKey, int32_t, CoordHash> seen;
    seen.reserve(size_t(nv));
    std::vector<int32_t> remap(static_cast<size_t>(nv));
    int64_t nu = 0;
    for (int64_t i = 0; i < nv; ++i) {
        const CoordKey k{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
        const bool has_nan = std::isnan(k.x) || std::isnan(k.y) || std::isnan(k.z);
        auto it = has_nan ? seen.end() : seen.find(k);
        if (it != seen.end()) {
            remap[size_t(i)] = it->second;
        } else {
            remap[size_t(i)] = int32_t(nu);
            if (!has_nan) seen.emplace(k, int32_t(nu));
            if (nu != i) {
                v[3 * nu] = k.x;
                v[3 * nu + 1] = k.y;
                v[3 * nu + 2] = k.z;
            }
            ++nu;
        }
    }
    if (nu == nv) return;
    int64_t kept = 0;
    for (int64_t j = 0; j < nf; ++j) {
        const int32_t a = remap[size_t(f[3 * j])], b = remap[size_t(f[3 * j + 1])], c = remap[size_t(f[3 * j + 2])];
        if (a == b || b == c || a == c) continue;
        f[3 * kept] = a;
        f[3 * kept + 1] = b;
        f[3 * kept + 2] = c;
        ++kept;
    }
    nv = nu;
    nf = kept;
}

/// Removes vertices with a non-finite coordinate and the faces touching them;
/// in place; returns how many vertices went.
int64_t drop_non_finite_arrays(double* v, int64_t& nv, int32_t* f, int64_t& nf) {
    std::vector<int32_t> remap(size_t(nv), -1);
    int64_t kept = 0;
    for (int64_t i = 0; i < nv; ++i) {
        const double x = v[3 * i], y = v[3 * i + 1], z = v[3 * i + 2];
        if (!(std::isfinite(x) && std::isfinite(y) && std::isfinite(z))) continue;
        remap[size_t(i)] = int32_t(kept);
        v[3 * kept] = x;
        v[3 * kept + 1] = y;
        v[3 * kept + 2] = z;
        ++kept;
    }
    const int64_t dropped = nv - kept;
    if (dropped == 0) return 0;
    int64_t kf = 0;
    for (int64_t j = 0; j < nf; ++j) {
        const int32_t a = remap[size_t(f[3 * j])], b = remap[size_t(f[3 * j + 1])], c = remap[size_t(f[3 * j + 2])];
        if (a < 0 || b < 0 || c < 0) continue;
        f[3 * kf] = a;
        f[3 * kf + 1] = b;
        f[3 * kf + 2] = c;
        ++kf;
    }
    nv = kept;
    nf = kf;
    return dropped;
}

// ---- files -------------------------------------------------------------------------

bool read_file(const char* path, std::vector<char>& buf) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return false;
    buf.clear();
    // A regular file in one read of its size, then whatever follows (a file
    // that grew meanwhile); anything else in chunks.
    struct stat st;
    if (fstat(fileno(fp), &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0) {
        buf.resize(size_t(st.st_size));
        buf.resize(std::fread(buf.data(), 1, buf.size(), fp));
    }
    char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof chunk, fp)) > 0) buf.insert(buf.end(), chunk, chunk + got);
    std::fclose(fp);
    return true;
}

std::string extension(const std::string& path) {
    const size_t dot = path.find_last_of('.');
    const size_t sep = path.find_last_of("/\\");
    if (dot == std::string::npos || (sep != std::string::npos && dot < sep)) return "";
    return lower(string_view(path).substr(dot));
}

const char* kFormats = "obj, off, ply, stl, xyz";

int host_threads() { return int(std::max(1u, std::thread::hardware_concurrency())); }

/// meshio::load: the reader by extension; `err` empty on success.  `threads`
/// parse a large "x y z" text file in pieces (the other formats are read in
/// one pass: their items depend on what came before).
void load_mesh(const std::string& path, Mesh& m, std::string& err, int threads) {
    err.clear();
    std::vector<char> buf;
    if (!read_file(path.c_str(), buf)) {
        err = "cannot open " + path;
        return;
    }
    Cursor in(string_view(buf.data(), buf.size()));
    const std::string ext = extension(path);
    if (ext == ".obj") {
        read_obj(in, m, err);
    } else if (ext == ".off") {
        read_off(in, m, err);
    } else if (ext == ".ply") {
        read_ply(in, m, err);
    } else if (ext == ".stl") {
        if (stl_binary(in)) read_stl_binary(in, m, err);
        else read_stl_ascii(in, m, err);
        int64_t nv = int64_t(m.nv()), nf = int64_t(m.f.size() / 3);
        weld_arrays(m.v.data(), nv, m.f.data(), nf);   // STL repeats every corner
        m.v.resize(size_t(nv) * 3);
        m.f.resize(size_t(nf) * 3);
    } else if (ext == ".xyz" || ext == ".txt" || ext == ".pts" || ext.empty()) {
        read_xyz_lines(string_view(buf.data(), buf.size()), m, err, threads);
    } else {
        err = "unknown extension '" + ext + "' (" + kFormats + ")";
    }
}

int fill_mesh(Mesh& m, d3g_mesh* out) {
    out->n_vertices = int64_t(m.nv());
    out->n_faces = int64_t(m.f.size() / 3);
    out->vertices = static_cast<double*>(std::malloc(std::max<size_t>(m.v.size(), 1) * sizeof(double)));
    out->faces = static_cast<int32_t*>(std::malloc(std::max<size_t>(m.f.size(), 1) * sizeof(int32_t)));
    if (!out->vertices || !out->faces) {
        std::free(out->vertices);
        std::free(out->faces);
        *out = d3g_mesh{};
        d3g::set_error("d3g_mesh_load: out of host memory");
        return D3G_ERR_OOM;
    }
    if (!m.v.empty()) std::memcpy(out->vertices, m.v.data(), m.v.size() * sizeof(double));
    if (!m.f.empty()) std::memcpy(out->faces, m.f.data(), m.f.size() * sizeof(int32_t));
    return D3G_OK;
}

}  // namespace

// ---- the reference's viewer interface (viewer/mesh_io.h) ---------------------------

namespace meshio {

Mesh load(const std::string& path, std::string& error) {
    ::Mesh m;
    load_mesh(path, m, error, host_threads());
    Mesh r;
    r.vertices.resize(m.nv());
    if (!m.v.empty()) std::memcpy(r.vertices.data(), m.v.data(), m.v.size() * sizeof(double));
    r.faces.resize(m.f.size() / 3);
    if (!m.f.empty()) std::memcpy(r.faces.data(), m.f.data(), m.f.size() * sizeof(int32_t));
    return r;
}

void weld(Mesh& m) {
    int64_t nv = int64_t(m.vertices.size()), nf = int64_t(m.faces.size());
    weld_arrays(m.vertices.empty() ? nullptr : m.vertices[0].data(), nv,
                m.faces.empty() ? nullptr : m.faces[0].data(), nf);
    m.vertices.resize(size_t(nv));
    m.faces.resize(size_t(nf));
}

std::size_t drop_non_finite(Mesh& m) {
    int64_t nv = int64_t(m.vertices.size()), nf = int64_t(m.faces.size());
    const int64_t dropped = drop_non_finite_arrays(m.vertices.empty() ? nullptr : m.vertices[0].data(), nv,
                                                   m.faces.empty() ? nullptr : m.faces[0].data(), nf);
    m.vertices.resize(size_t(nv));
    m.faces.resize(size_t(nf));
    return std::size_t(dropped);
}

const char* supported_formats() { return kFormats; }

}  // namespace meshio

// ---- C ABI -------------------------------------------------------------------------

/// Runs a C entry point's body; a C++ exception (out of memory) becomes a status.
template <class F>
int guarded(const char* where, F&& body) {
    try {
        return body();
    } catch (const std::bad_alloc&) {
        d3g::set_error(std::string(where) + ": out of host memory");
        return D3G_ERR_OOM;
    } catch (const std::exception& e) {
        d3g::set_error(std::string(where) + ": " + e.what());
        return D3G_ERR_INTERNAL;
    }
}

extern "C" {

static int d3g_mesh_load_impl(const char* path, d3g_mesh* out) {
    if (!path || !out) {
        d3g::set_error("d3g_mesh_load: null argument");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    *out = d3g_mesh{};
    Mesh m;
    std::string err;
    load_mesh(path, m, err, host_threads());
    const int st = fill_mesh(m, out);
    if (st != D3G_OK) return st;
    if (!err.empty()) {
        d3g::set_error(err);
        return D3G_ERR_INVALID_INPUT;
    }
    return D3G_OK;
}

static int d3g_read_xyz_impl(const char* path, d3g_mesh* out) {
    if (!path || !out) {
        d3g::set_error("d3g_read_xyz: null argument");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    *out = d3g_mesh{};
    std::vector<char> buf;
    if (!read_file(path, buf)) {
        d3g::set_error(std::string("cannot open ") + path);
        return D3G_ERR_INVALID_INPUT;
    }
    // examples/simple.cpp:17-23: triples until the first that does not parse
    Mesh m;
    Cursor in(string_view(buf.data(), buf.size()));
    double x, y, z;
    while (in.number(x) && in.number(y) && in.number(z)) m.vertex(x, y, z);
    return fill_mesh(m, out);
}

static int d3g_mesh_weld_impl(d3g_mesh* m) {
    if (!m || (m->n_vertices > 0 && !m->vertices) || (m->n_faces > 0 && !m->faces) || m->n_vertices < 0 ||
        m->n_faces < 0) {
        d3g::set_error("d3g_mesh_weld: bad mesh");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    for (int64_t i = 0; i < 3 * m->n_faces; ++i)
        if (m->faces[i] < 0 || m->faces[i] >= m->n_vertices) {
            d3g::set_error("d3g_mesh_weld: face index out of range");
            return D3G_ERR_INVALID_INPUT;
        }
    weld_arrays(m->vertices, m->n_vertices, m->faces, m->n_faces);
    return D3G_OK;
}

static int d3g_mesh_drop_non_finite_impl(d3g_mesh* m, int64_t* dropped) {
    if (!m || (m->n_vertices > 0 && !m->vertices) || (m->n_faces > 0 && !m->faces) || m->n_vertices < 0 ||
        m->n_faces < 0) {
        d3g::set_error("d3g_mesh_drop_non_finite: bad mesh");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    for (int64_t i = 0; i < 3 * m->n_faces; ++i)
        if (m->faces[i] < 0 || m->faces[i] >= m->n_vertices) {
            d3g::set_error("d3g_mesh_drop_non_finite: face index out of range");
            return D3G_ERR_INVALID_INPUT;
        }
    const int64_t d = drop_non_finite_arrays(m->vertices, m->n_vertices, m->faces, m->n_faces);
    if (dropped) *dropped = d;
    return D3G_OK;
}

void d3g_mesh_free(d3g_mesh* m) {
    if (!m) return;
    std::free(m->vertices);
    std::free(m->faces);
    *m = d3g_mesh{};
}

const char* d3g_mesh_supported_formats(void) { return kFormats; }

static int d3g_load_point_sets_impl(const char* const* paths, int n_paths, int threads, d3g_point_sets* out) {
    if (!out || n_paths < 0 || (n_paths > 0 && !paths)) {
        d3g::set_error("d3g_load_point_sets: bad argument");
        return D3G_ERR_INVALID_ARGUMENT;
    }
    *out = d3g_point_sets{};
    for (int i = 0; i < n_paths; ++i)
        if (!paths[i]) {
            d3g::set_error("d3g_load_point_sets: null path");
            return D3G_ERR_INVALID_ARGUMENT;
        }
    // Every file is parsed on a worker thread into its own buffer; then the
    // vertices are packed back to back into pinned host memory, ready for
    // d3g_build_batch or a host-to-device copy at full rate.
    std::vector<Mesh> meshes(static_cast<size_t>(n_paths));
    std::vector<std::string> errs(static_cast<size_t>(n_paths));
    std::vector<int64_t> dropped(size_t(n_paths), 0);
    const int want = threads > 0 ? threads : host_threads();
    const int nt = std::max(1, std::min(n_paths, want));
    const int per_file = std::max(1, want / std::max(n_paths, 1));   // few large files: split them too
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int i; (i = next.fetch_add(1)) < n_paths;) {
            Mesh& m = meshes[size_t(i)];
            try {
                load_mesh(paths[i], m, errs[size_t(i)], per_file);
                m.f.clear();
                int64_t nv = int64_t(m.nv()), nf = 0;
                dropped[size_t(i)] = drop_non_finite_arrays(m.v.data(), nv, nullptr, nf);
                m.v.resize(size_t(nv) * 3);
            } catch (const std::bad_alloc&) {
                m = Mesh();
                errs[size_t(i)] = "out of host memory";
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (std::thread& t : pool) t.join();
    for (int i = 0; i < n_paths; ++i)
        if (!errs[size_t(i)].empty()) {
            d3g::set_error(std::string(paths[i]) + ": " + errs[size_t(i)]);
            return D3G_ERR_INVALID_INPUT;
        }
    int64_t total = 0;
    for (const Mesh& m : meshes) total += int64_t(m.nv());
    out->xyz = static_cast<double*>(d3g::host_result_alloc(size_t(std::max<int64_t>(total, 1)) * 3 * sizeof(double)));
    out->set_offsets = static_cast<int64_t*>(std::malloc((size_t(n_paths) + 1) * sizeof(int64_t)));
    out->dropped = static_cast<int64_t*>(std::malloc(std::max<size_t>(size_t(n_paths), 1) * sizeof(int64_t)));
    if (!out->xyz || !out->set_offsets || !out->dropped) {
        d3g_point_sets_free(out);
        d3g::set_error("d3g_load_point_sets: out of host memory");
        return D3G_ERR_OOM;
    }
    int64_t off = 0;
    for (int i = 0; i < n_paths; ++i) {
        const Mesh& m = meshes[size_t(i)];
        out->set_offsets[i] = off;
        out->dropped[i] = dropped[size_t(i)];
        if (!m.v.empty()) std::memcpy(out->xyz + 3 * off, m.v.data(), m.v.size() * sizeof(double));
        off += int64_t(m.nv());
    }
    out->set_offsets[n_paths] = off;
    out->n_sets = n_paths;
    return D3G_OK;
}

void d3g_point_sets_free(d3g_point_sets* s) {
    if (!s) return;
    d3g::host_result_free(s->xyz);
    std::free(s->set_offsets);
    std::free(s->dropped);
    *s = d3g_point_sets{};
}

int d3g_mesh_load(const char* path, d3g_mesh* out) {
    return guarded("d3g_mesh_load", [&] { return d3g_mesh_load_impl(path, out); });
}

int d3g_read_xyz(const char* path, d3g_mesh* out) {
    return guarded("d3g_read_xyz", [&] { return d3g_read_xyz_impl(path, out); });
}

int d3g_mesh_weld(d3g_mesh* m) {
    return guarded("d3g_mesh_weld", [&] { return d3g_mesh_weld_impl(m); });
}

int d3g_mesh_drop_non_finite(d3g_mesh* m, int64_t* dropped) {
    return guarded("d3g_mesh_drop_non_finite", [&] { return d3g_mesh_drop_non_finite_impl(m, dropped); });
}

int d3g_load_point_sets(const char* const* paths, int n_paths, int threads, d3g_point_sets* out) {
    return guarded("d3g_load_point_sets", [&] { return d3g_load_point_sets_impl(paths, n_paths, threads, out); });
}

}  // extern "C"
