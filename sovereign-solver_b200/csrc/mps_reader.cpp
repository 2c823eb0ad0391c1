// mps_reader.cpp -- the MPS reader behind pdhg_read_mps / pdhg_read_mps_file.
//
// It reads the dialect of sov::read_mps_string (src/io/mps_reader.cpp:1-574,
// include/sovereign/io.hpp:14-66) and builds the same model: the same rows
// and columns in the same order, the same CSR (Problem::Builder::finish,
// src/io/problem.cpp:174-200, through CsrMatrix::from_triplets,
// src/l0/sparse.cpp:30-70: duplicates summed in file order, columns ascending,
// |sum| <= 1e-14 dropped), the same bounds, integrality, warnings (line,
// section, text) and error messages, the same fixed-column retry when the
// free-form read fails.
//
// It is laid out for models of tens of millions of nonzeros, where the
// reference's std::getline / per-token std::string / std::map of triplets
// dominate the time to the first iteration:
//   - the whole text is one buffer; threads over byte ranges find the section
//     header lines and count lines (for line numbers in messages);
//   - tokens are string_views, names live in two arenas with open-addressing
//     indexes, numbers go through std::from_chars (correctly rounded, like
//     glibc's strtod; anything it does not take whole falls back to strtod);
//   - COLUMNS data cards, nearly all of a file, are parsed by threads over
//     line-aligned chunks into chunk-local columns and triplets, then merged
//     in file order: new columns take their indices in order of first
//     appearance, objective coefficients are set in order (the last wins), the
//     integer markers' state is carried from chunk to chunk; the first error
//     in file order is the one reported;
//   - triplets become CSR through a stable counting sort by row (threads over
//     triplet ranges), then each row is ordered by column and its duplicates
//     summed in file order (threads over rows).
// Every other section runs card by card in file order, as in the reference.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <limits>
#include <memory>
#include <new>
#include <string>
#include <string_view>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/pdhg_b200.h"

namespace pdhg {
namespace mps {
namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr double kNumericZero = 1e-14;  // tol::numeric_zero (numeric.hpp:95)

// An error of the reference reader: sov::Error's message.
struct ReadError {
    std::string what;
};

// std::vector storage whose resize() leaves new elements of a trivial type
// uninitialised: the large arrays below are written in full by threads right
// after sizing, and zero-filling them first would be a serial pass over
// hundreds of MB.
template <class T>
struct NoInit : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInit<U>;
    };
    NoInit() = default;
    template <class U>
    NoInit(const NoInit<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... args) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(args)...);
    }
};
template <class T>
using bigvec = std::vector<T, NoInit<T>>;

// With PDHG_B200_PHASE_TIMES=1 in the environment, each phase's wall time on
// stderr.
struct HostClock {
    bool on;
    std::chrono::steady_clock::time_point t;
    HostClock() : t(std::chrono::steady_clock::now()) {
        const char* e = std::getenv("PDHG_B200_PHASE_TIMES");
        on = e != nullptr && e[0] != '\0' && e[0] != '0';
    }
    void mark(const char* what) {
        if (!on) return;
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[mps phase] %-22s %10.3f ms\n", what,
                     std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

// ---- lexing -----------------------------------------------------------------

inline bool is_space(char c) {  // std::isspace in the "C" locale
    return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

inline char up(char c) { return (c >= 'a' && c <= 'z') ? static_cast<char>(c - 32) : c; }

// upper(token) == word (word given in upper case)
bool ieq(std::string_view t, std::string_view word) {
    if (t.size() != word.size()) return false;
    for (size_t i = 0; i < t.size(); ++i)
        if (up(t[i]) != word[i]) return false;
    return true;
}

// upper(token) with every quote removed == word (the integer-marker test,
// mps_reader.cpp:254-262); all three marker words have six letters.
bool marker_eq(std::string_view t, std::string_view word) {
    if (t.size() < word.size()) return false;
    size_t k = 0;
    for (char c : t) {
        if (c == '\'') continue;
        if (k >= word.size() || up(c) != word[k]) return false;
        ++k;
    }
    return k == word.size();
}

std::string upper_copy(std::string_view t) {
    std::string s(t);
    for (char& c : s) c = up(c);
    return s;
}

// Free form: split on whitespace.
void tokenize_free(std::string_view line, std::vector<std::string_view>& out) {
    out.clear();
    size_t i = 0;
    const size_t n = line.size();
    while (i < n) {
        while (i < n && is_space(line[i])) ++i;
        if (i >= n) break;
        const size_t s = i;
        while (i < n && !is_space(line[i])) ++i;
        out.emplace_back(line.data() + s, i - s);
    }
}

// Fixed columns 2-3, 5-12, 15-22, 25-36, 40-47, 50-61, each trimmed, empty
// fields dropped (mps_reader.cpp:67-83).
void tokenize_fixed(std::string_view line, std::vector<std::string_view>& out) {
    static constexpr size_t kBegin[6] = {1, 4, 14, 24, 39, 49};
    static constexpr size_t kLen[6] = {2, 8, 8, 12, 8, 12};
    out.clear();
    for (int f = 0; f < 6; ++f) {
        if (kBegin[f] >= line.size()) break;
        std::string_view piece = line.substr(kBegin[f], std::min(kLen[f], line.size() - kBegin[f]));
        size_t b = 0, e = piece.size();
        while (b < e && is_space(piece[b])) ++b;
        while (e > b && is_space(piece[e - 1])) --e;
        if (e > b) out.push_back(piece.substr(b, e - b));
    }
}

// parse_real (mps_reader.cpp:85-92): strtod over the whole token.
bool parse_real(std::string_view t, double* out) {
    if (t.empty()) return false;
    const char* b = t.data();
    const char* e = t.data() + t.size();
    const char* s = b;
    if (*s == '+' && t.size() > 1 && s[1] != '-' && s[1] != '+') ++s;  // strtod takes a '+'
    double v = 0.0;
    const auto r = std::from_chars(s, e, v, std::chars_format::general);
    if (r.ec == std::errc() && r.ptr == e) {
        *out = v;
        return true;
    }
    // hex, out of range, or not a number: let strtod decide, as the reference does
    char small[128];
    std::string big;
    const char* z = nullptr;
    if (t.size() < sizeof small) {
        std::memcpy(small, b, t.size());
        small[t.size()] = '\0';
        z = small;
    } else {
        big.assign(t);
        z = big.c_str();
    }
    char* end = nullptr;
    const double w = std::strtod(z, &end);
    if (end == z || *end != '\0') return false;
    *out = w;
    return true;
}

// infinite_token (mps_reader.cpp:95-113)
bool infinite_token(std::string_view t, double* out) {
    std::string_view u = t;
    bool negative = false;
    if (!u.empty() && (u[0] == '+' || u[0] == '-')) {
        negative = u[0] == '-';
        u.remove_prefix(1);
    }
    if (ieq(u, "INF") || ieq(u, "INFINITY")) {
        *out = negative ? -kInf : kInf;
        return true;
    }
    double v = 0.0;
    if (parse_real(t, &v) && std::abs(v) >= 1e30) {
        *out = v > 0 ? kInf : -kInf;
        return true;
    }
    return false;
}

// ---- names --------------------------------------------------------------------

inline uint64_t hash_name(std::string_view s) {
    uint64_t h = 0x9e3779b97f4a7c15ull ^ (s.size() * 0xff51afd7ed558ccdull);
    size_t i = 0;
    for (; i + 8 <= s.size(); i += 8) {
        uint64_t w;
        std::memcpy(&w, s.data() + i, 8);
        h = (h ^ w) * 0xff51afd7ed558ccdull;
        h ^= h >> 29;
    }
    uint64_t w = 0;
    for (size_t k = 0; i < s.size(); ++i, ++k) w |= static_cast<uint64_t>(static_cast<unsigned char>(s[i])) << (8 * k);
    h ^= w;
    // MurmurHash3's 64-bit finalizer, so that the low bits (the slot) depend
    // on every byte of the name
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    return h;
}

// Names, each stored NUL-terminated.
struct Arena {
    std::vector<char> chars;
    std::vector<int64_t> off{0};
    int32_t size() const { return static_cast<int32_t>(off.size() - 1); }
    std::string_view get(int32_t i) const {
        return std::string_view(chars.data() + off[i], static_cast<size_t>(off[i + 1] - off[i] - 1));
    }
    const char* c_str(int32_t i) const { return chars.data() + off[i]; }
    int32_t add(std::string_view s) {
        chars.insert(chars.end(), s.begin(), s.end());
        chars.push_back('\0');
        off.push_back(static_cast<int64_t>(chars.size()));
        return size() - 1;
    }
};

// Open addressing over an Arena's indices.
struct NameIndex {
    const Arena* names = nullptr;
    std::vector<int32_t> slot;
    uint64_t mask = 0;
    int32_t count = 0;

    explicit NameIndex(const Arena* a = nullptr, size_t expect = 16) : names(a) { reserve(expect); }
    void reserve(size_t expect) {
        size_t cap = 16;
        while (cap < 2 * expect) cap <<= 1;
        if (cap <= slot.size()) return;
        std::vector<int32_t> old = std::move(slot);
        slot.assign(cap, -1);
        mask = cap - 1;
        for (int32_t idx : old)
            if (idx >= 0) place(idx, hash_name(names->get(idx)));
    }
    void place(int32_t idx, uint64_t h) {
        uint64_t p = h & mask;
        while (slot[p] >= 0) p = (p + 1) & mask;
        slot[p] = idx;
    }
    int32_t find(std::string_view s, uint64_t h) const {
        uint64_t p = h & mask;
        for (;;) {
            const int32_t idx = slot[p];
            if (idx < 0) return -1;
            if (names->get(idx) == s) return idx;
            p = (p + 1) & mask;
        }
    }
    int32_t find(std::string_view s) const { return find(s, hash_name(s)); }
    void insert(int32_t idx, uint64_t h) {
        if (2 * static_cast<size_t>(count + 1) > slot.size()) reserve(static_cast<size_t>(count + 1) * 2);
        place(idx, h);
        ++count;
    }
};

struct Triplet {
    int32_t row, col;
    double v;
};

// ---- the model under construction (Problem::Builder) ---------------------------

struct Builder {
    std::string name, objective_name;
    bool maximize = false;
    double obj_const = 0.0;
    Arena row_names, col_names;
    NameIndex row_idx{&row_names}, col_idx{&col_names};
    std::vector<double> row_lo, row_hi, col_lo, col_hi, obj;
    std::vector<uint8_t> is_int;
    std::vector<char> row_sense;     // L G E N, by row
    std::vector<double> row_rhs;     // the last RHS value, by row
    bigvec<Triplet> entries;         // file order
    Arena dropped_names;             // free rows dropped (keep_free_rows = 0)
    NameIndex dropped_idx{&dropped_names};

    int32_t add_row(std::string_view nm, double lo, double hi) {  // problem.cpp:119-128
        const uint64_t h = hash_name(nm);
        if (row_idx.find(nm, h) >= 0) throw ReadError{"duplicate row name '" + std::string(nm) + "'"};
        const int32_t i = row_names.add(nm);
        row_idx.insert(i, h);
        row_lo.push_back(lo);
        row_hi.push_back(hi);
        return i;
    }
    int32_t add_column(std::string_view nm, uint64_t h) {  // problem.cpp:130-144
        const int32_t j = col_names.add(nm);
        col_idx.insert(j, h);
        col_lo.push_back(0.0);
        col_hi.push_back(kInf);
        is_int.push_back(0);
        obj.push_back(0.0);
        return j;
    }
    int32_t column_for(std::string_view nm) {
        const uint64_t h = hash_name(nm);
        const int32_t j = col_idx.find(nm, h);
        return j >= 0 ? j : add_column(nm, h);
    }
    bool dropped(std::string_view nm) const { return dropped_idx.count > 0 && dropped_idx.find(nm) >= 0; }
};

struct Warning {
    int64_t line;
    std::string section, message;
};

enum class Section { None, Name, ObjSense, Rows, Columns, Rhs, Ranges, Bounds, Ignored };

struct Header {
    size_t pos;      // first byte of the header line
    int64_t line;    // its 1-based line number
};

// ---- threads ------------------------------------------------------------------------

// f(t, begin, end) over [0, count) split into min(threads, count) ranges; an
// exception in any range is rethrown here after every thread has joined.
template <class F>
void parallel_for(int threads, int64_t count, F&& f) {
    if (threads <= 1 || count < 2) {
        f(0, int64_t{0}, count);
        return;
    }
    const int T = static_cast<int>(std::min<int64_t>(threads, count));
    std::vector<std::exception_ptr> errs(static_cast<size_t>(T));
    auto run = [&](int t) {
        try {
            f(t, count * t / T, count * (t + 1) / T);
        } catch (...) {
            errs[static_cast<size_t>(t)] = std::current_exception();
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(static_cast<size_t>(T - 1));
    for (int t = 1; t < T; ++t) pool.emplace_back(run, t);
    run(0);
    for (auto& th : pool) th.join();
    for (auto& e : errs)
        if (e) std::rethrow_exception(e);
}

// Header lines (first byte neither blank nor '*') with their line numbers.
std::vector<Header> find_headers(const char* buf, size_t len, int threads) {
    const int T = len < (1u << 22) ? 1 : threads;
    std::vector<std::vector<std::pair<size_t, int64_t>>> found(T);  // pos, local line ordinal
    std::vector<int64_t> lines(T, 0);
    parallel_for(T, T, [&](int, int64_t tb, int64_t te) {
        for (int64_t t = tb; t < te; ++t) {
            const size_t b = len * t / T, e = len * (t + 1) / T;
            // line starts s in [b, e): s == 0 or buf[s - 1] == '\n'
            size_t s = b;
            if (b > 0) {
                const void* nl = std::memchr(buf + b - 1, '\n', len - (b - 1));
                s = nl ? static_cast<size_t>(static_cast<const char*>(nl) - buf) + 1 : len;
            }
            int64_t k = 0;
            while (s < e && s < len) {
                const char c = buf[s];
                if (!is_space(c) && c != '*') found[t].emplace_back(s, k);
                ++k;
                const void* nl = std::memchr(buf + s, '\n', len - s);
                if (!nl) break;
                s = static_cast<size_t>(static_cast<const char*>(nl) - buf) + 1;
            }
            lines[t] = k;
        }
    });
    std::vector<Header> out;
    int64_t base = 0;
    for (int t = 0; t < T; ++t) {
        for (auto& f : found[t]) out.push_back(Header{f.first, base + f.second + 1});
        base += lines[t];
    }
    return out;
}

// Lines of [b, e): callback(line without '\n' and without one trailing '\r').
template <class F>
void for_lines(const char* b, const char* e, F&& f) {
    while (b < e) {
        const char* nl = static_cast<const char*>(std::memchr(b, '\n', static_cast<size_t>(e - b)));
        const char* le = nl ? nl : e;
        std::string_view line(b, static_cast<size_t>(le - b));
        if (!line.empty() && line.back() == '\r') line.remove_suffix(1);
        if (!f(line)) return;
        b = nl ? nl + 1 : e;
    }
}

// ---- one read under one layout (MpsReader, mps_reader.cpp:119-500) -----------------

class Reader {
public:
    Reader(const pdhg_mps_options& o, std::string origin, bool fixed, int threads)
        : opt_(o), origin_(std::move(origin)), fixed_(fixed), threads_(threads) {}

    void read(const char* buf, size_t len, const std::vector<Header>& headers);

    Builder b;
    std::vector<Warning> warnings;

private:
    [[noreturn]] void error(const std::string& msg) const {
        throw ReadError{origin_ + ":" + std::to_string(line_no_) + ": " + msg};
    }
    void warn(const std::string& section, const std::string& msg) {
        warnings.push_back(Warning{line_no_, section, msg});
    }
    double require_real(std::string_view t) const {
        double v = 0.0;
        if (!parse_real(t, &v)) error("expected a number, got '" + std::string(t) + "'");
        return v;
    }
    double bound_value(std::string_view t) const {
        double v = 0.0;
        if (infinite_token(t, &v)) return v;
        return require_real(t);
    }
    void tokenize_data(std::string_view line, std::vector<std::string_view>& out) const {
        if (fixed_) tokenize_fixed(line, out);
        else tokenize_free(line, out);
    }

    void apply_objsense(std::string_view t);
    void header(const std::vector<std::string_view>& t, bool* stop);
    void data_card(const std::vector<std::string_view>& t);
    void handle_rows(const std::vector<std::string_view>& t);
    void handle_columns(const std::vector<std::string_view>& t);
    void handle_rhs(const std::vector<std::string_view>& t);
    void handle_ranges(const std::vector<std::string_view>& t);
    void handle_bounds(const std::vector<std::string_view>& t);
    void apply_bound(int32_t col, const std::string& type, const std::string_view* value_token);
    void apply_range(int32_t row, double range);
    void sequential(const char* b, const char* e, int64_t first_line, bool* stop);
    void columns_parallel(const char* b, const char* e, int64_t first_line);
    void bounds_parallel(const char* b, const char* e, int64_t first_line);

    pdhg_mps_options opt_;
    std::string origin_;
    bool fixed_ = false;
    int threads_ = 1;
    int64_t line_no_ = 0;
    Section section_ = Section::None;
    bool objective_seen_ = false;
    bool in_integer_block_ = false;
    std::vector<std::string_view> tok_;
};

void Reader::apply_objsense(std::string_view t) {
    if (ieq(t, "MAX") || ieq(t, "MAXIMIZE")) b.maximize = true;
    else if (ieq(t, "MIN") || ieq(t, "MINIMIZE")) b.maximize = false;
    else error("unknown OBJSENSE '" + std::string(t) + "'");
}

void Reader::header(const std::vector<std::string_view>& t, bool* stop) {
    const std::string head = upper_copy(t[0]);
    if (head == "NAME") {
        b.name = t.size() > 1 ? std::string(t[1]) : std::string();
        section_ = Section::Name;
    } else if (head == "OBJSENSE" || head == "OBJSENS") {
        if (t.size() > 1) {
            apply_objsense(t[1]);
            section_ = Section::None;
        } else {
            section_ = Section::ObjSense;
        }
    } else if (head == "ROWS") {
        section_ = Section::Rows;
    } else if (head == "COLUMNS") {
        section_ = Section::Columns;
    } else if (head == "RHS") {
        section_ = Section::Rhs;
    } else if (head == "RANGES") {
        section_ = Section::Ranges;
    } else if (head == "BOUNDS") {
        section_ = Section::Bounds;
    } else if (head == "ENDATA") {
        *stop = true;
    } else {
        warn(head, "unsupported section '" + head + "' ignored");
        section_ = Section::Ignored;
    }
}

void Reader::data_card(const std::vector<std::string_view>& t) {
    switch (section_) {
        case Section::ObjSense:
            apply_objsense(t[0]);
            section_ = Section::None;
            break;
        case Section::Rows: handle_rows(t); break;
        case Section::Columns: handle_columns(t); break;
        case Section::Rhs: handle_rhs(t); break;
        case Section::Ranges: handle_ranges(t); break;
        case Section::Bounds: handle_bounds(t); break;
        case Section::Ignored: break;
        case Section::Name: break;
        default: error("data card outside any section");
    }
}

void Reader::handle_rows(const std::vector<std::string_view>& t) {  // mps_reader.cpp:208-246
    if (t.size() < 2) error("ROWS card needs a type and a name");
    const std::string_view name = t[1];
    auto record = [&](char sense, double lo, double hi) {
        b.add_row(name, lo, hi);
        b.row_sense.push_back(sense);
        b.row_rhs.push_back(0.0);
    };
    if (ieq(t[0], "N")) {
        if (!objective_seen_) {
            objective_seen_ = true;
            b.objective_name = std::string(name);
            return;
        }
        if (!opt_.keep_free_rows) {
            warn("ROWS", "dropping free row '" + std::string(name) + "' (keep_free_rows = false)");
            const int32_t k = b.dropped_names.add(name);
            b.dropped_idx.insert(k, hash_name(name));
            return;
        }
        record('N', -kInf, kInf);
    } else if (ieq(t[0], "L")) {
        record('L', -kInf, 0.0);
    } else if (ieq(t[0], "G")) {
        record('G', 0.0, kInf);
    } else if (ieq(t[0], "E")) {
        record('E', 0.0, 0.0);
    } else {
        error("unknown row type '" + std::string(t[0]) + "'");
    }
}

void Reader::handle_columns(const std::vector<std::string_view>& t) {  // mps_reader.cpp:248-290
    bool has_marker = false, intorg = false, intend = false;
    for (std::string_view tok : t) {
        if (marker_eq(tok, "MARKER")) has_marker = true;
        else if (marker_eq(tok, "INTORG")) intorg = true;
        else if (marker_eq(tok, "INTEND")) intend = true;
    }
    if (has_marker && (intorg || intend)) {
        in_integer_block_ = intorg;
        return;
    }
    if (t.size() < 3) error("COLUMNS card needs a column, a row and a value");
    const int32_t col = b.column_for(t[0]);
    if (in_integer_block_) b.is_int[col] = 1;
    for (size_t k = 1; k + 1 < t.size(); k += 2) {
        const std::string_view row_name = t[k];
        const double value = require_real(t[k + 1]);
        if (objective_seen_ && row_name == b.objective_name) {
            b.obj[col] = value;
            continue;
        }
        const int32_t r = b.row_idx.find(row_name);
        if (r < 0) {
            if (b.dropped(row_name)) continue;
            error("unknown row '" + std::string(row_name) + "' in COLUMNS");
        }
        b.entries.push_back(Triplet{r, col, value});
    }
}

void Reader::handle_rhs(const std::vector<std::string_view>& t) {  // mps_reader.cpp:292-331
    if (t.size() < 2) error("RHS card needs a row and a value");
    size_t k = (t.size() % 2 == 1) ? 1 : 0;
    for (; k + 1 < t.size(); k += 2) {
        const std::string_view row_name = t[k];
        const double value = require_real(t[k + 1]);
        if (objective_seen_ && row_name == b.objective_name) {
            b.obj_const = -value;  // the RHS of the objective row is minus its constant
            continue;
        }
        const int32_t r = b.row_idx.find(row_name);
        if (r < 0) {
            if (b.dropped(row_name)) continue;
            error("unknown row '" + std::string(row_name) + "' in RHS");
        }
        b.row_rhs[r] = value;
        switch (b.row_sense[r]) {
            case 'L': b.row_lo[r] = -kInf; b.row_hi[r] = value; break;
            case 'G': b.row_lo[r] = value; b.row_hi[r] = kInf; break;
            case 'E': b.row_lo[r] = value; b.row_hi[r] = value; break;
            case 'N': warn("RHS", "RHS given for free row '" + std::string(row_name) + "'; ignored"); break;
            default: break;
        }
    }
}

void Reader::apply_range(int32_t row, double range) {  // mps_reader.cpp:333-360
    const double rhs = b.row_rhs[row];
    const double mag = std::abs(range);
    switch (b.row_sense[row]) {
        case 'L': b.row_lo[row] = rhs - mag; b.row_hi[row] = rhs; break;
        case 'G': b.row_lo[row] = rhs; b.row_hi[row] = rhs + mag; break;
        case 'E':
            if (range >= 0) {
                b.row_lo[row] = rhs;
                b.row_hi[row] = rhs + range;
            } else {
                b.row_lo[row] = rhs + range;
                b.row_hi[row] = rhs;
            }
            break;
        case 'N': warn("RANGES", "range given for a free row; ignored"); break;
        default: break;
    }
}

void Reader::handle_ranges(const std::vector<std::string_view>& t) {  // mps_reader.cpp:362-376
    if (t.size() < 2) error("RANGES card needs a row and a value");
    size_t k = (t.size() % 2 == 1) ? 1 : 0;
    for (; k + 1 < t.size(); k += 2) {
        const int32_t r = b.row_idx.find(t[k]);
        if (r < 0) {
            if (b.dropped(t[k])) continue;
            error("unknown row '" + std::string(t[k]) + "' in RANGES");
        }
        apply_range(r, require_real(t[k + 1]));
    }
}

void Reader::handle_bounds(const std::vector<std::string_view>& t) {  // mps_reader.cpp:378-405
    if (t.size() < 2) error("BOUNDS card needs a type and a column");
    const std::string type = upper_copy(t[0]);
    const bool valueless = type == "FR" || type == "MI" || type == "PL" || type == "BV";
    size_t col_pos = 0;
    if (valueless) {
        col_pos = t.size() - 1;
    } else {
        if (t.size() < 3) error("BOUNDS card of type " + type + " needs a value");
        col_pos = t.size() - 2;
    }
    const std::string_view col_name = t[col_pos];
    const uint64_t h = hash_name(col_name);
    int32_t col = b.col_idx.find(col_name, h);
    if (col < 0) {
        warn("BOUNDS", "bound on column '" + std::string(col_name) + "' which has no coefficients");
        col = b.add_column(col_name, h);
    }
    const std::string_view* value_token = valueless ? nullptr : &t[col_pos + 1];
    apply_bound(col, type, value_token);
}

void Reader::apply_bound(int32_t col, const std::string& type, const std::string_view* value_token) {
    // mps_reader.cpp:407-466
    const double lo = b.col_lo[col], hi = b.col_hi[col];
    auto value = [&]() -> double {
        if (value_token == nullptr) error("bound type " + type + " needs a value");
        return bound_value(*value_token);
    };
    auto set = [&](double l, double u) {
        b.col_lo[col] = l;
        b.col_hi[col] = u;
    };
    if (type == "UP") {
        const double v = value();
        set(lo, v);
        if (v < 0.0 && lo == 0.0) {
            if (opt_.negative_upper_bound == 0) {
                set(-kInf, v);
                warn("BOUNDS", "negative UP bound on a column with the default lower bound 0; "
                               "lower bound set to -infinity (the established-solver "
                               "convention; see MpsOptions::negative_upper_bound)");
            } else {
                warn("BOUNDS", "negative UP bound leaves crossed bounds (literal reading)");
            }
        }
    } else if (type == "LO") {
        set(value(), hi);
    } else if (type == "FX") {
        const double v = value();
        set(v, v);
    } else if (type == "FR") {
        set(-kInf, kInf);
    } else if (type == "MI") {
        set(-kInf, hi);
    } else if (type == "PL") {
        set(lo, kInf);
    } else if (type == "BV") {
        set(0.0, 1.0);
        b.is_int[col] = 1;
    } else if (type == "LI") {
        set(value(), hi);
        b.is_int[col] = 1;
    } else if (type == "UI") {
        set(lo, value());
        b.is_int[col] = 1;
    } else if (type == "SC") {
        error("semi-continuous bounds (SC) are not supported");
    } else {
        error("unknown bound type '" + type + "'");
    }
}

// Lines [b, e) one by one, first_line being the number of the first.
void Reader::sequential(const char* lb, const char* le, int64_t first_line, bool* stop) {
    line_no_ = first_line - 1;
    for_lines(lb, le, [&](std::string_view line) {
        ++line_no_;
        if (line.empty() || line[0] == '*') return true;
        const bool is_header = !is_space(line[0]);
        if (fixed_ && !is_header) tokenize_fixed(line, tok_);
        else tokenize_free(line, tok_);
        if (tok_.empty()) return true;
        if (is_header) {
            header(tok_, stop);
            return !*stop;
        }
        data_card(tok_);
        return true;
    });
}

// ---- COLUMNS by chunks ------------------------------------------------------------------

struct Chunk {
    const char* b = nullptr;
    const char* e = nullptr;
    int64_t lines = 0;                 // lines in [b, e)
    Arena names;                       // chunk-local columns, in order of first appearance
    std::vector<uint64_t> hash;        // their hashes
    NameIndex index{&names};
    std::vector<Triplet> entries;      // col = local column
    std::vector<std::pair<int32_t, double>> obj;   // (local column, value), file order
    std::vector<int32_t> int_if_incoming;          // local columns in the integer block if the
                                                   // state entering the chunk is "in"
    std::vector<int32_t> int_local;                // local columns in a block opened in the chunk
    int state_out = -1;                            // -1: as entering, 0 / 1: set by a marker
    bool failed = false;
    int64_t err_line = 0;                          // local line ordinal (1-based) of the error
    std::string err_msg;
};

void Reader::columns_parallel(const char* lb, const char* le, int64_t first_line) {
    const size_t bytes = static_cast<size_t>(le - lb);
    const int T = static_cast<int>(std::min<size_t>(static_cast<size_t>(threads_) * 4, bytes / (1u << 18) + 1));
    std::vector<Chunk> ch(T);
    // line-aligned chunk bounds
    const char* prev = lb;
    for (int t = 0; t < T; ++t) {
        const char* e = t + 1 == T ? le : lb + bytes * (t + 1) / T;
        if (e < le && e > prev) {
            const char* nl = static_cast<const char*>(std::memchr(e - 1, '\n', static_cast<size_t>(le - (e - 1))));
            e = nl ? nl + 1 : le;
        }
        if (e < prev) e = prev;
        ch[t].b = prev;
        ch[t].e = e;
        prev = e;
    }
    const std::string objective = b.objective_name;
    const bool have_objective = objective_seen_;
    const NameIndex& rows = b.row_idx;
    const Builder& cb = b;
    std::atomic<int> next{0};
    auto work = [&](int, int64_t, int64_t) {
        std::vector<std::string_view> t;
        for (int c = next.fetch_add(1); c < T; c = next.fetch_add(1)) {
            Chunk& k = ch[c];
            int state = -1;  // -1: as entering the chunk
            int32_t last_local = -1;
            std::string_view last_name;
            int64_t ord = 0;
            for_lines(k.b, k.e, [&](std::string_view line) {
                ++ord;
                if (line.empty() || line[0] == '*') return true;
                if (!is_space(line[0])) {  // a header cannot be inside the range
                    k.failed = true;
                    k.err_line = ord;
                    k.err_msg = "internal: header inside a COLUMNS range";
                    return false;
                }
                if (fixed_) tokenize_fixed(line, t);
                else tokenize_free(line, t);
                if (t.empty()) return true;
                auto fail = [&](std::string msg) {
                    k.failed = true;
                    k.err_line = ord;
                    k.err_msg = std::move(msg);
                    return false;
                };
                bool has_marker = false, intorg = false, intend = false;
                for (std::string_view tok : t) {
                    if (marker_eq(tok, "MARKER")) has_marker = true;
                    else if (marker_eq(tok, "INTORG")) intorg = true;
                    else if (marker_eq(tok, "INTEND")) intend = true;
                }
                if (has_marker && (intorg || intend)) {
                    state = intorg ? 1 : 0;
                    return true;
                }
                if (t.size() < 3) return fail("COLUMNS card needs a column, a row and a value");
                int32_t local = last_local;
                if (local < 0 || t[0] != last_name) {
                    const uint64_t h = hash_name(t[0]);
                    local = k.index.find(t[0], h);
                    if (local < 0) {
                        local = k.names.add(t[0]);
                        k.index.insert(local, h);
                        k.hash.push_back(h);
                    }
                    last_local = local;
                    last_name = t[0];  // a view into the text, which stays put
                }
                if (state == 1) k.int_local.push_back(local);
                else if (state < 0) k.int_if_incoming.push_back(local);
                for (size_t q = 1; q + 1 < t.size(); q += 2) {
                    const std::string_view row_name = t[q];
                    double value = 0.0;
                    if (!parse_real(t[q + 1], &value))
                        return fail("expected a number, got '" + std::string(t[q + 1]) + "'");
                    if (have_objective && row_name == objective) {
                        k.obj.emplace_back(local, value);
                        continue;
                    }
                    const int32_t r = rows.find(row_name);
                    if (r < 0) {
                        if (cb.dropped(row_name)) continue;
                        return fail("unknown row '" + std::string(row_name) + "' in COLUMNS");
                    }
                    k.entries.push_back(Triplet{r, local, value});
                }
                return true;
            });
            // lines in the chunk, for the numbers of later chunks' lines (a
            // chunk that stopped early failed, and its count is never used)
            k.lines = ord;
            k.state_out = state;
        }
    };
    HostClock clk;
    parallel_for(threads_, threads_, work);
    clk.mark("columns: chunks");

    // the first error in file order ends the read
    int64_t line_base = first_line - 1;
    for (int c = 0; c < T; ++c) {
        if (ch[c].failed) {
            line_no_ = line_base + ch[c].err_line;
            error(ch[c].err_msg);
        }
        line_base += ch[c].lines;
    }
    // Column indices in order of first appearance. Flat id f numbers every
    // chunk-local column in file order. Threads own hash shards: each walks
    // the flat ids of its shard in order and finds, for every name, the column
    // it already had (src >= 0) or the first flat id that carried it
    // (src = -2 - f0), else marks a first appearance (src = -1).
    std::vector<int64_t> base(static_cast<size_t>(T) + 1, 0);
    for (int c = 0; c < T; ++c) base[c + 1] = base[c] + ch[c].names.size();
    const int64_t F = base[T];
    std::vector<std::string_view> fname(static_cast<size_t>(F));  // by flat id
    bigvec<uint64_t> fhash(static_cast<size_t>(F));
    const int S = std::max(1, threads_);
    // flat ids of each chunk, bucketed by shard (file order inside a bucket)
    std::vector<std::vector<std::vector<int64_t>>> bucket(static_cast<size_t>(T));
    parallel_for(threads_, T, [&](int, int64_t cb0, int64_t ce) {
        for (int64_t c = cb0; c < ce; ++c) {
            auto& bk = bucket[static_cast<size_t>(c)];
            bk.assign(static_cast<size_t>(S), {});
            for (int32_t l = 0; l < ch[c].names.size(); ++l) {
                const int64_t f = base[c] + l;
                const uint64_t h = ch[c].hash[static_cast<size_t>(l)];
                fname[f] = ch[c].names.get(l);
                fhash[f] = h;
                bk[(h >> 40) % static_cast<uint64_t>(S)].push_back(f);
            }
        }
    });
    clk.mark("merge: flat ids");
    auto name_of = [&](int64_t f) { return fname[static_cast<size_t>(f)]; };
    auto hash_of = [&](int64_t f) { return fhash[static_cast<size_t>(f)]; };
    bigvec<int64_t> src(static_cast<size_t>(F));
    const bool have_cols = b.col_names.size() > 0;
    parallel_for(S, S, [&](int, int64_t sb, int64_t se) {
        for (int64_t sh = sb; sh < se; ++sh) {
            size_t count = 0;
            for (int c = 0; c < T; ++c) count += bucket[c][static_cast<size_t>(sh)].size();
            size_t cap = 16;
            while (cap < 2 * count) cap <<= 1;
            std::vector<int64_t> table(cap, -1);
            const uint64_t mask = cap - 1;
            for (int c = 0; c < T; ++c) {
                for (int64_t f : bucket[c][static_cast<size_t>(sh)]) {
                    const uint64_t h = hash_of(f);
                    const std::string_view nm = name_of(f);
                    if (have_cols) {
                        const int32_t j = b.col_idx.find(nm, h);
                        if (j >= 0) {
                            src[f] = j;
                            continue;
                        }
                    }
                    uint64_t q = h & mask;
                    for (;;) {
                        const int64_t g = table[q];
                        if (g < 0) {
                            table[q] = f;
                            src[f] = -1;
                            break;
                        }
                        if (name_of(g) == nm) {
                            src[f] = -2 - g;
                            break;
                        }
                        q = (q + 1) & mask;
                    }
                }
            }
        }
    });
    bucket.clear();
    clk.mark("merge: shards");
    // numbering in file order: first appearances counted per block, a prefix
    // over the blocks, then each block numbers its own; repeats take the
    // number of the first appearance they point at
    const int64_t n0 = b.col_names.size();
    bigvec<int32_t> id(static_cast<size_t>(F));
    const int64_t NB = std::max<int64_t>(1, std::min<int64_t>(F / 65536 + 1, 4 * threads_));
    std::vector<int64_t> firsts(static_cast<size_t>(NB) + 1, 0);
    parallel_for(threads_, NB, [&](int, int64_t bb, int64_t be) {
        for (int64_t q = bb; q < be; ++q) {
            int64_t k = 0;
            for (int64_t f = F * q / NB; f < F * (q + 1) / NB; ++f) k += src[f] == -1;
            firsts[q + 1] = k;
        }
    });
    for (int64_t q = 0; q < NB; ++q) firsts[q + 1] += firsts[q];
    const int64_t nn = firsts[NB];
    if (n0 + nn > std::numeric_limits<int32_t>::max() - 1)
        throw ReadError{"too many rows or columns for 32-bit indices"};
    bigvec<int64_t> fresh(static_cast<size_t>(nn));  // flat ids of the new columns, in order
    parallel_for(threads_, NB, [&](int, int64_t bb, int64_t be) {
        for (int64_t q = bb; q < be; ++q) {
            int64_t k = firsts[q];
            for (int64_t f = F * q / NB; f < F * (q + 1) / NB; ++f) {
                if (src[f] == -1) {
                    id[f] = static_cast<int32_t>(n0 + k);
                    fresh[k++] = f;
                } else if (src[f] >= 0) {
                    id[f] = static_cast<int32_t>(src[f]);
                }
            }
        }
    });
    parallel_for(threads_, NB, [&](int, int64_t bb, int64_t be) {
        for (int64_t q = bb; q < be; ++q)
            for (int64_t f = F * q / NB; f < F * (q + 1) / NB; ++f)
                if (src[f] <= -2) id[f] = id[-2 - src[f]];
    });
    clk.mark("merge: numbering");
    // new names into the arena (offsets by a blocked prefix, bytes by
    // threads) and into the index
    Arena& A = b.col_names;
    std::vector<int64_t>& off = A.off;
    off.resize(static_cast<size_t>(n0 + nn) + 1);
    const int64_t NK = std::max<int64_t>(1, std::min<int64_t>(nn / 65536 + 1, 4 * threads_));
    std::vector<int64_t> boff(static_cast<size_t>(NK) + 1, 0);
    parallel_for(threads_, NK, [&](int, int64_t bb, int64_t be) {
        for (int64_t q = bb; q < be; ++q) {
            int64_t t = 0;
            for (int64_t k = nn * q / NK; k < nn * (q + 1) / NK; ++k)
                t += static_cast<int64_t>(name_of(fresh[k]).size()) + 1;
            boff[q + 1] = t;
        }
    });
    boff[0] = off[n0];
    for (int64_t q = 0; q < NK; ++q) boff[q + 1] += boff[q];
    parallel_for(threads_, NK, [&](int, int64_t bb, int64_t be) {
        for (int64_t q = bb; q < be; ++q) {
            int64_t o = boff[q];
            for (int64_t k = nn * q / NK; k < nn * (q + 1) / NK; ++k) {
                o += static_cast<int64_t>(name_of(fresh[k]).size()) + 1;
                off[n0 + k + 1] = o;
            }
        }
    });
    A.chars.resize(static_cast<size_t>(off[n0 + nn]));
    b.col_idx.reserve(static_cast<size_t>(n0 + nn));
    int32_t* slots = b.col_idx.slot.data();
    const uint64_t smask = b.col_idx.mask;
    parallel_for(threads_, nn, [&](int, int64_t kb, int64_t ke) {
        for (int64_t k = kb; k < ke; ++k) {
            const std::string_view nm = name_of(fresh[k]);
            char* dst = A.chars.data() + off[n0 + k];
            std::memcpy(dst, nm.data(), nm.size());
            dst[nm.size()] = '\0';
            // the names are distinct: take the first free slot of the probe
            uint64_t q = hash_of(fresh[k]) & smask;
            for (;;) {
                int32_t expect = -1;
                if (__atomic_compare_exchange_n(slots + q, &expect, static_cast<int32_t>(n0 + k), false,
                                                __ATOMIC_RELAXED, __ATOMIC_RELAXED))
                    break;
                q = (q + 1) & smask;
            }
        }
    });
    clk.mark("merge: names");
    b.col_idx.count += static_cast<int32_t>(nn);
    b.col_lo.resize(static_cast<size_t>(n0 + nn), 0.0);
    b.col_hi.resize(static_cast<size_t>(n0 + nn), kInf);
    b.obj.resize(static_cast<size_t>(n0 + nn), 0.0);
    b.is_int.resize(static_cast<size_t>(n0 + nn), 0);
    // integrality (the marker state carried from chunk to chunk) and the
    // objective coefficients, in file order
    size_t total = b.entries.size();
    std::vector<size_t> at(T);
    for (int c = 0; c < T; ++c) {
        Chunk& k = ch[c];
        const int32_t* g = id.data() + base[c];
        if (in_integer_block_)
            for (int32_t l : k.int_if_incoming) b.is_int[g[l]] = 1;
        for (int32_t l : k.int_local) b.is_int[g[l]] = 1;
        if (k.state_out >= 0) in_integer_block_ = k.state_out == 1;
        for (auto& o : k.obj) b.obj[g[o.first]] = o.second;
        at[c] = total;
        total += k.entries.size();
    }
    line_no_ = line_base;
    clk.mark("columns: merge");
    b.entries.resize(total);
    parallel_for(threads_, T, [&](int, int64_t cb0, int64_t ce) {
        for (int64_t c = cb0; c < ce; ++c) {
            Triplet* out = b.entries.data() + at[c];
            const int32_t* g = id.data() + base[c];
            for (const Triplet& e : ch[c].entries) *out++ = Triplet{e.row, g[e.col], e.v};
        }
    });
    clk.mark("columns: triplets");
}

// ---- BOUNDS by chunks -------------------------------------------------------------------

enum BoundType : int8_t { kUP, kLO, kFX, kFR, kMI, kPL, kBV, kLI, kUI };

// One parsed BOUNDS card: its column (or, for a column COLUMNS never named,
// the name, resolved in file order), type and value.
struct BoundCard {
    int32_t col;               // -1: look the name up when applied
    int8_t type;
    double value;
    int64_t line;              // local line ordinal (1-based) in the chunk
    std::string_view name;
};

struct BoundChunk {
    const char* b = nullptr;
    const char* e = nullptr;
    int64_t lines = 0;
    std::vector<BoundCard> cards;
    bool failed = false;
    int64_t err_line = 0;
    std::string err_msg;
};

// The cards of [lb, le) parsed by threads (every error that does not depend
// on earlier cards found there: card shape, type, value), then applied in
// file order exactly as handle_bounds / apply_bound do, with their warnings.
void Reader::bounds_parallel(const char* lb, const char* le, int64_t first_line) {
    const size_t bytes = static_cast<size_t>(le - lb);
    const int T = static_cast<int>(std::min<size_t>(static_cast<size_t>(threads_) * 4, bytes / (1u << 18) + 1));
    std::vector<BoundChunk> ch(T);
    const char* prev = lb;
    for (int t = 0; t < T; ++t) {
        const char* e = t + 1 == T ? le : lb + bytes * (t + 1) / T;
        if (e < le && e > prev) {
            const char* nl = static_cast<const char*>(std::memchr(e - 1, '\n', static_cast<size_t>(le - (e - 1))));
            e = nl ? nl + 1 : le;
        }
        if (e < prev) e = prev;
        ch[t].b = prev;
        ch[t].e = e;
        prev = e;
    }
    const NameIndex& cols = b.col_idx;
    std::atomic<int> next{0};
    parallel_for(threads_, threads_, [&](int, int64_t, int64_t) {
        std::vector<std::string_view> t;
        for (int c = next.fetch_add(1); c < T; c = next.fetch_add(1)) {
            BoundChunk& k = ch[c];
            int64_t ord = 0;
            for_lines(k.b, k.e, [&](std::string_view line) {
                ++ord;
                if (line.empty() || line[0] == '*') return true;
                auto fail = [&](std::string msg) {
                    k.failed = true;
                    k.err_line = ord;
                    k.err_msg = std::move(msg);
                    return false;
                };
                if (!is_space(line[0])) return fail("internal: header inside a BOUNDS range");
                if (fixed_) tokenize_fixed(line, t);
                else tokenize_free(line, t);
                if (t.empty()) return true;
                if (t.size() < 2) return fail("BOUNDS card needs a type and a column");
                const std::string type = upper_copy(t[0]);
                const bool valueless = type == "FR" || type == "MI" || type == "PL" || type == "BV";
                if (!valueless && t.size() < 3) return fail("BOUNDS card of type " + type + " needs a value");
                const size_t col_pos = valueless ? t.size() - 1 : t.size() - 2;
                BoundCard card{-1, 0, 0.0, ord, t[col_pos]};
                static const char* const kNames[] = {"UP", "LO", "FX", "FR", "MI", "PL", "BV", "LI", "UI"};
                int code = -1;
                for (int q = 0; q < 9; ++q)
                    if (type == kNames[q]) code = q;
                if (type == "SC") return fail("semi-continuous bounds (SC) are not supported");
                if (code < 0) return fail("unknown bound type '" + type + "'");
                card.type = static_cast<int8_t>(code);
                if (!valueless) {
                    const std::string_view tok = t[col_pos + 1];
                    double v = 0.0;
                    if (!infinite_token(tok, &v) && !parse_real(tok, &v))
                        return fail("expected a number, got '" + std::string(tok) + "'");
                    card.value = v;
                }
                card.col = cols.find(card.name);
                k.cards.push_back(card);
                return true;
            });
            k.lines = ord;  // a chunk that stopped early failed: its count is not used
        }
    });
    // the first error in file order ends the read; else the cards apply in order
    int64_t line_base = first_line - 1;
    for (int c = 0; c < T; ++c) {
        BoundChunk& k = ch[c];
        if (k.failed) {
            line_no_ = line_base + k.err_line;
            error(k.err_msg);
        }
        line_base += k.lines;
    }
    line_base = first_line - 1;
    for (int c = 0; c < T; ++c) {
        for (const BoundCard& card : ch[c].cards) {
            line_no_ = line_base + card.line;
            int32_t col = card.col;
            if (col < 0) {  // a column COLUMNS never named: made by its first bound
                const uint64_t h = hash_name(card.name);
                col = b.col_idx.find(card.name, h);
                if (col < 0) {
                    warn("BOUNDS", "bound on column '" + std::string(card.name) + "' which has no coefficients");
                    col = b.add_column(card.name, h);
                }
            }
            const double lo = b.col_lo[col], v = card.value;
            switch (card.type) {
                case kUP:
                    b.col_hi[col] = v;
                    if (v < 0.0 && lo == 0.0) {
                        if (opt_.negative_upper_bound == 0) {
                            b.col_lo[col] = -kInf;
                            warn("BOUNDS", "negative UP bound on a column with the default lower bound 0; "
                                           "lower bound set to -infinity (the established-solver "
                                           "convention; see MpsOptions::negative_upper_bound)");
                        } else {
                            warn("BOUNDS", "negative UP bound leaves crossed bounds (literal reading)");
                        }
                    }
                    break;
                case kLO: b.col_lo[col] = v; break;
                case kFX: b.col_lo[col] = v; b.col_hi[col] = v; break;
                case kFR: b.col_lo[col] = -kInf; b.col_hi[col] = kInf; break;
                case kMI: b.col_lo[col] = -kInf; break;
                case kPL: b.col_hi[col] = kInf; break;
                case kBV: b.col_lo[col] = 0.0; b.col_hi[col] = 1.0; b.is_int[col] = 1; break;
                case kLI: b.col_lo[col] = v; b.is_int[col] = 1; break;
                case kUI: b.col_hi[col] = v; b.is_int[col] = 1; break;
                default: break;
            }
        }
        line_base += ch[c].lines;
    }
    line_no_ = line_base;
}

void Reader::read(const char* buf, size_t len, const std::vector<Header>& headers) {
    bool stop = false;
    // lines before the first header
    const size_t first = headers.empty() ? len : headers[0].pos;
    sequential(buf, buf + first, 1, &stop);
    for (size_t h = 0; h < headers.size() && !stop; ++h) {
        const size_t hb = headers[h].pos;
        const size_t he = h + 1 < headers.size() ? headers[h + 1].pos : len;
        const char* hl_end = static_cast<const char*>(std::memchr(buf + hb, '\n', he - hb));
        const char* data = hl_end ? hl_end + 1 : buf + he;
        sequential(buf + hb, data, headers[h].line, &stop);  // the header line itself
        if (stop) break;
        if (section_ == Section::Columns && (buf + he) - data > (1 << 20) && threads_ > 1)
            columns_parallel(data, buf + he, headers[h].line + 1);
        else if (section_ == Section::Bounds && (buf + he) - data > (1 << 20) && threads_ > 1)
            bounds_parallel(data, buf + he, headers[h].line + 1);
        else
            sequential(data, buf + he, headers[h].line + 1, &stop);
    }
    if (!objective_seen_)
        throw ReadError{origin_ + ": no objective row (no N row in the ROWS section)"};
}

// ---- the model -------------------------------------------------------------------------------

}  // namespace

struct Model {
    std::string name, objective_name;
    bool maximize = false;
    double obj_const = 0.0;
    int32_t m = 0, n = 0;
    std::vector<int32_t> rp;
    bigvec<int32_t> ci;
    bigvec<double> v;
    std::vector<double> c, col_lo, col_hi, row_lo, row_hi;
    std::vector<uint8_t> is_int;
    Arena row_names, col_names;
    std::vector<Warning> warnings;
    bool fixed_format = false;
};

namespace {

// CsrMatrix::from_triplets (sparse.cpp:30-70): rows by a stable counting sort,
// each row by column with duplicates summed in file order, |sum| <= 1e-14 dropped.
void build_csr(int32_t m, bigvec<Triplet>& ent, int threads, Model* out) {
    for (const Triplet& e : ent)
        if (!std::isfinite(e.v)) throw ReadError{"from_triplets: non-finite coefficient"};
    const int64_t nnz = static_cast<int64_t>(ent.size());
    int T = static_cast<int>(std::min<int64_t>(threads, nnz / 65536 + 1));
    while (T > 1 && static_cast<int64_t>(T) * (m + 1) > (int64_t{1} << 26)) --T;
    std::vector<std::vector<int64_t>> cnt(T, std::vector<int64_t>(static_cast<size_t>(m) + 1, 0));
    parallel_for(T, T, [&](int, int64_t tb, int64_t te) {
        for (int64_t t = tb; t < te; ++t)
            for (int64_t k = nnz * t / T; k < nnz * (t + 1) / T; ++k) ++cnt[t][ent[k].row];
    });
    std::vector<int64_t> start(static_cast<size_t>(m) + 1, 0);
    for (int32_t r = 0; r < m; ++r) {
        int64_t s = start[r];
        for (int t = 0; t < T; ++t) {
            const int64_t c = cnt[t][r];
            cnt[t][r] = s;
            s += c;
        }
        start[r + 1] = s;
    }
    bigvec<int32_t> col(static_cast<size_t>(nnz));
    bigvec<double> val(static_cast<size_t>(nnz));
    parallel_for(T, T, [&](int, int64_t tb, int64_t te) {
        for (int64_t t = tb; t < te; ++t)
            for (int64_t k = nnz * t / T; k < nnz * (t + 1) / T; ++k) {
                const int64_t p = cnt[t][ent[k].row]++;
                col[p] = ent[k].col;
                val[p] = ent[k].v;
            }
    });
    bigvec<Triplet>().swap(ent);
    cnt.clear();
    // order, sum and drop inside each row; keep[r] = entries kept
    std::vector<int64_t> keep(static_cast<size_t>(m) + 1, 0);
    parallel_for(threads, m, [&](int, int64_t rb, int64_t re) {
        std::vector<int64_t> idx;
        std::vector<int32_t> c2;
        std::vector<double> v2;
        for (int64_t r = rb; r < re; ++r) {
            const int64_t s = start[r], e = start[r + 1];
            bool sorted = true;
            for (int64_t k = s + 1; k < e; ++k)
                if (col[k - 1] >= col[k]) {
                    sorted = false;
                    break;
                }
            int64_t w = s;
            if (sorted) {
                for (int64_t k = s; k < e; ++k) {
                    const double sum = 0.0 + val[k];
                    if (std::abs(sum) <= kNumericZero) continue;
                    col[w] = col[k];
                    val[w] = sum;
                    ++w;
                }
            } else {
                idx.resize(static_cast<size_t>(e - s));
                for (int64_t k = s; k < e; ++k) idx[k - s] = k;
                std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b2) { return col[a] < col[b2]; });
                c2.clear();
                v2.clear();
                for (size_t q = 0; q < idx.size();) {
                    const int32_t cc = col[idx[q]];
                    double sum = 0.0;
                    for (; q < idx.size() && col[idx[q]] == cc; ++q) sum += val[idx[q]];
                    if (std::abs(sum) <= kNumericZero) continue;
                    c2.push_back(cc);
                    v2.push_back(sum);
                }
                for (size_t q = 0; q < c2.size(); ++q) {
                    col[s + static_cast<int64_t>(q)] = c2[q];
                    val[s + static_cast<int64_t>(q)] = v2[q];
                }
                w = s + static_cast<int64_t>(c2.size());
            }
            keep[r] = w - s;
        }
    });
    out->rp.assign(static_cast<size_t>(m) + 1, 0);
    int64_t total = 0;
    for (int32_t r = 0; r < m; ++r) {
        total += keep[r];
        if (total > std::numeric_limits<int32_t>::max()) throw ReadError{"too many nonzeros for 32-bit indices"};
        out->rp[r + 1] = static_cast<int32_t>(total);
    }
    out->ci.resize(static_cast<size_t>(total));
    out->v.resize(static_cast<size_t>(total));
    parallel_for(threads, m, [&](int, int64_t rb, int64_t re) {
        for (int64_t r = rb; r < re; ++r) {
            std::memcpy(out->ci.data() + out->rp[r], col.data() + start[r], sizeof(int32_t) * keep[r]);
            std::memcpy(out->v.data() + out->rp[r], val.data() + start[r], sizeof(double) * keep[r]);
        }
    });
}

// Problem::validate (problem.cpp:50-99) with the model's names; the matrix
// part cannot fail after build_csr.
bool validate(const Model& p, std::string* why) {
    if (!std::isfinite(p.obj_const)) {
        *why = "objective constant is not finite";
        return false;
    }
    for (int32_t j = 0; j < p.n; ++j) {
        if (!std::isfinite(p.c[j])) {
            *why = "non-finite objective coefficient in column " + std::string(p.col_names.get(j));
            return false;
        }
        if (std::isnan(p.col_lo[j]) || std::isnan(p.col_hi[j])) {
            *why = "NaN bound on column " + std::string(p.col_names.get(j));
            return false;
        }
        if (p.col_lo[j] > p.col_hi[j]) {
            *why = "crossed bounds on column " + std::string(p.col_names.get(j));
            return false;
        }
    }
    for (int32_t i = 0; i < p.m; ++i) {
        if (std::isnan(p.row_lo[i]) || std::isnan(p.row_hi[i])) {
            *why = "NaN bound on row " + std::string(p.row_names.get(i));
            return false;
        }
        if (p.row_lo[i] > p.row_hi[i]) {
            *why = "crossed bounds on row " + std::string(p.row_names.get(i));
            return false;
        }
    }
    for (int32_t j = 0; j < p.n; ++j) {
        if (!p.is_int[j]) continue;
        for (double bd : {p.col_lo[j], p.col_hi[j]}) {
            if (bd > -kInf && bd < kInf && std::abs(bd - std::round(bd)) > 1e-9) {
                *why = "integer column " + std::string(p.col_names.get(j)) + " has a fractional bound";
                return false;
            }
        }
    }
    return true;
}

std::unique_ptr<Model> read_once(const char* buf, size_t len, const std::vector<Header>& headers,
                                 const pdhg_mps_options& o, const std::string& origin, bool fixed,
                                 int threads) {
    HostClock clk;
    Reader rd(o, origin, fixed, threads);
    rd.read(buf, len, headers);
    clk.mark("parse");
    auto m = std::make_unique<Model>();
    Builder& b = rd.b;
    if (b.row_names.size() > std::numeric_limits<int32_t>::max() - 1 ||
        b.col_names.size() > std::numeric_limits<int32_t>::max() - 1)
        throw ReadError{"too many rows or columns for 32-bit indices"};
    m->name = std::move(b.name);
    m->objective_name = std::move(b.objective_name);
    m->maximize = b.maximize;
    m->obj_const = b.obj_const;
    m->m = b.row_names.size();
    m->n = b.col_names.size();
    build_csr(m->m, b.entries, threads, m.get());
    clk.mark("csr");
    m->c = std::move(b.obj);
    m->col_lo = std::move(b.col_lo);
    m->col_hi = std::move(b.col_hi);
    m->row_lo = std::move(b.row_lo);
    m->row_hi = std::move(b.row_hi);
    m->is_int = std::move(b.is_int);
    m->row_names = std::move(b.row_names);
    m->col_names = std::move(b.col_names);
    m->warnings = std::move(rd.warnings);
    std::string why;
    if (!validate(*m, &why)) throw ReadError{origin + ": model failed validation after parse: " + why};
    clk.mark("validate");
    return m;
}

}  // namespace

// read_mps_string (mps_reader.cpp:506-533): free form first, the fixed
// column layout when that fails, the free-form error when both fail.
std::unique_ptr<Model> read(const char* buf, size_t len, const pdhg_mps_options& o,
                            const std::string& origin) {
    int threads = o.threads > 0 ? o.threads : static_cast<int>(std::thread::hardware_concurrency());
    threads = std::max(1, std::min(threads, 64));
    HostClock clk;
    const std::vector<Header> headers = find_headers(buf, len, threads);
    clk.mark("headers");
    try {
        return read_once(buf, len, headers, o, origin, false, threads);
    } catch (const ReadError& free_form) {
        try {
            auto m = read_once(buf, len, headers, o, origin, true, threads);
            m->warnings.insert(m->warnings.begin(),
                               Warning{0, "FORMAT", "free-form parse failed (" + free_form.what +
                                                        "); re-read under fixed-column MPS rules"});
            m->fixed_format = true;
            return m;
        } catch (const ReadError&) {
            throw free_form;
        }
    }
}

}  // namespace mps
}  // namespace pdhg

// ---- C ABI ----------------------------------------------------------------------------------------

struct pdhg_model {
    std::unique_ptr<pdhg::mps::Model> m;
};

namespace {

void set_err(char* err, size_t cap, const std::string& msg) {
    if (err == nullptr || cap == 0) return;
    const size_t k = std::min(cap - 1, msg.size());
    std::memcpy(err, msg.data(), k);
    err[k] = '\0';
}

int read_common(const char* buf, size_t len, const char* origin, const pdhg_mps_options* opt,
                pdhg_model** out, char* err, size_t err_cap) {
    pdhg_mps_options o;
    pdhg_default_mps_options(&o);
    if (opt != nullptr) o = *opt;
    if (o.negative_upper_bound < 0 || o.negative_upper_bound > 1 || o.keep_free_rows < 0 ||
        o.keep_free_rows > 1 || o.threads < 0) {
        set_err(err, err_cap, "pdhg_read_mps: invalid options");
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    try {
        auto m = pdhg::mps::read(buf, len, o, origin);
        *out = new pdhg_model{std::move(m)};
        set_err(err, err_cap, "");
        return PDHG_OK;
    } catch (const pdhg::mps::ReadError& e) {
        set_err(err, err_cap, e.what);
        return PDHG_ERR_INVALID_ARGUMENT;
    } catch (const std::bad_alloc&) {
        set_err(err, err_cap, "pdhg_read_mps: out of host memory");
        return PDHG_ERR_OUT_OF_MEMORY;
    }
}

}  // namespace

extern "C" {

void pdhg_default_mps_options(pdhg_mps_options* o) {
    if (o == nullptr) return;
    o->negative_upper_bound = 0;
    o->keep_free_rows = 1;
    o->threads = 0;
}

int pdhg_read_mps(const char* text, size_t len, const char* origin, const pdhg_mps_options* opt,
                  pdhg_model** out, char* err, size_t err_cap) {
    if (out == nullptr || (text == nullptr && len > 0)) {
        set_err(err, err_cap, "pdhg_read_mps: null argument");
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    return read_common(text != nullptr ? text : "", len, origin != nullptr ? origin : "<string>", opt,
                       out, err, err_cap);
}

int pdhg_read_mps_file(const char* path, const pdhg_mps_options* opt, pdhg_model** out, char* err,
                       size_t err_cap) {
    if (out == nullptr || path == nullptr) {
        set_err(err, err_cap, "pdhg_read_mps_file: null argument");
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    std::FILE* f = std::fopen(path, "rb");
    if (f == nullptr) {
        set_err(err, err_cap, std::string("cannot open '") + path + "'");
        return PDHG_ERR_INVALID_ARGUMENT;
    }
    std::vector<char> buf;
    try {
        char tmp[1 << 16];
        if (std::fseek(f, 0, SEEK_END) == 0) {
            const long sz = std::ftell(f);
            if (sz > 0) buf.reserve(static_cast<size_t>(sz));
            std::fseek(f, 0, SEEK_SET);
        }
        size_t k;
        while ((k = std::fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + k);
    } catch (const std::bad_alloc&) {
        std::fclose(f);
        set_err(err, err_cap, "pdhg_read_mps_file: out of host memory");
        return PDHG_ERR_OUT_OF_MEMORY;
    }
    std::fclose(f);
    return read_common(buf.data(), buf.size(), path, opt, out, err, err_cap);
}

void pdhg_model_free(pdhg_model* m) { delete m; }

int pdhg_model_get_info(const pdhg_model* m, pdhg_model_info* info) {
    if (m == nullptr || info == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    info->m = m->m->m;
    info->n = m->m->n;
    info->nnz = static_cast<int64_t>(m->m->ci.size());
    info->obj_const = m->m->obj_const;
    info->maximize = m->m->maximize ? 1 : 0;
    info->warnings = static_cast<int32_t>(m->m->warnings.size());
    info->fixed_format = m->m->fixed_format ? 1 : 0;
    return PDHG_OK;
}

int pdhg_model_arrays(const pdhg_model* m, const int32_t** row_ptr, const int32_t** col_idx,
                      const double** values, const double** c, const double** col_lo,
                      const double** col_hi, const double** row_lo, const double** row_hi,
                      const uint8_t** is_integer) {
    if (m == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    const pdhg::mps::Model& p = *m->m;
    if (row_ptr) *row_ptr = p.rp.data();
    if (col_idx) *col_idx = p.ci.data();
    if (values) *values = p.v.data();
    if (c) *c = p.c.data();
    if (col_lo) *col_lo = p.col_lo.data();
    if (col_hi) *col_hi = p.col_hi.data();
    if (row_lo) *row_lo = p.row_lo.data();
    if (row_hi) *row_hi = p.row_hi.data();
    if (is_integer) *is_integer = p.is_int.data();
    return PDHG_OK;
}

const char* pdhg_model_name(const pdhg_model* m) { return m ? m->m->name.c_str() : ""; }
const char* pdhg_model_objective_name(const pdhg_model* m) { return m ? m->m->objective_name.c_str() : ""; }

const char* pdhg_model_row_name(const pdhg_model* m, int32_t i) {
    if (m == nullptr || i < 0 || i >= m->m->m) return nullptr;
    return m->m->row_names.c_str(i);
}

const char* pdhg_model_col_name(const pdhg_model* m, int32_t j) {
    if (m == nullptr || j < 0 || j >= m->m->n) return nullptr;
    return m->m->col_names.c_str(j);
}

int pdhg_model_name_table(const pdhg_model* m, int columns, const char** chars,
                          const int64_t** offsets) {
    if (m == nullptr || chars == nullptr || offsets == nullptr) return PDHG_ERR_INVALID_ARGUMENT;
    const pdhg::mps::Arena& a = columns ? m->m->col_names : m->m->row_names;
    *chars = a.chars.data();
    *offsets = a.off.data();
    return PDHG_OK;
}

int pdhg_model_warning(const pdhg_model* m, int32_t k, int64_t* line, const char** section,
                       const char** message) {
    if (m == nullptr || k < 0 || static_cast<size_t>(k) >= m->m->warnings.size())
        return PDHG_ERR_INVALID_ARGUMENT;
    const pdhg::mps::Warning& w = m->m->warnings[static_cast<size_t>(k)];
    if (line) *line = w.line;
    if (section) *section = w.section.c_str();
    if (message) *message = w.message.c_str();
    return PDHG_OK;
}

}  // extern "C"
