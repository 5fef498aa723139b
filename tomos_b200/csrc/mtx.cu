// mtx.cu -- MatrixMarket files on the host (tomos_mtx_*).
//
// The reference reads its matrices (the tall-thin test systems its MATLAB
// generator writes, scripts/generate_tall_thin_mtx.m) with the NIST mmio
// routines (src/io/mmio.c: mm_read_banner, mm_read_mtx_array_size,
// mm_read_mtx_crd_size) through read_mtx_host
// (benchmarks/solvers/cuda/lsqr_precision_runner.cu:101-125): an `array`
// file's values fill an m x n column-major FP64 buffer, one fscanf("%lf")
// per value.  Here the same files are read with the same number parsing
// (strtod), plus what the runner leaves out: `coordinate` files (1-based
// triplets), the `integer` and `pattern` fields, and symmetric /
// skew-symmetric storage (the stored lower triangle mirrored).  Complex and
// hermitian files are rejected, as the LSQR path has no complex type.
// Errors use the runner's wording ("could not open", "not a valid
// MatrixMarket file", "could not read array size", "truncated/malformed
// data").
//
// `array` files (the generator's format: one value per line, ~24 bytes a
// value, 24 GB for a 1e6 x 1000 system) are parsed by host threads over a
// read-only mapping of the file: the data section is cut into byte ranges,
// each thread counts the tokens that start in its range, a prefix sum gives
// every range its first value index, and each thread then parses its tokens
// with strtod.  Value t of the file sits at a position fixed by t alone, so
// every element is written exactly once and the result is the sequential
// read's bit for bit.  `general` coordinate files are read the same way by
// tomos_mtx_read_coo (entry e to slot e); into a dense matrix, and for
// symmetric storage, coordinate files stay sequential (repeated entries add
// in file order; mirrored entries shift the slots).  TOMOS_MTX_THREADS sets
// the thread count.
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "tomos_b200.h"

namespace {

struct MtxFile {
    FILE* f = nullptr;
    tomos_mtx_info info{};
    ~MtxFile() {
        if (f) std::fclose(f);
    }
};

std::string lower(const char* s) {
    std::string r(s);
    for (char& c : r) c = (char)std::tolower((unsigned char)c);
    return r;
}

// Reads one line (without the newline) into buf; false at end of file.
bool read_line(FILE* f, std::string& buf) {
    buf.clear();
    int c;
    bool any = false;
    while ((c = std::fgetc(f)) != EOF) {
        any = true;
        if (c == '\n') break;
        buf.push_back((char)c);
    }
    if (!buf.empty() && buf.back() == '\r') buf.pop_back();
    return any;
}

bool blank(const std::string& s) {
    for (char c : s)
        if (!std::isspace((unsigned char)c)) return false;
    return true;
}

// Opens the file, parses the banner and the size line; `f` is then at the
// first value.
tomos_status mtx_open(const char* path, MtxFile& m) {
    using tomos_b200::fail;
    const std::string p = path ? path : "";
    m.f = path ? std::fopen(path, "r") : nullptr;
    if (!m.f) return fail(TOMOS_ERR_INVALID, "could not open '" + p + "'");
    std::string line;
    char banner[64] = {0}, object[64] = {0}, format[64] = {0}, field[64] = {0}, sym[64] = {0};
    if (!read_line(m.f, line) ||
        std::sscanf(line.c_str(), "%63s %63s %63s %63s %63s", banner, object, format, field, sym) != 5 ||
        std::strcmp(banner, "%%MatrixMarket") != 0 || lower(object) != "matrix")
        return fail(TOMOS_ERR_INVALID, "'" + p + "': not a valid MatrixMarket file");
    const std::string fmt = lower(format), fld = lower(field), sy = lower(sym);
    tomos_mtx_info& in = m.info;
    if (fmt == "array") in.format = TOMOS_MTX_ARRAY;
    else if (fmt == "coordinate") in.format = TOMOS_MTX_COORDINATE;
    else return fail(TOMOS_ERR_INVALID, "'" + p + "': not a valid MatrixMarket file");
    if (fld == "real" || fld == "double") in.field = TOMOS_MTX_REAL;
    else if (fld == "integer") in.field = TOMOS_MTX_INTEGER;
    else if (fld == "pattern" && in.format == TOMOS_MTX_COORDINATE) in.field = TOMOS_MTX_PATTERN;
    else return fail(TOMOS_ERR_UNSUPPORTED, "'" + p + "': field '" + fld + "' is not supported (real, integer, pattern)");
    if (sy == "general") in.symmetry = TOMOS_MTX_GENERAL;
    else if (sy == "symmetric") in.symmetry = TOMOS_MTX_SYMMETRIC;
    else if (sy == "skew-symmetric") in.symmetry = TOMOS_MTX_SKEW;
    else return fail(TOMOS_ERR_UNSUPPORTED, "'" + p + "': symmetry '" + sy + "' is not supported");
    // comments, then the size line
    do {
        if (!read_line(m.f, line)) return fail(TOMOS_ERR_INVALID, "'" + p + "': could not read array size");
    } while (line.empty() || line[0] == '%' || blank(line));
    long long r = -1, c = -1, z = -1;
    const int got = std::sscanf(line.c_str(), "%lld %lld %lld", &r, &c, &z);
    if ((in.format == TOMOS_MTX_ARRAY && got < 2) || (in.format == TOMOS_MTX_COORDINATE && got < 3) || r < 0 ||
        c < 0 || (in.format == TOMOS_MTX_COORDINATE && z < 0))
        return fail(TOMOS_ERR_INVALID, "'" + p + "': could not read array size");
    if (in.symmetry != TOMOS_MTX_GENERAL && r != c)
        return fail(TOMOS_ERR_INVALID, "'" + p + "': a symmetric matrix must be square");
    in.rows = r;
    in.cols = c;
    if (in.format == TOMOS_MTX_COORDINATE) {
        in.entries = z;
    } else if (in.symmetry == TOMOS_MTX_SYMMETRIC) {
        in.entries = r * (r + 1) / 2;
    } else if (in.symmetry == TOMOS_MTX_SKEW) {
        in.entries = r * (r - 1) / 2;
    } else {
        in.entries = r * c;
    }
    return TOMOS_OK;
}

bool read_value(FILE* f, double* v) {
    char tok[128];
    if (std::fscanf(f, "%127s", tok) != 1) return false;
    // a token of 127 characters may have been cut: if more of it follows,
    // reject it, as the mapped reader rejects tokens over 127 characters
    if (std::strlen(tok) == 127) {
        const int c = std::fgetc(f);
        if (c != EOF) std::ungetc(c, f);
        if (c != EOF && !std::isspace(c)) return false;
    }
    errno = 0;
    char* end = nullptr;
    *v = std::strtod(tok, &end);
    return end && *end == '\0' && end != tok;
}

// A whole index token, as the mapped reader's parse_index: a decimal
// integer of at most 127 characters followed by whitespace or the end.
bool read_index(FILE* f, long long* v) {
    char tok[128];
    if (std::fscanf(f, "%127s", tok) != 1) return false;
    if (std::strlen(tok) == 127) {
        const int c = std::fgetc(f);
        if (c != EOF) std::ungetc(c, f);
        if (c != EOF && !std::isspace(c)) return false;
    }
    errno = 0;
    char* end = nullptr;
    *v = std::strtoll(tok, &end, 10);
    return end && *end == '\0' && end != tok && errno == 0;
}

// Visits every stored entry as (row, col, value), 0-based; symmetric parts
// are emitted once here (the callers mirror them).
template <class Fn>
tomos_status mtx_entries(MtxFile& m, const char* path, Fn&& fn) {
    using tomos_b200::fail;
    const tomos_mtx_info& in = m.info;
    const std::string bad = std::string("'") + path + "': truncated/malformed data";
    if (in.format == TOMOS_MTX_ARRAY) {
        for (int64_t j = 0; j < in.cols; ++j) {
            const int64_t i0 = in.symmetry == TOMOS_MTX_GENERAL ? 0 : (in.symmetry == TOMOS_MTX_SYMMETRIC ? j : j + 1);
            for (int64_t i = i0; i < in.rows; ++i) {
                double v;
                if (!read_value(m.f, &v)) return fail(TOMOS_ERR_INVALID, bad);
                fn(i, j, v);
            }
        }
        return TOMOS_OK;
    }
    for (int64_t e = 0; e < in.entries; ++e) {
        long long i, j;
        double v = 1.0;
        if (!read_index(m.f, &i) || !read_index(m.f, &j)) return fail(TOMOS_ERR_INVALID, bad);
        if (in.field != TOMOS_MTX_PATTERN && !read_value(m.f, &v)) return fail(TOMOS_ERR_INVALID, bad);
        if (i < 1 || j < 1 || i > in.rows || j > in.cols)
            return fail(TOMOS_ERR_INVALID, std::string("'") + path + "': entry " + std::to_string(e + 1) +
                                               " lies outside the matrix");
        fn((int64_t)(i - 1), (int64_t)(j - 1), v);
    }
    return TOMOS_OK;
}

inline bool is_space(char c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\f' || c == '\v'; }

// Parses one whitespace-free token [p, e) as a double, as strtod on the
// token alone; false if it is not entirely a number (or longer than 127
// characters, the sequential reader's token limit).
bool parse_token(const char* p, const char* e, double* v) {
    const size_t n = (size_t)(e - p);
    if (n == 0 || n > 127) return false;
    char tok[128];
    std::memcpy(tok, p, n);
    tok[n] = '\0';
    char* end = nullptr;
    *v = std::strtod(tok, &end);
    return end == tok + n;
}

// Host threads for n bytes of values: TOMOS_MTX_THREADS when set (1..256),
// else one per MiB up to the hardware threads.
int parse_threads(size_t bytes) {
    if (const char* e = std::getenv("TOMOS_MTX_THREADS")) {
        const long c = std::atol(e);
        if (c >= 1) return (int)std::min(c, 256L);
    }
    long hw = (long)std::thread::hardware_concurrency();
    if (hw < 1) hw = 1;
    const long want = (long)(bytes >> 20) + 1;
    return (int)std::max(1L, std::min(std::min(hw, want), 256L));
}

// The (row, col) of stored value t of an `array` file: column by column,
// the whole column for general storage, rows j.. (symmetric) or j+1..
// (skew-symmetric) of column j otherwise.
struct ArrayPos {
    int64_t rows, cols;
    int32_t sym;
    int64_t first(int64_t j) const {
        return sym == TOMOS_MTX_GENERAL ? 0 : (sym == TOMOS_MTX_SYMMETRIC ? j : j + 1);
    }
    void at(int64_t t, int64_t* i, int64_t* j) const {
        if (sym == TOMOS_MTX_GENERAL) {
            *j = t / rows;
            *i = t % rows;
            return;
        }
        int64_t c = 0;
        while (c < cols && t >= rows - first(c)) {
            t -= rows - first(c);
            ++c;
        }
        *j = c;
        *i = first(c) + t;
    }
    void next(int64_t* i, int64_t* j) const {
        if (++*i >= rows) {
            ++*j;
            *i = first(*j);
            while (*j < cols && *i >= rows) {  // empty trailing columns of skew storage
                ++*j;
                *i = first(*j);
            }
        }
    }
};

// The data section of an open file (positioned after its size line),
// mapped read-only and cut into one byte range per thread, with the index
// of the first token that starts in each range (cnt[k]; cnt[nt] = all).
struct MappedTokens {
    const char* d = nullptr;
    size_t size = 0, start = 0;
    int nt = 1;
    std::vector<size_t> lo, hi;
    std::vector<int64_t> cnt;
    void* map = nullptr;
    ~MappedTokens() {
        if (map) munmap(map, size);
    }
    bool starts_token(size_t p) const { return !is_space(d[p]) && (p == start || is_space(d[p - 1])); }
    // end of the token starting at p
    size_t token_end(size_t p) const {
        while (p < size && !is_space(d[p])) ++p;
        return p;
    }
    // start of the next token at or after p (size if none)
    size_t next_token(size_t p) const {
        while (p < size && is_space(d[p])) ++p;
        return p;
    }
    // body(k) for every range k, on up to nt threads
    template <class Body>
    void run(Body&& body) const {
        if (nt < 1) return;  // an empty data section has no ranges
        std::vector<std::thread> th;
        bool spawned = true;
        for (int k = 1; k < nt && spawned; ++k) {
            try {
                th.emplace_back(body, k);
            } catch (...) {
                spawned = false;
            }
        }
        const int done = (int)th.size() + 1;
        body(0);
        for (int k = done; k < nt; ++k) body(k);  // ranges no thread took
        for (auto& t : th) t.join();
    }
    bool open(FILE* f) {
        const long off = std::ftell(f);
        struct stat st;
        if (off < 0 || fstat(fileno(f), &st) != 0 || !S_ISREG(st.st_mode)) return false;
        size = (size_t)st.st_size;
        start = (size_t)off;
        if (start >= size) {
            size = 0;
            nt = 0;
            cnt.assign(1, 0);
            return true;
        }
        map = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fileno(f), 0);
        if (map == MAP_FAILED) {
            map = nullptr;
            return false;
        }
        madvise(map, size, MADV_SEQUENTIAL);
        d = static_cast<const char*>(map);
        const size_t bytes = size - start;
        nt = parse_threads(bytes);
        lo.resize(nt);
        hi.resize(nt);
        for (int k = 0; k < nt; ++k) {
            lo[k] = start + bytes * (size_t)k / (size_t)nt;
            hi[k] = start + bytes * (size_t)(k + 1) / (size_t)nt;
        }
        cnt.assign(nt + 1, 0);
        run([&](int k) {
            int64_t c = 0;
            for (size_t p = lo[k]; p < hi[k]; ++p) c += starts_token(p);
            cnt[k + 1] = c;
        });
        for (int k = 0; k < nt; ++k) cnt[k + 1] += cnt[k];
        return true;
    }
};

// The `array` values of the open file (positioned at its first value) into
// at(i, j) (and its mirror for symmetric storage), in parallel.  Returns
// kParsed, kMalformed (a malformed token or too few values) or kNoMap (not
// a regular file that maps: the caller reads it sequentially; the file
// position is untouched).
enum { kParsed = 0, kMalformed = 1, kNoMap = 2 };
template <class At>
int read_array_parallel(MtxFile& m, At&& at) {
    const tomos_mtx_info& in = m.info;
    const int64_t entries = in.entries;
    if (entries == 0) return kParsed;
    MappedTokens mt;
    if (!mt.open(m.f)) return kNoMap;
    if (mt.cnt.back() < entries) return kMalformed;
    std::atomic<bool> bad(false);
    const ArrayPos pos{in.rows, in.cols, in.symmetry};
    mt.run([&](int k) {
        int64_t t = mt.cnt[k];
        if (t >= entries) return;
        int64_t i, j;
        pos.at(t, &i, &j);
        for (size_t p = mt.lo[k]; p < mt.hi[k] && t < entries; ++p) {
            if (!mt.starts_token(p)) continue;
            const size_t e = mt.token_end(p);
            double v;
            if (!parse_token(mt.d + p, mt.d + e, &v)) {
                bad.store(true, std::memory_order_relaxed);
                return;
            }
            at(i, j, v);
            ++t;
            pos.next(&i, &j);
            p = e;  // the loop's ++p then steps past the whitespace at e
        }
    });
    return bad.load() ? kMalformed : kParsed;
}

// As parse_token, for a 1-based index: a whole decimal integer token.
bool parse_index(const char* p, const char* e, long long* v) {
    const size_t n = (size_t)(e - p);
    if (n == 0 || n > 127) return false;
    char tok[128];
    std::memcpy(tok, p, n);
    tok[n] = '\0';
    char* end = nullptr;
    errno = 0;
    *v = std::strtoll(tok, &end, 10);
    return end == tok + n && errno == 0;
}

void atomic_min(std::atomic<int64_t>& a, int64_t v) {
    int64_t cur = a.load(std::memory_order_relaxed);
    while (v < cur && !a.compare_exchange_weak(cur, v, std::memory_order_relaxed)) {
    }
}

// The entries of a `general` coordinate file (positioned at its first
// entry), in parallel: store(e, row, col, value), 0-based, once for every
// entry e.  An entry belongs to the range its first token starts in and is
// read to its end, past the range if need be.  Errors name the first bad
// entry in file order, as the sequential reader would meet it.
template <class Store>
tomos_status read_coord_parallel(MtxFile& m, const char* path, bool* nomap, Store&& store) {
    using tomos_b200::fail;
    const tomos_mtx_info& in = m.info;
    const int per = in.field == TOMOS_MTX_PATTERN ? 2 : 3;
    const int64_t entries = in.entries;
    const std::string bad = std::string("'") + path + "': truncated/malformed data";
    if (entries == 0) return TOMOS_OK;
    MappedTokens mt;
    *nomap = !mt.open(m.f);
    if (*nomap) return TOMOS_OK;  // the caller reads the file sequentially
    const int64_t have = std::min<int64_t>(entries, mt.cnt.back() / per);
    // no complete entry at all (a data section that is empty or ends at the
    // size line): nothing to parse, and too few entries
    if (mt.nt < 1 || have < 1) return fail(TOMOS_ERR_INVALID, bad);
    std::atomic<int64_t> first_bad(INT64_MAX), first_out(INT64_MAX);
    mt.run([&](int k) {
        int64_t t = mt.cnt[k];
        for (size_t p = mt.lo[k]; p < mt.hi[k]; ++p) {
            if (!mt.starts_token(p)) continue;
            if (t % per != 0) {  // inside an entry an earlier range reads
                p = mt.token_end(p);
                ++t;
                continue;
            }
            const int64_t e = t / per;
            if (e >= have) return;
            size_t q = p, qe = mt.token_end(q);
            long long i = 0, j = 0;
            double v = 1.0;
            bool ok = parse_index(mt.d + q, mt.d + qe, &i);
            q = mt.next_token(qe);
            qe = mt.token_end(q);
            ok = ok && parse_index(mt.d + q, mt.d + qe, &j);
            if (per == 3) {
                q = mt.next_token(qe);
                qe = mt.token_end(q);
                ok = ok && parse_token(mt.d + q, mt.d + qe, &v);
            }
            if (!ok) {
                atomic_min(first_bad, e);
                return;
            }
            if (i < 1 || j < 1 || i > in.rows || j > in.cols) {
                atomic_min(first_out, e);
                return;
            }
            store(e, (int64_t)(i - 1), (int64_t)(j - 1), v);
            t += per;
            p = qe;
        }
    });
    const int64_t b = first_bad.load(), o = first_out.load();
    if (b != INT64_MAX && b <= o) return fail(TOMOS_ERR_INVALID, bad);
    if (o != INT64_MAX)
        return fail(TOMOS_ERR_INVALID, std::string("'") + path + "': entry " + std::to_string(o + 1) +
                                           " lies outside the matrix");
    if (have < entries) return fail(TOMOS_ERR_INVALID, bad);
    return TOMOS_OK;
}

}  // namespace

extern "C" {

tomos_status tomos_mtx_read_info(const char* path, tomos_mtx_info* info) {
    if (!info) return tomos_b200::fail(TOMOS_ERR_INVALID, "tomos_mtx_read_info: null info");
    MtxFile m;
    tomos_status s = mtx_open(path, m);
    if (s) return s;
    *info = m.info;
    return TOMOS_OK;
}

tomos_status tomos_mtx_read_dense(const char* path, int32_t layout, double* out, int64_t ld) {
    using tomos_b200::fail;
    MtxFile m;
    tomos_status s = mtx_open(path, m);
    if (s) return s;
    const tomos_mtx_info& in = m.info;
    const int64_t need = layout == TOMOS_COL_MAJOR ? in.rows : in.cols;
    if (!out || ld < need || ld < 1)
        return fail(TOMOS_ERR_INVALID, "tomos_mtx_read_dense: null output or ld too small");
    auto at = [&](int64_t i, int64_t j) -> double& {
        return layout == TOMOS_COL_MAJOR ? out[(size_t)j * ld + i] : out[(size_t)i * ld + j];
    };
    for (int64_t j = 0; j < in.cols; ++j)
        for (int64_t i = 0; i < in.rows; ++i) at(i, j) = 0.0;
    const int32_t sym = in.symmetry;
    // in parallel where the file maps; otherwise (a pipe, say) sequentially
    // below, from the same file position
    if (in.format == TOMOS_MTX_ARRAY) {
        const int r = read_array_parallel(m, [&](int64_t i, int64_t j, double v) {
            at(i, j) = v;
            if (sym != TOMOS_MTX_GENERAL && i != j) at(j, i) = sym == TOMOS_MTX_SKEW ? -v : v;
        });
        if (r == kMalformed) return fail(TOMOS_ERR_INVALID, std::string("'") + path + "': truncated/malformed data");
        if (r == kParsed) return TOMOS_OK;
    } else if (sym == TOMOS_MTX_GENERAL) {
        // triplets parsed in parallel, then added in file order (repeated
        // entries sum as the sequential read sums them)
        std::vector<int64_t> ri, ci;
        std::vector<double> vi;
        try {
            ri.resize((size_t)in.entries);
            ci.resize((size_t)in.entries);
            vi.resize((size_t)in.entries);
        } catch (...) {
            return fail(TOMOS_ERR_ALLOC, "tomos_mtx_read_dense: no host memory for the entries");
        }
        bool nomap = false;
        s = read_coord_parallel(m, path, &nomap, [&](int64_t e, int64_t i, int64_t j, double v) {
            ri[(size_t)e] = i;
            ci[(size_t)e] = j;
            vi[(size_t)e] = v;
        });
        if (s) return s;
        if (!nomap) {
            for (size_t e = 0; e < vi.size(); ++e) at(ri[e], ci[e]) += vi[e];
            return TOMOS_OK;
        }
    }
    return mtx_entries(m, path, [&](int64_t i, int64_t j, double v) {
        if (in.format == TOMOS_MTX_COORDINATE) at(i, j) += v;  // repeated entries add
        else at(i, j) = v;
        if (sym != TOMOS_MTX_GENERAL && i != j) {
            const double w = sym == TOMOS_MTX_SKEW ? -v : v;
            if (in.format == TOMOS_MTX_COORDINATE) at(j, i) += w;
            else at(j, i) = w;
        }
    });
}

tomos_status tomos_mtx_read_coo(const char* path, int64_t cap, int64_t* rows, int64_t* cols, double* vals,
                                int64_t* count) {
    using tomos_b200::fail;
    MtxFile m;
    tomos_status s = mtx_open(path, m);
    if (s) return s;
    if (!count) return fail(TOMOS_ERR_INVALID, "tomos_mtx_read_coo: null count");
    int64_t k = 0;
    bool over = false;
    auto put = [&](int64_t i, int64_t j, double v) {
        if (k < cap && rows && cols && vals) {
            rows[k] = i;
            cols[k] = j;
            vals[k] = v;
        } else {
            over = true;
        }
        ++k;
    };
    const int32_t sym = m.info.symmetry;
    bool nomap = true;
    if (m.info.format == TOMOS_MTX_COORDINATE && sym == TOMOS_MTX_GENERAL) {
        std::atomic<bool> full(false);
        const bool room = rows && cols && vals;
        s = read_coord_parallel(m, path, &nomap, [&](int64_t e, int64_t i, int64_t j, double v) {
            if (room && e < cap) {
                rows[e] = i;
                cols[e] = j;
                vals[e] = v;
            } else {
                full.store(true, std::memory_order_relaxed);
            }
        });
        if (!nomap) {
            k = m.info.entries;
            over = full.load();
        }
    }
    if (nomap) {
        s = mtx_entries(m, path, [&](int64_t i, int64_t j, double v) {
            put(i, j, v);
            if (sym != TOMOS_MTX_GENERAL && i != j) put(j, i, sym == TOMOS_MTX_SKEW ? -v : v);
        });
    }
    if (s) return s;
    *count = k;
    if (over)
        return fail(TOMOS_ERR_INVALID, "tomos_mtx_read_coo: " + std::to_string(k) +
                                           " entries do not fit the given capacity");
    return TOMOS_OK;
}

tomos_status tomos_mtx_write_dense(const char* path, int32_t layout, int64_t rows, int64_t cols,
                                   const double* a, int64_t ld) {
    using tomos_b200::fail;
    const int64_t need = layout == TOMOS_COL_MAJOR ? rows : cols;
    if (rows < 0 || cols < 0 || (rows * cols > 0 && (!a || ld < need)))
        return fail(TOMOS_ERR_INVALID, "tomos_mtx_write_dense: bad shape, ld or null matrix");
    FILE* f = path ? std::fopen(path, "w") : nullptr;
    if (!f) return fail(TOMOS_ERR_INVALID, std::string("could not open '") + (path ? path : "") + "' for writing");
    bool ok = std::fprintf(f, "%%%%MatrixMarket matrix array real general\n%lld %lld\n", (long long)rows,
                           (long long)cols) > 0;
    // Values in file order (column by column), "%.17g" a line: host threads
    // format consecutive blocks of kBlock values into their own buffers,
    // which are then written in order, so the bytes are the sequential
    // fprintf's.
    constexpr int64_t kBlock = 1 << 18;
    const int64_t total = rows * cols;
    const int nt = parse_threads((size_t)(total * 24));
    std::vector<std::string> buf(nt);
    auto value = [&](int64_t t) {
        const int64_t i = t % rows, j = t / rows;
        return layout == TOMOS_COL_MAJOR ? a[(size_t)j * ld + i] : a[(size_t)i * ld + j];
    };
    for (int64_t t0 = 0; ok && t0 < total; t0 += kBlock * nt) {
        auto body = [&](int k) {
            std::string& b = buf[k];
            b.clear();
            const int64_t lo = t0 + kBlock * k, hi = std::min(total, lo + kBlock);
            char s[40];
            for (int64_t t = lo; t < hi; ++t) {
                const int n = std::snprintf(s, sizeof(s), "%.17g\n", value(t));
                b.append(s, (size_t)n);
            }
        };
        std::vector<std::thread> th;
        int spawned = 1;
        for (int k = 1; k < nt; ++k) {
            try {
                th.emplace_back(body, k);
                ++spawned;
            } catch (...) {
                break;
            }
        }
        body(0);
        for (int k = spawned; k < nt; ++k) body(k);
        for (auto& x : th) x.join();
        for (int k = 0; ok && k < nt; ++k)
            ok = buf[k].empty() || std::fwrite(buf[k].data(), 1, buf[k].size(), f) == buf[k].size();
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(TOMOS_ERR_INVALID, std::string("'") + path + "': write failed");
    return TOMOS_OK;
}

}  // extern "C"
