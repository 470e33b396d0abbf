// io.cu -- the reference's point-file format, parsed on the host (host code
// only; compiled with the rest of the library).
//
// load_points_fast (gprt-sandbox/src/io.rs:8-30) reads "x,y,z" lines: the
// file is split on '\n', empty lines are skipped, each line is split on ','
// and its first three fields, trimmed of white space, are parsed as f32; a
// line whose first three fields do not all parse is skipped, fields after
// the third are ignored.  This is the same format, parsed in parallel
// chunks by std::thread workers over a read-only mapping of the file, with
// the order of lines kept.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <rtdsl.h>

namespace rtd {
rtd_status fail(rtd_status s, const std::string &msg);
}

namespace {

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f' || c == '\n'; }

// One trimmed field as an f32, accepting what a Rust f32 parse accepts:
// optional sign, decimal digits with an optional fraction and exponent, or
// inf / infinity / nan in any case; nothing else (no hex, no inner spaces).
bool parse_f32(const char *b, const char *e, float *out) {
    while (b < e && is_space(*b)) ++b;
    while (e > b && is_space(e[-1])) --e;
    if (b == e) return false;
    const size_t len = (size_t)(e - b);
    char buf[64];
    if (len >= sizeof(buf)) return false;
    memcpy(buf, b, len);
    buf[len] = 0;
    const char *s = buf;
    if (*s == '+' || *s == '-') ++s;
    std::string word(s);
    std::transform(word.begin(), word.end(), word.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    if (word == "inf" || word == "infinity" || word == "nan") {
        const bool neg = buf[0] == '-';
        *out = word == "nan" ? NAN : (neg ? -INFINITY : INFINITY);
        return true;
    }
    // decimal form only: digits [. digits] [e|E [sign] digits]
    const char *p = s;
    bool digits = false;
    while (*p >= '0' && *p <= '9') { ++p; digits = true; }
    if (*p == '.') {
        ++p;
        while (*p >= '0' && *p <= '9') { ++p; digits = true; }
    }
    if (!digits) return false;
    if (*p == 'e' || *p == 'E') {
        ++p;
        if (*p == '+' || *p == '-') ++p;
        if (!(*p >= '0' && *p <= '9')) return false;
        while (*p >= '0' && *p <= '9') ++p;
    }
    if (*p != 0) return false;
    errno = 0;
    char *end = nullptr;
    const float v = strtof(buf, &end);   // correctly rounded, like the Rust parse
    if (end != buf + len) return false;
    *out = v;   // overflow gives +-inf, as a Rust f32 parse does
    return true;
}

// Parses the lines that start in [b, e) (a line starting inside runs to its
// '\n' even past e) into out.
void parse_chunk(const char *base, size_t size, size_t b, size_t e, std::vector<float> *out) {
    size_t i = b;
    while (i < e) {
        size_t j = i;
        while (j < size && base[j] != '\n') ++j;
        if (j > i) {
            float v[3];
            const char *p = base + i, *le = base + j;
            int f = 0;
            while (f < 3) {
                const char *c = p;
                while (c < le && *c != ',') ++c;
                if (!parse_f32(p, c, &v[f])) break;
                ++f;
                if (c == le) break;
                p = c + 1;
            }
            if (f == 3) out->insert(out->end(), v, v + 3);
        }
        i = j + 1;
    }
}

}  // namespace

extern "C" rtd_status rtd_load_points_csv(const char *path, float *out, uint64_t capacity,
                                          uint64_t *n_points) {
    if (!path || !n_points) return rtd::fail(RTD_ERR_INVALID_ARGUMENT, "NULL argument");
    if (capacity && !out) return rtd::fail(RTD_ERR_INVALID_ARGUMENT, "NULL output");
    *n_points = 0;
    const int fd = open(path, O_RDONLY);
    if (fd < 0) return rtd::fail(RTD_ERR_INVALID_ARGUMENT, "cannot open the point file");
    struct stat stt;
    if (fstat(fd, &stt) != 0) {
        close(fd);
        return rtd::fail(RTD_ERR_INVALID_ARGUMENT, "cannot stat the point file");
    }
    const size_t size = (size_t)stt.st_size;
    const char *base = nullptr;
    if (size) {
        void *m = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
        if (m == MAP_FAILED) {
            close(fd);
            return rtd::fail(RTD_ERR_INVALID_ARGUMENT, "cannot map the point file");
        }
        base = static_cast<const char *>(m);
    }
    close(fd);
    unsigned nt = std::thread::hardware_concurrency();
    if (nt == 0) nt = 1;
    if (size < (1u << 20)) nt = 1;
    // chunk c covers the lines starting in [start[c], start[c+1])
    std::vector<size_t> start(nt + 1, size);
    start[0] = 0;
    for (unsigned c = 1; c < nt; ++c) {
        size_t s = size * c / nt;
        while (s < size && base[s - 1] != '\n') ++s;
        start[c] = std::max(s, start[c - 1]);
    }
    std::vector<std::vector<float>> parts(nt);
    std::vector<std::thread> th;
    for (unsigned c = 0; c < nt; ++c)
        th.emplace_back(parse_chunk, base, size, start[c], start[c + 1], &parts[c]);
    for (auto &t : th) t.join();
    if (base) munmap(const_cast<char *>(base), size);
    uint64_t n = 0;
    for (auto &p : parts) n += p.size() / 3;
    *n_points = n;
    if (n > capacity) return rtd::fail(RTD_ERR_OVERFLOW, "point buffer smaller than the file's point count");
    uint64_t o = 0;
    for (auto &p : parts) {
        if (!p.empty()) memcpy(out + 3 * o, p.data(), p.size() * sizeof(float));
        o += p.size() / 3;
    }
    return RTD_OK;
}
